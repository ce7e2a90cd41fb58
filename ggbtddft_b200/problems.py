"""Run definitions: everything one atom-in-field run needs, built from the input producers.

A ``RunInputs`` holds the same arrays the reference's ``main.cu`` loads from ``workingData``
plus its compile-time scalars (``src/params.cuh:25-60``):

    grid (r, drdx, P)                    workingData/mesh/{r,drdx,P}.bin
    W [N_l][N_r][N_r] complex128         workingData/hamiltonian/propagators/propagatorL%03d.bin
    V/D per coupling [N_m][N_l][N_l]     workingData/hamiltonian/propagatorsL/<c>/V%03d.bin, D%03d.bin
    x0 [N_l][n_orb][N_r] complex128      workingData/eigenStates/active/<id>/eigenStatesL%03d.bin
    l/m/occ [n_orb] int32, rho_frozen    workingData/stateParameters/*.bin
    E [N_t]                              h_initialiseField (host-computed)

Named builders produce the benchmark configurations with seeded synthetic laser parameters.
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import inputs as I

# Wall-clock seconds spent in the one-time input producers (ground-state SCF, radial propagators,
# angular eigensystems) since the last ``reset_setup_seconds()``: set-up, reported beside the step rate.
SETUP_SECONDS: Dict[str, float] = {"ground_state": 0.0, "radial_propagators": 0.0, "angular": 0.0}


def reset_setup_seconds() -> None:
    for k in SETUP_SECONDS:
        SETUP_SECONDS[k] = 0.0


@dataclasses.dataclass
class RunInputs:
    grid: I.RadialGrid
    n_l: int
    dt: float
    W: np.ndarray
    V: Dict[str, np.ndarray]
    D: Dict[str, np.ndarray]
    x0: np.ndarray
    l_active: np.ndarray
    m_active: np.ndarray
    occ: np.ndarray
    rho_frozen: np.ndarray
    E: np.ndarray
    n_har: int = 4
    use_hartree: int = 1
    target_id: int = 0
    xc_correlation: bool = False
    xc_frozen: bool = False        # exchange-correlation potential held at its t = 0 value
    name: str = ""
    omega0: float = 0.057
    angular: str = "reference"     # "reference": the FF/FP/D/P/S chain; "theta": one phase at the P nodes

    @property
    def n_r(self) -> int:
        return self.grid.n_r

    @property
    def n_orb(self) -> int:
        return self.x0.shape[1]

    @property
    def n_t(self) -> int:
        return self.E.size

    @property
    def n_m(self) -> int:
        return int(self.m_active.max()) + 1

    def with_field(self, E: np.ndarray) -> "RunInputs":
        return dataclasses.replace(self, E=np.ascontiguousarray(E, dtype=np.float64))


def initial_orbitals(gs: I.GroundState, n_l: int) -> np.ndarray:
    """x[l][kso][r]: orbital kso placed in its own l, zero elsewhere (h_initialiseTDKSOSet.cuh:59-84)."""
    n_orb = len(gs.orbitals)
    x = np.zeros((n_l, n_orb, gs.u.shape[1]), dtype=np.complex128)
    for k, o in enumerate(gs.orbitals):
        x[o.l, k, :] = gs.u[k]
    return x


def build_run(grid: I.RadialGrid, n_l: int, dt: float, gs: I.GroundState, E: np.ndarray, *,
              absorber: str = "cap", cap_r_mask: Optional[float] = None, cap_passes: int = 2,
              mask_width: Optional[float] = None, n_har: int = 4, use_hartree: int = 1,
              target_id: int = 0, xc_correlation: bool = False, name: str = "",
              omega0: float = 0.057, device: Optional[str] = None,
              W: Optional[np.ndarray] = None, angular: str = "reference", xc_frozen: bool = False) -> RunInputs:
    """Assemble one run.

    absorber = "cap":  the reference's Manolopoulos CAP starting at ``cap_r_mask``, entering the
                       Hamiltonian ``cap_passes`` times (2 reproduces v0 - i W - i maskR,
                       groundState.py:27 + internal.py:253).
    absorber = "mask": a cos^(1/8) mask over the last ``mask_width`` a.u. folded into W's rows.
    """
    r = grid.r
    if absorber == "cap":
        r_mask = cap_r_mask if cap_r_mask is not None else grid.r_max / 1.5
        cap = I.cap_manolopoulos(r, r_mask, grid.r_max)
        v0 = gs.v_ion - 1j * cap * (cap_passes - 1)
        mask_r = cap
        row_mask = None
    elif absorber == "mask":
        v0 = gs.v_ion.astype(np.complex128)
        mask_r = np.zeros_like(r)
        row_mask = I.mask_cos8(r, grid.r_max, mask_width)
    elif absorber == "none":
        v0 = gs.v_ion.astype(np.complex128)
        mask_r = np.zeros_like(r)
        row_mask = None
    else:
        raise ValueError(absorber)
    if W is None:
        t0 = time.perf_counter()
        W = I.radial_propagators(grid, n_l, dt, v0, gs.vscf, mask_r, row_mask=row_mask, device=device)
        SETUP_SECONDS["radial_propagators"] += time.perf_counter() - t0
    n_m = int(max(o.m for o in gs.orbitals)) + 1
    t0 = time.perf_counter()
    ang = I.angular_eigensystems(n_l, n_m)
    SETUP_SECONDS["angular"] += time.perf_counter() - t0
    return RunInputs(
        grid=grid, n_l=n_l, dt=dt, W=W,
        V={c: ang[c][0] for c in I.COUPLINGS}, D={c: ang[c][1] for c in I.COUPLINGS},
        x0=initial_orbitals(gs, n_l),
        l_active=np.array([o.l for o in gs.orbitals], dtype=np.int32),
        m_active=np.array([o.m for o in gs.orbitals], dtype=np.int32),
        occ=np.array([o.occ for o in gs.orbitals], dtype=np.int32),
        rho_frozen=gs.rho_frozen.copy(), E=np.ascontiguousarray(E, dtype=np.float64),
        n_har=n_har, use_hartree=use_hartree, target_id=target_id,
        xc_correlation=xc_correlation, name=name, omega0=omega0, angular=angular, xc_frozen=xc_frozen)


# ----------------------------------------------------------------------------------------------
# small, reference-shaped problems (multiples of 32 so that the reference binary covers them too)
# ----------------------------------------------------------------------------------------------

def reference_like(n_r: int = 64, n_l: int = 32, n_t: int = 64, atom: str = "H", *,
                   r_mask: float = 30.0, zeta_ref: float = 1.0, dt_as: float = 20.0,
                   intensity: float = 2e14, omega0: float = 0.057, cycles: float = 1.0,
                   cep: float = 0.5 * math.pi, n_har: int = 4, use_hartree: int = 1,
                   seed: int = 0, perturb: float = 0.0, device: Optional[str] = None) -> RunInputs:
    """A run built the way the reference's init.py builds one (CAP twice, super-Gaussian, CN).

    atom "H": hydrogen-like 1s, targetID 0 (no Hartree/XC in the loop).
    atom "Ne3": a 3-orbital LDA atom (1s, 2p0, 2p1; occ 2,2,4; targetID 2) so that every
    coupling (P, FP, D, FF, S), the Hartree multipoles and the exchange potential are active.
    atom "Ar9": argon's nine orbitals (Z = 18, LDA), targetID 5, all couplings active: the size of
    the argon workloads on the reference's own code path.
    ``perturb`` mixes seeded random noise into the initial orbitals (then renormalises) so that
    the parity tests also exercise components that vanish for exact eigenstates.
    """
    r_max = 1.5 * r_mask
    grid = I.make_grid(n_r, r_max, zeta_ref)
    dt = dt_as * I.ATTOSECOND_AU
    if atom == "H":
        gs = I.ground_state(grid, 1.0, I.ORBITALS_H, interacting=False)
        target_id = 0
    elif atom == "Ne3":
        orbs = [I.Orbital(1, 0, 0, 2), I.Orbital(2, 1, 0, 2), I.Orbital(2, 1, 1, 4)]
        gs = I.ground_state(grid, 8.0, orbs, interacting=True, iterations=60)
        target_id = 2
    elif atom == "Ar9":
        gs = I.ground_state(grid, 18.0, I.ORBITALS_AR, interacting=True, device=device)
        target_id = 5
    else:
        raise ValueError(atom)
    if perturb:
        rng = np.random.default_rng(seed)
        u = gs.u + perturb * rng.standard_normal(gs.u.shape) * np.abs(gs.u).max(axis=1, keepdims=True)
        u /= np.sqrt((u ** 2).sum(axis=1, keepdims=True))
        gs = dataclasses.replace(gs, u=u)
    t = I.time_grid(n_t, dt)
    e0 = I.intensity_to_e0(intensity)
    tau0 = cycles * 2.0 * math.pi / omega0
    E = I.field_super_gaussian(t, e0, omega0, tau0, cep)
    return build_run(grid, n_l, dt, gs, E, absorber="cap", cap_r_mask=r_mask, cap_passes=2,
                     n_har=n_har, use_hartree=use_hartree, target_id=target_id,
                     name=f"{atom}-N{n_r}-L{n_l}", omega0=omega0, device=device)


# ----------------------------------------------------------------------------------------------
# benchmark configurations
# ----------------------------------------------------------------------------------------------

# Angular step of the benchmark configurations: "theta" (one phase per half-step at the Gauss nodes,
# the form these configurations are benchmarked in) or "reference" (the reference's FF/FP/D/P/S chain,
# the parity form).  The reference_like() runs always use the reference's chain.
BENCH_ANGULAR = "theta"


@dataclasses.dataclass
class LaserSpec:
    intensity: float      # W/cm^2
    wavelength_nm: float
    cycles: float
    cep: float = 0.0

    @property
    def omega(self) -> float:
        return I.wavelength_to_omega(self.wavelength_nm)

    @property
    def e0(self) -> float:
        return I.intensity_to_e0(self.intensity)


@dataclasses.dataclass
class AtomSpec:
    name: str
    Z: float
    orbitals: List[I.Orbital]
    interacting: bool
    correlation: bool


ATOMS = {
    "H": AtomSpec("H", 1.0, I.ORBITALS_H, False, False),
    "He": AtomSpec("He", 2.0, I.ORBITALS_HE, True, True),
    "Ar": AtomSpec("Ar", 18.0, I.ORBITALS_AR, True, True),
}


def baseline_run(atom: str, n_r: int, r_max: float, l_max: int, dt: float, laser: LaserSpec,
                 mask_width: float, zeta: float = 0.5, n_steps: Optional[int] = None,
                 device: Optional[str] = None, gs_cache: Optional[dict] = None,
                 W: Optional[np.ndarray] = None, angular: Optional[str] = None,
                 n_har: Optional[int] = None, xc_frozen: bool = False) -> RunInputs:
    """One of the benchmark configurations: sin^2 pulse, cos^(1/8) mask, Z = true nuclear charge.

    Hartree/XC runs use the reference's multipole treatment (L <= 3, N_har = 4) with Slater
    exchange plus PW92 correlation.
    """
    spec = ATOMS[atom]
    grid = I.make_grid(n_r, r_max, I.zeta_physical_to_ref(zeta, r_max))
    key = (atom, n_r, r_max)
    gs = None if gs_cache is None else gs_cache.get(key)
    if gs is None:
        t0 = time.perf_counter()
        gs = I.ground_state(grid, spec.Z, spec.orbitals, interacting=spec.interacting,
                            correlation=spec.correlation, device=device)
        SETUP_SECONDS["ground_state"] += time.perf_counter() - t0
        if gs_cache is not None:
            gs_cache[key] = gs
    full = I.steps_for_sin2(dt, laser.omega, laser.cycles)
    n_t = full if n_steps is None else n_steps
    E = I.field_sin2(n_t, dt, laser.e0, laser.omega, laser.cycles, laser.cep)
    target = 0 if not spec.interacting else 1
    if n_har is None:
        n_har = 4 if spec.interacting else 2
    return build_run(grid, l_max + 1, dt, gs, E, absorber="mask", mask_width=mask_width,
                     n_har=n_har, use_hartree=1 if spec.interacting else 0,
                     target_id=target, xc_correlation=spec.correlation,
                     name=f"{atom}-N{n_r}-L{l_max}", omega0=laser.omega, device=device, W=W,
                     angular=BENCH_ANGULAR if angular is None else angular, xc_frozen=xc_frozen)


def config_hydrogen(n_steps=None, device=None, angular=None) -> RunInputs:
    """H FP64: N_r=200, r_max=100, l_max=32, 800 nm, 1e14 W/cm^2, 4-cycle sin^2, dt=0.05, mask 20 a.u."""
    return baseline_run("H", 200, 100.0, 32, 0.05, LaserSpec(1e14, 800.0, 4.0, 0.0), 20.0,
                        n_steps=n_steps, device=device, angular=angular)


def config_helium(n_steps=None, device=None, angular=None) -> RunInputs:
    """He LDA FP64: N_r=400, r_max=200, l_max=64, 800 nm, 1.5e14, 8 cycles, dt=0.03, mask 40 a.u.;
    in the theta form the Hartree potential of every multipole L = 0 .. 2 l_max = 128."""
    a = BENCH_ANGULAR if angular is None else angular
    return baseline_run("He", 400, 200.0, 64, 0.03, LaserSpec(1.5e14, 800.0, 8.0, 0.0), 40.0,
                        n_steps=n_steps, device=device, angular=a, n_har=129 if a == "theta" else 4)


def config_argon(n_steps=None, device=None, angular=None, xc_frozen=False) -> RunInputs:
    """Ar LDA: N_r=600, r_max=300, l_max=96, 800 nm, 1.4e14, 10 cycles, dt=0.02, mask 60 a.u."""
    return baseline_run("Ar", 600, 300.0, 96, 0.02, LaserSpec(1.4e14, 800.0, 10.0, 0.0), 60.0,
                        n_steps=n_steps, device=device, angular=angular, xc_frozen=xc_frozen)


# ----------------------------------------------------------------------------------------------
# ensembles (focal-volume scans)
# ----------------------------------------------------------------------------------------------

@dataclasses.dataclass
class GridRung:
    n_r: int
    r_max: float
    l_max: int


# Grid ladders.  Runs are binned onto a few grids so that the runs of one grid share W (the radial
# propagators depend on the atom, the grid, dt and the absorber, not on the laser).  l_max 127 rather
# than 128: N_l = 128 channels fill one 128-row tensor-core tile of the int8 angular chain, where 129
# would need a second, nearly empty one (half the radii per CTA).
ARGON_LADDER = [GridRung(600, 300.0, 96), GridRung(700, 350.0, 112), GridRung(800, 400.0, 127),
                GridRung(900, 450.0, 144), GridRung(1000, 500.0, 160)]
HHE_LADDER = [GridRung(200, 100.0, 32), GridRung(400, 200.0, 64), GridRung(600, 300.0, 96),
              GridRung(800, 400.0, 127)]


def quiver_radius(laser: LaserSpec) -> float:
    return laser.e0 / laser.omega ** 2


@dataclasses.dataclass
class EnsembleDraws:
    """The seeded laser parameters of an ensemble and the ladder rung (grid) of each run."""
    atoms: List[str]
    intensity: np.ndarray
    wavelength_nm: np.ndarray
    cep: np.ndarray
    rung: np.ndarray
    cycles: float
    dt: float
    ladder: Sequence[GridRung]

    def grid_groups(self) -> Dict[tuple, List[int]]:
        """{(rung, atom): run indices}: the runs that share a grid and radial propagators (one grid
        group of the batched step), in ladder order."""
        out: Dict[tuple, List[int]] = {}
        for i, k in enumerate(self.rung):
            out.setdefault((int(k), self.atoms[i]), []).append(i)
        return dict(sorted(out.items()))


def argon_draws(n_runs: int = 64, seed: int = 0, ladder: Sequence[GridRung] = ARGON_LADDER) -> EnsembleDraws:
    """Argon LDA in-situ focal scan: I ~ U[0.8, 2]e14 W/cm^2, lambda ~ U[800, 1300] nm, 10-cycle sin^2,
    dt = 0.02, 9 orbitals; each run goes on the ladder rung indexed by its wavelength
    (longer wavelength -> larger excursion and higher cutoff -> larger grid and l_max)."""
    rng = np.random.default_rng(seed)
    I0 = rng.uniform(0.8e14, 2.0e14, n_runs)
    lam = rng.uniform(800.0, 1300.0, n_runs)
    rung = np.array([min(len(ladder) - 1, int((l - 800.0) / 100.0)) for l in lam])
    return EnsembleDraws(["Ar"] * n_runs, I0, lam, np.zeros(n_runs), rung, 10.0, 0.02, ladder)


def hhe_draws(n_runs: int = 256, seed: int = 0, ladder: Sequence[GridRung] = HHE_LADDER) -> EnsembleDraws:
    """H/He-like scan: I log-uniform in [0.5, 3]e14, CEP ~ U[0, 2 pi), lambda ~ U[800, 1800] nm,
    6-cycle sin^2, dt = 0.03; atoms alternate H / He; the rung is the smallest whose r_max covers
    3 quiver radii plus the absorber."""
    rng = np.random.default_rng(seed)
    I0 = np.exp(rng.uniform(np.log(0.5e14), np.log(3.0e14), n_runs))
    cep = rng.uniform(0.0, 2.0 * np.pi, n_runs)
    lam = rng.uniform(800.0, 1800.0, n_runs)

    def rung(i_run):
        a = quiver_radius(LaserSpec(I0[i_run], lam[i_run], 6.0))
        for k, g in enumerate(ladder):
            if g.r_max * 0.8 >= 3.0 * a:
                return k
        return len(ladder) - 1
    atoms = ["H" if i % 2 == 0 else "He" for i in range(n_runs)]
    return EnsembleDraws(atoms, I0, lam, cep, np.array([rung(i) for i in range(n_runs)]), 6.0, 0.03, ladder)


def argon_ensemble(n_runs: int = 64, seed: int = 0, n_steps: Optional[int] = None, device=None,
                   ladder: Sequence[GridRung] = ARGON_LADDER, only=None, xc_frozen: bool = False) -> List[RunInputs]:
    """The runs of ``argon_draws``; ``xc_frozen`` keeps each run's exchange-correlation potential at its
    ground-state value (the Hartree multipoles still follow the density)."""
    return _ensemble(argon_draws(n_runs, seed, ladder), n_steps, device, only=only, xc_frozen=xc_frozen)


def hhe_ensemble(n_runs: int = 256, seed: int = 0, n_steps: Optional[int] = None, device=None,
                 ladder: Sequence[GridRung] = HHE_LADDER, only=None) -> List[RunInputs]:
    """The runs of ``hhe_draws``."""
    return _ensemble(hhe_draws(n_runs, seed, ladder), n_steps, device, only=only)


def _ensemble(dr: EnsembleDraws, n_steps, device, only=None, xc_frozen: bool = False):
    """The runs of an ensemble from its drawn parameters; ``only`` = indices of the runs to build
    (the draws are made for the whole ensemble first, so a selected run equals its twin in the full
    ensemble)."""
    n_runs = len(dr.intensity)
    I0, lam, cep, cycles, dt, ladder = dr.intensity, dr.wavelength_nm, dr.cep, dr.cycles, dr.dt, dr.ladder
    runs: List[RunInputs] = []
    gs_cache: dict = {}
    w_cache: dict = {}
    for i in (range(n_runs) if only is None else only):
        a = dr.atoms[i]
        k = int(dr.rung[i])
        g = ladder[k]
        laser = LaserSpec(float(I0[i]), float(lam[i]), cycles, float(cep[i]))
        key = (a, g.n_r, g.r_max, g.l_max)
        run = baseline_run(a, g.n_r, g.r_max, g.l_max, dt, laser, 0.2 * g.r_max, n_steps=n_steps,
                           device=device, gs_cache=gs_cache, W=w_cache.get(key), xc_frozen=xc_frozen)
        w_cache[key] = run.W
        run.name = f"{a}-{i}-N{g.n_r}-L{g.l_max}"
        runs.append(run)
    return runs
