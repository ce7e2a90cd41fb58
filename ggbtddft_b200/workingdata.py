"""Reader/writer for the reference's file contract (workingData inputs, params.cuh, output files).

Input side (written by ``src/scripts/init.py:341-380`` and ``internal.py:141-198,326-331``,
read by ``main.cu`` through ``h_initialiseMesh.cuh``, ``h_initialisePropagators.cuh`` and
``h_initialiseTDKSOSet.cuh``), all raw little-endian:

    workingData/mesh/{r,drdx,P}.bin                                  f64[N_r]
    workingData/mesh/time.bin                                        f64[N_t]
    workingData/mesh/TD.bin                                          f64[N_scan]
    workingData/mesh/D1.bin                                          f64[N_r*N_r]  (unused by the loop)
    workingData/hamiltonian/propagators/propagatorL%03d.bin          c128[N_r][N_r]
    workingData/hamiltonian/propagatorsL/<P|FP|D|FF dir>/V%03d.bin   f64[N_l][N_l]  per m < N_m
    workingData/hamiltonian/propagatorsL/<...>/D%03d.bin             f64[N_l]
    workingData/eigenStates/active/%03d/eigenStatesL%03d.bin         c128[N_kso][N_r]  l = 0..L0
    workingData/stateParameters/{l,m,occ}_active.bin                 i32[N_kso]
    workingData/stateParameters/densityFrozen.bin                    f64[N_r]

Output side (``src/subFunctions/output/h_writeDipoleMoment.cuh:1-87``):

    ../output/%08d/%05d/timeDependent/observables/dipoleMoment/scan%03d/kso%03d/dipL%03d.bin  c128[N_t]
    ../output/%08d/%05d/timeDependent/field/E%03d.bin                                          f64[N_t]

``params.cuh`` is the generated compile-time header (``init.py:493-606``); ``write_params_cuh``
emits the same macro set, ``parse_params_cuh`` reads one back.
"""
from __future__ import annotations

import math
import os
import re
from typing import Dict, Optional

import numpy as np

from . import inputs as I
from .problems import RunInputs

_INCLUDES = [
    "./subFunctions/system/h_checkCUDADevice.cuh",
    "",
    "./subFunctions/output/h_writeMesh.cuh",
    "./subFunctions/output/h_writeDipoleMoment.cuh",
    "./subFunctions/output/h_writeHartreePotential.cuh",
    "./subFunctions/output/h_writeExchangePotential.cuh",
    "",
    "./subFunctions/mesh/h_initialiseMesh.cuh",
    "",
    "./subFunctions/field/h_initialiseField.cuh",
    "./subFunctions/field/h_resetField.cuh",
    "",
    "./subFunctions/potentials/hartree/angularCoefficients.cuh",
    "./subFunctions/potentials/hartree/hartreePotentialDensity.cuh",
    "./subFunctions/potentials/hartree/h_calculateHartreePotential.cuh",
    "./subFunctions/potentials/exchangeCorrelation/h_calculateExchangeCorrelationPotential.cuh",
    "",
    "./subFunctions/timePropagation/h_initialisePropagators.cuh",
    "./subFunctions/timePropagation/h_initialiseTDKSOSet.cuh",
    "./subFunctions/timePropagation/observables/dipoleMoment.cuh",
    "./subFunctions/timePropagation/observables/dipoleAcceleration.cuh",
    "./subFunctions/timePropagation/externalFieldCoupling/lengthGauge/couplingS.cuh",
    "./subFunctions/timePropagation/externalFieldCoupling/lengthGauge/couplingP.cuh",
    "./subFunctions/timePropagation/externalFieldCoupling/lengthGauge/couplingD.cuh",
    "./subFunctions/timePropagation/externalFieldCoupling/lengthGauge/couplingF.cuh",
    "./subFunctions/timePropagation/h_timePropagation.cuh",
]


def _w(path: str, arr: np.ndarray, dtype) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.ascontiguousarray(arr, dtype=dtype).tofile(path)


def write_working_data(run: RunInputs, root: str, *, n_scan: int = 1, target_id: Optional[int] = None,
                       t: Optional[np.ndarray] = None) -> None:
    """Write ``root/workingData`` for ``run`` in the reference's layout."""
    wd = os.path.join(root, "workingData")
    g = run.grid
    tid = run.target_id if target_id is None else target_id
    _w(f"{wd}/mesh/r.bin", g.r, np.float64)
    _w(f"{wd}/mesh/drdx.bin", g.drdx, np.float64)
    _w(f"{wd}/mesh/P.bin", g.P, np.float64)
    if t is None:
        t = I.time_grid(run.n_t, run.dt)
    _w(f"{wd}/mesh/time.bin", t, np.float64)
    _w(f"{wd}/mesh/TD.bin", np.zeros(max(n_scan, 1)), np.float64)
    _w(f"{wd}/mesh/D1.bin", np.zeros(g.n_r * g.n_r), np.float64)
    for l in range(run.n_l):
        _w(f"{wd}/hamiltonian/propagators/propagatorL{l:03d}.bin", run.W[l], np.complex128)
    for c in I.COUPLINGS:
        d = I.COUPLING_DIRS[c]
        for m in range(run.n_m):
            _w(f"{wd}/hamiltonian/propagatorsL/{d}/V{m:03d}.bin", run.V[c][m], np.float64)
            _w(f"{wd}/hamiltonian/propagatorsL/{d}/D{m:03d}.bin", run.D[c][m], np.float64)
    l0 = int(run.l_active.max())
    for l in range(l0 + 1):
        _w(f"{wd}/eigenStates/active/{tid:03d}/eigenStatesL{l:03d}.bin", run.x0[l], np.complex128)
    _w(f"{wd}/stateParameters/l_active.bin", run.l_active, np.int32)
    _w(f"{wd}/stateParameters/m_active.bin", run.m_active, np.int32)
    _w(f"{wd}/stateParameters/occ_active.bin", run.occ, np.int32)
    _w(f"{wd}/stateParameters/densityFrozen.bin", run.rho_frozen, np.float64)


def write_params_cuh(run: RunInputs, path: str, *, e0: float, omega0: float, tau0: float, cep0: float,
                     sim_date: int = 20000101, sim_index: int = 0, n_scan: int = 1, in_situ: int = 0,
                     Z: float = 1.0, target_id: Optional[int] = None, output_root: str = "../output") -> None:
    """Emit a params.cuh with the macro set of init.py:493-606 for this run."""
    tid = run.target_id if target_id is None else target_id
    base = f"{output_root}/{sim_date:08d}/{sim_index:05d}"
    theta = 30e-3
    L = []
    a = L.append
    a("// Simulation Parameters \n")
    a(f"#define SIM_DATE ({sim_date})  ")
    a(f"#define SIM_INDEX ({sim_index})  \n")
    a("#define TD_SIMULATION (1)")
    a(f"#define IN_SITU ({in_situ})\n")
    a("#define CUDA_DEVICE (0)   ")
    a("#define MTPB (32)   \n")
    a(f"#define attosecondAU ({I.ATTOSECOND_AU:.14E}) ")
    a(f"#define femtosecondAU ({I.FEMTOSECOND_AU:.14E}) ")
    a(f"#define cAU ({137.035999074:.14E}) ")
    a(f"#define intensityAU ({I.INTENSITY_AU:.14E}) ")
    a(f"#define electronVoltAU ({I.ELECTRONVOLT_AU:.14E}) \n")
    g = run.grid
    a(f"#define N_r ({g.n_r}) ")
    a(f"#define N_g ({g.n_g}) ")
    a(f"#define zeta ({g.zeta_ref:.15E}) ")
    a(f"#define R_MAX ({g.r_max:.15E}) \n")
    a(f"#define R_MASK ({g.r_max / 1.5:.15E}) ")
    a(f"#define ETA_MASK ({1e-3:.15E}) \n")
    a(f"#define N_l ({run.n_l}) ")
    a(f"#define N_m ({run.n_m}) \n")
    a(f"#define Z ({Z:.15E}) ")
    a(f"#define L0 ({int(run.l_active.max())}) ")
    a(f"#define targetID ({tid}) ")
    a(f"#define N_kso ({run.n_orb}) \n")
    a(f"#define N_t ({run.n_t}) ")
    a(f"#define dt ({run.dt:.15E}) \n")
    a(f"#define E0 ({e0:.15E}) ")
    a(f"#define omega0 ({omega0:.15E}) ")
    a(f"#define omegaX ({13.0 / 27.2114:.15E}) ")
    a(f"#define tau0 ({tau0:.15E}) ")
    a(f"#define CEP0 ({cep0:.15E}) \n")
    a(f"#define PERTURBATION_AMPLITUDE ({(0.01 if in_situ else 0.0):.15E}) ")
    a(f"#define dphi ({2.0 * math.pi / max(n_scan, 1):.15E}) ")
    a(f"#define COS_THETA ({math.cos(theta):.15E}) ")
    a(f"#define THETA ({theta:.15E}) \n")
    a(f"#define N_scan ({n_scan}) \n")
    a(f"#define N_har ({run.n_har}) ")
    a(f"#define USE_HARTREE ({run.use_hartree}) ")
    a(f"#define HARTREE_FACTOR ({1.0:.14E}) ")
    a("#define FUNCTIONAL (1) \n")
    for key, rel in (("R", "r"), ("P", "P"), ("DRDX", "drdx"), ("E", "E"), ("TIME", "time"), ("D1", "D1"), ("TD", "TD")):
        a(f'#define WORKING_DATA_MESH_{key} "./workingData/mesh/{rel}.bin"')
    a("")
    for l in range(run.n_l):
        a(f'#define WORKING_DATA_PROPAGATOR_L_{l:03d} "./workingData/hamiltonian/propagators/propagatorL{l:03d}.bin"')
    a("")
    a(f'#define LOCAL_OUTPUT_MESH_R "{base}/static/mesh/r.bin"')
    a(f'#define LOCAL_OUTPUT_MESH_DRDX "{base}/static/mesh/drdx.bin"')
    a(f'#define LOCAL_OUTPUT_MESH_TIME "{base}/static/mesh/time.bin"')
    a(f'#define LOCAL_OUTPUT_MESH_E "{base}/timeDependent/field/E.bin"')
    a(f'#define LOCAL_OUTPUT_VHAR_VHAR "{base}/timeDependent/observables/vhar/vhar.bin"')
    a(f'#define LOCAL_OUTPUT_VHAR_VHAR0 "{base}/timeDependent/observables/vhar/vhar0.bin"')
    a(f'#define LOCAL_OUTPUT_VEXC_VEXC "{base}/timeDependent/observables/vexc/vexc.bin"')
    a(f'#define LOCAL_OUTPUT_VEXC_VEXC0 "{base}/timeDependent/observables/vexc/vexc0.bin"\n')
    a("// Load Library Files \n")
    for inc in _INCLUDES:
        a(f'#include "{inc}"' if inc else "")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def output_dirs(root: str, sim_date: int, sim_index: int, n_scan: int, n_kso: int) -> None:
    """Create the output directories the reference writes into without creating them itself."""
    base = os.path.join(root, f"{sim_date:08d}", f"{sim_index:05d}")
    for sub in ("static/mesh", "timeDependent/field", "timeDependent/observables/vhar",
                "timeDependent/observables/vexc"):
        os.makedirs(os.path.join(base, sub), exist_ok=True)
    for s in range(n_scan):
        for k in range(n_kso):
            os.makedirs(os.path.join(base, f"timeDependent/observables/dipoleMoment/scan{s:03d}/kso{k:03d}"),
                        exist_ok=True)


_MACRO = re.compile(r"^\s*#define\s+(\w+)\s+(.*?)\s*$")


def parse_params_cuh(path: str) -> Dict[str, object]:
    """Read the scalar macros of a params.cuh (numbers in parentheses, strings in quotes)."""
    out: Dict[str, object] = {}
    with open(path) as f:
        for line in f:
            mm = _MACRO.match(line)
            if not mm:
                continue
            key, val = mm.group(1), mm.group(2)
            if val.startswith('"'):
                out[key] = val.strip('"')
                continue
            val = val.strip("()")
            try:
                out[key] = int(val)
            except ValueError:
                try:
                    out[key] = float(val)
                except ValueError:
                    out[key] = val
    return out


def read_working_data(root: str, params: Dict[str, object], E: Optional[np.ndarray] = None) -> RunInputs:
    """Load a reference workingData tree + params macros into a RunInputs (parity runs)."""
    wd = os.path.join(root, "workingData")
    n_r, n_l, n_m, n_kso, n_t = (int(params[k]) for k in ("N_r", "N_l", "N_m", "N_kso", "N_t"))
    tid = int(params["targetID"])
    l0 = int(params["L0"])
    rd = lambda p, dt, n: np.fromfile(os.path.join(wd, p), dtype=dt, count=n)
    r = rd("mesh/r.bin", np.float64, n_r)
    drdx = rd("mesh/drdx.bin", np.float64, n_r)
    P = rd("mesh/P.bin", np.float64, n_r)
    W = np.stack([rd(f"hamiltonian/propagators/propagatorL{l:03d}.bin", np.complex128, n_r * n_r).reshape(n_r, n_r)
                  for l in range(n_l)])
    V, D = {}, {}
    for c in I.COUPLINGS:
        d = I.COUPLING_DIRS[c]
        V[c] = np.stack([rd(f"hamiltonian/propagatorsL/{d}/V{m:03d}.bin", np.float64, n_l * n_l).reshape(n_l, n_l)
                         for m in range(n_m)])
        D[c] = np.stack([rd(f"hamiltonian/propagatorsL/{d}/D{m:03d}.bin", np.float64, n_l) for m in range(n_m)])
    l_act = rd("stateParameters/l_active.bin", np.int32, n_kso)
    m_act = rd("stateParameters/m_active.bin", np.int32, n_kso)
    occ = rd("stateParameters/occ_active.bin", np.int32, n_kso)
    rho_f = rd("stateParameters/densityFrozen.bin", np.float64, n_r)
    x0 = np.zeros((n_l, n_kso, n_r), dtype=np.complex128)
    for l in range(l0 + 1):
        x0[l] = rd(f"eigenStates/active/{tid:03d}/eigenStatesL{l:03d}.bin", np.complex128, n_kso * n_r).reshape(n_kso, n_r)
    for k in range(n_kso):        # h_initialiseTDKSOSet.cuh:69-84: keep only l == l_active[kso]
        for l in range(n_l):
            if l != l_act[k]:
                x0[l, k] = 0.0
    x_map = np.arange(n_r) * 0.0
    grid = I.RadialGrid(n_r, float(params.get("R_MAX", r[-1])), float(params.get("zeta", 0.0)), x_map, r, drdx, P,
                        np.zeros((0, 0)))
    if E is None:
        t = rd("mesh/time.bin", np.float64, n_t)
        E = I.field_super_gaussian(t, float(params["E0"]), float(params["omega0"]), float(params["tau0"]),
                                   float(params["CEP0"]))
    return RunInputs(grid=grid, n_l=n_l, dt=float(params["dt"]), W=W, V=V, D=D, x0=x0, l_active=l_act,
                     m_active=m_act, occ=occ, rho_frozen=rho_f, E=np.asarray(E, dtype=np.float64),
                     n_har=int(params["N_har"]), use_hartree=int(params["USE_HARTREE"]), target_id=tid)


def dipole_path(root: str, sim_date: int, sim_index: int, scan: int, kso: int, l: int) -> str:
    return os.path.join(root, f"{sim_date:08d}", f"{sim_index:05d}",
                        f"timeDependent/observables/dipoleMoment/scan{scan:03d}/kso{kso:03d}/dipL{l:03d}.bin")


def read_dipole_outputs(root: str, sim_date: int, sim_index: int, scan: int, n_kso: int, n_l: int) -> np.ndarray:
    """dipole[l][kso][t] from the reference's per-(kso, l) output files."""
    rows = []
    for l in range(n_l):
        rows.append(np.stack([np.fromfile(dipole_path(root, sim_date, sim_index, scan, k, l), dtype=np.complex128)
                              for k in range(n_kso)]))
    return np.stack(rows)


def write_dipole_outputs(root: str, sim_date: int, sim_index: int, scan: int, dipole: np.ndarray,
                         E: Optional[np.ndarray] = None) -> None:
    """Write dipole[l][kso][t] (and E) in the reference's output layout (h_writeDipoleMoment.cuh)."""
    n_l, n_kso, _ = dipole.shape
    for k in range(n_kso):
        for l in range(n_l):
            _w(dipole_path(root, sim_date, sim_index, scan, k, l), dipole[l, k], np.complex128)
    if E is not None:
        _w(os.path.join(root, f"{sim_date:08d}", f"{sim_index:05d}", f"timeDependent/field/E{scan:03d}.bin"),
           E, np.float64)
