"""Input producers for the split-operator time step (host side, FP64, one-time set-up).

These build the arrays that the reference's pre-processor ``src/scripts/init.py``
writes into ``workingData`` before ``main.cu`` runs: the mapped Gauss-Lobatto
radial grid, the complex absorbing potential, the per-l radial Crank-Nicolson
propagators W_l, the angular coupling matrices and their eigen-systems, the
time grid and the laser field.  The formulas restate

* ``src/scripts/phys/internal.py:524-556``  generateGaussLobattoGrid
* ``src/scripts/phys/internal.py:447-497``  getABCR (Manolopoulos CAP, ABC_TYPE=1)
* ``src/scripts/phys/internal.py:232-333``  propagatorsR (CN / EIG, smoothed l>256)
* ``src/scripts/phys/internal.py:88-198``   propagatorsL{P,FP,D,FF} + eigh per m
* ``src/scripts/phys/internal.py:51-86``    angular coefficients c, q, p3lm, f3lm, s2lm
* ``src/scripts/init.py:320``               t = (-N_t/2 .. N_t/2-1) * dt
* ``src/subFunctions/field/h_initialiseField.cuh:1-40``  super-Gaussian field (+ in-situ probe)

None of this runs per time step; the time step itself runs only in the CUDA
library (``ggbtddft_b200/csrc``).
"""
from __future__ import annotations

import dataclasses
import functools
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# Atomic-unit conversions used by the reference's init file (src/params.cuh:16-20).
ATTOSECOND_AU = 4.13413745757510e-02
FEMTOSECOND_AU = 4.13413745758000e01
INTENSITY_AU = 3.50900000000000e16
ELECTRONVOLT_AU = 2.72114000000000e01

COUPLINGS = ("P", "FP", "D", "FF")
# workingData sub-directories of the four angular couplings (src/subFunctions/timePropagation/h_initialisePropagators.cuh:26-117)
COUPLING_DIRS = {"P": "001/001", "FP": "001/003", "D": "002/002", "FF": "003/003"}


# ----------------------------------------------------------------------------------------------
# Legendre polynomials and the Gauss-Lobatto nodes
# ----------------------------------------------------------------------------------------------

def legendre_p_and_dp(n: int, x: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """P_n(x), P_{n-1}(x) and P_n'(x) by the three-term recurrence (|x| < 1)."""
    x = np.asarray(x, dtype=np.float64)
    p0 = np.ones_like(x)
    if n == 0:
        return p0, np.zeros_like(x), np.zeros_like(x)
    p1 = x.copy()
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    dp = n * (x * p1 - p0) / (x * x - 1.0)
    return p1, p0, dp


def lobatto_interior_nodes(n_r: int) -> np.ndarray:
    """The n_r interior Gauss-Lobatto nodes of order N_g = n_r + 1, ascending.

    They are the roots of P'_{N_g}(x); the reference reads them from
    ``workingData/mesh/legendreRoots/roots%05d.txt`` (internal.py:526), which
    ship only for n_r in {32, ..., 1024}.  Newton's method on
    P'_N(x) = 0 with the Chebyshev-Gauss-Lobatto starting points, using
    (1-x^2) P_N''(x) = 2 x P_N'(x) - N (N+1) P_N(x).
    """
    n_g = n_r + 1
    k = np.arange(1, n_g)
    # start from Chebyshev-Gauss-Lobatto points, then polish with Newton
    x = -np.cos(np.pi * k / n_g)
    for _ in range(100):
        p, _, dp = legendre_p_and_dp(n_g, x)
        d2p = (2.0 * x * dp - n_g * (n_g + 1) * p) / (1.0 - x * x)
        dx = dp / d2p
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    return np.sort(x)


@dataclasses.dataclass
class RadialGrid:
    """Mapped Lobatto grid r(x) = R zeta/2 (1+x)/(1-x+zeta) (internal.py:530-556)."""

    n_r: int
    r_max: float
    zeta_ref: float
    x: np.ndarray
    r: np.ndarray
    drdx: np.ndarray
    P: np.ndarray
    T: np.ndarray  # real N_r x N_r second-derivative matrix d_ij / (drdx_i drdx_j)

    @property
    def n_g(self) -> int:
        return self.n_r + 1


def make_grid(n_r: int, r_max: float, zeta_ref: float, x: Optional[np.ndarray] = None) -> RadialGrid:
    """Build the grid exactly as internal.py:524-556 does.

    ``zeta_ref`` is the reference's dimensionless zeta; the physical mapping
    r = zeta (1+x)/(1-x+2 zeta/r_max) of a length zeta maps to zeta_ref = 2 zeta / r_max.
    """
    if x is None:
        x = lobatto_interior_nodes(n_r)
    n_g = n_r + 1
    r = r_max * zeta_ref / 2.0 * (x + 1.0) / (1.0 - x + zeta_ref)
    drdx = r_max * zeta_ref / 2.0 * (2.0 + zeta_ref) / np.power(1.0 - x + zeta_ref, 2.0)
    xi = x[:, None]
    xj = x[None, :]
    with np.errstate(divide="ignore"):
        d = -2.0 / np.power(xi - xj, 2.0)
    np.fill_diagonal(d, -n_g * (n_g + 1.0) / (3.0 * (1.0 - np.power(x, 2.0))))
    T = d / (drdx[:, None] * drdx[None, :])
    P, _, _ = legendre_p_and_dp(n_g, x)
    return RadialGrid(n_r, float(r_max), float(zeta_ref), x, r, drdx, P, T)


def zeta_physical_to_ref(zeta: float, r_max: float) -> float:
    return 2.0 * zeta / r_max


# ----------------------------------------------------------------------------------------------
# Absorbers
# ----------------------------------------------------------------------------------------------

def cap_manolopoulos(r: np.ndarray, r_mask: float, r_max: float) -> np.ndarray:
    """Manolopoulos transmission-free CAP, ABC_TYPE = 1 (internal.py:447-475).  Real, >= 0."""
    n_r = r.size
    w = np.zeros(n_r, dtype=np.float64)
    min_dx = int(np.argmin(np.abs(r - r_mask)))
    rabc = r[min_dx:] - r_mask
    delta = 0.20
    c = 2.62206
    a = 1.0 - 16.0 / c ** 3
    b = (1.0 - 17.0 / c ** 3) / c ** 2
    kmin = c / (delta * 2.0 * (r_max - r_mask))
    emin = 0.5 * kmin ** 2
    x = 2.0 * delta * kmin * rabc
    y = a * x - b * x ** 3 + 4.0 / (c - x) ** 2 - 4.0 / (c + x) ** 2
    w[min_dx:] = emin * y * rabc
    return w


def mask_cos8(r: np.ndarray, r_max: float, width: float) -> np.ndarray:
    """Multiplicative absorbing mask cos^(1/8)(pi/2 (r - r0)/width) over the last ``width`` a.u.

    Not in the reference (which folds a CAP into W); the benchmark configurations use it.
    Applied once per radial step, folded into the radial propagator rows: W' = diag(mask) W.
    """
    r0 = r_max - width
    m = np.ones_like(r)
    sel = r > r0
    arg = 0.5 * np.pi * np.clip((r[sel] - r0) / width, 0.0, 1.0)
    m[sel] = np.power(np.cos(arg), 0.125)
    return m


# ----------------------------------------------------------------------------------------------
# Radial propagators
# ----------------------------------------------------------------------------------------------

def smoother_lr(r: np.ndarray, vmax: float) -> np.ndarray:
    """Smoothed 1/r^2 used for l > 256 (internal.py:222-230)."""
    a = np.exp(1) * vmax
    sig = 1.0 / np.sqrt(vmax)
    vc = np.power(r, -2.0)
    sel = vc > vmax
    vc[sel] = a * np.exp(-np.power(r[sel] / sig, 2.0))
    return vc


def radial_hamiltonian(grid: RadialGrid, l: int, v0: np.ndarray, vscf: np.ndarray,
                       mask_r: np.ndarray) -> np.ndarray:
    """H_l = -T/2 + diag(v0 + l(l+1)/2r^2 - i maskR) + diag(vscf)   (internal.py:249-257).

    ``v0`` may be complex (the reference's v0 = -Z/r - i W already carries the CAP once,
    groundState.py:27, and ``mask_r`` subtracts it a second time, internal.py:253).
    """
    if l <= 256:
        v = v0 + l * (l + 1) / 2.0 / np.power(grid.r, 2.0) - 1j * mask_r
    else:
        v = v0 - 1j * mask_r
    return -0.5 * grid.T.astype(np.complex128) + np.diag(v + vscf)


def radial_propagators(grid: RadialGrid, n_l: int, dt: float, v0: np.ndarray, vscf: np.ndarray,
                       mask_r: np.ndarray, method: str = "CN", row_mask: Optional[np.ndarray] = None,
                       device: Optional[str] = None) -> np.ndarray:
    """W_l = Wp^-1 Wm for l = 0..n_l-1, as the reference's file layout W[l][a][b] (internal.py:232-333).

    CN:  Wm = I - i dt/2 H,  Wp = I + i dt/2 H.
    EIG: Wm = exp(-i dt/2 H), Wp = exp(+i dt/2 H) via the eigen-decomposition.
    ``row_mask`` (optional) multiplies the rows: W' = diag(mask) W (the cos^(1/8) mask mode).
    ``device`` = "cuda" builds the matrices with torch.linalg on the GPU in complex128.
    """
    n_r = grid.n_r
    out = np.empty((n_l, n_r, n_r), dtype=np.complex128)
    if device is not None:
        import torch
        dev = torch.device(device)
        T = torch.from_numpy(grid.T).to(dev, torch.complex128)
        r = torch.from_numpy(grid.r).to(dev)
        eye = torch.eye(n_r, dtype=torch.complex128, device=dev)
        base = torch.from_numpy(np.asarray(v0 + vscf - 1j * mask_r, dtype=np.complex128)).to(dev)
        rm = None if row_mask is None else torch.from_numpy(row_mask).to(dev, torch.complex128)
        cn = [l for l in range(n_l) if l <= 256 and method == "CN"]
        # Crank-Nicolson for every l at once: a batch of N_r x N_r complex128 solves on the device,
        # in chunks that keep ~2 GB of matrices per solve
        chunk = max(1, int(2e9 // (3 * 16 * n_r * n_r)))
        for c0 in range(0, len(cn), chunk):
            ls = torch.tensor(cn[c0:c0 + chunk], dtype=torch.float64, device=dev)
            diag = base[None, :] + (ls * (ls + 1.0) / 2.0)[:, None] / (r ** 2)[None, :]
            H = -0.5 * T[None] + torch.diag_embed(diag)
            W = torch.linalg.solve(eye[None] + 0.5j * dt * H, eye[None] - 0.5j * dt * H)
            if rm is not None:
                W = rm[None, :, None] * W
            out[cn[c0]:cn[c0] + len(ls)] = W.cpu().numpy()
        for l in range(n_l):
            if l not in cn:
                out[l] = _propagator_from_h(radial_hamiltonian(grid, l, v0, vscf, mask_r), dt, method, l,
                                            grid.r, row_mask)
        return out
    for l in range(n_l):
        H = radial_hamiltonian(grid, l, v0, vscf, mask_r)
        out[l] = _propagator_from_h(H, dt, method, l, grid.r, row_mask)
    return out


def _propagator_from_h(H: np.ndarray, dt: float, method: str, l: int, r: np.ndarray,
                       row_mask: Optional[np.ndarray]) -> np.ndarray:
    n_r = H.shape[0]
    eye = np.eye(n_r)
    if method == "CN":
        Wm = eye - 0.5j * dt * H
        Wp = eye + 0.5j * dt * H
    elif method == "EIG":
        d, v = np.linalg.eig(H)
        vinv = np.linalg.inv(v)
        Wm = v @ np.diag(np.exp(-0.5j * dt * d)) @ vinv
        Wp = v @ np.diag(np.exp(0.5j * dt * d)) @ vinv
    else:
        raise ValueError(f"unknown propagator method {method!r}")
    prop = np.linalg.solve(Wp, Wm)
    if l > 256:
        vc = l * (l + 1) / 2.0 * smoother_lr(r.copy(), 100000.0 / l)
        e = np.exp(-0.5j * dt * vc)
        prop = e[:, None] * prop * e[None, :]
    if row_mask is not None:
        prop = row_mask[:, None] * prop
    return prop


# ----------------------------------------------------------------------------------------------
# Angular coupling coefficients and matrices
# ----------------------------------------------------------------------------------------------
# Closed-form <l m| P_L(cos theta) |l' m> couplings; each restates one __device__ function of
# src/subFunctions/potentials/hartree/angularCoefficients.cuh (and its Python twin in internal.py).

def coef_c(l, m):
    """d_c / d_cu  (angularCoefficients.cuh:57-93, internal.py:80-84)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = (m <= l) & (l >= 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l + 3.0)))
    return np.where(ok, v, 0.0)


coef_cu = coef_c


def coef_cd(l, m):
    """d_cd (angularCoefficients.cuh:95-111)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = (l >= 1) & (l - 1 >= m)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.sqrt((np.power(l, 2.0) - np.power(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l - 1.0)))
    return np.where(ok, v, 0.0)


def coef_p(l, m):
    """d_p (angularCoefficients.cuh:113-132), = s2lm (internal.py:68-69) for l >= 1."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = (m <= l) & (l >= 1)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = (l * (l + 1.0) - 3.0 * np.power(m, 2.0)) / ((2.0 * l - 1.0) * (2.0 * l + 3.0))
    return np.where(ok, v, 0.0)


def coef_q(l, m):
    """d_q / d_qu (angularCoefficients.cuh:134-166, internal.py:70-78)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = (m <= l) & (l >= 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = 1.50 / (2.0 * l + 3.0) * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0))
                                             * (np.power(l + 2.0, 2.0) - np.power(m, 2.0))
                                             / ((2.0 * l + 1.0) * (2.0 * l + 5.0)))
    return np.where(ok, v, 0.0)


coef_qu = coef_q


def coef_qd(l, m):
    """d_qd (angularCoefficients.cuh:168-174...)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = (m <= l - 2) & (l >= 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        v = 1.50 / (2.0 * l - 1.0) * np.sqrt((np.power(l, 2.0) - np.power(m, 2.0))
                                             * (np.power(l - 1.0, 2.0) - np.power(m, 2.0))
                                             / ((2.0 * l + 1.0) * (2.0 * l - 3.0)))
    return np.where(ok, v, 0.0)


def coef_p3lm(l, m):
    """d_p3lm (angularCoefficients.cuh:1-17, internal.py:58-62)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = l >= m
    with np.errstate(invalid="ignore", divide="ignore"):
        v = (1.50 * (l * (l + 2.0) - 5.0 * np.power(m, 2.0)) / (2.0 * l - 1.0) / (2.0 * l + 5.0)
             * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 3.0)))
    return np.where(ok, v, 0.0)


def coef_f3lm(l, m):
    """d_f3lm (angularCoefficients.cuh:19-35, internal.py:51-55)."""
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    ok = l >= m
    with np.errstate(invalid="ignore", divide="ignore"):
        v = (2.50 / (2.0 * l + 3.0) / (2.0 * l + 5.0)
             * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) * (np.power(l + 2.0, 2.0) - np.power(m, 2.0))
                       * (np.power(l + 3.0, 2.0) - np.power(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 7.0)))
    return np.where(ok, v, 0.0)


def coupling_matrix(coupling: str, n_l: int, m: int) -> np.ndarray:
    """Symmetric banded coupling matrix of one multipole for azimuthal number m (internal.py:88-120)."""
    u = np.zeros((n_l, n_l))
    if coupling == "P":
        k, f = 1, coef_c
    elif coupling == "FP":
        k, f = 1, coef_p3lm
    elif coupling == "D":
        k, f = 2, coef_q
    elif coupling == "FF":
        k, f = 3, coef_f3lm
    else:
        raise ValueError(coupling)
    for l in range(n_l - k):
        u[l, l + k] = f(l, m)
        u[l + k, l] = f(l, m)
    return u


@functools.lru_cache(maxsize=32)
def angular_eigensystems(n_l: int, n_m: int) -> Dict[str, Tuple[np.ndarray, np.ndarray]]:
    """V[m][l][j] and D[m][j] of each coupling, the workingData V%03d/D%03d files (internal.py:122-198).

    For each m the block l, j >= m of the coupling matrix is diagonalised with eigh; rows and
    columns below m are zero.  Cached per (n_l, n_m); the arrays are read-only.
    """
    out = {}
    for c in COUPLINGS:
        V = np.zeros((n_m, n_l, n_l))
        D = np.zeros((n_m, n_l))
        for m in range(n_m):
            L = coupling_matrix(c, n_l, m)
            d, v = np.linalg.eigh(L[m:, m:])
            D[m, m:] = d
            V[m, m:, m:] = v
        V.setflags(write=False)
        D.setflags(write=False)
        out[c] = (V, D)
    return out


def angular_eigensystems_device(n_l: int, n_m: int, device: str = "cuda") -> Dict[str, Tuple[np.ndarray, np.ndarray]]:
    """The same eigensystems with torch.linalg.eigh on ``device`` (FP64), every m of a coupling in one
    batched call: the m blocks l, j >= m are embedded in N_l x N_l matrices whose rows and columns below
    m carry distinct eigenvalues far outside [-1, 1] (2 + index), so that the m block's eigenpairs are the
    N_l - m eigenpairs inside [-1, 1]."""
    import torch
    dev = torch.device(device)
    out = {}
    for c in COUPLINGS:
        mats = np.zeros((n_m, n_l, n_l))
        for m in range(n_m):
            mats[m] = coupling_matrix(c, n_l, m)
            mats[m, :m, :] = 0.0
            mats[m, :, :m] = 0.0
            for k in range(m):
                mats[m, k, k] = 2.0 + k
        d, v = torch.linalg.eigh(torch.from_numpy(mats).to(dev))
        d, v = d.cpu().numpy(), v.cpu().numpy()
        V = np.zeros((n_m, n_l, n_l))
        D = np.zeros((n_m, n_l))
        for m in range(n_m):
            keep = np.argsort(d[m])[:n_l - m]          # the eigenvalues inside [-1, 1], ascending
            D[m, m:] = d[m][keep]
            V[m, m:, m:] = v[m][m:, keep]
        out[c] = (V, D)
    return out


# ----------------------------------------------------------------------------------------------
# Time grid and laser fields
# ----------------------------------------------------------------------------------------------

def time_grid(n_t: int, dt: float) -> np.ndarray:
    """t = linspace(-N_t/2, N_t/2 - 1, N_t) dt (init.py:320)."""
    return np.linspace(-0.5 * n_t, 0.5 * n_t - 1, n_t) * dt


def field_super_gaussian(t: np.ndarray, e0: float, omega0: float, tau0: float, cep0: float,
                         probe_amplitude: float = 0.0, cos_theta: float = 1.0, delay: float = 0.0) -> np.ndarray:
    """E(t) of h_initialiseField.cuh:1-40: E0 exp(-(2t/tau0)^10) cos(w0 t + CEP), plus the in-situ probe."""
    e = e0 * np.exp(-np.power(2.0 * t / tau0, 10.0)) * np.cos(omega0 * t + cep0)
    if probe_amplitude != 0.0:
        tp = t * cos_theta
        e = e + probe_amplitude * e0 * np.exp(-np.power(2.0 * tp / tau0, 10.0)) * np.cos(omega0 * (t + delay) + cep0)
    return e


def field_sin2(n_t: int, dt: float, e0: float, omega0: float, n_cycles: float, cep0: float = 0.0) -> np.ndarray:
    """sin^2-envelope pulse of n_cycles optical cycles sampled at t_k = k dt, k = 0..n_t-1.

    E(t) = E0 sin^2(pi t / T) cos(w0 (t - T/2) + CEP) for 0 <= t <= T = n_cycles 2 pi / w0, 0 after.
    Not in the reference (which uses a super-Gaussian); the benchmark configurations use it.
    """
    t = np.arange(n_t) * dt
    T = n_cycles * 2.0 * np.pi / omega0
    env = np.where(t <= T, np.power(np.sin(np.pi * t / T), 2.0), 0.0)
    return e0 * env * np.cos(omega0 * (t - 0.5 * T) + cep0)


def steps_for_sin2(dt: float, omega0: float, n_cycles: float) -> int:
    return int(math.ceil(n_cycles * 2.0 * np.pi / omega0 / dt))


def intensity_to_e0(intensity_w_cm2: float) -> float:
    return math.sqrt(intensity_w_cm2 / INTENSITY_AU)


def wavelength_to_omega(lambda_nm: float) -> float:
    return 45.5634 / lambda_nm


# ----------------------------------------------------------------------------------------------
# Ground states
# ----------------------------------------------------------------------------------------------

@dataclasses.dataclass
class Orbital:
    n: int
    l: int
    m: int
    occ: int


def bound_states(grid: RadialGrid, l: int, v: np.ndarray, count: int,
                 device: Optional[str] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Lowest ``count`` eigen-pairs of the real radial Hamiltonian -T/2 + v + l(l+1)/2r^2.

    Eigenvectors are the DVR coefficients u_i (sum |u_i|^2 = 1), sign fixed so that the
    largest-magnitude entry is positive.  ``device="cuda"`` diagonalises with torch in FP64.
    """
    H = -0.5 * grid.T + np.diag(v + l * (l + 1) / 2.0 / grid.r ** 2)
    H = 0.5 * (H + H.T)
    if device is not None:
        import torch
        e, u = torch.linalg.eigh(torch.from_numpy(H).to(device))
        e, u = e.cpu().numpy(), u.cpu().numpy()
    else:
        e, u = np.linalg.eigh(H)
    e = e[:count]
    u = u[:, :count]
    for k in range(u.shape[1]):
        if u[np.argmax(np.abs(u[:, k])), k] < 0:
            u[:, k] = -u[:, k]
    return e, u


def lda_exchange(n: np.ndarray) -> np.ndarray:
    """Slater exchange potential v_x = -(3 n / pi)^(1/3)."""
    return -np.cbrt(3.0 / np.pi * np.maximum(n, 0.0))


def pw92_correlation(n: np.ndarray) -> np.ndarray:
    """Perdew-Wang 1992 correlation potential of the unpolarised electron gas.

    e_c(rs) = -2A (1 + a1 rs) ln(1 + 1/(2A (b1 rs^1/2 + b2 rs + b3 rs^3/2 + b4 rs^2)))
    v_c = e_c - (rs/3) de_c/drs, with A=0.031091, a1=0.21370, b=(7.5957, 3.5876, 1.6382, 0.49294)
    (Phys. Rev. B 45, 13244, Table I, p = 1).
    """
    a, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    n = np.maximum(n, 1e-300)
    rs = np.cbrt(3.0 / (4.0 * np.pi * n))
    srs = np.sqrt(rs)
    q0 = -2.0 * a * (1.0 + a1 * rs)
    q1 = 2.0 * a * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs)
    q1p = a * (b1 / srs + 2.0 * b2 + 3.0 * b3 * srs + 4.0 * b4 * rs)
    lg = np.log1p(1.0 / q1)
    ec = q0 * lg
    dec = -2.0 * a * a1 * lg - q0 * q1p / (q1 * q1 + q1)
    return ec - rs / 3.0 * dec


def density_u_to_n(grid: RadialGrid, rho_u: np.ndarray) -> np.ndarray:
    """n(r) = N_g(N_g+1)/2 rho_u/drdx P^2 / r^2 with rho_u already divided by 4 pi.

    The DVR coefficients carry sqrt(w drdx); this undoes it the way the reference's exchange
    kernel does (h_calculateExchangeCorrelationPotential.cuh:33).
    """
    n_g = grid.n_g
    return n_g * (n_g + 1) / 2.0 * rho_u / grid.drdx * np.power(grid.P, 2.0) / np.power(grid.r, 2.0)


def hartree_monopole(grid: RadialGrid, rho0: np.ndarray) -> np.ndarray:
    """v(r_a) = sum_b rho0(b) / max(r_a, r_b)."""
    return (rho0[None, :] / np.maximum(grid.r[:, None], grid.r[None, :])).sum(axis=1)


@dataclasses.dataclass
class GroundState:
    orbitals: List[Orbital]
    u: np.ndarray            # [n_orb, N_r] real DVR coefficients
    energies: np.ndarray     # [n_orb]
    v_ion: np.ndarray        # -Z/r
    vscf: np.ndarray         # v_H + v_xc of the ground state (0 for one-electron atoms)
    rho_frozen: np.ndarray   # frozen-core density (u units, divided by 4 pi); 0 for all-electron runs


def ground_state(grid: RadialGrid, Z: float, orbitals: Sequence[Orbital], interacting: bool,
                 correlation: bool = False, iterations: int = 200, mix: float = 0.3,
                 tol: float = 1e-11, device: Optional[str] = None) -> GroundState:
    """Spherical Kohn-Sham LDA ground state on the grid (Slater exchange, optional PW92).

    The reference obtains its ground state from groundState.py (LDA + LB94 + Chachiyo), which is
    out of this path's scope; this self-consistent loop provides the same kind of input:
    occupied radial orbitals u and the static potential vscf that enters W_l.
    For ``interacting=False`` it diagonalises -T/2 - Z/r once (hydrogen-like).
    With ``device`` (a torch device name) the whole loop runs there (``ground_state_device``).
    """
    if device is not None:
        return ground_state_device(grid, Z, orbitals, interacting, correlation=correlation,
                                   iterations=iterations, mix=mix, tol=tol, device=device)
    v_ion = -Z / grid.r
    ls = sorted({o.l for o in orbitals})
    vscf = np.zeros(grid.n_r)

    def solve(vtot):
        u = np.zeros((len(orbitals), grid.n_r))
        en = np.zeros(len(orbitals))
        for l in ls:
            need = max(o.n - o.l for o in orbitals if o.l == l)
            e, vecs = bound_states(grid, l, vtot, need, device=device)
            for k, o in enumerate(orbitals):
                if o.l == l:
                    u[k] = vecs[:, o.n - o.l - 1]
                    en[k] = e[o.n - o.l - 1]
        return u, en

    u, en = solve(v_ion)
    if interacting:
        occ = np.array([o.occ for o in orbitals], dtype=np.float64)
        for _ in range(iterations):
            rho0 = (occ[:, None] * u ** 2).sum(axis=0)
            n = density_u_to_n(grid, rho0 / (4.0 * np.pi))
            v_new = hartree_monopole(grid, rho0) + lda_exchange(n)
            if correlation:
                v_new = v_new + pw92_correlation(n)
            dv = np.max(np.abs(v_new - vscf))
            vscf = (1.0 - mix) * vscf + mix * v_new
            u, en = solve(v_ion + vscf)
            if dv < tol:
                break
    return GroundState(list(orbitals), u, en, v_ion, vscf, np.zeros(grid.n_r))


def ground_state_device(grid: RadialGrid, Z: float, orbitals: Sequence[Orbital], interacting: bool,
                        correlation: bool = False, iterations: int = 200, mix: float = 0.3,
                        tol: float = 1e-11, device: str = "cuda") -> GroundState:
    """``ground_state`` with every array resident on ``device`` (torch, FP64).

    Per iteration: one batched symmetric eigensolve of the radial Hamiltonians of all occupied l,
    the orbital density, the Hartree monopole v(r_a) = sum_b rho0(b)/max(r_a, r_b), Slater exchange
    and PW92 correlation, linear mixing; one scalar (max |v_new - vscf|, the convergence test) is
    read back per iteration.  Same iteration, mixing and stopping rule as the host loop, so the two
    reach the same fixed point (to the eigensolvers' rounding).
    """
    import torch
    dev = torch.device(device)
    f64 = torch.float64
    r = torch.from_numpy(grid.r).to(dev, f64)
    T = torch.from_numpy(grid.T).to(dev, f64)
    ls = sorted({o.l for o in orbitals})
    lt = torch.tensor(ls, dtype=f64, device=dev)
    cent = lt[:, None] * (lt[:, None] + 1.0) / 2.0 / r[None, :] ** 2          # [n_ls, N_r]
    li = torch.tensor([ls.index(o.l) for o in orbitals], device=dev)
    ki = torch.tensor([o.n - o.l - 1 for o in orbitals], device=dev)
    rows = torch.arange(len(orbitals), device=dev)
    v_ion = -Z / r
    n_g = grid.n_g
    drdx = torch.from_numpy(grid.drdx).to(dev, f64)
    p2 = torch.from_numpy(np.power(grid.P, 2.0)).to(dev, f64)
    r2 = r ** 2
    inv_rmax = 1.0 / torch.maximum(r[:, None], r[None, :])

    def solve(vtot):
        H = -0.5 * T[None] + torch.diag_embed(vtot[None, :] + cent)
        H = 0.5 * (H + H.transpose(1, 2))
        e, U = torch.linalg.eigh(H)
        u = U[li, :, ki]                                       # [n_orb, N_r]
        big = u[rows, u.abs().argmax(dim=1)]
        u = torch.where((big < 0)[:, None], -u, u)
        return u, e[li, ki]

    def xc(n):
        v = -torch.pow(3.0 / math.pi * torch.clamp(n, min=0.0), 1.0 / 3.0)
        if correlation:
            a, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
            nc = torch.clamp(n, min=1e-300)
            rs = torch.pow(3.0 / (4.0 * math.pi * nc), 1.0 / 3.0)
            srs = torch.sqrt(rs)
            q0 = -2.0 * a * (1.0 + a1 * rs)
            q1 = 2.0 * a * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs)
            q1p = a * (b1 / srs + 2.0 * b2 + 3.0 * b3 * srs + 4.0 * b4 * rs)
            lg = torch.log1p(1.0 / q1)
            ec = q0 * lg
            dec = -2.0 * a * a1 * lg - q0 * q1p / (q1 * q1 + q1)
            v = v + (ec - rs / 3.0 * dec)
        return v

    u, en = solve(v_ion)
    vscf = torch.zeros_like(r)
    if interacting:
        occ = torch.tensor([float(o.occ) for o in orbitals], dtype=f64, device=dev)
        for _ in range(iterations):
            rho0 = (occ[:, None] * u ** 2).sum(dim=0)
            n = n_g * (n_g + 1) / 2.0 * (rho0 / (4.0 * math.pi)) / drdx * p2 / r2
            v_new = (rho0[None, :] * inv_rmax).sum(dim=1) + xc(n)
            dv = (v_new - vscf).abs().max()
            vscf = (1.0 - mix) * vscf + mix * v_new
            u, en = solve(v_ion + vscf)
            if float(dv) < tol:
                break
    return GroundState(list(orbitals), u.cpu().numpy(), en.cpu().numpy(), -Z / grid.r,
                       vscf.cpu().numpy(), np.zeros(grid.n_r))


# Orbital sets of the benchmark atoms.  m = -1 is stored as m = 1: the length-gauge couplings of a
# linearly polarised field depend on |m| only (angularCoefficients.cuh uses m^2).
ORBITALS_H = [Orbital(1, 0, 0, 1)]
ORBITALS_HE = [Orbital(1, 0, 0, 2)]
ORBITALS_AR = [Orbital(1, 0, 0, 2), Orbital(2, 0, 0, 2), Orbital(2, 1, 0, 2), Orbital(2, 1, 1, 2),
               Orbital(2, 1, 1, 2), Orbital(3, 0, 0, 2), Orbital(3, 1, 0, 2), Orbital(3, 1, 1, 2),
               Orbital(3, 1, 1, 2)]
