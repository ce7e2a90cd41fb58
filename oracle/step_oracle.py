"""CPU oracle: FP64 NumPy restatement of the reference's split-operator time loop.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``ggbtddft_b200``) imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, as
the checker.  It restates, operation by operation and in the same order, the reference's

* ``src/subFunctions/timePropagation/h_timePropagation.cuh:32-114``  step driver
* ``.../lengthGauge/couplingP.cuh:1-240``  P and FP couplings (rotate, phase, rotate back)
* ``.../lengthGauge/couplingD.cuh:1-114``  D coupling, ``couplingF.cuh:1-114`` FF coupling
* ``.../lengthGauge/couplingS.cuh:1-57``   l-diagonal phase
* ``src/subFunctions/timePropagation/h_timePropagation.cuh:1-30`` radial ZGEMM (column-major A)
* ``src/subFunctions/potentials/hartree/hartreePotentialDensity.cuh:1-222``  density multipoles
* ``src/subFunctions/potentials/hartree/h_calculateHartreePotential.cuh:1-136``  O(N_r^2) sum
* ``src/subFunctions/potentials/exchangeCorrelation/h_calculateExchangeCorrelationPotential.cuh``
* ``src/subFunctions/timePropagation/observables/dipoleMoment.cuh``, ``dipoleAcceleration.cuh``

Parity pin: this restatement is checked against the reference binary (``main.cu`` built for
sm_100a from the reference's own sources by ``oracle/build_ref.py``) on identical workingData;
the resulting dipole files are committed as golden fixtures under ``tests/golden/``.

Options beyond the reference (off by default, so the default reproduces the reference):
``xc_correlation`` (adds PW92 correlation to the TD exchange potential), ``xc_frozen`` (keeps the
exchange(-correlation) potential at its t = 0 value while the Hartree multipoles follow the density),
the ``norm`` output, and
``angular = "theta"``: the angular half-step as one diagonal phase at the Gauss nodes of the dipole
coupling (the eigenbasis of the reference's P coupling, couplingP.cuh:1-125), holding the laser term
and the Hartree potential of the multipoles L = 0 .. n_har - 1 (n_har up to 2 l_max + 1) with the
exchange(-correlation) change -- see ``OracleState.step_theta``.  With n_har <= 4 its multipoles are
the reference's l-space sums; beyond, exact Gauss-Legendre quadratures of the density on 2 N_l nodes.  The reference's truncation of every pointwise launch to
multiples of 32 (e.g. ``couplingP.cuh:117``) is NOT reproduced: full ranges are used, which
equals the reference whenever N_r and N_l are multiples of 32.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional

import numpy as np

# ---------------------------------------------------------------------------------------------
# angular coefficients (angularCoefficients.cuh:1-174) -- restated here so the oracle does not
# depend on the product package
# ---------------------------------------------------------------------------------------------


def _f(l, m):
    return np.asarray(l, dtype=np.float64), np.asarray(m, dtype=np.float64)


def c_u(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l + 3.0)))
    return np.where((l >= 0) & (l >= m), v, 0.0)


def c_d(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = np.sqrt((np.power(l, 2.0) - np.power(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l - 1.0)))
    return np.where((l >= 1) & (l - 1 >= m), v, 0.0)


def p_lm(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = (l * (l + 1.0) - 3.0 * np.power(m, 2.0)) / ((2.0 * l - 1.0) * (2.0 * l + 3.0))
    return np.where((m <= l) & (l >= 1), v, 0.0)


def q_u(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = 1.50 / (2.0 * l + 3.0) * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0))
                                             * (np.power(l + 2.0, 2.0) - np.power(m, 2.0))
                                             / ((2.0 * l + 1.0) * (2.0 * l + 5.0)))
    return np.where((m <= l) & (l >= 0), v, 0.0)


def q_d(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = 1.50 / (2.0 * l - 1.0) * np.sqrt((np.power(l, 2.0) - np.power(m, 2.0))
                                             * (np.power(l - 1.0, 2.0) - np.power(m, 2.0))
                                             / ((2.0 * l + 1.0) * (2.0 * l - 3.0)))
    return np.where((m <= l - 2) & (l >= 2), v, 0.0)


def p3lm(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = (1.50 * (l * (l + 2.0) - 5.0 * np.power(m, 2.0)) / (2.0 * l - 1.0) / (2.0 * l + 5.0)
             * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 3.0)))
    return np.where(l >= m, v, 0.0)


def f3lm(l, m):
    l, m = _f(l, m)
    with np.errstate(all="ignore"):
        v = (2.50 / (2.0 * l + 3.0) / (2.0 * l + 5.0)
             * np.sqrt((np.power(l + 1.0, 2.0) - np.power(m, 2.0)) * (np.power(l + 2.0, 2.0) - np.power(m, 2.0))
                       * (np.power(l + 3.0, 2.0) - np.power(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 7.0)))
    return np.where(l >= m, v, 0.0)


# ---------------------------------------------------------------------------------------------
# problem definition
# ---------------------------------------------------------------------------------------------

@dataclasses.dataclass
class OracleProblem:
    """Everything one reference run reads: params.cuh scalars + workingData arrays + E(t)."""

    r: np.ndarray            # [N_r]
    drdx: np.ndarray         # [N_r]
    P: np.ndarray            # [N_r]  P_{N_g}(x)
    W: np.ndarray            # [N_l, N_r, N_r] complex, file layout W[l][a][b]
    V: Dict[str, np.ndarray]  # coupling -> [N_m, N_l, N_l]   V[m][l][j]
    D: Dict[str, np.ndarray]  # coupling -> [N_m, N_l]
    x0: np.ndarray           # [N_l, N_kso, N_r] complex initial orbitals (already zeroed off l_active)
    m: np.ndarray            # [N_kso] int
    occ: np.ndarray          # [N_kso] int
    rho_frozen: np.ndarray   # [N_r]
    E: np.ndarray            # [N_t]
    dt: float
    n_har: int = 4
    use_hartree: int = 1
    target_id: int = 0
    # options beyond the reference (defaults reproduce it)
    xc_correlation: bool = False
    xc_frozen: bool = False          # exchange(-correlation) potential held at its t = 0 value
    angular: str = "reference"      # "reference" | "theta"

    @property
    def n_r(self):
        return self.r.size

    @property
    def n_l(self):
        return self.x0.shape[0]

    @property
    def n_kso(self):
        return self.x0.shape[1]

    @property
    def n_g(self):
        return self.n_r + 1


# ---------------------------------------------------------------------------------------------
# operators
# ---------------------------------------------------------------------------------------------

def _coupling(x, prob: OracleProblem, name: str, eta_r: Optional[np.ndarray]):
    """rotate -> phase -> rotate back, per orbital (couplingP.cuh:1-125 and twins).

    xROT[j] = sum_{l>=m} V[m][l][j] x[l]  (j >= m, else 0)         d_rotateL?1
    xROT[j] *= exp(-i eta(r) dt/2 D[m][j])   (j >= m)              d_propagateL?
    x[l]    = sum_{j>=m} V[m][l][j] xROT[j]  (l >= m, else 0)      d_rotateL?2
    ``eta_r`` = None means the phase kernel leaves xROT unchanged (e.g. FP without Hartree).
    """
    V = prob.V[name]
    D = prob.D[name]
    out = np.zeros_like(x)
    # the orbitals that share m share V, D and the phase: one product for all of them
    for m in sorted(set(int(v) for v in prob.m)):
        ks = [k for k in range(prob.n_kso) if int(prob.m[k]) == m]
        Vm = V[m][m:, m:]
        xm = x[m:][:, ks, :].reshape(prob.n_l - m, len(ks) * prob.n_r)
        xr = (Vm.T @ xm).reshape(prob.n_l - m, len(ks), prob.n_r)
        if eta_r is not None:
            eta = (eta_r[None, :] * ((0.5 * prob.dt) * D[m, m:])[:, None])[:, None, :]
            xr = (np.cos(eta) * xr.real + np.sin(eta) * xr.imag) + 1j * (np.cos(eta) * xr.imag - np.sin(eta) * xr.real)
        y = (Vm @ xr.reshape(prob.n_l - m, len(ks) * prob.n_r)).reshape(prob.n_l - m, len(ks), prob.n_r)
        out[m:, ks, :] = y
    return out


def legendre_table(x: np.ndarray, n: int) -> np.ndarray:
    """P_L(x) for L = 0 .. n-1 (rows), by the three-term recurrence (L+1) P_{L+1} = (2L+1) x P_L - L P_{L-1}."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((max(n, 1),) + x.shape)
    out[0] = 1.0
    if n > 1:
        out[1] = x
    for L in range(1, n - 1):
        out[L + 1] = ((2.0 * L + 1.0) * x * out[L] - L * out[L - 1]) / (L + 1.0)
    return out[:n]


def assoc_legendre_normalised(x: np.ndarray, n_l: int, m: int) -> np.ndarray:
    """Theta_l(x) for l = 0 .. n_l-1 (rows; zero for l < m): the associated Legendre functions of order
    m normalised to int_{-1}^{1} Theta_l^2 dx = 1, with the signs fixed by the recurrence of the
    dipole coupling, x Theta_l = c_u(l, m) Theta_{l+1} + c_d(l, m) Theta_{l-1} (angularCoefficients.cuh),
    so that an orbital's coefficients x_l are the coefficients of sum_l x_l Theta_l(cos theta)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((n_l,) + x.shape)
    if m >= n_l:
        return out
    # Theta_m = C (1 - x^2)^(m/2), C^2 = (2m+1)! / (2^(2m+1) (m!)^2), built as a product to stay finite
    c2 = 0.5
    for k in range(1, m + 1):
        c2 *= (2.0 * k + 1.0) * (2.0 * k) / (4.0 * k * k)
    out[m] = np.sqrt(c2) * np.power(1.0 - x * x, 0.5 * m)
    if m + 1 < n_l:
        out[m + 1] = x * out[m] / c_u(m, m)
    for l in range(m + 1, n_l - 1):
        out[l + 1] = (x * out[l] - c_d(l, m) * out[l - 1]) / c_u(l, m)
    return out


def hartree_multipoles_scaled(r: np.ndarray, dens: np.ndarray) -> np.ndarray:
    """v_L(r_a) = sum_b rho_L(b) r_<^L / r_>^(L+1) for every row L of ``dens``, evaluated as
    sum_b rho_L(b) (r_< / r_>)^L / r_> so that no power of r over- or underflows for large L
    (the reference's direct sum, h_calculateHartreePotential.cuh:22-51, extended past L = 3)."""
    rmax = np.maximum(r[:, None], r[None, :])
    ratio = np.minimum(r[:, None], r[None, :]) / rmax
    k = 1.0 / rmax
    v = np.zeros_like(dens)
    for L in range(dens.shape[0]):
        v[L] = k @ dens[L]
        k = k * ratio
    return v


class OracleState:
    def __init__(self, prob: OracleProblem):
        self.p = prob
        self.x = prob.x0.astype(np.complex128).copy()
        n_r = prob.n_r
        # hartree.d_v (real part), zeroed at set-up.  At least 4 rows: with N_har = 3 the reference's
        # FP phase reads d_v row 3 past the end of its N_har*N_r allocation; here that row is 0.
        self.v = np.zeros((max(prob.n_har, 4), n_r))
        self.v0 = np.zeros(n_r)
        self.vexc = np.zeros(n_r)
        self.vexc0 = np.zeros(n_r)
        self.density = np.zeros((max(prob.n_har, 4), n_r))
        self.density0 = np.zeros(n_r)
        self.hartree_on = bool(prob.use_hartree == 1 and prob.target_id > 0)
        l_idx = np.arange(prob.n_l)
        self._cu = np.stack([c_u(l_idx, mm) for mm in prob.m])     # [kso, l]
        self._cd = np.stack([c_d(l_idx, mm) for mm in prob.m])
        self._p = np.stack([p_lm(l_idx, mm) for mm in prob.m])
        self.theta = prob.angular == "theta"
        if self.theta:
            # Legendre values at each m's Gauss nodes (the P coupling's eigenvalues, j >= m):
            # pl[m][L][j] = P_L(D_P[m][j])
            n_m = int(np.max(prob.m)) + 1
            self.pl = np.stack([legendre_table(prob.D["P"][mm], max(prob.n_har, 1)) for mm in range(n_m)])
            self.htab = np.zeros((n_m, prob.n_l, n_r))     # H_m(r, j) as [m][j][r]
            if prob.n_har > 4:
                # exact multipoles: Gauss-Legendre quadrature on 2 N_l nodes (degree 4 l_max + 3 >= the
                # l + l' + L <= 4 l_max of every term)
                xq, wq = np.polynomial.legendre.leggauss(2 * prob.n_l)
                self.fine_t = np.stack([assoc_legendre_normalised(xq, prob.n_l, mm).T for mm in range(n_m)])
                self.fine_pw = legendre_table(xq, prob.n_har) * wq[None, :]      # [L][q]

    # ----- potentials -----
    def density_multipoles(self, x):
        """d_getHartreePotentialDensity (hartreePotentialDensity.cuh:1-181): the l ranges and
        coefficients of density_multipoles_literal, each range summed as one array expression."""
        p = self.p
        n_l = p.n_l
        out = np.zeros((max(p.n_har, 1), p.n_r))

        def xx(a, b, k):
            """x_a . x_b (real part of conj(x_b) x_a) for index arrays a, b; 0 where out of range."""
            a, b = np.atleast_1d(a), np.atleast_1d(b)
            ok = (a >= 0) & (a < n_l) & (b >= 0) & (b < n_l)
            ac, bc = np.where(ok, a, 0), np.where(ok, b, 0)
            v = x[ac, k].real * x[bc, k].real + x[ac, k].imag * x[bc, k].imag
            return np.where(ok[:, None], v, 0.0)

        def rng(lo, hi):
            return np.arange(lo, hi) if hi > lo else np.zeros(0, dtype=int)

        def term(c, a, b, k):
            """sum over the range of c[:, None] * xx(a, b)"""
            if np.size(a) == 0:
                return 0.0
            return (np.asarray(c, dtype=np.float64)[:, None] * xx(a, b, k)).sum(axis=0)

        for L in range(p.n_har):
            tot = np.zeros(p.n_r)
            for k in range(p.n_kso):
                m = int(p.m[k])
                d = np.zeros(p.n_r)
                if L == 0:
                    d += (x[m:, k].real ** 2 + x[m:, k].imag ** 2).sum(axis=0)
                elif L == 1:
                    lp = rng(m + 1, n_l - 1)
                    d += term(c_u(np.array([m]), m), [m + 1], [m], k)
                    d += term(c_u(lp, m), lp + 1, lp, k) + term(c_d(lp, m), lp - 1, lp, k)
                    d += term(c_d(np.array([n_l - 1]), m), [n_l - 2], [n_l - 1], k)
                elif L == 2:
                    lp = rng(m, m + 2)
                    d += term(q_u(lp, m), lp + 2, lp, k) + term(p_lm(lp, m), lp, lp, k)
                    lp = rng(m + 2, n_l - 2)
                    d += (term(q_u(lp, m), lp + 2, lp, k) + term(q_d(lp, m), lp - 2, lp, k)
                          + term(p_lm(lp, m), lp, lp, k))
                    lp = rng(n_l - 2, n_l)
                    d += term(q_d(lp, m), lp - 2, lp, k) + term(p_lm(lp, m), lp, lp, k)
                elif L == 3:
                    d += term(p3lm(np.array([m]), m), [m + 1], [m], k) + term(f3lm(np.array([m]), m), [m + 3], [m], k)
                    lp = rng(m + 1, m + 3)
                    d += (term(p3lm(lp - 1, m), lp - 1, lp, k) + term(p3lm(lp, m), lp + 1, lp, k)
                          + term(f3lm(lp, m), lp + 3, lp, k))
                    lp = rng(m + 3, n_l - 3)
                    d += (term(f3lm(lp - 3, m), lp - 3, lp, k) + term(p3lm(lp - 1, m), lp - 1, lp, k)
                          + term(p3lm(lp, m), lp + 1, lp, k) + term(f3lm(lp, m), lp + 3, lp, k))
                    # the reference's tail loop starts at N_l-4 again (hartreePotentialDensity.cuh:150)
                    lp = rng(n_l - 4, n_l - 1)
                    d += (term(f3lm(lp - 3, m), lp - 3, lp, k) + term(p3lm(lp - 1, m), lp - 1, lp, k)
                          + term(p3lm(lp, m), lp + 1, lp, k))
                    lp = np.array([n_l - 1])
                    d += term(f3lm(lp - 3, m), lp - 3, lp, k) + term(p3lm(lp - 1, m), lp - 1, lp, k)
                tot += float(p.occ[k]) * d
            out[L] = tot
        return out

    def density_multipoles_literal(self, x):
        """d_getHartreePotentialDensity (hartreePotentialDensity.cuh:1-181), literal l ranges."""
        p = self.p
        n_l = p.n_l
        out = np.zeros((max(p.n_har, 1), p.n_r))

        def xx(a, b, k):
            if a < 0 or a >= n_l or b < 0 or b >= n_l:
                return 0.0
            return x[a, k].real * x[b, k].real + x[a, k].imag * x[b, k].imag

        for L in range(p.n_har):
            tot = np.zeros(p.n_r)
            for k in range(p.n_kso):
                m = int(p.m[k])
                d = np.zeros(p.n_r)
                if L == 0:
                    for lp in range(m, n_l):
                        d += np.power(x[lp, k].real, 2.0) + np.power(x[lp, k].imag, 2.0)
                elif L == 1:
                    lp = m
                    d += c_u(lp, m) * xx(lp + 1, lp, k)
                    for lp in range(m + 1, n_l - 1):
                        d += c_u(lp, m) * xx(lp + 1, lp, k) + c_d(lp, m) * xx(lp - 1, lp, k)
                    lp = n_l - 1
                    d += c_d(lp, m) * xx(lp - 1, lp, k)
                elif L == 2:
                    for lp in range(m, m + 2):
                        d += q_u(lp, m) * xx(lp + 2, lp, k) + p_lm(lp, m) * xx(lp, lp, k)
                    for lp in range(m + 2, n_l - 2):
                        d += (q_u(lp, m) * xx(lp + 2, lp, k) + q_d(lp, m) * xx(lp - 2, lp, k)
                              + p_lm(lp, m) * xx(lp, lp, k))
                    for lp in range(n_l - 2, n_l):
                        d += q_d(lp, m) * xx(lp - 2, lp, k) + p_lm(lp, m) * xx(lp, lp, k)
                elif L == 3:
                    lp = m
                    d += p3lm(lp, m) * xx(lp + 1, lp, k) + f3lm(lp, m) * xx(lp + 3, lp, k)
                    for lp in range(m + 1, m + 3):
                        d += (p3lm(lp - 1, m) * xx(lp - 1, lp, k) + p3lm(lp, m) * xx(lp + 1, lp, k)
                              + f3lm(lp, m) * xx(lp + 3, lp, k))
                    for lp in range(m + 3, n_l - 3):
                        d += (f3lm(lp - 3, m) * xx(lp - 3, lp, k) + p3lm(lp - 1, m) * xx(lp - 1, lp, k)
                              + p3lm(lp, m) * xx(lp + 1, lp, k) + f3lm(lp, m) * xx(lp + 3, lp, k))
                    # the reference's tail loop starts at N_l-4 again (hartreePotentialDensity.cuh:150)
                    for lp in range(n_l - 4, n_l - 1):
                        d += (f3lm(lp - 3, m) * xx(lp - 3, lp, k) + p3lm(lp - 1, m) * xx(lp - 1, lp, k)
                              + p3lm(lp, m) * xx(lp + 1, lp, k))
                    lp = n_l - 1
                    d += f3lm(lp - 3, m) * xx(lp - 3, lp, k) + p3lm(lp - 1, m) * xx(lp - 1, lp, k)
                tot += float(p.occ[k]) * d
            out[L] = tot
        return out

    def hartree_from_density(self, dens):
        """d_calculateHartreePotential (h_calculateHartreePotential.cuh:1-56): direct O(N_r^2) sum."""
        p = self.p
        r = p.r
        rmax = np.maximum(r[:, None], r[None, :])   # [a, b]
        rmin = np.minimum(r[:, None], r[None, :])
        v = np.zeros_like(dens)
        for L in range(dens.shape[0]):
            if L == 0:
                v[L] = (dens[0][None, :] / rmax).sum(axis=1)
            elif L <= 3:
                v[L] = (dens[L][None, :] * np.power(rmin, float(L)) / np.power(rmax, float(L + 1))).sum(axis=1)
        return v

    def exchange(self, rho0, clamp):
        """d_exchangePotential[0] (h_calculateExchangeCorrelationPotential.cuh:1-45)."""
        p = self.p
        if clamp and p.xc_frozen:
            return self.vexc0.copy()
        dens = p.n_g * (p.n_g + 1) / 2.0 * (rho0 / 4.0 / np.pi + p.rho_frozen) / p.drdx * np.power(p.P, 2.0)
        if clamp:
            dens = np.maximum(dens, 0.0)
        vx = -np.cbrt(3.0 / np.pi * dens) / np.power(p.r, 2.0 / 3.0)
        if p.xc_correlation:
            n = dens / np.power(p.r, 2.0)
            vx = vx + _pw92(n)
        return vx

    # ----- theta mode -----
    def nodal_density(self, x):
        """rho_m(r, j) = sum over the orbitals with m of occ |(V_P,m^T x)_j(r)|^2: the density at the
        Gauss nodes of each m ([n_m][N_l][N_r]; rows j < m are zero)."""
        p = self.p
        n_m = self.pl.shape[0]
        out = np.zeros((n_m, p.n_l, p.n_r))
        V = p.V["P"]
        for k in range(p.n_kso):
            m = int(p.m[k])
            y = V[m][m:, m:].T @ x[m:, k, :]
            out[m, m:] += float(p.occ[k]) * (y.real ** 2 + y.imag ** 2)
        return out

    def theta_multipoles(self, x):
        """rho_L(r) = sum_m sum_j rho_m(r, j) P_L(x_j^m), L = 0 .. n_har-1: the quadrature of each m's
        density over its own N_l - m nodes.  Exact for L <= 1 only (for larger L the top multipoles
        alias by several per cent): a check, not what the theta form uses."""
        nd = self.nodal_density(x)
        return np.einsum("mlj,mjr->lr", self.pl, nd)

    def fine_multipoles(self, x):
        """rho_L(r) = sum_k occ_k int |sum_l x_l Theta_l^(m_k)(t)|^2 P_L(t) dt for L = 0 .. n_har-1, by
        Gauss-Legendre quadrature on 2 N_l nodes, exact for every L <= 2 l_max."""
        p = self.p
        rho_q = np.zeros((self.fine_pw.shape[1], p.n_r))
        for k in range(p.n_kso):
            f = self.fine_t[int(p.m[k])] @ x[:, k, :]            # [q][r]
            rho_q += float(p.occ[k]) * (f.real ** 2 + f.imag ** 2)
        return self.fine_pw @ rho_q

    def theta_density(self, x):
        """The theta form's multipoles: the reference's l-space sums for n_har <= 4, else exact."""
        if self.p.n_har <= 4:
            return self.density_multipoles(x)
        return self.fine_multipoles(x)

    def theta_hartree(self, dens):
        if self.p.n_har <= 4:
            return self.hartree_from_density(dens)
        return hartree_multipoles_scaled(self.p.r, dens)

    def theta_table(self):
        """H_m(r, j) = sum_{L>=1} v_L(r) P_L(x_j^m) + (v_0 - v_0^(0)) + (vxc - vxc^(0)): the potential
        change since t = 0 at the nodes (the ground state's spherical potential is inside W)."""
        s_r = self.v[0] - self.v0 + self.vexc - self.vexc0
        h = np.einsum("lr,mlj->mjr", self.v[1:], self.pl[:, 1:, :]) + s_r[None, None, :]
        for mm in range(h.shape[0]):
            h[mm, :mm] = 0.0
        self.htab = h

    def init_potentials(self):
        """h_timePropagation.cuh:47-57: Hartree0, XC0, Hartree, XC."""
        if self.theta:
            if self.hartree_on:
                self.density0 = self.theta_density(self.x)[0]
                self.v0 = self.theta_hartree(self.density0[None, :])[0]
            self.vexc0 = self.exchange(self.density0, clamp=False)
            self.update_potentials()
            return
        if self.hartree_on:
            self.density0 = self.density_multipoles(self.x)[0]
            self.v0 = self.hartree_from_density(self.density0[None, :])[0]
        self.vexc0 = self.exchange(self.density0, clamp=False)
        self.update_potentials()

    def update_potentials(self):
        if self.theta:
            if self.hartree_on:
                dens = self.theta_density(self.x)
                self.density = dens
                self.v = self.theta_hartree(dens)
                self.vexc = self.exchange(dens[0], clamp=True)
                self.theta_table()
            return
        if self.hartree_on:
            dens = self.density_multipoles(self.x)
            self.density[:dens.shape[0]] = dens
            self.v[:dens.shape[0]] = self.hartree_from_density(dens)
        self.vexc = self.exchange(self.density[0], clamp=True)

    # ----- observables -----
    def observables(self):
        """dipoleMoment.cuh:1-75 and dipoleAcceleration.cuh:1-71 (per l, per orbital), plus norm."""
        p = self.p
        x = self.x
        r = p.r
        n_l = p.n_l
        dip = np.zeros((n_l, p.n_kso), dtype=np.complex128)
        acc = np.zeros((n_l, p.n_kso), dtype=np.complex128)
        # sum of |terms| of each inner product: the scale that rounding errors of any summation
        # order (including the reference's cublasZdotc) are proportional to
        dip_scale = np.zeros((n_l, p.n_kso))
        acc_scale = np.zeros((n_l, p.n_kso))
        fr2 = np.power(r, -2.0)
        for k in range(p.n_kso):
            m = int(p.m[k])
            for l in range(n_l):
                if l < m:
                    continue
                cu = c_u(l, m)
                cd = c_d(l, m)
                if l == m:
                    z1 = r * cu * x[l + 1, k]
                    z2 = fr2 * cu * x[l + 1, k]
                elif l == n_l - 1:
                    z1 = r * cd * x[l - 1, k]
                    z2 = fr2 * cd * x[l - 1, k]
                else:
                    z1 = r * cu * x[l + 1, k] + r * cd * x[l - 1, k]
                    z2 = fr2 * (cu * x[l + 1, k] + cd * x[l - 1, k])
                dip[l, k] = np.vdot(x[l, k], z1)
                acc[l, k] = np.vdot(x[l, k], z2)
                dip_scale[l, k] = np.sum(np.abs(x[l, k]) * np.abs(z1))
                acc_scale[l, k] = np.sum(np.abs(x[l, k]) * np.abs(z2))
        norm = (np.abs(x) ** 2).sum(axis=(0, 2))
        self.last_scales = (dip_scale, acc_scale)
        return dip, acc, norm

    # ----- one step -----
    def _theta_half(self, x, E):
        """x <- V_P,m diag(exp(-i dt/2 (r E x_j + H_m(r, j)))) V_P,m^T x for every orbital (the P
        coupling of couplingP.cuh:1-125 with the whole angular potential in its phase)."""
        p = self.p
        V, D = p.V["P"], p.D["P"]
        out = np.zeros_like(x)
        for m in sorted(set(int(v) for v in p.m)):
            ks = [k for k in range(p.n_kso) if int(p.m[k]) == m]
            Vm = V[m][m:, m:]
            xm = x[m:][:, ks, :].reshape(p.n_l - m, len(ks) * p.n_r)
            xr = (Vm.T @ xm).reshape(p.n_l - m, len(ks), p.n_r)
            eta = ((p.r[None, :] * E) * D[m, m:][:, None] + (self.htab[m, m:] if self.hartree_on else 0.0))
            eta = (eta * (0.5 * p.dt))[:, None, :]
            xr = (np.cos(eta) * xr.real + np.sin(eta) * xr.imag) + 1j * (np.cos(eta) * xr.imag - np.sin(eta) * xr.real)
            out[m:, ks, :] = (Vm @ xr.reshape(p.n_l - m, len(ks) * p.n_r)).reshape(p.n_l - m, len(ks), p.n_r)
        return out

    def step_theta(self, tdx: int):
        """One step of the theta form: angular half, radial product, angular half (the reference's
        order, h_timePropagation.cuh:59-107, with the FF/FP/D/P/S couplings replaced by one diagonal
        phase at the nodes), then the potentials of the new orbitals (lagging one step, as there)."""
        E = self.p.E[tdx]
        x = self._theta_half(self.x, E)
        x = np.matmul(x, self.p.W)
        self.x = self._theta_half(x, E)
        self.update_potentials()
        return self.observables()

    def step(self, tdx: int):
        """One pass of the tdx loop body (h_timePropagation.cuh:59-107)."""
        if self.theta:
            return self.step_theta(tdx)
        p = self.p
        h = self.hartree_on
        E = p.E[tdx]
        r = p.r
        x = self.x
        use_d = p.n_har >= 3 and p.target_id > 0          # couplingD.cuh:103
        use_ff = p.n_har >= 4 and p.target_id > 0         # couplingF.cuh:103
        fp_phase = p.use_hartree == 1 and p.n_har >= 3 and p.target_id > 0   # couplingP.cuh:148
        s_on = p.n_har >= 3 and h                         # couplingS.cuh:18,49

        if p.use_hartree == 1 and p.n_har > 1 and p.target_id > 0:      # couplingP.cuh:83-97
            eta_p = r * E + self.v[1]
        else:
            eta_p = r * E

        def cP(x):
            return _coupling(x, p, "P", eta_p)

        def cFP(x):
            # the FP rotations run even when the phase is off (h_timePropagation.cuh:65,89)
            return _coupling(x, p, "FP", self.v[3] if fp_phase else None)

        def cD(x):
            return _coupling(x, p, "D", self.v[2]) if use_d else x

        def cFF(x):
            return _coupling(x, p, "FF", self.v[3]) if use_ff else x

        def cS(x):
            if not s_on:
                return x
            eta = (self.v[0] - self.v0 + self.vexc - self.vexc0)[None, None, :] \
                + self._p.T[:, :, None] * self.v[2][None, None, :]
            eta = eta * (0.5 * p.dt)                     # [l, kso, r]
            return (np.cos(eta) * x.real + np.sin(eta) * x.imag) + 1j * (np.cos(eta) * x.imag - np.sin(eta) * x.real)

        x = cFF(x)
        x = cFP(x)
        x = cD(x)
        x = cP(x)
        x = cS(x)
        # h_propagationH0: cublasZgemmBatched, A column-major => x_l <- W_l^T x_l (W is complex-symmetric):
        # out[l][k][a] = sum_b W[l][b][a] x[l][k][b], one BLAS product per l
        x = np.matmul(x, p.W)
        x = cS(x)
        x = cP(x)
        x = cD(x)
        x = cFP(x)
        x = cFF(x)
        self.x = x
        self.update_potentials()
        return self.observables()


def _pw92(n):
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


def propagate(prob: OracleProblem, n_steps: Optional[int] = None):
    """Run the reference time loop for ``n_steps`` steps (default N_t); return the time series.

    Returns a dict with ``dipole`` and ``acceleration`` [N_l, N_kso, n_steps] complex (the
    reference's h_dipoleMoment[l][kso][t] layout), their conditioning scales (sum of |terms| of
    each inner product), ``norm`` [N_kso, n_steps], the final orbitals ``x`` [N_l, N_kso, N_r]
    and the final potentials.
    """
    st = OracleState(prob)
    st.init_potentials()
    n = prob.E.size if n_steps is None else n_steps
    dip = np.zeros((prob.n_l, prob.n_kso, n), dtype=np.complex128)
    acc = np.zeros_like(dip)
    norm = np.zeros((prob.n_kso, n))
    dscale = np.zeros((prob.n_l, prob.n_kso, n))
    ascale = np.zeros_like(dscale)
    for t in range(n):
        d, a, nm = st.step(t)
        dip[:, :, t] = d
        acc[:, :, t] = a
        norm[:, t] = nm
        dscale[:, :, t], ascale[:, :, t] = st.last_scales
    return dict(dipole=dip, acceleration=acc, norm=norm, x=st.x, v=st.v, vexc=st.vexc,
                v0=st.v0, vexc0=st.vexc0, density=st.density, dipole_scale=dscale,
                acceleration_scale=ascale)
