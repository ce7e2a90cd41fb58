"""The oracle's theta form (one diagonal phase at the Gauss nodes, multipoles to 2 l_max) on CPU:
its parts against the reference form's, where they must agree."""
import dataclasses

import numpy as np

from ggbtddft_b200 import problems as P
from oracle.step_oracle import OracleState, hartree_multipoles_scaled, legendre_table, propagate
from tests.helpers import to_oracle


def test_legendre_table_against_numpy():
    x = np.linspace(-1.0, 1.0, 37)
    tab = legendre_table(x, 40)
    for L in (0, 1, 2, 7, 39):
        c = np.zeros(L + 1)
        c[L] = 1.0
        assert np.abs(tab[L] - np.polynomial.legendre.legval(x, c)).max() < 1e-12


def test_scaled_hartree_sum_equals_the_direct_sum_for_low_multipoles():
    run = P.reference_like(64, 16, 4, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=7)
    st = OracleState(to_oracle(run))
    dens = st.density_multipoles(st.x)
    a = st.hartree_from_density(dens)
    b = hartree_multipoles_scaled(run.grid.r, dens)
    for L in range(4):
        assert np.abs(a[L] - b[L]).max() <= 1e-13 * np.abs(a[L]).max()


def test_nodal_monopole_and_dipole_densities_are_exact():
    """At each m's Gauss nodes the quadrature of |psi|^2 P_L is exact for L <= 1: the theta form's
    rho_0 and rho_1 equal the reference's l-space sums."""
    run = P.reference_like(64, 16, 4, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=7)
    ref = OracleState(to_oracle(run))
    ref.init_potentials()
    for t in range(3):                 # orbitals spread over several l by the field
        ref.step(t)
    th = OracleState(dataclasses.replace(to_oracle(run), angular="theta", n_har=31))
    a = ref.density_multipoles(ref.x)
    b = th.theta_multipoles(ref.x)
    assert b.shape == (31, run.n_r)
    assert np.abs(a[1]).max() > 1e-6 * np.abs(a[0]).max()
    for L in range(2):
        assert np.abs(a[L] - b[L]).max() <= 1e-13 * np.abs(a[0]).max()


def test_theta_form_without_hartree_is_the_reference_p_coupling():
    """Hydrogen (no Hartree): the theta form's phase is the laser term alone, at the P coupling's
    eigenvalues -- the reference's chain with its P coupling only."""
    run = P.reference_like(64, 16, 24, "H", r_mask=20.0)
    a = propagate(to_oracle(run))
    b = propagate(dataclasses.replace(to_oracle(run), angular="theta"))
    assert np.abs(a["dipole"] - b["dipole"]).max() <= 1e-12 * np.abs(a["dipole"]).max()
    assert np.abs(a["x"] - b["x"]).max() <= 1e-12 * np.abs(a["x"]).max()


def test_theta_form_converges_to_the_reference_form_with_the_time_step():
    """With the same four multipoles both forms approximate the same equations; their difference is
    the splitting of the angular potential, which falls with dt (second order per unit time)."""
    diffs = []
    for dt_as, n in ((4.0, 40), (2.0, 80)):
        run = P.reference_like(48, 12, n, "Ne3", r_mask=15.0, dt_as=dt_as, perturb=0.05, seed=3)
        a = propagate(to_oracle(run))
        b = propagate(dataclasses.replace(to_oracle(run), angular="theta", n_har=4))
        diffs.append(np.abs(a["x"] - b["x"]).max() / np.abs(a["x"]).max())
    assert diffs[1] < 0.5 * diffs[0], diffs


def test_theta_form_conserves_the_norm_without_absorber_and_field():
    run = P.reference_like(48, 12, 30, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=3)
    prob = dataclasses.replace(to_oracle(run), angular="theta", n_har=23, E=np.zeros(30))
    # a propagator without the CAP: W from the same grid with the absorber off is not at hand here,
    # so compare the norm loss with the reference form's on the same W (the CAP is the only loss)
    a = propagate(dataclasses.replace(to_oracle(run), E=np.zeros(30)))
    b = propagate(prob)
    assert np.abs(a["norm"] - b["norm"]).max() < 1e-6


def _theta_half_parts(st, x, E, start=None):
    """The oracle's theta half-step (OracleState._theta_half) split at the node basis: returns the new
    orbitals and, per m, the node-basis vectors after the phase; ``start`` (a previous half's kept
    vectors) replaces V^T x."""
    p = st.p
    V, D = p.V["P"], p.D["P"]
    out = np.zeros_like(x)
    kept = {}
    for m in sorted(set(int(v) for v in p.m)):
        ks = [k for k in range(p.n_kso) if int(p.m[k]) == m]
        Vm = V[m][m:, m:]
        if start is None:
            xr = (Vm.T @ x[m:][:, ks, :].reshape(p.n_l - m, len(ks) * p.n_r)).reshape(p.n_l - m, len(ks), p.n_r)
        else:
            xr = start[m]
        eta = ((p.r[None, :] * E) * D[m, m:][:, None] + (st.htab[m, m:] if st.hartree_on else 0.0))
        xr = xr * np.exp(-1j * (eta * (0.5 * p.dt))[:, None, :])
        kept[m] = xr
        out[m:, ks, :] = (Vm @ xr.reshape(p.n_l - m, len(ks) * p.n_r)).reshape(p.n_l - m, len(ks), p.n_r)
    return out, kept


def test_basis_reuse_is_exact_in_fp64():
    """The int8 theta form's basis reuse (ggb_set_theta_reuse): each step's first half starts from the
    node-basis vectors the previous second half kept, skipping V^T V.  Nothing acts on the orbitals
    between the halves (the potentials computed there only enter the phase), so with orthogonal V the
    FP64 propagation is unchanged to rounding: an interacting atom with every Hartree and exchange
    phase on, 30 steps (the LDA feedback grows the rounding differences to ~2e-12)."""
    run = dataclasses.replace(P.reference_like(64, 16, 30, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=7),
                              angular="theta")
    prob = to_oracle(run)
    ref = propagate(prob)
    st = OracleState(prob)
    st.init_potentials()
    kept = None
    dip = []
    for t in range(run.n_t):
        E = prob.E[t]
        x, _ = _theta_half_parts(st, st.x, E, start=kept)
        x = np.matmul(x, prob.W)
        st.x, kept = _theta_half_parts(st, x, E)
        st.update_potentials()
        dip.append(st.observables()[0])
    assert st.hartree_on
    assert np.abs(st.x - ref["x"]).max() <= 1e-11 * np.abs(ref["x"]).max()
    d = np.stack(dip, axis=-1)
    assert np.abs(d - ref["dipole"]).max() <= 1e-11 * np.abs(ref["dipole"]).max()
