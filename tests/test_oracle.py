"""The oracle against the reference's own outputs and known-answer properties (CPU only)."""
import os

import numpy as np
import pytest

from ggbtddft_b200 import inputs as I
from ggbtddft_b200 import problems as P
from oracle.step_oracle import propagate
from tests.helpers import GOLDEN, load_ref_case, rel_err, to_oracle


@pytest.mark.parametrize("n", [32, 64, 128, 256, 512, 1024])
def test_lobatto_nodes_match_shipped_roots(n):
    ref = np.load(os.path.join(GOLDEN, "lobatto_roots.npz"))[f"n{n}"]
    assert np.max(np.abs(I.lobatto_interior_nodes(n) - ref)) < 5e-15


@pytest.mark.parametrize("case", ["h64", "ne3_64", "ne3_128", "ar9_256"])
def test_oracle_matches_reference_binary(case):
    """Dipole series of the reference main.cu (sm_100a build, same inputs) vs the oracle."""
    run, dref = load_ref_case(case)
    out = propagate(to_oracle(run))
    assert out["dipole"].shape == dref.shape
    assert rel_err(out["dipole"], dref) < 1e-10
    assert rel_err(out["dipole"].sum(axis=0), dref.sum(axis=0)) < 1e-10


def test_every_reference_case_has_its_fixture_and_its_pin():
    """Every case oracle/build_ref.py builds from the reference's sources has a committed fixture made
    from that binary's outputs, and the oracle test above covers it."""
    from oracle.build_ref import CASES
    pinned = test_oracle_matches_reference_binary.pytestmark[0].args[1]
    for name in CASES:
        assert os.path.exists(os.path.join(GOLDEN, f"ref_{name}.npz")), name
        assert name in pinned, name


def test_p_eigenvalues_are_gauss_legendre_nodes():
    V, D = I.angular_eigensystems(12, 1)["P"]
    nodes, _ = np.polynomial.legendre.leggauss(12)
    assert np.allclose(np.sort(D[0]), np.sort(nodes), atol=1e-14)


@pytest.mark.parametrize("coupling", I.COUPLINGS)
def test_angular_eigenvectors_orthogonal(coupling):
    V, D = I.angular_eigensystems(20, 3)[coupling]
    for m in range(3):
        B = V[m][m:, m:]
        assert np.allclose(B.T @ B, np.eye(20 - m), atol=1e-13)
        assert np.all(V[m][:m] == 0) and np.all(V[m][:, :m] == 0)


def test_radial_propagator_unitary_without_absorber():
    grid = I.make_grid(32, 30.0, 1.0)
    gs = I.ground_state(grid, 1.0, I.ORBITALS_H, interacting=False)
    W = I.radial_propagators(grid, 3, 0.05, gs.v_ion.astype(complex), gs.vscf, np.zeros(32))
    for l in range(3):
        s = np.linalg.svd(W[l], compute_uv=False)
        assert np.allclose(s, 1.0, atol=1e-12)
        assert np.allclose(W[l], W[l].T, atol=1e-13)  # complex-symmetric


def test_field_free_ground_state_is_stationary():
    run = P.reference_like(32, 8, 20, "H", intensity=1e-30)
    run = run.with_field(np.zeros(20))
    out = propagate(to_oracle(run))
    x0 = run.x0[0, 0]
    x = out["x"][0, 0]
    # |x(t)| unchanged away from the absorber, phase exp(-i e t)
    inner = run.grid.r < 10.0
    assert np.allclose(np.abs(x[inner]), np.abs(x0[inner]), atol=1e-6)


def test_oracle_quirk_tail_loop_of_octupole_density():
    """hartreePotentialDensity.cuh:150 restarts the L=3 tail loop at N_l-4: that l counts twice."""
    from oracle.step_oracle import OracleState
    run = P.reference_like(32, 10, 4, "Ne3", perturb=0.1)
    st = OracleState(to_oracle(run))
    x = np.zeros_like(run.x0)
    x[6, 0, :] = 1.0        # l = N_l - 4
    x[3, 0, :] = 1.0        # l - 3
    d = st.density_multipoles(x)[3]
    from oracle.step_oracle import f3lm
    # f3lm(3) x3.x6 is counted by the l=3 up-term, the middle loop's l=6 down-term and the tail's
    expect = float(run.occ[0]) * 3 * f3lm(3, 0)
    assert np.allclose(d, expect)


@pytest.mark.parametrize("n_l,ms", [(32, [0, 1, 0]), (8, [0, 1, 2]), (5, [0, 1]), (12, [0, 3, 1])])
def test_density_multipoles_equal_the_literal_loops(n_l, ms):
    """The array form of the density multipoles sums the same l ranges and coefficients as the
    literal loops of hartreePotentialDensity.cuh (including the L = 3 tail restart)."""
    from oracle.step_oracle import OracleState

    class _P:
        pass

    p = _P()
    p.n_l, p.n_r, p.n_kso, p.m, p.occ, p.n_har = n_l, 9, len(ms), np.array(ms), np.arange(1, len(ms) + 1), 4
    st = OracleState.__new__(OracleState)
    st.p = p
    rng = np.random.default_rng(n_l)
    x = rng.standard_normal((n_l, len(ms), 9)) + 1j * rng.standard_normal((n_l, len(ms), 9))
    a = st.density_multipoles_literal(x)
    b = st.density_multipoles(x)
    assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max()


def test_argon_exchange_feedback_amplifies_perturbations_and_frozen_xc_does_not():
    """All-electron argon in the adiabatic LDA exchange of the reference (Slater exchange of the
    monopole density, h_calculateExchangeCorrelationPotential.cuh:26-45) is unstable in field-free
    propagation: a 1e-10 perturbation of the self-consistent ground state grows by ~1e7 in 400 steps
    (8 a.u.).  With the exchange-correlation potential held at its ground-state value (the Hartree
    multipoles still follow the density) it stays at the size of the perturbation.  This is why no
    arithmetic other than the identical FP64 sequence can reproduce the argon LDA spectrum, and why
    the argon benchmark can freeze xc."""
    import numpy as np
    from ggbtddft_b200 import accuracy as A
    from ggbtddft_b200 import problems as P
    from oracle.step_oracle import OracleState
    grown = {}
    for frozen in (False, True):
        run = P.baseline_run("Ar", 100, 50.0, 8, 0.02, P.LaserSpec(1.4e14, 800.0, 10.0, 0.0), 10.0,
                             n_steps=400, xc_frozen=frozen).with_field(np.zeros(400))
        a = OracleState(to_oracle(run))
        b = OracleState(to_oracle(A.perturb_orbitals(run, 1e-10)))
        a.init_potentials()
        b.init_potentials()
        for t in range(400):
            a.step(t)
            b.step(t)
        grown[frozen] = np.abs(a.x - b.x).max() / np.abs(a.x).max()
    assert grown[False] > 1e-5, grown          # > 1e5-fold growth with the exchange following the density
    assert grown[True] < 1e-7, grown           # < 1e3-fold with it frozen
