"""The input producers (ggbtddft_b200.inputs) against the reference's own outputs, on CPU.

* the laser field against the E000.bin the reference binary wrote (h_initialiseField.cuh:1-40 on the
  time grid and params.cuh of the parity cases; tests/golden/ref_*.npz);
* the radial grid, the CAP, the Crank-Nicolson radial propagators and the angular eigensystems against
  what the reference's internal.py returned or wrote for the same inputs
  (tests/golden/internal_inputs.npz, made by tests/golden/make_internal_fixtures.py).
"""
import json
import os

import numpy as np
import pytest

from ggbtddft_b200 import inputs as I

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.fixture(scope="module")
def internal():
    return np.load(os.path.join(GOLDEN, "internal_inputs.npz"))


@pytest.mark.parametrize("case", ["h64", "ne3_64", "ne3_128", "ar9_256"])
def test_field_matches_the_reference_binary(case):
    z = np.load(os.path.join(GOLDEN, f"ref_{case}.npz"))
    c = json.loads(str(z["case"]))
    kw, fp = c["kwargs"], c["field"]
    dt = kw["dt_as"] * I.ATTOSECOND_AU
    t = I.time_grid(c["n_t"], dt)
    E = I.field_super_gaussian(t, fp["e0"], fp["omega0"], fp["tau0"], fp["cep0"])
    assert E.shape == z["E"].shape
    # relative to the amplitude E0: a short window near t = 0 with CEP pi/2 samples only E ~ E0 w t
    assert np.abs(E - z["E"]).max() <= 1e-14 * fp["e0"]


def test_grid_matches_internal_py(internal):
    z = internal
    g = I.make_grid(int(z["n_r"]), float(z["r_max"]), float(z["zeta"]))
    assert _rel(g.r, z["r"]) < 1e-14
    assert _rel(g.drdx, z["drdx"]) < 1e-14
    assert _rel(g.T, z["T"]) < 1e-13
    assert _rel(g.P, z["P"]) < 1e-12


def test_cap_matches_internal_py(internal):
    z = internal
    cap = I.cap_manolopoulos(z["r"], float(z["r_mask"]), float(z["r_max"]))
    assert _rel(cap, z["cap"]) < 1e-14


def test_radial_propagators_match_internal_py(internal):
    """W_l = (I + i dt/2 H_l)^-1 (I - i dt/2 H_l) with H_l = -T/2 + v0 + l(l+1)/2r^2 - i W + vscf."""
    z = internal
    g = I.make_grid(int(z["n_r"]), float(z["r_max"]), float(z["zeta"]))
    W = I.radial_propagators(g, int(z["n_l"]), float(z["dt"]), z["v0"], z["vscf"], z["cap"], method="CN")
    assert W.shape == z["W"].shape
    for l in range(int(z["n_l"])):
        assert _rel(W[l], z["W"][l]) < 1e-12, l


@pytest.mark.parametrize("coupling", ["P", "FP", "D", "FF"])
def test_angular_eigensystems_match_internal_py(internal, coupling):
    """Same eigenvalues, and the same operators V f(D) V^T (eigenvectors are defined up to sign, and
    within a degenerate eigenspace up to a rotation, so the operators are what must agree)."""
    z = internal
    n_l, n_m = int(z["n_l_ang"]), int(z["n_m"])
    V, D = I.angular_eigensystems(n_l, n_m)[coupling]
    Vr, Dr = z["V_" + coupling], z["D_" + coupling]
    for m in range(n_m):
        assert np.allclose(np.sort(D[m]), np.sort(Dr[m]), rtol=0, atol=1e-14)
        for a in (0.37, 2.9):
            U = V[m] @ np.diag(np.exp(-1j * a * D[m])) @ V[m].T
            Ur = Vr[m] @ np.diag(np.exp(-1j * a * Dr[m])) @ Vr[m].T
            assert np.abs(U - Ur).max() < 1e-13, (m, a)
        # rows and columns below m are zero in both
        assert np.all(V[m][:m] == 0) and np.all(Vr[m][:m] == 0)
