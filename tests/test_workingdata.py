"""The reference's file contract (CPU): workingData inputs, params.cuh and the dipole output files
written and read back in the reference's layout (ggbtddft_b200/workingdata.py)."""
import os

import numpy as np
import pytest

from ggbtddft_b200 import inputs as I
from ggbtddft_b200 import problems as P
from ggbtddft_b200 import workingdata as WD


def test_working_data_round_trip(tmp_path):
    run = P.reference_like(n_r=64, n_l=32, n_t=16, atom="H")
    root = str(tmp_path)
    WD.write_working_data(run, root)
    WD.write_params_cuh(run, str(tmp_path / "params.cuh"), e0=0.0534, omega0=0.057, tau0=200.0, cep0=0.0)
    params = WD.parse_params_cuh(str(tmp_path / "params.cuh"))
    assert (params["N_r"], params["N_l"], params["N_kso"], params["N_t"]) == (64, 32, run.n_orb, 16)
    assert params["WORKING_DATA_PROPAGATOR_L_000"] == "./workingData/hamiltonian/propagators/propagatorL000.bin"
    # the file sizes of the reference's contract
    wd = tmp_path / "workingData"
    assert (wd / "hamiltonian/propagators/propagatorL031.bin").stat().st_size == 64 * 64 * 16
    assert (wd / "mesh/r.bin").stat().st_size == 64 * 8
    assert (wd / "stateParameters/l_active.bin").stat().st_size == run.n_orb * 4
    back = WD.read_working_data(root, params, E=run.E)
    np.testing.assert_array_equal(back.W, run.W)
    for c in I.COUPLINGS:
        np.testing.assert_array_equal(back.V[c], run.V[c])
        np.testing.assert_array_equal(back.D[c], run.D[c])
    np.testing.assert_array_equal(back.grid.r, run.grid.r)
    np.testing.assert_array_equal(back.grid.drdx, run.grid.drdx)
    np.testing.assert_array_equal(back.grid.P, run.grid.P)
    np.testing.assert_array_equal(back.l_active, run.l_active)
    np.testing.assert_array_equal(back.m_active, run.m_active)
    np.testing.assert_array_equal(back.occ, run.occ)
    np.testing.assert_array_equal(back.rho_frozen, run.rho_frozen)
    # h_initialiseTDKSOSet keeps only l == l_active of each orbital
    x = np.zeros_like(run.x0)
    for k, l in enumerate(run.l_active):
        x[l, k] = run.x0[l, k]
    np.testing.assert_array_equal(back.x0, x)
    assert (back.n_har, back.use_hartree, back.target_id, back.dt) == (run.n_har, run.use_hartree,
                                                                        run.target_id, run.dt)


def test_dipole_outputs_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    d = rng.standard_normal((5, 2, 7)) + 1j * rng.standard_normal((5, 2, 7))
    E = rng.standard_normal(7)
    root = str(tmp_path)
    WD.output_dirs(root, 20000101, 3, 1, 2)
    WD.write_dipole_outputs(root, 20000101, 3, 0, d, E)
    p = tmp_path / "20000101/00003/timeDependent/observables/dipoleMoment/scan000/kso001/dipL004.bin"
    assert p.stat().st_size == 7 * 16
    np.testing.assert_array_equal(np.fromfile(p, dtype=np.complex128), d[4, 1])
    np.testing.assert_array_equal(WD.read_dipole_outputs(root, 20000101, 3, 0, 2, 5), d)
    np.testing.assert_array_equal(
        np.fromfile(tmp_path / "20000101/00003/timeDependent/field/E000.bin", dtype=np.float64), E)


REF_BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.mark.parametrize("case", ["h64", "ne3_64", "ne3_128"])
def test_reference_run_directory_reproduces_the_reference_binary(case):
    """The drop-in file contract end to end: the workingData tree and params.cuh that the reference
    binary of the case read (written by oracle/build_ref.py), loaded with read_working_data (the field
    generated from the params.cuh values, as h_initialiseField does) and propagated by the oracle, give
    the dipole files that binary wrote (the committed fixture)."""
    d = os.path.join(REF_BUILD, case)
    if not os.path.isdir(os.path.join(d, "run", "workingData")):
        pytest.skip("reference build of this case not present (oracle/build_ref.py needs the reference sources)")
    from oracle.step_oracle import propagate
    from tests.helpers import GOLDEN, rel_err, to_oracle
    params = WD.parse_params_cuh(os.path.join(d, "params.cuh"))
    ref = np.load(os.path.join(GOLDEN, f"ref_{case}.npz"))
    run = WD.read_working_data(os.path.join(d, "run"), params)      # the field from params.cuh
    out = propagate(to_oracle(run))
    assert out["dipole"].shape == ref["dipole"].shape
    assert rel_err(out["dipole"], ref["dipole"]) < 1e-10
