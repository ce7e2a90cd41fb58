"""Parity at the benchmark configurations' sizes and on the two-M-tile angular chain.

* FP64 form against the oracle at the helium (N_r 400, l_max 64) and argon (N_r 600, l_max 96, nine
  orbitals) configurations, over a window at the pulse centre, within 1e-10 (the bar of the other
  FP64 parity tests);
* the int8 form on the two-M-tile chain (N_l > 128: 16 radii per CTA, channels past 128 in the second
  tile) with the laser phase and the Hartree/exchange phases on, against the oracle over 48 steps,
  and the FP64 form on the same case within 1e-10;
* tile choices of the int8 radial product (ggb_set_tuning) give the same results bit for bit (the
  products accumulate exactly in int32, so tile width and pipeline depth cannot change them).
"""
import dataclasses

import numpy as np
import pytest

from ggbtddft_b200 import problems as P
from ggbtddft_b200.engine import TimePropagation
from oracle.step_oracle import propagate
from tests.helpers import obs_close, rel_err, to_oracle

pytestmark = pytest.mark.gpu

TOL = 1e-10        # FP64 form vs the oracle, relative to the series maximum
TOL_I8 = 3e-5      # int8 form vs the oracle over 48 steps of an interacting atom (as test_gpu_int8)


def _fp64_vs_oracle(run, n):
    ref = propagate(to_oracle(run), n)
    tp = TimePropagation([run])
    tp.step(n)
    got = tp.observables(0, per_l=True, n_steps=n)
    x = tp.orbitals(0)
    pot = tp.potentials(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert obs_close(got["dipole"], ref["dipole"], ref["dipole_scale"], rel=TOL)
    assert obs_close(got["acceleration"], ref["acceleration"], ref["acceleration_scale"], rel=TOL)
    assert rel_err(got["norm"], ref["norm"]) < TOL
    assert rel_err(x, ref["x"]) < TOL
    if run.use_hartree and run.target_id > 0:
        nv = min(run.n_har, 4)
        assert rel_err(pot["v"][:nv], ref["v"][:nv]) < TOL
        assert rel_err(pot["vexc"], ref["vexc"]) < TOL


def _centre(run, n):
    mid = run.n_t // 2
    return run.with_field(run.E[mid:mid + n])


def test_fp64_helium_configuration_at_the_pulse_centre():
    """He LDA, N_r 400, r_max 200, l_max 64, PW92 correlation, cos^(1/8) mask: 16 steps."""
    run = _centre(P.config_helium(device="cuda", angular="reference"), 16)
    _fp64_vs_oracle(run, 16)


def test_fp64_argon_configuration_at_the_pulse_centre():
    """Ar LDA, N_r 600, r_max 300, l_max 96, nine orbitals, all couplings active: 12 steps."""
    run = _centre(P.config_argon(device="cuda", angular="reference"), 12)
    _fp64_vs_oracle(run, 12)


def _two_tile_case(atom, n_l):
    if atom == "H":
        return P.reference_like(96, n_l, 48, "H", r_mask=25.0, intensity=3e14)
    return P.reference_like(64, n_l, 48, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=7)


@pytest.mark.parametrize("atom,n_l", [("H", 150), ("Ne3", 161)])
def test_int8_two_tile_chain_with_phases_tracks_the_oracle(atom, n_l):
    """N_l > 128 takes the two-M-tile chain.  E != 0 (laser phase on every step) and, for the
    3-orbital LDA atom, the P/FP/D/FF/S Hartree and exchange phases; 48 steps."""
    run = _two_tile_case(atom, n_l)
    assert np.abs(run.E).max() > 0.01
    ref = propagate(to_oracle(run))
    tp = TimePropagation([run], precision="split_int8")
    tp.step(run.n_t)
    got = tp.observables(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert rel_err(got["norm"], ref["norm"]) < TOL_I8
    assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_I8
    assert rel_err(got["acceleration"].sum(axis=0), ref["acceleration"].sum(axis=0)) < TOL_I8


@pytest.mark.parametrize("n_l", [150, 161])
def test_fp64_two_tile_sizes_match_the_oracle(n_l):
    run = _two_tile_case("Ne3", n_l)
    _fp64_vs_oracle(run, 24)


def test_int8_radial_tiles_do_not_change_results():
    """ggb_set_tuning: tile widths 16/32/64 and 2-3 pipeline stages, against the built-in choice."""
    base = P.reference_like(64, 16, 12, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=2)
    runs = [base.with_field(base.E * s) for s in (1.0, 0.7, 1.3, 0.4)]     # 12 orbital columns
    ref = TimePropagation(runs, precision="split_int8")
    ref.step(12)
    want = [ref.observables(i) for i in range(len(runs))]
    want_x = [ref.orbitals(i) for i in range(len(runs))]
    ref.close()
    for tune in ((16, 2), (16, 3), (32, 3), (64, 2), (64, 3)):
        tp = TimePropagation(runs, precision="split_int8", tuning={0: tune})
        tp.step(12)
        st, msg = tp.status()
        assert st == 0, (tune, msg)
        for i in range(len(runs)):
            got = tp.observables(i)
            assert np.array_equal(got["dipole"], want[i]["dipole"]), tune
            assert np.array_equal(got["norm"], want[i]["norm"]), tune
            assert np.array_equal(tp.orbitals(i), want_x[i]), tune
        tp.close()


def test_set_tuning_is_refused_by_the_fp64_form():
    from ggbtddft_b200.engine import GGBError
    run = P.reference_like(32, 8, 4, "H")
    with pytest.raises(GGBError, match="split_int8"):
        TimePropagation([run], precision="fp64", tuning={0: (16, 2)})


# ---------------------------------------------------------------------------------------------
# theta form (GGB_RUN_THETA): one phase per half-step at the P coupling's nodes
# ---------------------------------------------------------------------------------------------

def _theta(run, n_har=None):
    return dataclasses.replace(run, angular="theta", n_har=run.n_har if n_har is None else n_har)


@pytest.mark.parametrize("n_r,n_l,n_har", [(45, 9, 4), (70, 17, 3), (64, 33, 2)])
def test_fp64_theta_form_matches_the_oracle(n_r, n_l, n_har):
    run = _theta(P.reference_like(n_r, n_l, 20, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=3), n_har)
    _fp64_vs_oracle(run, 20)


def test_fp64_theta_form_argon_configuration():
    run = _theta(_centre(P.config_argon(device="cuda"), 10))
    _fp64_vs_oracle(run, 10)


@pytest.mark.parametrize("n_l", [32, 161])
def test_int8_theta_form_tracks_the_oracle(n_l):
    run = _theta(_two_tile_case("Ne3", n_l))
    ref = propagate(to_oracle(run))
    tp = TimePropagation([run], precision="split_int8")
    tp.step(run.n_t)
    got = tp.observables(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert rel_err(got["norm"], ref["norm"]) < TOL_I8
    assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_I8


def test_theta_runs_and_reference_runs_do_not_share_a_group():
    from ggbtddft_b200.engine import GGBError
    base = P.reference_like(32, 8, 4, "Ne3", r_mask=12.0, dt_as=10.0)
    with pytest.raises(GGBError):
        TimePropagation([base, _theta(base)], groups=[[0, 1]])


@pytest.mark.parametrize("n_r,n_l,n_har", [(45, 9, 17), (70, 17, 9)])
def test_fp64_theta_form_every_multipole_matches_the_oracle(n_r, n_l, n_har):
    """n_har > 4: multipoles by exact quadrature on 2 N_l nodes (17 = 2 l_max + 1 for N_l = 9)."""
    run = _theta(P.reference_like(n_r, n_l, 20, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=3), n_har)
    _fp64_vs_oracle(run, 20)


def test_fp64_theta_helium_with_multipoles_to_2_lmax():
    """The helium configuration as asked: LDA + PW92, multipoles L = 0 .. 2 l_max = 128."""
    run = _theta(_centre(P.config_helium(device="cuda"), 12), 129)
    _fp64_vs_oracle(run, 12)


def test_int8_theta_form_every_multipole_tracks_the_oracle():
    run = _theta(_two_tile_case("Ne3", 40), 79)
    ref = propagate(to_oracle(run))
    tp = TimePropagation([run], precision="split_int8")
    tp.step(run.n_t)
    got = tp.observables(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert rel_err(got["norm"], ref["norm"]) < TOL_I8
    assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_I8


@pytest.mark.parametrize("angular", ["reference", "theta"])
def test_fp64_frozen_xc_matches_the_oracle(angular):
    """GGB_RUN_XC_FROZEN: the exchange-correlation potential stays at its t = 0 value."""
    run = P.reference_like(45, 9, 20, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=3)
    run = dataclasses.replace(run, xc_frozen=True, angular=angular)
    _fp64_vs_oracle(run, 20)


# the int8 form with its angular products on the FP64 tensor cores (ggb_set_angular_fp64): the radial
# product keeps its int8 slices, so the difference from the oracle is the radial product's alone
@pytest.mark.parametrize("angular,n_l", [("theta", 32), ("theta", 161), ("reference", 161)])
def test_int8_with_fp64_angular_tracks_the_oracle(angular, n_l):
    run = dataclasses.replace(_two_tile_case("Ne3", n_l), angular=angular)
    ref = propagate(to_oracle(run))
    tp = TimePropagation([run], precision="split_int8", angular_fp64=True)
    tp.step(run.n_t)
    got = tp.observables(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert rel_err(got["norm"], ref["norm"]) < TOL_I8
    assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_I8


def test_set_angular_fp64_is_refused_by_the_fp64_form():
    from ggbtddft_b200.engine import GGBError
    run = P.reference_like(32, 8, 4, "H")
    tp = TimePropagation([run])
    with pytest.raises(GGBError):
        tp._call("ggb_set_angular_fp64", 0, 1)
    tp.close()
