"""Basis reuse of the int8 theta form (ggb_set_theta_reuse, on by default).

A half-step is x <- V diag(phase) V^T x with V orthogonal, and nothing acts on the orbitals between
a step's second half and the next step's first half, so the first half starts from the node-basis
vectors the second half kept and runs one product instead of two.  The tests check that

* the reuse path runs (its results differ in the last bits from the two-product chain, which
  applies V^T V, the identity up to the operands' rounding) and tracks the oracle as closely as the
  two-product chain, on one and two M tiles, with the laser, Hartree and exchange phases on, and
  with every multipole from the exact quadrature (n_har > 4);
* after new orbitals are set the steps equal a fresh context's (the kept vectors are invalidated and
  the step counter restarts);
* batching runs in one grid group, or on several grid groups stepped on concurrent streams, still
  changes nothing at all;
* the switch is refused by the FP64 form.
"""
import dataclasses

import numpy as np
import pytest

from ggbtddft_b200 import problems as P
from ggbtddft_b200.engine import GGBError, TimePropagation
from oracle.step_oracle import propagate
from tests.helpers import rel_err, to_oracle

pytestmark = pytest.mark.gpu

TOL_I8 = 3e-5      # int8 form vs the oracle over 48 steps of an interacting atom (as the other int8 tests)


def _case(n_l, n_har=None, seed=7):
    run = P.reference_like(64, n_l, 48, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=seed)
    return dataclasses.replace(run, angular="theta", n_har=run.n_har if n_har is None else n_har)


def _run(run, reuse, n=None):
    tp = TimePropagation([run], precision="split_int8", theta_reuse=reuse)
    tp.step(run.n_t if n is None else n)
    got = tp.observables(0)
    x = tp.orbitals(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    return got, x


@pytest.mark.parametrize("n_l,n_har", [(32, 4), (161, 4), (40, 79)])
def test_reuse_runs_and_tracks_the_oracle(n_l, n_har):
    run = _case(n_l, n_har)
    assert np.abs(run.E).max() > 0.01
    ref = propagate(to_oracle(run))
    on, x_on = _run(run, True)
    off, x_off = _run(run, False)
    assert not np.array_equal(x_on, x_off)       # the one-product first half ran
    for got in (on, off):
        assert rel_err(got["norm"], ref["norm"]) < TOL_I8
        assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_I8
        assert rel_err(got["acceleration"].sum(axis=0), ref["acceleration"].sum(axis=0)) < TOL_I8
    assert rel_err(x_on, x_off) < TOL_I8


def test_set_orbitals_invalidates_the_kept_vectors():
    run = _case(161)
    n = 12
    _, want = _run(run, True, n)
    tp = TimePropagation([run], precision="split_int8")
    tp.step(n)
    tp.set_orbitals(0, run.x0)      # back to the initial orbitals, the step counter to 0
    tp.step(n)
    got = tp.orbitals(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert np.array_equal(got, want)


def test_reuse_in_a_group_equals_single_runs():
    base = _case(32, seed=2)
    runs = [base.with_field(base.E * s) for s in (1.0, 0.5, 1.5)]
    ens = TimePropagation(runs, precision="split_int8")
    ens.step(20)
    for i, r in enumerate(runs):
        one = TimePropagation([r], precision="split_int8")
        one.step(20)
        assert np.array_equal(ens.orbitals(i), one.orbitals(0))
        assert np.array_equal(ens.observables(i)["dipole"], one.observables(0)["dipole"])
        one.close()
    ens.close()


def test_reuse_with_grid_groups_on_concurrent_streams_equals_single_runs():
    """Runs on different grids form separate groups stepped on their own streams, each with its own
    kept vectors and step counter: every run equals the run stepped alone."""
    runs = [_case(32, seed=2),
            dataclasses.replace(P.reference_like(48, 161, 48, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=5),
                                angular="theta")]
    ens = TimePropagation(runs, precision="split_int8")
    assert len(ens.groups) == 2
    ens.step(20)
    for i, r in enumerate(runs):
        one = TimePropagation([r], precision="split_int8")
        one.step(20)
        assert np.array_equal(ens.orbitals(i), one.orbitals(0))
        one.close()
    st, msg = ens.status()
    ens.close()
    assert st == 0, msg


def test_theta_reuse_is_refused_by_the_fp64_form():
    run = P.reference_like(32, 8, 4, "H")
    tp = TimePropagation([run])
    with pytest.raises(GGBError, match="split_int8"):
        tp._call("ggb_set_theta_reuse", 0, 0)
    tp.close()
