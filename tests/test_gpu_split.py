"""Split-precision form (complex64 orbitals, 3xBF16 tcgen05 radial GEMM) against the FP64 oracle."""
import dataclasses

import numpy as np
import pytest

from ggbtddft_b200 import problems as P
from ggbtddft_b200.engine import TimePropagation
from oracle.step_oracle import propagate
from tests.helpers import rel_err, to_oracle

pytestmark = pytest.mark.gpu

# 3xBF16 products keep ~16 significant bits of each operand (hi + lo) and drop lo*lo: one radial
# product is accurate to a few 1e-5 of the vector norm; the bounds below allow for that per step.
TOL_ONE_STEP = 2e-4
TOL_MULTI = 3e-3


@pytest.mark.parametrize("n_r,n_l", [(64, 16), (200, 33), (37, 5)])
def test_radial_tensor_core_product_one_step(n_r, n_l):
    """E = 0 and no Hartree: the angular half-steps are V V^T = 1, so one step is x <- A x."""
    run = P.reference_like(n_r, n_l, 4, "H", r_mask=20.0)
    run = run.with_field(np.zeros(4))
    rng = np.random.default_rng(0)
    x0 = np.zeros_like(run.x0)
    x0[:, 0, :] = rng.standard_normal((n_l, n_r)) + 1j * rng.standard_normal((n_l, n_r))
    run = dataclasses.replace(run, x0=x0)
    tp = TimePropagation([run], precision="split_bf16")
    tp.step(1)
    got = tp.orbitals(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    expect = np.einsum("lba,lkb->lka", run.W, x0)
    for l in range(n_l):
        assert rel_err(got[l, 0], expect[l, 0]) < TOL_ONE_STEP, l


@pytest.mark.parametrize("atom", ["H", "Ne3"])
def test_split_bf16_tracks_fp64_oracle(atom):
    if atom == "H":
        run = P.reference_like(64, 32, 48, "H", r_mask=30.0)
    else:
        run = P.reference_like(64, 32, 48, "Ne3", r_mask=20.0, dt_as=10.0, perturb=0.05, seed=7)
    ref = propagate(to_oracle(run))
    tp = TimePropagation([run], precision="split_bf16")
    tp.step(run.n_t)
    got = tp.observables(0)
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg
    assert rel_err(got["norm"], ref["norm"]) < TOL_MULTI
    assert rel_err(got["dipole"].sum(axis=0), ref["dipole"].sum(axis=0)) < TOL_MULTI
    assert rel_err(got["acceleration"].sum(axis=0), ref["acceleration"].sum(axis=0)) < TOL_MULTI


def test_split_ensemble_group_equals_single_runs():
    base = P.reference_like(64, 16, 20, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=2)
    runs = [base.with_field(base.E * s) for s in (1.0, 0.5, 1.5, 0.8)]
    ens = TimePropagation(runs, precision="split_bf16")
    ens.step(20)
    for i, r in enumerate(runs):
        one = TimePropagation([r], precision="split_bf16")
        one.step(20)
        # same arithmetic in the same order: the grouped GEMM must not mix columns
        assert rel_err(ens.observables(i)["dipole"], one.observables(0)["dipole"]) < 1e-6
        one.close()
    ens.close()
