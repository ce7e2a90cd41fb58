"""Shared test helpers: fixtures loading and conversion of RunInputs to the oracle's problem."""
import json
import os

import numpy as np

from ggbtddft_b200 import problems as P
from oracle.step_oracle import OracleProblem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def to_oracle(run: P.RunInputs) -> OracleProblem:
    return OracleProblem(r=run.grid.r, drdx=run.grid.drdx, P=run.grid.P, W=run.W, V=run.V, D=run.D,
                         x0=run.x0, m=run.m_active, occ=run.occ, rho_frozen=run.rho_frozen, E=run.E,
                         dt=run.dt, n_har=run.n_har, use_hartree=run.use_hartree, target_id=run.target_id,
                         xc_correlation=run.xc_correlation, xc_frozen=run.xc_frozen, angular=run.angular)


def load_ref_case(name):
    """(RunInputs rebuilt from the case's generator arguments with the reference's own E, ref dipole)."""
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    case = json.loads(str(z["case"]))
    run = P.reference_like(**case["kwargs"]).with_field(z["E"])
    return run, z["dipole"]


def rel_err(a, b):
    """max |a - b| / max |b| (size-independent, robust to near-zero entries)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def obs_close(got, ref, scale, rel=1e-10, cond=1e-13):
    """|got - ref| <= rel * max|ref| + cond * scale, elementwise.

    ``scale`` is the sum of |terms| of each inner product: per-(l, t) dipole and acceleration sums
    cancel (terms ~1e-2 summing to ~1e-8 near t = 0), so any two summation orders -- the
    reference's cublasZdotc included -- differ by ~1e-16 * scale there.
    """
    got = np.asarray(got)
    ref = np.asarray(ref)
    bound = rel * np.abs(ref).max() + cond * np.asarray(scale)
    return bool(np.all(np.abs(got - ref) <= bound))
