"""Error of the split-precision form against the FP64 form, per result, over a full pulse.

    python -m ggbtddft_b200.accuracy --config argon [--precision split_bf16] [--steps N] [--out report.json]

Both forms run the same inputs on the GPU (the FP64 form is the one held to the reference to 1e-10).
Reported: norm drift (max |norm_split - norm_fp64| per orbital), relative L2 error of the total
dipole and of the total dipole acceleration <cos(theta)/r^2>, and the relative error of every
harmonic intensity up to the semiclassical cutoff, from the HHG spectrum of the total dipole
computed with the reference's recipe (spectrum.py).
"""
from __future__ import annotations

import argparse
import json
import time
from typing import Optional

import numpy as np

from . import problems as P
from . import spectrum as S
from .engine import TimePropagation

IONISATION_POTENTIAL = {"H": 0.5, "He": 0.9036, "Ar": 0.5792}   # Ha (experimental first Ip)


def _run(run: P.RunInputs, precision: str, n_steps: int, chunk: int = 4096):
    tp = TimePropagation([run], precision=precision, per_l=True, n_t=n_steps)
    t0 = time.perf_counter()
    done = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        tp.step(k)
        done += k
    obs = tp.observables(0, per_l=True, n_steps=n_steps)
    st, msg = tp.status()
    tp.close()
    obs["seconds"] = time.perf_counter() - t0
    obs["status"] = (st, msg)
    return obs


def compare_forms(run: P.RunInputs, atom: str, precision: str = "split_bf16", n_steps: Optional[int] = None,
                  e0: Optional[float] = None) -> dict:
    n = run.n_t if n_steps is None else n_steps
    ref = _run(run, "fp64", n)
    tst = _run(run, precision, n)
    d_ref = S.total_dipole(ref["dipole"], run.l_active, run.m_active, run.occ)
    d_tst = S.total_dipole(tst["dipole"], run.l_active, run.m_active, run.occ)
    a_ref = (run.occ[None, :, None] * ref["acceleration"]).real.sum(axis=(0, 1))
    a_tst = (run.occ[None, :, None] * tst["acceleration"]).real.sum(axis=(0, 1))
    w, s_ref = S.hhg_spectrum(d_ref, run.dt)
    _, s_tst = S.hhg_spectrum(d_tst, run.dt)
    e0 = float(np.abs(run.E).max()) if e0 is None else e0
    q_cut = S.cutoff_order(IONISATION_POTENTIAL[atom], e0, run.omega0)
    herr = S.harmonic_errors(s_tst, s_ref, w, run.omega0, q_cut)
    odd = herr[0::2]
    return dict(
        config=run.name, precision=precision, steps=n, dt=run.dt, omega0=run.omega0, cutoff_order=q_cut,
        seconds=dict(fp64=ref["seconds"], split=tst["seconds"]),
        status=dict(fp64=ref["status"], split=tst["status"]),
        final_norm_fp64=ref["norm"][:, -1].tolist(),
        final_norm_split=tst["norm"][:, -1].tolist(),
        norm_drift_max=float(np.abs(tst["norm"] - ref["norm"]).max()),
        dipole_rel_l2=float(np.linalg.norm(d_tst - d_ref) / np.linalg.norm(d_ref)),
        acceleration_rel_l2=float(np.linalg.norm(a_tst - a_ref) / np.linalg.norm(a_ref)),
        harmonic_rel_err=herr.tolist(),
        odd_harmonic_rel_err_max=float(odd.max()),
        all_harmonics_within_1e3=bool(np.all(herr <= 1e-3)),
        odd_harmonics_within_1e3=bool(np.all(odd <= 1e-3)),
    )


CONFIGS = {
    "hydrogen": ("H", P.config_hydrogen),
    "helium": ("He", P.config_helium),
    "argon": ("Ar", P.config_argon),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="argon", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="split_bf16")
    ap.add_argument("--steps", type=int, default=None, help="default: the full pulse")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    atom, builder = CONFIGS[args.config]
    run = builder(n_steps=args.steps, device="cuda")
    rep = compare_forms(run, atom, args.precision)
    line = json.dumps(rep)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    print(json.dumps({k: v for k, v in rep.items() if k != "harmonic_rel_err"}))


if __name__ == "__main__":
    main()
