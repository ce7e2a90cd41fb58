"""Time the reference's own main.cu on this GPU (test infrastructure, like the rest of oracle/).

The binaries of ``oracle/build_ref.py``'s TIMED_CASES are compiled from the reference's sources with
a cudaEvent wrapper around its ``h_timePropagation`` (h_timePropagation.cuh:32-114: the initial
potentials and the whole tdx loop, with the reference's per-kernel synchronisations and per-(orbital,
l) dot products).  This script writes the case's workingData next to the binary (the same generator
arguments as the build, so the same sizes and parameters), runs the binary, and reports
orbital-steps/s = N_kso * N_t / event time.

    python oracle/time_ref.py <case> <out.json>        # e.g. ar9_608
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.build_ref import OUT, SIM_DATE, SIM_INDEX, TIMED_CASES  # noqa: E402


def main(case: str, out_path: str) -> int:
    from ggbtddft_b200 import problems as P, workingdata as WD
    kw = TIMED_CASES[case]
    d = os.path.join(OUT, case)
    binary = os.path.join(d, "ggb_ref")
    if not os.access(binary, os.X_OK):
        raise SystemExit(f"{binary} is missing: build it with oracle/build_ref.py where the reference sources are")
    t0 = time.perf_counter()
    run = P.reference_like(**kw, device="cuda")
    WD.write_working_data(run, os.path.join(d, "run"))
    WD.output_dirs(os.path.join(d, "output"), SIM_DATE, SIM_INDEX, 1, run.n_orb)
    setup_s = time.perf_counter() - t0
    t1 = time.perf_counter()
    proc = subprocess.run([binary], cwd=os.path.join(d, "run"), capture_output=True, text=True, timeout=1800)
    wall_s = time.perf_counter() - t1
    m = re.findall(r"GGB_REF_TIMING scan=(\d+) steps=(\d+) ms=([0-9.]+)", proc.stdout)
    if proc.returncode != 0 or not m:
        sys.stderr.write(proc.stdout[-2000:] + proc.stderr[-2000:])
        raise SystemExit(f"reference binary failed (exit {proc.returncode})")
    steps, ms = int(m[0][1]), float(m[0][2])
    res = dict(case=case, generator=kw, n_r=run.n_r, n_l=run.n_l, n_kso=run.n_orb, n_t=steps,
               event_ms=ms, ms_per_step=ms / steps, orbital_steps_per_s=run.n_orb * steps / (ms / 1e3),
               process_wall_s=wall_s, inputs_setup_s=setup_s,
               how="reference main.cu (sm_100a build of its own sources), cudaEvents around h_timePropagation")
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit("usage: python oracle/time_ref.py <case> <out.json>")
    raise SystemExit(main(sys.argv[1], sys.argv[2]))
