"""Autotuner of the int8 radial product's tiles, per grid group.

The split_int8 radial product (`k_radial_i8`) has two free choices per grid group: the tile width
bn (orbital columns per tile: 16, 32 or 64) and the number of TMA pipeline stages (2 up to what fits
in shared memory).  The library's built-in choice takes bn from the group's column count and the
most stages that fit.  The tuner times every candidate on the group's own runs (the radial phase
launched alone, CUDA events, after warm-up) and keeps the fastest.  Results are cached in a JSON
file keyed on the GPU's name, the library version and the group's (N_r, l_max, orbital columns), so
a grid shape is timed once per GPU model and kernel version; the cache is $GGB_AUTOTUNE_CACHE, else
~/.cache/ggbtddft_b200/autotune.json, read over the tunings shipped in tuning/autotune_b200.json.

    TimePropagation(runs, precision="split_int8", autotune=True)   # cached or tuned tiles
    tuning_for(runs, groups)                                         # {group: (bn, stages)}
"""
from __future__ import annotations

import json
import os
import tempfile
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

BN_CHOICES = (16, 32, 64)
# one stage of k_radial_i8: eight int8 W planes of 128 x 32 and twelve x planes of bn x 32
R8_BM, R8_BK, R8_W_PLANES, R8_X_PLANES = 128, 32, 8, 12
SMEM_BUDGET = 200 * 1024


def max_stages(bn: int) -> int:
    """Pipeline stages of the radial product that fit in shared memory (the library's r8_stages)."""
    stage = R8_W_PLANES * R8_BM * R8_BK + R8_X_PLANES * bn * R8_BK
    return max(2, min(8, SMEM_BUDGET // stage))


# Every k_radial_i8 CTA allocates 512 tensor-memory columns (all of an SM's).  A CTA whose shared
# memory leaves room for a second one on its SM (<= 113 KB of the SM's 228 KB, with the 1 KB the
# runtime reserves per CTA) can be placed beside another radial CTA -- of its own grid or of another
# grid group's concurrent launch -- which then waits in tcgen05.alloc until the first one exits.
# Timed alone such a tile looks fine and is slower in the real step, so it is not a candidate.
SM_SMEM = 228 * 1024
CTA_RESERVED = 1024


def smem_bytes(bn: int, stages: int) -> int:
    """Dynamic shared memory of one k_radial_i8 CTA (the library's r8_smem)."""
    return stages * (R8_W_PLANES * R8_BM * R8_BK + R8_X_PLANES * bn * R8_BK) + 1024


def one_cta_per_sm(bn: int, stages: int) -> bool:
    return 2 * (smem_bytes(bn, stages) + CTA_RESERVED) > SM_SMEM


def candidates(n_cols: int) -> List[Tuple[int, int]]:
    """(bn, stages) pairs worth timing: tile widths up to the first one that covers all columns
    (a wider tile only adds padding), each with the stage counts from 2 to max_stages(bn) whose
    shared memory keeps one CTA per SM."""
    out = []
    for bn in BN_CHOICES:
        out.extend((bn, st) for st in range(2, max_stages(bn) + 1) if one_cta_per_sm(bn, st))
        if bn >= n_cols:
            break
    return out


# tunings measured on B200 for the benchmark ensembles' grid groups, shipped with the package
PACKAGED_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "autotune_b200.json")


def cache_path() -> str:
    """$GGB_AUTOTUNE_CACHE, else the user cache ~/.cache/ggbtddft_b200/autotune.json."""
    return os.environ.get("GGB_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "ggbtddft_b200", "autotune.json")


def library_version() -> str:
    """ggb_version() of the loaded library, so that tunings of older kernels are not reused."""
    try:
        from .engine import load_library
        return load_library().ggb_version().decode()
    except Exception:
        return "unknown"


def cache_key(n_r: int, l_max: int, n_cols: int, device_name: str, version: Optional[str] = None) -> str:
    v = library_version() if version is None else version
    return f"{device_name}|{v}|N_r={n_r}|l_max={l_max}|cols={n_cols}"


def load_cache(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: Dict[str, dict]) -> None:
    """Write the cache atomically (a temporary file renamed over the old one)."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(path)), suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_candidate(runs, cand: Tuple[int, int], warmup: int = 3, reps: int = 10) -> float:
    """Milliseconds of one radial product of these runs (one grid group) with tiles ``cand``."""
    import torch
    from .engine import TimePropagation
    n_t = warmup + 8
    short = [r.with_field(np.asarray(r.E)[:n_t]) for r in runs]   # few steps of observables
    tp = TimePropagation(short, precision="split_int8", per_l=True, n_t=n_t, groups=[list(range(len(short)))],
                         tuning={0: cand})
    try:
        stream = torch.cuda.current_stream()
        tp.step(warmup, stream.cuda_stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tp.launch_phase(1, stream.cuda_stream)
        a.record(stream)
        for _ in range(reps):
            tp.launch_phase(1, stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps
    finally:
        tp.close()


def tune_group(runs, timer: Callable = time_candidate) -> Tuple[Tuple[int, int], Dict[str, float]]:
    """Time every candidate for one grid group; returns the fastest (bn, stages) and the table."""
    n_cols = sum(r.n_orb for r in runs)
    table = {f"{bn}x{st}": float(timer(runs, (bn, st))) for bn, st in candidates(n_cols)}
    best = min(table, key=table.get)
    bn, st = (int(v) for v in best.split("x"))
    return (bn, st), table


def tuning_for(runs: Sequence, groups: Sequence[Sequence[int]], cache_file: Optional[str] = None,
               timer: Callable = time_candidate, device_name: Optional[str] = None) -> Dict[int, Tuple[int, int]]:
    """{group index: (bn, stages)} from the cache, timing the groups that miss it."""
    path = cache_file or cache_path()
    cache = load_cache(PACKAGED_CACHE)
    cache.update(load_cache(path))
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name()
    out, dirty = {}, False
    for gi, members in enumerate(groups):
        rs = [runs[i] for i in members]
        key = cache_key(rs[0].n_r, rs[0].n_l - 1, sum(r.n_orb for r in rs), device_name)
        if key not in cache:
            (bn, st), table = tune_group(rs, timer)
            cache[key] = dict(bn=bn, stages=st, ms=table)
            dirty = True
        out[gi] = (int(cache[key]["bn"]), int(cache[key]["stages"]))
    if dirty:
        save_cache(path, cache)
    return out


def main(argv=None):
    """Tune the grid groups of the benchmark ensembles on this GPU and write them to the packaged cache:
    python -m ggbtddft_b200.autotune [--out PATH]"""
    import argparse
    import dataclasses
    from . import problems as P
    from .engine import group_runs
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=PACKAGED_CACHE)
    args = ap.parse_args(argv)
    for runs in (P.argon_ensemble(64, seed=0, n_steps=16, device="cuda"),
                 P.hhe_ensemble(256, seed=0, n_steps=16, device="cuda")):
        runs = [dataclasses.replace(r, angular="theta") for r in runs]
        groups = group_runs(runs)
        print(json.dumps({str(k): v for k, v in tuning_for(runs, groups, cache_file=args.out).items()}))


if __name__ == "__main__":
    main()
