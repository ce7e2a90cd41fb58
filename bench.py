"""Throughput of the split-operator time step on B200: orbital-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A "step" is one time step of every run of the workload (both angular half-steps, the radial
propagator, density, Hartree/exchange potentials and the dipole/acceleration/norm reductions).
``value`` = sum over runs of (orbitals x steps) / device time of the K timed steps, all inputs
resident in HBM, steps replayed from a captured CUDA graph.  ``e2e`` is the same metric through
the C ABI from host buffers: orbitals and field uploaded from pinned host memory, K steps, per-l
dipole/acceleration and norm series downloaded, wall clock.

Multi-GPU (torchrun): every rank runs an independent replica of the workload (the runs of an
ensemble are independent; there is no exchange step), ``value`` = all ranks' orbital-steps / the
slowest rank's device time.

``--impl reference`` times the reference algorithm on the host CPU: the FP64 NumPy restatement of
the reference time loop (``oracle/step_oracle.py``; the reference itself is a CUDA program with no
CPU path), on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


# ---------------------------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------------------------

POTENTIALS = {
    "adiabatic": "Hartree multipoles and exchange-correlation follow the density (the reference's loop)",
    "xc-frozen": "Hartree multipoles follow the density; exchange-correlation held at the ground state",
    "frozen": "all potentials held at the LDA ground state (USE_HARTREE = 0): a linear propagation",
}


def workload_runs(name: str, n_t: int, device=None, split: str = "split_int8", only=None,
                  angular: str = "theta", potentials: str = "adiabatic"):
    """Return (runs, precision, description dict); ``split`` is the form of the non-FP64 workloads;
    ``only`` builds just those runs of an ensemble workload (the CPU sample needs one); ``angular``
    and ``potentials`` (POTENTIALS) set every run's angular step and potential treatment."""
    runs, precision, desc = _workload_runs(name, n_t, device, split, only)
    import dataclasses
    runs = [dataclasses.replace(r, angular=angular, xc_frozen=potentials == "xc-frozen" or r.xc_frozen,
                                use_hartree=0 if potentials == "frozen" else r.use_hartree) for r in runs]
    if runs and any(r.n_har > 4 for r in runs) and angular != "theta":
        runs = [dataclasses.replace(r, n_har=4) for r in runs]
    desc = dict(desc, angular=angular + (" (one phase per half-step at the P coupling's Gauss nodes)"
                                         if angular == "theta" else " (the reference's FF/FP/D/P/S chain)"),
                potentials=f"{potentials}: {POTENTIALS[potentials]}")
    return runs, precision, desc


def _workload_runs(name: str, n_t: int, device=None, split: str = "split_int8", only=None):
    from ggbtddft_b200 import problems as P
    if name.startswith("ar-ens64"):
        precision = "fp64" if name.endswith("fp64") else split
        runs = P.argon_ensemble(64, seed=0, n_steps=n_t, device=device, only=only)
        ladder = ", ".join(f"{g.n_r}/{g.r_max:.0f}/{g.l_max}" for g in P.ARGON_LADDER)
        return runs, precision, dict(
            workload="64-run argon LDA in-situ focal scan: I U[0.8,2]e14 W/cm^2, lambda U[800,1300] nm, "
                     "10-cycle sin^2, dt=0.02, 9 orbitals per run; grids N_r/r_max/l_max on the ladder " + ladder +
                     " (runs of one grid share W); first steps of the pulse",
            runs=64, n_orb=9, precision=precision, seed=0)
    if name.startswith("hhe-ens256"):
        precision = "fp64" if name.endswith("fp64") else split
        runs = P.hhe_ensemble(256, seed=0, n_steps=n_t, device=device, only=only)
        return runs, precision, dict(
            workload="256-run H/He scan: I log-U[0.5,3]e14, CEP U[0,2pi), lambda U[800,1800] nm, 6-cycle sin^2, "
                     "dt=0.03; grids N_r 200-800, l_max 32-128 on a ladder", runs=256, n_orb=1,
            precision=precision, seed=0)
    if name == "ar16-n600":
        base = P.config_argon(n_steps=n_t, device=device)
        runs = [base.with_field(base.E * s) for s in np.linspace(0.8, 1.2, 16)]
        return runs, split, dict(workload="16 argon LDA runs on one grid (N_r=600, r_max=300, l_max=96, dt=0.02; "
                                          "9 orbitals each), 800 nm 10-cycle sin^2 at 0.8-1.2 x 1.4e14 W/cm^2; "
                                          "first steps of the pulse", runs=16, n_r=600, l_max=96, n_orb=9,
                                 precision=split)
    if name == "ar16-n400-l160":
        # the angular size of the largest rung of the ensemble (N_l = 161: two M tiles of channels)
        # on a shorter radial grid, small enough for a full ncu capture
        base = P.baseline_run("Ar", 400, 200.0, 160, 0.02, P.LaserSpec(1.4e14, 800.0, 10.0, 0.0), 40.0,
                              n_steps=n_t, device=device)
        runs = [base.with_field(base.E * s) for s in np.linspace(0.8, 1.2, 16)]
        return runs, split, dict(workload="16 argon LDA runs on one grid (N_r=400, r_max=200, l_max=160, dt=0.02; "
                                          "9 orbitals each), 800 nm 10-cycle sin^2 at 0.8-1.2 x 1.4e14 W/cm^2; "
                                          "first steps of the pulse", runs=16, n_r=400, l_max=160, n_orb=9,
                                 precision=split)
    if name == "ar-split":
        run = P.config_argon(n_steps=n_t, device=device)
        return [run], split, dict(workload="Ar LDA, 9 orbitals, N_r=600, r_max=300, l_max=96, dt=0.02",
                                  runs=1, n_r=600, l_max=96, n_orb=9, precision=split)
    if name == "ar-fp64":
        run = P.config_argon(n_steps=n_t, device=device)
        return [run], "fp64", dict(workload="Ar LDA, 9 orbitals, N_r=600, r_max=300, l_max=96, dt=0.02, "
                                            "800 nm 1.4e14 W/cm^2 10-cycle sin^2 (first steps of the pulse)",
                                   runs=1, n_r=600, l_max=96, n_orb=9, precision="fp64")
    if name == "he-fp64":
        run = P.config_helium(n_steps=n_t, device=device, angular="theta")
        return [run], "fp64", dict(workload="He LDA, 1 orbital, N_r=400, r_max=200, l_max=64, dt=0.03",
                                   runs=1, n_r=400, l_max=64, n_orb=1, precision="fp64")
    if name == "h-fp64":
        run = P.config_hydrogen(n_steps=n_t, device=device)
        return [run], "fp64", dict(workload="H, 1 orbital, N_r=200, r_max=100, l_max=32, dt=0.05",
                                   runs=1, n_r=200, l_max=32, n_orb=1, precision="fp64")
    raise SystemExit(f"unknown workload {name}")


def workload_groups(name: str):
    """[(representative run index, runs in the group, label)] for the grid groups of a workload, without
    building its runs: the CPU legs time one run per group and weight it by the group's size."""
    from ggbtddft_b200 import problems as P
    if name.startswith("ar-ens64") or name.startswith("hhe-ens256"):
        dr = P.argon_draws(64, seed=0) if name.startswith("ar-ens64") else P.hhe_draws(256, seed=0)
        out = []
        for (k, atom), members in dr.grid_groups().items():
            g = dr.ladder[k]
            out.append((members[0], len(members), f"{atom} N_r {g.n_r} l_max {g.l_max}"))
        return out
    runs = {"ar16-n600": 16, "ar16-n400-l160": 16}.get(name, 1)
    return [(0, runs, name)]


DEFAULT_WORKLOAD = "ar-ens64"
# the headline: the theta form (the form the benchmark configurations are built for) with the
# potentials frozen at the LDA ground state -- adiabatic all-electron argon amplifies any rounding
# exponentially over a pulse (in FP64 too), so its harmonics cannot carry a 1e-3 bound in any
# arithmetic; the frozen-potential ensemble can, and is checked instance by instance
DEFAULT_ANGULAR = "theta"
DEFAULT_POTENTIALS = "frozen"
DEFAULT_ANGULAR_ARITH = "int8"
# tensor-core products executed per algorithmic real product, and the peak they run against
SPLIT_PRODUCTS = {"split_bf16": 5,    # W_h x_h + W_h x_l + W_m x_h + W_m x_l + W_l x_h (BF16)
                  "split_int8": 10}   # int8 slice pairs (j, m), 0-based, with j + m <= 3
W_BYTES = {"fp64": 16, "split_bf16": 12, "split_int8": 8}   # per complex element of W as streamed
# kernels launched per grid group and step: fp64 angular, radial, angular (+ partials), finalize;
# split_bf16 angular, radial, angular, partials, finalize; split_int8 angular, operand slicing,
# radial, angular (+ partials), finalize
LAUNCHES_PER_GROUP_STEP = {"fp64": 4, "split_bf16": 5, "split_int8": 5}


# ---------------------------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------------------------

def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def reference_binary_record():
    """The reference's own main.cu timed on a B200 (a committed record of oracle/time_ref.py's run;
    nothing under oracle/ is executed here)."""
    p = os.path.join(ROOT, "profiles", "reference_main_cu__ar9_n608_l96.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return dict(value=d["orbital_steps_per_s"], unit="orbital-steps/s", ms_per_step=d["ms_per_step"],
                config=f"argon, {d['n_kso']} orbitals, N_r {d['n_r']}, N_l {d['n_l']}, {d['n_t']} steps",
                how=d["how"] + "; recorded in profiles/reference_main_cu__ar9_n608_l96.json")


def compute_peaks(stream_handle):
    """FP64 FMA and tcgen05 int8 peaks of this GPU from the library's own microbenchmarks
    (ggb_measure_peaks), taken once before the timed region."""
    from ggbtddft_b200.engine import measure_peaks
    return measure_peaks(stream_handle)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region: the sampler is started and its
    first sample awaited before the region opens; only the samples written after that count."""

    def __init__(self, index: int, path: str = None, period_ms: int = 50):
        self.index = index
        self.proc = None
        self.period_ms = period_ms
        self.skip = 0
        self.path = path or os.path.join(tempfile.mkdtemp(prefix="ggb_clocks_"), f"clocks_gpu{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)], stdout=self.f,
                stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 10.0 and self.proc.poll() is None:
                with open(self.path) as fh:
                    n = sum(1 for line in fh if line.endswith("\n"))
                if n > 0:
                    self.skip = n
                    break
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = open(self.path).readlines()
        # the samples of the timed region; if it was shorter than one period, the one just before it
        lines = lines[self.skip:] if len(lines) > self.skip else lines[-1:]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM traffic per algorithmic byte, dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture
# (--set full, cold caches) over the launch's algorithmic bytes, for the split_int8 kernels of the
# committed profiling workloads: ar16-n600 (N_l = 97, the one-M-tile kernel, and the radial product)
# and ar16-n400-l160 (N_l = 161, the two-M-tile kernel).  The ensemble is too large to capture whole;
# its traffic is estimated group by group from these ratios (orbital traffic grows in proportion to
# N_r N_l columns; W in proportion to N_r^2 N_l).  The two-M-tile angular ratios come from the capture
# with basis reuse (first half: kept vectors in, orbitals out; second half: orbitals in and out, kept
# vectors out); the one-M-tile ones from a capture of the two-product form of both halves.
MEASURED_TRAFFIC_RATIO = {
    ("split_int8", "radial", 1): 554.63 / 514.02, ("split_int8", "radial", 2): 554.63 / 514.02,
    ("split_int8", "angular_first", 1): 212.18 / 268.19, ("split_int8", "angular_second", 1): 241.05 / 268.19,
    ("split_int8", "angular_first", 2): (149.01 + 104.49) / 296.76,
    ("split_int8", "angular_second", 2): (150.63 + 279.10) / 445.15,
}
TRAFFIC_SOURCE = ("per group: algorithmic bytes x (DRAM bytes / algorithmic bytes) of an ncu capture of the same "
                  "kernel on ar16-n600 (one M tile, radial) or ar16-n400-l160 (two M tiles)")


def measured_traffic(runs, groups, precision, phase, theta_reuse: bool = False):
    """Estimated DRAM bytes of one launch of `phase` (all groups), or None without a capture."""
    total = 0.0
    for members in groups:
        sub = phase_traffic(runs, [members], precision, theta_reuse)[phase]["bytes"]
        m_tiles = 1 if runs[members[0]].n_l <= 128 else 2
        ratio = MEASURED_TRAFFIC_RATIO.get((precision, phase, m_tiles))
        if ratio is None:
            return None
        total += sub * ratio
    return total


def chain_products(run) -> int:
    """Products of one angular half-step: the theta form's two (to the P coupling's eigenbasis and
    back); the reference chain's active couplings + 1 (adjacent rotations pre-multiplied): FF with
    N_har >= 4, FP and D with N_har >= 3 when Hartree is on, always P."""
    if getattr(run, "angular", "reference") == "theta":
        return 2
    h = run.use_hartree == 1 and run.target_id > 0
    k = 1 + (2 if h and run.n_har >= 3 else 0) + (1 if h and run.n_har >= 4 else 0)
    return k + 1


def phase_traffic(runs, groups, precision, theta_reuse: bool = False):
    """Algorithmic bytes and flops of each phase of one step, summed over the grid groups.

    radial: W once per group (16 B per complex FP64, 12 B as three BF16 planes per real part, 8 B as
    four int8 slices per real part) + the orbital operand in (cb B per complex value; the int8 form
    reads its 12 B of Xr, Xi, -Xi slices) + the result out (cb B); flops 8 N_r^2 N_l per orbital
    column (the split products are not counted).
    angular half: orbitals in and out (cb B each); (#chain GEMMs) x 4 N_l^2 N_r flops per column.
    cb = 16 B for the FP64 and int8 forms (complex128 orbitals), 8 B for the BF16 form.
    theta_reuse (split_int8, theta form, ggb_set_theta_reuse): the first half runs one product
    fewer (it starts from the node-basis vectors the second half kept), and the second half also
    writes those vectors (cb B per value).
    """
    cb = 8 if precision == "split_bf16" else 16
    xin = 12 if precision == "split_int8" else cb
    wb = W_BYTES[precision]
    out = {k: dict(bytes=0.0, flops=0.0) for k in ("radial", "angular_first", "angular_second")}
    for members in groups:
        r0 = runs[members[0]]
        n_r, n_l = r0.n_r, r0.n_l
        cols = sum(runs[i].n_orb for i in members)
        elems = n_r * n_l * cols
        n_gemm = chain_products(r0)
        out["radial"]["bytes"] += wb * n_r * n_r * n_l + (xin + cb) * elems
        out["radial"]["flops"] += 8.0 * n_r * n_r * n_l * cols
        reuse = theta_reuse and precision == "split_int8" and getattr(r0, "angular", "reference") == "theta"
        for k in ("angular_first", "angular_second"):
            out[k]["bytes"] += 2 * cb * elems
            out[k]["flops"] += (n_gemm - (1 if reuse and k == "angular_first" else 0)) * 4.0 * n_l * n_l * n_r * cols
        if reuse:
            out["angular_second"]["bytes"] += cb * elems
    return out


def phase_bound_seconds(tf, hbm_gbs: float, arith_tera: float) -> float:
    """Roofline time of one step whose phases run one after another: sum over phases of
    max(algorithmic bytes / HBM peak, algorithmic flops / arithmetic peak)."""
    return sum(max(v["bytes"] / (hbm_gbs * 1e9), v["flops"] / (arith_tera * 1e12)) for v in tf.values())


# ---------------------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------------------

def max_over_ranks(ms: float, dist: bool, device: str = "cuda") -> float:
    """The slowest rank's timed milliseconds; every rank calls this once, at the same point."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_step: int, steps: int, ms_max: float) -> float:
    """Orbital-steps/s of the whole job: every replica's units over the slowest replica's time."""
    return world * units_per_step * steps / (ms_max / 1e3)


def run_ours(args, rank, world, dist):
    import torch
    from ggbtddft_b200.engine import TimePropagation
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    n_t = args.warmup + args.steps + 8
    from ggbtddft_b200 import problems as P
    P.reset_setup_seconds()
    t_setup = time.perf_counter()
    runs, precision, desc = workload_runs(args.workload, n_t, device="cuda", split=args.precision,
                                          angular=args.angular, potentials=args.potentials)
    setup = dict(seconds=round(time.perf_counter() - t_setup, 3),
                 parts={k: round(v, 3) for k, v in P.SETUP_SECONDS.items()}, device="cuda",
                 how="wall clock of building the workload's inputs, excluded from the step rate: ground-state "
                     "SCF per grid (device-resident loop, batched eigensolves), radial Crank-Nicolson "
                     "propagators per grid (batched linear solves on the GPU), angular eigensystems (host, "
                     "closed form), the rest is the laser fields and initial orbitals")
    units_per_step = sum(r.n_orb for r in runs)
    tp = TimePropagation(runs, precision=precision, per_l=True, n_t=n_t,
                         autotune=bool(args.autotune) and precision == "split_int8",
                         angular_fp64=args.angular_arith == "fp64", theta_reuse=bool(args.theta_reuse))
    # basis reuse is active where the int8 angular chain runs the theta form
    reuse = tp.theta_reuse and not tp.angular_fp64 and args.angular == "theta"
    if precision == "split_int8":
        desc = dict(desc, angular_products="FP64 tensor cores (mma.sync m8n8k4 f64)" if tp.angular_fp64 else
                    "int8 slice products on tcgen05 (31-bit operands, exact int32 accumulation)")
        if args.angular == "theta" and not tp.angular_fp64:
            desc = dict(desc, basis_reuse=("on: each first half starts from the node-basis vectors the previous "
                                           "second half kept (3 angular products per step instead of 4)")
                        if reuse else "off: 4 angular products per step")
    stream = torch.cuda.Stream()
    h = stream.cuda_stream
    hbm_peak, _, peak_kind = read_peaks()
    peaks = compute_peaks(h)

    # warm-up (also captures the step graph)
    tp.step(args.warmup, h)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev, args.clocks_csv) as clk:
        e0.record(stream)
        tp.step(args.steps, h)
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    st, msg = tp.status()
    if st != 0:
        raise SystemExit(f"device status {st}: {msg}")
    ms_max = max_over_ranks(ms, dist)
    value = whole_job_rate(world, units_per_step, args.steps, ms_max)

    # per-kernel durations (each phase launched alone, CUDA events on the launching stream)
    reps = 20
    phase_ms = {}
    for ph, name in ((1, "radial"), (0, "angular_first"), (2, "angular_second"), (3, "finalize")):
        tp.launch_phase(ph, h)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            tp.launch_phase(ph, h)
        b.record(stream)
        torch.cuda.synchronize()
        phase_ms[name] = a.elapsed_time(b) / reps
    tp.close()

    # end to end through the C ABI from host buffers: every run's orbitals and field from pinned
    # (page-locked) host memory, filled before the timed region; the observables into host arrays
    if not args.e2e:
        e2e_value, h2d, d2h = None, 0, 0
    tp2 = TimePropagation(runs, precision=precision, per_l=True, n_t=n_t, tuning=tp.tuning,
                          angular_fp64=tp.angular_fp64, theta_reuse=tp.theta_reuse) if args.e2e else None
    if tp2 is not None:
        pin_x = [torch.from_numpy(np.ascontiguousarray(r.x0, dtype=np.complex128)).pin_memory().numpy()
                 for r in runs]
        pin_E = [torch.from_numpy(np.ascontiguousarray(r.E, dtype=np.float64)).pin_memory().numpy() for r in runs]
        tp2.step(args.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h2d = 0
        for i in range(len(runs)):
            tp2.set_orbitals(i, pin_x[i])
            tp2.set_field(i, pin_E[i])
            h2d += pin_x[i].nbytes + pin_E[i].nbytes
        tp2.step(args.steps)
        d2h = 0
        for i in range(len(runs)):
            o = tp2.observables(i, per_l=True, n_steps=args.steps)
            d2h += o["dipole"].nbytes + o["acceleration"].nbytes + o["norm"].nbytes
        e2e_s = time.perf_counter() - t0
        tp2.close()
        e2e_value = world * units_per_step * args.steps / e2e_s

    # roofline of the dominant kernel (the phase with the longest device time per step), by the
    # algorithmic bytes and flops of each phase: frac = max(bytes / t / HBM peak, flops / t / the
    # precision's peak).  The peaks of the arithmetic are this GPU's, measured by the library's own
    # microbenchmarks before the timed region; the HBM peak is the measured copy bandwidth.  The int8
    # form's executed slice products (10 per algorithmic real product) are a secondary figure.
    tf = phase_traffic(runs, tp.groups, precision, reuse)
    dom = max(("radial", "angular_first", "angular_second"), key=lambda k: phase_ms[k])
    arith_peak = {"fp64": peaks["fp64_tflops"], "split_int8": peaks["int8_tops"],
                  "split_bf16": read_peaks()[1]}[precision]
    arith_unit = {"fp64": "TFLOP/s (FP64 FMA)", "split_int8": "TOP/s (tcgen05 kind::i8)",
                  "split_bf16": "TFLOP/s (bf16, cuBLAS-measured)"}[precision]
    sp = SPLIT_PRODUCTS.get(precision, 1)
    # each phase's arithmetic against the peak of the unit it runs on (the int8 form with FP64
    # angular products: the angular phases against the FP64 peak)
    phase_peak = {k: arith_peak for k in ("radial", "angular_first", "angular_second")}
    phase_split = {k: sp for k in phase_peak}
    if tp.angular_fp64:
        for k in ("angular_first", "angular_second"):
            phase_peak[k], phase_split[k] = peaks["fp64_tflops"], 1
    kernels = {}
    for k in ("radial", "angular_first", "angular_second"):
        sec = phase_ms[k] / 1e3
        kernels[k] = dict(ms=round(phase_ms[k], 5), algorithmic_bytes=int(tf[k]["bytes"]),
                          algorithmic_flops=int(tf[k]["flops"]),
                          gbs=round(tf[k]["bytes"] / sec / 1e9, 1), tflops=round(tf[k]["flops"] / sec / 1e12, 3),
                          hbm_frac=round(tf[k]["bytes"] / sec / 1e9 / hbm_peak, 4),
                          arith_frac=round(tf[k]["flops"] / sec / 1e12 / phase_peak[k], 4))
        if precision != "fp64" and phase_split[k] > 1:
            kernels[k]["tensor_frac_executed"] = round(phase_split[k] * tf[k]["flops"] / sec / 1e12 / phase_peak[k], 4)
    kernels["finalize"] = dict(ms=round(phase_ms["finalize"], 5))
    names = {"radial": {"fp64": "k_radial_fp64", "split_bf16": "k_radial_tc_persistent (tcgen05 kind::f16)",
                        "split_int8": "k_radial_i8 (tcgen05 kind::i8, int8 slices, int32 accumulation)"},
             "angular": {"fp64": "k_angular_fp64 (mma.sync f64)", "split_bf16": "k_angular_tc (tcgen05 kind::f16)",
                         "split_int8": ("k_angular_fp64 (mma.sync f64)" if tp.angular_fp64 else
                                        "k_angular_i8 (tcgen05 kind::i8 chain, FP64 phases)")}}
    d = kernels[dom]
    kname = names["radial" if dom == "radial" else "angular"][precision]
    est = measured_traffic(runs, tp.groups, precision, dom, reuse)
    roofline = dict(bound="hbm", kernel=f"{dom} ({kname})", achieved=d["gbs"], peak=hbm_peak, unit="GB/s",
                    frac=d["hbm_frac"], traffic=None if est is None else int(est),
                    traffic_source=None if est is None else TRAFFIC_SOURCE,
                    peak_kind=f"{peak_kind} hbm_gbs", dominant_by_time=dom,
                    peaks_measured=dict(hbm_gbs=hbm_peak, fp64_tflops=round(peaks["fp64_tflops"], 2),
                                        fp64_fma_tflops=round(peaks["fp64_fma_tflops"], 2),
                                        fp64_mma_tflops=round(peaks["fp64_mma_tflops"], 2),
                                        int8_tops=round(peaks["int8_tops"], 1),
                                        how="FP64 FMA, FP64 mma.sync and tcgen05 kind::i8 microbenchmarks of "
                                            "this library (ggb_measure_peaks, ggb_measure_peak_fp64_mma; the FP64 "
                                            "roofline takes the larger FP64 figure); HBM: copy bandwidth of "
                                            "MEASURED_PEAKS.json"),
                    kernels=kernels)
    if d["arith_frac"] > d["hbm_frac"]:
        fp64_unit = tp.angular_fp64 and dom != "radial"
        roofline.update(bound="tensor" if precision != "fp64" else "fp64", achieved=d["tflops"],
                        peak=round(phase_peak[dom], 2), unit=arith_unit if not fp64_unit else "TFLOP/s (FP64)",
                        frac=d["arith_frac"], peak_kind="measured (ggb_measure_peaks)")
    if "tensor_frac_executed" in d:
        roofline["tensor_frac_executed"] = d["tensor_frac_executed"]
    # the whole step against its own bound: the phases run one after another, so the bound is the
    # sum over phases of each phase's own bound (algorithmic bytes at the HBM peak or flops at the
    # arithmetic peak, whichever takes longer)
    step_bytes = sum(tf[k]["bytes"] for k in tf)
    step_flops = sum(tf[k]["flops"] for k in tf)
    step_s = ms_max / args.steps / 1e3 / world
    step_bound = sum(phase_bound_seconds({k: v}, hbm_peak, phase_peak.get(k, arith_peak)) for k, v in tf.items())
    roofline["step"] = dict(ms=round(ms_max / args.steps, 4), algorithmic_bytes=int(step_bytes),
                            algorithmic_flops=int(step_flops), bound_ms=round(1e3 * step_bound, 4),
                            frac=round(step_bound / step_s, 4),
                            bound_how="sum over phases of max(bytes / HBM peak, flops / arithmetic peak)")
    # the same runs stepped one at a time in the plain FP64 form (per-instance launches), on this GPU,
    # with that form's own roofline (its step's algorithmic bytes and flops against the HBM and the
    # measured FP64 peak)
    fp64_inst = None
    if args.compare_fp64 and (len(runs) > 1 or precision != "fp64"):
        from ggbtddft_b200.engine import group_runs
        total_s, units, bound_s = 0.0, 0, 0.0
        for members in group_runs(runs):
            one = TimePropagation([runs[members[0]]], precision="fp64", per_l=True, n_t=n_t)
            one.step(args.warmup, h)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k = min(args.steps, 64)
            a.record(stream)
            one.step(k, h)
            b.record(stream)
            torch.cuda.synchronize()
            per_step = a.elapsed_time(b) / 1e3 / k
            one.close()
            t1 = phase_traffic([runs[members[0]]], [[0]], "fp64")
            bound_s += len(members) * phase_bound_seconds(t1, hbm_peak, peaks["fp64_tflops"])
            total_s += per_step * len(members)
            units += sum(runs[i].n_orb for i in members)
        rate = units / total_s
        fp64_inst = dict(value=rate, unit="orbital-steps/s",
                         how="each run of the workload stepped alone in the FP64 form (one time per grid, "
                             "weighted by the runs on it), same GPU", speedup=round(value / rate, 2),
                         roofline_frac=round(bound_s / total_s, 4),
                         roofline_how="per run-step: sum over its phases of max(algorithmic bytes / HBM peak, "
                                      "algorithmic flops / measured FP64 peak), over the measured time, weighted "
                                      "like the rate")
    return dict(value=value, ms=ms_max, units_per_step=units_per_step, desc=desc, precision=precision,
                clocks=clk.summary(), roofline=roofline,
                e2e=None if e2e_value is None else dict(
                    value=e2e_value, unit="orbital-steps/s", h2d_bytes_per_step=int(h2d / args.steps),
                    d2h_bytes_per_step=int(d2h / args.steps),
                    how="wall clock through the C ABI: every run's orbitals and field copied in from pinned host "
                        "memory, the K steps, every run's per-l dipole, acceleration and norm series copied out"),
                gpu_launches=args.steps * sum(LAUNCHES_PER_GROUP_STEP[precision] +
                                              (4 if runs[m[0]].angular == "theta" and runs[m[0]].n_har > 4
                                               and runs[m[0]].use_hartree else 0) for m in tp.groups),
                fp64_per_instance=fp64_inst, setup=setup)


def cpu_port_rate(runs, n_steps: int, warmup: int = 1):
    """Orbital-steps/s and seconds of the CPU oracle on ``n_steps`` steps of the first of ``runs``."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle.step_oracle import OracleProblem, OracleState
    r = runs[0]
    prob = OracleProblem(r=r.grid.r, drdx=r.grid.drdx, P=r.grid.P, W=r.W, V=r.V, D=r.D, x0=r.x0, m=r.m_active,
                         occ=r.occ, rho_frozen=r.rho_frozen, E=r.E, dt=r.dt, n_har=r.n_har,
                         use_hartree=r.use_hartree, target_id=r.target_id, xc_correlation=r.xc_correlation)
    st = OracleState(prob)
    st.init_potentials()
    for t in range(warmup):
        st.step(t)
    t0 = time.perf_counter()
    for t in range(warmup, warmup + n_steps):
        st.step(t)
    dt = time.perf_counter() - t0
    return r.n_orb * n_steps / dt, dt


def cpu_workload_rate(name: str, n_steps: int, warmup: int, angular: str = "theta", potentials: str = "adiabatic"):
    """The CPU oracle on a bounded sample of the workload: one run per grid group, ``n_steps`` timed
    steps each (after ``warmup``), weighted by the runs in its group.  Returns (orbital-steps/s of the
    whole workload, seconds timed, estimated CPU seconds of one whole-workload step, sample text, the
    workload's description)."""
    units, step_s, timed, parts, desc = 0.0, 0.0, 0.0, [], None
    for idx, count, label in workload_groups(name):
        runs, _, desc = workload_runs(name, n_steps + warmup + 8, only=[idx], angular=angular, potentials=potentials)
        runs = runs[:1] if idx == 0 else runs
        rate, sec = cpu_port_rate(runs, n_steps, warmup)
        per_step = sec / n_steps
        units += count * runs[0].n_orb
        step_s += count * per_step
        timed += sec
        parts.append(f"{label} (run {idx}, weight {count}): {1e3 * per_step:.0f} ms/step")
    text = (f"oracle (FP64 NumPy restatement of the reference loop), one run per grid group, {n_steps} steps "
            f"each after {warmup} warm-up, weighted by the runs per group; " + "; ".join(parts))
    return units / step_s, timed, step_s, text, desc


# the reference arm's bounded sample: at most this many timed steps per grid group, after at most two
# warm-up steps
REF_SAMPLE_STEPS = 6


def run_reference(args, rank, world):
    """CPU arm: the oracle (FP64 NumPy restatement of the reference loop) on the host cores, on a
    bounded sample of the workload (one run per grid group, weighted by the group's runs)."""
    if rank != 0:
        return None
    n, w = min(args.steps, REF_SAMPLE_STEPS), min(args.warmup, 2)
    rate, timed, step_s, text, desc = cpu_workload_rate(args.workload, n, w, args.angular, args.potentials)
    return dict(value=rate, desc=desc, seconds=timed, step_seconds=step_s, steps_timed=n, sample=text)


# ---------------------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=40)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split_int8", choices=["split_int8", "split_bf16"],
                    help="form of the split-precision workloads (FP64 workloads end in -fp64)")
    ap.add_argument("--cpu-sample-steps", type=int, default=4,
                    help="oracle steps timed per grid group for cpu_baseline (0: skip)")
    ap.add_argument("--angular", default=DEFAULT_ANGULAR, choices=["reference", "theta"],
                    help="angular step of every run: theta (one phase per half-step at the Gauss nodes) or the "
                         "reference's coupling chain")
    ap.add_argument("--potentials", default=DEFAULT_POTENTIALS, choices=sorted(POTENTIALS),
                    help="how the runs' potentials evolve: " + "; ".join(f"{k}: {v}" for k, v in POTENTIALS.items()))
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: radial tiles of the int8 form from the autotuner (shipped B200 tunings; times the "
                         "candidates of a group shape it has not seen)")
    ap.add_argument("--angular-arith", default=DEFAULT_ANGULAR_ARITH, choices=["int8", "fp64"],
                    help="split_int8 form: the angular products as int8 slice products on tcgen05 (int8) or on "
                         "the FP64 tensor cores with mma.sync (fp64); the radial product stays int8")
    ap.add_argument("--theta-reuse", type=int, default=1,
                    help="split_int8 theta form: 1 starts each step's first angular half from the node-basis "
                         "vectors kept by the previous second half (one product instead of two; "
                         "ggb_set_theta_reuse), 0 runs both products of every half")
    ap.add_argument("--clocks-csv", default=None,
                    help="where to keep the nvidia-smi clock samples of the timed region (default: a temp dir)")
    ap.add_argument("--e2e", type=int, default=1, help="also measure the end-to-end (host buffers) number")
    ap.add_argument("--compare-fp64", type=int, default=1,
                    help="also time the runs one at a time in the FP64 form (per-instance baseline)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = world > 1
    metric = "orbital-steps/s (batched time step, one B200)"
    cores = os.cpu_count()

    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if rank == 0:
            line = dict(metric=metric, value=res["value"], unit="orbital-steps/s", n_gpus=args.gpus,
                        steps=args.steps, warmup=args.warmup, ms_per_step=1e3 * res["step_seconds"],
                        higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
                        data="synthetic (seeded laser parameters; LDA ground state computed at set-up)",
                        config=dict(res["desc"], l2="n/a (CPU)"), impl="reference",
                        cpu_baseline=dict(value=res["value"], unit="orbital-steps/s", cores=cores, kind="port",
                                          sample=res["sample"]),
                        e2e=dict(value=res["value"], unit="orbital-steps/s", h2d_bytes_per_step=0,
                                 d2h_bytes_per_step=0))
            print(json.dumps(line))
        return

    import torch
    if dist:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = run_ours(args, rank, world, dist)
    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample_steps > 0:
        rate, timed, _, text, _ = cpu_workload_rate(args.workload, args.cpu_sample_steps, 1, args.angular,
                                                    args.potentials)
        cpu = dict(value=rate, unit="orbital-steps/s", cores=cores, kind="port", sample=f"{text}; {timed:.1f} s timed")
    if rank == 0:
        desc = dict(res["desc"])
        desc["l2"] = "inputs larger than L2 (radial propagators stream from HBM every step)"
        desc["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
        line = dict(metric=metric, value=res["value"], unit="orbital-steps/s", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=res["ms"] / args.steps, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype={"fp64": "f64", "split_bf16": "f32+split-bf16", "split_int8": "f64+split-int8"}[res["precision"]],
                    data="synthetic (seeded laser parameters; LDA ground state computed at set-up)", config=desc,
                    roofline=res["roofline"], cpu_baseline=cpu, e2e=res["e2e"], clocks=res["clocks"],
                    gpu_launches=res["gpu_launches"], fp64_per_instance=res["fp64_per_instance"],
                    reference_main_cu_b200=reference_binary_record(), setup=res["setup"])
        print(json.dumps(line))
    if dist:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
