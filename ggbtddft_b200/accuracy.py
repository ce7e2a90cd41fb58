"""Error of the split-precision form against the FP64 form, per result, over a full pulse.

    python -m ggbtddft_b200.accuracy --config argon [--precision split_int8] [--steps N] [--frozen]
                                     [--sensitivity 1e-10] [--out report.json]

Both forms run the same inputs on the GPU (the FP64 form is the one held to the reference to 1e-10).
Reported: norm drift (max |norm_split - norm_fp64| per orbital), relative L2 error of the total
dipole and of the total dipole acceleration <cos(theta)/r^2>, and the relative error of every
harmonic intensity up to the semiclassical cutoff, from the HHG spectrum of the total dipole
computed with the reference's recipe (spectrum.py).

Conditioning: with Hartree and exchange in the loop the time step feeds the density of one step
into the potential of the next, and that feedback amplifies small differences (in the FP64 form
too: a 1e-10 change of the initial orbitals of the argon configuration changes its dipole by tens
of per cent within a few thousand steps).  ``--sensitivity eps`` runs the FP64 form a second time
from initial orbitals perturbed by eps (relative, seeded) and reports the same errors for that pair:
the floor below which no arithmetic other than the identical FP64 sequence can agree with it.
``--frozen`` runs the same configuration with the potentials frozen at the ground state
(USE_HARTREE = 0), a linear and well-conditioned propagation on the same grid, orbitals and pulse.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time
from typing import Optional

import numpy as np

from . import problems as P
from . import spectrum as S
from .engine import TimePropagation

IONISATION_POTENTIAL = {"H": 0.5, "He": 0.9036, "Ar": 0.5792}   # Ha (experimental first Ip)


def _run(run: P.RunInputs, precision: str, n_steps: int, chunk: int = 4096, angular_fp64: bool = False,
         theta_reuse: bool = True):
    tp = TimePropagation([run], precision=precision, per_l=True, n_t=n_steps, angular_fp64=angular_fp64,
                         theta_reuse=theta_reuse)
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


def perturb_orbitals(run: P.RunInputs, eps: float, seed: int = 1) -> P.RunInputs:
    """Initial orbitals + eps * max|x| * complex Gaussian noise, renormalised per orbital."""
    rng = np.random.default_rng(seed)
    x = run.x0 + eps * np.abs(run.x0).max() * (rng.standard_normal(run.x0.shape)
                                                + 1j * rng.standard_normal(run.x0.shape))
    x = x / np.sqrt((np.abs(x) ** 2).sum(axis=(0, 2)))[None, :, None]
    return dataclasses.replace(run, x0=x)


def _errors(run, ref, tst, atom, e0):
    d_ref = S.total_dipole(ref["dipole"], run.l_active, run.m_active, run.occ)
    d_tst = S.total_dipole(tst["dipole"], run.l_active, run.m_active, run.occ)
    a_ref = (run.occ[None, :, None] * ref["acceleration"]).real.sum(axis=(0, 1))
    a_tst = (run.occ[None, :, None] * tst["acceleration"]).real.sum(axis=(0, 1))
    w, s_ref = S.hhg_spectrum(d_ref, run.dt)
    _, s_tst = S.hhg_spectrum(d_tst, run.dt)
    q_cut = S.cutoff_order(IONISATION_POTENTIAL[atom], e0, run.omega0)
    herr = S.harmonic_errors(s_tst, s_ref, w, run.omega0, q_cut)
    return dict(norm_drift_max=float(np.abs(tst["norm"] - ref["norm"]).max()),
                dipole_rel_l2=float(np.linalg.norm(d_tst - d_ref) / np.linalg.norm(d_ref)),
                acceleration_rel_l2=float(np.linalg.norm(a_tst - a_ref) / np.linalg.norm(a_ref)),
                harmonic_rel_err=herr.tolist(), odd_harmonic_rel_err_max=float(herr[0::2].max()),
                harmonic_rel_err_max=float(herr.max()))


def compare_forms(run: P.RunInputs, atom: str, precision: str = "split_int8", n_steps: Optional[int] = None,
                  e0: Optional[float] = None, sensitivity: float = 0.0, angular_fp64: bool = False,
                  theta_reuse: bool = True) -> dict:
    """``angular_fp64``: the split form with its angular products on the FP64 tensor cores;
    ``theta_reuse`` = False: the split theta form without basis reuse (ggb_set_theta_reuse)."""
    n = run.n_t if n_steps is None else n_steps
    ref = _run(run, "fp64", n)
    tst = _run(run, precision, n, angular_fp64=angular_fp64, theta_reuse=theta_reuse)
    e0 = float(np.abs(run.E).max()) if e0 is None else e0
    fp64_self = None
    if sensitivity > 0:
        pert = _run(perturb_orbitals(run, sensitivity), "fp64", n)
        fp64_self = dict(eps=sensitivity, **{k: v for k, v in _errors(run, ref, pert, atom, e0).items()
                                             if k != "harmonic_rel_err"})
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
        config=run.name, precision=precision, theta_reuse=bool(theta_reuse), steps=n, dt=run.dt,
        omega0=run.omega0, cutoff_order=q_cut,
        use_hartree=int(run.use_hartree), fp64_self_sensitivity=fp64_self,
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


def compare_ensemble(n_steps: int, precision: str = "split_int8", n_runs: int = 64, seed: int = 0,
                     sensitivity: float = 0.0) -> dict:
    """Every instance of the argon focal-scan ensemble: the batched `precision` form (all runs in one
    context, grid groups on concurrent streams) against each run stepped alone in the FP64 form, over
    the first `n_steps` steps of its pulse.  Reports, per instance, the relative L2 difference of the
    total dipole and the largest orbital-norm difference (a window this short has no harmonic
    spectrum; the full pulses would take hours in the per-instance FP64 form).  With ``sensitivity``
    > 0 each run is also stepped in FP64 from orbitals perturbed by that relative amount, and the
    same two numbers are reported for that pair: the FP64 self-sensitivity of each instance over the
    same window."""
    runs = P.argon_ensemble(n_runs, seed=seed, n_steps=n_steps, device="cuda")
    tp = TimePropagation(runs, precision=precision, per_l=True, n_t=n_steps)
    done = 0
    while done < n_steps:
        k = min(4096, n_steps - done)
        tp.step(k)
        done += k
    batched_status = tp.status()
    per = []
    for i, r in enumerate(runs):
        tst = tp.observables(i, per_l=True, n_steps=n_steps)
        ref = _run(r, "fp64", n_steps)
        d_ref = S.total_dipole(ref["dipole"], r.l_active, r.m_active, r.occ)
        d_tst = S.total_dipole(tst["dipole"], r.l_active, r.m_active, r.occ)
        row = dict(run=i, n_r=r.n_r, l_max=r.n_l - 1,
                   dipole_rel_l2=float(np.linalg.norm(d_tst - d_ref) / np.linalg.norm(d_ref)),
                   norm_drift_max=float(np.abs(tst["norm"] - ref["norm"]).max()),
                   fp64_status=ref["status"][0])
        if sensitivity > 0:
            pert = _run(perturb_orbitals(r, sensitivity), "fp64", n_steps)
            d_p = S.total_dipole(pert["dipole"], r.l_active, r.m_active, r.occ)
            row["fp64_self_dipole_rel_l2"] = float(np.linalg.norm(d_p - d_ref) / np.linalg.norm(d_ref))
            row["fp64_self_norm_drift_max"] = float(np.abs(pert["norm"] - ref["norm"]).max())
        per.append(row)
    tp.close()
    return dict(config=f"argon ensemble, {n_runs} runs (seed {seed})", precision=precision, steps=n_steps,
                batched_status=batched_status, per_instance=per,
                dipole_rel_l2_max=max(q["dipole_rel_l2"] for q in per),
                dipole_rel_l2_median=float(np.median([q["dipole_rel_l2"] for q in per])),
                norm_drift_max=max(q["norm_drift_max"] for q in per),
                fp64_self_sensitivity=None if sensitivity <= 0 else dict(
                    eps=sensitivity, dipole_rel_l2_max=max(q["fp64_self_dipole_rel_l2"] for q in per),
                    dipole_rel_l2_median=float(np.median([q["fp64_self_dipole_rel_l2"] for q in per]))))


def _run_totals(run: P.RunInputs, n_steps: int, chunk: int = 8192):
    """FP64 form, one run, totals over l only (per-l series of long fine-step runs would take GBs)."""
    tp = TimePropagation([run], precision="fp64", per_l=False, n_t=n_steps)
    t0 = time.perf_counter()
    done = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        tp.step(k)
        done += k
    obs = tp.observables(0, per_l=False, n_steps=n_steps)
    st, msg = tp.status()
    tp.close()
    d = (run.occ[:, None] * obs["dipole"].real).sum(axis=0)
    return dict(dipole=d, norm=obs["norm"], seconds=time.perf_counter() - t0, status=(st, msg))


def sensitivity_sweep(variants=((0.02, 4), (0.01, 4), (0.005, 4), (0.02, 3), (0.02, 2)), eps: float = 1e-10,
                      windows: int = 10) -> dict:
    """Where the argon LDA self-sensitivity comes from: for each (dt, N_har) the FP64 form is run twice
    over the whole pulse (same physical time), from the ground state and from it perturbed by ``eps``,
    and the growth of the difference is recorded per tenth of the pulse.  A growth rate that falls
    with dt is a property of the time stepping (potentials lagging one step behind the orbitals);
    one that does not is a property of the equations.  N_har = 2 keeps only the dipole Hartree term
    (the S phase, which carries the monopole Hartree and exchange changes, runs only for N_har >= 3;
    couplingS.cuh:49), N_har = 3 adds S and the quadrupole, N_har = 4 the octupole.
    Also reported: the dipole of each finer step against the dt = 0.02 run at the common times
    (time-step convergence of the trajectory itself)."""
    laser = P.LaserSpec(1.4e14, 800.0, 10.0, 0.0)
    gs_cache: dict = {}
    rows, by_dt = [], {}
    for dt, n_har in variants:
        run = P.baseline_run("Ar", 600, 300.0, 96, dt, laser, 60.0, device="cuda", gs_cache=gs_cache)
        run = dataclasses.replace(run, n_har=n_har, name=f"{run.name}-dt{dt}-nhar{n_har}")
        n = run.n_t
        ref = _run_totals(run, n)
        pert = _run_totals(perturb_orbitals(run, eps), n)
        d_r, d_p = ref["dipole"], pert["dipole"]
        scale = float(np.abs(d_r).max())
        edges = np.linspace(0, n, windows + 1).astype(int)
        growth = [float(np.abs(d_p[a:b] - d_r[a:b]).max() / scale) for a, b in zip(edges[:-1], edges[1:])]
        rows.append(dict(dt=dt, n_har=n_har, steps=n, seconds=ref["seconds"] + pert["seconds"],
                         status=[ref["status"][0], pert["status"][0]], eps=eps,
                         diff_per_tenth_of_pulse=growth,
                         dipole_rel_l2=float(np.linalg.norm(d_p - d_r) / np.linalg.norm(d_r)),
                         norm_diff_max=float(np.abs(pert["norm"] - ref["norm"]).max())))
        if n_har == 4:
            by_dt[dt] = d_r
    conv = {}
    if 0.02 in by_dt:
        base = by_dt[0.02]
        for dt, d in by_dt.items():
            if dt == 0.02:
                continue
            k = int(round(0.02 / dt))
            sub = d[k - 1::k][:base.size]
            m = min(sub.size, base.size)
            conv[str(dt)] = float(np.linalg.norm(sub[:m] - base[:m]) / np.linalg.norm(base[:m]))
    return dict(config="Ar LDA, N_r 600, r_max 300, l_max 96, 800 nm 1.4e14 10-cycle sin^2", variants=rows,
                dipole_vs_dt002_rel_l2=conv)


def _batched_totals(runs, precision: str, n_steps: int, chunk: int = 4096, angular_fp64: bool = False):
    """All runs in one context (grid groups on concurrent streams); occupation-weighted total dipole
    (sum over every l) and norms of each run, and the seconds the stepping took."""
    tp = TimePropagation(runs, precision=precision, per_l=False, n_t=n_steps, angular_fp64=angular_fp64)
    t0 = time.perf_counter()
    done = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        tp.step(k)
        done += k
    st = tp.status()
    out = []
    for i, r in enumerate(runs):
        o = tp.observables(i, per_l=False, n_steps=n_steps)
        out.append(dict(dipole=(r.occ[:, None] * o["dipole"].real).sum(axis=0), norm=o["norm"]))
    tp.close()
    return out, time.perf_counter() - t0, st


def compare_hhe_ensemble(precision: str = "split_int8", n_runs: int = 256, seed: int = 0,
                         angular: str = "reference", angular_fp64: bool = False) -> dict:
    """The 256-run H/He focal scan over every run's whole pulse: the batched ``precision`` form against
    the batched FP64 form (the same runs, grid groups and field samples).  Each run's pulse is
    followed by zero field up to the longest pulse; each run's spectrum is taken over its own
    pulse.  Reported per instance: the largest relative error of the harmonic intensities up to its
    semiclassical cutoff, the dipole L2 difference and the norm difference.  The total dipole is
    the occupation-weighted sum over every l (the reference's analysis leaves out l = l_kso and
    the top four l; both forms are summed the same way here)."""
    runs = P.hhe_ensemble(n_runs, seed=seed, device="cuda")
    if angular != "reference":
        runs = [dataclasses.replace(r, angular=angular) for r in runs]
    n = max(r.n_t for r in runs)
    ref, t_ref, st_ref = _batched_totals(runs, "fp64", n)
    tst, t_tst, st_tst = _batched_totals(runs, precision, n, angular_fp64=angular_fp64)
    per = []
    for i, r in enumerate(runs):
        m = r.n_t
        atom = "H" if r.name.startswith("H-") else "He"
        d_r, d_t = ref[i]["dipole"][:m], tst[i]["dipole"][:m]
        w, s_r = S.hhg_spectrum(d_r, r.dt)
        _, s_t = S.hhg_spectrum(d_t, r.dt)
        e0 = float(np.abs(r.E).max())
        q_cut = S.cutoff_order(IONISATION_POTENTIAL[atom], e0, r.omega0)
        herr = S.harmonic_errors(s_t, s_r, w, r.omega0, q_cut)
        per.append(dict(run=i, atom=atom, n_r=r.n_r, l_max=r.n_l - 1, steps=m, cutoff_order=q_cut,
                        harmonic_rel_err_max=float(herr.max()),
                        dipole_rel_l2=float(np.linalg.norm(d_t - d_r) / np.linalg.norm(d_r)),
                        norm_drift_max=float(np.abs(tst[i]["norm"][:, :m] - ref[i]["norm"][:, :m]).max())))
    worst = max(per, key=lambda q: q["harmonic_rel_err_max"])
    return dict(config=f"H/He focal scan, {n_runs} runs (seed {seed}), whole pulses", precision=precision,
                angular=angular, angular_products="FP64 (mma.sync)" if angular_fp64 else "int8 slices", steps_stepped=n, seconds=dict(fp64=t_ref, split=t_tst),
                status=dict(fp64=st_ref, split=st_tst), per_instance=per,
                harmonic_rel_err_max=worst["harmonic_rel_err_max"], worst_instance=worst,
                instances_within_1e3=int(sum(q["harmonic_rel_err_max"] <= 1e-3 for q in per)),
                dipole_rel_l2_max=max(q["dipole_rel_l2"] for q in per),
                norm_drift_max=max(q["norm_drift_max"] for q in per))


def compare_argon_ensemble_full(precision: str = "split_int8", n_runs: int = 64, seed: int = 0,
                                angular: str = "theta", xc_frozen: bool = True, per_rung: int = 1,
                                frozen: bool = False, angular_fp64: bool = False) -> dict:
    """Whole pulses of the argon focal scan: all runs batched in ``precision`` (one context, grid groups
    on concurrent streams, each run followed by zero field up to the longest pulse) against the FP64
    form of ``per_rung`` runs per grid rung, each stepped alone over its own pulse.  Per checked
    instance: the largest relative error of the harmonic intensities up to its cutoff (total dipole
    summed over every l), the dipole L2 difference and the norm difference."""
    dr = P.argon_draws(n_runs, seed)
    runs = P.argon_ensemble(n_runs, seed=seed, device="cuda", xc_frozen=xc_frozen)
    runs = [dataclasses.replace(r, angular=angular, use_hartree=0 if frozen else r.use_hartree) for r in runs]
    n = max(r.n_t for r in runs)
    tst, t_tst, st_tst = _batched_totals(runs, precision, n, angular_fp64=angular_fp64)
    checked = [i for members in dr.grid_groups().values() for i in members[:per_rung]]
    per = []
    t_ref = 0.0
    for i in checked:
        r = runs[i]
        ref, t1, st1 = _batched_totals([r], "fp64", r.n_t)
        t_ref += t1
        m = r.n_t
        d_r, d_t = ref[0]["dipole"][:m], tst[i]["dipole"][:m]
        w, s_r = S.hhg_spectrum(d_r, r.dt)
        _, s_t = S.hhg_spectrum(d_t, r.dt)
        q_cut = S.cutoff_order(IONISATION_POTENTIAL["Ar"], float(np.abs(r.E).max()), r.omega0)
        herr = S.harmonic_errors(s_t, s_r, w, r.omega0, q_cut)
        per.append(dict(run=i, n_r=r.n_r, l_max=r.n_l - 1, steps=m, cutoff_order=q_cut, fp64_status=st1[0],
                        harmonic_rel_err_max=float(herr.max()), harmonic_rel_err=herr.tolist(),
                        dipole_rel_l2=float(np.linalg.norm(d_t - d_r) / np.linalg.norm(d_r)),
                        norm_drift_max=float(np.abs(tst[i]["norm"][:, :m] - ref[0]["norm"][:, :m]).max())))
    pot = "all potentials frozen at the ground state" if frozen else (
        "xc frozen at the ground state" if xc_frozen else "adiabatic")
    return dict(config=f"argon focal scan, {n_runs} runs (seed {seed}), whole pulses, angular {angular}, {pot}",
                precision=precision, steps_stepped=n, seconds=dict(batched=t_tst, fp64_checked=t_ref),
                batched_status=st_tst, per_instance=per,
                harmonic_rel_err_max=max(q["harmonic_rel_err_max"] for q in per),
                instances_within_1e3=int(sum(q["harmonic_rel_err_max"] <= 1e-3 for q in per)),
                dipole_rel_l2_max=max(q["dipole_rel_l2"] for q in per),
                norm_drift_max=max(q["norm_drift_max"] for q in per))


CONFIGS = {
    "hydrogen": ("H", P.config_hydrogen),
    "helium": ("He", P.config_helium),
    "argon": ("Ar", P.config_argon),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="argon", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="split_int8")
    ap.add_argument("--steps", type=int, default=None, help="default: the full pulse")
    ap.add_argument("--frozen", action="store_true", help="potentials frozen at the ground state (USE_HARTREE=0)")
    ap.add_argument("--sensitivity", type=float, default=0.0,
                    help="also run FP64 from initial orbitals perturbed by this relative amount")
    ap.add_argument("--out", default=None)
    ap.add_argument("--ensemble-steps", type=int, default=0,
                    help="instead: every run of the 64-run argon ensemble, batched, against each run alone in "
                         "FP64, over this many steps")
    ap.add_argument("--hhe-ensemble", action="store_true",
                    help="instead: the 256-run H/He ensemble over whole pulses, batched, against batched FP64")
    ap.add_argument("--angular", default="reference", choices=["reference", "theta"])
    ap.add_argument("--argon-ensemble-full", action="store_true",
                    help="instead: whole pulses of the 64-run argon ensemble, batched, against FP64 runs of "
                         "one run per grid rung")
    ap.add_argument("--xc-frozen", action="store_true", help="exchange-correlation held at the ground state")
    ap.add_argument("--per-rung", type=int, default=1, help="--argon-ensemble-full: FP64 runs checked per rung")
    ap.add_argument("--hhe-run", type=int, default=-1,
                    help="instead: run N of the 256-run H/He scan alone, split form against FP64 (with "
                         "--sensitivity: FP64 against FP64 from perturbed orbitals too)")
    ap.add_argument("--argon-run", type=int, default=-1,
                    help="instead: run N of the 64-run argon focal scan alone over its whole pulse, split form "
                         "against FP64 (with --frozen, --xc-frozen and --angular as given)")
    ap.add_argument("--theta-reuse", type=int, default=1,
                    help="split theta form: 1 with basis reuse (the default), 0 both products of every half")
    ap.add_argument("--angular-fp64", action="store_true",
                    help="the split form's angular products on the FP64 tensor cores (ggb_set_angular_fp64)")
    ap.add_argument("--sweep", action="store_true",
                    help="instead: FP64 self-sensitivity of argon LDA for dt in {0.02, 0.01, 0.005} and N_har "
                         "in {2, 3, 4} over the whole pulse")
    args = ap.parse_args(argv)
    if args.argon_ensemble_full:
        rep = compare_argon_ensemble_full(args.precision, angular=args.angular, xc_frozen=args.xc_frozen,
                                          frozen=args.frozen, per_rung=args.per_rung,
                                          angular_fp64=args.angular_fp64)
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps({k: v for k, v in rep.items() if k != "per_instance"}))
        return
    if args.argon_run >= 0:
        run = P.argon_ensemble(64, seed=0, device="cuda", only=[args.argon_run], xc_frozen=args.xc_frozen)[0]
        run = dataclasses.replace(run, angular=args.angular, use_hartree=0 if args.frozen else run.use_hartree)
        rep = compare_forms(run, "Ar", args.precision, sensitivity=args.sensitivity, angular_fp64=args.angular_fp64,
                            theta_reuse=bool(args.theta_reuse))
        pot = "all potentials frozen" if args.frozen else ("xc frozen" if args.xc_frozen else "adiabatic")
        rep["config"] = (f"argon scan run {args.argon_run}: {run.name}, N_r {run.n_r}, l_max {run.n_l - 1}, "
                         f"angular {args.angular}, {pot}")
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps({k: v for k, v in rep.items() if k != "harmonic_rel_err"}))
        return
    if args.hhe_run >= 0:
        run = P.hhe_ensemble(256, seed=0, device="cuda", only=[args.hhe_run])[0]
        run = dataclasses.replace(run, angular=args.angular)
        atom = "H" if run.name.startswith("H-") else "He"
        rep = compare_forms(run, atom, args.precision, sensitivity=args.sensitivity, angular_fp64=args.angular_fp64,
                            theta_reuse=bool(args.theta_reuse))
        rep["config"] = f"H/He scan run {args.hhe_run}: {run.name}, angular {args.angular}"
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps({k: v for k, v in rep.items() if k != "harmonic_rel_err"}))
        return
    if args.hhe_ensemble:
        rep = compare_hhe_ensemble(args.precision, angular=args.angular, angular_fp64=args.angular_fp64)
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps({k: v for k, v in rep.items() if k != "per_instance"}))
        return
    if args.sweep:
        rep = sensitivity_sweep(eps=args.sensitivity or 1e-10)
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps(rep))
        return
    if args.ensemble_steps > 0:
        rep = compare_ensemble(args.ensemble_steps, args.precision, sensitivity=args.sensitivity)
        if args.out:
            with open(args.out, "w") as f:
                f.write(json.dumps(rep) + "\n")
        print(json.dumps({k: v for k, v in rep.items() if k != "per_instance"}))
        return
    atom, builder = CONFIGS[args.config]
    run = builder(n_steps=args.steps, device="cuda")
    if args.angular != "reference":
        run = dataclasses.replace(run, angular=args.angular, n_har=129 if atom == "He" else run.n_har)
    if args.xc_frozen:
        run = dataclasses.replace(run, xc_frozen=True, name=run.name + "-xcfrozen")
    if args.frozen:
        run = dataclasses.replace(run, use_hartree=0, name=run.name + "-frozen")
    rep = compare_forms(run, atom, args.precision, sensitivity=args.sensitivity, angular_fp64=args.angular_fp64,
                        theta_reuse=bool(args.theta_reuse))
    line = json.dumps(rep)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    print(json.dumps({k: v for k, v in rep.items() if k != "harmonic_rel_err"}))


if __name__ == "__main__":
    main()
