"""Host-side driver of the CUDA time step, over the C ABI of libggbtddft.so (include/ggbtddft.h).

``TimePropagation`` plays the role of the reference's ``h_timePropagation`` plus the loaders and
buffers ``main.cu`` sets up around it (src/main.cu:228-481): give it one or more runs
(``problems.RunInputs``), call ``step(n)``, read the dipole / acceleration / norm series in the
reference's layout.  Runs that share a grid, N_l and the radial-propagator array (the same
``W`` object) are placed in one grid group and advance in the same launches.

There is no CPU fallback: if the library is missing or no CUDA device is present, construction
raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import inputs as I
from .problems import RunInputs

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libggbtddft.so")

PRECISIONS = {"fp64": 0, "split_bf16": 1, "split_tf32": 2, "split_int8": 3}
COUPLING_IDS = {"P": 0, "FP": 1, "D": 2, "FF": 3}
RUN_XC_PW92 = 1
RUN_THETA = 2
RUN_XC_FROZEN = 4


class GGBError(RuntimeError):
    pass


class _GroupDesc(ctypes.Structure):
    _fields_ = [("n_r", ctypes.c_int), ("n_l", ctypes.c_int), ("n_m", ctypes.c_int)]


class _RunDesc(ctypes.Structure):
    _fields_ = [("group", ctypes.c_int), ("n_orb", ctypes.c_int), ("n_har", ctypes.c_int),
                ("use_hartree", ctypes.c_int), ("target_id", ctypes.c_int), ("flags", ctypes.c_int),
                ("dt", ctypes.c_double)]


class _Dims(ctypes.Structure):
    _fields_ = [("n_groups", ctypes.c_int), ("n_runs", ctypes.c_int), ("precision", ctypes.c_int),
                ("n_t", ctypes.c_int), ("per_l", ctypes.c_int)]


_lib = None

EXPORTS = ("ggb_create", "ggb_set_grid", "ggb_set_radial_propagators", "ggb_set_angular", "ggb_set_orbitals",
           "ggb_set_field", "ggb_step", "ggb_get_step", "ggb_get_observables", "ggb_get_orbitals",
           "ggb_get_potentials", "ggb_status", "ggb_destroy", "ggb_version", "ggb_launch_phase",
           "ggb_set_tuning", "ggb_observables_noalloc", "ggb_measure_peaks", "ggb_measure_peak_fp64_mma",
           "ggb_set_angular_fp64", "ggb_set_theta_reuse")


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libggbtddft.so and declare the C signatures.  Raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise GGBError(f"{path} is missing: build it with `python -m ggbtddft_b200.build` "
                       "(there is no CPU fallback for the time step)")
    lib = ctypes.CDLL(path)
    P, I_, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    pp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "ggb_create": ([ctypes.POINTER(_Dims), ctypes.POINTER(_GroupDesc), ctypes.POINTER(_RunDesc), pp], I_),
        "ggb_set_grid": ([P, I_, P, P, P, I_], I_),
        "ggb_set_radial_propagators": ([P, I_, P], I_),
        "ggb_set_angular": ([P, I_, I_, I_, P, P], I_),
        "ggb_set_orbitals": ([P, I_, P, P, P, P, P], I_),
        "ggb_set_field": ([P, I_, P, I_], I_),
        "ggb_step": ([P, I_, P], I_),
        "ggb_get_step": ([P, ctypes.POINTER(ctypes.c_int)], I_),
        "ggb_launch_phase": ([P, I_, P], I_),
        "ggb_set_tuning": ([P, I_, I_, I_], I_),
        "ggb_set_angular_fp64": ([P, I_, I_], I_),
        "ggb_set_theta_reuse": ([P, I_, I_], I_),
        "ggb_get_observables": ([P, I_, P, P, P, I_, I_], I_),
        "ggb_get_orbitals": ([P, I_, P], I_),
        "ggb_get_potentials": ([P, I_, P, P, P, P], I_),
        "ggb_status": ([P, ctypes.c_char_p, I_], I_),
        "ggb_destroy": ([P], None),
        "ggb_version": ([], ctypes.c_char_p),
        "ggb_observables_noalloc": ([P, P, P, I_, I_, I_, P, P, P, P], I_),
        "ggb_measure_peaks": ([ctypes.POINTER(D), ctypes.POINTER(D), P], I_),
        "ggb_measure_peak_fp64_mma": ([ctypes.POINTER(D), P], I_),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def measure_peaks(stream: Optional[int] = None) -> Dict[str, float]:
    """Peaks of the current GPU from the library's microbenchmarks: FP64 FMA and FP64 mma.sync
    (TFLOP/s; ``fp64_tflops`` is the larger, the FP64 roofline) and tcgen05 int8 (TOP/s)."""
    lib = load_library()
    f, i, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    h = ctypes.c_void_p(stream) if stream else None
    rc = lib.ggb_measure_peaks(ctypes.byref(f), ctypes.byref(i), h)
    if rc != 0:
        raise GGBError(f"ggb_measure_peaks failed: {rc}")
    rc = lib.ggb_measure_peak_fp64_mma(ctypes.byref(d), h)
    if rc != 0:
        raise GGBError(f"ggb_measure_peak_fp64_mma failed: {rc}")
    return dict(fp64_tflops=max(f.value, d.value), fp64_fma_tflops=f.value, fp64_mma_tflops=d.value,
                int8_tops=i.value)


def group_runs(runs: Sequence[RunInputs]) -> List[List[int]]:
    """Runs sharing the same W array object (and therefore grid and N_l) form one grid group."""
    groups: Dict[int, List[int]] = {}
    order: List[int] = []
    for i, r in enumerate(runs):
        k = id(r.W)
        if k not in groups:
            groups[k] = []
            order.append(k)
        groups[k].append(i)
    return [groups[k] for k in order]


class TimePropagation:
    """All runs of an ensemble on one GPU; FP64 parity form or a split-precision form."""

    def __init__(self, runs: Sequence[RunInputs], precision: str = "fp64", per_l: bool = True,
                 n_t: Optional[int] = None, groups: Optional[List[List[int]]] = None, W_device=None,
                 tuning: Optional[Dict[int, Tuple[int, int]]] = None, autotune: bool = False,
                 angular_fp64: bool = False, theta_reuse: bool = True):
        """``tuning`` = {group: (radial_bn, radial_stages)} (ggb_set_tuning); ``autotune`` = True
        takes each group's tiles from the autotuner's cache, timing the candidates on a miss
        (split_int8 form only); ``angular_fp64`` = True runs the split_int8 form's angular products
        on the FP64 tensor cores (ggb_set_angular_fp64), the radial product staying int8;
        ``theta_reuse`` = False runs both products of every angular half in the split_int8 theta
        form (ggb_set_theta_reuse; by default a step's first half starts from the node-basis
        vectors its predecessor's second half kept)."""
        self.lib = load_library()
        self.runs = list(runs)
        self.precision = precision
        self.per_l = per_l
        self.groups = groups if groups is not None else group_runs(self.runs)
        self.n_t = int(n_t if n_t is not None else max(r.n_t for r in self.runs))
        if autotune and precision == "split_int8" and tuning is None:
            # before this context allocates anything: the tuner times its candidates in contexts
            # of its own, one grid group at a time
            from . import autotune as AT
            tuning = AT.tuning_for(self.runs, self.groups)
        self.tuning = tuning
        run_group = {}
        for gi, members in enumerate(self.groups):
            for ri in members:
                run_group[ri] = gi
        gd = (_GroupDesc * len(self.groups))()
        for gi, members in enumerate(self.groups):
            r0 = self.runs[members[0]]
            gd[gi] = _GroupDesc(r0.n_r, r0.n_l, max(self.runs[i].n_m for i in members))
        rd = (_RunDesc * len(self.runs))()
        for i, r in enumerate(self.runs):
            rd[i] = _RunDesc(run_group[i], r.n_orb, r.n_har, r.use_hartree, r.target_id,
                             (RUN_XC_PW92 if r.xc_correlation else 0) |
                             (RUN_THETA if getattr(r, "angular", "reference") == "theta" else 0) |
                             (RUN_XC_FROZEN if getattr(r, "xc_frozen", False) else 0), r.dt)
        dims = _Dims(len(self.groups), len(self.runs), PRECISIONS[precision], self.n_t, 1 if per_l else 0)
        ctx = ctypes.c_void_p()
        self._check(self.lib.ggb_create(ctypes.byref(dims), gd, rd, ctypes.byref(ctx)), None)
        self.ctx = ctx
        for gi, members in enumerate(self.groups):
            r0 = self.runs[members[0]]
            g = r0.grid
            self._call("ggb_set_grid", gi, _ptr(_c(g.r, np.float64)), _ptr(_c(g.drdx, np.float64)),
                       _ptr(_c(g.P, np.float64)), g.n_r)
            W = _c(r0.W, np.complex128)
            self._call("ggb_set_radial_propagators", gi, _ptr(W))
            n_m = gd[gi].n_m
            for c, cid in COUPLING_IDS.items():
                for m in range(n_m):
                    self._call("ggb_set_angular", gi, cid, m, _ptr(_c(r0.V[c][m], np.float64)),
                               _ptr(_c(r0.D[c][m], np.float64)))
        for gi, (bn, stages) in (tuning or {}).items():
            self._call("ggb_set_tuning", int(gi), int(bn), int(stages))
        self.angular_fp64 = bool(angular_fp64) and precision == "split_int8"
        if self.angular_fp64:
            for gi in range(len(self.groups)):
                self._call("ggb_set_angular_fp64", gi, 1)
        self.theta_reuse = bool(theta_reuse) and precision == "split_int8"
        if precision == "split_int8" and not self.theta_reuse:
            for gi in range(len(self.groups)):
                self._call("ggb_set_theta_reuse", gi, 0)
        for i in range(len(self.runs)):
            self.set_orbitals(i, self.runs[i].x0)
            self.set_field(i, self.runs[i].E)

    # ---------------------------------------------------------------- helpers
    def _check(self, rc, ctx):
        if rc < 0:
            msg = ctypes.create_string_buffer(512)
            if ctx is not None:
                self.lib.ggb_status(ctx, msg, 512)
            raise GGBError(f"libggbtddft error {rc}: {msg.value.decode()}")
        return rc

    def _call(self, name, *args):
        return self._check(getattr(self.lib, name)(self.ctx, *args), self.ctx)

    # ---------------------------------------------------------------- set-up
    def set_orbitals(self, run: int, x0: np.ndarray, rho_frozen: Optional[np.ndarray] = None):
        r = self.runs[run]
        x = _c(x0, np.complex128)
        self._call("ggb_set_orbitals", run, _ptr(x), _ptr(_c(r.l_active, np.int32)),
                   _ptr(_c(r.m_active, np.int32)), _ptr(_c(r.occ, np.int32)),
                   _ptr(_c(r.rho_frozen if rho_frozen is None else rho_frozen, np.float64)))

    def set_field(self, run: int, E: np.ndarray):
        E = _c(E, np.float64)
        self._call("ggb_set_field", run, _ptr(E), E.size)

    # ---------------------------------------------------------------- stepping
    def step(self, n_steps: int, stream: Optional[int] = None):
        """Advance every run by n_steps (asynchronous on ``stream``, a cudaStream_t handle)."""
        self._call("ggb_step", int(n_steps), ctypes.c_void_p(stream) if stream else None)

    def launch_phase(self, phase: int, stream: Optional[int] = None):
        """Profiling only: launch one phase of the step alone (see ggb_launch_phase)."""
        self._call("ggb_launch_phase", int(phase), ctypes.c_void_p(stream) if stream else None)

    @property
    def current_step(self) -> int:
        s = ctypes.c_int()
        self._call("ggb_get_step", ctypes.byref(s))
        return s.value

    def status(self):
        msg = ctypes.create_string_buffer(512)
        st = self.lib.ggb_status(self.ctx, msg, 512)
        return st, msg.value.decode()

    # ---------------------------------------------------------------- results
    def observables(self, run: int, per_l: bool = True, n_steps: Optional[int] = None):
        """dipole, acceleration ([N_l][n_orb][t] if per_l else [n_orb][t]) and norm [n_orb][t]."""
        r = self.runs[run]
        n = self.current_step if n_steps is None else n_steps
        shape = (r.n_l, r.n_orb, n) if per_l else (r.n_orb, n)
        dip = np.zeros(shape, dtype=np.complex128)
        acc = np.zeros(shape, dtype=np.complex128)
        norm = np.zeros((r.n_orb, n))
        self._call("ggb_get_observables", run, _ptr(dip), _ptr(acc), _ptr(norm), 1 if per_l else 0, n)
        return dict(dipole=dip, acceleration=acc, norm=norm)

    def orbitals(self, run: int) -> np.ndarray:
        r = self.runs[run]
        x = np.zeros((r.n_l, r.n_orb, r.n_r), dtype=np.complex128)
        self._call("ggb_get_orbitals", run, _ptr(x))
        return x

    def potentials(self, run: int):
        r = self.runs[run]
        v = np.zeros((4, r.n_r))
        v0, vx, vx0 = (np.zeros(r.n_r) for _ in range(3))
        self._call("ggb_get_potentials", run, _ptr(v), _ptr(v0), _ptr(vx), _ptr(vx0))
        return dict(v=v, v0=v0, vexc=vx, vexc0=vx0)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.ggb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def h_time_propagation(run: RunInputs, n_steps: Optional[int] = None, precision: str = "fp64"):
    """One run through the whole loop, as the reference's h_timePropagation (h_timePropagation.cuh:32-114).

    Returns the reference's observable layout: dipole[l][kso][t] (h_dipoleMoment, main.cu:395),
    acceleration[l][kso][t], plus norm[kso][t] and the final orbitals.
    """
    tp = TimePropagation([run], precision=precision, per_l=True)
    try:
        n = run.n_t if n_steps is None else n_steps
        tp.step(n)
        out = tp.observables(0, per_l=True, n_steps=n)
        out["x"] = tp.orbitals(0)
        st, msg = tp.status()
        if st != 0:
            raise GGBError(f"device status {st}: {msg}")
        return out
    finally:
        tp.close()
