"""Python host API over libmarfa_gpu.so.

`Context` plays the part of the reference's opened line database and TIPS
table (main.f90:54, 196-212); `Context.compute` replaces the level and
subinterval loops of main.f90:81-180 and returns the PT records that
`marfa` would write, one [n_sub, 20481] float32 array per level.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MarfaError, MarfaRun, MARFA_NT
from .io import LINE_DTYPE, species_code


@dataclass
class Run:
    """The 7-argument command line (plus the options the reference fixes at
    compile time): molecule, start_wv, end_wv, cutoff, target, chi, shape,
    precision."""
    start_wv: float
    end_wv: float
    cutoff: float
    target: str = "ACS"
    molecule: str = "CO2"
    chi: str = "none"
    shape: str = "voigt"
    precision: str = "fp64"

    def c(self) -> MarfaRun:
        code = species_code(self.molecule)
        if code == 0:
            raise MarfaError(8, f"unsupported molecule {self.molecule!r}")
        if self.target not in _lib.TARGET:
            raise MarfaError(2, f"target must be ACS or VAC, got {self.target!r}")
        return MarfaRun(float(self.start_wv), float(self.end_wv), float(self.cutoff),
                        _lib.TARGET[self.target], code, _lib.CHI[self.chi],
                        _lib.SHAPE[self.shape], _lib.PRECISION[self.precision])

    @property
    def n_sub(self) -> int:
        return num_subintervals(self.start_wv, self.end_wv)


def num_subintervals(start_wv: float, end_wv: float) -> int:
    return _lib.load().marfa_num_subintervals(float(start_wv), float(end_wv))


def plan_windows(nu: np.ndarray, start_wv: float, end_wv: float, cutoff: float):
    """Line window [lo, hi) (0-based) of every subinterval: the line-loop
    recurrence of LBL.f90:41-61 with capWV (main.f90:138-144).  Host only."""
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    ns = num_subintervals(start_wv, end_wv)
    lo = np.zeros(ns, dtype=np.int64)
    hi = np.zeros(ns, dtype=np.int64)
    rc = _lib.load().marfa_plan_windows(nu.ctypes.data, len(nu), float(start_wv), float(end_wv),
                                        float(cutoff), lo.ctypes.data, hi.ctypes.data)
    if rc:
        raise MarfaError(rc, "plan_windows")
    return lo, hi


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class Context:
    """Device-resident line list + TIPS table on one GPU."""

    def __init__(self, lines: np.ndarray, tips: np.ndarray, device: int = 0):
        lib = _lib.load()
        self._lines = np.ascontiguousarray(lines, dtype=LINE_DTYPE)
        self._tips = np.ascontiguousarray(tips, dtype=np.float64)
        h = ctypes.c_void_p()
        rc = lib.marfa_ctx_create(self._lines.ctypes.data, len(self._lines),
                                  self._tips.ctypes.data, self._tips.shape[0],
                                  self._tips.shape[1], int(device), ctypes.byref(h))
        if rc:
            raise MarfaError(rc, "context creation failed")
        self._h = h
        self._lib = lib

    def close(self):
        if getattr(self, "_h", None):
            self._lib.marfa_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            msg = self._lib.marfa_last_error(self._h)
            raise MarfaError(rc, msg.decode() if msg else "")

    @property
    def handle(self):
        return self._h

    def compute(self, run: Run, pressure, temperature, density, out=None, want64=False):
        """One profile: returns float32 records [n_levels, n_sub, 20481]
        (and the float64 values before rounding when want64)."""
        return self.compute_batched(run, [len(pressure)], pressure, temperature, density,
                                    out=out, want64=want64)

    def compute_batched(self, run: Run, level_counts, pressure, temperature, density,
                        out=None, want64=False):
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        counts = np.ascontiguousarray(level_counts, dtype=np.int32)
        L = int(counts.sum())
        shape = (L, run.n_sub, MARFA_NT)
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        out64 = np.empty(shape, dtype=np.float64) if want64 else None
        r = run.c()
        self._check(self._lib.marfa_compute_batched(
            self._h, ctypes.byref(r), len(counts), counts.ctypes.data, P.ctypes.data,
            T.ctypes.data, n.ctypes.data, ctypes.c_void_p(_ptr(out)),
            ctypes.c_void_p(out64.ctypes.data if want64 else 0)))
        return (out, out64) if want64 else out

    def compute_device(self, run: Run, level_counts, pressure, temperature, density,
                       device_ptr: int, stream: int = 0):
        """Asynchronous form writing into a device buffer (e.g. a torch
        tensor's data_ptr()) on `stream` (a cudaStream_t as int)."""
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        counts = np.ascontiguousarray(level_counts, dtype=np.int32)
        r = run.c()
        self._check(self._lib.marfa_compute_device(
            self._h, ctypes.byref(r), len(counts), counts.ctypes.data, P.ctypes.data,
            T.ctypes.data, n.ctypes.data, ctypes.c_void_p(device_ptr), ctypes.c_void_p(stream)))

    def synchronize(self):
        self._check(self._lib.marfa_synchronize(self._h))

    def graph(self, run: Run, level_counts, pressure, temperature, density, device_ptr: int) -> "Graph":
        """Compute into the device buffer at `device_ptr` and capture the
        launches into a CUDA graph, replayed by Graph.launch for new profiles
        of the same level counts."""
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        counts = np.ascontiguousarray(level_counts, dtype=np.int32)
        r = run.c()
        h = ctypes.c_void_p()
        self._check(self._lib.marfa_graph_create(
            self._h, ctypes.byref(r), len(counts), counts.ctypes.data, P.ctypes.data, T.ctypes.data,
            n.ctypes.data, ctypes.c_void_p(device_ptr), ctypes.byref(h)))
        return Graph(self, h)

    def autotune(self, run: Run, pressure, temperature, density) -> dict:
        """Time the launch-parameter candidates on a few levels of this
        profile and keep the fastest for later calls."""
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        fc, ck = ctypes.c_int(), ctypes.c_int()
        r = run.c()
        self._check(self._lib.marfa_autotune(self._h, ctypes.byref(r), len(P), P.ctypes.data,
                                             T.ctypes.data, n.ctypes.data, ctypes.byref(fc),
                                             ctypes.byref(ck)))
        return self.launch()

    def launch(self) -> dict:
        """The context's launch parameters: lines per far-kernel block,
        coarse fine grids summed by lane groups, and the FP32c fine-block
        shape (0: one 1024-thread block per SM, 1: two of 512)."""
        fc, ck, fp = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.marfa_ctx_get_launch(self._h, ctypes.byref(fc), ctypes.byref(ck),
                                                   ctypes.byref(fp)))
        return {"far_chunk": fc.value, "coop_k": ck.value, "fine_pair": fp.value}

    def set_launch(self, far_chunk: int, coop_k: int, fine_pair: int) -> None:
        """Pin the launch parameters (as returned by autotune or launch)."""
        self._check(self._lib.marfa_ctx_set_launch(self._h, int(far_chunk), int(coop_k), int(fine_pair)))

    @property
    def n_lines(self) -> int:
        return len(self._lines)

    def set_line_params(self, S=None, gamma_air=None):
        """Double-precision reference intensities and air-broadening
        coefficients for every line (None: the database record's value)."""
        self._S64 = None if S is None else _f64(S)
        self._g64 = None if gamma_air is None else _f64(gamma_air)
        for a in (self._S64, self._g64):
            if a is not None and a.shape != (self.n_lines,):
                raise ValueError(f"expected {self.n_lines} values, got {a.shape}")
        self._check(self._lib.marfa_ctx_set_line_params(
            self._h, ctypes.c_void_p(0 if self._S64 is None else self._S64.ctypes.data),
            ctypes.c_void_p(0 if self._g64 is None else self._g64.ctypes.data)))

    def set_tips_grid(self, t_first: float, t_step: float):
        """Temperature grid of the context's TIPS table (node j at t_first +
        j t_step K; the reference's table: 20 K, 2 K)."""
        self._check(self._lib.marfa_ctx_set_tips_grid(self._h, float(t_first), float(t_step)))

    def vjp(self, run: Run, pressure, temperature, density, cotangent) -> dict:
        """Vector-Jacobian product of the FP64 records for `cotangent`
        [n_levels, n_sub, 20481]: dict of dT, dP [n_levels] and dS,
        dgamma_air [n_lines] (float64)."""
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        cot = _f64(cotangent)
        if cot.shape != (len(P), run.n_sub, MARFA_NT):
            raise ValueError(f"cotangent shape {cot.shape} != {(len(P), run.n_sub, MARFA_NT)}")
        dT = np.zeros(len(P))
        dP = np.zeros(len(P))
        dS = np.zeros(self.n_lines)
        dg = np.zeros(self.n_lines)
        r = run.c()
        self._check(self._lib.marfa_vjp(self._h, ctypes.byref(r), P.ctypes.data, T.ctypes.data,
                                        n.ctypes.data, len(P), cot.ctypes.data, dT.ctypes.data,
                                        dP.ctypes.data, dS.ctypes.data, dg.ctypes.data))
        return {"dT": dT, "dP": dP, "dS": dS, "dgamma_air": dg}

    def eval_count(self, run: Run, pressure, temperature, density, far=False):
        """Line-shape evaluations of the reference schedule per level (and,
        with far=True, also the part made by the far-line kernel)."""
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        ev = np.zeros(len(P), dtype=np.int64)
        evf = np.zeros(len(P), dtype=np.int64)
        r = run.c()
        self._check(self._lib.marfa_eval_count(self._h, ctypes.byref(r), len(P), P.ctypes.data,
                                               T.ctypes.data, n.ctypes.data, ev.ctypes.data,
                                               evf.ctypes.data))
        return (ev, evf) if far else ev

    def accumulators(self, run: Run, pressure, temperature, density, level, isub) -> np.ndarray:
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        d = np.zeros(MARFA_NT + 3 * 10230, dtype=np.float64)
        r = run.c()
        self._check(self._lib.marfa_debug_accumulators(
            self._h, ctypes.byref(r), P.ctypes.data, T.ctypes.data, n.ctypes.data, len(P),
            int(level), int(isub), d.ctypes.data))
        return d

    def timings(self) -> dict:
        """Milliseconds per kernel family of the last compute call (CUDA
        events on its stream) and its kernel-launch counts."""
        t = np.zeros(8, dtype=np.float64)
        self._check(self._lib.marfa_last_timings(self._h, t.ctypes.data))
        return dict(zip(("prep", "sort", "far", "fine", "cascade", "total", "launches",
                         "far_launches"), t.tolist()))


class Graph:
    """A captured compute call (marfa_graph_*)."""

    def __init__(self, ctx: Context, handle):
        self._ctx = ctx
        self._h = handle

    def launch(self, pressure, temperature, density, stream: int = 0):
        P, T, n = _f64(pressure), _f64(temperature), _f64(density)
        self._ctx._check(self._ctx._lib.marfa_graph_launch(self._h, P.ctypes.data, T.ctypes.data,
                                                           n.ctypes.data, ctypes.c_void_p(stream)))

    def close(self):
        if getattr(self, "_h", None):
            self._ctx._lib.marfa_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        if not (a.flags.c_contiguous and a.dtype == np.float32):
            raise ValueError("output must be a C-contiguous float32 array")
        return a.ctypes.data
    return int(a.data_ptr())  # a pinned torch tensor
