"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C restatement of the reference Fortran line-by-line core
(see marfa_oracle.h for provenance and the parity-pin status).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "liboracle.so"

NT = 20481
NCELLS = 10230
DUMP_LEN = NT + 3 * NCELLS
MIXED, FP64 = 0, 1
CHI = {"none": 0, "tonkov": 1, "pollack": 2, "perrin": 3}
SHAPE = {"voigt": 0, "lorentz": 1, "one": 100, "absx": 101}
TARGET = {"ACS": 0, "VAC": 1}


class OracleArgs(ctypes.Structure):
    _fields_ = [
        ("records", ctypes.c_void_p), ("n_lines", ctypes.c_int64),
        ("tips", ctypes.c_void_p), ("n_iso", ctypes.c_int), ("n_temp", ctypes.c_int),
        ("tips_t0", ctypes.c_double), ("tips_dt", ctypes.c_double),
        ("pressure", ctypes.c_void_p), ("temperature", ctypes.c_void_p),
        ("density", ctypes.c_void_p), ("n_levels", ctypes.c_int),
        ("start_wv", ctypes.c_double), ("end_wv", ctypes.c_double),
        ("cutoff", ctypes.c_double), ("target", ctypes.c_int), ("chi", ctypes.c_int),
        ("mol_code", ctypes.c_int), ("shape", ctypes.c_int), ("precision", ctypes.c_int),
        ("nthreads", ctypes.c_int),
    ]


def build():
    """Compile the oracle library (make in this folder)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_run.restype = ctypes.c_int
        _lib.oracle_unit_accumulators.restype = ctypes.c_int
        _lib.oracle_shape_value.restype = ctypes.c_int
        _lib.oracle_windows.restype = ctypes.c_int
        _lib.oracle_num_subintervals.restype = ctypes.c_int
        _lib.oracle_num_subintervals.argtypes = [ctypes.c_double, ctypes.c_double]
        _lib.oracle_record_number.restype = ctypes.c_int
        _lib.oracle_record_number.argtypes = [ctypes.c_double, ctypes.c_int]
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code):
        super().__init__(f"oracle status {code}")
        self.code = code


class Oracle:
    """Holds the arrays an oracle call points into."""

    def __init__(self, lines, tips, pressure, temperature, density, start_wv, end_wv,
                 cutoff, target="ACS", chi="none", mol_code=2, shape="voigt",
                 precision=FP64, nthreads=None, tips_grid=(20.0, 2.0)):
        self.lines = np.ascontiguousarray(lines)
        assert self.lines.dtype.itemsize == 36
        self.tips = np.ascontiguousarray(tips, dtype=np.float64)
        self.P = np.ascontiguousarray(pressure, dtype=np.float64)
        self.T = np.ascontiguousarray(temperature, dtype=np.float64)
        self.n = np.ascontiguousarray(density, dtype=np.float64)
        a = OracleArgs()
        a.records = self.lines.ctypes.data
        a.n_lines = len(self.lines)
        a.tips = self.tips.ctypes.data
        a.n_iso, a.n_temp = self.tips.shape
        a.tips_t0, a.tips_dt = float(tips_grid[0]), float(tips_grid[1])
        a.pressure = self.P.ctypes.data
        a.temperature = self.T.ctypes.data
        a.density = self.n.ctypes.data
        a.n_levels = len(self.P)
        a.start_wv, a.end_wv, a.cutoff = float(start_wv), float(end_wv), float(cutoff)
        a.target = TARGET[target] if isinstance(target, str) else int(target)
        a.chi = CHI[chi] if isinstance(chi, str) else int(chi)
        a.mol_code = int(mol_code)
        a.shape = SHAPE[shape] if isinstance(shape, str) else int(shape)
        a.precision = int(precision)
        a.nthreads = int(nthreads or os.cpu_count() or 1)
        self.args = a

    @property
    def n_sub(self):
        return lib().oracle_num_subintervals(self.args.start_wv, self.args.end_wv)

    def run(self, want64=True):
        """Returns (records float32 [L, n_sub, NT], records64 or None, evals [L])."""
        L, ns = self.args.n_levels, self.n_sub
        out = np.zeros((L, ns, NT), dtype=np.float32)
        out64 = np.zeros((L, ns, NT), dtype=np.float64) if want64 else None
        ev = np.zeros(L, dtype=np.int64)
        rc = lib().oracle_run(ctypes.byref(self.args), ctypes.c_void_p(out.ctypes.data),
                              ctypes.c_void_p(out64.ctypes.data if want64 else 0),
                              ctypes.c_void_p(ev.ctypes.data))
        if rc:
            raise OracleError(rc)
        return out, out64, ev

    def accumulators(self, level, isub):
        """Raw accumulators of one (level, subinterval): dict of RK [NT] and
        P, M, L [10230] (grid k at offset 10*(2^k-1))."""
        d = np.zeros(DUMP_LEN, dtype=np.float64)
        rc = lib().oracle_unit_accumulators(ctypes.byref(self.args), int(level), int(isub),
                                            ctypes.c_void_p(d.ctypes.data))
        if rc:
            raise OracleError(rc)
        return d

    def shape_value(self, level, line, X):
        v = ctypes.c_double()
        r = ctypes.c_int()
        rc = lib().oracle_shape_value(ctypes.byref(self.args), int(level), ctypes.c_int64(line),
                                      ctypes.c_double(X), ctypes.byref(v), ctypes.byref(r))
        if rc:
            raise OracleError(rc)
        return v.value, r.value

    def windows(self):
        ns = self.n_sub
        lo = np.zeros(ns, dtype=np.int64)
        hi = np.zeros(ns, dtype=np.int64)
        rc = lib().oracle_windows(ctypes.byref(self.args), ctypes.c_void_p(lo.ctypes.data),
                                  ctypes.c_void_p(hi.ctypes.data))
        if rc:
            raise OracleError(rc)
        return lo, hi


def from_workload(w, profile_index=0, **kw):
    """Oracle for a marfa_b200.synth.Workload and one of its profiles."""
    from marfa_b200.io import read_tips, species_code
    from marfa_b200 import data_path
    p = w.profiles[profile_index]
    tips = kw.pop("tips", None)
    if tips is None:
        tips = read_tips(data_path("TIPS_subset.dat"))
    return Oracle(w.lines, tips, p.pressure, p.temperature, p.density, w.start_wv,
                  w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                  mol_code=species_code(w.molecule), **kw)
