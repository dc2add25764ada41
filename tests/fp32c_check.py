"""Accuracy check of the FP32-compensated records against the FP64 oracle.

The reference's cascade interpolation (Grids.f90:91, 98, 125, 133) replaces
the quadratic quarter-point value by the half sum whenever it falls below
either neighbour: a discontinuous decision.  When the FP64 oracle itself
finds such a decision within 1e-6 (relative) of its threshold, any
perturbation of the sums at the 1e-7 level of FP32 may take the other branch
and move the finest points below that cell by up to the jump.  Those points
are identified here from the oracle's own accumulators; every other
significant point must agree to 1e-5.
"""
import numpy as np

NT = 20481


def tainted_points(dump, rel=1e-6, want_record=False):
    """Finest points of one (level, subinterval) that sit below a near-tie
    clamp decision of the cascade run on the oracle's accumulators (and,
    with want_record, the cascaded record itself)."""
    ncell = 10230
    RK = dump[:NT].copy()
    P = dump[NT:NT + ncell].copy()
    M = dump[NT + ncell:NT + 2 * ncell].copy()
    L = dump[NT + 2 * ncell:].copy()
    taint = np.zeros(10, dtype=bool)
    for k in range(10):
        b = 10 * ((1 << k) - 1)
        n = 10 << k
        cP, cM, cL = P[b:b + n], M[b:b + n], L[b:b + n]
        scale = np.maximum(np.maximum(np.abs(cP), np.abs(cM)), np.abs(cL)) + 1e-300
        A1 = 0.375 * cP + 0.75 * cM - 0.125 * cL
        A2 = 0.375 * cL + 0.75 * cM - 0.125 * cP
        t1 = np.abs(A1 - np.maximum(cP, cM)) < rel * scale
        t2 = np.abs(A2 - np.maximum(cL, cM)) < rel * scale
        A1 = np.where((A1 < cP) | (A1 < cM), 0.5 * (cP + cM), A1)
        A2 = np.where((A2 < cL) | (A2 < cM), 0.5 * (cL + cM), A2)
        child = np.empty(2 * n, dtype=bool)
        child[0::2] = taint | t1
        child[1::2] = taint | t2
        if k < 9:
            bf = 10 * ((1 << (k + 1)) - 1)
            P[bf:bf + 2 * n:2] += cP
            M[bf:bf + 2 * n:2] += A1
            L[bf:bf + 2 * n:2] += cM
            P[bf + 1:bf + 2 * n:2] += cM
            M[bf + 1:bf + 2 * n:2] += A2
            L[bf + 1:bf + 2 * n:2] += cL
            taint = child
        else:
            RK[1::4][:n] += A1
            RK[2::4][:n] += cM
            RK[3::4][:n] += A2
            RK[4::4][:n] += cL
            pts = np.zeros(NT, dtype=bool)
            pts[1::4][:n] = child[0::2]        # RK(4J-2)
            pts[2::4][:n] = taint               # RK(4J-1) = M: no decision of its own
            pts[3::4][:n] = child[1::2]        # RK(4J)
            pts[4::4][:n] = taint               # RK(4J+1) = L
            return (pts, RK) if want_record else pts


def check_fp32c(got, ref, oracle, tol=1e-5, floor=1e-6):
    """got/ref: [levels, n_sub, NT]; oracle: the FP64 Oracle that made ref.
    Returns (max error on untainted points, number of tainted points)."""
    got = np.asarray(got, dtype=np.float64)
    m = ref > floor * ref.max()
    err = np.zeros_like(ref)
    err[m] = np.abs(got[m] - ref[m]) / ref[m]
    if err.max() <= tol:
        return float(err.max()), 0
    bad_units = np.argwhere(err.max(axis=2) > tol)
    n_taint = 0
    for lvl, isub in bad_units:
        t = tainted_points(oracle.accumulators(lvl, isub))
        n_taint += int((t & m[lvl, isub]).sum())
        err[lvl, isub][t] = 0.0
    return float(err.max()), n_taint
