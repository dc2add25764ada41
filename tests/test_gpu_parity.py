"""Parity of the CUDA library (through its C ABI) with the CPU oracle.

Tolerances: the FP64 drop-in agrees with the all-double oracle to 1e-12
relative on every point; the FP32-compensated form agrees with it to 1e-5
relative on points where k > 1e-6 max(k) (the accuracy target of the FP32
form).  The multigrid placement is checked exactly with diagnostic shapes.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from marfa_b200 import synth
from marfa_b200.api import Context, Run

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32C_TOL = 1e-5


def run_for(w, **kw):
    d = dict(start_wv=w.start_wv, end_wv=w.end_wv, cutoff=w.cutoff, target=w.target,
             molecule=w.molecule, chi=w.chi)
    d.update(kw)
    return Run(**d)


@pytest.fixture(scope="module")
def cfg0(gpu, tips):
    w = synth.config(0)
    ctx = Context(w.lines, tips)
    o = O.from_workload(w, precision=O.FP64, tips=tips)
    ref, ref64, ev = o.run()
    yield w, ctx, o, ref64, ev
    ctx.close()


def test_config0_fp64_matches_oracle(cfg0):
    w, ctx, o, ref64, _ = cfg0
    p = w.profiles[0]
    out, out64 = ctx.compute(run_for(w, precision="fp64"), p.pressure, p.temperature, p.density,
                             want64=True)
    err, n = rel_err(out64, ref64, floor_frac=0.0)
    assert n == ref64.size
    assert err <= FP64_TOL, err
    assert np.array_equal(out, out64.astype(np.float32))


def test_config0_fp32c_within_tolerance(cfg0):
    w, ctx, o, ref64, _ = cfg0
    p = w.profiles[0]
    out = ctx.compute(run_for(w, precision="fp32c"), p.pressure, p.temperature, p.density)
    err, n = rel_err(out, ref64)
    assert err <= FP32C_TOL, err


def test_config0_eval_count_exact(cfg0):
    w, ctx, o, _, ev = cfg0
    p = w.profiles[0]
    g = ctx.eval_count(run_for(w), p.pressure, p.temperature, p.density)
    assert g.tolist() == ev.tolist()


@pytest.mark.parametrize("shape", ["one", "absx"])
@pytest.mark.parametrize("isub", [0, 4, 9])
def test_placement_matches_oracle(cfg0, tips, shape, isub):
    """Diagnostic shapes F = 1 (per-accumulator line counts, exact) and
    F = |X| (sum of offsets) expose every (line, grid, cell, slot, X) the
    multigrid schedule touches."""
    w, ctx, _, _, _ = cfg0
    p = w.profiles[0]
    o = O.from_workload(w, precision=O.FP64, shape=shape, tips=tips)
    ref = o.accumulators(0, isub)
    got = ctx.accumulators(run_for(w, precision="fp64", shape=shape), p.pressure,
                           p.temperature, p.density, 0, isub)
    if shape == "one":
        assert np.array_equal(got, ref), np.flatnonzero(got != ref)[:20]
    else:
        assert np.array_equal(got > 0, ref > 0)
        m = ref > 0
        assert np.max(np.abs(got[m] - ref[m]) / ref[m]) <= 1e-12
