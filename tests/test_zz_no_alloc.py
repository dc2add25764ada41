"""marfa_compute_record_static: one PT record computed without any memory
allocation (all device working storage in the library's static array), for
callers that cannot call cudaMalloc, e.g. applications whose device memory is
owned by a pool allocator that reserves the GPU at start-up.

Checked through the C ABI against the regular entry point (marfa_compute) on
two calls in a row, in both precisions; this file is collected last so that a
run stopping at its first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from marfa_b200 import _lib, synth
from marfa_b200._lib import MarfaRun
from marfa_b200.api import Context, Run

pytestmark = pytest.mark.gpu

NT = 20481


def static_record(lib, lines, tips, run, P, T, n, isub):
    rec = np.full(NT, np.nan, dtype=np.float32)
    msg = ctypes.create_string_buffer(256)
    r = run.c()
    rc = lib.marfa_compute_record_static(lines.ctypes.data, len(lines), tips.ctypes.data,
                                         tips.shape[0], tips.shape[1], ctypes.byref(r), P, T, n,
                                         isub, rec.ctypes.data, None, msg, len(msg))
    return rc, rec, msg.value.decode()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32c", 1e-6)])
def test_static_record_matches_regular_entry_point(gpu, tips, prec, tol):
    lib = gpu
    t = np.ascontiguousarray(tips)
    for w, level, subs in ((synth.config(0), 0, (3, 7)), (synth.config(1, scale=0.3), 5, (12, 2))):
        lines = np.ascontiguousarray(w.lines)
        p = w.profiles[0]
        run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule,
                  chi=w.chi, precision=prec)
        with Context(lines, t) as ctx:
            full = ctx.compute(run, p.pressure[level:level + 1], p.temperature[level:level + 1],
                               p.density[level:level + 1])[0]
        for isub in subs:                       # two calls in a row share the static array
            rc, rec, msg = static_record(lib, lines, t, run, p.pressure[level],
                                         p.temperature[level], p.density[level], isub)
            assert rc == 0, msg
            assert rel_err(rec, full[isub], 0.0)[0] <= tol


def test_static_record_rejects_windows_beyond_capacity(gpu, tips):
    lib = gpu
    dense = synth.make_lines(synth.LineSpec(n=80_000, nu_lo=4000.0, nu_hi=4100.0, seed=9))
    run = Run(4000.0, 4100.0, 25.0, molecule="CO2", precision="fp32c")
    rc, rec, msg = static_record(lib, dense, np.ascontiguousarray(tips), run, 1.0, 296.0, 2.39e24, 4)
    assert rc == 15 and "static capacity" in msg


def regular_record(lines, tips, run, P, T, n, isub):
    f = lambda x: np.asarray([x], dtype=np.float64)
    with Context(lines, tips) as ctx:
        return ctx.compute(run, f(P), f(T), f(n))[0][isub]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32c", 1e-6)])
def test_static_record_dense_band_stages_in_the_static_array(gpu, tips, prec, tol):
    """5,000 lines within [4049, 4061]: more near lines than either precision
    stages on chip, so the static array's staging region is used."""
    lib = gpu
    t = np.ascontiguousarray(tips)
    lines = np.ascontiguousarray(synth.make_lines(synth.LineSpec(n=5000, nu_lo=4049.0, nu_hi=4061.0, seed=5)))
    run = Run(4040.0, 4070.0, 25.0, molecule="CO2", precision=prec)
    P, T = 1.0, 296.0
    n = float(synth.ideal_gas_density(synth.f32([P]), synth.f32([T]))[0])
    full = [regular_record(lines, t, run, P, T, n, isub) for isub in (1,)]
    for _ in range(2):
        rc, rec, msg = static_record(lib, lines, t, run, P, T, n, 1)
        assert rc == 0, msg
        assert rel_err(rec, full[0], 0.0)[0] <= tol


def test_static_record_empty_window(gpu, tips):
    """A subinterval whose window holds no line (a gap in the line list wider
    than twice the cutoff) gives an all-zero record, like the regular entry
    point."""
    lib = gpu
    t = np.ascontiguousarray(tips)
    a = synth.make_lines(synth.LineSpec(n=500, nu_lo=4000.0, nu_hi=4050.0, seed=6))[:-1]
    b = synth.make_lines(synth.LineSpec(n=500, nu_lo=4200.0, nu_hi=4300.0, seed=7))
    lines = np.ascontiguousarray(np.concatenate([a, b]))
    run = Run(4100.0, 4200.0, 25.0, molecule="CO2", precision="fp32c")
    P, T = 1.0, 296.0
    n = float(synth.ideal_gas_density(synth.f32([P]), synth.f32([T]))[0])
    full = regular_record(lines, t, run, P, T, n, 1)
    rc, rec, msg = static_record(lib, lines, t, run, P, T, n, 1)
    assert rc == 0, msg
    assert not np.any(full) and not np.any(rec)


def test_static_record_rejects_windows_beyond_line_capacity(gpu, tips):
    """A window of more than MARFA_STATIC_MAX_WINDOW_LINES lines."""
    lib = gpu
    lines = synth.make_lines(synth.LineSpec(n=200_000, nu_lo=4000.0, nu_hi=4100.0, seed=8))
    run = Run(4000.0, 4100.0, 25.0, molecule="CO2", precision="fp64")
    rc, rec, msg = static_record(lib, lines, np.ascontiguousarray(tips), run, 1.0, 296.0, 2.39e24, 5)
    assert rc == 15 and "window of" in msg and "static capacity" in msg


FIRST_CALL = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import numpy as np
from test_zz_no_alloc import static_record, regular_record
from marfa_b200 import _lib, synth, data_path
from marfa_b200.io import read_tips
from marfa_b200.api import Run
lib = _lib.load()
tips = np.ascontiguousarray(read_tips(data_path("TIPS_subset.dat")))
w = synth.config(0)
lines = np.ascontiguousarray(w.lines)
p = w.profiles[0]
run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi, precision="fp64")
rc, rec, msg = static_record(lib, lines, tips, run, p.pressure[0], p.temperature[0], p.density[0], 4)
assert rc == 0, msg
full = regular_record(lines, tips, run, p.pressure[0], p.temperature[0], p.density[0], 4)
err = float(np.max(np.abs(rec.astype(np.float64) - full) / np.maximum(np.abs(full), 1e-300)))
assert err <= 1e-12, err
print("first call ok", err)
"""


def test_static_record_as_first_call_of_a_process(gpu):
    """A process whose first library call is the allocation-free one (no
    context exists yet on the device)."""
    import subprocess
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parent.parent)
    r = subprocess.run([sys.executable, "-c", FIRST_CALL, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "first call ok" in r.stdout
