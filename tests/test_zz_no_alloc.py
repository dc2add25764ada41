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
