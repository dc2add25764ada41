"""The C-ABI library: exports, host-side logic, loud failure without a GPU (CPU)."""
import ctypes
import re

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from marfa_b200 import _lib, build, synth
from marfa_b200.api import num_subintervals, plan_windows
from test_oracle import edge_lines


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    header = (ROOT / "include" / "marfa_gpu.h").read_text()
    declared = set(re.findall(r"\b(marfa_[a-z0-9_]+)\s*\(", header))
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert getattr(lib, name)


def test_plan_windows_matches_oracle(lib, tips):
    cases = [(synth.config(0).lines, 4000.0, 4100.0, 25.0),
             (synth.config(0).lines, 4003.5, 4097.0, 13.0),
             (edge_lines(), 4050.0, 4060.0, 25.0),
             (edge_lines(), 4020.0, 4080.0, 0.75),
             (synth.config(2, 0.1).lines, 10.0, 300.0, 25.0)]
    for lines, a, b, cut in cases:
        o = O.Oracle(lines, tips, [1.0], [296.0], [1e20], a, b, cut)
        lo, hi = o.windows()
        glo, ghi = plan_windows(lines["nu"], a, b, cut)
        assert np.array_equal(glo, lo - 1) and np.array_equal(ghi, hi - 1)


def test_plan_windows_without_sentinel_is_status_9(lib):
    lines = synth.config(0).lines[:-1]
    with pytest.raises(_lib.MarfaError) as e:
        plan_windows(lines["nu"], 4000.0, 4100.0, 25.0)
    assert e.value.code == 9


def test_subinterval_counts_and_records(lib):
    for a, b in ((4000.0, 4100.0), (4000.0, 4095.0), (10.0, 3000.0), (4003.7, 4050.2)):
        assert num_subintervals(a, b) == O.lib().oracle_num_subintervals(a, b)
        for i in range(num_subintervals(a, b)):
            assert lib.marfa_record_number(a, i) == O.lib().oracle_record_number(a, i)


def test_no_cpu_fallback_without_gpu(lib, tips):
    """Without a CUDA device the library refuses to run (status 110)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    lines = synth.config(0).lines
    h = ctypes.c_void_p()
    t = np.ascontiguousarray(tips)
    rc = lib.marfa_ctx_create(lines.ctypes.data, len(lines), t.ctypes.data, 74, 501, 0, ctypes.byref(h))
    assert rc == 110


@pytest.mark.parametrize("name,start,end", [("co_hitran2020_1900_2400.lines", 2000.0, 2300.0),
                                            ("o2_hitran2020_12900_13300.lines", 13000.0, 13200.0)])
def test_plan_windows_on_reference_databases(lib, tips, name, start, end):
    """Windows of the host planner on slices of the reference's own line
    databases (tests/golden/make_real_golden.py) equal the oracle's."""
    from marfa_b200.io import read_lines
    lines = read_lines(ROOT / "tests" / "golden" / name)
    lo, hi = plan_windows(lines["nu"], start, end, 25.0)
    o = O.Oracle(lines, tips, [1.0], [296.0], [1e10], start, end, 25.0)
    olo, ohi = o.windows()
    assert np.array_equal(lo + 1, olo) and np.array_equal(hi + 1, ohi)

