"""GPU parity on the reference's own inputs: its CO line database (the
1900-2400 cm-1 slice of data/databases/HITRAN2020.05: six isotopologues,
HITRAN pressure shifts down to -0.019 cm-1/atm) and its Haus 2015 Venus
profile (data/Atmospheres/VenusCO2-3.dat), as fixtures made by
tests/golden/make_real_golden.py.

Over 2000-2300 cm-1 with a 25 cm-1 cutoff, at six levels from the surface
(91 atm, 733 K: shifts of up to -1.7 cm-1 reorder the lines and move them
across subinterval edges) to the top of the profile, for both targets:
- line windows equal to the oracle's;
- evaluation counts equal to the oracle's;
- FP64 records within 1e-12 of the all-double oracle on every point;
- FP32c within 1e-5 where k > 1e-6 max(k), outside cascade near-ties."""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from fp32c_check import check_fp32c
from marfa_b200.api import Context, Run, plan_windows
from marfa_b200.io import read_lines, read_profile

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
START, END, CUT = 2000.0, 2300.0, 25.0


@pytest.fixture(scope="module")
def real():
    lines = read_lines(GOLD / "co_hitran2020_1900_2400.lines")
    _, _, P, T, n = read_profile(GOLD / "VenusCO2-3.dat")
    lv = np.arange(0, len(P), 13)
    return lines, P[lv], T[lv], n[lv]


@pytest.mark.parametrize("target", ["ACS", "VAC"])
def test_real_co_band_matches_oracle(gpu, tips, real, target):
    lines, P, T, n = real
    orc = O.Oracle(lines, tips, P, T, n, START, END, CUT, target=target, chi="none", mol_code=5,
                   precision=O.FP64)
    _, ref, ev_ref = orc.run()
    lo_ref, hi_ref = orc.windows()
    lo, hi = plan_windows(lines["nu"], START, END, CUT)      # 0-based; the oracle's are 1-based
    assert np.array_equal(lo + 1, lo_ref) and np.array_equal(hi + 1, hi_ref)
    run = dict(start_wv=START, end_wv=END, cutoff=CUT, target=target, molecule="CO", chi="none")
    with Context(lines, tips) as ctx:
        _, g64 = ctx.compute(Run(precision="fp64", **run), P, T, n, want64=True)
        g32 = ctx.compute(Run(precision="fp32c", **run), P, T, n)
        ev = ctx.eval_count(Run(precision="fp64", **run), P, T, n)
    assert np.array_equal(np.asarray(ev), ev_ref), (ev, ev_ref)
    err, npts = rel_err(g64, ref, 0.0)
    assert npts == ref.size and err <= 1e-12, err
    e32, taint = check_fp32c(g32, ref, orc, tol=1e-5)
    print(f"{target}: {int(ev_ref.sum())} evaluations, FP64 max err {err:.2e}, "
          f"FP32c max err {e32:.2e} outside {taint} near-tie points")
    assert e32 <= 1e-5 and taint <= 1e-4 * ref.size
