"""GPU parity on the reference's own inputs: slices of its CO and O2 line
databases (data/databases/HITRAN2020.05, 1900-2400 cm-1: six isotopologues,
HITRAN pressure shifts down to -0.019 cm-1/atm; HITRAN2020.07, 12900-13300
cm-1: the A band of three isotopologues, centres near 1.3e4 cm-1) and its
Haus 2015 Venus profile (data/Atmospheres/VenusCO2-3.dat), as fixtures made
by tests/golden/make_real_golden.py.

Over 2000-2300 cm-1 (CO, both targets) and 13000-13200 cm-1 (O2) with a 25
cm-1 cutoff, at six levels from the surface (91 atm, 733 K: shifts of up to
-1.7 cm-1 reorder the lines and move them across subinterval edges) to the
top of the profile:
- line windows equal to the oracle's;
- evaluation counts equal to the oracle's;
- FP64 records within 1e-12 of the all-double oracle on every point;
- FP32c within 1e-5 where k > 1e-6 max(k), outside cascade near-ties.
And the `marfa` command run on the same files in the reference's directory
layout writes PT files equal to the oracle's records within float32
rounding at every level of the profile."""
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
CUT = 25.0
# (fixture, molecule, HITRAN molecule number, interval): the CO fundamental
# band and the O2 A band (centres near 1.3e4 cm-1, against grid offsets of
# 5e-4 cm-1)
BANDS = {"co": ("co_hitran2020_1900_2400.lines", "CO", 5, 2000.0, 2300.0),
         "o2": ("o2_hitran2020_12900_13300.lines", "O2", 7, 13000.0, 13200.0)}


def levels():
    _, _, P, T, n = read_profile(GOLD / "VenusCO2-3.dat")
    lv = np.arange(0, len(P), 13)
    return P[lv], T[lv], n[lv]


@pytest.mark.parametrize("band,target", [("co", "ACS"), ("co", "VAC"), ("o2", "VAC")])
def test_real_band_matches_oracle(gpu, tips, band, target):
    name, molecule, mol_code, start, end = BANDS[band]
    lines = read_lines(GOLD / name)
    P, T, n = levels()
    orc = O.Oracle(lines, tips, P, T, n, start, end, CUT, target=target, chi="none", mol_code=mol_code,
                   precision=O.FP64)
    _, ref, ev_ref = orc.run()
    lo_ref, hi_ref = orc.windows()
    lo, hi = plan_windows(lines["nu"], start, end, CUT)      # 0-based; the oracle's are 1-based
    assert np.array_equal(lo + 1, lo_ref) and np.array_equal(hi + 1, hi_ref)
    run = dict(start_wv=start, end_wv=end, cutoff=CUT, target=target, molecule=molecule, chi="none")
    with Context(lines, tips) as ctx:
        _, g64 = ctx.compute(Run(precision="fp64", **run), P, T, n, want64=True)
        g32 = ctx.compute(Run(precision="fp32c", **run), P, T, n)
        ev = ctx.eval_count(Run(precision="fp64", **run), P, T, n)
    assert np.array_equal(np.asarray(ev), ev_ref), (ev, ev_ref)
    err, npts = rel_err(g64, ref, 0.0)
    assert npts == ref.size and err <= 1e-12, err
    e32, taint = check_fp32c(g32, ref, orc, tol=1e-5)
    print(f"{band} {target}: {int(ev_ref.sum())} evaluations, FP64 max err {err:.2e}, "
          f"FP32c max err {e32:.2e} outside {taint} near-tie points")
    assert e32 <= 1e-5 and taint <= 1e-4 * ref.size


def test_marfa_command_on_reference_inputs(gpu, tips, tmp_path):
    """`marfa CO 2000 2100 HITRAN2020 25 VAC VenusCO2-3.dat fp64` in a tree of
    the reference's layout (its CO line slice as data/databases/HITRAN2020.05,
    its profile, the TIPS rows in the full-table layout) writes one PT file
    per level of the 66-level profile; every record equals the all-double
    oracle's within float32 rounding (1e-6)."""
    import subprocess
    from marfa_b200 import build, data_path
    from marfa_b200.io import RECORD_BYTES, pt_name, record_number, subinterval_starts
    for d in ("data/Atmospheres", "data/databases", "data/TIPS", "output/ptTables"):
        (tmp_path / d).mkdir(parents=True)
    (tmp_path / "data/databases/HITRAN2020.05").write_bytes((GOLD / "co_hitran2020_1900_2400.lines").read_bytes())
    (tmp_path / "data/Atmospheres/VenusCO2-3.dat").write_bytes((GOLD / "VenusCO2-3.dat").read_bytes())
    sub = data_path("TIPS_subset.dat").read_text().splitlines()
    rows = {int(l.split(":")[0]): l.split(":", 1)[1].strip() for l in sub[1:]}
    zero = ", ".join(["0.0"] * 501)
    (tmp_path / "data/TIPS/TIPS.dat").write_text(
        "74, 501\n" + "\n".join(rows.get(i, zero) for i in range(1, 75)) + "\n")
    build.build()
    marfa = Path(__file__).resolve().parent.parent / "marfa_b200" / "marfa"
    r = subprocess.run([str(marfa), "CO", "2000", "2100", "HITRAN2020", "25", "VAC", "VenusCO2-3.dat", "fp64"],
                       cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    latest = (tmp_path / "output/ptTables/latest_run.txt").read_text().strip()
    out = tmp_path / "output/ptTables" / latest
    lines = read_lines(GOLD / "co_hitran2020_1900_2400.lines")
    _, _, P, T, n = read_profile(GOLD / "VenusCO2-3.dat")
    orc = O.Oracle(lines, tips, P, T, n, 2000.0, 2100.0, 25.0, target="VAC", chi="none", mol_code=5,
                   precision=O.FP64)
    _, ref, _ = orc.run()
    starts = subinterval_starts(2000.0, 2100.0)
    worst = 0.0
    for lev in range(len(P)):
        raw = (out / pt_name(lev + 1)).read_bytes()
        for i, s in enumerate(starts):
            k = record_number(s) - 1
            rec = np.frombuffer(raw[k * RECORD_BYTES:(k + 1) * RECORD_BYTES], dtype="<f4")
            worst = max(worst, rel_err(rec, ref[lev, i], 0.0)[0])
    print(f"{len(P)} levels x {len(starts)} records: max err {worst:.2e}")
    assert worst <= 1e-6
