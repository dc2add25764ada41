"""The `marfa` command: argument and input errors with the reference's exit
codes (CPU), and a full run writing PT-tables (GPU)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, rel_err
from marfa_b200 import build, synth, data_path
from marfa_b200.io import (NT, RECORD_BYTES, pt_name, record_number, subinterval_starts,
                           write_lines, write_profile)

MARFA = ROOT / "marfa_b200" / "marfa"


def make_tree(tmp: Path, w, tips_path=None, levels=None):
    (tmp / "data" / "Atmospheres").mkdir(parents=True)
    (tmp / "data" / "databases").mkdir(parents=True)
    (tmp / "data" / "TIPS").mkdir(parents=True)
    (tmp / "output" / "ptTables").mkdir(parents=True)
    p = w.profiles[0]
    sl = slice(None) if levels is None else levels
    write_profile(tmp / "data" / "Atmospheres" / "syn.dat", "synthetic", p.height[sl],
                  p.pressure[sl], p.temperature[sl], p.density[sl])
    write_lines(tmp / "data" / "databases" / "SYN.02", w.lines)
    # full-layout TIPS file built from the subset (rows not used stay zero)
    sub = data_path("TIPS_subset.dat").read_text().splitlines()
    rows = {int(l.split(":")[0]): l.split(":", 1)[1].strip() for l in sub[1:]}
    zero = ", ".join(["0.0"] * 501)
    (tmp / "data" / "TIPS" / "TIPS.dat").write_text(
        "74, 501\n" + "\n".join(rows.get(i, zero) for i in range(1, 75)) + "\n")


def run(tmp, *args):
    build.build()
    return subprocess.run([str(MARFA), *map(str, args)], cwd=tmp, capture_output=True, text=True)


def test_exit_codes(tmp_path):
    w = synth.config(0)
    make_tree(tmp_path, w)
    assert run(tmp_path, "CO2", 4000).returncode == 1
    assert run(tmp_path, "CO2", 4000, 4100, "SYN", 25, "XYZ", "syn.dat").returncode == 2
    assert run(tmp_path, "CO2", 4000, 4100, "SYN", 25, "ACS", "missing.dat").returncode == 7
    (tmp_path / "data" / "Atmospheres" / "big.dat").write_text("t\n201\n" + "1 1 300 1\n" * 201)
    assert run(tmp_path, "CO2", 4000, 4100, "SYN", 25, "ACS", "big.dat").returncode == 6
    (tmp_path / "data" / "Atmospheres" / "bad.dat").write_text("t\n2\n1 1 300 1\n1 1 x\n")
    assert run(tmp_path, "CO2", 4000, 4100, "SYN", 25, "ACS", "bad.dat").returncode == 7
    assert run(tmp_path, "XE", 4000, 4100, "SYN", 25, "ACS", "syn.dat").returncode == 8
    assert run(tmp_path, "H2O", 4000, 4100, "SYN", 25, "ACS", "syn.dat").returncode == 9


@pytest.mark.gpu
def test_full_run_writes_reference_pt_tables(tmp_path, gpu, tips):
    w = synth.config(0)
    make_tree(tmp_path, w)
    r = run(tmp_path, "CO2", 4000, 4100, "SYN", 25, "ACS", "syn.dat", "fp64")
    assert r.returncode == 0, r.stdout + r.stderr
    latest = (tmp_path / "output" / "ptTables" / "latest_run.txt").read_text().strip()
    d = tmp_path / "output" / "ptTables" / latest
    assert latest.startswith("CO2_4000-4100_")
    info = (d / "info.txt").read_text().splitlines()
    assert info[0] == "Command-Line Arguments:" and "Cut Off: 25" in info
    raw = (d / pt_name(1)).read_bytes()
    assert len(raw) == (record_number(4090.0)) * RECORD_BYTES
    o = O.from_workload(w, precision=O.FP64, tips=tips)
    ref = o.run()[0][0]
    for i, s in enumerate(subinterval_starts(4000.0, 4100.0)):
        k = record_number(s) - 1
        rec = np.frombuffer(raw[k * RECORD_BYTES:(k + 1) * RECORD_BYTES], dtype="<f4")
        assert rel_err(rec, ref[i], 0.0)[0] <= 1e-6
