"""File formats and the reference's own fixture (CPU)."""
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from marfa_b200 import data_path
from marfa_b200.ingest import decimal_to_f32, parse_par, isotopologue_number
from marfa_b200.io import (LINE_DTYPE, MarfaFormatError, NT, RECORD_BYTES, pt_name, read_lines,
                           read_profile, read_pt_table, read_tips, record_number,
                           subinterval_starts, write_profile, write_pt_table)

GOLDEN = ROOT / "tests" / "golden"


def test_par_conversion_matches_reference_fixture_bytes():
    """test/testDB.txt -> test/testDB.02 of the reference: the five CO2 .par
    lines convert to exactly the reference's 180 database bytes."""
    recs = parse_par((GOLDEN / "testDB.par").read_text().splitlines(True), "CO2")
    ref = (GOLDEN / "testDB.02").read_bytes()
    assert len(ref) == 180
    assert recs.tobytes() == ref


def test_line_record_layout():
    recs = read_lines(GOLDEN / "testDB.02")
    assert recs.dtype.itemsize == 36
    assert recs["jmi"].tolist() == [1002] * 5            # CO2 626: isotopologue 10, molecule 2
    assert recs["nu"][0] == 648.888078
    assert recs["delta"][4] == np.float32(-0.005872)


def test_isotopologue_numbers():
    assert isotopologue_number(1, 1) == 1        # H2O 161
    assert isotopologue_number(2, 1) == 10       # CO2 626
    assert isotopologue_number(12, 2) == 74      # last HNO3
    assert isotopologue_number(2, 14) == 0


def test_decimal_to_f32_is_correctly_rounded():
    for s in ["0.0705", ".096", "-.000709", "0.73", "1.4", "3.1415926"]:
        v = decimal_to_f32(s)
        ex = Fraction(s if not s.startswith((".", "-.")) else s.replace(".", "0.", 1))
        up = np.nextafter(v, np.float32(np.inf))
        dn = np.nextafter(v, np.float32(-np.inf))
        err = abs(Fraction(float(v)) - ex)
        assert err <= abs(Fraction(float(up)) - ex) and err <= abs(Fraction(float(dn)) - ex)


def test_tips_values_round_identically_through_double():
    """The library takes TIPS as doubles; a value parsed via double and then
    rounded to float must equal the direct decimal->float rounding the
    reference's list-directed read performs (no double rounding)."""
    text = data_path("TIPS_subset.dat").read_text().splitlines()[1:]
    for line in text:
        for tok in line.split(":", 1)[1].replace(",", " ").split():
            assert np.float32(float(tok)) == decimal_to_f32(tok)


def test_tips_subset_rows():
    t = read_tips(data_path("TIPS_subset.dat"))
    assert t.shape == (74, 501)
    assert np.isfinite(t[0]).all() and np.isfinite(t[9]).all()
    assert np.isnan(t[1]).all()


def test_pt_names_and_records():
    assert pt_name(1) == "1__.ptbin" and pt_name(12) == "12_.ptbin" and pt_name(123) == "123.ptbin"
    assert record_number(4000.0) == 400 and record_number(10.0) == 1 and record_number(560.0) == 56
    assert subinterval_starts(4000, 4100) == [4000.0 + 10 * i for i in range(10)]
    assert len(subinterval_starts(4000, 4095)) == 10


def test_pt_table_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    recs = rng.random((3, NT), dtype=np.float32)
    f = tmp_path / "1__.ptbin"
    write_pt_table(f, 4000.0, recs)
    assert f.stat().st_size == 402 * RECORD_BYTES           # records 400..402, leading holes
    assert not np.frombuffer(f.read_bytes()[:RECORD_BYTES], np.float32).any()
    wv, vals = read_pt_table(f, 4000.0, 4030.0)
    assert np.array_equal(vals, recs.ravel())
    assert wv[0] == np.float32(4000.0) and wv[NT] == np.float32(4010.0)


def test_profile_roundtrip_and_errors(tmp_path):
    from marfa_b200.synth import venus_profile
    p = venus_profile(40)
    f = tmp_path / "v.dat"
    write_profile(f, "Venus test", p.height, p.pressure, p.temperature, p.density)
    title, h, P, T, n = read_profile(f)
    assert np.array_equal(P, p.pressure) and np.array_equal(T, p.temperature)
    assert np.array_equal(n, p.density)
    f.write_text("t\n201\n" + "1 1 300 1\n" * 201)
    with pytest.raises(MarfaFormatError) as e:
        read_profile(f)
    assert e.value.code == 6
    f.write_text("t\n2\n1 1 300 1\n1 x 300 1\n")
    with pytest.raises(MarfaFormatError) as e:
        read_profile(f)
    assert e.value.code == 7


def test_pt_reader_and_converter_match_reference_handlers(tmp_path):
    """The reader and the text converter against golden vectors that the
    reference's own handlers (parsers.base_parser, convert.convert_pttable)
    produced for the same run directory (tests/golden/make_pt_golden.py):
    wavenumbers and values bit for bit, the converted text byte for byte, and
    the reference's error for a range beyond the file."""
    import hashlib
    import json
    import sys
    sys.path.insert(0, str(GOLDEN))
    from make_pt_golden import make_run
    from marfa_b200.io import convert_pt_table
    gold = json.loads((GOLDEN / "pt_convert.json").read_text())
    sha = lambda b: hashlib.sha256(b).hexdigest()
    run = tmp_path / "run"
    run.mkdir()
    make_run(run)
    level = gold["run"]["level"]
    assert sha((run / pt_name(level)).read_bytes()) == gold["ptbin_sha256"]
    for case in gold["cases"]:
        if "index_error" in case:
            with pytest.raises(IndexError) as e:
                read_pt_table(run / pt_name(level), case["v1"], case["v2"])
            assert str(e.value) == case["index_error"]
            continue
        wv, vals = read_pt_table(run / pt_name(level), case["v1"], case["v2"])
        assert len(wv) == case["points"]
        assert sha(wv.astype(np.float32).tobytes()) == case["wv_sha256"]
        assert sha(vals.astype(np.float32).tobytes()) == case["values_sha256"]
    out = tmp_path / "processed"
    out.mkdir()
    txt = convert_pt_table(run, level, out)
    assert txt.name == gold["converted_name"]
    assert sha(txt.read_bytes()) == gold["converted_sha256"]
