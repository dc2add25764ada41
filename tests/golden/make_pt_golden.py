"""Golden vectors of the PT-table reader and text converter, made by the
reference's own Python handlers (handlers/parsers.py:base_parser,
handlers/convert.py:convert_pttable), which are plain numpy.

The input is a run directory that this repository's writers produce from a
seeded record set (write_info, write_pt_table: the CLI's output format).  The
reference reads and converts it; the SHA-256 of its results (float32 bytes of
the wavenumbers and values, the converted text) and its error message for a
range beyond the file go to pt_convert.json.  tests/test_formats.py rebuilds
the same input and checks the library's reader and converter against them.

    python tests/golden/make_pt_golden.py /path/to/reference
"""
import hashlib
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

# v1, v2 of the reads: the run's range, one starting a record before the first
# written record (a hole of zeros), one ending beyond the file
CASES = [(4000.0, 4030.0), (3990.0, 4015.0), (4000.0, 4041.0)]
RUN = {"molecule": "CO2", "start": 4000.0, "end": 4030.0, "level": 7, "seed": 11}


def make_run(directory: Path):
    """The seeded run directory: info.txt and the level's PT table."""
    from marfa_b200.io import pt_name, write_info, write_pt_table
    rng = np.random.default_rng(RUN["seed"])
    recs = (np.exp(rng.uniform(-40, -20, (3, 20481)))).astype(np.float32)
    write_info(directory, RUN["molecule"], RUN["start"], RUN["end"], 25.0, "ACS", "syn.dat")
    write_pt_table(directory / pt_name(RUN["level"]), RUN["start"], recs)


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def main():
    ref = Path(sys.argv[1])
    sys.path.insert(0, str(ref))
    from handlers import convert, parsers  # the reference's modules
    from marfa_b200.io import pt_name
    out = {"run": RUN, "cases": []}
    with tempfile.TemporaryDirectory() as tmp:
        run = Path(tmp) / "run"
        run.mkdir()
        make_run(run)
        out["ptbin_sha256"] = sha((run / pt_name(RUN["level"])).read_bytes())
        for v1, v2 in CASES:
            case = {"v1": v1, "v2": v2}
            try:
                wv, vals = parsers.base_parser(run / pt_name(RUN["level"]), v1, v2)
                case["wv_sha256"] = sha(np.asarray(wv, dtype=np.float32).tobytes())
                case["values_sha256"] = sha(np.asarray(vals, dtype=np.float32).tobytes())
                case["points"] = len(wv)
            except IndexError as e:
                case["index_error"] = str(e)
            out["cases"].append(case)
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            Path("output/processedData").mkdir(parents=True)
            convert.convert_pttable(run, RUN["level"])
            (txt,) = Path("output/processedData").iterdir()
            out["converted_name"] = txt.name
            out["converted_sha256"] = sha(txt.read_bytes())
        finally:
            os.chdir(cwd)
    (HERE / "pt_convert.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
