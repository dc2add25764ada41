"""Real-data fixtures for the GPU parity test on the reference's own inputs:
the 1900-2400 cm-1 slice of the reference's CO line database
(data/databases/HITRAN2020.05: the fundamental band of six isotopologues,
with HITRAN's pressure shifts) as 36-byte records plus the sentinel record
the library expects at the end of a line list, and the reference's Venus
profile data/Atmospheres/VenusCO2-3.dat (Haus 2015, 66 levels), copied
unchanged.  Run where the reference tree is present:
    python tests/golden/make_real_golden.py /path/to/reference
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from marfa_b200.io import LINE_DTYPE, read_lines, write_lines  # noqa: E402

LO, HI = 1900.0, 2400.0


def main():
    ref = Path(sys.argv[1])
    lines = read_lines(ref / "data" / "databases" / "HITRAN2020.05")
    keep = lines[(lines["nu"] >= LO) & (lines["nu"] <= HI)]
    sentinel = np.zeros(1, dtype=LINE_DTYPE)
    sentinel["nu"] = 1e5
    sentinel["jmi"] = keep["jmi"][-1]
    write_lines(HERE / "co_hitran2020_1900_2400.lines", np.concatenate([keep, sentinel]))
    prof = (ref / "data" / "Atmospheres" / "VenusCO2-3.dat").read_bytes()
    (HERE / "VenusCO2-3.dat").write_bytes(prof)
    print(len(keep), "lines")


if __name__ == "__main__":
    main()
