"""Real-data fixtures for the GPU parity test on the reference's own inputs:
slices of two of the reference's line databases as 36-byte records, each
followed by the sentinel record the library expects at the end of a line
list -- 1900-2400 cm-1 of data/databases/HITRAN2020.05 (the CO fundamental
band, six isotopologues) and 12900-13300 cm-1 of HITRAN2020.07 (the O2 A
band, three isotopologues), both with HITRAN's pressure shifts -- and the
reference's Venus profile data/Atmospheres/VenusCO2-3.dat (Haus 2015, 66
levels), copied unchanged.  Run where the reference tree is present:
    python tests/golden/make_real_golden.py /path/to/reference
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from marfa_b200.io import LINE_DTYPE, read_lines, write_lines  # noqa: E402

SLICES = (("HITRAN2020.05", 1900.0, 2400.0, "co_hitran2020_1900_2400.lines"),
          ("HITRAN2020.07", 12900.0, 13300.0, "o2_hitran2020_12900_13300.lines"))


def main():
    ref = Path(sys.argv[1])
    for db, lo, hi, name in SLICES:
        lines = read_lines(ref / "data" / "databases" / db)
        keep = lines[(lines["nu"] >= lo) & (lines["nu"] <= hi)]
        sentinel = np.zeros(1, dtype=LINE_DTYPE)
        sentinel["nu"] = 1e5
        sentinel["jmi"] = keep["jmi"][-1]
        write_lines(HERE / name, np.concatenate([keep, sentinel]))
        print(name, len(keep), "lines")
    prof = (ref / "data" / "Atmospheres" / "VenusCO2-3.dat").read_bytes()
    (HERE / "VenusCO2-3.dat").write_bytes(prof)


if __name__ == "__main__":
    main()
