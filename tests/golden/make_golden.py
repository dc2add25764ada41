"""Regenerate the golden fixtures of tests/golden from the reference tree.

The reference's only fixture pair for this path is test/testDB.txt (five CO2
lines in HITRAN .par format) and test/testDB.02 (their 36-byte database
records written by app/processParFile.f90).  This script copies both, byte
for byte, into tests/golden so the tests run where the reference is absent:
    python tests/golden/make_golden.py /path/to/reference
"""
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main():
    ref = Path(sys.argv[1])
    shutil.copyfile(ref / "test" / "testDB.txt", HERE / "testDB.par")
    shutil.copyfile(ref / "test" / "testDB.02", HERE / "testDB.02")


if __name__ == "__main__":
    main()
