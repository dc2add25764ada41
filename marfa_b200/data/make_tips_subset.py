"""Extract the TIPS rows used by the workloads (isotopologue 1, H2O 161, and
10, CO2 626, of the synthetic ones; 46-51, the six CO isotopologues, and
59-61, the three O2 isotopologues, of the real-data tests) from a reference
TIPS table into TIPS_subset.dat.

The partition sums are physical data (Gamache et al. 2017, as shipped in the
reference's data/TIPS/TIPS.dat) that the intensity scaling must reproduce
exactly, so the values are copied as text, unchanged.  Run where the
reference tree is present:
    python marfa_b200/data/make_tips_subset.py /path/to/data/TIPS/TIPS.dat
"""
import sys
from pathlib import Path

ROWS = (1, 10, 46, 47, 48, 49, 50, 51, 59, 60, 61)


def main():
    src = Path(sys.argv[1]).read_text().splitlines()
    head = src[0]
    out = [head]
    for r in ROWS:
        out.append(f"{r}: {src[r].strip()}")
    Path(__file__).with_name("TIPS_subset.dat").write_text("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
