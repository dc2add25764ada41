"""Generate marfa_wiso.h: the isotopologue molar-mass table WISO(124).

The values are physical data that the line-shape arithmetic must reproduce
exactly (Doppler half-width uses WISO(jointMolIso/100)), so they are taken
verbatim, in order, from the reference's MolarMasses.f90:9-145 (the WISO array
is the concatenation of the per-molecule arrays, MolarMasses.f90:140-145).

Run once, where the reference tree is present:
    python marfa_b200/csrc/gen_tables.py /path/to/reference/src/MolarMasses.f90
"""
import re
import sys
from pathlib import Path


def parse(path):
    src = Path(path).read_text()
    arrays = {}
    for m in re.finditer(r"real, parameter :: (WISO_\w+)\((\d+)\) = \[(.*?)\]", src, re.S):
        vals = [v.strip() for v in m.group(3).replace("&", "").split(",") if v.strip()]
        if len(vals) != int(m.group(2)):
            raise ValueError(f"{m.group(1)}: expected {m.group(2)} values, got {len(vals)}")
        arrays[m.group(1)] = vals
    order = re.search(r"WISO\(124\) = \[(.*?)\]", src, re.S).group(1).replace("&", "").split(",")
    out = []
    for name in (o.strip() for o in order if o.strip()):
        out += arrays[name]
    if len(out) != 124:
        raise ValueError("WISO must have 124 entries")
    return out


def literal(v, suffix):
    if "." not in v and "e" not in v.lower():
        v += ".0"
    return v + suffix


def main():
    vals = parse(sys.argv[1])
    lines = [
        "/* marfa_wiso.h -- generated by gen_tables.py; do not edit.",
        " * Isotopologue molar masses [g/mol], WISO(1..124) of the reference",
        " * (MolarMasses.f90:9-145), index = jointMolIso / 100. */",
        "#ifndef MARFA_WISO_H",
        "#define MARFA_WISO_H",
        "#define MARFA_WISO_LEN 124",
    ]
    for name, suffix in (("MARFA_WISO_F", "f"), ("MARFA_WISO_D", "")):
        ctype = "float" if suffix else "double"
        lines.append(f"static const {ctype} {name}[MARFA_WISO_LEN] = {{")
        for i in range(0, 124, 6):
            lines.append("    " + ", ".join(literal(v, suffix) for v in vals[i:i + 6]) + ",")
        lines.append("};")
    lines.append("#endif")
    out = Path(__file__).with_name("marfa_wiso.h")
    out.write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
