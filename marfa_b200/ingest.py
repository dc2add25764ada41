"""HITRAN .par -> 36-byte line database conversion.

Restates app/processParFile.f90: the fixed-format read of
'(I2, A1, F12.6, 2E10.3, 2F5.4, F10.4, F4.2, F8.6, ...)' (:94), the
isotopologue letter code (convert_ISO, :226-271), the internal isotopologue
number N_MOL_ISO(ISO, MOL) (:69-93) and jointMolIso = iso*100 + mol (:171-174).
Fields read into double (wavenumber, and intensity and lower-state energy,
which the reference then narrows to float, :167-168) go through double; the
fields read straight into default reals are rounded once from their decimal
text, as a Fortran formatted read does.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

from .io import LINE_DTYPE, SPECIES_CODES

# internal isotopologue numbers per molecule (processParFile.f90:69-93):
# molecule m owns a contiguous block, in HITRAN isotopologue order.
_ISO_COUNTS = (9, 13, 18, 5, 9, 4, 6, 3, 2, 1, 2, 2)
_ISO_BASE = np.concatenate([[0], np.cumsum(_ISO_COUNTS)[:-1]])

_ISO_CODES = {**{str(d): d for d in range(1, 10)}, "0": 10,
              **{c: 11 + i for i, c in enumerate("ABCDEFGHI")}}


def isotopologue_number(mol: int, iso: int) -> int:
    """N_MOL_ISO(iso, mol); 0 for an isotopologue the table does not hold."""
    if not 1 <= mol <= len(_ISO_COUNTS) or not 1 <= iso <= _ISO_COUNTS[mol - 1]:
        return 0
    return int(_ISO_BASE[mol - 1]) + iso


def decimal_to_f32(text: str) -> np.float32:
    """Correctly rounded decimal -> float32 (one rounding from the exact
    decimal value, as a formatted read into a default real)."""
    t = text.strip()
    if not t:
        return np.float32(0.0)
    if t.startswith("."):
        t = "0" + t
    elif t.startswith("-.") or t.startswith("+."):
        t = t[0] + "0" + t[1:]
    exact = Fraction(t.replace("D", "E").replace("d", "e"))
    guess = np.float32(float(exact))
    best = guess
    for cand in (np.nextafter(guess, np.float32(-np.inf)), guess,
                 np.nextafter(guess, np.float32(np.inf))):
        if abs(Fraction(float(cand)) - exact) < abs(Fraction(float(best)) - exact):
            best = cand
        elif abs(Fraction(float(cand)) - exact) == abs(Fraction(float(best)) - exact):
            # ties to even
            if int(np.array(cand, dtype=np.float32).view(np.uint32)) % 2 == 0:
                best = cand
    return np.float32(best)


def _f(line: str, a: int, b: int) -> str:
    return line[a:b]


def parse_par(lines, molecule: str):
    """Convert .par text lines to database records.  Lines with an unknown
    isotopologue letter leave an empty (all-zero) record, like the `cycle`
    of processParFile.f90:160-165 after the record counter was advanced."""
    if molecule.strip() not in SPECIES_CODES:
        raise ValueError(f"unsupported molecule {molecule!r}")  # reference: stop 2
    recs = []
    for raw in lines:
        line = raw.rstrip("\n").ljust(160)
        if not line.strip():
            continue
        mol = int(_f(line, 0, 2))
        iso = _ISO_CODES.get(line[2], 99)
        rec = np.zeros(1, dtype=LINE_DTYPE)[0]
        if iso == 99 or isotopologue_number(mol, iso) == 0:
            recs.append(rec)
            continue
        rec["nu"] = float(_f(line, 3, 15))
        rec["S"] = np.float32(float(_f(line, 15, 25)))            # read as DP, narrowed
        rec["gair"] = decimal_to_f32(_f(line, 35, 40))
        rec["gself"] = decimal_to_f32(_f(line, 40, 45))
        rec["E"] = np.float32(float(_f(line, 45, 55)))            # read as DP, narrowed
        rec["nair"] = decimal_to_f32(_f(line, 55, 59))
        rec["jmi"] = isotopologue_number(mol, iso) * 100 + mol
        rec["delta"] = decimal_to_f32(_f(line, 59, 67))
        recs.append(rec)
    return np.array(recs, dtype=LINE_DTYPE)


def convert_par_file(par_path, out_path, molecule: str) -> int:
    with open(par_path) as f:
        recs = parse_par(f.readlines(), molecule)
    recs.tofile(out_path)
    return len(recs)
