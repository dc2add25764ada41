"""File formats of the MARFA line-by-line core.

All readers and writers here follow the reference's on-disk formats, so files
written by one program are read by the other:

* line database: 36-byte little-endian direct-access records, one per line,
  sorted by wavenumber (README.md:361-365; processParFile.f90:140-176;
  read in LBL.f90:43-44);
* atmospheric profile: a 20-character title line, a level count N <= 200, then
  N rows "height pressure[atm] temperature[K] density[1/(cm^2 km)]"
  (Atmsosphere.f90:29-60);
* TIPS table: header "n_iso, n_temp", then one row of n_temp partition sums
  per isotopologue for T = 20, 22, ... K (EnvironmentSetup.f90:169-184);
* PT-table: one file per level, named '1__.ptbin', '12_.ptbin', '123.ptbin',
  records of 20481 float32 (81,924 bytes), record number int((start+1)/10)
  of the subinterval (main.f90:99-112, 126, 163-168; handlers/constants.py;
  handlers/parsers.py:17-65).
"""
from __future__ import annotations

import os
import shutil
from pathlib import Path

import numpy as np

LINE_DTYPE = np.dtype([
    ("nu", "<f8"),      # transition wavenumber [cm-1]
    ("S", "<f4"),       # intensity at 296 K [cm-1/(molecule cm-2)]
    ("gair", "<f4"),    # air (foreign) broadened HWHM at 296 K [cm-1/atm]
    ("gself", "<f4"),   # self broadened HWHM [cm-1/atm]
    ("E", "<f4"),       # lower-state energy [cm-1]
    ("nair", "<f4"),    # temperature exponent of gair
    ("jmi", "<i4"),     # isotopologue index * 100 + molecule number
    ("delta", "<f4"),   # pressure shift [cm-1/atm]
])
assert LINE_DTYPE.itemsize == 36

NT = 20481                      # points per PT record (Grids.f90:16)
RECORD_BYTES = NT * 4           # 81,924 bytes
RECORD_SPAN = 10.0              # cm-1 per record (Grids.f90:20)
MAX_LEVELS = 200                # Atmsosphere.f90:64

# getSpeciesCode (EnvironmentSetup.f90:187-235)
SPECIES_CODES = {"H2O": 1, "CO2": 2, "O3": 3, "N2O": 4, "CO": 5, "CH4": 6, "O2": 7,
                 "NO": 8, "SO2": 9, "NO2": 10, "NH3": 11, "HNO3": 12}


class MarfaFormatError(RuntimeError):
    """A file did not match the reference format; .code is the reference's
    `stop` code for the same failure."""

    def __init__(self, message: str, code: int):
        super().__init__(message)
        self.code = code


def species_code(name: str) -> int:
    """HITRAN molecule number of `name`, 0 when unsupported (the reference
    then stops with code 8, main.f90:68-72)."""
    return SPECIES_CODES.get(name.strip(), 0)


def read_lines(path) -> np.ndarray:
    """Read a 36-byte-record line database."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size % LINE_DTYPE.itemsize:
        raise MarfaFormatError(f"{path}: size {raw.size} is not a multiple of 36", 9)
    return raw.view(LINE_DTYPE).copy()


def write_lines(path, lines: np.ndarray) -> None:
    np.asarray(lines, dtype=LINE_DTYPE).tofile(path)


def read_profile(path):
    """Parse an atmospheric profile; returns (title, height, P, T, n) with
    the four columns as float64 arrays.  Raises MarfaFormatError with code 6
    (more than 200 levels) or 7 (malformed row), like Atmsosphere.f90:40,55."""
    with open(path) as f:
        title = f.readline().rstrip("\n")[:20]
        levels = int(f.readline().split()[0])
        if levels > MAX_LEVELS:
            raise MarfaFormatError(f"{path}: {levels} levels > {MAX_LEVELS}", 6)
        rows = []
        for _ in range(levels):
            parts = f.readline().replace(",", " ").split()
            try:
                rows.append([float(v) for v in parts[:4]])
                if len(parts) < 4:
                    raise ValueError
            except ValueError:
                raise MarfaFormatError(f"{path}: bad data row", 7) from None
    a = np.array(rows, dtype=np.float64).reshape(levels, 4)
    return title, a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy(), a[:, 3].copy()


def write_profile(path, title, height, P, T, n) -> None:
    """Write a profile whose values are float32 numbers printed exactly (the
    reference parses them into default reals; a double parse of the text
    gives the same value)."""
    with open(path, "w") as f:
        f.write(f"{title[:20]}\n{len(P)}\n")
        for h, p, t, d in zip(height, P, T, n):
            f.write(" ".join(repr(float(np.float32(v))) for v in (h, p, t, d)) + "\n")


def read_tips(path):
    """Read a TIPS table: returns a float64 array [n_iso, n_temp].  Besides the
    reference layout (one row per isotopologue), a subset layout is accepted in
    which each row starts with 'iso:'; rows not listed are NaN and any line
    using them is rejected by the library."""
    with open(path) as f:
        head = f.readline().replace(",", " ").split()
        n_iso, n_temp = int(head[0]), int(head[1])
        table = np.full((n_iso, n_temp), np.nan)
        row = 0
        for line in f:
            if not line.strip():
                continue
            if ":" in line:
                key, rest = line.split(":", 1)
                idx = int(key) - 1
            else:
                idx, rest = row, line
                row += 1
            vals = [float(v) for v in rest.replace(",", " ").split()]
            if len(vals) != n_temp:
                raise MarfaFormatError(f"{path}: row {idx + 1} has {len(vals)} values", 9)
            table[idx] = vals
    return table


def pt_name(level: int) -> str:
    """PT-table file name of 1-based `level` (main.f90:99-108)."""
    label = str(level)
    return label + "_" * (3 - len(label)) + ".ptbin"


def record_number(start_wv: float) -> int:
    """outputRecNum of the subinterval starting at start_wv (main.f90:126)."""
    return int((start_wv + 1.0) / 10.0)


def subinterval_starts(start_wv: float, end_wv: float) -> list:
    """Left edges of the 10 cm-1 subintervals (main.f90:117-122, 171)."""
    starts = []
    s = float(start_wv)
    while s < end_wv:
        starts.append(s)
        s = s + RECORD_SPAN
    return starts


def write_pt_table(path, start_wv: float, records: np.ndarray) -> None:
    """Write the records of one level (array [n_sub, NT] float32) at their
    record numbers; leading records stay holes, as in a Fortran direct-access
    file."""
    records = np.ascontiguousarray(records, dtype="<f4")
    starts = subinterval_starts(start_wv, start_wv + RECORD_SPAN * records.shape[0])
    fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)
    try:
        for s, rec in zip(starts, records):
            os.pwrite(fd, rec.tobytes(), (record_number(s) - 1) * RECORD_BYTES)
    finally:
        os.close(fd)


def read_pt_table(path, v1: float, v2: float):
    """Restatement of handlers/parsers.py:17-65 (base_parser): returns
    (wavenumbers, values) as float32 arrays for records int(v1/10) ..
    int((v2-1)/10), the wavenumber of point i of record r being
    10*r + i*10/20480."""
    start_rec = int(v1 / 10.0)
    end_rec = int((v2 - 1) / 10.0)
    step = RECORD_SPAN / (NT - 1)
    size = os.path.getsize(path)
    wv, vals = [], []
    with open(path, "rb") as f:
        for rec in range(start_rec, end_rec + 1):
            pos = (rec - 1) * RECORD_BYTES
            if pos >= size:
                raise IndexError(f"Record number {rec} exceeds a file size.")
            f.seek(pos)
            data = np.frombuffer(f.read(RECORD_BYTES), dtype="<f4")
            wv.append((RECORD_SPAN * rec + np.arange(NT) * step).astype(np.float32))
            vals.append(data.astype(np.float32))
    return np.concatenate(wv), np.concatenate(vals)


CONVERTED_DIRECTORY = Path("output") / "processedData"   # handlers/constants.py


def read_info(directory) -> dict:
    """The run parameters a converter needs from info.txt: start and end
    wavenumber and the molecule (handlers/convert.py:28-40)."""
    v1 = v2 = molecule = None
    with open(Path(directory) / "info.txt") as info:
        for line in info.readlines():
            if line.startswith("Start Wavenumber"):
                v1 = float(line.split(":")[1])
            if line.startswith("End Wavenumber"):
                v2 = float(line.split(":")[1])
            if line.startswith("Input Molecule"):
                molecule = line.split(":")[1]
    if v1 is None or v2 is None:
        raise ValueError("Corrupted info file: start or end wavenumbers are not defined")
    return {"start": v1, "end": v2, "molecule": molecule}


def convert_pt_table(directory, level: int, out_directory=None) -> Path:
    """Restatement of convert_pttable (handlers/convert.py:12-53): the PT
    table of `level` in a run directory as text.  The output file
    `<molecule>_<int(v1)>-<int(v2)>_<level>level.dat` in `out_directory`
    (default output/processedData, relative to the working directory) starts
    with a copy of info.txt, followed by one line per point,
    '%15.5f %17.7e' of (wavenumber, value) as float32 (handlers/parsers.py:17-65
    gives the points).  Returns the path of the written file."""
    directory = Path(directory)
    info = read_info(directory)
    v1, v2 = info["start"], info["end"]
    wv, vals = read_pt_table(directory / pt_name(level), v1, v2)
    out_dir = Path(out_directory) if out_directory is not None else CONVERTED_DIRECTORY
    out = out_dir / f"{info['molecule'].strip()}_{int(v1)}-{int(v2)}_{level}level.dat"
    shutil.copyfile(directory / "info.txt", out)
    with open(out, "a") as f:
        # the same conversions as the reference's f-string on numpy float32:
        # each value widened to a Python float, then formatted
        f.write("".join(f"{w:15.5f} {a:17.7e}\n" for w, a in zip(wv.tolist(), vals.tolist())))
    return out


def write_info(directory: Path, molecule, start, end, cutoff, target, profile) -> None:
    """info.txt of a run (EnvironmentSetup.f90:136-154)."""
    with open(Path(directory) / "info.txt", "w") as f:
        f.write("Command-Line Arguments:\n")
        f.write(f"Input Molecule: {molecule}\n")
        f.write(f"Start Wavenumber: {start}\n")
        f.write(f"End Wavenumber: {end}\n")
        f.write(f"Cut Off: {cutoff}\n")
        f.write(f"Target Value: {target}\n")
        f.write(f"Atmospheric Profile File: {profile}\n")
