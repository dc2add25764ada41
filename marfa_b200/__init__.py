"""marfa_b200 -- B200-native line-by-line absorption core with the
interfaces of MARFA (Razumovskyy/MARFA).

The compute path is the CUDA library libmarfa_gpu.so (C ABI declared in
include/marfa_gpu.h); this package holds its ctypes binding, the file formats
and the host-side driver that mirrors the reference's command line.
"""
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent


def data_path(name: str) -> Path:
    return PACKAGE_DIR / "data" / name
