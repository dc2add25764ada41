"""Seeded synthetic line lists and atmospheric profiles.

The reference's benchmark rows use HITRAN2020 CO2/H2O databases that are not
available here; these generators stand in for them with the distributions
below (uniform centres, log-uniform intensities, uniform broadening, shift and
lower-state energy).  No HITRAN record is reproduced.

Every list is sorted by wavenumber and ends with a sentinel record (nu = 1e5,
S = 0): the reference's line loop only leaves a subinterval when it reads a
line beyond the window (LBL.f90:41-57), so a list must extend past the last
window.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .io import LINE_DTYPE

BOLTZMANN_SI = 1.3806503e-23
ATM_PA = 101325.0
SENTINEL_NU = 1.0e5

# isotopologue index * 100 + molecule number (processParFile.f90:171-174)
JMI_CO2_626 = 10 * 100 + 2
JMI_H2O_161 = 1 * 100 + 1


@dataclass
class LineSpec:
    n: int
    nu_lo: float
    nu_hi: float
    s_lo: float = 1e-26
    s_hi: float = 1e-20
    gair: tuple = (0.02, 0.09)
    gself: tuple = (0.05, 0.12)
    nair: tuple = (0.5, 0.8)
    elow: tuple = (0.0, 4000.0)
    delta: tuple = (-0.008, 0.0)
    jmi: int = JMI_CO2_626
    seed: int = 0


def make_lines(spec: LineSpec) -> np.ndarray:
    rng = np.random.default_rng(spec.seed)
    n = spec.n
    lines = np.zeros(n + 1, dtype=LINE_DTYPE)
    nu = np.sort(rng.uniform(spec.nu_lo, spec.nu_hi, n))
    lines["nu"][:n] = nu
    lines["S"][:n] = np.exp(rng.uniform(np.log(spec.s_lo), np.log(spec.s_hi), n))
    lines["gair"][:n] = rng.uniform(*spec.gair, n)
    lines["gself"][:n] = rng.uniform(*spec.gself, n)
    lines["E"][:n] = rng.uniform(*spec.elow, n)
    lines["nair"][:n] = rng.uniform(*spec.nair, n)
    lines["jmi"][:n] = spec.jmi
    lines["delta"][:n] = rng.uniform(*spec.delta, n)
    lines["nu"][n] = SENTINEL_NU
    lines["jmi"][n] = spec.jmi
    return lines


def f32(x):
    """Round to the nearest float32 and return float64 (profile values are
    Fortran default reals in the reference)."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def ideal_gas_density(P, T, mixing=0.965):
    """Number density [1/(cm^2 km)] of a gas with the given mixing ratio at
    P [atm], T [K]; chosen so that the reference's pSelf = n*10*k*T/101325
    (main.f90:92) equals mixing * P."""
    return mixing * np.asarray(P) * ATM_PA / (10.0 * BOLTZMANN_SI * np.asarray(T))


@dataclass
class Profile:
    pressure: np.ndarray
    temperature: np.ndarray
    density: np.ndarray
    height: np.ndarray = field(default=None)

    def __post_init__(self):
        self.pressure = f32(self.pressure)
        self.temperature = f32(self.temperature)
        self.density = f32(self.density)
        if self.height is None:
            self.height = f32(np.arange(len(self.pressure)) * 2.0)

    @property
    def n_levels(self):
        return len(self.pressure)


def venus_profile(n_levels=40, p_top=1e-4, p_bottom=92.0, t_bottom=735.0, t_top=170.0):
    """Venus-like profile: P log-spaced bottom to top, T linear, 96.5% CO2."""
    P = np.geomspace(p_bottom, p_top, n_levels)
    T = np.linspace(t_bottom, t_top, n_levels)
    return Profile(P, T, ideal_gas_density(f32(P), f32(T)))


def random_profile(seed, p_range=(1e-4, 100.0), t_range=(150.0, 750.0), n_range=(10, 100)):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(n_range[0], n_range[1] + 1))
    P = np.exp(rng.uniform(np.log(p_range[0]), np.log(p_range[1]), n))
    T = rng.uniform(*t_range, n)
    return Profile(P, T, ideal_gas_density(f32(P), f32(T)))


@dataclass
class Workload:
    """One benchmark configuration: a line list, one or more profiles and the
    run parameters of the 7-argument command line."""
    name: str
    lines: np.ndarray
    profiles: list
    start_wv: float
    end_wv: float
    cutoff: float
    target: str          # "ACS" or "VAC"
    chi: str             # "none", "tonkov", "pollack", "perrin"
    molecule: str        # "CO2" / "H2O"


def config(index: int, scale: float = 1.0) -> Workload:
    """The five configurations of the benchmark plan.  `scale` < 1 shrinks
    line counts and spectral spans proportionally (parity-test sizes)."""
    if index == 0:
        lines = make_lines(LineSpec(n=int(2000 * scale) or 1, nu_lo=4000.0, nu_hi=4100.0, seed=0))
        prof = Profile([1.0], [296.0], ideal_gas_density(f32([1.0]), f32([296.0])))
        return Workload("plain-2k-lines-1-level", lines, [prof], 4000.0, 4100.0, 25.0,
                        "ACS", "none", "CO2")
    if index == 1:
        span = max(10.0, round(1000.0 * scale / 10.0) * 10.0)
        lines = make_lines(LineSpec(n=max(1, int(200_000 * span / 1000.0)), nu_lo=4000.0,
                                    nu_hi=4000.0 + span, seed=1))
        return Workload("venus-200k-lines-40-levels", lines, [venus_profile(40)], 4000.0,
                        4000.0 + span, 125.0, "VAC", "tonkov", "CO2")
    if index == 2:
        lines = make_lines(LineSpec(n=int(30_000 * scale) or 1, nu_lo=10.0, nu_hi=3000.0,
                                    s_lo=1e-27, s_hi=1e-18, gair=(0.01, 0.11),
                                    jmi=JMI_H2O_161, seed=2))
        profs = [random_profile(1000 + i) for i in range(max(1, int(64 * scale)))]
        return Workload("uneven-64-profiles", lines, profs, 10.0, 3000.0, 25.0,
                        "VAC", "none", "H2O")
    if index == 3:
        span = 200.0
        lines = make_lines(LineSpec(n=int(40_000 * scale) or 1, nu_lo=4000.0,
                                    nu_hi=4000.0 + span, seed=1))
        return Workload("diff-40k-lines-10-levels", lines, [venus_profile(10)], 4000.0,
                        4000.0 + span, 125.0, "ACS", "tonkov", "CO2")
    if index == 4:
        lines = make_lines(LineSpec(n=int(2_000_000 * scale) or 1, nu_lo=500.0, nu_hi=10000.0,
                                    s_lo=1e-30, s_hi=1e-19, seed=4))
        return Workload("stress-2M-lines-100-levels", lines, [venus_profile(100)], 500.0,
                        10000.0, 250.0, "VAC", "tonkov", "CO2")
    raise ValueError(index)
