"""The CPU oracle: internal consistency, Voigt accuracy, schedule counts (CPU)."""
import math

import numpy as np
import pytest
from scipy.special import wofz

import oracle as O
from marfa_b200 import synth
from marfa_b200.io import LINE_DTYPE

H = 2.0 ** -11
NT = 20481


def count_line(nu_s, s, cut):
    """Closed form of the number of FSHAPE calls one line makes in one
    subinterval (LineGridCalc.f90), written independently of the oracle's
    walk and of the CUDA count kernel."""
    se = s + 10.0
    if nu_s < s:
        D = -(nu_s - s)
        if D > cut:
            return 0
        if not D < 1.0:
            return 21
        for k in range(1, 10):
            if not D < 2.0 ** -k:
                return 21 + 2 * k
        return 41
    if nu_s > se:
        U = (nu_s - s) - 10.0
        if U >= cut:
            return 0
        if not U < 1.0:
            return 21
        for k in range(1, 9):
            if not U < 2.0 ** -k:
                return 21 + 2 * k
        return 40 if not U < 2.0 ** -9 else 42
    UU = nu_s - s
    if UU >= 10.0:
        return 0
    n = 2
    I = cells = 0
    if UU >= H:
        for k in range(10):
            hk = 2.0 ** -k
            if k:
                I *= 2
            if UU >= 2 * hk:
                Ik = math.floor(UU / hk) - 1
                cells += Ik - I
                I = Ik
        n += 2 * cells + math.floor(UU / H) - 4 * I
    V = 10.0 - UU
    III = rc = 0
    for k in range(10):
        hk = 2.0 ** -k
        if k:
            III *= 2
        if V >= 2 * hk:
            Ik = math.floor(V / hk) - 1
            rc += Ik - III
            III = Ik
    npoint = math.floor(UU / H) + 2
    return n + 1 + 2 * rc + (NT - 4 * III) - npoint + 1


def edge_lines():
    """Lines at exact and near-exact multigrid distances on both sides of
    4050-4060 plus a random population; exercises every branch of the
    placement."""
    rng = np.random.default_rng(5)
    s = 4050.0
    offs = [0.0, 1e-9, H / 2, H, 3 * H, 2.0 ** -9, 2.0 ** -9 * 1.5, 2.0 ** -8, 0.3, 0.5, 0.75, 1.0,
            1.5, 2.0, 4.999, 5.0, 7.25, 9.99, 10.0 - H, 10.0 - 1e-9]
    nus = [s + o for o in offs] + [s - o for o in offs[1:]] + [s + 10 + o for o in offs[1:]]
    nus += list(rng.uniform(4020, 4090, 300))
    nus = np.sort(np.array(nus))
    L = np.zeros(len(nus) + 1, dtype=LINE_DTYPE)
    L["nu"][:-1] = nus
    L["S"][:-1] = 1e-21
    L["gair"][:-1] = 0.07
    L["gself"][:-1] = 0.09
    L["E"][:-1] = 500.0
    L["nair"][:-1] = 0.7
    L["jmi"] = 1002
    L["nu"][-1] = 1e5
    return L


@pytest.fixture(scope="module")
def cfg0():
    return synth.config(0)


def test_mixed_and_fp64_maps_agree(cfg0, tips):
    a = O.from_workload(cfg0, precision=O.MIXED, tips=tips).run()[1]
    b = O.from_workload(cfg0, precision=O.FP64, tips=tips).run()[1]
    m = b > 1e-6 * b.max()
    assert np.max(np.abs(a[m] - b[m]) / b[m]) < 1e-5


def test_eval_counts_match_closed_form(cfg0, tips):
    from pathlib import Path
    from marfa_b200.io import read_lines
    real = read_lines(Path(__file__).resolve().parent / "golden" / "co_hitran2020_1900_2400.lines")
    for lines, start, end, cut in ((cfg0.lines, 4000.0, 4100.0, 25.0),
                                   (edge_lines(), 4050.0, 4060.0, 25.0),
                                   (edge_lines(), 4050.0, 4060.0, 0.75),
                                   (real, 2000.0, 2100.0, 25.0)):
        o = O.Oracle(lines, tips, [1.0], [296.0], [2.39e24], start, end, cut)
        _, _, ev = o.run(want64=False)
        lo, hi = o.windows()
        s = start
        total = 0
        for isub in range(len(lo)):
            for i in range(lo[isub] - 1, hi[isub] - 1):
                nus = lines["nu"][i] + float(np.float32(lines["delta"][i]) * np.float32(1.0))
                total += count_line(nus, s, float(np.float32(cut)))
            s += 10.0
        assert total == int(ev[0])


def test_voigt_close_to_faddeeva(tips):
    """The oracle's shape of one line across its whole profile against the
    exact Voigt, Re w(x + iy) sqrt(ln 2) / (sqrt(pi) alpha) S
    (scipy.special.wofz), at the accuracy of the reference's approximation:
    the Kuntz rational regions 1 and 2 within 1e-4, region 3 within 2e-3
    (1.0e-3 is reached near its outer edge, x + y close to 5.5), and the
    branches where the reference drops correction terms -- region 0 (pure
    Lorentz beyond VX = 15), the Lorentz asymptote beyond VX = 5, the Doppler
    core and its tabulated wing at small Y -- within 1e-2 (6.3e-3 at most).
    Every region the profile crosses is checked (the region codes are the
    oracle's)."""
    L = np.zeros(2, dtype=LINE_DTYPE)
    L[0] = (4000.0, 1e-20, 0.07, 0.09, 0.0, 0.7, 1002, 0.0)
    L[1] = (1e5, 0, 0, 0, 0, 0, 1002, 0)
    sqln2 = math.sqrt(math.log(2.0))
    dop = math.sqrt(2 * 6.02214076e23 * 1.3806503e-16 * math.log(2.0)) / 2.99792458e10
    alpha = dop * 4000.0 * math.sqrt(296.0 / 43.98983)
    seen = set()
    for P in (1e-4, 1e-2, 1.0):
        o = O.Oracle(L, tips, [P], [296.0], [1e10], 3990.0, 4010.0, 25.0, precision=O.FP64)
        y = sqln2 * 0.07 * P / alpha
        for X in np.geomspace(1e-5, 20.0, 400):
            v, region = o.shape_value(0, 0, X)
            x = sqln2 * X / alpha
            exact = wofz(x + 1j * y).real / math.sqrt(3.1415926) * sqln2 / alpha * 1e-20
            tol = 1e-4 if region in (1, 2) else (2e-3 if region == 3 else 1e-2)
            assert abs(v - exact) / exact <= tol, (P, X, region, v, exact)
            seen.add(region)
    assert seen >= {0, 1, 2, 3, 40, 41, 42}, seen


def test_region_formulas_against_wofz(tips):
    """Direct check of the Kuntz regions: K(x, y) from the oracle's voigt
    divided by the intensity scale equals Re w(x + iy)/sqrt(pi)... within
    the approximation accuracy in regions 1-3."""
    L = np.zeros(2, dtype=LINE_DTYPE)
    L[0] = (4000.0, 1e-20, 0.07, 0.09, 0.0, 0.7, 1002, 0.0)
    L[1] = (1e5, 0, 0, 0, 0, 0, 1002, 0)
    for P in (1e-3, 0.05, 1.0, 10.0):
        o = O.Oracle(L, tips, [P], [296.0], [1e10], 3990.0, 4010.0, 25.0, precision=O.FP64)
        # alpha from the oracle's Doppler formula; probe with X giving VX values
        sqln2 = math.sqrt(math.log(2.0))
        dop = math.sqrt(2 * 6.02214076e23 * 1.3806503e-16 * math.log(2.0)) / 2.99792458e10
        alpha = dop * 4000.0 * math.sqrt(296.0 / 43.98983)
        gamma = 0.07 * P  # pSelf ~ 0 (tiny density), T = Tref
        y = sqln2 * gamma / alpha
        S = 1e-20
        for x in (0.0, 0.5, 2.0, 4.0, 8.0, 12.0):
            X = x * alpha / sqln2
            v, region = o.shape_value(0, 0, X)
            exact = wofz(x + 1j * y).real / math.sqrt(3.1415926) * sqln2 / alpha * S
            if region in (1, 2, 3):
                assert abs(v - exact) / exact < 2e-4, (P, x, region)


def test_self_pressure_above_total_makes_negative_shapes(cfg0, tips):
    """With pSelf > P the Lorentz width can turn negative and the reference's
    `IF(FF < EPS) RETURN` exits fire (the eval count drops); physical
    profiles never reach them.  The library rejects such levels (status 7)."""
    ok = O.Oracle(cfg0.lines, tips, [1.0], [296.0], [2.39e24], 4000.0, 4100.0, 25.0)
    bad = O.Oracle(cfg0.lines, tips, [1.0], [296.0], [2.4e25], 4000.0, 4100.0, 25.0)
    assert bad.run(want64=False)[2][0] < ok.run(want64=False)[2][0]


def test_windows_recurrence_and_eof(cfg0, tips):
    o = O.from_workload(cfg0, tips=tips)
    lo, hi = o.windows()
    assert np.all(np.diff(lo) >= 0) and np.all(hi > lo)
    nu = cfg0.lines["nu"]
    for s, a, b in zip(np.arange(4000.0, 4100.0, 10.0), lo, hi):
        assert nu[b - 1] >= s + 10 + 25 and nu[b - 2] < s + 10 + 25
    bad = cfg0.lines[:-1]                       # drop the sentinel
    ob = O.Oracle(bad, tips, [1.0], [296.0], [2.4e25], 4000.0, 4100.0, 25.0)
    with pytest.raises(O.OracleError) as e:
        ob.run()
    assert e.value.code == 9


def test_temperature_outside_tips_is_rejected(cfg0, tips):
    o = O.Oracle(cfg0.lines, tips, [1.0], [10.0], [2.4e25], 4000.0, 4010.0, 25.0)
    with pytest.raises(O.OracleError) as e:
        o.run()
    assert e.value.code == 11


def test_cascade_is_exact_at_grid0_lattice_points(tips):
    """A single line far from every grid-0 point: the record equals the
    directly evaluated shape at the integer positions (the cascade carries
    grid-0 edge values unchanged)."""
    L = np.zeros(2, dtype=LINE_DTYPE)
    L[0] = (4053.3, 1e-20, 0.07, 0.09, 100.0, 0.7, 1002, 0.0)
    L[1] = (1e5, 0, 0, 0, 0, 0, 1002, 0)
    o = O.Oracle(L, tips, [1.0], [296.0], [1.0], 4050.0, 4060.0, 25.0)
    rec = o.run()[1][0, 0]
    for j in range(11):
        v, _ = o.shape_value(0, 0, 4050.0 + j - 4053.3)
        assert abs(rec[2048 * j] - v) <= 1e-12 * v


def test_cascade_restatement_used_by_the_fp32c_check(cfg0, tips):
    """The vectorised cascade of tests/fp32c_check.py reproduces the oracle's
    records from the oracle's raw accumulators."""
    from fp32c_check import tainted_points
    o = O.from_workload(cfg0, precision=O.FP64, tips=tips)
    rec = o.run()[1][0]
    for isub in (0, 5, 9):
        _, rk = tainted_points(o.accumulators(0, isub), want_record=True)
        assert np.max(np.abs(rk - rec[isub]) / rec[isub]) < 1e-13


def test_tips_grid_resampled_to_1k_steps(tips):
    """The oracle's TIPSofT on a 1 K grid, with the 2 K table resampled so
    that linear interpolation gives the same partition sums, reproduces the
    reference grid's records (all-double map)."""
    w = synth.config(0, scale=0.25)
    t = np.asarray(tips, dtype=np.float64)
    t1 = np.empty((t.shape[0], 2 * t.shape[1] - 1))
    t1[:, 0::2] = t
    t1[:, 1::2] = 0.5 * (t[:, :-1] + t[:, 1:])
    P, T = synth.f32([1.0]), synth.f32([251.3])
    n = synth.ideal_gas_density(P, T)
    kw = dict(target="ACS", chi="none", precision=O.FP64)
    a = O.Oracle(w.lines, t, P, T, n, w.start_wv, w.end_wv, w.cutoff, **kw).run()[1]
    b = O.Oracle(w.lines, t1, P, T, n, w.start_wv, w.end_wv, w.cutoff, tips_grid=(20.0, 1.0), **kw).run()[1]
    m = a > 0
    assert np.max(np.abs(a[m] - b[m]) / a[m]) <= 1e-12
