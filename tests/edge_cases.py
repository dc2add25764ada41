"""Line lists that place lines exactly on the decision boundaries of the
reference's multigrid schedule (LineGridCalc.f90) and of its line window
(LBL.f90:41-61, main.f90:133-144, 196-248).

Every boundary below is a power of two or a sum of powers of two, exactly
representable in double, so the reference's comparisons (`UU >= H_k`,
`-UU > cutOff`, `UU >= cutOff`, the walk decrements `UUU - H_k`) meet exact
ties, and the neighbours one ulp away flip them.
"""
import numpy as np

from marfa_b200.io import LINE_DTYPE

H = 2.0 ** -11
SUB = 4050.0          # the subinterval [SUB, SUB + 10) whose ties are placed
START, END = 4040.0, 4070.0


def _ulps(x):
    return [np.nextafter(x, -np.inf), x, np.nextafter(x, np.inf)]


def tie_offsets():
    """Offsets from the subinterval start of lines inside it: every bin edge
    j * H_k of every grid (k = 0..9 and the finest step) near both ends and
    in the middle, each with its two neighbouring doubles."""
    offs = set()
    for k in list(range(10)) + [11]:
        hk = 2.0 ** -k
        for j in (0, 1, 2, 3, 4, 5, 7, 8):
            for base in (0.0, 5.0, 10.0 - (j + 1) * hk):
                o = base + j * hk
                if 0.0 <= o < 10.0:
                    offs.update(v for v in _ulps(o) if 0.0 <= v < 10.0)
        offs.add(10.0 - hk)
        offs.add(hk / 2)
    return sorted(offs)


def side_offsets():
    """Distances of lines outside the subinterval: D = H_k and its
    neighbours (leftLBL / rightLBL branch points), H_k / 2, and 1e-9."""
    d = set([1e-9, 0.3, 0.75, 1.5])
    for k in range(10):
        hk = 2.0 ** -k
        d.update(v for v in _ulps(hk) if v > 0)
        d.add(hk / 2)
        d.add(1.5 * hk)
    return sorted(d)


def tie_lines(cutoff, delta=0.0, n_random=300, seed=5):
    """A sorted list (with sentinel) for the run START..END at `cutoff`:
    tie lines inside [SUB, SUB+10), lines at the exact distances of
    side_offsets() on both sides of it, lines exactly at SUB - cutoff (kept:
    leftLBL returns only for D > cutOff) and SUB + 10 + cutoff (dropped:
    rightLBL returns for U >= cutOff) and their neighbours, and a random
    population over the whole window."""
    rng = np.random.default_rng(seed)
    nus = [SUB + o for o in tie_offsets()]
    nus += [SUB - d for d in side_offsets()]
    nus += [SUB + 10.0 + d for d in side_offsets()]
    for x in (SUB - cutoff, SUB + 10.0 + cutoff, START + 10.0 - cutoff):
        nus += _ulps(x)
    nus += list(rng.uniform(START - cutoff - 2.0, END + cutoff + 2.0, n_random))
    nus = np.unique(np.array(nus))
    n = len(nus)
    L = np.zeros(n + 1, dtype=LINE_DTYPE)
    L["nu"][:n] = nus
    L["S"][:n] = np.exp(rng.uniform(np.log(1e-23), np.log(1e-20), n))
    L["gair"][:n] = rng.uniform(0.02, 0.09, n)
    L["gself"][:n] = rng.uniform(0.05, 0.12, n)
    L["E"][:n] = rng.uniform(0.0, 3000.0, n)
    L["nair"][:n] = rng.uniform(0.5, 0.8, n)
    L["delta"][:n] = delta
    L["jmi"] = 1002
    L["nu"][n] = 1e5
    return L
