"""The adjoint (marfa_vjp) against FP64 central finite differences.

Workload: the differentiation configuration -- 40,000 synthetic CO2-like
lines over 4000-4200 cm-1, a 10-level Venus-like profile (92 atm / 735 K down
to 1e-4 atm / 170 K), cutoff 125 cm-1, tonkov chi-factor, ACS, and a
Gaussian cotangent (seed 3) on every finest-grid point.

The records are piecewise smooth: a line's multigrid placement jumps when its
shifted centre crosses a multiple of 2^-11 cm-1 (pressure shift), the
Humlicek approximation jumps at its region boundaries and the cascade clamp
switches on near-ties.  A difference quotient that straddles such a point is
not a derivative, so
  * pressure steps are shrunk until no line crosses a 2^-11 lattice point;
  * each parameter is compared over a ladder of relative steps, and the
    closest difference quotient must agree within 1e-4 (truncation and jump
    errors shrink with the step, rounding grows: the ladder brackets the
    usable range);
  * temperatures on a TIPS knot (T = 20 + 2j K, where the partition sum has a
    kink) are compared with the one-sided quotient from above, the branch the
    reference's truncating index selects.
Per level, only that level's records change, so the quotient is formed from
the difference of that level's records before the cotangent sum.
"""
import numpy as np
import pytest

from marfa_b200 import synth, data_path
from marfa_b200.api import Context, Run
from marfa_b200.io import read_tips

pytestmark = pytest.mark.gpu

TOL = 1e-4
LADDER = (1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8)


@pytest.fixture(scope="module")
def case(gpu):
    tips = read_tips(data_path("TIPS_subset.dat"))
    w = synth.config(3)
    p = w.profiles[0]
    P, T, n = (np.asarray(a, dtype=np.float64) for a in (p.pressure, p.temperature, p.density))
    ctx = Context(w.lines, tips)
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp64")
    cot = np.random.default_rng(3).standard_normal((len(P), run.n_sub, 20481))
    g = ctx.vjp(run, P, T, n, cot)
    yield dict(w=w, ctx=ctx, run=run, P=P, T=T, n=n, cot=cot, g=g)
    ctx.set_line_params(None, None)
    ctx.close()


def level_records(c, l, P, T):
    _, o = c["ctx"].compute(c["run"], [P], [T], [c["n"][l]], want64=True)
    return o[0]


def straddles(c, P, h):
    nu = c["w"].lines["nu"].astype(np.float64)
    de = c["w"].lines["delta"].astype(np.float64)
    a = np.floor((nu + de * (P + h)) * 2048.0)
    b = np.floor((nu + de * (P - h)) * 2048.0)
    return int(np.count_nonzero(a != b))


def best_rel(estimates, value):
    return min(abs(e / value - 1.0) for e in estimates)


def test_homogeneity_in_intensity(case):
    """The records are positively homogeneous of degree 1 in the vector of
    line intensities (the clamp decisions are scale invariant), so
    sum_q S_q dL/dS_q = L exactly: this checks every (line, slot) pair of the
    adjoint's placement and the backward cascade against the forward."""
    c = case
    ctx = c["ctx"]
    ctx.set_line_params(None, None)
    _, o = ctx.compute(c["run"], c["P"], c["T"], c["n"], want64=True)
    terms = c["cot"] * o
    L = float(terms.sum())
    S = c["w"].lines["S"].astype(np.float64)
    assert abs(float(S @ c["g"]["dS"]) - L) <= 1e-12 * float(np.abs(terms).sum())


def test_temperature(case):
    c = case
    cot, T, P = c["cot"], c["T"], c["P"]
    for l in range(len(T)):
        base = level_records(c, l, P[l], T[l])
        knot = float((T[l] - 20.0) / 2.0).is_integer()
        est = []
        for rel in LADDER:
            h = rel * T[l]
            up = level_records(c, l, P[l], T[l] + h)
            if knot:
                est.append(float(np.sum(cot[l] * (up - base))) / h)
            else:
                dn = level_records(c, l, P[l], T[l] - h)
                est.append(float(np.sum(cot[l] * (up - dn))) / (2 * h))
        r = best_rel(est, c["g"]["dT"][l])
        assert r <= TOL, (l, T[l], c["g"]["dT"][l], est)


def test_pressure(case):
    c = case
    cot, T, P = c["cot"], c["T"], c["P"]
    for l in range(len(P)):
        est = []
        for rel in LADDER:
            h = rel * P[l]
            if straddles(c, P[l], h):
                continue
            up = level_records(c, l, P[l] + h, T[l])
            dn = level_records(c, l, P[l] - h, T[l])
            est.append(float(np.sum(cot[l] * (up - dn))) / (2 * h))
        assert est, f"level {l}: every step moves a line across the 2^-11 lattice"
        r = best_rel(est, c["g"]["dP"][l])
        assert r <= TOL, (l, P[l], c["g"]["dP"][l], est)


def _L(c, S=None, G=None):
    c["ctx"].set_line_params(S, G)
    try:
        _, o = c["ctx"].compute(c["run"], c["P"], c["T"], c["n"], want64=True)
    finally:
        c["ctx"].set_line_params(None, None)
    return o


def test_line_parameters(case):
    """Directional derivatives along a random direction of all intensities
    and all air-broadening coefficients, and the five lines with the largest
    gamma_air gradient one by one."""
    c = case
    S0 = c["w"].lines["S"].astype(np.float64)
    G0 = c["w"].lines["gair"].astype(np.float64)
    v = np.random.default_rng(5).standard_normal(len(S0))
    cot = c["cot"]
    for name, base, key in (("S", S0, "dS"), ("gamma_air", G0, "dgamma_air")):
        an = float(c["g"][key] @ (base * v))
        est = []
        for rel in (1e-5, 1e-6, 1e-7):
            if name == "S":
                d = _L(c, S=base * (1 + rel * v)) - _L(c, S=base * (1 - rel * v))
            else:
                d = _L(c, G=base * (1 + rel * v)) - _L(c, G=base * (1 - rel * v))
            est.append(float(np.sum(cot * d)) / (2 * rel))
        assert best_rel(est, an) <= TOL, (name, an, est)
    for i in np.argsort(-np.abs(c["g"]["dgamma_air"]))[:5]:
        h = 1e-6 * G0[i]
        Gp, Gm = G0.copy(), G0.copy()
        Gp[i] += h
        Gm[i] -= h
        fd = float(np.sum(cot * (_L(c, G=Gp) - _L(c, G=Gm)))) / (2 * h)
        assert abs(fd / c["g"]["dgamma_air"][i] - 1.0) <= TOL, (i, fd, c["g"]["dgamma_air"][i])


def test_autograd_function(case):
    """torch.autograd.Function: the forward equals the FP64 records and the
    backward of sum(cot * records) equals the library's VJP."""
    torch = pytest.importorskip("torch")
    from marfa_b200.autograd import Spectrum
    c = case
    model = Spectrum(c["ctx"], c["run"], c["n"])
    T = torch.tensor(c["T"], requires_grad=True)
    P = torch.tensor(c["P"], requires_grad=True)
    S = torch.tensor(c["w"].lines["S"].astype(np.float64), requires_grad=True)
    G = torch.tensor(c["w"].lines["gair"].astype(np.float64), requires_grad=True)
    rec = model(T, P, S, G)
    _, o = c["ctx"].compute(c["run"], c["P"], c["T"], c["n"], want64=True)
    assert np.array_equal(rec.detach().numpy(), o)
    (rec * torch.from_numpy(c["cot"])).sum().backward()
    for t, key in ((T, "dT"), (P, "dP"), (S, "dS"), (G, "dgamma_air")):
        assert np.allclose(t.grad.numpy(), c["g"][key], rtol=1e-9, atol=0.0), key
    c["ctx"].set_line_params(None, None)
