"""The adjoint (marfa_vjp) against FP64 central finite differences.

Workload: the differentiation configuration -- 40,000 synthetic CO2-like
lines over 4000-4200 cm-1, a 10-level Venus-like profile (92 atm / 735 K down
to 1e-4 atm / 170 K), cutoff 125 cm-1, tonkov chi-factor, ACS, and a
Gaussian cotangent (seed 3) on every finest-grid point.

The records are piecewise smooth: a line's multigrid placement jumps when its
shifted centre crosses a multiple of 2^-11 cm-1 (pressure shift), the
Humlicek approximation jumps at its region boundaries and the cascade clamp
switches on near-ties (a jump of the order of the value itself).  Among
4 million points per level, some such point always lies within a relative
step of 1e-6, so a difference quotient there is not a derivative.  So
  * the points where the map is not differentiable inside the step are found
    from the records themselves -- where the one-sided quotients
    (f(x+h) - f(x)) / h and (f(x) - f(x-h)) / h disagree by more than 1e-3 of
    their size -- the cotangent is zeroed there and the VJP recomputed with
    it: the VJP is linear in the cotangent, so both sides leave out exactly
    the same points (how many is printed);
  * every quotient starts at the relative step 1e-6 and must agree within
    1e-4.  Where the records' rounding dominates a 1e-6 step -- the
    low-pressure levels, whose records depend on P only through gamma_L,
    proportional to P, a small part of a Doppler-dominated profile -- the
    quotients at h and 10 h disagree; the step then grows by 10 until they
    agree within 5e-5, a choice made from the quotients alone (rounding
    error falls as 1/h and truncation error grows as h^2, so that agreement
    bounds the error at h by about 5.6e-5; the steps used are printed);
  * a temperature on a TIPS knot (T = 20 + 2j K: the partition sum has a
    kink there, at every point) uses the second-order one-sided quotient from
    above, (-3 f(x) + 4 f(x+h) - f(x+2h)) / 2h, the branch the reference's
    truncating index selects.
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
STEP = 1e-6


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


def kinks(up, base, dn, h):
    """Points whose one-sided quotients disagree: a jump inside +-h."""
    qp = (up - base) / h
    qm = (base - dn) / h
    return np.abs(qp - qm) > 1e-3 * np.maximum(np.abs(qp), np.abs(qm))


def rel(estimate, value):
    return abs(estimate / value - 1.0)


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


def level_fd(c, l, rec, x, one_sided):
    """Difference quotient of level l's cotangent-weighted records in the
    parameter x (rec(value) -> records), the jump mask and the relative step
    used, by the rules of the module docstring."""
    cot = c["cot"][l]
    base = rec(x)
    for r in (1e-6, 1e-5, 1e-4, 1e-3):
        est = []
        mask = np.zeros(cot.shape, dtype=bool)
        for h in (r * x, 10 * r * x):
            up = rec(x + h)
            if one_sided:
                up2 = rec(x + 2 * h)
                mask |= kinks(up2, up, base, h)
                est.append((4.0 * up - 3.0 * base - up2) / (2 * h))
            else:
                dn = rec(x - h)
                mask |= kinks(up, base, dn, h)
                est.append((up - dn) / (2 * h))
        fd = [float(np.sum(np.where(mask, 0.0, cot) * e)) for e in est]
        if abs(fd[0] - fd[1]) <= 5e-5 * abs(fd[0]):
            break
    return fd[0], mask, r


def test_temperature(case):
    c = case
    T, P = c["T"], c["P"]
    masked = c["cot"].copy()
    fd, steps = np.zeros(len(T)), []
    for l in range(len(T)):
        knot = float((T[l] - 20.0) / 2.0).is_integer()
        fd[l], mask, r = level_fd(c, l, lambda t: level_records(c, l, P[l], t), T[l], knot)
        masked[l][mask] = 0.0
        steps.append(r)
    g = c["ctx"].vjp(c["run"], P, T, c["n"], masked)
    print(f"\ntemperature: {int((masked == 0).sum())} of {masked.size} points left out; steps {steps}")
    for l in range(len(T)):
        assert rel(fd[l], g["dT"][l]) <= TOL, (l, T[l], g["dT"][l], fd[l])


def test_pressure(case):
    c = case
    T, P = c["T"], c["P"]
    masked = c["cot"].copy()
    fd, steps = np.zeros(len(P)), []
    for l in range(len(P)):
        fd[l], mask, r = level_fd(c, l, lambda p: level_records(c, l, p, T[l]), P[l], False)
        masked[l][mask] = 0.0
        steps.append(r)
    g = c["ctx"].vjp(c["run"], P, T, c["n"], masked)
    print(f"\npressure: {int((masked == 0).sum())} of {masked.size} points left out; steps {steps}")
    for l in range(len(P)):
        assert rel(fd[l], g["dP"][l]) <= TOL, (l, P[l], g["dP"][l], fd[l])


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
    base = _L(c)

    def check(what, up, dn, h, key, weights):
        masked = cot.copy()
        masked[kinks(up, base, dn, h)] = 0.0
        g = c["ctx"].vjp(c["run"], c["P"], c["T"], c["n"], masked)
        fd = float(np.sum(masked * (up - dn))) / (2 * h)
        an = float(g[key] @ weights)
        print(f"\n{what}: {int((masked == 0).sum())} of {cot.size} points left out")
        assert rel(fd, an) <= TOL, (what, an, fd)

    check("S direction", _L(c, S=S0 * (1 + STEP * v)), _L(c, S=S0 * (1 - STEP * v)), STEP, "dS", S0 * v)
    check("gamma_air direction", _L(c, G=G0 * (1 + STEP * v)), _L(c, G=G0 * (1 - STEP * v)), STEP,
          "dgamma_air", G0 * v)
    for i in np.argsort(-np.abs(c["g"]["dgamma_air"]))[:5]:
        h = STEP * G0[i]
        Gp, Gm = G0.copy(), G0.copy()
        Gp[i] += h
        Gm[i] -= h
        e = np.zeros(len(G0))
        e[i] = 1.0
        check(f"gamma_air of line {i}", _L(c, G=Gp), _L(c, G=Gm), h, "dgamma_air", e)


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
