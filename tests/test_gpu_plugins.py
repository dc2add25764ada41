"""The plugin surface beyond the Voigt: lorentzShape (Shapes.f90:135-141, the
chi-corrected Lorentz at every offset) and a TIPS table on another
temperature grid (the 1 K steps of Gamache's 2021 partition sums, which the
reference plans: README.md:458-460).

Lorentz: FP64 records within 1e-12 of the all-double oracle on every point,
FP32c within 1e-5 where k > 1e-6 max(k) (outside cascade near-ties), with
and without a chi-factor.  TIPS grid: the reference's 2 K table resampled to
1 K steps (each odd node the mean of its neighbours, so that linear
interpolation gives the same Q(T)) reproduces the 2 K results to 1e-12 and
agrees with the oracle on the same grid."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from fp32c_check import check_fp32c
from marfa_b200 import synth
from marfa_b200._lib import MarfaError
from marfa_b200.api import Context, Run

pytestmark = pytest.mark.gpu


def tips_1k(tips):
    """The 2 K table (T = 20 + 2j) on 1 K steps (T = 20 + j)."""
    t = np.asarray(tips, dtype=np.float64)
    out = np.empty((t.shape[0], 2 * t.shape[1] - 1))
    out[:, 0::2] = t
    out[:, 1::2] = 0.5 * (t[:, :-1] + t[:, 1:])
    return out


@pytest.mark.parametrize("chi", ["none", "tonkov"])
def test_lorentz_shape_matches_oracle(gpu, tips, chi):
    w = synth.config(1, scale=0.03)     # 30 cm-1 of the Venus list, 40 levels
    p = w.profiles[0]
    lv = slice(0, 40, 6)
    P, T, n = p.pressure[lv], p.temperature[lv], p.density[lv]
    orc = O.Oracle(w.lines, tips, P, T, n, w.start_wv, w.end_wv, w.cutoff, target=w.target, chi=chi,
                   shape="lorentz", precision=O.FP64)
    _, ref, _ = orc.run()
    run = dict(start_wv=w.start_wv, end_wv=w.end_wv, cutoff=w.cutoff, target=w.target,
               molecule=w.molecule, chi=chi, shape="lorentz")
    with Context(w.lines, tips) as ctx:
        _, g64 = ctx.compute(Run(precision="fp64", **run), P, T, n, want64=True)
        g32 = ctx.compute(Run(precision="fp32c", **run), P, T, n)
    err, npts = rel_err(g64, ref, 0.0)
    assert npts == ref.size and err <= 1e-12, err
    e32, taint = check_fp32c(g32, ref, orc, tol=1e-5)
    assert e32 <= 1e-5 and taint <= 1e-4 * ref.size


def test_lorentz_differs_from_voigt_near_line_centres(gpu, tips):
    """At low pressure the Doppler core makes the two shapes differ near the
    line centres and agree in the far wings."""
    w = synth.config(0)
    p = synth.Profile(synth.f32([1e-3]), synth.f32([200.0]),
                      synth.ideal_gas_density(synth.f32([1e-3]), synth.f32([200.0])))
    with Context(w.lines, tips) as ctx:
        v = ctx.compute(Run(w.start_wv, w.end_wv, w.cutoff, precision="fp64"), p.pressure,
                        p.temperature, p.density)
        l = ctx.compute(Run(w.start_wv, w.end_wv, w.cutoff, precision="fp64", shape="lorentz"),
                        p.pressure, p.temperature, p.density)
    assert np.max(np.abs(l - v) / np.maximum(v, 1e-300)) > 0.1


def test_tips_on_1k_grid(gpu, tips):
    w = synth.config(0)
    p = w.profiles[0]
    prof = synth.Profile(synth.f32([1.0, 0.1]), synth.f32([296.0, 251.3]),
                         synth.ideal_gas_density(synth.f32([1.0, 0.1]), synth.f32([296.0, 251.3])))
    t1 = tips_1k(tips)
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp64")
    with Context(w.lines, tips) as ctx:
        _, base = ctx.compute(run, prof.pressure, prof.temperature, prof.density, want64=True)
    with Context(w.lines, t1) as ctx:
        ctx.set_tips_grid(20.0, 1.0)
        _, g = ctx.compute(run, prof.pressure, prof.temperature, prof.density, want64=True)
        with pytest.raises(MarfaError) as e:          # 296 K outside a table starting at 300 K
            ctx.set_tips_grid(300.0, 1.0)
        assert e.value.code == 10
        t_hot = 20.0 + (t1.shape[1] - 1) + 1.0      # 1 K past the table's last node
        hot = synth.Profile(synth.f32([1.0]), synth.f32([t_hot]),
                            synth.ideal_gas_density(synth.f32([1.0]), synth.f32([t_hot])))
        with pytest.raises(MarfaError) as e:          # beyond the last node
            ctx.compute(run, hot.pressure, hot.temperature, hot.density)
        assert e.value.code == 11
    orc = O.Oracle(w.lines, t1, prof.pressure, prof.temperature, prof.density, w.start_wv, w.end_wv,
                   w.cutoff, target=w.target, chi=w.chi, precision=O.FP64, tips_grid=(20.0, 1.0))
    _, ref, _ = orc.run()
    assert rel_err(g, base, 0.0)[0] <= 1e-12
    assert rel_err(g, ref, 0.0)[0] <= 1e-12
