"""Parity of the CUDA library with the CPU oracle across the benchmark
configurations (reduced sizes), chi-factors, targets, batching, output paths
and error statuses.  FP64: 1e-12 relative on every point; FP32c: 1e-5
relative where k > 1e-6 max(k)."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from fp32c_check import check_fp32c
from marfa_b200 import synth
from marfa_b200.api import Context, Run
from marfa_b200._lib import MarfaError
from marfa_b200.io import species_code

pytestmark = pytest.mark.gpu


def make_oracle(w, tips, prof, **kw):
    return O.Oracle(w.lines, tips, prof.pressure, prof.temperature, prof.density, w.start_wv,
                    w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                    mol_code=species_code(w.molecule), precision=O.FP64, **kw)


def oracle_ref(w, tips, prof, **kw):
    return make_oracle(w, tips, prof, **kw).run()[1]


def check(ctx, w, tips, prof=None, fp64_tol=1e-12, fp32c_tol=1e-5, **run_kw):
    prof = prof or w.profiles[0]
    orc = make_oracle(w, tips, prof)
    ref = orc.run()[1]
    d = dict(start_wv=w.start_wv, end_wv=w.end_wv, cutoff=w.cutoff, target=w.target,
             molecule=w.molecule, chi=w.chi)
    d.update(run_kw)
    _, g64 = ctx.compute(Run(precision="fp64", **d), prof.pressure, prof.temperature,
                         prof.density, want64=True)
    assert rel_err(g64, ref, 0.0)[0] <= fp64_tol
    g32 = ctx.compute(Run(precision="fp32c", **d), prof.pressure, prof.temperature, prof.density)
    err, n_tainted = check_fp32c(g32, ref, orc, tol=fp32c_tol)
    assert err <= fp32c_tol
    assert n_tainted <= 1e-4 * ref.size
    return ref


def test_venus_all_levels_short_span(gpu, tips):
    w = synth.config(1, scale=0.03)                  # 6,000 lines over 30 cm-1, 40 levels
    with Context(w.lines, tips) as ctx:
        check(ctx, w, tips)


@pytest.mark.parametrize("chi", ["tonkov", "pollack", "perrin"])
@pytest.mark.parametrize("target", ["ACS", "VAC"])
def test_chi_factors_and_targets(gpu, tips, chi, target):
    w = synth.config(0)
    w.chi, w.target = chi, target
    with Context(w.lines, tips) as ctx:
        check(ctx, w, tips)


def test_chi_factor_applies_only_to_co2(gpu, tips):
    w = synth.config(0)
    w.chi, w.molecule = "tonkov", "H2O"              # factor disabled for H2O
    w.lines = w.lines.copy()
    with Context(w.lines, tips) as ctx:
        ref = check(ctx, w, tips)
        w.chi = "none"
        assert np.array_equal(ref, oracle_ref(w, tips, w.profiles[0]))


def test_stress_weak_intensities_and_long_cutoff(gpu, tips):
    """S down to 1e-30 (float underflow without the intensity scaling),
    cutoff 250, 100 levels."""
    w = synth.config(4, scale=0.002)                 # 4,000 lines over 500-10000
    w.start_wv, w.end_wv = 5000.0, 5100.0
    with Context(w.lines, tips) as ctx:
        check(ctx, w, tips)


def test_uneven_batch_matches_per_profile(gpu, tips):
    w = synth.config(2, scale=0.05)                  # H2O-like, 1,500 lines, 3 profiles
    w.end_wv = 300.0
    profs = [synth.random_profile(1000 + i, n_range=(3, 12)) for i in range(3)]
    counts = [p.n_levels for p in profs]
    cat = lambda f: np.concatenate([getattr(p, f) for p in profs])
    with Context(w.lines, tips) as ctx:
        for prec in ("fp64", "fp32c"):
            run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule,
                      precision=prec)
            batch = ctx.compute_batched(run, counts, cat("pressure"), cat("temperature"),
                                        cat("density"))
            off = 0
            for p in profs:
                ref = oracle_ref(w, tips, p)
                got = batch[off:off + p.n_levels]
                tol = 1e-6 if prec == "fp64" else 1e-5     # float32 records
                assert rel_err(got, ref, 1e-6)[0] <= tol
                off += p.n_levels


def test_device_output_equals_host_output_and_is_deterministic(gpu, tips):
    import torch
    w = synth.config(1, scale=0.02)
    p = w.profiles[0]
    with Context(w.lines, tips) as ctx:
        run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule,
                  chi=w.chi, precision="fp32c")
        host = ctx.compute(run, p.pressure, p.temperature, p.density)
        dev = torch.empty(host.shape, dtype=torch.float32, device="cuda")
        st = torch.cuda.Stream()
        ctx.compute_device(run, [p.n_levels], p.pressure, p.temperature, p.density,
                           dev.data_ptr(), st.cuda_stream)
        st.synchronize()
        assert np.array_equal(dev.cpu().numpy(), host)
        again = ctx.compute(run, p.pressure, p.temperature, p.density)
        assert np.array_equal(again, host)


def test_error_statuses(gpu, tips):
    w = synth.config(0)
    p = w.profiles[0]
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule)
    with Context(w.lines, tips) as ctx:
        with pytest.raises(MarfaError) as e:                   # outside the TIPS table
            ctx.compute(run, [1.0], [10.0], [1e20])
        assert e.value.code == 11
        with pytest.raises(MarfaError) as e:                   # pSelf > P
            ctx.compute(run, [1.0], [296.0], [1e26])
        assert e.value.code == 7
        with pytest.raises(MarfaError) as e:                   # more than 200 levels
            ctx.compute_batched(run, [201], np.ones(201), np.full(201, 296.0), np.ones(201))
        assert e.value.code == 6
        with pytest.raises(MarfaError) as e:
            Run(4000, 4100, 25, molecule="XE").c()
        assert e.value.code == 8
    with Context(w.lines[:-1], tips) as ctx:                   # no line beyond the last window
        with pytest.raises(MarfaError) as e:
            ctx.compute(run, p.pressure, p.temperature, p.density)
        assert e.value.code == 9
    unsorted = w.lines.copy()
    unsorted["nu"][[3, 4]] = unsorted["nu"][[4, 3]]
    with pytest.raises(MarfaError) as e:
        Context(unsorted, tips)
    assert e.value.code == 12
    lines = w.lines.copy()
    lines["jmi"][10] = 1502                                   # isotopologue 15: no TIPS row
    with Context(lines, tips) as ctx, pytest.raises(MarfaError) as e:
        ctx.compute(run, p.pressure, p.temperature, p.density)
    assert e.value.code == 13
