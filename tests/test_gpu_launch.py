"""Launch parameters (marfa_ctx_set_launch / marfa_ctx_get_launch): values
outside the tuned sets are refused, and the FP32c fine-kernel block shapes
(one 1024-thread block per SM, or two of 512) both give the method's
results: within 1e-5 of the FP64 oracle where k > 1e-6 max(k) (outside
cascade near-ties), on a workload whose densest units stage in global
memory under the paired shape.  FP64 ignores the shape (bit-identical
records), and every far-kernel chunk size and lane-group setting keeps the
FP64 records within 1e-12 of the oracle."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from fp32c_check import check_fp32c
from marfa_b200 import synth
from marfa_b200._lib import MarfaError
from marfa_b200.api import Context, Run

pytestmark = pytest.mark.gpu


def test_set_launch_validates_and_round_trips(gpu, tips):
    w = synth.config(0)
    with Context(w.lines, tips) as ctx:
        default = ctx.launch()
        assert default["fine_pair"] == 0
        ctx.set_launch(4096, 3, 1)
        assert ctx.launch() == {"far_chunk": 4096, "coop_k": 3, "fine_pair": 1}
        for bad in ((3000, 3, 0), (4096, 0, 0), (4096, 6, 0), (4096, 3, 2)):
            with pytest.raises(MarfaError) as e:
                ctx.set_launch(*bad)
            assert e.value.code == 10
        assert ctx.launch() == {"far_chunk": 4096, "coop_k": 3, "fine_pair": 1}


def test_fine_block_shapes_match_oracle(gpu, tips):
    # 60 cm-1 of the Venus list (about 2,400 near lines per unit) plus a band
    # of 3,000 lines in 4 cm-1: units on both sides of the 2,304 lines a
    # paired block stages on chip (and of the 2,688 of a 1024-thread block)
    w = synth.config(1, scale=0.06)
    rng = np.random.default_rng(11)
    band = w.lines[rng.choice(len(w.lines) - 1, 3000)].copy()
    band["nu"] = np.sort(rng.uniform(w.start_wv + 21.0, w.start_wv + 25.0, 3000))
    lines = np.concatenate([w.lines[:-1], band])
    lines = np.concatenate([lines[np.argsort(lines["nu"], kind="stable")], w.lines[-1:]])
    p = w.profiles[0]
    lv = slice(0, 40, 8)
    P, T, n = p.pressure[lv], p.temperature[lv], p.density[lv]
    orc = O.Oracle(lines, tips, P, T, n, w.start_wv, w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                   precision=O.FP64)
    _, ref, _ = orc.run()
    run = dict(start_wv=w.start_wv, end_wv=w.end_wv, cutoff=w.cutoff, target=w.target,
               molecule=w.molecule, chi=w.chi)
    recs, r64 = {}, {}
    with Context(lines, tips) as ctx:
        for pair in (0, 1):
            ctx.set_launch(16384, 5, pair)
            recs[pair] = ctx.compute(Run(precision="fp32c", **run), P, T, n)
            _, r64[pair] = ctx.compute(Run(precision="fp64", **run), P, T, n, want64=True)
    for pair in (0, 1):
        e32, taint = check_fp32c(recs[pair], ref, orc, tol=1e-5)
        print(f"fine_pair={pair}: max err {e32:.3e} outside {taint} near-tie points")
        assert e32 <= 1e-5 and taint <= 1e-4 * ref.size
    assert np.array_equal(r64[0], r64[1])


@pytest.mark.parametrize("far_chunk,coop_k", [(2048, 1), (4096, 3), (8192, 5), (16384, 2)])
def test_launch_parameters_keep_fp64_parity(gpu, tips, far_chunk, coop_k):
    """Every far-kernel chunk size (the cp.async tiles then end inside a
    tile at many chunk boundaries) and lane-group setting gives FP64 records
    within 1e-12 of the all-double oracle."""
    w = synth.config(1, scale=0.03)
    p = w.profiles[0]
    lv = slice(0, 40, 13)
    P, T, n = p.pressure[lv], p.temperature[lv], p.density[lv]
    orc = O.Oracle(w.lines, tips, P, T, n, w.start_wv, w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                   precision=O.FP64)
    _, ref, _ = orc.run()
    with Context(w.lines, tips) as ctx:
        ctx.set_launch(far_chunk, coop_k, 0)
        _, g64 = ctx.compute(Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule,
                                 chi=w.chi, precision="fp64"), P, T, n, want64=True)
    err, npts = rel_err(g64, ref, 0.0)
    assert npts == ref.size and err <= 1e-12, err
