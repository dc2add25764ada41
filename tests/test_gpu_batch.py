"""Batched execution: CUDA-graph capture and replay, and the launch-parameter
autotuner (marfa_graph_*, marfa_autotune)."""
import numpy as np
import pytest

from marfa_b200 import synth, data_path
from marfa_b200._lib import MarfaError
from marfa_b200.api import Context, Run
from marfa_b200.io import read_tips

pytestmark = pytest.mark.gpu


def _uneven(scale=0.05):
    """The uneven-batch configuration (H2O-like lines, profiles of 10-100
    levels) at a reduced size: profiles concatenated level-wise."""
    w = synth.config(2, scale)
    counts = [len(p.pressure) for p in w.profiles]
    cat = lambda f: np.concatenate([np.asarray(getattr(p, f), dtype=np.float64) for p in w.profiles])
    return w, counts, cat("pressure"), cat("temperature"), cat("density")


def test_graph_replay_matches_direct_calls(gpu):
    torch = pytest.importorskip("torch")
    tips = read_tips(data_path("TIPS_subset.dat"))
    w, counts, P, T, n = _uneven()
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp32c")
    L = sum(counts)
    with Context(w.lines, tips) as ctx:
        out_g = torch.empty((L, run.n_sub, 20481), dtype=torch.float32, device="cuda")
        out_d = torch.empty_like(out_g)
        g = ctx.graph(run, counts, P, T, n, out_g.data_ptr())
        ctx.compute_device(run, counts, P, T, n, out_d.data_ptr())
        ctx.synchronize()
        assert torch.equal(out_g, out_d)
        for dT in (3.0, -7.5):  # replays for new profiles of the same shape
            T2 = T + dT
            g.launch(P, T2, n)
            ctx.compute_device(run, counts, P, T2, n, out_d.data_ptr())
            ctx.synchronize()
            assert torch.equal(out_g, out_d)
            assert float(out_g.abs().sum()) > 0.0
        g.close()


def test_graph_refuses_a_changed_launch_plan(gpu):
    torch = pytest.importorskip("torch")
    tips = read_tips(data_path("TIPS_subset.dat"))
    w, counts, P, T, n = _uneven()
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp32c")
    with Context(w.lines, tips) as ctx:
        out = torch.empty((sum(counts), run.n_sub, 20481), dtype=torch.float32, device="cuda")
        g = ctx.graph(run, counts, P, T, n, out.data_ptr())
        # a larger computation grows the context's buffers: the graph's
        # captured addresses are gone, and its launch must say so
        big = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
                  precision="fp64")
        ctx.compute(big, P, T, n)
        with pytest.raises(MarfaError) as e:
            g.launch(P, T, n)
        assert e.value.code == 10
        g.close()


def test_autotune_keeps_results(gpu):
    torch = pytest.importorskip("torch")
    tips = read_tips(data_path("TIPS_subset.dat"))
    w = synth.config(1, 0.03)
    p = w.profiles[0]
    lv = [0, 13, 26, 39]
    P, T, n = (np.asarray(a, dtype=np.float64)[lv] for a in (p.pressure, p.temperature, p.density))
    for prec, tol in (("fp32c", 1e-5), ("fp64", 1e-12)):
        run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
                  precision=prec)
        with Context(w.lines, tips) as ctx:
            before = ctx.compute(run, P, T, n, want64=True)[1]
            choice = ctx.autotune(run, P, T, n)
            assert choice["far_chunk"] in (2048, 4096, 8192)
            assert 1 <= choice["coop_k"] <= 5
            after = ctx.compute(run, P, T, n, want64=True)[1]
        big = before > 1e-6 * before.max()
        rel = np.abs(after[big] - before[big]) / before[big]
        assert rel.max() <= tol, (prec, choice, rel.max())


def test_host_record_chunks_keep_results(gpu):
    """Records copied to host memory come in level chunks whose sizes follow
    the copy/kernel time ratio measured on the previous call; every schedule
    gives the records of the device-memory path."""
    torch = pytest.importorskip("torch")
    tips = read_tips(data_path("TIPS_subset.dat"))
    w = synth.config(1, 0.03)
    p = w.profiles[0]
    P, T, n = (np.asarray(a, dtype=np.float64) for a in (p.pressure, p.temperature, p.density))
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp32c")
    with Context(w.lines, tips) as ctx:
        dev = torch.empty((len(P), run.n_sub, 20481), dtype=torch.float32, device="cuda")
        ctx.compute_device(run, [len(P)], P, T, n, dev.data_ptr())
        ctx.synchronize()
        ref = dev.cpu()
        for _ in range(3):
            host = torch.empty_like(ref).pin_memory()
            ctx.compute(run, P, T, n, out=host)
            assert torch.equal(host, ref)
        assert float(ref.abs().sum()) > 0.0
