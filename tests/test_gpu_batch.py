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
    """The tuned launch parameters change only the order of summation: FP64
    records stay within 1e-12 of the untuned ones, FP32c records within the
    FP32c contract of the FP64 oracle (1e-5 away from near-tie clamps) with
    and without tuning."""
    import oracle as O
    from fp32c_check import check_fp32c
    from marfa_b200.io import species_code
    tips = read_tips(data_path("TIPS_subset.dat"))
    w = synth.config(1, 0.03)
    p = w.profiles[0]
    lv = [0, 13, 26, 39]
    P, T, n = (np.asarray(a, dtype=np.float64)[lv] for a in (p.pressure, p.temperature, p.density))
    orc = O.Oracle(w.lines, tips, P, T, n, w.start_wv, w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                   mol_code=species_code(w.molecule), precision=O.FP64)
    ref = orc.run()[1]
    for prec in ("fp32c", "fp64"):
        run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
                  precision=prec)
        with Context(w.lines, tips) as ctx:
            before = ctx.compute(run, P, T, n, want64=True)
            choice = ctx.autotune(run, P, T, n)
            assert choice["far_chunk"] in (2048, 4096, 8192, 16384)
            assert 1 <= choice["coop_k"] <= 5
            after = ctx.compute(run, P, T, n, want64=True)
        if prec == "fp64":
            b, a = before[1], after[1]
            big = b > 1e-6 * b.max()
            rel = np.abs(a[big] - b[big]) / b[big]
            assert rel.max() <= 1e-12, (choice, rel.max())
        else:
            for got in (before[0], after[0]):
                err, n_tainted = check_fp32c(got, ref, orc)
                assert err <= 1e-5, (choice, err)
                assert n_tainted <= 1e-4 * ref.size


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


def test_queued_device_calls(gpu):
    """Device calls queue on the stream without waiting (a ring of pinned
    staging buffers carries their tables): six calls with different profiles
    enqueued back to back give the records of the same calls made one at a
    time."""
    torch = pytest.importorskip("torch")
    tips = read_tips(data_path("TIPS_subset.dat"))
    w = synth.config(1, 0.03)
    p = w.profiles[0]
    P, T, n = (np.asarray(a, dtype=np.float64) for a in (p.pressure, p.temperature, p.density))
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp32c")
    shape = (len(P), run.n_sub, 20481)
    pressures = [P * (1.0 + 0.05 * i) for i in range(6)]
    with Context(w.lines, tips) as ctx:
        one = []
        for Pi in pressures:
            o = torch.empty(shape, dtype=torch.float32, device="cuda")
            ctx.compute_device(run, [len(P)], Pi, T, n, o.data_ptr())
            ctx.synchronize()
            one.append(o)
        queued = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in pressures]
        for Pi, o in zip(pressures, queued):
            ctx.compute_device(run, [len(P)], Pi, T, n, o.data_ptr())
        ctx.synchronize()
        for a, b in zip(one, queued):
            assert torch.equal(a, b)
        assert not torch.equal(one[0], one[5])
