"""Run one benchmark configuration, or a subset of its levels, a few times.

    python -m marfa_b200.run_case [--config 1] [--levels 0,20] [--precision fp32c]
                                  [--shape voigt] [--iters 2]

The small cases this makes (a few levels of the Venus-like workload) are the
ones to put under a profiler: every kernel of the full computation runs, on a
fraction of the device memory.  Prints the per-family kernel times of every
iteration (CUDA events on the computation's stream).
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--levels", default="", help="comma-separated level indices (default: all)")
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--shape", default="voigt", choices=["voigt", "one", "absx"])
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--vjp", action="store_true",
                    help="run the adjoint (FP64) for a Gaussian cotangent instead of the forward")
    args = ap.parse_args(argv)

    import torch
    from . import build, data_path, synth
    from .api import Context, Run
    from .io import read_tips

    build.build()
    w = synth.config(args.config)
    p = w.profiles[0]
    lv = [int(x) for x in args.levels.split(",")] if args.levels else list(range(len(p.pressure)))
    P, T, n = (np.asarray(a)[lv] for a in (p.pressure, p.temperature, p.density))
    ctx = Context(w.lines, read_tips(data_path("TIPS_subset.dat")))
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision=args.precision, shape=args.shape)
    if args.vjp:
        cot = np.random.default_rng(3).standard_normal((len(P), run.n_sub, 20481))
        for it in range(args.iters):
            g = ctx.vjp(run, P, T, n, cot)
            print(json.dumps({"iter": it, "dT": g["dT"].tolist(), "dP": g["dP"].tolist()}), flush=True)
        ctx.close()
        return
    out = torch.empty((len(P), run.n_sub, 20481), dtype=torch.float32, device="cuda")
    for it in range(args.iters):
        ctx.compute_device(run, [len(P)], P, T, n, out.data_ptr(), 0)
        ctx.synchronize()
        print(json.dumps({"iter": it, **{k: round(v, 4) for k, v in ctx.timings().items()}}), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
