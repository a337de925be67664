"""Launch-shape autotuner for the persistent integrator kernels.

For one (view set, integrator) pair it times every candidate launch shape --
threads per block, resident blocks per SM, and the number of sample slots a
lane takes per work-queue fetch -- with CUDA events and keeps the fastest.
For the gradient calls it then times the round size of the split kernels
(sample slots per set-up/body round of the boundary terms, paths per round
of the interior adjoint: smaller rounds need smaller queues, larger ones give
each edge more samples per sort and fewer kernel tails) with that shape.
Results are cached per (integrator, slot-count bucket, scene size bucket).
Gradient passes write into the scene's gradient buffers, so the caller clears
them after tuning (tune() does it).
"""
from __future__ import annotations

import math

import torch

from . import api

BLOCKS = (128, 256)
PER_SM = (2, 4, 8)
CHUNKS = (1, 4)
ROUND_LOG2 = (20, 22)   # tried against the library default (16M boundary slots, 2M paths)

_cache: dict = {}


def _key(vs: api.ViewSet, integrator: int) -> tuple:
    slots = vs.slots(integrator)
    return (integrator, int(math.log2(max(slots, 1))), int(math.log2(max(vs.scene.num_triangles, 1))))


def tune(vs: api.ViewSet, integrator: int, options: api.RenderOptions, dLdI: torch.Tensor | None = None,
         reps: int = 1, candidates=None) -> api.TrnLaunch:
    """Return the fastest launch shape for this integrator on this view set."""
    key = _key(vs, integrator)
    if key in _cache:
        return _cache[key]
    cands = candidates or [(b, p, c) for b in BLOCKS for p in PER_SM for c in CHUNKS if b * p <= 2048]
    if dLdI is None:
        g = torch.Generator(device="cpu").manual_seed(0)
        dLdI = (torch.rand(vs.npix, 3, generator=g) - 0.5).to(vs.scene.device)

    def run(ln):
        vs.render_grad(integrator, options, dLdI, launch=ln)

    best, best_ms = None, float("inf")
    for b, p, c in cands:
        ln = api.launch_config(b, p, c)
        run(ln)  # warm
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run(ln)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        if ms < best_ms:
            best, best_ms = ln, ms
    # round size of the split kernels, with the best shape (only sizes below
    # the call's slot count change anything)
    slots = vs.slots(integrator)
    for r in ROUND_LOG2:
        if (1 << r) >= slots:
            continue
        ln = api.launch_config(best.block, best.blocks_per_sm, best.chunk, r)
        run(ln)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run(ln)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        if ms < best_ms:
            best, best_ms = ln, ms
    vs.scene.clear_grads()
    _cache[key] = best
    return best


def tune_forward(vs: api.ViewSet, options: api.RenderOptions, reps: int = 1) -> api.TrnLaunch:
    key = ("fwd",) + _key(vs, api.TRN_PATH_TRACER)
    if key in _cache:
        return _cache[key]
    out = torch.empty(vs.npix, 3, device=vs.scene.device)
    best, best_ms = None, float("inf")
    for b in BLOCKS:
        for p in PER_SM:
            for c in CHUNKS:
                if b * p > 2048:
                    continue
                ln = api.launch_config(b, p, c)
                vs.render(api.TRN_PATH_TRACER, options, launch=ln, out=out)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    vs.render(api.TRN_PATH_TRACER, options, launch=ln, out=out)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                if ms < best_ms:
                    best, best_ms = ln, ms
    _cache[key] = best
    return best
