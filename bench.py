#!/usr/bin/env python
"""Benchmark: grad path-samples/sec of render + gradient on one B200 per rank.

Workload (default): the 100K-triangle config -- a sphere displaced by 3-octave
value noise, GGX microfacet (roughness 0.3) with a 512x512 albedo texture,
ground quad and quad light, 512x512 pixels, 64 spp per term, depth 5, all
boundary terms (primary, direct, indirect, pixel), gradients w.r.t. every
vertex position and the texture. One step = parameter upload to the scene +
Scene::Configure (geometry chain + LBVH rebuild) + PathTracer.renderC +
dL/dI of 0.5*|I - I_target|^2 + renderD of all five integrators + the
geometry adjoint. A grad path-sample is one sample slot processed forward +
adjoint by one integrator: W*H*spp per enabled term.

With --gpus N (torchrun) every rank renders its own seeds of the same view
and the gradient buffers are summed with one NCCL all-reduce (weak scaling).
--impl reference times the CPU oracle (the port of the reference path) on a
bounded sample of the same workload on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

# algorithmic bytes per counted unit (the roofline model of the path):
# closest-hit query = 32 B ray + 16 B hit + 48 B hit-triangle fetch; shadow
# query = 32 B + 4 B + 48 B; smooth-shaded vertex +36 B normals +12 B normal
# indices; textured vertex +24 B uv +12 B uv indices +12 B texel; light
# sample = 4 B per CDF probe + 48 B emitter triangle; one vertex gradient
# update = 12 B read-modify-write (24 B); texel update 24 B; pixel access 12 B.
B_CLOSEST, B_SHADOW, B_SMOOTH, B_TEX, B_LIGHT_TRI = 96, 84, 48, 48, 48
B_VSCATTER, B_NSCATTER, B_TSCATTER, B_PIXEL = 24, 24, 24, 12
CNT_NAMES = ["closest", "shadow", "shade", "smooth", "tex", "light", "vscatter", "nscatter", "tscatter", "pixel"]


def algorithmic_bytes(c: dict, n_emit: int) -> int:
    light = 4 * max(1, math.ceil(math.log2(max(n_emit, 2)))) + B_LIGHT_TRI
    return (c["closest"] * B_CLOSEST + c["shadow"] * B_SHADOW + c["smooth"] * B_SMOOTH + c["tex"] * B_TEX +
            c["light"] * light + c["vscatter"] * B_VSCATTER + c["nscatter"] * B_NSCATTER +
            c["tscatter"] * B_TSCATTER + c["pixel"] * B_PIXEL)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="trn", choices=["trn", "reference"])
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--tris", type=int, default=100_000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched-views and served-requests legs of the default run")
    ap.add_argument("--quick", action="store_true", help="small smoke-sized run")
    ap.add_argument("--no-path-cache", action="store_true",
                    help="gradient calls re-trace the interior paths instead of reusing the forward's records")
    ap.add_argument("--requests", type=int, default=48, help="serve workload: number of requests")
    ap.add_argument("--guide-depth", type=int, default=0,
                    help="inverse workload: refinement passes of the direct boundary's guiding tree")
    ap.add_argument("--workload", default="single", choices=["single", "icosphere", "views", "serve", "inverse"],
                    help="single: the 100K-triangle single-view config; icosphere: the 1280-triangle "
                         "config (translation gradient); views: 32 batched views "
                         "of the icosphere scene against the plain per-view form; serve: Poisson "
                         "render+gradient requests over four resident scenes; inverse: the 2M-triangle "
                         "16-view inverse-rendering loop (refit + guided direct boundary + Adam)")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling during the timed region. start() may come before
    the warm-up (nvidia-smi's own start-up then stays out of the timed
    steps); mark() at the start of the timed region keeps only the samples
    taken after it."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.t_mark = None
        # raw samples go to TRN_CLOCKS_DIR when set (kept for inspection),
        # else to the temporary directory
        d = os.environ.get("TRN_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, f"clocks_{os.getpid()}.csv")

    def mark(self):
        self.t_mark = time.time()

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], [], set()
        from datetime import datetime
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            if self.t_mark is not None:
                try:
                    if datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp() < self.t_mark:
                        continue
                except ValueError:
                    pass
            p = p[1:]
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_name(a) -> str:
    return (f"displaced sphere {a.tris // 1000}K tris, GGX r=0.3 + 512^2 texture, {a.res}x{a.res}, "
            f"{a.spp} spp x 5 terms (interior+primary+direct+indirect+pixel), depth {a.depth}, "
            f"grads: all vertex positions + texels")


# ---------------------------------------------------------------------------
# reference arm: the CPU oracle on a bounded sample
# ---------------------------------------------------------------------------
CPU_RES = 32  # pixel window of the bounded CPU sample (1 spp per term)


def cpu_oracle_rate(a, budget_s: float = 20.0, res: int = CPU_RES, spp: int = 1):
    from oracle import tr_oracle as O
    from tensorray_b200 import api, scenes
    torch.set_num_threads(os.cpu_count() or 1)
    spec = scenes.config2_scene(res, res, tris=a.tris)
    sc = O.OracleScene(spec, requires_grad=("positions", "texels"))
    c = spec.cameras[0]
    cam = O.camera_matrices(c.pos, c.target, c.up, c.width, c.height, c.fov)
    D = a.depth
    units = 0
    t0 = time.perf_counter()
    it = 0
    while True:
        target = torch.zeros(res * res, 3)
        for integ in range(5):
            smp = O.hash_table(it, integ, api.sample_dims(integ, D), api.sample_slots(integ, res, res, spp))
            dLdI = target + 0.5
            O.grads(sc, cam, integ, spp, D, smp, dLdI)
            units += res * res * spp
        it += 1
        if time.perf_counter() - t0 > budget_s or it >= 50:
            break
    dt = time.perf_counter() - t0
    return units / dt, units, dt, torch.get_num_threads()


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = []
    tot_units = 0
    t_all = 0.0
    for _ in range(a.warmup):
        cpu_oracle_rate(a, budget_s=2.0)
    for _ in range(a.steps):
        rate, units, dt, cores = cpu_oracle_rate(a, budget_s=10.0)
        steps.append(dt)
        tot_units += units
        t_all += dt
    value = tot_units / t_all
    sample = f"{tot_units // a.steps} grad path-samples per step: {CPU_RES}x{CPU_RES} px, 1 spp per term, 5 terms, same scene"
    line = {"metric": "grad path-samples/sec", "value": value, "unit": "grad path-samples/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_all / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene)", "impl": "reference",
            "config": {"workload": workload_name(a), "sample": sample},
            "cpu_baseline": {"value": value, "unit": "grad path-samples/s", "cores": torch.get_num_threads(),
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "grad path-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# trn arm
# ---------------------------------------------------------------------------
def main():
    a = parse()
    if a.quick:
        a.res, a.spp, a.tris = 128, 4, 20_000
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "views":
        return run_views(a)
    if a.workload == "inverse":
        return run_inverse(a)
    if a.workload == "serve":
        return run_serve(a)
    if a.workload == "icosphere":
        return run_icosphere(a)
    line, world = run_single(a)
    if line is not None and world == 1 and not a.no_extra:
        # the metric's comparison legs at N=1: the batched multi-view
        # configuration and the served request stream, each against the plain
        # per-view / one-at-a-time form of the same kernels
        import copy
        import gc
        ax = copy.copy(a)
        ax.steps, ax.warmup = min(a.steps, 10), max(3, min(a.warmup, 5))
        gc.collect()
        torch.cuda.empty_cache()
        ic = run_icosphere(ax, quiet=True)
        line["icosphere_plain"] = {"workload": ic["config"]["workload"], "value": ic["value"], "unit": ic["unit"],
                                   "ms_per_step": ic["ms_per_step"], "e2e": ic["e2e"]}
        gc.collect()
        torch.cuda.empty_cache()
        v = run_views(ax, quiet=True)
        line["batched_vs_plain"] = {
            "workload": v["config"]["workload"], "batched_over_plain": v["batched_over_plain"],
            "batched": {"value": v["value"], "unit": v["unit"], "ms_per_step": v["ms_per_step"]},
            "plain_per_view": {"value": v["plain_per_view"]["value"], "unit": v["unit"],
                               "ms_per_step": v["plain_per_view"]["ms_per_step"]},
            "split_ms": v["split_ms"], "graph_vs_eager_grad_rel_l2": v["graph_vs_eager_grad_rel_l2"],
            "steps": ax.steps, "warmup": ax.warmup}
        gc.collect()
        torch.cuda.empty_cache()
        sv = run_serve(ax, quiet=True)
        pl = sv["plain_one_at_a_time"]
        line["served_vs_plain"] = {
            "workload": sv["config"]["workload"],
            "served": {"latency_s": sv["latency_s"], "value": sv["value"], "unit": sv["unit"],
                       "requests_per_s": sv["requests_per_s"]},
            "plain_one_at_a_time": {"latency_s": pl["latency_s"], "value": pl["value"], "unit": sv["unit"],
                                    "requests_per_s": pl["requests_per_s"]},
            "plain_one_at_a_time_path_cache": sv["plain_one_at_a_time_path_cache"],
            "throughput_over_plain": sv["value"] / pl["value"],
            "p50_plain_over_served": pl["latency_s"]["p50"] / sv["latency_s"]["p50"],
            "clocks": sv["clocks"]}
    if line is not None:
        print(json.dumps(line), flush=True)


def run_single(a):
    """The 100K-triangle single-view configuration (the headline line);
    returns (line on rank 0 else None, world size)."""
    import torch.distributed as dist
    from tensorray_b200 import api, scenes
    from tensorray_b200 import autograd as tra
    from tensorray_b200 import _abi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    lib = _abi.load()

    spec = scenes.config2_scene(a.res, a.res, tris=a.tris)
    scene = api.Scene(spec)
    scene.configure()
    if a.no_path_cache:
        scene.set_path_cache(0)
    sphere = scene.shapes[0]
    D = a.depth
    from tensorray_b200 import dist as trd
    base_seed = trd.rank_seed(0, rank)
    opts = api.RenderOptions(base_seed, D, a.spp, a.spp, a.spp, a.spp, a.spp)
    integrators = [api.PathTracer(), api.PrimaryEdgeIntegrator(), api.DirectEdgeIntegrator(),
                   api.IndirectEdgeIntegrator(), api.PixelBoundaryIntegrator()]
    # timed spans: the interior forward and one span per renderD call; each
    # span is the term's production kernels (set-up rounds, edge keys and
    # their radix sort, body stages)
    kernel_names = ["interior_fwd", "interior_adj", "primary", "direct", "indirect", "pixel"]
    term_kernels = {
        "interior_fwd": ["k_path_fwd_rec_regen"] if not a.no_path_cache else ["k_path_fwd"],
        "interior_adj": (["k_path_reverse<8,true> (over the forward's path records)"] if not a.no_path_cache
                         else ["k_path_replay", "k_path_reverse"]),
        "primary": ["k_edge_keys", "cub radix sort", "k_primary_setup", "k_primary_body_regen"],
        "direct": ["k_edge_keys", "cub radix sort", "k_direct_setup", "k_direct_body"],
        "indirect": ["k_edge_keys", "cub radix sort", "k_indirect_setup", "k_indirect_sensor_regen",
                     "k_indirect_emitter_regen"],
        "pixel": ["k_pixel_setup", "k_primary_body_regen"],
    }
    units_per_step = a.res * a.res * a.spp * 5
    V0 = scene._raw_positions.clone()
    tex0 = torch.as_tensor(np.ascontiguousarray(spec.textures[0]), device=dev).reshape(-1, 3).clone()
    # target: same view rendered with perturbed geometry
    g = torch.Generator(device="cpu").manual_seed(7)
    Vt = V0.clone()
    sl = sphere.vertex_slice()
    Vt[sl] += (torch.randn(Vt[sl].shape, generator=g) * 0.01).to(dev)
    scene.set_vertex_positions(Vt)
    scene.configure()
    target = integrators[0].renderC(scene, api.RenderOptions(12345, D, a.spp, 0, 0, 0, 0)).clone()
    scene.set_vertex_positions(V0)
    scene.configure()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream()

    def step(ev=None):
        # parameter update -> Scene::Configure
        scene.set_vertex_positions(V0)
        scene.set_texels(tex0)
        scene.configure()
        if ev: ev["interior_fwd"][0].record(stream)
        img = integrators[0].renderC(scene, opts)
        if ev: ev["interior_fwd"][1].record(stream)
        dLdI = img - target
        scene.clear_grads()
        for i, it in enumerate(integrators):
            if ev: ev[kernel_names[i + 1]][0].record(stream)
            it.renderD(scene, opts, dLdI)
            if ev: ev[kernel_names[i + 1]][1].record(stream)
        gr = scene.get_grads(clear=True)
        return trd.allreduce_grads(gr)

    # the clock sampler starts before the warm-up, so that nvidia-smi's own
    # start-up does not fall into a timed step; only samples taken during the
    # timed steps count
    clocks = Clocks(local)
    clocks.start()
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    ev_keys = kernel_names
    per_kernel = {k: [] for k in ev_keys}
    clocks.mark()
    launches0 = lib.trn_kernel_launches()
    total_ms = 0.0
    step_ms = []
    for s in range(a.steps):
        if world > 1:
            dist.barrier()
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for k in ev_keys}
        e0.record(stream)
        step(ev)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        step_ms.append(round(e0.elapsed_time(e1), 2))
        for k in ev_keys:
            per_kernel[k].append(ev[k][0].elapsed_time(ev[k][1]))
    launches = lib.trn_kernel_launches() - launches0
    clk = clocks.stop()
    ms = torch.tensor([total_ms / a.steps], device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_per_step = float(ms)
    value = units_per_step * world / (ms_per_step / 1e3)

    # ---- the replay form: the gradient calls re-trace the interior paths
    # from their seeds instead of reading the forward's path records ----
    replay = None
    if not a.no_path_cache:
        scene.set_path_cache(0)
        rsteps = min(a.steps, 10)
        for _ in range(2):
            step()
        tot = 0.0
        for _ in range(rsteps):
            if world > 1:
                dist.barrier()
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        t = torch.tensor([tot / rsteps], device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        replay = {"value": units_per_step * world / (float(t) / 1e3), "unit": "grad path-samples/s",
                  "ms_per_step": float(t), "steps": rsteps,
                  "kernels": {"interior_fwd": ["k_path_fwd"], "interior_adj": ["k_path_replay", "k_path_reverse"]}}
        scene.set_path_cache(16 << 30)

    # ---- e2e: through the autograd.Function with host buffers ----
    e2e = None
    if not a.no_e2e:
        ctx = tra.RenderContext(scene, opts)
        Vh = V0.cpu().pin_memory()
        th = tex0.cpu().pin_memory()
        gVh = torch.empty_like(Vh).pin_memory()
        gth = torch.empty_like(th).pin_memory()
        lossh = torch.empty(1).pin_memory()

        def e2e_step():
            V = Vh.to(dev, non_blocking=True).requires_grad_(True)
            T = th.to(dev, non_blocking=True).requires_grad_(True)
            img = tra.render(V, T, ctx)
            loss = 0.5 * ((img - target) ** 2).sum()
            loss.backward()
            gv, gt = V.grad, T.grad
            if world > 1:
                flat = torch.cat([gv.reshape(-1), gt.reshape(-1)])
                dist.all_reduce(flat)
            gVh.copy_(gv, non_blocking=True)
            gth.copy_(gt, non_blocking=True)
            lossh.copy_(loss.detach().reshape(1), non_blocking=True)

        for _ in range(a.warmup):
            e2e_step()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(a.steps):
            if world > 1:
                dist.barrier()
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        t = torch.tensor([tot / a.steps], device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = {"value": units_per_step * world / (float(t) / 1e3), "unit": "grad path-samples/s",
               "h2d_bytes_per_step": int(Vh.numel() * 4 + th.numel() * 4),
               "d2h_bytes_per_step": int(gVh.numel() * 4 + gth.numel() * 4 + 4),
               "ms_per_step": float(t)}

    # ---- roofline of the dominant kernel: counters from one instrumented step ----
    lib.trn_stats_enable(scene.handle, 1)
    import ctypes as C
    buf = (C.c_ulonglong * 16)()
    lib.trn_stats_read(scene.handle, buf, 1, C.c_void_p(stream.cuda_stream))
    counts = {}
    scene.set_vertex_positions(V0)
    scene.configure()
    img = integrators[0].renderC(scene, opts)
    lib.trn_stats_read(scene.handle, buf, 1, C.c_void_p(stream.cuda_stream))
    counts["interior_fwd"] = dict(zip(CNT_NAMES, list(buf)[:10]))
    dLdI = img - target
    for i, it in enumerate(integrators):
        it.renderD(scene, opts, dLdI)
        lib.trn_stats_read(scene.handle, buf, 1, C.c_void_p(stream.cuda_stream))
        counts[kernel_names[i + 1]] = dict(zip(CNT_NAMES, list(buf)[:10]))
    scene.get_grads(clear=True)
    lib.trn_stats_enable(scene.handle, 0)
    avg = {k: sum(v) / len(v) for k, v in per_kernel.items()}
    dom = max(avg, key=avg.get)
    n_emit = 2
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    per_kernel_roof = {}
    for k in ev_keys:
        by = algorithmic_bytes(counts[k], n_emit)
        per_kernel_roof[k] = {"ms": avg[k], "alg_bytes": by, "gbs": by / (avg[k] / 1e3) / 1e9,
                              "counts": counts[k]}
    ach = per_kernel_roof[dom]["gbs"]
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(dom)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": traffic, "kernel": f"{dom} term: " + " + ".join(term_kernels[dom]),
                "peak_source": peak_src}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        rate, units, dt, cores = cpu_oracle_rate(a, budget_s=15.0)
        cpu = {"value": rate, "unit": "grad path-samples/s", "cores": cores, "kind": "port",
               "sample": f"{units} grad path-samples in {dt:.1f}s: {CPU_RES}x{CPU_RES} px, 1 spp per term, 5 terms, same scene"}

    line = None
    if rank == 0:
        line = {
            "metric": "grad path-samples/sec", "value": value, "unit": "grad path-samples/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": workload_name(a), "global_batch_samples": units_per_step * world,
                       "res": a.res, "spp_per_term": a.spp, "depth": D, "triangles": scene.num_triangles,
                       "l2": "flushed between timed steps (256 MB write)", "parallelism": f"seeds x{world}"},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "roofline": roofline, "step_ms": step_ms,
            "replay_form": replay,
            "kernels": {k: {"ms": v["ms"], "GB/s": v["gbs"], "launches_of": term_kernels[k], "counts": v["counts"]}
                        for k, v in per_kernel_roof.items()},
            "cpu_baseline": cpu,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line, world


# ---------------------------------------------------------------------------
# batched multi-view workload: one graph-captured launch per integrator for
# all views vs the same kernels launched one view at a time
# ---------------------------------------------------------------------------
def run_views(a, quiet: bool = False):
    from tensorray_b200 import api, autotune, scenes
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rng = np.random.default_rng(0)
    nviews = 8 if a.quick else 32
    res_choices = [64, 96] if a.quick else [128, 256, 384, 512]
    spec = scenes.config1_scene(256, 256)
    scene = api.Scene(spec)
    scene.configure()
    cams_spec = scenes.fibonacci_cameras(nviews, 4.0, res_choices, seed=1)
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov) for c in cams_spec]
    spps = [int(x) for x in rng.choice([8, 16, 32, 64] if not a.quick else [4, 8], size=nviews)]
    D = 3
    terms = [api.TRN_PATH_TRACER, api.TRN_PRIMARY_EDGE, api.TRN_DIRECT_EDGE]
    vs = api.ViewSet(scene, cams, spps)
    opts = api.RenderOptions(1, D, 0, 0, 0, 0, 0)
    # targets: the same views with the sphere shifted
    scene.shapes[0].translation = torch.tensor([0.05, -0.03, 0.02])
    scene.configure()
    targets = vs.render(api.TRN_PATH_TRACER, api.RenderOptions(77, D, 0, 0, 0, 0, 0)).clone()
    scene.shapes[0].translation = torch.zeros(3)
    scene.configure()
    units = sum(c.width * c.height * s for c, s in zip(cams, spps)) * len(terms)
    # launch shapes: the library defaults and the per-integrator autotuned
    # ones; the whole captured step is timed with both and the faster is kept
    shapes = {"default": (None, {t: None for t in terms}),
              "autotuned": (autotune.tune_forward(vs, opts, reps=2),
                            {t: autotune.tune(vs, t, opts, reps=2) for t in terms})}
    img = torch.empty(vs.npix, 3, device=scene.device)
    dLdI = torch.empty(vs.npix, 3, device=scene.device)
    ln_f, ln_g = shapes["default"]

    def batched_step():
        vs.render(api.TRN_PATH_TRACER, opts, launch=ln_f, out=img)
        loss = vs.loss(img, targets, dLdI)
        for t in terms:
            vs.render_grad(t, opts, dLdI, launch=ln_g[t])
        g = scene.get_grads(clear=True)
        return loss, g["positions"]

    # plain form: one view set per view, same kernels, launched view by view
    singles = [api.ViewSet(scene, [c], [s], seeds=[i]) for i, (c, s) in enumerate(zip(cams, spps))]
    tgt_v = [vs.view_image(targets, i).reshape(-1, 3).contiguous() for i in range(nviews)]

    def plain_step():
        # the reference's multi-view loop (pyTensorRay/renderer_multi_view.py:
        # 53-98): per view a forward, its loss, every integrator's renderD
        # and get_grads, summed into the vertex gradient
        losses = []
        gsum = torch.zeros(scene.num_vertices, 3, device=scene.device)
        for i, sv in enumerate(singles):
            im = sv.render(api.TRN_PATH_TRACER, opts)
            d = torch.empty_like(im)
            losses.append(sv.loss(im, tgt_v[i], d))
            for t in terms:
                sv.render_grad(t, opts, d)
            gsum += scene.get_grads(clear=True)["positions"]
        return losses, gsum

    for _ in range(a.warmup):
        batched_step()
        plain_step()
    torch.cuda.synchronize()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=scene.device)
    graphs = {}
    for name, (lf, lg) in shapes.items():
        ln_f, ln_g = lf, lg
        graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            batched_step()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            out_loss, out_grad = batched_step()
        graphs[name] = (graph, out_loss, out_grad)

    def timed(fn):
        tot = 0.0
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / a.steps

    shape_ms = {}
    for name, (graph, _, _) in graphs.items():
        for _ in range(a.warmup):
            graph.replay()
        shape_ms[name] = timed(graph.replay)
    best = min(shape_ms, key=shape_ms.get)
    graph, out_loss, out_grad = graphs[best]
    ln_f, ln_g = shapes[best]
    ms_batched = shape_ms[best]
    ms_plain = timed(plain_step)
    # the graph-captured step computes what the eager batched step computes
    graph.replay()
    torch.cuda.synchronize()
    g_graph = out_grad.clone()
    _, g_eager = batched_step()
    rel = float((g_graph - g_eager).norm() / g_eager.norm().clamp_min(1e-30))
    # per-integrator split of one eager batched step and one plain step
    def split(fn_list):
        out = {}
        for name, fn in fn_list:
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            out[name] = round(e0.elapsed_time(e1), 2)
        return out
    scene.clear_grads()
    split_b = split([("fwd", lambda: vs.render(api.TRN_PATH_TRACER, opts, launch=ln_f, out=img))] +
                    [(str(t), (lambda t=t: vs.render_grad(t, opts, dLdI, launch=ln_g[t]))) for t in terms])
    split_bd = split([("fwd", lambda: vs.render(api.TRN_PATH_TRACER, opts, out=img))] +
                     [(str(t), (lambda t=t: vs.render_grad(t, opts, dLdI))) for t in terms])
    pimgs = [sv.render(api.TRN_PATH_TRACER, opts) for sv in singles]
    pd = [torch.empty_like(im) for im in pimgs]
    for i, sv in enumerate(singles):
        sv.loss(pimgs[i], tgt_v[i], pd[i])
    split_p = split([("fwd", lambda: [sv.render(api.TRN_PATH_TRACER, opts) for sv in singles])] +
                    [(str(t), (lambda t=t: [sv.render_grad(t, opts, pd[i]) for i, sv in enumerate(singles)]))
                     for t in terms])
    scene.clear_grads()
    line = {"metric": "grad path-samples/sec", "value": units / (ms_batched / 1e3), "unit": "grad path-samples/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_batched, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": f"{nviews} views of the 1280-tri icosphere scene, res {res_choices}, "
                                   f"spp {sorted(set(spps))}, depth {D}, interior+primary+direct, one "
                                   "graph-captured launch per integrator",
                       "views": nviews, "samples_per_step": units},
            "plain_per_view": {"value": units / (ms_plain / 1e3), "ms_per_step": ms_plain},
            "batched_over_plain": ms_plain / ms_batched,
            "graph_vs_eager_grad_rel_l2": rel,
            "split_ms": {"batched": split_b, "batched_default_shape": split_bd, "plain": split_p},
            "launch": {"shape": best, "ms_by_shape": shape_ms,
                       "fwd": [ln_f.block, ln_f.blocks_per_sm, ln_f.chunk] if ln_f else "default",
                       **{str(t): ([ln_g[t].block, ln_g[t].blocks_per_sm, ln_g[t].chunk, ln_g[t].round_log2] if ln_g[t] else "default")
                          for t in terms}}}
    if not quiet:
        print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------------------
# inverse-rendering loop: 2M-triangle target, 16 views at 1024^2, depth 8,
# AQ-guided direct boundary, start = target + N(0, 0.02^2) per vertex, Adam
# lr 1e-3; a step = refit + batched forward + loss + batched adjoints + Adam
# ---------------------------------------------------------------------------
def run_icosphere(a, quiet: bool = False):
    """The icosphere configuration: 1280-triangle Lambertian icosphere over the
    ground quad, 256x256, 16 spp, depth 3, interior + primary + direct terms,
    gradient of the L2 image loss w.r.t. the sphere's 3-float translation.
    A step = translation upload + Scene::Configure + renderC + dL/dI + renderD
    of the three integrators + get_grads. `value` times it on resident
    inputs; `e2e` copies the translation from pinned host memory and the
    gradient and loss back every step."""
    from tensorray_b200 import api, scenes
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    res, spp, D = (64, 4, 3) if a.quick else (256, 16, 3)
    scene = api.Scene(scenes.config1_scene(res, res))
    scene.configure()
    dev = scene.device
    sphere = scene.shapes[0]
    its = [api.PathTracer(), api.PrimaryEdgeIntegrator(), api.DirectEdgeIntegrator()]
    opts = api.RenderOptions(1, D, spp, spp, spp, 0, 0)
    sphere.translation = torch.tensor([0.05, -0.03, 0.02])
    scene.configure()
    target = its[0].renderC(scene, api.RenderOptions(777, D, 4 * spp, 0, 0, 0, 0)).clone()
    t0 = torch.zeros(3, device=dev)
    units = res * res * spp * len(its)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def step(t):
        scene._translation[0].copy_(t)
        scene.configure()
        img = its[0].renderC(scene, opts)
        dLdI = img - target
        loss = 0.5 * (dLdI * dLdI).sum()
        scene.clear_grads()
        for it in its:
            it.renderD(scene, opts, dLdI)
        return loss, scene.get_grads(clear=True)["translation"][0]

    th = torch.zeros(3).pin_memory()
    gh = torch.empty(3).pin_memory()
    lh = torch.empty(1).pin_memory()

    def e2e_step():
        loss, g = step(th.to(dev, non_blocking=True))
        gh.copy_(g, non_blocking=True)
        lh.copy_(loss.reshape(1), non_blocking=True)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        tot = []
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot.append(e0.elapsed_time(e1))
        return sum(tot) / len(tot)

    ms = timed(lambda: step(t0))
    ms_e2e = timed(e2e_step)
    line = {"metric": "grad path-samples/sec", "value": units / (ms / 1e3), "unit": "grad path-samples/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": f"icosphere 1280 tris + ground, {res}x{res}, {spp} spp x 3 terms "
                                   f"(interior+primary+direct), depth {D}, grad: sphere translation",
                       "samples_per_step": units, "l2": "flushed between timed steps (256 MB write)"},
            "e2e": {"value": units / (ms_e2e / 1e3), "unit": "grad path-samples/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": 12, "d2h_bytes_per_step": 16}}
    if not quiet:
        print(json.dumps(line), flush=True)
    return line


def run_inverse(a):
    """The inverse-rendering loop. Under torchrun (N > 1) every rank holds a
    replica of the scene and renders its cost-balanced share of the views;
    the vertex gradient is summed with one NCCL all-reduce per step."""
    import torch.distributed as dist
    from tensorray_b200 import api, inverse, scenes
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    tris, nviews, res, D = (20_000, 4, 128, 4) if a.quick else (2_000_000, 16, 1024, 8)
    spp = 2 if a.quick else min(a.spp, 4)
    spec = scenes.served_scene(tris, seed=5)
    scene = api.Scene(spec)
    scene.configure()
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(nviews, 4.0, [res], seed=2)]
    topts = api.RenderOptions(1234, D, 16, 0, 0, 0, 0)
    targets = inverse.render_targets(scene, cams, [16] * nviews, topts).clone()
    raw = torch.as_tensor(spec.arrays()["positions"]).clone()
    nv = len(spec.meshes[0].positions)
    g = torch.Generator().manual_seed(7)
    raw[:nv] += 0.02 * torch.randn(nv, 3, generator=g)
    scene.set_vertex_positions(raw)
    scene.configure()
    opts = api.RenderOptions(0, D, spp, spp, spp, 0, 0)
    opts.g_direct, opts.g_direct_spp, opts.g_eps = True, 16, 0.01
    opts.g_direct_depth = a.guide_depth
    # the forward render keeps its interior path records for the interior
    # gradient of the same step (about 42 GB at 16 x 1024^2 x 4 spp, depth 8)
    inv = inverse.InverseRenderer(scene, cams, [spp] * nviews, targets, opts, lr=1e-3,
                                  path_cache_bytes=0 if a.no_path_cache else 64 << 30)
    units = inv.samples_per_step()
    if world > 1:
        u = torch.tensor([float(units)], device="cuda")
        dist.all_reduce(u)
        units = int(u.item())
    losses = []
    for _ in range(a.warmup):
        losses.append(float(inv.step().sum()))
    # one probe step per BVH policy (refit of the first topology vs rebuild),
    # timed per phase; the timed steps use the refit the workload names
    probe = {}
    for policy in ("refit", "rebuild"):
        inv.refit = policy == "refit"
        ph = {}
        losses.append(float(inv.step(phases=ph).sum()))
        probe[policy] = {k: round(v, 2) for k, v in inverse.phase_ms(ph).items()}
    inv.refit = True
    # work counters of one step per integrator (ray queries, shading vertices)
    import ctypes as C
    lib = scene._lib
    buf = (C.c_ulonglong * 16)()
    lib.trn_stats_enable(scene.handle, 1)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib.trn_stats_read(scene.handle, buf, 1, st)
    work = {}
    if inv.views is not None:
        inv.views.render(api.TRN_PATH_TRACER, inv.options, out=inv.image)
        lib.trn_stats_read(scene.handle, buf, 1, st)
        work["forward"] = dict(zip(CNT_NAMES, list(buf)[:10]))
        for i in inv.integrators:
            inv.views.render_grad(i, inv.options, inv.dLdI)
            lib.trn_stats_read(scene.handle, buf, 1, st)
            work[f"grad_{i}"] = dict(zip(CNT_NAMES, list(buf)[:10]))
    lib.trn_stats_enable(scene.handle, 0)
    scene.clear_grads()
    torch.cuda.synchronize()
    clk = Clocks(torch.cuda.current_device())
    clk.start()
    ms = []
    for _ in range(a.steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        l = inv.step()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        losses.append(float(l.sum()))
    clocks = clk.stop()
    mean_ms = sum(ms) / len(ms)
    if world > 1:
        t = torch.tensor([mean_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mean_ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return
    line = {"metric": "grad path-samples/sec", "value": units / (mean_ms / 1e3), "unit": "grad path-samples/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": mean_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded displaced sphere target, seeded vertex perturbation)",
            "config": {"workload": f"inverse rendering, {tris} tris target, {nviews} views {res}^2, {spp} spp x "
                                   f"3 terms (interior+primary+guided direct, guiding tree depth {a.guide_depth}), depth {D}, Adam lr 1e-3, "
                                   "LBVH refit per step; inputs larger than L2",
                       "samples_per_step": units,
                       "parallelism": f"views sharded by cost over {world} rank(s), gradient all-reduce"},
            "loss": {"first": losses[0], "last": losses[-1], "per_step": losses},
            "phases_ms": probe, "work": work, "clocks": clocks}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# served workload: Poisson arrivals of render+gradient requests over four
# resident scenes, continuous batching vs one request at a time
# ---------------------------------------------------------------------------
def run_serve(a, quiet: bool = False):
    from tensorray_b200 import api, scenes, serve
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rng = np.random.default_rng(0)
    sizes = {"s1k": 1_000, "s50k": 50_000, "s300k": 300_000, "s1m": 1_000_000}
    if a.quick:
        sizes = {"s1k": 1_000, "s20k": 20_000}
    world = {k: api.Scene(scenes.served_scene(n, seed=i)) for i, (k, n) in enumerate(sizes.items())}
    for sc in world.values():
        sc.configure()
    names = list(world)
    nreq = a.requests if not a.quick else 12
    rate = 200.0
    gaps = rng.exponential(1.0 / rate, size=nreq)
    arrivals = np.cumsum(gaps) - gaps[0]
    rmax = 256 if a.quick else 1024

    def make(i):
        name = names[int(rng.integers(len(names)))]
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        pos = tuple(float(x) for x in 4.0 * u)
        up = (0.0, 1.0, 0.0) if abs(u[1]) < 0.99 else (1.0, 0.0, 0.0)
        res = int(rng.integers(128, rmax + 1))
        spp = int(rng.integers(4, 65))
        depth = int(rng.integers(3, 7))
        cam = api.Camera(pos, (0.0, 0.0, 0.0), up, res, res, 45.0)
        tgt = torch.zeros(res * res, 3, device="cuda")
        return serve.RenderRequest(name, cam, spp, depth, tgt, seed=i)

    reqs = [make(i) for i in range(nreq)]
    budget = 120e9
    # the server's own view sets and every kernel warmed up before timing
    srv = serve.Server(world, hbm_budget_bytes=budget, chunk_spp=8)
    srv.warmup()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    t0 = time.perf_counter()
    stats = srv.run(reqs, list(arrivals))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    lat = [r.latency for r in stats.completed]
    samples = sum(r.samples() for r in stats.completed)
    # plain: one request at a time through the single-view API, no batching.
    # Like the server (and the reference's RenderD) its gradient call
    # re-traces the interior paths; a second pass lets the single-view calls
    # keep the forward's path records (not possible across the server's
    # interleaved chunks, whose forward completes before any gradient chunk)
    def one_at_a_time(path_cache: bool):
        for sc in world.values():
            sc.set_path_cache((16 << 30) if path_cache else 0)
        lat = []
        t1 = time.perf_counter()
        tq = 0.0
        for r, at in zip(reqs, arrivals):
            start = max(at, tq)
            sc = world[r.scene]
            e0 = time.perf_counter()
            opts = api.RenderOptions(r.seed, r.depth, r.spp, r.spp, r.spp, 0, 0)
            img = api.PathTracer().renderC(sc, opts, camera=r.camera)
            d = img.reshape(-1, 3) - r.target
            sc.clear_grads()
            for it in (api.PathTracer(), api.PrimaryEdgeIntegrator(), api.DirectEdgeIntegrator()):
                it.renderD(sc, opts, d.reshape(img.shape), camera=r.camera)
            sc.get_grads()
            torch.cuda.synchronize()
            dur = time.perf_counter() - e0
            tq = start + dur
            lat.append(tq - at)
        return lat, time.perf_counter() - t1

    plain_lat, plain_wall = one_at_a_time(False)
    cached_lat, cached_wall = one_at_a_time(True)
    line = {"metric": "grad path-samples/sec", "value": samples / wall, "unit": "grad path-samples/s", "n_gpus": 1,
            "steps": 1, "warmup": 1, "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes, Poisson arrivals)",
            "config": {"workload": f"{nreq} render+gradient requests at {rate:.0f} req/s over scenes "
                                   f"{list(sizes.values())} tris, res 128-{rmax}^2, spp 4-64, depth 3-6, "
                                   "interior+primary+direct, continuous batching, 120 GB budget"},
            "requests_per_s": len(stats.completed) / wall,
            "latency_s": {"p50": serve.percentile(lat, 50), "p99": serve.percentile(lat, 99),
                          "mean": float(np.mean(lat))},
            "plain_one_at_a_time": {"requests_per_s": nreq / plain_wall, "value": samples / plain_wall,
                                    "latency_s": {"p50": serve.percentile(plain_lat, 50),
                                                  "p99": serve.percentile(plain_lat, 99)}},
            "plain_one_at_a_time_path_cache": {"requests_per_s": nreq / cached_wall, "value": samples / cached_wall,
                                               "latency_s": {"p50": serve.percentile(cached_lat, 50),
                                                             "p99": serve.percentile(cached_lat, 99)}},
            "peak_request_bytes": stats.peak_bytes, "iterations": stats.iterations, "clocks": clk}
    if not quiet:
        print(json.dumps(line), flush=True)
    return line


if __name__ == "__main__":
    main()
