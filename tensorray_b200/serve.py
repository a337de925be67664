"""Continuous-batching render + gradient server.

Requests (scene, camera, spp, depth, target image) arrive over time. The
server keeps every scene's BVH, geometry and textures resident, admits a
request when its device buffers fit in the HBM budget, and advances all
admitted requests in batches. Each iteration issues, per scene, one batched
launch for the next forward chunk of every request still rendering and one
batched launch per gradient term for every request in its gradient phase:
iteration-level continuous batching, so a request that arrives while others
are on the GPU joins at the next iteration instead of waiting for them to
finish. An iteration carries at most `iter_samples` path samples, filled
shortest-remaining-work first (SRPT), so small requests are not held behind
large ones while the GPU stays saturated. Every scene has its own CUDA stream,
so launches of different scenes
overlap on the device. A request's samples depend only on its own seed and
chunk offsets, never on the batch it shares, so its result is the same alone
and in the mix (up to float atomic ordering).

The reference has no serving mode; its closest pattern is the per-view loop
of pyTensorRay/renderer_multi_view.py:53-61.
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field

import torch

from . import api
from ._abi import (TRN_DIRECT_EDGE, TRN_INDIRECT_EDGE, TRN_PATH_TRACER, TRN_PIXEL_EDGE, TRN_PRIMARY_EDGE,
                   TrnView)

PHASE_FWD, PHASE_GRAD, PHASE_FINISH, PHASE_DONE = 0, 1, 2, 3

# the gradient terms a request may ask for (RenderRequest.terms): the
# interior path tracer and the four boundary terms
ALL_TERMS = (TRN_PATH_TRACER, TRN_PRIMARY_EDGE, TRN_DIRECT_EDGE, TRN_INDIRECT_EDGE, TRN_PIXEL_EDGE)

# Device bytes a gradient view set holds for the queues of the split
# integrator kernels (one round: 16M boundary samples, at most about 312 bytes
# each at depth <= 8) and for the boundary set-up's run order (16 bytes per
# slot plus the sort's temporary storage). Forward view sets hold none.
VIEWSET_QUEUE_BYTES = 5_600_000_000


@dataclass
class RenderRequest:
    scene: str
    camera: api.Camera
    spp: int
    depth: int
    target: torch.Tensor                      # (H*W, 3) on the device
    seed: int = 0
    terms: tuple = (TRN_PATH_TRACER, TRN_PRIMARY_EDGE, TRN_DIRECT_EDGE)
    arrival: float | None = None
    rid: int = -1
    # results / state (filled by the server)
    image: torch.Tensor | None = None
    dLdI: torch.Tensor | None = None
    grad_positions: torch.Tensor | None = None
    grad_vertex_normals: torch.Tensor | None = None
    loss: torch.Tensor | None = None
    phase: int = PHASE_FWD
    chunk: int = 0
    nbytes: int = 0
    t_admit: float | None = None
    t_done: float | None = None
    done_event: object = None

    @property
    def latency(self) -> float | None:
        return None if self.t_done is None else self.t_done - self.arrival

    def samples(self) -> int:
        return self.camera.width * self.camera.height * self.spp * len(self.terms)


@dataclass
class ServerStats:
    completed: list = field(default_factory=list)
    peak_bytes: int = 0
    iterations: int = 0


class Server:
    def __init__(self, scenes: dict, hbm_budget_bytes: float = 120e9, chunk_spp: int = 8, max_active: int = 256,
                 clock=time.perf_counter, iter_samples: int = 1 << 25, max_depth: int = 8):
        self.scenes = scenes
        # gradient view sets reserve their round buffers for this depth when
        # created (deeper requests still run; their first batch grows them)
        self.max_depth = int(max_depth)
        # the gradient view set of every scene holds one round of queues
        self.reserve = len(scenes) * VIEWSET_QUEUE_BYTES
        self.budget = int(hbm_budget_bytes) - self.reserve
        self.chunk_spp = chunk_spp
        self.iter_samples = int(iter_samples)
        self.max_active = max_active
        self.clock = clock
        self.streams = {k: torch.cuda.Stream() for k in scenes}
        self.vsets: dict = {}
        self.pending: deque = deque()
        self.active: list = []
        self.used = 0
        self.stats = ServerStats()
        self._next_id = 0
        for sc in scenes.values():
            sc._ensure()

    # -- memory model --------------------------------------------------------------
    def request_bytes(self, req: RenderRequest) -> int:
        sc = self.scenes[req.scene]
        npix = req.camera.width * req.camera.height
        # image + dL/dI + two gradient buffers + this view's silhouette workspace
        return 4 * (2 * 3 * npix + 2 * 3 * sc.num_vertices + 2 * sc.num_edges + 1)

    # -- API --------------------------------------------------------------------------
    def submit(self, req: RenderRequest) -> RenderRequest:
        if req.arrival is None:
            req.arrival = self.clock()
        req.rid = self._next_id
        self._next_id += 1
        req.nbytes = self.request_bytes(req)
        if req.nbytes > self.budget:
            raise RuntimeError(f"request {req.rid} needs {req.nbytes} bytes, above the HBM budget {self.budget}")
        self.pending.append(req)
        return req

    def warmup(self) -> None:
        """Serve one small request per scene, so that this server's view sets
        exist (with their round buffers reserved) and every kernel has run
        once before the first real request; then reset the statistics."""
        for name, sc in self.scenes.items():
            cam = api.Camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 64, 64, 45.0)
            self.submit(RenderRequest(name, cam, self.chunk_spp, 3, torch.zeros(64 * 64, 3, device=sc.device),
                                      seed=999))
        while not self.idle():
            self.step()
        torch.cuda.synchronize()
        self.stats = ServerStats()
        self._next_id = 0

    def idle(self) -> bool:
        return not self.pending and not self.active

    def _remaining(self, r: RenderRequest) -> int:
        """Path samples a request still needs (forward chunks + gradient chunks)."""
        npix = r.camera.width * r.camera.height
        per_chunk = npix * self.chunk_spp
        n = self._nchunks(r)
        if r.phase == PHASE_FWD:
            return per_chunk * ((n - r.chunk) + n * len(r.terms))
        if r.phase == PHASE_GRAD:
            return per_chunk * (n - r.chunk) * len(r.terms)
        return 0

    def _chunk_samples(self, r: RenderRequest) -> int:
        npix = r.camera.width * r.camera.height
        k0 = r.chunk * self.chunk_spp
        spp = min(self.chunk_spp, r.spp - k0)
        return npix * spp * (1 if r.phase == PHASE_FWD else len(r.terms))

    def _select(self) -> list:
        """Requests that advance this iteration: shortest remaining work first,
        until the iteration's sample budget is used (at least one request)."""
        runnable = [r for r in self.active if r.phase in (PHASE_FWD, PHASE_GRAD)]
        runnable.sort(key=lambda r: (self._remaining(r), r.arrival, r.rid))
        chosen, used = [], 0
        for r in runnable:
            cs = self._chunk_samples(r)
            if chosen and used + cs > self.iter_samples:
                continue
            chosen.append(r)
            used += cs
        return chosen

    def step(self) -> None:
        """One scheduling iteration: admit, launch one chunk for each selected
        request, retire."""
        self._admit()
        chosen = set(id(r) for r in self._select())
        for name, sc in self.scenes.items():
            reqs = [r for r in self.active if r.scene == name and id(r) in chosen]
            if not reqs:
                continue
            with torch.cuda.stream(self.streams[name]):
                self._forward(name, sc, [r for r in reqs if r.phase == PHASE_FWD])
                self._gradient(name, sc, [r for r in reqs if r.phase == PHASE_GRAD])
        self._retire()
        self.stats.iterations += 1

    def run(self, requests: list, arrival_times: list | None = None) -> ServerStats:
        """Feed requests at their (relative) arrival times and serve until all
        are done. Returns the completed requests with latencies."""
        t0 = self.clock()
        order = list(zip(arrival_times or [0.0] * len(requests), requests))
        order.sort(key=lambda x: x[0])
        i = 0
        while i < len(order) or not self.idle():
            now = self.clock() - t0
            while i < len(order) and order[i][0] <= now:
                order[i][1].arrival = t0 + order[i][0]
                self.submit(order[i][1])
                i += 1
            if self.idle():
                time.sleep(max(0.0, min(0.001, order[i][0] - now)) if i < len(order) else 0.0)
                continue
            self.step()
        return self.stats

    # -- internals ----------------------------------------------------------------------
    def _admit(self) -> None:
        while self.pending and len(self.active) < self.max_active:
            req = self.pending[0]
            if self.used + req.nbytes > self.budget:
                break
            self.pending.popleft()
            sc = self.scenes[req.scene]
            npix = req.camera.width * req.camera.height
            with torch.cuda.stream(self.streams[req.scene]):
                d = sc.device
                req.image = torch.zeros(npix, 3, device=d)
                req.dLdI = torch.empty(npix, 3, device=d)
                req.grad_positions = torch.zeros(sc.num_vertices, 3, device=d)
                req.grad_vertex_normals = torch.zeros(sc.num_vertices, 3, device=d)
            req.phase, req.chunk = PHASE_FWD, 0
            req.t_admit = self.clock()
            self.used += req.nbytes
            self.stats.peak_bytes = max(self.stats.peak_bytes, self.used)
            self.active.append(req)

    def _nchunks(self, req: RenderRequest) -> int:
        return (req.spp + self.chunk_spp - 1) // self.chunk_spp

    def _views(self, reqs: list, grad: bool):
        arr = (TrnView * len(reqs))()
        spps = []
        for i, r in enumerate(reqs):
            c = r.camera
            k0 = r.chunk * self.chunk_spp
            spp = min(self.chunk_spp, r.spp - k0)
            spps.append(spp)
            arr[i] = TrnView(c.c, spp, int(r.seed), -1, k0 * c.width * c.height, 1.0 / r.spp, int(r.depth),
                             C.c_void_p(r.grad_positions.data_ptr()) if grad else None,
                             C.c_void_p(r.grad_vertex_normals.data_ptr()) if grad else None, None,
                             None if grad else C.c_void_p(r.image.data_ptr()),
                             C.c_void_p(r.dLdI.data_ptr()) if grad else None)
        return arr, spps

    def _viewset(self, name: str, phase: int, reqs: list, arr, spps):
        key = (name, phase)
        cams = [r.camera for r in reqs]
        vs = self.vsets.get(key)
        if vs is None:
            vs = api.ViewSet(self.scenes[name], cams, spps, views=arr)
            if phase != PHASE_FWD:
                vs.reserve(self.max_depth)
            self.vsets[key] = vs
        else:
            vs.update(cams, spps, arr)
        return vs

    def _forward(self, name: str, sc: api.Scene, reqs: list) -> None:
        if not reqs:
            return
        arr, spps = self._views(reqs, grad=False)
        vs = self._viewset(name, PHASE_FWD, reqs, arr, spps)
        vs.render(TRN_PATH_TRACER, api.RenderOptions(0, 0, 0, 0, 0, 0, 0), out=False)
        for r in reqs:
            r.chunk += 1
            if r.chunk >= self._nchunks(r):
                # loss 0.5 |I - T|^2 and dL/dI (pyTensorRay/loss.py:34-38)
                torch.sub(r.image, r.target, out=r.dLdI)
                r.loss = 0.5 * (r.dLdI * r.dLdI).sum()
                r.phase, r.chunk = PHASE_GRAD, 0

    def _gradient(self, name: str, sc: api.Scene, reqs: list) -> None:
        if not reqs:
            return
        groups: dict = {}
        for r in reqs:
            groups.setdefault(tuple(r.terms), []).append(r)
        for gi, (terms, grp) in enumerate(sorted(groups.items())):
            arr, spps = self._views(grp, grad=True)
            vs = self._viewset(name, (PHASE_GRAD, gi), grp, arr, spps)
            for t in terms:
                vs.render_grad(t, api.RenderOptions(0, 0, 0, 0, 0, 0, 0), None)
        for r in reqs:
            r.chunk += 1
            if r.chunk >= self._nchunks(r):
                sc.finalize_grads(r.grad_positions, r.grad_vertex_normals)
                r.done_event = torch.cuda.Event()
                r.done_event.record()
                r.phase = PHASE_FINISH

    def _retire(self) -> None:
        keep = []
        for r in self.active:
            if r.phase == PHASE_FINISH and r.done_event.query():
                r.t_done = self.clock()
                r.phase = PHASE_DONE
                self.used -= r.nbytes
                r.dLdI = None
                r.grad_vertex_normals = None
                self.stats.completed.append(r)
            else:
                keep.append(r)
        self.active = keep


def percentile(xs: list, q: float) -> float:
    if not xs:
        return float("nan")
    ys = sorted(xs)
    k = min(len(ys) - 1, max(0, int(round(q / 100.0 * (len(ys) - 1)))))
    return ys[k]
