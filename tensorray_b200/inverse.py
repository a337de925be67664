"""Multi-view inverse rendering loop on the GPU.

The reference optimises scene parameters from Python: per view it calls
RenderFunction (forward renderC, backward renderD of every integrator,
pyTensorRay/renderer_multi_view.py:40-98), reads the gradients through the
parameter manager (pyTensorRay/parameter_manager.py:36-101) and steps a torch
optimiser. Here one step is: new vertex positions -> geometry chain + LBVH
refit (Scene::Update, Scene.cpp:535-546) -> one batched forward launch over
all views -> per-view loss and dL/dI in one launch -> one batched adjoint
launch per integrator -> geometry adjoint -> Adam on the device. Nothing
leaves the GPU inside a step; the loss stays a device tensor until read.
"""
from __future__ import annotations

import torch

from . import api
from . import dist as trd
from . import loss as trl
from . import optim as tro


class InverseRenderer:
    """Optimise the raw vertex positions of a scene against target images.

    integrators: ids of the terms whose gradients drive the step (the forward
    image is always the interior path tracer's). options: one RenderOptions for
    every term (its seed advances each step so sample noise decorrelates).
    path_cache_bytes: bound on the interior path records the forward render
    keeps for the interior gradient of the same step (0 = re-trace them).

    loss: "l2" (0.5 |I - T|^2 per view in one launch, the default), or "l1",
    "pyramid_l1", "pyramid_l2" (pyTensorRay/loss.py:41-83, evaluated per view
    on the device by tensorray_b200.loss). optimizer: "adam" (torch Adam, the
    default) or "largesteps" (tensorray_b200.optim.LargeSteps,
    pyTensorRay/optimizer.py:149-180, with `lmbda`). shapes: indices of the
    meshes whose vertices are optimised (None: every vertex). The reference
    optimises one shape's vertices (DiffAllVertexPos, Primitive.cpp:385-388);
    LargeSteps needs this, since its uniform second moment would otherwise be
    set by the largest gradient anywhere in the scene.

    With an initialised torch.distributed process group (one process per GPU,
    each with its own replica of the scene), the views are split over the
    ranks by cost (trd.ViewShard); each rank renders its views, the vertex
    gradient is summed over ranks with one all-reduce before the identical
    Adam update on every rank, and step() returns the losses of all views."""

    def __init__(self, scene: api.Scene, cameras: list, spps: list, targets: torch.Tensor,
                 options: api.RenderOptions, integrators=(api.TRN_PATH_TRACER, api.TRN_PRIMARY_EDGE,
                                                          api.TRN_DIRECT_EDGE),
                 lr: float = 1e-3, refit: bool = True, launch=None, path_cache_bytes: int = 0, group=None,
                 loss: str = "l2", optimizer: str = "adam", lmbda: float = 0.1, shapes=None):
        if loss not in ("l2",) + tuple(trl.LOSSES):
            raise ValueError(f"unknown loss {loss!r}")
        self.scene = scene
        self.loss_kind = loss
        self.group = group
        npix_all = sum(c.width * c.height for c in cameras)
        if targets.numel() != 3 * npix_all:
            raise RuntimeError("targets must hold npix x 3 values (all views concatenated)")
        self.shard = trd.ViewShard.of(cameras, spps, options.max_bounces, group)
        offs = [0]
        for c in cameras:
            offs.append(offs[-1] + c.width * c.height)
        tg = targets.reshape(-1, 3).to(scene.device, torch.float32)
        self.targets = torch.cat([tg[offs[i]:offs[i + 1]] for i in self.shard.local]).contiguous() \
            if self.shard.local else tg[:0].contiguous()
        # every view keeps its global index as its seed: the sharded run draws
        # the samples of the unsharded one
        self.views = api.ViewSet(scene, self.shard.pick(cameras), self.shard.pick(spps), seeds=list(self.shard.local)) \
            if self.shard.local else None
        if path_cache_bytes and self.views is not None:
            self.views.set_path_cache(path_cache_bytes)
        self.options = options
        self.integrators = tuple(integrators)
        self.refit = refit
        self.launch = launch
        dev = scene.device
        self.x = scene._raw_positions.detach().clone().requires_grad_(True)
        # the optimised vertices: all, or those of the chosen meshes
        self._sel = None
        self._xs = self.x
        faces = None
        if shapes is not None:
            meshes = scene.spec.meshes
            starts = [0]
            for m in meshes:
                starts.append(starts[-1] + len(m.positions))
            sel, fl, base = [], [], 0
            for i in shapes:
                sel.append(torch.arange(starts[i], starts[i + 1]))
                fl.append(torch.as_tensor(meshes[i].faces, dtype=torch.int64) + base)
                base += starts[i + 1] - starts[i]
            self._sel = torch.cat(sel).to(dev)
            faces = torch.cat(fl).to(dev)
            self._xs = self.x.detach()[self._sel].clone().requires_grad_(True)
        if optimizer == "adam":
            self.opt = torch.optim.Adam([self._xs], lr=lr)
        elif optimizer == "largesteps":
            if faces is None:
                faces = torch.as_tensor(scene.spec.arrays()["indices"], device=dev).reshape(-1, 3)
            self.opt = tro.LargeSteps(self._xs, faces, lr=lr, lmbda=lmbda)
        else:
            raise ValueError(f"unknown optimizer {optimizer!r}")
        # target pyramids of the pyramid losses, per local view
        self._target_levels = None
        if loss.startswith("pyramid"):
            self._target_levels = [trl.build_pyramid(self._view(self.targets, i)) for i in range(len(self.shard.local))]
        npix = self.views.npix if self.views is not None else 0
        self.image = torch.empty(npix, 3, device=dev)
        self.dLdI = torch.empty(npix, 3, device=dev)
        self.loss = torch.zeros(len(cameras), device=dev)
        self.steps = 0

    def _view(self, flat: torch.Tensor, i: int) -> torch.Tensor:
        """Local view i of a concatenated [npix, 3] buffer as (H, W, 3)."""
        c = self.views.cameras[i]
        off = self.views.offsets[i]
        return flat[off:off + c.width * c.height].view(c.height, c.width, 3)

    def _loss_and_dLdI(self) -> torch.Tensor:
        if self.loss_kind == "l2":
            return self.views.loss(self.image, self.targets, self.dLdI)
        losses = []
        for i in range(len(self.views.cameras)):
            tgt = self._target_levels[i] if self._target_levels is not None else self._view(self.targets, i)
            l, g = trl.loss_and_grad(self.loss_kind, self._view(self.image, i), tgt)
            self._view(self.dLdI, i).copy_(g)
            losses.append(l)
        return torch.stack(losses)

    def samples_per_step(self) -> int:
        """Grad path-samples of one step on this rank: its views' W*H*spp per term."""
        if self.views is None:
            return 0
        n = sum(c.width * c.height * s for c, s in zip(self.views.cameras, self.views.spps))
        return n * len(self.integrators)

    def step(self, phases: dict | None = None) -> torch.Tensor:
        """One optimisation step; returns the per-view losses (device tensor)
        of the parameters before the update. With `phases` (a dict), CUDA
        events around each phase are stored there under its name."""
        def mark(name):
            if phases is not None:
                ev = torch.cuda.Event(enable_timing=True)
                ev.record()
                phases.setdefault("_order", []).append((name, ev))

        sc = self.scene
        mark("start")
        sc.set_vertex_positions(self.x.detach())
        sc.configure(refit=self.refit and self.steps > 0)
        mark("configure")
        self.options.seed = self.steps
        sc.clear_grads()
        if self.views is not None:
            self.views.render(api.TRN_PATH_TRACER, self.options, launch=self.launch, out=self.image)
            mark("forward")
            local_loss = self._loss_and_dLdI()
            for i in self.integrators:
                self.views.render_grad(i, self.options, self.dLdI, launch=self.launch)
                mark(f"grad_{i}")
        else:
            local_loss = torch.zeros(0, device=sc.device)
        g = sc.get_grads()["positions"]
        # non-finite entries are zeroed, as the reference's multi-view bridge
        # does (pyTensorRay/renderer_multi_view.py:94)
        g = torch.nan_to_num(g, nan=0.0, posinf=0.0, neginf=0.0)
        self.x.grad = trd.allreduce_grads({"positions": g}, self.group)["positions"]
        self.loss = trd.gather_view_values(self.shard, local_loss, self.group)
        mark("exchange")
        if self._sel is None:
            self.opt.step()
        else:
            self._xs.grad = self.x.grad[self._sel]
            self.opt.step()
            with torch.no_grad():
                self.x[self._sel] = self._xs.detach()
        mark("update")
        self.steps += 1
        return self.loss


def phase_ms(phases: dict) -> dict:
    """Milliseconds between consecutive marks recorded by step(phases=...)."""
    torch.cuda.synchronize()
    order = phases.get("_order", [])
    return {name: order[i - 1][1].elapsed_time(ev) for i, (name, ev) in enumerate(order) if i > 0}


def render_targets(scene: api.Scene, cameras: list, spps: list, options: api.RenderOptions,
                   launch=None) -> torch.Tensor:
    """Forward images of all views (concatenated [npix, 3]) for the current
    scene parameters, e.g. the targets of an inverse-rendering run."""
    vs = api.ViewSet(scene, cameras, spps)
    return vs.render(api.TRN_PATH_TRACER, options, launch=launch)
