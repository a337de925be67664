"""torch.autograd bridge, mirroring pyTensorRay's RenderFunctionSingleView /
RenderFunction (pyTensorRay/renderer_single_view.py:40-85,
renderer_multi_view.py:40-98).

forward(V, texels) sets the scene parameters, re-configures the scene (the
reference's context.update + Scene::Configure) and returns the PathTracer
image. backward(dL/dI) replays the same seeds through renderD of the interior
integrator and every enabled edge integrator, finishes the geometry adjoint
and returns dL/dV and dL/dtexels. Tensors stay on the GPU (zero-copy), where
the reference copies images through host pointers (pyTensorRay/utils.py:60-80).
"""
from __future__ import annotations

import torch

from . import api


class RenderContext:
    def __init__(self, scene: api.Scene, options: api.RenderOptions, edge_integrators=None, camera=None):
        self.scene = scene
        self.options = options
        self.integrator = api.PathTracer()
        if edge_integrators is None:
            edge_integrators = []
            if options.sppe:
                edge_integrators.append(api.PrimaryEdgeIntegrator())
            if options.sppse0:
                edge_integrators.append(api.DirectEdgeIntegrator())
            if options.sppse1:
                edge_integrators.append(api.IndirectEdgeIntegrator())
            if options.sppe0:
                edge_integrators.append(api.PixelBoundaryIntegrator())
        self.edge_integrators = edge_integrators
        self.camera = camera


class RenderFunction(torch.autograd.Function):
    """image = render(V, texels); V are raw vertex positions [V, 3], texels
    the concatenated texture texels [N, 3] (or an empty tensor)."""

    @staticmethod
    def forward(ctx, V: torch.Tensor, texels: torch.Tensor, context: RenderContext):
        scene = context.scene
        scene.set_vertex_positions(V)
        if texels.numel():
            scene.set_texels(texels)
        scene.configure()
        ctx.context = context
        ctx.has_tex = texels.numel() > 0
        return context.integrator.renderC(scene, context.options, camera=context.camera)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        c = ctx.context
        scene = c.scene
        scene.clear_grads()
        c.integrator.renderD(scene, c.options, grad_out, camera=c.camera)
        for e in c.edge_integrators:
            e.renderD(scene, c.options, grad_out, camera=c.camera)
        g = scene.get_grads(clear=True)
        gv = torch.nan_to_num(g["positions"], nan=0.0)  # renderer_single_view.py:82
        gt = torch.nan_to_num(g["texels"], nan=0.0) if ctx.has_tex else None
        return gv, gt, None


def render(V: torch.Tensor, texels: torch.Tensor, context: RenderContext) -> torch.Tensor:
    return RenderFunction.apply(V, texels, context)
