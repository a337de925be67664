"""tensorray_b200: B200-native path-space differentiable rendering.

Drop-in for TensorRay's integrator/scene execution layer: a C-ABI library
(include/trn.h, built from tensorray_b200/csrc for sm_100a) behind a Python
mirror of the reference's ``TensorRay`` module and its torch.autograd bridge.
"""
from .api import (BSDF, Camera, DirectEdgeIntegrator, IndirectEdgeIntegrator, Integrator, PathTracer,
                  PixelBoundaryIntegrator, PrimaryEdgeIntegrator, RenderOptions, Scene, Shape, ViewSet,
                  env_create, env_release, launch_config, sample_dims, sample_slots)
from . import scenes

__all__ = [
    "BSDF", "Camera", "DirectEdgeIntegrator", "IndirectEdgeIntegrator", "Integrator", "PathTracer",
    "PixelBoundaryIntegrator", "PrimaryEdgeIntegrator", "RenderOptions", "Scene", "Shape", "env_create",
    "env_release", "sample_dims", "sample_slots", "scenes", "ViewSet", "launch_config",
]
