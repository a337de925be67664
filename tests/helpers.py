"""Shared helpers for the parity tests: scenes, oracle cameras, samples."""
import numpy as np
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes


def oracle_camera_from(cam: "api.Camera") -> dict:
    """The oracle consumes the library's float camera so primary rays are
    bit-identical; oracle.camera_matrices is checked against it separately."""
    return cam.matrices()


def sample_table(integrator: int, width: int, height: int, spp: int, D: int, seed: int) -> torch.Tensor:
    dims = api.sample_dims(integrator, D)
    slots = api.sample_slots(integrator, width, height, spp)
    return O.uniform_table(seed * 10 + integrator, dims, slots)


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a, b = a.double().reshape(-1), b.double().reshape(-1)
    den = max(float(b.norm()), 1e-30)
    return float((a - b).norm()) / den
