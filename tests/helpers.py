"""Shared helpers for the parity tests: scenes, oracle cameras, samples."""
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


# Parity tolerance of the CUDA path against the oracle on the same samples:
# images per pixel and channel, gradients as relative L2 and as the largest
# element error relative to the largest element.
PARITY_TOL = 1e-4
# measured errors, printed in the terminal summary (tests/conftest.py)
PARITY_LOG: list = []


def assert_image_parity(img_gpu: torch.Tensor, img_oracle: torch.Tensor, label: str) -> None:
    """Every pixel channel within PARITY_TOL relative (plus a 1e-7 floor for
    pixels that are black up to float noise)."""
    a = img_gpu.reshape(-1, 3).cpu().double()
    b = img_oracle.reshape(-1, 3).cpu().double()
    assert float(b.abs().sum()) > 0, f"{label}: the oracle image is black"
    err = (a - b).abs()
    scale = torch.maximum(a.abs(), b.abs())
    rel = float((err / (scale + 1e-7)).max())
    bad = int((err > PARITY_TOL * scale + 1e-7).any(-1).sum())
    PARITY_LOG.append((label, "image max rel", rel, f"{bad} of {a.shape[0]} pixels beyond tolerance"))
    assert bad == 0, f"{label}: {bad} pixels beyond {PARITY_TOL} relative (max {rel:.2e})"


def assert_grad_parity(g_gpu: torch.Tensor, g_oracle: torch.Tensor, label: str) -> None:
    a = g_gpu.detach().cpu().double().reshape(-1)
    b = g_oracle.detach().cpu().double().reshape(-1)
    assert float(b.abs().sum()) > 0, f"{label}: the oracle gradient is zero"
    l2 = rel_l2(a, b)
    mx = float((a - b).abs().max()) / float(b.abs().max())
    PARITY_LOG.append((label, "grad rel L2", l2, f"max elem err / max elem {mx:.2e}"))
    assert l2 <= PARITY_TOL, f"{label}: relative L2 {l2:.2e}"
    assert mx <= PARITY_TOL, f"{label}: largest element error {mx:.2e} of the largest element"
