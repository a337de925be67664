"""Optimiser side of the inverse-rendering loop on the CPU: the image losses
against golden vectors from the reference's own loss module
(pyTensorRay/loss.py:34-83; tests/golden/make_loss_goldens.py made them),
and LargeSteps (pyTensorRay/optimizer.py:149-180) against a float64 dense
restatement of the published method (Nicolet et al. 2021)."""
import os

import numpy as np
import pytest
import torch

from tensorray_b200 import loss as L
from tensorray_b200 import optim, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "loss_pyramid.pt")


@pytest.mark.parametrize("kind", ["l1", "l2", "pyramid_l1", "pyramid_l2"])
def test_losses_match_reference_goldens(kind):
    for case in torch.load(GOLDEN):
        img, tgt, w = case["img"], case["target"], case["weight"]
        target = L.build_pyramid(tgt) if kind.startswith("pyramid") else tgt
        assert len(L.build_pyramid(tgt)) == case["levels"]
        loss, grad = L.loss_and_grad(kind, img, target, w)
        ref_loss, ref_grad = case[kind]
        assert abs(float(loss) - ref_loss) <= 1e-6 * abs(ref_loss), (kind, float(loss), ref_loss)
        torch.testing.assert_close(grad, ref_grad, rtol=1e-6, atol=1e-7)


def _mesh():
    P, F = scenes.icosphere(2, 1.0)
    return torch.as_tensor(P, dtype=torch.float32), torch.as_tensor(F, dtype=torch.int64)


def _dense_M(F, n, lmbda):
    A = np.zeros((n, n))
    for a, b, c in F.tolist():
        for i, j in ((a, b), (b, c), (c, a)):
            A[i, j] = A[j, i] = 1.0
    return np.eye(n) + lmbda * (np.diag(A.sum(1)) - A)


def test_system_matrix_is_identity_plus_lambda_uniform_laplacian():
    V, F = _mesh()
    M = optim.SystemMatrix(F, V.shape[0], 0.37)
    ref = _dense_M(F, V.shape[0], 0.37)
    np.testing.assert_allclose(M.M.to_dense().double().numpy(), ref, rtol=1e-6, atol=1e-7)
    b = torch.randn(V.shape[0], 3, generator=torch.Generator().manual_seed(1))
    x = M.solve(b, tol=1e-7)
    np.testing.assert_allclose(x.double().numpy(), np.linalg.solve(ref, b.double().numpy()), rtol=1e-4, atol=1e-5)


def test_largesteps_step_matches_float64_restatement():
    V, F = _mesh()
    n, lmbda, lr, b1, b2 = V.shape[0], 2.0, 0.05, 0.9, 0.999
    g = torch.Generator().manual_seed(2)
    grads = [torch.randn(n, 3, generator=g) for _ in range(3)]
    Vp = V.clone().requires_grad_(True)
    opt = optim.LargeSteps(Vp, F, lr=lr, betas=(b1, b2), lmbda=lmbda, tol=1e-8)
    M = _dense_M(F, n, lmbda)
    u = M @ V.double().numpy()
    m1 = np.zeros_like(u)
    m2 = np.zeros_like(u)
    for t, gr in enumerate(grads, 1):
        Vp.grad = gr.clone()
        opt.step()
        gu = np.linalg.solve(M, gr.double().numpy())
        m1 = b1 * m1 + (1 - b1) * gu
        m2 = b2 * m2 + (1 - b2) * gu * gu
        u = u - lr * (m1 / (1 - b1 ** t)) / (1e-8 + np.sqrt((m2 / (1 - b2 ** t)).max()))
        np.testing.assert_allclose(Vp.detach().double().numpy(), np.linalg.solve(M, u), rtol=1e-4, atol=1e-5)


def test_largesteps_takes_large_smooth_steps():
    """Growing a unit sphere to a stretched ellipsoid under 0.5|V - T|^2: the
    smooth deformation is reached in few steps and the surface stays smooth
    (the neighbours of a vertex move together)."""
    V, F = _mesh()
    T = V * torch.tensor([1.3, 0.8, 1.1])
    Vp = V.clone().requires_grad_(True)
    opt = optim.LargeSteps(Vp, F, lr=0.02, lmbda=5.0)
    losses = []
    for _ in range(40):
        Vp.grad = (Vp.detach() - T)
        losses.append(float(0.5 * ((Vp.detach() - T) ** 2).sum()))
        opt.step()
    assert losses[-1] < 0.1 * losses[0], losses[::8]
    # no vertex strays from its neighbours: the Laplacian of the result is
    # as small as the target's
    M = optim.SystemMatrix(F, V.shape[0], 1.0)
    lap = lambda X: (M @ X - X).norm()
    assert float(lap(Vp.detach())) < 2.0 * float(lap(T))
