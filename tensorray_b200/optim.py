"""LargeSteps optimiser of vertex positions, on the device.

The reference's LargeSteps (pyTensorRay/optimizer.py:149-180) wraps the
third-party `largesteps` package (PyPI; the reference's docs install it
without a pinned version, docs/python_intro.rst:34-35; it is not part of the
reference tree). This module restates the package's published method,
Nicolet, Jacobson and Jakob, "Large Steps in Inverse Rendering of Geometry",
ACM TOG 40(6), 2021:

* M = I + lambda * L, with L = D - A the combinatorial (uniform) Laplacian of
  the mesh's undirected edges (D the vertex degrees).
* The optimised variable is u = M V (to_differential). The positions are
  V = M^-1 u (from_differential).
* The gradient w.r.t. u is M^-1 dL/dV, since M is symmetric.
* The step is Adam with a uniform second moment: the bias-corrected first
  moment divided by 1e-8 + sqrt(max over all entries of the bias-corrected
  second moment) (the package's AdamUniform).

The package solves with a sparse Cholesky factorisation (cholespy) on the
host. Here M is symmetric positive definite and well conditioned (its
eigenvalues lie in [1, 1 + 2 lambda max_degree]), so both solves per step
run as Jacobi-preconditioned conjugate gradients on the device. They are
warm-started from the previous step's solution and stop at a relative
residual of `tol`.
"""
from __future__ import annotations

import warnings

import torch


def uniform_laplacian_edges(faces: torch.Tensor, num_vertices: int):
    """Unique undirected edges (i < j) of a triangle list and the degrees."""
    f = faces.long()
    e = torch.cat([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
    e = torch.stack([e.min(1).values, e.max(1).values], 1)
    e = torch.unique(e, dim=0)
    deg = torch.zeros(num_vertices, dtype=torch.float32, device=faces.device)
    ones = torch.ones(e.shape[0], dtype=torch.float32, device=faces.device)
    deg.index_add_(0, e[:, 0], ones)
    deg.index_add_(0, e[:, 1], ones)
    return e, deg


class SystemMatrix:
    """M = I + lambda (D - A) as a CSR matrix on the positions' device."""

    def __init__(self, faces: torch.Tensor, num_vertices: int, lmbda: float):
        e, deg = uniform_laplacian_edges(faces, num_vertices)
        n = num_vertices
        dev = faces.device
        rows = torch.cat([e[:, 0], e[:, 1], torch.arange(n, device=dev)])
        cols = torch.cat([e[:, 1], e[:, 0], torch.arange(n, device=dev)])
        vals = torch.cat([torch.full((2 * e.shape[0],), -float(lmbda), device=dev), 1.0 + float(lmbda) * deg])
        with warnings.catch_warnings():
            # torch flags its sparse CSR support as beta
            warnings.simplefilter("ignore", UserWarning)
            coo = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (n, n), check_invariants=True).coalesce()
            self.M = coo.to_sparse_csr()
        self.diag = 1.0 + float(lmbda) * deg
        self.n = n

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        return self.M @ x

    def solve(self, b: torch.Tensor, x0: torch.Tensor | None = None, tol: float = 1e-7,
              max_iter: int = 1000) -> torch.Tensor:
        """M x = b for every column of b by Jacobi-preconditioned conjugate
        gradients (columns are independent systems with the same matrix)."""
        x = torch.zeros_like(b) if x0 is None else x0.clone()
        inv_d = (1.0 / self.diag)[:, None]
        r = b - self.M @ x
        z = r * inv_d
        p = z.clone()
        rz = (r * z).sum(0)
        bnorm = b.norm(dim=0).clamp_min(1e-30)
        for _ in range(max_iter):
            if bool((r.norm(dim=0) <= tol * bnorm).all()):
                break
            Ap = self.M @ p
            alpha = rz / (p * Ap).sum(0).clamp_min(1e-30)
            x = x + p * alpha
            r = r - Ap * alpha
            z = r * inv_d
            rz_new = (r * z).sum(0)
            p = z + p * (rz_new / rz.clamp_min(1e-30))
            rz = rz_new
        return x


class AdamUniform:
    """Adam whose denominator is the square root of the largest bias-corrected
    second moment over all entries (the package's AdamUniform)."""

    def __init__(self, lr: float, betas=(0.9, 0.999), eps: float = 1e-8):
        self.lr, (self.b1, self.b2), self.eps = float(lr), betas, eps
        self.t = 0
        self.m1 = self.m2 = None

    def step(self, param: torch.Tensor, grad: torch.Tensor) -> None:
        if self.m1 is None:
            self.m1 = torch.zeros_like(param)
            self.m2 = torch.zeros_like(param)
        self.t += 1
        self.m1.mul_(self.b1).add_(grad, alpha=1.0 - self.b1)
        self.m2.mul_(self.b2).add_(grad.square(), alpha=1.0 - self.b2)
        m1 = self.m1 / (1.0 - self.b1 ** self.t)
        m2 = self.m2 / (1.0 - self.b2 ** self.t)
        param.sub_(m1 / (self.eps + m2.sqrt().max()), alpha=self.lr)


class LargeSteps(torch.optim.Optimizer):
    """LargeSteps(V, F, lr=0.1, betas=(0.9, 0.999), lmbda=0.1)
    (pyTensorRay/optimizer.py:149-180): V is the [n, 3] vertex-position
    parameter (its .grad is dL/dV), F the [m, 3] triangle indices. step()
    maps the gradient to the differential coordinates u = M V, takes one
    AdamUniform step on u and writes V = M^-1 u back into V."""

    def __init__(self, V: torch.Tensor, F: torch.Tensor, lr: float = 0.1, betas=(0.9, 0.999), lmbda: float = 0.1,
                 tol: float = 1e-7):
        if V.dim() != 2 or V.shape[1] != 3:
            raise ValueError("V must be an [n, 3] tensor of vertex positions")
        super().__init__([V], dict(lr=lr, betas=betas))
        self.V = V
        self.tol = tol
        self.M = SystemMatrix(F.to(V.device), V.shape[0], lmbda)
        self.u = (self.M @ V.detach().float()).contiguous()
        self.adam = AdamUniform(lr, betas)
        self._gu = None
        self._x = V.detach().float().clone()

    @torch.no_grad()
    def step(self, closure=None):
        loss = closure() if closure is not None else None
        if self.V.grad is None:
            return loss
        g = self.V.grad.detach().float()
        # dL/du = M^-T dL/dV (M is symmetric)
        self._gu = self.M.solve(g, self._gu, self.tol)
        self.adam.lr = self.param_groups[0]["lr"]
        self.adam.b1, self.adam.b2 = self.param_groups[0]["betas"]
        self.adam.step(self.u, self._gu)
        self._x = self.M.solve(self.u, self._x, self.tol)
        self.V.copy_(self._x.to(self.V.dtype))
        return loss
