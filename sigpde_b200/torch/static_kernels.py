"""Static kernels on path points, with the duck-typed protocol of
sigpde/torch/static_kernels.py:

    .pairwise(X, Y) -> (B, M, N)      X: (B, M, d), Y: (B, N, d)
    .gram(X, Y)     -> (A, B, M, N)   X: (A, M, d), Y: (B, N, d)

`LinearKernel` is recognised by the solvers and never materialised: its
increments <dx_i, dy_j> are contracted inside the CUDA wavefront kernel.
Every other kernel (RBF, L1-RBF, or any object with this protocol) goes
through the generic-increment entry points: torch builds the 4-term second
difference of its static Gram and the CUDA kernel solves the PDE.
"""
from __future__ import annotations

import torch


class LinearKernel:
    """k(x, y) = scale * <x, y>  (sigpde/torch/static_kernels.py:3-11)."""

    fused = True

    def __init__(self, scale=1.0):
        self.scale = scale

    def pairwise(self, X, Y):
        return self.scale * torch.matmul(X, Y.transpose(1, 2))

    def gram(self, X, Y):
        A, M, d = X.shape
        B, N, _ = Y.shape
        G = torch.matmul(X.reshape(A * M, d), Y.reshape(B * N, d).t())  # (A*M, B*N)
        return self.scale * G.reshape(A, M, B, N).permute(0, 2, 1, 3)


def _sq_dist(X, Y, batched: bool):
    """|x - y|^2 = |x|^2 + |y|^2 - 2 <x, y> over the point axes."""
    xn = (X * X).sum(-1)
    yn = (Y * Y).sum(-1)
    if batched:  # (B,M,d) x (B,N,d) -> (B,M,N)
        return xn[:, :, None] + yn[:, None, :] - 2.0 * torch.matmul(X, Y.transpose(1, 2))
    A, M, d = X.shape
    B, N, _ = Y.shape
    ip = torch.matmul(X.reshape(A * M, d), Y.reshape(B * N, d).t()).reshape(A, M, B, N).permute(0, 2, 1, 3)
    return xn[:, None, :, None] + yn[None, :, None, :] - 2.0 * ip


class RBFKernel:
    """k(x, y) = exp(-|x - y|^2 / sigma)  (sigpde/torch/static_kernels.py:13-36)."""

    fused = False

    def __init__(self, sigma=1.0):
        self.sigma = sigma

    def pairwise(self, X, Y):
        return torch.exp(-_sq_dist(X, Y, True) / self.sigma)

    def gram(self, X, Y):
        return torch.exp(-_sq_dist(X, Y, False) / self.sigma)


class L1RBFKernel:
    """k(x, y) = exp(-|x - y|_1 / sigma)  (sigpde/torch/static_kernels.py:38-53)."""

    fused = False

    def __init__(self, sigma=1.0):
        self.sigma = sigma

    def pairwise(self, X, Y):
        return torch.exp(-torch.cdist(X, Y, p=1) / self.sigma)

    def gram(self, X, Y):
        A, M, d = X.shape
        B, N, _ = Y.shape
        dist = torch.cdist(X.reshape(1, A * M, d), Y.reshape(1, B * N, d), p=1)[0]
        return torch.exp(-dist.reshape(A, M, B, N).permute(0, 2, 1, 3) / self.sigma)
