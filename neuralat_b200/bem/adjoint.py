"""Differentiable listener pressures with a hand-written adjoint.

``listener_pressure(vertices, neumann, triangles, points, k)`` returns
p = -S g + D u with (1/2 M - K) u = -V g (the reference's CBIE followed by
``boundary2potential``, src/bem/solver.py:97-104,140-147) as a
``torch.autograd.Function``.  Its backward is written by hand:

    lambda   = (1/2 M - K)^{-H} D^H pbar            adjoint GMRES
    dL/dg*   = -S^H pbar - V^H lambda
    dL/dx    = Re[-pbar^H dS g + pbar^H dD u - lambda^H dV g
                  - 1/2 lambda^H dM u + lambda^H dK u]

The vertex gradient is one kernel-derivative pass over all triangle pairs,
touching pairs (Sauter-Schwab) and listener-triangle pairs
(``bem_vertex_gradient``): derivative matrices are never formed.  With
``store_matrices=False`` the forward keeps only u and V, A are re-assembled in
the backward (memory for time).
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib as L
from .solver import BEM_Solver, _stream, _vp, cmatmul, gmres


def cmatmul_adjoint(A: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
    """Y = A^H X (complex64) on the library's kernel."""
    n = A.shape[0]
    Xc = X.reshape(n, -1).contiguous()
    Y = torch.empty_like(Xc)
    with torch.cuda.device(A.device):
        L.check(L.lib().bem_cmatmul_adjoint(_vp(A), n, _vp(Xc), Xc.shape[1], _vp(Y), _stream(A.device)),
                "bem_cmatmul_adjoint")
    return Y.reshape(X.shape)


def conj_transpose(A: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(A)
    with torch.cuda.device(A.device):
        L.check(L.lib().bem_conj_transpose(_vp(A), A.shape[0], _vp(out), _stream(A.device)), "bem_conj_transpose")
    return out


class _ListenerPressure(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vertices, neumann, triangles, points, k, precision, rtol, store_matrices):
        solver = BEM_Solver(vertices.detach().float().contiguous(), triangles)
        g = neumann.detach().to(torch.complex64).contiguous()
        pts = points.detach().float().contiguous()
        V, A = solver.assemble_vk(k)
        u = gmres(A, -cmatmul(V, g), rtol=rtol, precision=precision)
        p = solver.boundary2potential(k, g, u, pts)
        ctx.solver, ctx.k, ctx.pts, ctx.precision, ctx.rtol = solver, float(k), pts, precision, rtol
        ctx.g, ctx.u = g, u
        ctx.V, ctx.A = (V, A) if store_matrices else (None, None)
        return p

    @staticmethod
    def backward(ctx, pbar):
        s, k, pts = ctx.solver, ctx.k, ctx.pts
        pbar = pbar.to(torch.complex64).contiguous()
        V, A = ctx.V, ctx.A
        if V is None:
            V, A = s.assemble_vk(k)
        lib = L.lib()
        nv = s.geometry.nv
        sh = torch.empty(nv, dtype=torch.complex64, device=pbar.device)
        dh = torch.empty_like(sh)
        with torch.cuda.device(pbar.device):
            L.check(lib.bem_boundary2potential_adjoint(s.geometry.ptr, _vp(pts), int(pts.shape[0]), float(k),
                                                       _vp(pbar), _vp(sh), _vp(dh), _stream(pbar.device)),
                    "bem_boundary2potential_adjoint")
        lam = gmres(conj_transpose(A), dh, rtol=min(ctx.rtol, 1e-7), precision=ctx.precision)
        grad_x = grad_g = None
        if ctx.needs_input_grad[1]:
            grad_g = -sh - cmatmul_adjoint(V, lam)
        if ctx.needs_input_grad[0]:
            gx = torch.empty((nv, 3), dtype=torch.float64, device=pbar.device)
            with torch.cuda.device(pbar.device):
                L.check(lib.bem_vertex_gradient(s.geometry.ptr, float(k), _vp(lam), _vp(ctx.g), _vp(ctx.u), _vp(pts),
                                                int(pts.shape[0]), _vp(pbar), _vp(gx), _stream(pbar.device)),
                        "bem_vertex_gradient")
            grad_x = gx.to(torch.float32)
        return grad_x, grad_g, None, None, None, None, None, None


def listener_pressure(vertices: torch.Tensor, neumann: torch.Tensor, triangles: torch.Tensor, points: torch.Tensor,
                      k: float, *, precision: str = "fp16x3", rtol: float = 1e-7, store_matrices: bool = True):
    """Listener pressures (P,) complex64, differentiable w.r.t. ``vertices``
    (float32 (N,3)) and ``neumann`` (complex64 (N,))."""
    return _ListenerPressure.apply(vertices, neumann, triangles, points, float(k), precision, rtol, store_matrices)
