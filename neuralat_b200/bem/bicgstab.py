"""BiCGSTAB kept for parity with the reference's solver (src/bem/BiCGSTAB.py:5-107).

Same iteration as the reference -- van der Vorst's BiCGSTAB with the
reference's *unconjugated* inner products for rho, alpha and omega
(BiCGSTAB.py:60,69,74), the stopping test ||r||^2 < tol ||b||^2 or
||r||^2 < atol (BiCGSTAB.py:40-41,53-54), and the rho == 0 exit (:103) -- so
that ``solve_linear_equation(..., solver="bicgstab")`` reproduces the
reference's iterates.  The operator is whatever callable is passed (the
drop-in wraps matrices with the library's complex matmul).  The default
solver of this package is the device-resident GMRES instead.
"""
from __future__ import annotations

import torch


class BiCGSTAB:
    def __init__(self, Ax_gen, device="cuda"):
        self.Ax_gen = Ax_gen
        self.device = device

    def _residual(self, x):
        r = self.b - self.Ax_gen(x)
        rr = torch.vdot(r, r).real
        return bool(rr < self.residual_tol or rr < self.atol), r

    def solve(self, b, x=None, nsteps=None, tol=1e-10, atol=1e-16):
        self.b = b.clone().detach()
        self.x = torch.zeros_like(b) if x is None else x
        self.residual_tol = tol * torch.vdot(self.b, self.b).real
        self.atol = torch.tensor(atol, device=b.device)
        steps = b.shape[0] if nsteps is None else nsteps
        self.iterations = 0
        done, r = self._residual(self.x)
        if done:
            return self.x
        r_hat = r.clone()
        rho_prev = torch.tensor(1.0, dtype=b.dtype, device=b.device)
        alpha = torch.tensor(1.0, dtype=b.dtype, device=b.device)
        omega = torch.tensor(1.0, dtype=b.dtype, device=b.device)
        v = torch.zeros_like(b)
        p = torch.zeros_like(b)
        while steps:
            rho = torch.dot(r, r_hat)
            beta = (rho / rho_prev) * (alpha / omega)
            rho_prev = rho
            p = r + beta * (p - omega * v)
            v = self.Ax_gen(p)
            alpha = rho_prev / torch.dot(r_hat, v)
            s = r - alpha * v
            t = self.Ax_gen(s)
            omega = torch.dot(t, s) / torch.dot(t, t)
            self.x = self.x + alpha * p + omega * s
            self.iterations += 1
            done, _ = self._residual(self.x)
            if done:
                return self.x
            r = s - omega * t
            if rho_prev == 0:
                break
            steps -= 1
        return self.x
