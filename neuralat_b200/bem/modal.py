"""Acoustic transfer of many vibration modes of one object.

The reference's ``EditableModalSound.solve`` (src/scene.py:384-397) loops
over the modes: for mode i, ``neumann2dirichlet(ks[i], neumann_vtx[i])`` and
``boundary2potential(ks[i], neumann_vtx[i], dirichlet, trg_points)``, then
stacks the listener pressures (modes, P).  ``solve_modes`` computes the same
through the batch runner: the Burton-Miller matrices of all modes of a wave
in one launch family, the solves on concurrent streams, the listener
evaluation on the solver's fused kernel.
"""
from __future__ import annotations

import torch

from .batch import shared_runner
from .solver import BEM_Solver


def solve_modes(solver: BEM_Solver, ks, neumanns, points, *, precision: str = "fp32", rtol: float = 1e-5,
                max_iters: int = 500, restart: int = 200, workers: int = 4, memory_budget_bytes: int | None = None,
                return_dirichlet: bool = False, info: list | None = None):
    """Listener pressures (modes, P) complex64 of every mode.

    ks: (modes,) wavenumbers; neumanns: (modes, N) complex normal velocities
    (one row per mode); points: (P, 3).  The defaults follow the reference's
    ``solve_linear_equation`` (relative residual 1e-5, at most 500 steps).
    With ``return_dirichlet`` also the (modes, N) boundary pressures.
    ``info`` (a list) receives the solver info of every mode."""
    ks = [float(k) for k in (ks.tolist() if torch.is_tensor(ks) else ks)]
    if len(ks) == 0:
        raise ValueError("no modes")
    rows = [neumanns[i] for i in range(len(ks))]
    with torch.cuda.device(solver.device):
        runner = shared_runner(memory_budget_bytes=memory_budget_bytes, workers=workers, precision=precision,
                               rtol=rtol, restart=restart, formulation="burton_miller", max_iters=max_iters)
        res = runner.run([solver], [ks], [rows], points, return_dirichlet=return_dirichlet)
    order = sorted(range(len(res.index)), key=lambda i: res.index[i][1])
    p = torch.stack([res.pressure[i][:, 0] for i in order])
    if info is not None:
        info.extend(res.info[i] for i in order)
    if return_dirichlet:
        return p, torch.stack([res.dirichlet[i][:, 0] for i in order])
    return p
