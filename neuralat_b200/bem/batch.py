"""Batched BEM: many meshes of uneven size x many wavenumbers x many RHS.

For every (mesh, wavenumber) problem the path is the same as ``BEM_Solver``
(fused V / (1/2 M - K) assembly, -V g, CBIE solve, listener evaluation); the
batch runner changes how the work reaches the GPU:

* problems are processed in waves sized to a device-memory budget (each
  problem's matrices are released before the next wave), so a batch larger
  than HBM streams through it;
* the assembly of a whole wave is ONE persistent launch of the regular-pair
  kernel (CTAs drain a single queue of (problem, test group, trial chunk)
  items, so a 320-triangle mesh and a 20 480-triangle mesh share the GPU
  without launch-per-problem overhead) plus one launch per touching-pair
  type (``bem_batch_matrices_vk``);
* the solves of a wave run concurrently, one CUDA stream per worker thread,
  each Arnoldi step replayed from a captured CUDA graph;
* launch shapes come from the autotuner (``neuralat_b200.bem.autotune``).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from .. import _lib as L
from .solver import BEM_Solver, _stream, _vp, cmatmul, gmres


@dataclass
class BatchResult:
    dirichlet: list = field(default_factory=list)  # per problem: (N, m) complex64 (or None)
    pressure: list = field(default_factory=list)   # per problem: (P, m) complex64
    info: list = field(default_factory=list)       # per problem: solver info dict
    index: list = field(default_factory=list)      # per problem: (mesh index, k index)


def assemble_batch(solvers, ks, mass_coeff=0.5, k_coeff=-1.0, stream=None):
    """Assemble (V, mass_coeff M + k_coeff K) for each (solver, k) in one launch family."""
    assert len(solvers) == len(ks) and len(ks) > 0
    lib = L.lib()
    dev = solvers[0].device
    n = len(ks)
    probs = (L.BatchProblem * n)()
    outs = []
    for i, (s, k) in enumerate(zip(solvers, ks)):
        V, A = s._new_matrix(), s._new_matrix()
        outs.append((V, A))
        probs[i].geom = s.geometry.ptr.value
        probs[i].k = float(k)
        probs[i].v_out = V.data_ptr()
        probs[i].k_out = A.data_ptr()
    nbytes = int(lib.bem_batch_workspace_bytes(n))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else _stream(dev)
        L.check(lib.bem_batch_matrices_vk(probs, n, float(mass_coeff), float(k_coeff), _vp(ws), nbytes, st),
                "bem_batch_matrices_vk")
    return outs


def problem_bytes(nv: int, m: int, restart: int = 200) -> int:
    """Device bytes one problem holds while it is solved (V, LHS, tensor-core
    planes, Krylov basis and vectors)."""
    return 3 * 8 * nv * nv + 8 * m * (restart + 1) * nv + 64 * m * nv


class BatchRunner:
    """Run a list of meshes x wavenumbers x RHS through the GPU in waves."""

    def __init__(self, memory_budget_bytes: int | None = None, workers: int = 4, precision: str = "fp16x3",
                 rtol: float = 1e-6, restart: int = 200):
        if memory_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            memory_budget_bytes = int(0.6 * free)
        self.budget = memory_budget_bytes
        self.workers = max(1, workers)
        self.precision, self.rtol, self.restart = precision, rtol, restart
        self._streams = [torch.cuda.Stream() for _ in range(self.workers)]

    def _solve_one(self, widx, A, rhs, solver, k, g, pts, want_u):
        st = self._streams[widx % self.workers]
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            info = {}
            u = gmres(A, rhs, rtol=self.rtol, restart=self.restart, precision=self.precision, info=info)
            p = solver.boundary2potential(k, g, u, pts)
            st.synchronize()
        return (u if want_u else None), p, info

    def run(self, meshes, ks_per_mesh, neumann_per_mesh, points, return_dirichlet=False) -> BatchResult:
        """meshes: list of (vertices, triangles) numpy arrays; ks_per_mesh: list
        of wavenumber lists; neumann_per_mesh: list of (N, m) arrays; points (P, 3)."""
        dev = torch.device("cuda", torch.cuda.current_device())
        pts = torch.as_tensor(np.asarray(points, np.float32), device=dev).contiguous()
        solvers = [BEM_Solver(np.asarray(v, np.float32), np.asarray(t, np.int32)) for v, t in meshes]
        gs = [torch.as_tensor(np.asarray(g, np.complex64), device=dev).contiguous() for g in neumann_per_mesh]
        jobs = [(mi, ki) for mi in range(len(meshes)) for ki in range(len(ks_per_mesh[mi]))]
        # largest first: big problems start early and small ones fill the tail
        jobs.sort(key=lambda j: -solvers[j[0]].geometry.nv)
        res = BatchResult()
        wave, used = [], 0
        waves = []
        for j in jobs:
            b = problem_bytes(solvers[j[0]].geometry.nv, gs[j[0]].shape[1], self.restart)
            if wave and used + b > self.budget:
                waves.append(wave)
                wave, used = [], 0
            wave.append(j)
            used += b
        if wave:
            waves.append(wave)
        pool = cf.ThreadPoolExecutor(max_workers=self.workers)
        try:
            for wave in waves:
                ss = [solvers[mi] for mi, _ in wave]
                ks = [float(ks_per_mesh[mi][ki]) for mi, ki in wave]
                mats = assemble_batch(ss, ks)
                rhss = []
                for (mi, _), (V, A) in zip(wave, mats):
                    rhss.append(-cmatmul(V, gs[mi]))
                mats = [A for _, A in mats]  # V is no longer needed
                futs = [pool.submit(self._solve_one, w, A, rhs, solvers[mi], k, gs[mi], pts, return_dirichlet)
                        for w, ((mi, ki), A, rhs, k) in enumerate(zip(wave, mats, rhss, ks))]
                for (mi, ki), f in zip(wave, futs):
                    u, p, info = f.result()
                    res.dirichlet.append(u)
                    res.pressure.append(p)
                    res.info.append(info)
                    res.index.append((mi, ki))
                del mats, rhss
        finally:
            pool.shutdown(wait=True)
        return res
