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
  each Arnoldi step replayed from a captured CUDA graph; the concurrency
  follows the problem size (a 10k-unknown solve already keeps every SM busy,
  so problems of 4096 unknowns or more run two at a time, smaller ones on
  every worker);
* launch shapes come from the autotuner (``neuralat_b200.bem.autotune``).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .. import _lib as L
from .solver import BEM_Solver, _order, _stream, _vp, cmatmul, gmres


@dataclass
class BatchResult:
    dirichlet: list = field(default_factory=list)  # per problem: (N, m) complex64 (or None)
    pressure: list = field(default_factory=list)   # per problem: (P, m) complex64
    info: list = field(default_factory=list)       # per problem: solver info dict
    index: list = field(default_factory=list)      # per problem: (mesh index, k index)
    waves: list = field(default_factory=list)      # per wave: size, problems, concurrency, seconds


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


def assemble_batch_bm(solvers, ks, stream=None, approx=True):
    """Fused Burton-Miller (lhs, rhs) matrices of ``neumann2dirichlet`` (or,
    with approx=False, of ``HBIE``) for each (solver, k) in one launch family."""
    assert len(solvers) == len(ks) and len(ks) > 0
    lib = L.lib()
    dev = solvers[0].device
    n = len(ks)
    probs = (L.BmProblem * n)()
    outs = []
    for i, (s, k) in enumerate(zip(solvers, ks)):
        lhs, rhs = s._new_matrix(), s._new_matrix()
        outs.append((lhs, rhs))
        probs[i].geom = s.geometry.ptr.value
        probs[i].k = float(k)
        probs[i].lhs_out = lhs.data_ptr()
        probs[i].rhs_out = rhs.data_ptr()
    nbytes = int(lib.bem_batch_workspace_bytes(n))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else _stream(dev)
        L.check(lib.bem_batch_matrices_bm(probs, n, _order(approx), _vp(ws), nbytes, st), "bem_batch_matrices_bm")
    return outs


def problem_bytes(nv: int, m: int, restart: int = 200) -> int:
    """Device bytes one problem holds while it is solved (V, LHS, tensor-core
    planes, Krylov basis and vectors)."""
    return 3 * 8 * nv * nv + 8 * m * (restart + 1) * nv + 64 * m * nv


FORMULATIONS = ("cbie", "burton_miller")


def plan_waves(sizes, budget: int, concurrency) -> list:
    """Group jobs into waves: ``sizes`` is a list of (job, nv, bytes) in the
    order the jobs should run; a wave holds jobs of one concurrency class
    (``concurrency(nv)``) whose bytes fit ``budget`` together.  Returns
    [(jobs, concurrency)].  Raises ``MemoryError`` (before anything is
    allocated) when one job alone needs more than the budget."""
    waves, wave, used, conc = [], [], 0, None
    for job, nv, b in sizes:
        if b > budget:
            raise MemoryError(f"a problem of {nv} unknowns needs {b / 2**30:.2f} GiB of device memory, more than "
                              f"the batch budget of {budget / 2**30:.2f} GiB")
        c = concurrency(nv)
        if wave and (used + b > budget or c != conc):
            waves.append((wave, conc))
            wave, used = [], 0
        wave.append(job)
        used += b
        conc = c
    if wave:
        waves.append((wave, conc))
    return waves


class BatchRunner:
    """Run a list of meshes x wavenumbers x RHS through the GPU in waves.

    formulation "cbie": (1/2 I - K) u = -V g (``BEM_Solver.CBIE``);
    "burton_miller": the <2,3> Burton-Miller system of
    ``BEM_Solver.neumann2dirichlet`` (free of interior resonances)."""

    def __init__(self, memory_budget_bytes: int | None = None, workers: int = 4, precision: str = "fp16x3",
                 rtol: float = 1e-6, restart: int = 200, formulation: str = "cbie", max_iters: int = 1000):
        if formulation not in FORMULATIONS:
            raise ValueError(f"formulation must be one of {FORMULATIONS}")
        if memory_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            memory_budget_bytes = int(0.6 * free)
        if memory_budget_bytes <= 0:
            raise ValueError("memory_budget_bytes must be positive")
        self.budget = int(memory_budget_bytes)
        self.workers = max(1, workers)
        self.precision, self.rtol, self.restart = precision, rtol, restart
        self.formulation, self.max_iters = formulation, max_iters
        self._local = threading.local()
        # persistent workers: each keeps its stream and the solver's per-thread
        # host buffers for the runner's lifetime
        self._pool = cf.ThreadPoolExecutor(max_workers=self.workers)

    def close(self) -> None:
        self._pool.shutdown(wait=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def concurrency(self, nv: int) -> int:
        """Concurrent solves for problems of nv unknowns."""
        return min(2, self.workers) if nv >= 4096 else self.workers

    def _stream(self):
        st = getattr(self._local, "stream", None)
        if st is None:
            st = self._local.stream = torch.cuda.Stream()
        return st

    def _solve_lane(self, tasks, want_u, ready):
        """Solve tasks [(A, rhs, solver, k, g, points)] one after another on this worker's stream."""
        st = self._stream()
        st.wait_event(ready)
        out = []
        with torch.cuda.stream(st):
            for A, rhs, solver, k, g, pts in tasks:
                info = {}
                u = gmres(A, rhs, rtol=self.rtol, restart=self.restart, max_iters=self.max_iters,
                          precision=self.precision, info=info)
                p = solver.boundary2potential(k, g, u, pts)
                out.append(((u if want_u else None), p, info))
            st.synchronize()
        return out

    def run(self, meshes, ks_per_mesh, neumann_per_mesh, points, return_dirichlet=False) -> BatchResult:
        """meshes: list of (vertices, triangles) numpy arrays or ``BEM_Solver``s;
        ks_per_mesh: list of wavenumber lists; neumann_per_mesh: per mesh an
        (N,) or (N, m) array shared by its wavenumbers, or a list with one
        such array per wavenumber (a vibration mode per wavenumber); points
        (P, 3) for every problem, or a list with one (P_i, 3) array per mesh.
        Results are (N, m) / (P, m) per problem, m = 1 for (N,)."""
        dev = torch.device("cuda", torch.cuda.current_device())

        def dev_points(x):
            return (x.to(device=dev, dtype=torch.float32) if torch.is_tensor(x)
                    else torch.as_tensor(np.asarray(x, np.float32), device=dev)).contiguous()

        per_mesh_points = isinstance(points, (list, tuple))
        if per_mesh_points and len(points) != len(meshes):
            raise ValueError(f"{len(points)} point sets for {len(meshes)} meshes")
        pts = [dev_points(x) for x in points] if per_mesh_points else dev_points(points)
        solvers = [m if isinstance(m, BEM_Solver) else BEM_Solver(np.asarray(m[0], np.float32),
                                                                   np.asarray(m[1], np.int32)) for m in meshes]

        def dev_c64(g):
            g = g if torch.is_tensor(g) else torch.from_numpy(np.asarray(g, np.complex64))
            g = g.to(device=dev, dtype=torch.complex64)
            return (g.reshape(-1, 1) if g.dim() == 1 else g).contiguous()

        gs = []
        for mi, g in enumerate(neumann_per_mesh):
            if isinstance(g, (list, tuple)):
                if len(g) != len(ks_per_mesh[mi]):
                    raise ValueError(f"mesh {mi}: {len(g)} Neumann arrays for {len(ks_per_mesh[mi])} wavenumbers")
                gs.append([dev_c64(x) for x in g])
            else:
                gs.append(dev_c64(g))

        def neumann(mi, ki):
            return gs[mi][ki] if isinstance(gs[mi], list) else gs[mi]

        jobs = [(mi, ki) for mi in range(len(meshes)) for ki in range(len(ks_per_mesh[mi]))]
        # largest first: big problems start early and small ones fill the tail
        jobs.sort(key=lambda j: -solvers[j[0]].geometry.nv)
        res = BatchResult()
        # waves: one size class (same concurrency) and within the memory budget,
        # which must itself fit the device: a budget above the free memory is
        # an error here, not an out-of-memory failure in the middle of a wave
        free, _ = torch.cuda.mem_get_info(dev)
        budget = self.budget
        sizes = [(j, solvers[j[0]].geometry.nv,
                  problem_bytes(solvers[j[0]].geometry.nv, neumann(*j).shape[1], self.restart)) for j in jobs]
        waves = plan_waves(sizes, budget, self.concurrency)
        bytes_of = {j: b for j, _, b in sizes}
        peak = max(sum(bytes_of[j] for j in w) for w, _ in waves)
        if peak > free:
            raise MemoryError(f"a wave needs {peak / 2**30:.2f} GiB of device memory but only {free / 2**30:.2f} GiB "
                              f"are free: lower memory_budget_bytes (now {budget / 2**30:.2f} GiB)")
        for wave, conc in waves:
            t0 = time.perf_counter()
            ss = [solvers[mi] for mi, _ in wave]
            ks = [float(ks_per_mesh[mi][ki]) for mi, ki in wave]
            # keep only the left-hand sides once the right-hand sides are formed
            if self.formulation == "cbie":
                pairs = assemble_batch(ss, ks)  # (V, 1/2 I - K)
                rhss = [-cmatmul(V, neumann(*j)) for j, (V, _) in zip(wave, pairs)]
                mats = [A for _, A in pairs]
            else:
                pairs = assemble_batch_bm(ss, ks)  # (lhs, rhs operator)
                rhss = [cmatmul(R, neumann(*j)) for j, (_, R) in zip(wave, pairs)]
                mats = [A for A, _ in pairs]
            del pairs
            ready = torch.cuda.Event()
            ready.record()
            tasks = [(A, rhs, solvers[mi], k, neumann(mi, ki), pts[mi] if per_mesh_points else pts)
                     for (mi, ki), A, rhs, k in zip(wave, mats, rhss, ks)]
            lanes = [list(range(w, len(wave), conc)) for w in range(conc)]  # round-robin over workers
            futs = [self._pool.submit(self._solve_lane, [tasks[i] for i in lane], return_dirichlet, ready)
                    for lane in lanes if lane]
            out = [None] * len(wave)
            for lane, f in zip([ln for ln in lanes if ln], futs):
                for i, r in zip(lane, f.result()):
                    out[i] = r
            for sv in {id(x): x for x in ss}.values():  # a bounded wait of the wave's assembly expired?
                sv.geometry.check_status()
            for (mi, ki), (u, p, info) in zip(wave, out):
                res.dirichlet.append(u)
                res.pressure.append(p)
                res.info.append(info)
                res.index.append((mi, ki))
            res.waves.append({"vertices": int(ss[0].geometry.nv), "problems": len(wave), "concurrency": conc,
                              "seconds": time.perf_counter() - t0})
            del mats, rhss, tasks
        return res


# Runners (with their worker threads, streams and per-thread host buffers)
# kept across calls, one per device and setting.
_SHARED: dict = {}
_SHARED_LOCK = threading.Lock()


def shared_runner(**kw) -> BatchRunner:
    """A process-wide BatchRunner for these settings on the current device,
    created on first use and reused by later calls."""
    key = (torch.cuda.current_device(),) + tuple(sorted(kw.items()))
    with _SHARED_LOCK:
        r = _SHARED.get(key)
        if r is None:
            r = _SHARED[key] = BatchRunner(**kw)
        return r
