#!/usr/bin/env python
"""Benchmark: BEM assemble + solve + evaluate, seconds per problem at 20k triangles.

Workload (one "problem" = one step): icosphere subdivision 5 (N = 10 242 P1
unknowns, T = 20 480 triangles), radius 0.15 m with axes scaled by seeded
U[0.7, 1.3], k at 4 kHz, 8 smoothed complex Gaussian Neumann fields, 256
listeners on a 0.5 m sphere.  A step builds the mesh geometry, assembles V
and 0.5 I - K (fused), forms -V g, solves the exterior-Neumann CBIE for all 8
right-hand sides to rtol 1e-6 (FP64 refinement) and evaluates the listener
pressures.  Inputs are synthetic (seeded); the matrices (839 MB each) exceed
the 126 MB L2, so no extra L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank solves its own replica ("replicas only":
the path has no data exchange); times are the max over ranks.
``--impl reference`` times the FP64 CPU restatement of the reference's
algorithm (the reference has no CPU implementation of its own) on a bounded
sample of the same workload.

Besides the metric line: ``roofline`` (fused assembly, FP32 issue) and
``roofline_matvec`` (tensor-core matvec timed alone, HBM).  Other workloads,
one JSON line each: ``--batch-case`` (meshes x wavenumbers through the batch
runner), ``--modal-case`` (many vibration modes of one object, Burton-Miller),
``--grad-case`` (forward + adjoint backward), ``--large-case`` (s6, 64 RHS),
``--kernel-case assemble|assemble_bm|solve|eval`` (one stage on a smaller
mesh, for profiler captures), ``--validate`` (listener error against the FP64
oracle).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "assemble+solve+eval s/problem @20k tris (icosphere s5, 8 RHS, 4 kHz, 256 listeners), 1 B200"
WORKLOAD = ("icosphere s5 N=10242 T=20480, r=0.15 m axes*U[0.7,1.3] (seed 1), k=2pi*4000/343, "
            "8 smoothed complex Gaussian Neumann RHS (seed 2), 256 listeners r=0.5 m (seed 0), CBIE rtol 1e-6")
F_VK = 63.0  # FP32 flops per regular quadrature-point pair, fused V+K (algorithmic count)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", default="fp16x3", choices=["fp32", "bf16x3", "bf16", "fp16x3"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-FP32 comparison timing")
    ap.add_argument("--plain-steps", type=int, default=5, help="timed steps of the plain-FP32 comparison (>= 5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own GPU kernels (B0) beside the CPU line")
    ap.add_argument("--validate", action="store_true", help="also compare against the FP64 oracle (minutes)")
    ap.add_argument("--kernel-case", choices=["assemble", "assemble_bm", "solve", "eval"], default=None,
                    help="profiling case: one stage on an icosphere of --subdiv, after one warm-up launch")
    ap.add_argument("--subdiv", type=int, default=4)
    ap.add_argument("--cpu-validate", action="store_true",
                    help="sampled CPU model vs one whole measured FP64 CPU problem on an icosphere of --subdiv")
    ap.add_argument("--large-case", action="store_true",
                    help="large multi-RHS configuration: icosphere s6 (N=40962) with 5%% radial noise, 64 RHS, "
                         "8 kHz, 4096 listeners (stage times, solver info, FP64 residual)")
    ap.add_argument("--grad-case", action="store_true",
                    help="differentiation configuration: icosphere s4, 2 kHz, one RHS, 128 listeners, "
                         "L = sum |p|^2, forward + hand-written adjoint backward (dL/dvertices, dL/dneumann)")
    ap.add_argument("--batch-case", action="store_true",
                    help="batching workload: meshes x wavenumbers through the batch runner vs one at a time")
    ap.add_argument("--batch-meshes", type=int, default=16)
    ap.add_argument("--batch-k", type=int, default=4)
    ap.add_argument("--batch-max-subdiv", type=int, default=4)
    ap.add_argument("--modal-case", action="store_true",
                    help="multi-mode workload (EditableModalSound.solve): one object, --modal-modes modes at "
                         "log-uniform 200-8000 Hz, Burton-Miller solve per mode, 256 listeners")
    ap.add_argument("--modal-subdiv", type=int, default=4)
    ap.add_argument("--modal-modes", type=int, default=64)
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
def workload():
    from neuralat_b200.bem import meshes as M

    w = M.precision_large(m=8)
    return (w["vertices"].astype(np.float32), w["triangles"].astype(np.int32), float(w["k"]),
            w["neumann"].astype(np.complex64), w["points"].astype(np.float32))


def regular_pair_evals(triangles) -> float:
    """36 x (ordered triangle pairs sharing no vertex)."""
    t = np.asarray(triangles)
    nt = t.shape[0]
    nv = int(t.max()) + 1
    star = [[] for _ in range(nv)]
    for i, tri in enumerate(t):
        for a in tri:
            star[a].append(i)
    touching = 0
    for i, tri in enumerate(t):
        touching += len(set(star[tri[0]]) | set(star[tri[1]]) | set(star[tri[2]]))
    return 36.0 * (nt * nt - touching)


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json beside
    this file), else the earlier pool measurement."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return {"gbs": float(json.load(f)["hbm_gbs"]), "source": "measured copy bandwidth (MEASURED_PEAKS.json)"}
    except (OSError, ValueError, KeyError):
        return {"gbs": 6650.0, "source": "fallback 6.65 TB/s (earlier measurement on this pool)"}


def fp32_peak_tflops(sm_max_mhz=None):
    import torch

    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    mhz = sm_max_mhz or 1965.0
    return props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12


# ---------------------------------------------------------------------------
def host_cpu():
    """CPU model and logical core count of this host (for the CPU baseline record)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


# The sampled CPU model below was checked against one full FP64 problem on an
# icosphere s4 workload (``--cpu-validate``): the ratio model / full is
# recorded in the line of that case and quoted in ``sample``.
CPU_MODEL_CHECK = "model checked against a full FP64 s4 problem by bench.py --cpu-validate"


def cpu_baseline(v, t, k, g, pts, rows_sampled=48):
    """FP64 CPU restatement (oracle) timed on a bounded sample, extrapolated to
    one full problem: assembly of sampled rows of V and K, a dense complex128
    LU solve of a smaller system (scaled by n^3), listener evaluation for a
    subset of listeners."""
    from oracle import oracle as O

    O.build()
    nv, nt = v.shape[0], t.shape[0]
    v64 = v.astype(np.float64)
    rows = np.linspace(0, nv - 1, min(rows_sampled, nv)).astype(np.int32)
    mask = np.zeros(nv, bool)
    mask[rows] = True
    frac_tris = float(np.any(mask[t], axis=1).sum()) / nt
    t0 = time.perf_counter()
    O.boundary_matrix("single", v64, t, k, rows=rows)
    O.boundary_matrix("double", v64, t, k, rows=rows)
    t_asm = (time.perf_counter() - t0) / frac_tris
    ns = min(2048, nv)
    rng = np.random.default_rng(0)
    A = rng.standard_normal((ns, ns)) + 1j * rng.standard_normal((ns, ns))
    B = rng.standard_normal((ns, g.shape[1])) + 1j * rng.standard_normal((ns, g.shape[1]))
    t0 = time.perf_counter()
    np.linalg.solve(A, B)
    t_solve = (time.perf_counter() - t0) * (nv / ns) ** 3
    pp = pts[:8]
    t0 = time.perf_counter()
    O.potential_matrix("single", v64, t, pp, k)
    O.potential_matrix("double", v64, t, pp, k)
    t_eval = (time.perf_counter() - t0) * pts.shape[0] / pp.shape[0]
    total = t_asm + t_solve + t_eval
    return {
        "value": total, "unit": "s/problem", "cores": int(O.num_threads()), "kind": "port",
        "sample": (f"FP64 oracle: V+K rows of {rows.size} vertices ({frac_tris:.4f} of test triangles) "
                   f"extrapolated; complex128 LU {ns}x{ns} x{g.shape[1]} RHS scaled by (N/{ns})^3; "
                   f"{pp.shape[0]} of {pts.shape[0]} listeners scaled; {CPU_MODEL_CHECK}"),
        "stages_s": {"assemble": t_asm, "solve": t_solve, "eval": t_eval},
        **host_cpu(),
    }


def cpu_full(v, t, k, g, pts):
    """One whole FP64 CPU problem on the oracle, every stage measured: full V,
    K and M assembly, the dense complex128 solve of the CBIE (LAPACK) and all
    listeners."""
    from oracle import oracle as O

    O.build()
    v64 = v.astype(np.float64)
    t0 = time.perf_counter()
    V = O.boundary_matrix("single", v64, t, k)
    K = O.boundary_matrix("double", v64, t, k)
    M = O.identity_matrix(v64, t)
    t1 = time.perf_counter()
    u = np.linalg.solve(0.5 * M - K, -V @ g.astype(np.complex128))
    t2 = time.perf_counter()
    p = O.boundary2potential(v64, t, k, g.astype(np.complex128), u, pts.astype(np.float64))
    t3 = time.perf_counter()
    return {"value": t3 - t0, "stages_s": {"assemble": t1 - t0, "solve": t2 - t1, "eval": t3 - t2},
            "cores": int(O.num_threads()), "pressure_norm": float(np.linalg.norm(p))}


# Multi-rank plumbing ("replicas only": every rank solves its own problem, no
# collective on the data path).
def rank_barrier(dist, cuda: bool = True) -> None:
    if dist is not None:
        dist.barrier()
    if cuda:
        import torch

        torch.cuda.synchronize()


def max_over_ranks_of(x: float, dist, device) -> float:
    """The slowest rank's time (device timings are compared as the max over ranks)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_problem(ms_per_step: float, world: int) -> float:
    """World replicas each finish one problem per step (max-over-ranks step
    time), so the whole job solves `world` problems per step."""
    return (ms_per_step / 1e3) / world


def reference_preprocess(torch, vertices, triangles):
    """Unit normals and surface curls as the reference's ``preprocess``
    computes them with torch (src/bem/solver.py:40-58): edge vectors, the
    batched inverse metric, gradients of the three P1 functions, n x grad."""
    v0, v1, v2 = (vertices[triangles[:, i].long()] for i in range(3))
    n = torch.linalg.cross(v1 - v0, v2 - v0, dim=1)
    n = n / torch.norm(n, dim=1, keepdim=True)
    J = torch.stack([v1 - v0, v2 - v0], dim=2)
    jit = torch.bmm(J, torch.inverse(torch.bmm(J.transpose(1, 2), J)))
    rg = torch.tensor([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]], dtype=torch.float32, device=vertices.device)
    grads = torch.matmul(jit, rg).transpose(1, 2)
    return n.contiguous(), torch.linalg.cross(n.unsqueeze(1), grads, dim=2).contiguous()


def reference_gpu(v, t, k, g, pts, steps=1):
    """B0: the reference's own CUDA kernels (src/bem/cuda/bind.cu, built
    unmodified into oracle/_ref by oracle/build_ref.py) on this workload,
    driven the way its ``BEM_Solver.CBIE`` + ``boundary2potential`` drive
    them (src/bem/solver.py:83-147): torch preprocess, identity / single /
    double boundary matrices, 0.5 I - K and -V g with torch (cuBLAS), the
    reference's BiCGSTAB per right-hand side with its defaults (500 steps,
    tol 1e-10 on ||r||^2 / ||b||^2), then the two potential matrices and
    their products.  Per-stage CUDA-event times after one warm-up problem,
    and the listener error against the same FP64 fixture as our line."""
    import torch

    from neuralat_b200.bem.bicgstab import BiCGSTAB
    from oracle import build_ref

    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    ref = build_ref.load_prebuilt()
    if ref is None:
        return {"unavailable": "oracle/_ref/neuralat_ref_bem.so not built"}
    dev = torch.device("cuda", 0)
    vt = torch.from_numpy(v).to(dev)
    tt = torch.from_numpy(t).to(dev)
    gt = torch.from_numpy(g).to(dev)
    pt = torch.from_numpy(pts).to(dev)
    kf = float(k)

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    def problem(tol=1e-10, atol=1e-16):
        e = [ev()]
        normals, curls = reference_preprocess(torch, vt, tt)
        e.append(ev())
        identity = ref.identity_matrix(vt, tt)
        V = ref.single_boundary_matrix(vt, tt, normals, curls, kf)
        K = ref.double_boundary_matrix(vt, tt, normals, curls, kf)
        e.append(ev())
        A = 0.5 * identity - K
        del identity, K
        b = -V @ gt
        del V
        e.append(ev())
        iters = []
        us = []
        for j in range(gt.shape[1]):
            solver = BiCGSTAB(lambda x: A @ x)
            us.append(solver.solve(b[:, j].contiguous(), nsteps=500, tol=tol, atol=atol))
            iters.append(solver.iterations)
        u = torch.stack(us, dim=1)
        del A
        e.append(ev())
        S = ref.single_boundary_potential(vt, tt, pt, kf)
        D = ref.double_boundary_potential(vt, tt, pt, kf)
        p = -S @ gt + D @ u
        e.append(ev())
        torch.cuda.synchronize()
        return e, p, iters

    names = ["preprocess", "assemble", "rhs", "solve", "eval"]

    def timed(**kw):
        problem(**kw)
        times, p, iters = [], None, None
        for _ in range(max(1, steps)):
            e, p, iters = problem(**kw)
            times.append([e[i].elapsed_time(e[i + 1]) for i in range(len(e) - 1)])
        stage_ms = {n: float(np.mean([tm[i] for tm in times])) for i, n in enumerate(names)}
        return {"s_per_problem": sum(stage_ms.values()) / 1e3, "stages_ms": stage_ms, "steps": len(times),
                "bicgstab_iterations": iters,
                "listener_err_vs_fp64": listener_error_vs_fixture(v, t, k, g, p, None).get("mixed")}

    out = timed()
    out["what"] = ("reference src/bem kernels (bind.cu, unmodified, oracle/_ref) + torch/cuBLAS + the reference's "
                   "BiCGSTAB per RHS with its defaults (tol 1e-10 on ||r||^2/||b||^2, atol 1e-16 on ||r||^2: on this "
                   "workload's scale the absolute test stops it near relative residual 1e-3); FP32; one B200")
    # the same path with the absolute test off, so that only the relative one
    # (1e-5 in ||r||) stops it: the reference's own kernels at their best accuracy
    out["relative_tol_only"] = timed(atol=0.0)
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    v, t, k, g, pts = workload()
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(v, t, k, g, pts)
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(v, t, k, g, pts)
        vals.append(cb["value"])
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s/problem", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": "s/problem", "cores": cb["cores"], "kind": cb["kind"],
                         "sample": cb["sample"], "cpu_model": cb["cpu_model"], "nproc": cb["nproc"]},
        "e2e": {"value": value, "unit": "s/problem", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        try:
            line["reference_gpu"] = reference_gpu(v, t, k, g, pts)
        except Exception as e:  # a reported side measurement; the CPU line stands
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from neuralat_b200 import _lib as L
    from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
    from neuralat_b200.bem.solver import _stream, _vp

    lib = L.lib()
    v, t, k, g, pts = workload()
    dev = torch.device("cuda", local)
    v_d = torch.from_numpy(v).to(dev)
    t_d = torch.from_numpy(t).to(dev)
    g_d = torch.from_numpy(g).to(dev)
    p_d = torch.from_numpy(pts).to(dev)
    n_eval = regular_pair_evals(t)
    stream = torch.cuda.current_stream(dev)

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    stage_names = ["geometry", "assemble", "rhs", "solve", "eval"]

    def step(record=None, info=None):
        e0 = ev()
        s = BEM_Solver(v_d, t_d)
        e1 = ev()
        # the assembly's bounded-wait status is read once after the timed region
        V, A = s.assemble_vk(k, check=False)
        e2 = ev()
        rhs = -cmatmul(V, g_d)
        del V
        e3 = ev()
        u = gmres(A, rhs, rtol=1e-6, precision=args.precision, info=info)
        e4 = ev()
        p = s.boundary2potential(k, g_d, u, p_d)
        e5 = ev()
        if record is not None:
            record.append((e0, e1, e2, e3, e4, e5))
        return u, p

    def barrier():
        rank_barrier(dist, cuda=True)

    def max_over_ranks(x: float) -> float:
        return max_over_ranks_of(x, dist, dev)

    # ---- warm-up --------------------------------------------------------------
    info = {}
    for _ in range(max(args.warmup, 0)):
        step(info=info)
    barrier()

    # ---- timed region (device-resident inputs) --------------------------------
    rec = []
    infos = []
    with ClockSampler(local) as clk:
        barrier()
        l0 = lib.bem_kernel_launches()
        t_start = ev()
        last_p = None
        for _ in range(args.steps):
            inf = {}
            _, last_p = step(rec, inf)
            infos.append(inf)
        t_end = ev()
        barrier()
        l1 = lib.bem_kernel_launches()
    # no bounded wait of any assembly kernel expired in the timed steps
    L.check(lib.bem_assembly_status(_stream(dev)), "assembly in the timed steps")
    total_ms = max_over_ranks(t_start.elapsed_time(t_end))
    ms_per_step = total_ms / args.steps
    value = whole_job_seconds_per_problem(ms_per_step, world)
    stages = {n: float(np.mean([r[i].elapsed_time(r[i + 1]) for r in rec])) for i, n in enumerate(stage_names)}
    asm_ms = stages["assemble"]

    # ---- end to end through the public API from host buffers -------------------
    v_h = torch.from_numpy(v).pin_memory()
    t_h = torch.from_numpy(t).pin_memory()
    g_h = torch.from_numpy(g).pin_memory()
    p_h = torch.from_numpy(pts).pin_memory()
    h2d = sum(x.numel() * x.element_size() for x in (v_h, t_h, g_h, p_h))
    d2h = pts.shape[0] * g.shape[1] * 8
    barrier()
    e_s = ev()
    for _ in range(args.steps):
        vd = v_h.to(dev, non_blocking=True)
        td = t_h.to(dev, non_blocking=True)
        gd = g_h.to(dev, non_blocking=True)
        pd = p_h.to(dev, non_blocking=True)
        s = BEM_Solver(vd, td)
        _, p = s.solve_and_evaluate(k, gd, pd, precision=args.precision, rtol=1e-6)
        p.cpu()
    e_e = ev()
    barrier()
    e2e_ms = max_over_ranks(e_s.elapsed_time(e_e)) / args.steps

    # ---- plain FP32 form (reference-shaped pipeline on our kernels) ------------
    plain = None
    if not args.no_plain and rank == 0:
        def plain_step():
            s = BEM_Solver(v_d, t_d)
            I = s.identity_matrix()
            V = s.assemble_boundary_matrix(k, "single")
            K = s.assemble_boundary_matrix(k, "double")
            A = (0.5 * I - K).contiguous()
            del I, K
            rhs = -cmatmul(V, g_d)
            del V
            us = [gmres(A, rhs[:, j].contiguous(), rtol=1e-6, precision="fp32") for j in range(rhs.shape[1])]
            u = torch.stack(us, dim=1)
            del A
            S = s.potential_matrix(k, p_d, "single")
            D = s.potential_matrix(k, p_d, "double")
            return -(S @ g_d) + D @ u  # (P x N) products as the reference forms them (solver.py:147)

        plain_step()
        torch.cuda.synchronize()
        ps = ev()
        nplain = max(5, args.plain_steps)
        for _ in range(nplain):
            p_plain = plain_step()
        pe = ev()
        torch.cuda.synchronize()
        plain = {"s_per_problem": ps.elapsed_time(pe) / nplain / 1e3, "steps": nplain, "warmup": 1,
                 "form": "separate V, K, M assembly; explicit 0.5M-K; one FP32 single-RHS GMRES per RHS; "
                         "explicit S, D potential matrices"}
    err = listener_error_vs_fixture(v, t, k, g, last_p, p_plain if plain else None)

    # ---- roofline of the dominant kernel (fused regular V+K assembly) ----------
    clocks = clk.summary()
    peak = fp32_peak_tflops(clocks.get("sm_max_mhz"))
    achieved = F_VK * n_eval / (asm_ms / 1e3) / 1e12
    # DRAM traffic of regular_sym_kernel: 167.4 MB per launch measured by ncu at
    # icosphere s4 (N = 2562: the atomic read-modify-write of the two output
    # matrices), scaled by the units processed, (10242 / 2562)^2, to this mesh
    traffic = 167.4e6 * (v.shape[0] / 2562.0) ** 2
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic,
                "kernel": "bem_boundary_matrices_vk (regular_sym_kernel + singular + memset, timed as one stage), "
                          f"63 flop x {n_eval:.4e} ordered regular quadrature-point pairs per launch (the kernel "
                          "evaluates each unordered pair once); peak = nominal FP32 (SMs x 128 FMA x 2 x max SM "
                          "clock; no measured FP32 peak available); traffic scaled from an s4 ncu capture"}

    # ---- roofline of the solve's dominant kernel (tensor-core matvec) ----------
    roofline_matvec = None
    if args.precision in ("fp16x3", "bf16x3", "bf16"):
        prec = {"fp16x3": L.PREC_FP16X3, "bf16x3": L.PREC_BF16X3, "bf16": L.PREC_BF16}[args.precision]
        s = BEM_Solver(v_d, t_d)
        _, A = s.assemble_vk(k, single=False)
        n, m = A.shape[0], g.shape[1]
        nbytes = int(lib.bem_tc_operator_bytes(n, m, prec))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        L.check(lib.bem_tc_operator_prepare(_vp(A), n, prec, _vp(ws), nbytes, _stream(dev)))
        del A
        X = torch.randn(n, m, dtype=torch.complex64, device=dev)
        Y = torch.empty_like(X)
        for _ in range(3):
            L.check(lib.bem_tc_matmul(_vp(ws), nbytes, n, prec, _vp(X), m, _vp(Y), _stream(dev)))
        nrep = 20
        m0 = ev()
        for _ in range(nrep):  # the 16-bit planes (839 MB at s5) are far larger than L2
            L.check(lib.bem_tc_matmul(_vp(ws), nbytes, n, prec, _vp(X), m, _vp(Y), _stream(dev)))
        m1 = ev()
        torch.cuda.synchronize()
        L.check(lib.bem_tc_status(_vp(ws), _stream(dev)))
        us = m0.elapsed_time(m1) / nrep * 1e3
        planes = 2 if args.precision != "bf16" else 1
        alg = planes * 2 * n * (2 * n)  # 16-bit planes of the (n x 2n) real form of A
        hbm = measured_hbm_gbs()
        # DRAM reads of tc_gemm_kernel (fp16x3, 8 RHS): 53.7 MB per launch by ncu
        # at icosphere s4 (N = 2562, the two planes once), scaled by (N / 2562)^2
        traffic = 53.7e6 * (n / 2562.0) ** 2 if args.precision == "fp16x3" and m == 8 else None
        roofline_matvec = {"bound": "hbm", "achieved": alg / (us * 1e-6) / 1e9, "peak": hbm["gbs"], "unit": "GB/s",
                           "frac": alg / (us * 1e-6) / 1e9 / hbm["gbs"], "traffic": traffic, "us_per_launch": us,
                           "kernel": f"tc_gemm_kernel ({args.precision}, {m} RHS), {alg / 1e6:.0f} MB of operator "
                                     f"planes per launch, timed alone over {nrep} launches; peak = {hbm['source']}; "
                                     "traffic scaled from an s4 ncu capture"}
        del ws

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(v, t, k, g, pts)
        cpu = {kk: cb[kk] for kk in ("value", "unit", "cores", "kind", "sample", "cpu_model", "nproc")}

    if rank == 0:
        it = infos[-1] if infos else {}
        line = {
            "metric": METRIC, "value": value, "unit": "s/problem", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": f"f32 assembly + {args.precision} matvec + f64 refinement",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (two 839 MB matrices per step)"},
            "roofline": roofline, "roofline_matvec": roofline_matvec, "cpu_baseline": cpu,
            "e2e": {"value": e2e_ms / 1e3 / world, "unit": "s/problem", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(l1 - l0),
            "clocks": clocks,
            "stages_ms": stages,
            "solver": {kk: it.get(kk) for kk in ("iterations", "refinements", "matvecs", "rel_residual", "status")},
            "plain_fp32": plain,
            "speedup_vs_plain_fp32": (plain["s_per_problem"] / (ms_per_step / 1e3)) if plain else None,
            "listener_err_vs_fp64": err,
        }
        if args.validate:
            line["validation"] = validate(v, t, k, g, pts, dev, args.precision)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


FIXTURE = os.path.join(ROOT, "tests", "golden", "cfg2_pressures.npz")
ERR_BAR = 1e-4


def listener_error_vs_fixture(v, t, k, g, p_mixed, p_plain):
    """Listener-pressure error of the timed pipeline's last step (and of one
    plain-FP32 step) against the committed FP64-oracle pressures of this
    workload (tests/golden/make_cfg2_reference.py): the max over right-hand
    sides of ||p - p_fp64|| / ||p_fp64|| over the listeners."""
    if not os.path.exists(FIXTURE):
        return {"unavailable": f"{os.path.relpath(FIXTURE, ROOT)} missing"}
    f = np.load(FIXTURE)
    same = (int(f["nv"]) == v.shape[0] and int(f["nt"]) == t.shape[0] and abs(float(f["k"]) - float(np.float32(k))) <
            1e-9 * abs(k) and abs(float(f["vertex_checksum"]) - float(np.abs(v.astype(np.float64)).sum())) <
            1e-9 * float(f["vertex_checksum"]))
    if not same:
        return {"unavailable": "fixture was made for another workload"}
    ref = f["pressures"]

    def rel(p):
        if p is None:
            return None
        p = p.detach().cpu().numpy().astype(np.complex128)
        return float((np.linalg.norm(p - ref, axis=0) / np.linalg.norm(ref, axis=0)).max())

    e_mixed, e_plain = rel(p_mixed), rel(p_plain)
    return {"mixed": e_mixed, "plain": e_plain, "bar": ERR_BAR,
            "both_within_bar": bool(e_mixed is not None and e_mixed <= ERR_BAR and
                                    (e_plain is None or e_plain <= ERR_BAR)),
            "measure": "max over the RHS of ||p - p_fp64||_2 / ||p_fp64||_2 over the listeners; p_fp64 = FP64 "
                       "oracle (dense CBIE solve) on the same float32 inputs, tests/golden/cfg2_pressures.npz"}


def validate(v, t, k, g, pts, dev, precision):
    """Listener-pressure error of the GPU path against the FP64 oracle (minutes)."""
    import torch

    from neuralat_b200.bem import BEM_Solver
    from oracle import oracle as O

    s = BEM_Solver(torch.from_numpy(v).to(dev), torch.from_numpy(t).to(dev))
    _, p = s.solve_and_evaluate(k, torch.from_numpy(g).to(dev), torch.from_numpy(pts).to(dev), precision=precision,
                                rtol=1e-6)
    p = p.cpu().numpy()
    u_ref = O.cbie_solve(v, t, k, g)
    p_ref = O.boundary2potential(v, t, k, g, u_ref, pts)
    err = np.linalg.norm(p - p_ref, axis=0) / np.linalg.norm(p_ref, axis=0)
    return {"listener_rel_err_per_rhs": err.tolist(), "max": float(err.max())}


def run_cpu_validate(args):
    """The sampled CPU model (``cpu_baseline``) against one whole measured
    FP64 CPU problem on the same box: the benchmark workload's recipe on an
    icosphere of --subdiv (default 4: N = 2562), where the full problem takes
    about a minute."""
    from neuralat_b200.bem import meshes as M

    v, t = M.icosphere(args.subdiv, 0.15)
    v = (v * np.random.default_rng(1).uniform(0.7, 1.3, size=3)).astype(np.float32)
    t = t.astype(np.int32)
    k = M.wavenumber(4000.0)
    g = M.smoothed_gaussian_field(v.shape[0], t, 8, seed=2).astype(np.complex64)
    pts = M.sphere_points(256, 0.5, seed=0).astype(np.float32)
    model = cpu_baseline(v, t, k, g, pts)
    full = cpu_full(v, t, k, g, pts)
    line = {"case": "cpu_model_check", "N": int(v.shape[0]), "T": int(t.shape[0]), "rhs": 8, "listeners": 256,
            "model_s": model["value"], "full_s": full["value"], "model_over_full": model["value"] / full["value"],
            "model_stages_s": model["stages_s"], "full_stages_s": full["stages_s"], "cores": full["cores"],
            **host_cpu()}
    print(json.dumps(line), flush=True)


def run_kernel_case(args):
    """One stage of the path on a smaller mesh (for ncu captures): warm-up once, then run once."""
    import torch

    from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
    from neuralat_b200.bem import meshes as M

    v, t = M.icosphere(args.subdiv, 0.15)
    v = (v * np.random.default_rng(1).uniform(0.7, 1.3, size=3)).astype(np.float32)
    k = M.wavenumber(4000.0)
    g = torch.from_numpy(M.smoothed_gaussian_field(v.shape[0], t, 8, seed=2).astype(np.complex64)).cuda()
    pts = torch.from_numpy(M.sphere_points(256, 0.5, seed=0).astype(np.float32)).cuda()
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    rhs = -cmatmul(V, g)
    for _ in range(2):
        if args.kernel_case == "assemble":
            s.assemble_vk(k)
        elif args.kernel_case == "assemble_bm":
            s.assemble_bm(k)
        elif args.kernel_case == "solve":
            gmres(A, rhs, rtol=1e-6, precision=args.precision)
        else:
            s.boundary2potential(k, g, rhs, pts)
    torch.cuda.synchronize()
    print(f"kernel case {args.kernel_case} subdiv {args.subdiv} N={v.shape[0]} T={t.shape[0]} ok")


def run_batch_case(args):
    """Meshes of subdivision U{2..max} x log-uniform frequencies x 16 RHS x 512
    listeners: the batch runner (one batched assembly launch family per wave,
    concurrent solves on worker streams, autotuned launch shape) against the
    same problems solved one at a time through ``BEM_Solver``."""
    import torch

    from neuralat_b200.bem import BEM_Solver, autotune
    from neuralat_b200.bem import meshes as M
    from neuralat_b200.bem.batch import BatchRunner

    probs, pts = M.batching(n_meshes=args.batch_meshes, n_k=args.batch_k, n_rhs=16,
                            max_subdiv=args.batch_max_subdiv)
    meshes = [(p["vertices"].astype(np.float32), p["triangles"].astype(np.int32)) for p in probs]
    ks = [p["ks"] for p in probs]
    gs = [p["neumann"].astype(np.complex64) for p in probs]
    nprob = sum(len(x) for x in ks)
    pts_d = torch.from_numpy(pts.astype(np.float32)).cuda()

    def one_at_a_time():
        infos = []
        for (v, t), kk, g in zip(meshes, ks, gs):
            s = BEM_Solver(v, t)
            gd = torch.from_numpy(g).cuda()
            for k in kk:
                infos.append({})
                s.solve_and_evaluate(k, gd, pts_d, precision=args.precision, rtol=1e-6, info=infos[-1])
        torch.cuda.synchronize()
        return infos

    tuned = autotune.tune_assembly([BEM_Solver(v, t) for v, t in meshes[:8]], [k[0] for k in ks[:8]], repeats=2)
    runner = BatchRunner(workers=4, precision=args.precision, rtol=1e-6)
    # warm-up: a few problems of every mesh size, so each worker thread has its stream and buffers
    warm, seen = [], {}
    for i, (v, _) in enumerate(meshes):
        if seen.get(v.shape[0], 0) < 4:
            seen[v.shape[0]] = seen.get(v.shape[0], 0) + 1
            warm.append(i)
    runner.run([meshes[i] for i in warm], [ks[i][:1] for i in warm], [gs[i] for i in warm], pts)
    one_at_a_time()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq_infos = one_at_a_time()
    t_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = runner.run(meshes, ks, gs, pts)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    runner.close()
    by_conc = {}
    for w in res.waves:
        c = by_conc.setdefault(str(w["concurrency"]), {"problems": 0, "seconds": 0.0})
        c["problems"] += w["problems"]
        c["seconds"] += w["seconds"]
    line = {
        "case": "batching", "problems": nprob, "meshes": len(meshes),
        "vertices": sorted({int(m[0].shape[0]) for m in meshes}), "rhs": 16, "listeners": int(pts.shape[0]),
        "precision": args.precision, "tuning": {k: tuned[k] for k in ("chunk", "ctas_per_sm")},
        "one_at_a_time_problems_per_s": nprob / t_seq, "batched_problems_per_s": nprob / t_batch,
        "speedup": t_seq / t_batch,
        "max_rel_residual_converged": max((i.get("rel_residual", 0.0) for i in res.info if i.get("status") == 0),
                                          default=None),
        "not_converged": sum(1 for i in res.info if i.get("status") != 0),
        "one_at_a_time_not_converged": sum(1 for i in seq_infos if i.get("status") != 0),
        "waves_by_concurrency": by_conc,
    }
    print(json.dumps(line), flush=True)


def run_large_case(args):
    """One problem of the large multi-RHS configuration through the public API
    (BEM_Solver -> fused assembly -> -V g -> GMRES -> listeners), timed per
    stage with CUDA events after one warm-up problem."""
    import torch

    from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
    from neuralat_b200.bem import meshes as M

    w = M.large_multi_rhs(m=64)
    v = torch.from_numpy(w["vertices"].astype(np.float32)).cuda()
    t = torch.from_numpy(w["triangles"].astype(np.int32)).cuda()
    g = torch.from_numpy(w["neumann"].astype(np.complex64)).cuda()
    pts = torch.from_numpy(w["points"].astype(np.float32)).cuda()
    k = float(w["k"])

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    def problem(info):
        e = [ev()]
        s = BEM_Solver(v, t)
        e.append(ev())
        V, A = s.assemble_vk(k)
        e.append(ev())
        rhs = -cmatmul(V, g)
        del V
        e.append(ev())
        u = gmres(A, rhs, rtol=1e-6, precision=args.precision, info=info)
        e.append(ev())
        p = s.boundary2potential(k, g, u, pts)
        e.append(ev())
        torch.cuda.synchronize()
        problem.last_u = u
        return e, p

    problem({})
    info = {}
    e, p = problem(info)
    u_timed = problem.last_u
    names = ["geometry", "assemble", "rhs", "solve", "eval"]
    stages = {n: e[i].elapsed_time(e[i + 1]) for i, n in enumerate(names)}
    line = {"case": "large_multi_rhs", "N": int(v.shape[0]), "T": int(t.shape[0]), "rhs": int(g.shape[1]),
            "listeners": int(pts.shape[0]), "k": k, "precision": args.precision,
            "s_per_problem": e[0].elapsed_time(e[-1]) / 1e3, "stages_ms": stages,
            "solver": {kk: info.get(kk) for kk in ("iterations", "refinements", "matvecs", "rel_residual", "status")},
            "pressure_finite": bool(torch.isfinite(torch.view_as_real(p)).all()),
            "peak_device_gb": torch.cuda.max_memory_allocated() / 1e9}
    line["validation"] = validate_large(w, v, t, g, pts, k, u_timed, args.precision)
    print(json.dumps(line), flush=True)


CFG5_ROWS = os.path.join(ROOT, "tests", "golden", "cfg5_rows.npz")


def validate_large(w, v, t, g, pts, k, u, precision):
    """Error of the large multi-RHS problem against FP64 references (after the
    timed problem, not timed):
      * rows: 64 seeded rows of V and 1/2 M - K against the FP64 oracle's,
        through 16 random projections per row (tests/golden/cfg5_rows.npz,
        made by tests/golden/make_cfg5_rows.py);
      * per right-hand side, the FP64 residual ||b - A x|| / ||b|| of the
        timed solution against the FP32-stored operator;
      * an analytic monopole at the centre of the same-size sphere without the
        radial noise (icosphere s6, r = 0.2 m, same k): the listener pressures
        against e^{ikr}/(4 pi r) (P1 discretisation error).  On the noisy
        surface itself neighbouring vertices differ in radius by up to 2 cm,
        k x 2 cm ~ 3 rad, so the monopole's surface field is not resolved
        there and its error says nothing about the solver."""
    import torch

    from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
    from neuralat_b200.bem import meshes as M

    out = {}
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    if os.path.exists(CFG5_ROWS):
        f = np.load(CFG5_ROWS)
        if int(f["nv"]) == v.shape[0] and abs(float(f["k"]) - float(np.float32(k))) < 1e-6 * abs(k):
            rows = torch.from_numpy(f["rows"].astype(np.int64)).cuda()
            rng = np.random.default_rng(66)
            nv = v.shape[0]
            Z = (rng.standard_normal((nv, 16)) + 1j * rng.standard_normal((nv, 16))) / np.sqrt(2.0)
            pv = V[rows].cpu().numpy().astype(np.complex128) @ Z
            pa = A[rows].cpu().numpy().astype(np.complex128) @ Z
            out["rows_rel_err"] = {
                "V": float(np.linalg.norm(pv - f["V_proj"]) / np.linalg.norm(f["V_proj"])),
                "half_M_minus_K": float(np.linalg.norm(pa - f["A_proj"]) / np.linalg.norm(f["A_proj"])),
                "rows": int(rows.numel()), "measure": "16 complex Gaussian projections per row, relative Frobenius"}
    b = -cmatmul(V, g)
    # FP64 residual per column, in row blocks (complex128 copies of 4096 rows at a time)
    r2 = torch.zeros(g.shape[1], dtype=torch.float64, device=g.device)
    u64 = u.to(torch.complex128)
    for r0 in range(0, A.shape[0], 4096):
        blk = A[r0:r0 + 4096].to(torch.complex128)
        r2 += ((b[r0:r0 + 4096].to(torch.complex128) - blk @ u64).abs() ** 2).sum(dim=0)
        del blk
    rel = (r2.sqrt() / b.to(torch.complex128).abs().pow(2).sum(dim=0).sqrt()).cpu().numpy()
    out["fp64_residual_per_rhs"] = {"max": float(rel.max()), "median": float(np.median(rel)), "all": rel.tolist()}
    del V, A, s, b, u64
    torch.cuda.empty_cache()
    # analytic monopole (exact for any closed surface around the source)
    vs, ts = M.icosphere(6, 0.2)
    vd = vs.astype(np.float32).astype(np.float64)
    nrm = M.vertex_normals(vd, ts)
    rr = np.linalg.norm(vd, axis=1)
    ikr = 1j * k * rr
    gm = (-np.exp(ikr) / (4 * np.pi * rr ** 3) * (1 - ikr) * np.sum(vd * nrm, axis=1)).astype(np.complex64)
    gm_d = torch.from_numpy(gm).cuda()
    s = BEM_Solver(vs.astype(np.float32), ts)
    V, A = s.assemble_vk(k)
    um = gmres(A, -cmatmul(V, gm_d), rtol=1e-6, precision=precision)
    pm = s.boundary2potential(k, gm_d, um, pts).cpu().numpy()
    pp = pts.cpu().numpy().astype(np.float64)
    rp = np.linalg.norm(pp, axis=1)
    exact = np.exp(1j * k * rp) / (4 * np.pi * rp)
    out["monopole_listener_rel_err"] = float(np.linalg.norm(pm - exact) / np.linalg.norm(exact))
    del V, A
    return out


def run_grad_case(args):
    """Forward and backward time of the differentiable listener pressures
    (neuralat_b200.bem.listener_pressure) on the differentiation workload."""
    import torch

    from neuralat_b200.bem import listener_pressure
    from neuralat_b200.bem import meshes as M

    w = M.differentiation()
    v0 = torch.from_numpy(w["vertices"].astype(np.float32)).cuda()
    t = torch.from_numpy(w["triangles"].astype(np.int32)).cuda()
    g0 = torch.from_numpy(w["neumann"].astype(np.complex64)).cuda()
    pts = torch.from_numpy(w["points"].astype(np.float32)).cuda()
    k = float(w["k"])

    def once():
        v = v0.clone().requires_grad_(True)
        g = g0.clone().requires_grad_(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record()
        p = listener_pressure(v, g, t, pts, k)
        loss = (p.real ** 2 + p.imag ** 2).sum()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), e1.elapsed_time(e2), v.grad, g.grad

    for _ in range(max(args.warmup, 1)):
        once()
    runs = [once() for _ in range(max(args.steps, 1))]
    fwd = float(np.median([r[0] for r in runs]))
    bwd = float(np.median([r[1] for r in runs]))
    vg, gg = runs[-1][2], runs[-1][3]
    line = {"case": "differentiation", "N": int(v0.shape[0]), "T": int(t.shape[0]), "listeners": int(pts.shape[0]),
            "k": k, "forward_ms": fwd, "backward_ms": bwd, "steps": len(runs),
            "grad_finite": bool(torch.isfinite(vg).all() and torch.isfinite(torch.view_as_real(gg)).all()),
            "grad_vertices_norm": float(vg.norm()), "grad_neumann_norm": float(gg.abs().norm())}
    line["fd_check"] = grad_vs_fixture(w, vg.double().cpu().numpy(), gg.cpu().numpy())
    print(json.dumps(line), flush=True)


CFG4_FD = os.path.join(ROOT, "tests", "golden", "cfg4_fd.npz")


def grad_vs_fixture(w, gx, gg):
    """Adjoint gradient against FP64 central differences of the oracle at 64
    seeded vertex coordinates and 16 Neumann entries (tests/golden/cfg4_fd.npz,
    made by tests/golden/make_cfg4_fd.py)."""
    if not os.path.exists(CFG4_FD):
        return {"unavailable": "tests/golden/cfg4_fd.npz missing"}
    f = np.load(CFG4_FD)
    if int(f["nv"]) != gx.shape[0]:
        return {"unavailable": "fixture was made for another workload"}
    adj_v = np.array([gx[a, c] for a, c in f["coords"]])
    adj_g = np.stack([gg[f["neumann_index"]].real, gg[f["neumann_index"]].imag], axis=1)
    return {"fd_rel_err_vertices": float(np.linalg.norm(adj_v - f["fd_vertices"]) / np.linalg.norm(f["fd_vertices"])),
            "fd_rel_err_neumann": float(np.linalg.norm(adj_g - f["fd_neumann"]) / np.linalg.norm(f["fd_neumann"])),
            "coordinates": int(len(f["coords"])), "neumann_entries": int(len(f["neumann_index"])), "bar": 1e-3,
            "step": "1e-4 relative (mesh radius; max |g|), FP64 central differences on the oracle"}


def run_modal_case(args):
    """The reference's multi-mode loop (src/scene.py:384-397) three ways, each
    mode a Burton-Miller solve plus listener evaluation: the reference's
    operator structure on this library's kernels (bm_lhs, bm_rhs and the
    identity assembled separately and combined elementwise, FP32 GMRES), the
    fused assembly per mode (``neumann2dirichlet``), and ``solve_modes``."""
    import torch

    from neuralat_b200.bem import BEM_Solver, solve_linear_equation, solve_modes
    from neuralat_b200.bem import meshes as M

    rng = np.random.default_rng(11)
    v, t = M.icosphere(args.modal_subdiv, 0.15)
    v = (v * rng.uniform(0.7, 1.3, size=3)).astype(np.float32)
    nm = args.modal_modes
    ks = [M.wavenumber(f) for f in np.sort(10.0 ** rng.uniform(np.log10(200.0), np.log10(8000.0), nm))]
    neu = torch.from_numpy(M.smoothed_gaussian_field(v.shape[0], t, nm, seed=3).T.copy().astype(np.complex64)).cuda()
    pts = torch.from_numpy(M.sphere_points(256, 0.5, seed=0).astype(np.float32)).cuda()
    s = BEM_Solver(v, t)

    def operator_path():
        out = []
        for i, k in enumerate(ks):
            Id = s.identity_matrix()
            lhs = (s.assemble_boundary_matrix(k, "bm_lhs", approx=True) + 0.5 * Id).contiguous()
            rhs_m = (s.assemble_boundary_matrix(k, "bm_rhs", approx=True) - (0.5j / k) * Id).contiguous()
            u = solve_linear_equation(lhs, rhs_m @ neu[i])
            out.append(s.boundary2potential(k, neu[i], u, pts))
        return torch.stack(out)

    def fused_loop():
        return torch.stack([s.boundary2potential(k, neu[i], s.neumann2dirichlet(k, neu[i]), pts)
                            for i, k in enumerate(ks)])

    def batched():
        return solve_modes(s, ks, neu, pts)

    times, outs = {}, {}
    for name, fn in (("operator_path", operator_path), ("fused_loop", fused_loop), ("solve_modes", batched)):
        fn()  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs[name] = fn()
        torch.cuda.synchronize()
        times[name] = time.perf_counter() - t0
    ref = outs["operator_path"]
    line = {"case": "modal", "N": int(v.shape[0]), "T": int(t.shape[0]), "modes": nm, "listeners": int(pts.shape[0]),
            "modes_per_s": {k_: nm / t_ for k_, t_ in times.items()},
            "speedup_vs_operator_path": {k_: times["operator_path"] / t_ for k_, t_ in times.items()},
            "max_rel_diff_vs_operator_path": {k_: float(((o - ref).abs().max(dim=1).values /
                                                          ref.abs().max(dim=1).values).max())
                                              for k_, o in outs.items()}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.modal_case:
        run_modal_case(args)
    elif args.grad_case:
        run_grad_case(args)
    elif args.large_case:
        run_large_case(args)
    elif args.batch_case:
        run_batch_case(args)
    elif args.kernel_case:
        run_kernel_case(args)
    elif args.cpu_validate:
        run_cpu_validate(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
