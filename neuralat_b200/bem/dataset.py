"""Acoustic-transfer sample generator in the reference's dataset format.

The reference's audio experiment (experiments/neuPAT_audio/generate.py:75-116)
moves a vibrating object by a random offset next to a static one, draws
listener points on a spherical shell and a log-uniform frequency, solves the
Burton-Miller BIE (``BEM_Solver.neumann2dirichlet``) and stores |p| at the
listeners:

    torch.save({"x": x, "y": y}, path)
    x: (S, P, 5) float32 = (three shell coordinates in [0, 1), the vertical
       displacement fraction, the frequency fraction) per listener
    y: (S, P, 1) float32 = |p| at the listener

This module produces the same tensors on this package's CUDA path.  The
random numbers come from a seeded ``numpy`` generator (the reference draws
from torch's unseeded CUDA generator), so a dataset is reproducible; the
mapping from the uniform draws to positions and frequencies is the
reference's.  The meshes and the solver settings are arguments (the
reference reads them from a dataset directory that is not part of it).
With ``batch_size`` the samples go through the batch runner in groups (the
Burton-Miller matrices of a group assembled in one launch family, the solves
on concurrent streams); the draws and the outputs are the same.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .batch import shared_runner
from .solver import BEM_Solver

SPEED_OF_SOUND = 343.2  # generate.py:99


def shell_points(base: np.ndarray, bbox_center, bbox_r: float, r_max: float) -> np.ndarray:
    """Listener positions from uniform draws base (P, 3) in [0, 1)
    (generate.py:85-94): radius in [bbox_r, r_max * bbox_r], azimuth in
    [-pi, pi), polar angle in [0, pi)."""
    base = np.asarray(base, np.float64)
    rs = (base[:, 0] * (r_max - 1.0) + 1.0) * bbox_r
    theta = base[:, 1] * 2.0 * math.pi - math.pi
    phi = base[:, 2] * math.pi
    c = np.asarray(bbox_center, np.float64)
    return np.stack([rs * np.sin(phi) * np.cos(theta) + c[0], rs * np.sin(phi) * np.sin(theta) + c[1],
                     rs * np.cos(phi) + c[2]], axis=-1)


def log_frequency(fraction: float, freq_min: float, freq_max: float) -> float:
    """Frequency from a uniform draw in [0, 1), log-uniform in [freq_min, freq_max] (generate.py:96-99)."""
    lo, hi = math.log10(freq_min), math.log10(freq_max)
    return 10.0 ** (fraction * (hi - lo) + lo)


def generate_audio_samples(vib_vertices, vib_triangles, static_vertices, static_triangles, *, src_pos_min,
                           src_pos_max, bbox_center, bbox_r: float, r_max: float, freq_min: float = 100.0,
                           freq_max: float = 10000.0, trg_sample_num: int = 1000, src_sample_num: int = 1000,
                           vib_neumann=None, seed: int = 0, device=None, solve_kw: dict | None = None,
                           batch_size: int = 0, workers: int = 4):
    """Return {"x": (S, P, 5) float32, "y": (S, P, 1) float32} as the reference writes them.

    vib_neumann: (Nv,) normal velocity of the vibrating object (default 1
    everywhere; the reference zeroes part of its specific mesh); the static
    object is rigid (0).  solve_kw: options of ``neumann2dirichlet`` (the
    linear solver's tolerance, precision, ...).  batch_size > 0: solve the
    samples in groups of that size through the batch runner (GMRES with the
    relative stopping test sqrt(tol) of ``solve_linear_equation``; ``nsteps``,
    ``precision`` and ``restart`` as there)."""
    device = torch.device("cuda") if device is None else torch.device(device)
    vv = np.asarray(vib_vertices, np.float32)
    vt = np.asarray(vib_triangles, np.int32)
    sv = np.asarray(static_vertices, np.float32)
    st = np.asarray(static_triangles, np.int32)
    nvib = vv.shape[0]
    triangles = torch.from_numpy(np.concatenate([vt, st + nvib], axis=0)).to(device)
    neu = np.ones(nvib, np.complex64) if vib_neumann is None else np.asarray(vib_neumann, np.complex64)
    neumann = torch.from_numpy(np.concatenate([neu, np.zeros(sv.shape[0], np.complex64)])).to(device)
    lo = np.asarray(src_pos_min, np.float64)
    hi = np.asarray(src_pos_max, np.float64)
    rng = np.random.default_rng(seed)
    S, P = int(src_sample_num), int(trg_sample_num)
    x = torch.zeros(S, P, 5, dtype=torch.float32)
    y = torch.zeros(S, P, 1, dtype=torch.float32)
    static_d = torch.from_numpy(sv).to(device)
    if batch_size and batch_size > 0:
        kw = dict(solve_kw or {})
        if kw.get("solver", "gmres") != "gmres":
            raise ValueError("batched generation solves with GMRES")
        tri_np = np.concatenate([vt, st + nvib], axis=0)
        with torch.cuda.device(device):
            runner = shared_runner(workers=workers, precision=kw.get("precision", "fp32"),
                                   rtol=math.sqrt(max(float(kw.get("tol", 1e-10)), 0.0)),
                                   restart=int(kw.get("restart", 200)), max_iters=int(kw.get("nsteps", 500)),
                                   formulation="burton_miller")
            for b0 in range(0, S, batch_size):
                meshes, ks, pts = [], [], []
                for i in range(b0, min(S, b0 + batch_size)):
                    src_base = rng.random(3)
                    displacement = src_base * (hi - lo) + lo
                    base = rng.random((P, 3))
                    freq_base = float(rng.random())
                    meshes.append((np.concatenate([(vv + displacement).astype(np.float32), sv]), tri_np))
                    pts.append(shell_points(base, bbox_center, bbox_r, r_max).astype(np.float32))
                    ks.append([2.0 * math.pi * log_frequency(freq_base, freq_min, freq_max) / SPEED_OF_SOUND])
                    x[i, :, :3] = torch.from_numpy(base.astype(np.float32))
                    x[i, :, 3] = float(src_base[1])
                    x[i, :, 4] = freq_base
                res = runner.run(meshes, ks, [neumann] * len(meshes), pts)
                for (mi, _), p in zip(res.index, res.pressure):
                    y[b0 + mi, :, 0] = p[:, 0].abs().cpu()
        return {"x": x, "y": y}
    for i in range(S):
        src_base = rng.random(3)
        displacement = src_base * (hi - lo) + lo
        vertices = torch.cat([torch.from_numpy((vv + displacement).astype(np.float32)).to(device), static_d])
        base = rng.random((P, 3))
        points = torch.from_numpy(shell_points(base, bbox_center, bbox_r, r_max).astype(np.float32)).to(device)
        freq_base = float(rng.random())
        k = 2.0 * math.pi * log_frequency(freq_base, freq_min, freq_max) / SPEED_OF_SOUND
        x[i, :, :3] = torch.from_numpy(base.astype(np.float32))
        x[i, :, 3] = float(src_base[1])
        x[i, :, 4] = freq_base
        solver = BEM_Solver(vertices.contiguous(), triangles)
        dirichlet = solver.neumann2dirichlet(k, neumann, **(solve_kw or {}))
        p = solver.boundary2potential(k, neumann, dirichlet, points)
        y[i, :, 0] = p.abs().cpu()
    return {"x": x, "y": y}


def save_audio_dataset(path: str, data: dict) -> None:
    """Write the samples as the reference does (generate.py:116)."""
    torch.save({"x": data["x"], "y": data["y"]}, path)
