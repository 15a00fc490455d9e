"""Autotuner for the assembly launch shape.

Times the batched fused assembly (``bem_batch_matrices_vk``) of a sample of
problems for every candidate (used (test group, trial tile) units per work
item, persistent CTAs per SM), keeps the fastest, and installs it with ``bem_set_tuning``.  Results are
cached per GPU model and problem-size signature in a JSON file
(``$NEURALAT_B200_CACHE`` or ``~/.cache/neuralat_b200/autotune.json``), so a
later process reuses them without re-timing.
"""
from __future__ import annotations

import json
import os

import torch

from .. import _lib as L
from .batch import assemble_batch

CHUNKS = (2, 4, 8, 16, 32, 64)
CTAS = (1, 2)  # persistent CTAs per SM of the symmetric regular-pair kernel (at most two fit)


def _cache_path() -> str:
    base = os.environ.get("NEURALAT_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "neuralat_b200")
    return os.path.join(base, "autotune.json")


def _signature(solvers) -> str:
    sizes = sorted(s.geometry.nt for s in solvers)
    gpu = torch.cuda.get_device_name()
    bucket = [1 << max(0, (n - 1).bit_length()) for n in sizes]
    return f"{gpu}|asm-sym|{len(sizes)}|{bucket[0]}-{bucket[-1]}"


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def apply(config) -> None:
    lib = L.lib()
    L.check(lib.bem_set_tuning(L.TUNE_ASSEMBLY_CHUNK, int(config["chunk"])), "bem_set_tuning")
    L.check(lib.bem_set_tuning(L.TUNE_ASSEMBLY_CTAS_PER_SM, int(config["ctas_per_sm"])), "bem_set_tuning")


def tune_assembly(solvers, ks, repeats: int = 2, use_cache: bool = True, verbose: bool = False) -> dict:
    """Pick the fastest (chunk, ctas_per_sm) for batched assembly of these problems."""
    key = _signature(solvers)
    cache = _load() if use_cache else {}
    if key in cache:
        apply(cache[key])
        return dict(cache[key], cached=True)
    timings = []
    for ctas in CTAS:
        for chunk in CHUNKS:
            apply({"chunk": chunk, "ctas_per_sm": ctas})
            assemble_batch(solvers, ks)  # warm-up
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                mats = assemble_batch(solvers, ks)
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
                del mats
            timings.append((best, chunk, ctas))
            if verbose:
                print(f"autotune chunk={chunk:2d} ctas/SM={ctas}: {best:8.3f} ms", flush=True)
    best_ms, chunk, ctas = min(timings)
    config = {"chunk": chunk, "ctas_per_sm": ctas, "ms": best_ms}
    apply(config)
    cache = _load()
    cache[key] = config
    _store(cache)
    return dict(config, cached=False, timings=[list(t) for t in timings])


def reset() -> None:
    apply({"chunk": 0, "ctas_per_sm": 0})
