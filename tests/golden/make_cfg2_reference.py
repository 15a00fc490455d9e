"""FP64 listener pressures of the 20 480-triangle precision workload (fixture generator).

Runs the FP64 CPU oracle (``oracle/oracle.py``) once on the exact benchmark
workload of ``bench.py`` -- icosphere s5 (N = 10 242, T = 20 480), r = 0.15 m
with axes scaled by seeded U[0.7, 1.3], k at 4 kHz, 8 smoothed complex
Gaussian Neumann fields, 256 listeners on a 0.5 m sphere -- and writes the
256 x 8 listener pressures p = -S g + D u, u the dense FP64 solution of the
CBIE (1/2 M - K) u = -V g (the reference's ``BEM_Solver.CBIE`` and
``boundary2potential``, src/bem/solver.py:97-104,140-147).

The inputs are the float32 values the GPU path receives (vertices, Neumann
data, listener points and the wavenumber rounded to float32, then widened),
so the fixture isolates the GPU path's arithmetic error.  ``bench.py`` reads
the fixture after its timed region and reports the listener error of both the
mixed-precision and the plain-FP32 pipeline against it.

Usage:  python tests/golden/make_cfg2_reference.py [out.npz]
        (default tests/golden/cfg2_pressures.npz; ~5-10 minutes on 8 cores)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DEFAULT_OUT = os.path.join(HERE, "cfg2_pressures.npz")


def workload_f32():
    """The benchmark inputs exactly as the GPU path sees them (float32 / complex64)."""
    from neuralat_b200.bem import meshes as M

    w = M.precision_large(m=8)
    return (w["vertices"].astype(np.float32), w["triangles"].astype(np.int32), np.float32(w["k"]),
            w["neumann"].astype(np.complex64), w["points"].astype(np.float32))


def main(out=DEFAULT_OUT):
    from oracle import oracle as O

    v, t, k, g, pts = workload_f32()
    v64, k64 = v.astype(np.float64), float(k)
    t0 = time.perf_counter()
    u = O.cbie_solve(v64, t, k64, g.astype(np.complex128))
    t1 = time.perf_counter()
    p = O.boundary2potential(v64, t, k64, g.astype(np.complex128), u, pts.astype(np.float64))
    t2 = time.perf_counter()
    np.savez_compressed(out, pressures=p, k=np.float64(k64), nv=np.int64(v.shape[0]), nt=np.int64(t.shape[0]),
                        vertex_checksum=np.float64(np.abs(v64).sum()),
                        neumann_checksum=np.float64(np.abs(g.astype(np.complex128)).sum()),
                        u_norms=np.linalg.norm(u, axis=0))
    print(f"wrote {out}: p {p.shape}, solve {t1 - t0:.1f} s, listeners {t2 - t1:.1f} s, "
          f"{O.num_threads()} threads")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_OUT)
