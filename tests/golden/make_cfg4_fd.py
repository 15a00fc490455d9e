"""Central finite differences of the listener loss on the differentiation workload (fixture generator).

Workload: icosphere s4 (N = 2562, T = 5120), r = 0.1 m, k at 2 kHz, one
smoothed complex Gaussian Neumann field, 128 listeners on a 0.5 m sphere
(``neuralat_b200.bem.meshes.differentiation``); loss L = sum |p|^2 of the
listener pressures of the reference's CBIE + ``boundary2potential``
(src/bem/solver.py:97-104,140-147).

On the FP64 CPU oracle (``oracle.ListenerLoss``: base LU factorisation plus
an exact low-rank update for each moved vertex), this writes
  * dL/dx at 64 seeded vertex coordinates, central differences with a step
    of 1e-4 relative to the mesh radius;
  * dL/d(Re g_j), dL/d(Im g_j) at 16 seeded Neumann entries, step 1e-4
    relative to max |g|.
The inputs are the float32 values the GPU path receives.  The adjoint
gradient of ``neuralat_b200.bem.listener_pressure`` is compared with these
values by tests/test_gpu_adjoint.py and by ``bench.py --grad-case``.

Usage:  python tests/golden/make_cfg4_fd.py [out.npz]   (default tests/golden/cfg4_fd.npz)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DEFAULT_OUT = os.path.join(HERE, "cfg4_fd.npz")
RADIUS = 0.1
N_COORDS, N_NEUMANN = 64, 16


def workload_f32():
    from neuralat_b200.bem import meshes as M

    w = M.differentiation()
    return (w["vertices"].astype(np.float32), w["triangles"].astype(np.int32), np.float32(w["k"]),
            w["neumann"].astype(np.complex64), w["points"].astype(np.float32))


def coordinates(nv):
    rng = np.random.default_rng(64)
    coords = np.stack([rng.integers(nv, size=N_COORDS), rng.integers(3, size=N_COORDS)], axis=1)
    nidx = np.random.default_rng(16).choice(nv, N_NEUMANN, replace=False)
    return coords.astype(np.int64), nidx.astype(np.int64)


def main(out=DEFAULT_OUT):
    from oracle import oracle as O

    v, t, k, g, pts = workload_f32()
    t0 = time.perf_counter()
    F = O.ListenerLoss(v.astype(np.float64), t, float(k), g.astype(np.complex128), pts.astype(np.float64))
    t1 = time.perf_counter()
    coords, nidx = coordinates(v.shape[0])
    h = 1e-4 * RADIUS
    fd_v = np.array([(F.vertex_loss(a, c, h) - F.vertex_loss(a, c, -h)) / (2 * h) for a, c in coords])
    t2 = time.perf_counter()
    hg = 1e-4 * float(np.abs(g).max())
    fd_g = np.array([[(F.neumann_loss(j, hg * unit) - F.neumann_loss(j, -hg * unit)) / (2 * hg) for unit in (1.0, 1j)]
                     for j in nidx])
    np.savez_compressed(out, loss=np.float64(F.loss), coords=coords, fd_vertices=fd_v, neumann_index=nidx,
                        fd_neumann=fd_g, step_vertices=np.float64(h), step_neumann=np.float64(hg),
                        k=np.float64(k), nv=np.int64(v.shape[0]), nt=np.int64(t.shape[0]),
                        vertex_checksum=np.float64(np.abs(v.astype(np.float64)).sum()))
    print(f"wrote {out}: base {t1 - t0:.1f} s, {len(coords)} vertex coordinates {t2 - t1:.1f} s, "
          f"{O.num_threads()} threads")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_OUT)
