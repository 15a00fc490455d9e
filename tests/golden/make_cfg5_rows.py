"""Sampled rows of the s6 operators, as random projections (fixture generator).

Workload: icosphere s6 (N = 40 962, T = 81 920) with 5 % seeded radial noise,
r = 0.2 m, k at 8 kHz (``neuralat_b200.bem.meshes.large_multi_rhs``).  One
complex64 operator is 13.4 GB here and its FP64 counterpart does not fit in
host memory, so the FP64 oracle assembles only 64 seeded rows of V and of the
CBIE left-hand side 1/2 M - K (src/bem/solver.py:97-104), and the fixture
keeps each row's projections onto 16 seeded complex Gaussian vectors Z
(N x 16) plus the row norms: a checksum of every row entry whose relative
error estimates the rows' relative Frobenius error.

The mass rows use the closed form of the P1 mass matrix (the 6-point rule
integrates phi_a phi_b exactly: M_ab = sum over triangles holding a and b of
area (1 + [a = b]) / 12), checked here against the oracle's
``identity_matrix`` on a small mesh first.

Usage:  python tests/golden/make_cfg5_rows.py [out.npz]   (default tests/golden/cfg5_rows.npz)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DEFAULT_OUT = os.path.join(HERE, "cfg5_rows.npz")
N_ROWS, N_PROJ = 64, 16


def sample_rows(nv):
    return np.sort(np.random.default_rng(65).choice(nv, N_ROWS, replace=False)).astype(np.int32)


def projection_vectors(nv):
    rng = np.random.default_rng(66)
    return (rng.standard_normal((nv, N_PROJ)) + 1j * rng.standard_normal((nv, N_PROJ))) / np.sqrt(2.0)


def mass_rows(v, t, rows):
    """Rows of the P1 mass matrix, closed form (exact for the 6-point rule)."""
    v = np.asarray(v, np.float64)
    area = 0.5 * np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1)
    slot = -np.ones(v.shape[0], np.int64)
    slot[rows] = np.arange(len(rows))
    out = np.zeros((len(rows), v.shape[0]))
    for a in range(3):
        ra = slot[t[:, a]]
        for b in range(3):
            sel = ra >= 0
            np.add.at(out, (ra[sel], t[sel, b]), area[sel] * (2.0 if a == b else 1.0) / 12.0)
    return out


def main(out=DEFAULT_OUT):
    from neuralat_b200.bem import meshes as M
    from oracle import oracle as O

    # the closed-form mass rows equal the oracle's mass matrix
    vs, ts = M.icosphere(2, 0.2)
    rs = np.arange(0, vs.shape[0], 7).astype(np.int32)
    ref = O.identity_matrix(vs, ts)[rs]
    assert np.abs(mass_rows(vs, ts, rs) - ref).max() <= 1e-12 * np.abs(ref).max()

    w = M.large_multi_rhs(m=1)
    v = w["vertices"].astype(np.float32).astype(np.float64)
    t = w["triangles"].astype(np.int32)
    k = float(np.float32(w["k"]))
    rows = sample_rows(v.shape[0])
    Z = projection_vectors(v.shape[0])
    t0 = time.perf_counter()
    Vr = O.boundary_matrix("single", v, t, k, rows=rows)
    Ar = 0.5 * mass_rows(v, t, rows) - O.boundary_matrix("double", v, t, k, rows=rows)
    t1 = time.perf_counter()
    np.savez_compressed(out, rows=rows, V_proj=Vr @ Z, A_proj=Ar @ Z, V_row_norms=np.linalg.norm(Vr, axis=1),
                        A_row_norms=np.linalg.norm(Ar, axis=1), k=np.float64(k), nv=np.int64(v.shape[0]),
                        nt=np.int64(t.shape[0]), vertex_checksum=np.float64(np.abs(v).sum()))
    print(f"wrote {out}: {rows.size} rows of V and 1/2 M - K in {t1 - t0:.1f} s, {O.num_threads()} threads")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_OUT)
