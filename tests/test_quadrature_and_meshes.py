"""Quadrature rules, mesh generators and host-side helpers (CPU only)."""
import math

import numpy as np
import pytest
import torch

from neuralat_b200.bem import BiCGSTAB
from neuralat_b200.bem import meshes as M
from oracle import oracle as O


@pytest.mark.parametrize("s", [0, 1, 2, 3])
def test_icosphere_counts_and_orientation(s):
    v, t = M.icosphere(s, 0.3)
    assert v.shape == (10 * 4 ** s + 2, 3) and t.shape == (20 * 4 ** s, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 0.3)
    p0, p1, p2 = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    n = np.cross(p1 - p0, p2 - p0)
    assert (np.einsum("ij,ij->i", n, p0 + p1 + p2) > 0).all()  # outward
    # closed 2-manifold: every edge shared by exactly two triangles
    e = np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert (cnt == 2).all()


def test_mass_matrix_closed_form():
    """P1 mass on a triangle: area/12 * (1 + delta_ab); 6-point rule is exact."""
    v, t = M.icosphere(1, 0.5)
    Mo = O.identity_matrix(v, t).real
    ref = np.zeros_like(Mo)
    for tri in t:
        p = v[tri]
        area = 0.5 * np.linalg.norm(np.cross(p[1] - p[0], p[2] - p[0]))
        for a in range(3):
            for b in range(3):
                ref[tri[a], tri[b]] += area / 12.0 * (2.0 if a == b else 1.0)
    assert np.abs(Mo - ref).max() < 1e-14


def test_triangle_rule_exact_for_degree_four():
    """Oracle potential of a constant density is the area-weighted rule; check
    the 6-point rule integrates x^a y^b (a+b<=4) on the unit triangle exactly."""
    import ctypes  # noqa: F401
    r10 = math.sqrt(10.0)
    tt = math.sqrt(38.0 - 44.0 * math.sqrt(2.0 / 5.0))
    a1, a2 = (8 - r10 + tt) / 18, (8 - r10 - tt) / 18
    w1 = (620 + math.sqrt(213125 - 53320 * r10)) / 3720
    w2 = (620 - math.sqrt(213125 - 53320 * r10)) / 3720
    pts = [(a1, a1), (1 - 2 * a1, a1), (a1, 1 - 2 * a1), (a2, a2), (1 - 2 * a2, a2), (a2, 1 - 2 * a2)]
    ws = [w1] * 3 + [w2] * 3
    for a in range(5):
        for b in range(5 - a):
            q = sum(w * x ** a * y ** b for w, (x, y) in zip(ws, pts)) * 0.5
            exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
            assert abs(q - exact) < 1e-14


def test_oracle_monopole_known_answer():
    v, t = M.icosphere(2, 0.1)
    k = M.wavenumber(1000.0)
    g = O.monopole_neumann(v, M.vertex_normals(v, t), k)
    u = O.cbie_solve(v, t, k, g)
    assert np.linalg.norm(u - O.monopole(v, k)) / np.linalg.norm(O.monopole(v, k)) < 3e-2


def test_smoothed_field_is_smooth_and_seeded():
    v, t = M.icosphere(2, 1.0)
    a = M.smoothed_gaussian_field(v.shape[0], t, 3, seed=4)
    b = M.smoothed_gaussian_field(v.shape[0], t, 3, seed=4)
    assert a.shape == (v.shape[0], 3) and np.array_equal(a, b)
    raw = np.random.default_rng(4).standard_normal((v.shape[0], 3))
    assert np.std(a.real) < np.std(raw)


def test_bicgstab_matches_dense_solve_on_cpu():
    """The reference-parity BiCGSTAB (unconjugated dots) is generic torch code."""
    rng = np.random.default_rng(0)
    n = 60
    A = (np.eye(n) * 3 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n))
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    At = torch.from_numpy(A)
    x = BiCGSTAB(lambda z: At @ z, device="cpu").solve(torch.from_numpy(b), nsteps=200, tol=1e-24, atol=0.0)
    assert np.linalg.norm(x.numpy() - np.linalg.solve(A, b)) / np.linalg.norm(np.linalg.solve(A, b)) < 1e-10


def test_named_workloads_shapes():
    w = M.plain_small()
    assert w["vertices"].shape == (642, 3) and w["points"].shape == (256, 3)
    assert abs(w["k"] - 2 * math.pi * 1000 / 343) < 1e-12
