"""Fused Burton-Miller assembly and the multi-mode solve.

``bem_boundary_matrices_bm`` computes both matrices of the reference's
``neumann2dirichlet`` (src/bem/solver.py:118-126) in one pass:
lhs = bm_lhs_approx + 1/2 I and rhs = bm_rhs_approx - (i/(2k)) I.  Checked
against the reference's own kernels (golden fixtures), the FP64 oracle and
the per-operator path; the batched assembly against the single one;
``solve_modes`` against the reference's per-mode loop (src/scene.py:384-397).
"""
import glob
import os

import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, solve_modes
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.batch import assemble_batch_bm
from neuralat_b200.bem.solver import _stream
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "reference_*.npz")))


def relfro(a, b):
    a = a.cpu().numpy() if torch.is_tensor(a) else a
    b = b.cpu().numpy() if torch.is_tensor(b) else b
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def ellipsoid(sub=2, scale=(1.25, 0.75, 1.0)):
    v, t = M.icosphere(sub, 0.15)
    return (v * np.array(scale)).astype(np.float32), t.astype(np.int32)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(f) for f in GOLDEN])
def test_fused_bm_matches_reference_kernels(path):
    z = dict(np.load(path))
    s = BEM_Solver(z["vertices"], z["triangles"])
    I = z["identity"]
    for ki, k in enumerate(z["ks"]):
        lhs, rhs = s.assemble_bm(float(k))
        # the golden matrices are the reference's FP32 kernels (atomics); 3e-5 as for every operator
        assert relfro(lhs, z[f"k{ki}_bm_lhs_approx"] + 0.5 * I) <= 3e-5, k
        assert relfro(rhs, z[f"k{ki}_bm_rhs_approx"] - (0.5j / k) * I) <= 3e-5, k


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(f) for f in GOLDEN])
def test_fused_exact_order_is_the_reference_hbie_system(path):
    """<4,6>: lhs = 1/2 I - K + (i/k) W, rhs = -V - (i/k)(K' + 1/2 I) from the
    reference's own kernels (solver.py:106-116); <2,1> against its bm_*_approx_1."""
    z = dict(np.load(path))
    s = BEM_Solver(z["vertices"], z["triangles"])
    I = z["identity"]
    for ki, k in enumerate(z["ks"]):
        beta = 1j / k
        lhs, rhs = s.assemble_bm(float(k), approx=False)
        ref_l = 0.5 * I - z[f"k{ki}_double"] + beta * z[f"k{ki}_hypersingular"]
        ref_r = -z[f"k{ki}_single"] - beta * (z[f"k{ki}_adjointdouble"] + 0.5 * I)
        assert relfro(lhs, ref_l) <= 3e-5, k
        assert relfro(rhs, ref_r) <= 3e-5, k
        lhs1, rhs1 = s.assemble_bm(float(k), approx="1")
        assert relfro(lhs1, z[f"k{ki}_bm_lhs_approx_1"] + 0.5 * I) <= 3e-5, k
        assert relfro(rhs1, z[f"k{ki}_bm_rhs_approx_1"] - (0.5j / k) * I) <= 3e-5, k


@pytest.mark.parametrize("k", [18.3, -100.6])
def test_fused_exact_order_matches_oracle(k):
    v, t = ellipsoid(2)
    s = BEM_Solver(v, t)
    vd = v.astype(np.float64)
    I = O.identity_matrix(vd, t)
    beta = 1j / k
    lhs, rhs = s.assemble_bm(k, approx=False)
    ref_l = 0.5 * I - O.boundary_matrix("double", vd, t, k) + beta * O.boundary_matrix("hypersingular", vd, t, k)
    ref_r = -O.boundary_matrix("single", vd, t, k) - beta * (O.boundary_matrix("adjointdouble", vd, t, k) + 0.5 * I)
    assert relfro(lhs, ref_l) <= 1e-5
    assert relfro(rhs, ref_r) <= 1e-5
    (lb, rb), = assemble_batch_bm([s], [k], approx=False)
    assert relfro(lb, lhs) <= 1e-6 and relfro(rb, rhs) <= 1e-6


@pytest.mark.parametrize("k", [18.3, 73.27, -100.6])
def test_fused_bm_matches_oracle_and_operator_path(k):
    v, t = ellipsoid(2)
    s = BEM_Solver(v, t)
    lhs, rhs = s.assemble_bm(k)
    vd = v.astype(np.float64)
    I = O.identity_matrix(vd, t)
    assert relfro(lhs, O.boundary_matrix("bm_lhs", vd, t, k, approx="_approx") + 0.5 * I) <= 1e-5
    assert relfro(rhs, O.boundary_matrix("bm_rhs", vd, t, k, approx="_approx") - (0.5j / k) * I) <= 1e-5
    Id = s.identity_matrix()
    sep_l = s.assemble_boundary_matrix(k, "bm_lhs", approx=True) + 0.5 * Id
    sep_r = s.assemble_boundary_matrix(k, "bm_rhs", approx=True) - (0.5j / k) * Id
    assert relfro(lhs, sep_l) <= 1e-5
    assert relfro(rhs, sep_r) <= 1e-5
    assert L.lib().bem_assembly_status(_stream(s.device)) == L.BEM_OK


def test_fused_bm_larger_mesh_matches_operator_path():
    v, t = ellipsoid(4, (1.1, 0.9, 1.0))  # 5120 triangles: many tiles and work-item boundaries
    s = BEM_Solver(v, t)
    k = 60.0
    lhs, rhs = s.assemble_bm(k)
    Id = s.identity_matrix()
    sep_l = s.assemble_boundary_matrix(k, "bm_lhs", approx=True) + 0.5 * Id
    assert relfro(lhs, sep_l) <= 1e-5
    del sep_l
    sep_r = s.assemble_boundary_matrix(k, "bm_rhs", approx=True) - (0.5j / k) * Id
    assert relfro(rhs, sep_r) <= 1e-5


def test_batched_bm_matches_single():
    meshes = [ellipsoid(1), ellipsoid(3, (0.9, 1.2, 1.0)), ellipsoid(2)]
    solvers = [BEM_Solver(v, t) for v, t in meshes]
    ks = [40.0, -73.3, 11.0]
    out = assemble_batch_bm(solvers, ks)
    for s, k, (lhs, rhs) in zip(solvers, ks, out):
        l1, r1 = s.assemble_bm(k)
        assert relfro(lhs, l1) <= 1e-6
        assert relfro(rhs, r1) <= 1e-6


def test_zero_wavenumber_rejected():
    v, t = ellipsoid(1)
    s = BEM_Solver(v, t)
    with pytest.raises(L.BEMError) as e:
        s.assemble_bm(0.0)
    assert e.value.status == L.BEM_ERR_INVALID_ARGUMENT


def test_neumann2dirichlet_fused_equals_operator_path():
    v, t = ellipsoid(3)
    s = BEM_Solver(v, t)
    k = 50.0
    g = torch.from_numpy(M.smoothed_gaussian_field(v.shape[0], t, 3, seed=2)[:, 0].astype(np.complex64)).cuda()
    u = s.neumann2dirichlet(k, g, tol=1e-14)
    Id = s.identity_matrix()
    lhs = (s.assemble_boundary_matrix(k, "bm_lhs", approx=True) + 0.5 * Id).cpu().numpy().astype(np.complex128)
    rhs = (s.assemble_boundary_matrix(k, "bm_rhs", approx=True) - (0.5j / k) * Id).cpu().numpy().astype(np.complex128)
    u_ref = np.linalg.solve(lhs, rhs @ g.cpu().numpy().astype(np.complex128))
    assert relfro(u.cpu().numpy(), u_ref) <= 5e-5  # matrices agree to ~1e-6; the system is well conditioned


@pytest.mark.parametrize("precision", ["fp32", "fp16x3"])
def test_solve_modes_matches_per_mode_loop(precision):
    v, t = ellipsoid(3, (1.0, 0.8, 1.2))
    s = BEM_Solver(v, t)
    rng = np.random.default_rng(5)
    ks = [M.wavenumber(f) for f in (300.0, 900.0, 2500.0, 4100.0, 7000.0)]
    fields = M.smoothed_gaussian_field(v.shape[0], t, 3, seed=7)
    neu = np.stack([fields[:, i % fields.shape[1]] * (1 + 0.1 * rng.standard_normal()) for i in range(len(ks))])
    neu_d = torch.from_numpy(neu.astype(np.complex64)).cuda()
    pts = torch.from_numpy(M.sphere_points(96, 1.0, seed=4).astype(np.float32)).cuda()
    info = []
    p = solve_modes(s, ks, neu_d, pts, precision=precision, rtol=1e-7, workers=3, info=info)
    assert p.shape == (len(ks), pts.shape[0])
    assert all(i["status"] == 0 for i in info)
    for i, k in enumerate(ks):  # src/scene.py:387-393
        u = s.neumann2dirichlet(k, neu_d[i], tol=1e-14)
        p1 = s.boundary2potential(k, neu_d[i], u, pts)
        assert relfro(p[i], p1) <= 1e-5, (i, k)


def test_solve_modes_vs_oracle():
    """EditableModalSound.solve's loop (src/scene.py:384-397) through
    solve_modes against the FP64 oracle: per mode the <2,3> Burton-Miller
    system (bm_lhs + 1/2 M) u = (bm_rhs - (i/2k) M) g solved densely
    (solver.py:118-126), then the listener pressures (solver.py:140-147)."""
    v, t = ellipsoid(2, (1.0, 0.8, 1.2))
    vd = v.astype(np.float32).astype(np.float64)
    s = BEM_Solver(v, t)
    ks = [M.wavenumber(f) for f in (400.0, 2500.0, 6000.0)]
    neu = M.smoothed_gaussian_field(v.shape[0], t, 3, seed=8).T.astype(np.complex64)
    pts = M.sphere_points(40, 1.0, seed=6).astype(np.float32)
    p = solve_modes(s, ks, torch.from_numpy(neu).cuda(), torch.from_numpy(pts).cuda(), precision="fp32", rtol=1e-7,
                    workers=2)
    I = O.identity_matrix(vd, t)
    for i, k in enumerate(ks):
        k32 = float(np.float32(k))
        lhs = O.boundary_matrix("bm_lhs", vd, t, k32, approx="_approx") + 0.5 * I
        rhs = O.boundary_matrix("bm_rhs", vd, t, k32, approx="_approx") - (0.5j / k32) * I
        g = neu[i].astype(np.complex128)
        u = np.linalg.solve(lhs, rhs @ g)
        p_ref = O.boundary2potential(vd, t, k32, g, u, pts)
        assert relfro(p[i].cpu().numpy(), p_ref) <= 1e-4, (i, k)


def test_high_frequency_assembly_accuracy():
    """10 kHz on an r = 0.3 m ellipsoid (k r up to ~130): the fused V/K and
    Burton-Miller kernels (fast sincos of k r) stay within 1e-5 of the FP64
    oracle; the error grows with k r like the FP32 rounding of k r itself."""
    v, t = M.icosphere(3, 0.3)
    v = (v * np.array([1.2, 0.9, 1.0])).astype(np.float32)
    vd = v.astype(np.float64)
    k = M.wavenumber(10000.0)
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    I = O.identity_matrix(vd, t)
    assert relfro(V, O.boundary_matrix("single", vd, t, k)) <= 1e-5
    assert relfro(A, 0.5 * I - O.boundary_matrix("double", vd, t, k)) <= 1e-5
    lhs, rhs = s.assemble_bm(k)
    assert relfro(lhs, O.boundary_matrix("bm_lhs", vd, t, k, approx="_approx") + 0.5 * I) <= 1e-5
    assert relfro(rhs, O.boundary_matrix("bm_rhs", vd, t, k, approx="_approx") - (0.5j / k) * I) <= 1e-5
