"""Failure detection and robustness on the GPU, through the C ABI.

The reference reports no errors at all: a NaN right-hand side or an
iteration cap ends BiCGSTAB silently (src/bem/BiCGSTAB.py:106), and its
singular-pair kernel keeps the touching triangles of a vertex in a fixed
`__shared__ int adj[64]` (src/bem/cuda/bind.cu:83), which a vertex shared by
more than 64 triangles overflows.  Here:
  * a non-finite right-hand side is reported as BEM_ERR_NONFINITE and an
    iteration cap as BEM_ERR_NOT_CONVERGED (with the solver info filled), and
    the context stays usable for the next solve;
  * the geometry status word (bounded waits of the assembly kernels) and the
    process-wide flag read clean after ordinary assemblies;
  * a geometry workspace whose address was released is read from the device
    again, so a buffer that holds no geometry is refused (BEM_ERR_WORKSPACE);
  * a fan mesh with a vertex of valence 80 assembles and solves like the FP64
    oracle (touching pairs come from exact host-built lists, no cap);
  * the normals and surface curls of the geometry equal the reference's own
    preprocess output (tests/golden/reference_*.npz);
  * batch budgets that cannot be met raise MemoryError before any matrix is
    allocated.
No test here faults or hangs the GPU: every failure is made on the host
(invalid data, a cap, a released address).
"""
import ctypes
import glob
import os

import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.batch import BatchRunner
from neuralat_b200.bem.solver import _stream, _vp
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "reference_*.npz")))


def relfro(a, b):
    a = a.cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def small():
    v, t = M.icosphere(2, 0.1)
    v = (v * np.array([1.2, 0.9, 1.0])).astype(np.float32)
    s = BEM_Solver(v, t)
    k = M.wavenumber(2000.0)
    V, A = s.assemble_vk(k)
    b = -cmatmul(V, torch.ones(V.shape[0], dtype=torch.complex64, device="cuda"))
    return s, k, A, b


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_geometry_normals_and_curls_match_reference_preprocess(path):
    f = np.load(path)
    s = BEM_Solver(f["vertices"], f["triangles"])
    n, c = s.geometry.normals_and_curls()
    assert np.abs(n.cpu().numpy() - f["normals"]).max() < 1e-6
    assert np.abs(c.cpu().numpy() - f["curls"]).max() <= 1e-5 * np.abs(f["curls"]).max()


def test_nonfinite_right_hand_side_is_reported(small):
    _, _, A, b = small
    bad = b.clone()
    bad[3] = complex(float("nan"), 0.0)
    info = {}
    with pytest.raises(L.BEMError) as e:
        gmres(A, bad, rtol=1e-6, info=info)
    assert e.value.status == L.BEM_ERR_NONFINITE
    assert info["status"] == L.BEM_ERR_NONFINITE
    info = {}
    gmres(A, b, rtol=1e-6, info=info)  # the next solve on the same context is clean
    assert info["status"] == L.BEM_OK and info["rel_residual"] <= 1e-6


def test_iteration_cap_is_reported_as_not_converged(small):
    _, _, A, b = small
    info = {}
    gmres(A, b, rtol=1e-12, max_iters=3, info=info)
    assert info["status"] == L.BEM_ERR_NOT_CONVERGED
    assert 1 <= info["iterations"] <= 3
    assert info["rel_residual"] > 1e-12
    with pytest.raises(L.BEMError) as e:
        gmres(A, b, rtol=1e-12, max_iters=3, raise_on_failure=True)
    assert e.value.status == L.BEM_ERR_NOT_CONVERGED
    # through the C ABI: status returned and info filled
    lib = L.lib()
    n = A.shape[0]
    p = L.SolverParams(precision=L.PREC_FP32, restart=3, max_iters=3, max_refine=2, rtol=1e-12, atol=0.0,
                       inner_rtol=1e-3)
    nb = int(lib.bem_gmres_workspace_bytes(n, 1, ctypes.byref(p)))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    X = torch.zeros_like(b)
    out = L.SolverInfo()
    st = lib.bem_gmres_solve(_vp(A), n, _vp(b), 1, _vp(X), 0, ctypes.byref(p), _vp(ws), nb, ctypes.byref(out),
                             _stream())
    assert st == L.BEM_ERR_NOT_CONVERGED and out.status == st and out.iterations == 3


def test_assembly_status_words_read_clean(small):
    s, k, _, _ = small
    s.assemble_bm(k, check=False)
    lib = L.lib()
    assert lib.bem_geometry_status(s.geometry.ptr, _stream()) == L.BEM_OK
    assert lib.bem_assembly_status(_stream()) == L.BEM_OK
    s.geometry.check_status()


def test_released_geometry_address_is_read_again():
    v, t = M.icosphere(1, 0.1)
    vd = torch.from_numpy(v.astype(np.float32)).cuda()
    td = torch.from_numpy(t.astype(np.int32)).cuda()
    lib = L.lib()
    nbytes = ctypes.c_size_t(0)
    L.check(lib.bem_geometry_bytes(_vp(vd), v.shape[0], _vp(td), t.shape[0], ctypes.byref(nbytes), _stream()))
    buf = torch.empty(int(nbytes.value), dtype=torch.uint8, device="cuda")
    L.check(lib.bem_geometry_build(_vp(vd), v.shape[0], _vp(td), t.shape[0], _vp(buf), int(nbytes.value), _stream()))
    out = torch.empty((v.shape[0], v.shape[0]), dtype=torch.complex64, device="cuda")
    assert lib.bem_identity_matrix(_vp(buf), _vp(out), _stream()) == L.BEM_OK
    ref = O.identity_matrix(v.astype(np.float32).astype(np.float64), t)
    assert relfro(out, ref) <= 1e-6
    L.check(lib.bem_geometry_release(_vp(buf)))
    buf.zero_()
    torch.cuda.synchronize()
    assert lib.bem_identity_matrix(_vp(buf), _vp(out), _stream()) == L.BEM_ERR_WORKSPACE
    assert lib.bem_geometry_release(ctypes.c_void_p(0)) == L.BEM_ERR_INVALID_ARGUMENT


def fan_mesh(n_ring=80, r=0.1, h=0.08):
    """Closed bipyramid over an n_ring-gon: each apex is a vertex of n_ring
    triangles (valence above the reference's 64-entry adjacency buffer)."""
    ang = 2 * np.pi * np.arange(n_ring) / n_ring
    ring = np.stack([r * np.cos(ang), r * np.sin(ang), 0.03 * np.sin(3 * ang)], axis=1)
    v = np.concatenate([[[0.0, 0.0, h], [0.0, 0.0, -h]], ring])
    tris = []
    for i in range(n_ring):
        a, b = 2 + i, 2 + (i + 1) % n_ring
        tris += [(a, b, 0), (b, a, 1)]
    t = np.array(tris, dtype=np.int32)
    p0, p1, p2 = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    flip = np.einsum("ij,ij->i", np.cross(p1 - p0, p2 - p0), p0 + p1 + p2) < 0
    t[flip] = t[flip][:, [0, 2, 1]]
    return v.astype(np.float32), t


def test_high_valence_fan_mesh_matches_oracle():
    v, t = fan_mesh()
    assert np.bincount(t.reshape(-1)).max() == 80
    vd = v.astype(np.float64)
    k = M.wavenumber(1000.0)
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    assert relfro(V, O.boundary_matrix("single", vd, t, k)) <= 1e-5
    ref_A = 0.5 * O.identity_matrix(vd, t) - O.boundary_matrix("double", vd, t, k)
    assert relfro(A, ref_A) <= 1e-5
    Kd = s.assemble_boundary_matrix(k, "double")
    assert relfro(Kd, O.boundary_matrix("double", vd, t, k)) <= 1e-5
    g = M.smoothed_gaussian_field(v.shape[0], t, 2, seed=9).astype(np.complex64)
    pts = M.sphere_points(64, 0.5, seed=3).astype(np.float32)
    u, p = s.solve_and_evaluate(k, torch.from_numpy(g).cuda(), torch.from_numpy(pts).cuda(), precision="fp32")
    u_ref = O.cbie_solve(vd, t, k, g)
    p_ref = O.boundary2potential(vd, t, k, g, u_ref, pts)
    assert relfro(u, u_ref) <= 1e-4
    assert relfro(p, p_ref) <= 1e-4


def test_batch_budget_below_one_problem_raises_before_allocating():
    v, t = M.icosphere(2, 0.1)
    g = M.smoothed_gaussian_field(v.shape[0], t, 16, seed=1)
    pts = M.sphere_points(32, 1.0, seed=1)
    before = torch.cuda.memory_allocated()
    with BatchRunner(memory_budget_bytes=1 << 20) as r:
        with pytest.raises(MemoryError):
            r.run([(v, t)], [[10.0, 20.0]], [g], pts)
    assert torch.cuda.memory_allocated() - before < (1 << 20)


def test_batch_wave_above_free_memory_raises_before_allocating():
    v, t = M.icosphere(4, 0.1)
    s = BEM_Solver(v.astype(np.float32), t)
    g = M.smoothed_gaussian_field(v.shape[0], t, 16, seed=1)
    pts = M.sphere_points(32, 1.0, seed=1)
    ks = list(np.linspace(10.0, 100.0, 1000))  # ~224 MB each: ~220 GB in one wave
    with BatchRunner(memory_budget_bytes=1 << 50) as r:
        with pytest.raises(MemoryError):
            r.run([s], [ks], [g], pts)
    # the runner's device stays usable
    with BatchRunner(memory_budget_bytes=1 << 32) as r:
        res = r.run([s], [ks[:2]], [g[:, :2]], pts)
    assert all(i["status"] == 0 for i in res.info)
