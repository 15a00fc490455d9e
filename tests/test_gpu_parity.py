"""Parity of the CUDA path against the FP64 CPU oracle (and the analytic monopole).

Every call goes through the C ABI of libbemb200.so (via the drop-in
``BEM_Solver``).  Tolerances: relative Frobenius <= 1e-5 for matrices,
<= 1e-4 for listener pressures (FP32 kernels vs FP64 oracle).
"""
import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, cmatmul, gmres, map_triangle2vertex, solve_linear_equation
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.solver import _stream
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAT_TOL = 1e-5
PRESSURE_TOL = 1e-4


def relfro(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _mesh(name):
    if name == "s1":
        v, t = M.icosphere(1, 0.2)
    elif name == "s2_ellipsoid":
        v, t = M.icosphere(2, 0.15)
        v = v * np.array([1.25, 0.75, 1.0])
    elif name == "s3":
        v, t = M.icosphere(3, 0.1)
    else:
        raise KeyError(name)
    return v.astype(np.float32), t


_oracle_cache = {}


def oracle_matrix(layer, name, k):
    key = (layer, name, k)
    if key not in _oracle_cache:
        v, t = _mesh(name)
        _oracle_cache[key] = O.boundary_matrix(layer, v.astype(np.float64), t, k)
    return _oracle_cache[key]


@pytest.fixture(scope="module")
def solvers():
    return {n: BEM_Solver(*_mesh(n)) for n in ("s1", "s2_ellipsoid", "s3")}


@pytest.mark.parametrize("name", ["s1", "s2_ellipsoid"])
@pytest.mark.parametrize("k", [18.318, 73.27, -100.6])
@pytest.mark.parametrize("layer", ["single", "double"])
def test_boundary_matrix_vs_oracle(solvers, name, k, layer):
    A = solvers[name].assemble_boundary_matrix(k, layer).cpu().numpy()
    assert np.isfinite(A).all()
    assert relfro(A, oracle_matrix(layer, name, k)) <= MAT_TOL


def test_s3_vk_vs_oracle(solvers):
    k = M.wavenumber(1000.0)
    s = solvers["s3"]
    V, lhs = s.assemble_vk(k)
    assert L.lib().bem_assembly_status(_stream()) == L.BEM_OK  # no bounded wait expired
    Mo = O.identity_matrix(*_mesh("s3"))
    assert relfro(V.cpu().numpy(), oracle_matrix("single", "s3", k)) <= MAT_TOL
    assert relfro(lhs.cpu().numpy(), 0.5 * Mo - oracle_matrix("double", "s3", k)) <= MAT_TOL


@pytest.mark.parametrize("name", ["s1", "s2_ellipsoid"])
def test_fused_equals_separate(solvers, name):
    s = solvers[name]
    k = 37.0
    V, lhs = s.assemble_vk(k)
    V1 = s.assemble_boundary_matrix(k, "single")
    K1 = s.assemble_boundary_matrix(k, "double")
    I1 = s.identity_matrix()
    assert relfro(V.cpu(), V1.cpu()) <= 1e-6
    assert relfro(lhs.cpu(), (0.5 * I1 - K1).cpu()) <= 1e-6


@pytest.mark.parametrize("name", ["s1", "s2_ellipsoid", "s3"])
def test_identity_vs_oracle(solvers, name):
    v, t = _mesh(name)
    assert relfro(solvers[name].identity_matrix().cpu().numpy(), O.identity_matrix(v, t)) <= 1e-6


@pytest.mark.parametrize("layer", ["single", "double"])
def test_potential_matrix_vs_oracle(solvers, layer):
    v, t = _mesh("s2_ellipsoid")
    pts = M.sphere_points(40, 0.5, seed=3).astype(np.float32)
    k = 73.27
    P = solvers["s2_ellipsoid"].potential_matrix(k, torch.from_numpy(pts).cuda(), layer).cpu().numpy()
    assert relfro(P, O.potential_matrix(layer, v, t, pts, k)) <= MAT_TOL


@pytest.mark.parametrize("m", [1, 3, 9])
def test_boundary2potential_vs_oracle(solvers, m):
    v, t = _mesh("s2_ellipsoid")
    k = 73.27
    pts = M.sphere_points(70, 0.5, seed=4).astype(np.float32)
    rng = np.random.default_rng(m)
    g = (rng.standard_normal((v.shape[0], m)) + 1j * rng.standard_normal((v.shape[0], m))).astype(np.complex64)
    u = (rng.standard_normal((v.shape[0], m)) + 1j * rng.standard_normal((v.shape[0], m))).astype(np.complex64)
    s = solvers["s2_ellipsoid"]
    p = s.boundary2potential(k, torch.from_numpy(g).cuda(), torch.from_numpy(u).cuda(),
                             torch.from_numpy(pts).cuda()).cpu().numpy()
    S = O.potential_matrix("single", v, t, pts, k)
    D = O.potential_matrix("double", v, t, pts, k)
    ref = -S @ g + D @ u
    assert relfro(p, ref) <= PRESSURE_TOL
    p1 = s.single_potential(k, torch.from_numpy(g[:, 0]).cuda(), torch.from_numpy(pts).cuda()).cpu().numpy()
    assert relfro(p1, S @ g[:, 0]) <= PRESSURE_TOL


@pytest.mark.parametrize("m", [1, 2, 5, 8, 13])
def test_cmatmul(m):
    rng = np.random.default_rng(m)
    n = 777
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    X = (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)
    Y = cmatmul(torch.from_numpy(A).cuda(), torch.from_numpy(X).cuda()).cpu().numpy()
    ref = A.astype(np.complex128) @ X.astype(np.complex128)
    assert relfro(Y, ref) <= 1e-5


@pytest.mark.parametrize("m", [1, 4])
def test_gmres_random_system(m):
    rng = np.random.default_rng(7 + m)
    n = 500
    A = (np.eye(n) * 4 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)).astype(
        np.complex64)
    b = (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)
    info = {}
    x = gmres(torch.from_numpy(A).cuda(), torch.from_numpy(b).cuda(), rtol=1e-6, restart=20, info=info).cpu().numpy()
    ref = np.linalg.solve(A.astype(np.complex128), b.astype(np.complex128))
    assert info["status"] == L.BEM_OK
    assert info["rel_residual"] <= 1e-6
    assert relfro(x, ref) <= 1e-5


def _cbie_reference(name, k, g):
    v, t = _mesh(name)
    lhs = 0.5 * O.identity_matrix(v, t) - oracle_matrix("double", name, k)
    return np.linalg.solve(lhs, -oracle_matrix("single", name, k) @ g)


@pytest.mark.parametrize("name", ["s2_ellipsoid", "s3"])
def test_cbie_vs_oracle(solvers, name):
    k = 73.27 if name == "s2_ellipsoid" else M.wavenumber(1000.0)
    v, t = _mesh(name)
    g = M.smoothed_gaussian_field(v.shape[0], t, 3, seed=5)
    info = {}
    u = solvers[name].CBIE(k, torch.from_numpy(g.astype(np.complex64)).cuda(), rtol=1e-6, info=info).cpu().numpy()
    assert info["status"] == L.BEM_OK
    assert relfro(u, _cbie_reference(name, k, g)) <= 1e-4


def test_monopole_known_answer(solvers):
    """Analytic pulsating-sphere solution (scripts/unit_test.py:27-39) at 1 kHz."""
    v, t = _mesh("s3")
    k = M.wavenumber(1000.0)
    vn = M.vertex_normals(v, t)
    g = O.monopole_neumann(v, vn, k).astype(np.complex64)
    s = solvers["s3"]
    pts = M.sphere_points(256, 0.5, seed=0).astype(np.float32)
    u, p = s.solve_and_evaluate(k, torch.from_numpy(g).cuda(), torch.from_numpy(pts).cuda(), precision="fp32")
    u, p = u.cpu().numpy(), p.cpu().numpy()
    assert relfro(u, O.monopole(v, k)) < 1e-2
    assert relfro(p, O.monopole(pts, k)) < 1e-2


def test_solve_linear_equation_bicgstab_and_gmres(solvers):
    """Default stopping test as the reference: ||r||^2 < tol ||b||^2 (tol 1e-10)."""
    s = solvers["s2_ellipsoid"]
    k = 30.0
    v, t = _mesh("s2_ellipsoid")
    g = torch.from_numpy(M.smoothed_gaussian_field(v.shape[0], t, 1, seed=9)[:, 0].astype(np.complex64)).cuda()
    V, lhs = s.assemble_vk(k)
    rhs = -cmatmul(V, g)
    A = lhs.cpu().numpy().astype(np.complex128)
    b = rhs.cpu().numpy().astype(np.complex128)
    ref = np.linalg.solve(A, b)
    # GMRES verifies its stopping test with an FP64 residual
    x = solve_linear_equation(lhs, rhs).cpu().numpy()
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1.05e-5
    # BiCGSTAB (matrix or callable) measures ||r|| in FP32 like the reference
    for x in (solve_linear_equation(lhs, rhs, solver="bicgstab"),
              solve_linear_equation(lambda z: cmatmul(lhs, z), rhs)):
        x = x.cpu().numpy()
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-4
    x_t = solve_linear_equation(lhs, rhs, tol=1e-14).cpu().numpy()
    assert relfro(x_t, ref) <= 1e-5


def test_triangle2vertex():
    v, t = _mesh("s2_ellipsoid")
    rng = np.random.default_rng(2)
    f = (rng.standard_normal(t.shape[0]) + 1j * rng.standard_normal(t.shape[0])).astype(np.complex64)
    out = map_triangle2vertex(torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(f).cuda())
    assert relfro(out.cpu().numpy(), O.triangle2vertex(v.shape[0], t, f)) <= 1e-6


def test_mesh_errors_raise():
    v, t = _mesh("s1")
    bad = t.copy()
    bad[3, 1] = v.shape[0] + 5
    with pytest.raises(L.BEMError) as e:
        BEM_Solver(v, bad)
    assert e.value.status == L.BEM_ERR_INDEX
    deg = t.copy()
    deg[0, 1] = deg[0, 0]
    with pytest.raises(L.BEMError) as e:
        BEM_Solver(v, deg)
    assert e.value.status == L.BEM_ERR_DEGENERATE
    vn = v.copy()
    vn[2, 0] = np.nan
    with pytest.raises(L.BEMError) as e:
        BEM_Solver(vn, t)
    assert e.value.status == L.BEM_ERR_NONFINITE
