"""Batched assembly and the batch runner against the single-problem path.

One persistent launch assembles (V, 0.5 M - K) for problems of different mesh
sizes and wavenumbers; each must equal the single-problem fused assembly
(relative Frobenius <= 1e-5: only the order of FP32 atomic additions differs)
and the FP64 oracle (<= 1e-5).  The batch runner's listener pressures must
equal the per-problem CBIE + evaluation (<= 1e-4).
"""
import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, autotune
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.batch import BatchRunner, assemble_batch
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def relfro(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _meshes():
    rng = np.random.default_rng(11)
    out = []
    for s, r in ((1, 0.2), (3, 0.1), (2, 0.15), (4, 0.12)):
        v, t = M.icosphere(s, r)
        v = (v * rng.uniform(0.7, 1.3, size=3)) @ M.random_rotation(rng).T
        out.append((v.astype(np.float32), t))
    return out


@pytest.fixture(scope="module")
def solvers():
    return [BEM_Solver(v, t) for v, t in _meshes()]


PROBLEMS = [(0, 18.3), (1, 73.3), (2, -40.0), (1, 120.5), (3, 55.0), (0, 150.0)]


@pytest.mark.parametrize("chunk", [0, 1, 3, 32])
def test_batched_assembly_equals_single(solvers, chunk):
    L.check(L.lib().bem_set_tuning(L.TUNE_ASSEMBLY_CHUNK, chunk))
    try:
        ss = [solvers[i] for i, _ in PROBLEMS]
        ks = [k for _, k in PROBLEMS]
        mats = assemble_batch(ss, ks)
        torch.cuda.synchronize()
        for s, k, (V, A) in zip(ss, ks, mats):
            V1, A1 = s.assemble_vk(k)
            assert relfro(V.cpu(), V1.cpu()) <= 1e-5
            assert relfro(A.cpu(), A1.cpu()) <= 1e-5
    finally:
        autotune.reset()


def test_batched_assembly_vs_oracle(solvers):
    ss = [solvers[0], solvers[2], solvers[0]]
    ks = [18.3, -40.0, 150.0]
    mats = assemble_batch(ss, ks)
    for s, k, (V, A) in zip(ss, ks, mats):
        v = s.vertices.cpu().numpy().astype(np.float64)
        t = s.triangles.cpu().numpy()
        Vo = O.boundary_matrix("single", v, t, k)
        Ko = O.boundary_matrix("double", v, t, k)
        Io = O.identity_matrix(v, t)
        assert relfro(V.cpu(), Vo) <= 1e-5
        assert relfro(A.cpu(), 0.5 * Io - Ko) <= 1e-5


def test_batched_assembly_custom_coefficients(solvers):
    s = solvers[2]
    (V, A), = assemble_batch([s], [33.0], mass_coeff=0.0, k_coeff=1.0)
    K = s.assemble_boundary_matrix(33.0, "double")
    assert relfro(A.cpu(), K.cpu()) <= 1e-5


def test_batch_runner_matches_per_problem(solvers):
    ms = _meshes()[:3]
    ks = [[18.3, 90.0], [73.3], [-40.0, 20.0]]
    gs = [M.smoothed_gaussian_field(v.shape[0], t, 3, seed=i) for i, (v, t) in enumerate(ms)]
    pts = M.sphere_points(64, 1.0, seed=3)
    # a tiny budget forces several waves
    with BatchRunner(memory_budget_bytes=3 * 8 * 642 * 642 * 2, workers=3, precision="fp32", rtol=1e-7) as runner:
        res = runner.run(ms, ks, gs, pts, return_dirichlet=True)
        assert all(w["concurrency"] == runner.concurrency(w["vertices"]) for w in res.waves)
    assert sorted(res.index) == sorted((mi, ki) for mi in range(3) for ki in range(len(ks[mi])))
    assert sum(w["problems"] for w in res.waves) == len(res.index)
    ptt = torch.as_tensor(pts, dtype=torch.float32, device="cuda")
    for (mi, ki), p, u, info in zip(res.index, res.pressure, res.dirichlet, res.info):
        s = BEM_Solver(*ms[mi])
        g = torch.as_tensor(gs[mi], dtype=torch.complex64, device="cuda")
        u1 = s.CBIE(ks[mi][ki], g, rtol=1e-7)  # both solves tight: the solutions may differ by cond x rtol
        p1 = s.boundary2potential(ks[mi][ki], g, u1, ptt)
        assert info["rel_residual"] <= 1e-7
        assert relfro(u.cpu(), u1.cpu()) <= 1e-4
        assert relfro(p.cpu(), p1.cpu()) <= 1e-4


def test_batch_runner_vs_oracle_on_mixed_sizes():
    """The runner's own output (both formulations' CBIE path, two meshes of
    different size, two wavenumbers on one of them, tensor-core precision)
    against the FP64 oracle's dense CBIE solve and listener evaluation."""
    ms = [_meshes()[0], _meshes()[2]]  # 42 and 162 vertices
    ks = [[18.3, 90.0], [55.0]]
    gs = [M.smoothed_gaussian_field(v.shape[0], t, 2, seed=20 + i) for i, (v, t) in enumerate(ms)]
    pts = M.sphere_points(48, 1.0, seed=7)
    with BatchRunner(workers=2, precision="fp16x3", rtol=1e-7) as runner:
        res = runner.run(ms, ks, gs, pts, return_dirichlet=True)
    for (mi, ki), p, u in zip(res.index, res.pressure, res.dirichlet):
        v, t = ms[mi]
        vd = v.astype(np.float32).astype(np.float64)
        k = float(np.float32(ks[mi][ki]))
        g = gs[mi].astype(np.complex64)
        u_ref = O.cbie_solve(vd, t, k, g)
        p_ref = O.boundary2potential(vd, t, k, g, u_ref, pts.astype(np.float32))
        assert relfro(u.cpu(), u_ref) <= 1e-4, (mi, ki)
        assert relfro(p.cpu(), p_ref) <= 1e-4, (mi, ki)


def test_autotune_installs_and_caches(solvers, tmp_path, monkeypatch):
    monkeypatch.setenv("NEURALAT_B200_CACHE", str(tmp_path))
    ss = [solvers[1], solvers[2], solvers[3]]
    ks = [40.0, 60.0, 80.0]
    try:
        cfg = autotune.tune_assembly(ss, ks, repeats=1)
        assert not cfg["cached"]
        lib = L.lib()
        assert lib.bem_get_tuning(L.TUNE_ASSEMBLY_CHUNK) == cfg["chunk"]
        assert lib.bem_get_tuning(L.TUNE_ASSEMBLY_CTAS_PER_SM) == cfg["ctas_per_sm"]
        assert len(cfg["timings"]) == len(autotune.CHUNKS) * len(autotune.CTAS)
        again = autotune.tune_assembly(ss, ks)
        assert again["cached"] and again["chunk"] == cfg["chunk"]
        mats = assemble_batch(ss, ks)
        for s, k, (V, A) in zip(ss, ks, mats):
            V1, A1 = s.assemble_vk(k)
            assert relfro(A.cpu(), A1.cpu()) <= 1e-5
    finally:
        autotune.reset()
