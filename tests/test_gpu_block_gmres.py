"""Block GMRES: one block Krylov space for several right-hand sides.

bem_gmres_solve with 2..16 right-hand sides extends one block Krylov space by
all columns at each operator application (CholQR of the block, FP64 block
Gram-Schmidt, the small least-squares problem solved on the host); 17..64
right-hand sides are split into groups of at most 16 columns, each group its
own block space, all groups sharing one matvec per step.  Against
the FP64 oracle's dense CBIE solve it must give the same solutions as the
per-column spaces, with far fewer operator applications; a right-hand-side
block that has lost rank (equal or zero columns) falls back to per-column
spaces and still converges.
"""
import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
from neuralat_b200.bem import meshes as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    v, t = M.icosphere(3, 0.15)
    v = (v * np.array([1.2, 0.8, 1.0])).astype(np.float32)
    k = M.wavenumber(4000.0)
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    lhs, Vo = O.cbie_system(v.astype(np.float64), t, np.float32(k))
    return s, V, A, lhs, Vo


@pytest.mark.parametrize("m", [2, 8, 16, 17, 33, 64])
@pytest.mark.parametrize("precision", ["fp32", "fp16x3"])
def test_block_solve_matches_fp64_oracle(system, m, precision):
    s, V, A, lhs, Vo = system
    g = M.smoothed_gaussian_field(A.shape[0], s.triangles.cpu().numpy(), m, seed=30 + m).astype(np.complex64)
    rhs = -cmatmul(V, torch.from_numpy(g).cuda())
    info = {}
    u = gmres(A, rhs, rtol=1e-6, precision=precision, info=info).cpu().numpy()
    assert info["status"] == 0 and info["rel_residual"] <= 1e-6
    lib = L.lib()
    try:
        L.check(lib.bem_set_tuning(L.TUNE_GMRES_BLOCK, 1))
        info1 = {}
        u1 = gmres(A, rhs, rtol=1e-6, precision=precision, info=info1).cpu().numpy()
    finally:
        L.check(lib.bem_set_tuning(L.TUNE_GMRES_BLOCK, 0))
    assert info1["status"] == 0
    # against the FP64 oracle's dense solve: within 1e-4, or (a column whose
    # FP32 operator is worse conditioned) no further than the per-column solve
    u_ref = np.linalg.solve(lhs, -Vo @ g.astype(np.complex128))
    err = np.linalg.norm(u - u_ref, axis=0) / np.linalg.norm(u_ref, axis=0)
    err1 = np.linalg.norm(u1 - u_ref, axis=0) / np.linalg.norm(u_ref, axis=0)
    assert np.all(err <= np.maximum(1e-4, 1.1 * err1 + 1e-6)), (err.max(), err1.max())
    # both solve the same FP32 system to residual 1e-6
    assert np.linalg.norm(u - u1) / np.linalg.norm(u1) <= 1e-4
    assert info["iterations"] < info1["iterations"], (info, info1)


def test_rank_deficient_block_falls_back_to_separate_spaces(system):
    s, V, A, lhs, Vo = system
    g = M.smoothed_gaussian_field(A.shape[0], s.triangles.cpu().numpy(), 4, seed=9).astype(np.complex64)
    g[:, 2] = g[:, 0]  # two equal right-hand sides
    g[:, 3] = 0.0      # and a zero one
    rhs = -cmatmul(V, torch.from_numpy(g).cuda())
    info = {}
    u = gmres(A, rhs, rtol=1e-6, precision="fp32", info=info).cpu().numpy()
    assert info["status"] == 0
    u_ref = np.linalg.solve(lhs, -Vo @ g.astype(np.complex128))
    for c in range(3):
        assert np.linalg.norm(u[:, c] - u_ref[:, c]) / np.linalg.norm(u_ref[:, c]) <= 1e-4
    assert np.abs(u[:, 3]).max() == 0.0


def test_block_mode_key():
    lib = L.lib()
    assert lib.bem_get_tuning(L.TUNE_GMRES_BLOCK) == 0
    assert lib.bem_set_tuning(L.TUNE_GMRES_BLOCK, 2) == L.BEM_ERR_INVALID_ARGUMENT
