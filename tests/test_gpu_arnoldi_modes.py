"""The Arnoldi step variants of the device GMRES give the same solves.

With 2 to 64 right-hand sides the default is block GMRES (one block Krylov
space per group of at most 16 columns, BEM_TUNE_GMRES_BLOCK = 0); the
per-column variants below are run with it switched off.

The default is the cluster kernel (one launch per step, a thread-block
cluster per right-hand side) with one classical Gram-Schmidt pass whose
projections are formed with FP64 products; two passes (CGS2) are the stable
reference.  The streamed step (launches over all SMs, a second pass where the
first one cancels most of w) and the cooperative kernel (one launch over all
SMs, two grid barriers) are selected with BEM_TUNE_ARNOLDI_MODE.  The odd-sized 3 kHz case here is one where
single-pass Gram-Schmidt with FP32 products needed up to 1.7 times the steps;
it also exercises the padding entry of an odd number of unknowns."""
import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
from neuralat_b200.bem import meshes as M

pytestmark = pytest.mark.gpu


def relfro(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.fixture(scope="module")
def system():
    v, t = M.icosphere(3, 0.15)
    v = (v * np.array([1.2, 0.8, 1.0])).astype(np.float32)
    # split one triangle at its centroid: a closed mesh with an odd number of unknowns (padding entry)
    a, b, c = t[0]
    nv = v.shape[0]
    v = np.concatenate([v, v[[a, b, c]].mean(axis=0, keepdims=True)]).astype(np.float32)
    t = np.concatenate([[[a, b, nv], [b, c, nv], [c, a, nv]], t[1:]]).astype(np.int32)
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(M.wavenumber(3000.0))
    return s, V, A


@pytest.mark.parametrize("m", [1, 8, 64])
@pytest.mark.parametrize("precision", ["fp32", "fp16x3"])
def test_arnoldi_variants_match_two_pass_reference(system, m, precision):
    s, V, A = system
    n = A.shape[0]
    g = torch.from_numpy(M.smoothed_gaussian_field(n, s.triangles.cpu().numpy(), m, seed=m).astype(np.complex64)).cuda()
    rhs = -cmatmul(V, g)
    lib = L.lib()
    out = {}
    try:
        for name, mode, reorth, blk in (("cgs2", 1, 2, 1), ("default", 0, 0, 0), ("cluster", 1, 0, 1),
                                        ("streamed", 2, 0, 1), ("cooperative", 3, 0, 1)):
            L.check(lib.bem_set_tuning(L.TUNE_ARNOLDI_MODE, mode))
            L.check(lib.bem_set_tuning(L.TUNE_GMRES_REORTH, reorth))
            L.check(lib.bem_set_tuning(L.TUNE_GMRES_BLOCK, blk))
            info = {}
            out[name] = (gmres(A, rhs, rtol=1e-6, precision=precision, info=info), info)
    finally:
        L.check(lib.bem_set_tuning(L.TUNE_ARNOLDI_MODE, 0))
        L.check(lib.bem_set_tuning(L.TUNE_GMRES_REORTH, 0))
        L.check(lib.bem_set_tuning(L.TUNE_GMRES_BLOCK, 0))
    u_ref, i_ref = out["cgs2"]
    assert i_ref["status"] == 0
    if 2 <= m <= 64:  # the default is block Krylov spaces: far fewer operator applications
        assert out["default"][1]["iterations"] <= 0.5 * i_ref["iterations"], (out["default"][1], i_ref)
    for name in ("default", "cluster", "streamed", "cooperative"):
        u, info = out[name]
        assert info["status"] == 0, name
        assert info["iterations"] <= 1.1 * i_ref["iterations"] + 2, (name, info["iterations"], i_ref["iterations"])
        res = torch.linalg.norm(cmatmul(A, u) - rhs) / torch.linalg.norm(rhs)
        assert float(res) <= 2e-6, name
        # two solutions with residual <= 1e-6 differ by up to cond(A) x 2e-6
        assert relfro(u, u_ref) <= 1e-4, name


def test_arnoldi_mode_key():
    lib = L.lib()
    assert lib.bem_get_tuning(L.TUNE_ARNOLDI_MODE) == 0
    assert lib.bem_set_tuning(L.TUNE_ARNOLDI_MODE, 4) == L.BEM_ERR_INVALID_ARGUMENT
