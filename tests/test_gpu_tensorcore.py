"""Tensor-core (tcgen05) complex matvec and the mixed-precision solve.

bem_tc_matmul against an FP64 numpy product; GMRES with the bf16 operators
(FP64 refinement against the FP32 matrix) against the FP32-operator solve.
"""
import ctypes

import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver, cmatmul, gmres
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.solver import _stream, _vp

pytestmark = pytest.mark.gpu


def tc_matmul(A, X, precision):
    lib = L.lib()
    n, m = A.shape[0], X.shape[1]
    nbytes = int(lib.bem_tc_operator_bytes(n, m, precision))
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    L.check(lib.bem_tc_operator_prepare(_vp(A), n, precision, _vp(ws), nbytes, _stream()))
    Y = torch.empty_like(X)
    L.check(lib.bem_tc_matmul(_vp(ws), nbytes, n, precision, _vp(X), m, _vp(Y), _stream()))
    L.check(lib.bem_tc_status(_vp(ws), _stream()))
    return Y


@pytest.mark.parametrize("n,m", [(1000, 8), (517, 3), (129, 1), (300, 16), (640, 37), (256, 64), (200, 128)])
@pytest.mark.parametrize("precision,tol", [(L.PREC_BF16X3, 5e-5), (L.PREC_BF16, 1e-2), (L.PREC_FP16X3, 3e-6)])
def test_tc_matmul_vs_fp64(n, m, precision, tol):
    rng = np.random.default_rng(n + m)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    X = (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)
    Y = tc_matmul(torch.from_numpy(A).cuda(), torch.from_numpy(X).cuda(), precision).cpu().numpy()
    ref = A.astype(np.complex128) @ X.astype(np.complex128)
    err = np.linalg.norm(Y - ref) / np.linalg.norm(ref)
    assert err <= tol, err


def test_fp16x3_scales_rows_and_columns_of_any_magnitude():
    """fp16 has a narrow exponent range: rows of A spanning 1e-9..1e3 and
    right-hand sides spanning 1e-6..1e6 must keep FP32-level accuracy per
    row and per column (power-of-two scales per row / column)."""
    rng = np.random.default_rng(11)
    n, m = 700, 6
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    A *= 10.0 ** rng.uniform(-9, 3, size=(n, 1))
    X = (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))) * 10.0 ** np.linspace(-6, 6, m)
    A, X = A.astype(np.complex64), X.astype(np.complex64)
    Y = tc_matmul(torch.from_numpy(A).cuda(), torch.from_numpy(X).cuda(), L.PREC_FP16X3).cpu().numpy()
    ref = A.astype(np.complex128) @ X.astype(np.complex128)
    scale = np.abs(A).astype(np.float64) @ np.abs(X).astype(np.float64)
    assert np.isfinite(Y).all()
    assert np.max(np.abs(Y - ref) / scale) <= 3e-6


@pytest.mark.parametrize("m", [8, 64])
def test_fp16x3_matvec_of_a_bem_matrix_matches_fp32(m):
    """On a Galerkin CBIE matrix (dominant mass diagonal, oscillatory far
    field) the fp16x3 operator with short accumulator segments is as accurate
    as an FP32 matvec (relative error <= 2e-6; a long in-place tensor-memory
    accumulation gives ~3e-5 here)."""
    v, t = M.icosphere(4, 0.15)
    v = (v * np.array([1.2, 0.8, 1.0])).astype(np.float32)
    s = BEM_Solver(v, t)
    _, A = s.assemble_vk(M.wavenumber(4000.0))
    rng = np.random.default_rng(4)
    X = torch.from_numpy((rng.standard_normal((A.shape[0], m)) + 1j * rng.standard_normal((A.shape[0], m)))
                         .astype(np.complex64)).cuda()
    Y = tc_matmul(A, X, L.PREC_FP16X3).to(torch.complex128)
    ref = A.to(torch.complex128) @ X.to(torch.complex128)
    assert float(torch.linalg.norm(Y - ref) / torch.linalg.norm(ref)) <= 2e-6


def test_tc_matmul_repeat_is_deterministic_enough():
    rng = np.random.default_rng(5)
    n, m = 800, 8
    A = torch.from_numpy((rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)).cuda()
    X = torch.from_numpy((rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)).cuda()
    y1 = tc_matmul(A, X, L.PREC_BF16X3)
    y2 = tc_matmul(A, X, L.PREC_BF16X3)
    assert torch.allclose(y1, y2, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("precision", ["bf16x3", "bf16", "fp16x3"])
def test_mixed_precision_cbie_matches_fp32(precision):
    v, t = M.icosphere(3, 0.15)
    v = (v * np.array([1.2, 0.8, 1.0])).astype(np.float32)
    k = M.wavenumber(4000.0)
    g = torch.from_numpy(M.smoothed_gaussian_field(v.shape[0], t, 8, seed=2).astype(np.complex64)).cuda()
    s = BEM_Solver(v, t)
    V, A = s.assemble_vk(k)
    rhs = -cmatmul(V, g)
    i32, imx = {}, {}
    x32 = gmres(A, rhs, rtol=1e-6, precision="fp32", info=i32)
    xmx = gmres(A, rhs, rtol=1e-6, precision=precision, info=imx)
    assert i32["status"] == L.BEM_OK and imx["status"] == L.BEM_OK, (i32, imx)
    assert imx["rel_residual"] <= 1e-6
    Ad = A.cpu().numpy().astype(np.complex128)
    b = rhs.cpu().numpy().astype(np.complex128)
    ref = np.linalg.solve(Ad, b)
    for x in (x32, xmx):
        xx = x.cpu().numpy()
        assert np.linalg.norm(xx - ref) / np.linalg.norm(ref) <= 1e-4  # residual 1e-6 times the conditioning


@pytest.mark.parametrize("fill", [1, 4])
def test_expired_bounded_wait_is_reported_and_the_next_call_is_clean(fill):
    """A bounded wait that runs out, made on the host: the test hook leaves one
    pipeline fill of CTA 0 unissued, so its tensor-core consumer waits on a
    stage that never fills.  With a 1 ms limit the wait expires, the kernel
    lets its other copies land, releases tensor memory and returns (no fault,
    no hang); bem_tc_status reports BEM_ERR_CUDA once, and the next call on the
    same workspace is exact again."""
    lib = L.lib()
    rng = np.random.default_rng(3)
    n, m = 4000, 8  # 32 row blocks x 125 K blocks: ~27 pipeline fills per CTA
    A = torch.from_numpy((rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)).cuda()
    X = torch.from_numpy((rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)).cuda()
    ref = A.cpu().numpy().astype(np.complex128) @ X.cpu().numpy().astype(np.complex128)
    prec = L.PREC_FP16X3
    nbytes = int(lib.bem_tc_operator_bytes(n, m, prec))
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    L.check(lib.bem_tc_operator_prepare(_vp(A), n, prec, _vp(ws), nbytes, _stream()))
    Y = torch.empty_like(X)
    try:
        L.check(lib.bem_set_tuning(L.TUNE_TC_WAIT_US, 1000))
        L.check(lib.bem_set_tuning(L.TUNE_TC_TEST_SKIP_FILL, fill))
        L.check(lib.bem_tc_matmul(_vp(ws), nbytes, n, prec, _vp(X), m, _vp(Y), _stream()))
        assert lib.bem_get_tuning(L.TUNE_TC_TEST_SKIP_FILL) == 0  # one launch only
        assert lib.bem_tc_status(_vp(ws), _stream()) == L.BEM_ERR_CUDA
        assert lib.bem_tc_status(_vp(ws), _stream()) == L.BEM_OK  # read once, then clear
    finally:
        lib.bem_set_tuning(L.TUNE_TC_TEST_SKIP_FILL, 0)
        lib.bem_set_tuning(L.TUNE_TC_WAIT_US, 0)
    L.check(lib.bem_tc_matmul(_vp(ws), nbytes, n, prec, _vp(X), m, _vp(Y), _stream()))
    assert lib.bem_tc_status(_vp(ws), _stream()) == L.BEM_OK
    err = np.linalg.norm(Y.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= 3e-6, err
