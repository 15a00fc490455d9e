"""The C ABI library loads and exports every entry point of include/bem_b200.h
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

from neuralat_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms.update(re.findall(r"\b(bem_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(L.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert set(L.EXPORTED) <= syms


def test_status_strings_and_version():
    lib = L.lib()
    assert b"sm_100a" in lib.bem_version()
    for st in range(10):
        assert lib.bem_status_string(st)
    assert L.BEMError(L.BEM_ERR_INDEX).status == L.BEM_ERR_INDEX


def test_host_side_sizes():
    lib = L.lib()
    p = L.SolverParams(precision=L.PREC_FP32, restart=30, max_iters=100, max_refine=2, rtol=1e-6, atol=0.0,
                       inner_rtol=1e-3)
    n, m = 1000, 4
    b = lib.bem_gmres_workspace_bytes(n, m, ctypes.byref(p))
    assert b > 8 * m * 31 * n  # complex64 Krylov basis of restart + 1 vectors per column
    p.restart = 0
    assert lib.bem_gmres_workspace_bytes(n, m, ctypes.byref(p)) == 0
    assert lib.bem_boundary2potential_scratch_bytes(100, 3) == 2 * 8 * 100 * 6 * 3
    assert lib.bem_boundary2potential_scratch_bytes(0, 3) == 0


def test_invalid_arguments_rejected_before_any_device_work():
    lib = L.lib()
    nbytes = ctypes.c_size_t(0)
    assert lib.bem_geometry_bytes(None, 3, None, 1, ctypes.byref(nbytes), None) == L.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_cmatmul(None, -1, None, 1, None, None) == L.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_boundary_matrix(None, 0, 0, 1.0, None, None, None, None) == L.BEM_ERR_WORKSPACE


def test_no_cpu_fallback_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    lib = L.lib()
    nbytes = ctypes.c_size_t(0)
    st = lib.bem_geometry_bytes(ctypes.c_void_p(16), 3, ctypes.c_void_p(16), 1, ctypes.byref(nbytes), None)
    assert st == L.BEM_ERR_CUDA


def test_tuning_knobs_and_batch_sizes():
    lib = L.lib()
    assert lib.bem_get_tuning(L.TUNE_ASSEMBLY_CHUNK) == 0
    assert lib.bem_set_tuning(L.TUNE_ASSEMBLY_CHUNK, 4) == L.BEM_OK
    assert lib.bem_get_tuning(L.TUNE_ASSEMBLY_CHUNK) == 4
    assert lib.bem_set_tuning(L.TUNE_ASSEMBLY_CTAS_PER_SM, 1) == L.BEM_OK
    assert lib.bem_get_tuning(L.TUNE_ASSEMBLY_CTAS_PER_SM) == 1
    assert lib.bem_set_tuning(99, 1) == L.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_set_tuning(L.TUNE_ASSEMBLY_CHUNK, -1) == L.BEM_ERR_INVALID_ARGUMENT
    assert lib.bem_get_tuning(99) == -1
    for key in (L.TUNE_ASSEMBLY_CHUNK, L.TUNE_ASSEMBLY_CTAS_PER_SM):
        assert lib.bem_set_tuning(key, 0) == L.BEM_OK
    assert lib.bem_batch_workspace_bytes(1) >= 256
    assert lib.bem_batch_workspace_bytes(1000) > lib.bem_batch_workspace_bytes(10)
    assert lib.bem_batch_matrices_vk(None, 1, 0.5, -1.0, None, 0, None) == L.BEM_ERR_INVALID_ARGUMENT
    probs = (L.BatchProblem * 1)()
    assert lib.bem_batch_matrices_vk(probs, 0, 0.5, -1.0, None, 0, None) == L.BEM_ERR_INVALID_ARGUMENT


def test_burton_miller_entry_points_reject_bad_arguments_on_host():
    lib = L.lib()
    # no geometry: rejected before any device work, whatever the order
    for order in (L.ORDER_EXACT, L.ORDER_APPROX, L.ORDER_APPROX_1):
        assert lib.bem_boundary_matrices_bm(None, order, 10.0, None, None, None) == L.BEM_ERR_WORKSPACE
    assert lib.bem_batch_matrices_bm(None, 1, L.ORDER_APPROX, None, 0, None) == L.BEM_ERR_INVALID_ARGUMENT
    probs = (L.BmProblem * 1)()
    assert lib.bem_batch_matrices_bm(probs, 0, L.ORDER_APPROX, None, 0, None) == L.BEM_ERR_INVALID_ARGUMENT
    # the batch workspace covers both batched assemblies
    assert lib.bem_batch_workspace_bytes(64) >= 64 * ctypes.sizeof(L.BmProblem)
