"""ctypes binding of ``libbemb200.so`` (the C ABI declared in include/bem_b200.h).

The shared library is built in-tree by ``neuralat_b200/build.py`` (called by
``__graft_entry__.build()``).  There is no fallback: if the library is absent
or no CUDA device is usable, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libbemb200.so")

# status codes (bem_status)
BEM_OK = 0
BEM_ERR_INVALID_ARGUMENT = 1
BEM_ERR_INDEX = 2
BEM_ERR_DEGENERATE = 3
BEM_ERR_WORKSPACE = 4
BEM_ERR_NONFINITE = 5
BEM_ERR_NOT_CONVERGED = 6
BEM_ERR_BREAKDOWN = 7
BEM_ERR_CUDA = 8
BEM_ERR_UNSUPPORTED = 9

# layers and orders
SINGLE_LAYER, DOUBLE_LAYER, ADJOINT_DOUBLE_LAYER, HYPERSINGULAR, BM_LHS, BM_RHS = range(6)
ORDER_EXACT, ORDER_APPROX, ORDER_APPROX_1 = range(3)
PREC_FP32, PREC_BF16X3, PREC_BF16, PREC_FP16X3 = range(4)

# every symbol include/bem_b200.h declares
EXPORTED = (
    "bem_status_string", "bem_version", "bem_kernel_launches",
    "bem_geometry_bytes", "bem_geometry_build", "bem_geometry_normals",
    "bem_boundary_matrix", "bem_boundary_matrices_vk", "bem_identity_matrix", "bem_triangle2vertex",
    "bem_potential_matrix", "bem_boundary2potential_scratch_bytes", "bem_boundary2potential",
    "bem_cmatmul", "bem_gmres_workspace_bytes", "bem_gmres_solve",
    "bem_tc_operator_bytes", "bem_tc_operator_prepare", "bem_tc_matmul", "bem_tc_status",
    "bem_boundary2potential_noalloc_max", "bem_boundary2potential_noalloc",
    "bem_cmatmul_adjoint", "bem_conj_transpose", "bem_boundary2potential_adjoint", "bem_vertex_gradient",
    "bem_batch_workspace_bytes", "bem_batch_matrices_vk", "bem_set_tuning", "bem_assembly_status", "bem_get_tuning",
    "bem_boundary_matrices_bm", "bem_batch_matrices_bm", "bem_geometry_status", "bem_geometry_release",
)


class BEMError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = int(status)
        msg = _status_string(self.status)
        super().__init__(f"{what}: {msg} (status {self.status})" if what else f"{msg} (status {self.status})")


TUNE_ASSEMBLY_CHUNK, TUNE_ASSEMBLY_CTAS_PER_SM, TUNE_TC_PROMOTE, TUNE_GMRES_REORTH, TUNE_ARNOLDI_CLUSTER = 1, 2, 3, 4, 5
TUNE_ARNOLDI_MODE = 6
TUNE_TC_WAIT_US = 7
TUNE_TC_TEST_SKIP_FILL = 8
TUNE_GMRES_BLOCK = 9


class BatchProblem(ctypes.Structure):
    _fields_ = [("geom", ctypes.c_void_p), ("k", ctypes.c_float), ("v_out", ctypes.c_void_p),
                ("k_out", ctypes.c_void_p)]


class BmProblem(ctypes.Structure):
    _fields_ = [("geom", ctypes.c_void_p), ("k", ctypes.c_float), ("lhs_out", ctypes.c_void_p),
                ("rhs_out", ctypes.c_void_p)]


class SolverParams(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("restart", ctypes.c_int),
        ("max_iters", ctypes.c_int),
        ("max_refine", ctypes.c_int),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("inner_rtol", ctypes.c_double),
    ]


class SolverInfo(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("matvecs", ctypes.c_int),
        ("rel_residual", ctypes.c_double),
    ]


_lib = None


def _status_string(st: int) -> str:
    try:
        return lib().bem_status_string(int(st)).decode()
    except Exception:  # pragma: no cover - library missing
        return "error"


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built; run neuralat_b200/build.py (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, f, d, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
    P = ctypes.POINTER
    sigs = {
        "bem_status_string": ([i], ctypes.c_char_p),
        "bem_version": ([], ctypes.c_char_p),
        "bem_kernel_launches": ([], ctypes.c_ulonglong),
        "bem_geometry_bytes": ([vp, i, vp, i, P(sz), vp], i),
        "bem_geometry_build": ([vp, i, vp, i, vp, sz, vp], i),
        "bem_geometry_normals": ([vp, vp, vp, vp], i),
        "bem_boundary_matrix": ([vp, i, i, f, vp, vp, vp, vp], i),
        "bem_boundary_matrices_vk": ([vp, f, vp, vp, f, f, vp], i),
        "bem_identity_matrix": ([vp, vp, vp], i),
        "bem_triangle2vertex": ([vp, vp, vp, vp, vp], i),
        "bem_potential_matrix": ([vp, i, vp, i, f, vp, vp], i),
        "bem_boundary2potential_scratch_bytes": ([i, i], sz),
        "bem_boundary2potential": ([vp, vp, i, f, vp, vp, i, vp, vp, sz, vp], i),
        "bem_cmatmul": ([vp, i, vp, i, vp, vp], i),
        "bem_gmres_workspace_bytes": ([i, i, P(SolverParams)], sz),
        "bem_gmres_solve": ([vp, i, vp, i, vp, i, P(SolverParams), vp, sz, P(SolverInfo), vp], i),
        "bem_tc_operator_bytes": ([i, i, i], sz),
        "bem_tc_operator_prepare": ([vp, i, i, vp, sz, vp], i),
        "bem_tc_matmul": ([vp, sz, i, i, vp, i, vp, vp], i),
        "bem_tc_status": ([vp, vp], i),
        "bem_boundary2potential_noalloc_max": ([], ctypes.c_longlong),
        "bem_boundary2potential_noalloc": ([vp, vp, i, f, vp, vp, i, vp, vp], i),
        "bem_cmatmul_adjoint": ([vp, i, vp, i, vp, vp], i),
        "bem_conj_transpose": ([vp, i, vp, vp], i),
        "bem_boundary2potential_adjoint": ([vp, vp, i, f, vp, vp, vp, vp], i),
        "bem_vertex_gradient": ([vp, f, vp, vp, vp, vp, i, vp, vp, vp], i),
        "bem_batch_workspace_bytes": ([i], sz),
        "bem_batch_matrices_vk": ([P(BatchProblem), i, f, f, vp, sz, vp], i),
        "bem_set_tuning": ([i, i], i),
        "bem_assembly_status": ([vp], i),
        "bem_get_tuning": ([i], i),
        "bem_boundary_matrices_bm": ([vp, i, f, vp, vp, vp], i),
        "bem_batch_matrices_bm": ([P(BmProblem), i, i, vp, sz, vp], i),
        "bem_geometry_status": ([vp, vp], i),
        "bem_geometry_release": ([vp], i),
    }
    for name, (argt, rest) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = argt
        fn.restype = rest
    _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != BEM_OK:
        raise BEMError(status, what)
