"""Python face of the FP64 CPU oracle (test infrastructure only).

Loads ``oracle/_build/libbem_oracle.so`` (built from ``oracle/bem_oracle.cpp``
by ``oracle/Makefile``) through ctypes and adds the FP64 dense solve and the
analytic monopole.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module; the product path never does.

Layer codes follow the reference's ``PotentialType`` order
(``src/bem/cuda/include/potential.h:7-15``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libbem_oracle.so")

SINGLE, DOUBLE, ADJOINT_DOUBLE, HYPERSINGULAR, BM_LHS, BM_RHS = range(6)
LAYER_CODES = {
    "single": SINGLE,
    "double": DOUBLE,
    "adjointdouble": ADJOINT_DOUBLE,
    "hypersingular": HYPERSINGULAR,
    "bm_lhs": BM_LHS,
    "bm_rhs": BM_RHS,
}
# (line rule, triangle rule) per reference binding suffix (bind.cu:180-215)
ORDERS = {"": (4, 6), "_approx": (2, 3), "_approx_1": (2, 1)}

_lib = None


def build() -> str:
    """Compile the oracle library if it is missing or stale."""
    src = os.path.join(HERE, "bem_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.oracle_boundary_matrix.argtypes = [c_int, c_int, c_int, dp, c_int, ip, c_int, c_double, ip, c_int, dp]
        L.oracle_pair_block.argtypes = [c_int, c_int, c_int, dp, c_int, ip, c_int, c_int, c_int, c_double, dp]
        L.oracle_identity_matrix.argtypes = [dp, c_int, ip, c_int, dp]
        L.oracle_potential_matrix.argtypes = [c_int, dp, c_int, ip, c_int, dp, c_int, c_double, dp]
        L.oracle_triangle2vertex.argtypes = [c_int, ip, c_int, dp, dp]
        for f in ("oracle_boundary_matrix", "oracle_pair_block", "oracle_identity_matrix",
                  "oracle_potential_matrix", "oracle_triangle2vertex", "oracle_num_threads"):
            getattr(L, f).restype = c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _mesh(vertices, triangles):
    v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, 3))
    t = np.ascontiguousarray(np.asarray(triangles, dtype=np.int32).reshape(-1, 3))
    return v, t


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def boundary_matrix(layer, vertices, triangles, k, approx: str = "", rows=None) -> np.ndarray:
    """Dense complex128 Galerkin matrix (or the requested rows of it)."""
    code = LAYER_CODES[layer] if isinstance(layer, str) else int(layer)
    line_n, tri_n = ORDERS[approx]
    v, t = _mesh(vertices, triangles)
    nv = v.shape[0]
    if rows is None:
        out = np.zeros((nv, nv), dtype=np.complex128)
        rp, nr = None, nv
    else:
        rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int32))
        out = np.zeros((rows.size, nv), dtype=np.complex128)
        rp, nr = _ip(rows), rows.size
    rc = lib().oracle_boundary_matrix(code, line_n, tri_n, _dp(v), nv, _ip(t), t.shape[0], float(k), rp, nr,
                                      _dp(out.view(np.float64)))
    if rc:
        raise ValueError(f"oracle_boundary_matrix failed ({rc})")
    return out


def pair_block(layer, vertices, triangles, i, j, k, approx: str = "") -> np.ndarray:
    code = LAYER_CODES[layer] if isinstance(layer, str) else int(layer)
    line_n, tri_n = ORDERS[approx]
    v, t = _mesh(vertices, triangles)
    out = np.zeros(10, dtype=np.complex128)
    rc = lib().oracle_pair_block(code, line_n, tri_n, _dp(v), v.shape[0], _ip(t), t.shape[0], int(i), int(j),
                                 float(k), _dp(out.view(np.float64)))
    if rc:
        raise ValueError("oracle_pair_block failed")
    return out


def identity_matrix(vertices, triangles) -> np.ndarray:
    v, t = _mesh(vertices, triangles)
    nv = v.shape[0]
    out = np.zeros((nv, nv), dtype=np.complex128)
    lib().oracle_identity_matrix(_dp(v), nv, _ip(t), t.shape[0], _dp(out.view(np.float64)))
    return out


def potential_matrix(layer, vertices, triangles, points, k) -> np.ndarray:
    code = LAYER_CODES[layer] if isinstance(layer, str) else int(layer)
    v, t = _mesh(vertices, triangles)
    p = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    out = np.zeros((p.shape[0], v.shape[0]), dtype=np.complex128)
    rc = lib().oracle_potential_matrix(code, _dp(v), v.shape[0], _ip(t), t.shape[0], _dp(p), p.shape[0], float(k),
                                       _dp(out.view(np.float64)))
    if rc:
        raise ValueError("oracle_potential_matrix failed")
    return out


def triangle2vertex(nv, triangles, values) -> np.ndarray:
    t = np.ascontiguousarray(np.asarray(triangles, dtype=np.int32).reshape(-1, 3))
    vals = np.ascontiguousarray(np.asarray(values, dtype=np.complex128))
    out = np.zeros(nv, dtype=np.complex128)
    with np.errstate(all="ignore"):
        lib().oracle_triangle2vertex(int(nv), _ip(t), t.shape[0], _dp(vals.view(np.float64)),
                                     _dp(out.view(np.float64)))
    return out


# ---- composite operations (solver.py:97-147) ------------------------------

def cbie_system(vertices, triangles, k):
    """(LHS, V) of the CBIE: LHS = M/2 - K, RHS = -V g (solver.py:97-104)."""
    M = identity_matrix(vertices, triangles)
    V = boundary_matrix("single", vertices, triangles, k)
    K = boundary_matrix("double", vertices, triangles, k)
    return 0.5 * M - K, V


def cbie_solve(vertices, triangles, k, neumann) -> np.ndarray:
    """FP64 dense solve of the exterior Neumann CBIE; neumann (N,) or (N, m)."""
    lhs, V = cbie_system(vertices, triangles, k)
    return np.linalg.solve(lhs, -V @ np.asarray(neumann, dtype=np.complex128))


def boundary2potential(vertices, triangles, k, neumann, dirichlet, points) -> np.ndarray:
    S = potential_matrix("single", vertices, triangles, points, k)
    D = potential_matrix("double", vertices, triangles, points, k)
    return -S @ np.asarray(neumann, np.complex128) + D @ np.asarray(dirichlet, np.complex128)


def monopole(points, k, x0=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Analytic pressure e^{ikr}/(4 pi r) of a unit monopole (scripts/unit_test.py:27-31)."""
    d = np.asarray(points, np.float64) - np.asarray(x0, np.float64)
    r = np.linalg.norm(d, axis=-1)
    return np.exp(1j * k * r) / (4 * np.pi * r)


def monopole_neumann(points, normals, k, x0=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Normal derivative of the monopole (scripts/unit_test.py:33-39)."""
    d = np.asarray(points, np.float64) - np.asarray(x0, np.float64)
    r = np.linalg.norm(d, axis=-1)
    ikr = 1j * k * r
    return -np.exp(ikr) / (4 * np.pi * r ** 3) * (1 - ikr) * np.sum(d * np.asarray(normals, np.float64), axis=-1)
