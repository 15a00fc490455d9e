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
        L.oracle_boundary_matrix_cols.argtypes = [c_int, c_int, c_int, dp, c_int, ip, c_int, c_double, ip, c_int,
                                                  dp]
        L.oracle_pair_block.argtypes = [c_int, c_int, c_int, dp, c_int, ip, c_int, c_int, c_int, c_double, dp]
        L.oracle_identity_matrix.argtypes = [dp, c_int, ip, c_int, dp]
        L.oracle_potential_matrix.argtypes = [c_int, dp, c_int, ip, c_int, dp, c_int, c_double, dp]
        L.oracle_triangle2vertex.argtypes = [c_int, ip, c_int, dp, dp]
        for f in ("oracle_boundary_matrix", "oracle_boundary_matrix_cols", "oracle_pair_block", "oracle_identity_matrix",
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


def boundary_matrix_cols(layer, vertices, triangles, k, cols, approx: str = "") -> np.ndarray:
    """Columns ``cols`` of the dense complex128 Galerkin matrix: (nv, len(cols))."""
    code = LAYER_CODES[layer] if isinstance(layer, str) else int(layer)
    line_n, tri_n = ORDERS[approx]
    v, t = _mesh(vertices, triangles)
    cols = np.ascontiguousarray(np.asarray(cols, dtype=np.int32))
    out = np.zeros((v.shape[0], cols.size), dtype=np.complex128)
    rc = lib().oracle_boundary_matrix_cols(code, line_n, tri_n, _dp(v), v.shape[0], _ip(t), t.shape[0], float(k),
                                           _ip(cols), cols.size, _dp(out.view(np.float64)))
    if rc:
        raise ValueError(f"oracle_boundary_matrix_cols failed ({rc})")
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


class ListenerLoss:
    """L = sum |p|^2 of the listener pressures p = -S g + D u, (1/2 M - K) u =
    -V g (solver.py:97-104,140-147), in FP64, for a base problem and for
    perturbations of one vertex coordinate or one Neumann entry: the checker
    of the hand-written adjoint by central finite differences.

    Moving vertex a changes only the integrals over the triangles around a,
    hence only the rows and columns of V, K and M that belong to their
    vertices R.  The perturbed solve is the base LU factorisation plus a
    Woodbury correction of rank 2|R| (exact, up to rounding), so one
    evaluation costs a few matrix rows instead of a full re-assembly."""

    def __init__(self, vertices, triangles, k, neumann, points):
        import scipy.linalg as sla

        self.v, self.t = _mesh(vertices, triangles)
        self.k = float(k)
        self.g = np.asarray(neumann, np.complex128).reshape(-1)
        self.pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
        v, t, k = self.v, self.t, self.k
        self.V = boundary_matrix("single", v, t, k)
        self.K = boundary_matrix("double", v, t, k)
        self.M = identity_matrix(v, t)
        self.lu = sla.lu_factor(0.5 * self.M - self.K)
        self._sla = sla
        self.b = -self.V @ self.g
        self.u = sla.lu_solve(self.lu, self.b)
        self.S = potential_matrix("single", v, t, self.pts, k)
        self.D = potential_matrix("double", v, t, self.pts, k)
        self.p = -self.S @ self.g + self.D @ self.u
        self.loss = float(np.sum(np.abs(self.p) ** 2))
        self._stars = {}

    def _rows_of(self, a):
        if a not in self._stars:
            star = np.any(self.t == a, axis=1)
            self._stars[a] = np.unique(self.t[star])
        return self._stars[a]

    def _rows_cols(self, v, R):
        """Rows R and columns R of V and of A = 1/2 M - K on mesh v."""
        t, k = self.t, self.k
        Vr = boundary_matrix("single", v, t, k, rows=R)
        Vc = boundary_matrix_cols("single", v, t, k, R)
        Kr = boundary_matrix("double", v, t, k, rows=R)
        Kc = boundary_matrix_cols("double", v, t, k, R)
        M = identity_matrix(v, t)
        return Vr, Vc, 0.5 * M[R, :] - Kr, 0.5 * M[:, R] - Kc

    def vertex_loss(self, a, c, delta):
        """L with vertex a's coordinate c moved by delta."""
        R = self._rows_of(int(a))
        v2 = self.v.copy()
        v2[a, c] += delta
        Vr0, Vc0, Ar0, Ac0 = self._rows_cols(self.v, R)
        Vr1, Vc1, Ar1, Ac1 = self._rows_cols(v2, R)
        n, r = self.v.shape[0], R.size
        inR = np.zeros(n, bool)
        inR[R] = True
        dVr, dVc = Vr1 - Vr0, (Vc1 - Vc0) * (~inR)[:, None]
        dAr, dAc = Ar1 - Ar0, (Ac1 - Ac0) * (~inR)[:, None]
        # b' = -(V + E dVr + dVc E^T) g
        b2 = self.b.copy()
        b2[R] -= dVr @ self.g
        b2 -= dVc @ self.g[R]
        # A' = A + U W with U = [E, dAc], W = [dAr; E^T]
        E = np.zeros((n, r), np.complex128)
        E[R, np.arange(r)] = 1.0
        U = np.concatenate([E, dAc], axis=1)
        W = np.concatenate([dAr, E.T], axis=0)
        Z = self._sla.lu_solve(self.lu, U)
        y = self._sla.lu_solve(self.lu, b2)
        cap = np.eye(2 * r) + W @ Z
        u2 = y - Z @ np.linalg.solve(cap, W @ y)
        S2 = potential_matrix("single", v2, self.t, self.pts, self.k)
        D2 = potential_matrix("double", v2, self.t, self.pts, self.k)
        p2 = -S2 @ self.g + D2 @ u2
        return float(np.sum(np.abs(p2) ** 2))

    def neumann_loss(self, j, delta):
        """L with Neumann entry j changed by the complex delta (p is linear in g)."""
        e = np.zeros_like(self.g)
        e[j] = delta
        du = self._sla.lu_solve(self.lu, -self.V @ e)
        p2 = self.p + (-self.S @ e + self.D @ du)
        return float(np.sum(np.abs(p2) ** 2))
