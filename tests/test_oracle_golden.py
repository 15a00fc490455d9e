"""The FP64 CPU oracle pinned against the reference's own src/bem kernels.

tests/golden/reference_*.npz hold outputs of every binding of the reference
extension (bind.cu:178-223), produced on a B200 by tests/golden/make_golden.py
from the unmodified reference sources.  The reference computes in FP32 with
atomics, so agreement is at FP32 rounding level (relative Frobenius).
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "reference_*.npz")))
LAYERS = ["single", "double", "adjointdouble", "hypersingular", "bm_lhs", "bm_rhs"]
SUFFIXES = ["", "_approx", "_approx_1"]
TOL = 2e-5


def relfro(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=FILES, ids=[os.path.basename(f) for f in FILES])
def golden(request):
    return dict(np.load(request.param))


def test_fixtures_present():
    assert len(FILES) >= 2


@pytest.mark.parametrize("layer", LAYERS)
@pytest.mark.parametrize("suffix", SUFFIXES)
def test_boundary_matrices(golden, layer, suffix):
    v, t = golden["vertices"], golden["triangles"]
    for ki, k in enumerate(golden["ks"]):
        ref = golden[f"k{ki}_{layer}{suffix}"]
        assert relfro(O.boundary_matrix(layer, v, t, k, approx=suffix), ref) <= TOL, (layer, suffix, k)


def test_identity_and_potentials(golden):
    v, t = golden["vertices"], golden["triangles"]
    assert relfro(O.identity_matrix(v, t), golden["identity"]) <= 1e-6
    for ki, k in enumerate(golden["ks"]):
        for lay in ("single", "double"):
            ref = golden[f"k{ki}_{lay}_potential"]
            assert relfro(O.potential_matrix(lay, v, t, golden["points"], k), ref) <= TOL


def test_triangle2vertex(golden):
    t = golden["triangles"]
    out = O.triangle2vertex(golden["vertices"].shape[0], t, golden["t2v_in"])
    assert relfro(out, golden["t2v_out"]) <= 1e-6


def fp64_normals_and_curls(v, t):
    """Unit normals and surface curls n x grad(phi_b) of the P1 hat functions
    in FP64: grad phi_b from the inverse metric (J^T J)^-1 of the edge
    vectors, the quantities of the reference's preprocess (solver.py:40-58)."""
    v = v.astype(np.float64)
    p0, p1, p2 = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    e1, e2 = p1 - p0, p2 - p0
    n = np.cross(e1, e2)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    J = np.stack([e1, e2], axis=2)                       # (T, 3, 2)
    G = np.linalg.inv(np.einsum("tia,tib->tab", J, J))  # (T, 2, 2)
    d = np.einsum("tia,tab->tib", J, G)                  # columns: grad of the 2nd and 3rd barycentric
    grads = np.stack([-(d[:, :, 0] + d[:, :, 1]), d[:, :, 0], d[:, :, 1]], axis=1)  # (T, 3 functions, 3)
    curls = np.cross(n[:, None, :], grads)
    return n, curls


def test_normals_and_curls_match_reference_preprocess(golden):
    """Unit normals and surface curls (used by the hypersingular and
    Burton-Miller operators) against the reference's own preprocess output."""
    n, curls = fp64_normals_and_curls(golden["vertices"], golden["triangles"])
    assert np.abs(n - golden["normals"]).max() < 1e-6
    scale = np.abs(golden["curls"]).max()
    assert np.abs(curls - golden["curls"]).max() <= 1e-5 * scale


@pytest.mark.parametrize("suffix", SUFFIXES)
def test_burton_miller_operators_are_the_hbie_combination(golden, suffix):
    """bm_lhs = -K + (i/k) W and bm_rhs = -V - (i/k) K' at every order: the
    identity behind assembling HBIE (solver.py:106-116) as the Burton-Miller
    pair.  Exact to rounding in the FP64 restatement (all operators share
    their quadrature points), within FP32 rounding in the reference's own
    kernels."""
    v, t = golden["vertices"], golden["triangles"]
    for ki, k in enumerate(golden["ks"]):
        beta = 1j / k
        mats = {l: O.boundary_matrix(l, v, t, k, approx=suffix) for l in LAYERS}
        assert relfro(mats["bm_lhs"], -mats["double"] + beta * mats["hypersingular"]) <= 1e-12, (suffix, k)
        assert relfro(mats["bm_rhs"], -mats["single"] - beta * mats["adjointdouble"]) <= 1e-12, (suffix, k)
        g = {l: golden[f"k{ki}_{l}{suffix}"] for l in LAYERS}
        assert relfro(g["bm_lhs"], -g["double"] + beta * g["hypersingular"]) <= TOL, (suffix, k)
        assert relfro(g["bm_rhs"], -g["single"] - beta * g["adjointdouble"]) <= TOL, (suffix, k)
