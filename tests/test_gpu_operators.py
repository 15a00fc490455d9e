"""All reference operator types and quadrature orders through the C ABI.

Compared with the reference's own kernels (golden fixtures produced by the
unmodified src/bem extension on a B200) and with the FP64 oracle; HBIE and
Burton-Miller solves against the analytic pulsating sphere
(scripts/unit_test.py:27-39,110-123).
"""
import glob
import os

import numpy as np
import pytest
import torch

from neuralat_b200.bem import BEM_Solver
from neuralat_b200.bem import meshes as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "reference_*.npz")))
LAYERS = ["single", "double", "adjointdouble", "hypersingular", "bm_lhs", "bm_rhs"]
APPROX = {"": False, "_approx": True, "_approx_1": "1"}


def relfro(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=GOLDEN, ids=[os.path.basename(f) for f in GOLDEN])
def golden(request):
    z = dict(np.load(request.param))
    z["solver"] = BEM_Solver(z["vertices"], z["triangles"])
    return z


@pytest.mark.parametrize("layer", LAYERS)
@pytest.mark.parametrize("suffix", list(APPROX))
def test_operator_matches_reference_kernels(golden, layer, suffix):
    s = golden["solver"]
    for ki, k in enumerate(golden["ks"]):
        ref = golden[f"k{ki}_{layer}{suffix}"]
        got = s.assemble_boundary_matrix(float(k), layer, approx=APPROX[suffix]).cpu().numpy()
        # the reference is itself FP32 with atomics; both sit within 2e-5 of FP64
        assert relfro(got, ref) <= 3e-5, (layer, suffix, k)


@pytest.mark.parametrize("layer", LAYERS)
@pytest.mark.parametrize("suffix", list(APPROX))
def test_operator_matches_oracle_on_ellipsoid(layer, suffix):
    v, t = M.icosphere(2, 0.15)
    v = (v * np.array([1.25, 0.75, 1.0])).astype(np.float32)
    k = 73.27
    s = BEM_Solver(v, t)
    got = s.assemble_boundary_matrix(k, layer, approx=APPROX[suffix]).cpu().numpy()
    ref = O.boundary_matrix(layer, v.astype(np.float64), t, k, approx=suffix)
    assert relfro(got, ref) <= 1e-5


@pytest.mark.parametrize("method", ["HBIE", "neumann2dirichlet"])
def test_hbie_and_burton_miller_monopole(method):
    v, t = M.icosphere(3, 0.1)
    v = v.astype(np.float32)
    k = -M.wavenumber(1000.0)  # negative k as in scripts/unit_test.py:24
    g = O.monopole_neumann(v, M.vertex_normals(v, t), k).astype(np.complex64)
    s = BEM_Solver(v, t)
    u = getattr(s, method)(k, torch.from_numpy(g).cuda(), tol=1e-14).cpu().numpy()
    assert relfro(u, O.monopole(v, k)) < 2e-2
