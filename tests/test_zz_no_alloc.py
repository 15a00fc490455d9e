"""The listener-evaluation entry point that allocates nothing.

Callers that cannot allocate device memory while they run (a real-time audio
loop synthesising sound from listener pressures must not block on the
allocator; a C plug-in may have no device allocator at all) use
bem_boundary2potential_noalloc, whose scratch is a fixed array inside the
library.  This file is collected last on purpose: if it fails, a run that stops
at the first failure has already run every other test.  It checks, through
the C ABI, that two calls in a row agree with the scratch-buffer entry point
bem_boundary2potential within the listener-pressure tolerance, that the
result matches the FP64 oracle (with both densities, and with only a
Dirichlet density, the double-layer potential), and that an oversized
request is refused before any work.
"""
import ctypes

import numpy as np
import pytest
import torch

from neuralat_b200 import _lib as L
from neuralat_b200.bem import BEM_Solver
from neuralat_b200.bem import meshes as M
from neuralat_b200.bem.solver import _stream, _vp
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PRESSURE_TOL = 1e-4


def _case(seed, m):
    rng = np.random.default_rng(seed)
    nv = _SOLVER.geometry.nv
    g = (rng.standard_normal((nv, m)) + 1j * rng.standard_normal((nv, m))).astype(np.complex64)
    u = (rng.standard_normal((nv, m)) + 1j * rng.standard_normal((nv, m))).astype(np.complex64)
    pts = M.sphere_points(90, 0.5, seed=seed).astype(np.float32)
    return torch.from_numpy(g).cuda(), torch.from_numpy(u).cuda(), torch.from_numpy(pts).cuda()


_SOLVER = None


_MESH = None


@pytest.fixture(scope="module", autouse=True)
def solver():
    global _SOLVER, _MESH
    v, t = M.icosphere(2, 0.15)
    v = (v * np.array([1.25, 0.75, 1.0])).astype(np.float32)
    _MESH = (v.astype(np.float64), t)
    _SOLVER = BEM_Solver(v, t)
    yield _SOLVER


def _noalloc(k, g, u, pts):
    lib = L.lib()
    m = (g if g is not None else u).shape[1]
    out = torch.empty((pts.shape[0], m), dtype=torch.complex64, device="cuda")
    st = lib.bem_boundary2potential_noalloc(_SOLVER.geometry.ptr, _vp(pts), int(pts.shape[0]), float(k), _vp(g),
                                            _vp(u), m, _vp(out), _stream())
    L.check(st, "bem_boundary2potential_noalloc")
    return out


def test_noalloc_matches_scratch_entry_point_on_two_calls():
    for call, (seed, m, k) in enumerate([(1, 3, 73.27), (2, 9, 18.3)]):
        g, u, pts = _case(seed, m)
        ref = _SOLVER.boundary2potential(k, g, u, pts)  # bem_boundary2potential with a scratch buffer
        got = _noalloc(k, g, u, pts)
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
        assert err <= PRESSURE_TOL, (call, err)


def test_noalloc_matches_fp64_oracle():
    k = 40.0
    g, u, pts = _case(3, 2)
    got = _noalloc(k, g, u, pts).cpu().numpy()
    v, t = _MESH
    ref = O.boundary2potential(v, t, np.float32(k), g.cpu().numpy(), u.cpu().numpy(), pts.cpu().numpy())
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= PRESSURE_TOL, err


def test_noalloc_dirichlet_density_only_is_the_double_layer_potential():
    """neumann = NULL: the call evaluates D u alone (solver.py:134-138)."""
    k = 25.0
    _, u, pts = _case(4, 3)
    got = _noalloc(k, None, u, pts)
    ref = _SOLVER.double_potential(k, u, pts)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref)) <= PRESSURE_TOL
    v, t = _MESH
    D = O.potential_matrix("double", v, t, pts.cpu().numpy(), np.float32(k))
    ref64 = D @ u.cpu().numpy().astype(np.complex128)
    err = np.linalg.norm(got.cpu().numpy() - ref64) / np.linalg.norm(ref64)
    assert err <= PRESSURE_TOL, err


def test_noalloc_rejects_oversized_request():
    lib = L.lib()
    limit = int(lib.bem_boundary2potential_noalloc_max())
    nt = _SOLVER.geometry.nt
    m = limit // (6 * nt) + 1
    pts = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    out = torch.empty((4, m), dtype=torch.complex64, device="cuda")
    st = lib.bem_boundary2potential_noalloc(_SOLVER.geometry.ptr, _vp(pts), 4, 1.0, ctypes.c_void_p(0),
                                            ctypes.c_void_p(0), m, _vp(out), _stream())
    assert st == L.BEM_ERR_WORKSPACE
