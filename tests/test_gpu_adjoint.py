"""Hand-written adjoint of the listener pressures vs central finite differences.

L = sum |p|^2 over listeners (differentiation workload, scaled down to an
icosphere s2 so that the FP64 oracle can evaluate 2 x 64 perturbed problems
in seconds).  Finite differences are taken on the FP64 CPU oracle (full
re-assembly, dense solve) with a step of 1e-4 relative to the mesh radius,
at 64 seeded vertex coordinates and 16 seeded Neumann entries; the adjoint
gradient (FP32 kernels, FP64 reductions) must agree to 1e-3 relative.
"""
import numpy as np
import pytest
import torch

from neuralat_b200.bem import listener_pressure
from neuralat_b200.bem import meshes as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _problem():
    v, t = M.icosphere(2, 0.1)
    v = (v * np.array([1.2, 0.9, 1.0])).astype(np.float32).astype(np.float64)
    k = M.wavenumber(2000.0)
    g = M.smoothed_gaussian_field(v.shape[0], t, 1, seed=3)[:, 0].astype(np.complex64).astype(np.complex128)
    pts = M.sphere_points(128, 0.5, seed=4).astype(np.float32).astype(np.float64)
    return v, t, k, g, pts


def oracle_loss(v, t, k, g, pts):
    u = O.cbie_solve(v, t, k, g)
    p = O.boundary2potential(v, t, k, g, u, pts)
    return float(np.sum(np.abs(p) ** 2))


def _adjoint_grads(v, t, k, g, pts, store=True):
    vt = torch.tensor(v, dtype=torch.float32, device="cuda", requires_grad=True)
    gt = torch.tensor(g, dtype=torch.complex64, device="cuda", requires_grad=True)
    tt = torch.from_numpy(t.astype(np.int32)).cuda()
    pt = torch.tensor(pts, dtype=torch.float32, device="cuda")
    p = listener_pressure(vt, gt, tt, pt, k, store_matrices=store)
    loss = (p.abs() ** 2).sum()
    loss.backward()
    return float(loss), vt.grad.double().cpu().numpy(), gt.grad.cpu().numpy().astype(np.complex128)


def test_forward_loss_matches_oracle():
    v, t, k, g, pts = _problem()
    loss, _, _ = _adjoint_grads(v, t, k, g, pts)
    ref = oracle_loss(v, t, k, g, pts)
    assert abs(loss - ref) / ref < 1e-4


def test_vertex_gradient_vs_finite_differences():
    v, t, k, g, pts = _problem()
    _, gx, _ = _adjoint_grads(v, t, k, g, pts)
    rng = np.random.default_rng(64)
    coords = [(int(rng.integers(v.shape[0])), int(rng.integers(3))) for _ in range(64)]
    h = 1e-4 * 0.1
    fd, adj = [], []
    for vi, c in coords:
        vp = v.copy(); vp[vi, c] += h
        vm = v.copy(); vm[vi, c] -= h
        fd.append((oracle_loss(vp, t, k, g, pts) - oracle_loss(vm, t, k, g, pts)) / (2 * h))
        adj.append(gx[vi, c])
    fd, adj = np.array(fd), np.array(adj)
    err = np.linalg.norm(fd - adj) / np.linalg.norm(fd)
    assert err <= 1e-3, (err, np.abs(fd - adj).max(), np.abs(fd).max())


def test_neumann_gradient_vs_finite_differences():
    v, t, k, g, pts = _problem()
    _, _, gg = _adjoint_grads(v, t, k, g, pts)
    rng = np.random.default_rng(16)
    idx = rng.choice(v.shape[0], 16, replace=False)
    h = 1e-4 * np.abs(g).max()
    fd, adj = [], []
    for j in idx:
        for unit in (1.0, 1j):
            gp = g.copy(); gp[j] += h * unit
            gm = g.copy(); gm[j] -= h * unit
            fd.append((oracle_loss(v, t, k, gp, pts) - oracle_loss(v, t, k, gm, pts)) / (2 * h))
            adj.append(gg[j].real if unit == 1.0 else gg[j].imag)
    fd, adj = np.array(fd), np.array(adj)
    assert np.linalg.norm(fd - adj) / np.linalg.norm(fd) <= 1e-3


def test_recompute_matches_stored():
    v, t, k, g, pts = _problem()
    _, gx1, gg1 = _adjoint_grads(v, t, k, g, pts, store=True)
    _, gx2, gg2 = _adjoint_grads(v, t, k, g, pts, store=False)
    assert np.linalg.norm(gx1 - gx2) / np.linalg.norm(gx1) < 1e-5
    assert np.linalg.norm(gg1 - gg2) / np.linalg.norm(gg1) < 1e-5


# ---- the differentiation workload itself: icosphere s4 (N = 2562), 2 kHz, 128 listeners ----
import os  # noqa: E402

CFG4_FD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cfg4_fd.npz")


def _cfg4():
    w = M.differentiation()
    return (w["vertices"].astype(np.float32).astype(np.float64), w["triangles"].astype(np.int32), float(w["k"]),
            w["neumann"].astype(np.complex64).astype(np.complex128), w["points"].astype(np.float32).astype(np.float64))


@pytest.fixture(scope="module")
def cfg4_grads():
    v, t, k, g, pts = _cfg4()
    return _adjoint_grads(v, t, k, g, pts)


def test_cfg4_gradients_vs_committed_finite_differences(cfg4_grads):
    """Adjoint gradient at all 64 seeded vertex coordinates and 16 Neumann
    entries of the s4 workload against FP64 central differences of the
    oracle (tests/golden/make_cfg4_fd.py): relative error <= 1e-3."""
    f = np.load(CFG4_FD)
    loss, gx, gg = cfg4_grads
    assert abs(loss - float(f["loss"])) / float(f["loss"]) < 1e-4
    adj_v = np.array([gx[a, c] for a, c in f["coords"]])
    err_v = np.linalg.norm(adj_v - f["fd_vertices"]) / np.linalg.norm(f["fd_vertices"])
    assert err_v <= 1e-3, err_v
    adj_g = np.stack([gg[f["neumann_index"]].real, gg[f["neumann_index"]].imag], axis=1)
    err_g = np.linalg.norm(adj_g - f["fd_neumann"]) / np.linalg.norm(f["fd_neumann"])
    assert err_g <= 1e-3, err_g


def test_cfg4_vertex_gradient_vs_live_finite_differences(cfg4_grads):
    """Eight of those coordinates, differenced live on the oracle (base LU
    plus an exact low-rank update per moved vertex)."""
    v, t, k, g, pts = _cfg4()
    F = O.ListenerLoss(v, t, k, g, pts)
    _, gx, _ = cfg4_grads
    coords = np.load(CFG4_FD)["coords"][:8]
    h = 1e-4 * 0.1
    fd = np.array([(F.vertex_loss(a, c, h) - F.vertex_loss(a, c, -h)) / (2 * h) for a, c in coords])
    adj = np.array([gx[a, c] for a, c in coords])
    assert np.linalg.norm(fd - adj) / np.linalg.norm(fd) <= 1e-3
