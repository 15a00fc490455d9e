"""The audio-dataset generator on the CUDA path against the FP64 oracle:
Burton-Miller solve (the <2,3> rules) of a displaced vibrating sphere next to
a static one, |p| at shell listeners (relative error <= 1e-4), and the x
layout of the reference's format recomputed from the same seed."""
import math

import numpy as np
import pytest
import torch

from neuralat_b200.bem import dataset as D
from neuralat_b200.bem import meshes as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scene():
    vv, vt = M.icosphere(2, 0.05)
    sv, st = M.icosphere(1, 0.08)
    sv = sv + np.array([0.25, 0.0, 0.0])
    return vv.astype(np.float32), vt, sv.astype(np.float32), st


def test_generated_samples_match_fp64_oracle_and_layout(tmp_path):
    vv, vt, sv, st = _scene()
    cfg = dict(src_pos_min=[-0.05, -0.02, -0.03], src_pos_max=[0.05, 0.02, 0.03], bbox_center=[0.1, 0.0, 0.0],
               bbox_r=0.4, r_max=2.0, freq_min=200.0, freq_max=4000.0, trg_sample_num=24, src_sample_num=2)
    vib_neumann = (vv[:, 1] <= 0.0).astype(np.complex64)  # part of the object vibrates, as in the reference
    data = D.generate_audio_samples(vv, vt, sv, st, vib_neumann=vib_neumann, seed=7,
                                    solve_kw=dict(tol=1e-14), **cfg)
    x, y = data["x"].numpy(), data["y"].numpy()
    assert x.shape == (2, 24, 5) and y.shape == (2, 24, 1)
    assert x.dtype == np.float32 and y.dtype == np.float32
    rng = np.random.default_rng(7)
    for i in range(2):
        src_base = rng.random(3)
        disp = src_base * (np.array(cfg["src_pos_max"]) - cfg["src_pos_min"]) + cfg["src_pos_min"]
        base = rng.random((24, 3))
        fb = float(rng.random())
        np.testing.assert_allclose(x[i, :, :3], base, rtol=0, atol=1e-7)
        assert np.allclose(x[i, :, 3], src_base[1]) and np.allclose(x[i, :, 4], fb)
        # FP64 oracle: (BM_lhs + I/2) u = (BM_rhs - (i/k) I/2) g, p = D u - S g
        k = 2 * math.pi * D.log_frequency(fb, cfg["freq_min"], cfg["freq_max"]) / D.SPEED_OF_SOUND
        v = np.concatenate([(vv + disp).astype(np.float32), sv]).astype(np.float64)  # the vertices the GPU saw
        t = np.concatenate([vt, st + vv.shape[0]])
        g = np.concatenate([vib_neumann, np.zeros(sv.shape[0])]).astype(np.complex128)
        I = O.identity_matrix(v, t)
        lhs = O.boundary_matrix("bm_lhs", v, t, k, approx="_approx") + 0.5 * I
        rhs = (O.boundary_matrix("bm_rhs", v, t, k, approx="_approx") - 0.5j / k * I) @ g
        u = np.linalg.solve(lhs, rhs)
        pts = D.shell_points(base, cfg["bbox_center"], cfg["bbox_r"], cfg["r_max"]).astype(np.float32)
        p = O.boundary2potential(v, t, k, g, u, pts.astype(np.float64))
        ref = np.abs(p)
        assert np.linalg.norm(y[i, :, 0] - ref) / np.linalg.norm(ref) <= 1e-4
    path = tmp_path / "samples.pt"
    D.save_audio_dataset(str(path), data)
    back = torch.load(str(path))
    assert set(back) == {"x", "y"} and torch.equal(back["x"], data["x"])


def test_batched_generation_matches_sequential():
    vv, vt, sv, st = _scene()
    cfg = dict(src_pos_min=[-0.05, -0.02, -0.03], src_pos_max=[0.05, 0.02, 0.03], bbox_center=[0.1, 0.0, 0.0],
               bbox_r=0.4, r_max=2.0, freq_min=200.0, freq_max=4000.0, trg_sample_num=32, src_sample_num=7)
    seq = D.generate_audio_samples(vv, vt, sv, st, seed=3, solve_kw=dict(tol=1e-14), **cfg)
    bat = D.generate_audio_samples(vv, vt, sv, st, seed=3, solve_kw=dict(tol=1e-14), batch_size=3, workers=2, **cfg)
    assert torch.equal(seq["x"], bat["x"])  # same draws, same layout
    ys, yb = seq["y"].numpy(), bat["y"].numpy()
    for i in range(cfg["src_sample_num"]):
        assert np.linalg.norm(yb[i] - ys[i]) / np.linalg.norm(ys[i]) <= 1e-5, i
