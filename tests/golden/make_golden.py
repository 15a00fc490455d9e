"""Generate golden fixtures from the reference's own src/bem CUDA kernels.

Runs on a CUDA machine with the prebuilt reference extension
(``oracle/_ref/neuralat_ref_bem.so``, built by ``oracle/build_ref.py`` from the
unmodified ``src/bem/cuda/bind.cu``).  For each small mesh and wavenumber it
records the outputs of every reference binding (bind.cu:178-223): the 18
boundary matrices, the identity, the two listener potential matrices and
triangle2vertex, with the reference's own preprocess (solver.py:40-58) for
the normals/curls it passes in.

Usage:  python tests/golden/make_golden.py [out_dir]   (default: tests/golden/reference_*.npz)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

LAYERS = ["single", "double", "adjointdouble", "hypersingular", "bm_lhs", "bm_rhs"]
SUFFIXES = ["", "_approx", "_approx_1"]
KS = [1.0, 10.0, 100.0, -100.6]
POINTS = np.array([[0.0, 0.0, 2.0], [0.0, 2.0, 0.0], [2.0, 0.0, 0.0],
                   [0.31, -0.42, 0.27], [-0.5, 0.1, -0.35]], dtype=np.float32)


def meshes():
    from neuralat_b200.bem import meshes as M

    v0, t0 = M.icosphere(0, 1.0)  # the 12-vertex icosahedron of check_with_bempp.py:19
    v1, t1 = M.icosphere(1, 0.2)
    v1 = v1 * np.array([1.3, 0.8, 1.0])  # ellipsoid, non-uniform triangles
    return {"s0": (v0.astype(np.float32), t0), "s1": (v1.astype(np.float32), t1)}


def reference_preprocess(torch, vertices, triangles):
    """The reference's preprocess (solver.py:40-58), re-expressed with torch."""
    v0 = vertices[triangles[:, 0].long()]
    v1 = vertices[triangles[:, 1].long()]
    v2 = vertices[triangles[:, 2].long()]
    rg = torch.tensor([[-1, 1, 0], [-1, 0, 1]], dtype=torch.float32, device=vertices.device)
    n = torch.cross(v1 - v0, v2 - v0, dim=1)
    n = n / torch.norm(n, dim=1, keepdim=True)
    J = torch.stack([v1 - v0, v2 - v0], dim=2)
    JtJ = torch.bmm(J.transpose(1, 2), J)
    jit = torch.bmm(J, torch.inverse(JtJ))
    grads = torch.matmul(jit, rg).transpose(1, 2)
    curls = torch.linalg.cross(n.unsqueeze(1), grads)
    return n.contiguous(), curls.contiguous()


def main(out_dir=HERE):
    import torch

    from oracle import build_ref

    ref = build_ref.load_prebuilt()
    if ref is None:
        raise SystemExit("reference extension not built (oracle/_ref)")
    for name, (v, t) in meshes().items():
        vt = torch.from_numpy(v).cuda()
        tt = torch.from_numpy(t.astype(np.int32)).cuda()
        normals, curls = reference_preprocess(torch, vt, tt)
        out = {"vertices": v, "triangles": t.astype(np.int32), "points": POINTS, "ks": np.array(KS),
               "normals": normals.cpu().numpy(), "curls": curls.cpu().numpy()}
        out["identity"] = ref.identity_matrix(vt, tt).cpu().numpy()
        rng = np.random.default_rng(11)
        tv = (rng.standard_normal(t.shape[0]) + 1j * rng.standard_normal(t.shape[0])).astype(np.complex64)
        out["t2v_in"] = tv
        out["t2v_out"] = ref.triangle2vertex(vt, tt, torch.from_numpy(tv).cuda()).cpu().numpy()
        pts = torch.from_numpy(POINTS).cuda()
        for ki, k in enumerate(KS):
            for layer in LAYERS:
                for suf in SUFFIXES:
                    fn = getattr(ref, f"{layer}_boundary_matrix{suf}")
                    out[f"k{ki}_{layer}{suf}"] = fn(vt, tt, normals, curls, float(k)).cpu().numpy()
            out[f"k{ki}_single_potential"] = ref.single_boundary_potential(vt, tt, pts, float(k)).cpu().numpy()
            out[f"k{ki}_double_potential"] = ref.double_boundary_potential(vt, tt, pts, float(k)).cpu().numpy()
        torch.cuda.synchronize()
        path = os.path.join(out_dir, f"reference_{name}.npz")
        np.savez_compressed(path, **out)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
