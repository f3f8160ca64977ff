"""Generate golden three-body + self velocities from the reference's own HIGNN model classes.

Run in a container where the reference checkout is available (it is not needed afterwards). It
imports python/HIGNN/model_structure.py (Three_body_net, Two_body_self_net and the HIGNN model's
forward, :41-139) with a stand-in for the absent torch_scatter package (scatter with
reduce='add' as an index_add), loads the shipped python/Saved_Model/Unbounded networks, and
evaluates the forward with no two-body edges -- as python/gravity_field.py:31-52 does -- on
seeded filament suspensions, in torch FP32 and FP64. The edge lists are the oracle's
NeighborLists restatement at the three-body epsilon. Outputs: ``three_body_velocity.npz``.

    python tests/golden/make_three_body_golden.py /path/to/reference
"""
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402


def scatter(src, index, dim=0, dim_size=None, reduce="add"):
    assert dim == 0 and reduce == "add"
    out = torch.zeros((dim_size,) + tuple(src.shape[1:]), dtype=src.dtype)
    return out.index_add_(0, index, src)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python " + os.path.relpath(__file__) + " /path/to/reference  (the reference checkout)")
    ref = sys.argv[1]
    sys.modules["torch_scatter"] = types.SimpleNamespace(scatter=scatter)
    sys.path.insert(0, os.path.join(ref, "python"))
    import HIGNN.model_structure as ms

    model_cls = getattr(ms, "HIGNN_model", None) or getattr(ms, "HIGNN_mdoel")
    saved = os.path.join(ref, "python", "Saved_Model", "Unbounded")
    load = lambda name: torch.load(os.path.join(saved, name), weights_only=False, map_location="cpu")  # noqa: E731
    model = model_cls(load("HIGNN_nn_2body.pkl"), load("HIGNN_nn_3body.pkl"), load("HIGNN_nn_self.pkl"))
    out = {}
    for name, (nf, nc, eps, seed) in {"filaments": (24, 32, 5.0, 31), "dense": (48, 16, 4.0, 32)}.items():
        x = S.filaments(nf, nc, 2.2, 0.08, seed)
        x = (x + np.random.default_rng(seed).normal(0, 0.2, x.shape)).astype(np.float32)
        f = S.sedimenting_forces(len(x), seed)
        off, nbr = O.neighbour_csr(x, eps)
        tri, _ = O.three_body_edge_info(off, nbr)
        pairs = O.two_body_edge_info(off, nbr)
        for dtype, tag in ((torch.float32, "v32"), (torch.float64, "v64")):
            m = model.to(dtype)
            X = torch.tensor(x, dtype=torch.float32).to(dtype)
            F = torch.tensor(f, dtype=torch.float32).to(dtype)
            e2 = torch.zeros((2, 0), dtype=torch.long)
            e3 = torch.tensor(tri.astype(np.int64))
            es = torch.tensor(pairs.astype(np.int64))
            e1 = torch.arange(len(x)).reshape(1, -1)
            with torch.no_grad():
                v = m(X, e2, e3, es, e1, F[e2[0]], F[e3[0]], F[es[1]], F)
            out[f"{name}_{tag}"] = v.numpy()
        out[f"{name}_x"], out[f"{name}_f"], out[f"{name}_eps"] = x, f, np.float32(eps)
        print(name, len(x), "triplets", tri.shape[1], "pairs", pairs.shape[1])
    np.savez_compressed(os.path.join(HERE, "three_body_velocity.npz"), **out)


if __name__ == "__main__":
    main()
