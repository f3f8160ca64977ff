"""Generate golden vectors for the two-body mobility kernel from the reference itself.

Run in a container where the reference checkout is available (it is not needed
afterwards): it imports the reference's own ``Net`` wrapper
(python/convert.py:6-20) around the shipped ``nn/two_body_unbounded.pkl`` and
evaluates it in torch FP32 (the path libtorch runs in src/CloseDot.cpp:233,
src/FarDot.cpp:414,739) and in FP64 on seeded inputs. The outputs are committed
as ``two_body_net.npz`` next to this script.

    python tests/golden/make_golden.py /path/to/reference
"""
import hashlib
import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_reference_net(ref_root):
    spec = importlib.util.spec_from_file_location("ref_convert", os.path.join(ref_root, "python", "convert.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)  # defines Net; the CLI part sits under __main__
    seq = torch.load(os.path.join(ref_root, "nn", "two_body_unbounded.pkl"), weights_only=False, map_location="cpu")
    return mod.Net, seq


def seeded_inputs(seed=20240):
    rng = np.random.default_rng(seed)

    def dirs(n):
        v = rng.normal(size=(n, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    parts = []
    # near field: contact to a few leaf diameters (sphere radius 1, contact at 2)
    d = rng.uniform(2.0, 30.0, size=512)
    parts.append(dirs(512) * d[:, None])
    # admissible separations, log-uniform in [4, 400]
    d = np.exp(rng.uniform(np.log(4.0), np.log(400.0), size=512))
    parts.append(dirs(512) * d[:, None])
    # grid-aligned and coincident cases: |r| < 1e-5 maps to the identity
    special = np.array([[0, 0, 0], [1e-6, 0, 0], [0, -3e-6, 2e-6], [2.05, 0, 0], [0, 0, -2.05],
                        [1, 1, 1], [-10, 4, 0.5], [300, -200, 100]], dtype=np.float64)
    parts.append(special)
    # overlapping spheres (clustered configurations have them): |r| in [1e-3, 2]
    d = rng.uniform(1e-3, 2.0, size=64)
    parts.append(dirs(64) * d[:, None])
    return np.concatenate(parts).astype(np.float32)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python " + os.path.relpath(__file__) + " /path/to/reference  (the reference checkout)")
    ref_root = sys.argv[1]
    Net, seq = load_reference_net(ref_root)
    r = seeded_inputs()
    with torch.no_grad():
        y32 = Net(seq.float())(torch.from_numpy(r.copy())).numpy()
        # the inner network alone (what a student network is trained to reproduce)
        inner64 = seq.double()(torch.from_numpy(r.astype(np.float64))).numpy()
    # Net.forward only runs in FP32 (its index_put of a float32 identity fails on a
    # float64 tensor), so the FP64 values apply the same wrapper to the FP64 inner net.
    r64 = r.astype(np.float64)
    nrm = np.sqrt((r64 * r64).sum(1))
    y64 = inner64.copy()
    y64[:, [0, 4, 8]] += 1.0
    with np.errstate(divide="ignore", invalid="ignore"):
        y64 /= nrm[:, None]
    y64[nrm < 1e-5] = np.eye(3).reshape(9)
    wpath = os.path.join(REPO, "hignn_b200", "data", "two_body_unbounded.hgnw")
    sha = hashlib.sha256(open(wpath, "rb").read()).hexdigest() if os.path.exists(wpath) else ""
    np.savez_compressed(os.path.join(HERE, "two_body_net.npz"), r=r, y_fp32=y32, y_fp64=y64,
                        inner_fp64=inner64, weights_sha256=np.array(sha))
    print("wrote", len(r), "cases; weights sha256", sha[:16])


if __name__ == "__main__":
    main()
