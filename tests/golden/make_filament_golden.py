"""Generate golden filament forces from the reference's own chain_bending / chain_tension.

Run in a container where the reference checkout is available (it is not needed afterwards).
python/simulate.py imports hignn, mpi4py and h5py at module level, so only its two force
functions are compiled from its source (python/simulate.py:14-88) and called, per filament, the
way velocity_update assembles the force (python/simulate.py:130-142): a float32 body force,
then += bending, then += tension. The outputs are committed as ``filament_forces.npz``.

    python tests/golden/make_filament_golden.py /path/to/reference
"""
import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from hignn_b200 import synthetic as S  # noqa: E402


def load_reference_forces(ref_root):
    path = os.path.join(ref_root, "python", "simulate.py")
    tree = ast.parse(open(path).read(), path)
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ("chain_bending", "chain_tension")]
    ns = {"np": np}
    exec(compile(ast.Module(body=defs, type_ignores=[]), path, "exec"), ns)
    return ns["chain_bending"], ns["chain_tension"]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python " + os.path.relpath(__file__) + " /path/to/reference  (the reference checkout)")
    ref_root = sys.argv[1]
    bending, tension = load_reference_forces(ref_root)
    cases = {}
    rng = np.random.default_rng(7)
    # (n_filament, n_chain, rest length, k_t, k_b, position jitter, free particles)
    for name, (nf, nc, L, kt, kb, jit, free) in {
        "chains": (64, 32, 2.2, 100.0, 10.0, 0.3, 0),
        "short": (40, 3, 2.0, 50.0, 5.0, 0.5, 17),
        "pairs": (30, 2, 2.5, 1.0, 1.0, 0.2, 0),
        "single": (5, 1, 2.2, 100.0, 10.0, 0.1, 3),
    }.items():
        x = S.filaments(nf, nc, L, 0.05, 100 + nc)
        x = (x + rng.normal(0, jit, x.shape)).astype(np.float32)
        if free:
            x = np.concatenate([x, rng.uniform(0, 50, (free, 3)).astype(np.float32)])
        f0 = np.zeros((len(x), 3), np.float32)
        f0 += np.float32([0.0, 0.0, -1.0])
        f = f0.copy()
        for i in range(nf):
            pos3 = x[nc * i:nc * i + nc, :3]
            f[nc * i:nc * i + nc, :] += bending(pos3, kb)
            f[nc * i:nc * i + nc, :] += tension(pos3, kt, L)
        cases[name] = dict(x=x, f0=f0, f=f, params=np.array([nf, nc, L, kt, kb]))
    out = {}
    for name, c in cases.items():
        for k, v in c.items():
            out[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "filament_forces.npz"), **out)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
