"""Seeded synthetic suspensions with the shapes of the benchmark workloads.

No public dataset is involved: every workload is generated here from a seed.
All coordinates are in sphere radii (radius 1, contact at separation 2).
"""
from __future__ import annotations

import math

import numpy as np


def cube_side(n: int, phi: float) -> float:
    """Side of the cube holding n unit spheres at volume fraction phi."""
    return (n * 4.0 * math.pi / 3.0 / phi) ** (1.0 / 3.0)


def uniform_min_dist(n: int, phi: float, seed: int, min_dist: float = 2.05) -> np.ndarray:
    """Uniform centres in a cube sized for ``phi``; random sequential rejection to ``min_dist``.

    A candidate is accepted iff no previously accepted centre lies within
    ``min_dist`` (candidates are visited in draw order).
    """
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    L = cube_side(n, phi)
    acc = np.empty((0, 3))
    while acc.shape[0] < n:
        m = max(4096, 4 * (n - acc.shape[0]))
        cand = rng.uniform(0.0, L, size=(m, 3))
        if acc.shape[0]:
            d, _ = cKDTree(acc).query(cand, k=1, distance_upper_bound=min_dist)
            cand = cand[~(d < min_dist)]
        if cand.shape[0] == 0:
            continue
        pairs = cKDTree(cand).query_pairs(min_dist, output_type="ndarray")
        removed = np.zeros(cand.shape[0], bool)
        if len(pairs):
            pairs = pairs[np.lexsort((pairs[:, 0], pairs[:, 1]))]  # by j, then i
            for i, j in pairs:
                if not removed[i]:
                    removed[j] = True
        keep = cand[~removed][: n - acc.shape[0]]
        acc = np.concatenate([acc, keep])
    return acc.astype(np.float32)


def clustered(n: int, phi: float, seed: int, n_clusters: int = 64, sigma: float = 8.0,
              background: float = 0.5) -> np.ndarray:
    """Gaussian clusters (``sigma`` radii) plus a uniform background fraction, in the phi cube."""
    rng = np.random.default_rng(seed)
    L = cube_side(n, phi)
    n_bg = int(round(n * background))
    n_cl = n - n_bg
    centres = rng.uniform(0.0, L, size=(n_clusters, 3))
    which = rng.integers(0, n_clusters, size=n_cl)
    pts_cl = centres[which] + rng.normal(0.0, sigma, size=(n_cl, 3))
    pts_bg = rng.uniform(0.0, L, size=(n_bg, 3))
    pts = np.concatenate([pts_cl, pts_bg])
    return pts[rng.permutation(n)].astype(np.float32)


def uniform(n: int, phi: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, cube_side(n, phi), size=(n, 3)).astype(np.float32)


def filaments(n_filament: int, n_chain: int, bond: float, phi: float, seed: int) -> np.ndarray:
    """Straight chains of ``n_chain`` beads ``bond`` apart, random starts and directions in a cube
    sized for ``phi`` (filament f holds rows f * n_chain .. (f + 1) * n_chain - 1)."""
    rng = np.random.default_rng(seed)
    n = n_filament * n_chain
    side = cube_side(n, phi)
    start = rng.uniform(0.0, side, size=(n_filament, 1, 3))
    d = rng.normal(size=(n_filament, 1, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    k = np.arange(n_chain, dtype=np.float64)[None, :, None]
    return (start + bond * k * d).reshape(n, 3).astype(np.float32)


def sedimenting_forces(n: int, seed: int) -> np.ndarray:
    """F_i = (0, 0, -1) + N(0, 0.1^2) per component, FP32."""
    rng = np.random.default_rng(seed + 1000)
    f = rng.normal(0.0, 0.1, size=(n, 3))
    f[:, 2] -= 1.0
    return f.astype(np.float32)


def workload(name: str):
    """(coords, forces, params) for a named workload.

    ``small``:   N=4,096, phi=0.05, seed 0, min separation 2.05, eps 1e-5.
    ``medium``:  N=131,072, phi=0.10, seed 1, min separation 2.05, eps 1e-4.
    ``large``:   N=1,048,576, phi=0.10, seed 2, 64 Gaussian clusters (sigma 8) + 50% uniform.
    """
    if name == "small":
        x = uniform_min_dist(4096, 0.05, 0)
        return x, sedimenting_forces(4096, 0), dict(leaf=128, epsilon=1e-5, max_iter=100)
    if name == "medium":
        x = uniform_min_dist(131072, 0.10, 1)
        return x, sedimenting_forces(131072, 1), dict(leaf=128, epsilon=1e-4, max_iter=100)
    if name == "large":
        x = clustered(1048576, 0.10, 2)
        return x, sedimenting_forces(1048576, 2), dict(leaf=128, epsilon=1e-3, max_iter=100)
    raise ValueError(name)
