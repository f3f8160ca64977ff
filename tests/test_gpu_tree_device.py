"""The device build of the cluster tree and the close/far lists against the host build.

Both builds restate HignnModel::Divide / Build / CloseFarCheck (src/HignnModel.cpp:119-198,
src/Build.cpp:17-265, src/CloseFarCheck.cpp:11-465) with the same arithmetic; the host build is
pinned against the oracle (tests/test_tree_lists.py). The device build must give the same tree
rows, permutation and lists, element for element and in the same order, on uniform, clustered,
lattice (exact projection ties), duplicated, planar and ragged inputs, with and without symmetry
and with the size gate max_relative_coord active.
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402


def build(x, leaf, device_tree, **params):
    m = capi.Model(x, leaf, device=0)
    m.set(capi.P_TREE_DEVICE, 1 if device_tree else 0)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    t, p = m.tree()
    lists = m.lists()
    ms = m.stats()["t_build_ms"]
    m.close()
    return t, p, lists, ms


def same(x, leaf, **params):
    th, ph, lh, _ = build(x, leaf, False, **params)
    td, pd, ld, _ = build(x, leaf, True, **params)
    assert np.array_equal(th, td)
    assert np.array_equal(ph, pd)
    for a, b in zip(lh, ld):
        assert np.array_equal(a, b)


def lattice(n_side, spacing=2.5):
    g = np.arange(n_side, dtype=np.float32) * np.float32(spacing)
    return np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)


@pytest.mark.parametrize("case", ["uniform4k", "uniform131k", "clustered262k", "lattice", "duplicates", "plane",
                                  "ragged"])
def test_device_tree_and_lists_match_host(case):
    if case == "uniform4k":
        same(S.uniform_min_dist(4096, 0.05, 0), 128)
    elif case == "uniform131k":
        same(S.uniform(131072, 0.1, 1), 128)
    elif case == "clustered262k":
        same(S.clustered(262144, 0.1, 2), 128)
    elif case == "lattice":  # exact ties in the projections
        same(lattice(24), 64)
    elif case == "duplicates":  # coincident pairs
        same(np.repeat(S.uniform(5000, 0.1, 4), 2, axis=0), 64)
    elif case == "plane":
        x = S.uniform(20000, 0.1, 5)
        x[:, 2] = 0.0
        same(x, 128)
    else:  # sizes around the leaf size
        for n in (1, 50, 128, 129, 1000, 3001):
            same(S.uniform(n, 0.1, n), 128)


def test_device_lists_symmetry_off_and_size_gate():
    x = S.uniform(30000, 0.1, 8)
    same(x, 64, use_symmetry=0)
    same(x, 128, max_relative_coord=3000)
    same(x, 128, max_relative_coord=3000, use_symmetry=0)


@pytest.mark.slow
def test_device_tree_1m_matches_host_and_is_faster():
    x = S.clustered(1048576, 0.10, 2)
    th, ph, lh, ms_host = build(x, 128, False)
    build(x, 128, True)  # first device build: allocations and module loading
    td, pd, ld, ms_dev = build(x, 128, True)
    print("TREE_BUILD_1M " + json.dumps({"host_ms": ms_host, "device_ms": ms_dev}))
    assert np.array_equal(th, td) and np.array_equal(ph, pd)
    for a, b in zip(lh, ld):
        assert np.array_equal(a, b)
    assert ms_dev < ms_host
