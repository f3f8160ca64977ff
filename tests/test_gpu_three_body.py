"""Three-body + self near field on the tensor cores (C ABI hignn_tb_*) against the reference's
own model classes (golden vectors) and the FP64 oracle.

Layers 2 and 3 take FP16 operands (FP32 accumulation), so the velocities carry the FP16
rounding of the weights and activations: relative L2 error below 3e-3 of the FP64 result over
many edges. A single edge is held to 2e-2 of its velocity: its small matrix entries carry an
error of order 1e-3 of the largest entry.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from hignn_b200.weights import default_three_body_paths  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "three_body_velocity.npz")
TOL = 3e-3


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def tb():
    return capi.ThreeBody(0)


@pytest.mark.parametrize("case", ["filaments", "dense"])
def test_matches_reference_golden(tb, case):
    g = np.load(GOLD)
    tb.set_epsilon(float(g[f"{case}_eps"]))
    u = tb.velocity(g[f"{case}_x"], g[f"{case}_f"])
    err = rel(u, g[f"{case}_v64"])
    print(case, "relative error vs the reference (FP64)", err, tb.stats())
    assert err < TOL


def test_matches_oracle_and_is_repeatable(tb):
    x = S.filaments(96, 32, 2.2, 0.05, 41)
    x = (x + np.random.default_rng(4).normal(0, 0.2, x.shape)).astype(np.float32)
    f = S.sedimenting_forces(len(x), 41)
    tb.set_epsilon(5.0)
    u = tb.velocity(x, f)
    st = tb.stats()
    assert st["triplets"] % 128 != 0  # a ragged last tile
    p3, ps = default_three_body_paths()
    ref = O.three_body_velocity(x, f, 5.0, O.DenseTanh.from_hgnw(p3), O.DenseTanh.from_hgnw(ps))
    err = rel(u, ref)
    print("relative error vs the oracle", err, st)
    assert err < TOL
    u2 = tb.velocity(x, f)
    assert rel(u2, u) < 1e-5  # float atomics: only the order of the sums may differ


def test_caller_edge_lists(tb):
    # the reference's usage (python/gravity_field.py): edge lists from NeighborLists, any order
    g = np.load(GOLD)
    x, f, eps = g["filaments_x"], g["filaments_f"], float(g["filaments_eps"])
    off, nbr = O.neighbour_csr(x, eps)
    tri, _ = O.three_body_edge_info(off, nbr)
    pairs = O.two_body_edge_info(off, nbr)
    rng = np.random.default_rng(5)
    tri = tri[:, rng.permutation(tri.shape[1])]
    pairs = pairs[:, rng.permutation(pairs.shape[1])]
    u = tb.velocity_edges(x, f, tri, pairs)
    assert rel(u, g["filaments_v64"]) < TOL
    tb.set_epsilon(eps)
    assert rel(u, tb.velocity(x, f)) < 1e-5  # the same edges in another order: float sums only
    with pytest.raises(capi.HignnError):
        tb.velocity_edges(x, f, np.array([[0], [1], [len(x)]], np.uint64), pairs)


def test_sparse_and_empty_lists(tb):
    tb.set_epsilon(5.0)
    x = np.array([[0, 0, 0], [100, 0, 0], [0, 100, 0]], np.float32)  # no neighbours at all
    u = tb.velocity(x, np.ones_like(x))
    assert np.array_equal(u, np.zeros_like(x))
    x = np.array([[0, 0, 0], [3, 0, 0], [100, 0, 0]], np.float32)  # one pair, no triplet
    f = np.array([[0, 0, -1], [0, 0, -1], [0, 0, -1]], np.float32)
    u = tb.velocity(x, f)
    p3, ps = default_three_body_paths()
    ref = O.three_body_velocity(x, f, 5.0, O.DenseTanh.from_hgnw(p3), O.DenseTanh.from_hgnw(ps))
    assert tb.stats()["triplets"] == 0 and tb.stats()["pairs"] == 2
    assert rel(u, ref) < 2e-2 and np.all(u[2] == 0)


def test_errors():
    t = capi.ThreeBody(0)
    with pytest.raises(capi.HignnError):
        t.set_epsilon(0.0)
    with pytest.raises(capi.HignnError):
        t.velocity(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))
