"""Device neighbour lists (C ABI hignn_nbl_*) against the oracle: bit-exact edge lists.

Each particle's neighbours come out in ascending order on both sides, so the (rows, E) arrays
must be equal element for element; the reference's own order within a particle is its kd-tree's
traversal order, so parity with it is parity of the per-particle sets.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402


def build(x, eps2, eps3):
    nl = capi.NeighborLists(0)
    nl.update_coord(x)
    nl.set_two_body_epsilon(eps2)
    nl.set_three_body_epsilon(eps3)
    nl.build_two_body_info()
    nl.build_three_body_info()
    return nl


def check_all(x, eps2, eps3, index):
    nl = build(x, eps2, eps3)
    off2, nbr2 = O.neighbour_csr(x, eps2)
    off3, nbr3 = O.neighbour_csr(x, eps3)
    trip, toff = O.three_body_edge_info(off3, nbr3)
    self3 = O.two_body_edge_info(off3, nbr3)
    assert np.array_equal(nl.edges(capi.EDGES_TWO_BODY), O.two_body_edge_info(off2, nbr2))
    assert np.array_equal(nl.edges(capi.EDGES_THREE_BODY), trip)
    assert np.array_equal(nl.edges(capi.EDGES_THREE_BODY_SELF), self3)
    assert np.array_equal(nl.edges(capi.EDGES_THREE_BODY, index), O.edge_info_by_index(trip, toff, index))
    assert np.array_equal(nl.edges(capi.EDGES_THREE_BODY_SELF, index), O.edge_info_by_index(self3, off3, index))
    assert np.array_equal(nl.edges(capi.EDGES_TWO_BODY, index), O.two_body_edge_info_by_index(len(x), index))
    return nl


def test_filaments_config_shape():
    # filaments of 32 beads 2.2 apart at volume fraction 0.05, three-body cutoff 5
    x = S.filaments(512, 32, 2.2, 0.05, 3)
    idx = np.random.default_rng(0).integers(0, len(x), 300).astype(np.uint64)
    nl = check_all(x, 3.0, 5.0, idx)
    assert nl.edges(capi.EDGES_THREE_BODY).shape[1] > 10 * len(x)


def test_uniform_and_clustered():
    check_all(S.uniform_min_dist(20000, 0.1, 11), 2.5, 4.0, np.array([0, 19999, 7, 7], np.uint64))
    check_all(S.clustered(30000, 0.1, 12), 2.1, 3.0, np.arange(0, 30000, 97, dtype=np.uint64))


def test_edge_cases():
    # float-squared radius: a pair exactly float(0.1) apart is a neighbour at eps 0.1
    x = np.array([[0, 0, 0], [np.float32(0.1), 0, 0], [0, 0.2, 0]], np.float32)
    nl = build(x, 0.1, 0.1)
    assert nl.edges(capi.EDGES_TWO_BODY).tolist() == [[0, 1], [1, 0]]
    assert nl.edges(capi.EDGES_THREE_BODY).shape == (3, 0)
    # coincident particles are neighbours of each other; an isolated particle has no edges
    x = np.array([[1, 1, 1], [1, 1, 1], [1, 1, 1.5], [40, 40, 40]], np.float32)
    check_all(x, 1.0, 1.0, np.array([3, 0], np.uint64))
    # one particle, and widely spread coordinates (the cell grid is capped)
    check_all(np.array([[5, 5, 5]], np.float32), 1.0, 2.0, np.array([0], np.uint64))
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.random((2000, 3)) * 10, rng.random((50, 3)) * 1e5]).astype(np.float32)
    check_all(x, 1.0, 1.5, np.arange(0, 2050, 41, dtype=np.uint64))


def test_errors_and_lifetime():
    nl = capi.NeighborLists(0)
    nl.update_coord(S.uniform(100, 0.1, 1))
    with pytest.raises(capi.HignnError):
        nl.build_two_body_info()  # epsilon 0: the reference's lists underflow here
    assert nl.edges(capi.EDGES_TWO_BODY).shape == (2, 0)  # nothing built yet
    nl.set_two_body_epsilon(4.0)
    nl.build_two_body_info()
    with pytest.raises(capi.HignnError):
        nl.edges(capi.EDGES_THREE_BODY, np.array([100], np.uint64))  # index out of range
    before = nl.edges(capi.EDGES_TWO_BODY)
    nl.update_coord(S.uniform(100, 0.1, 2))  # lists stay until the next build
    assert np.array_equal(nl.edges(capi.EDGES_TWO_BODY), before)
    ptr, e = nl.device_edges(capi.EDGES_TWO_BODY)
    assert ptr and e == before.shape[1]


def test_pybind_neighbor_lists():
    from hignn_b200 import hignn

    x = S.filaments(64, 32, 2.2, 0.05, 4)
    nl = hignn.NeighborLists()
    nl.update_coord(x)
    nl.set_two_body_epsilon(3.0)
    nl.set_three_body_epsilon(5.0)
    nl.build_two_body_info()
    nl.build_three_body_info()
    off2, nbr2 = O.neighbour_csr(x, 3.0)
    off3, nbr3 = O.neighbour_csr(x, 5.0)
    trip, toff = O.three_body_edge_info(off3, nbr3)
    idx = np.array([5, 1000, 5], np.uint64)
    assert np.array_equal(nl.get_two_body_edge_info(), O.two_body_edge_info(off2, nbr2))
    assert np.array_equal(nl.get_three_body_edge_info(), trip)
    assert np.array_equal(nl.get_three_body_edge_self_info(), O.two_body_edge_info(off3, nbr3))
    assert np.array_equal(nl.get_three_body_edge_info_by_index(idx), O.edge_info_by_index(trip, toff, idx))
    assert np.array_equal(nl.get_three_body_edge_self_info_by_index(idx),
                          O.edge_info_by_index(O.two_body_edge_info(off3, nbr3), off3, idx))
    assert np.array_equal(nl.get_two_body_edge_info_by_index(idx[:1]), O.two_body_edge_info_by_index(len(x), idx[:1]))
    assert nl.get_two_body_edge_info().dtype == np.uint64
    with pytest.raises(RuntimeError):
        nl.set_periodic(True)
