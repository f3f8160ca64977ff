"""The oracle's neighbour lists (include/NeighborLists.hpp restated) against independent forms.

The reference has no test of its own for NeighborLists, so the restatement is checked against an
all-pairs search with the same metric, the reference's loop structure for the triplets, and the
float-squared radius rule. CPU only.
"""
import numpy as np

from hignn_b200 import synthetic as S
from oracle import hignn_oracle as O


def test_candidate_search_matches_all_pairs():
    rng = np.random.default_rng(0)
    x = (rng.random((600, 3)) * 25).astype(np.float32)
    x[10] = x[11]  # a coincident pair: distance 0 < eps^2, a neighbour both ways
    for eps in (0.5, 3.0, 5.0):
        off, nbr = O.neighbour_csr(x, eps)
        off2, nbr2 = O.neighbour_csr_brute(x, eps)
        assert np.array_equal(off, off2) and np.array_equal(nbr, nbr2)
    off, nbr = O.neighbour_csr(x, 3.0)
    assert 11 in nbr[off[10]:off[11]] and 10 in nbr[off[11]:off[12]]


def test_radius_is_squared_in_float():
    # float(0.1)^2 rounded in float (0.0100000007) exceeds the double square (0.0100000003), so a
    # pair exactly float(0.1) apart is a neighbour under the reference's rule
    x = np.array([[0, 0, 0], [np.float32(0.1), 0, 0], [0, 0.2, 0]], np.float32)
    off, nbr = O.neighbour_csr(x, 0.1)
    assert list(nbr[off[0]:off[1]]) == [1] and list(nbr[off[1]:off[2]]) == [0]
    assert off[3] - off[2] == 0


def test_triplets_follow_the_reference_loops():
    x = S.filaments(12, 16, 2.2, 0.05, 3)
    off, nbr = O.neighbour_csr(x, 5.0)
    info, off3 = O.three_body_edge_info(off, nbr)
    assert np.array_equal(info, O.three_body_edge_info_loops(off, nbr))
    # per-particle counts: sum over j in N(i) of |N(j)| - 1 (include/NeighborLists.hpp:520-529)
    deg = np.diff(off)
    cnt = np.array([sum(deg[j] - 1 for j in nbr[off[i]:off[i + 1]]) for i in range(len(x))])
    assert np.array_equal(np.diff(off3), cnt)


def test_by_index_forms():
    x = S.filaments(4, 8, 2.2, 0.05, 5)
    off, nbr = O.neighbour_csr(x, 5.0)
    info, off3 = O.three_body_edge_info(off, nbr)
    idx = np.array([3, 0, 3, 31], np.uint64)
    got = O.edge_info_by_index(info, off3, idx)
    want = np.concatenate([info[::-1, off3[p]:off3[p + 1]] for p in (3, 0, 3, 31)], axis=1)
    assert np.array_equal(got, want)
    two = O.two_body_edge_info_by_index(5, [2, 4])
    assert two.tolist() == [[0, 1, 3, 4, 0, 1, 2, 3], [2, 2, 2, 2, 4, 4, 4, 4]]
