"""Native host tree and close/far lists against the oracle restatement (bit-exact)."""
import numpy as np
import pytest

from hignn_b200 import capi
from hignn_b200 import synthetic as S
from oracle import hignn_oracle as O


def native(x, leaf, sym=True, max_rel=500000):
    m = capi.Model(x, leaf, device=-1)
    m.set(capi.P_USE_SYMMETRY, sym)
    m.set(capi.P_MAX_RELATIVE_COORD, max_rel)
    t, p = m.tree()
    return t, p, m.lists(), m


def oracle(x, leaf, sym=True, max_rel=500000):
    t, p = O.build_tree(x, leaf)
    aux = O.compute_aux(t, x[p])
    ci, cj, fi, fj, lv = O.close_far_lists(t, aux, max_rel, sym)
    return t, p, (ci, cj, fi, fj)


CASES = [
    ("small_min_dist", lambda: S.uniform_min_dist(4096, 0.05, 0), 128),
    ("uniform_20k", lambda: S.uniform(20000, 0.1, 7), 128),
    ("clustered_30k", lambda: S.clustered(30000, 0.1, 2), 128),
    ("leaf_64", lambda: S.uniform(5000, 0.1, 3), 64),
    ("ragged_1001", lambda: S.uniform(1001, 0.2, 4), 50),
    # exact ties and signed zeros among the projections: the sort must keep input order for equal keys
    ("lattice_ties", lambda: (np.stack(np.meshgrid(*[np.arange(32)] * 3, indexing="ij"), -1)
                              .reshape(-1, 3).astype(np.float32) - np.float32(15.5)), 100),
    # the benchmark's workload: nodes of >= 2^18 particles take the threaded radix sort
    ("clustered_1m", lambda: S.clustered(1048576, 0.10, 2), 128),
]


@pytest.mark.parametrize("name,gen,leaf", CASES, ids=[c[0] for c in CASES])
def test_tree_and_lists_bit_exact(name, gen, leaf):
    x = gen()
    t, p, lists, _ = native(x, leaf)
    ot, op, olists = oracle(x, leaf)
    assert np.array_equal(t, ot)
    assert np.array_equal(p, op)
    for a, b in zip(lists, olists):
        assert np.array_equal(a, b)


def test_no_symmetry_and_size_gate():
    x = S.uniform(8000, 0.1, 11)
    for sym, max_rel in ((False, 500000), (True, 1500), (False, 700)):
        _, _, lists, _ = native(x, 100, sym, max_rel)
        _, _, olists = oracle(x, 100, sym, max_rel)
        for a, b in zip(lists, olists):
            assert np.array_equal(a, b)


def test_tree_invariants():
    x = S.clustered(20000, 0.1, 5)
    t, p, (ci, cj, fi, fj), m = native(x, 128)
    assert np.array_equal(np.sort(p), np.arange(len(x)))
    # one-rank layout: root children re-pointed to rows 3, 4; rows 1, 2 orphaned
    assert t[0, 0] == 3 and t[0, 1] == 4 and t[0, 2] == 0 and t[0, 3] == len(x)
    leaves = [i for i in range(len(t)) if t[i, 0] == 0 and i not in (1, 2)]
    assert max(t[i, 3] - t[i, 2] for i in leaves) <= 128
    for i in range(3, len(t)):
        if t[i, 0]:
            c0, c1 = t[i, 0], t[i, 1]
            assert t[c0, 2] == t[i, 2] and t[c0, 3] == t[c1, 2] and t[c1, 3] == t[i, 3]
            assert t[c0, 4] == t[i, 4] + 1
    assert np.all(cj >= ci) and np.all(fj >= fi)


def test_coverage_exactly_once():
    x = S.uniform(3000, 0.1, 9)
    t, p, (ci, cj, fi, fj), _ = native(x, 64)
    n = len(x)
    cover = np.zeros((n, n), np.int16)
    for I, J in zip(list(ci) + list(fi), list(cj) + list(fj)):
        a, b, c, d = t[I, 2], t[I, 3], t[J, 2], t[J, 3]
        cover[a:b, c:d] += 1
        if J != I:
            cover[c:d, a:b] += 1
    assert np.all(cover == 1)


def test_edge_cases():
    # fewer particles than a leaf: the root is one leaf (the reference reads past its tree here)
    x = S.uniform(40, 0.1, 1)
    t, p, (ci, cj, fi, fj), _ = native(x, 128)
    assert t.shape == (1, 5) and list(ci) == [0] and list(cj) == [0] and len(fi) == 0
    ot, op, ol = oracle(x, 128)
    assert np.array_equal(t, ot)
    # coincident points: splits that would leave a child empty make a leaf instead of looping
    x = np.zeros((500, 3), np.float32)
    x[250:] = 5.0
    t, p, lists, _ = native(x, 100)
    ot, op, ol = oracle(x, 100)
    assert np.array_equal(t, ot) and np.array_equal(p, op)
    # one particle
    t, p, (ci, cj, fi, fj), _ = native(np.ones((1, 3), np.float32), 4)
    assert list(ci) == [0]
    with pytest.raises(capi.HignnError):
        capi.Model(np.zeros((0, 3), np.float32), 4, device=-1)
    with pytest.raises(capi.HignnError):
        capi.Model(np.array([[np.nan, 0, 0]], np.float32), 4, device=-1)


def test_tree_does_not_depend_on_the_thread_count(monkeypatch):
    # 300k particles: the root's divisions take the threaded radix sort (nodes of >= 2^18)
    x = S.clustered(300000, 0.1, 6)
    out = []
    for threads in ("1", "5", "16"):
        monkeypatch.setenv("HIGNN_HOST_THREADS", threads)
        t, p, lists, _ = native(x, 128)
        out.append((t, p, lists))
    for t, p, lists in out[1:]:
        assert np.array_equal(t, out[0][0]) and np.array_equal(p, out[0][1])
        for a, b in zip(lists, out[0][2]):
            assert np.array_equal(a, b)
