"""GPU parity of the plain FP32 path against the CPU oracle (calls go through the C ABI).

Tolerances: the plain FP32 path must be within 1e-5 relative L2 of the
restated reference path on the same inputs and weights; the H-matrix error
against the dense FP64 evaluation is reported and bounded by 1e-3.
"""
import numpy as np
import pytest

from conftest import GOLDEN, WEIGHTS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def make_model(x, leaf=128, **params):
    m = capi.Model(x, leaf, device=0)
    m.load_two_body(WEIGHTS)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    return m


def test_two_body_eval_matches_golden():
    d = np.load(GOLDEN)
    r = torch.from_numpy(d["r"]).cuda()
    y = torch.empty((r.shape[0], 9), dtype=torch.float32, device="cuda")
    m = make_model(np.random.default_rng(0).uniform(0, 50, (256, 3)))
    m.two_body_eval(r.data_ptr(), y.data_ptr(), r.shape[0], 0)
    y = y.cpu().numpy().astype(np.float64)
    err = np.linalg.norm(y - d["y_fp64"], axis=1) / np.linalg.norm(d["y_fp64"], axis=1)
    assert err.max() < 2e-5, err.max()
    err32 = np.linalg.norm(y - d["y_fp32"], axis=1) / np.linalg.norm(d["y_fp32"], axis=1)
    assert err32.max() < 2e-5
    # |r| < 1e-5 gives the identity exactly
    assert np.array_equal(y[1024:1027], np.tile(np.eye(3).reshape(1, 9), (3, 1)))


def test_near_field_matches_oracle(small_workload, oracle_net):
    x, f = small_workload
    m = make_model(x, fields=1)
    u = m.dot(f)
    om = O.OracleModel(x, 128, oracle_net)
    ft = f[om.rmap]
    uc = O.close_dot(om.tree, om.xt, ft, om.closeI, om.closeJ, oracle_net)
    ref = np.empty_like(uc)
    ref[om.rmap] = uc
    assert rel(u, ref) < 1e-6


def _oracle_parts(x, f, net, eps, replays=None, collect=None, leaf=128):
    om = O.OracleModel(x, leaf, net, epsilon=eps, max_iter=100)
    ft = f[om.rmap]
    uc = O.close_dot(om.tree, om.xt, ft, om.closeI, om.closeJ, net)
    uf = O.far_dot(om.tree, om.xt, ft, om.farI, om.farJ, net, eps, 100, collect=collect, replays=replays)
    back = lambda v: v[np.argsort(om.rmap)]
    return back(uc), back(uf), om


def _far_parity(x, f, net, eps):
    """GPU far field vs the oracle replaying the GPU's pivots, and vs the free-running oracle."""
    m = make_model(x, epsilon=eps, record_pivots=1)
    u = m.dot(f)
    rk, rows, cols = m.far_pivots()
    col = []
    uc, uf_free, om = _oracle_parts(x, f, net, eps, collect=col)
    _, uf_rep, _ = _oracle_parts(x, f, net, eps, replays=list(zip(rows, cols)))
    same = np.mean([c[2] == rk[b] and list(c[3]) == list(rows[b]) for b, c in enumerate(col)])
    return u, uc, uf_rep, uf_free, same


def test_dot_matches_oracle_eps_1e2(small_workload, oracle_net_exact):
    """eps 1e-2 (the reference's production setting, python/simulate.py:198): plain FP32 within
    1e-5 of the free-running oracle.

    ACA picks its pivots as the argmax of signed 3x3 determinants (src/FarDot.cpp:557-573), so
    two FP32 networks that round differently choose other, equally valid pivots at near-ties.
    The oracle's FP32 network (TwoBodyF32Exact) performs the device network's operations in the
    same order, so the network outputs agree bit for bit, every block follows the same pivot
    path, and the products agree free-running; the replayed comparison is kept as well.
    """
    x, f = small_workload
    u, uc, uf_rep, uf_free, same = _far_parity(x, f, oracle_net_exact, 1e-2)
    assert rel(u, uc + uf_rep) < 1e-5
    assert rel(u, uc + uf_free) < 1e-5
    assert same >= 0.99, same


@pytest.mark.slow
def test_dot_small_config_eps_1e5(small_workload, oracle_net_exact):
    """N=4,096, phi=0.05, min separation 2.05, leaf 128, eps 1e-5: plain FP32 within 1e-5 of the
    free-running oracle, and within 1e-3 of the FP64 dense evaluation."""
    x, f = small_workload
    u, uc, uf_rep, uf_free, same = _far_parity(x, f, oracle_net_exact, 1e-5)
    assert rel(u, uc + uf_rep) < 1e-5
    assert rel(u, uc + uf_free) < 1e-5
    assert same >= 0.99, same
    rows = np.arange(0, 4096, 16)
    ud = O.dense_rows(x, f, rows, oracle_net_exact, fp64=True)
    assert rel(u[rows], ud) < 1e-3


def test_plain_network_is_bit_exact_with_the_oracle(oracle_net_exact):
    """The plain device network (hignn_two_body_eval, precision 0) and the oracle's FP32
    restatement give identical bits, over the golden features and a wide spread of separations
    (including |r| below 1e-5, where M is the identity)."""
    d = np.load(GOLDEN)
    rng = np.random.default_rng(11)
    v = rng.normal(size=(60000, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    rr = (v * np.exp(rng.uniform(np.log(1e-6), np.log(900.0), 60000))[:, None]).astype(np.float32)
    r = np.concatenate([d["r"], rr]).astype(np.float32)
    rt = torch.from_numpy(r).cuda()
    y = torch.empty((r.shape[0], 9), dtype=torch.float32, device="cuda")
    m = make_model(np.random.default_rng(0).uniform(0, 50, (256, 3)))
    m.two_body_eval(rt.data_ptr(), y.data_ptr(), r.shape[0], 0)
    dev = y.cpu().numpy()
    ora = oracle_net_exact.eval32(r)
    diff = np.flatnonzero(dev.view(np.uint32).ravel() != ora.view(np.uint32).ravel())
    assert diff.size == 0, (diff.size, diff[:10])


def test_dense_dot_matches_oracle(small_workload, oracle_net):
    x, f = small_workload
    m = make_model(x)
    u = m.dense_dot(f)
    rows = np.arange(0, 4096, 97)
    ref = O.dense_rows(x, f, rows, oracle_net, fp64=True)
    assert rel(u[rows], ref) < 1e-5
    ur = m.dense_rows(f, rows, 0)
    assert rel(ur, ref) < 1e-5


def test_symmetry_off_and_small_leaves(oracle_net):
    x = S.uniform(3000, 0.1, 21)
    f = S.sedimenting_forces(3000, 21)
    for sym in (0, 1):
        m = make_model(x, 64, epsilon=1e-2, use_symmetry=sym, record_pivots=1)
        u = m.dot(f)
        rk, rows, cols = m.far_pivots()
        om = O.OracleModel(x, 64, oracle_net, epsilon=1e-2, use_symmetry=bool(sym))
        ft = f[om.rmap]
        ut = O.close_dot(om.tree, om.xt, ft, om.closeI, om.closeJ, oracle_net, bool(sym))
        ut += O.far_dot(om.tree, om.xt, ft, om.farI, om.farJ, oracle_net, 1e-2, 100, bool(sym),
                        replays=list(zip(rows, cols)))
        assert rel(u, ut[np.argsort(om.rmap)]) < 1e-5


def test_edge_cases_single_leaf_and_coincident(oracle_net):
    # N below the leaf size: one close pair, no far field
    x = S.uniform(50, 0.1, 3)
    f = S.sedimenting_forces(50, 3)
    m = make_model(x)
    om = O.OracleModel(x, 128, oracle_net)
    assert rel(m.dot(f), om.dot(f)) < 1e-6
    # coincident particles: M = I for |r| < 1e-5
    x = np.repeat(S.uniform(100, 0.1, 4), 2, axis=0)
    f = S.sedimenting_forces(200, 4)
    m = make_model(x, 32, epsilon=1e-2, fields=1)
    uc, _, _ = _oracle_parts(x, f, oracle_net, 1e-2, leaf=32)
    assert rel(m.dot(f), uc) < 1e-6
    # single particle: u = f
    m = make_model(np.ones((1, 3), np.float32))
    f1 = np.array([[0.3, -0.2, 1.0]], np.float32)
    assert np.allclose(m.dot(f1), f1)


def test_update_coord_and_repeat_deterministic(small_workload):
    x, f = small_workload
    m = make_model(x, epsilon=1e-2)
    u1 = m.dot(f)
    x2 = x + np.float32(0.3)
    m.update_coord(x2)
    u2 = m.dot(f)
    m.update_coord(x)
    u3 = m.dot(f)
    assert rel(u3, u1) < 1e-6  # same inputs: only the FP64 atomic summation order may differ
    assert rel(u2, u1) < 1e-3  # translation invariance of M(x_j - x_i), up to float rounding of x


def test_errors_are_reported():
    m = capi.Model(S.uniform(300, 0.1, 1), 64, device=0)
    with pytest.raises(capi.HignnError) as e:
        m.dot(np.zeros((300, 3), np.float32))
    assert e.value.code == -3  # no weights loaded
    m.load_two_body(WEIGHTS)
    with pytest.raises(ValueError):
        m.dot(np.zeros((299, 3), np.float32))
    with pytest.raises(TypeError):
        m.dot(np.zeros((300, 3), np.float32), u=np.zeros((300, 3), np.float64))


def test_pybind_module_matches_capi(small_workload):
    from hignn_b200 import hignn

    x, f = small_workload
    hm = hignn.HignnModel(x, 128)
    hm.load_two_body_model(WEIGHTS)
    hm.set_epsilon(1e-2)
    hm.update_coord(x)
    u = np.zeros((len(x), 3), np.float32)
    hm.dot(u, f)
    m = make_model(x, epsilon=1e-2)
    assert rel(u, m.dot(f)) < 1e-6
    with pytest.raises(Exception):
        hm.dot(np.zeros((len(x), 3)), f)  # float64 output is rejected, not silently lost


def test_failed_rebuild_leaves_model_unready():
    """A tree the device kernels cannot take (here 300 coincident points: one leaf above the
    256-particle staging limit whatever the block size) is refused on the host, before any
    launch, and leaves the model without a tree: later calls are refused too, none runs on the
    lists of the previous positions."""
    n = 2000
    x = S.uniform(n, 0.1, 7)
    f = S.sedimenting_forces(n, 7)
    m = make_model(x, epsilon=1e-2)
    m.dot(f)
    bad = x.copy()
    bad[:300] = bad[0]
    with pytest.raises(capi.HignnError) as e:
        m.update_coord(bad)
    assert e.value.code == -1
    with pytest.raises(capi.HignnError) as e:
        m.dense_rows_noalloc(f, np.arange(10))
    assert e.value.code == -3
    with pytest.raises(capi.HignnError) as e:
        m.dot(f)  # the rebuild is tried again and refused again
    assert e.value.code == -1
    m.update_coord(x)  # good positions: the model works again
    u = m.dot(f)
    assert np.isfinite(u).all()
    with pytest.raises(capi.HignnError):
        capi.Model(x, 512, device=0)  # block_size above the staging limit


def test_dense_rows_f64_matches_oracle(small_workload, oracle_net):
    """The FP64 dense rows (the network in FP64) against the oracle's FP64 dense evaluation
    (FP64 network, FP64 sums): only summation order and the last bits of tanh may differ."""
    x, f = small_workload
    m = make_model(x)
    rows = np.random.default_rng(3).choice(len(x), 24, replace=False)
    ref = O.dense_rows(x, f, rows, oracle_net, fp64=True)
    u64 = m.dense_rows(f, rows, capi.DENSE_F64)
    assert rel(u64, ref) < 1e-11
    u32 = m.dense_rows(f, rows, 0)  # FP32 network, FP64 sums: FP32 rounding of the network only
    assert rel(u32, ref) < 1e-5


def test_post_check_flag_prints_dense_error(small_workload, capfd):
    """set_post_check_flag(True) (interface/HignnInterface.cpp:27): every dot also computes the
    dense product and prints the relative L2 error of the H-matrix result against it
    (src/PostCheckDot.cpp:351-377); the printed figure matches the error computed here."""
    import re

    x, f = small_workload
    m = make_model(x, epsilon=1e-2)
    m.set(capi.P_POST_CHECK_FLAG, 1)
    u = m.dot(f)
    out = capfd.readouterr().out
    hits = re.findall(r"relative error of the H-matrix product vs the dense product: ([0-9.eE+-]+)", out)
    assert len(hits) == 1, out
    printed = float(hits[0])
    expect = rel(u, m.dense_dot(f))
    assert 1e-6 < printed < 1e-3
    assert abs(printed - expect) <= 0.02 * expect  # float32 rounding of both results only
    m.set(capi.P_POST_CHECK_FLAG, 0)
    u2 = m.dot(f)
    assert "relative error" not in capfd.readouterr().out
    assert rel(u2, u) < 1e-6
