"""Tensor-core (tcgen05, BF16 with FP32 accumulation) path against the FP64 oracle.

Tolerances: a BF16 network is not expected to match FP32 to 1e-5. Per 3x3
block the BF16 evaluation stays within 1e-2 relative (typical 1e-3); summed
into velocities the error must stay below 1e-3 relative L2 against the dense
FP64 evaluation, the bar of the mixed-precision form.
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


def eval_tc(m, r, precision):
    rt = torch.from_numpy(np.ascontiguousarray(r, np.float32)).cuda()
    y = torch.empty((rt.shape[0], 9), dtype=torch.float32, device="cuda")
    m.two_body_eval(rt.data_ptr(), y.data_ptr(), rt.shape[0], precision)
    return y.cpu().numpy().astype(np.float64)


def test_tc_eval_matches_golden():
    d = np.load(GOLDEN)
    m = make_model(np.random.default_rng(0).uniform(0, 50, (256, 3)))
    y = eval_tc(m, d["r"], 1)
    ref = d["y_fp64"]
    err = np.linalg.norm(y - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) < 3e-3 and err.max() < 1e-2, (np.median(err), err.max())
    assert np.array_equal(y[1024:1027], np.tile(np.eye(3).reshape(1, 9), (3, 1)))


def test_tc_eval_many_tiles_and_ragged_tail(oracle_net):
    rng = np.random.default_rng(3)
    n = 148 * 128 * 3 + 77  # several tiles per CTA and a partial last tile
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = (v * np.exp(rng.uniform(np.log(2.0), np.log(300.0), n))[:, None]).astype(np.float32)
    m = make_model(np.random.default_rng(0).uniform(0, 50, (256, 3)))
    y = eval_tc(m, r, 1)
    ref = oracle_net.eval64(r)
    assert rel(y, ref) < 2e-3
    y2 = eval_tc(m, r, 1)
    assert np.array_equal(y, y2)  # deterministic


def test_tc_near_field(small_workload, oracle_net):
    x, f = small_workload
    m = make_model(x, fields=1, precision=1)
    u = m.dot(f)
    om = O.OracleModel(x, 128, oracle_net)
    ft = f[om.rmap]
    # FP64 near field of the same lists
    uc = np.zeros((len(x), 3))
    for I, J in zip(om.closeI, om.closeJ):
        a, b, c, d = om.tree[I, 2], om.tree[I, 3], om.tree[J, 2], om.tree[J, 3]
        r = (om.xt[c:d][None, :, :] - om.xt[a:b][:, None, :]).reshape(-1, 3)
        M = oracle_net.eval64(r).reshape(b - a, d - c, 3, 3)
        uc[a:b] += np.einsum("ijrc,jc->ir", M, ft[c:d].astype(np.float64))
        if J > I:
            uc[c:d] += np.einsum("ijrc,ic->jr", M, ft[a:b].astype(np.float64))
    ref = uc[np.argsort(om.rmap)]
    assert rel(u, ref) < 1e-3


def test_tc_dot_vs_dense_fp64(small_workload, oracle_net):
    x, f = small_workload
    m = make_model(x, epsilon=1e-2, precision=1)
    u = m.dot(f)
    rows = np.arange(0, 4096, 16)
    ud = O.dense_rows(x, f, rows, oracle_net, fp64=True)
    assert rel(u[rows], ud) < 1e-3
    mp = make_model(x, epsilon=1e-2, precision=0)
    assert rel(u, mp.dot(f)) < 1e-3
