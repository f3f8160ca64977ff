"""Far-field student network: device gradients against autograd on the CPU, training, and use inside ACA.

The student (3-32-32-32-9 SiLU on x = r_hat ln(|r|/2), predicting the teacher's
inner output minus the Rotne-Prager-Yamakawa tensor) is trained by the
library's own forward/backward/Adam kernels. Per entry it stays within a few
1e-3 of the teacher (the teacher carries ~2e-3 rms of structure that no small
smooth network reproduces); summed into velocities that deviation averages out.
"""
import time

import numpy as np
import pytest

from conftest import WEIGHTS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def student_torch(params):
    """The student as a float64 torch module over the flat parameter layout of the C ABI."""
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    offs = [(0, (32, 3)), (96, (32,)), (128, (32, 32)), (1152, (32,)), (1184, (32, 32)), (2208, (32,)),
            (2240, (9, 32)), (2528, (9,))]

    def get(i):
        o, sh = offs[i]
        return p[o:o + int(np.prod(sh))].reshape(sh)

    def fwd(r):
        r = torch.as_tensor(r, dtype=torch.float64)
        d = torch.linalg.norm(r, dim=1, keepdim=True)
        x = r / d * torch.log(d / 2.0)
        h = torch.nn.functional.silu(x @ get(0).T + get(1))
        h = torch.nn.functional.silu(h @ get(2).T + get(3))
        h = torch.nn.functional.silu(h @ get(4).T + get(5))
        return h @ get(6).T + get(7)

    return p, fwd


def features(n, seed, lo=4.0, hi=400.0):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * np.exp(rng.uniform(np.log(lo), np.log(hi), n))[:, None]).astype(np.float32)


def make_model(x, **params):
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    return m


def test_student_gradient_matches_autograd():
    m = make_model(S.uniform(500, 0.1, 1))
    rng = np.random.default_rng(7)
    params = (rng.normal(size=capi.STUDENT_PARAMS) * 0.2).astype(np.float32)
    m.set_student(params)
    n = 1000  # several CTAs of 128 and a partial one
    r = features(n, 3)
    t = (rng.normal(size=(n, 9)) * 0.01).astype(np.float32)
    # keep the device copies alive: a temporary's memory goes back to the caching allocator at once
    rd, td = torch.from_numpy(r).cuda(), torch.from_numpy(t).cuda()
    g_dev, loss_dev = m.student_grad(rd.data_ptr(), td.data_ptr(), n)
    p, fwd = student_torch(params)
    loss = ((fwd(r) - torch.as_tensor(t, dtype=torch.float64)) ** 2).mean()
    loss.backward()
    g = p.grad.numpy()
    assert abs(loss_dev - loss.item()) / loss.item() < 1e-5
    assert rel(g_dev, g) < 1e-4, rel(g_dev, g)


def test_student_eval_matches_cpu_forward():
    m = make_model(S.uniform(500, 0.1, 1))
    params = (np.random.default_rng(9).normal(size=capi.STUDENT_PARAMS) * 0.2).astype(np.float32)
    m.set_student(params)
    r = features(4096, 4)
    y = torch.empty((4096, 9), device="cuda")
    rd = torch.from_numpy(r).cuda()
    m.student_eval(rd.data_ptr(), y.data_ptr(), 4096)
    _, fwd = student_torch(params)
    d = np.linalg.norm(r.astype(np.float64), axis=1, keepdims=True)
    rh = r / d
    rpy = 0.75 * ((1 + 2 / (3 * d[:, :, None] ** 2)) * np.eye(3)[None]
                  + (1 - 2 / d[:, :, None] ** 2) * rh[:, :, None] * rh[:, None, :]) - np.eye(3)[None]
    with torch.no_grad():
        inner = fwd(r).numpy() + rpy.reshape(-1, 9)
    ref = (inner + np.eye(3).reshape(1, 9)) / d
    assert rel(y.cpu().numpy(), ref) < 1e-5


@pytest.fixture(scope="module")
def trained():
    m = make_model(S.uniform(500, 0.1, 1))
    t0 = time.time()
    loss = m.train_student(steps=4000, batch=16384, nsamples=2_000_000, lr=1e-3, seed=3)
    return m.get_student(), loss, time.time() - t0


def test_student_training_fits_teacher(trained, oracle_net):
    params, loss, seconds = trained
    assert loss < 1e-5, loss  # the residual targets have ~4e-6 mean square
    m = make_model(S.uniform(500, 0.1, 1))
    m.set_student(params)
    r = features(8192, 11)
    y = torch.empty((8192, 9), device="cuda")
    rd = torch.from_numpy(r).cuda()
    m.student_eval(rd.data_ptr(), y.data_ptr(), 8192)
    ref = oracle_net.eval64(r)
    err = np.linalg.norm(y.cpu().numpy() - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) < 6e-3 and np.percentile(err, 99) < 2e-2, (np.median(err), np.percentile(err, 99))


def test_student_far_field_accuracy_and_gain(trained, oracle_net):
    """What the student gains over the same method without it: far-field time at the same velocity accuracy."""
    params, _, _ = trained
    x = S.uniform(30000, 0.1, 21)
    f = S.sedimenting_forces(30000, 21)
    rows = np.random.default_rng(2).choice(len(x), 96, replace=False)
    ud = O.dense_rows(x, f, rows, oracle_net, fp64=True)
    res = {}
    for prec in (1, 2):
        m = make_model(x, epsilon=1e-2, precision=prec, timing=1)
        if prec == 2:
            m.set_student(params)
        m.dot(f)
        u = m.dot(f)
        st = m.stats()
        res[prec] = (rel(u[rows], ud), st["t_far_ms"], st["far_evals"])
    err_teacher, far_teacher, _ = res[1]
    err_student, far_student, _ = res[2]
    assert err_student < 1e-3, res
    assert err_student < err_teacher + 3e-4, res
    assert far_student < far_teacher, res
