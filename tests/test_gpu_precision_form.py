"""Precision form at full size: N = 131,072 spheres (phi 0.10, minimum separation 2.05, seed 1), eps 1e-4.

The BF16 tensor-core form (two-body network in BF16 with FP32 accumulation, ACA with the FP64
stopping-norm estimate) and the plain FP32 form run on the same inputs. Both are compared with
the dense product on a random 16,384-particle sub-sample of target rows, each row summed over
all N sources (hignn_dense_rows: FP32 network, FP64 accumulation). That dense kernel is itself
pinned at this size against the oracle's FP64 dense rows on 24 of the sampled rows.
At this tolerance the ACA of the largest blocks stops at max_iter = 100, as the reference's
does, so both forms are bounded by their measured error with a margin, the BF16 one by the
1e-3 of the workload's specification.
"""
import json

import numpy as np
import pytest

from conftest import WEIGHTS

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_precision_form_131k(oracle_net):
    x, f, p = S.workload("medium")
    rows = np.sort(np.random.default_rng(1).choice(len(x), 16384, replace=False))
    u, st = {}, {}
    for prec in (0, 1):
        m = capi.Model(x, p["leaf"], device=0)
        m.load_two_body(WEIGHTS)
        m.set(capi.P_PRECISION, prec)
        m.set(capi.P_EPSILON, p["epsilon"])
        m.set(capi.P_MAX_ITER, p["max_iter"])
        m.set(capi.P_TIMING, 1)
        m.dot(f)  # records the ranks of the plan
        u[prec] = m.dot(f)
        st[prec] = m.stats()
    ud = m.dense_rows(f, rows, 0)
    pin = O.dense_rows(x, f, rows[:24], oracle_net, fp64=True)
    e_pin = rel(ud[:24], pin)
    e_plain, e_bf16 = rel(u[0][rows], ud), rel(u[1][rows], ud)
    print(json.dumps({"n": len(x), "epsilon": p["epsilon"], "rel_l2_plain_fp32": e_plain, "rel_l2_bf16": e_bf16,
                      "dense_rows_vs_oracle_fp64": e_pin,
                      "dot_ms": {"plain_fp32": st[0]["t_dot_ms"], "bf16": st[1]["t_dot_ms"]},
                      "far_rank_max": {"plain_fp32": st[0]["far_rank_max"], "bf16": st[1]["far_rank_max"]}}))
    assert e_pin < 1e-5, e_pin
    # At eps 1e-4 the largest blocks reach max_iter (rank 100) before the stopping rule holds, so
    # the plain form's error sits above eps (2.3e-4 measured); the BF16 network adds its own
    # rounding (7.1e-4 measured).
    assert e_plain < 5e-4, e_plain
    assert e_bf16 < 1e-3, e_bf16
