"""Learned far field at full size: N = 4,194,304 spheres uniform at volume fraction 0.10 (seed 4).

The student (3-32-32-32-9 SiLU) is trained on the device with the workload's own settings (Adam,
lr 1e-3, batch 65,536, 20,000 steps, 10M teacher samples at separations 4-400 radii, log-uniform
in distance, uniform directions) and then queried inside ACA for every admissible block; each
converged block is checked on 64 sampled entries against the teacher and sent back to it when
the relative residual exceeds 1e-3 (the library's default student tolerance).

Checks, through the C ABI:
* the velocities of the BF16 + student form are within 1e-3 relative L2 of the dense sum over
  all N sources on 512 sampled rows (FP32 network, FP64 accumulation: hignn_dense_rows, which
  test_gpu_parity.py pins against the oracle's FP64 dense rows at small N);
* the second H-matvec, run on the rank plan that the first one recorded, reproduces the first;
* the student carries the far field (no more than 1 % of the blocks go back to the teacher).
"""
import gc
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

N = 4_194_304


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_learned_far_field_4m():
    x = S.uniform(N, 0.10, 4)
    f = S.sedimenting_forces(N, 4)
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    m.set(capi.P_PRECISION, 2)
    m.set(capi.P_EPSILON, 1e-2)
    m.set(capi.P_TIMING, 1)
    loss = m.train_student(steps=20000, batch=65536, nsamples=10_000_000, lr=1e-3, seed=3)
    assert loss < 1e-5, loss
    u1 = m.dot(f)  # ACA at full pool capacity; records every block's rank
    s1 = m.stats()
    u2 = m.dot(f)  # rank-planned batches
    s2 = m.stats()
    rows = np.random.default_rng(4).choice(N, 512, replace=False)
    ud = m.dense_rows(f, rows, 0)
    err = rel(u2[rows], ud)
    print(json.dumps({"n": N, "rel_l2_vs_dense": err, "student_loss": loss, "near_ms": s2["t_close_ms"],
                      "far_ms": s2["t_far_ms"], "dot_ms": s2["t_dot_ms"], "num_close": s2["num_close"],
                      "num_far": s2["num_far"], "far_rank_max": s2["far_rank_max"],
                      "far_iterations": s2["far_iterations"], "fallback_blocks": s2["student_fallback_blocks"],
                      "far_ms_unplanned": s1["t_far_ms"]}))
    assert err < 1e-3, err
    assert rel(u2, u1) < 1e-6
    assert s2["far_rank_sum"] == s1["far_rank_sum"]
    assert s2["student_fallback_blocks"] <= 0.01 * s2["num_far"], s2
    del m
    gc.collect()
