"""Student ablation at the benchmark's size: what the trained far-field network adds to its base.

The student predicts the teacher's inner output minus the Rotne-Prager-Yamakawa (RPY) tensor,
so the same network with every parameter zero is RPY alone. On the benchmark workload
(N = 1,048,576 clustered spheres, seed 2, leaf 128, eps 1e-2) three far fields are compared,
each on the rank plan recorded by its own first H-matvec:
* teacher: the two-body network on the tensor cores for every ACA query (precision 1);
* RPY: the student form with all-zero parameters;
* trained: the student form after the workload's training (20,000 Adam steps, batch 65,536,
  10M teacher samples at 4-400 radii).
Each is checked against FP64 dense rows (the network in FP64, all N sources) on 512 seeded rows.
Recorded per arm: far-field ms, mean and max ACA rank, blocks sent back to the teacher, relative
L2 error. Asserted: every arm is within 1e-3 of the dense rows, and the residual check keeps the
student forms honest (a block whose sampled student error exceeds eps goes back to the teacher).
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

N = 1_048_576


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_student_ablation_1m():
    x = S.clustered(N, 0.10, 2)
    f = S.sedimenting_forces(N, 2)
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    m.set(capi.P_EPSILON, 1e-2)
    m.set(capi.P_TIMING, 1)
    rows = np.sort(np.random.default_rng(7).choice(N, 512, replace=False))
    ud = m.dense_rows(f, rows, capi.DENSE_F64)
    arms = {}

    def run(name, precision, params=None):
        m.set(capi.P_PRECISION, precision)
        if params is not None:
            m.set_student(params)
        m.dot(f)  # records the ranks of this form
        u = m.dot(f)
        st = m.stats()
        arms[name] = {"far_ms": st["t_far_ms"], "near_ms": st["t_close_ms"],
                      "rank_mean": st["far_rank_sum"] / max(1, st["num_far"]), "rank_max": st["far_rank_max"],
                      "fallback_blocks": st["student_fallback_blocks"], "far_evals": st["far_evals"],
                      "rel_l2_vs_fp64_dense": rel(u[rows], ud)}

    run("teacher", 1)
    run("rpy", 2, np.zeros(2537, np.float32))
    loss = m.train_student(steps=20000, batch=65536, nsamples=10_000_000, lr=1e-3, seed=3)
    run("trained", 2, m.get_student())
    arms["trained"]["train_mse"] = loss
    print("STUDENT_ABLATION " + json.dumps(arms))
    for name, a in arms.items():
        assert a["rel_l2_vs_fp64_dense"] < 1e-3, (name, a)
    for name in ("rpy", "trained"):
        assert arms[name]["fallback_blocks"] <= 0.05 * m.stats()["num_far"], (name, arms[name])
    m.close()
