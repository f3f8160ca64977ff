"""ACA planning and the student fallback on the GPU (calls through the C ABI).

The far field records every block's ACA rank; the next far field on the same
tree plans its batches from those ranks (exact pool capacities, blocks sorted
by rank, no counter read-back inside a batch). A block that would need more
terms than recorded is deferred and rerun with its full capacity, so the
result never depends on the plan: the tests compare plans against each other
to 1e-7 relative L2 (FP64 sums in another order, rounded to the float32 output).
"""
import numpy as np
import pytest

from conftest import WEIGHTS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402


def rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def make_model(x, leaf=128, **params):
    m = capi.Model(x, leaf, device=0)
    m.load_two_body(WEIGHTS)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    return m


@pytest.fixture(scope="module")
def workload():
    x = S.uniform(12000, 0.1, 31)
    f = S.sedimenting_forces(12000, 31)
    return x, f


@pytest.mark.parametrize("precision", [0, 1])
def test_rank_plan_reuses_ranks(workload, precision):
    x, f = workload
    m = make_model(x, epsilon=1e-2, precision=precision)
    u1 = m.dot(f)
    s1 = m.stats()
    u2 = m.dot(f)
    s2 = m.stats()
    assert rel(u2, u1) < 1e-7
    assert s2["far_rank_sum"] == s1["far_rank_sum"] and s2["far_evals"] == s1["far_evals"]
    assert s2["far_iterations"] <= s1["far_iterations"]


def test_deferred_blocks_are_rerun(workload):
    x, f = workload
    m = make_model(x, epsilon=1e-2, precision=1)
    u1 = m.dot(f)
    s1 = m.stats()
    m.set(capi.P_RANK_HINT_OFFSET, -2)  # plan two terms short of every recorded rank
    u2 = m.dot(f)
    s2 = m.stats()
    assert rel(u2, u1) < 1e-7
    assert s2["far_rank_sum"] == s1["far_rank_sum"]
    m.set(capi.P_RANK_HINT_OFFSET, 0)
    assert rel(m.dot(f), u1) < 1e-7


def test_small_pool_budget_many_batches(workload):
    x, f = workload
    ref = make_model(x, epsilon=1e-2, precision=1).dot(f)
    m = make_model(x, epsilon=1e-2, precision=1, far_pool_mb=2)
    assert rel(m.dot(f), ref) < 1e-7
    assert rel(m.dot(f), ref) < 1e-7  # planned from ranks, still 2 MiB per batch


def test_student_fallback_to_teacher(workload):
    """An all-zero student is the Rotne-Prager-Yamakawa tensor, about 3e-3 (relative) from the teacher.

    The fallback threshold is max(student_tol, epsilon): at epsilon 1e-4 and tol 0 every block goes
    back to the teacher and the result is the teacher's; with a huge tol none does.
    """
    x, f = workload
    u_teacher = make_model(x, epsilon=1e-4, precision=1).dot(f)
    m = make_model(x, epsilon=1e-4, precision=2)
    m.set_student(np.zeros(capi.STUDENT_PARAMS, np.float32))
    m.set(capi.P_STUDENT_TOL, 0.0)
    u = m.dot(f)
    st = m.stats()
    assert st["student_fallback_blocks"] == st["num_far"]
    assert rel(u, u_teacher) < 1e-7
    m.set(capi.P_STUDENT_TOL, 1e9)
    u_rpy = m.dot(f)
    assert m.stats()["student_fallback_blocks"] == 0
    assert 1e-9 < rel(u_rpy, u_teacher) < 1e-1


def test_student_fallback_threshold_follows_epsilon(workload):
    """At epsilon 1e-2 the RPY student's ~3e-3 sampled error is within the block's own accuracy."""
    x, f = workload
    m = make_model(x, epsilon=1e-2, precision=2)
    m.set_student(np.zeros(capi.STUDENT_PARAMS, np.float32))
    m.dot(f)
    st = m.stats()
    assert st["student_fallback_blocks"] < 0.05 * st["num_far"], st


def test_shards_sum_to_the_whole_product(workload):
    """Two shards computed one after the other on this GPU add up to the unsharded H-matvec."""
    x, f = workload
    full = make_model(x, epsilon=1e-2, precision=1).dot(f).astype(np.float64)
    parts = []
    for r in range(2):
        m = make_model(x, epsilon=1e-2, precision=1)
        m.set_shard(r, 2)
        parts.append(m.dot(f).astype(np.float64))
    assert rel(parts[0] + parts[1], full) < 1e-6  # float32 partial results
    assert rel(parts[0], full) > 1e-2  # each shard alone is only part of the product


def test_ranks_carried_across_a_rebuild(workload):
    """A rebuild on moved positions keeps the recorded rank of every block that joins the same two
    nodes (HIGNN_P_KEEP_RANKS, default on); the product on the new tree equals that of a model
    that plans nothing (a fresh model, and the same model with the ranks forgotten)."""
    x, f = workload
    x2 = (x + np.random.default_rng(9).normal(0, 0.05, x.shape)).astype(np.float32)
    for prec in (0, 1):
        m = make_model(x, epsilon=1e-2, precision=prec)
        m.dot(f)  # records the ranks on the first tree
        m.update_coord(x2)
        u_carried = m.dot(f)
        fresh = make_model(x2, epsilon=1e-2, precision=prec)
        u_fresh = fresh.dot(f)
        assert rel(u_carried, u_fresh) < 1e-6
        m.set(capi.P_KEEP_RANKS, 0)
        m.update_coord(x)
        m.update_coord(x2)
        assert rel(m.dot(f), u_fresh) < 1e-6
        m.close()
        fresh.close()
