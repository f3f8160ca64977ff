"""The CUDA-graph form of the rank-planned H-matvec against the eager form.

The first product on a tree runs eagerly and records every far block's ACA rank; later products
on the same tree and settings run as one captured graph (HIGNN_P_GRAPH) whose only host read-back
is the status at the end. Checked for the three precision forms: the graph products equal the
eager ones (only the order of FP64 atomic additions differs), the replay equals the capture, and
the two paths the host takes after the graph -- blocks deferred past their recorded rank and
blocks the student check sends back to the teacher -- give the eager results too.
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
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def model(x, graph, precision, student=None, **params):
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    m.set(capi.P_EPSILON, 1e-2)
    m.set(capi.P_GRAPH, 1 if graph else 0)
    if student is not None:
        m.set_student(student)
    m.set(capi.P_PRECISION, precision)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    return m


@pytest.fixture(scope="module")
def case():
    x = S.uniform(40000, 0.1, 31)
    f = S.sedimenting_forces(40000, 31)
    trainer = capi.Model(x[:2000], 128, device=0)
    trainer.load_two_body(WEIGHTS)
    trainer.train_student(steps=1500, batch=16384, nsamples=1_000_000, lr=1e-3, seed=3)
    student = trainer.get_student()
    trainer.close()
    return x, f, student


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_graph_matches_eager(case, precision):
    x, f, student = case
    st = student if precision == 2 else None
    me = model(x, False, precision, st)
    mg = model(x, True, precision, st)
    ue1 = me.dot(f)
    ue2 = me.dot(f)  # eager, rank-planned
    ug1 = mg.dot(f)  # eager: records the ranks
    s1 = mg.stats()
    ug2 = mg.dot(f)  # captured and launched
    s2 = mg.stats()
    ug3 = mg.dot(f)  # replayed
    assert rel(ue2, ue1) < 1e-6
    assert rel(ug1, ue1) < 1e-6
    assert rel(ug2, ue2) < 1e-6
    assert rel(ug3, ug2) < 1e-6
    assert s2["far_rank_sum"] == s1["far_rank_sum"] and s2["far_rank_max"] == s1["far_rank_max"]
    assert s2["gpu_launches"] > 0
    # the graph through the device-pointer call as well
    fd = torch.from_numpy(f).cuda()
    ud = torch.empty_like(fd)
    mg.dot_device(ud.data_ptr(), fd.data_ptr())
    assert rel(ud.cpu().numpy(), ug3) < 1e-6
    me.close()
    mg.close()


def test_graph_deferred_blocks_are_rerun(case):
    """Planned capacities two terms below the recorded ranks: blocks are deferred inside the
    graph and rerun at full capacity afterwards; the product does not change."""
    x, f, _ = case
    ref = model(x, False, 1)
    ref.dot(f)
    u_ref = ref.dot(f)
    mg = model(x, True, 1)
    mg.dot(f)
    mg.set(capi.P_RANK_HINT_OFFSET, -2)
    u = mg.dot(f)
    assert rel(u, u_ref) < 1e-6
    u2 = mg.dot(f)
    assert rel(u2, u_ref) < 1e-6
    ref.close()
    mg.close()


def test_graph_student_fallback_is_rerun(case):
    """A student far from the teacher (random parameters): the residual check sends blocks back
    to the teacher inside the graph; after the graph they are recomputed with the teacher."""
    x, f, _ = case
    bad = np.random.default_rng(0).normal(0, 0.3, 2537).astype(np.float32)
    ref = model(x, False, 2, bad)
    ref.dot(f)
    u_ref = ref.dot(f)
    n_back = ref.stats()["student_fallback_blocks"]
    assert n_back > 0
    mg = model(x, True, 2, bad)
    mg.dot(f)
    u = mg.dot(f)
    assert mg.stats()["student_fallback_blocks"] == n_back
    assert rel(u, u_ref) < 1e-6
    ref.close()
    mg.close()
