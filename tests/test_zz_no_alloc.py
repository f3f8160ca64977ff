"""hignn_dense_rows_noalloc against hignn_dense_rows, through the C ABI.

hignn_dense_rows_noalloc serves callers that cannot allocate device memory once
they are running (a fixed device-memory budget, or a host framework whose own
allocator owns the GPU). It keeps its per-call scratch in one static device
array that every call shares and that keeps the previous call's contents, so
the test makes two calls in a row -- the second with other forces and fewer
rows, over the first call's leftovers -- and checks each against the
allocating entry point within the tolerance of the FP64-accumulated dense rows
(only the order of FP64 atomic additions differs), and that the device's free
memory is the same before and after the second call.

This file is named to be collected last.
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


def test_noalloc_dense_rows_matches_allocating_entry_point_twice():
    n = 6000
    x = S.uniform(n, 0.1, 17)
    f1 = S.sedimenting_forces(n, 17)
    f2 = S.sedimenting_forces(n, 18) * np.float32(2.5)
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    m.set(capi.P_EPSILON, 1e-2)
    m.dot(f1)  # builds the tree and the model's device buffers (may allocate)
    rng = np.random.default_rng(5)
    rows1 = rng.choice(n, 700, replace=False)
    rows2 = rng.choice(n, 300, replace=False)
    out1 = m.dense_rows_noalloc(f1, rows1)
    ref1 = m.dense_rows(f1, rows1)
    assert rel(out1, ref1) < 1e-6
    # the second call runs with every kernel loaded: the device's free memory must not change
    torch.cuda.synchronize(0)
    free_before = torch.cuda.mem_get_info(0)[0]
    out2 = m.dense_rows_noalloc(f2, rows2)
    free_after = torch.cuda.mem_get_info(0)[0]
    assert free_after == free_before, f"device free memory changed by {free_before - free_after} bytes"
    ref2 = m.dense_rows(f2, rows2)
    assert rel(out2, ref2) < 1e-6


def test_noalloc_rejects_oversized_requests():
    n = 2000
    x = S.uniform(n, 0.1, 3)
    f = S.sedimenting_forces(n, 3)
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    with pytest.raises(capi.HignnError) as e:  # no tree yet: building it may allocate
        m.dense_rows_noalloc(f, np.arange(10))
    assert e.value.code == -3
    m.dot(f)
    too_many = np.zeros(131073, np.int64)  # one above HIGNN_NOALLOC_MAX_ROWS
    with pytest.raises(capi.HignnError) as e:
        m.dense_rows_noalloc(f, too_many)
    assert e.value.code == -1
