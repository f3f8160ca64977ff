"""The C-ABI library loads and exports every entry point declared in include/hignn_b200.h (no GPU calls)."""
import ctypes
import os
import re

from conftest import REPO


def declared_symbols():
    src = open(os.path.join(REPO, "include", "hignn_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|void)\s+(hignn_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("hignn_create", "hignn_dot", "hignn_update_coord", "hignn_dense_dot", "hignn_load_two_body"):
        assert s in syms


def test_library_exports_all_declared_symbols():
    from hignn_b200 import capi

    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_errors_without_device():
    import numpy as np

    from hignn_b200 import capi

    assert capi.lib.hignn_version() >= 100
    m = capi.Model(np.random.default_rng(0).uniform(0, 10, (300, 3)), 64, device=-1)
    try:
        m.dot(np.zeros((300, 3), np.float32))
        raise AssertionError("dot on a host-only model must fail")
    except capi.HignnError as e:
        assert e.code == -6
    try:
        m.set(capi.P_MAX_ITER, 10_000)
        raise AssertionError("max_iter above the cap must be rejected")
    except capi.HignnError as e:
        assert e.code == -1
    for key, bad in ((capi.P_FAR_BATCH_ROWS, 2.0 ** 31), (capi.P_FAR_BATCH_ROWS, float("nan")),
                     (capi.P_FAR_BATCH_ROWS, 100), (capi.P_FAR_POOL_MB, 1e30), (capi.P_FAR_POOL_MB, 0)):
        try:
            m.set(key, bad)
            raise AssertionError(f"key {key} = {bad} must be rejected")
        except capi.HignnError as e:
            assert e.code == -1
    m.set(capi.P_FAR_BATCH_ROWS, 2.0 ** 30)
    try:
        m.set(12345, 1.0)
        raise AssertionError("unknown key must be rejected")
    except capi.HignnError as e:
        assert e.code == -1
    m.set(capi.P_EPSILON, 1e-3)
    assert m.get(capi.P_EPSILON) == 1e-3
    assert m.get(capi.P_MAX_ITER) == 100 and m.get(capi.P_USE_SYMMETRY) == 1.0


def test_bad_weight_file(tmp_path):
    import numpy as np

    from hignn_b200 import capi

    m = capi.Model(np.zeros((10, 3)) + np.arange(10)[:, None], 4, device=-1)
    p = tmp_path / "bad.hgnw"
    p.write_bytes(b"nope")
    try:
        m.load_two_body(str(p))
        raise AssertionError("malformed weights must be rejected")
    except capi.HignnError as e:
        assert e.code == -4


def test_neighbour_lists_and_three_body_need_a_device():
    import ctypes as C

    import pytest

    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from hignn_b200 import capi

    h = C.c_void_p()
    assert capi.lib.hignn_nbl_create(0, C.byref(h)) == -6  # HIGNN_ERR_NODEV
    assert capi.lib.hignn_tb_create(0, C.byref(h)) == -6
    assert not h.value
    capi.lib.hignn_nbl_destroy(None)  # a null handle is accepted
    capi.lib.hignn_tb_destroy(None)


def test_weights_from_memory_are_shape_checked_first():
    """hignn_load_two_body_mem checks the layer shapes before it reads any weight, so a wrong
    shape is an error (not a read past the caller's array); the right shape loads on a
    host-only model."""
    import ctypes as C

    import numpy as np

    from hignn_b200 import capi

    m = capi.Model(np.random.default_rng(1).uniform(0, 20, (400, 3)), 64, device=-1)
    good = np.array([3, 128, 512, 9], np.int32)
    params = np.random.default_rng(2).standard_normal(3 * 128 + 128 + 128 * 512 + 512 + 512 * 9 + 9).astype(np.float32)
    fp = params.ctypes.data_as(C.POINTER(C.c_float))

    def load(dims, layers, act=1):
        d = np.ascontiguousarray(dims, np.int32)
        return capi.lib.hignn_load_two_body_mem(m._h, layers, d.ctypes.data_as(C.POINTER(C.c_int32)), fp, act)

    assert load(good, 3) == 0
    assert load(good, 2) == -1
    assert load(good, -5) == -1
    assert load([3, 1 << 30, 512, 9], 3) == -1  # would read far past `params` if read first
    assert load(good, 3, act=2) == -1
