"""The C-ABI library loads and exports every entry point declared in include/hignn_b200.h (no GPU calls)."""
import ctypes
import os
import re

from conftest import REPO


def declared_symbols():
    src = open(os.path.join(REPO, "include", "hignn_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(hignn_\w+)\s*\(", src)))


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
