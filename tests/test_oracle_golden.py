"""The oracle's two-body kernel against golden vectors from the reference's own Net (python/convert.py)."""
import numpy as np

from conftest import GOLDEN


def _rowrel(a, b):
    # error relative to the Frobenius norm of each 3x3 block
    return np.max(np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30))


def test_fp64_matches_golden(oracle_net):
    d = np.load(GOLDEN)
    y = oracle_net.eval64(d["r"])
    assert _rowrel(y, d["y_fp64"]) < 1e-12


def test_fp32_matches_reference_torch_fp32(oracle_net):
    d = np.load(GOLDEN)
    y = oracle_net.eval32(d["r"])
    # two FP32 evaluations of the same network differ by summation order only
    assert _rowrel(y, d["y_fp32"]) < 2e-5


def test_identity_below_cutoff(oracle_net):
    r = np.array([[0, 0, 0], [9e-6, 0, 0], [0, 5e-6, -5e-6]], np.float32)
    for y in (oracle_net.eval32(r), oracle_net.eval64(r)):
        assert np.array_equal(y, np.tile(np.eye(3).reshape(1, 9), (3, 1)).astype(y.dtype))


def test_inner_network(oracle_net):
    d = np.load(GOLDEN)
    assert np.max(np.abs(oracle_net.inner64(d["r"]) - d["inner_fp64"])) < 1e-12


def test_weights_file_matches_golden():
    import hashlib

    from conftest import WEIGHTS

    d = np.load(GOLDEN)
    assert hashlib.sha256(open(WEIGHTS, "rb").read()).hexdigest() == str(d["weights_sha256"])
