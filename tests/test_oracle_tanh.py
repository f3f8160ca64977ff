"""The plain form's FP32 tanh (the oracle's C restatement of the device method): accuracy against
a double-precision tanh, odd symmetry and the special values. The device computes the same
operations (tests/test_gpu_parity.py checks the two networks bit for bit)."""
import numpy as np

from oracle import hignn_oracle as O


def ulp_error(t, x):
    ref = np.tanh(x.astype(np.float64))
    rf = ref.astype(np.float32)
    ulp = np.abs(np.nextafter(rf, np.float32(2)) - rf).astype(np.float64)
    ulp[rf == 1.0] = 2.0 ** -24
    ok = rf != 0
    return np.abs(t.astype(np.float64) - ref)[ok] / ulp[ok]


def test_tanh_accuracy_within_1_05_ulp():
    rng = np.random.default_rng(0)
    # dense near the branch points (0.8, 9.5) and across the range, both signs
    x = np.concatenate([rng.uniform(-12, 12, 3_000_000), rng.uniform(0.7, 0.9, 500_000),
                        rng.uniform(9.3, 9.7, 100_000), np.exp(rng.uniform(-40, 2, 500_000))]).astype(np.float32)
    t = O.tanh_f32_exact(x)
    e = ulp_error(np.abs(t), np.abs(x))
    assert e.max() <= 1.05, e.max()
    assert np.array_equal(O.tanh_f32_exact(-x), -t)


def test_tanh_special_values():
    x = np.array([0.0, -0.0, 1e-30, 9.5, 1e30, np.inf, -np.inf, np.nan], np.float32)
    t = O.tanh_f32_exact(x)
    assert t[0] == 0 and np.signbit(t[1]) and t[2] == np.float32(1e-30)
    assert t[3] == 1 and t[4] == 1 and t[5] == 1 and t[6] == -1 and np.isnan(t[7])
