"""Time integrators of the `hignn` module (ExplicitEuler, ExplicitRk4) against the oracle.

The integrators call a Python velocity function, as the reference's do
(include/TimeIntegrator.hpp:92-141), so they are tested on the CPU with
analytic velocity fields; the GPU H-matvec behind a real velocity function is
covered by the parity tests. Euler is float32 arithmetic in a fixed order and
must match the restatement bit for bit; the adaptive Dormand-Prince step
differs from it only in the order of the error-norm sum.
"""
import numpy as np
import pytest

from oracle import hignn_oracle as O

hignn = pytest.importorskip("hignn_b200.hignn")


def linear_field(n, seed):
    rng = np.random.default_rng(seed)
    A = (0.3 * rng.standard_normal((3, 3))).astype(np.float32)
    b = rng.standard_normal(3).astype(np.float32)

    def vel(t, pos6):
        p = np.asarray(pos6, np.float32)[:, :3]
        return (p @ A.T + b * np.float32(1.0 + 0.5 * np.sin(t))).astype(np.float32)

    return vel


def f32(v):
    return float(np.float32(v))


def run_native(cls, x0, vel, dt, tf, lim=None, output_step=1, threshold=None):
    integ = cls()
    integ.set_time_step(dt)
    integ.set_final_time(tf)
    integ.set_num_rigid_body(len(x0))
    integ.set_velocity_func(vel)
    outs = []
    integ.set_output_func(lambda p, v: outs.append((np.array(p), np.array(v))))
    integ.set_output_step(output_step)
    if threshold is not None:
        integ.set_threshold(threshold)
    if lim is not None:
        integ.set_x_lim([lim[0][0], lim[1][0]])
        integ.set_y_lim([lim[0][1], lim[1][1]])
        integ.set_z_lim([lim[0][2], lim[1][2]])
    integ.initialize(x0)
    integ.run()
    return outs, integ.get_func_count()


def test_euler_bit_exact():
    rng = np.random.default_rng(0)
    x0 = rng.uniform(-5, 5, (64, 3)).astype(np.float32)
    vel = linear_field(64, 1)
    outs, count = run_native(hignn.ExplicitEuler, x0, vel, 0.01, 0.25, output_step=3)
    ref = []
    _, rcount = O.euler_run(x0, vel, f32(0.01), f32(0.25), output=lambda p, v: ref.append((p, v)), output_step=3)
    assert count == rcount == 25
    assert len(outs) == len(ref) == 9
    for (p, v), (rp, rv) in zip(outs, ref):
        assert np.array_equal(p, rp)
        assert np.array_equal(v, rv)


def test_euler_periodic_box():
    rng = np.random.default_rng(2)
    x0 = rng.uniform(-1, 1, (40, 3)).astype(np.float32)
    lim = ([-1.0, -1.0, -1.0], [1.0, 1.0, 1.0])

    def vel(t, pos6):  # uniform drift: particles leave the box and are wrapped
        p = np.asarray(pos6, np.float32)[:, :3]
        assert np.all(p >= -1.0 - 1e-6) and np.all(p <= 1.0 + 1e-6), "positions passed out of the box"
        return np.tile(np.array([[3.0, -2.0, 0.5]], np.float32), (len(p), 1))

    outs, count = run_native(hignn.ExplicitEuler, x0, vel, 0.05, 1.0, lim=lim)
    ref = []
    O.euler_run(x0, vel, f32(0.05), f32(1.0), lim=lim, output=lambda p, v: ref.append((p, v)))
    assert count == 20 and len(outs) == len(ref)
    for (p, _), (rp, _) in zip(outs, ref):
        assert np.array_equal(p, rp)


def test_euler_last_step_is_shortened():
    x0 = np.zeros((3, 3), np.float32)
    times = []

    def vel(t, pos6):
        times.append(float(t))
        return np.ones((len(pos6), 3), np.float32)

    _, count = run_native(hignn.ExplicitEuler, x0, vel, 0.3, 1.0)
    assert count == 4
    assert times[-1] == pytest.approx(1.0, abs=1e-6)


def test_dp45_matches_restatement():
    rng = np.random.default_rng(3)
    x0 = rng.uniform(-2, 2, (32, 3)).astype(np.float32)
    vel = linear_field(32, 4)
    outs, count = run_native(hignn.ExplicitRk4, x0, vel, 0.05, 0.5, threshold=1e-4)
    ref = []
    _, rcount = O.dp45_run(x0, vel, f32(0.05), f32(0.5), threshold=1e-4, output=lambda p, v: ref.append((p, v)))
    assert count == rcount and len(outs) == len(ref) > 0
    for (p, _), (rp, _) in zip(outs, ref):
        np.testing.assert_allclose(p, rp, rtol=0, atol=1e-6)


def test_dp45_first_step_starts_from_zero_k1():
    """The reference never initialises k1 before the first step (include/TimeIntegrator.hpp:608)."""
    x0 = np.zeros((4, 3), np.float32)
    calls = []

    def vel(t, pos6):
        calls.append(np.array(pos6[:, :3]))
        return np.ones((len(pos6), 3), np.float32)

    run_native(hignn.ExplicitRk4, x0, vel, 0.1, 0.1, threshold=1.0)
    # call 0 is the initial evaluation; call 1 is stage 1 at x0 + k1 * a21 dt with k1 = 0
    assert np.array_equal(calls[1], x0)


def test_integrator_input_errors():
    integ = hignn.ExplicitEuler()
    integ.set_num_rigid_body(5)
    with pytest.raises(RuntimeError):
        integ.initialize(np.zeros((4, 3), np.float32))
    with pytest.raises(RuntimeError):
        integ.initialize(np.zeros(15, np.float32))
