"""The oracle's Dormand-Prince (ExplicitRk4::Run, include/TimeIntegrator.hpp:602-860) pinned
against an independent integrator.

The reference cannot be built here, so its integrator is pinned through what the method must
do: on a smooth linear system x' = A x + B sin(2t), x(0) = 0, the oracle's result at t = 1 must
agree with scipy's 8th-order Dormand-Prince (DOP853, rtol 1e-13) to float32 rounding. The
initial state has zero velocity, so the reference's zero k1 on the first step (a quirk the
oracle reproduces) is exact here. A wrong tableau entry (a52 off by 0.3 %, b1 by 3 %) leaves
errors of 5e-4 to 6e-3 on this problem, far above the 5e-6 bound.
"""
import math

import numpy as np
import pytest

from oracle import hignn_oracle as O

scipy_integrate = pytest.importorskip("scipy.integrate")

N = 16


def system(seed):
    rng = np.random.default_rng(seed)
    A = 0.8 * rng.standard_normal((3, 3))
    B = rng.standard_normal((N, 3))

    def vel(t, pos6):
        p = np.asarray(pos6, np.float64)[:, :3]
        return (p @ A.T + B * math.sin(2.0 * t)).astype(np.float32)

    def rhs(t, y):
        return (y.reshape(N, 3) @ A.T + B * math.sin(2.0 * t)).ravel()

    return vel, rhs


@pytest.mark.parametrize("dt,threshold", [(0.05, 1e-3), (0.2, 1e-3), (0.05, 1e-5)])
def test_dp45_against_dop853(dt, threshold):
    vel, rhs = system(5)
    tf = 1.0
    exact = scipy_integrate.solve_ivp(rhs, (0.0, tf), np.zeros(3 * N), method="DOP853", rtol=1e-13,
                                      atol=1e-15).y[:, -1].reshape(N, 3)
    x, steps = O.dp45_run(np.zeros((N, 3), np.float32), vel, dt, tf, threshold=threshold)
    assert steps == math.ceil(tf / dt - 1e-9)  # the field is smooth: no step is rejected
    assert np.abs(x - exact).max() < 5e-6, np.abs(x - exact).max()


def test_dp45_rejects_and_shrinks_steps():
    """A step whose error estimate exceeds the threshold is retried with
    h * max(0.8 (err / threshold)^-0.2, 0.1), and the next step restarts from min(h0, tf - t),
    so a tight threshold on a large h0 takes more, shorter steps and stays accurate."""
    vel, rhs = system(6)
    tf = 1.0
    exact = scipy_integrate.solve_ivp(rhs, (0.0, tf), np.zeros(3 * N), method="DOP853", rtol=1e-13,
                                      atol=1e-15).y[:, -1].reshape(N, 3)
    x_loose, n_loose = O.dp45_run(np.zeros((N, 3), np.float32), vel, 0.5, tf, threshold=1e-1)
    x_tight, n_tight = O.dp45_run(np.zeros((N, 3), np.float32), vel, 0.5, tf, threshold=1e-6)
    assert n_loose == 2 and n_tight > n_loose
    assert np.abs(x_tight - exact).max() < 5e-6
