"""Device time step: pair forces on the cell list and the explicit Euler loop (C ABI).

Pair forces are compared with the oracle's restatement of PotentialForce::GetPotentialForce
(include/PotentialForce.hpp:468-593) to 1e-4 relative per particle (float sums of up to a few
dozen terms of both signs, in another order).
The device Euler loop must equal the same loop driven from the host through the C ABI
(hignn_pair_forces, hignn_dot / hignn_update_coord_keep_tree, x += u dt in float32): to 1e-5 of
the displacement with the FP32 network, 1e-4 with the BF16 one. The two loops sum the Morse terms
in different orders (tree order on the device, input order on the host), so after the first step
the positions differ in the last bits; the BF16 network rounds its hidden activations to 8 bits,
which turns those last-bit differences into differences at the BF16 level in some evaluations.
"""
import os

import numpy as np
import pytest

from conftest import WEIGHTS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402
from oracle import hignn_oracle as O  # noqa: E402

MORSE = dict(De=1.0, a=5.0, re=2.1, cutoff=3.0)  # a Morse repulsion of the clustered suspension
G = (0.0, 0.0, -1.0)


def make_model(x, **params):
    m = capi.Model(x, 128, device=0)
    m.load_two_body(WEIGHTS)
    for k, v in params.items():
        m.set(getattr(capi, "P_" + k.upper()), v)
    return m


def rel_rows(a, b):
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-6)))


def test_pair_forces_match_oracle():
    x = S.uniform_min_dist(6000, 0.15, 5)  # separations >= 2.05: finite Morse forces
    m = make_model(x)
    f = m.pair_forces(x, G, **MORSE)
    ref = O.pair_forces(x, G, **MORSE)
    assert rel_rows(f, ref) < 1e-4
    # gravity only, and the reference's hard-coded parameters (De = 1, a = 1, re = 2.5)
    assert np.array_equal(m.pair_forces(x, G), np.tile(np.float32(G), (len(x), 1)))
    f2 = m.pair_forces(x, (0, 0, 0), 1.0, 1.0, 2.5, 4.0)
    assert rel_rows(f2, O.pair_forces(x, (0, 0, 0), 1.0, 1.0, 2.5, 4.0)) < 1e-4


def test_pair_forces_clustered_and_coincident():
    x = np.concatenate([S.uniform_min_dist(3000, 0.1, 6), np.zeros((2, 3), np.float32) + 5.0])
    m = make_model(x)
    f = m.pair_forces(x, G, **MORSE)
    ref = O.pair_forces(x, G, **MORSE)
    assert np.all(np.isfinite(f))
    assert rel_rows(f, ref) < 1e-4  # the coincident pair (|r| < 1e-3) contributes nothing


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "filament_forces.npz")
FIL = dict(n_filament=100, n_chain=32, rest_length=2.2, k_t=100.0, k_b=10.0)


@pytest.mark.parametrize("case", ["chains", "short", "pairs", "single"])
def test_filament_forces_match_reference_golden(case):
    # bit-exact with the reference's own chain_bending / chain_tension (numpy arithmetic)
    g = np.load(GOLD)
    nf, nc, L, kt, kb = g[f"{case}_params"]
    x = g[f"{case}_x"]
    m = make_model(x)
    f = m.forces(x, gravity=(0.0, 0.0, -1.0), n_filament=int(nf), n_chain=int(nc), rest_length=L, k_t=kt, k_b=kb)
    assert np.array_equal(f, g[f"{case}_f"])


def test_filaments_compose_with_pair_forces():
    x = S.filaments(100, 32, 2.2, 0.05, 21)
    x = (x + np.random.default_rng(2).normal(0, 0.2, x.shape)).astype(np.float32)
    m = make_model(x)
    both = m.forces(x, gravity=G, **MORSE, **FIL)
    pair = m.forces(x, gravity=G, **MORSE)
    assert np.array_equal(both, O.filament_forces(x, pair, 100, 32, 2.2, 100.0, 10.0))


@pytest.mark.parametrize("precision", [0, 1])
def test_device_euler_matches_host_loop(precision):
    x0 = S.uniform_min_dist(8000, 0.1, 7)
    # 100 slightly bent filaments along x on a 10 x 10 grid 6 apart, beside the free particles
    yz = np.stack(np.meshgrid(np.arange(10), np.arange(10)), -1).reshape(100, 1, 2) * 6.0
    fil = np.concatenate([np.broadcast_to(200.0 + 2.2 * np.arange(32)[None, :, None], (100, 32, 1)),
                          np.broadcast_to(yz, (100, 32, 2))], axis=2).reshape(3200, 3)
    x0[:3200] = fil + np.random.default_rng(3).normal(0, 0.05, fil.shape)
    steps, dt, k = 4, 1e-3, 2
    m = make_model(x0, epsilon=1e-2, precision=precision)
    xd = m.run_euler(x0, steps, dt, rebuild_every=k, gravity=G, **MORSE, **FIL)
    h = make_model(x0, epsilon=1e-2, precision=precision)
    x = x0.copy()
    for s in range(steps):
        if s > 0 and s % k == 0:
            h.update_coord(x)
        elif s > 0:
            h.update_coord_keep_tree(x)
        f = h.forces(x, gravity=G, **MORSE, **FIL)
        u = h.dot(f)
        x = (x + u * np.float32(dt)).astype(np.float32)
    disp = np.linalg.norm(x - x0)
    assert disp > 0
    assert np.linalg.norm(xd - x) / disp < (1e-5 if precision == 0 else 1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_device_rk2_matches_host_loop(precision):
    x0 = S.uniform_min_dist(6000, 0.1, 17)
    steps, dt, k = 3, 1e-3, 2
    m = make_model(x0, epsilon=1e-2, precision=precision)
    xd = m.run_rk2(x0, steps, dt, rebuild_every=k, gravity=G, **MORSE)
    h = make_model(x0, epsilon=1e-2, precision=precision)
    x = x0.copy()
    for s in range(steps):
        if s > 0 and s % k == 0:
            h.update_coord(x)
        elif s > 0:
            h.update_coord_keep_tree(x)
        u1 = h.dot(h.forces(x, gravity=G, **MORSE))
        xm = (x + u1 * np.float32(0.5 * dt)).astype(np.float32)
        h.update_coord_keep_tree(xm)
        u2 = h.dot(h.forces(xm, gravity=G, **MORSE))
        x = (x + u2 * np.float32(dt)).astype(np.float32)
    disp = np.linalg.norm(x - x0)
    assert disp > 0
    assert np.linalg.norm(xd - x) / disp < (1e-5 if precision == 0 else 1e-4)
    # a different integrator from Euler on the same forces
    xe = make_model(x0, epsilon=1e-2, precision=precision).run_euler(x0, steps, dt, rebuild_every=k,
                                                                      gravity=G, **MORSE)
    assert np.linalg.norm(xe - xd) > 0


def filament_suspension():
    x0 = S.uniform_min_dist(8000, 0.1, 7)
    # 100 slightly bent filaments along x on a 10 x 10 grid 6 apart, beside the free particles
    yz = np.stack(np.meshgrid(np.arange(10), np.arange(10)), -1).reshape(100, 1, 2) * 6.0
    fil = np.concatenate([np.broadcast_to(200.0 + 2.2 * np.arange(32)[None, :, None], (100, 32, 1)),
                          np.broadcast_to(yz, (100, 32, 2))], axis=2).reshape(3200, 3)
    x0[:3200] = fil + np.random.default_rng(3).normal(0, 0.05, fil.shape)
    return x0


@pytest.mark.parametrize("precision", [0, 1])
def test_device_rk2_with_three_body(precision):
    # the whole HIGNN velocity in the device loop: H-matrix two-body term + three-body + self terms
    x0 = filament_suspension()
    steps, dt, k = 2, 1e-3, 2
    tb = capi.ThreeBody(0, epsilon=5.0)
    m = make_model(x0, epsilon=1e-2, precision=precision)
    m.set_three_body(tb)
    xd = m.run_rk2(x0, steps, dt, rebuild_every=k, gravity=G, **MORSE, **FIL)
    h = make_model(x0, epsilon=1e-2, precision=precision)
    tbh = capi.ThreeBody(0, epsilon=5.0)

    def vel(x):
        f = h.forces(x, gravity=G, **MORSE, **FIL)
        return h.dot(f) + tbh.velocity(x, f)

    x = x0.copy()
    for s in range(steps):
        if s > 0 and s % k == 0:
            h.update_coord(x)
        elif s > 0:
            h.update_coord_keep_tree(x)
        xm = (x + vel(x) * np.float32(0.5 * dt)).astype(np.float32)
        h.update_coord_keep_tree(xm)
        x = (x + vel(xm) * np.float32(dt)).astype(np.float32)
    disp = np.linalg.norm(x - x0)
    assert tbh.stats()["triplets"] > 0
    # The device sums the two-body and three-body velocities in FP64 and rounds once; the host loop
    # rounds each to FP32 and adds them. The positions then differ in the last bits, and ACA's
    # signed-determinant pivots (src/FarDot.cpp:557-573) turn such differences into other, equally
    # valid block approximations at eps 1e-2: 1e-4 of the displacement for both forms.
    assert np.linalg.norm(xd - x) / disp < 1e-4
    m.set_three_body(None)  # detached: the two-body loop alone moves the particles differently
    xn = m.run_rk2(x0, steps, dt, rebuild_every=k, gravity=G, **MORSE, **FIL)
    assert np.linalg.norm(xn - xd) / disp > 1e-4


@pytest.mark.parametrize("precision,morse", [(0, False), (0, True), (1, False)])
def test_device_dp45_matches_reference_integrator(precision, morse):
    # ExplicitRk4 (include/TimeIntegrator.hpp:602-860) as the oracle restates it, driven from the host
    # through the C ABI on the same kept tree, against the device loop
    x0 = S.uniform_min_dist(5000, 0.1, 23)
    forces = dict(gravity=G, **(MORSE if morse else {}))
    tf, dt0, thr = 4e-3, 1.5e-3, 2e-4
    m = make_model(x0, epsilon=1e-2, precision=precision)
    xd, steps = m.run_dp45(x0, tf, dt0, threshold=thr, **forces)
    h = make_model(x0, epsilon=1e-2, precision=precision)

    def velocity(t, inp):
        p = np.ascontiguousarray(inp[:, :3])
        h.update_coord_keep_tree(p)
        return h.dot(h.forces(p, **forces))

    x, count = O.dp45_run(x0, velocity, dt0, tf, threshold=thr)
    assert steps == count >= 3
    disp = np.linalg.norm(x - x0)
    assert disp > 0
    # FP32 network: last-bit differences only (FP64 atomic order of the matvec, order of the Morse
    # sums). BF16 network: a last-bit difference of a stage position can flip the BF16 rounding of
    # its network inputs, and six stages per accepted step compound it (1.4e-4 measured), so the
    # bound is 3e-4; the step counts must still agree exactly.
    assert np.linalg.norm(xd - x) / disp < (1e-5 if precision == 0 else 3e-4)


def test_device_dp45_with_tree_rebuilds():
    """A rebuild between Dormand-Prince steps must carry the stage vector k1 (the previous step's
    k7, first-same-as-last), which lives in tree order, over to the new tree's order. On this
    workload one step of motion reorders 94 % of the tree (the root's PCA axis turns), and a k1
    left in the old order errs by ~3e-3 of the displacement per rebuild (both figures from the
    oracle's velocity field on the CPU; the velocity is mostly the collective sedimentation, so
    particles' velocities differ little). Rebuilt every step, the run must agree with the
    kept-tree run up to the two H-matrix approximations, which at eps 1e-5 are each within
    ~2e-4 of the dense product."""
    x0 = S.uniform_min_dist(5000, 0.1, 23)
    forces = dict(gravity=G, **MORSE)
    tf, dt0, thr = 4e-3, 1.5e-3, 2e-4
    xa, na = make_model(x0, epsilon=1e-5).run_dp45(x0, tf, dt0, threshold=thr, rebuild_every=1, **forces)
    xb, nb = make_model(x0, epsilon=1e-5).run_dp45(x0, tf, dt0, threshold=thr, rebuild_every=0, **forces)
    disp = np.linalg.norm(xb - x0)
    assert na >= 3 and nb >= 3 and disp > 0
    assert np.linalg.norm(xa - xb) / disp < 1e-3, (np.linalg.norm(xa - xb) / disp, na, nb)


def test_keep_tree_is_close_to_rebuild():
    x0 = S.uniform_min_dist(8000, 0.1, 8)
    f = S.sedimenting_forces(8000, 8)
    x1 = x0 + np.float32(0.05) * np.random.default_rng(1).standard_normal(x0.shape).astype(np.float32)
    a = make_model(x0, epsilon=1e-2)
    a.dot(f)
    a.update_coord_keep_tree(x1)
    ua = a.dot(f)
    b = make_model(x1, epsilon=1e-2)
    ub = b.dot(f)
    assert np.linalg.norm(ua - ub) / np.linalg.norm(ub) < 2e-3  # two H-matrix approximations at eps 1e-2
    dense = b.dense_rows(f, np.arange(0, 8000, 40), 0)
    assert np.linalg.norm(ua[::40] - dense) / np.linalg.norm(dense) < 2e-3


def test_pybind_potential_force():
    from hignn_b200 import hignn

    x = S.uniform_min_dist(3000, 0.15, 9)
    pf = hignn.PotentialForce()
    pf.set_two_body_epsilon(4.0)
    f = pf.get_potential_force(x)  # the reference's constants De = 1, a = 1, re = 2.5
    assert rel_rows(f, O.pair_forces(x, (0, 0, 0), 1.0, 1.0, 2.5, 4.0)) < 1e-4
    pf.set_parameters(1.0, 5.0, 2.1)
    f = pf.get_potential_force(x)
    assert rel_rows(f, O.pair_forces(x, (0, 0, 0), 1.0, 5.0, 2.1, 4.0)) < 1e-4
    with pytest.raises(RuntimeError):
        pf.set_periodic(True)
