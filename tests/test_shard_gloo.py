"""Sharding of the block lists over processes, on the CPU (gloo, world size 2).

Each rank computes its shard of the close and far lists -- here with the
oracle, since the ranks have no GPU -- and the partial velocities are summed
with an all-reduce, as the multi-GPU product sums its ranks' partial results
over NCCL (the reference all-reduces u over MPI, src/HignnModel.cpp:602). The
sum must equal the unsharded product to 1e-8 relative L2: the oracle's FP32
network is evaluated in batches of other shapes per shard, and BLAS rounds
those differently in the last bit.
"""
import os
import socket

import numpy as np
import pytest

from conftest import WEIGHTS

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from hignn_b200 import capi  # noqa: E402
from hignn_b200 import synthetic as S  # noqa: E402

N, LEAF, EPS = 2500, 64, 1e-2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from oracle import hignn_oracle as O

        x = S.uniform(N, 0.1, 9)
        f = S.sedimenting_forces(N, 9)
        m = capi.Model(x, LEAF, device=-1)
        m.set_shard(rank, world)
        c0, c1, f0, f1 = m.shard()
        net = O.TwoBody.from_hgnw(WEIGHTS)
        om = O.OracleModel(x, LEAF, net, epsilon=EPS)
        ft = f[om.rmap]
        u = O.close_dot(om.tree, om.xt, ft, om.closeI[c0:c1], om.closeJ[c0:c1], net)
        u = u + O.far_dot(om.tree, om.xt, ft, om.farI[f0:f1], om.farJ[f0:f1], net, EPS, 100)
        t = torch.from_numpy(np.ascontiguousarray(u))
        dist.all_reduce(t)
        q.put((rank, (c0, c1, f0, f1), t.numpy() if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_to_the_whole_product():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, ranges, u = q.get(timeout=600)
        out[rank] = (ranges, u)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    from oracle import hignn_oracle as O

    x = S.uniform(N, 0.1, 9)
    f = S.sedimenting_forces(N, 9)
    net = O.TwoBody.from_hgnw(WEIGHTS)
    om = O.OracleModel(x, LEAF, net, epsilon=EPS)
    ft = f[om.rmap]
    ref = O.close_dot(om.tree, om.xt, ft, om.closeI, om.closeJ, net)
    ref = ref + O.far_dot(om.tree, om.xt, ft, om.farI, om.farJ, net, EPS, 100)
    u = out[0][1]
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-8
    (a0, a1, b0, b1), (c0, c1, d0, d1) = out[0][0], out[1][0]
    assert a0 == 0 and a1 == c0 and c1 == len(om.closeI)
    assert b0 == 0 and b1 == d0 and d1 == len(om.farI)


@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_shards_partition_the_lists_with_balanced_cost(world):
    x = S.uniform(20000, 0.1, 4)
    base = capi.Model(x, 128, device=-1)
    t, _ = base.tree()
    ci, cj, fi, fj = base.lists()
    sz = t[:, 3] - t[:, 2]
    close_cost = sz[ci] * sz[cj]
    ends_c, ends_f, costs = [0], [0], []
    for r in range(world):
        m = capi.Model(x, 128, device=-1)
        m.set_shard(r, world)
        c0, c1, f0, f1 = m.shard()
        assert c0 == ends_c[-1] and f0 == ends_f[-1]
        ends_c.append(c1)
        ends_f.append(f1)
        costs.append(close_cost[c0:c1].sum())
    assert ends_c[-1] == len(ci) and ends_f[-1] == len(fi)
    assert max(costs) <= close_cost.sum() / world + close_cost.max()
    with pytest.raises(capi.HignnError):
        base.set_shard(world, world)
