"""The C++/OpenMP restatement of the H-matvec (oracle/hmatvec_cpu.cpp, the CPU baseline) against
the numpy restatement: the same close field to FP64 summation order, the same ACA ranks and pivots
block for block, and the same far field."""
import numpy as np

from conftest import WEIGHTS
from hignn_b200 import synthetic as S
from oracle import hignn_oracle as O


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_cpu_hmatvec_matches_numpy_restatement():
    net = O.TwoBodyF32Exact.from_hgnw(WEIGHTS)
    x = S.uniform_min_dist(4096, 0.05, 0)
    f = S.sedimenting_forces(4096, 0)
    om = O.OracleModel(x, 128, net, epsilon=1e-2)
    ft = f[om.rmap]
    cpu = O.CpuHMatvec(om.tree, om.xt, net)
    uc_ref = O.close_dot(om.tree, om.xt, ft, om.closeI, om.closeJ, net)
    uc = cpu.close_dot(ft, om.closeI, om.closeJ)
    assert rel(uc, uc_ref) < 1e-12
    col = []
    uf_ref = O.far_dot(om.tree, om.xt, ft, om.farI, om.farJ, net, 1e-2, 100, collect=col)
    uf, ranks, evals = cpu.far_dot(ft, om.farI, om.farJ, 1e-2)
    assert np.array_equal(ranks, np.array([c[2] for c in col]))
    assert evals == sum(c[2] * (om.tree[c[0], 3] - om.tree[c[0], 2] + om.tree[c[1], 3] - om.tree[c[1], 2])
                        for c in col)
    assert rel(uf, uf_ref) < 1e-10
    # a sample of the lists (the benchmark's CPU baseline times such samples)
    u2 = cpu.close_dot(ft, om.closeI, om.closeJ, 10, 50)
    ref2 = O.close_dot(om.tree, om.xt, ft, om.closeI[10:50], om.closeJ[10:50], net)
    assert rel(u2, ref2) < 1e-12
