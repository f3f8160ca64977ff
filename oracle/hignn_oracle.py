"""CPU oracle for the H-HIGNN mobility matvec U = M(x) F -- TEST INFRASTRUCTURE ONLY.

This module is a numpy restatement of the reference algorithm. It is used by
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg as
the checker; the product (``hignn_b200``) never imports it.

Pinning. The two-body kernel is pinned against golden vectors produced by the
reference's own ``Net`` wrapper (python/convert.py:6-20) on the shipped
``nn/two_body_unbounded.pkl`` (tests/golden/two_body_net.npz). The H-matrix
parts (tree, admissibility, CloseDot, FarDot/ACA, DenseDot) restate the C++
sources line by line; the reference's own tests pin none of them (its only
tests are docker smoke tests) and its C++ cannot be built here (Kokkos, Eigen,
MPI, VTK are absent), so for those parts parity is unpinned against the
reference binary and rests on this restatement. Also pinned: the three-body and
self terms against the reference's own model classes
(python/HIGNN/model_structure.py; tests/golden/three_body_velocity.npz), the
filament forces against its chain_bending / chain_tension (python/simulate.py;
tests/golden/filament_forces.npz), and the Dormand-Prince integrator against
scipy's DOP853 on a smooth system (tests/test_oracle_dp45.py).

Declared choices where the reference is solver-defined:
* PCA direction: the reference takes U(:,0) of an Eigen JacobiSVD of the
  centred 3xL float matrix (src/HignnModel.cpp:149-151). Here it is the
  dominant eigenvector of the 3x3 covariance (FP64 sums of the float centred
  coordinates) from a cyclic Jacobi solve, rounded to float, with the sign
  fixed so that its largest-magnitude component is positive. Eigen's sign is
  implementation-defined (it swaps child order and reverses in-node order).
* The mean (FP32) and the covariance (FP64) of a node are summed in blocks of
  SUM_BLOCK consecutive particles, then over the block sums; the reference sums
  the mean sequentially (src/HignnModel.cpp:130-135).
* The ACA factors C_l, Q_l are stored in FP32 (the reference: FP64), every
  operation on them in FP64.
* The FP32 network of the plain form (TwoBodyF32Exact, oracle/twobody_f32.c)
  performs the operations of the library's plain network in the same order,
  with the same tanh; the FP64 network (TwoBody.eval64) is the dense oracle's.
* ``std::sort`` with ``par_unseq`` is not stable (src/HignnModel.cpp:165-171);
  ties in the projection are ordered by position here (stable sort).
* Team reductions (Kokkos MaxLoc / Sum) are sequential here; MaxLoc takes the
  first index among equal maxima.
"""
from __future__ import annotations

import math
import os
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_NTHREADS = max(1, os.cpu_count() or 1)
_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(_NTHREADS)
    return _POOL


# ----------------------------------------------------------------------------------------------
# Two-body kernel: python/convert.py:11-20 (Net.forward over the reference nn.Sequential)
# ----------------------------------------------------------------------------------------------
class TwoBody:
    """y = W3 tanh(W2 tanh(W1 r + b1) + b2) + b3; y[0,4,8] += 1; y /= |r|; |r| < 1e-5 -> I."""

    def __init__(self, weights, biases):
        self.w32 = [np.ascontiguousarray(w, np.float32) for w in weights]
        self.b32 = [np.ascontiguousarray(b, np.float32) for b in biases]
        self.w64 = [w.astype(np.float64) for w in self.w32]
        self.b64 = [b.astype(np.float64) for b in self.b32]

    @classmethod
    def from_hgnw(cls, path):
        import sys

        sys.path.insert(0, os.path.dirname(_HERE))
        from hignn_b200.weights import load_hgnw  # file-format reader only

        m = load_hgnw(path)
        return cls(m.weights, m.biases)

    def _inner(self, r, ws, bs):
        h = r
        for li, (w, b) in enumerate(zip(ws, bs)):
            h = h @ w.T + b
            if li + 1 < len(ws):
                h = np.tanh(h)
        return h

    def _chunked(self, r, fn, out_dtype, chunk=32768):
        n = r.shape[0]
        out = np.empty((n, 9), out_dtype)
        if n <= chunk:
            out[:] = fn(r)
            return out
        starts = list(range(0, n, chunk))

        def work(s):
            out[s:s + chunk] = fn(r[s:s + chunk])

        list(_pool().map(work, starts))
        return out

    def inner64(self, r):
        r = np.asarray(r, np.float64)
        return self._chunked(r, lambda x: self._inner(x, self.w64, self.b64), np.float64)

    def eval32(self, r):
        """FP32 mirror of the libtorch forward used by CloseDot/FarDot (src/CloseDot.cpp:233)."""
        r = np.ascontiguousarray(r, np.float32)

        def fn(x):
            y = self._inner(x, self.w32, self.b32).astype(np.float32)
            y[:, 0] += np.float32(1)
            y[:, 4] += np.float32(1)
            y[:, 8] += np.float32(1)
            nr = np.sqrt((x * x).sum(1, dtype=np.float32)).astype(np.float32)
            with np.errstate(divide="ignore", invalid="ignore"):
                y = y / nr[:, None]
            y[nr < 1e-5] = np.eye(3, dtype=np.float32).reshape(9)
            return y

        return self._chunked(r, fn, np.float32)

    def eval64(self, r):
        """FP64 evaluation of the same network and wrapper (the dense oracle's kernel)."""
        r = np.asarray(r, np.float64)

        def fn(x):
            y = self._inner(x, self.w64, self.b64)
            y[:, 0] += 1.0
            y[:, 4] += 1.0
            y[:, 8] += 1.0
            nr = np.sqrt((x * x).sum(1))
            with np.errstate(divide="ignore", invalid="ignore"):
                y = y / nr[:, None]
            y[nr < 1e-5] = np.eye(3).reshape(9)
            return y

        return self._chunked(r, fn, np.float64)


class TwoBodyF32Exact(TwoBody):
    """TwoBody whose FP32 evaluation is the C restatement (oracle/twobody_f32.c) of the plain
    device network: the same correctly rounded FP32 operations in the same order and the same
    tanh, so its outputs equal the device's bit for bit. The FP64 evaluation is TwoBody's."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            import ctypes

            import importlib

            build = importlib.import_module("oracle.build")
            path = build.build()
            lib = ctypes.CDLL(path)
            fp = ctypes.POINTER(ctypes.c_float)
            lib.oracle_twobody_eval32.argtypes = [fp] * 7 + [ctypes.c_int64, fp, ctypes.c_int]
            lib.oracle_twobody_eval32.restype = None
            lib.oracle_tanh_f32.argtypes = [fp, ctypes.c_int64, fp]
            lib.oracle_tanh_f32.restype = None
            cls._lib = lib
        return cls._lib

    def __init__(self, weights, biases, threads=None):
        super().__init__(weights, biases)
        self.threads = threads or os.cpu_count() or 1

    def eval32(self, r):
        import ctypes

        fp = ctypes.POINTER(ctypes.c_float)
        r = np.ascontiguousarray(r, np.float32)
        y = np.empty((r.shape[0], 9), np.float32)
        w = [np.ascontiguousarray(a, np.float32) for a in (self.w32[0], self.b32[0], self.w32[1], self.b32[1],
                                                           self.w32[2], self.b32[2])]
        if r.shape[0]:
            self.lib().oracle_twobody_eval32(*[a.ctypes.data_as(fp) for a in w], r.ctypes.data_as(fp), r.shape[0],
                                             y.ctypes.data_as(fp), int(self.threads))
        return y


def _cpu_lib():
    import ctypes

    lib = TwoBodyF32Exact.lib()
    if not getattr(lib, "_hmatvec_ready", False):
        fp, dp, lp = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
        i64, c_int = ctypes.c_int64, ctypes.c_int
        lib.oracle_close_dot.argtypes = [fp] * 8 + [lp] * 4 + [i64, i64, c_int, c_int, dp]
        lib.oracle_close_dot.restype = None
        lib.oracle_far_dot.argtypes = ([fp] * 8 + [lp] * 4 + [i64, i64, ctypes.c_double, c_int, c_int, c_int, dp,
                                       ctypes.POINTER(ctypes.c_int32)])
        lib.oracle_far_dot.restype = ctypes.c_int64
        lib._hmatvec_ready = True
    return lib


class CpuHMatvec:
    """The C++/OpenMP restatement of the H-matvec (oracle/hmatvec_cpu.cpp) on a built tree: the
    same blocks and ACA rules as close_dot / aca_blocks / aca_apply, the FP32 network of
    TwoBodyF32Exact, every block on one host thread (dynamic schedule over the threads)."""

    def __init__(self, tree, xt, net, threads=None):
        self.tree = tree
        self.xt = np.ascontiguousarray(xt, np.float32)
        self.net = net
        self.threads = int(threads or os.cpu_count() or 1)
        self.nstart = np.ascontiguousarray(tree[:, 2], np.int64)
        self.nend = np.ascontiguousarray(tree[:, 3], np.int64)
        self.w = [np.ascontiguousarray(a, np.float32) for a in (net.w32[0], net.b32[0], net.w32[1], net.b32[1],
                                                               net.w32[2], net.b32[2])]

    def _common(self, ft):
        import ctypes

        fp = ctypes.POINTER(ctypes.c_float)
        lp = ctypes.POINTER(ctypes.c_int64)
        self._ft = np.ascontiguousarray(ft, np.float32)
        return ([a.ctypes.data_as(fp) for a in self.w] + [self.xt.ctypes.data_as(fp), self._ft.ctypes.data_as(fp),
                self.nstart.ctypes.data_as(lp), self.nend.ctypes.data_as(lp)])

    def close_dot(self, ft, closeI, closeJ, p0=0, p1=None, use_symmetry=True, u=None):
        import ctypes

        ci = np.ascontiguousarray(closeI, np.int64)
        cj = np.ascontiguousarray(closeJ, np.int64)
        p1 = len(ci) if p1 is None else p1
        u = np.zeros((self.xt.shape[0], 3), np.float64) if u is None else u
        lp = ctypes.POINTER(ctypes.c_int64)
        _cpu_lib().oracle_close_dot(*self._common(ft), ci.ctypes.data_as(lp), cj.ctypes.data_as(lp), int(p0), int(p1),
                                    int(bool(use_symmetry)), self.threads,
                                    u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return u

    def far_dot(self, ft, farI, farJ, epsilon, max_iter=100, p0=0, p1=None, use_symmetry=True, u=None):
        """Adds the far field of far pairs [p0, p1) into u; returns (u, ranks, ACA evaluations)."""
        import ctypes

        fi = np.ascontiguousarray(farI, np.int64)
        fj = np.ascontiguousarray(farJ, np.int64)
        p1 = len(fi) if p1 is None else p1
        u = np.zeros((self.xt.shape[0], 3), np.float64) if u is None else u
        ranks = np.zeros(max(0, p1 - p0), np.int32)
        lp = ctypes.POINTER(ctypes.c_int64)
        ev = _cpu_lib().oracle_far_dot(*self._common(ft), fi.ctypes.data_as(lp), fj.ctypes.data_as(lp), int(p0),
                                       int(p1), float(epsilon), int(max_iter), int(bool(use_symmetry)), self.threads,
                                       u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       ranks.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return u, ranks, int(ev)


def tanh_f32_exact(x):
    """The plain form's FP32 tanh (oracle/twobody_f32.c) on an array."""
    import ctypes

    fp = ctypes.POINTER(ctypes.c_float)
    x = np.ascontiguousarray(x, np.float32)
    t = np.empty_like(x)
    TwoBodyF32Exact.lib().oracle_tanh_f32(x.ctypes.data_as(fp), x.size, t.ctypes.data_as(fp))
    return t


def symmetrize_f32(y32):
    """Far-field block symmetrisation, src/FarDot.cpp:445-456: diag copied, off-diag 0.5*(a+b).

    ``a + b`` is a float32 sum; the product with 0.5 is formed in double.
    """
    y = np.asarray(y32, np.float32)
    out = y.astype(np.float64)
    for row in range(3):
        for col in range(3):
            if row != col:
                l1, l2 = 3 * row + col, 3 * col + row
                out[:, l1] = 0.5 * (y[:, l1] + y[:, l2]).astype(np.float32).astype(np.float64)
    return out


# ----------------------------------------------------------------------------------------------
# Cluster tree: HignnModel::Divide (src/HignnModel.cpp:119-198), HignnModel::Build (src/Build.cpp:17-265)
# ----------------------------------------------------------------------------------------------
def jacobi_dominant_axis(cov):
    """Dominant eigenvector of a symmetric 3x3 (cyclic Jacobi, FP64), sign: max |component| > 0.

    The identical sequence of IEEE operations is used by the native tree builder,
    so the two agree bit for bit.
    """
    a = [[float(cov[i][j]) for j in range(3)] for i in range(3)]
    v = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
    for _sweep in range(50):
        off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2]
        diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2]
        if off <= 1e-36 * diag or off == 0.0:
            break
        for p, q in ((0, 1), (0, 2), (1, 2)):
            apq = a[p][q]
            if apq == 0.0:
                continue
            theta = (a[q][q] - a[p][p]) / (2.0 * apq)
            t = 1.0 / (abs(theta) + math.sqrt(theta * theta + 1.0))
            if theta < 0.0:
                t = -t
            c = 1.0 / math.sqrt(t * t + 1.0)
            s = t * c
            for k in range(3):
                akp = a[k][p]
                akq = a[k][q]
                a[k][p] = c * akp - s * akq
                a[k][q] = s * akp + c * akq
            for k in range(3):
                apk = a[p][k]
                aqk = a[q][k]
                a[p][k] = c * apk - s * aqk
                a[q][k] = s * apk + c * aqk
            for k in range(3):
                vkp = v[k][p]
                vkq = v[k][q]
                v[k][p] = c * vkp - s * vkq
                v[k][q] = s * vkp + c * vkq
    best = 0
    for k in (1, 2):
        if a[k][k] > a[best][best]:
            best = k
    u = [v[0][best], v[1][best], v[2][best]]
    big = 0
    for k in (1, 2):
        if abs(u[k]) > abs(u[big]):
            big = k
    if u[big] < 0.0:
        u = [-x for x in u]
    return u


SUM_BLOCK = 256


def _blocked_sum(v, dtype):
    """Column sums of v (L, k): each block of SUM_BLOCK consecutive rows is summed sequentially
    from zero in ``dtype``, then the block sums are summed sequentially from zero."""
    v = np.asarray(v, dtype)
    L = v.shape[0]
    nfull = L // SUM_BLOCK
    parts = []
    if nfull:
        parts.append(np.cumsum(v[:nfull * SUM_BLOCK].reshape(nfull, SUM_BLOCK, -1), axis=1, dtype=dtype)[:, -1])
    if L > nfull * SUM_BLOCK:
        parts.append(np.cumsum(v[nfull * SUM_BLOCK:], axis=0, dtype=dtype)[-1:])
    blocks = np.concatenate(parts, axis=0)
    return np.cumsum(blocks, axis=0, dtype=dtype)[-1]


def divide(coords, rmap, first, last):
    """Split [first,last) of ``rmap`` at the mean along the principal axis; returns the split index.

    src/HignnModel.cpp:125-197: float mean (sum in map order), centred float coordinates,
    principal axis, float projection t_i, sort by t, split at upper_bound(t, 0), i.e. the
    left child is {t <= 0}. The reference sums the mean sequentially; here the mean and the
    covariance sums run in blocks of SUM_BLOCK consecutive particles (see _blocked_sum), so a
    parallel device build forms the same values.
    """
    L = last - first
    pts = coords[rmap[first:last]]  # float32 (L,3)
    mean = (_blocked_sum(pts, np.float32) / np.float32(L)).astype(np.float32)
    vh = (pts - mean).astype(np.float32)
    vh64 = vh.astype(np.float64)
    cov = [[0.0] * 3 for _ in range(3)]
    prods = np.stack([vh64[:, i] * vh64[:, j] for i in range(3) for j in range(i, 3)], axis=1)
    sums = _blocked_sum(prods, np.float64)
    q = 0
    for i in range(3):
        for j in range(i, 3):
            cov[i][j] = cov[j][i] = float(sums[q])
            q += 1
    u = np.array(jacobi_dominant_axis(cov), np.float64).astype(np.float32)
    t = (u[0] * vh[:, 0]).astype(np.float32)
    t = (t + (u[1] * vh[:, 1]).astype(np.float32)).astype(np.float32)
    t = (t + (u[2] * vh[:, 2]).astype(np.float32)).astype(np.float32)
    order = np.argsort(t, kind="stable")
    rmap[first:last] = rmap[first:last][order]
    ts = t[order]
    return int(np.searchsorted(ts, np.float32(0.0), side="right")) + first


def _split_ok(d, first, last):
    # The reference treats a returned index of 0 as "leaf" (src/Build.cpp:71,160); an
    # empty child (d == first or d == last, coincident points) would make it recurse
    # forever, so it is a leaf here as well.
    return d != 0 and d != first and d != last


def build_tree(coords, leaf):
    """Tree rows [child0, child1, start, end, level] and the particle permutation, one rank.

    With one MPI rank the root is divided in the sequential stage (nodes 1, 2) and
    again at the start of the parallel stage (src/Build.cpp:31-33,112-114); the
    parallel-stage nodes are appended from row 3 (ids shifted by +2,
    src/Build.cpp:211-220) and the root is re-pointed to rows 3, 4
    (src/Build.cpp:239-240), leaving rows 1, 2 orphaned.
    """
    coords = np.ascontiguousarray(coords, np.float32)
    N = coords.shape[0]
    rmap = np.arange(N, dtype=np.int64)
    init = np.zeros((3, 5), np.int64)
    init[0] = [0, 0, 0, N, 0]
    if N > leaf:
        d = divide(coords, rmap, 0, N)
        if _split_ok(d, 0, N):
            init[0, 0:2] = [1, 2]
            init[1] = [0, 0, 0, d, 1]
            init[2] = [0, 0, d, N, 1]
    local = [list(init[0])]
    queue = deque([0])
    while queue:
        node = queue.popleft()
        s, e, lvl = local[node][2], local[node][3], local[node][4]
        d = divide(coords, rmap, s, e) if (e - s) > leaf else 0
        if not _split_ok(d, s, e):
            local[node][0] = local[node][1] = 0
        else:
            c0 = len(local)
            local.append([0, 0, s, d, lvl + 1])
            local.append([0, 0, d, e, lvl + 1])
            local[node][0], local[node][1] = c0, c0 + 1
            queue.append(c0)
            queue.append(c0 + 1)
    nloc = len(local) - 1
    if nloc == 0:
        # N <= leaf: the reference would point the root at rows 3, 4 of a 3-row tree
        # (src/Build.cpp:239-240) and read past it; here the root is a single leaf.
        tree = np.zeros((1, 5), np.int64)
        tree[0] = [0, 0, 0, N, 0]
        return tree, rmap
    tree = np.zeros((nloc + 3, 5), np.int64)
    tree[0:3] = init
    for i in range(nloc):
        row = local[i + 1]
        c0, c1 = (row[0] + 2, row[1] + 2) if row[0] != 0 else (0, 0)
        tree[3 + i] = [c0, c1, row[2], row[3], row[4]]
    tree[0, 0], tree[0, 1] = 3, 4
    return tree, rmap


# ----------------------------------------------------------------------------------------------
# Bounding boxes and close/far lists: src/CloseFarCheck.cpp:11-465, src/HignnModel.cpp:482-518
# ----------------------------------------------------------------------------------------------
def reachable_nodes(tree):
    out, st = [], [0]
    while st:
        n = st.pop()
        out.append(n)
        if tree[n, 0] != 0:
            st.append(int(tree[n, 0]))
            st.append(int(tree[n, 1]))
    return out


def compute_aux(tree, xt):
    """[xmin,xmax,ymin,ymax,zmin,zmax] per reachable node over its (tree-ordered) range.

    Leaves use ComputeAux (src/HignnModel.cpp:76-95); internal nodes take min/max of
    their children (src/CloseFarCheck.cpp:70-108), which is the same exact value.
    """
    aux = np.zeros((tree.shape[0], 6), np.float32)
    aux[:, 0] = -np.finfo(np.float32).max
    for n in reachable_nodes(tree):
        s, e = int(tree[n, 2]), int(tree[n, 3])
        if e > s:
            p = xt[s:e]
            aux[n, 0::2] = p.min(0)
            aux[n, 1::2] = p.max(0)
        else:
            aux[n, 0::2] = np.finfo(np.float32).max
            aux[n, 1::2] = -np.finfo(np.float32).max
    return aux


def is_far(aux, n1, n2):
    """HignnModel::CloseFarCheck(aux, node1, node2), src/HignnModel.cpp:482-518 (float arithmetic)."""
    a, b = aux[n1], aux[n2]
    if not (a[0] > b[1] or a[1] < b[0] or a[2] > b[3] or a[3] < b[2] or a[4] > b[5] or a[5] < b[4]):
        return False
    f = np.float32
    d0 = f(0)
    d1 = f(0)
    dist = f(0)
    for j in range(3):
        t = f(a[2 * j] - a[2 * j + 1])
        d0 = f(d0 + f(t * t))
        t = f(b[2 * j] - b[2 * j + 1])
        d1 = f(d1 + f(t * t))
        t = f(f(f(a[2 * j] + a[2 * j + 1]) - b[2 * j]) - b[2 * j + 1])
        dist = f(dist + f(t * t))
    dist = f(dist * f(0.25))
    return bool(dist > d0 and dist > d1)


def _diam2(aux):
    """Squared box diagonal per node with the float32 operation order of src/HignnModel.cpp:500-504."""
    d = np.zeros(aux.shape[0], np.float32)
    with np.errstate(over="ignore", invalid="ignore"):  # unreachable rows 1, 2 hold -FLT_MAX
        for j in range(3):
            t = (aux[:, 2 * j] - aux[:, 2 * j + 1]).astype(np.float32)
            d = (d + (t * t).astype(np.float32)).astype(np.float32)
    return d


def is_far_many(aux, diam2, i, js):
    """Vectorised HignnModel::CloseFarCheck(aux, i, j) over candidate nodes js (same float32 rounding)."""
    js = np.asarray(js, np.int64)
    a, b = aux[i], aux[js]
    disjoint = ((a[0] > b[:, 1]) | (a[1] < b[:, 0]) | (a[2] > b[:, 3]) | (a[3] < b[:, 2])
                | (a[4] > b[:, 5]) | (a[5] < b[:, 4]))
    dist = np.zeros(len(js), np.float32)
    for j in range(3):
        t = ((np.float32(a[2 * j] + a[2 * j + 1]) - b[:, 2 * j]).astype(np.float32) - b[:, 2 * j + 1]).astype(np.float32)
        dist = (dist + (t * t).astype(np.float32)).astype(np.float32)
    dist = (dist * np.float32(0.25)).astype(np.float32)
    return disjoint & (dist > diam2[i]) & (dist > diam2[js])


def close_far_lists(tree, aux, max_relative_coord=500000, use_symmetry=True):
    """Dual traversal (src/CloseFarCheck.cpp:179-290) and flattening (:292-454).

    Returns (closeI, closeJ, farI, farJ, leaf_list) in the reference's order.
    """
    nn = tree.shape[0]
    sizes = (tree[:, 3] - tree[:, 2]).astype(np.int64)
    d2 = _diam2(aux)
    far = [[] for _ in range(nn)]
    close = [[] for _ in range(nn)]
    close[0] = [0]
    leaves = []
    q = deque([0])
    while q:
        i = q.popleft()
        cand = close[i]
        fl = is_far_many(aux, d2, i, cand).tolist() if cand else []
        if tree[i, 0] != 0:
            child_close = []
            for j, fr in zip(cand, fl):
                if fr and sizes[i] < max_relative_coord and sizes[j] < max_relative_coord:
                    far[i].append(j)
                elif tree[j, 0] != 0:
                    child_close.append(int(tree[j, 0]))
                    child_close.append(int(tree[j, 1]))
                else:
                    child_close.append(j)
            close[int(tree[i, 0])] = list(child_close)
            close[int(tree[i, 1])] = list(child_close)
            q.append(int(tree[i, 0]))
            q.append(int(tree[i, 1]))
        else:
            new_close = []
            for j, fr in zip(cand, fl):
                if fr:
                    if sizes[j] < max_relative_coord:
                        far[i].append(j)
                    else:
                        st = [j]
                        while st:
                            c = st.pop()
                            if sizes[c] < max_relative_coord:
                                far[i].append(c)
                            else:
                                st.append(int(tree[c, 0]))
                                st.append(int(tree[c, 1]))
                else:
                    if tree[j, 0] == 0:
                        new_close.append(j)
                    else:
                        st = [j]
                        while st:
                            c = st.pop()
                            if tree[c, 0] != 0:
                                st.append(int(tree[c, 0]))
                                st.append(int(tree[c, 1]))
                            else:
                                new_close.append(c)
            close[i] = new_close
            leaves.append(i)
    cI, cJ = [], []
    for i in leaves:
        for j in close[i]:
            if (not use_symmetry) or j >= i:
                cI.append(i)
                cJ.append(j)
    fI, fJ = [], []
    for i in range(nn):
        for j in far[i]:
            if (not use_symmetry) or j >= i:
                fI.append(i)
                fJ.append(j)
    return (np.array(cI, np.int64), np.array(cJ, np.int64), np.array(fI, np.int64),
            np.array(fJ, np.int64), np.array(leaves, np.int64))


# ----------------------------------------------------------------------------------------------
# CloseDot: src/CloseDot.cpp:177-299
# ----------------------------------------------------------------------------------------------
def close_dot(tree, xt, ft, closeI, closeJ, net, use_symmetry=True, max_batch=1 << 20):
    """u_I[j] += M(x_J[k] - x_I[j]) f_J[k]; if J > I also u_J[k] += (same M) f_I[j]. FP64 accumulation."""
    u = np.zeros((xt.shape[0], 3), np.float64)
    f64 = ft.astype(np.float64)
    pairs = list(zip(closeI.tolist(), closeJ.tolist()))
    p0 = 0
    while p0 < len(pairs):
        batch, tot = [], 0
        while p0 < len(pairs):
            I, J = pairs[p0]
            n = int((tree[I, 3] - tree[I, 2]) * (tree[J, 3] - tree[J, 2]))
            if batch and tot + n > max_batch:
                break
            batch.append((I, J))
            tot += n
            p0 += 1
        rs = []
        for I, J in batch:
            xI = xt[tree[I, 2]:tree[I, 3]]
            xJ = xt[tree[J, 2]:tree[J, 3]]
            rs.append((xJ[None, :, :] - xI[:, None, :]).reshape(-1, 3))
        M = net.eval32(np.concatenate(rs)).astype(np.float64)
        off = 0
        for I, J in batch:
            sI, eI, sJ, eJ = (int(v) for v in (tree[I, 2], tree[I, 3], tree[J, 2], tree[J, 3]))
            nI, nJ = eI - sI, eJ - sJ
            m = M[off:off + nI * nJ].reshape(nI, nJ, 3, 3)
            off += nI * nJ
            u[sI:eI] += np.einsum("ijrc,jc->ir", m, f64[sJ:eJ])
            if use_symmetry and J > I:
                u[sJ:eJ] += np.einsum("ijrc,ic->jr", m, f64[sI:eI])
    return u


# ----------------------------------------------------------------------------------------------
# FarDot: adaptive cross approximation per admissible block, src/FarDot.cpp:191-1388
# ----------------------------------------------------------------------------------------------
def det3(m):
    """Signed determinant exactly as src/FarDot.cpp:557-558 (double, no fused multiply-add)."""
    a, b, c, d, e, f, g, h, i = (m[:, k] for k in range(9))
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)


def inv3(m):
    """Adjugate / det inverse of one 3x3 (src/FarDot.cpp:588-609)."""
    a, b, c, d, e, f, g, h, i = (float(x) for x in m)
    det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)
    return np.array([(e * i - f * h) / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                     -(d * i - f * g) / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                     (d * h - e * g) / det, -(a * h - b * g) / det, (a * e - b * d) / det])


def _first_argmax(v, excluded):
    """Kokkos MaxLoc with a strict '>' over unused indices: the first maximal index wins."""
    vv = np.array(v, np.float64, copy=True)
    if excluded:
        vv[list(excluded)] = -np.inf
    if vv.size == 0 or not np.any(vv > -np.inf):
        return -1
    return int(np.argmax(vv))


def _f32(v):
    """Values rounded to FP32 and widened again: the ACA factors are stored in FP32 (the
    reference stores FP64, src/FarDot.cpp:104-107; every operation on them is FP64 either way),
    and the pivot searches, norms and the apply see the stored values."""
    return np.asarray(v, np.float64).astype(np.float32).astype(np.float64)


def _orth_col(C, Q, k, jk, Ck):
    """C_k(i) -= sum_{l<k} C_l(i) Q_l(jk)  (src/FarDot.cpp:502-511).

    FP64 sums here may associate differently from the reference's sequential loop
    (a 1e-16 relative effect, far below the FP32 network's own rounding).
    """
    if k == 0:
        return Ck
    nI = Ck.shape[0]
    A = C[:k].reshape(k, nI, 3, 3).transpose(1, 2, 0, 3).reshape(nI * 3, k * 3)  # (i,row) x (l,m)
    B = Q[:k, jk].reshape(k * 3, 3)                                               # (l,m) x col
    return Ck - (A @ B).reshape(Ck.shape)


def _orth_row(C, Q, k, ik, Qk):
    """Q_k(j) -= sum_{l<k} C_l(ik) Q_l(j)  (src/FarDot.cpp:827-839)."""
    if k == 0:
        return Qk
    nJ = Qk.shape[0]
    A = C[:k, ik].reshape(k, 3, 3).transpose(1, 0, 2).reshape(3, k * 3)          # row x (l,m)
    B = Q[:k].reshape(k, nJ, 3, 3).transpose(0, 2, 1, 3).reshape(k * 3, nJ * 3)  # (l,m) x (j,col)
    s = (A @ B).reshape(3, nJ, 3).transpose(1, 0, 2)
    return Qk - s.reshape(Qk.shape)


def _mul_inv(Ck, inv):
    """C_k <- C_k * inv, each entry sum_k a*b accumulated left to right (src/FarDot.cpp:645-654)."""
    A = Ck.reshape(-1, 3, 3)
    B = inv.reshape(3, 3)
    out = np.empty_like(A)
    for row in range(3):
        for col in range(3):
            acc = A[:, row, 0] * B[0, col]
            acc = acc + A[:, row, 1] * B[1, col]
            acc = acc + A[:, row, 2] * B[2, col]
            out[:, row, col] = acc
    return out.reshape(Ck.shape)


def _norm_terms(Ck, Qk, C, Q, k):
    """nu2 and the mu2 increment of src/FarDot.cpp:948-1077 for iteration k (0-based)."""
    cn = [np.sum(Ck[:, c] * Ck[:, c] + Ck[:, c + 3] * Ck[:, c + 3] + Ck[:, c + 6] * Ck[:, c + 6]) for c in range(3)]
    cd = [np.sum(Ck[:, c] * Ck[:, (c + 1) % 3] + Ck[:, c + 3] * Ck[:, (c + 1) % 3 + 3]
                 + Ck[:, c + 6] * Ck[:, (c + 1) % 3 + 6]) for c in range(3)]
    qn = [np.sum(Qk[:, 3 * d] * Qk[:, 3 * d] + Qk[:, 3 * d + 1] * Qk[:, 3 * d + 1]
                 + Qk[:, 3 * d + 2] * Qk[:, 3 * d + 2]) for d in range(3)]
    qd = [np.sum(Qk[:, 0] * Qk[:, 3] + Qk[:, 1] * Qk[:, 4] + Qk[:, 2] * Qk[:, 5]),
          np.sum(Qk[:, 3] * Qk[:, 6] + Qk[:, 4] * Qk[:, 7] + Qk[:, 5] * Qk[:, 8]),
          np.sum(Qk[:, 6] * Qk[:, 0] + Qk[:, 7] * Qk[:, 1] + Qk[:, 8] * Qk[:, 2])]
    nu2 = float(cn[0] * qn[0] + cn[1] * qn[1] + cn[2] * qn[2]
                + 2.0 * qd[0] * cd[0] + 2.0 * qd[1] * cd[1] + 2.0 * qd[2] * cd[2])
    cross = np.zeros(0)
    if k >= 2:
        Cl = C[:k - 1].reshape(k - 1, -1, 3, 3)
        Ql = Q[:k - 1].reshape(k - 1, -1, 3, 3)
        nI, nJ = Ck.shape[0], Qk.shape[0]
        # column d1 of C_k . column d2 of C_l, and row d1 of Q_k . row d2 of Q_l
        ckd = np.matmul(Ck.reshape(nI * 3, 3).T[None], Cl.reshape(k - 1, nI * 3, 3))
        qkd = np.matmul(Qk.reshape(nJ, 3, 3).transpose(1, 0, 2).reshape(3, nJ * 3)[None],
                        Ql.transpose(0, 1, 3, 2).reshape(k - 1, nJ * 3, 3))
        cross = (2.0 * np.abs(ckd) * np.abs(qkd)).reshape(-1)
    return nu2, cross


class _AcaState:
    def __init__(self, xI, xJ, replay, max_iter):
        self.xI, self.xJ = xI, xJ
        self.nI, self.nJ = xI.shape[0], xJ.shape[0]
        kmax = max(1, min(max_iter, self.nI, self.nJ)) if replay is None else len(replay[0])
        self.C = np.zeros((kmax, self.nI, 9))
        self.Q = np.zeros((kmax, self.nJ, 9))
        self.rows, self.cols = [], [self.nJ // 2]
        self.mu2 = 0.0
        self.nu2 = 0.0
        self.k = 0
        self.done = False
        self.replay = replay


def aca_blocks(blocks, net, epsilon, max_iter, replays=None):
    """ACA of symmetrised blocks A(i,j) = sym(M(x_j - x_i)) for a list of far pairs (xI, xJ).

    All blocks advance in lock-step with one batched network query per half
    step, like the reference's batches. Per block this follows
    src/FarDot.cpp:257 (first column |J|/2), :348-458 (column query and
    symmetrisation), :474-512 (C orthogonalisation over all previous
    iterations), :520-611 (row pivot = max signed det over unused rows, adjugate
    inverse), :614-656 (C_k <- C_k inv(C_k(ik))), :672-781 (row query),
    :797-841 (Q orthogonalisation), :846-903 (column pivot excluding the current
    and earlier columns), :919-1109 (nu2, mu2 with |.| cross terms that skip
    l = k-1; stop if nu2 < mu2 eps^2, k >= maxIter or k >= min(|I|,|J|)).
    ``replays[b]`` = (rows, cols) forces a pivot sequence, for comparing two
    implementations whose FP32 network outputs differ in the last bits.
    Returns one dict per block: C (k, nI, 9), Q (k, nJ, 9), rows, cols, rank.
    """
    eps2 = epsilon * epsilon
    st = [_AcaState(xI, xJ, None if replays is None else replays[b], max_iter) for b, (xI, xJ) in enumerate(blocks)]
    while True:
        act = [s for s in st if not s.done]
        if not act:
            break
        feats = [(s.xJ[s.cols[s.k]][None, :] - s.xI).astype(np.float32) for s in act]
        Y = symmetrize_f32(net.eval32(np.concatenate(feats)))
        off = 0
        for s in act:
            Ck = _f32(_orth_col(s.C, s.Q, s.k, s.cols[s.k], Y[off:off + s.nI]))
            off += s.nI
            dets = det3(Ck)
            ik = _first_argmax(dets, set(s.rows)) if s.replay is None else int(s.replay[0][s.k])
            s.rows.append(ik)
            s.Ck = _f32(_mul_inv(Ck, inv3(Ck[ik])))
        feats = [(s.xJ - s.xI[s.rows[s.k]][None, :]).astype(np.float32) for s in act]
        Y = symmetrize_f32(net.eval32(np.concatenate(feats)))
        off = 0
        for s in act:
            k = s.k
            Qk = _f32(_orth_row(s.C, s.Q, k, s.rows[k], Y[off:off + s.nJ]))
            off += s.nJ
            if s.replay is None:
                s.cols.append(_first_argmax(det3(Qk), set(s.cols[:k + 1])))
            else:
                s.cols.append(int(s.replay[1][k + 1]) if k + 1 < len(s.replay[1]) else -1)
            nu2, cross = _norm_terms(s.Ck, Qk, s.C, s.Q, k)
            s.nu2 = nu2
            s.mu2 = float(np.cumsum(np.concatenate([[s.mu2, nu2], cross]))[-1])
            s.C[k] = s.Ck
            s.Q[k] = Qk
            s.k = k + 1
            if s.replay is not None:
                s.done = s.k >= len(s.replay[0])
            else:
                s.done = (s.nu2 < s.mu2 * eps2) or s.k >= max_iter or s.k >= min(s.nI, s.nJ)
    return [dict(C=s.C[:s.k].copy(), Q=s.Q[:s.k].copy(), rows=s.rows, cols=s.cols, rank=s.k, nu2=s.nu2,
                 mu2=s.mu2) for s in st]


def aca_block(xI, xJ, net, epsilon, max_iter, replay=None):
    return aca_blocks([(xI, xJ)], net, epsilon, max_iter, None if replay is None else [replay])[0]


def aca_apply(res, fI, fJ, use_symmetry=True):
    """Low-rank apply (src/FarDot.cpp:1194-1388): u_I = sum_l C_l (Q_l f_J); u_J = sum_l Q_l^T (C_l^T f_I)."""
    C = res["C"].reshape(res["rank"], -1, 3, 3)
    Q = res["Q"].reshape(res["rank"], -1, 3, 3)
    mid = np.einsum("ljrc,jc->lr", Q, fJ)
    uI = np.einsum("lirc,lc->ir", C, mid)
    uJ = None
    if use_symmetry:
        mid2 = np.einsum("licr,ic->lr", C, fI)
        uJ = np.einsum("ljcr,lc->jr", Q, mid2)
    return uI, uJ


def far_dot(tree, xt, ft, farI, farJ, net, epsilon, max_iter, use_symmetry=True, collect=None,
            batch_rows=200000, replays=None):
    """FarDot over all far pairs; blocks are processed in batches of at most ``batch_rows`` rows."""
    u = np.zeros((xt.shape[0], 3), np.float64)
    f64 = ft.astype(np.float64)
    pairs = list(zip(farI.tolist(), farJ.tolist()))
    rng = lambda n: (int(tree[n, 2]), int(tree[n, 3]))
    p0 = 0
    while p0 < len(pairs):
        batch, tot = [], 0
        while p0 < len(pairs):
            (sI, eI), (sJ, eJ) = rng(pairs[p0][0]), rng(pairs[p0][1])
            if batch and tot + (eI - sI) + (eJ - sJ) > batch_rows:
                break
            batch.append(p0)
            tot += (eI - sI) + (eJ - sJ)
            p0 += 1
        blocks = [(xt[slice(*rng(pairs[b][0]))], xt[slice(*rng(pairs[b][1]))]) for b in batch]
        rep = None if replays is None else [replays[b] for b in batch]
        res = aca_blocks(blocks, net, epsilon, max_iter, rep)
        for b, r in zip(batch, res):
            I, J = pairs[b]
            (sI, eI), (sJ, eJ) = rng(I), rng(J)
            uI, uJ = aca_apply(r, f64[sI:eI], f64[sJ:eJ], use_symmetry)
            u[sI:eI] += uI
            if uJ is not None:
                u[sJ:eJ] += uJ
            if collect is not None:
                collect.append((I, J, r["rank"], list(r["rows"]), list(r["cols"])))
    return u


# ----------------------------------------------------------------------------------------------
# DenseDot (src/DenseDot.cpp:141-247): u_i = sum_j 0.5 (M + M^T)(x_j - x_i) f_j
# ----------------------------------------------------------------------------------------------
def dense_rows(x, f, rows, net, fp64=True, chunk_sources=4096):
    """Dense symmetrised matvec for the given target rows over all sources (original order)."""
    x64 = np.asarray(x, np.float64 if fp64 else np.float32)
    f64 = np.asarray(f, np.float64)
    out = np.zeros((len(rows), 3), np.float64)
    for a, i in enumerate(rows):
        acc = np.zeros(3)
        for s in range(0, x64.shape[0], chunk_sources):
            r = x64[s:s + chunk_sources] - x64[i][None, :]
            M = net.eval64(r) if fp64 else net.eval32(r).astype(np.float64)
            Ms = 0.5 * (M.reshape(-1, 3, 3) + M.reshape(-1, 3, 3).transpose(0, 2, 1))
            acc += np.einsum("jrc,jc->r", Ms, f64[s:s + chunk_sources])
        out[a] = acc
    return out


# ----------------------------------------------------------------------------------------------
# HignnModel::Dot (src/HignnModel.cpp:545-634) for one rank
# ----------------------------------------------------------------------------------------------
class OracleModel:
    def __init__(self, coords, leaf, net, epsilon=0.05, max_iter=100, max_relative_coord=500000,
                 use_symmetry=True):
        self.net = net
        self.leaf = leaf
        self.epsilon = epsilon
        self.max_iter = max_iter
        self.max_relative_coord = max_relative_coord
        self.use_symmetry = use_symmetry
        self.update_coord(coords)

    def update_coord(self, coords):
        self.x = np.ascontiguousarray(coords, np.float32)
        self.tree, self.rmap = build_tree(self.x, self.leaf)
        self.xt = self.x[self.rmap]
        self.aux = compute_aux(self.tree, self.xt)
        (self.closeI, self.closeJ, self.farI, self.farJ,
         self.leaves) = close_far_lists(self.tree, self.aux, self.max_relative_coord, self.use_symmetry)

    def dot_parts(self, f):
        ft = np.asarray(f, np.float32)[self.rmap]
        uc = close_dot(self.tree, self.xt, ft, self.closeI, self.closeJ, self.net, self.use_symmetry)
        uf = far_dot(self.tree, self.xt, ft, self.farI, self.farJ, self.net, self.epsilon, self.max_iter,
                     self.use_symmetry)
        return uc, uf

    def dot(self, f):
        uc, uf = self.dot_parts(f)
        ut = uc + uf
        u = np.empty_like(ut)
        u[self.rmap] = ut  # BackwardReorder: vCopy(map(i)) = v(i)
        return u.astype(np.float32)


# ----------------------------------------------------------------------------------------------
# Time integration: include/TimeIntegrator.hpp (float positions, double t and dt)
# ----------------------------------------------------------------------------------------------
def _periodic_offsets(x, lo, hi):
    """Per-component offset that wraps a position back into [lo, hi] (TimeIntegrator.hpp:105-115)."""
    off = np.zeros_like(x)
    span = (np.asarray(lo, np.float32) - np.asarray(hi, np.float32)).astype(np.float32)
    off = np.where(x > np.asarray(hi, np.float32), span, off)
    off = np.where(x < np.asarray(lo, np.float32), -span, off)
    return off.astype(np.float32)


def euler_run(x0, velocity, dt, tf, lim=None, output=None, output_step=1):
    """ExplicitEuler::Run (include/TimeIntegrator.hpp:431-488), float32 positions.

    ``velocity(t, pos6)`` gets t rounded to float32 and an (n, 6) array (positions wrapped
    into the box when ``lim`` = (lo, hi) is given; angles zero) and returns (n, 3).
    ``output(pos, vel)`` is called every ``output_step`` steps before the wrap is
    applied to the stored positions, as the reference does.
    """
    x = np.array(x0, np.float32, copy=True)
    n = len(x)
    t, count = 0.0, 0
    while t < tf - 1e-5:
        h = min(dt, tf - t)
        inp = np.zeros((n, 6), np.float32)
        inp[:, :3] = x if lim is None else x + _periodic_offsets(x, *lim)
        v = np.asarray(velocity(float(np.float32(t + h)), inp), np.float32)[:, :3]  # t passed as float
        x = (x + v * np.float32(h)).astype(np.float32)
        off = None if lim is None else _periodic_offsets(x, *lim)
        t += h
        if output is not None and count % output_step == 0:
            output(x.copy(), v.copy())
        if off is not None:
            x = (x + off).astype(np.float32)
        count += 1
    return x, count


def dp45_run(x0, velocity, dt, tf, threshold=1e-3, output=None, output_step=1):
    """ExplicitRk4::Run (include/TimeIntegrator.hpp:602-860): adaptive Dormand-Prince 5(4)
    with FSAL, float32 stage arithmetic, no periodic box.

    Reproduced quirks: k1 is zero on the first step (the initial evaluation writes the
    velocity, :608); the step size grown at the end of a step is discarded because the
    next step starts from min(h0, tf - t) (:616).
    """
    f32 = np.float32
    a = {
        21: f32(1) / f32(5), 31: f32(3) / f32(40), 32: f32(9) / f32(40),
        41: f32(44) / f32(45), 42: f32(-56) / f32(15), 43: f32(32) / f32(9),
        51: f32(19372) / f32(6561), 52: f32(-25360) / f32(2187), 53: f32(64448) / f32(6561),
        54: f32(-212) / f32(729),
        61: f32(9017) / f32(3168), 62: f32(-355) / f32(33), 63: f32(46732) / f32(5247), 64: f32(49) / f32(176),
        65: f32(-5103) / f32(18656),
    }
    b1, b3, b4 = f32(35) / f32(384), f32(500) / f32(1113), f32(125) / f32(192)
    b5, b6 = f32(-2187) / f32(6784), f32(11) / f32(84)
    dc = [b1 - f32(5179) / f32(57600), None, b3 - f32(7571) / f32(16695), b4 - f32(393) / f32(640),
          b5 - f32(-92097) / f32(339200), b6 - f32(187) / f32(2100), f32(-1) / f32(40)]
    c = [f32(0), f32(1) / f32(5), f32(3) / f32(10), f32(4) / f32(5), f32(8) / f32(9), f32(1), f32(1)]
    rows = {1: [(1, a[21])], 2: [(1, a[31]), (2, a[32])], 3: [(1, a[41]), (2, a[42]), (3, a[43])],
            4: [(1, a[51]), (2, a[52]), (3, a[53]), (4, a[54])],
            5: [(1, a[61]), (2, a[62]), (3, a[63]), (4, a[64]), (5, a[65])],
            6: [(1, b1), (3, b3), (4, b4), (5, b5), (6, b6)]}
    x = np.array(x0, np.float32, copy=True)
    n = len(x)
    k = {i: np.zeros((n, 3), np.float32) for i in range(1, 8)}

    def vel(t, p):
        inp = np.zeros((n, 6), np.float32)
        inp[:, :3] = p
        return np.asarray(velocity(float(np.float32(t)), inp), np.float32)[:, :3]  # t passed as float

    v = vel(0.0, x)
    t, count = 0.0, 0
    while t < tf - 1e-5:
        h = min(dt, tf - t)
        x0s = x.copy()
        err = 100.0
        while err > threshold:
            for i in range(1, 7):
                p = x0s.copy()
                for j, coef in rows[i]:
                    p = (p + k[j] * f32(float(coef) * h)).astype(np.float32)  # (a_ij * dt) in double, then float
                x = p
                v = vel(t + float(c[i]) * h, x)
                k[i + 1] = v
            ve = (k[1] * dc[0] + k[3] * dc[2] + k[4] * dc[3] + k[5] * dc[4] + k[6] * dc[5] + k[7] * dc[6])
            ve = (ve.astype(np.float32) * f32(h)).astype(np.float32)
            sq = (ve[:, 0] * ve[:, 0] + ve[:, 1] * ve[:, 1] + ve[:, 2] * ve[:, 2]).astype(np.float32)
            err = math.sqrt(float(np.sum(sq.astype(np.float64))))
            if err > threshold:
                h = h * max(0.8 * (err / threshold) ** -0.2, 0.1)
                h = max(h, 1e-6)
        t += h
        if output is not None and count % output_step == 0:
            output(x.copy(), v.copy())
        k[1] = k[7].copy()
        count += 1
    return x, count


# ----------------------------------------------------------------------------------------------
# Pair forces: PotentialForce::GetPotentialForce (include/PotentialForce.hpp:468-593) with the
# Morse force of CalculatePotentialForce (:115-140), parameters instead of De = 1, a = 1, re = 2.5
# ----------------------------------------------------------------------------------------------
def pair_forces(x, gravity=(0.0, 0.0, 0.0), De=1.0, a=1.0, re=2.5, cutoff=0.0):
    """f_i = gravity + sum over neighbours j != i of r fMag / |r|, r = x_i - x_j (float32).

    Neighbours: sqrt(sum (double)(x_j - x_i)^2) squared < cutoff^2 (the kd-tree radius search's
    metric, include/PointCloudSearch.hpp:231-240, strict <), and |r| > 1e-3 (float).
    fMag = -2 a De (exp(-a (|r| - re)) - exp(-2 a (|r| - re))): the exponentials in float, the
    product with -2 a De in double, stored as float (include/PotentialForce.hpp:125-131).
    """
    from scipy.spatial import cKDTree

    x = np.asarray(x, np.float32)
    n = len(x)
    f = np.zeros((n, 3), np.float32)
    if cutoff > 0:
        pairs = cKDTree(x.astype(np.float64)).query_pairs(cutoff * (1 + 1e-6), output_type="ndarray")
        if len(pairs):
            ii = np.concatenate([pairs[:, 0], pairs[:, 1]])
            jj = np.concatenate([pairs[:, 1], pairs[:, 0]])
            d = x[jj].astype(np.float64) - x[ii].astype(np.float64)
            dist = np.sqrt(np.sum(d * d, axis=1))
            keep = dist * dist < float(np.float32(cutoff) * np.float32(cutoff))  # float radius, squared in float
            ii, jj = ii[keep], jj[keep]
            r = (x[ii] - x[jj]).astype(np.float32)
            rn = np.sqrt(np.sum(r * r, axis=1, dtype=np.float32)).astype(np.float32)
            keep = rn > np.float32(1e-3)
            ii, r, rn = ii[keep], r[keep], rn[keep]
            a32, re32, de32 = np.float32(a), np.float32(re), np.float32(De)
            e1 = np.exp((-a32 * (rn - re32)).astype(np.float32)).astype(np.float32)
            e2 = np.exp((np.float32(-2.0) * a32 * (rn - re32)).astype(np.float32)).astype(np.float32)
            fmag = (-2.0 * float(a32) * float(de32) * (e1 - e2).astype(np.float64)).astype(np.float32)
            ratio = (fmag / rn).astype(np.float32)
            np.add.at(f, ii, (r * ratio[:, None]).astype(np.float32))
    return (f + np.asarray(gravity, np.float32)[None, :]).astype(np.float32)


# ---------------------------------------------------------------- neighbour lists
def radius_sq(eps):
    """The reference's squared search radius: eps squared in float, then widened
    (include/PointCloudSearch.hpp:395-397: epsilons(i) * epsilons(i) of a float view)."""
    e = np.float32(eps)
    return float(np.float32(e * e))


def neighbour_csr(x, eps):
    """Per particle i the neighbours j != i, ascending: (off int64[n + 1], nbr int64[E]).

    A neighbour is any j with sqrt(sum((double)x_j - (double)x_i)^2)^2 < radius_sq(eps): the vendored
    nanoflann metric (include/nanoflann.hpp:387-399 squares PointCloudSearch::kdtree_distance,
    include/PointCloudSearch.hpp:231-240) and RadiusResultSet::addPoint's strict test
    (include/PointCloudSearch.hpp:56-72). The particle itself (distance 0) is the entry the reference
    swaps to the front and skips (include/NeighborLists.hpp:207-224, 496-506).
    """
    from scipy.spatial import cKDTree

    x = np.asarray(x, np.float32)
    n = len(x)
    if n == 0:
        return np.zeros(1, np.int64), np.zeros(0, np.int64)
    x64 = x.astype(np.float64)
    c2 = radius_sq(eps)
    pairs = cKDTree(x64).query_pairs(math.sqrt(c2) * (1 + 1e-6), output_type="ndarray")
    if len(pairs) == 0:
        return np.zeros(n + 1, np.int64), np.zeros(0, np.int64)
    ii = np.concatenate([pairs[:, 0], pairs[:, 1]])
    jj = np.concatenate([pairs[:, 1], pairs[:, 0]])
    d = x64[jj] - x64[ii]
    dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    keep = dist * dist < c2
    ii, jj = ii[keep], jj[keep]
    order = np.lexsort((jj, ii))
    ii, jj = ii[order], jj[order]
    off = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(ii, minlength=n), out=off[1:])
    return off, jj.astype(np.int64)


def neighbour_csr_brute(x, eps):
    """neighbour_csr by an all-pairs loop over rows (checks the kd-tree candidate search)."""
    x = np.asarray(x, np.float32)
    x64 = x.astype(np.float64)
    c2 = radius_sq(eps)
    off, nbr = [0], []
    for i in range(len(x)):
        d = x64 - x64[i]
        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        js = np.nonzero(dist * dist < c2)[0]
        js = js[js != i]
        nbr.extend(js.tolist())
        off.append(len(nbr))
    return np.asarray(off, np.int64), np.asarray(nbr, np.int64)


def two_body_edge_info(off, nbr):
    """BuildTwoBodyInfo + GetTwoBodyEdgeInfo (include/NeighborLists.hpp:466-510, 289-307):
    uint64 (2, E), rows (i, j) for j in N(i) \\ {i}."""
    n = len(off) - 1
    i = np.repeat(np.arange(n, dtype=np.uint64), np.diff(off))
    return np.stack([i, nbr.astype(np.uint64)]) if len(nbr) else np.zeros((2, 0), np.uint64)


def three_body_edge_info(off, nbr):
    """BuildThreeBodyInfo + GetThreeBodyEdgeInfo (include/NeighborLists.hpp:512-585, 342-360):
    uint64 (3, E), rows (i, j, k) for j in N(i) \\ {i}, k in N(j) \\ {j}, k != i; and the
    triplet offsets per particle (int64[n + 1]). Vectorised form of the loops over i, j, k."""
    n = len(off) - 1
    deg = np.diff(off)
    ei = np.repeat(np.arange(n, dtype=np.int64), deg)  # the (i, j) edges in order
    ej = nbr
    dj = deg[ej] if len(ej) else np.zeros(0, np.int64)
    tot = int(dj.sum())
    ti = np.repeat(ei, dj)
    tj = np.repeat(ej, dj)
    first = np.repeat(off[ej] - np.concatenate([[0], np.cumsum(dj)[:-1]]) if len(ej) else np.zeros(0, np.int64), dj)
    tk = nbr[first + np.arange(tot, dtype=np.int64)] if tot else np.zeros(0, np.int64)
    keep = tk != ti
    ti, tj, tk = ti[keep], tj[keep], tk[keep]
    off3 = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(ti, minlength=n), out=off3[1:])
    info = np.stack([ti, tj, tk]).astype(np.uint64) if len(ti) else np.zeros((3, 0), np.uint64)
    return info, off3


def three_body_edge_info_loops(off, nbr):
    """three_body_edge_info by the reference's own loops (small inputs)."""
    rows = []
    n = len(off) - 1
    for i in range(n):
        for t in range(off[i], off[i + 1]):
            j = int(nbr[t])
            for q in range(off[j], off[j + 1]):
                k = int(nbr[q])
                if k != i:
                    rows.append((i, j, k))
    return np.asarray(rows, np.uint64).T.reshape(3, -1)


def two_body_edge_info_by_index(n, index):
    """GetTwoBodyEdgeInfoByIndex (include/NeighborLists.hpp:309-340): for each target p all
    j != p in order, rows (j, p)."""
    rows0, rows1 = [], []
    for p in np.asarray(index, np.uint64):
        j = np.arange(n, dtype=np.uint64)
        j = j[j != p]
        rows0.append(j)
        rows1.append(np.full(len(j), p, np.uint64))
    if not rows0:
        return np.zeros((2, 0), np.uint64)
    return np.stack([np.concatenate(rows0), np.concatenate(rows1)])


def edge_info_by_index(info, off, index):
    """GetThreeBodyEdgeInfoByIndex / GetThreeBodyEdgeSelfInfoByIndex (include/NeighborLists.hpp:
    362-403, 424-464): each target's edges in turn, rows reversed."""
    parts = [info[::-1, off[p]:off[p + 1]] for p in np.asarray(index, np.int64)]
    if not parts:
        return np.zeros((info.shape[0], 0), np.uint64)
    return np.concatenate(parts, axis=1)


# ---------------------------------------------------------------- filament forces
def _cross32(a, b):
    """np.cross of float32 3-vectors: each product rounded, then the difference."""
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _norm32(v):
    """np.linalg.norm(v, axis=-1) of float32 3-vectors: sqrt((x^2 + y^2) + z^2) in float32."""
    s = v * v
    return np.sqrt((s[..., 0] + s[..., 1]) + s[..., 2])


def chain_bending(X, k_b):
    """python/simulate.py:14-54 for chains X (..., N, 3) float32 -> float64 (..., N, 3)."""
    N = X.shape[-2]
    F = np.zeros(X.shape, np.float64)
    if N < 3:
        return F
    arm1 = X[..., 1:N - 1, :] - X[..., 0:N - 2, :]
    arm2 = X[..., 2:N, :] - X[..., 1:N - 1, :]
    arm1 = arm1 / _norm32(arm1)[..., None]
    arm2 = arm2 / _norm32(arm2)[..., None]
    p = arm1 * arm2
    cos = (p[..., 0] + p[..., 1]) + p[..., 2]
    tmp = np.float32(1) - cos * cos
    tmp[tmp < 0] = np.float32(0)
    sin = np.sqrt(tmp)[..., None]
    torque = -_cross32(arm1, arm2) * sin
    f21 = _cross32(torque, arm1)
    f23 = _cross32(torque, arm2)
    F[..., 0:N - 2, :] += f21
    F[..., 1:N - 1, :] -= f21 + f23
    F[..., 2:N, :] += f23
    return k_b * F


def chain_tension(X, k_t, rest_length):
    """python/simulate.py:56-88 for chains X (..., N, 3) float32 -> float64 (..., N, 3); rest_length
    and k_t meet float32 arrays there and act as float32."""
    N = X.shape[-2]
    F = np.zeros(X.shape, np.float64)
    if N < 2:
        return F
    r = X[..., 0:N - 1, :] - X[..., 1:N, :]
    rn = _norm32(r)[..., None]
    r = r / rn
    fm = np.float32(k_t) * (rn - np.float32(rest_length))
    nodal = r * fm
    F[..., 0:N - 1, :] -= nodal
    F[..., 1:N, :] += nodal
    return F


def filament_forces(x, f0, n_filament, n_chain, rest_length, k_t, k_b):
    """velocity_update's force assembly (python/simulate.py:130-142): f0 (float32) += bending, then
    += tension, per filament of n_chain consecutive rows; all filaments at once (elementwise the same)."""
    f = np.array(f0, np.float32, copy=True)
    rows = n_filament * n_chain
    if rows == 0:
        return f
    X = np.asarray(x, np.float32)[:rows].reshape(n_filament, n_chain, 3)
    with np.errstate(divide="ignore", invalid="ignore"):
        fb = chain_bending(X, float(k_b)).reshape(rows, 3)
        ft = chain_tension(X, k_t, rest_length).reshape(rows, 3)
    f[:rows] = (f[:rows].astype(np.float64) + fb).astype(np.float32)
    f[:rows] = (f[:rows].astype(np.float64) + ft).astype(np.float32)
    return f


# ---------------------------------------------------------------- three-body near field
class DenseTanh:
    """A tanh MLP (W: out x in, row-major) as python/HIGNN/model_structure.py's nn.Sequential."""

    def __init__(self, weights, biases):
        self.w64 = [np.asarray(w, np.float64) for w in weights]
        self.b64 = [np.asarray(b, np.float64) for b in biases]

    @classmethod
    def from_hgnw(cls, path):
        import sys

        sys.path.insert(0, os.path.dirname(_HERE))
        from hignn_b200.weights import load_hgnw  # file-format reader only

        m = load_hgnw(path)
        return cls(m.weights, m.biases)

    def __call__(self, z, chunk=8192):
        z = np.asarray(z, np.float64)
        out = np.empty((len(z), self.w64[-1].shape[0]), np.float64)
        for s in range(0, len(z), chunk):
            h = z[s:s + chunk]
            for li, (w, b) in enumerate(zip(self.w64, self.b64)):
                h = h @ w.T + b
                if li + 1 < len(self.w64):
                    h = np.tanh(h)
            out[s:s + chunk] = h
        return out


def three_body_velocity(x, f, eps, net3, net_self):
    """The three-body and self terms of HIGNN_model.forward (python/HIGNN/model_structure.py:94-139)
    on the edge lists of NeighborLists at the three-body epsilon, in FP64 from float32 positions:
      triplet rows (a, b, c) (read as (j, k, i)): x_in = (x_b - x_a, x_c - x_b) in float32,
        M = net3(x_in) / |x_b - x_a| / |x_c - x_b|  (Three_body_net, :41-55),  u_c += M f_a;
      self rows (a, b) (read as (j, i)): x_in = x_a - x_b,
        M = net_self(x_in) / |x_in| / |x_in|  (Two_body_self_net, :58-70),  u_b += M f_b."""
    x = np.asarray(x, np.float32)
    f = np.asarray(f, np.float32).astype(np.float64)
    n = len(x)
    off, nbr = neighbour_csr(x, eps)
    info, _ = three_body_edge_info(off, nbr)
    pairs = two_body_edge_info(off, nbr)
    u = np.zeros((n, 3), np.float64)
    if info.shape[1]:
        a, b, c = (info[k].astype(np.int64) for k in range(3))
        d1 = x[b] - x[a]
        d2 = x[c] - x[b]
        y = net3(np.concatenate([d1, d2], axis=1))
        r1 = np.linalg.norm(d1.astype(np.float64), axis=1)
        r2 = np.linalg.norm(d2.astype(np.float64), axis=1)
        M = (y / r1[:, None] / r2[:, None]).reshape(-1, 3, 3)
        np.add.at(u, c, np.einsum("eij,ej->ei", M, f[a]))
    if pairs.shape[1]:
        a, b = (pairs[k].astype(np.int64) for k in range(2))
        d = x[a] - x[b]
        y = net_self(d)
        r = np.linalg.norm(d.astype(np.float64), axis=1)
        M = (y / r[:, None] / r[:, None]).reshape(-1, 3, 3)
        np.add.at(u, b, np.einsum("eij,ej->ei", M, f[b]))
    return u
