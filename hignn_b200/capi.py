"""ctypes binding of the C ABI in ``include/hignn_b200.h`` (``libhignn_b200.so``).

Tests and the benchmark call the native library through this module. It
raises at import time when the library has not been built: there is no
Python or CPU fallback for any operation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhignn_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hignn_b200.build`")

lib = C.CDLL(LIB_PATH)

# parameter keys (enum hignn_param)
P_EPSILON = 0
P_ETA = 1
P_MAX_ITER = 2
P_MAT_POOL_SIZE_FACTOR = 3
P_MAX_FAR_DOT_WORK_NODE_SIZE = 4
P_MAX_RELATIVE_COORD = 5
P_POST_CHECK_FLAG = 6
P_USE_SYMMETRY = 7
P_MAX_FAR_FIELD_DISTANCE = 8
P_PRECISION = 100
P_FAR_BATCH_ROWS = 101
P_TIMING = 102
P_STUDENT_TOL = 103
P_FIELDS = 104
P_RECORD_PIVOTS = 105
P_FAR_POOL_MB = 106
P_RANK_HINT_OFFSET = 107
P_TREE_DEVICE = 108
P_GRAPH = 109
P_KEEP_RANKS = 110
DENSE_F64 = 64  # hignn_dense_rows precision: the network in FP64

STUDENT_PARAMS = 2537

ERR_NAMES = {-1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_STATE", -4: "ERR_IO", -5: "ERR_LIMIT", -6: "ERR_NODEV"}


class HignnStats(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("num_nodes", C.c_int64), ("num_leaves", C.c_int64), ("num_close", C.c_int64),
        ("num_far", C.c_int64), ("close_evals", C.c_int64), ("far_evals", C.c_int64), ("far_rank_sum", C.c_int64),
        ("far_rank_max", C.c_int32), ("far_iterations", C.c_int32), ("student_fallback_blocks", C.c_int64),
        ("t_build_ms", C.c_double), ("t_close_ms", C.c_double), ("t_far_ms", C.c_double), ("t_dot_ms", C.c_double),
        ("gpu_launches", C.c_int64), ("t_far_query_ms", C.c_double), ("t_far_pivot_ms", C.c_double),
        ("t_far_active_ms", C.c_double), ("t_far_check_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_u64p = C.POINTER(C.c_uint64)

# edge list kinds (HIGNN_EDGES_*)
EDGES_TWO_BODY = 0
EDGES_THREE_BODY = 1
EDGES_THREE_BODY_SELF = 2

SIGNATURES = {
    "hignn_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
    "hignn_version": ([], C.c_int),
    "hignn_create": ([_fp, C.c_int64, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "hignn_destroy": ([_P], C.c_int),
    "hignn_load_two_body": ([_P, C.c_char_p], C.c_int),
    "hignn_load_two_body_mem": ([_P, C.c_int, C.POINTER(C.c_int32), _fp, C.c_int], C.c_int),
    "hignn_set_param": ([_P, C.c_int, C.c_double], C.c_int),
    "hignn_get_param": ([_P, C.c_int, _dp], C.c_int),
    "hignn_update_coord": ([_P, _fp, C.c_int64], C.c_int),
    "hignn_dot": ([_P, _fp, _fp, C.c_int64], C.c_int),
    "hignn_dot_device": ([_P, C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "hignn_dense_dot": ([_P, _fp, _fp, C.c_int64], C.c_int),
    "hignn_dense_rows": ([_P, _dp, _fp, _i64p, C.c_int64, C.c_int], C.c_int),
    "hignn_dense_rows_noalloc": ([_P, _dp, _fp, _i64p, C.c_int64, C.c_int], C.c_int),
    "hignn_two_body_eval": ([_P, C.c_void_p, C.c_void_p, C.c_int64, C.c_int], C.c_int),
    "hignn_get_stats": ([_P, C.POINTER(HignnStats)], C.c_int),
    "hignn_get_tree": ([_P, _i64p, _i64p], C.c_int),
    "hignn_get_lists": ([_P, _i64p, _i64p, _i64p, _i64p], C.c_int),
    "hignn_train_student": ([_P, C.c_int, C.c_int, C.c_int64, C.c_double, C.c_uint64, _dp], C.c_int),
    "hignn_set_student": ([_P, _fp, C.c_int], C.c_int),
    "hignn_get_student": ([_P, _fp, C.c_int], C.c_int),
    "hignn_student_eval": ([_P, C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "hignn_student_grad": ([_P, C.c_void_p, C.c_void_p, C.c_int64, _fp, _dp], C.c_int),
    "hignn_set_shard": ([_P, C.c_int, C.c_int], C.c_int),
    "hignn_update_coord_keep_tree": ([_P, _fp, C.c_int64], C.c_int),
    "hignn_pair_forces": ([_P, _fp, _fp, C.c_int64, _fp, C.c_double, C.c_double, C.c_double, C.c_double], C.c_int),
    "hignn_forces": ([_P, _fp, _fp, C.c_int64, C.c_void_p], C.c_int),
    "hignn_run_euler": ([_P, _fp, C.c_int64, C.c_int, C.c_double, C.c_int, C.c_void_p], C.c_int),
    "hignn_run_rk2": ([_P, _fp, C.c_int64, C.c_int, C.c_double, C.c_int, C.c_void_p], C.c_int),
    "hignn_set_three_body": ([_P, _P], C.c_int),
    "hignn_run_dp45": ([_P, _fp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p, _i64p],
                       C.c_int),
    "hignn_get_shard": ([_P, _i64p], C.c_int),
    "hignn_get_far_pivots": ([_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int], C.c_int),
    "hignn_synchronize": ([_P], C.c_int),
    "hignn_get_stream": ([_P, C.POINTER(C.c_void_p)], C.c_int),
    "hignn_nbl_create": ([C.c_int, C.POINTER(_P)], C.c_int),
    "hignn_nbl_destroy": ([_P], None),
    "hignn_nbl_update_coord": ([_P, _fp, C.c_int64], C.c_int),
    "hignn_nbl_set_two_body_epsilon": ([_P, C.c_float], C.c_int),
    "hignn_nbl_set_three_body_epsilon": ([_P, C.c_float], C.c_int),
    "hignn_nbl_build_two_body_info": ([_P], C.c_int),
    "hignn_nbl_build_three_body_info": ([_P], C.c_int),
    "hignn_nbl_get_edge_info": ([_P, C.c_int, C.c_int, _u64p, C.c_int64, _u64p, C.c_int64, _i64p], C.c_int),
    "hignn_nbl_edge_info_device": ([_P, C.c_int, C.POINTER(C.c_void_p), _i64p], C.c_int),
    "hignn_nbl_last_build_ms": ([_P, _dp], C.c_int),
    "hignn_nbl_get_stream": ([_P, C.POINTER(C.c_void_p)], C.c_int),
    "hignn_tb_create": ([C.c_int, C.POINTER(_P)], C.c_int),
    "hignn_tb_destroy": ([_P], None),
    "hignn_tb_load": ([_P, C.c_int, C.c_char_p], C.c_int),
    "hignn_tb_load_mem": ([_P, C.c_int, C.c_int, C.POINTER(C.c_int32), _fp], C.c_int),
    "hignn_tb_set_epsilon": ([_P, C.c_float], C.c_int),
    "hignn_tb_velocity": ([_P, _fp, _fp, _fp, C.c_int64], C.c_int),
    "hignn_tb_velocity_edges": ([_P, _fp, _fp, _fp, C.c_int64, _u64p, C.c_int64, _u64p, C.c_int64], C.c_int),
    "hignn_tb_stats": ([_P, _dp, _dp, _dp, _i64p, _i64p], C.c_int),
    "hignn_tb_wait_profile": ([_P, C.POINTER(C.c_uint64)], C.c_int),
    "hignn_near_wait_profile": ([_P, C.POINTER(C.c_uint64)], C.c_int),
    "hignn_loop_profile": ([_P, _dp], C.c_int),
}

for _name, (_args, _res) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res


class ForceModel(C.Structure):
    """hignn_force_model: body force, Morse pair forces, filament bending and tension."""

    _fields_ = [
        ("gravity", C.c_float * 3),
        ("morse_De", C.c_double),
        ("morse_a", C.c_double),
        ("morse_re", C.c_double),
        ("morse_cutoff", C.c_double),
        ("n_filament", C.c_int64),
        ("n_chain", C.c_int32),
        ("rest_length", C.c_double),
        ("k_t", C.c_double),
        ("k_b", C.c_double),
    ]


def force_model(gravity=(0.0, 0.0, 0.0), De=1.0, a=1.0, re=2.5, cutoff=0.0, n_filament=0, n_chain=0,
                rest_length=0.0, k_t=0.0, k_b=0.0):
    fm = ForceModel()
    fm.gravity[:] = [float(v) for v in gravity]
    fm.morse_De, fm.morse_a, fm.morse_re, fm.morse_cutoff = float(De), float(a), float(re), float(cutoff)
    fm.n_filament, fm.n_chain = int(n_filament), int(n_chain)
    fm.rest_length, fm.k_t, fm.k_b = float(rest_length), float(k_t), float(k_b)
    return fm


class HignnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib.hignn_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != 0:
        raise HignnError(status, last_error())


def _f32(a, shape=None, writable=False):
    if writable:
        if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous and a.flags.writeable):
            raise TypeError("output must be a writable C-contiguous float32 array")
        arr = a
    else:
        arr = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and arr.shape != shape:
        raise ValueError(f"expected shape {shape}, got {arr.shape}")
    return arr


def fptr(a):
    return a.ctypes.data_as(_fp)


class Model:
    """Thin owner of a ``hignn_model*`` (one device, one stream)."""

    def __init__(self, xyz, block_size=128, device=0):
        x = _f32(xyz)
        if x.ndim != 2 or x.shape[1] != 3:
            raise ValueError("coordinates must have shape (n, 3)")
        self.n = x.shape[0]
        self._h = _P()
        check(lib.hignn_create(fptr(x), self.n, int(block_size), int(device), C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None):
            lib.hignn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_two_body(self, path):
        check(lib.hignn_load_two_body(self._h, os.fsencode(path)))

    def set(self, key, value):
        check(lib.hignn_set_param(self._h, int(key), float(value)))

    def get(self, key):
        v = C.c_double()
        check(lib.hignn_get_param(self._h, int(key), C.byref(v)))
        return v.value

    def update_coord(self, xyz):
        x = _f32(xyz, (self.n, 3))
        check(lib.hignn_update_coord(self._h, fptr(x), self.n))

    def dot(self, f, u=None):
        f = _f32(f, (self.n, 3))
        if u is None:
            u = np.empty((self.n, 3), np.float32)
        _f32(u, (self.n, 3), writable=True)
        check(lib.hignn_dot(self._h, fptr(u), fptr(f), self.n))
        return u

    def dot_ptr(self, u_ptr, f_ptr):
        """Host pointers (e.g. pinned buffers) of (n, 3) float32 arrays."""
        check(lib.hignn_dot(self._h, C.cast(u_ptr, _fp), C.cast(f_ptr, _fp), self.n))

    def dot_device(self, d_u_ptr, d_f_ptr):
        check(lib.hignn_dot_device(self._h, C.c_void_p(d_u_ptr), C.c_void_p(d_f_ptr), self.n))

    def dense_dot(self, f):
        f = _f32(f, (self.n, 3))
        u = np.empty((self.n, 3), np.float32)
        check(lib.hignn_dense_dot(self._h, fptr(u), fptr(f), self.n))
        return u

    def dense_rows(self, f, rows, precision=0):
        f = _f32(f, (self.n, 3))
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.empty((rows.shape[0], 3), np.float64)
        check(lib.hignn_dense_rows(self._h, out.ctypes.data_as(_dp), fptr(f), rows.ctypes.data_as(_i64p),
                                   rows.shape[0], int(precision)))
        return out

    def dense_rows_noalloc(self, f, rows, precision=0):
        """hignn_dense_rows without device allocation (scratch in a static device array)."""
        f = _f32(f, (self.n, 3))
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.empty((rows.shape[0], 3), np.float64)
        check(lib.hignn_dense_rows_noalloc(self._h, out.ctypes.data_as(_dp), fptr(f), rows.ctypes.data_as(_i64p),
                                           rows.shape[0], int(precision)))
        return out

    def two_body_eval(self, d_r_ptr, d_y_ptr, n, precision=0):
        check(lib.hignn_two_body_eval(self._h, C.c_void_p(d_r_ptr), C.c_void_p(d_y_ptr), int(n), int(precision)))

    def stats(self):
        s = HignnStats()
        check(lib.hignn_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def tree(self):
        s = self.stats()
        t = np.empty((s["num_nodes"], 5), np.int64)
        p = np.empty(self.n, np.int64)
        check(lib.hignn_get_tree(self._h, t.ctypes.data_as(_i64p), p.ctypes.data_as(_i64p)))
        return t, p

    def lists(self):
        s = self.stats()
        ci = np.empty(s["num_close"], np.int64)
        cj = np.empty(s["num_close"], np.int64)
        fi = np.empty(s["num_far"], np.int64)
        fj = np.empty(s["num_far"], np.int64)
        check(lib.hignn_get_lists(self._h, ci.ctypes.data_as(_i64p), cj.ctypes.data_as(_i64p),
                                  fi.ctypes.data_as(_i64p), fj.ctypes.data_as(_i64p)))
        return ci, cj, fi, fj

    def update_coord_keep_tree(self, x):
        """New positions on the existing cluster tree (lists and ACA plan kept)."""
        x = np.ascontiguousarray(x, np.float32)
        check(lib.hignn_update_coord_keep_tree(self._h, fptr(x), len(x)))

    def pair_forces(self, x, gravity=(0.0, 0.0, 0.0), De=1.0, a=1.0, re=2.5, cutoff=0.0):
        """gravity + Morse pair forces of positions x (n, 3) on the device."""
        x = np.ascontiguousarray(x, np.float32)
        f = np.empty_like(x)
        g = np.ascontiguousarray(gravity, np.float32)
        check(lib.hignn_pair_forces(self._h, fptr(x), fptr(f), len(x), fptr(g), float(De), float(a), float(re),
                                    float(cutoff)))
        return f

    def forces(self, x, **model):
        """Forces of force_model(**model) at positions x (n, 3), on the device."""
        x = np.ascontiguousarray(x, np.float32)
        f = np.empty_like(x)
        fm = force_model(**model)
        check(lib.hignn_forces(self._h, fptr(x), fptr(f), len(x), C.addressof(fm)))
        return f

    def run_euler(self, x, steps, dt, rebuild_every=1, gravity=(0.0, 0.0, -1.0), **model):
        """Explicit Euler on the device with the forces of force_model(gravity, **model); returns the final positions."""
        x = np.array(x, np.float32, copy=True)
        fm = force_model(gravity=gravity, **model)
        check(lib.hignn_run_euler(self._h, fptr(x), len(x), int(steps), float(dt), int(rebuild_every),
                                  C.addressof(fm)))
        return x

    def run_rk2(self, x, steps, dt, rebuild_every=1, gravity=(0.0, 0.0, -1.0), **model):
        """Explicit midpoint rule on the device with the forces of force_model(gravity, **model)."""
        x = np.array(x, np.float32, copy=True)
        fm = force_model(gravity=gravity, **model)
        check(lib.hignn_run_rk2(self._h, fptr(x), len(x), int(steps), float(dt), int(rebuild_every),
                                C.addressof(fm)))
        return x

    def run_dp45(self, x, tf, dt0, threshold=1e-3, rebuild_every=0, gravity=(0.0, 0.0, -1.0), **model):
        """Adaptive Dormand-Prince on the device (the reference's ExplicitRk4); returns (positions, steps)."""
        x = np.array(x, np.float32, copy=True)
        fm = force_model(gravity=gravity, **model)
        steps = C.c_int64()
        check(lib.hignn_run_dp45(self._h, fptr(x), len(x), float(tf), float(dt0), float(threshold),
                                 int(rebuild_every), C.addressof(fm), C.byref(steps)))
        return x, steps.value

    def set_three_body(self, tb):
        """Add the three-body and self terms of `tb` (a ThreeBody, or None) to the device time loops."""
        check(lib.hignn_set_three_body(self._h, tb._h if tb is not None else None))
        self._tb = tb  # keep it alive while attached

    def set_shard(self, rank, world):
        """Compute only shard `rank` of `world` of the block lists; dot then returns partial velocities."""
        check(lib.hignn_set_shard(self._h, int(rank), int(world)))

    def shard(self):
        """(close begin, close end, far begin, far end) of this model's shard, in list order."""
        r = np.empty(4, np.int64)
        check(lib.hignn_get_shard(self._h, r.ctypes.data_as(_i64p)))
        return tuple(int(v) for v in r)

    # ---- far-field student network
    def train_student(self, steps=20000, batch=65536, nsamples=10_000_000, lr=1e-3, seed=1):
        loss = C.c_double()
        check(lib.hignn_train_student(self._h, int(steps), int(batch), int(nsamples), float(lr), int(seed),
                                      C.byref(loss)))
        return loss.value

    def set_student(self, params):
        p = np.ascontiguousarray(params, np.float32)
        check(lib.hignn_set_student(self._h, fptr(p), p.size))

    def loop_profile(self):
        """Phases of the last hignn_run_euler / hignn_run_rk2 call (milliseconds and counts)."""
        v = np.zeros(8, np.float64)
        check(lib.hignn_loop_profile(self._h, v.ctypes.data_as(_dp)))
        keys = ("wall_ms", "rebuild_ms", "forces_ms", "matvec_ms", "three_body_ms", "steps", "evaluations",
                "eager_matvecs")
        return {k: float(x) for k, x in zip(keys, v)}

    def near_wait_profile(self):
        """Wait cycles of the tensor-core near field by barrier (HIGNN_P_TIMING >= 3), then reset."""
        c = (C.c_uint64 * 16)()
        check(lib.hignn_near_wait_profile(self._h, c))
        names = {0: "mma_first_features", 1: "mma_a1", 2: "mma_q0_in_a2", 3: "mma_d3_free", 4: "mma_q1_in_a2",
                 5: "mma_q2_in_a2", 6: "mma_next_features", 7: "mma_q3_in_a2", 8: "epi_layer1_acc",
                 9: "epi_layer2_acc", 10: "epi_layer3_acc", 11: "epi_a2_free", 12: "epi_total_warp0", 13: "tiles"}
        return {names[i]: int(c[i]) for i in names}

    def get_student(self):
        p = np.empty(STUDENT_PARAMS, np.float32)
        check(lib.hignn_get_student(self._h, fptr(p), p.size))
        return p

    def student_eval(self, d_r_ptr, d_y_ptr, n):
        check(lib.hignn_student_eval(self._h, C.c_void_p(d_r_ptr), C.c_void_p(d_y_ptr), int(n)))

    def student_grad(self, d_r_ptr, d_t_ptr, n):
        g = np.empty(STUDENT_PARAMS, np.float32)
        loss = C.c_double()
        check(lib.hignn_student_grad(self._h, C.c_void_p(d_r_ptr), C.c_void_p(d_t_ptr), int(n), fptr(g),
                                     C.byref(loss)))
        return g, loss.value

    def far_pivots(self):
        """(ranks, rows, cols) of the last far field; rows/cols are per-block lists."""
        nf = self.stats()["num_far"]
        ld = int(self.get(P_MAX_ITER)) + 1
        rk = np.empty(nf, np.int32)
        rows = np.empty((nf, ld), np.int32)
        cols = np.empty((nf, ld), np.int32)
        i32 = C.POINTER(C.c_int32)
        check(lib.hignn_get_far_pivots(self._h, rk.ctypes.data_as(i32), rows.ctypes.data_as(i32),
                                       cols.ctypes.data_as(i32), ld))
        return rk, [list(rows[b, :rk[b]]) for b in range(nf)], [list(cols[b, :rk[b] + 1]) for b in range(nf)]

    def synchronize(self):
        check(lib.hignn_synchronize(self._h))

    def stream(self):
        s = C.c_void_p()
        check(lib.hignn_get_stream(self._h, C.byref(s)))
        return s.value


class NeighborLists:
    """Owner of a ``hignn_nbl*``: the reference's NeighborLists (include/NeighborLists.hpp) on one device.

    Getters return uint64 arrays of shape (rows, E), as the reference's do.
    """

    def __init__(self, device=0):
        h = _P()
        check(lib.hignn_nbl_create(int(device), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.hignn_nbl_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def update_coord(self, x):
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 2 or x.shape[1] != 3:
            raise ValueError("coordinates must be (n, 3)")
        check(lib.hignn_nbl_update_coord(self._h, fptr(x), len(x)))

    def set_two_body_epsilon(self, eps):
        check(lib.hignn_nbl_set_two_body_epsilon(self._h, float(eps)))

    def set_three_body_epsilon(self, eps):
        check(lib.hignn_nbl_set_three_body_epsilon(self._h, float(eps)))

    def build_two_body_info(self):
        check(lib.hignn_nbl_build_two_body_info(self._h))

    def build_three_body_info(self):
        check(lib.hignn_nbl_build_three_body_info(self._h))

    def last_build_ms(self):
        v = C.c_double()
        check(lib.hignn_nbl_last_build_ms(self._h, C.byref(v)))
        return v.value

    def edges(self, kind, index=None):
        """(rows, E) uint64 edge list of `kind` (EDGES_*), or its ByIndex variant for `index`."""
        rows = 3 if kind == EDGES_THREE_BODY else 2
        by = index is not None
        idx = np.ascontiguousarray(index if by else np.zeros(0), np.uint64)
        ip = idx.ctypes.data_as(_u64p)
        e = C.c_int64()
        check(lib.hignn_nbl_get_edge_info(self._h, kind, int(by), ip, len(idx), None, 0, C.byref(e)))
        out = np.empty((rows, e.value), np.uint64)
        check(lib.hignn_nbl_get_edge_info(self._h, kind, int(by), ip, len(idx), out.ctypes.data_as(_u64p), out.size,
                                          C.byref(e)))
        return out

    def device_edges(self, kind):
        """(device pointer, E) of a whole list; the pointer is owned by this object."""
        p, e = C.c_void_p(), C.c_int64()
        check(lib.hignn_nbl_edge_info_device(self._h, kind, C.byref(p), C.byref(e)))
        return p.value, e.value


TB_THREE_BODY = 0
TB_SELF = 1


class ThreeBody:
    """Owner of a ``hignn_tb*``: the three-body and self terms of the reference's HIGNN model
    (python/HIGNN/model_structure.py:76-139) on one device."""

    def __init__(self, device=0, three_body_path=None, self_path=None, epsilon=5.0):
        from .weights import default_three_body_paths

        h = _P()
        check(lib.hignn_tb_create(int(device), C.byref(h)))
        self._h = h
        d3, ds = default_three_body_paths()
        check(lib.hignn_tb_load(self._h, TB_THREE_BODY, (three_body_path or d3).encode()))
        check(lib.hignn_tb_load(self._h, TB_SELF, (self_path or ds).encode()))
        self.set_epsilon(epsilon)

    def close(self):
        if getattr(self, "_h", None):
            lib.hignn_tb_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_epsilon(self, eps):
        check(lib.hignn_tb_set_epsilon(self._h, float(eps)))

    def velocity(self, x, f):
        x = _f32(x)
        f = _f32(f, x.shape)
        u = np.empty_like(x)
        check(lib.hignn_tb_velocity(self._h, fptr(x), fptr(f), fptr(u), len(x)))
        return u

    def velocity_edges(self, x, f, tri, self_edges):
        """The same two terms on caller-given edge lists: tri (3, E3) and self_edges (2, Es), the
        rows of NeighborLists.get_three_body_edge_info / get_three_body_edge_self_info."""
        x = _f32(x)
        f = _f32(f, x.shape)
        tri = np.ascontiguousarray(tri, np.uint64).reshape(3, -1)
        se = np.ascontiguousarray(self_edges, np.uint64).reshape(2, -1)
        u = np.empty_like(x)
        check(lib.hignn_tb_velocity_edges(self._h, fptr(x), fptr(f), fptr(u), len(x), tri.ctypes.data_as(_u64p),
                                          tri.shape[1], se.ctypes.data_as(_u64p), se.shape[1]))
        return u

    def stats(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        t, p = C.c_int64(), C.c_int64()
        check(lib.hignn_tb_stats(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(t), C.byref(p)))
        return dict(ms_lists=a.value, ms_three=b.value, ms_self=c.value, triplets=t.value, pairs=p.value)

    def wait_profile(self):
        """Clocks the three-body (then self) kernel's MMA lane waited for act1, weight stages, layer-2
        epilogues, the layer-3 accumulator; its total; the producer's waits for free slots."""
        c = (C.c_uint64 * 12)()
        check(lib.hignn_tb_wait_profile(self._h, c))
        keys = ["wait_act1", "wait_stage", "wait_epilogue", "wait_d3", "total", "producer_wait"]
        return {"three_body": dict(zip(keys, c[:6])), "self": dict(zip(keys, c[6:]))}
