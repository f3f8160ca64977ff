"""Kernel-level timings of the native library (CUDA events), for tuning and profiler captures.

    python -m hignn_b200.microbench eval --n 378880 --precision 1
    python -m hignn_b200.microbench dot --workload medium --precision 1 --fields 1
    python -m hignn_b200.microbench three_body --filaments 4096

`three_body` times the three-body + self near field on filaments of 32 beads 2.2 apart at volume
fraction 0.05 (seed 3) with three-body cutoff 5, against the measured bf16 tensor peak.

Prints one JSON line: milliseconds per call and evaluations per second.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
WEIGHTS = os.path.join(HERE, "data", "two_body_unbounded.hgnw")
FLOP_PER_EVAL = 2 * (3 * 128 + 128 * 512 + 512 * 9)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["eval", "dot", "three_body"])
    ap.add_argument("--filaments", type=int, default=4096)
    ap.add_argument("--n", type=int, default=148 * 128 * 20)
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--workload", default="medium", choices=["small", "medium", "large", "uniform1m", "uniform4m"])
    ap.add_argument("--fields", type=int, default=3)
    ap.add_argument("--epsilon", type=float, default=1e-2)
    ap.add_argument("--timing", type=int, default=2,
                    help="2 = far-field breakdown by kernel category, 3 = also the near-field wait profile")
    ap.add_argument("--pool-mb", type=int, default=0, help="ACA pool memory per batch (0: the default)")
    ap.add_argument("--student-steps", type=int, default=4000, help="training steps when --precision 2")
    ap.add_argument("--student-batch", type=int, default=16384)
    ap.add_argument("--student-samples", type=int, default=2_000_000)
    ap.add_argument("--student-tol", type=float, nargs="*", default=[1e-3],
                    help="sampled-residual tolerances to time (precision 2)")
    a = ap.parse_args()

    import torch

    from hignn_b200 import capi
    from hignn_b200 import synthetic as S

    out = {"what": a.what, "precision": a.precision}
    if a.what == "three_body":
        out.update(three_body(a))
    elif a.what == "eval":
        rng = np.random.default_rng(1)
        v = rng.normal(size=(a.n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        r = (v * np.exp(rng.uniform(np.log(2.0), np.log(300.0), a.n))[:, None]).astype(np.float32)
        m = capi.Model(rng.uniform(0, 50, (256, 3)), 128, device=0)
        m.load_two_body(WEIGHTS)
        rt = torch.from_numpy(r).cuda()
        y = torch.empty((a.n, 9), device="cuda")
        stream = torch.cuda.ExternalStream(m.stream())
        m.two_body_eval(rt.data_ptr(), y.data_ptr(), a.n, a.precision)
        ts = []
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            m.two_body_eval(rt.data_ptr(), y.data_ptr(), a.n, a.precision)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.min(ts))
        out.update(n=a.n, ms=ms, evals_per_s=a.n / ms * 1e3, tflops=a.n * FLOP_PER_EVAL / ms / 1e9)
    else:
        if a.workload == "uniform1m":
            x, f = S.uniform(1048576, 0.1, 2), S.sedimenting_forces(1048576, 2)
        elif a.workload == "uniform4m":
            # the learned-far-field workload: 4,194,304 spheres uniform at volume fraction 0.10, seed 4
            x, f = S.uniform(4194304, 0.1, 4), S.sedimenting_forces(4194304, 4)
        elif a.workload == "large":
            x, f = S.clustered(1048576, 0.10, 2), S.sedimenting_forces(1048576, 2)
        else:
            x, f, _ = S.workload(a.workload)
        m = capi.Model(x, 128, device=0)
        m.load_two_body(WEIGHTS)
        m.set(capi.P_PRECISION, a.precision)
        m.set(capi.P_FIELDS, a.fields)
        m.set(capi.P_EPSILON, a.epsilon)
        m.set(capi.P_TIMING, a.timing)
        if a.pool_mb:
            m.set(capi.P_FAR_POOL_MB, a.pool_mb)
        if a.precision == 2:
            import time

            t0 = time.time()
            out["student_loss"] = m.train_student(steps=a.student_steps, batch=a.student_batch,
                                                  nsamples=a.student_samples, lr=1e-3, seed=3)
            out["student_train_s"] = time.time() - t0
            out["per_tol"] = {}
            for tol in a.student_tol:
                m.set(capi.P_STUDENT_TOL, tol)
                m.dot(f)
                m.dot(f)
                st = m.stats()
                out["per_tol"][str(tol)] = {"far_ms": st["t_far_ms"], "fallback_blocks": st["student_fallback_blocks"],
                                            "num_far": st["num_far"], "far_iterations": st["far_iterations"]}
            m.set(capi.P_STUDENT_TOL, a.student_tol[-1])
        m.dot(f)
        first = m.stats()
        if a.timing >= 3:
            m.near_wait_profile()  # reset: the profile below covers the timed repetitions only
        near, far = [], []
        for _ in range(a.reps):
            m.dot(f)
            st = m.stats()
            near.append(st["t_close_ms"])
            far.append(st["t_far_ms"])
        st = m.stats()
        if a.timing >= 3 and a.precision >= 1:
            out["near_wait_profile"] = m.near_wait_profile()
        out["first_far_ms"] = first["t_far_ms"]
        out["first_far_iterations"] = first["far_iterations"]
        out.update(workload=a.workload, n=len(x), near_ms=float(np.min(near)), far_ms=float(np.min(far)),
                   close_evals=st["close_evals"], far_evals=st["far_evals"],
                   near_evals_per_s=st["close_evals"] / max(1e-9, np.min(near)) * 1e3,
                   near_tflops=st["close_evals"] * FLOP_PER_EVAL / max(1e-9, np.min(near)) / 1e9,
                   far_evals_per_s=st["far_evals"] / max(1e-9, np.min(far)) * 1e3 if st["far_evals"] else None,
                   far_iterations=st["far_iterations"], far_rank_max=st["far_rank_max"],
                   student_fallback_blocks=st["student_fallback_blocks"], gpu_launches=st["gpu_launches"],
                   num_far=st["num_far"], far_query_ms=st["t_far_query_ms"], far_pivot_ms=st["t_far_pivot_ms"],
                   far_active_ms=st["t_far_active_ms"], far_check_ms=st["t_far_check_ms"])
    print(json.dumps(out), flush=True)


TB_FLOP = 2 * (6 * 256 + 256 * 1024 + 1024 * 512 + 512 * 9)    # per triplet
TB_SELF_FLOP = 2 * (3 * 256 + 256 * 1024 + 1024 * 512 + 512 * 9)


def three_body(a, reps=None):
    import time

    from hignn_b200 import capi
    from hignn_b200 import synthetic as S
    x = S.filaments(a.filaments, 32, 2.2, 0.05, 3)
    f = S.sedimenting_forces(len(x), 3)
    tb = capi.ThreeBody(0)
    tb.set_epsilon(5.0)
    for _ in range(3):
        tb.velocity(x, f)
    runs = []
    for _ in range(max(1, reps or a.reps)):
        t0 = time.perf_counter()
        tb.velocity(x, f)
        st = tb.stats()
        st["wall_ms"] = (time.perf_counter() - t0) * 1e3
        runs.append(st)
    best = min(runs, key=lambda r: r["ms_three"] + r["ms_self"])
    flop = best["triplets"] * TB_FLOP + best["pairs"] * TB_SELF_FLOP
    kernel_ms = best["ms_three"] + best["ms_self"]
    peaks = {}
    pk = os.path.join(os.path.dirname(HERE), "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = peaks.get("bf16_tflops", 1590.0)
    tflops = best["triplets"] * TB_FLOP / best["ms_three"] / 1e9
    out = dict(n=len(x), triplets=best["triplets"], pairs=best["pairs"], ms_lists=best["ms_lists"],
               ms_three=best["ms_three"], ms_self=best["ms_self"], e2e_ms=best["wall_ms"],
               edges_per_s=(best["triplets"] + best["pairs"]) / kernel_ms * 1e3,
               roofline={"bound": "tensor", "kernel": "k_three_body<0>", "achieved": tflops, "peak": peak,
                         "unit": "TFLOP/s", "frac": tflops / peak,
                         "peak_source": "measured" if peaks else "fallback"},
               total_tflops=flop / kernel_ms / 1e9, wait_profile=tb.wait_profile())
    out["triplets_per_s"] = best["triplets"] / best["ms_three"] * 1e3
    return out


if __name__ == "__main__":
    main()
