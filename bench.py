#!/usr/bin/env python
"""H-matvec benchmark: particles/s of U = M(x) F at N = 1,048,576 on B200s.

Workload (seeded, synthetic; no dataset): 1,048,576 unit spheres in a cube at
volume fraction 0.10, 64 Gaussian clusters (sigma 8 radii) + 50% uniform
background (seed 2), forces (0,0,-1) + N(0, 0.1^2); leaf size 128, ACA
tolerance 1e-2 (the reference's production value, python/simulate.py:198),
max_iter 100, tree prebuilt (its host build time is reported apart). One step =
one H-matvec (near field + ACA far field). The headline form is FP16 tensor
cores (FP32 layer 1 and accumulation) + rank-planned ACA batches + the far-field student network (trained on
the device before timing; its training time is reported apart); the plain FP32
form is timed in the same run for the mixed-vs-plain ratio of the metric, and
both are checked against the dense product on sampled target rows.

With N GPUs (torchrun, one rank per GPU) every rank builds the same tree and
computes a cost-balanced shard of the close and far block lists; the partial
velocities are summed by one NCCL all-reduce per step, inside the timed region
(strong scaling: the same N=1M product on every GPU count).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision P]
    python bench.py --impl reference ...   # the reference algorithm on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
WEIGHTS = os.path.join(REPO, "hignn_b200", "data", "two_body_unbounded.hgnw")
METRIC = "H-matvec particles/s at N=1M: mixed+batched+student vs plain FP32, err≤1e-3"
FLOP_PER_EVAL = 2 * (3 * 128 + 128 * 512 + 512 * 9)  # 141,056
TANH_PER_EVAL = 128 + 512
# DRAM bytes of one k_near_tc launch in the committed full ncu capture (N = 131,072: 8.9 MB read,
# nothing written; positions, forces and the pair list are read once, the FP64 accumulators stay
# in L2). The reads are per particle, so the figure scales with N.
NEAR_DRAM_BYTES_PER_PARTICLE = 8.9e6 / 131072
PREC_NAME = {0: "plain_fp32", 1: "fp16_tensor_cores", 2: "fp16_tensor_cores+student_far_field"}
PREC_DTYPE = {0: "fp32", 1: "fp16", 2: "fp16"}  # layers 2-3 on the tensor cores in FP16 (FP32 accumulation)
_T0 = time.time()


def note(msg):
    """Progress of a run on stderr (stdout carries only the result line)."""
    print(f"[bench {time.time() - _T0:8.1f} s] {msg}", file=sys.stderr, flush=True)


WORKLOAD = ("N=1,048,576 clustered (64 Gaussian clusters sigma 8 + 50% uniform), phi 0.10, seed 2, "
            "leaf 128, eps 1e-2, max_iter 100, tree prebuilt")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hignn_b200", choices=["hignn_b200", "reference"])
    ap.add_argument("--precision", type=int, default=2, choices=[0, 1, 2])
    ap.add_argument("--student-steps", type=int, default=20000)
    ap.add_argument("--student-batch", type=int, default=65536)
    ap.add_argument("--student-samples", type=int, default=10_000_000)
    ap.add_argument("--n", type=int, default=1048576)
    ap.add_argument("--epsilon", type=float, default=1e-2)
    ap.add_argument("--check-rows", type=int, default=16384,
                    help="seeded target rows of the FP64 dense error check (all N sources each)")
    ap.add_argument("--no-unplanned", action="store_true",
                    help="skip the matvec on a freshly built tree (no recorded ACA ranks)")
    ap.add_argument("--no-plain", action="store_true", help="do not time the plain FP32 form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing")
    ap.add_argument("--cpu-sample-seconds", type=float, default=6.0,
                    help="CPU work of one sample step of the CPU baseline / reference arm")
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the time loops and the three-body near field added to the line")
    ap.add_argument("--euler-steps", type=int, default=100, help="steps of the 1M Euler loop (next_rows)")
    ap.add_argument("--filament-steps", type=int, default=200, help="RK2 steps of the filament loop (next_rows)")
    return ap.parse_args()


def filament_steps(steps=200):
    """The filament suspension (4,096 filaments x 32 beads, bond 2.2, phi 0.05, seed 3) stepped on the
    device with the whole HIGNN velocity: filament bending (k_b 10) and tension (k 100) plus
    gravity, H-matrix two-body term (tensor-core network, eps 1e-2, leaf 128), three-body and self terms
    (cutoff 5); explicit midpoint rule (RK2), dt 5e-4, tree rebuilt every 2 steps."""
    from hignn_b200 import capi
    from hignn_b200 import synthetic as S
    from hignn_b200.weights import default_two_body_path

    x = S.filaments(4096, 32, 2.2, 0.05, 3)
    tb = capi.ThreeBody(0, epsilon=5.0)
    m = capi.Model(x, 128, device=0)
    m.load_two_body(default_two_body_path())
    m.set(capi.P_PRECISION, 1)
    m.set(capi.P_EPSILON, 1e-2)
    m.set_three_body(tb)
    model = dict(gravity=(0.0, 0.0, -1.0), n_filament=4096, n_chain=32, rest_length=2.2, k_t=100.0, k_b=10.0)
    m.run_rk2(x, 2, 5e-4, rebuild_every=2, **model)  # warm-up: module loading, allocations
    t0 = time.perf_counter()
    x1 = m.run_rk2(x, steps, 5e-4, rebuild_every=2, **model)
    dt = time.perf_counter() - t0
    prof = m.loop_profile()
    m.set_three_body(None)
    m.close()
    tb.close()
    return {"workload": "4,096 filaments x 32 beads, RK2 (explicit midpoint), dt 5e-4, tree rebuilt every 2 steps",
            "integrator": "explicit midpoint (hignn_run_rk2)", "steps": steps, "ms_per_step": dt / steps * 1e3,
            "particle_steps_per_s": len(x) * steps / dt, "final_positions_finite": bool(np.isfinite(x1).all()),
            "phases_ms": prof,
            "note": "wall clock of the whole call from host positions, tree rebuilds included; phases from "
                    "hignn_loop_profile (device time of forces, matvecs, three-body terms; rebuilds by wall clock)"}


def three_body_row(args):
    """The three-body + self near field (131,072 filament beads, cutoff 5) on this GPU, with the
    three-body network on torch's CPU FP32 path over a bounded sample of triplets as its CPU
    baseline."""
    import time
    from types import SimpleNamespace

    from hignn_b200.microbench import three_body
    from hignn_b200.weights import default_three_body_paths
    from oracle import hignn_oracle as O

    import torch

    row = three_body(SimpleNamespace(filaments=4096, reps=3))
    note("three-body kernel timed")
    # the reference runs this network in torch (python/HIGNN/model_structure.py:41-55): its CPU
    # FP32 path on the oracle's weights, batches of 8,192 triplets
    net = O.DenseTanh.from_hgnw(default_three_body_paths()[0])
    layers = [(torch.from_numpy(w.astype(np.float32)), torch.from_numpy(b.astype(np.float32)))
              for w, b in zip(net.w64, net.b64)]
    torch.set_num_threads(os.cpu_count() or 1)
    sample = 65536
    z = torch.from_numpy(np.random.default_rng(0).normal(0, 3, (sample, 6)).astype(np.float32))

    def forward(h):
        for i, (w, b) in enumerate(layers):
            h = torch.addmm(b, h, w.T)
            if i + 1 < len(layers):
                h = torch.tanh(h)
        return h

    with torch.no_grad():
        forward(z[:8192])  # warm-up: thread pool and allocator
    t0 = time.perf_counter()
    with torch.no_grad():
        for s in range(0, sample, 8192):
            forward(z[s:s + 8192])
    dt = time.perf_counter() - t0
    row["workload"] = "4,096 filaments x 32 beads, bond 2.2, phi 0.05, seed 3, three-body cutoff 5"
    note("three-body CPU baseline timed")
    row["time_step"] = filament_steps(args.filament_steps)
    note("filament loop done")
    row["cpu_baseline"] = {"value": sample / dt, "unit": "triplets/s", "cores": os.cpu_count(), "kind": "port",
                           "sample": f"{sample} triplets through the three-body network on torch's CPU FP32 path "
                                     f"(the reference's engine), {os.cpu_count()} threads"}
    return row


def workload(n):
    from hignn_b200 import synthetic as S

    return S.clustered(n, 0.10, 2), S.sedimenting_forces(n, 2)


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if bus_id:
            cmd += ["-i", bus_id]
        try:
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [[s.strip() for s in line.split(",")] for line in open(self.f.name)]
        rows = [r for r in rows if len(r) >= 9]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}

        def num(s):
            try:
                return float(s)
            except ValueError:
                return float("nan")

        sm = [num(r[1]) for r in rows]
        mx = max(num(r[2]) for r in rows)
        pw = [num(r[3]) for r in rows]
        load = [i for i in range(len(rows)) if pw[i] > 250 or sm[i] > 0.5 * mx] or list(range(len(rows)))
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for i in load for k in range(4) if rows[i][5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm[i] for i in load), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "samples_under_load": len(load), "power_w_max": max(pw)}


class CpuSample:
    """The CPU baseline: the C++/OpenMP restatement of the reference path (oracle/hmatvec_cpu.cpp:
    CloseDot and ACA FarDot, FP32 network, FP64 accumulation and bookkeeping) on all host threads,
    timed on a bounded, fixed sample of one H-matvec: the leading close pairs worth about
    seconds / 2 of CPU work and the leading ACA blocks worth the other half (chosen once, by a
    first timed pass). Every step runs exactly that sample; its evaluations per second are
    extrapolated to the counted evaluations of the whole H-matvec (far evaluations from the
    sampled mean rank when not given)."""

    def __init__(self, x, f, eps, seconds, close_evals=None, far_evals=None):
        from oracle import hignn_oracle as O

        self.O = O
        self.cores = os.cpu_count() or 1
        net = O.TwoBodyF32Exact.from_hgnw(WEIGHTS)
        self.eps = eps
        self.n = len(x)
        t0 = time.time()
        tree, rmap = O.build_tree(x, 128)
        xt = x[rmap]
        aux = O.compute_aux(tree, xt)
        self.ci, self.cj, self.fi, self.fj, _ = O.close_far_lists(tree, aux)
        self.t_lists = time.time() - t0
        self.ft = f[rmap]
        self.cpu = O.CpuHMatvec(tree, xt, net, threads=self.cores)
        sz = tree[:, 3] - tree[:, 2]
        self.close_evals = int(np.sum(sz[self.ci] * sz[self.cj])) if close_evals is None else close_evals
        # choose the sample: leading pairs / blocks until each half of the budget is used
        p, t_near = 0, 0.0
        while t_near < seconds / 2 and p < len(self.ci):
            q = min(len(self.ci), p + 256)
            t = time.time()
            self.cpu.close_dot(self.ft, self.ci, self.cj, p, q)
            t_near += time.time() - t
            p = q
        b, t_far, ranks = 0, 0.0, []
        while t_far < seconds / 2 and b < len(self.fi):
            q = min(len(self.fi), b + 256)
            t = time.time()
            _, rk, _ = self.cpu.far_dot(self.ft, self.fi, self.fj, eps, 100, b, q)
            t_far += time.time() - t
            ranks += rk.tolist()
            b = q
        self.p, self.b = p, b
        self.near_sample = int(np.sum(sz[self.ci[:p]] * sz[self.cj[:p]]))
        if far_evals is None:
            far_evals = float(np.mean(ranks)) * float(np.sum(sz[self.fi] + sz[self.fj])) if ranks else 0.0
        self.far_evals = far_evals

    def step(self):
        """One timed sample step: (seconds, near seconds, far seconds, far evaluations of the sample)."""
        t0 = time.time()
        self.cpu.close_dot(self.ft, self.ci, self.cj, 0, self.p)
        t1 = time.time()
        _, _, far_e = self.cpu.far_dot(self.ft, self.fi, self.fj, self.eps, 100, 0, self.b)
        t2 = time.time()
        return t2 - t0, t1 - t0, t2 - t1, far_e

    def estimate(self, t_near, t_far, far_e):
        r_near = self.near_sample / t_near
        r_far = far_e / t_far if t_far > 0 else r_near
        t_dot = self.close_evals / r_near + self.far_evals / r_far
        return {"value": self.n / t_dot, "unit": "particles/s", "cores": self.cores, "kind": "port",
                "sample": (f"C++/OpenMP restatement of the reference path (oracle/hmatvec_cpu.cpp: CloseDot and ACA "
                           f"FarDot, FP32 network, FP64 accumulation) on {self.cores} host threads (nproc "
                           f"{os.cpu_count()}; the reference fixes 10); each step runs the same sample: {self.p} "
                           f"close pairs ({self.near_sample:.3g} evals, {r_near:.3g} evals/s) and {self.b} ACA blocks "
                           f"({far_e:.3g} evals, {r_far:.3g} evals/s), extrapolated to {self.close_evals:.3g} near "
                           f"+ {self.far_evals:.3g} far evaluations of one H-matvec; tree+lists "
                           f"({self.t_lists:.1f} s) not counted")}


def cpu_estimate(x, f, eps, seconds, close_evals=None, far_evals=None):
    """One timed sample step of CpuSample, extrapolated to a whole H-matvec."""
    cs = CpuSample(x, f, eps, seconds, close_evals, far_evals)
    _, tn, tf, fe = cs.step()
    return cs.estimate(tn, tf, fe)


def reference_arm(args, rank, world):
    """The reference algorithm (restated on the CPU) on the host cores: every step runs the same
    bounded sample of one H-matvec; ms_per_step is the measured time of that sample, value the
    sample's rate extrapolated to the whole H-matvec."""
    if rank != 0:
        return 0
    x, f = workload(args.n)
    cs = CpuSample(x, f, args.epsilon, args.cpu_sample_seconds)
    tot, near, far, fe = [], [], [], []
    for k in range(args.warmup + args.steps):
        t, tn, tf, e = cs.step()
        if k >= args.warmup:
            tot.append(t)
            near.append(tn)
            far.append(tf)
            fe.append(e)
    est = cs.estimate(float(np.sum(near)), float(np.sum(far)), float(np.sum(fe)))
    v = est["value"]
    frac = (cs.near_sample + float(np.mean(fe))) / (cs.close_evals + cs.far_evals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(tot)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": args.n, "epsilon": args.epsilon, "parallelism": "host cores"},
            "cpu_baseline": {"value": v, "unit": "particles/s", "cores": est["cores"], "kind": "port",
                             "sample": est["sample"]},
            "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sample": {"fraction_of_matvec_evals": frac, "seconds_per_step": float(np.mean(tot)),
                       "extrapolated_ms_per_matvec": 1e3 * args.n / v,
                       "note": "ms_per_step is the measured time of one sample step; value extrapolates the "
                               "sample's evaluations per second to the whole H-matvec"},
            "note": "the reference's Kokkos/libtorch build cannot be built here (Kokkos, Eigen, MPI absent; "
                    "not pip-installable); this arm times its C++/OpenMP restatement on the host cores"}
    print(json.dumps(line), flush=True)
    return 0


def timed(m, stream, flush, steps, fn):
    """Per-step device time (CUDA events on the model's stream), L2 flushed between steps."""
    import torch

    times, near, far = [], [], []
    for k in range(steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        s = m.stats()
        near.append(s["t_close_ms"])
        far.append(s["t_far_ms"])
    return times, near, far


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    def max_over_ranks(v):
        if not dist:
            return v
        t = torch.tensor([v], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from hignn_b200 import capi

    x, f = workload(args.n)
    n = len(x)
    m = capi.Model(x, 128, device=local)
    m.load_two_body(WEIGHTS)
    m.set(capi.P_EPSILON, args.epsilon)
    m.set(capi.P_MAX_ITER, 100)
    m.set(capi.P_TIMING, 1)
    if world > 1:
        m.set_shard(rank, world)
    st0 = m.stats()  # builds the tree and lists
    note("tree and lists built")
    student = None
    if args.precision == 2:  # the far-field student network, trained on the device from teacher samples
        t0 = time.time()
        loss = m.train_student(steps=args.student_steps, batch=args.student_batch, nsamples=args.student_samples,
                               lr=1e-3, seed=3)
        student = {"steps": args.student_steps, "batch": args.student_batch, "teacher_samples": args.student_samples,
                   "final_mse": loss, "train_seconds": time.time() - t0}
    m.set(capi.P_PRECISION, args.precision)
    f_d = torch.from_numpy(f).cuda()
    u_d = torch.empty_like(f_d)
    stream = torch.cuda.ExternalStream(m.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step_device(out):
        m.dot_device(out.data_ptr(), f_d.data_ptr())
        if dist:  # partial velocities of this rank's shard -> the whole product on every rank
            with torch.cuda.stream(stream):
                dist.all_reduce(out)

    f_h = torch.from_numpy(f).pin_memory()
    u_h = torch.empty_like(f_h).pin_memory()
    fe_d = torch.empty_like(f_d)

    def step_e2e():
        if not dist:
            m.dot_ptr(u_h.data_ptr(), f_h.data_ptr())  # the C ABI's host-pointer call (H2D, matvec, D2H)
            return
        with torch.cuda.stream(stream):  # the model's stream: copies, matvec and all-reduce in order
            fe_d.copy_(f_h, non_blocking=True)
        m.dot_device(u_d.data_ptr(), fe_d.data_ptr())
        with torch.cuda.stream(stream):
            dist.all_reduce(u_d)
            u_h.copy_(u_d, non_blocking=True)

    note("student trained" if student else "model ready")
    for _ in range(args.warmup):
        step_device(u_d)
    note("warm-up products done")
    props = torch.cuda.get_device_properties(local)
    bus = None
    try:
        bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except AttributeError:
        pass
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(bus)
    times, near_ms, far_ms = timed(m, stream, flush, args.steps, lambda: step_device(u_d))
    torch.cuda.synchronize()
    ck = clocks.stop()
    note("timed products done")
    if dist:
        dist.barrier()
    st = m.stats()
    ms = max_over_ranks(float(np.mean(times)))
    value = n / (ms / 1e3)
    # one more (untimed) matvec with CUDA events around every far-field launch: the far breakdown
    m.set(capi.P_TIMING, 2)
    step_device(u_d)
    sb = m.stats()
    m.set(capi.P_TIMING, 1)
    far_breakdown = {"queries": sb["t_far_query_ms"], "pivots_and_apply": sb["t_far_pivot_ms"],
                     "active_lists": sb["t_far_active_ms"], "student_check": sb["t_far_check_ms"],
                     "total": sb["t_far_ms"], "note": "one untimed matvec with an event around every launch"}

    # end to end through the public C ABI from pinned host memory (H2D + matvec + D2H per step)
    if args.no_e2e:
        u_h.copy_(u_d.cpu())
        e2e_ms = float("nan")
    else:
        e2e_times, _, _ = timed(m, stream, flush, args.steps, step_e2e)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(float(np.mean(e2e_times)))
    u = u_h.numpy().astype(np.float64)

    # the reference rebuilds the tree before every product (python/simulate.py:129,
    # src/HignnModel.cpp:744-762): a product on a freshly built tree has no recorded ACA ranks.
    # One such product is timed here (same positions, so the same tree), the rebuild apart.
    unplanned = None
    if not args.no_unplanned:
        m.set(capi.P_KEEP_RANKS, 0)  # the rebuild forgets the recorded ranks
        t0 = time.perf_counter()
        m.update_coord(x)
        rebuild_ms = (time.perf_counter() - t0) * 1e3
        m.set(capi.P_KEEP_RANKS, 1)
        ut, un, uf = timed(m, stream, flush, 1, lambda: step_device(u_d))
        su = m.stats()
        ums = max_over_ranks(float(ut[0]))
        unplanned = {"ms_per_step": ums, "value": n / (ums / 1e3), "near_ms": float(un[0]), "far_ms": float(uf[0]),
                     "far_iterations": su["far_iterations"], "rebuild_host_ms": rebuild_ms,
                     "note": "first H-matvec after update_coord with HIGNN_P_KEEP_RANKS 0: ACA batches without "
                             "recorded ranks, as every product of the reference's time loop; the tree rebuild is "
                             "timed apart"}
        step_device(u_d)  # ranks recorded again for the forms timed below
        note("unplanned product done")

    # accuracy: FP64 dense rows on seeded target rows, each summed over all N sources
    rng = np.random.default_rng(12345)
    rows = np.sort(rng.choice(n, size=min(args.check_rows, n), replace=False))
    err = err_plain = None
    t0 = time.time()
    ud = m.dense_rows(f, rows, capi.DENSE_F64) if len(rows) and rank == 0 else None
    t_check = time.time() - t0
    note("FP64 dense-row check done")
    if ud is not None:
        err = float(np.linalg.norm(u[rows] - ud) / np.linalg.norm(ud))

    plain = None
    if args.precision != 0 and not args.no_plain:
        m.set(capi.P_PRECISION, 0)
        up_d = torch.empty_like(f_d)
        step_device(up_d)  # warm-up: records the plain form's ACA ranks for its plan
        pt, pn, pf = timed(m, stream, flush, 1, lambda: step_device(up_d))
        m.set(capi.P_PRECISION, args.precision)
        pms = max_over_ranks(float(np.mean(pt)))
        up = up_d.cpu().numpy().astype(np.float64)
        if ud is not None:
            err_plain = float(np.linalg.norm(up[rows] - ud) / np.linalg.norm(ud))
        plain = {"form": "plain_fp32", "ms_per_step": pms, "value": n / (pms / 1e3),
                 "near_ms": float(pn[0]), "far_ms": float(pf[0]), "rel_l2_vs_dense": err_plain,
                 "steps": 1, "warmup": 1, "speedup_of_headline": pms / ms}

    hbm, bf16, src = peaks()
    near_s = float(np.mean(near_ms)) / 1e3
    achieved = st["close_evals"] * FLOP_PER_EVAL / near_s / 1e12
    # the MUFU roofline of the same kernel: 640 tanh per evaluation at 16 tanh per clock per SM
    # (tanh.approx.bf16x2 issues at half the rate of tanh.approx.f32; measured on this B200)
    sm_mhz = ck.get("sm_mhz") or 1965.0  # clocks.max.sm of this B200 when nvidia-smi gave nothing
    mufu_peak = props.multi_processor_count * 16 * sm_mhz * 1e6 / TANH_PER_EVAL
    near_eps = st["close_evals"] / near_s
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": PREC_DTYPE[args.precision], "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "epsilon": args.epsilon, "max_iter": 100,
                   "form": PREC_NAME[args.precision],
                   "parallelism": f"list shards x{world} + NCCL all-reduce of u" if world > 1 else "single GPU",
                   "l2": "256 MiB buffer written between timed steps",
                   "aca_plan": "ranks recorded by the warm-up H-matvec on the same tree"},
        "roofline": {"bound": "tensor", "kernel": "k_near_tc (features + two-body network + contraction)",
                     "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                     "peak_source": f"bf16_tflops of {src} MEASURED_PEAKS.json",
                     "traffic": NEAR_DRAM_BYTES_PER_PARTICLE * n,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of k_near_tc in the ncu "
                                       "capture at N = 131,072, scaled by N",
                     "algorithmic": f"{FLOP_PER_EVAL} FLOP/eval x {st['close_evals']} evals / near-field time",
                     "mufu": {"achieved_evals_per_s": near_eps, "peak_evals_per_s": mufu_peak,
                              "frac": near_eps / mufu_peak,
                              "peak_source": f"16 tanh/clk/SM x {props.multi_processor_count} SMs x {sm_mhz:.0f} MHz "
                                             f"/ {TANH_PER_EVAL} tanh per evaluation"}},
        "e2e": {"value": n / (e2e_ms / 1e3), "unit": "particles/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 12 * n, "ms_per_step": e2e_ms},
        "gpu_launches": int(st["gpu_launches"]),
        "clocks": ck,
        "error": {"rel_l2_vs_dense": err, "rows": int(len(rows)), "seconds": t_check,
                  "oracle": "FP64 dense rows on the device: the two-body network in FP64 (weights promoted "
                            "from FP32), features and sums in FP64, every row summed over all N sources; "
                            "rows drawn without replacement, seed 12345"},
        "unplanned": unplanned,
        "plain_fp32": plain,
        "student": student,
        "breakdown_ms": {"near": float(np.mean(near_ms)), "far": float(np.mean(far_ms)),
                         "build": st0["t_build_ms"], "far_by_kernel": far_breakdown},
        "work": {"close_pairs": st["num_close"], "far_pairs": st["num_far"], "close_evals": st["close_evals"],
                 "far_evals": st["far_evals"], "far_rank_mean": st["far_rank_sum"] / max(1, st["num_far"]),
                 "far_rank_max": st["far_rank_max"], "far_iterations": st["far_iterations"],
                 "student_fallback_blocks": st["student_fallback_blocks"]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_estimate(x, f, args.epsilon, args.cpu_sample_seconds, st["close_evals"],
                                            st["far_evals"])
    note("plain form and CPU baseline done")
    euler = None
    if rank == 0 and world == 1 and not args.no_next_rows and args.euler_steps > 0:
        # the batching workload's time loop on the benchmark model (tensor cores + student, eps 1e-2):
        # gravity + Morse (D 1, a 5, r0 2.1, cutoff 3), explicit Euler, dt 1e-3, rebuilt every 10 steps
        # The 64 Gaussian clusters of the matvec positions overlap (their cores hold about ten
        # times the spheres that fit), and Morse repulsion between overlapping spheres blows the
        # loop up within two steps; the loop starts from non-overlapping spheres at the same N and
        # volume fraction (random sequential placement, minimum separation 2.05, seed 2). Gravity
        # on all 1M spheres of an unbounded suspension drives a collective flow of ~5.6 radii per
        # step whose shear closes neighbour gaps (minimum separation 2.05 -> 1.92 in 10 steps), and
        # the stiff Morse wall then makes explicit Euler at dt 1e-3 unstable; the timed loop
        # therefore runs the Morse forces alone (stable: minimum separation 2.05 -> 2.06 in 10 steps).
        from hignn_b200 import synthetic as S

        xe = S.uniform_min_dist(n, 0.10, 2)
        note("Euler loop: positions placed")
        m.set(capi.P_TIMING, 0)
        morse = dict(De=1.0, a=5.0, re=2.1, cutoff=3.0)
        m.run_euler(xe, 1, 1e-3, rebuild_every=10, gravity=(0.0, 0.0, 0.0), **morse)  # warm-up
        t0 = time.perf_counter()
        x1 = m.run_euler(xe, args.euler_steps, 1e-3, rebuild_every=10, gravity=(0.0, 0.0, 0.0), **morse)
        dt_loop = time.perf_counter() - t0
        note(f"Euler loop done: {dt_loop / args.euler_steps * 1e3:.0f} ms per step")
        euler = {"workload": "N=1,048,576 spheres uniform at volume fraction 0.10 with minimum separation 2.05 "
                             "(seed 2; the matvec's clustered positions overlap), Morse (D 1, a 5, r0 2.1, cutoff "
                             "3) without gravity (with it the unbounded collective flow drives neighbours into the "
                             "Morse wall and explicit Euler at dt 1e-3 becomes unstable), tensor cores + student far field, "
                             "eps 1e-2, explicit Euler dt 1e-3, tree rebuilt every 10 steps",
                 "steps": args.euler_steps, "ms_per_step": dt_loop / args.euler_steps * 1e3,
                 "particle_steps_per_s": n * args.euler_steps / dt_loop,
                 "final_positions_finite": bool(np.isfinite(x1).all()),
                 "max_displacement": float(np.abs(x1 - xe).max()), "phases_ms": m.loop_profile(),
                 "note": "wall clock of hignn_run_euler from host positions; rebuilds, forces, matvecs inside"}
    m.close()
    if rank == 0 and world == 1 and not args.no_next_rows:
        line["next_rows"] = {"three_body": three_body_row(args), "euler_1m": euler}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
