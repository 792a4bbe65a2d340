#!/usr/bin/env python3
"""Solves/s of the NEC2++ thin-wire hot path on one B200 (or N replicas).

A step is one pass of the hot path -- interaction-matrix fill, dense complex
LU, solve (with FP64 refinement in mixed precision), current coefficients and
the 91 x 72 far-field pattern -- for the 8 x 8 axial-mode helix array
(11,520 segments, dense complex Z of 11,520^2, 1 GHz, 64 feeds with seeded
phases).  Synthetic seeded geometry; no dataset.

  value   mixed-precision solves/s with all inputs resident in HBM
          (structure tables, right-hand side, direction list), all ranks
  fp64    the same step in plain complex128 (reported beside it)
  e2e     solves/s through the NEC2++ C API with host buffers: create the
          context, build the geometry, cards, nec_rp_card (fill, factor,
          solve, pattern), read Zin and gains, delete -- every byte moved
          between host and device inside the timed region
  cpu_baseline  the reference's own CPU implementation (oracle/_ref),
          timed on a bounded sample of the same workload

``--impl reference`` times the reference's CPU path alone (rank 0).
Under torchrun each rank runs an independent replica (no collective on the
data path); value is the total over ranks and the step time the max.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Solves/s at N=11520, mixed vs FP64 on B200 at ≤1e-6 Zin err; grad/fwd cost"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--k", type=int, default=8, help="helix array is k x k (k=8: N=11520)")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-gradient", action="store_true")
    p.add_argument("--no-sweep", action="store_true")
    p.add_argument("--trace", default=None,
                   help="write a launch trace (every kernel with its stream, start and end) of one mixed step "
                        "to this JSON file")
    return p.parse_args()


def load_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- reference CPU path
def _workloads():
    """The card sequences of necpp_b200/workloads.py, loaded from the file
    itself: importing the package would map libnecpp_b200.so into the
    reference arm's process."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("necpp_workloads", os.path.join(HERE, "necpp_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(args, world):
    """The `config` of both arms' lines (identical by construction)."""
    n = args.k * args.k * 180
    return {"workload": "helix_array_%dx%d N=%d 1GHz seed=%d, 91x72 pattern" % (args.k, args.k, n, args.seed),
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (Z: 16 N^2 = %.2f GB rewritten every step)" % (16 * n * n / 1e9)}


def reference_solve_in_steps(ref, W, k, seed, steps):
    """One complete solve of the k x k helix array through the reference's
    C API, run as `steps` real pieces that add up to exactly that solve.
    Piece 1 builds the structure (helix, GM, geometry completion, FR, the
    64 EX cards) and runs nec_xq_card: cmset, factrs and the solve
    (src/nec_context.cpp:1523-1558, 4850-4935).  Pieces 2..steps each run
    one RP card over a contiguous share of the 72 phi cuts of the 91 x 72
    pattern (src/nec_radiation_pattern.cpp:209-450); after XQ the
    reference's RP card evaluates only the far field on the held currents.
    With steps = 1 the whole pattern follows XQ in the one piece."""
    t_piece = []
    t0 = time.perf_counter()
    ctx = ref.nec_create()
    n = W.helix_array(ref, ctx, k=k, seed=seed, execute=False)
    t_build = time.perf_counter() - t0
    t1 = time.perf_counter()
    if ref.nec_xq_card(ctx, 0) != 0:
        raise RuntimeError("reference nec_xq_card: " + ref.error())
    t_xq = time.perf_counter() - t1
    zin = [complex(ref.nec_impedance_real_indexed(ctx, 0, f), ref.nec_impedance_imag_indexed(ctx, 0, f))
           for f in range(k * k)]
    chunks = np.array_split(np.arange(72), max(steps - 1, 1))
    t_pattern = 0.0
    for c, ph in enumerate(chunks):
        if steps > 1:  # the previous piece ends here
            t_piece.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
        t1 = time.perf_counter()
        if len(ph) and ref.nec_rp_card(ctx, 0, 91, len(ph), 1, 0, 0, 0, 0.0, 5.0 * ph[0], 2.0, 5.0, 0.0, 0.0) != 0:
            raise RuntimeError("reference nec_rp_card: " + ref.error())
        t_pattern += time.perf_counter() - t1
    t_piece.append(time.perf_counter() - t0)
    gmax = max(ref.nec_gain_max(ctx, i) for i in range(len(chunks)) if len(chunks[i]))
    ref.nec_delete(ctx)
    return {"n": n, "piece_s": t_piece, "build_s": t_build, "xq_s": t_xq,
            "pattern_s": t_pattern, "zin_feed1": [zin[0].real, zin[0].imag], "gain_max_dbi": gmax}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    os.environ["OMP_NUM_THREADS"] = str(cores)  # read when libgomp loads
    from oracle import refwrap
    world = int(os.environ.get("WORLD_SIZE", "1"))
    omp = refwrap.available(omp=True)
    if not refwrap.available(omp=omp):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference compiled from its "
                          "sources) is not built on this host"}), flush=True)
        return 0
    W = _workloads()
    ref = refwrap.RefAPI(omp=omp)
    # warm-up: whole solves of the 2 x 2 array (N = 720): loads the library,
    # starts the OpenMP pool, touches the allocator
    for _ in range(args.warmup):
        ctx = ref.nec_create()
        W.helix_array(ref, ctx, k=2, seed=args.seed)
        ref.nec_delete(ctx)
    r = reference_solve_in_steps(ref, W, args.k, args.seed, args.steps)
    t = float(sum(r["piece_s"]))
    v = 1.0 / t
    sample = ("one full solve of the %dx%d helix array (N=%d) through the reference's C API, run as the %d "
              "timed steps: step 1 = structure + nec_xq_card (fill, factor, solve), steps 2..%d = RP cards over "
              "contiguous shares of the 91x72 pattern; Eigen with OpenMP over %d threads, fill and pattern serial"
              % (args.k, args.k, r["n"], args.steps, args.steps, cores if omp else 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": workload_config(args, world),
        "precision": "fp64 (Eigen PartialPivLU)",
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores if omp else 1,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "stages_s": {"structure_and_cards": r["build_s"], "xq_fill_factor_solve": r["xq_s"],
                     "pattern": r["pattern_s"]},
        "step_s": r["piece_s"],
        "check": {"zin_feed1": r["zin_feed1"], "gain_max_dbi": r["gain_max_dbi"]},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(seed):
    """The reference's one-thread build (oracle/_ref/libnecpp_ref.so) on a
    bounded sample of the workload: the 4 x 4 corner of the helix array
    (N = 2880, the same helices, pitch, frequency and feeds), each stage
    timed and scaled to N = 11520 by its own operation count: the fill by
    the pair count (N^2, x16), the factorisation and solve by the LU's flops
    (N^3, x64), the pattern by the segment count (N, x4), the structure and
    cards by N (x4).  A full-size one-thread run of the same build measured
    the scaled figure within the error recorded in the design notes."""
    from oracle import refwrap
    W = _workloads()
    ref = refwrap.RefAPI(omp=False)
    k = 4
    t0 = time.perf_counter()
    ctx = ref.nec_create()
    n = W.helix_array(ref, ctx, k=k, seed=seed, execute=False)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.nec_xq_card(ctx, 0)
    t_xq = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.nec_rp_card(ctx, *W.PATTERN_91x72)
    t_pat = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.fill(ctx)  # the reference's cmset again, alone (plus an N^2 copy out)
    t_fill = time.perf_counter() - t0
    ref.nec_delete(ctx)
    t_lu = max(t_xq - t_fill, 0.0)
    r = 11520.0 / n
    t_full = t_build * r + t_fill * r ** 2 + t_lu * r ** 3 + t_pat * r
    return {"n_sample": n, "t_sample_s": t_build + t_xq + t_pat, "t_build_s": t_build, "t_fill_s": t_fill,
            "t_factor_solve_s": t_lu, "t_pattern_s": t_pat, "t_scaled_s": t_full}


# ---------------------------------------------------------------- B200 path
class Stats(C.Structure):
    _fields_ = [("refine_iters", C.c_int), ("refine_residual", C.c_double),
                ("ms_fill", C.c_double), ("ms_factor", C.c_double), ("ms_solve", C.c_double),
                ("ms_pattern", C.c_double), ("launches", C.c_int64), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("k_ms", C.c_double * 9), ("k_launches", C.c_int64 * 9),
                ("k_flops", C.c_double * 9), ("pivoting", C.c_int), ("near_passes", C.c_int)]


K_NAMES = ["fill", "lu_panel", "lu_laswp", "lu_trsm", "lu_gemm", "trsv", "refine_residual",
           "pattern", "other"]
# roofline class of each kernel: (bound, unit of the recorded work)
K_BOUND = {"fill": ("compute", "pair evaluations"), "lu_gemm": ("tensor", "flops"),
           "lu_panel": ("latency", "flops"), "lu_trsm": ("compute", "flops"),
           "trsv": ("hbm", "bytes"), "refine_residual": ("hbm", "bytes"),
           "pattern": ("compute", "terms"), "lu_laswp": ("hbm", "bytes"), "other": ("hbm", "bytes")}


def gradient_cost(nb, W, reps=5):
    """grad/fwd cost on the adjoint workload: the seeded 9-element Yagi, 21
    segments per element, 10 m over Sommerfeld ground, 145 MHz; outputs Re Zin,
    Im Zin and gain at theta 80, phi 0; 27 parameters.  forward = one solve
    through the C API with the gain direction (cards, fill, factorisation,
    solve, far field); gradient = all 27 x 3 derivatives after it (perturbed
    structures, 3 transposed solves, contracted perturbed fills, assembly).
    Wall clock of the synchronous API calls, median of `reps`."""
    from necpp_b200 import adjoint
    p = W.yagi_ground_params(0)
    build = lambda ctx, q: W.yagi_ground_cards(nb, ctx, q)

    def forward():
        t0 = time.perf_counter()
        ctx = nb.nec_create()
        nb.nec_set_precision(ctx, 1)
        build(ctx, p)
        nb.nec_fr_card(ctx, 0, 1, 145.0, 0.0)
        if nb.nec_rp_card(ctx, 0, 1, 1, 1, 0, 0, 0, 80.0, 0.0, 0.0, 0.0, 0.0, 0.0) != 0:
            raise RuntimeError(nb.nec_error_message())
        g = nb.nec_gain(ctx, 0, 0, 0)
        dt = time.perf_counter() - t0
        nb.nec_delete(ctx)
        return dt, g

    forward()
    adjoint.gradient(build, p, 145.0, 80.0, 0.0)  # warm-up
    fw, gr = [], []
    for _ in range(reps):
        fw.append(forward()[0])
        tm = {}
        value, jac = adjoint.gradient(build, p, 145.0, 80.0, 0.0, timings=tm)
        gr.append(tm["gradient_s"])
    f, g = statistics.median(fw), statistics.median(gr)
    return {"workload": "yagi9 over Sommerfeld ground, N=189, 145 MHz, 27 params x (Re Zin, Im Zin, gain)",
            "forward_ms": f * 1e3, "gradient_ms": g * 1e3, "grad_fwd_cost": g / f,
            "value": [float(v) for v in value], "timing": "wall clock of the synchronous C-API calls, median of %d"
            % reps}


def gradient_population_cost(nb, W, rank, world, replicas, m=64):
    """The population check of the adjoint workload: m seeded designs
    (yagi_ground_params(seed), seeds 0..m-1), shared out over the ranks.
    adjoint_s: wall clock of this rank's adjoint gradients (27 x 3 each);
    batched_fd_s: the same designs' central differences, all m x 55 base
    and perturbed structures in one batched solve; agreement: the largest
    |adjoint - difference| over each output's largest derivative."""
    from necpp_b200 import adjoint
    build = lambda ctx, q: W.yagi_ground_cards(nb, ctx, q)
    P = np.array([W.yagi_ground_params(s) for s in range(m)])
    t0 = time.perf_counter()
    idx, vals, jacs = adjoint.gradient_population(build, P, 145.0, 80.0, 0.0, world=world, rank=rank)
    t_adj = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, fd = adjoint.batched_fd(build, P[idx], 145.0, 80.0, 0.0)
    t_fd = time.perf_counter() - t0
    err = max(float(np.max(np.max(np.abs(jacs[k] - fd[k]), axis=1) / np.max(np.abs(fd[k]), axis=1)))
              for k in range(len(idx)))
    rate, total, slowest = replicas.whole_job_rate(len(idx), t_adj, device="cuda")
    return {"designs": int(total), "adjoint_s": slowest, "gradients_per_s": rate, "batched_fd_s": t_fd,
            "batched_fd_structures": len(idx) * 55, "max_rel_err_vs_batched_fd": err,
            "partition": "%d design(s) on rank %d of %d" % (len(idx), rank, world)}


def batched_sweep(nb, rank, world, replicas, reps=3, ref_sample=16):
    """The batched sweep: 256 seeded Yagi-Uda variants x 32 frequencies
    (140-160 MHz) = 8192 solves of fill, LU, FP64-refined solve, currents
    and a 91x72 gain pattern.  Problems are dealt to ranks by N^3
    (round-robin in decreasing cost); the job rate is all solves over the
    slowest rank's time.  `value` times the batched call from host
    structures to host results (copies included); host_prep_s is building
    the 8192 structures from cards; device_ms the kernels' CUDA-event time."""
    import ctypes as _C
    from necpp_b200 import batch as B
    t0 = time.perf_counter()
    problems, labels = B.yagi_problems(256, 32, seed=0)
    prep = time.perf_counter() - t0
    mine = replicas.partition_by_cost([float(p[0]["n"]) ** 3 for p in problems], world, rank)
    sub = [problems[i] for i in mine]
    th, ph = B.pattern_grid()
    B.sweep(sub[:64], th, ph)  # warm-up (pool, module)
    B.sweep(sub, th, ph)
    ts = []
    for _ in range(reps):
        t = time.perf_counter()
        res = B.sweep(sub, th, ph)
        ts.append(time.perf_counter() - t)
    # kernel time of one more pass with per-launch events
    eng = B._get_engine()
    L = nb.lib
    L.necgpu_enable_timing.argtypes = [_C.c_void_p, _C.c_int]
    L.necgpu_reset_kernel_stats.argtypes = [_C.c_void_p]
    L.necgpu_get_stats.argtypes = [_C.c_void_p, _C.POINTER(Stats)]
    L.necgpu_enable_timing(eng, 2)
    L.necgpu_reset_kernel_stats(eng)
    B.sweep(sub, th, ph)
    st = Stats()
    L.necgpu_get_stats(eng, _C.byref(st))
    L.necgpu_enable_timing(eng, 0)
    dev = {K_NAMES[i]: st.k_ms[i] for i in range(9) if st.k_launches[i]}
    t = statistics.median(ts)
    rate, total, slowest = replicas.whole_job_rate(len(sub), t, device="cuda")
    out = {"workload": "256 Yagi-Uda variants (3-15 elements, 11-41 segments each, N 33-615) x 32 "
                       "frequencies 140-160 MHz, 91x72 gain pattern each",
           "solves": int(total), "value": rate, "unit": "solves/s", "seconds": slowest,
           "host_prep_s": prep, "device_ms": {"fill": dev.get("fill"), "lu_and_refined_solve": dev.get("lu_panel"),
                                               "pattern": dev.get("pattern"), "other": dev.get("other")},
           "status_ok": int(np.sum(res["status"] == 0)), "max_residual": float(np.max(res["residual"])),
           "n_range": [int(min(p[0]["n"] for p in problems)), int(max(p[0]["n"] for p in problems))],
           "partition": "N^3 round-robin over %d rank(s)" % world}
    if rank == 0 and ref_sample:
        from oracle import refwrap
        if refwrap.available():
            out["reference_cpu"] = reference_sweep_sample(problems, labels, ref_sample)
    return out


def reference_sweep_sample(problems, labels, k):
    """The reference (oracle/_ref, one thread) on k of the sweep's problems
    spread over its size range; solves/s = k / their total time."""
    from oracle.refwrap import RefAPI
    from necpp_b200 import workloads as W
    ref = RefAPI()
    order = sorted(range(len(problems)), key=lambda i: problems[i][0]["n"])
    pick = [order[int(j * (len(order) - 1) / (k - 1))] for j in range(k)]
    rng = np.random.default_rng(0)
    params = [W.yagi_params(rng) for _ in range(256)]
    t = 0.0
    for i in pick:
        v, f = labels[i]
        half, xs, rad, segs = params[v]
        ctx = ref.nec_create()
        t0 = time.perf_counter()
        for e in range(len(half)):
            ref.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                         float(half[e]), float(rad[e]), 1.0, 1.0)
        ref.nec_geometry_complete(ctx, 0)
        ref.nec_fr_card(ctx, 0, 1, f, 0.0)
        ref.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        ref.nec_rp_card(ctx, 0, 91, 72, 1, 0, 0, 0, 0.0, 0.0, 2.0, 5.0, 0.0, 0.0)
        t += time.perf_counter() - t0
        ref.nec_delete(ctx)
    return {"value": k / t, "unit": "solves/s", "cores": 1, "kind": "reference",
            "sample": "%d problems spread over the size range (N %d-%d), each cards + fill + LU + solve + "
                      "91x72 pattern; the sweep's mix of sizes differs, so this is indicative"
                      % (k, problems[pick[0]][0]["n"], problems[pick[-1]][0]["n"])}


class TraceRec(C.Structure):
    _fields_ = [("cls", C.c_int), ("stream", C.c_int), ("start_ms", C.c_float), ("end_ms", C.c_float),
                ("work", C.c_double), ("name", C.c_char * 48)]


def measure_tf32_peak(torch, n=8192, iters=300):
    """Dense TF32 rate of this GPU: a cuBLAS FP32 GEMM with TF32 allowed
    (n^3, about half a second of back-to-back launches), TFLOP/s.  The
    tensor-core update's TF32 form is measured against it, as its split-BF16
    form is against the measured BF16 GEMM rate."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        g = torch.Generator(device="cuda").manual_seed(7)
        a = torch.randn(n, n, device="cuda", generator=g)
        b = torch.randn(n, n, device="cuda", generator=g)
        c = torch.empty(n, n, device="cuda")
        for _ in range(5):
            torch.matmul(a, b, out=c)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(iters):
            torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) * 1e-3
        del a, b, c
        return 2.0 * n ** 3 * iters / secs / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def write_trace(L, eng, path, check):
    """One resident mixed step at timing level 3: every launch with its
    class, stream, start and end (ms from the step's first launch).  The
    events around each launch slow the step; the order and overlap of the
    launches are what the trace is for."""
    L.necgpu_get_trace.argtypes = [C.c_void_p, C.POINTER(TraceRec), C.c_int]
    check(eng, L.necgpu_enable_timing(eng, 3))
    check(eng, L.necgpu_step_resident(eng, 1))  # warm
    L.necgpu_reset_kernel_stats(eng)
    check(eng, L.necgpu_step_resident(eng, 1))
    cnt = L.necgpu_get_trace(eng, None, 0)
    buf = (TraceRec * cnt)()
    L.necgpu_get_trace(eng, buf, cnt)
    L.necgpu_enable_timing(eng, 0)
    recs = [{"cls": K_NAMES[r.cls] if 0 <= r.cls < len(K_NAMES) else r.cls, "stream": r.stream,
             "start_ms": r.start_ms, "end_ms": r.end_ms, "work": r.work,
             "name": r.name.decode(errors="replace").split("<<<")[0]} for r in buf]
    with open(path, "w") as f:
        json.dump(recs, f)


def run_b200(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ["NECPP_B200_DEVICE"] = str(local)
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    import necpp_b200 as nb
    from necpp_b200 import replicas
    from necpp_b200 import workloads as W
    L = nb.lib
    L.nec_gpu_engine.restype = C.c_void_p
    L.nec_gpu_engine.argtypes = [C.c_void_p]
    for nm in ("necgpu_set_stream",):
        getattr(L, nm).argtypes = [C.c_void_p, C.c_void_p]
    L.necgpu_step_resident.argtypes = [C.c_void_p, C.c_int]
    L.necgpu_reuse_last_inputs.argtypes = [C.c_void_p]
    L.necgpu_enable_timing.argtypes = [C.c_void_p, C.c_int]
    L.necgpu_reset_kernel_stats.argtypes = [C.c_void_p]
    L.necgpu_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    L.necgpu_last_error.restype = C.c_char_p
    L.necgpu_last_error.argtypes = [C.c_void_p]
    L.necgpu_read_resident.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.necgpu_measure_peak.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]

    class API:
        def __getattr__(self, k):
            return getattr(nb, k)

        def helix(self, ctx, *a):
            return nb.nec_helix(ctx, *a)

    api = API()
    stream = torch.cuda.Stream()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, device="cuda")

    def check(eng, rc):
        if rc != 0:
            raise RuntimeError(L.necgpu_last_error(eng).decode())

    def prepare(precision):
        ctx = nb.nec_create()
        nb.nec_set_precision(ctx, precision)
        W.helix_array(api, ctx, k=args.k, seed=args.seed)
        eng = L.nec_gpu_engine(ctx)
        check(eng, L.necgpu_set_stream(eng, C.c_void_p(stream.cuda_stream)))
        check(eng, L.necgpu_reuse_last_inputs(eng))
        return ctx, eng

    def zin_all(ctx):
        nfeed = args.k * args.k
        return np.array([complex(nb.nec_impedance_real_indexed(ctx, 0, f),
                                 nb.nec_impedance_imag_indexed(ctx, 0, f)) for f in range(nfeed)])

    def timed(eng, precision, steps, warmup, sampler=None, level=0):
        """Device time per step over `steps` resident steps.  level 2 adds an
        event pair around every launch (per-kernel-class times for the
        roofline); the headline number is taken with level 0."""
        for _ in range(warmup):
            check(eng, L.necgpu_step_resident(eng, precision))
        st0 = Stats()
        L.necgpu_get_stats(eng, C.byref(st0))
        check(eng, L.necgpu_enable_timing(eng, level))
        L.necgpu_reset_kernel_stats(eng)
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            check(eng, L.necgpu_step_resident(eng, precision))
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop() if sampler else None
        ms = e0.elapsed_time(e1) / steps
        st = Stats()
        L.necgpu_get_stats(eng, C.byref(st))
        L.necgpu_enable_timing(eng, 0)
        return ms, st, st.launches - st0.launches, clocks

    peaks, peak_src = load_peaks()
    out = {}

    # ---- mixed precision, resident inputs
    ctx_m, eng_m = prepare(1)
    z_mixed = zin_all(ctx_m)
    iters, resid = nb.last_refinement(ctx_m)
    L.necgpu_update_format.argtypes = [C.c_void_p]
    update_format = {1: "split_bf16x3", 2: "tf32"}.get(L.necgpu_update_format(eng_m), "none")
    sampler = ClockSampler(local)
    ms_m, _, launches_m, clocks = timed(eng_m, 1, args.steps, args.warmup, sampler)
    value, _, secs = replicas.whole_job_rate(args.steps, ms_m * args.steps / 1e3, device="cuda")
    ms_m_max = secs * 1e3 / args.steps
    # the same steps again with per-launch events, for the per-kernel roofline
    ms_inst, st_m, _, _ = timed(eng_m, 1, args.steps, 1, None, level=2)

    if args.trace:
        write_trace(L, eng_m, args.trace, check)

    # ---- plain FP64
    ms_f_max, z_fp64 = None, None
    if not args.no_fp64:
        ctx_f, eng_f = prepare(0)
        z_fp64 = zin_all(ctx_f)
        fsteps = max(1, min(args.steps, 5))
        ms_f, _, _, _ = timed(eng_f, 0, fsteps, min(args.warmup, 3))
        ms_f_max = max_over_ranks(ms_f)
        _, st_f, _, _ = timed(eng_f, 0, 1, 0, None, level=2)
        out["fp64_kernels_ms_per_step"] = {K_NAMES[i]: st_f.k_ms[i] for i in range(9) if st_f.k_launches[i]}
        # measured FP64 peaks (register-only loops) and the FP64 path's update against them
        pk = {}
        for kind, nm in ((0, "fp64_fma"), (1, "fp64_tensor_mma")):
            v = C.c_double(0.0)
            check(eng_f, L.necgpu_measure_peak(eng_f, kind, C.byref(v)))
            pk[nm] = v.value
        out["fp64_peaks_tflops"] = pk
        gi = K_NAMES.index("lu_gemm")
        if st_f.k_launches[gi]:
            ach = st_f.k_flops[gi] / (st_f.k_ms[gi] * 1e-3) / 1e12
            out["fp64_roofline"] = {"kernel": "gemm_dmma_kernel (FP64 trailing update)", "achieved": ach,
                                    "peak": pk["fp64_tensor_mma"], "unit": "TFLOP/s",
                                    "frac": ach / pk["fp64_tensor_mma"],
                                    "peak_source": "measured here: mma.sync m8n8k4 f64 register loop"}
        nb.nec_delete(ctx_f)

    # ---- end to end through the C API (host buffers)
    # two untimed passes: the first creates the engine that later contexts
    # take from the pool, the second captures its LU graph
    e2e_ms = []
    h2d = d2h = 0
    e2e_warm = 2
    for s in range(args.e2e_steps + e2e_warm if args.e2e_steps > 0 else 0):
        barrier()
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        ctx = nb.nec_create()
        nb.nec_set_precision(ctx, 1)
        W.helix_array(api, ctx, k=args.k, seed=args.seed)
        z = zin_all(ctx)
        g = nb.nec_gain_max(ctx, 0)
        eng = L.nec_gpu_engine(ctx)
        st = Stats()
        L.necgpu_get_stats(eng, C.byref(st))
        nb.nec_delete(ctx)
        a1.record(stream)
        torch.cuda.synchronize()
        if s >= e2e_warm:
            e2e_ms.append(a0.elapsed_time(a1))
            h2d, d2h = st.h2d_bytes, st.d2h_bytes
        if not np.all(np.isfinite(z)) or not math.isfinite(g):
            raise RuntimeError("e2e produced non-finite results")
    e2e_ms_max = max_over_ranks(statistics.mean(e2e_ms)) if e2e_ms else float("nan")

    # ---- roofline of the dominant kernel of the mixed step
    shares = {K_NAMES[i]: st_m.k_ms[i] for i in range(9) if st_m.k_launches[i]}
    tot = sum(shares.values()) or 1.0
    # the roofline kernel: the largest class with a throughput bound (tensor
    # or HBM).  The latency-bound panel classes run on side streams beside
    # the updates; their summed time counts overlapped work and has no peak
    # to be a fraction of, so the largest class by time is reported beside
    dom_time = max(shares, key=shares.get)
    thr = {k: v for k, v in shares.items() if K_BOUND[k][0] in ("tensor", "hbm")}
    dom = max(thr, key=thr.get) if thr else dom_time
    di = K_NAMES.index(dom)
    avg_ms = st_m.k_ms[di] / st_m.k_launches[di]
    work = st_m.k_flops[di] / st_m.k_launches[di]
    bound, unit_kind = K_BOUND[dom]
    traffic, traffic_src = None, None
    tfile = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        traffic = tj.get(dom)
        if traffic is not None:
            traffic_src = "ncu capture, not this run: %s (%s)" % (tj.get("_source"), tj.get("_captured"))
    if bound == "hbm":
        achieved = work / (avg_ms * 1e-3) / 1e9
        peak, unit = peaks["hbm_gbs"], "GB/s"
    else:
        achieved = work / (avg_ms * 1e-3) / 1e12
        peak, unit = peaks["bf16_tflops_sustained"], "TFLOP/s"
    peak_source = peak_src + (" bf16 dense sustained" if unit != "GB/s" else " copy")
    extra = {}
    if dom == "lu_gemm" and update_format == "tf32":
        # the update computes in TF32, whose tensor-core rate is half of
        # BF16's: its fraction of a TF32 rate measured here, beside the
        # fraction of the measured BF16 peak
        tf32 = measure_tf32_peak(torch)
        extra = {"tf32_rate": tf32, "frac_of_tf32_rate": achieved / tf32,
                 "tf32_rate_source": "measured here: cuBLAS TF32 GEMM 8192^3 (torch.matmul, allow_tf32), "
                                     "300 back-to-back launches"}
    roofline = {"kernel": dom, "bound": "hbm" if bound == "hbm" else "tensor", "achieved": achieved,
                "peak": peak, "unit": unit, "frac": achieved / peak, **extra, "traffic": traffic,
                "traffic_source": traffic_src, "peak_source": peak_source,
                "avg_launch_ms": avg_ms, "work_per_launch": work, "work_unit": unit_kind,
                "launches_per_step": st_m.k_launches[di] / args.steps,
                "largest_class_by_time": {"kernel": dom_time, "bound": K_BOUND[dom_time][0],
                                          "share": round(shares[dom_time] / tot, 4)},
                "share": {k: round(v / tot, 4) for k, v in sorted(shares.items(), key=lambda kv: -kv[1])},
                "ms_per_step_by_kernel": {k: v / args.steps for k, v in shares.items()},
                "ms_per_step_instrumented": ms_inst}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_m_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 LU (%s tensor-core update) + c128 fill/refinement" % update_format, "data": "synthetic",
        "config": workload_config(args, world), "precision": "mixed",
        "gpu_launches": int(launches_m / args.steps * args.steps),
        "clocks": clocks,
        "refine": {"iters": iters, "residual": resid, "update_format": update_format},
        "e2e": {"value": world * 1000.0 / e2e_ms_max, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": roofline,
    }
    if ms_f_max is not None:
        line["fp64"] = {"value": world * 1000.0 / ms_f_max, "ms_per_step": ms_f_max}
        line["mixed_vs_fp64"] = ms_f_max / ms_m_max
        rel = np.abs(z_mixed - z_fp64) / np.abs(z_fp64)
        line["zin_rel_err_mixed_vs_fp64"] = float(np.max(rel))
    gold = os.path.join(HERE, "tests", "golden", "helix_array_%dx%d.npz" % (args.k, args.k))
    if args.seed == 0 and os.path.exists(gold):
        # the reference's own solve of this workload (committed fixture)
        zr = np.load(gold)["zin"][0]
        line["zin_rel_err_mixed_vs_ref"] = float(np.max(np.abs(z_mixed - zr) / np.abs(zr)))
        if z_fp64 is not None:
            line["zin_rel_err_fp64_vs_ref"] = float(np.max(np.abs(z_fp64 - zr) / np.abs(zr)))
    line.update(out)

    if rank == 0 and not args.no_gradient:
        line["gradient"] = gradient_cost(nb, W)
    if not args.no_gradient:
        pop = gradient_population_cost(nb, W, rank, world, replicas)
        if rank == 0:
            line.setdefault("gradient", {})["population"] = pop
    if not args.no_sweep:
        sw = batched_sweep(nb, rank, world, replicas, ref_sample=0 if args.no_cpu_baseline else 16)
        if rank == 0:
            line["batched_sweep"] = sw

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import refwrap
        if refwrap.available():
            r = cpu_baseline_sample(args.seed)
            line["cpu_baseline"] = {
                "value": 1.0 / r["t_scaled_s"], "unit": "solves/s", "cores": 1, "kind": "reference",
                "sample": "4x4 corner of the helix array (N=%d) through the reference's one-thread build "
                          "(%.1f s); each stage scaled to N=11520 by its operation count: fill x16 (pairs), "
                          "factor+solve x64 (LU flops), pattern and cards x4 (segments)"
                          % (r["n_sample"], r["t_sample_s"]),
                "detail": r}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                                    "sample": "oracle/_ref not built on this host"}
    nb.nec_delete(ctx_m)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
