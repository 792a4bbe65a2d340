"""Autotuner of the mixed-precision LU's blocking (necgpu_tuning).

For each problem size it times the resident hot-path step (fill, block-
pivoted complex64 LU with tensor-core updates, refined solve, pattern) of
the seeded k x k helix array over a grid of

  outer          columns per outer block (inner dimension of the trailing
                 tensor-core update): 128, 256, 384, 512
  lookahead_sms  SMs kept for the next outer block's panels while the far
                 update runs beside them: 0 (no lookahead), 32, 48, 64
  gemm_group     m-tiles per band of the tensor-core update's tile walk:
                 8, 16, 32

and writes the fastest per size as rows of the tuning table the engine
reads when it factors (tuning.tsv beside libnecpp_b200.so):

    python -m necpp_b200.tune --sizes 2,4,6,8 --out necpp_b200/tuning.tsv

Each row covers the sizes up to the geometric mean of its size and the
next tuned one; the last row covers everything larger.  Needs one GPU.
"""
import argparse
import ctypes as C
import itertools
import math
import os
import statistics
import time

OUTER = (128, 256, 384, 512)
LOOKAHEAD_SMS = (0, 32, 48, 64)
GEMM_GROUP = (8, 16, 32)
DEFAULT = (256, 48, 16)


class Tuning(C.Structure):
    _fields_ = [("outer", C.c_int), ("lookahead_sms", C.c_int), ("gemm_group", C.c_int)]


def _bind(lib):
    lib.nec_gpu_engine.restype = C.c_void_p
    lib.nec_gpu_engine.argtypes = [C.c_void_p]
    lib.necgpu_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.necgpu_reuse_last_inputs.argtypes = [C.c_void_p]
    lib.necgpu_step_resident.argtypes = [C.c_void_p, C.c_int]
    lib.necgpu_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    lib.necgpu_last_error.restype = C.c_char_p
    lib.necgpu_last_error.argtypes = [C.c_void_p]


def time_candidates(k, candidates, steps=3, seed=0, precision=1):
    """ms per resident step of the k x k helix array for each candidate
    (outer, lookahead_sms, gemm_group); returns (n, {candidate: ms})."""
    import torch

    import necpp_b200 as nb
    from necpp_b200 import workloads as W
    L = nb.lib
    _bind(L)

    class API:
        def __getattr__(self, name):
            return getattr(nb, name)

        def helix(self, ctx, *a):
            return nb.nec_helix(ctx, *a)

    stream = torch.cuda.Stream()
    ctx = nb.nec_create()
    try:
        nb.nec_set_precision(ctx, precision)
        n = W.helix_array(API(), ctx, k=k, seed=seed)
        eng = L.nec_gpu_engine(ctx)

        def check(rc):
            if rc != 0:
                raise RuntimeError(L.necgpu_last_error(eng).decode())

        check(L.necgpu_set_stream(eng, C.c_void_p(stream.cuda_stream)))
        check(L.necgpu_reuse_last_inputs(eng))
        out = {}
        for cand in candidates:
            t = Tuning(*cand)
            check(L.necgpu_set_tuning(eng, C.byref(t)))
            check(L.necgpu_step_resident(eng, precision))  # warm-up (operand buffers, streams)
            ms = []
            for _ in range(steps):
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                check(L.necgpu_step_resident(eng, precision))
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            out[cand] = statistics.median(ms)
        check(L.necgpu_set_tuning(eng, None))
        return n, out
    finally:
        nb.nec_delete(ctx)


def tune(sizes, steps=3, precision=1, log=print):
    """Rows (n, best candidate, its ms, the default's ms) per helix array size k."""
    cands = list(itertools.product(OUTER, LOOKAHEAD_SMS, GEMM_GROUP))
    rows = []
    for k in sizes:
        t0 = time.perf_counter()
        n, res = time_candidates(k, cands, steps=steps, precision=precision)
        best = min(res, key=res.get)
        rows.append((n, best, res[best], res[DEFAULT]))
        log("k=%d N=%d best outer=%d lookahead_sms=%d gemm_group=%d: %.2f ms (default %.2f ms) [%d candidates, %.0f s]"
            % (k, n, *best, res[best], res[DEFAULT], len(cands), time.perf_counter() - t0))
    return rows


def write_table(rows, path, precision=1, device=""):
    """Tuning table rows 'precision n_max outer lookahead_sms gemm_group # ...'."""
    rows = sorted(rows)
    prec = "mixed" if precision == 1 else "fp64"
    lines = ["# necgpu tuning table, written by necpp_b200/tune.py%s" % (" on " + device if device else ""),
             "# precision  n_max  outer  lookahead_sms  gemm_group  # tuned at N: best ms, default ms"]
    for i, (n, best, ms, ms_default) in enumerate(rows):
        nmax = int(math.sqrt(n * rows[i + 1][0])) if i + 1 < len(rows) else 1 << 30
        lines.append("%s %d %d %d %d  # N=%d: %.3f ms, default %.3f ms" % (prec, nmax, *best, n, ms, ms_default))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="2,4,6,8", help="helix array sizes k (N = 180 k^2)")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.tsv"))
    a = ap.parse_args()
    import torch
    # the table being written must not steer the timings
    os.environ["NECPP_B200_TUNING"] = "none"
    rows = tune([int(x) for x in a.sizes.split(",")], steps=a.steps)
    write_table(rows, a.out, device=torch.cuda.get_device_name(0))
    print("wrote", a.out)


if __name__ == "__main__":
    main()
