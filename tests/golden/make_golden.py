"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs every case of tests/cases.py through the reference NEC2++ library built
from its own sources by oracle/Makefile (oracle/_ref/libnecpp_ref.so) and
stores, per case: connection tables, the scaled segment arrays and trio basis
tables of the last frequency, every antenna-input impedance, every pattern's
gain grid and statistics, the last solve's currents and current
coefficients, and the unfactored interaction matrix (full for N <= 200,
otherwise a seeded sample of elements).

    make -C oracle ref && python tests/golden/make_golden.py
    python tests/golden/make_golden.py helix_array_8x8 wire_mesh_41   # full size
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import refwrap  # noqa: E402
from oracle.refwrap import RefAPI  # noqa: E402
from cases import CASES, LARGE_CASES  # noqa: E402


def collect(ref, name, builder, grid, compact=False):
    """compact (the full-size workloads): no segment arrays, basis tables or
    current coefficients (the host tables are compared with the live
    reference by the CPU tests), Z as a sample plus its diagonal."""
    ctx = ref.nec_create()
    t0 = time.perf_counter()
    builder(ref, ctx)
    t_solve = time.perf_counter() - t0
    out = {}
    seg = ref.segments(ctx)
    n = len(seg["x"])
    if not compact:
        for k, v in seg.items():
            out["seg_" + k] = v
    out["wavelength"] = np.array(ref.ref_wavelength(ctx))
    # antenna inputs
    zin = []
    i = 0
    while True:
        feeds = []
        f = 0
        while True:
            re = ref.nec_impedance_real_indexed(ctx, i, f)
            if re == -999.0:
                break
            feeds.append(complex(re, ref.nec_impedance_imag_indexed(ctx, i, f)))
            f += 1
        if not feeds:
            break
        zin.append(feeds)
        i += 1
    nfeed = max((len(z) for z in zin), default=0)
    out["zin"] = np.array([z + [np.nan] * (nfeed - len(z)) for z in zin], dtype=complex).reshape(len(zin), nfeed)
    # patterns
    if grid is not None:
        nth, nph = grid
        gains, stats = [], []
        i = 0
        while ref.nec_gain_max(ctx, i) != -999.0:
            g = np.array([[ref.nec_gain(ctx, i, t, p) for p in range(nph)] for t in range(nth)])
            gains.append(g)
            stats.append([getattr(ref, "nec_gain_" + pre + s)(ctx, i)
                          for pre in ("", "rhcp_", "lhcp_") for s in ("max", "min", "mean", "sd")])
            i += 1
        out["gains"] = np.array(gains).reshape(len(gains), nth, nph)
        out["gain_stats"] = np.array(stats).reshape(len(stats), 12)
    # near-field patterns
    nf = ref.near_fields(ctx)
    if nf:
        out["near_nfeh"] = np.array([k for k, _, _ in nf], dtype=np.int32)
        out["near_np"] = np.array([len(x) for _, x, _ in nf], dtype=np.int32)
        out["near_xyz"] = np.concatenate([x for _, x, _ in nf])
        out["near_f"] = np.concatenate([f for _, _, f in nf])
    # last solution
    cur, abc = ref.currents(ctx)
    out["current_vector"] = cur
    if not compact:
        out["abc"] = abc
        # trio tables at the last frequency scaling
        ptr, basis, coef = [0], [], []
        for j in range(1, n + 1):
            jco, ax, bx, cx = ref.trio(ctx, j)
            basis.extend(jco.tolist())
            coef.extend(zip(ax, bx, cx))
            ptr.append(len(basis))
        out["trio_ptr"] = np.array(ptr, dtype=np.int32)
        out["trio_basis"] = np.array(basis, dtype=np.int32)
        out["trio_abc"] = np.array(coef, dtype=np.float64).reshape(-1, 3)
    # Sommerfeld tables of the last frequency (zero when the case has none)
    tab, eps = ref.somm_tables(ctx)
    if np.any(tab != 0):
        out["somm_tables"] = tab
        out["somm_epscf"] = np.array(eps)
    # interaction matrix (refilled by the reference's cmset, its table
    # interpolation cache reset to the state of a new context)
    ref.ref_somm_interp_reset(ctx)
    t0 = time.perf_counter()
    z = ref.fill(ctx)
    t_fill = time.perf_counter() - t0
    if n <= 200:
        out["Z"] = z
    else:
        rng = np.random.default_rng(1234)
        idx = rng.integers(0, n, size=(4000, 2))
        out["Z_idx"] = idx.astype(np.int32)
        out["Z_val"] = z[idx[:, 0], idx[:, 1]]
        out["Z_diag"] = np.diag(z).copy()
    out["n"] = np.array(n)
    ref.nec_delete(ctx)
    print("  %s: reference solve %.1f s, refill %.1f s" % (name, t_solve, t_fill), flush=True)
    return out


def main():
    # the full-size workloads run the reference's OpenMP build (Eigen's LU
    # over all cores); its results agree with the one-thread build to
    # rounding, far inside the parity tolerances
    args = sys.argv[1:]
    large = [a for a in args if a in LARGE_CASES]
    names = [a for a in args if a not in LARGE_CASES] if args else list(CASES)
    jobs = [(nm, CASES[nm], False) for nm in names] + [(nm, LARGE_CASES[nm], True) for nm in large]
    refs = {}
    for name, (builder, grid), compact in jobs:
        if compact not in refs:
            refs[compact] = RefAPI(omp=compact and refwrap.available(omp=True))
        out = collect(refs[compact], name, builder, grid, compact=compact)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print("%-22s N=%-5d zin=%s -> %s (%d KB)" % (name, int(out["n"]), out["zin"].shape,
                                                    os.path.basename(path), os.path.getsize(path) // 1024))


if __name__ == "__main__":
    main()
