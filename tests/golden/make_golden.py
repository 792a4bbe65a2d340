"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs every case of tests/cases.py through the reference NEC2++ library built
from its own sources by oracle/Makefile (oracle/_ref/libnecpp_ref.so) and
stores, per case: connection tables, the scaled segment arrays and trio basis
tables of the last frequency, every antenna-input impedance, every pattern's
gain grid and statistics, the last solve's currents and current
coefficients, and the unfactored interaction matrix (full for N <= 200,
otherwise a seeded sample of elements).

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.refwrap import RefAPI  # noqa: E402
from cases import CASES  # noqa: E402


def collect(ref, name, builder, grid):
    ctx = ref.nec_create()
    builder(ref, ctx)
    out = {}
    seg = ref.segments(ctx)
    n = len(seg["x"])
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
    z = ref.fill(ctx)
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
    return out


def main():
    ref = RefAPI()
    names = sys.argv[1:] or list(CASES)
    for name in names:
        builder, grid = CASES[name]
        out = collect(ref, name, builder, grid)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print("%-22s N=%-5d zin=%s -> %s (%d KB)" % (name, int(out["n"]), out["zin"].shape,
                                                    os.path.basename(path), os.path.getsize(path) // 1024))


if __name__ == "__main__":
    main()
