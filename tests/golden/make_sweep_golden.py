"""Reference fixtures for the batched Yagi-Uda sweep (tests/test_batch.py).

The sweep is 256 seeded variants (seed 0) x 32 frequencies, 140-160 MHz.
Twelve of its problems, spread over the range of segment counts and over
the frequency grid, are solved here by the reference NEC2++ built from its
own sources (oracle/_ref/libnecpp_ref.so), each with the sweep's 91 x 72
pattern.  Stored: the (variant, frequency index) pairs, N, Zin and the gain
grid (float32 dB, phi-major: index phi * 91 + theta).

    make -C oracle ref && python tests/golden/make_sweep_golden.py
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refwrap import RefAPI  # noqa: E402

NVAR, NFREQ, SEED, NPICK = 256, 32, 0, 12


def _workloads():
    spec = importlib.util.spec_from_file_location("necpp_workloads", os.path.join(ROOT, "necpp_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def variants(W):
    rng = np.random.default_rng(SEED)
    return [W.yagi_params(rng) for _ in range(NVAR)]


def picks(params):
    """NPICK (variant, frequency index) pairs: variants at evenly spaced
    ranks of N, frequencies stepping through the grid."""
    n = np.array([int(np.sum(p[3])) for p in params])
    order = np.argsort(n, kind="stable")
    vs = [int(order[int(round(k * (NVAR - 1) / (NPICK - 1)))]) for k in range(NPICK)]
    fis = [(7 * k) % NFREQ for k in range(NPICK)]
    return list(zip(vs, fis))


def main():
    W = _workloads()
    params = variants(W)
    freqs = np.linspace(140.0, 160.0, NFREQ)
    ref = RefAPI()
    out = {"pick": [], "n": [], "zin": [], "gain": []}
    for v, fi in picks(params):
        half, xs, rad, segs = params[v]
        ctx = ref.nec_create()
        for e in range(len(half)):
            ref.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                         float(half[e]), float(rad[e]), 1.0, 1.0)
        ref.nec_geometry_complete(ctx, 0)
        ref.nec_fr_card(ctx, 0, 1, float(freqs[fi]), 0.0)
        ref.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        if ref.nec_rp_card(ctx, *W.PATTERN_91x72) != 0:
            raise RuntimeError(ref.error())
        out["pick"].append((v, fi))
        out["n"].append(int(np.sum(segs)))
        out["zin"].append(complex(ref.nec_impedance_real(ctx, 0), ref.nec_impedance_imag(ctx, 0)))
        out["gain"].append([[ref.nec_gain(ctx, 0, t, p) for t in range(91)] for p in range(72)])
        ref.nec_delete(ctx)
        print("variant %3d  f = %.4f MHz  N = %3d  Zin = %s" % (v, freqs[fi], out["n"][-1], out["zin"][-1]))
    np.savez_compressed(os.path.join(HERE, "yagi_sweep.npz"), pick=np.array(out["pick"], dtype=np.int32),
                        n=np.array(out["n"], dtype=np.int32), zin=np.array(out["zin"]),
                        gain=np.array(out["gain"], dtype=np.float32).reshape(NPICK, -1))


if __name__ == "__main__":
    main()
