"""Generate the gradient golden fixture (tests/golden/yagi_grad.npz) from the
reference itself: the seeded 9-element Yagi, 21 segments per element, 10 m
over Sommerfeld ground (eps_r 13, sigma 0.005 S/m), 145 MHz, element 2
centre-fed with 1 V.  Outputs (Re Zin, Im Zin, gain dB at theta 80, phi 0)
and their central finite differences with h = 1e-6 m for each of the 27
parameters (9 half lengths, 9 x positions, 9 radii), each from a full FP64
solve of the reference NEC2++ built from its own sources (oracle/Makefile).

    make -C oracle ref && python tests/golden/make_grad_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refwrap import RefAPI  # noqa: E402

H = 1e-6
FREQ = 145.0
THETA, PHI = 80.0, 0.0


def yagi_params(seed=0):
    # same draws as necpp_b200.workloads.yagi_params(rng, n_elements=9, nseg=21)
    rng = np.random.default_rng(seed)
    half, xs, rad = [], [], []
    x = 0.0
    for e in range(9):
        hl = rng.uniform(0.40, 0.55)
        sp = rng.uniform(0.1, 0.7)
        r = rng.uniform(0.5e-3, 3e-3)
        rng.integers(5, 21)
        if e > 0:
            x += sp
        half.append(hl)
        xs.append(x)
        rad.append(r)
    return np.concatenate([half, xs, rad])


def outputs(ref, p):
    ctx = ref.nec_create()
    ne = len(p) // 3
    for e in range(ne):
        assert ref.nec_wire(ctx, e + 1, 21, p[ne + e], 0.0, 10.0 - p[e], p[ne + e], 0.0, 10.0 + p[e],
                            p[2 * ne + e], 1.0, 1.0) == 0
    assert ref.nec_geometry_complete(ctx, 0) == 0
    assert ref.nec_gn_card(ctx, 2, 0, 13.0, 0.005, 0.0, 0.0, 0.0, 0.0) == 0
    assert ref.nec_fr_card(ctx, 0, 1, FREQ, 0.0) == 0
    assert ref.nec_ex_card(ctx, 0, 2, 11, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0) == 0
    assert ref.nec_rp_card(ctx, 0, 1, 1, 1, 0, 0, 0, THETA, PHI, 0.0, 0.0, 0.0, 0.0) == 0
    v = np.array([ref.nec_impedance_real(ctx, 0), ref.nec_impedance_imag(ctx, 0), ref.nec_gain(ctx, 0, 0, 0)])
    ref.nec_delete(ctx)
    return v


def main():
    ref = RefAPI()
    p = yagi_params(0)
    v0 = outputs(ref, p)
    fd = np.zeros((3, len(p)))
    for k in range(len(p)):
        q = p.copy()
        q[k] += H
        vp = outputs(ref, q)
        q[k] -= 2 * H
        vm = outputs(ref, q)
        fd[:, k] = (vp - vm) / (2 * H)
    np.savez(os.path.join(HERE, "yagi_grad.npz"), params=p, value=v0, fd=fd, h=np.array(H))
    print("value", v0)
    print("fd", fd)


if __name__ == "__main__":
    main()
