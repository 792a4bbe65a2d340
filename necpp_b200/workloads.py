"""Seeded synthetic workloads of the thin-wire hot path, as NEC2++ C-API call
sequences.

Each builder takes an ``api`` object exposing the C-API names (``nec_wire``,
``nec_geometry_complete``, ...) plus ``helix(ctx, ...)`` and drives a context
to the point where the hot path has run.  The same sequence drives this
library and the reference build, so their results are directly comparable.

Workloads (sizes as stated):
  dipole        centre-fed straight dipole, 1.0 m, radius 1 mm, 51 segments,
                150 MHz, 1 V on segment 26, 91 x 72 pattern (N = 51)
  wire_mesh     square mesh 2 m side, 41 + 41 wires of 40 segments, radius
                1 mm, 150 MHz, plane wave theta=30 phi=0 theta-polarised,
                181 x 72 bistatic pattern (N = 3280)
  helix_array   k x k axial-mode helices on 0.5 m pitch, 6 turns,
                circumference 0.3 m, pitch angle 12.5 deg, wire radius 1 mm,
                180 segments per helix, 1 GHz, each fed at its base segment
                with 1 V at a seeded uniform phase, 91 x 72 pattern
                (k = 8: N = 11520)
  yagi          seeded Yagi-Uda variant (3-15 elements parallel to z, half
                lengths 0.40-0.55 m, spacings 0.1-0.7 m, radii 0.5-3 mm, odd
                11-41 segments per element), element 2 centre-fed with 1 V,
                swept over 32 frequencies 140-160 MHz, 91 x 72 pattern
  yagi_ground   9-element seeded Yagi (21 segments per element) at 10 m over
                Sommerfeld ground (eps_r 13, sigma 0.005), 145 MHz, gain at
                theta=80 phi=0 (N = 189)
"""
import math

import numpy as np

PATTERN_91x72 = (0, 91, 72, 1, 0, 0, 0, 0.0, 0.0, 2.0, 5.0, 0.0, 0.0)


def _check(api, ctx, r, what):
    if r != 0:
        raise RuntimeError("%s failed: %s" % (what, api.nec_error_message()))


def dipole(api, ctx, pattern=PATTERN_91x72):
    c = lambda r, w: _check(api, ctx, r, w)
    c(api.nec_wire(ctx, 1, 51, 0.0, 0.0, -0.5, 0.0, 0.0, 0.5, 1e-3, 1.0, 1.0), "wire")
    c(api.nec_geometry_complete(ctx, 0), "geometry_complete")
    c(api.nec_fr_card(ctx, 0, 1, 150.0, 0.0), "fr")
    c(api.nec_ex_card(ctx, 0, 1, 26, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0), "ex")
    if pattern is not None:
        c(api.nec_rp_card(ctx, *pattern), "rp")
    else:
        c(api.nec_xq_card(ctx, 0), "xq")
    return 51


def wire_mesh(api, ctx, nwires=41, nseg=40, side=2.0, pattern=(0, 181, 72, 1, 0, 0, 0, 0.0, 0.0, 1.0, 5.0, 0.0, 0.0)):
    c = lambda r, w: _check(api, ctx, r, w)
    h = side / 2.0
    step = side / (nwires - 1)
    for k in range(nwires):
        y = -h + step * k
        c(api.nec_wire(ctx, k + 1, nseg, -h, y, 0.0, h, y, 0.0, 1e-3, 1.0, 1.0), "wire")
    for k in range(nwires):
        x = -h + step * k
        c(api.nec_wire(ctx, nwires + k + 1, nseg, x, -h, 0.0, x, h, 0.0, 1e-3, 1.0, 1.0), "wire")
    c(api.nec_geometry_complete(ctx, 0), "geometry_complete")
    c(api.nec_fr_card(ctx, 0, 1, 150.0, 0.0), "fr")
    c(api.nec_ex_card(ctx, 1, 1, 1, 0, 30.0, 0.0, 0.0, 0.0, 0.0, 0.0), "ex")
    if pattern is not None:
        c(api.nec_rp_card(ctx, *pattern), "rp")
    else:
        c(api.nec_xq_card(ctx, 0), "xq")
    return 2 * nwires * nseg


def helix_geometry():
    circ = 0.3
    a = circ / (2.0 * math.pi)
    s = circ * math.tan(math.radians(12.5))
    return a, s, 6.0 * s


def helix_array(api, ctx, k=8, seed=0, nseg=180, pattern=PATTERN_91x72, freq_mhz=1000.0, execute=True):
    """execute=False stops after the EX cards (no XQ or RP card)."""
    c = lambda r, w: _check(api, ctx, r, w)
    a, s, hl = helix_geometry()
    c(api.helix(ctx, 1, nseg, s, hl, a, a, a, a, 1e-3), "helix")
    if k > 1:
        c(api.nec_gm_card(ctx, 1, k - 1, 0.0, 0.0, 0.0, 0.5, 0.0, 0.0, 1), "gm x")
        c(api.nec_gm_card(ctx, k, k - 1, 0.0, 0.0, 0.0, 0.0, 0.5, 0.0, 1), "gm y")
    c(api.nec_geometry_complete(ctx, 0), "geometry_complete")
    c(api.nec_fr_card(ctx, 0, 1, freq_mhz, 0.0), "fr")
    phases = np.random.default_rng(seed).uniform(0.0, 2.0 * math.pi, size=k * k)
    for t in range(k * k):
        c(api.nec_ex_card(ctx, 0, t + 1, 1, 0, math.cos(phases[t]), math.sin(phases[t]), 0.0, 0.0, 0.0, 0.0), "ex")
    if not execute:
        return k * k * nseg
    if pattern is not None:
        c(api.nec_rp_card(ctx, *pattern), "rp")
    else:
        c(api.nec_xq_card(ctx, 0), "xq")
    return k * k * nseg


def yagi_params(rng, n_elements=None, nseg=None):
    """Draw one Yagi variant: (half_lengths, x_positions, radii, segments)."""
    n = int(rng.integers(3, 16)) if n_elements is None else n_elements
    half, xs, rad, segs = [], [], [], []
    x = 0.0
    for e in range(n):
        hl = rng.uniform(0.40, 0.55)
        sp = rng.uniform(0.1, 0.7)
        r = rng.uniform(0.5e-3, 3e-3)
        sg = int(rng.integers(5, 21)) * 2 + 1
        if e > 0:
            x += sp
        half.append(hl)
        xs.append(x)
        rad.append(r)
        segs.append(sg if nseg is None else nseg)
    return np.array(half), np.array(xs), np.array(rad), np.array(segs, dtype=int)


def yagi(api, ctx, params, height=0.0, nfreq=32, f0=140.0, df=20.0 / 31.0, ground=None,
         pattern=PATTERN_91x72):
    c = lambda r, w: _check(api, ctx, r, w)
    half, xs, rad, segs = params
    for e in range(len(half)):
        c(api.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, height - float(half[e]),
                       float(xs[e]), 0.0, height + float(half[e]), float(rad[e]), 1.0, 1.0), "wire")
    c(api.nec_geometry_complete(ctx, 0), "geometry_complete")
    if ground is not None:
        c(api.nec_gn_card(ctx, *ground), "gn")
    c(api.nec_fr_card(ctx, 0, nfreq, f0, df), "fr")
    c(api.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0), "ex")
    if pattern is not None:
        c(api.nec_rp_card(ctx, *pattern), "rp")
    else:
        c(api.nec_xq_card(ctx, 0), "xq")
    return int(np.sum(segs))


def yagi_ground(api, ctx, seed=0):
    params = yagi_params(np.random.default_rng(seed), n_elements=9, nseg=21)
    return yagi(api, ctx, params, height=10.0, nfreq=1, f0=145.0, df=0.0,
                ground=(2, 0, 13.0, 0.005, 0.0, 0.0, 0.0, 0.0),
                pattern=(0, 1, 1, 1, 0, 0, 0, 80.0, 0.0, 0.0, 0.0, 0.0, 0.0))


def yagi_ground_cards(api, ctx, p, nseg=21, height=10.0, ground=(2, 0, 13.0, 0.005, 0.0, 0.0, 0.0, 0.0)):
    """Cards of the 9-element Yagi over Sommerfeld ground without frequency
    or solve: p = (half lengths [m], x positions [m], radii [m]), element 2
    centre-fed with 1 V.  For adjoint gradients (necpp_b200.adjoint)."""
    c = lambda r, w: _check(api, ctx, r, w)
    p = np.asarray(p, dtype=float)
    ne = len(p) // 3
    half, xs, rad = p[:ne], p[ne:2 * ne], p[2 * ne:]
    for e in range(ne):
        c(api.nec_wire(ctx, e + 1, nseg, float(xs[e]), 0.0, height - float(half[e]), float(xs[e]), 0.0,
                       height + float(half[e]), float(rad[e]), 1.0, 1.0), "wire")
    c(api.nec_geometry_complete(ctx, 0), "geometry_complete")
    if ground is not None:
        c(api.nec_gn_card(ctx, *ground), "gn")
    c(api.nec_ex_card(ctx, 0, 2, (nseg + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0), "ex")
    return ne * nseg


def yagi_ground_params(seed=0):
    """The 27 parameters of the seeded 9-element Yagi (config of yagi_ground)."""
    half, xs, rad, _ = yagi_params(np.random.default_rng(seed), n_elements=9, nseg=21)
    return np.concatenate([half, xs, rad])
