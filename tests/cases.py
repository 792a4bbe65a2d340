"""Parity cases: NEC2++ C-API call sequences run identically against this
library and the reference build.  Each case is (builder, description); a
builder takes (api, ctx) and returns the frequency (MHz) of its last run.
"""
import numpy as np

from necpp_b200 import workloads as W


def _ex1(api, ctx):
    # reference testharness/python/test_examples.py:27-31 (example 1, unloaded part)
    api.nec_wire(ctx, 0, 7, 0., 0., .75, 0., 0., 1.25, .001, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 1)
    api.nec_ex_card(ctx, 0, 0, 4, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_xq_card(ctx, 0)
    return None


def _ex3_perfect(api, ctx):
    # test_examples.py:110-121 (example 3: EK, perfect ground)
    api.nec_wire(ctx, 0, 9, 0., 0.0, 2.0, 0.0, 0.0, 7.0, 0.03, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 1)
    api.nec_ek_card(ctx, 0)
    api.nec_fr_card(ctx, 0, 1, 30., 0)
    api.nec_ex_card(ctx, 0, 0, 5, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_gn_card(ctx, 1, 0, 0, 0, 0, 0, 0, 0)
    api.nec_rp_card(ctx, 0, 10, 2, 1, 3, 0, 1, 0.0, 0.0, 10.0, 90.0, 0, 0)
    return 30.0


def _ex3_finite(api, ctx):
    # test_examples.py:123-128 (example 3 continued: reflection-coefficient ground)
    _ex3_perfect(api, ctx)
    api.nec_gn_card(ctx, 0, 0, 6.0, 1.000E-03, 0, 0, 0, 0)
    api.nec_rp_card(ctx, 0, 10, 2, 1, 3, 0, 1, 0.0, 0.0, 10.0, 90.0, 0, 0)
    return 30.0


def _dipole(api, ctx):
    W.dipole(api, ctx)
    return 150.0


def _helix1(api, ctx):
    W.helix_array(api, ctx, k=1, seed=1)
    return 1000.0


def _helix2(api, ctx):
    W.helix_array(api, ctx, k=2, seed=2)
    return 1000.0


def _mesh_small(api, ctx):
    W.wire_mesh(api, ctx, nwires=11, nseg=10, side=1.0,
                pattern=(0, 19, 8, 1, 0, 0, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0))
    return 150.0


def _yagi(seed, nfreq=3):
    def build(api, ctx):
        p = W.yagi_params(np.random.default_rng(seed))
        W.yagi(api, ctx, p, nfreq=nfreq, pattern=(0, 19, 8, 1, 0, 0, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0))
        return 140.0 + (nfreq - 1) * 20.0 / 31.0
    return build


def _yagi_ground(api, ctx):
    W.yagi_ground(api, ctx, seed=5)
    return 145.0


def _yagi_ek_perfect(api, ctx):
    p = W.yagi_params(np.random.default_rng(7), n_elements=4, nseg=15)
    W.yagi(api, ctx, p, height=2.0, nfreq=1, f0=145.0, df=0.0, ground=(1, 0, 0, 0, 0, 0, 0, 0),
           pattern=(0, 10, 4, 1, 0, 0, 1, 0.0, 0.0, 10.0, 90.0, 0.0, 0.0))
    return 145.0


def _plane_wave_reflection(api, ctx):
    p = W.yagi_params(np.random.default_rng(11), n_elements=3, nseg=13)
    half, xs, rad, segs = p
    for e in range(len(half)):
        api.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, 3.0 - float(half[e]), float(xs[e]), 0.0,
                     3.0 + float(half[e]), float(rad[e]), 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    api.nec_gn_card(ctx, 0, 0, 10.0, 0.01, 0, 0, 0, 0)
    api.nec_fr_card(ctx, 0, 1, 145.0, 0.0)
    api.nec_ex_card(ctx, 1, 2, 2, 0, 60.0, 0.0, 30.0, 15.0, 90.0, 0.0)
    api.nec_rp_card(ctx, 0, 10, 4, 1, 0, 0, 0, 0.0, 0.0, 10.0, 90.0, 0.0, 0.0)
    return 145.0


def _yagi_loaded(api, ctx):
    """Every load type: series / parallel RLC (lumped and per metre), fixed
    impedance and wire conductivity, by tag, tag range and absolute segment
    numbers; two frequencies (the loads are recomputed per frequency)."""
    p = W.yagi_params(np.random.default_rng(3), n_elements=5, nseg=11)
    half, xs, rad, segs = p
    for e in range(len(half)):
        api.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                     float(half[e]), float(rad[e]), 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    api.nec_ld_card(ctx, 0, 2, 6, 6, 5.0, 2.0e-8, 3.0e-11)      # series RLC at the feed
    api.nec_ld_card(ctx, 1, 3, 4, 8, 1.0e3, 4.0e-7, 2.0e-12)    # parallel RLC, segments 4-8 of tag 3
    api.nec_ld_card(ctx, 2, 1, 0, 0, 0.5, 1.0e-7, 0.0)          # series per metre, all of tag 1
    api.nec_ld_card(ctx, 3, 4, 2, 3, 2.0e4, 1.0e-6, 1.0e-12)    # parallel per metre
    api.nec_ld_card(ctx, 4, 0, 50, 52, 3.0, -7.0, 0.0)          # fixed impedance, absolute segments 50-52
    api.nec_ld_card(ctx, 5, 5, 0, 0, 3.7e7, 0.0, 0.0)           # aluminium wire, tag 5
    api.nec_fr_card(ctx, 0, 2, 140.0, 10.0)
    api.nec_ex_card(ctx, 0, 2, 6, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    # directive gain: normalised by the radiated power, input minus load loss
    api.nec_rp_card(ctx, 0, 19, 8, 1, 0, 1, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0)
    return 150.0


def _dipoles_conductivity(api, ctx):
    """Wire conductivity in the three ranges of the internal-impedance
    approximation (x <= 8, 8 < x <= 110, x > 110) on three dipoles."""
    for t, sig in enumerate((1.0e4, 5.0e5, 5.8e7)):
        api.nec_wire(ctx, t + 1, 21, 0.8 * t, 0.0, -0.5, 0.8 * t, 0.0, 0.5, 1.0e-3, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    for t, sig in enumerate((1.0e4, 5.0e5, 5.8e7)):
        api.nec_ld_card(ctx, 5, t + 1, 0, 0, sig, 0.0, 0.0)
    api.nec_fr_card(ctx, 0, 1, 150.0, 0.0)
    api.nec_ex_card(ctx, 0, 2, 11, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_rp_card(ctx, 0, 19, 8, 1, 0, 0, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0)
    return 150.0


def _array_tl(api, ctx):
    """Three dipoles fed through transmission lines from a source on the
    first: a straight line of given length from the source, a crossed line
    of computed length (0) with shunt admittances, and an NT two-port
    between two non-source ports; two frequencies."""
    for t in range(3):
        api.nec_wire(ctx, t + 1, 21, 0.5 * t, 0.0, -0.48, 0.5 * t, 0.0, 0.48, 1.0e-3, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    api.nec_tl_card(ctx, 1, 11, 2, 11, 50.0, 0.6, 0.0, 0.0, 0.0, 0.0)
    api.nec_tl_card(ctx, 2, 11, 3, 11, -75.0, 0.0, 1.0e-3, 2.0e-3, 0.0, -1.0e-3)
    api.nec_nt_card(ctx, 2, 4, 3, 18, 2.0e-3, -1.0e-3, -5.0e-4, 2.0e-4, 1.0e-3, 3.0e-3)
    api.nec_fr_card(ctx, 0, 2, 145.0, 10.0)
    api.nec_ex_card(ctx, 0, 1, 11, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_rp_card(ctx, 0, 19, 8, 1, 0, 1, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0)
    return 150.0


def _dipole_nt(api, ctx):
    """A two-port network between two segments of a driven dipole, the
    source off the network (the plain input path with network loss)."""
    api.nec_wire(ctx, 1, 31, 0.0, 0.0, -0.5, 0.0, 0.0, 0.5, 1.0e-3, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    api.nec_nt_card(ctx, 1, 6, 1, 26, 1.0e-2, 5.0e-3, -2.0e-3, 1.0e-3, 4.0e-3, -6.0e-3)
    api.nec_fr_card(ctx, 0, 1, 150.0, 0.0)
    api.nec_ex_card(ctx, 0, 1, 16, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_rp_card(ctx, 0, 19, 8, 1, 0, 1, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0)
    return 150.0


def _near_ground(api, ctx):
    """A dipole 0.05 wavelength above Sommerfeld ground and a tilted wire
    touching down near it: most pairs are within a wavelength of their
    image, so the fill integrates the interpolated Sommerfeld tables; two
    frequencies (new tables, the interpolation cache carried over)."""
    api.nec_wire(ctx, 1, 21, -0.5, 0.0, 0.1, 0.5, 0.0, 0.1, 1.0e-3, 1.0, 1.0)
    api.nec_wire(ctx, 2, 9, 0.6, 0.0, 0.05, 0.6, 0.3, 0.4, 1.0e-3, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 1)
    api.nec_gn_card(ctx, 2, 0, 10.0, 0.01, 0, 0, 0, 0)
    api.nec_fr_card(ctx, 0, 2, 150.0, 12.0)
    api.nec_ex_card(ctx, 0, 1, 11, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    # near field over the ground at both frequencies: its table reads move
    # the interpolation cache the next fill starts from
    api.nec_ne_card(ctx, 0, 3, 2, 2, -0.4, 0.1, 0.02, 0.4, 0.2, 0.15)
    api.nec_rp_card(ctx, 0, 10, 4, 1, 0, 0, 0, 0.0, 0.0, 10.0, 90.0, 0.0, 0.0)
    return 150.0


def _dipole_fields(api, ctx):
    """Near electric field on a rectangular grid through and around a
    dipole (points inside a segment's volume included) and the magnetic
    field on a spherical grid, free space."""
    api.nec_wire(ctx, 1, 21, 0.0, 0.0, -0.5, 0.0, 0.0, 0.5, 1.0e-3, 1.0, 1.0)
    api.nec_geometry_complete(ctx, 0)
    api.nec_fr_card(ctx, 0, 1, 150.0, 0.0)
    api.nec_ex_card(ctx, 0, 1, 11, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_ne_card(ctx, 0, 4, 3, 5, 0.0, -0.0005, -0.6, 0.1, 0.0005, 0.3)
    api.nec_nh_card(ctx, 1, 3, 4, 3, 0.8, 0.0, 10.0, 0.5, 30.0, 40.0)
    api.nec_rp_card(ctx, 0, 10, 4, 1, 0, 0, 0, 0.0, 0.0, 20.0, 90.0, 0.0, 0.0)
    return 150.0


def _yagi_fields_ground(api, ctx, gn):
    p = W.yagi_params(np.random.default_rng(17), n_elements=3, nseg=11)
    half, xs, rad, segs = p
    for e in range(len(half)):
        api.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, 1.5 - float(half[e]), float(xs[e]), 0.0,
                     1.5 + float(half[e]), float(rad[e]), 1.0, 1.0)
    api.nec_geometry_complete(ctx, 1)
    api.nec_gn_card(ctx, *gn)
    api.nec_fr_card(ctx, 0, 1, 145.0, 0.0)
    api.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    api.nec_ne_card(ctx, 0, 3, 2, 4, -0.5, 0.3, 0.2, 0.6, 0.5, 0.7)
    api.nec_nh_card(ctx, 0, 3, 2, 4, -0.5, 0.3, 0.2, 0.6, 0.5, 0.7)
    api.nec_rp_card(ctx, 0, 10, 4, 1, 0, 0, 0, 0.0, 0.0, 10.0, 90.0, 0.0, 0.0)
    return 145.0


def _yagi_fields_reflection(api, ctx):
    """Near E and H over a finite ground in the reflection-coefficient
    approximation (the image terms of efld and hsfld)."""
    return _yagi_fields_ground(api, ctx, (0, 0, 13.0, 0.005, 0, 0, 0, 0))


def _yagi_fields_perfect(api, ctx):
    return _yagi_fields_ground(api, ctx, (1, 0, 0, 0, 0, 0, 0, 0))


# name: (builder, pattern grid (n_theta, n_phi) or None)
CASES = {
    "ex1": (_ex1, None),
    "ex3_perfect": (_ex3_perfect, (10, 2)),
    "ex3_finite": (_ex3_finite, (10, 2)),
    "dipole": (_dipole, (91, 72)),
    "helix1": (_helix1, (91, 72)),
    "helix2": (_helix2, (91, 72)),
    "mesh_small": (_mesh_small, (19, 8)),
    "yagi_s1": (_yagi(1), (19, 8)),
    "yagi_s2": (_yagi(2), (19, 8)),
    "yagi_ground": (_yagi_ground, (1, 1)),
    "yagi_ek_perfect": (_yagi_ek_perfect, (10, 4)),
    "plane_wave_reflection": (_plane_wave_reflection, (10, 4)),
    "yagi_loaded": (_yagi_loaded, (19, 8)),
    "dipoles_conductivity": (_dipoles_conductivity, (19, 8)),
    "array_tl": (_array_tl, (19, 8)),
    "dipole_nt": (_dipole_nt, (19, 8)),
    "near_ground": (_near_ground, (10, 4)),
    "dipole_fields": (_dipole_fields, (10, 4)),
    "yagi_fields_reflection": (_yagi_fields_reflection, (10, 4)),
    "yagi_fields_perfect": (_yagi_fields_perfect, (10, 4)),
}


def _helix_array_8x8(api, ctx):
    """The benchmark workload: 8 x 8 axial-mode helix array, N = 11520,
    1 GHz, 64 feeds with seeded phases (seed 0), 91 x 72 pattern."""
    W.helix_array(api, ctx, k=8, seed=0)
    return 1000.0


def _wire_mesh_41(api, ctx):
    """Square wire mesh, 41 + 41 wires of 40 segments (N = 3280, 4-way
    junctions at the crossings), 150 MHz, plane wave at theta 30 deg,
    theta-polarised, bistatic 181 x 72 pattern."""
    W.wire_mesh(api, ctx)
    return 150.0


# full-size workloads: compact fixtures (no full Z, no host tables)
LARGE_CASES = {
    "helix_array_8x8": (_helix_array_8x8, (91, 72)),
    "wire_mesh_41": (_wire_mesh_41, (181, 72)),
}
