"""Batched sweeps on the GPU: many small structures solved in one pass
(necgpu_batch_solve): an FR-card frequency sweep of several designs, or an
optimiser's population.

    res = sweep(problems, theta, phi)   # res["zin"], res["gain"], ...

`problems` is a list of (structure, rhs, feed, voltage, wavelength) tuples
as produced by `host_problem(ctx, freq_mhz, feed_tag, feed_seg)`, built on
the host through the C API (geometry and excitation cards, no solve).
`yagi_sweep()` builds the seeded Yagi-Uda sweep (256 variants x 32
frequencies) and solves it.
"""
import ctypes as _C
import math as _math
import os as _os

import numpy as _np

from . import lib, nec_create, nec_delete, nec_error_message, structure, rhs as _rhs

_dp = _C.POINTER(_C.c_double)
_ip = _C.POINTER(_C.c_int32)

# wave impedance and light speed as the host library computes them
# (truncated pi, mu0 = 4 pi 1e-7, eps0 = 8.854e-12)
_PI = 3.1415926536
_C0 = 1.0 / _math.sqrt(4.0 * _PI * 1e-7 * 8.854e-12)


class NecgpuStructure(_C.Structure):
    """ctypes mirror of necgpu_structure (include/necgpu.h)."""
    _fields_ = [("n", _C.c_int64)] + [(k, _dp) for k in ("x", "y", "z", "length", "radius", "cab", "sab", "salp")] + [
        ("trio_ptr", _ip), ("trio_basis", _ip), ("trio_a", _dp), ("trio_b", _dp), ("trio_c", _dp),
        ("ek_ind1", _ip), ("ek_ind2", _ip), ("rkh", _C.c_double), ("use_exk", _C.c_int32), ("ground", _C.c_int32),
        ("zrati_re", _C.c_double), ("zrati_im", _C.c_double), ("frati_re", _C.c_double), ("frati_im", _C.c_double),
        ("eta", _C.c_double)]


def to_struct(st):
    """NecgpuStructure over the arrays of a structure() dict (kept alive by
    the returned tuple)."""
    n = st["n"]
    s = NecgpuStructure()
    s.n = n
    seg = st["seg"]
    for k, name in enumerate(("x", "y", "z", "length", "radius", "cab", "sab", "salp")):
        setattr(s, name, seg[k * n:(k + 1) * n].ctypes.data_as(_dp))
    nt = len(st["tbasis"])
    abc = st["tabc"]
    s.trio_ptr = st["tptr"].ctypes.data_as(_ip)
    s.trio_basis = st["tbasis"].ctypes.data_as(_ip)
    s.trio_a = abc[:nt].ctypes.data_as(_dp)
    s.trio_b = abc[nt:2 * nt].ctypes.data_as(_dp)
    s.trio_c = abc[2 * nt:].ctypes.data_as(_dp)
    s.ek_ind1 = st["ind"][:n].ctypes.data_as(_ip)
    s.ek_ind2 = st["ind"][n:].ctypes.data_as(_ip)
    p = st["params"]
    s.rkh, s.use_exk, s.ground = p[0], int(p[1]), int(p[2])
    s.zrati_re, s.zrati_im, s.frati_re, s.frati_im, s.eta = p[3], p[4], p[5], p[6], p[7]
    return s, st


def _struct_dtype():
    """numpy record layout of necgpu_structure (offsets from the ctypes mirror)."""
    names, formats, offsets = [], [], []
    for name, ctype in NecgpuStructure._fields_:
        names.append(name)
        offsets.append(getattr(NecgpuStructure, name).offset)
        if ctype is _C.c_int64:
            formats.append(_np.int64)
        elif ctype is _C.c_int32:
            formats.append(_np.int32)
        elif ctype is _C.c_double:
            formats.append(_np.float64)
        else:
            formats.append(_np.uint64)  # pointer
    return _np.dtype({"names": names, "formats": formats, "offsets": offsets,
                      "itemsize": _C.sizeof(NecgpuStructure)})


_SDT = None


def struct_array(structs):
    """A contiguous array of necgpu_structure over structure() dicts (the
    dicts must outlive its use)."""
    global _SDT
    if _SDT is None:
        _SDT = _struct_dtype()
    out = _np.zeros(len(structs), dtype=_SDT)
    addr = lambda a: a.__array_interface__["data"][0]
    for k, st in enumerate(structs):
        n = st["n"]
        seg, tabc, ind = addr(st["seg"]), addr(st["tabc"]), addr(st["ind"])
        nt = len(st["tbasis"])
        p = st["params"]
        out[k] = (n, seg, seg + 8 * n, seg + 16 * n, seg + 24 * n, seg + 32 * n, seg + 40 * n, seg + 48 * n,
                  seg + 56 * n, addr(st["tptr"]), addr(st["tbasis"]), tabc, tabc + 8 * nt, tabc + 16 * nt, ind,
                  ind + 4 * n, p[0], int(p[1]), int(p[2]), p[3], p[4], p[5], p[6], p[7])
    return out


def host_problem(ctx, freq_mhz, feed_index, voltage=1.0 + 0j):
    """Tables and right-hand side of context ctx at freq_mhz (host only);
    feed_index: 0-based segment of the voltage source."""
    st = structure(ctx, freq_mhz)
    if _np.any(st["zload"] != 0):
        raise ValueError("batched sweeps do not carry impedance loading (LD cards)")
    if st["networks"]:
        raise ValueError("batched sweeps do not carry networks or transmission lines (NT/TL cards)")
    b = _rhs(ctx)
    return st, b, int(feed_index), complex(voltage), _C0 / (freq_mhz * 1e6)


_engine = None


def _get_engine():
    global _engine
    if _engine is None:
        lib.necgpu_create.argtypes = [_C.POINTER(_C.c_void_p), _C.c_int]
        lib.necgpu_last_error.restype = _C.c_char_p
        lib.necgpu_last_error.argtypes = [_C.c_void_p]
        lib.necgpu_batch_solve.argtypes = [_C.c_void_p, _C.c_int, _C.c_void_p, _C.c_void_p, _C.c_void_p,
                                           _C.c_void_p, _C.c_void_p, _C.c_int, _C.c_void_p, _C.c_void_p,
                                           _C.c_void_p, _C.c_void_p, _C.c_void_p, _C.c_void_p, _C.c_void_p,
                                           _C.c_void_p]
        h = _C.c_void_p()
        dev = int(_os.environ.get("NECPP_B200_DEVICE", "0"))
        rc = lib.necgpu_create(_C.byref(h), dev)
        if rc != 0:
            raise RuntimeError("necgpu_create: %s" % lib.necgpu_last_error(h))
        _engine = h
    return _engine


def sweep(problems, theta=None, phi=None, fields=False):
    """Solve every problem.  Returns a dict: zin (complex per problem),
    cur (all problems' segment currents in amperes, concatenated) with
    offsets, gain (nprob x ndir float32 power gain in dB, normalised by each
    problem's one voltage source), eth / eph (complex fields, only with
    fields=True), status and residual."""
    eng = _get_engine()
    nprob = len(problems)
    for p in problems:  # the structure array points into these arrays
        st = p[0]
        for key in ("seg", "tabc", "ind", "tptr", "tbasis"):
            if not st[key].flags["C_CONTIGUOUS"]:
                st[key] = _np.ascontiguousarray(st[key])
    arr = struct_array([p[0] for p in problems])
    ns = _np.fromiter((p[0]["n"] for p in problems), dtype=_np.int64, count=nprob)
    off = _np.concatenate([[0], _np.cumsum(ns)])
    rhs = _np.concatenate([_np.asarray(p[1], dtype=_np.complex128) for p in problems])
    feed = _np.fromiter((p[2] for p in problems), dtype=_np.int32, count=nprob)
    volt = _np.array([p[3] for p in problems], dtype=_np.complex128)
    lam = _np.fromiter((p[4] for p in problems), dtype=_np.float64, count=nprob)
    cur = _np.zeros(off[-1], dtype=_np.complex128)
    th = _np.ascontiguousarray(theta if theta is not None else [], dtype=_np.float64)
    ph = _np.ascontiguousarray(phi if phi is not None else [], dtype=_np.float64)
    ndir = len(th)
    gain = _np.zeros((nprob, max(ndir, 1)), dtype=_np.float32)
    eth = eph = None
    if fields and ndir:
        eth = _np.zeros((nprob, ndir), dtype=_np.complex128)
        eph = _np.zeros((nprob, ndir), dtype=_np.complex128)
    status = _np.zeros(nprob, dtype=_np.int32)
    resid = _np.zeros(nprob)
    rc = lib.necgpu_batch_solve(eng, nprob, arr.ctypes.data, rhs.ctypes.data, feed.ctypes.data,
                                volt.ctypes.data, lam.ctypes.data, ndir, th.ctypes.data, ph.ctypes.data,
                                cur.ctypes.data, gain.ctypes.data if ndir else None,
                                eth.ctypes.data if eth is not None else None,
                                eph.ctypes.data if eph is not None else None, status.ctypes.data, resid.ctypes.data)
    if rc != 0:
        raise RuntimeError("necgpu_batch_solve: %s" % lib.necgpu_last_error(eng).decode())
    cur_amps = cur * _np.repeat(lam, ns)
    zin = volt / cur_amps[off[:-1] + feed]
    return {"zin": zin, "cur": cur_amps, "offsets": off, "gain": gain[:, :ndir], "eth": eth, "eph": eph,
            "status": status, "residual": resid}


def yagi_problems(nvariants=256, nfreq=32, f0=140.0, f1=160.0, seed=0):
    """The seeded Yagi-Uda sweep: nvariants designs (3-15 elements, 11-41
    segments each, half lengths 0.40-0.55 m, spacings 0.1-0.7 m, radii
    0.5-3 mm, element 2 centre-fed with 1 V) at nfreq frequencies from f0 to
    f1 MHz.  Returns (problems, per-problem (variant, frequency) labels)."""
    from . import workloads as W
    from . import nec_wire, nec_geometry_complete, nec_ex_card
    rng = _np.random.default_rng(seed)
    freqs = _np.linspace(f0, f1, nfreq)
    problems, labels = [], []
    for v in range(nvariants):
        half, xs, rad, segs = W.yagi_params(rng)
        ctx = nec_create()
        try:
            for e in range(len(half)):
                if nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                            float(half[e]), float(rad[e]), 1.0, 1.0) != 0:
                    raise RuntimeError(nec_error_message())
            nec_geometry_complete(ctx, 0)
            nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
            feed = int(segs[0]) + (int(segs[1]) + 1) // 2 - 1
            for f in freqs:
                problems.append(host_problem(ctx, float(f), feed))
                labels.append((v, float(f)))
        finally:
            nec_delete(ctx)
    return problems, labels


def pattern_grid(nth=91, nph=72, dth=2.0, dph=5.0):
    """Directions (radians) of the RP grid theta 0..180 step 2, phi 0..355
    step 5, theta fastest (the reference's cell order)."""
    th = _np.radians(_np.arange(nth) * dth)
    ph = _np.radians(_np.arange(nph) * dph)
    T, P = _np.meshgrid(th, ph)
    return T.ravel(), P.ravel()
