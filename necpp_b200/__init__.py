"""necpp_b200 -- B200 thin-wire method-of-moments hot path behind the NEC2++ C API.

Python binding of libnecpp_b200.so through ctypes.  The functions keep the
names and argument order of the NEC2++ C API (src/libnecpp.h), which is what
the reference's own Python wrapper exposes, so code written against
``necpp`` runs unchanged::

    from necpp_b200 import *
    nec = nec_create()
    nec_wire(nec, 1, 51, 0, 0, -0.5, 0, 0, 0.5, 1e-3, 1, 1)
    nec_geometry_complete(nec, 0)
    nec_fr_card(nec, 0, 1, 150.0, 0)
    nec_ex_card(nec, 0, 1, 26, 0, 1.0, 0, 0, 0, 0, 0)
    nec_rp_card(nec, 0, 91, 72, 1, 0, 0, 0, 0, 0, 2, 5, 0, 0)
    zin = complex(nec_impedance_real(nec, 0), nec_impedance_imag(nec, 0))

The fill, factorisation, solve and far-field sum run on the GPU; there is no
CPU path.  Loading fails loudly when the shared library is missing.
"""
import ctypes as _C
import os as _os

import numpy as _np

_HERE = _os.path.dirname(_os.path.abspath(__file__))
_LIBPATH = _os.path.join(_HERE, "libnecpp_b200.so")

if not _os.path.exists(_LIBPATH):
    raise ImportError(
        "libnecpp_b200.so is not built (run python necpp_b200/build.py or "
        "__graft_entry__.build()); there is no CPU fallback")

lib = _C.CDLL(_LIBPATH)

_d = _C.c_double
_i = _C.c_int
_l = _C.c_long
_p = _C.c_void_p
_dp = _C.POINTER(_C.c_double)
_ip = _C.POINTER(_C.c_int)


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("nec_create", _p, [])
_sig("nec_delete", _l, [_p])
_sig("nec_error_message", _C.c_char_p, [])
_sig("nec_wire", _l, [_p, _i, _i] + [_d] * 9)
_sig("nec_helix", _l, [_p, _i, _i] + [_d] * 7)
_sig("nec_gm_card", _l, [_p, _i, _i] + [_d] * 6 + [_i])
_sig("nec_geometry_complete", _l, [_p, _i])
_sig("nec_medium_parameters", _l, [_p, _d, _d])
_sig("nec_gn_card", _l, [_p, _i, _i] + [_d] * 6)
_sig("nec_fr_card", _l, [_p, _i, _i, _d, _d])
_sig("nec_ek_card", _l, [_p, _i])
_sig("nec_ld_card", _l, [_p, _i, _i, _i, _i, _d, _d, _d])
_sig("nec_ex_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
_sig("nec_excitation_voltage", _l, [_p, _i, _i, _d, _d])
_sig("nec_excitation_current", _l, [_p] + [_d] * 6)
_sig("nec_excitation_planewave", _l, [_p, _i, _i] + [_d] * 6)
_sig("nec_xq_card", _l, [_p, _i])
_sig("nec_rp_card", _l, [_p] + [_i] * 7 + [_d] * 6)
_sig("nec_pt_card", _l, [_p, _i, _i, _i, _i])
_sig("nec_pq_card", _l, [_p, _i, _i, _i, _i])
_sig("nec_kh_card", _l, [_p, _d])
for _name in ("nec_sp_card", "nec_sc_card"):
    _sig(_name, _l, [_p, _i] + [_d] * 6)
_sig("nec_gx_card", _l, [_p, _i, _i])
_sig("nec_tl_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
_sig("nec_nt_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
_sig("nec_ne_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
_sig("nec_nh_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
_sig("nec_gd_card", _l, [_p] + [_d] * 4)
_sig("nec_cp_card", _l, [_p, _i, _i, _i, _i])
_sig("nec_gain", _d, [_p, _i, _i, _i])
for _stat in ("max", "min", "mean", "sd"):
    for _pre in ("nec_gain_", "nec_gain_rhcp_", "nec_gain_lhcp_"):
        _sig(_pre + _stat, _d, [_p, _i])
_sig("nec_impedance_real", _d, [_p, _i])
_sig("nec_impedance_imag", _d, [_p, _i])
_sig("nec_impedance_real_indexed", _d, [_p, _i, _i])
_sig("nec_impedance_imag_indexed", _d, [_p, _i, _i])
_sig("nec_set_precision", _l, [_p, _i])
_sig("nec_set_intersection_check", _l, [_p, _i, _i])
_sig("nec_segment_count", _l, [_p])
_sig("nec_frequency_scale", _l, [_p, _d])
_sig("nec_get_currents", _l, [_p, _i, _dp, _l])
_sig("nec_get_segments", _l, [_p] + [_dp] * 8 + [_ip] * 3)
_sig("nec_get_trio", _l, [_p, _i, _ip, _dp, _dp, _dp, _l])
_sig("nec_last_refinement", _l, [_p, _ip, _dp])
_sig("nec_get_loads", _l, [_p, _dp])
_sig("nec_network_count", _l, [_p])
_sig("nec_near_field", _l, [_p, _i, _C.POINTER(_i), _dp, _dp])
_sig("nec_gradient", _l, [_p, _i, _C.POINTER(_p), _C.POINTER(_p), _dp, _d, _d, _dp, _dp])
_sig("nec_prepare_structure", _l, [_p, _d])
_sig("nec_get_structure", _l, [_p, _dp, _ip, _ip, _dp, _ip, _dp])
_sig("nec_gpu_engine", _p, [_p])
_sig("nec_get_rhs", _l, [_p, _dp])
_sig("nec_get_pattern_fields", _l, [_p, _i, _dp, _dp, _l])


def _wrap(name):
    f = getattr(lib, name)

    def call(*args):
        return f(*args)

    call.__name__ = name
    return call


_PUBLIC = [
    "nec_create", "nec_delete", "nec_wire", "nec_helix", "nec_gm_card", "nec_geometry_complete",
    "nec_medium_parameters", "nec_gn_card", "nec_fr_card", "nec_ek_card", "nec_ld_card",
    "nec_ex_card", "nec_excitation_voltage", "nec_excitation_current", "nec_excitation_planewave",
    "nec_xq_card", "nec_rp_card", "nec_pt_card", "nec_pq_card", "nec_kh_card", "nec_sp_card",
    "nec_sc_card", "nec_gx_card", "nec_tl_card", "nec_nt_card", "nec_ne_card", "nec_nh_card",
    "nec_gd_card", "nec_cp_card", "nec_gain", "nec_impedance_real", "nec_impedance_imag",
    "nec_impedance_real_indexed", "nec_impedance_imag_indexed", "nec_set_precision",
    "nec_set_intersection_check", "nec_segment_count", "nec_frequency_scale", "nec_network_count",
] + [p + s for s in ("max", "min", "mean", "sd")
     for p in ("nec_gain_", "nec_gain_rhcp_", "nec_gain_lhcp_")]

for _n in _PUBLIC:
    globals()[_n] = _wrap(_n)


def nec_error_message():
    m = lib.nec_error_message()
    return m.decode() if m else ""


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


def segments(nec):
    """Segment tables after geometry_complete (metres) as a dict of arrays."""
    n = lib.nec_segment_count(nec)
    arr = {k: _np.zeros(n) for k in ("x", "y", "z", "si", "bi", "cab", "sab", "salp")}
    ints = {k: _np.zeros(n, dtype=_np.int32) for k in ("tags", "icon1", "icon2")}
    r = lib.nec_get_segments(nec, *[_dptr(arr[k]) for k in ("x", "y", "z", "si", "bi", "cab", "sab", "salp")],
                             *[_iptr(ints[k]) for k in ("tags", "icon1", "icon2")])
    if r < 0:
        raise RuntimeError("geometry not complete")
    arr.update(ints)
    return arr


def trio(nec, j, cap=64):
    """Basis table of source segment j (1-based) at the last scaling."""
    jco = _np.zeros(cap, dtype=_np.int32)
    ax, bx, cx = _np.zeros(cap), _np.zeros(cap), _np.zeros(cap)
    k = lib.nec_get_trio(nec, j, _iptr(jco), _dptr(ax), _dptr(bx), _dptr(cx), cap)
    if k < 0:
        raise RuntimeError(nec_error_message())
    return jco[:k].copy(), ax[:k].copy(), bx[:k].copy(), cx[:k].copy()


def currents(nec, index=0):
    """Segment-centre currents (amperes, complex) of result index."""
    n = lib.nec_segment_count(nec)
    out = _np.zeros(2 * n)
    k = lib.nec_get_currents(nec, index, _dptr(out), 2 * n)
    if k < 0:
        raise IndexError("no currents for index %d" % index)
    return out[0::2] + 1j * out[1::2]


def pattern_fields(nec, index, n_cells):
    eth = _np.zeros(2 * n_cells)
    eph = _np.zeros(2 * n_cells)
    k = lib.nec_get_pattern_fields(nec, index, _dptr(eth), _dptr(eph), n_cells)
    if k < 0:
        raise IndexError("no pattern for index %d" % index)
    return eth[0::2] + 1j * eth[1::2], eph[0::2] + 1j * eph[1::2]


def near_fields(nec):
    """Every near-field pattern of the context: list of (nfeh, points (m,
    np x 3), fields (np x 3 complex))."""
    out = []
    k = 0
    while True:
        nfeh = _i(0)
        np_ = lib.nec_near_field(nec, k, _C.byref(nfeh), None, None)
        if np_ < 0:
            return out
        xyz, f = _np.zeros(3 * np_), _np.zeros(6 * np_)
        lib.nec_near_field(nec, k, _C.byref(nfeh), _dptr(xyz), _dptr(f))
        out.append((nfeh.value, xyz.reshape(-1, 3), (f[0::2] + 1j * f[1::2]).reshape(-1, 3)))
        k += 1


def structure(nec, freq_mhz=None):
    """The structure tables the GPU receives (wavelengths): dict with n, seg
    (8n), tptr, tbasis, tabc (3nt), ind (2n), params (10).  With freq_mhz the
    tables are (re)built on the host at that frequency first."""
    if freq_mhz is not None and lib.nec_prepare_structure(nec, freq_mhz) != 0:
        raise RuntimeError(nec_error_message())
    n = lib.nec_segment_count(nec)
    nt = lib.nec_get_structure(nec, None, None, None, None, None, None)
    if nt < 0:
        raise RuntimeError("no structure tables built")
    st = {"n": n, "seg": _np.zeros(8 * n), "tptr": _np.zeros(n + 1, dtype=_np.int32),
          "tbasis": _np.zeros(max(nt, 1), dtype=_np.int32), "tabc": _np.zeros(3 * max(nt, 1)),
          "ind": _np.zeros(2 * n, dtype=_np.int32), "params": _np.zeros(10)}
    lib.nec_get_structure(nec, _dptr(st["seg"]), _iptr(st["tptr"]), _iptr(st["tbasis"]), _dptr(st["tabc"]),
                          _iptr(st["ind"]), _dptr(st["params"]))
    st["tbasis"] = st["tbasis"][:nt]
    st["tabc"] = st["tabc"][:3 * nt].copy()
    zl = _np.zeros(2 * n)
    lib.nec_get_loads(nec, _dptr(zl))
    st["zload"] = zl[0::2] + 1j * zl[1::2]
    st["networks"] = int(lib.nec_network_count(nec))
    return st


def rhs(nec):
    """Applied-field vector (complex, n) of the current excitation at the
    frequency of the last structure()/nec_prepare_structure call."""
    n = lib.nec_segment_count(nec)
    out = _np.zeros(2 * n)
    if lib.nec_get_rhs(nec, _dptr(out)) != 0:
        raise RuntimeError(nec_error_message())
    return out[0::2] + 1j * out[1::2]


def last_refinement(nec):
    it = _C.c_int(0)
    res = _C.c_double(0)
    lib.nec_last_refinement(nec, _C.byref(it), _C.byref(res))
    return it.value, res.value


__all__ = _PUBLIC + ["nec_error_message", "segments", "trio", "currents", "pattern_fields",
                     "last_refinement", "structure", "rhs", "lib"]
