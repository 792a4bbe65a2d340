"""ctypes wrapper of the reference NEC2++ library built by oracle/Makefile.

Test infrastructure: only tests/, the fixture generator and bench.py's
CPU-baseline / reference arm load it.  It exposes the C API names of
src/libnecpp.h plus the shim entry points of oracle/ref_shim.cpp.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libnecpp_ref.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libnecpp_ref_omp.so")

_d, _i, _l, _p = C.c_double, C.c_int, C.c_long, C.c_void_p
_dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


def available(omp=False):
    return os.path.exists(REF_OMP_SO if omp else REF_SO)


class RefAPI:
    """The reference's C API (plus shim) under the same names as necpp_b200."""

    def __init__(self, omp=False):
        path = REF_OMP_SO if omp else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run make -C oracle ref)")
        L = C.CDLL(path)
        self.lib = L

        def sig(name, res, args):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
            setattr(self, name, f)

        sig("nec_create", _p, [])
        sig("nec_delete", _l, [_p])
        sig("nec_wire", _l, [_p, _i, _i] + [_d] * 9)
        sig("nec_gm_card", _l, [_p, _i, _i] + [_d] * 6 + [_i])
        sig("nec_geometry_complete", _l, [_p, _i])
        sig("nec_gn_card", _l, [_p, _i, _i] + [_d] * 6)
        sig("nec_ld_card", _l, [_p, _i, _i, _i, _i] + [_d] * 3)
        sig("nec_nt_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
        sig("nec_tl_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
        sig("nec_fr_card", _l, [_p, _i, _i, _d, _d])
        sig("nec_ek_card", _l, [_p, _i])
        sig("nec_ex_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
        sig("nec_xq_card", _l, [_p, _i])
        sig("nec_rp_card", _l, [_p] + [_i] * 7 + [_d] * 6)
        sig("nec_kh_card", _l, [_p, _d])
        sig("nec_pt_card", _l, [_p, _i, _i, _i, _i])
        sig("nec_gain", _d, [_p, _i, _i, _i])
        for stat in ("max", "min", "mean", "sd"):
            for pre in ("nec_gain_", "nec_gain_rhcp_", "nec_gain_lhcp_"):
                sig(pre + stat, _d, [_p, _i])
        sig("nec_impedance_real", _d, [_p, _i])
        sig("nec_impedance_imag", _d, [_p, _i])
        sig("nec_impedance_real_indexed", _d, [_p, _i, _i])
        sig("nec_impedance_imag_indexed", _d, [_p, _i, _i])
        sig("nec_error_message", C.c_char_p, [])
        sig("ref_helix", _l, [_p, _i, _i] + [_d] * 7)
        sig("ref_n_segments", _l, [_p])
        sig("ref_segments", None, [_p] + [_dp] * 8 + [_ip] * 3)
        sig("ref_segment_ends", None, [_p] + [_dp] * 6)
        sig("ref_trio", _i, [_p, _i, _ip, _dp, _dp, _dp])
        sig("ref_tbf", _i, [_p, _i, _i, _ip, _dp, _dp, _dp])
        sig("ref_wavelength", _d, [_p])
        sig("ref_fill", _l, [_p, _dp])
        sig("ref_lu", None, [_p, _dp, _ip])
        sig("ref_somm_tables", None, [_p, _dp, _dp])
        sig("ref_near_field", _l, [_p, _l, C.POINTER(C.c_int), _dp, _dp])
        sig("nec_ne_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
        sig("nec_nh_card", _l, [_p, _i, _i, _i, _i] + [_d] * 6)
        sig("ref_somm_interp_reset", None, [_p])
        sig("ref_somm_interpolate", None, [_p, _d, _d, _dp])
        sig("ref_currents", None, [_p] + [_dp] * 7)
        sig("ref_ffld", None, [_p, _d, _d, _dp, _dp])

    def helix(self, ctx, *args):
        return self.ref_helix(ctx, *args)

    def error(self):
        m = self.nec_error_message()
        return m.decode() if m else ""

    # ---- shim helpers ----
    def segments(self, ctx):
        n = self.ref_n_segments(ctx)
        arr = {k: np.zeros(n) for k in ("x", "y", "z", "si", "bi", "cab", "sab", "salp")}
        ints = {k: np.zeros(n, dtype=np.int32) for k in ("tags", "icon1", "icon2")}
        self.ref_segments(ctx, *[arr[k].ctypes.data_as(_dp) for k in ("x", "y", "z", "si", "bi", "cab", "sab", "salp")],
                          *[ints[k].ctypes.data_as(_ip) for k in ("tags", "icon1", "icon2")])
        arr.update(ints)
        return arr

    def trio(self, ctx, j, cap=64):
        jco = np.zeros(cap, dtype=np.int32)
        ax, bx, cx = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        k = self.ref_trio(ctx, j, jco.ctypes.data_as(_ip), ax.ctypes.data_as(_dp),
                          bx.ctypes.data_as(_dp), cx.ctypes.data_as(_dp))
        return jco[:k].copy(), ax[:k].copy(), bx[:k].copy(), cx[:k].copy()

    def fill(self, ctx):
        """Unfactored Z at the last simulated frequency, Z[obs, basis]."""
        n = self.ref_n_segments(ctx)
        out = np.zeros(2 * n * n)
        if self.ref_fill(ctx, out.ctypes.data_as(_dp)) != 0:
            raise RuntimeError(self.error())
        z = out[0::2] + 1j * out[1::2]
        return z.reshape(n, n)  # row = obs, column = basis (cm[basis + obs*n])

    def somm_tables(self, ctx):
        """Sommerfeld tables (1068 complex) of the last frequency and their
        complex permittivity."""
        out, eps = np.zeros(2 * 1068), np.zeros(2)
        self.ref_somm_tables(ctx, out.ctypes.data_as(_dp), eps.ctypes.data_as(_dp))
        return out[0::2] + 1j * out[1::2], complex(eps[0], eps[1])

    def somm_interpolate(self, ctx, x, y):
        f = np.zeros(8)
        self.ref_somm_interpolate(ctx, x, y, f.ctypes.data_as(_dp))
        return f[0::2] + 1j * f[1::2]

    def near_fields(self, ctx):
        """Every near-field pattern: list of (nfeh, points (m, np x 3),
        fields (np x 3 complex))."""
        out = []
        k = 0
        while True:
            nfeh = C.c_int(0)
            np_ = self.ref_near_field(ctx, k, C.byref(nfeh), None, None)
            if np_ < 0:
                return out
            xyz, f = np.zeros(3 * np_), np.zeros(6 * np_)
            self.ref_near_field(ctx, k, C.byref(nfeh), xyz.ctypes.data_as(_dp), f.ctypes.data_as(_dp))
            out.append((nfeh.value, xyz.reshape(-1, 3), (f[0::2] + 1j * f[1::2]).reshape(-1, 3)))
            k += 1

    def currents(self, ctx):
        n = self.ref_n_segments(ctx)
        cur = np.zeros(2 * n)
        abc = [np.zeros(n) for _ in range(6)]
        self.ref_currents(ctx, cur.ctypes.data_as(_dp), *[a.ctypes.data_as(_dp) for a in abc])
        return cur[0::2] + 1j * cur[1::2], np.stack(abc)

    def ffld(self, ctx, thet, phi):
        a, b = np.zeros(2), np.zeros(2)
        self.ref_ffld(ctx, thet, phi, a.ctypes.data_as(_dp), b.ctypes.data_as(_dp))
        return complex(a[0], a[1]), complex(b[0], b[1])
