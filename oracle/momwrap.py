"""ctypes wrapper of oracle/liboracle.so (the C restatement of the hot path).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class MoStructure(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(k, _dp) for k in ("x", "y", "z", "s", "b", "cab", "sab", "salp")] + [
        ("trio_ptr", _ip), ("trio_basis", _ip), ("trio_a", _dp), ("trio_b", _dp), ("trio_c", _dp),
        ("ind1", _ip), ("ind2", _ip), ("rkh", C.c_double), ("use_exk", C.c_int), ("ground", C.c_int),
        ("zrati_re", C.c_double), ("zrati_im", C.c_double), ("frati_re", C.c_double),
        ("frati_im", C.c_double), ("eta", C.c_double), ("zload", _dp), ("somm", _dp),
        ("interp", C.c_void_p), ("interp_stateful", C.c_int)]


def build():
    """Compile liboracle.so (gcc, no contraction) if missing or stale."""
    src = [os.path.join(HERE, f) for f in ("mom_oracle.c", "somm_oracle.c", "mom_oracle.h")]
    if not os.path.exists(SO) or any(os.path.getmtime(s) > os.path.getmtime(SO) for s in src):
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        subprocess.run([cc, "-std=c11", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        "-o", SO, os.path.join(HERE, "mom_oracle.c"), os.path.join(HERE, "somm_oracle.c"),
                        "-lm"], check=True)
    return SO


class Oracle:
    def __init__(self):
        build()
        L = C.CDLL(SO)
        L.mo_fill.argtypes = [C.POINTER(MoStructure), _dp]
        L.mo_fill.restype = C.c_int
        L.mo_lu.argtypes = [C.c_int64, _dp, _ip]
        L.mo_lu.restype = C.c_int
        L.mo_solve.argtypes = [C.c_int64, _dp, _ip, _dp]
        L.mo_coefficients.argtypes = [C.POINTER(MoStructure), _dp, _dp, _dp]
        L.mo_ffld.argtypes = [C.POINTER(MoStructure), _dp, C.c_double, C.c_double, _dp, _dp]
        L.mo_nefld.argtypes = [C.POINTER(MoStructure), _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.mo_nhfld.argtypes = [C.POINTER(MoStructure), _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.mo_sommerfeld.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.mo_sommerfeld.restype = C.c_int
        L.mo_interp_size.restype = C.c_int64
        L.mo_interp_init.argtypes = [C.c_void_p]
        L.mo_interpolate.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double, C.c_int, _dp]
        self.L = L

    def sommerfeld(self, epr, sig, wavelength, eta):
        """Sommerfeld tables (1068 complex) and the complex permittivity used."""
        t = np.zeros(2 * 1068)
        eps = np.zeros(2)
        bad = self.L.mo_sommerfeld(epr, sig, wavelength, eta, t.ctypes.data_as(_dp), eps.ctypes.data_as(_dp))
        assert bad == 0, "Sommerfeld integral did not converge"
        return t[0::2] + 1j * t[1::2], complex(eps[0], eps[1])

    def new_interp(self):
        """A fresh interpolation cache (the state a new context starts with)."""
        buf = np.zeros(self.L.mo_interp_size(), dtype=np.uint8)
        self.L.mo_interp_init(buf.ctypes.data_as(C.c_void_p))
        return buf

    def interpolate(self, interp, tables, x, y, stateful=True):
        t = np.ascontiguousarray(tables, dtype=np.complex128).view(np.float64)
        f = np.zeros(8)
        self.L.mo_interpolate(interp.ctypes.data_as(C.c_void_p), t.ctypes.data_as(_dp), x, y, int(stateful),
                              f.ctypes.data_as(_dp))
        return f[0::2] + 1j * f[1::2]

    def structure(self, st):
        """st: dict from tests.helpers.export_structure (kept alive by the caller)."""
        s = MoStructure()
        s.n = st["n"]
        seg = st["seg"]
        n = st["n"]
        for k, name in enumerate(("x", "y", "z", "s", "b", "cab", "sab", "salp")):
            setattr(s, name, seg[k * n:(k + 1) * n].ctypes.data_as(_dp))
        s.trio_ptr = st["tptr"].ctypes.data_as(_ip)
        s.trio_basis = st["tbasis"].ctypes.data_as(_ip)
        nt = len(st["tbasis"])
        s.trio_a = st["tabc"][:nt].ctypes.data_as(_dp)
        s.trio_b = st["tabc"][nt:2 * nt].ctypes.data_as(_dp)
        s.trio_c = st["tabc"][2 * nt:].ctypes.data_as(_dp)
        s.ind1 = st["ind"][:n].ctypes.data_as(_ip)
        s.ind2 = st["ind"][n:].ctypes.data_as(_ip)
        p = st["params"]
        s.rkh, s.use_exk, s.ground = p[0], int(p[1]), int(p[2])
        s.zrati_re, s.zrati_im, s.frati_re, s.frati_im, s.eta = p[3], p[4], p[5], p[6], p[7]
        zl = st.get("zload")
        if zl is not None and np.any(zl != 0):
            st["_zload_ri"] = np.ascontiguousarray(np.asarray(zl, dtype=np.complex128)).view(np.float64)
            s.zload = st["_zload_ri"].ctypes.data_as(_dp)
        somm = st.get("somm")
        if somm is not None:
            st["_somm_ri"] = np.ascontiguousarray(np.asarray(somm, dtype=np.complex128)).view(np.float64)
            s.somm = st["_somm_ri"].ctypes.data_as(_dp)
            if st.get("interp") is None:
                st["interp"] = self.new_interp()
            s.interp = st["interp"].ctypes.data_as(C.c_void_p)
            s.interp_stateful = int(st.get("interp_stateful", True))
        return s

    def fill(self, st):
        s = self.structure(st)
        n = st["n"]
        z = np.zeros(2 * n * n)
        status = self.L.mo_fill(C.byref(s), z.ctypes.data_as(_dp))
        return (z[0::2] + 1j * z[1::2]).reshape(n, n), status

    def solve(self, z, rhs):
        n = z.shape[0]
        a = np.ascontiguousarray(z, dtype=np.complex128).copy()
        piv = np.zeros(n, dtype=np.int32)
        bad = self.L.mo_lu(n, a.view(np.float64).ctypes.data_as(_dp), piv.ctypes.data_as(_ip))
        b = np.ascontiguousarray(rhs, dtype=np.complex128).copy()
        self.L.mo_solve(n, a.view(np.float64).ctypes.data_as(_dp), piv.ctypes.data_as(_ip),
                        b.view(np.float64).ctypes.data_as(_dp))
        return b, bad

    def coefficients(self, st, x):
        s = self.structure(st)
        n = st["n"]
        xx = np.ascontiguousarray(x, dtype=np.complex128)
        abc = np.zeros(6 * n)
        cur = np.zeros(2 * n)
        self.L.mo_coefficients(C.byref(s), xx.view(np.float64).ctypes.data_as(_dp),
                               abc.ctypes.data_as(_dp), cur.ctypes.data_as(_dp))
        return abc, cur[0::2] + 1j * cur[1::2]

    def near_field(self, st, abc, pts, magnetic=False):
        """Near E (or H) at points (wavelengths, np x 3) in order: np x 3 complex."""
        s = self.structure(st)
        f = self.L.mo_nhfld if magnetic else self.L.mo_nefld
        out = np.zeros((len(pts), 6))
        a = np.ascontiguousarray(abc, dtype=np.float64)
        for k, (x, y, z) in enumerate(pts):
            f(C.byref(s), a.ctypes.data_as(_dp), float(x), float(y), float(z), out[k].ctypes.data_as(_dp))
        return out[:, 0::2] + 1j * out[:, 1::2]

    def ffld(self, st, abc, thet, phi):
        s = self.structure(st)
        a, b = np.zeros(2), np.zeros(2)
        self.L.mo_ffld(C.byref(s), abc.ctypes.data_as(_dp), thet, phi, a.ctypes.data_as(_dp),
                       b.ctypes.data_as(_dp))
        return complex(a[0], a[1]), complex(b[0], b[1])
