"""ctypes access to the necgpu C-ABI (include/necgpu.h) for the GPU tests."""
import ctypes as C

import numpy as np

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class NecgpuStructure(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(k, _dp) for k in ("x", "y", "z", "length", "radius", "cab", "sab", "salp")] + [
        ("trio_ptr", _ip), ("trio_basis", _ip), ("trio_a", _dp), ("trio_b", _dp), ("trio_c", _dp),
        ("ek_ind1", _ip), ("ek_ind2", _ip), ("rkh", C.c_double), ("use_exk", C.c_int32), ("ground", C.c_int32),
        ("zrati_re", C.c_double), ("zrati_im", C.c_double), ("frati_re", C.c_double), ("frati_im", C.c_double),
        ("eta", C.c_double)]


class NecgpuStats(C.Structure):
    _fields_ = [("refine_iters", C.c_int), ("refine_residual", C.c_double),
                ("ms_fill", C.c_double), ("ms_factor", C.c_double), ("ms_solve", C.c_double),
                ("ms_pattern", C.c_double), ("launches", C.c_int64), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("k_ms", C.c_double * 9), ("k_launches", C.c_int64 * 9),
                ("k_flops", C.c_double * 9), ("pivoting", C.c_int), ("near_passes", C.c_int)]


class Engine:
    def __init__(self, lib, device=0):
        self.lib = lib
        L = lib
        L.necgpu_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
        L.necgpu_destroy.argtypes = [C.c_void_p]
        L.necgpu_last_error.restype = C.c_char_p
        L.necgpu_last_error.argtypes = [C.c_void_p]
        L.necgpu_set_structure.argtypes = [C.c_void_p, C.POINTER(NecgpuStructure)]
        L.necgpu_fill.argtypes = [C.c_void_p]
        L.necgpu_factor.argtypes = [C.c_void_p, C.c_int]
        L.necgpu_solve.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.necgpu_pattern.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        L.necgpu_copy_z.argtypes = [C.c_void_p, _dp]
        L.necgpu_set_refinement.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.necgpu_set_pivoting.argtypes = [C.c_void_p, C.c_int]
        L.necgpu_set_loads.argtypes = [C.c_void_p, _dp]
        L.necgpu_set_sommerfeld.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.necgpu_copy_sommerfeld.argtypes = [C.c_void_p, _dp]
        L.necgpu_reset_interpolation.argtypes = [C.c_void_p]
        L.necgpu_get_stats.argtypes = [C.c_void_p, C.POINTER(NecgpuStats)]
        self.h = C.c_void_p()
        rc = L.necgpu_create(C.byref(self.h), device)
        if rc != 0:
            raise RuntimeError("necgpu_create: %d %s" % (rc, L.necgpu_last_error(self.h)))
        self._keep = None

    def err(self):
        return self.lib.necgpu_last_error(self.h).decode()

    def check(self, rc):
        if rc != 0:
            raise RuntimeError("necgpu rc=%d: %s" % (rc, self.err()))

    def set_structure(self, st, tables=True):
        """Structure tables of st; for Sommerfeld ground also its tables
        (unless tables=False)."""
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
        self.check(self.lib.necgpu_set_structure(self.h, C.byref(s)))
        zl = np.ascontiguousarray(st.get("zload", np.zeros(n, complex)), dtype=complex)
        self._keep = (st, s, zl)
        if np.any(zl != 0):
            self.check(self.lib.necgpu_set_loads(self.h, zl.ctypes.data_as(_dp)))
        if tables and int(p[2]) == 3:
            self.check(self.lib.necgpu_set_sommerfeld(self.h, p[8], p[9]))
        self.n = n

    def sommerfeld_tables(self):
        t = np.zeros(2 * 1068)
        self.check(self.lib.necgpu_copy_sommerfeld(self.h, t.ctypes.data_as(_dp)))
        return t[0::2] + 1j * t[1::2]

    def reset_interpolation(self):
        self.check(self.lib.necgpu_reset_interpolation(self.h))

    def fill(self):
        self.check(self.lib.necgpu_fill(self.h))

    def copy_z(self):
        z = np.zeros(2 * self.n * self.n)
        self.check(self.lib.necgpu_copy_z(self.h, z.ctypes.data_as(_dp)))
        return (z[0::2] + 1j * z[1::2]).reshape(self.n, self.n)

    def factor(self, precision):
        self.check(self.lib.necgpu_factor(self.h, precision))

    def solve(self, rhs):
        b = np.ascontiguousarray(rhs, dtype=np.complex128)
        cur = np.zeros(2 * self.n)
        abc = np.zeros(6 * self.n)
        self.check(self.lib.necgpu_solve(self.h, b.view(np.float64).ctypes.data_as(_dp), cur.ctypes.data_as(_dp),
                                         abc.ctypes.data_as(_dp)))
        return cur[0::2] + 1j * cur[1::2], abc

    def pattern(self, theta, phi):
        th = np.ascontiguousarray(theta, dtype=np.float64)
        ph = np.ascontiguousarray(phi, dtype=np.float64)
        nd = len(th)
        eth, eph = np.zeros(2 * nd), np.zeros(2 * nd)
        self.check(self.lib.necgpu_pattern(self.h, nd, th.ctypes.data_as(_dp), ph.ctypes.data_as(_dp),
                                           eth.ctypes.data_as(_dp), eph.ctypes.data_as(_dp)))
        return eth[0::2] + 1j * eth[1::2], eph[0::2] + 1j * eph[1::2]

    def set_pivoting(self, mode):
        self.check(self.lib.necgpu_set_pivoting(self.h, mode))

    def set_update_format(self, fmt):
        """0: chosen by size, 1: split BF16, 2: TF32 (necgpu_set_update_format)."""
        self.check(self.lib.necgpu_set_update_format(self.h, fmt))

    def update_format(self):
        return self.lib.necgpu_update_format(self.h)

    def stats(self):
        st = NecgpuStats()
        self.check(self.lib.necgpu_get_stats(self.h, C.byref(st)))
        return st

    def close(self):
        if self.h:
            self.lib.necgpu_destroy(self.h)
            self.h = C.c_void_p()
