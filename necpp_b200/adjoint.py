"""Adjoint gradients of input impedance and gain (extension of the C API,
nec_gradient).

    value, jac = gradient(build, p, freq_mhz=145.0, theta_deg=80.0, phi_deg=0.0)

`build(ctx, p)` issues the geometry cards (ending with geometry complete),
the ground card and the single voltage-source EX card for parameter vector
p; the frequency is set here.  value = (Re Zin, Im Zin, gain dB at
(theta, phi)); jac[i, k] = d value[i] / d p[k].  The forward solve runs in
mixed precision on the GPU; every parameter costs two host-side structure
builds, and the GPU work is one transposed solve per output on the held
factors plus one batched fill of the perturbed structures contracted on the
fly (the derivative of the interaction matrix is never stored).
"""
import ctypes as _C

import numpy as _np

from . import lib, nec_create, nec_delete, nec_error_message, nec_fr_card, nec_set_precision, nec_xq_card

__all__ = ["gradient", "gradient_population", "batched_outputs", "batched_fd", "ZinGain"]


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s: %s" % (what, nec_error_message()))


def gradient(build, params, freq_mhz, theta_deg, phi_deg, h=1e-6, timings=None):
    """See the module docstring.  If `timings` is a dict it receives the
    wall-clock seconds of the forward solve ('forward_s': cards, fill,
    factorisation, solve) and of everything after it ('gradient_s':
    perturbed structures, adjoint solves, contractions, assembly)."""
    import time
    p = _np.asarray(params, dtype=_np.float64)
    npar = len(p)
    hs = _np.broadcast_to(_np.asarray(h, dtype=_np.float64), (npar,)).copy()
    ctxs = []
    try:
        t0 = time.perf_counter()
        base = nec_create()
        ctxs.append(base)
        _check(nec_set_precision(base, 1), "set_precision")
        build(base, p)
        _check(nec_fr_card(base, 0, 1, float(freq_mhz), 0.0), "fr card")
        _check(nec_xq_card(base, 0), "forward solve")
        t1 = time.perf_counter()
        plus, minus = [], []
        for k in range(npar):
            for sign, lst in ((1.0, plus), (-1.0, minus)):
                q = p.copy()
                q[k] += sign * hs[k]
                c = nec_create()
                ctxs.append(c)
                build(c, q)
                lst.append(c)
        parr = (_C.c_void_p * npar)(*plus)
        marr = (_C.c_void_p * npar)(*minus)
        value = _np.zeros(3)
        grad = _np.zeros(3 * npar)
        _check(lib.nec_gradient(base, npar, parr, marr, hs.ctypes.data_as(_C.POINTER(_C.c_double)),
                                float(theta_deg), float(phi_deg), value.ctypes.data_as(_C.POINTER(_C.c_double)),
                                grad.ctypes.data_as(_C.POINTER(_C.c_double))), "gradient")
        if timings is not None:
            timings["forward_s"] = t1 - t0
            timings["gradient_s"] = time.perf_counter() - t1
        return value, grad.reshape(npar, 3).T.copy()
    finally:
        for c in ctxs:
            nec_delete(c)


def gradient_population(build, P, freq_mhz, theta_deg, phi_deg, h=1e-6, world=1, rank=0):
    """Adjoint gradients of a population of designs (the rows of P), each
    as `gradient` computes it.  With world > 1 the designs are shared out
    over the ranks (equal costs: round robin) and each rank returns only
    its own: (indices, values (m, 3), jacobians (m, 3, npar))."""
    from .replicas import partition_by_cost
    P = _np.atleast_2d(_np.asarray(P, dtype=_np.float64))
    mine = partition_by_cost([1.0] * len(P), world, rank)
    vals = _np.zeros((len(mine), 3))
    jacs = _np.zeros((len(mine), 3, P.shape[1]))
    for k, i in enumerate(mine):
        vals[k], jacs[k] = gradient(build, P[i], freq_mhz, theta_deg, phi_deg, h=h)
    return mine, vals, jacs


def batched_outputs(build, params, freq_mhz, theta_deg, phi_deg):
    """(Re Zin, Im Zin, gain dB at (theta, phi)) of every parameter vector in
    `params`, all solved in ONE batched call (necgpu_batch_solve: one fill
    launch over all structures, persistent per-structure LU with FP64
    refinement, far field).  `build(ctx, p)` as for `gradient`, with one
    voltage source."""
    import math
    from . import batch as B
    from . import rhs as _rhs
    from . import structure as _structure
    problems = []
    for p in params:
        c = nec_create()
        try:
            build(c, _np.asarray(p, dtype=_np.float64))
            st = _structure(c, float(freq_mhz))
            b = _rhs(c)
        finally:
            nec_delete(c)
        feeds = _np.flatnonzero(b)
        if len(feeds) != 1:
            raise ValueError("batched_outputs: exactly one voltage source is supported")
        f = int(feeds[0])
        lam = B._C0 / (float(freq_mhz) * 1e6)
        n = st["n"]
        v = -b[f] * st["seg"][3 * n + f] * lam  # e_f = -V / (s_f lambda), s in wavelengths
        problems.append((st, b, f, complex(v), lam))
    res = B.sweep(problems, [math.radians(theta_deg)], [math.radians(phi_deg)], fields=True)
    bad = _np.flatnonzero(res["status"] != 0)
    if len(bad):
        raise RuntimeError("batched_outputs: problems %s failed (status %s)" % (bad[:8], res["status"][bad[:8]]))
    out = _np.zeros((len(problems), 3))
    for k, (st, b, f, v, lam) in enumerate(problems):
        z = res["zin"][k]
        i = res["cur"][res["offsets"][k] + f]
        pin = 0.5 * (v * _np.conj(i)).real
        gcop = lam * lam * 2.0 * B._PI / (st["params"][7] * pin)
        e2 = abs(res["eth"][k][0]) ** 2 + abs(res["eph"][k][0]) ** 2
        out[k] = (z.real, z.imag, 10.0 * math.log10(gcop * e2))
    return out


def batched_fd(build, P, freq_mhz, theta_deg, phi_deg, h=1e-6):
    """Central finite differences of (Re Zin, Im Zin, gain dB) for every
    design in P (rows), every one of its parameters moved by +-h: all
    len(P) * (2 npar + 1) structures in one batched solve.  Returns
    (values (m, 3), fd (m, 3, npar))."""
    P = _np.atleast_2d(_np.asarray(P, dtype=_np.float64))
    m, npar = P.shape
    params = []
    for p in P:
        params.append(p)
        for k in range(npar):
            for sign in (1.0, -1.0):
                q = p.copy()
                q[k] += sign * h
                params.append(q)
    out = batched_outputs(build, params, freq_mhz, theta_deg, phi_deg).reshape(m, 2 * npar + 1, 3)
    vals = out[:, 0, :]
    fd = (out[:, 1::2, :] - out[:, 2::2, :]) / (2.0 * h)  # (m, npar, 3)
    return vals, _np.transpose(fd, (0, 2, 1)).copy()


def _make_function():
    import torch

    class ZinGain(torch.autograd.Function):
        """(Re Zin, Im Zin, gain dB) of the structure build(ctx, p) as a
        differentiable function of the parameter tensor p; the backward pass
        applies the adjoint Jacobian computed with the forward pass."""

        @staticmethod
        def forward(ctx, p, build, freq_mhz, theta_deg, phi_deg, h=1e-6):
            value, jac = gradient(build, p.detach().cpu().double().numpy(), freq_mhz, theta_deg, phi_deg, h)
            ctx.save_for_backward(torch.as_tensor(jac, dtype=p.dtype, device=p.device))
            return torch.as_tensor(value, dtype=p.dtype, device=p.device)

        @staticmethod
        def backward(ctx, g):
            (jac,) = ctx.saved_tensors
            return g @ jac, None, None, None, None, None

    return ZinGain


_zin_gain = None


def __getattr__(name):
    global _zin_gain
    if name == "ZinGain":
        if _zin_gain is None:
            _zin_gain = _make_function()
        return _zin_gain
    raise AttributeError(name)
