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

__all__ = ["gradient", "ZinGain"]


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
