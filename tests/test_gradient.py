"""Adjoint gradients (nec_gradient): the seeded 9-element Yagi over
Sommerfeld ground at 145 MHz, 27 parameters (half lengths, x positions,
radii), outputs Re Zin, Im Zin and gain at theta 80, phi 0.

The reference fixture holds the reference's own FP64 outputs and their
central finite differences (h = 1e-6 m, one full reference solve per side);
those differences are reproducible to ~1e-6 of each output's largest
derivative (h = 1e-7 agrees to that level), so the adjoint gradients are
held to 1e-5 of it.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN

TOL_GRAD = 1e-5


def _golden():
    return dict(np.load(os.path.join(GOLDEN, "yagi_grad.npz")))


def test_golden_params_match_workload():
    from necpp_b200 import workloads as W
    assert np.array_equal(_golden()["params"], W.yagi_ground_params(0))


def test_gradient_needs_a_forward_solve(nb):
    """Host-side argument and state checks (no device needed)."""
    from necpp_b200 import workloads as W
    base = nb.nec_create()
    W.yagi_ground_cards(nb, base, W.yagi_ground_params(0))
    arr = (C.c_void_p * 1)(base)
    h = np.array([1e-6])
    v, g = np.zeros(3), np.zeros(3)
    rc = nb.lib.nec_gradient(base, 1, arr, arr, h.ctypes.data_as(C.POINTER(C.c_double)), 80.0, 0.0,
                             v.ctypes.data_as(C.POINTER(C.c_double)), g.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 1 and "forward solve" in nb.nec_error_message()
    nb.nec_delete(base)


@pytest.mark.gpu
def test_adjoint_gradient_matches_reference_fd(nb):
    from necpp_b200 import adjoint, workloads as W
    g = _golden()
    build = lambda ctx, p: W.yagi_ground_cards(nb, ctx, p)
    value, jac = adjoint.gradient(build, g["params"], 145.0, 80.0, 0.0, h=float(g["h"]))
    ref = g["value"]
    zin, zref = complex(value[0], value[1]), complex(ref[0], ref[1])
    assert abs(zin - zref) / abs(zref) <= 1e-6
    assert abs(value[2] - ref[2]) <= 0.01
    fd = g["fd"]
    scale = np.max(np.abs(fd), axis=1)
    err = np.max(np.abs(jac - fd), axis=1) / scale
    assert np.all(err <= TOL_GRAD), err


@pytest.mark.gpu
def test_adjoint_solve_is_the_transposed_solve(nb, oracle):
    """Z^T w = phi through the C-ABI, checked against the oracle's Z."""
    from cases import CASES
    from gpu_helpers import Engine
    from helpers import host_case
    ctx, st, rhs, _ = host_case(nb, CASES["yagi_ground"][0])
    e = Engine(nb.lib)
    try:
        e.set_structure(st)
        e.fill()
        e.factor(1)
        e.solve(rhs)
        n = st["n"]
        rng = np.random.default_rng(3)
        phi = rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))
        w = np.zeros((2, n), dtype=np.complex128)
        L = nb.lib
        L.necgpu_adjoint_solve.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        pin = np.ascontiguousarray(phi)
        e.check(L.necgpu_adjoint_solve(e.h, 2, pin.ctypes.data, w.ctypes.data))
        Z, _ = oracle.fill(st)
        for k in range(2):
            r = Z.T @ w[k] - phi[k]
            assert np.linalg.norm(r) / np.linalg.norm(phi[k]) <= 1e-12
        # after an FP64 factorisation (Z overwritten) the adjoint is refused
        e.fill()
        e.factor(0)
        assert L.necgpu_adjoint_solve(e.h, 2, pin.ctypes.data, w.ctypes.data) == 6
    finally:
        e.close()
        nb.nec_delete(ctx)


@pytest.mark.gpu
def test_torch_autograd_wrapper(nb):
    import torch
    from necpp_b200 import adjoint, workloads as W
    g = _golden()
    build = lambda ctx, p: W.yagi_ground_cards(nb, ctx, p)
    p = torch.tensor(g["params"], dtype=torch.float64, requires_grad=True)
    out = adjoint.ZinGain.apply(p, build, 145.0, 80.0, 0.0, float(g["h"]))
    loss = out[0] - 0.5 * out[2]
    loss.backward()
    expect = g["fd"][0] - 0.5 * g["fd"][2]
    assert np.max(np.abs(p.grad.numpy() - expect)) <= 2 * TOL_GRAD * np.max(np.abs(g["fd"]))


@pytest.mark.gpu
def test_population_adjoint_matches_batched_differences(nb):
    """A population of 64 seeded designs (yagi_ground_params(seed), seeds
    0..63): the adjoint gradients of every design against central
    differences of all 64 x 55 base and perturbed structures solved in ONE
    batched call (necgpu_batch_solve), within 1e-5 of each output's largest
    derivative; the batched differences of design 0 against the reference's
    own FP64 differences at the same tolerance."""
    from necpp_b200 import adjoint, workloads as W
    build = lambda ctx, p: W.yagi_ground_cards(nb, ctx, p)
    P = np.array([W.yagi_ground_params(s) for s in range(64)])
    idx, vals, jacs = adjoint.gradient_population(build, P, 145.0, 80.0, 0.0)
    assert idx == list(range(64))
    bvals, fd = adjoint.batched_fd(build, P, 145.0, 80.0, 0.0)
    zrel = np.abs((vals[:, 0] + 1j * vals[:, 1]) - (bvals[:, 0] + 1j * bvals[:, 1])) / np.abs(bvals[:, 0] + 1j * bvals[:, 1])
    assert np.max(zrel) <= 1e-9
    assert np.max(np.abs(vals[:, 2] - bvals[:, 2])) <= 1e-6
    for i in range(64):
        scale = np.max(np.abs(fd[i]), axis=1)
        err = np.max(np.abs(jacs[i] - fd[i]), axis=1) / scale
        assert np.all(err <= TOL_GRAD), (i, err)
    g = _golden()
    assert np.array_equal(P[0], g["params"])
    scale = np.max(np.abs(g["fd"]), axis=1)
    assert np.all(np.max(np.abs(fd[0] - g["fd"]), axis=1) / scale <= TOL_GRAD)
