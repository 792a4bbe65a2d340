"""The precision argument behind the mixed LU's two update formats, on the
CPU: a blocked complex64 LU of the 2 x 2 helix array (720 unknowns, Z from
the oracle) whose trailing updates see their operands rounded as each
tensor-core format rounds them, then FP64 iterative refinement.

* split BF16 (hi + lo parts, three products: hi*hi + hi*lo + lo*hi);
* TF32 (operands rounded to 10 explicit mantissa bits, nearest; the update
  kernel rounds with cvt.rna.tf32.f32 before the MMA).

Split BF16 contracts the residual by ~1e-5 or better per step, TF32 by
~1e-3: TF32 needs one more step to reach the engine's 1e-13 tolerance on
this structure, which is what the engine's choice of format (TF32 only
for large systems, where the update's saving outweighs a step) rests on.
This emulates the formats' rounding, not the kernels: the kernels are
tested on the GPU (test_gpu_parity, test_tuning)."""
import numpy as np
import pytest
import scipy.linalg as sl

from cases import CASES
from helpers import host_case


def _bf16(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + np.uint32(0x7FFF) + ((u >> 16) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return u.view(np.float32).astype(np.float64)


def _tf32(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + np.uint32(0xFFF) + ((u >> 13) & np.uint32(1))) & np.uint32(0xFFFFE000)
    return u.view(np.float32).astype(np.float64)


def _update(A, B, fmt):
    if fmt == "tf32":
        qa = _tf32(A.real) + 1j * _tf32(A.imag)
        qb = _tf32(B.real) + 1j * _tf32(B.imag)
        return qa @ qb
    ah = _bf16(A.real) + 1j * _bf16(A.imag)
    bh = _bf16(B.real) + 1j * _bf16(B.imag)
    al = _bf16(A.real - ah.real) + 1j * _bf16(A.imag - ah.imag)
    bl = _bf16(B.real - bh.real) + 1j * _bf16(B.imag - bh.imag)
    return ah @ bh + ah @ bl + al @ bh


def _lu(Z, fmt, kb=64):
    A = Z.astype(np.complex64)
    n = A.shape[0]
    perm = np.arange(n)
    for k0 in range(0, n, kb):
        k1 = min(k0 + kb, n)
        for j in range(k0, k1):
            p = j + int(np.argmax(np.abs(A[j:, j])))
            if p != j:
                A[[j, p]] = A[[p, j]]
                perm[[j, p]] = perm[[p, j]]
            A[j + 1:, j] /= A[j, j]
            A[j + 1:, j + 1:k1] -= np.outer(A[j + 1:, j], A[j, j + 1:k1])
        if k1 < n:
            L11 = np.tril(A[k0:k1, k0:k1], -1) + np.eye(k1 - k0, dtype=np.complex64)
            A[k0:k1, k1:] = sl.solve_triangular(L11, A[k0:k1, k1:], lower=True, unit_diagonal=True)
            A[k1:, k1:] = (A[k1:, k1:] - _update(A[k1:, k0:k1], A[k0:k1, k1:], fmt)).astype(np.complex64)
    return A, perm


def _refine(Z, A, perm, b, steps=6):
    L = np.tril(A, -1).astype(np.complex128) + np.eye(A.shape[0])
    U = np.triu(A).astype(np.complex128)
    x = np.zeros_like(b)
    hist = []
    for _ in range(steps):
        r = b - Z @ x
        hist.append(np.linalg.norm(r) / np.linalg.norm(b))
        y = sl.solve_triangular(L, r[perm], lower=True, unit_diagonal=True)
        x = x + sl.solve_triangular(U, y)
    hist.append(np.linalg.norm(b - Z @ x) / np.linalg.norm(b))
    return hist


def _steps_to(hist, tol=1e-13):
    return next(i for i, v in enumerate(hist) if v <= tol)


@pytest.fixture(scope="module")
def helix2(nb, oracle):
    ctx, st, rhs, _ = host_case(nb, CASES["helix2"][0])
    Z, _ = oracle.fill(st)
    nb.nec_delete(ctx)
    return np.asarray(Z, dtype=np.complex128), np.asarray(rhs, dtype=np.complex128)


def test_update_formats_refinement_contraction(helix2):
    Z, b = helix2
    hist = {}
    for fmt in ("bf16x3", "tf32"):
        A, perm = _lu(Z, fmt)
        hist[fmt] = _refine(Z, A, perm, b)
    # first correction: the factor's error shows directly
    assert hist["bf16x3"][1] <= 1e-5, hist["bf16x3"]
    assert 1e-6 <= hist["tf32"][1] <= 1e-3, hist["tf32"]
    # both reach the FP64 floor; TF32 one step later
    assert _steps_to(hist["bf16x3"]) == 3, hist["bf16x3"]
    assert _steps_to(hist["tf32"]) == 4, hist["tf32"]
