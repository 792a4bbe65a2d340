"""Failure and fallback paths of the dense solve, on caller matrices
(necgpu_matrix_solve), checked on the host.  Nothing here faults the GPU:
every failure is an exact zero pivot or a refinement cap, reported through
the engine's status codes.

The reference warns about a near-singular factorisation and carries on
(src/matrix_algebra.cpp:140-161); this path stops with an error instead of
returning non-finite currents.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_SINGULAR, ERR_NONFINITE, ERR_REFINE = 3, 4, 5


@pytest.fixture
def engine(nb):
    from gpu_helpers import Engine
    e = Engine(nb.lib)
    L = nb.lib
    L.necgpu_matrix_solve.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                      C.POINTER(C.c_double)]
    yield e
    e.close()


def _solve(e, z, b, precision):
    n = len(b)
    z = np.ascontiguousarray(z, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    x = np.full(n, np.nan, dtype=np.complex128)
    res = C.c_double(-1.0)
    rc = e.lib.necgpu_matrix_solve(e.h, n, z.ctypes.data, b.ctypes.data, precision, x.ctypes.data, C.byref(res))
    return rc, x, res.value


def _matrix(n, seed):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    z += n * np.eye(n)  # well conditioned
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return z, b


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [50, 300, 1000])
def test_matrix_solve_matches_numpy(engine, n, precision):
    z, b = _matrix(n, n)
    rc, x, res = _solve(engine, z, b, precision)
    assert rc == 0, engine.err()
    ref = np.linalg.solve(z, b)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= 1e-12
    if precision == 1:
        assert res <= 1e-12


def test_singular_diagonal_block_takes_partial_pivot_refactor(engine):
    """Rows 0 and 1 agree inside the first 64 x 64 diagonal block but not
    beyond it: the matrix is regular, the block is not.  Block-local
    pivoting meets an exact zero pivot there, the engine refactors with
    partial pivoting, and the refined solution is the FP64 one."""
    n = 300
    z, b = _matrix(n, 11)
    z[1, :64] = z[0, :64]
    rc, x, res = _solve(engine, z, b, 1)
    assert rc == 0, engine.err()
    assert engine.stats().pivoting == 0
    assert res <= 1e-12
    ref = np.linalg.solve(z, b)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_exactly_singular_matrix_is_an_error(engine, precision):
    """A zero row (an equation without coefficients): an exact zero pivot,
    reported as NECGPU_ERR_SINGULAR with a message."""
    n = 200
    z, b = _matrix(n, 5)
    z[137, :] = 0.0
    rc, x, _ = _solve(engine, z, b, precision)
    assert rc == ERR_SINGULAR, (rc, engine.err())
    assert "singular" in engine.err() or "pivot" in engine.err()


def test_refinement_cap_forces_the_fallback(engine, nb):
    """One refinement step only (max_iter 0): the residual stays at the
    complex64 level, above the fallback threshold, so the engine refactors
    with partial pivoting and refines once more; the result is accepted at
    the 1e-6 gate of the mixed path."""
    L = nb.lib
    n = 400
    z, b = _matrix(n, 21)
    engine.check(L.necgpu_set_refinement(engine.h, 1e-13, 0))
    try:
        rc, x, res = _solve(engine, z, b, 1)
        st = engine.stats()
    finally:
        engine.check(L.necgpu_set_refinement(engine.h, 1e-13, 30))
    assert rc == 0, engine.err()
    assert st.pivoting == 0 and st.refine_iters == 2
    assert 1e-10 < res <= 1e-6
    ref = np.linalg.solve(z, b)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= 1e-5
