"""Engine reuse between contexts (necgpu_acquire / necgpu_release): a
released engine that kept its default settings serves the next context of
its device, with nothing of the previous context's results, tables or
interpolation state carried over; a changed engine is not pooled."""
import ctypes as C

import numpy as np
import pytest

from cases import CASES
from test_gpu_parity import our_zin, run_case


def _lib(nb):
    L = nb.lib
    L.necgpu_acquire.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    L.necgpu_release.argtypes = [C.c_void_p]
    L.necgpu_set_refinement.argtypes = [C.c_void_p, C.c_double, C.c_int]
    L.nec_gpu_engine.restype = C.c_void_p
    L.nec_gpu_engine.argtypes = [C.c_void_p]
    return L


def test_pool_symbols_exported(nb):
    L = nb.lib
    for name in ("necgpu_acquire", "necgpu_release"):
        assert hasattr(L, name)


@pytest.mark.gpu
def test_released_engine_is_reacquired(nb):
    L = _lib(nb)
    a, b = C.c_void_p(), C.c_void_p()
    assert L.necgpu_acquire(C.byref(a), 0) == 0
    assert L.necgpu_release(a) == 0
    assert L.necgpu_acquire(C.byref(b), 0) == 0
    assert b.value == a.value  # the pooled engine, still alive while pooled
    # a changed setting: destroyed on release, not pooled
    assert L.necgpu_set_refinement(b, 1e-12, 20) == 0
    assert L.necgpu_release(b) == 0
    c = C.c_void_p()
    assert L.necgpu_acquire(C.byref(c), 0) == 0
    d = C.c_void_p()
    assert L.necgpu_acquire(C.byref(d), 0) == 0  # the pool is empty: a second, new engine
    assert d.value != c.value
    L.necgpu_release(c)
    L.necgpu_release(d)


def _zin(nb, api, name, precision=1):
    ctx = run_case(nb, api, name, precision)
    try:
        return np.array(our_zin(nb, ctx), dtype=complex)
    finally:
        nb.nec_delete(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["near_ground", "yagi_ground", "helix2"])
def test_contexts_in_sequence_match(nb, api, name):
    """The same case in a fresh context after other structures (a Sommerfeld
    ground, a reflection ground, a helix array) ran on the pooled engine
    gives the same impedances as the first time (to 1e-13; state carried
    over, such as the Sommerfeld interpolation cache, would show at 1e-8 or
    more): the tables, the interpolation cache and the factors start
    afresh."""
    first = _zin(nb, api, name)
    for other in ("helix2", "near_ground", "yagi_ground"):
        _zin(nb, api, other)
    again = _zin(nb, api, name)
    assert first.shape == again.shape
    assert np.max(np.abs(first - again) / np.abs(first)) <= 1e-13
