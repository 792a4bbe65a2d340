"""necgpu_solve_noalloc: the allocation-free solve (static device scratch)
against necgpu_solve on the same held factors.

Two calls in a row per case: the second call reuses the scratch and the next
sweep epochs, so a stale flag word or an uncleared vector shows up as a
mismatch.  The file is named to be collected last, and also runs alone.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from cases import CASES
from helpers import host_case

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)
# the two paths run the same kernels in the same order; the mixed residual
# norm is summed with atomics, so allow for a different stopping step there
TOL = {0: 1e-12, 1: 1e-10}
MAX_N = 16384


@pytest.fixture(scope="module")
def engine(nb):
    from gpu_helpers import Engine
    e = Engine(nb.lib)
    nb.lib.necgpu_solve_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    yield e
    e.close()


def _noalloc(engine, rhs_t, cur_t, abc_t):
    import torch
    torch.cuda.synchronize()
    rc = engine.lib.necgpu_solve_noalloc(engine.h, C.c_void_p(rhs_t.data_ptr()), C.c_void_p(cur_t.data_ptr()),
                                         None if abc_t is None else C.c_void_p(abc_t.data_ptr()))
    return rc


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["yagi_ground", "helix2", "mesh_small"])
def test_noalloc_matches_solve(nb, engine, name, precision):
    import torch
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    n = st["n"]
    engine.set_structure(st)
    engine.fill()
    engine.factor(precision)
    cur_ref, abc_ref = engine.solve(rhs)
    scale = np.max(np.abs(cur_ref))
    rhs_t = torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.complex128).view(np.float64)).cuda()
    for call in range(2):
        cur_t = torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda")
        abc_t = torch.full((6 * n,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _noalloc(engine, rhs_t, cur_t, abc_t)
        assert rc == 0, (call, engine.err())
        c = cur_t.cpu().numpy()
        cur = c[0::2] + 1j * c[1::2]
        assert np.max(np.abs(cur - cur_ref)) <= TOL[precision] * scale, call
        abc = abc_t.cpu().numpy()
        assert np.max(np.abs(abc - abc_ref)) <= TOL[precision] * np.max(np.abs(abc_ref)), call
    # coefficients may be left out (they go to the static scratch)
    cur_t = torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda")
    assert _noalloc(engine, rhs_t, cur_t, None) == 0, engine.err()
    c = cur_t.cpu().numpy()
    assert np.max(np.abs(c[0::2] + 1j * c[1::2] - cur_ref)) <= TOL[precision] * scale
    # the input is not modified
    assert np.array_equal(rhs_t.cpu().numpy(), np.ascontiguousarray(rhs, dtype=np.complex128).view(np.float64))
    nb.nec_delete(ctx)


def test_noalloc_rejects_host_memory_and_overlap(nb, engine):
    import torch
    ctx, st, rhs, _ = host_case(nb, CASES["helix2"][0])
    n = st["n"]
    engine.set_structure(st)
    engine.fill()
    engine.factor(0)
    host = np.zeros(2 * n)
    dev = torch.zeros(4 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = engine.lib.necgpu_solve_noalloc(engine.h, host.ctypes.data, C.c_void_p(dev.data_ptr()), None)
    assert rc == 2 and "not device memory" in engine.err()
    rc = engine.lib.necgpu_solve_noalloc(engine.h, C.c_void_p(dev.data_ptr()), C.c_void_p(dev.data_ptr()), None)
    assert rc == 2 and "overlap" in engine.err()
    nb.nec_delete(ctx)


def test_noalloc_rejects_beyond_static_limit(nb, engine):
    """n = 16385 (one above the static scratch) is refused before any work."""
    import torch
    n = MAX_N + 1
    z = np.linspace(-0.5, 0.5, n + 1)
    seg = np.concatenate([np.zeros(n), np.zeros(n), 0.5 * (z[:-1] + z[1:]), np.diff(z), np.full(n, 1e-6),
                          np.zeros(n), np.zeros(n), np.ones(n)])
    st = {"n": n, "seg": seg, "tptr": np.arange(n + 1, dtype=np.int32), "tbasis": np.arange(n, dtype=np.int32),
          "tabc": np.concatenate([np.zeros(n), np.zeros(n), np.ones(n)]), "ind": np.zeros(2 * n, dtype=np.int32),
          "params": np.array([1e-4, 0, 0, 0, 0, 0, 0, 376.73])}
    engine.set_structure(st)
    rhs_t = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    cur_t = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    rc = _noalloc(engine, rhs_t, cur_t, None)
    assert rc == 2
    assert "16384" in engine.err()


def test_noalloc_rejects_buffer_past_its_allocation(nb, engine):
    """A right-hand side that runs 16 bytes past the end of its cudaMalloc
    allocation is refused (the extent comes from cuMemGetAddressRange)."""
    import torch
    ctx, st, rhs, _ = host_case(nb, CASES["helix2"][0])
    n = st["n"]
    engine.set_structure(st)
    engine.fill()
    engine.factor(0)
    torch.cuda.init()
    rt = C.CDLL("libcudart.so.12")  # the runtime torch has loaded
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaFree.argtypes = [C.c_void_p]
    size = 2 << 20
    vec = 16 * n
    base = C.c_void_p()
    assert rt.cudaMalloc(C.byref(base), size) == 0
    try:
        cur = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        inside = base.value + size - vec
        rc = engine.lib.necgpu_solve_noalloc(engine.h, C.c_void_p(inside), C.c_void_p(cur.data_ptr()), None)
        assert rc == 0, engine.err()
        rc = engine.lib.necgpu_solve_noalloc(engine.h, C.c_void_p(inside + 16), C.c_void_p(cur.data_ptr()), None)
        assert rc == 2 and "beyond its allocation" in engine.err()
    finally:
        torch.cuda.synchronize()
        rt.cudaFree(base)
    nb.nec_delete(ctx)


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
import necpp_b200 as nb
from cases import CASES
from gpu_helpers import Engine
from helpers import host_case
e = Engine(nb.lib)
nb.lib.necgpu_solve_noalloc.argtypes = [C.c_void_p] * 4
ctx, st, rhs, _ = host_case(nb, CASES["helix2"][0])
n = st["n"]
rhs_t = torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.complex128).view(np.float64)).cuda()
cur_t = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
abc_t = torch.zeros(6 * n, dtype=torch.float64, device="cuda")
def call():
    torch.cuda.synchronize()
    rc = nb.lib.necgpu_solve_noalloc(e.h, rhs_t.data_ptr(), cur_t.data_ptr(), abc_t.data_ptr())
    assert rc == 0, e.err()
e.set_structure(st)
e.fill()
e.factor(0)
call()                      # first call on the device: the set-up
e.fill()                    # the FP64 factorisation overwrote Z
e.factor(1)                 # mixed factors; no mixed solve has run in this process
torch.cuda.synchronize()
free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
call()                      # mixed refinement kernels, loaded by the set-up
free1, reserved1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
assert free1 == free0, ("device memory taken by the second call", free0 - free1)
assert reserved1 == reserved0
c = cur_t.cpu().numpy()
cur_ref, _ = e.solve(rhs)
err = np.max(np.abs(c[0::2] + 1j * c[1::2] - cur_ref)) / np.max(np.abs(cur_ref))
assert err <= 1e-10, err
print("fresh-process noalloc ok", err)
"""


def test_noalloc_allocates_nothing_after_the_first_call():
    """In a fresh process (lazy module loading as by default): FP64 factors,
    the first call (set-up), then mixed factors with no mixed solve run
    before; the second call must leave the device's free memory and
    PyTorch's reserved memory unchanged and match necgpu_solve."""
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([os.path.dirname(here), here, env.get("PYTHONPATH", "")])
    env.pop("CUDA_MODULE_LOADING", None)
    r = subprocess.run([sys.executable, "-c", _FRESH], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "fresh-process noalloc ok" in r.stdout
