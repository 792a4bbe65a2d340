"""Tuning of the mixed LU (necgpu_tuning): the table lookup on the host, the
committed table, and parity of the mixed path under tuned blockings."""
import ctypes as C
import os

import numpy as np
import pytest

from cases import CASES
from conftest import golden


class Tuning(C.Structure):
    _fields_ = [("outer", C.c_int), ("lookahead_sms", C.c_int), ("gemm_group", C.c_int)]


def _lookup(nb, path, precision, n):
    L = nb.lib
    L.necgpu_tuning_lookup.argtypes = [C.c_char_p, C.c_int, C.c_int64, C.POINTER(Tuning)]
    t = Tuning()
    rc = L.necgpu_tuning_lookup(None if path is None else path.encode(), precision, n, C.byref(t))
    return rc, (t.outer, t.lookahead_sms, t.gemm_group)


def test_table_lookup_bands(nb, tmp_path):
    p = tmp_path / "t.tsv"
    p.write_text("# comment\n"
                 "mixed 1000 128 0 8  # small\n"
                 "mixed 5000 256 32 16\n"
                 "  mixed 1073741824 512 64 32\n"
                 "fp64 100000 64 0 4\n")
    assert _lookup(nb, str(p), 1, 500) == (0, (128, 0, 8))
    assert _lookup(nb, str(p), 1, 1000) == (0, (128, 0, 8))
    assert _lookup(nb, str(p), 1, 1001) == (0, (256, 32, 16))
    assert _lookup(nb, str(p), 1, 11520) == (0, (512, 64, 32))
    assert _lookup(nb, str(p), 0, 11520) == (0, (64, 0, 4))
    assert _lookup(nb, str(p), 0, 10 ** 6) == (0, (64, 0, 4))  # beyond every row: the largest


def test_table_rejects_bad_rows(nb, tmp_path):
    defaults = (256, 48, 16)
    for bad in ("mixed 1000 100 0 8\n",        # outer not a multiple of 64
                "mixed 1000 256 200 8\n",      # lookahead beyond 127
                "mixed 1000 256 48\n",         # a field missing
                "double 1000 256 48 16\n"):    # unknown precision
        p = tmp_path / "bad.tsv"
        p.write_text(bad)
        assert _lookup(nb, str(p), 1, 500) == (2, defaults), bad
    assert _lookup(nb, str(tmp_path / "missing.tsv"), 1, 500) == (2, defaults)
    p = tmp_path / "fp64only.tsv"
    p.write_text("fp64 1000 256 48 16\n")
    assert _lookup(nb, str(p), 1, 500) == (2, defaults)


def test_committed_table_parses(nb):
    path = os.path.join(os.path.dirname(nb.__file__), "tuning.tsv")
    if not os.path.exists(path):
        pytest.skip("no tuning table committed")
    for n in (180, 720, 2880, 11520, 40000):
        rc, t = _lookup(nb, path, 1, n)
        assert rc == 0 and t[0] % 64 == 0, (n, t)


TUNINGS = [(128, 0, 8), (512, 64, 32), (384, 32, 1)]


def _set_tuning(nb, e, tuning):
    L = nb.lib
    L.necgpu_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    L.necgpu_get_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.POINTER(Tuning)]
    t = Tuning(*tuning)
    e.check(L.necgpu_set_tuning(e.h, C.byref(t)))
    got = Tuning()
    e.check(L.necgpu_get_tuning(e.h, 1, 1000, C.byref(got)))
    assert (got.outer, got.lookahead_sms, got.gemm_group) == tuning


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", TUNINGS)
@pytest.mark.parametrize("name", ["helix2", "mesh_small", "yagi_ground"])
def test_tuned_blocking_keeps_parity(nb, oracle, name, tuning):
    """The mixed path under non-default blockings refines to the FP64 floor
    and matches the oracle's currents to 1e-9, as with the defaults."""
    from gpu_helpers import Engine
    from helpers import host_case
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur_o = oracle.coefficients(st, x)
    e = Engine(nb.lib)
    try:
        _set_tuning(nb, e, tuning)
        e.set_structure(st)
        e.fill()
        e.factor(1)
        cur, _ = e.solve(rhs)
        assert e.stats().refine_residual <= 1e-12
        assert np.max(np.abs(cur - cur_o)) / np.max(np.abs(cur_o)) <= 1e-9
    finally:
        e.close()
        nb.nec_delete(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", TUNINGS)
def test_tuned_block_lu_backward_error(nb, tuning):
    """The block-pivoted LU self-check (P A = L U on a seeded random matrix of
    3,000 unknowns) under each tuned blocking."""
    from gpu_helpers import Engine
    e = Engine(nb.lib)
    try:
        _set_tuning(nb, e, tuning)
        L = nb.lib
        L.necgpu_check_block_lu.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double), C.POINTER(C.c_int)]
        be, mx, moved = C.c_double(), C.c_double(), C.c_int()
        e.check(L.necgpu_check_block_lu(e.h, 3000, 7, C.byref(be), C.byref(mx), C.byref(moved)))
        assert be.value <= 5e-4 and moved.value > 1000
    finally:
        e.close()


@pytest.mark.gpu
def test_lu_graph_replay_matches_eager(nb, oracle):
    """The block-pivoted LU runs eagerly the first time a size, tuning and
    buffer set are seen, is captured as a CUDA graph the second time and
    replayed after that: all three give the same currents bit for bit, and
    they match the oracle."""
    from gpu_helpers import Engine
    from helpers import host_case
    ctx, st, rhs, _ = host_case(nb, CASES["helix2"][0])
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur_o = oracle.coefficients(st, x)
    e = Engine(nb.lib)
    try:
        e.set_structure(st)
        curs, launches = [], []
        for _ in range(4):
            e.fill()
            l0 = e.stats().launches
            e.factor(1)
            launches.append(e.stats().launches - l0)
            cur, _ = e.solve(rhs)
            curs.append(cur)
        for c in curs[1:]:
            assert np.array_equal(c, curs[0])
        assert np.max(np.abs(curs[0] - cur_o)) / np.max(np.abs(cur_o)) <= 1e-9
        # the replays account for the launches the graph holds
        assert launches[2] == launches[1] == launches[3] and launches[0] >= launches[1] > 0
    finally:
        e.close()
        nb.nec_delete(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("clusters", ["16", "8", "0"])
@pytest.mark.parametrize("name", ["helix2", "mesh_small"])
def test_sweep_forms_keep_parity(nb, oracle, name, clusters, monkeypatch):
    """The refinement sweeps in clusters of 16 or 8 CTAs (blocks handed over
    in shared memory) and without clusters (every block polled in global
    memory, the form taken when the clustered launch is refused) refine to
    the FP64 floor and match the oracle's currents to 1e-9."""
    from gpu_helpers import Engine
    from helpers import host_case
    monkeypatch.setenv("NECPP_B200_SWEEP_CLUSTER", clusters)
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur_o = oracle.coefficients(st, x)
    e = Engine(nb.lib)
    try:
        e.set_structure(st)
        e.fill()
        e.factor(1)
        cur, _ = e.solve(rhs)
        assert e.stats().refine_residual <= 1e-12
        assert np.max(np.abs(cur - cur_o)) / np.max(np.abs(cur_o)) <= 1e-9
    finally:
        e.close()
        nb.nec_delete(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [1, 2])
@pytest.mark.parametrize("name", ["helix2", "mesh_small", "yagi_ground"])
def test_update_formats_keep_parity(nb, oracle, name, fmt):
    """Both operand formats of the mixed LU's tensor-core update (1: split
    BF16, 2: TF32) refine to the FP64 floor and match the oracle's currents
    to 1e-9; the held factors report the format they were made in."""
    from gpu_helpers import Engine
    from helpers import host_case
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur_o = oracle.coefficients(st, x)
    e = Engine(nb.lib)
    try:
        e.set_update_format(fmt)
        e.set_structure(st)
        e.fill()
        assert e.update_format() == 0  # nothing factored yet
        e.factor(1)
        assert e.update_format() == fmt
        cur, _ = e.solve(rhs)
        assert e.stats().refine_residual <= 1e-12
        assert np.max(np.abs(cur - cur_o)) / np.max(np.abs(cur_o)) <= 1e-9
    finally:
        e.close()
        nb.nec_delete(ctx)


@pytest.mark.gpu
def test_update_format_choice_and_demotion(nb, monkeypatch):
    """The engine's own choice: split BF16 below the TF32 threshold; with
    the threshold lowered, TF32 first, and after a TF32 factorisation whose
    refinement took more than five steps (the 41 + 41-wire mesh of 3,280
    unknowns takes about twelve, against six with split BF16) split BF16
    for the engine's later factorisations, with the same currents."""
    from gpu_helpers import Engine
    from helpers import host_case
    from cases import LARGE_CASES
    ctx, st, rhs, _ = host_case(nb, LARGE_CASES["wire_mesh_41"][0])
    e = Engine(nb.lib)
    try:
        e.set_structure(st)
        e.fill()
        e.factor(1)
        assert e.update_format() == 1  # 3,280 unknowns: below the threshold
        cur_ref, _ = e.solve(rhs)
        iters_bf16 = e.stats().refine_iters
    finally:
        e.close()
    monkeypatch.setenv("NECPP_B200_TF32_MIN_N", "1000")
    e = Engine(nb.lib)
    try:
        e.set_structure(st)
        e.fill()
        e.factor(1)
        assert e.update_format() == 2
        cur1, _ = e.solve(rhs)
        s1 = e.stats()
        assert s1.refine_residual <= 1e-12 and s1.refine_iters > max(5, iters_bf16)
        e.fill()
        e.factor(1)
        assert e.update_format() == 1  # demoted for the rest of the engine's life
        cur2, _ = e.solve(rhs)
        assert e.stats().refine_iters == iters_bf16
        for c in (cur1, cur2):
            assert np.max(np.abs(c - cur_ref)) / np.max(np.abs(cur_ref)) <= 1e-9
    finally:
        e.close()
        nb.nec_delete(ctx)
