"""Batched sweeps (necgpu_batch_solve): a small seeded Yagi-Uda sweep
against the single-structure path through the C API on the same cards.
Both refine to the FP64 floor, so input impedances agree to 1e-9 and gains
to 1e-6 dB."""
import numpy as np
import pytest


def test_yagi_problems_host_tables(nb):
    from necpp_b200 import batch as B
    problems, labels = B.yagi_problems(nvariants=3, nfreq=2, seed=5)
    assert len(problems) == 6 and len(labels) == 6
    for (st, b, feed, v, lam), (var, f) in zip(problems, labels):
        n = st["n"]
        assert 33 <= n <= 615 and len(b) == n and 0 <= feed < n
        assert abs(b[feed]) > 0 and np.count_nonzero(b) == 1  # one voltage source
        assert abs(lam - 299.8e6 / (f * 1e6)) / lam < 1e-3


def test_struct_array_matches_ctypes_layout(nb):
    """The record array handed to necgpu_batch_solve is byte for byte the
    ctypes necgpu_structure of each problem."""
    from necpp_b200 import batch as B
    problems, _ = B.yagi_problems(nvariants=3, nfreq=2, seed=2)
    arr = B.struct_array([p[0] for p in problems])
    for k, p in enumerate(problems):
        s, _ = B.to_struct(p[0])
        assert bytes(memoryview(s)) == arr[k].tobytes()


def _single(nb, params, f, nth, nph, dth, dph):
    half, xs, rad, segs = params
    ctx = nb.nec_create()
    for e in range(len(half)):
        assert nb.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                           float(half[e]), float(rad[e]), 1.0, 1.0) == 0
    nb.nec_geometry_complete(ctx, 0)
    nb.nec_fr_card(ctx, 0, 1, f, 0.0)
    nb.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    assert nb.nec_rp_card(ctx, 0, nth, nph, 1, 0, 0, 0, 0.0, 0.0, dth, dph, 0.0, 0.0) == 0, nb.nec_error_message()
    z = complex(nb.nec_impedance_real(ctx, 0), nb.nec_impedance_imag(ctx, 0))
    g = np.array([[nb.nec_gain(ctx, 0, t, p) for t in range(nth)] for p in range(nph)]).ravel()
    nb.nec_delete(ctx)
    return z, g


@pytest.mark.gpu
def test_batch_matches_single_path(nb):
    from necpp_b200 import batch as B
    from necpp_b200 import workloads as W
    nvar, nfreq, seed = 5, 3, 11
    problems, labels = B.yagi_problems(nvariants=nvar, nfreq=nfreq, f0=140.0, f1=160.0, seed=seed)
    nth, nph, dth, dph = 10, 8, 10.0, 45.0
    th, ph = B.pattern_grid(nth, nph, dth, dph)
    res = B.sweep(problems, th, ph, fields=True)
    assert np.all(res["status"] == 0), res["status"]
    assert np.all(res["residual"] <= 1e-12), res["residual"]
    rng = np.random.default_rng(seed)
    params = [W.yagi_params(rng) for _ in range(nvar)]
    for k, (v, f) in enumerate(labels):
        z, g = _single(nb, params[v], f, nth, nph, dth, dph)
        assert abs(res["zin"][k] - z) / abs(z) <= 1e-9, (k, res["zin"][k], z)
        strong = g > np.max(g) - 60.0
        # gains are returned in float32 (dB): 1e-4 dB resolution at these levels
        assert np.max(np.abs(res["gain"][k][strong] - g[strong])) <= 1e-4
        # the complex fields give the FP64 gains
        eta = problems[k][0]["params"][7]
        lam = problems[k][4]
        i = res["cur"][res["offsets"][k] + problems[k][2]]
        pin = 0.5 * (problems[k][3] * np.conj(i)).real
        gcop = lam * lam * 2.0 * 3.1415926536 / (eta * pin)
        pw = gcop * (np.abs(res["eth"][k]) ** 2 + np.abs(res["eph"][k]) ** 2)
        with np.errstate(divide="ignore"):
            g64 = 10 * np.log10(pw)
        assert np.max(np.abs(g64[strong] - g[strong])) <= 1e-6


@pytest.mark.gpu
def test_batch_rejects_oversized_problem(nb):
    from necpp_b200 import batch as B
    ctx = nb.nec_create()
    nb.nec_wire(ctx, 1, 641, 0.0, 0.0, -5.0, 0.0, 0.0, 5.0, 1e-3, 1.0, 1.0)
    nb.nec_geometry_complete(ctx, 0)
    nb.nec_ex_card(ctx, 0, 1, 321, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    prob = B.host_problem(ctx, 30.0, 320)
    nb.nec_delete(ctx)
    with pytest.raises(RuntimeError, match="640"):
        B.sweep([prob])


@pytest.mark.gpu
def test_batch_matches_reference_sweep(nb):
    """Twelve problems of the seeded 256 x 32 Yagi sweep (seed 0), spread
    over its range of N, solved in one batched call and compared with the
    reference's own solves of the same problems (tests/golden/yagi_sweep.npz,
    made by make_sweep_golden.py): Zin within 1e-9 relative, the float32
    gain grid within 1e-4 dB where the gain is within 60 dB of its peak."""
    import os
    from necpp_b200 import batch as B
    from necpp_b200 import workloads as W
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "yagi_sweep.npz"))
    rng = np.random.default_rng(0)
    params = [W.yagi_params(rng) for _ in range(256)]
    freqs = np.linspace(140.0, 160.0, 32)
    problems = []
    for v, fi in g["pick"]:
        half, xs, rad, segs = params[v]
        ctx = nb.nec_create()
        for e in range(len(half)):
            assert nb.nec_wire(ctx, e + 1, int(segs[e]), float(xs[e]), 0.0, -float(half[e]), float(xs[e]), 0.0,
                               float(half[e]), float(rad[e]), 1.0, 1.0) == 0
        nb.nec_geometry_complete(ctx, 0)
        nb.nec_ex_card(ctx, 0, 2, (int(segs[1]) + 1) // 2, 0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        feed = int(segs[0]) + (int(segs[1]) + 1) // 2 - 1
        problems.append(B.host_problem(ctx, float(freqs[fi]), feed))
        nb.nec_delete(ctx)
    assert [p[0]["n"] for p in problems] == list(g["n"])
    th, ph = B.pattern_grid()
    res = B.sweep(problems, th, ph)
    assert np.all(res["status"] == 0), res["status"]
    rel = np.abs(res["zin"] - g["zin"]) / np.abs(g["zin"])
    assert np.max(rel) <= 1e-9, rel
    for k in range(len(problems)):
        ref = g["gain"][k].astype(np.float64)
        strong = ref > np.max(ref) - 60.0
        assert np.max(np.abs(res["gain"][k][strong] - ref[strong])) <= 1e-4, k
