"""The oracle (oracle/mom_oracle.c, a CPU restatement of the reference's
algorithm) pinned against the reference: its fill, solve, current
coefficients and far field against the golden fixtures the reference
produced (tests/golden/), and the published full-precision values of the
reference's own tests (testharness/python/test_examples.py)."""
import math

import numpy as np
import pytest

from cases import CASES
from conftest import golden
from helpers import host_case

NAMES = list(CASES)
NETWORK_CASES = ("array_tl", "dipole_nt")
PLAIN = [n for n in NAMES if n not in NETWORK_CASES]
ETA = math.sqrt((4.0 * 3.1415926536 * 1.0e-7) / 8.854e-12)


def _zcheck(g, Z):
    if "Z" in g:
        ref = g["Z"]
        return np.max(np.abs(Z - ref)) / np.max(np.abs(ref)), np.mean(Z == ref)
    idx = g["Z_idx"]
    vals = Z[idx[:, 0], idx[:, 1]]
    d = np.abs(vals - g["Z_val"]) / np.max(np.abs(g["Z_diag"]))
    dd = np.abs(np.diag(Z) - g["Z_diag"]) / np.max(np.abs(g["Z_diag"]))
    return max(d.max(), dd.max()), np.mean(vals == g["Z_val"])


# Sommerfeld-ground cases with pairs near their image: ground constants
# (relative permittivity, conductivity S/m) of their GN card
SOMM_GROUND = {"near_ground": (10.0, 0.01)}


def _sweep(api):
    from helpers import default_freq_mhz
    if api.fr is None:
        return [default_freq_mhz()]
    ifrq, nfrq, f, df = api.fr
    out = [f]
    for _ in range(max(nfrq, 1) - 1):
        f = f * df if ifrq == 1 else f + df
        out.append(f)
    return out


def _wavelength(f_mhz):
    return (1.0 / math.sqrt(((4.0 * 3.1415926536) * 1.0e-7) * 8.854e-12)) / (1.0e6 * f_mhz)


def _oracle_sweep(nb, oracle, name, ctx, api):
    """The case's frequency sweep on the oracle, in the reference's order:
    per frequency the fill, the solve and the near-field requests at the
    golden points.  Near-ground cases integrate the oracle's tables through
    one interpolation cache over the whole sweep.  Returns per frequency
    (Z, status, structure, abc, currents, near fields)."""
    g = golden(name)
    interp = oracle.new_interp()
    nearf = list(zip(g["near_nfeh"], np.split(g["near_xyz"], np.cumsum(g["near_np"])[:-1]))) \
        if "near_nfeh" in g else []
    freqs = _sweep(api)
    per = len(nearf) // len(freqs) if nearf else 0
    out = []
    for k, f in enumerate(freqs):
        sf = nb.structure(ctx, f)
        if name in SOMM_GROUND:
            epr, sig = SOMM_GROUND[name]
            sf["somm"], _ = oracle.sommerfeld(epr, sig, _wavelength(f), ETA)
            sf["interp"] = interp
        Z, status = oracle.fill(sf)
        rhs = nb.rhs(ctx)
        x, bad = oracle.solve(Z, rhs)
        assert bad == 0
        abc, cur = oracle.coefficients(sf, x)
        fields = [(nfeh, oracle.near_field(sf, abc, xyz / _wavelength(f), magnetic=nfeh == 1))
                  for nfeh, xyz in nearf[k * per:(k + 1) * per]]
        out.append((Z, status, sf, abc, cur, fields))
    return out


def _oracle_fill(nb, oracle, name, ctx, st, api, fresh=False):
    """The oracle's fill of the case's last frequency.  For near-ground
    cases the interpolation cache carries over from the earlier work of the
    sweep, as in the reference; fresh=True starts the last fill from a new
    cache instead."""
    if name not in SOMM_GROUND:
        return oracle.fill(st)
    if fresh:
        epr, sig = SOMM_GROUND[name]
        st["somm"], _ = oracle.sommerfeld(epr, sig, _wavelength(_sweep(api)[-1]), ETA)
        return oracle.fill(st)
    Z, status = _oracle_sweep(nb, oracle, name, ctx, api)[-1][:2]
    return Z, status


@pytest.mark.parametrize("name", NAMES)
def test_oracle_fill_matches_reference(nb, oracle, name):
    ctx, st, _, api = host_case(nb, CASES[name][0])
    Z, status = _oracle_fill(nb, oracle, name, ctx, st, api, fresh=True)
    # 1: rom2 reached its finest step (the reference prints a warning)
    assert status & ~1 == 0 and (status == 0 or name in SOMM_GROUND)
    err, exact = _zcheck(golden(name), Z)
    assert err <= 1e-14, err
    assert exact >= 0.999, exact  # the restatement rounds as the reference does
    nb.nec_delete(ctx)


@pytest.mark.parametrize("name", list(SOMM_GROUND))
def test_oracle_sommerfeld_tables_and_cache(nb, oracle, ref, name):
    """Sommerfeld tables (c_ggrid::sommerfeld) bit for bit, and the
    interpolation cache through a long random sequence of points, against
    the reference's own."""
    g = golden(name)
    ctx, st, _, api = host_case(nb, CASES[name][0])
    epr, sig = SOMM_GROUND[name]
    lam = float(g["wavelength"])
    tab, eps = oracle.sommerfeld(epr, sig, lam, ETA)
    assert eps == complex(g["somm_epscf"])
    assert np.array_equal(tab, g["somm_tables"])
    rc = ref.nec_create()
    CASES[name][0](ref, rc)
    ref.ref_somm_interp_reset(rc)
    interp = oracle.new_interp()
    rng = np.random.default_rng(3)
    # points wander between the three grids, below their starts included
    for x, y in zip(rng.uniform(0.0005, 0.99, 4000), rng.uniform(0.0, 1.5707963, 4000)):
        assert np.array_equal(oracle.interpolate(interp, tab, x, y), ref.somm_interpolate(rc, x, y))
    ref.nec_delete(rc)
    nb.nec_delete(ctx)


def _solve_case(nb, oracle, name):
    ctx, st, rhs, api = host_case(nb, CASES[name][0])
    Z, _ = _oracle_fill(nb, oracle, name, ctx, st, api)
    x, bad = oracle.solve(Z, rhs)
    assert bad == 0
    abc, cur = oracle.coefficients(st, x)
    return ctx, st, rhs, abc, cur


@pytest.mark.parametrize("name", [n for n in PLAIN if n != "plane_wave_reflection"])
def test_oracle_solution_matches_reference(nb, oracle, name):
    """LU + solve + current coefficients of the oracle against the
    reference's current_vector and coefficients of its last solve."""
    ctx, st, rhs, abc, cur = _solve_case(nb, oracle, name)
    g = golden(name)
    scale = np.max(np.abs(g["current_vector"]))
    assert np.max(np.abs(cur - g["current_vector"])) / scale <= 1e-10
    assert np.max(np.abs(abc.reshape(6, -1) - g["abc"])) / np.max(np.abs(g["abc"])) <= 1e-10
    nb.nec_delete(ctx)


def _zin(g, nb, st, rhs, cur):
    # voltage sources: e[seg] = -V / (s * lambda)  ->  V = -e * s * lambda
    lam = float(g["wavelength"])
    n = st["n"]
    s = st["seg"][3 * n:4 * n]
    feeds = np.nonzero(rhs)[0]
    v = -rhs[feeds] * s[feeds] * lam
    return v / (cur[feeds] * lam), v, feeds


@pytest.mark.parametrize("name", [n for n in PLAIN if n not in ("mesh_small", "plane_wave_reflection")])
def test_oracle_zin_matches_reference(nb, oracle, name):
    ctx, st, rhs, abc, cur = _solve_case(nb, oracle, name)
    g = golden(name)
    zin, _, _ = _zin(g, nb, st, rhs, cur)
    ref = g["zin"][-1]
    ref = ref[~np.isnan(ref)]
    assert np.max(np.abs(zin - ref) / np.abs(ref)) <= 1e-10
    nb.nec_delete(ctx)


def _oracle_network(nb, oracle, name):
    from oracle import network as NW
    ctx, st, rhs, api = host_case(nb, CASES[name][0])
    g = golden(name)
    tags = g["seg_tags"]

    def absolute(tag, m):
        return m if tag == 0 else int(np.nonzero(tags == tag)[0][m - 1]) + 1

    nets = []
    for card, t1, s1, t2, s2, x in api.networks:
        x = list(x)
        typ = 1 if card == "NT" else 2
        if typ == 2 and x[0] <= 0.0:
            typ, x[0] = 3, -x[0]
        nets.append((typ, absolute(t1, s1), absolute(t2, s2), x))
    lam = float(g["wavelength"])
    nets = NW.tl_lengths(st, lam, nets)
    n = st["n"]
    s = st["seg"][3 * n:4 * n]
    feeds = np.nonzero(rhs)[0]
    sources = [(int(f) + 1, -rhs[f] * s[f] * lam) for f in feeds]
    Z, _ = oracle.fill(st)
    return ctx, g, NW.netwk(oracle, st, Z, rhs, lam, nets, sources)


@pytest.mark.parametrize("name", NETWORK_CASES)
def test_oracle_network_matches_reference(nb, oracle, name):
    """Network equations (NT two-ports, straight and crossed transmission
    lines, computed line length) restated in numpy over the C oracle's
    solves, against the reference's input impedances and last currents."""
    ctx, g, (cur, abc, zin, pin, loss) = _oracle_network(nb, oracle, name)
    ref = g["zin"][-1]
    ref = ref[~np.isnan(ref)]
    assert np.max(np.abs(zin - ref) / np.abs(ref)) <= 1e-10
    scale = np.max(np.abs(g["current_vector"]))
    assert np.max(np.abs(cur - g["current_vector"])) / scale <= 1e-10
    assert np.max(np.abs(abc.reshape(6, -1) - g["abc"])) / np.max(np.abs(g["abc"])) <= 1e-10
    # the ports really carry network current
    assert abs(loss) > 1e-6 * pin
    nb.nec_delete(ctx)


NEAR_CASES = [n for n in NAMES if "near_nfeh" in golden(n)]


@pytest.mark.parametrize("name", NEAR_CASES)
def test_oracle_near_fields_match_reference(nb, oracle, name):
    """Near E and H fields (nefld / nhfld over the nfpat grid) of the oracle
    against the reference's near-field patterns, every frequency."""
    ctx, st, rhs, api = host_case(nb, CASES[name][0])
    g = golden(name)
    ours = [f for step in _oracle_sweep(nb, oracle, name, ctx, api) for f in step[5]]
    offs = np.cumsum(np.concatenate([[0], g["near_np"]]))
    assert len(ours) == len(g["near_nfeh"])
    for k, (nfeh, f) in enumerate(ours):
        ref = g["near_f"][offs[k]:offs[k + 1]]
        assert nfeh == g["near_nfeh"][k]
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(f - ref)) <= 1e-10 * scale, (k, np.max(np.abs(f - ref)) / scale)
    nb.nec_delete(ctx)


def _gains(oracle, st, abc, lam, power, grid, th0=0.0, dth=10.0, ph0=0.0, dph=90.0, ground=False):
    nth, nph = grid
    gcon = lam * lam * 2.0 * 3.1415926536 / (ETA * power)
    rad = (2 * 3.1415926536) / 360.0
    out = np.full((nth, nph), np.nan)
    for p in range(nph):
        for t in range(nth):
            th = th0 + dth * t
            if ground and th > 90.01:
                continue
            eth, eph = oracle.ffld(st, abc, th * rad, (ph0 + dph * p) * rad)
            x = gcon * (abs(eth) ** 2 + abs(eph) ** 2)
            out[t, p] = -999.99 if x < 1e-20 else 10 * math.log10(x)  # db10, math_util.h:134-139
    return out


def test_published_example1_zin(nb, oracle):
    """test_examples.py:35-36: Zin = 82.69792906662622 + j46.30603888063429."""
    ctx, st, rhs, abc, cur = _solve_case(nb, oracle, "ex1")
    zin, _, _ = _zin(golden("ex1"), nb, st, rhs, cur)
    want = complex(82.69792906662622, 46.30603888063429)
    assert abs(zin[0] - want) / abs(want) <= 1e-12
    nb.nec_delete(ctx)


@pytest.mark.parametrize("name,zin_want,gmax_want,places", [
    # test_examples.py:119-121 (EK, perfect ground) and 126-128 (finite ground)
    ("ex3_perfect", complex(83.7552291016712, 45.32205265591289), 8.393875976328134, 12),
    ("ex3_finite", complex(86.415, 47.822), 1.44837, 3),
])
def test_published_example3(nb, oracle, name, zin_want, gmax_want, places):
    ctx, st, rhs, abc, cur = _solve_case(nb, oracle, name)
    g = golden(name)
    zin, v, feeds = _zin(g, nb, st, rhs, cur)
    lam = float(g["wavelength"])
    power = float(np.sum(0.5 * np.real(v * np.conj(cur[feeds] * lam))))
    gains = _gains(oracle, st, abc, lam, power, (10, 2), ground=True)
    if places >= 12:
        assert abs(zin[0] - zin_want) / abs(zin_want) <= 1e-12
        assert abs(np.nanmax(gains) - gmax_want) <= 1e-10
    else:
        assert abs(zin[0].real - zin_want.real) < 10 ** -places * 0.5 * 10
        assert abs(zin[0].imag - zin_want.imag) < 10 ** -places * 0.5 * 10
        assert abs(np.nanmax(gains) - gmax_want) < 10 ** -places * 0.5 * 10
    nb.nec_delete(ctx)


def test_oracle_far_field_matches_reference(nb, oracle, ref):
    """Direct comparison of the far-field sum with the reference's ffld."""
    from necpp_b200 import workloads as W
    ctx, st, rhs, abc, cur = _solve_case(nb, oracle, "yagi_ek_perfect")
    rc = ref.nec_create()
    CASES["yagi_ek_perfect"][0](ref, rc)
    rng = np.random.default_rng(0)
    for th, ph in rng.uniform(0, 1.5, size=(8, 2)):
        a = oracle.ffld(st, abc, th, ph * 4)
        b = ref.ffld(rc, th, ph * 4)
        assert abs(a[0] - b[0]) <= 1e-11 * (abs(b[0]) + 1e-30)
        assert abs(a[1] - b[1]) <= 1e-11 * (abs(b[1]) + 1e-30) + 1e-14
    ref.nec_delete(rc)
    nb.nec_delete(ctx)
