"""Host side of the boundary (CPU): geometry, connection tables and trio
basis tables against the reference's golden fixtures, bit for bit; the C
API's error behaviour; the exported symbol set."""
import os
import re

import numpy as np
import pytest

from cases import CASES
from conftest import ROOT, golden
from helpers import host_case

NAMES = list(CASES)


@pytest.mark.parametrize("name", NAMES)
def test_connection_tables_bit_exact(nb, name):
    ctx, st, _, _ = host_case(nb, CASES[name][0])
    g = golden(name)
    seg = nb.segments(ctx)
    for k in ("tags", "icon1", "icon2"):
        assert np.array_equal(seg[k], g["seg_" + k]), k
    nb.nec_delete(ctx)


@pytest.mark.parametrize("nw,nseg,offset", [(11, 12, 0.0), (9, 16, 0.37)])
def test_connection_grid_search_matches_reference(nb, ref, nw, nseg, offset):
    """Structures above 256 segments use the bucketed endpoint search: a
    wire mesh (4-way junctions, several candidate ends per end) and its
    connection tables against the reference's cyclic scan, run here."""
    from necpp_b200 import workloads as W
    ctxs = []
    for api in (nb, ref):
        ctx = api.nec_create()
        for k in range(nw):
            y = -1.0 + 2.0 * k / (nw - 1) + offset
            assert api.nec_wire(ctx, k + 1, nseg, -1.0 + offset, y, 0.2, 1.0 + offset, y, 0.2, 1e-3, 1.0, 1.0) == 0
            x = -1.0 + 2.0 * k / (nw - 1) + offset
            assert api.nec_wire(ctx, nw + k + 1, nseg, x, -1.0 + offset, 0.2, x, 1.0 + offset, 0.2, 1e-3, 1.0,
                                1.0) == 0
        assert api.nec_geometry_complete(ctx, 0) == 0
        ctxs.append((api, ctx))
    ours = nb.segments(ctxs[0][1])
    theirs = ref.segments(ctxs[1][1])
    assert len(ours["icon1"]) == 2 * nw * nseg > 256
    for k in ("icon1", "icon2"):
        assert np.array_equal(ours[k], theirs[k]), k
    nb.nec_delete(ctxs[0][1])
    ref.nec_delete(ctxs[1][1])


@pytest.mark.parametrize("name", NAMES)
def test_scaled_segments_bit_exact(nb, name):
    ctx, st, _, _ = host_case(nb, CASES[name][0])
    g = golden(name)
    n = st["n"]
    for k, key in enumerate(("x", "y", "z", "si", "bi", "cab", "sab", "salp")):
        assert np.array_equal(st["seg"][k * n:(k + 1) * n], g["seg_" + key]), key
    nb.nec_delete(ctx)


@pytest.mark.parametrize("name", NAMES)
def test_trio_tables_bit_exact(nb, name):
    ctx, st, _, _ = host_case(nb, CASES[name][0])
    g = golden(name)
    assert np.array_equal(st["tptr"], g["trio_ptr"])
    assert np.array_equal(st["tbasis"] + 1, g["trio_basis"])
    nt = len(st["tbasis"])
    abc = np.stack([st["tabc"][:nt], st["tabc"][nt:2 * nt], st["tabc"][2 * nt:]], axis=1)
    assert np.array_equal(abc, g["trio_abc"])
    nb.nec_delete(ctx)


def test_helix_array_full_size_tables(nb):
    """8 x 8 helix array (N = 11520): connectivity of every helix is a single
    open chain; tables are built in well under a second."""
    from helpers import HostOnly
    from necpp_b200 import workloads as W
    api = HostOnly(nb)
    ctx = nb.nec_create()
    W.helix_array(api, ctx, k=8)
    st = nb.structure(ctx, 1000.0)
    seg = nb.segments(ctx)
    n = st["n"]
    assert n == 11520
    # each helix: end 1 of its first and end 2 of its last segment are free
    assert np.sum(seg["icon1"] == 0) == 64 and np.sum(seg["icon2"] == 0) == 64
    assert np.all(np.diff(st["tptr"]) <= 3)
    nb.nec_delete(ctx)


# ---------------------------------------------------------------- errors
def test_errors_and_sentinels(nb):
    ctx = nb.nec_create()
    assert nb.nec_impedance_real(ctx, 0) == -999.0
    assert nb.nec_gain_max(ctx, 0) == -999.0
    assert nb.nec_gain(ctx, 0, 0, 0) == -999.0
    # one segment only: geometry_complete refuses (c_geometry.cpp:1340-1342)
    assert nb.nec_wire(ctx, 1, 1, 0, 0, 0, 0, 0, 1, 1e-3, 1, 1) == 0
    assert nb.nec_geometry_complete(ctx, 0) == 1
    assert "ONE OR FEWER SEGMENTS" in nb.nec_error_message()
    nb.nec_delete(ctx)

    ctx = nb.nec_create()
    assert nb.nec_geometry_complete(ctx, 0) == 1  # no wires
    nb.nec_delete(ctx)

    ctx = nb.nec_create()
    nb.nec_wire(ctx, 1, 9, 0, 0, -1, 0, 0, 1, 1e-3, 1, 1)
    # overlapping second wire: segment centre inside the first wire
    nb.nec_wire(ctx, 2, 9, 0, 0.0005, -1, 0, 0.0005, 1, 1e-3, 1, 1)
    assert nb.nec_geometry_complete(ctx, 0) == 1
    assert "MIDPOINT LIES WITHIN" in nb.nec_error_message()
    nb.nec_delete(ctx)

    ctx = nb.nec_create()
    nb.nec_wire(ctx, 1, 9, 0, 0, -1, 0, 0, 1, 1e-3, 1, 1)
    assert nb.nec_geometry_complete(ctx, 0) == 0
    # source segment beyond the tag's range
    assert nb.nec_ex_card(ctx, 0, 1, 10, 0, 1.0, 0, 0, 0, 0, 0) == 1
    assert "NO SEGMENT HAS AN ITAG" in nb.nec_error_message()
    assert nb.nec_ex_card(ctx, 0, 7, 1, 0, 1.0, 0, 0, 0, 0, 0) == 1
    # cards outside the hot path exist and refuse
    for call in (lambda: nb.nec_sp_card(ctx, 0, 0, 0, 0, 0, 0, 0),
                 lambda: nb.nec_cp_card(ctx, 1, 1, 1, 2)):
        assert call() == 1
        assert "not part of the B200" in nb.nec_error_message()
    # NT port on a tag that does not exist (c_geometry.cpp:76-99)
    assert nb.nec_nt_card(ctx, 1, 1, 4, 2, 0, 0, 0, 0, 0, 0) == 1
    assert "NO SEGMENT HAS AN ITAG OF 4" in nb.nec_error_message()
    assert nb.nec_network_count(ctx) == 0
    assert nb.nec_tl_card(ctx, 1, 2, 1, 8, 50.0, 0, 0, 0, 0, 0) == 0
    assert nb.nec_network_count(ctx) == 1
    # LD range reversed (nec_context.cpp:465-470)
    assert nb.nec_ld_card(ctx, 0, 1, 5, 3, 10.0, 0, 0) == 1
    assert "ITAG STEP1: 5 IS GREATER THAN ITAG STEP2: 3" in nb.nec_error_message()
    # GN with zero conductivity (nec_ground.cpp:111-117)
    assert nb.nec_gn_card(ctx, 0, 0, 10.0, 0.0, 0, 0, 0, 0) == 1
    assert "CONDUCTIVITY IS ZERO" in nb.nec_error_message()
    nb.nec_delete(ctx)


def test_below_ground_rejected(nb):
    ctx = nb.nec_create()
    nb.nec_wire(ctx, 1, 5, 0, 0, -1, 0, 0, 1, 1e-3, 1, 1)
    assert nb.nec_geometry_complete(ctx, 1) == 1
    assert "EXTENDS BELOW GROUND" in nb.nec_error_message()
    nb.nec_delete(ctx)


# ---------------------------------------------------------------- exports
def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b((?:nec|necgpu)_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol(nb):
    import ctypes
    lib = ctypes.CDLL(nb._LIBPATH)
    names = _declared("libnecpp.h") | _declared("necgpu.h")
    assert len(names) > 60
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("along_x", [False, True])
@pytest.mark.parametrize("nseg", [9, 200, 1500])
@pytest.mark.parametrize("z0", [-1.0, 0.3])
def test_overlap_check_matches_reference(nb, ref, nseg, z0, along_x):
    """The segment-overlap check (a midpoint inside another segment) gives
    the reference's message, segment pair and distance both below the grid
    search's size (the scan) and above it (cell grids over the ends and the
    centres, end cells of four times the contact distance).  With several
    overlapping pairs the reported one is the first of the reference's
    sweep along the widest axis (z, or x when the wires lie along x)."""
    def p(u, v, w):  # (offset, offset, position along the wires)
        return (w, u, v) if along_x else (u, v, w)
    msgs = []
    for api in (nb, ref):
        ctx = api.nec_create()
        api.nec_wire(ctx, 1, nseg, *p(0, 0, -1), *p(0, 0, 1), 1e-3, 1, 1)
        api.nec_wire(ctx, 2, nseg, *p(0, 0.0005, z0), *p(0, 0.0005, 1 + (1 + z0)), 1e-3, 1, 1)
        rc = api.nec_geometry_complete(ctx, 0)
        msgs.append((rc, nb.nec_error_message() if api is nb else ref.error()))
        api.nec_delete(ctx)
    assert msgs[0][0] == 1 and "MIDPOINT LIES WITHIN" in msgs[0][1]
    assert msgs[0] == msgs[1]
