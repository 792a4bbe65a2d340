"""NumPy restatement of the reference's network solve (NT/TL cards).

Test infrastructure: only tests/ use it, as the checker of the product's
network path.  It follows src/nec_context.cpp:
  calculate_network_data  1210-1243   (transmission-line lengths)
  netwk_solve_and_check   4638-4845   (port rows, admittances, unit solves)
  netwk_compute_currents  4850-4925   (port voltages, final solve, losses)
  netwk_compute_inputs    4930-5003   (source currents with network terms)
and the un-transposed lu_decompose / solve of src/matrix_algebra.cpp:217-307
for the network equations.  Structure solves go through the C oracle
(mo_lu / mo_solve / mo_coefficients).
"""
import math

import numpy as np

TWO_PI = 2.0 * 3.1415926536


def tl_lengths(st, lam, networks):
    """Lengths (m) of transmission lines given with length <= 0: the
    distance between the two port segment centres."""
    n = st["n"]
    x, y, z = st["seg"][0:n], st["seg"][n:2 * n], st["seg"][2 * n:3 * n]
    out = []
    for typ, s1, s2, p in networks:
        p = list(p)
        if typ >= 2 and p[1] <= 0.0:
            a, b = s1 - 1, s2 - 1
            p[1] = lam * math.sqrt((x[b] - x[a]) ** 2 + (y[b] - y[a]) ** 2 + (z[b] - z[a]) ** 2)
        out.append((typ, s1, s2, p))
    return out


def _admittances(typ, p, lam):
    if typ <= 1:
        return complex(p[0], p[1]), complex(p[2], p[3]), complex(p[4], p[5])
    bl = TWO_PI * p[1] / lam
    b12 = 1.0 / (p[0] * math.sin(bl))
    b11 = -b12 * math.cos(bl)
    y12 = complex(0.0, b12 if typ == 2 else -b12)
    return complex(p[2], b11 + p[3]), y12, complex(p[4], b11 + p[5])


def netwk(oracle, st, Z, einc, lam, networks, sources):
    """networks: [(type 1|2|3, seg1, seg2, [x11r, x11i, x12r, x12i, x22r,
    x22i])] with 1-based segments and resolved line lengths (metres);
    sources: [(seg, voltage)].  Returns the segment currents, the current
    coefficients, per-source input impedances, the input power and the
    network power loss."""
    n = st["n"]
    seglen = st["seg"][3 * n:4 * n]

    def solve(rhs):
        x, bad = oracle.solve(Z, rhs)
        assert bad == 0
        abc, cur = oracle.coefficients(st, x)
        return cur, abc

    nsrc = len(sources)
    ndimn = 2 * len(networks) + nsrc
    cmn = np.zeros((ndimn, ndimn), complex)   # cmn[c, r]: row r, column c
    rhnx = np.zeros(ndimn, complex)
    nteqa, ntsca, vsrc = [], [], []
    src_seg = [s for s, _ in sources]

    def row(seg):
        if seg in src_seg:
            isc = src_seg.index(seg)
            if seg not in ntsca:
                ntsca.append(seg)
                vsrc.append(sources[isc][1])
            return ndimn - (ntsca.index(seg) + 1), isc
        if seg not in nteqa:
            nteqa.append(seg)
        return nteqa.index(seg), -1

    for typ, s1, s2, p in networks:
        y11, y12, y22 = _admittances(typ, p, lam)
        r1, i1 = row(s1)
        r2, i2 = row(s2)
        if i1 == -1:
            cmn[r1, r1] -= y11 * seglen[s1 - 1]
            cmn[r1, r2] -= y12 * seglen[s1 - 1]
        else:
            rhnx[r1] += y11 * sources[i1][1] / lam
            rhnx[r2] += y12 * sources[i1][1] / lam
        if i2 == -1:
            cmn[r2, r2] -= y22 * seglen[s2 - 1]
            cmn[r2, r1] -= y12 * seglen[s2 - 1]
        else:
            rhnx[r1] += y12 * sources[i2][1] / lam
            rhnx[r2] += y22 * sources[i2][1] / lam
    nteq = len(nteqa)
    for i in range(nteq):
        e = np.zeros(n, complex)
        e[nteqa[i] - 1] = 1.0
        cur, _ = solve(e)
        for j in range(nteq):
            cmn[i, j] += cur[nteqa[j] - 1]
    e = np.array(einc, complex)
    cur, abc = solve(e)
    rhnt = np.zeros(ndimn, complex)
    if nteq:
        a = cmn[:nteq, :nteq].T   # row r, column c
        rhnt[:nteq] = np.linalg.solve(a, rhnx[:nteq] + np.array([cur[s - 1] for s in nteqa]))
        for i in range(nteq):
            e[nteqa[i] - 1] -= rhnt[i]
        cur, abc = solve(e)
    loss = 0.0
    for i in range(nteq):
        s = nteqa[i] - 1
        loss -= 0.5 * (rhnt[i] * seglen[s] * lam * np.conj(cur[s] * lam)).real
    for v, s in zip(vsrc, ntsca):
        loss -= 0.5 * (v * np.conj(cur[s - 1] * lam)).real
    zin, pin = [], 0.0
    for s, v in sources:
        c = cur[s - 1] * lam
        if ntsca:
            r = ndimn - (ntsca.index(s) + 1)
            t = rhnx[r] - np.dot(cmn[:nteq, r], rhnt[:nteq])
            c = (cur[s - 1] + t) * lam
            loss += 0.5 * (v * np.conj(c)).real
        pin += 0.5 * (v * np.conj(c)).real
        zin.append(v / c)
    return cur, abc, np.array(zin), pin, loss
