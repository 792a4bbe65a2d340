"""Shared test helpers: host-only case driver, reference default frequency."""
import math

import numpy as np


def default_freq_mhz():
    """calc_prepare's default frequency, c / 1e6 with the reference's constants
    (src/electromag.cpp:22-29, src/nec_context.cpp:150)."""
    mu = (4.0 * 3.1415926536) * 1.0e-7
    eps = 8.854e-12
    return (1.0 / math.sqrt(mu * eps)) / 1.0e6


class HostOnly:
    """Runs a case's card sequence on the host library without simulating:
    rp/xq cards are recorded, not executed, so geometry, tables and the
    right-hand side can be built and inspected without a GPU."""

    def __init__(self, nb):
        self.nb = nb
        self.fr = None
        self.networks = []   # (card, tag1, seg1, tag2, seg2, six reals)

    def nec_nt_card(self, ctx, t1, s1, t2, s2, *x):
        self.networks.append(("NT", t1, s1, t2, s2, x))
        return self.nb.nec_nt_card(ctx, t1, s1, t2, s2, *x)

    def nec_tl_card(self, ctx, t1, s1, t2, s2, *x):
        self.networks.append(("TL", t1, s1, t2, s2, x))
        return self.nb.nec_tl_card(ctx, t1, s1, t2, s2, *x)

    def __getattr__(self, k):
        return getattr(self.nb, k)

    def helix(self, ctx, *a):
        return self.nb.nec_helix(ctx, *a)

    def nec_fr_card(self, ctx, ifrq, nfrq, f, df):
        self.fr = (ifrq, nfrq, f, df)
        return self.nb.nec_fr_card(ctx, ifrq, nfrq, f, df)

    def nec_rp_card(self, ctx, *a):
        return 0

    def nec_xq_card(self, ctx, *a):
        return 0

    def last_freq(self):
        """Frequency of the last step of the sweep, stepped as simulate does."""
        if self.fr is None:
            return default_freq_mhz()
        ifrq, nfrq, f, df = self.fr
        for _ in range(max(nfrq, 1) - 1):
            f = f * df if ifrq == 1 else f + df
        return f


def host_case(nb, builder):
    """Build a case on the host only; return (ctx, structure tables, rhs)."""
    api = HostOnly(nb)
    ctx = nb.nec_create()
    builder(api, ctx)
    st = nb.structure(ctx, api.last_freq())
    return ctx, st, nb.rhs(ctx), api


def zin_from_currents(cur_amps, feeds, voltages):
    return np.array([v / cur_amps[s] for s, v in zip(feeds, voltages)])
