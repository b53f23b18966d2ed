"""The precision form keeps only the q row types of the angular interpolation
grid (nGrid = 10 nDir rows repeat every q = nGrid / gcd(nDir, nGrid) rows,
shifted by p = nDir / gcd directions) and rebuilds row g as type g mod q
shifted by p (g div q).  This checks, on the reference's own interpolation
tables for every direction count the tests use, that the rebuilt 5-direction
windows (rows g and g+1 blended in t) act on the same directions with the
same weights as the rows themselves -- the property the context set-up
verifies before it uploads the table."""
import ctypes as C
from math import gcd

import numpy as np
import pytest


def host_rows(grlbm, nd):
    ng = 10 * nd
    idx = np.zeros(4 * ng, dtype=np.int64)
    w = np.zeros(4 * ng)
    rc = grlbm.lib().grlbm_host_stencil(nd, 1, None, None, None, None, idx.ctypes.data_as(C.POINTER(C.c_int64)),
                                        w.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return idx.reshape(ng, 4), w.reshape(ng, 4)


def window(idx, w, g, t, nd):
    """IntensityAt's blend of rows g and g+1 as weights over all directions."""
    ng = len(idx)
    out = np.zeros(nd)
    g1 = (g + 1) % ng
    for k in range(4):
        out[idx[g, k]] += (1 - t) * w[g, k]
        out[idx[g1, k]] += t * w[g1, k]
    return out


@pytest.mark.parametrize("nd", [4, 5, 8, 12, 16, 20, 24, 32, 48, 64, 200, 256])
def test_row_types_rebuild_every_row(grlbm, nd):
    idx, w = host_rows(grlbm, nd)
    ng = 10 * nd
    q, p = ng // gcd(nd, ng), nd // gcd(nd, ng)
    assert q <= 32
    rng = np.random.default_rng(nd)
    for g in range(ng):
        r, m = g % q, g // q
        for t in (0.0, float(rng.uniform()), 1.0):
            want = window(idx, w, g, t, nd)
            got = np.roll(window(idx, w, r, t, nd), p * m)
            assert np.abs(got - want).max() <= 1e-12, (g, t)
