"""The allocation-free plane-moments entry point against the context path.

chan_avg_spatial_noalloc serves callers that cannot allocate device memory,
such as the reference's Fortran post-processing programs, which have no
binding to cudaMalloc and keep no solver context.  It stages the field
through a static 32 MiB device array.  Its moments must equal those of the
existing entry points chan_avg_spatial + chan_stats on the same field bit for
bit (both reduce every plane in the same order), and must stay equal on a
second call that reuses the same array.  The relative difference against the
parity tolerance used everywhere (1e-12 per moment row) is reported when they
differ.
"""
import ctypes

import numpy as np
import pytest

from chan_cases import make_case
from compchan3dmpi_b200 import Channel, _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(var, nP):
    L = _lib.load()
    n3 = nP[2]
    s1 = np.full((7, n3), np.nan); s2 = np.full((7, n3), np.nan); c = np.full((9, n3), np.nan)
    nPc = (ctypes.c_int32 * 3)(*nP)
    rc = L.chan_avg_spatial_noalloc(_lib.dptr(np.ascontiguousarray(var)), nPc, _lib.dptr(s1), _lib.dptr(s2),
                                    _lib.dptr(c), 0)
    return rc, s1, s2, c


def _close(a, b):
    for r in range(a.shape[0]):
        den = max(np.max(np.abs(b[r])), 1e-300)
        rel = np.max(np.abs(a[r] - b[r])) / den
        assert np.array_equal(a[r], b[r]), f"row {r}: not bitwise equal, relative difference {rel:.3e} (tolerance {TOL})"


@pytest.mark.parametrize("nP", [(40, 24, 33), (160, 96, 65)])   # one slab, and two slabs of the 32 MiB area
def test_noalloc_moments_match_context_path_twice(nP):
    p, x3, jac, inv, var = make_case(nP=nP, quantize=False, istat=0)
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    g.step(2)
    field = g.download()
    g.avg_spatial()
    _, e1, e2, ec = g.stats()
    for call in range(2):
        rc, s1, s2, c = _noalloc(field, p.nP)
        assert rc == 0, _lib.load().chan_last_error(None)
        _close(s1, e1)
        _close(s2, e2)
        _close(c, ec)
    g.close()


def test_noalloc_rejects_grids_beyond_the_fixed_area():
    L = _lib.load()
    nP = (1100, 560, 7)       # 7*nP1*nP2 = 4.31M doubles > 4,194,304
    dummy = np.zeros(8)
    out = np.zeros(64)
    nPc = (ctypes.c_int32 * 3)(*nP)
    rc = L.chan_avg_spatial_noalloc(_lib.dptr(dummy), nPc, _lib.dptr(out), _lib.dptr(out), _lib.dptr(out), 0)
    assert rc == -1
    assert b"exceeds the fixed area" in L.chan_last_error(None)
