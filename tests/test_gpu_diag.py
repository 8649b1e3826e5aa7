"""Diagnostics series, fluctuation field and Q-criterion of the sm_100a
library against the oracle.

Tolerance: <= 1e-12 relative to each series' scale.  The GPU sums in a tree
order, the reference sums sequentially; both are FP64.
"""
import numpy as np
import pytest

from chan_cases import CASES, make_case, rel_err
from compchan3dmpi_b200 import Channel
from compchan3dmpi_b200.channel import q_criterion
from compchan3dmpi_b200.mesh import periodic_coords
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12
PLANES = (3, 5, 10, 18, 70)        # 3 and nP1-2 = 18 are the edges kept on a 20-point x grid


def _pair(case):
    p, x3, jac, inv, var = case
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    return g, o


def _close(a, b, what):
    a = np.asarray(a); b = np.asarray(b)
    scale = max(np.max(np.abs(b)), 1e-300)
    assert np.max(np.abs(a - b)) <= TOL * scale, f"{what}: {a} vs {b}"


@pytest.mark.parametrize("name", ["ref_rk2_cosine", "rk3_tanh"])
def test_series_every_5_steps(name):
    case = make_case(**CASES[name])
    p, x3 = case[0], case[1]
    g, o = _pair(case)
    g.diag_enable(PLANES, every=5)
    dy = p.Ly / (p.nP[1] - 1)
    x2end = periodic_coords(p.nP[1], p.Ly)[-1]
    want = []
    for _ in range(3):
        o.step(5)
        want.append((o.nstep, o.time, O.diagnostics(o.download(), PLANES, x3, dy, x2end)))
    g.step(15)
    d = g.diag_read()
    assert d["lost"] == 0 and list(d["nstep"]) == [5, 10, 15]
    for r, (n, t, ref) in enumerate(want):
        assert d["time"][r] == t
        _close(d["ke"][r], ref[0], "KE")
        npl = len(PLANES)
        _close(d["rho_b"][r], ref[1:1 + npl], "rho_b")
        _close(d["u_b"][r], ref[1 + npl:1 + 2 * npl], "U_b")
        _close(d["rhou_b"][r], ref[1 + 2 * npl:], "massflow")
    assert d["rho_b"][0][-1] == 0.0          # plane 70 lies outside the grid
    assert g.diag_read()["nstep"].size == 0  # drained


def test_series_ring_and_custom_coordinates():
    case = make_case(**CASES["ref_rk2_cosine"])
    p, x3 = case[0], case[1]
    g, o = _pair(case)
    x3q = np.round(x3, 6)                    # the deck's F10.6 column after a restart
    g.diag_enable((5, 10), every=2, x3q=x3q, x2end=4.18879, capacity=2)
    g.step(10)
    d = g.diag_read()
    assert d["lost"] == 3 and list(d["nstep"]) == [8, 10]
    o.step(10)
    ref = O.diagnostics(o.download(), (5, 10), x3q, p.Ly / (p.nP[1] - 1), 4.18879)
    _close(d["ke"][-1], ref[0], "KE")
    _close(d["rhou_b"][-1], ref[5:7], "massflow")
    g.diag_enable((), every=0)
    g.step(2)
    assert g.diag_read()["nstep"].size == 0


def test_fluctuation_and_q():
    case = make_case(**CASES["rk3_tanh"])
    p, x3 = case[0], case[1]
    g, o = _pair(case)
    g.step(3)
    o.step(3)
    var = g.download()
    mean = var.mean(axis=(2, 3))
    fl, Q = g.fluctuation_q(mean)
    assert np.array_equal(fl, var - mean[:, :, None, None])
    x1 = periodic_coords(p.nP[0], p.Lx); x2 = periodic_coords(p.nP[1], p.Ly)
    ofl = O.fluctuation(o.download(), mean)
    Qo = O.qcrit(ofl[1], ofl[2], ofl[3], x1, x2, x3)
    assert rel_err(Q[None], Qo[None]).max() <= TOL
    # explicit (F10.6-rounded) coordinates, Q only
    xr = [np.round(a, 6) for a in (x1, x2, x3)]
    _, Q2 = g.fluctuation_q(mean, *xr, want_fluc=False)
    Qr = O.qcrit(fl[1], fl[2], fl[3], *xr)
    assert rel_err(Q2[None], Qr[None]).max() <= TOL


def test_q_criterion_standalone():
    rng = np.random.default_rng(5)
    n1, n2, n3 = 33, 17, 21
    u, v, w = (rng.normal(size=(n3, n2, n1)) for _ in range(3))
    x = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n1 - 1)])
    y = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n2 - 1)])
    z = np.cumsum(np.r_[0, rng.uniform(0.5, 1.5, n3 - 1)])
    Q = q_criterion(u, v, w, x, y, z)
    Qo = O.qcrit(u, v, w, x, y, z)
    assert rel_err(Q[None], Qo[None]).max() <= TOL
