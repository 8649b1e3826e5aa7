"""Wall-BC builders and the oracle's wall-BC block against the reference's
formulas (CPU only)."""
import math

import numpy as np
import pytest

from chan_cases import CASES, make_case
from compchan3dmpi_b200 import wallbc as W
from compchan3dmpi_b200.mesh import periodic_coords, wall_coeffs
from oracle import oracle as O


def test_spanwise_stripe_mask():
    # mod(6*j/nP2, 2) == 0 with integer division (v1.9_groov/v1.9_g1:609)
    nP = (5, 48, 9)
    bc = W.spanwise_stripes(nP)
    for j in range(1, 49):
        want = ((6 * j) // 48) % 2 == 0
        assert np.all(bc.mask[j - 1] == want)
    assert bc.mask.shape == (48, 5) and bc.mask.dtype == np.uint8


def test_diagonal_and_sinusoidal_masks():
    x1 = periodic_coords(33, 4 * math.pi)
    x2 = periodic_coords(17, 4 * math.pi / 3)
    d = W.diagonal_stripes(x1, x2)
    w = (x1[-1] + x2[-1]) / 8.0
    for j in (0, 5, 16):
        for i in (0, 7, 32):
            assert d.mask[j, i] == (math.floor((x1[i] - x2[j] + x2[-1]) / w) % 2 == 0)
    s = W.sinusoidal_stripes(x1, x2)
    r = x2[-1] / 8.0
    for j in (0, 3, 16):
        for i in (0, 9, 31):
            assert s.mask[j, i] == ((math.floor((x2[j] - r * math.sin(x1[i])) / r) + 1) % 3 == 0)


def test_myatand_quadrants():
    a1 = np.array([1.0, -1.0, -1.0, 1.0, 0.3])
    a2 = np.array([1.0, 1.0, -1.0, -1.0, 2.0])
    got = W._myatand(a1, a2)
    want = np.mod(np.arctan2(a2, a1), 2 * math.pi)
    assert np.allclose(got, want, rtol=0, atol=4e-16)


def test_rotating_discs_velocity():
    x1 = periodic_coords(64, 4 * math.pi)
    x2 = periodic_coords(48, 4 * math.pi / 3)
    bc = W.rotating_discs(x1, x2, 3.0)
    R = x2[-1] / 10.0
    u, v = bc.uv
    for j in range(48):
        for i in range(64):
            r = [math.hypot(x1[i] - 2 * R, x2[j] - c * R) for c in (2, 5, 8)]
            if min(r) >= R:
                assert u[j, i] == 0.0 and v[j, i] == 0.0
            else:
                c = (2, 5, 8)[[n for n in range(3) if r[n] < R][0]]
                # solid-body rotation: (u, v) = omega x (dx, dy)
                dx, dy = x1[i] - 2 * R, x2[j] - c * R
                assert abs(u[j, i] + 3.0 * dy) < 1e-13 and abs(v[j, i] - 3.0 * dx) < 1e-13


def test_phase_literal():
    assert W.PHASE_314 == 3.140000104904175
    assert W.PHASE_314 != 3.14


def _oracle(case):
    p, x3, jac, inv, var = case
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    return o, p, x3


def test_default_bc_set_explicitly_is_identity():
    case = make_case(**CASES["ref_rk2_cosine"])
    a, p, _ = _oracle(case)
    b, _, _ = _oracle(case)
    b.set_wall_bc(0, W.isothermal(p.Tw[0]))
    b.set_wall_bc(1, W.isothermal(p.Tw[1]))
    a.step(3)
    b.step(3)
    assert np.array_equal(a.download(), b.download())


def test_fixed_gradient_holds_at_wall():
    case = make_case(**CASES["ref_rk2_cosine"])
    o, p, x3 = _oracle(case)
    o.set_wall_bc(0, W.fixed_gradient(2.0))
    o.step(2)
    v = o.download()
    c = wall_coeffs(x3)
    T = v[5]
    g = c["f1d2c0"] * T[0] + c["f1d2c1"] * T[1] + c["f1d2c2"] * T[2]
    assert np.allclose(g, 2.0, rtol=0, atol=1e-10)
    # E = T + gamma(gamma-1)Ma^2/2 |u|^2 and rho = gamma Ma^2 p / T on the wall
    ggM = p.gama * (p.gama - 1.0) * p.Mac ** 2
    assert np.allclose(v[4][0], T[0] + ggM * 0.5 * (v[1][0] ** 2 + v[2][0] ** 2), rtol=1e-14, atol=0)


def test_slip_mask_and_wave_formulas():
    case = make_case(**CASES["ref_rk2_cosine"])
    o, p, x3 = _oracle(case)
    bc = W.spanwise_stripes(p.nP, 6, Tw=0.3, slip_grad=0.5)
    o.set_wall_bc(0, bc)
    o.step(2)
    v = o.download()
    c = wall_coeffs(x3)
    for m in (1, 2):
        g = c["f1d2c0"] * v[m][0] + c["f1d2c1"] * v[m][1] + c["f1d2c2"] * v[m][2]
        m1 = bc.mask.astype(bool)
        assert np.allclose(g[m1], 0.5, rtol=0, atol=1e-10)
        assert np.all(v[m][0][~m1] == 0.0)
    assert np.all(v[5][0] == 0.3)

    case = make_case(**CASES["ragged"])
    o, p, x3 = _oracle(case)
    bc = W.travelling_wave(0.5, 10.0, -3.0, W.PHASE_314)
    o.set_wall_bc(0, bc)
    o.step(3)
    v = o.download()
    x1 = periodic_coords(p.nP[0], p.Lx)
    t = o.time
    for j in range(p.nP[1]):
        ph = W.PHASE_314 if (j + 1) % 2 == 1 else 0.0
        want = 0.5 * np.sin(10.0 * x1 - 3.0 * t + ph)
        assert np.allclose(v[2][0, j], want, rtol=0, atol=1e-15)
    assert np.all(v[1][0] == 0.0) and np.all(v[3][0] == 0.0)
