"""CPU tests of the oracle (the checker) against the reference's own data."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from compchan3dmpi_b200 import mesh_cosine, wall_coeffs

GOLD = Path(__file__).with_name("golden")


def test_fd_coeff_kat():
    """Reference KAT: v1.8_validation/codes/nohupDebug.out:23-26.  The logged
    values come from an ifort -O3 build; the near-wall stencils amplify
    rounding by ~1e7, hence 1e-10 (1st derivative) and 1e-8 (2nd)."""
    kat = json.loads((GOLD / "fd_coeff_kat.json").read_text())
    n3 = kat["mesh"]["nP3"]
    x3, _, _ = O.mesh_cosine(n3)
    c = O.coeffs(x3)
    pl = [x ** 3.0 - 5.0 * x ** 2.0 + 3.0 * x - 10.0 for x in x3]
    got = {
        "Bottom 1st Derivative": (c[0] * pl[0] + c[1] * pl[1]) + c[2] * pl[2],
        "Top    1st Derivative": (c[6] * pl[-1] + c[7] * pl[-2]) + c[8] * pl[-3],
        "Bottom 2nd Derivative": (c[3] * pl[0] + c[4] * pl[1]) + c[5] * pl[2],
        "Top    2nd Derivative": (c[9] * pl[-1] + c[10] * pl[-2]) + c[11] * pl[-3],
    }
    for name, row in kat["rows"].items():
        tol = 1e-10 if "1st" in name else 1e-8
        assert abs(got[name] - row["logged"]) <= tol * abs(row["logged"]), (name, got[name], row)
        # and the stencil is a derivative: exact value within its truncation error
        assert abs(got[name] - row["exact"]) < 2e-3 * abs(row["exact"])


def test_host_mesh_and_coeffs_match_oracle():
    for n3 in (9, 65, 160):
        x3, jac, inv = mesh_cosine(n3)
        ox3, ojac, oinv = O.mesh_cosine(n3)
        np.testing.assert_allclose(x3, ox3, rtol=0, atol=4e-16)
        np.testing.assert_allclose(jac, ojac, rtol=1e-15, atol=1e-17)
        c = wall_coeffs(ox3)
        oc = O.coeffs(ox3)
        names = ["f1d2c0", "f1d2c1", "f1d2c2", "f2d1c0", "f2d1c1", "f2d1c2",
                 "b1d2c0", "b1d2c1", "b1d2c2", "b2d1c0", "b2d1c1", "b2d1c2", "dz1", "dzN"]
        for i, n in enumerate(names):
            assert c[n] == oc[i], n   # same formula, same operation order: bit-identical


def test_coefficients_are_derivatives():
    # one-sided 2nd-order first derivative is exact for quadratics; 2nd derivative for quadratics too
    x3, _, _ = O.mesh_cosine(33)
    c = O.coeffs(x3)
    f = lambda x: 2.0 * x * x - 3.0 * x + 1.0
    d1 = c[0] * f(x3[0]) + c[1] * f(x3[1]) + c[2] * f(x3[2])
    d2 = c[3] * f(x3[0]) + c[4] * f(x3[1]) + c[5] * f(x3[2])
    assert abs(d1 - (-3.0)) < 1e-9 and abs(d2 - 4.0) < 1e-6
    b1 = c[6] * f(x3[-1]) + c[7] * f(x3[-2]) + c[8] * f(x3[-3])
    assert abs(b1 - (4.0 * 2.0 - 3.0)) < 1e-9


def _quiescent(p, x3):
    n1, n2, n3 = p.nP
    var = np.zeros((7, n3, n2, n1))
    var[0] = 1.0
    var[5] = 1.0
    var[4] = 1.0
    var[6] = 1.0 / (p.gama * p.Mac * p.Mac)
    return var


def test_quiescent_state_is_steady():
    """u=v=w=0, rho=T=1, uniform p is an exact steady state of the scheme."""
    from chan_cases import make_case
    p, x3, jac, inv, _ = make_case(nP=(12, 10, 11), quantize=False, dt=1e-3)
    var = _quiescent(p, x3)
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    assert o.step(3) == 0
    out = o.download()
    np.testing.assert_allclose(out, var, rtol=0, atol=5e-14)


def test_oracle_deterministic_and_thread_independent():
    from chan_cases import make_case
    p, x3, jac, inv, var = make_case(nP=(16, 10, 13), quantize=False)
    outs = []
    for th in (1, 3):
        o = O.Oracle(p, x3, jac, inv, threads=th)
        o.upload(var)
        o.step(4)
        outs.append(o.download())
    assert np.array_equal(outs[0], outs[1])


def test_oracle_blowup_detection():
    from chan_cases import make_case
    p, x3, jac, inv, var = make_case(nP=(12, 10, 11), quantize=False)
    var = var.copy()
    var[0, 5, 4, 6] = -1.0   # negative density at one interior point
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    assert o.step(5) == 1
    f, ijk = o.blown()
    assert f == 1 and o.nstep == 1


def test_plane_mass_conserved_by_one_scheme():
    """With w = 0 the z continuity flux vanishes; central (Pe thresholds never
    exceeded) and QUICK (always exceeded) face fluxes telescope over the periodic
    points, so each interior plane's mass is kept by a stage.  The hybrid switch
    mixes the two and does not telescope."""
    from chan_cases import conservation_case, plane_mass
    for Pe in ((1e300, 1e300, 1e300), (0.0, 0.0, 0.0)):
        p, x3, jac, inv, var = conservation_case(Pe=Pe)
        o = O.Oracle(p, x3, jac, inv)
        o.upload(var)
        m0 = plane_mass(var)
        o.stage(1)
        m1 = plane_mass(o.download())
        rel = np.abs(m1[1:-1] - m0[1:-1]) / m0[1:-1]
        assert rel.max() <= 1e-13, (Pe, rel.max())
    p, x3, jac, inv, var = conservation_case()
    o = O.Oracle(p, x3, jac, inv)
    o.upload(var)
    o.stage(1)
    rel = np.abs(plane_mass(o.download())[1:-1] - plane_mass(var)[1:-1]) / plane_mass(var)[1:-1]
    assert rel.max() > 1e-12    # the hybrid switch is not conservative


def test_oracle_buoyancy_source_is_the_stated_term():
    """One RK2 first stage (Q <- Q + dt/2 R) with and without the buoyancy
    term: rho*w changes by dt/2*Ri*rho*(T - Tref) and rho*E by ggM*w times
    that; rho, rho*u and rho*v are untouched, bit for bit."""
    from chan_cases import make_case
    p, x3, jac, inv, var = make_case(nP=(12, 10, 13), quantize=False)
    p = p.with_(Tw=(0.9, 1.1))
    Ri, Tref = 0.5, 1.05
    a = O.Oracle(p, x3, jac, inv, threads=1)
    b = O.Oracle(p, x3, jac, inv, threads=1)
    b.set_buoyancy(Ri, Tref)
    for o in (a, b):
        o.upload(var)
        o.stage(1)
    qa, qb = a.download_solv(0), b.download_solv(0)
    a.close(); b.close()
    n1, n2, n3 = p.nP
    sl = (slice(1, n3 - 1), slice(1, n2 - 1), slice(1, n1 - 1))   # interior k, j, i (0-based)
    rho, w, T = var[0][sl], var[3][sl], var[5][sl]
    bq = Ri * (rho * (T - Tref))
    cdt = 0.5 * p.dt
    for m in (0, 1, 2):
        assert np.array_equal(qa[m][sl], qb[m][sl]), m
    dw = qb[3][sl] - qa[3][sl]
    dE = qb[4][sl] - qa[4][sl]
    assert np.max(np.abs(bq)) > 1e-3
    assert np.max(np.abs(dw - cdt * bq)) <= 1e-12 * np.max(np.abs(qa[3][sl])) + 1e-15
    assert np.max(np.abs(dE - cdt * p.ggM * w * bq)) <= 1e-12 * np.max(np.abs(qa[4][sl])) + 1e-15


def test_closure_oracle_gradient_matches_finite_differences():
    """The oracle's MLP backward pass (without its BF16 roundings) is the
    derivative of its loss: checked by central differences in float64."""
    from oracle import closure_oracle as C
    rng = np.random.default_rng(3)
    params = rng.standard_normal(C.N_PARAM) * 0.3
    norm = np.concatenate([np.zeros(13), np.ones(13), np.zeros(9), np.ones(9)])
    X = rng.standard_normal((40, 13))
    T = rng.standard_normal((40, 9))
    ident = lambda x: np.asarray(x, dtype=np.float64)   # noqa: E731
    orig = C.bf16
    C.bf16 = ident
    try:
        loss, g = C.grad(params, norm, X, T)
        for idx in list(range(0, C.N_PARAM, 97)) + [C.OFF_B1 + 3, C.OFF_B3 + 2, C.OFF_W3 + 5]:
            e = np.zeros(C.N_PARAM)
            e[idx] = 1e-6
            lp, _ = C.grad(params + e, norm, X, T)
            lm, _ = C.grad(params - e, norm, X, T)
            fd = (lp - lm) / (2e-6) / (9.0 * 40)
            assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(g[idx])), (idx, fd, g[idx])
    finally:
        C.bf16 = orig


def test_v19_alias_changes_only_the_edge_points_of_one_stage():
    """The v1.9 aliasing switch: with the central branch everywhere, one stage
    differs from main19fix's only at the points whose x or spanwise 4th-order
    stencil reaches past the ghost-free var (i = 2, nP1-1 or j = 2, nP2-1) and
    their periodic duplicates; everywhere else the two agree bit for bit.  At such a point the
    difference is the one the aliased reads imply: var(0,j,k) is var(nP1,j-1,k)
    instead of var(nP1-2,j,k)."""
    from chan_cases import make_case
    p, x3, jac, inv, var = make_case(nP=(12, 10, 9), Pe=(1e300, 1e300, 1e300), quantize=False)
    a = O.Oracle(p, x3, jac, inv)
    b = O.Oracle(p, x3, jac, inv)
    b.set_v19_alias(True)
    for o in (a, b):
        o.upload(var)
        o.stage(1)
    qa, qb = a.download_solv(0), b.download_solv(0)
    n1, n2, n3 = p.nP
    d = np.any(qa != qb, axis=0)            # [k][j][i], 0-based
    edge = np.zeros_like(d)                 # the edge points and their periodic duplicates
    for i in (0, 1, n1 - 2, n1 - 1):
        edge[1:n3 - 1, :, i] = True
    for j in (0, 1, n2 - 2, n2 - 1):
        edge[1:n3 - 1, j, :] = True
    assert not np.any(d & ~edge)
    assert np.all(d[1:n3 - 1, 2:n2 - 2, 1])     # every interior-row point at i = 2 changes
    # the x-flux difference at (i=2, j, k) from the two wraps of var(0, j, k)
    k, j = 3, 4                                 # 1-based interior point (2, j, k)
    u = var[1]                                  # [k][j][i] 0-based
    rho = var[0]
    diff_u0 = u[k - 1, j - 2, n1 - 1] - u[k - 1, j - 1, n1 - 3]   # var(nP1,j-1,k) - var(nP1-2,j,k)
    Q0 = rho[k - 1, j - 1, n1 - 3]              # solV(0,j,k,1) = its periodic image (nP1-2,j,k)
    dF = diff_u0 * Q0 * (1.0 / p.dx) / 12.0     # F(:,1) gains +var(i-2)*solV(i-2)/(12 dx)
    cdt = 0.5 * p.dt                            # RK2 stage 1: Q <- Q + dt/2 * R, R = -dF
    got = qb[0, k - 1, j - 1, 1] - qa[0, k - 1, j - 1, 1]
    assert abs(got - (-cdt * dF)) <= 1e-12 * abs(cdt * dF) + 1e-15, (got, -cdt * dF)
