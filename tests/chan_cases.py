"""Shared test cases: seeded inputs for the oracle and the GPU library."""
from __future__ import annotations

import numpy as np

from compchan3dmpi_b200 import ChanParams, RK2, RK3, FORCE_WALLSHEAR, make_mesh, laminar_noise, cfl_dt
from compchan3dmpi_b200.deck import quantize_deck


def make_case(nP=(20, 14, 19), mesh="cosine", beta=2.0, rk=RK2, Pr=0.71, dt=None, cfl=0.5, istat=2,
              forcing=FORCE_WALLSHEAR, seed=1234, amp=0.1, quantize=True, **kw):
    """(params, x3, jac, invJac, var).  dt from CFL unless given."""
    x3, jac, inv = make_mesh(nP[2], mesh, beta)
    p = ChanParams(nP=tuple(nP), Pr=Pr, rk_scheme=rk, istat=istat, forcing=forcing, **kw)
    var = laminar_noise(p, x3, seed=seed, amp=amp)
    if quantize:
        var = quantize_deck(var)
    if dt is None:
        dt = cfl_dt(var, p, jac, cfl)
    p = p.with_(dt=dt)
    return p, x3, jac, inv, var


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-variable normwise relative error max|a-b| / max|b| (7 entries)."""
    a = np.asarray(a); b = np.asarray(b)
    out = []
    for m in range(a.shape[0]):
        den = np.max(np.abs(b[m]))
        num = np.max(np.abs(a[m] - b[m]))
        out.append(num / den if den > 0 else num)
    return np.array(out)


def worst(a: np.ndarray, b: np.ndarray):
    """(variable, k, j, i) of the largest absolute difference, for messages."""
    d = np.abs(np.asarray(a) - np.asarray(b))
    return np.unravel_index(np.argmax(d), d.shape)


# reference-semantics and production-physics cases used by the parity tests
CASES = {
    "ref_rk2_cosine": dict(nP=(20, 14, 19), mesh="cosine", rk=RK2, Pr=0.71),
    "rk3_tanh": dict(nP=(22, 12, 21), mesh="tanh", beta=2.2, rk=RK3, Pr=0.72),
    "ragged": dict(nP=(39, 7, 11), mesh="cosine", rk=RK2, Pr=0.71),
    "tiny": dict(nP=(8, 6, 9), mesh="tanh", beta=2.0, rk=RK3, Pr=0.72),
}


def conservation_case(nP=(20, 14, 19), Pe=(2.0, 2.0, 0.2), seed=77):
    """Field with w = 0 everywhere and a perturbed density: the continuity flux
    in z vanishes, so with one inviscid scheme everywhere (telescoping face
    fluxes) every plane's mass over its periodic points is conserved by a stage."""
    from compchan3dmpi_b200.ic import uniform_pm1, periodic_fill
    p, x3, jac, inv, var = make_case(nP=nP, Pe=Pe, quantize=False)
    n1, n2, n3 = p.nP
    kk, jj, ii = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
    rho = 1.0 + 0.05 * uniform_pm1(seed, 9, ii, jj, kk)
    periodic_fill(rho)
    rho[0] = 1.0
    rho[-1] = 1.0
    var = var.copy()
    var[3] = 0.0
    u, v, T = var[1], var[2], var[5]
    var[0] = rho
    var[4] = T + p.ggM * 0.5 * (u * u + v * v)
    var[6] = rho * T / (p.gama * p.Mac * p.Mac)
    return p, x3, jac, inv, var


def plane_mass(var):
    """Sum of rho over the periodic points i = 2..nP1-1, j = 2..nP2-1 of each plane."""
    return var[0][:, 1:-1, 1:-1].sum(axis=(1, 2))
