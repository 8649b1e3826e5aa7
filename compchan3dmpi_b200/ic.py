"""Seeded initial condition: laminar Poiseuille flow plus uniform noise.

The reference ships no initial-condition generator: it restarts from an
external Tecplot file (v1.8/codes/comData.f90:30).  This generator defines
the synthetic start used by the tests and benchmarks.

* rho = 1, T = T_w = 1 everywhere.
* u = u_lam(z) * (1 + a*r1), v = a*u_lam(z)*r2, w = a*u_lam(z)*r3, with
  u_lam = 1.5*(1-(z-1)^2) (bulk velocity 1) and r uniform on [-1, 1).
  The noise is scaled by u_lam, so the velocity is exactly 0 at the walls.
* p = rho*T/(gama*Ma^2) and E = T + 0.5*ggM*(u^2+v^2+w^2), as in
  v1.9/codes/main_v1.9.f90:603-606.
* The noise is a counter-based hash of (seed, i, j, k, component) on the
  UNIQUE periodic points.  The same grid and seed always give the same bits.
  Duplicate periodic points copy their partner, so q(1)=q(nP-1) and q(nP)=q(2)
  (v1.8_validation/codes/mainV1.8_serial.f90:162-170).

Layout: ``var[m, k, j, i]`` of shape (7, nP3, nP2, nP1), i.e. the Fortran
array var(1:nP1,1:nP2,1:nP3,1:7).
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
    return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, comp: int, ii: np.ndarray, jj: np.ndarray, kk: np.ndarray) -> np.ndarray:
    """Uniform [-1, 1) from a 64-bit hash of (seed, comp, i, j, k)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x100000001B3)) & M64
        key = key ^ (np.uint64(comp) << np.uint64(56))
        x = key ^ (kk.astype(np.uint64) << np.uint64(40)) ^ (jj.astype(np.uint64) << np.uint64(20)) \
            ^ ii.astype(np.uint64)
        h = _splitmix64(_splitmix64(x))
    # 53 random bits -> [0,1) -> [-1,1)
    return ((h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0


def periodic_fill(a: np.ndarray) -> np.ndarray:
    """Copy periodic duplicates in the last two axes (i, j) from the unique points."""
    a[..., :, 0] = a[..., :, -2]
    a[..., :, -1] = a[..., :, 1]
    a[..., 0, :] = a[..., -2, :]
    a[..., -1, :] = a[..., 1, :]
    return a


def laminar_noise(params, x3, seed: int = 1234, amp: float = 0.1) -> np.ndarray:
    n1, n2, n3 = params.nP
    x3 = np.asarray(x3, dtype=np.float64)
    kk, jj, ii = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
    ulam = (1.5 * (1.0 - (x3 - 1.0) ** 2))[:, None, None] * np.ones((1, n2, n1))
    ulam[0] = 0.0
    ulam[-1] = 0.0
    r1 = uniform_pm1(seed, 1, ii, jj, kk)
    r2 = uniform_pm1(seed, 2, ii, jj, kk)
    r3 = uniform_pm1(seed, 3, ii, jj, kk)
    u = ulam * (1.0 + amp * r1)
    v = amp * ulam * r2
    w = amp * ulam * r3
    for a in (u, v, w):
        periodic_fill(a)
    var = np.empty((7, n3, n2, n1))
    rho = np.ones((n3, n2, n1))
    T = np.empty((n3, n2, n1))
    T[...] = 1.0
    T[0] = params.Tw[0]
    T[-1] = params.Tw[1]
    ggM = params.ggM
    var[0] = rho
    var[1] = u
    var[2] = v
    var[3] = w
    var[5] = T
    var[4] = T + ggM * 0.5 * ((u * u + v * v) + w * w)
    var[6] = rho * T / (params.gama * (params.Mac * params.Mac))
    return var
