"""Mesh, wall coefficients and the CFL time step (host side).

* ``mesh_cosine``: the reference map x3 = 1 - cos(pi*xi/2), xi uniform on
  [0, 2], analytic Jacobian (v1.9/codes/comdata.f90:70-110).
* ``mesh_tanh``: x3 = 1 + tanh(beta*(xi-1))/tanh(beta), the production-grid
  stretching; no reference counterpart.
* ``wall_coeffs``: one-sided 1st/2nd-derivative coefficients on the three
  wall-adjacent non-uniform points (v1.10/codes/main_v1.9.f90:59-83).
* ``cfl_dt``: time step from a CFL number, evaluated once on a field.  The
  reference uses a fixed dt from its deck; this formula is this project's.
"""
from __future__ import annotations

import math

import numpy as np


def _xi(n3: int) -> np.ndarray:
    # Xi(k+1) = Xi(k) + dXi, accumulated as in comdata.f90:101-103
    dXi = 2.0 / float(n3 - 1)
    xi = np.zeros(n3)
    acc = 0.0
    for k in range(1, n3):
        acc = acc + dXi
        xi[k] = acc
    return xi


def mesh_cosine(n3: int):
    """x3, jac, invJac (0-based arrays of length nP3).  invJac[0] = 0 because
    the reference only sets invJac(2:nP3)."""
    xi = _xi(n3)
    x3 = 1.0 - np.cos(0.50 * xi * math.pi)
    jac = 0.50 * math.pi * np.sin(0.50 * xi * math.pi)
    inv = np.zeros(n3)
    inv[1:] = 1.0 / jac[1:]
    return x3, jac, inv


def mesh_tanh(n3: int, beta: float):
    xi = _xi(n3)
    tb = math.tanh(beta)
    th = np.tanh(beta * (xi - 1.0))
    x3 = 1.0 + th / tb
    x3[0] = 0.0
    x3[-1] = 2.0
    jac = beta * (1.0 - th * th) / tb
    inv = 1.0 / jac
    return x3, jac, inv


def make_mesh(n3: int, kind: str = "cosine", beta: float = 2.0):
    if kind == "cosine":
        return mesh_cosine(n3)
    if kind == "tanh":
        return mesh_tanh(n3, beta)
    raise ValueError(f"unknown mesh kind {kind!r}")


def periodic_coords(n: int, L: float) -> np.ndarray:
    """x1 or x2 of comdata.f90:93-99 (x(1)=0, x(i+1)=x(i)+dx)."""
    d = L / float(n - 1)
    x = np.zeros(n)
    acc = 0.0
    for i in range(1, n):
        acc = acc + d
        x[i] = acc
    return x


def wall_coeffs(x3) -> dict:
    """v1.10/codes/main_v1.9.f90:59-83.  ``x3`` is 0-based (x3[0] is x3(1))."""
    x = [0.0] + [float(v) for v in x3]
    n3 = len(x3)
    one, haf = 1.0, 0.5
    c = {}
    dz1 = x[2] - x[1]
    alpha = (x[3] - x[2]) / dz1
    t = dz1 * alpha * (alpha + one)
    c["f1d2c0"] = (one - (alpha + one) * (alpha + one)) / t
    c["f1d2c1"] = ((alpha + one) * (alpha + one)) / t
    c["f1d2c2"] = -one / t
    t = haf * (dz1 * dz1) * alpha * (alpha + one)
    c["f2d1c0"] = alpha / t
    c["f2d1c1"] = -(alpha + one) / t
    c["f2d1c2"] = one / t
    dzN = x[n3] - x[n3 - 1]
    alpha = (x[n3 - 1] - x[n3 - 2]) / dzN
    t = dzN * alpha * (alpha + one)
    c["b1d2c0"] = ((alpha + one) * (alpha + one) - one) / t
    c["b1d2c1"] = -((alpha + one) * (alpha + one)) / t
    c["b1d2c2"] = one / t
    t = haf * (dzN * dzN) * alpha * (alpha + one)
    c["b2d1c0"] = alpha / t
    c["b2d1c1"] = -(alpha + one) / t
    c["b2d1c2"] = one / t
    c["dz1"] = dz1
    c["dzN"] = dzN
    return c


def cfl_dt(var: np.ndarray, params, jac: np.ndarray, cfl: float) -> float:
    """dt = CFL / max over interior points of (lambda_conv + lambda_visc).

    lambda_conv = (|u|+c)/dx + (|v|+c)/dy + (|w|+c)/dz_k,  c = sqrt(T)/Ma
    lambda_visc = 2 * max(4/3, gama/Pr) * mu/(rho*Re) * (1/dx^2 + 1/dy^2 + 1/dz_k^2)
    with dz_k = dXi * jac(k) and mu = T^0.7.  ``var`` is (7, nP3, nP2, nP1).
    """
    rho, u, v, w, _E, T, _p = (var[m, 1:-1, 1:-1, 1:-1] for m in range(7))
    dz = (params.dXi * np.asarray(jac)[1:-1])[:, None, None]
    c = np.sqrt(np.maximum(T, 0.0)) / params.Mac
    lam_c = (np.abs(u) + c) / params.dx + (np.abs(v) + c) / params.dy + (np.abs(w) + c) / dz
    nu = np.power(np.maximum(T, 0.0), 0.7) / (rho * params.Re)
    kv = 2.0 * max(4.0 / 3.0, params.gama / params.Pr)
    lam_v = kv * nu * (1.0 / params.dx ** 2 + 1.0 / params.dy ** 2 + 1.0 / dz ** 2)
    return float(cfl / np.max(lam_c + lam_v))
