"""Wall boundary conditions: the reference's wall-BC variants as data.

The reference ships every wall treatment as a separate copy of the solver
that differs only in the wall block of the stage (lines ~605-640 of each
main_v1.9_*.f90).  Here one generic plug-in, ``chan_set_wall_bc``, takes a
``WallBC`` per wall, and the builders below reproduce each variant:

    isothermal(Tw)                   v1.9 (Tw=1), v1.9_strat/v1.9_st1 (0.2), st2 (1.8)
    fixed_gradient(G)                v1.9_strat/v1.9_st3 (G=2), st4 (G=12)
    spanwise_stripes(nP, ...)        v1.9_groov/v1.9_g1 (Tw=1), v1.9_groov_strat/gst1 (Tw=0.3),
                                     gst2 (slip gradient 0.5, Tw=0.3)
    diagonal_stripes(x1, x2, ...)    v1.9_groov_strat/gst3, gst4
    sinusoidal_stripes(x1, x2, ...)  v1.9_groov_strat/gst5
    travelling_wave(A, k, omega, ph) v1.9_STWNV/s1..s6
    rotating_discs(x1, x2, omega)    v1.9_RD/rd1 (omega=3), rd3 (omega=2)

Arrays are (nP2, nP1), i fastest, 1-based reference (i, j) at [j-1, i-1].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NOSLIP, SLIP_MASK, UV_FIELD, WAVE = 0, 1, 2, 3
ISOTHERMAL, FIXED_GRADIENT = 0, 1


@dataclass
class WallBC:
    velocity: int = NOSLIP
    thermal: int = ISOTHERMAL
    Tw: float = 1.0
    dTdz: float = 0.0
    slip_grad: float = 0.0
    wave: tuple = (0.0, 0.0, 0.0, 0.0)     # A, k, omega, phase on odd j
    mask: np.ndarray | None = None        # uint8 (nP2, nP1)
    uv: np.ndarray | None = None          # float64 (2, nP2, nP1)
    x1: np.ndarray | None = None          # float64 (nP1,)


def isothermal(Tw=1.0):
    return WallBC(Tw=float(Tw))


def fixed_gradient(G, Tw_guess=1.0):
    """c0*T1 + c1*T2 + c2*T3 = G (v1.9_strat/v1.9_st3:612, st4:612)."""
    return WallBC(thermal=FIXED_GRADIENT, dTdz=float(G), Tw=float(Tw_guess))


def spanwise_stripes(nP, nstripes=6, Tw=1.0, slip_grad=0.0):
    """Slip where mod(nstripes*j/nP2, 2) == 0 with integer division
    (v1.9_groov/v1.9_g1/codes/main_v1.9_g1.f90:609)."""
    n1, n2 = nP[0], nP[1]
    j = np.arange(1, n2 + 1)
    m = ((nstripes * j) // n2) % 2 == 0
    mask = np.repeat(m[:, None], n1, axis=1).astype(np.uint8)
    return WallBC(velocity=SLIP_MASK, Tw=float(Tw), slip_grad=float(slip_grad), mask=mask)


def diagonal_stripes(x1, x2, Tw=0.3):
    """Slip where mod(floor((x1-x2+x2(nP2))/w), 2) == 0, w = (x1(nP1)+x2(nP2))/8
    (v1.9_groov_strat/v1.9_gst3/codes/main_v1.9_gst3.f90)."""
    x1 = np.asarray(x1); x2 = np.asarray(x2)
    w = (x1[-1] + x2[-1]) / 8.0
    X1, X2 = np.meshgrid(x1, x2)
    mask = (np.mod(np.floor((X1 - X2 + x2[-1]) / w), 2) == 0).astype(np.uint8)
    return WallBC(velocity=SLIP_MASK, Tw=float(Tw), mask=mask)


def sinusoidal_stripes(x1, x2, Tw=0.3):
    """Slip where mod(floor((x2 - w*sin(x1))/w)+1, 3) == 0, w = x2(nP2)/8
    (v1.9_groov_strat/v1.9_gst5/codes/main_v1.9_gst5.f90)."""
    x1 = np.asarray(x1); x2 = np.asarray(x2)
    w = x2[-1] / 8.0
    X1, X2 = np.meshgrid(x1, x2)
    mask = (np.mod(np.floor((X2 - w * np.sin(X1)) / w) + 1, 3) == 0).astype(np.uint8)
    return WallBC(velocity=SLIP_MASK, Tw=float(Tw), mask=mask)


def travelling_wave(A, k, omega, phase_odd=0.0, Tw=1.0, x1=None):
    """v_w = A*sin(k*x1(i) + omega*time [+ phase on odd j])
    (v1.9_STWNV/v1.9_s1:609 A=0.7 k=10 omega=3; s3:609-610 omega=-3, phase 3.14)."""
    return WallBC(velocity=WAVE, Tw=float(Tw), wave=(float(A), float(k), float(omega), float(phase_odd)),
                  x1=None if x1 is None else np.asarray(x1, dtype=np.float64))


def _myatand(a1, a2):
    """Angle of (a1, a2) in [0, 2*pi) by quadrant from atan(|a2/a1|)
    (v1.9_RD/v1.9_rd1/codes/comdata.f90:185-196).  The reference leaves the
    axes (a1 == 0 or a2 == 0) undefined; atan2 covers those points here."""
    a1 = np.asarray(a1, dtype=np.float64); a2 = np.asarray(a2, dtype=np.float64)
    pi = 4.0 * np.arctan(1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.arctan(np.abs(a2 / a1))
    out = np.mod(np.arctan2(a2, a1), 2.0 * pi)
    out = np.where((a1 > 0) & (a2 > 0), t, out)
    out = np.where((a1 < 0) & (a2 > 0), pi - t, out)
    out = np.where((a1 < 0) & (a2 < 0), pi + t, out)
    out = np.where((a1 > 0) & (a2 < 0), 2.0 * pi - t, out)
    return out


def rotating_discs(x1, x2, omega=3.0, Tw=1.0):
    """Three discs of radius R = x2(nP2)/10 centred at (2R, 2R), (2R, 5R),
    (2R, 8R) turning at omega: u = -r*omega*sin(theta), v = r*omega*cos(theta)
    (v1.9_RD/v1.9_rd1/codes/main_v1.9_rd1.f90:607-633)."""
    x1 = np.asarray(x1); x2 = np.asarray(x2)
    R = x2[-1] / 10.0
    X1, X2 = np.meshgrid(x1, x2)
    u = np.zeros_like(X1); v = np.zeros_like(X1)
    done = np.zeros(X1.shape, dtype=bool)
    for cy in (2.0 * R, 5.0 * R, 8.0 * R):
        dxp = X1 - 2.0 * R
        dyp = X2 - cy
        r = np.sqrt(dxp ** 2 + dyp ** 2)
        inside = (r < R) & ~done
        th = _myatand(dxp, dyp)
        u = np.where(inside, -r * omega * np.sin(th), u)
        v = np.where(inside, r * omega * np.cos(th), v)
        done |= inside
    return WallBC(velocity=UV_FIELD, Tw=float(Tw), uv=np.stack([u, v]))


# Fortran's default-real literal 3.14 (single precision) widened to double,
# as the odd-j phase of v1.9_STWNV/v1.9_s3:610 and s4:610 evaluates it.
PHASE_314 = float(np.float32(3.14))

# bottom-wall BC of each reference variant; the top wall stays no-slip, Tw=1
VARIANTS = {
    "v1.9": lambda nP, x1, x2: isothermal(1.0),
    "st1": lambda nP, x1, x2: isothermal(0.2),
    "st2": lambda nP, x1, x2: isothermal(1.8),
    "st3": lambda nP, x1, x2: fixed_gradient(2.0),
    "st4": lambda nP, x1, x2: fixed_gradient(12.0),
    "g1": lambda nP, x1, x2: spanwise_stripes(nP, 6, Tw=1.0),
    "gst1": lambda nP, x1, x2: spanwise_stripes(nP, 6, Tw=0.3),
    "gst2": lambda nP, x1, x2: spanwise_stripes(nP, 6, Tw=0.3, slip_grad=0.5),
    "gst3": lambda nP, x1, x2: diagonal_stripes(x1, x2, Tw=0.3),
    "gst4": lambda nP, x1, x2: diagonal_stripes(x1, x2, Tw=0.3),
    "gst5": lambda nP, x1, x2: sinusoidal_stripes(x1, x2, Tw=0.3),
    "s1": lambda nP, x1, x2: travelling_wave(0.7, 10.0, 3.0, x1=x1),
    "s2": lambda nP, x1, x2: travelling_wave(0.5, 10.0, 3.0, x1=x1),
    "s3": lambda nP, x1, x2: travelling_wave(0.5, 10.0, -3.0, PHASE_314, x1=x1),
    "s4": lambda nP, x1, x2: travelling_wave(0.5, 3.75, 3.0, PHASE_314, x1=x1),
    "s5": lambda nP, x1, x2: travelling_wave(0.7, 3.75, -3.0, x1=x1),
    "s6": lambda nP, x1, x2: travelling_wave(0.3, 10.0, 3.0, x1=x1),
    "rd1": lambda nP, x1, x2: rotating_discs(x1, x2, 3.0),
    "rd2": lambda nP, x1, x2: rotating_discs(x1, x2, 3.0),
    "rd3": lambda nP, x1, x2: rotating_discs(x1, x2, 2.0),
}


def reference_variant(name, params):
    """(bottom, top) WallBC of a reference variant for a ChanParams."""
    from .mesh import periodic_coords
    n1, n2, _ = params.nP
    x1 = periodic_coords(n1, params.Lx)
    x2 = periodic_coords(n2, params.Ly)
    return VARIANTS[name](params.nP, x1, x2), isothermal(params.Tw[1])
