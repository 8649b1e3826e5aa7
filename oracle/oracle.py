"""ctypes wrapper of the C restatement in ``chan_oracle.c``.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the GPU library and
the CPU baseline of ``bench.py``; it is never on the product path.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline and
``--impl reference`` legs) may import it.

Field layout used everywhere on the Python side: ``var[m, k, j, i]`` (C order,
shape ``(7, nP3, nP2, nP1)``) which is byte-for-byte the reference's Fortran
array ``var(1:nP1, 1:nP2, 1:nP3, 1:7)`` (v1.9/codes/main_v1.9.f90:38).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "chan_oracle.c"
BUILD_DIR = HERE / "_build"
LIB = BUILD_DIR / "liboracle.so"

# parameter vector layout (enum in chan_oracle.c)
P_RE, P_MAC, P_DT, P_PR, P_GAMA, P_PEX, P_PEY, P_PEZ, P_LX, P_LY, P_TWB, P_TWT, \
    P_ISTAT, P_RK, P_FORCING, P_NPARAM = range(16)

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> Path:
    """Compile the restatement with gcc (OpenMP, no FMA contraction)."""
    BUILD_DIR.mkdir(exist_ok=True)
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = BUILD_DIR / f"liboracle.{os.getpid()}.so"
    cmd = ["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
           "-shared", "-std=c99", "-o", str(tmp), str(SRC), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [_I, _D, _D, _D, _D]
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_upload.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, ctypes.c_double]
        L.orc_stage.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_step.restype = ctypes.c_int
        L.orc_check.argtypes = [ctypes.c_void_p]
        L.orc_check.restype = ctypes.c_int
        L.orc_tau_wall.argtypes = [ctypes.c_void_p]
        L.orc_avg_spatial.argtypes = [ctypes.c_void_p]
        L.orc_download.argtypes = [ctypes.c_void_p, _D]
        L.orc_download_solv.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_get_stats.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        L.orc_set_forcing.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D]
        L.orc_set_buoyancy.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.orc_set_v19_alias.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_wall_bc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, _D, ctypes.c_void_p, _D, _D]
        L.orc_diagnostics.argtypes = [_D, _I, _I, ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, _D]
        L.orc_qcrit.argtypes = [_I, _D, _D, _D, _D, _D, _D, _D]
        L.orc_nstep.argtypes = [ctypes.c_void_p]
        L.orc_nstep.restype = ctypes.c_long
        L.orc_time.argtypes = [ctypes.c_void_p]
        L.orc_time.restype = ctypes.c_double
        L.orc_blown.argtypes = [ctypes.c_void_p, _I]
        L.orc_blown.restype = ctypes.c_int
        L.orc_coeffs.argtypes = [ctypes.c_int, _D, _D]
        L.orc_setup_mesh_cosine.argtypes = [ctypes.c_int, _D, _D, _D]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def coeffs(x3: np.ndarray) -> np.ndarray:
    """14 numbers: f1d2c0..2, f2d1c0..2, b1d2c0..2, b2d1c0..2, dz1, dzN
    (v1.10/codes/main_v1.9.f90:59-83).  ``x3`` is 0-based."""
    x = np.zeros(len(x3) + 1)
    x[1:] = x3
    out = np.zeros(14)
    lib().orc_coeffs(len(x3), _dp(x), _dp(out))
    return out


def mesh_cosine(n3: int):
    """x3, jac, invJac (0-based) of v1.9/codes/comdata.f90:101-110."""
    x3 = np.zeros(n3 + 1); jac = np.zeros(n3 + 1); inv = np.zeros(n3 + 1)
    lib().orc_setup_mesh_cosine(n3, _dp(x3), _dp(jac), _dp(inv))
    return x3[1:].copy(), jac[1:].copy(), inv[1:].copy()


def param_vector(p) -> np.ndarray:
    """Pack a ``compchan3dmpi_b200.ChanParams``-like object into the oracle's vector."""
    v = np.zeros(P_NPARAM)
    v[P_RE] = p.Re; v[P_MAC] = p.Mac; v[P_DT] = p.dt; v[P_PR] = p.Pr; v[P_GAMA] = p.gama
    v[P_PEX], v[P_PEY], v[P_PEZ] = p.Pe
    v[P_LX] = p.Lx; v[P_LY] = p.Ly; v[P_TWB], v[P_TWT] = p.Tw
    v[P_ISTAT] = p.istat; v[P_RK] = p.rk_scheme; v[P_FORCING] = p.forcing
    return v


class Oracle:
    """One reference-semantics solver instance (single MPI rank, periodic x,y)."""

    def __init__(self, params, x3, jac, invJac, threads: int | None = None):
        L = lib()
        if threads:
            L.orc_set_num_threads(int(threads))
        self.nP = tuple(int(n) for n in params.nP)
        self.params = params
        nP = (ctypes.c_int * 3)(*self.nP)
        pv = param_vector(params)
        self._x3 = np.ascontiguousarray(x3, dtype=np.float64)
        self._jac = np.ascontiguousarray(jac, dtype=np.float64)
        self._inv = np.ascontiguousarray(invJac, dtype=np.float64)
        self._h = L.orc_create(nP, _dp(pv), _dp(self._x3), _dp(self._jac), _dp(self._inv))
        if not self._h:
            raise MemoryError("oracle allocation failed")

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_free(self._h)
            self._h = None

    __del__ = close

    @property
    def shape(self):
        n1, n2, n3 = self.nP
        return (7, n3, n2, n1)

    def upload(self, var: np.ndarray, nstep: int = 0, time: float = 0.0):
        v = np.ascontiguousarray(var, dtype=np.float64)
        assert v.shape == self.shape
        lib().orc_upload(self._h, _dp(v), int(nstep), float(time))

    def stage(self, it: int):
        lib().orc_stage(self._h, int(it))

    def step(self, n: int = 1) -> int:
        return lib().orc_step(self._h, int(n))

    def download(self) -> np.ndarray:
        out = np.empty(self.shape)
        lib().orc_download(self._h, _dp(out))
        return out

    def download_solv(self, lev: int = 0) -> np.ndarray:
        n1, n2, n3 = self.nP
        out = np.empty((5, n3, n2, n1))
        lib().orc_download_solv(self._h, int(lev), _dp(out))
        return out

    def stats(self):
        n3 = self.nP[2]
        tau = np.zeros(2); s1 = np.zeros((7, n3)); s2 = np.zeros((7, n3)); c = np.zeros((9, n3))
        lib().orc_get_stats(self._h, _dp(tau), _dp(s1), _dp(s2), _dp(c))
        return tau, s1, s2, c

    def tau_wall(self):
        lib().orc_tau_wall(self._h)

    def avg_spatial(self):
        lib().orc_avg_spatial(self._h)

    def set_forcing(self, tauL, tauU, rhobar):
        rb = np.ascontiguousarray(rhobar, dtype=np.float64)
        lib().orc_set_forcing(self._h, float(tauL), float(tauU), _dp(rb))

    def set_v19_alias(self, on=True):
        """The canonical v1.9 binary's single-rank semantics: its 4th-order
        central fluxes read var(i+-2) / var(j+-2) beyond var's bounds, which land
        on the neighbouring column or plane (chan_oracle.c, var_c).  Off by
        default: main19fix's periodic ghosts."""
        lib().orc_set_v19_alias(self._h, 1 if on else 0)

    def set_buoyancy(self, Ri, Tref=1.0):
        """Same buoyancy body force as Channel.set_buoyancy."""
        lib().orc_set_buoyancy(self._h, float(Ri), float(Tref))

    def set_wall_bc(self, wall, bc):
        """Same WallBC description as Channel.set_wall_bc."""
        wave = np.ascontiguousarray(bc.wave, dtype=np.float64)
        mask = None if bc.mask is None else np.ascontiguousarray(bc.mask, dtype=np.uint8)
        uv = None if bc.uv is None else np.ascontiguousarray(bc.uv, dtype=np.float64)
        x1 = None if bc.x1 is None else np.ascontiguousarray(bc.x1, dtype=np.float64)
        lib().orc_set_wall_bc(self._h, int(wall), int(bc.velocity), int(bc.thermal), float(bc.Tw), float(bc.dTdz),
                              float(bc.slip_grad), _dp(wave), None if mask is None else mask.ctypes.data,
                              None if uv is None else _dp(uv), None if x1 is None else _dp(x1))

    @property
    def nstep(self):
        return lib().orc_nstep(self._h)

    @property
    def time(self):
        return lib().orc_time(self._h)

    def blown(self):
        ijk = (ctypes.c_int * 3)()
        f = lib().orc_blown(self._h, ijk)
        return f, tuple(ijk)


def diagnostics(var, planes, x3q, dy, x2end):
    """[KE, rho_b[np], U_b[np], rhoU_b[np]] of var (7, nP3, nP2, nP1):
    main_v1.9.f90:799-906 on one rank."""
    v = np.ascontiguousarray(var, dtype=np.float64)
    _, n3, n2, n1 = v.shape
    nP = (ctypes.c_int * 3)(n1, n2, n3)
    pl = (ctypes.c_int * max(1, len(planes)))(*[int(p) for p in planes])
    z = np.ascontiguousarray(x3q, dtype=np.float64)
    out = np.zeros(1 + 3 * len(planes))
    lib().orc_diagnostics(_dp(v), nP, pl, len(planes), _dp(z), float(dy), float(x2end), _dp(out))
    return out


def fluctuation(var, mean):
    """var(i,j,k,:) - mean(k,:) (fluc.f90:63-69); mean is (7, nP3)."""
    return np.asarray(var, dtype=np.float64) - np.asarray(mean, dtype=np.float64)[:, :, None, None]


def qcrit(u, v, w, x, y, z):
    """Q-criterion of qInvariant.f90:26-81; u, v, w are (nP3, nP2, nP1)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    n3, n2, n1 = u.shape
    v = np.ascontiguousarray(v, dtype=np.float64); w = np.ascontiguousarray(w, dtype=np.float64)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    Q = np.empty_like(u)
    lib().orc_qcrit((ctypes.c_int * 3)(n1, n2, n3), _dp(u), _dp(v), _dp(w), _dp(x), _dp(y), _dp(z), _dp(Q))
    return Q


def num_threads() -> int:
    return lib().orc_num_threads()
