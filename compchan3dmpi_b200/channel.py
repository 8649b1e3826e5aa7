"""Host-side mirror of the reference's solver interface.

The reference drives its hot path from a Fortran main program through these
subroutines (v1.10/codes/main_v1.10.f90:20-53):

    readParam, calcMeshParam, calcCoeffs   -> Channel(params, x3, jac, invJac)
    readInputFile + initSolV + share2P     -> Channel.init_sol_v(var) / read_input_file(path)
    calcFlux, calcSolV, share2P, calcPrim,
    share2P, calcBC (one RK stage)         -> Channel.stage(iter)
    the time loop                          -> Channel.step(n)
    checkSoln                              -> Channel.check_soln()
    calcTauWall                            -> Channel.calc_tau_wall()
    avgSpatial                             -> Channel.avg_spatial()
    writeSoln                              -> Channel.write_soln(path)

Every call goes through the C ABI of ``libchanrhs.so``.  Errors are raised
where the reference would ``stop``: ``BlowUpError`` for rho<0 or T<0
(v1.9/codes/main_v1.9.f90:709-743), ``ChanError`` for usage/IO/CUDA errors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import ChanParams


class ChanError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"chanrhs error {code}: {msg}")
        self.code = code


class BlowUpError(ChanError):
    def __init__(self, code, msg, ijk, nstep):
        super().__init__(code, msg)
        self.ijk = ijk
        self.nstep = nstep


def to_c_params(p: ChanParams) -> _lib.ChanParamsC:
    c = _lib.ChanParamsC()
    c.nP[:] = [int(n) for n in p.nP]
    c.istat = int(p.istat)
    c.rk_scheme = int(p.rk_scheme)
    c.forcing = int(p.forcing)
    c.device = int(p.device)
    c.flags = _lib.CHAN_MIXED if getattr(p, "mixed", False) else 0
    c.Re = float(p.Re); c.Mac = float(p.Mac); c.dt = float(p.dt); c.Pr = float(p.Pr); c.gama = float(p.gama)
    c.Pe[:] = [float(x) for x in p.Pe]
    c.Lx = float(p.Lx); c.Ly = float(p.Ly)
    c.Tw[:] = [float(x) for x in p.Tw]
    return c


class Channel:
    def __init__(self, params: ChanParams, x3, jac, invJac):
        self.L = _lib.load()
        self.params = params
        self.nP = tuple(int(n) for n in params.nP)
        self.x3 = np.ascontiguousarray(x3, dtype=np.float64)
        self.jac = np.ascontiguousarray(jac, dtype=np.float64)
        self.invJac = np.ascontiguousarray(invJac, dtype=np.float64)
        if self.x3.shape != (self.nP[2],) or self.jac.shape != self.x3.shape or self.invJac.shape != self.x3.shape:
            raise ValueError("x3, jac, invJac must have nP3 entries")
        self._cp = to_c_params(params)
        h = ctypes.c_void_p()
        r = self.L.chan_init(ctypes.byref(self._cp), _lib.dptr(self.x3), _lib.dptr(self.jac),
                             _lib.dptr(self.invJac), ctypes.byref(h))
        if r != 0:
            raise ChanError(r, self.L.chan_last_error(None).decode())
        self._h = h

    # -------------------------------------------------------------- plumbing
    def _check(self, r):
        if r == 0:
            return 0
        if r == _lib.CHAN_BLOWUP:
            ijk, n, _ = self.status_detail()
            raise BlowUpError(r, f"blow-up (rho<0 or T<0) at i,j,k={ijk} in step {n}", ijk, n)
        if r == _lib.CHAN_NONFINITE:
            return r
        raise ChanError(r, self.L.chan_last_error(self._h).decode())

    def close(self):
        ens = getattr(self, "_ensemble", None)
        if ens is not None:   # an ensemble is freed before its members
            ens.close()
        if getattr(self, "_h", None):
            self.L.chan_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        n1, n2, n3 = self.nP
        return (7, n3, n2, n1)

    # ------------------------------------------------------ reference names
    def init_sol_v(self, var: np.ndarray, nstep: int = 0, time: float = 0.0):
        v = np.ascontiguousarray(var, dtype=np.float64)
        if v.shape != self.shape:
            raise ValueError(f"var must have shape {self.shape}")
        self._check(self.L.chan_upload(self._h, _lib.dptr(v), int(nstep), float(time)))

    def read_input_file(self, path):
        from .deck import read_3d_dat_native
        var, time, nstep, *_ = read_3d_dat_native(path, self.nP)
        self.init_sol_v(var, nstep, time)
        return var

    def checkpoint_write(self, path):
        """Exact binary checkpoint of the device state (between steps)."""
        self._check(self.L.chan_checkpoint_write(self._h, str(path).encode()))

    def checkpoint_read(self, path):
        self._check(self.L.chan_checkpoint_read(self._h, str(path).encode()))

    def stage(self, it: int):
        return self._check(self.L.chan_stage(self._h, int(it)))

    def step(self, n: int = 1):
        return self._check(self.L.chan_step(self._h, int(n)))

    def step_async(self, n: int = 1):
        return self._check(self.L.chan_step_async(self._h, int(n)))

    def sync(self):
        return self._check(self.L.chan_sync(self._h))

    def check_soln(self):
        return self._check(self.L.chan_check(self._h))

    def calc_tau_wall(self):
        return self._check(self.L.chan_tau_wall(self._h))

    def avg_spatial(self):
        return self._check(self.L.chan_avg_spatial(self._h))

    def stats(self):
        n3 = self.nP[2]
        tau = np.zeros(2); s1 = np.zeros((7, n3)); s2 = np.zeros((7, n3)); c = np.zeros((9, n3))
        self._check(self.L.chan_stats(self._h, _lib.dptr(tau), _lib.dptr(s1), _lib.dptr(s2), _lib.dptr(c)))
        return tau, s1, s2, c

    def time_avg_start(self):
        """Start device-side time averaging of the statistics steps."""
        self._check(self.L.chan_time_avg_start(self._h))

    def time_average(self):
        """avg_v1.7.f90 over the statistics steps since time_avg_start:
        dict with mean, rms, covar, tau (means), samples, t0, t1."""
        from .stats import time_average
        n3 = self.nP[2]
        s1 = np.zeros((7, n3)); s2 = np.zeros((7, n3)); sc = np.zeros((9, n3)); st = np.zeros(2)
        n = ctypes.c_int64(); t0 = ctypes.c_double(); t1 = ctypes.c_double()
        self._check(self.L.chan_time_avg(self._h, _lib.dptr(s1), _lib.dptr(s2), _lib.dptr(sc), _lib.dptr(st),
                                         ctypes.byref(n), ctypes.byref(t0), ctypes.byref(t1)))
        mean, rms, covar, tau = time_average(s1, s2, sc, st, n.value)
        return {"mean": mean, "rms": rms, "covar": covar, "tau": tau, "samples": n.value,
                "t0": t0.value, "t1": t1.value}

    def set_wall_bc(self, wall: int, bc):
        """Wall-BC plug-in for wall 0 (k=1) or 1 (k=nP3); ``bc`` is a wallbc.WallBC."""
        c = _lib.ChanWallBCC()
        c.velocity = int(bc.velocity); c.thermal = int(bc.thermal)
        c.Tw = float(bc.Tw); c.dTdz = float(bc.dTdz); c.slip_grad = float(bc.slip_grad)
        c.wave[:] = [float(x) for x in bc.wave]
        keep = []
        if bc.mask is not None:
            m = np.ascontiguousarray(bc.mask, dtype=np.uint8); keep.append(m)
            c.mask = m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        if bc.uv is not None:
            uv = np.ascontiguousarray(bc.uv, dtype=np.float64); keep.append(uv)
            c.uv = _lib.dptr(uv)
        if bc.x1 is not None:
            x1 = np.ascontiguousarray(bc.x1, dtype=np.float64); keep.append(x1)
            c.x1 = _lib.dptr(x1)
        self._check(self.L.chan_set_wall_bc(self._h, int(wall), ctypes.byref(c)))

    def diag_enable(self, planes=(5, 10, 70, 100, 125), every: int = 10, x3q=None, x2end=None,
                    capacity: int = 4096):
        """Diagnostics series of main_v1.9.f90:799-906 every ``every`` steps, kept on
        the device (0 turns it off).  x3q / x2end: the coordinates the reference
        holds when it writes the series (after a restart, the deck's F10.6
        columns); defaults: the mesh x3 and x2(nP2) accumulated from Ly."""
        from .mesh import periodic_coords
        pl = (ctypes.c_int32 * max(1, len(planes)))(*[int(p) for p in planes])
        if x2end is None:
            x2end = float(periodic_coords(self.nP[1], self.params.Ly)[-1])
        z = None if x3q is None else np.ascontiguousarray(x3q, dtype=np.float64)
        self._diag_np = len(planes)
        self._check(self.L.chan_diag_enable(self._h, pl, len(planes), int(every),
                                            None if z is None else _lib.dptr(z), float(x2end), int(capacity)))

    def diag_read(self):
        """Drain the device series: dict with nstep, time, ke (n,), rho_b, u_b,
        rhou_b (n, nplanes) and lost (records the ring overwrote)."""
        n = ctypes.c_int32(); lost = ctypes.c_int64()
        self._check(self.L.chan_diag_read(self._h, None, 0, ctypes.byref(n), ctypes.byref(lost)))
        npl = getattr(self, "_diag_np", 0)
        rec = np.zeros((max(n.value, 1), 3 + 3 * npl))
        self._check(self.L.chan_diag_read(self._h, _lib.dptr(rec), rec.shape[0], ctypes.byref(n),
                                          ctypes.byref(lost)))
        rec = rec[:n.value]
        return {"nstep": rec[:, 0].astype(np.int64), "time": rec[:, 1], "ke": rec[:, 2],
                "rho_b": rec[:, 3:3 + npl], "u_b": rec[:, 3 + npl:3 + 2 * npl],
                "rhou_b": rec[:, 3 + 2 * npl:3 + 3 * npl], "lost": lost.value}

    def fluctuation_q(self, mean, x1=None, x2=None, x3=None, want_fluc=True, want_q=True):
        """(fluc, Q) of the current state on the device: fluc.f90:63-69 and
        qInvariant.f90:26-81.  mean is (7, nP3); either output may be skipped."""
        m = np.ascontiguousarray(mean, dtype=np.float64)
        assert m.shape == (7, self.nP[2])
        fl = np.empty(self.shape) if want_fluc else None
        q = np.empty(self.shape[1:]) if want_q else None
        cs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x1, x2, x3)]
        self._check(self.L.chan_fluctuation_q(self._h, _lib.dptr(m), *[None if a is None else _lib.dptr(a) for a in cs],
                                              None if fl is None else _lib.dptr(fl),
                                              None if q is None else _lib.dptr(q)))
        return fl, q

    def set_buoyancy(self, Ri: float, Tref: float = 1.0):
        """Buoyancy body force Ri*rho*(T - Tref) on the wall-normal momentum
        (and its work on the energy); Ri = 0 switches it off."""
        self._check(self.L.chan_set_buoyancy(self._h, float(Ri), float(Tref)))

    def set_launch(self, tile: int = 0, nchunks: int = 0):
        """Stage-kernel launch shape: tile 0 (32x8), 1 (32x4), 2 (16x16) or 3 (32x16), k-chunks (0: automatic)."""
        self._check(self.L.chan_set_launch(self._h, int(tile), int(nchunks)))

    def launch(self):
        """(tile, nchunks, planes per chunk) of the stage kernel."""
        t, n, k = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self.L.chan_get_launch(self._h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(k)))
        return t.value, n.value, k.value

    def set_forcing(self, tauL: float, tauU: float, rhobar):
        rb = np.ascontiguousarray(rhobar, dtype=np.float64)
        self._check(self.L.chan_set_forcing(self._h, float(tauL), float(tauU), _lib.dptr(rb)))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape)
        assert out.shape == self.shape and out.dtype == np.float64 and out.flags.c_contiguous
        self._check(self.L.chan_download(self._h, _lib.dptr(out)))
        return out

    def write_soln(self, path):
        from .deck import write_3d_dat_native
        from .mesh import periodic_coords
        var = self.download()
        _, n, t = self.status_detail()
        write_3d_dat_native(path, var, periodic_coords(self.nP[0], self.params.Lx),
                            periodic_coords(self.nP[1], self.params.Ly), self.x3, t, n)

    def status_detail(self):
        ijk = (ctypes.c_int32 * 3)()
        n = ctypes.c_int64()
        t = ctypes.c_double()
        self.L.chan_status(self._h, ijk, ctypes.byref(n), ctypes.byref(t))
        return tuple(ijk), n.value, t.value

    def status(self) -> int:
        ijk = (ctypes.c_int32 * 3)()
        return self.L.chan_status(self._h, ijk, None, None)

    @property
    def nstep(self):
        return self.status_detail()[1]

    @property
    def time(self):
        return self.status_detail()[2]

    # -------------------------------------------------------- measurement
    def profile(self, enable: bool):
        self._check(self.L.chan_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        ms = np.zeros(3)
        cnt = np.zeros(3, dtype=np.int64)
        self._check(self.L.chan_profile_read(self._h, _lib.dptr(ms), cnt.ctypes.data_as(_lib._I64)))
        return ms, cnt

    def stream_handle(self) -> int:
        return int(self.L.chan_stream(self._h) or 0)

    def debug_canaries(self) -> int:
        """Guard words around the state buffers that changed (0: no stray writes)."""
        n = ctypes.c_int64()
        self._check(self.L.chan_debug_canaries(self._h, ctypes.byref(n)))
        return n.value

    def device_bytes(self) -> int:
        return int(self.L.chan_device_bytes(self._h))


def q_criterion(u, v, w, x1, x2, x3, device: int = 0):
    """Q-criterion (qInvariant.f90:26-81) of host velocity arrays (nP3, nP2, nP1) on a GPU."""
    L = _lib.load()
    u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
    n3, n2, n1 = u.shape
    x1, x2, x3 = (np.ascontiguousarray(a, dtype=np.float64) for a in (x1, x2, x3))
    Q = np.empty_like(u)
    nP = (ctypes.c_int32 * 3)(n1, n2, n3)
    r = L.chan_q_criterion(nP, _lib.dptr(u), _lib.dptr(v), _lib.dptr(w), _lib.dptr(x1), _lib.dptr(x2),
                           _lib.dptr(x3), _lib.dptr(Q), int(device))
    if r != 0:
        raise ChanError(r, L.chan_last_error(None).decode())
    return Q


def version() -> str:
    return _lib.load().chan_version().decode()
