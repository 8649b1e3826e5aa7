"""Ensembles of channel cases stepped together on one GPU, and the stratified
parameter sweep they are built for.

``Ensemble`` wraps chan_ensemble_* (include/chanrhs.h): a block of L steps
of every member (L = least common multiple of the members' istat) is
captured once into a CUDA graph and replayed.  By default that graph holds
every member's kernels, one branch per member on its own stream
(``mode="graph"``); ``mode="persistent"`` captures instead one persistent
kernel which runs every member's work units from one work list, ordered by
per-member device counters with bounded waits.  Results are bit for bit
those of stepping each member alone.  ``Ensemble.tune`` runs the
launch-shape autotuner.

``sweep_cases`` builds the sweep: cases of uneven grid sizes with per-case
Mach and Reynolds numbers, a top-bottom wall temperature difference and a
buoyancy body force of bulk Richardson number Ri (Channel.set_buoyancy).
The reference runs one case per MPI job and has no buoyancy term; its
stratified variants (v1.9_strat) change only the wall temperature.
"""
from __future__ import annotations

import ctypes
import itertools
from dataclasses import dataclass

import numpy as np

from . import _lib
from .channel import Channel, ChanError
from .ic import laminar_noise, uniform_pm1
from .mesh import cfl_dt, mesh_tanh
from .params import ChanParams, RK3


class Ensemble:
    def __init__(self, channels):
        self.L = _lib.load()
        self.members = list(channels)
        n = len(self.members)
        if n < 1:
            raise ValueError("an ensemble needs at least one member")
        arr = (ctypes.c_void_p * n)(*[c._h for c in self.members])
        h = ctypes.c_void_p()
        r = self.L.chan_ensemble_create(arr, n, ctypes.byref(h))
        if r != 0:
            raise ChanError(r, "chan_ensemble_create: " + (self.L.chan_ensemble_last_error(None) or b"").decode())
        self._h = h
        for c in self.members:
            c._ensemble = self

    @property
    def block(self) -> int:
        """Steps per graph replay."""
        return int(self.L.chan_ensemble_block(self._h))

    def step(self, n: int = 1):
        """n steps of every member; returns the members' status codes (0 = ok,
        CHAN_BLOWUP / CHAN_NONFINITE for a member whose state blew up)."""
        st = (ctypes.c_int32 * len(self.members))()
        r = self.L.chan_ensemble_step(self._h, int(n), st)
        if r < 0:
            raise ChanError(r, self.L.chan_ensemble_last_error(self._h).decode())
        return list(st)

    def tune(self, reps: int = 3) -> float:
        """Autotune the members' launch shapes; returns ms per trial step."""
        ms = ctypes.c_double()
        r = self.L.chan_ensemble_tune(self._h, int(reps), ctypes.byref(ms))
        if r != 0:
            raise ChanError(r, self.L.chan_ensemble_last_error(self._h).decode())
        return ms.value

    MODES = {"graph": _lib.CHAN_ENSEMBLE_GRAPH, "persistent": _lib.CHAN_ENSEMBLE_PERSISTENT,
             "persistent-stall-test": _lib.CHAN_ENSEMBLE_PERSISTENT_STALL_TEST}

    def set_mode(self, mode: str):
        """"graph" (default), "persistent", or "persistent-stall-test" (host-side
        fault injection: a dependency that is never met, for tests)."""
        r = self.L.chan_ensemble_set_mode(self._h, self.MODES[mode])
        if r != 0:
            raise ChanError(r, self.L.chan_ensemble_last_error(self._h).decode())

    def mode_in_use(self):
        """("persistent" | "graph" | None before the first block, fallback reason)."""
        m, why = ctypes.c_int32(), ctypes.c_char_p()
        self.L.chan_ensemble_get_mode(self._h, ctypes.byref(m), ctypes.byref(why))
        name = {_lib.CHAN_ENSEMBLE_GRAPH: "graph", _lib.CHAN_ENSEMBLE_PERSISTENT: "persistent"}.get(m.value)
        return name, (why.value or b"").decode()

    def counters(self):
        """(graph replays, graph captures) so far."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self.L.chan_ensemble_counters(self._h, ctypes.byref(a), ctypes.byref(b), None)
        return a.value, b.value

    def last_replay_ms(self) -> float:
        """Device time (CUDA events) of the graph replays of the last step() call."""
        ms = ctypes.c_double()
        self.L.chan_ensemble_counters(self._h, None, None, ctypes.byref(ms))
        return ms.value

    def launch_shapes(self):
        return [c.launch() for c in self.members]

    def close(self):
        if getattr(self, "_h", None):
            self.L.chan_ensemble_free(self._h)
            self._h = None
            for c in self.members:
                c._ensemble = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ the sweep
MACH = (0.5, 1.5)
REYNOLDS = (2000.0, 3000.0, 4000.0)
RICHARDSON = (0.0, 0.1, 0.5)
DELTA_T = (0.0, 0.2)


@dataclass
class SweepCase:
    params: ChanParams
    x3: np.ndarray
    jac: np.ndarray
    inv: np.ndarray
    var: np.ndarray
    Ri: float
    dT: float
    Tref: float


def sweep_grids(n: int):
    """n uneven grids from nP = (64, 64, 65) to (160, 128, 129): x and y in
    steps of 8 points, an odd wall-normal count, sizes spread linearly."""
    out = []
    for c in range(n):
        f = c / max(n - 1, 1)
        n1 = 64 + 8 * int(round(12 * f))
        n2 = 64 + 8 * int(round(8 * ((c * 5) % n) / max(n - 1, 1)))   # y sizes shuffled against x
        n3 = 65 + 8 * int(round(8 * ((c * 3) % n) / max(n - 1, 1)))
        out.append((n1, n2, n3))
    return out


def stratified_start(p: ChanParams, x3, Tb: float, Tt: float, seed: int, amp: float = 0.1):
    """The seeded laminar start (ic.laminar_noise) with a linear temperature
    profile between the wall temperatures Tb (k=1) and Tt (k=nP3) at uniform
    pressure: rho = 1/T, p = 1/(gama Ma^2), E = T + ggM/2 |u|^2."""
    var = laminar_noise(p, x3, seed=seed, amp=amp)
    x3 = np.asarray(x3, dtype=np.float64)
    T = (Tb + (Tt - Tb) * (x3 - x3[0]) / (x3[-1] - x3[0]))[:, None, None] * np.ones_like(var[0])
    rho = 1.0 / T
    u, v, w = var[1], var[2], var[3]
    var[0] = rho
    var[5] = T
    var[4] = T + 0.5 * p.ggM * ((u * u + v * v) + w * w)
    var[6] = (rho * T) / (p.gama * p.Mac * p.Mac)
    return var


def sweep_cases(n: int = 16, seed: int = 2024, cfl: float = 0.6, beta: float = 2.2, mixed: bool = True,
                istat: int = 10, grids=None):
    """n cases: grids from sweep_grids; (Ma, Re, Ri, dT) drawn without
    repetition from the 36 combinations by a seeded shuffle; stable
    stratification (the top wall hotter by dT about Tref = 1); SSP-RK3 at the
    given CFL; each case's own seeded start."""
    combos = list(itertools.product(MACH, REYNOLDS, RICHARDSON, DELTA_T))
    key = uniform_pm1(seed, 0, np.arange(len(combos)), np.zeros(len(combos), np.int64),
                      np.zeros(len(combos), np.int64))
    order = np.argsort(key, kind="stable")
    grids = grids or sweep_grids(n)
    cases = []
    for c in range(n):
        Ma, Re, Ri, dT = combos[int(order[c % len(combos)])]
        nP = tuple(grids[c])
        Tb, Tt = 1.0 - 0.5 * dT, 1.0 + 0.5 * dT
        x3, jac, inv = mesh_tanh(nP[2], beta)
        p = ChanParams(nP=nP, Re=Re, Mac=Ma, Pr=0.72, rk_scheme=RK3, istat=istat, Tw=(Tb, Tt), mixed=mixed)
        var = stratified_start(p, x3, Tb, Tt, seed=seed + 7 * c)
        p = p.with_(dt=cfl_dt(var, p, jac, cfl))
        cases.append(SweepCase(p, x3, jac, inv, var, Ri, dT, 1.0))
    return cases


def open_case(case: SweepCase) -> Channel:
    """A Channel for one sweep case, uploaded, with its buoyancy term set."""
    ch = Channel(case.params, case.x3, case.jac, case.inv)
    ch.set_buoyancy(case.Ri, case.Tref)
    ch.init_sol_v(case.var)
    return ch
