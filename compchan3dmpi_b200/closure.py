"""Learned subgrid closure: a small MLP trained on box-filtered DNS snapshots
that lets a coarse run stand in for the DNS.

The reference (theparvezahmad/compChan3Dmpi) resolves every scale and has no
closure; this module adds one around the same solver:

* ``Closure`` wraps chan_closure_* (include/chanrhs.h): a device-resident
  dataset of (features, subgrid fluxes) samples, the 13 -> 64 -> 64 -> 9 GELU
  MLP with BF16 weights and F32 accumulation on the tensor cores, Adam.
* ``attach`` (chan_set_closure) puts it on a plain FP64 coarse context: every
  stage adds the divergence of the predicted subgrid fluxes.
* ``run_with_fallback`` steps a closure run and falls back to the plain
  method (restoring the last good checkpoint) if the closure diverges: a
  blow-up, a non-finite state, or a normalised output beyond its limit.
* ``main`` is the whole experiment: DNS from a smooth perturbation, snapshots
  filtered into the dataset, training, the coarse run with and without the
  closure from the filtered DNS state, and their statistics against the DNS.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import tempfile
import time

import numpy as np

from . import _lib
from .channel import Channel, ChanError, BlowUpError
from .ic import laminar_noise
from .mesh import cfl_dt, mesh_tanh, periodic_coords
from .params import ChanParams, RK3, production_params
from .stats import wall_units

N_IN, N_OUT = 13, 9
FEATURES = ["du/dx", "du/dy", "du/dz", "dv/dx", "dv/dy", "dv/dz", "dw/dx", "dw/dy", "dw/dz",
            "dT/dx", "dT/dy", "dT/dz", "y+"]
FLUXES = ["tau_uu", "tau_vv", "tau_ww", "tau_uv", "tau_uw", "tau_vw", "q_u", "q_v", "q_w"]


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Closure:
    def __init__(self, capacity: int = 0, device: int = 0):
        self.L = _lib.load()
        h = ctypes.c_void_p()
        r = self.L.chan_closure_create(int(device), int(capacity), ctypes.byref(h))
        if r != 0:
            raise ChanError(r, self.L.chan_closure_last_error(None).decode())
        self._h = h
        self.nparams = int(self.L.chan_closure_nparams())

    def _check(self, r):
        if r != 0:
            raise ChanError(r, self.L.chan_closure_last_error(self._h).decode())

    # ---------------------------------------------------------------- data
    def sample(self, dns: Channel, strides=(4, 3, 3), width: int = 4) -> int:
        n = ctypes.c_int64()
        self._check(self.L.chan_closure_sample(self._h, dns._h, *[int(s) for s in strides], int(width),
                                               ctypes.byref(n)))
        return n.value

    def add_data(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        assert X.shape[1] == N_IN and T.shape == (X.shape[0], N_OUT)
        self._check(self.L.chan_closure_add_data(self._h, _fp(X), _fp(T), X.shape[0]))

    @property
    def count(self) -> int:
        n = ctypes.c_int64()
        self._check(self.L.chan_closure_count(self._h, ctypes.byref(n)))
        return n.value

    def data(self, first: int = 0, n: int | None = None):
        n = self.count - first if n is None else n
        X = np.empty((n, N_IN), np.float32)
        T = np.empty((n, N_OUT), np.float32)
        self._check(self.L.chan_closure_get_data(self._h, int(first), int(n), _fp(X), _fp(T)))
        return X, T

    # ---------------------------------------------------------- parameters
    def fit_normalization(self):
        out = np.empty(44, np.float32)
        self._check(self.L.chan_closure_fit_normalization(self._h, _fp(out)))
        return out

    @property
    def norm(self):
        out = np.empty(44, np.float32)
        self._check(self.L.chan_closure_get_normalization(self._h, _fp(out)))
        return out

    @norm.setter
    def norm(self, v):
        v = np.ascontiguousarray(v, dtype=np.float32)
        assert v.shape == (44,)
        self._check(self.L.chan_closure_set_normalization(self._h, _fp(v)))

    def init(self, seed: int = 1):
        self._check(self.L.chan_closure_init(self._h, ctypes.c_uint64(seed)))

    @property
    def params(self):
        out = np.empty(self.nparams, np.float32)
        self._check(self.L.chan_closure_get_params(self._h, _fp(out)))
        return out

    @params.setter
    def params(self, v):
        v = np.ascontiguousarray(v, dtype=np.float32)
        assert v.shape == (self.nparams,)
        self._check(self.L.chan_closure_set_params(self._h, _fp(v)))

    def save(self, path):
        np.savez(path, params=self.params, norm=self.norm)

    def load(self, path):
        d = np.load(path)
        self.norm = d["norm"]
        self.params = d["params"]

    # ------------------------------------------------------------ learning
    def train(self, epochs: int, batch: int = 65536, lr: float = 1e-3, seed: int = 7):
        losses = np.zeros(max(epochs, 1))
        self._check(self.L.chan_closure_train(self._h, int(epochs), int(batch), float(lr), ctypes.c_uint64(seed),
                                              losses.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return losses[:epochs]

    def grad(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.empty(self.nparams, np.float32)
        loss = ctypes.c_double()
        self._check(self.L.chan_closure_grad(self._h, _fp(X), _fp(T), X.shape[0], _fp(g), ctypes.byref(loss)))
        return loss.value, g

    def infer(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.empty((X.shape[0], N_OUT), np.float32)
        self._check(self.L.chan_closure_infer(self._h, _fp(X), X.shape[0], _fp(Y)))
        return Y

    def close(self):
        if getattr(self, "_h", None):
            self.L.chan_closure_free(self._h)
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


def attach(ch: Channel, cl: Closure | None, on: bool = True, every_stage: bool = False):
    """Switch the closure of a coarse context on or off; by default its source
    is evaluated once per step (at the first stage) and held for the others."""
    mode = (2 if every_stage else 1) if on else 0
    r = ch.L.chan_set_closure(ch._h, cl._h if (cl is not None and on) else None, mode)
    ch._check(r)
    ch._closure = cl if on else None


def closure_flag(ch: Channel, reset: bool = True) -> int:
    f = ctypes.c_int32()
    ch._check(ch.L.chan_closure_flag(ch._h, ctypes.byref(f), 1 if reset else 0))
    return f.value


def run_with_fallback(ch: Channel, cl: Closure, steps: int, check_every: int = 100, workdir=None):
    """``steps`` steps with the closure, checking every ``check_every`` steps.
    On divergence (blow-up, non-finite state, or the closure's output flag)
    the last good checkpoint is restored and the remaining steps run with the
    plain method.  Returns {"fallback_step": step or None, "reason": ...,
    "plain_failed": None or the plain method's own failure}: if the plain
    continuation blows up too, the report says so (with its step) instead of
    the exception replacing it.  The checkpoint lives in ``workdir``, or in a
    temporary directory removed on return."""
    if workdir is None:
        with tempfile.TemporaryDirectory(prefix="closure_") as tmp:
            return run_with_fallback(ch, cl, steps, check_every, tmp)
    attach(ch, cl, True)
    closure_flag(ch, reset=True)
    ckp = os.path.join(workdir, "last_good.ckp")
    ch.checkpoint_write(ckp)
    done, report = 0, {"fallback_step": None, "reason": None, "plain_failed": None}
    while done < steps:
        n = min(check_every, steps - done)
        reason = None
        try:
            st = ch.step(n)
            if st:
                reason = "non-finite state"
        except BlowUpError:
            reason = "blow-up"
        if reason is None and closure_flag(ch, reset=True):
            reason = "closure output beyond its limit"
        if reason is not None:
            ch.checkpoint_read(ckp)
            attach(ch, None, False)
            report = {"fallback_step": int(ch.nstep), "reason": reason, "plain_failed": None}
            try:
                if ch.step(steps - done):
                    report["plain_failed"] = {"reason": "non-finite state", "step": int(ch.nstep)}
            except BlowUpError as e:
                report["plain_failed"] = {"reason": "blow-up", "step": int(e.nstep), "ijk": list(e.ijk)}
            return report
        done += n
        ch.checkpoint_write(ckp)
    return report


# ------------------------------------------------------------------ experiment
def smooth_start(p: ChanParams, x3, amp: float = 0.2, modes: int = 4, seed: int = 7, noise: float = 0.02):
    """Laminar start plus smooth perturbations that drive transition: every
    (kx, kz) wavenumber pair up to ``modes`` in x and spanwise with a seeded
    phase per velocity component, shaped (1 - (x3 - 1)^2)^2 across the channel
    and scaled to ``amp``; plus the seeded grid-scale noise of amplitude
    ``noise`` (ic.laminar_noise)."""
    var = laminar_noise(p, x3, seed=1234, amp=noise)
    n1, n2, n3 = p.nP
    x1, x2 = periodic_coords(n1, p.Lx), periodic_coords(n2, p.Ly)
    Z, Y, X = np.meshgrid(np.asarray(x3), x2, x1, indexing="ij")
    f = (1.0 - (Z - 1.0) ** 2) ** 2
    rng = np.random.default_rng(seed)
    for comp in (1, 2, 3):
        d = np.zeros_like(X)
        for kx in range(1, modes + 1):
            for kz in range(1, modes + 1):
                d += np.cos(2 * np.pi * kx * X / p.Lx + 2 * np.pi * kz * Y / p.Ly + rng.uniform(0, 2 * np.pi))
        var[comp] += amp * (4.0 / (modes * modes)) * f * d
    var[4] = var[5] + 0.5 * p.ggM * (var[1] ** 2 + var[2] ** 2 + var[3] ** 2)
    var[6] = var[0] * var[5] / (p.gama * p.Mac ** 2)
    return var


def _interp_periodic(a, n_src, n_dst, axis):
    """Linear interpolation along a periodic axis stored with duplicates
    (unique points 2..n-1 of period n-2), onto the destination's unique points."""
    a = np.moveaxis(a, axis, -1)
    src = a[..., 1:n_src - 1]                       # unique points, period n_src - 2
    ms, md = n_src - 2, n_dst - 2
    pos = np.arange(md) * (ms / md)                 # destination unique points in source units
    i0 = np.floor(pos).astype(int)
    w = pos - i0
    out = src[..., i0 % ms] * (1 - w) + src[..., (i0 + 1) % ms] * w
    full = np.concatenate([out[..., -1:], out, out[..., :1]], axis=-1)
    return np.moveaxis(full, -1, axis)


def coarsen(var, p_dns: ChanParams, p_c: ChanParams, kstride: int):
    """A coarse-grid state from a DNS field: linear periodic interpolation in x
    and spanwise, every ``kstride``-th wall-normal plane (the tanh map of the
    coarse grid with the same beta samples the same stretched coordinates);
    E and p recomputed, the walls at rest at their temperature."""
    n1, n2, n3 = p_dns.nP
    c1, c2, c3 = p_c.nP
    assert (n3 - 1) % kstride == 0 and (n3 - 1) // kstride == c3 - 1
    prim = var[[0, 1, 2, 3, 5]][:, ::kstride]
    prim = _interp_periodic(prim, n1, c1, axis=-1)
    prim = _interp_periodic(prim, n2, c2, axis=-2)
    out = np.empty((7, c3, c2, c1))
    out[0], out[1], out[2], out[3], out[5] = prim
    for k, Tw in ((0, p_c.Tw[0]), (c3 - 1, p_c.Tw[1])):
        out[1:4, k] = 0.0
        out[5, k] = Tw
    out[4] = out[5] + 0.5 * p_c.ggM * (out[1] ** 2 + out[2] ** 2 + out[3] ** 2)
    out[6] = out[0] * out[5] / (p_c.gama * p_c.Mac ** 2)
    return out


def _profiles(avg, x3, Re):
    wu = wall_units(avg["mean"], avg["tau"], x3, Re)
    return {"Cf": wu["Cf"], "Re_tau": wu["Re_tau"], "u_tau": wu["u_tau"], "yplus": wu["yplus"].tolist(),
            "uplus": np.asarray(wu["uplus"]).tolist(), "u_rms": avg["rms"][1].tolist(),
            "w_rms": avg["rms"][3].tolist(), "uw": avg["covar"][3].tolist()}


def _errors(les, dns):
    """Relative errors of a coarse run's statistics against the DNS's at the
    same wall-normal points."""
    u_l, u_d = np.asarray(les["uplus"]), np.asarray(dns["uplus"])
    pk = lambda a: float(np.max(np.abs(np.asarray(a))))   # noqa: E731
    return {"Cf": abs(les["Cf"] - dns["Cf"]) / abs(dns["Cf"]),
            "uplus_max": float(np.max(np.abs(u_l - u_d)) / np.max(np.abs(u_d))),
            "u_rms_peak": abs(pk(les["u_rms"]) - pk(dns["u_rms"])) / pk(dns["u_rms"]),
            "uw_peak": abs(pk(les["uw"]) - pk(dns["uw"])) / pk(dns["uw"])}


def _seeds(s):
    """A seed or a sequence of seeds, as a tuple."""
    return tuple(int(x) for x in s) if isinstance(s, (tuple, list)) else (int(s),)


def mean_stats(stats):
    """The statistics of several coarse runs averaged run by run: Cf, Re_tau and
    u_tau, and each profile point by point (the same grid for every run)."""
    out = {}
    for k in stats[0]:
        v = [st[k] for st in stats]
        out[k] = np.mean(np.asarray(v, dtype=np.float64), axis=0).tolist() if isinstance(v[0], list) \
            else float(np.mean(v))
    return out


def seed_runs(runs):
    """Coarse runs from several seeds as one result: the statistics averaged
    over the runs (None if any run blew up or fell back), the first fallback
    report, the mean wall time of a run, and the runs themselves."""
    ok = all(r["stats"] is not None and r["report"]["fallback_step"] is None for r in runs)
    rep = next((r["report"] for r in runs if r["report"]["fallback_step"] is not None or r["report"]["reason"]),
               runs[0]["report"])
    return {"steps": runs[0]["steps"], "wall_s": float(np.mean([r["wall_s"] for r in runs])), "report": rep,
            "stats": mean_stats([r["stats"] for r in runs]) if ok else None, "per_seed": runs}


def wall_shear_history(ch: Channel, steps: int, every: int):
    """Step ``steps`` steps in chunks of ``every`` (a multiple of istat) and
    record (time, wall shear (tauL - tauU)/2) after each chunk."""
    out = []
    done = 0
    while done < steps:
        n = min(every, steps - done)
        ch.step(n)
        done += n
        tau = ch.stats()[0]
        out.append((ch.time, 0.5 * (tau[0] - tau[1])))
    return out


def stationarity(hist):
    """Drift of the wall shear over a window: the least-squares slope times the
    window length over the mean, and the relative difference of its two halves."""
    t = np.array([h[0] for h in hist]); w = np.array([h[1] for h in hist])
    if len(t) < 4:
        return {"drift": None, "halves": None}
    slope = np.polyfit(t - t[0], w, 1)[0]
    h = len(w) // 2
    return {"tau_w_mean": float(w.mean()), "drift": float(slope * (t[-1] - t[0]) / w.mean()),
            "halves": float((w[h:].mean() - w[:h].mean()) / w.mean()), "records": len(w)}


def scaled_norm(norm, alpha: float):
    """The closure's normalisation with its outputs scaled by alpha (output
    means and standard deviations times alpha): the closure's magnitude knob."""
    n = np.array(norm, dtype=np.float32, copy=True)
    n[26:44] *= alpha
    return n


def coarse_run(pc: ChanParams, x3, jac, inv, var, steps: int, cl: Closure | None = None, avg_from: float = 0.5,
               check_every: int = 200, sample_into: Closure | None = None, sample_every: int = 200):
    """A coarse run of ``steps`` steps from ``var``, statistics time-averaged over
    the steps after ``avg_from`` of the run; with ``cl`` the closure is on, with
    fallback to the plain method.  With ``sample_into`` (plain runs) the run's
    own closure inputs -- every interior point, no filter, the features the
    closure would see -- are sampled every ``sample_every`` steps of the
    averaging window."""
    ch = Channel(pc, x3, jac, inv)
    ch.init_sol_v(var)
    first = int(steps * avg_from) // max(pc.istat, 1) * max(pc.istat, 1)
    t0 = time.time()
    rep = {"fallback_step": None, "reason": None, "plain_failed": None}
    try:
        if cl is None:
            nonfinite = ch.step(first) != 0
            ch.time_avg_start()
            if sample_into is None:
                nonfinite = nonfinite or ch.step(steps - first) != 0
            else:
                done = first
                while done < steps and not nonfinite:
                    n = min(sample_every, steps - done)
                    nonfinite = ch.step(n) != 0
                    done += n
                    sample_into.sample(ch, strides=(1, 1, 1), width=0)
            if nonfinite:
                rep = {"fallback_step": None, "reason": "blew up: non-finite state", "plain_failed": None}
        else:
            rep = run_with_fallback(ch, cl, first, check_every=check_every)
            ch.time_avg_start()
            if rep["fallback_step"] is None:
                r2 = run_with_fallback(ch, cl, steps - first, check_every=check_every)
                if r2["fallback_step"] is not None:
                    rep = r2
            else:
                ch.step(steps - first)
    except BlowUpError as e:
        rep = {"fallback_step": None, "reason": f"blew up: {e}", "plain_failed": None}
    wall = time.time() - t0
    st = None
    if not (rep["reason"] or "").startswith("blew up") and rep.get("plain_failed") is None:
        st = _profiles(ch.time_average(), x3, pc.Re)
    ch.close()
    return {"steps": steps, "wall_s": wall, "report": rep, "stats": st}


def add_shear_deficit(src: Closure, dst: Closure, deficit, per_snapshot: int, per_plane: int, chunk: int = 1 << 22):
    """Copy the dataset of ``src`` into ``dst`` with the mean Reynolds-shear-
    stress deficit of the coarse solver added to each sample's tau_uw target:
    samples come in snapshots of ``per_snapshot`` (per_plane samples per
    coarse interior plane, planes in order), so sample s sits on coarse plane
    ((s mod per_snapshot) // per_plane) + 1, whose deficit is added."""
    n = src.count
    d = np.asarray(deficit, dtype=np.float64)
    for first in range(0, n, chunk):
        m = min(chunk, n - first)
        X, T = src.data(first, m)
        idx = np.arange(first, first + m)
        kc = (idx % per_snapshot) // per_plane + 1
        T[:, 4] += d[kc].astype(np.float32)
        dst.add_data(X, T)


def _train_and_calibrate(name, sources, deficit, pcc, x3c, jacc, invc, start, cal_seed, coarse_steps, dns_c, epochs,
                         batch, lr, seed, alphas, log):
    """One training set: the samples of ``sources`` (closure datasets with their
    snapshot layout) with the coarse solver's shear-stress deficit added to
    tau_uw; training; the magnitude alpha picked by coarse runs from the
    calibration seeds (their statistics averaged over the runs).  Returns
    (closure, normalisation, alpha, report)."""
    cl = Closure(capacity=sum(src.count for src, _, _ in sources))
    for src, per_snap, per_plane in sources:
        add_shear_deficit(src, cl, deficit, per_snap, per_plane)
    cl.fit_normalization()
    norm0 = cl.norm
    cl.init(seed=seed)
    t0 = time.time()
    losses = cl.train(epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.time() - t0
    log(json.dumps({"phase": f"training ({name})", "epochs": epochs, "samples": cl.count,
                    "loss_first": float(losses[0]), "loss_last": float(losses[-1]), "wall_s": train_s}))
    cal = {}
    for a in alphas:
        cl.norm = scaled_norm(norm0, a)
        runs = []
        for sd in _seeds(cal_seed):
            runs.append(coarse_run(pcc, x3c, jacc, invc, start(sd), coarse_steps, cl))
            if runs[-1]["report"]["fallback_step"] is not None or runs[-1]["stats"] is None:
                break   # this alpha is out: the other seeds need not run
        r = seed_runs(runs)
        e = _errors(r["stats"], dns_c) if r["stats"] else None
        cal[a] = {"report": r["report"], "errors": e, "wall_s": r["wall_s"], "seeds_run": len(runs)}
        log(json.dumps({"phase": f"calibration ({name})", "alpha": a, **cal[a]}))
    ok = {a: c for a, c in cal.items() if c["errors"] is not None}
    best = min(ok, key=lambda a: ok[a]["errors"]["Cf"] + ok[a]["errors"]["uw_peak"]) if ok else None
    rep = {"samples": cl.count, "losses": [float(x) for x in losses], "train_s": train_s,
           "calibration": {str(a): c for a, c in cal.items()}, "alpha": best,
           "score": (ok[best]["errors"]["Cf"] + ok[best]["errors"]["uw_peak"]) if best is not None else None}
    return cl, norm0, best, rep


def experiment(dns_grid=(256, 192, 193), coarse_grid=(64, 64, 65), spinup=150000, snapshots=200, snap_every=200,
               coarse_steps=20000, epochs=20, batch=65536, lr=1e-3, cfl=0.6, beta=2.2, seed=7, cal_seed=21,
               eval_seed=33, alphas=(0.5, 1.0, 2.0, 3.0), fp64_probe=400, filter_width=4, rec_every=1000,
               coarse_snapshots=50, Re=None, log=print):
    """The closure experiment.

    1. DNS (mixed precision) from a smooth seeded perturbation, ``spinup``
       steps, then a window of ``snapshots`` x ``snap_every`` steps in which the
       width-``filter_width`` filtered DNS is sampled into the dataset and the
       statistics are time-averaged; the wall shear is recorded every
       ``rec_every`` steps to show whether the window is stationary.
    2. Plain coarse runs (``coarse_steps`` steps from seeded smooth
       perturbations, one per calibration seed, statistics over each run's
       second half, averaged over the runs) give what the coarse solver
       misses: the deficit of its mean Reynolds shear stress rho<u'w'> against
       the DNS at its wall-normal points.  ``coarse_snapshots`` of each run's
       own closure inputs are sampled over the same half.
    3. Two training sets, each with that deficit added to tau_uw plane by
       plane: the filtered-DNS samples with their subgrid fluxes, and those plus
       the coarse run's own inputs (deficit targets only), which are the inputs
       the closure meets in a coarse run.
    4. For each, the closure's magnitude alpha (its outputs scaled by alpha) is
       chosen by coarse runs from the calibration seeds; the better training
       set by that score is then compared, plain against closure, in coarse
       runs from the evaluation seeds (statistics averaged over the runs, and
       each run's own errors).  ``cal_seed`` and ``eval_seed`` are a seed or a
       sequence of seeds.
    """
    t_all = time.time()
    kst = (dns_grid[2] - 1) // (coarse_grid[2] - 1)
    x3d, jacd, invd = mesh_tanh(dns_grid[2], beta)
    pd = production_params(dns_grid).with_(mixed=True)
    if Re is not None:
        pd = pd.with_(Re=Re)
    var0 = smooth_start(pd, x3d, seed=seed)
    pd = pd.with_(dt=cfl_dt(var0, pd, jacd, cfl))
    dns = Channel(pd, x3d, jacd, invd)
    dns.init_sol_v(var0)
    rec = max(rec_every // pd.istat, 1) * pd.istat
    hist_spin = wall_shear_history(dns, spinup, rec)
    log(json.dumps({"phase": "dns spin-up", "steps": spinup, "t": dns.time,
                    "last_half": stationarity(hist_spin[len(hist_spin) // 2:])}))
    x3c, jacc, invc = mesh_tanh(coarse_grid[2], beta)
    pc = production_params(coarse_grid)
    if Re is not None:
        pc = pc.with_(Re=Re)
    window = snapshots * snap_every * pd.dt
    per_plane = ((dns_grid[0] - 3) // 4 + 1) * ((dns_grid[1] - 3) // 3 + 1)
    per_snap = per_plane * ((dns_grid[2] - 1) // kst - 1)
    raw = Closure(capacity=snapshots * per_snap)
    dns.time_avg_start()
    hist_win = []
    t0 = time.time()
    for s in range(snapshots):
        hist_win += wall_shear_history(dns, snap_every, snap_every)
        raw.sample(dns, strides=(4, 3, kst), width=filter_width)
    dns_wall = time.time() - t0
    avg_d = dns.time_average()
    dns_stats = _profiles(avg_d, x3d, pd.Re)
    rho_d = np.asarray(avg_d["mean"][0])
    f64 = Channel(pd.with_(mixed=False), x3d, jacd, invd)
    f64.init_sol_v(dns.download())
    f64.step(20)
    t0 = time.time()
    f64.step(fp64_probe)
    fp64_ms = (time.time() - t0) / fp64_probe * 1e3
    f64.close()
    dns_c = {k: (np.asarray(v)[::kst].tolist() if isinstance(v, list) else v) for k, v in dns_stats.items()}
    dns.close()
    stat = stationarity(hist_win)
    log(json.dumps({"phase": "dns window", "samples": raw.count, "window_t": window, "wall_s": dns_wall,
                    "Cf": dns_stats["Cf"], "Re_tau": dns_stats["Re_tau"], "stationarity": stat}))

    # coarse starts and dt: seeded smooth perturbations on the coarse grid
    def start(sd):
        return smooth_start(pc, x3c, seed=sd)
    cal_seeds, eval_seeds = _seeds(cal_seed), _seeds(eval_seed)
    dtc = cfl_dt(start(cal_seeds[0]), pc, jacc, cfl)
    pcc = pc.with_(dt=dtc)
    c1, c2, c3 = coarse_grid
    cper_plane, cper_snap = (c1 - 2) * (c2 - 2), (c1 - 2) * (c2 - 2) * (c3 - 2)
    craw = Closure(capacity=(coarse_snapshots + 1) * cper_snap * len(cal_seeds))
    every = max(((coarse_steps - coarse_steps // 2) // max(coarse_snapshots, 1)) // pcc.istat, 1) * pcc.istat
    plain_cal = seed_runs([coarse_run(pcc, x3c, jacc, invc, start(sd), coarse_steps, sample_into=craw,
                                      sample_every=every) for sd in cal_seeds])
    log(json.dumps({"phase": "coarse plain (calibration seeds)", "wall_s": plain_cal["wall_s"],
                    "samples": craw.count,
                    "errors": _errors(plain_cal["stats"], dns_c) if plain_cal["stats"] else None}))
    if plain_cal["stats"] is None:
        raise RuntimeError(f"the plain coarse run failed ({plain_cal['report']['reason']}): "
                           "no deficit to train on; try a smaller CFL or a finer coarse grid")
    # what the coarse solver misses: rho <u'w'> deficit at the coarse points
    uw_d = np.asarray(dns_c["uw"]) * rho_d[::kst]
    uw_c = np.asarray(plain_cal["stats"]["uw"]) * rho_d[::kst]
    deficit = uw_d - uw_c
    sets = {"filtered DNS": [(raw, per_snap, per_plane)],
            "filtered DNS + coarse inputs": [(raw, per_snap, per_plane), (craw, cper_snap, cper_plane)]}
    trained = {}
    for name, srcs in sets.items():
        trained[name] = _train_and_calibrate(name, srcs, deficit, pcc, x3c, jacc, invc, start, cal_seed,
                                             coarse_steps, dns_c, epochs, batch, lr, seed, alphas, log)
    ok = {n: t for n, t in trained.items() if t[2] is not None}
    chosen = min(ok, key=lambda n: ok[n][3]["score"]) if ok else None
    # evaluation from other seeds: plain against the calibrated closure
    runs = {"plain": seed_runs([coarse_run(pcc, x3c, jacc, invc, start(sd), coarse_steps) for sd in eval_seeds])}
    if chosen is not None:
        cl, norm0, best, _ = trained[chosen]
        cl.norm = scaled_norm(norm0, best)
        runs["closure"] = seed_runs([coarse_run(pcc, x3c, jacc, invc, start(sd), coarse_steps, cl)
                                     for sd in eval_seeds])
    for name, r in runs.items():
        r["errors_vs_dns"] = _errors(r["stats"], dns_c) if r["stats"] else None
        for q in r["per_seed"]:
            q["errors_vs_dns"] = _errors(q["stats"], dns_c) if q["stats"] else None
        log(json.dumps({"phase": f"coarse {name} (evaluation seeds)", "wall_s": r["wall_s"], "report": r["report"],
                        "errors": r["errors_vs_dns"], "per_seed": [q["errors_vs_dns"] for q in r["per_seed"]]}))
    fp64_window_s = fp64_ms * 1e-3 * snapshots * snap_every
    fp64_coarse_equiv_s = fp64_ms * 1e-3 * (coarse_steps * pcc.dt / pd.dt)
    out = {"dns": {"nP": list(dns_grid), "Re": pd.Re, "dt": pd.dt, "spinup_steps": spinup,
                   "window_steps": snapshots * snap_every, "window_t": window, "wall_s": dns_wall, "stats": dns_c,
                   "precision": "mixed FP32/FP64", "stationarity_window": stat,
                   "stationarity_spinup_last_half": stationarity(hist_spin[len(hist_spin) // 2:]),
                   "fp64_ms_per_step": fp64_ms, "fp64_window_s": fp64_window_s},
           "coarse": {"nP": list(coarse_grid), "dt": pcc.dt, "steps": coarse_steps,
                      "seeds": {"calibration": list(cal_seeds), "evaluation": list(eval_seeds)},
                      "deficit_rho_uw": deficit.tolist(), "training_sets": {n: t[3] for n, t in trained.items()},
                      "chosen": chosen, "alpha": trained[chosen][2] if chosen else None, "runs": runs},
           "wall_time_fp64_dns_same_physical_time_over_closure":
               (fp64_coarse_equiv_s / runs["closure"]["wall_s"]) if "closure" in runs else None,
           "total_s": time.time() - t_all}
    if chosen is not None:
        cl, norm0, best, _ = trained[chosen]
        params, norm = cl.params, scaled_norm(norm0, best)
    else:
        params, norm = None, None
    for t in trained.values():
        t[0].close()
    raw.close()
    craw.close()
    return out, params, norm


def synthetic_train(n: int, epochs: int, batch: int = 65536, seed: int = 4):
    """Training throughput on a synthetic dataset of n samples (a smooth map of
    Gaussian inputs): the tensor-core training kernel alone, for measurement."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, N_IN)).astype(np.float32)
    A = rng.standard_normal((N_IN, N_OUT)) * 0.5
    T = (np.tanh(X @ A) + 0.1 * X[:, :N_OUT] ** 2).astype(np.float32)
    with Closure(capacity=n) as cl:
        cl.add_data(X, T)
        cl.fit_normalization()
        cl.init(seed=seed)
        cl.train(1, batch=batch, seed=seed)          # warm-up epoch
        t0 = time.time()
        losses = cl.train(epochs, batch=batch, seed=seed + 1)
        dt = time.time() - t0
    steps = epochs * (n // batch)
    return {"samples": n, "epochs": epochs, "batch": batch, "steps": steps, "ms_per_step": dt / steps * 1e3,
            "samples_per_s": steps * batch / dt, "loss_first": float(losses[0]), "loss_last": float(losses[-1])}


def main(argv=None):
    ap = argparse.ArgumentParser(description="learned subgrid closure: DNS -> dataset -> training -> coarse runs")
    ap.add_argument("--synthetic-train", type=int, default=0, metavar="N",
                    help="only time training on N synthetic samples (the tensor-core kernel alone)")
    ap.add_argument("--spinup", type=int, default=150000)
    ap.add_argument("--snapshots", type=int, default=200)
    ap.add_argument("--coarse-steps", type=int, default=20000)
    ap.add_argument("--alphas", type=float, nargs="+", default=[0.5, 1.0, 2.0, 3.0])
    ap.add_argument("--snap-every", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--dns-grid", type=int, nargs=3, default=[256, 192, 193])
    ap.add_argument("--coarse-grid", type=int, nargs=3, default=[64, 64, 65])
    ap.add_argument("--filter-width", type=int, default=4,
                    help="box-filter width (even, in DNS points) in x and spanwise for the training targets")
    ap.add_argument("--cfl", type=float, default=0.6)
    ap.add_argument("--re", type=float, default=None, help="Reynolds number (default: the production 3000)")
    ap.add_argument("--coarse-snapshots", type=int, default=50)
    ap.add_argument("--rec-every", type=int, default=1000)
    ap.add_argument("--cal-seeds", type=int, nargs="+", default=[21, 27, 29],
                    help="seeds of the coarse runs that give the deficit and pick alpha")
    ap.add_argument("--eval-seeds", type=int, nargs="+", default=[33, 41, 47],
                    help="seeds of the held-out coarse runs, plain against closure")
    ap.add_argument("--out", default=None, help="write the JSON report here")
    ap.add_argument("--weights", default=None, help="save the trained closure (npz) here")
    a = ap.parse_args(argv)
    if a.synthetic_train:
        print(json.dumps(synthetic_train(a.synthetic_train, a.epochs, a.batch)), flush=True)
        return 0
    res, params, norm = experiment(tuple(a.dns_grid), tuple(a.coarse_grid), a.spinup, a.snapshots, a.snap_every,
                                   a.coarse_steps, a.epochs, a.batch, a.lr, cfl=a.cfl, alphas=tuple(a.alphas),
                                   filter_width=a.filter_width, rec_every=a.rec_every,
                                   coarse_snapshots=a.coarse_snapshots, Re=a.re, cal_seed=tuple(a.cal_seeds),
                                   eval_seed=tuple(a.eval_seeds), log=lambda s: print(s, flush=True))
    if a.weights and params is not None:
        np.savez(a.weights, params=params, norm=norm)
    s = json.dumps(res)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")
    print(json.dumps({k: v for k, v in res.items() if k not in ("coarse", "dns")} | {
        "alpha": res["coarse"]["alpha"], "chosen": res["coarse"]["chosen"],
        "errors": {n: r["errors_vs_dns"] for n, r in res["coarse"]["runs"].items()},
        "fallback": {n: r["report"] for n, r in res["coarse"]["runs"].items()}}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
