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


def experiment(dns_grid=(256, 192, 193), coarse_grid=(64, 64, 65), spinup=60000, snapshots=100, snap_every=200,
               epochs=20, batch=65536, lr=1e-3, cfl=0.6, beta=2.2, seed=7, fp64_probe=400, filter_width=4,
               log=print):
    t_all = time.time()
    kst = (dns_grid[2] - 1) // (coarse_grid[2] - 1)
    x3d, jacd, invd = mesh_tanh(dns_grid[2], beta)
    pd = production_params(dns_grid).with_(mixed=True)
    var0 = smooth_start(pd, x3d, seed=seed)
    pd = pd.with_(dt=cfl_dt(var0, pd, jacd, cfl))
    dns = Channel(pd, x3d, jacd, invd)
    dns.init_sol_v(var0)
    dns.step(spinup)
    log(json.dumps({"phase": "dns spin-up", "steps": spinup, "t": dns.time}))
    # the coarse start: the DNS state at the start of the sampling window
    x3c, jacc, invc = mesh_tanh(coarse_grid[2], beta)
    pc = production_params(coarse_grid)
    varc = coarsen(dns.download(), pd, pc, kst)
    pc = pc.with_(dt=cfl_dt(varc, pc, jacc, cfl))
    window = snapshots * snap_every * pd.dt
    # DNS window: snapshots into the dataset, statistics time-averaged
    cap = snapshots * ((dns_grid[0] - 3) // 4 + 1) * ((dns_grid[1] - 3) // 3 + 1) * ((dns_grid[2] - 1) // kst - 1)
    cl = Closure(capacity=cap)
    dns.time_avg_start()
    t0 = time.time()
    for s in range(snapshots):
        dns.step(snap_every)
        cl.sample(dns, strides=(4, 3, kst), width=filter_width)
    dns_wall = time.time() - t0
    avg_d = dns.time_average()
    dns_stats = _profiles(avg_d, x3d, pd.Re)
    # plain FP64 DNS on the same GPU: time a few hundred steps from the window's end state
    f64 = Channel(pd.with_(mixed=False), x3d, jacd, invd)
    f64.init_sol_v(dns.download())
    f64.step(20)
    t0 = time.time()
    f64.step(fp64_probe)
    fp64_ms = (time.time() - t0) / fp64_probe * 1e3
    f64.close()
    # the DNS statistics at the coarse grid's wall-normal points
    dns_c = {k: (np.asarray(v)[::kst].tolist() if isinstance(v, list) else v) for k, v in dns_stats.items()}
    dns.close()
    log(json.dumps({"phase": "dns window", "samples": cl.count, "window_t": window, "wall_s": dns_wall,
                    "Cf": dns_stats["Cf"], "Re_tau": dns_stats["Re_tau"]}))
    # training
    cl.fit_normalization()
    cl.init(seed=seed)
    t0 = time.time()
    losses = cl.train(epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.time() - t0
    log(json.dumps({"phase": "training", "epochs": epochs, "loss_first": float(losses[0]),
                    "loss_last": float(losses[-1]), "wall_s": train_s}))
    # coarse runs over the same window, with and without the closure
    nc = int(math.ceil(window / pc.dt))
    runs = {}
    for name, use in (("closure", True), ("plain", False)):
        ch = Channel(pc.with_(dt=window / nc), x3c, jacc, invc)
        ch.init_sol_v(varc)
        ch.time_avg_start()
        t0 = time.time()
        if use:
            rep = run_with_fallback(ch, cl, nc, check_every=200)
        else:
            try:
                ch.step(nc)
                rep = {"fallback_step": None, "reason": None}
            except BlowUpError as e:
                rep = {"fallback_step": None, "reason": f"plain coarse run blew up: {e}"}
        wall = time.time() - t0
        st = _profiles(ch.time_average(), x3c, pc.Re) if rep["reason"] is None or use else None
        runs[name] = {"steps": nc, "dt": window / nc, "wall_s": wall, "report": rep,
                      "stats": st, "errors_vs_dns": _errors(st, dns_c) if st else None}
        ch.close()
        log(json.dumps({"phase": f"coarse {name}", "steps": nc, "wall_s": wall, "report": rep,
                        "errors": runs[name]["errors_vs_dns"]}))
    fp64_window_s = fp64_ms * 1e-3 * snapshots * snap_every
    out = {"dns": {"nP": list(dns_grid), "dt": pd.dt, "window_steps": snapshots * snap_every, "window_t": window,
                   "wall_s": dns_wall, "stats": dns_c, "precision": "mixed FP32/FP64",
                   "fp64_ms_per_step": fp64_ms, "fp64_window_s": fp64_window_s},
           "coarse": {"nP": list(coarse_grid), "runs": runs},
           "training": {"samples": cl.count, "epochs": epochs, "batch": batch, "lr": lr, "filter_width": filter_width,
                        "losses": [float(x) for x in losses], "wall_s": train_s},
           "wall_time_ratio_dns_over_closure": dns_wall / runs["closure"]["wall_s"],
           "wall_time_ratio_fp64_dns_over_closure": fp64_window_s / runs["closure"]["wall_s"],
           "total_s": time.time() - t_all}
    params, norm = cl.params, cl.norm
    cl.close()
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
    ap.add_argument("--spinup", type=int, default=60000)
    ap.add_argument("--snapshots", type=int, default=100)
    ap.add_argument("--snap-every", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--dns-grid", type=int, nargs=3, default=[256, 192, 193])
    ap.add_argument("--coarse-grid", type=int, nargs=3, default=[64, 64, 65])
    ap.add_argument("--filter-width", type=int, default=4,
                    help="box-filter width (even, in DNS points) in x and spanwise for the training targets")
    ap.add_argument("--out", default=None, help="write the JSON report here")
    ap.add_argument("--weights", default=None, help="save the trained closure (npz) here")
    a = ap.parse_args(argv)
    if a.synthetic_train:
        print(json.dumps(synthetic_train(a.synthetic_train, a.epochs, a.batch)), flush=True)
        return 0
    res, params, norm = experiment(tuple(a.dns_grid), tuple(a.coarse_grid), a.spinup, a.snapshots, a.snap_every,
                                   a.epochs, a.batch, a.lr, filter_width=a.filter_width,
                                   log=lambda s: print(s, flush=True))
    if a.weights:
        np.savez(a.weights, params=params, norm=norm)
    s = json.dumps(res)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")
    print(json.dumps({k: v for k, v in res.items() if k != "coarse"} | {
        "errors": {n: r["errors_vs_dns"] for n, r in res["coarse"]["runs"].items()},
        "fallback": {n: r["report"] for n, r in res["coarse"]["runs"].items()}}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
