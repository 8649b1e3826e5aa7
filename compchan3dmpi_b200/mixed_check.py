"""Long-run check of the mixed FP32/FP64 path against the plain FP64 path.

Both paths start from the same seeded state and step in lockstep.  Every
``every`` steps the instantaneous fields are compared (relative L2 per
variable).  From step ``avg_from`` on, both contexts time-average their
statistics steps on the device (chan_time_avg, the avg_v1.7.f90 formulas);
at the end the mean profiles are put in wall units (stats.wall_units) and
compared: Cf, u+(y+), the rms profiles and the Reynolds shear stress <u'w'>.
The host wall time of each path's chan_step calls is reported beside them.

    python -m compchan3dmpi_b200.mixed_check --grid 256 192 193 --steps 20000 --avg-from 10000

The plain FP64 path is the reference here: it matches the restatement of the
reference's stage (main_v1.9.f90:313-704) to 1e-12 per step.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import Channel, cfl_dt, laminar_noise, mesh_tanh, production_params
from .stats import wall_units

VARS = ["rho", "u", "v", "w", "E", "T", "p"]


def _rel_max(a, b):
    """max_k |a - b| / max_k |b| (0 when b vanishes identically)."""
    d = float(np.max(np.abs(np.asarray(a) - np.asarray(b))))
    s = float(np.max(np.abs(np.asarray(b))))
    return d / s if s > 0 else d


def _rel_l2(a, b):
    n = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / n if n > 0 else float(np.linalg.norm(a - b))


def _profiles(ch, p, x3):
    av = ch.time_average()
    wu = wall_units(av["mean"], av["tau"], x3, p.Re)
    return av, wu


def compare(p, x3, jac, inv, var, steps, avg_from, every):
    """Run both paths; returns the comparison as a dict (see the module doc)."""
    if avg_from % every or steps % every or not 0 <= avg_from < steps:
        raise ValueError("steps and avg_from must be multiples of every, with 0 <= avg_from < steps")
    if every % p.istat:
        raise ValueError("every must be a multiple of istat")
    d = Channel(p.with_(mixed=False), x3, jac, inv)
    m = Channel(p.with_(mixed=True), x3, jac, inv)
    try:
        d.init_sol_v(var)
        m.init_sol_v(var)
        wall = {"fp64": 0.0, "mixed": 0.0}
        series = []
        done = 0
        while done < steps:
            if done == avg_from:
                d.time_avg_start()
                m.time_avg_start()
            for name, ch in (("fp64", d), ("mixed", m)):
                t0 = time.perf_counter()
                ch.step(every)
                wall[name] += time.perf_counter() - t0
            done += every
            fd, fm = d.download(), m.download()
            series.append({"step": done, "rel_l2": [_rel_l2(fm[v], fd[v]) for v in range(7)]})
        avd, wud = _profiles(d, p, x3)
        avm, wum = _profiles(m, p, x3)
    finally:
        d.close()
        m.close()
    uw = 3   # <u'w'>: CORR_PAIRS[3] = (u, w), w the wall-normal velocity
    prof = {
        "Cf": {"fp64": wud["Cf"], "mixed": wum["Cf"], "rel_err": abs(wum["Cf"] - wud["Cf"]) / abs(wud["Cf"])},
        "Re_tau": {"fp64": wud["Re_tau"], "mixed": wum["Re_tau"]},
        "uplus_rel_err": _rel_max(wum["uplus"], wud["uplus"]),
        "mean_rel_err": {VARS[v]: _rel_max(avm["mean"][v], avd["mean"][v]) for v in range(7)},
        "rms_rel_err": {VARS[v]: _rel_max(avm["rms"][v], avd["rms"][v]) for v in range(7)},
        "rms_peak": {VARS[v]: {"fp64": float(np.max(avd["rms"][v])), "mixed": float(np.max(avm["rms"][v]))}
                     for v in (1, 2, 3, 5)},
        "uw_rel_err": _rel_max(avm["covar"][uw], avd["covar"][uw]),
        "samples": avd["samples"],
        "window": [avd["t0"], avd["t1"]],
    }
    return {"steps": steps, "avg_from": avg_from, "every": every, "series": series, "profiles": prof,
            "wall_s": wall, "wall_ratio_fp64_over_mixed": wall["fp64"] / wall["mixed"]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 192, 193], metavar=("NP1", "NP2", "NP3"))
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--avg-from", type=int, default=10000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--beta", type=float, default=2.2)
    ap.add_argument("--cfl", type=float, default=0.6)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--out", default=None, help="also write the JSON here")
    a = ap.parse_args(argv)
    nP = tuple(a.grid)
    x3, jac, inv = mesh_tanh(nP[2], a.beta)
    p = production_params(nP)
    var = laminar_noise(p, x3, seed=a.seed)
    p = p.with_(dt=cfl_dt(var, p, jac, a.cfl))
    r = compare(p, x3, jac, inv, var, a.steps, a.avg_from, a.every)
    r["config"] = {"nP": list(nP), "beta": a.beta, "cfl": a.cfl, "dt": p.dt, "seed": a.seed,
                   "Ma": p.Mac, "Re": p.Re, "Pr": p.Pr, "istat": p.istat, "scheme": "SSP-RK3"}
    s = json.dumps(r)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")
    print(s, flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
