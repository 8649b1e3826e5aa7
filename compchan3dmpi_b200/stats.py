"""Time-averaged statistics and wall units.

Reference: the solver appends plane moments every istat steps
(v1.9/codes/main_v1.9.f90:993-1061 -> moment1st.dat, moment2nd.dat,
momentJoint.dat; :929-987 -> tauWall.dat).  The offline program
v1.9/codes/avg_v1.7.f90 time-averages them (lines 239-274):

    mean  = <stat1Spc>                          mean.dat  (x3, 7 columns, F22.18)
    rms   = sqrt(<stat2Spc> - mean**2)          rms.dat
    covar = <corrSpc> - products of the means   corr.dat  (x3, 9 columns, F10.5)
            in the order rho*w, rho*T, u*v, u*w, v*w, v*T, T*w, p*w, p*T

The GPU library keeps the running sums on the device (chan_time_avg); this
module applies the formulas above and adds the derived wall quantities the
validation plots use (u+(y+), Cf).  Layouts follow chan_stats: [p][k].
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

# pairs of corrSpc (1-based var indices rho,u,v,w,E,T,p), main_v1.9.f90:1014-1022
CORR_PAIRS = [(1, 4), (1, 6), (2, 3), (2, 4), (3, 4), (3, 6), (6, 4), (7, 4), (7, 6)]


def time_average(sum1, sum2, sumc, sumtau, n):
    """(mean[7,n3], rms[7,n3], covar[9,n3], tau_mean[2]) from running sums over n samples."""
    if n <= 0:
        raise ValueError("no statistics samples accumulated")
    mean = np.asarray(sum1) / n
    stat2 = np.asarray(sum2) / n
    rms = np.sqrt(np.maximum(stat2 - mean ** 2, 0.0))
    corr = np.asarray(sumc) / n
    covar = np.empty_like(corr)
    for c, (a, b) in enumerate(CORR_PAIRS):
        covar[c] = corr[c] - mean[a - 1] * mean[b - 1]
    return mean, rms, covar, np.asarray(sumtau) / n


def average_snapshots(snaps):
    """Same result from a list of (stat1, stat2, corr, tau2) snapshots."""
    n = len(snaps)
    s1 = sum(np.asarray(s[0]) for s in snaps)
    s2 = sum(np.asarray(s[1]) for s in snaps)
    sc = sum(np.asarray(s[2]) for s in snaps)
    st = sum(np.asarray(s[3]) for s in snaps)
    return time_average(s1, s2, sc, st, n)


def _trapz(y, x):
    y = np.asarray(y, dtype=np.float64); x = np.asarray(x, dtype=np.float64)
    return float(np.sum(0.5 * (y[1:] + y[:-1]) * np.diff(x)))


def wall_units(mean, tau_mean, x3, Re, Tw=(1.0, 1.0)):
    """Wall-scaled quantities of the mean profiles.

    tau_w   = (tauL - tauU)/2 (both walls; tauU is negative by orientation)
    rho_w   = mean density of the two wall planes; mu_w = Tw**0.7
    u_tau   = sqrt(tau_w / rho_w);  Re_tau = rho_w u_tau h Re / mu_w with h = 1
    rho_b, U_b = wall-normal averages of the mean density and velocity
                 (the area averages the solver's rhobulk/Ubulk series use)
    Cf      = 2 tau_w / (rho_b U_b^2)
    y+      = rho_w u_tau d Re / mu_w, d the distance to the nearer wall
    u+      = mean u / u_tau
    """
    x3 = np.asarray(x3, dtype=np.float64)
    tau_w = 0.5 * (tau_mean[0] - tau_mean[1])
    rho_w = 0.5 * (mean[0][0] + mean[0][-1])
    mu_w = 0.5 * (Tw[0] ** 0.7 + Tw[1] ** 0.7)
    u_tau = math.sqrt(max(tau_w, 0.0) / rho_w)
    H = x3[-1] - x3[0]
    rho_b = _trapz(mean[0], x3) / H
    U_b = _trapz(mean[1], x3) / H
    Cf = 2.0 * tau_w / (rho_b * U_b * U_b)
    d = np.minimum(x3 - x3[0], x3[-1] - x3)
    yplus = rho_w * u_tau * d * Re / mu_w
    uplus = mean[1] / u_tau if u_tau > 0 else np.full_like(x3, np.nan)
    return {"tau_w": tau_w, "rho_w": rho_w, "mu_w": mu_w, "u_tau": u_tau,
            "Re_tau": rho_w * u_tau * (H / 2.0) * Re / mu_w, "rho_b": rho_b, "U_b": U_b, "Cf": Cf,
            "yplus": yplus, "uplus": uplus}


# ------------------------------------------------------------------ writers
def _f(x, w, d):
    return f"{x:{w}.{d}f}"


def moment_line(time, stat, ncol):
    """One line of moment1st/2nd.dat (1X,F15.7 time then ncol (1X,F15.7) per k)."""
    n3 = stat.shape[1]
    parts = [" " + _f(time, 15, 7)]
    for k in range(n3):
        parts.append("".join(" " + _f(stat[c, k], 15, 7) for c in range(ncol)))
    return "".join(parts)


def append_series(outdir, time, tau2, stat1, stat2, corr):
    """Append one statistics step to tauWall.dat, moment1st.dat, moment2nd.dat
    and momentJoint.dat in the reference's formats (main_v1.9.f90:980-1058)."""
    d = Path(outdir)
    d.mkdir(parents=True, exist_ok=True)
    with open(d / "tauWall.dat", "a") as f:
        f.write(" " + _f(time, 15, 7) + " " + _f(tau2[0], 15, 7) + " " + _f(tau2[1], 15, 7) + "\n")
    with open(d / "moment1st.dat", "a") as f:
        f.write(moment_line(time, stat1, 7) + "\n")
    with open(d / "moment2nd.dat", "a") as f:
        f.write(moment_line(time, stat2, 7) + "\n")
    with open(d / "momentJoint.dat", "a") as f:
        f.write(moment_line(time, corr, 9) + "\n")


def write_profiles(outdir, x3, mean, rms, covar):
    """mean.dat, rms.dat (8(1X,F22.18)) and corr.dat (10(1X,F10.5)) as avg_v1.7.f90:241-283."""
    d = Path(outdir)
    d.mkdir(parents=True, exist_ok=True)
    with open(d / "mean.dat", "w") as f:
        for k in range(len(x3)):
            f.write("".join(" " + _f(v, 22, 18) for v in [x3[k], *mean[:, k]]) + "\n")
    with open(d / "rms.dat", "w") as f:
        for k in range(len(x3)):
            f.write("".join(" " + _f(v, 22, 18) for v in [x3[k], *rms[:, k]]) + "\n")
    with open(d / "corr.dat", "w") as f:
        for k in range(len(x3)):
            f.write("".join(" " + _f(v, 10, 5) for v in [x3[k], *covar[:, k]]) + "\n")


def read_series(path, ncol, n3):
    """Parse moment*.dat lines back into (times[n], values[n, ncol, n3])."""
    times, vals = [], []
    for ln in Path(path).read_text().splitlines():
        if not ln.strip():
            continue
        nums = [float(ln[1 + 16 * c: 16 + 16 * c]) for c in range(1 + ncol * n3)]
        times.append(nums[0])
        vals.append(np.array(nums[1:]).reshape(n3, ncol).T)
    return np.array(times), np.array(vals)


# ------------------------------------------------------------ diagnostics series
def _f15_7(x):
    return f"{float(x):15.7f}"


def append_diag_series(outdir, d):
    """Append a diag_read() result to KE.dat (format 2(1X,F15.7)) and
    rhobulk.dat, Ubulk.dat, massflow.dat (6(1X,F15.7)): time then one column
    per plane (main_v1.9.f90:813-906)."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    with open(out / "KE.dat", "a") as f:
        for t, ke in zip(d["time"], d["ke"]):
            f.write(" " + _f15_7(t) + " " + _f15_7(ke) + "\n")
    for name, key in (("rhobulk.dat", "rho_b"), ("Ubulk.dat", "u_b"), ("massflow.dat", "rhou_b")):
        with open(out / name, "a") as f:
            for t, row in zip(d["time"], d[key]):
                f.write(" " + _f15_7(t) + "".join(" " + _f15_7(v) for v in row) + "\n")


def write_q_invariant(path, x1, x2, x3, Q):
    """qInvariant.dat as qInvariant.f90:84-95 writes it: list-directed header
    lines, then x,y,z,Q records 3(1X,F10.6),1X,E22.15 with i fastest."""
    from .deck import fmt_e22_15
    n3, n2, n1 = Q.shape
    lines = [' TITLE ="qInvariant"', ' Variables = "x","y","z","Q"',
             f'ZONE i={n1:3d},j={n2:3d},k={n3:3d},DATAPACKING="POINT"']
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                lines.append(f" {x1[i]:10.6f} {x2[j]:10.6f} {x3[k]:10.6f} " + fmt_e22_15(float(Q[k, j, i])))
    Path(path).write_text("\n".join(lines) + "\n")
