"""The reference's time loop (v1.9/codes/main_v1.9.f90:304-1049) on the GPU library.

    python -m compchan3dmpi_b200.run CASE_DIR --nP 64 48 65 [--maxstep N] [--rk 2]
                                     [--mesh cosine|tanh] [--beta B] [--variant NAME]

CASE_DIR is laid out as the reference expects around its ``codes/`` folder:
``CASE_DIR/param.dat`` is the fixed-column run deck (comdata.f90:31-68) and
paths in it are relative to ``CASE_DIR/codes``.  The input deck is
param.dat's input path for resOp = 1, or ``output/3D001.dat`` for resOp = 2
(main_v1.9.f90:211-262; one device holds the whole grid, so the per-rank file
is the rank-0 file).  Outputs, with the reference's cadences and formats:

  output/3D001.dat, output/3D001_.dat   every 1000 steps, alternating (:749-773)
  output/KE.dat, rhobulk.dat, Ubulk.dat, massflow.dat   every 10 steps (:799-906)
  output/tauWall.dat, moment1st.dat, moment2nd.dat, momentJoint.dat
                                        every istat steps (:957-1037)
  debug/3D001.dat                       on a blow-up, then exit status 1 (:709-743)

and a progress line every 10 steps (:1042-1047).  The diagnostics series use
the coordinates read from the deck (the reference overwrites x1, x2, x3 with
the file's F10.6 columns); the solver uses the analytic mesh.
"""
from __future__ import annotations

import argparse
import datetime
import sys
import time as _time
from pathlib import Path

import numpy as np

from .channel import BlowUpError, Channel
from .deck import fmt_e, read_3d_dat_native, read_param_dat, write_3d_dat_native
from .mesh import make_mesh, periodic_coords
from .stats import append_diag_series, append_series

PLANES = (5, 10, 70, 100, 125)   # main_v1.9.f90:10
OUTPUT_EVERY = 1000
DIAG_EVERY = 10


def _next_event(nstep, maxstep, istat):
    cands = [maxstep, (nstep // DIAG_EVERY + 1) * DIAG_EVERY, (nstep // OUTPUT_EVERY + 1) * OUTPUT_EVERY]
    if istat > 0:
        cands.append((nstep // istat + 1) * istat)
    return min(cands)


def write_debug_dump(path, var, x1, x2, x3, time, nstep):
    """debug/3D001.dat of a blow-up: records 3(1X,F7.4),7(1X,E12.5) (main_v1.9.f90:722-739)."""
    _, n3, n2, n1 = var.shape
    out = [f'TITLE ="{time:20.10f}{nstep:9d}"', ' Variables ="x","y","z","Rho","U","V","W","E","T","P"',
           f'ZONE k={n3:3d},j={n2:3d},i={n1:3d},DATAPACKING="POINT"']
    for k in range(n3):
        out.append("")
        for j in range(n2):
            out.append("")
            for i in range(n1):
                out.append(f" {x1[i]:7.4f} {x2[j]:7.4f} {x3[k]:7.4f}" +
                           "".join(" " + fmt_e(float(var[m, k, j, i]), 12, 5) for m in range(7)))
    Path(path).write_text("\n".join(out) + "\n")


def run(case_dir, nP, maxstep=None, rk=2, mesh="cosine", beta=2.0, variant=None, log=print):
    case = Path(case_dir)
    codes = case / "codes"
    out = case / "output"
    dbg = case / "debug"
    out.mkdir(parents=True, exist_ok=True)
    params, extra = read_param_dat(case / "param.dat", nP=tuple(nP), rk_scheme=rk)
    if extra["resOp"] == 2:
        deck = out / "3D001.dat"
    else:
        deck = (codes / extra["inputPath"]).resolve()
    x3, jac, inv = make_mesh(nP[2], mesh, beta)
    var, t0, n0, fx1, fx2, fx3 = read_3d_dat_native(deck, nP)
    ch = Channel(params, x3, jac, inv)
    ch.init_sol_v(var, n0, t0)
    if variant:
        from .wallbc import reference_variant
        bottom, top = reference_variant(variant, params)
        ch.set_wall_bc(0, bottom)
        ch.set_wall_bc(1, top)
    ch.diag_enable(PLANES, every=DIAG_EVERY, x3q=fx3, x2end=float(fx2[-1]), capacity=OUTPUT_EVERY // DIAG_EVERY + 1)
    maxstep = int(5e7) if maxstep is None else int(maxstep)   # comdata.f90:9
    x1 = periodic_coords(nP[0], params.Lx)
    x2 = periodic_coords(nP[1], params.Ly)
    nstep, tic = n0, _time.perf_counter()
    while nstep < maxstep:
        nxt = _next_event(nstep, maxstep, params.istat)
        try:
            ch.step(nxt - nstep)
        except BlowUpError as e:
            dbg.mkdir(parents=True, exist_ok=True)
            v = ch.download()
            i, j, k = e.ijk
            log(f"{e.nstep:10d}{0:4d}{i:4d}{j:4d}{k:4d}{v[0, k - 1, j - 1, i - 1]:8.4f}{v[5, k - 1, j - 1, i - 1]:8.4f}")
            write_debug_dump(dbg / "3D001.dat", v, fx1, fx2, fx3, ch.time, ch.nstep)
            append_diag_series(out, ch.diag_read())
            return 1
        nstep = nxt
        if params.istat > 0 and nstep % params.istat == 0:
            tau, s1, s2, c = ch.stats()
            append_series(out, ch.time, tau, s1, s2, c)
        if nstep % DIAG_EVERY == 0:
            append_diag_series(out, ch.diag_read())
            toc = _time.perf_counter()
            stamp = datetime.datetime.now().strftime("%d %b %Y  %H:%M:%S")
            log(f"{nstep:10d}{ch.time:10.5f} | CPU Time:{toc - tic:6.3f} sec for 10 iters | {stamp}")
            log("-" * 83)
            tic = toc
        if nstep % OUTPUT_EVERY == 0:
            name = "3D001.dat" if (nstep // OUTPUT_EVERY) % 2 == 0 else "3D001_.dat"
            write_3d_dat_native(out / name, ch.download(), x1, x2, x3, ch.time, nstep)
    append_diag_series(out, ch.diag_read())
    ch.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case_dir")
    ap.add_argument("--nP", type=int, nargs=3, required=True, help="nP1 nP2 nP3 (x, spanwise, wall-normal)")
    ap.add_argument("--maxstep", type=int, default=None)
    ap.add_argument("--rk", type=int, default=2, choices=(2, 3))
    ap.add_argument("--mesh", default="cosine", choices=("cosine", "tanh"))
    ap.add_argument("--beta", type=float, default=2.0)
    ap.add_argument("--variant", default=None, help="a wall-BC variant of the reference (wallbc.VARIANTS)")
    a = ap.parse_args(argv)
    return run(a.case_dir, a.nP, a.maxstep, a.rk, a.mesh, a.beta, a.variant)


if __name__ == "__main__":
    sys.exit(main())
