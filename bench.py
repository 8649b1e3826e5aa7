"""Benchmark: grid-point RK-stage updates/s of the plain FP64 channel DNS on B200.

Workload (one GPU): the production grid nP = (256, 192, 193) (x, spanwise,
wall-normal; 256 x 193 x 192 in the x / wall-normal / spanwise order), i.e.
9,486,336 points with 9,217,660 updated.  SSP-RK3 with dt from CFL 0.6,
tanh wall stretching beta = 2.2, Ma 1.5, Re 3000, Pr 0.72, mu ~ T^0.7,
isothermal walls, periodic x and z, lagged wall-shear forcing with
statistics every 10 steps.  It starts from the seeded laminar +-10 % start.

One "step" is one full RK3 time step (3 stages).  The metric counts
interior points x stages per second, summed over all GPUs (replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--mixed]

--mixed measures the mixed-precision path (float stage states and fluxes,
double accumulation) on the same workload and adds its error against the
FP64 path.

--ensemble measures the stratified parameter sweep (16 mixed-precision cases
of uneven grids) stepped as one ensemble with autotuned launch shapes -- every
member's kernels replayed from one graph per block of steps, and for
comparison one persistent kernel per block -- next to the same cases run one
at a time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "grid-point RK-stage updates/s"
UNIT = "stage-updates/s"
GRID = (256, 192, 193)
BETA = 2.2
CFL = 0.6
ISTAT = 10


def workload(nP=GRID):
    from compchan3dmpi_b200 import production_params, mesh_tanh, laminar_noise, cfl_dt
    x3, jac, inv = mesh_tanh(nP[2], BETA)
    p = production_params(nP, istat=ISTAT)
    var = laminar_noise(p, x3, seed=1234)
    p = p.with_(dt=cfl_dt(var, p, jac, CFL))
    return p, x3, jac, inv, var


def config_dict(p, n_gpus):
    n1, n2, n3 = p.nP
    kind = "mixed FP32/FP64 DNS" if getattr(p, "mixed", False) else "plain FP64 DNS"
    return {
        "workload": f"{kind} {n1}x{n3}x{n2} (x*wall-normal*spanwise), SSP-RK3 CFL {CFL}, "
                    f"tanh beta {BETA}",
        "nP": list(p.nP),
        "points": n1 * n2 * n3,
        "updated_points": p.n_interior,
        "stages_per_step": p.stages,
        "dt": p.dt,
        "Ma": p.Mac, "Re": p.Re, "Pr": p.Pr,
        "istat": p.istat,
        "parallelism": f"replicas x{n_gpus}",
        "l2_policy": "inputs larger than L2 (state 3 x 400 MB per GPU, L2 126 MB); no flush",
    }


# --------------------------------------------------------------- clocks
class Clocks:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML (the library behind nvidia-smi) is polled every few milliseconds from
    a thread, so that even a timed region of a few tens of milliseconds gets
    samples; nvidia-smi's own loop (200 ms at best, block-buffered when piped)
    is the fallback.  Only reads: no clock or other setting is changed."""
    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu: int, period_s: float = 0.004):
        self.gpu = gpu
        self.period = period_s
        self.sm, self.mx, self.bits = [], [], []
        self.nv = self.h = None
        self._stop = threading.Event()
        self.t = None
        self.source = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.gpu)
        try:
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip().isdigit()]
            idx = int(ids[self.gpu]) if self.gpu < len(ids) else self.gpu
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _sample(self):
        nv, h = self.nv, self.h
        self.sm.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
        self.mx.append(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        self.bits.append(int(nv.nvmlDeviceGetCurrentClocksEventReasons(h)))

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            self._stop.wait(self.period)

    def start(self):
        try:
            self.nv, self.h = self._handle()
            self._sample()
            self.source = "nvml"
        except Exception:
            self.nv = None
            return self._start_smi()
        self.t = threading.Thread(target=self._loop, daemon=True)
        self.t.start()

    def _start_smi(self):
        fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True, bufsize=1)
            self.source = "nvidia-smi"
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read_smi(self):
        for ln in self.proc.stdout:
            f = [x.strip() for x in ln.split(",")]
            try:
                sm, mx = float(f[0]), float(f[1])
            except (ValueError, IndexError):
                continue
            b = 0
            for (name, bit), v in zip(self.REASONS, f[2:6]):
                if v.lower() == "active":
                    b |= bit
            self.sm.append(sm); self.mx.append(mx); self.bits.append(b)

    def stop(self):
        self._stop.set()
        if self.source == "nvml":
            self.t.join(timeout=2)
            try:
                self._sample()   # one more sample at the end of the region
            except Exception:
                pass
        elif self.source == "nvidia-smi" and self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)
        if not self.sm:
            return None
        reasons = sorted({name for b in self.bits for name, bit in self.REASONS if b & bit})
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": max(self.mx), "reasons": reasons,
                "samples": len(self.sm), "source": self.source}


# --------------------------------------------------------------- peaks
def hbm_peak():
    f = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(f) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_traffic(p, n_int):
    """Per-launch DRAM bytes of the stage kernel: the per-point figure that
    profiles/stage_kernel_traffic.json records from an ncu capture
    (dram__bytes_read.sum + dram__bytes_write.sum over one RK3 step of a
    smaller grid, per updated point and launch) scaled by this workload's
    updated points.  Returns (bytes or None, provenance)."""
    f = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    key = "mixed" if getattr(p, "mixed", False) else "fp64"
    try:
        with open(f) as fh:
            rec = json.load(fh)[key]
        return float(rec["bytes_per_updated_point_per_launch"]) * n_int, rec.get("capture")
    except (OSError, KeyError, ValueError, TypeError):
        return None, None


def upload_bytes(nP):
    """Bytes chan_upload copies from the host: rho, u, v, w, E everywhere; T
    and p on the two wall planes and the four corner columns."""
    n1, n2, n3 = nP
    return 8 * (5 * n1 * n2 * n3 + 2 * (2 * n1 * n2 + 4 * n3))


# --------------------------------------------------------------- CPU
def cpu_baseline(nP=GRID, budget_s=20.0, threads=None):
    """The oracle (C restatement, OpenMP) on the host cores: one RK3 stage at
    a time on a wall-normal slab of the grid, sized to the time budget."""
    from oracle import oracle as O
    p, x3, jac, inv, var = workload(nP)
    O.build()
    nthreads = threads or os.cpu_count()
    o = O.Oracle(p, x3, jac, inv, threads=nthreads)
    o.upload(var)
    t0 = time.perf_counter()
    o.stage(1)
    t1 = time.perf_counter()
    per_stage = t1 - t0
    n = max(1, min(3, int(budget_s / max(per_stage, 1e-3))))
    t0 = time.perf_counter()
    for it in range(n):
        o.stage(2 if it % 2 == 0 else 3)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": p.n_interior * n / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"{n} RK3 stage(s) of the full {nP} grid after 1 untimed stage, "
                      f"C restatement with OpenMP ({O.num_threads()} threads); not the Fortran binary "
                      f"(no Fortran compiler on this image)"}


def mixed_error(p, x3, jac, inv, var, steps=200, every=50):
    """Relative L2 error per variable of the mixed-precision path against the
    plain FP64 path (which matches the oracle to 1e-12) from the same start."""
    import torch
    from compchan3dmpi_b200 import Channel
    a = Channel(p, x3, jac, inv)
    b = Channel(p.with_(mixed=False), x3, jac, inv)
    a.init_sol_v(var)
    b.init_sol_v(var)
    out = []
    for s in range(every, steps + 1, every):
        a.step(every)
        b.step(every)
        ga = torch.from_numpy(a.download()).cuda()
        gb = torch.from_numpy(b.download()).cuda()
        e = [float(torch.linalg.vector_norm(ga[m] - gb[m]) / torch.linalg.vector_norm(gb[m])) for m in range(7)]
        out.append({"step": s, "rel_l2": e})
        del ga, gb
    a.close()
    b.close()
    return {"reference": "plain FP64 path, same start", "per_step": out,
            "max_rel_l2": max(max(r["rel_l2"]) for r in out)}


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (the oracle port) on the
    host cores, same metric/config; rank 0 only."""
    from compchan3dmpi_b200.replicas import from_env
    r = from_env()
    if r.rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    nthreads = os.cpu_count()
    p, x3, jac, inv, var = workload(GRID)
    o = O.Oracle(p, x3, jac, inv, threads=nthreads)
    o.upload(var)
    # each bench step is one RK3 stage on the full grid; the budget caps the count
    t0 = time.perf_counter()
    o.stage(1)
    per = time.perf_counter() - t0
    budget = float(os.environ.get("CHAN_REF_BUDGET_S", "150"))
    K, W = args.steps, args.warmup
    total = K + W
    if total * per > budget:
        scale = budget / (total * per)
        K = max(3, int(K * scale))
        W = max(1, min(W, int(W * scale) or 1))
    for s in range(W):
        o.stage(2 + s % 2)
    t0 = time.perf_counter()
    for s in range(K):
        o.stage(2 + s % 2)
    dt = time.perf_counter() - t0
    o.close()
    val = p.n_interior * K / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": K, "warmup": W, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": dt / K * 1e3 * p.stages,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded laminar Poiseuille +-10%)", "config": config_dict(p, 1),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                         "sample": f"{K} timed RK3 stages (after {W} warm-up) of the full {GRID} grid, "
                                   "C restatement of the reference with OpenMP; the Fortran reference "
                                   "cannot be built (no Fortran compiler or MPI on this image)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU
def run_ours(args):
    import torch
    from compchan3dmpi_b200 import Channel
    from compchan3dmpi_b200 import replicas as R

    ranks = R.init("nccl" if args.gpus > 1 else "gloo")
    dev = ranks.local_rank
    torch.cuda.set_device(dev)
    p, x3, jac, inv, var = workload(tuple(args.grid))
    p = p.with_(device=dev, mixed=bool(args.mixed))
    n_int = p.n_interior
    K, W = args.steps, args.warmup

    ch = Channel(p, x3, jac, inv)
    stream = torch.cuda.ExternalStream(ch.stream_handle(), device=torch.device("cuda", dev))

    # ---------------- device-timed region (inputs resident in HBM)
    ch.init_sol_v(var)
    ch.step(W)
    ch.profile(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks = Clocks(dev)
    R.barrier(ranks)
    torch.cuda.synchronize()
    ch.sync()
    clocks.start()
    ev0.record(stream)
    ch.step_async(K)
    ev1.record(stream)
    st = ch.sync()
    torch.cuda.synchronize()
    ck = clocks.stop()
    R.barrier(ranks)
    ms = ev0.elapsed_time(ev1)
    prof_ms, prof_cnt = ch.profile_read()
    ch.profile(False)
    ms_max = R.max_over_ranks(ranks, ms)
    stage_ms = prof_ms[0] / max(int(prof_cnt[0]), 1)
    stage_ms_max = R.max_over_ranks(ranks, stage_ms)

    # ---------------- end to end through the C ABI with host buffers
    # the reference's driver loop: restart read (upload), steps in calls of
    # istat steps that each return the status (a blow-up freezes the state at
    # its step, so this reports what a per-step check would), statistics read
    # every istat steps, final field write
    host_in = torch.empty(var.shape, dtype=torch.float64).pin_memory()
    host_in.numpy()[...] = var
    host_out = torch.empty(var.shape, dtype=torch.float64).pin_memory()
    host_out.numpy().fill(0.0)   # the buffer's pages are touched once, as a reused output buffer's are
    n3 = p.nP[2]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    R.barrier(ranks)
    torch.cuda.synchronize()
    e0.record(stream)
    ch.init_sol_v(host_in.numpy())
    nstats = ncalls = 0
    done = 0
    while done < K:
        chunk = min(p.istat - done % p.istat if p.istat > 0 else K, K - done)
        ch.step(chunk)
        ncalls += 1
        done += chunk
        if p.istat > 0 and done % p.istat == 0:
            tau, s1, s2, cc = ch.stats()
            nstats += 1
    ch.download(out=host_out.numpy())
    e1.record(stream)
    torch.cuda.synchronize()
    R.barrier(ranks)
    e2e_ms = R.max_over_ranks(ranks, e0.elapsed_time(e1))
    n_pts = p.nP[0] * p.nP[1] * p.nP[2]
    h2d = upload_bytes(p.nP)
    d2h = 7 * n_pts * 8 + ncalls * 48 + nstats * (23 * n3 + 2) * 8

    status_ok = (st == 0)
    ch.close()

    if ranks.is_root:
        stages = p.stages
        value = ranks.world * n_int * stages * K / (ms_max / 1e3)
        e2e_val = ranks.world * n_int * stages * K / (e2e_ms / 1e3)
        if p.mixed:
            # stage 1 reads the double state and writes float; middle stages read float and
            # the double base and write float; the last writes the double state
            bpp = ((40 + 20) + (20 + 40 + 20) * (stages - 2) + (20 + 40 + 40)) / stages
        else:
            bpp = (80 + 120 * (stages - 1)) / stages   # algorithmic bytes per updated point per stage launch
        achieved = n_int * bpp / (stage_ms_max / 1e3) / 1e9
        peak, peak_kind = hbm_peak()
        traffic, traffic_src = measured_traffic(p, n_int)
        # stage + wall-BC kernels per stage, plus the two statistics passes on their cadence
        launches = K * 2 * stages + 2 * sum(1 for s in range(W + 1, W + K + 1) if s % p.istat == 0)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if p.mixed else "f64", "data": "synthetic (seeded laminar Poiseuille +-10%)",
            "config": config_dict(p, ranks.world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                         "kernel": "k_stage<32,8>", "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_launch": n_int * bpp,
                         "stage_kernel_ms": stage_ms_max,
                         "stage_share_of_step": prof_ms[0] / max(sum(prof_ms), 1e-12)},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
                    "calls": "chan_upload(var) + K/istat x chan_step(istat) + chan_stats every istat + chan_download(var)"},
            "gpu_launches": int(launches),
            "status_ok": status_ok,
        }
        if ck:
            line["clocks"] = ck
        if p.mixed:
            line["mixed_error"] = mixed_error(p, x3, jac, inv, var)
        if ranks.world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(tuple(args.grid), budget_s=args.cpu_budget)
        print(json.dumps(line), flush=True)
    R.finalize(ranks)
    return 0


def run_ensemble(args):
    """--ensemble: the stratified parameter sweep (compchan3dmpi_b200.ensemble:
    16 mixed-precision cases of uneven grids, per-case Ma, Re, Ri, dT) as one
    ensemble -- graph replays of all members concurrently, launch shapes from
    the autotuner -- against the same cases run one at a time."""
    import torch
    from compchan3dmpi_b200 import replicas as R
    from compchan3dmpi_b200.ensemble import Ensemble, open_case, sweep_cases

    ranks = R.init("nccl" if args.gpus > 1 else "gloo")
    dev = ranks.local_rank
    torch.cuda.set_device(dev)
    cases = sweep_cases(args.members)
    for c in cases:
        c.params = c.params.with_(device=dev)
    L = ISTAT
    K = max(L, (args.steps + L - 1) // L * L)   # whole graph blocks
    W = max(args.warmup, 3)
    per_step = sum(c.params.n_interior * c.params.stages for c in cases)

    # one at a time: each case alone with its default launch shape
    solo_ms = 0.0
    for c in cases:
        ch = open_case(c)
        ch.step(W)
        stream = torch.cuda.ExternalStream(ch.stream_handle(), device=torch.device("cuda", dev))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ch.sync()
        ev0.record(stream)
        ch.step_async(K)
        ev1.record(stream)
        ch.sync()
        torch.cuda.synchronize()
        solo_ms += ev0.elapsed_time(ev1)
        ch.close()

    chans = [open_case(c) for c in cases]
    e = Ensemble(chans)
    clocks = Clocks(dev)
    e.step(W)
    R.barrier(ranks)
    clocks.start()
    st0 = e.step(K)
    untuned_ms = e.last_replay_ms()
    tune_ms = e.tune(reps=3)
    e.step(W)
    st1 = e.step(K)
    tuned_ms = e.last_replay_ms()
    mode, fallback = e.mode_in_use()
    # the same tuned shapes in the other mode: one persistent kernel per block
    e.set_mode("persistent")
    e.step(W)
    stg = e.step(K)
    pers_ms = e.last_replay_ms()
    pmode, pfallback = e.mode_in_use()
    e.set_mode("graph")
    ck = clocks.stop()
    shapes = e.launch_shapes()
    replays, captures = e.counters()

    # end to end: upload every member from pinned host memory, K steps, download every member
    host_in = [torch.empty(c.var.shape, dtype=torch.float64).pin_memory() for c in cases]
    host_out = [torch.empty(c.var.shape, dtype=torch.float64).pin_memory() for c in cases]
    for h, o, c in zip(host_in, host_out, cases):
        h.numpy()[...] = c.var
        o.numpy().fill(0.0)   # pages touched once, as a reused output buffer's are
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for ch, h in zip(chans, host_in):
        ch.init_sol_v(h.numpy())
    st2 = e.step(K)
    for ch, h in zip(chans, host_out):
        ch.download(out=h.numpy())
    e2e_s = time.perf_counter() - t0
    e.close()
    for ch in chans:
        ch.close()
    R.barrier(ranks)
    tuned_max = R.max_over_ranks(ranks, tuned_ms)
    solo_max = R.max_over_ranks(ranks, solo_ms)
    e2e_max = R.max_over_ranks(ranks, e2e_s)
    if ranks.is_root:
        value = ranks.world * per_step * K / (tuned_max / 1e3)
        solo = ranks.world * per_step * K / (solo_max / 1e3)
        bpp = 240.0 / 3.0   # mixed RK3: algorithmic bytes per updated point per stage
        achieved = per_step * bpp * K / (tuned_max / 1e3) / 1e9
        peak, peak_kind = hbm_peak()
        n_pts = sum(int(np.prod(c.params.nP)) for c in cases)
        launches = K * sum(1 + 2 * c.params.stages for c in cases) + (K // L) * 2 * len(cases)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": K, "warmup": W,
            "ms_per_step": tuned_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded stratified laminar starts, +-10% noise)",
            "config": {
                "workload": f"stratified sweep ensemble: {len(cases)} mixed-precision SSP-RK3 cases, "
                            f"grids nP (64,64,65)..(160,128,129), CFL 0.6, tanh beta 2.2",
                "members": [{"nP": list(c.params.nP), "Ma": c.params.Mac, "Re": c.params.Re, "Ri": c.Ri,
                             "dT": c.dT} for c in cases],
                "updated_points": per_step // 3, "istat": ISTAT, "graph_block_steps": L,
                "parallelism": f"replicas x{ranks.world}",
                "l2_policy": "members' states together larger than L2 (126 MB); no flush"},
            "one_at_a_time": {"value": solo, "ms_per_step": solo_max / K,
                              "how": "each case alone, default launch shape, CUDA events on its stream"},
            "speedup_vs_one_at_a_time": value / solo,
            "mode": mode,
            "persistent_mode": {"value": per_step * K / (pers_ms / 1e3), "ms_per_step": pers_ms / K,
                                "mode_in_use": pmode, "fallback_reason": pfallback,
                                "how": "same members and shapes, one persistent kernel per block of steps"},
            "untuned": {"value": per_step * K / (untuned_ms / 1e3), "ms_per_step": untuned_ms / K},
            "autotuner": {"trial_ms": tune_ms, "shapes": [list(x) for x in shapes]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "every member's k_stage (whole ensemble step)",
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "e2e": {"value": ranks.world * per_step * K / e2e_max, "unit": UNIT,
                    "h2d_bytes_per_step": sum(upload_bytes(c.params.nP) for c in cases) / K,
                    "d2h_bytes_per_step": 7 * 8 * n_pts / K,
                    "calls": "chan_upload of every member + chan_ensemble_step(K) + chan_download of every "
                             "member (host wall clock around the synchronous calls)"},
            "gpu_launches": int(launches),
            "graph": {"replays": replays, "captures": captures},
            "status_ok": all(x == 0 for x in st0 + st1 + st2 + stg),
        }
        if ck:
            line["clocks"] = ck
        print(json.dumps(line), flush=True)
    R.finalize(ranks)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, nargs=3, default=list(GRID))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--mixed", action="store_true",
                    help="mixed precision: float stage storage and fluxes, double accumulation")
    ap.add_argument("--ensemble", action="store_true",
                    help="the stratified parameter sweep as one graph-replayed ensemble vs one case at a time")
    ap.add_argument("--members", type=int, default=16, help="ensemble size for --ensemble")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.ensemble:
        return run_ensemble(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
