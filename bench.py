#!/usr/bin/env python
"""Throughput of the B200 Godunov step on the 3-D 256^3 ideal-MHD blast.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mhd3d_blast|ensemble|serve|rmhd]

Workload (one "step" = one full RK2 step of the grid): 3-D ideal MHD, 256^3
periodic on [0,1]^3, PLM with the MC limiter, HLLD, UCT_HLLD constrained
transport, RK2, CFL 0.4, gamma 5/3; seeded blast initial condition (rho=1,
p=0.1, p=10 inside r<0.1, uniform B at beta 0.1 along a seeded direction,
divergence-free random velocity at rms 0.1).  Plain FP64 form; the mixed
FP32-flux form is timed beside it.  Inputs are far larger than L2 (the
state alone is ~2.5 GB), so no L2 flush is needed between steps.

Multi-GPU: replicas only (one independent grid per rank, no data-path
collective); value = zone updates of all ranks / max-over-ranks time.

The default line also carries the CPU baseline (the reference serial build,
one thread, on this same 256^3 grid: one timed step after one untimed, run
beside the GPU measurements), the end-to-end rate through the C ABI with
host buffers in the drop-in driver's loop, and three short legs of the
other workloads: the batched ensemble (all 512 grids, K steps), the serving
loop (64 requests at 8 requests/s: p50/p99 latency and Mzone-updates/s) and
the 3-D RMHD 192^3 grid (FP64 and mixed, min(K, 10) steps).

``--impl reference`` times the reference gPLUTO serial build (compiled from
the reference sources into oracle/_ref by __graft_entry__.build()) on this
same workload, the 256^3 blast: as many concurrent single-thread processes
as the host's cores and memory hold (at most 16; ~18 GB each), each one
untimed and one timed RK2 step of the full grid -- a bounded sample, since
one step takes the reference 40-60 s on one core.

``--workload ensemble`` (default 200 steps): 512 independent 2-D ideal-MHD
grids (sides log-uniform 64..512, square and 2:1, half FP64 / half mixed,
per-grid dt), advanced by the batched step -- per RK stage one persistent
sweep launch and one persistent EMF/finish launch over all grids, the steps
replayed from a CUDA graph -- with tile
shapes picked per size bin by gpluto_dev_b200.autotune on a sample of the
grids first.  value = zone updates of all grids / device time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mzone-updates/s"
WORKLOAD = "3d_ideal_mhd_blast_256^3"
SCHEME = dict(limiter="mc", riemann="hlld", ct_emf="uct_hlld", cfl=0.4, cfl_max_var=1.1)
FIRST_DT = 1e-4
N = 256
# algorithmic bytes per zone-update of the RK2 step (state read/written once
# per stage: 5 x 8 B x (NVAR + n_face)) for 3-D ideal MHD
ALG_BYTES_ZONE = 440
# compulsory bytes per cell of each kernel of the FP64 3-D MHD step (arrays
# it must read and write once, 8 B each), indexed by (kernel, stage):
#   sweep  V(8) + Bs_n(1) -> dU_dir(5) + C_dir(1) + UCT(6)            21 x 8
#   emf    UCT(18) + Bs(3) -> Ee(3)                                    24 x 8
#   finish stage 1: dU(15) + C(3) + U0(5) + Ee(3) + Bs(3)
#          -> Bs'(3) + U(5: the field components of the intermediate state
#          are never read, so not stored) + V(8)                        45 x 8
#   finish stage 2: dU(15) + U0(5) + Uc(5) + Ee(3) + Bs(3) + Bs0(3)
#          -> Bs'(3) + U(8) + V(8)                                      53 x 8
KERNEL_BYTES = {
    ("sweep_x", 1): 168, ("sweep_x", 2): 168,
    ("sweep_y", 1): 168, ("sweep_y", 2): 168,
    ("sweep_z", 1): 168, ("sweep_z", 2): 168,
    ("emf", 1): 192, ("emf", 2): 192,
    ("finish", 1): 360, ("finish", 2): 424,
}
# the same for the mixed form, whose flux differences, inverse-dt terms, UCT
# data and edge EMFs are 4-byte floats (state, faces and V stay 8 bytes)
KERNEL_BYTES_MIXED = {
    ("sweep_x", 1): 120, ("sweep_x", 2): 120,
    ("sweep_y", 1): 120, ("sweep_y", 2): 120,
    ("sweep_z", 1): 120, ("sweep_z", 2): 120,
    ("emf", 1): 108, ("emf", 2): 108,
    ("finish", 1): 300, ("finish", 2): 352,
}
REF_BINARY = os.path.join(ROOT, "oracle", "_ref", "mhd3d_mc_lim_hlld_uct_hlld", "pluto")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# reference (CPU) timing: the reference serial build, one process per core
# --------------------------------------------------------------------------
def _ref_available() -> bool:
    return os.path.exists(REF_BINARY)


REF_RSS_256 = 18 << 30     # resident bytes of one reference process at 256^3 (measured)


def _mem_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


class ReferenceRun:
    """`nproc` concurrent reference processes (serial build, one thread
    each), every one advancing the bench's own 256^3 grid: `nwarm` untimed
    steps, then `ntimed` timed ones (the wall stamps the problem file logs
    before every step).  Started at construction, collected by result()."""

    def __init__(self, st, nproc: int, nwarm: int, ntimed: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
        from gpluto_dev_b200 import ics
        import build_ref as br
        self.br, self.nwarm, self.ntimed, self.ncell = br, nwarm, ntimed, st.ncells
        total = nwarm + ntimed
        nx, ny, nz = st.shape
        cfg = br.RefConfig(name="bench", physics="MHD", ndim=3, n=(nx, ny, nz),
                           limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                           first_dt=FIRST_DT)
        self.tmp = tempfile.TemporaryDirectory()
        icp = os.path.join(self.tmp.name, "ic.bin")
        ics.write_ic(icp, st)
        self.procs = []
        for r in range(nproc):
            d = os.path.join(self.tmp.name, f"p{r}")
            os.makedirs(d)
            open(os.path.join(d, "pluto.ini"), "w").write(cfg.ini())
            env = dict(os.environ, GPLUTO_FTZ_DAZ="0", GP_IC_FILE=icp,
                       GP_DUMP_STEP=str(total), GP_DUMP_FILE=os.path.join(d, "out.dump"))
            self.procs.append((d, subprocess.Popen(
                [REF_BINARY, "-no-write", "-maxsteps", str(total)], cwd=d, env=env,
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)))

    def result(self):
        """(Mzone-updates/s summed over processes, mean s/step)."""
        per = []
        for d, p in self.procs:
            p.wait()
            w = self.br.read_dump(os.path.join(d, "out.dump")).wall
            per.append((w[self.nwarm + self.ntimed] - w[self.nwarm]) / self.ntimed)
        self.tmp.cleanup()
        return sum(self.ncell / t for t in per) / 1e6, statistics.mean(per)


def reference_processes(cap: int) -> int:
    """Concurrent 256^3 reference processes the host can hold: one per core,
    at most `cap`, and no more than 80% of the available memory allows."""
    cores = os.cpu_count() or 1
    by_mem = max(1, int(0.8 * _mem_available() // REF_RSS_256))
    return max(1, min(cores, by_mem, cap))


def _oracle_rate(n, nwarm, ntimed):
    """The oracle port on one n^3 blast grid, one thread (when the reference
    build is absent)."""
    t = _oracle_worker((n, nwarm + ntimed, nwarm, 0))
    return n ** 3 / t / 1e6, t


def _oracle_worker(args):
    n, total, nwarm, r = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from gpluto_dev_b200 import ics
    o = orc.Oracle(ics.mhd3d_blast(n=(n, n, n), seed=1 + r), limiter="mc", solver="hlld",
                   ct="uct_hlld")
    dt = FIRST_DT
    for _ in range(nwarm):
        inv, _ = o.step(dt)
        dt = orc.lib().orc_next_dt(inv, 0.4, 1.1, dt)
    t0 = time.perf_counter()
    for _ in range(total - nwarm):
        inv, _ = o.step(dt)
        dt = orc.lib().orc_next_dt(inv, 0.4, 1.1, dt)
    return (time.perf_counter() - t0) / (total - nwarm)


def config_block(n=N):
    return {"workload": f"3d_ideal_mhd_blast_{n}^3", "grid": [n, n, n], "physics": "ideal MHD",
            "scheme": "PLM-MC + HLLD + UCT_HLLD + RK2, CFL 0.4, gamma 5/3",
            "boundary": "periodic", "ic": "seeded blast (seed 1 + rank)",
            "l2": "inputs larger than L2 (state ~2.5 GB), no flush"}


def impl_reference(args):
    """The reference serial build on the bench's own workload (the seeded
    256^3 blast, the same scheme): as many concurrent single-thread
    processes as the host's cores and memory hold (at most 16), each one
    untimed step then one timed step -- a bounded sample, since one step of
    this grid takes the reference about 40-60 s on one core."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from gpluto_dev_b200 import ics
    n = args.n
    st = ics.mhd3d_blast(n=(n, n, n), seed=1)
    if _ref_available():
        nproc = reference_processes(16)
        v, sps = ReferenceRun(st, nproc, 1, 1).result()
        kind, cores = "reference", nproc
        sample = (f"{nproc} concurrent single-thread processes of the reference serial build, "
                  f"each advancing the {n}^3 blast grid of this workload (seed 1): 1 untimed "
                  f"RK2 step, then 1 timed step; Mzone-updates/s summed over processes")
    else:
        v, sps = _oracle_rate(n, 1, 1)
        kind, cores = "port", 1
        sample = f"the C oracle on the {n}^3 blast grid, one thread, 1 timed step after 1"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC,
            "n_gpus": args.gpus, "steps": 1, "warmup": 1, "steps_requested": args.steps,
            "ms_per_step": sps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block(n),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def mixed_error(make_solver, nsteps, st):
    """Both forms for nsteps steps on the FP64 run's dt sequence; per
    conserved variable the relative L1 (sum|d|/sum|fp64|) and L-infinity
    (max|d|/max|fp64|) error of the mixed form, and its div(B)."""
    import torch
    from gpluto_dev_b200 import api
    a = make_solver(api.FP64)
    _, hist, _ = a.run(nsteps, FIRST_DT)
    _, Ua, _ = a.download()
    a.close()
    del a
    torch.cuda.empty_cache()
    b = make_solver(api.MIXED)
    for dt in hist:
        b.AdvanceStep(float(dt))
    _, Ub, Bb = b.download()
    b.close()
    del b
    torch.cuda.empty_cache()
    l1, linf = [], []
    for nv in range(Ua.shape[0]):
        den = float(np.abs(Ua[nv]).sum())
        d = np.abs(Ub[nv] - Ua[nv])
        l1.append(float(d.sum()) / den if den else 0.0)
        linf.append(float(d.max()) / float(np.abs(Ua[nv]).max()) if den else 0.0)
    nx, ny, nz = st.shape
    dx = [1.0 / nx, 1.0 / ny, 1.0 / nz]
    axes = {0: 2, 1: 1, 2: 0}
    div = sum((np.roll(Bb[d], -1, axis=axes[d]) - Bb[d]) / dx[d] for d in range(3))
    bmax = max(float(np.abs(x).max()) for x in Bb)
    return {"steps": nsteps, "variables": ["rho", "mx", "my", "mz", "Bx", "By", "Bz", "E"],
            "l1_rel": l1, "linf_rel": linf, "l1_rel_max": max(l1),
            "divB_rel_max": float(np.abs(div).max()) / (bmax / min(dx))}


def measure_e2e(make_solver, ncell, steps, ranks):
    """End to end through the C ABI with host buffers (pinned), three ways.

    The headline is the drop-in driver's loop (oracle/ref/gp_dropin.cpp
    around the reference's Src/main.cpp:444-463): the full reference-layout
    state (Uc, Vc, Vs with ghost zones, as Data holds it) goes up once;
    every step is one gp_advance_step (dt from the host, gp_step_out back)
    followed by gp_download_state of the whole state into the host arrays,
    so that output, analysis and the log read the new state.
    `roundtrip` also uploads the whole state before every step (Data
    changed on the host between steps); `resident` downloads it once after
    K steps (the loop between outputs)."""
    import torch
    from gpluto_dev_b200 import api
    se = make_solver(api.FP64)
    cshape, fshapes = se.reference_shapes()
    hU = torch.empty(cshape, dtype=torch.float64, pin_memory=True)
    hV = torch.empty(cshape, dtype=torch.float64, pin_memory=True)
    hB = [torch.empty(f, dtype=torch.float64, pin_memory=True) for f in fshapes]
    hB += [None] * (3 - len(hB))
    L = api.lib()
    out = api.GpStepOut()

    def up():
        api._check(L.gp_upload_state(se._h, api.LAYOUT_REFERENCE, api._dp(hU), api._dp(hV),
                                     api._dp(hB[0]), api._dp(hB[1]), api._dp(hB[2])))

    def dl():
        api._check(L.gp_download_state(se._h, api.LAYOUT_REFERENCE, api._dp(hU), api._dp(hV),
                                       api._dp(hB[0]), api._dp(hB[1]), api._dp(hB[2])))

    def timed(fn):
        torch.cuda.synchronize()
        ranks.barrier()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return ranks.max_over_ranks(time.perf_counter() - t0)

    dl()
    nbytes = (hU.numel() + hV.numel() + sum(b.numel() for b in hB if b is not None)) * 8
    so = ctypes.sizeof(out)

    k = max(1, steps)   # drop-in loop

    def dropin():
        up()
        de = FIRST_DT
        for _ in range(k):
            api._check(L.gp_advance_step(se._h, de, ctypes.byref(out)))
            de = out.dt_next
            dl()
    td = timed(dropin)

    kt = max(1, min(steps, 10))   # whole state both ways every step

    def roundtrip():
        de = FIRST_DT
        for _ in range(kt):
            up()
            api._check(L.gp_advance_step(se._h, de, ctypes.byref(out)))
            de = out.dt_next
            dl()
    tt = timed(roundtrip)

    def resident():
        up()
        de = FIRST_DT
        for _ in range(k):
            api._check(L.gp_advance_step(se._h, de, ctypes.byref(out)))
            de = out.dt_next
        dl()
    tr = timed(resident)
    se.close()
    return {"value": ranks.world * ncell * k / td / 1e6, "unit": METRIC,
            "h2d_bytes_per_step": nbytes / k + 8, "d2h_bytes_per_step": nbytes + so,
            "steps": k,
            "path": "state up once (gp_upload_state, reference layout, pinned host); per "
                    "step gp_advance_step (dt in, gp_step_out back) + gp_download_state "
                    "(reference layout) into the host Data arrays: the drop-in driver's loop",
            "roundtrip": {"value": ranks.world * ncell * kt / tt / 1e6, "unit": METRIC,
                          "steps": kt, "h2d_bytes_per_step": nbytes + 8,
                          "d2h_bytes_per_step": nbytes + so,
                          "path": "gp_upload_state + gp_advance_step + gp_download_state "
                                  "(reference layout, pinned host) every step"},
            "resident": {"value": ranks.world * ncell * k / tr / 1e6, "unit": METRIC,
                         "steps": k, "h2d_bytes_per_step": nbytes / k + 8,
                         "d2h_bytes_per_step": nbytes / k + so,
                         "path": "state up once (pinned, reference layout), K x "
                                 "gp_advance_step with its gp_step_out read by the host, "
                                 "state down once: the drop-in loop between outputs"}}

def fp64_roofline(per_kernel, top, ncell, ms_step, clocks):
    """The FP64 pipe as the roof of the FP64 form: FP64 flops per cell of
    each kernel (2 x DFMA + DADD + DMUL thread instructions counted by ncu on
    the same kernels, profiles/fp64_ops.json) x cells / the kernel's CUDA-event
    time, against the hardware's DFMA rate (ncu's peak_sustained DFMA thread
    instructions per cycle, x 2 flop) at the SM clock sampled in the run."""
    path = os.path.join(ROOT, "profiles", "fp64_ops.json")
    if not os.path.exists(path):
        return None
    ops = json.load(open(path))
    mhz = (clocks or {}).get("sm_mhz") or ops["sm_mhz_nominal"]
    peak = 2.0 * ops["dfma_per_cycle"] * mhz * 1e6 / 1e12
    per = ops["flop_per_cell"]

    def key(k):
        return f"{k['kernel']}_stage{k['stage']}" if k["kernel"] == "finish" else k["kernel"]
    step_flop = sum(per.get(key(k), 0.0) for k in per_kernel) * ncell
    top_flop = per.get(key(top), 0.0) * ncell
    ach = top_flop / (top["ms"] * 1e-3) / 1e12
    step_ach = step_flop / (ms_step * 1e-3) / 1e12
    return {"bound": "fp64", "kernel": f"{top['kernel']} (stage {top['stage']})",
            "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "flop_per_cell": per.get(key(top)),
            "pipe_active_pct_ncu": ops.get("pipe_active_pct", {}).get(key(top)),
            "peak_kind": "hardware DFMA rate (ncu peak_sustained) at the sampled SM clock",
            "step": {"flop_per_zone_update": step_flop / ncell, "achieved": step_ach,
                     "frac": step_ach / peak}}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def impl_ours(args):
    import torch
    from gpluto_dev_b200 import api, ics, replicas

    ranks = replicas.init("nccl")          # replicas: one grid (set) per GPU
    world, rank, local = ranks.world, ranks.rank, ranks.local
    torch.cuda.set_device(local)
    barrier = ranks.barrier

    n = args.n
    st = ics.mhd3d_blast(n=(n, n, n), seed=replicas.replica_seed(1, rank))
    ncell = n ** 3

    def solver(precision):
        sch = api.Scheme(physics=api.MHD, precision=precision, gamma=st.gamma, **SCHEME)
        return api.Solver.from_state(st, sch)

    # ---- CPU baseline: the reference serial build on this same grid, one
    # core, started now so that it runs beside the GPU measurements ------
    ref_run = None
    want_cpu = rank == 0 and world == 1 and not args.no_cpu
    if want_cpu and _ref_available():
        ref_run = ReferenceRun(st, 1, 1, 1)

    # ---- plain FP64 form: timed region ---------------------------------
    s64 = solver(api.FP64)
    dt = FIRST_DT
    dt, _, _ = s64.run(args.warmup, dt, history=False)
    clock = ClockSampler(local)
    torch.cuda.synchronize()
    barrier()
    clock.start()
    time.sleep(0.25)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    dt_after, _, out = s64.run(args.steps, dt, history=False)
    e1.record()
    torch.cuda.synchronize()
    clocks = clock.stop()
    barrier()
    t_ms = e0.elapsed_time(e1)
    t_ms = ranks.max_over_ranks(t_ms)
    ms_step = t_ms / args.steps
    value = replicas.whole_job_rate(world, ncell, args.steps, t_ms)
    launches = args.steps * s64.launches_per_step

    # ---- per-kernel timing (CUDA events around every launch) -----------
    prof, _ = s64.profile(3, dt_after)
    peak, peak_kind = peaks()
    per_kernel = []
    for name, stage, ms in prof:
        b = KERNEL_BYTES.get((name, stage), 0) * ncell
        per_kernel.append({"kernel": name, "stage": stage, "ms": ms,
                           "gbs": b / (ms * 1e-3) / 1e9 if ms > 0 else None})
    top = max(per_kernel, key=lambda k: k["ms"])
    top_bytes = KERNEL_BYTES[(top["kernel"], top["stage"])] * ncell
    achieved = top_bytes / (top["ms"] * 1e-3) / 1e9
    step_gbs = ALG_BYTES_ZONE * ncell / (ms_step * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        traffic = tj.get(f"{top['kernel']}_stage{top['stage']}")
    roofline = {"bound": "hbm", "kernel": f"{top['kernel']} (stage {top['stage']})",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": top_bytes, "launch_ms": top["ms"],
                "step": {"alg_bytes_per_zone_update": ALG_BYTES_ZONE, "achieved": step_gbs,
                         "frac": step_gbs / peak}}
    fp64 = fp64_roofline(per_kernel, top, ncell, ms_step, clocks)
    if fp64 is not None:
        roofline["fp64"] = fp64

    # ---- mixed FP32-flux form ------------------------------------------
    mixed = None
    if not args.no_mixed:
        s64 = None
        torch.cuda.empty_cache()
        smx = solver(api.MIXED)
        d2, _, _ = smx.run(args.warmup, FIRST_DT, history=False)
        torch.cuda.synchronize()
        barrier()
        e0.record()
        smx.run(args.steps, d2, history=False)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        tm = e0.elapsed_time(e1)
        tm = ranks.max_over_ranks(tm)
        mixed = {"value": replicas.whole_job_rate(world, ncell, args.steps, tm),
                 "ms_per_step": tm / args.steps}
        mixed["speedup_vs_fp64"] = mixed["value"] / value
        mprof, _ = smx.profile(3, d2)
        mixed["kernels"] = [{"kernel": nm, "stage": stg, "ms": ms} for nm, stg, ms in mprof]
        # the mixed form's HBM-bound kernel (its finish) against the HBM peak
        mtop = max(mixed["kernels"], key=lambda k: k["ms"])
        mbytes = KERNEL_BYTES_MIXED.get((mtop["kernel"], mtop["stage"]), 0) * ncell
        mach = mbytes / (mtop["ms"] * 1e-3) / 1e9
        mixed["roofline"] = {"bound": "hbm", "kernel": f"{mtop['kernel']} (stage {mtop['stage']})",
                             "achieved": mach, "peak": peak, "unit": "GB/s",
                             "frac": mach / peak, "peak_kind": peak_kind,
                             "alg_bytes_per_launch": mbytes, "launch_ms": mtop["ms"]}
        del smx
        torch.cuda.empty_cache()

    # ---- mixed-form error against the FP64 form (the FP64 oracle) --------
    if mixed is not None:
        mixed["error_vs_fp64"] = mixed_error(solver, args.error_steps, st)

    # ---- end to end through the C ABI with host buffers (measure_e2e) ----
    e2e = None if args.no_e2e else measure_e2e(solver, ncell, args.steps, ranks)

    # ---- the other workloads, short: the batched ensemble (all 512 grids,
    # K steps), the serving loop (64 requests at one rate) and RMHD 192^3 ---
    legs = {}
    if world == 1 and not args.no_legs:
        s64 = None
        torch.cuda.empty_cache()
        ens = ensemble_leg(args, ranks, args.steps, 3, with_e2e=False, with_cpu=False)
        legs["ensemble"] = {k: ens[k] for k in ("value", "unit", "steps", "ms_per_step",
                                               "roofline", "err_bits", "steps_done_min",
                                               "ctas")}
        legs["ensemble"]["workload"] = ens["config"]["workload"]
        legs["ensemble"]["cells_total"] = ens["config"]["cells_total"]
        torch.cuda.empty_cache()
        sweep, table, _, work = serve_leg(args, [SERVE_DEFAULT_RATE], args.requests)
        legs["serve"] = dict(sweep[0], workload=f"serve_poisson_{args.requests}req",
                             work_zone_updates=work)
        torch.cuda.empty_cache()
        legs["rmhd"] = rmhd_leg(min(args.steps, 10), 3)

    cpu = None
    if want_cpu:
        if ref_run is not None:
            v, sps = ref_run.result()
            cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": "reference",
                   "sample": f"the reference serial build (one thread) on this workload's own "
                             f"{n}^3 grid: 1 untimed RK2 step, then 1 timed step",
                   "s_per_step": sps}
        else:
            v, sps = _oracle_rate(n, 1, 1)
            cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": "port",
                   "sample": f"the C oracle (one thread) on this workload's {n}^3 grid: 1 "
                             f"timed RK2 step after 1", "s_per_step": sps}

    ranks.close()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 3-D MHD blast initial conditions)",
            "config": dict(config_block(args.n), parallelism=f"replicas x{world}"),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks,
            "forms": {"fp64": {"value": value, "ms_per_step": ms_step}, "mixed": mixed},
            "kernels": per_kernel, "err_bits": out.err_bits, **legs}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# batched ensemble: many uneven 2-D grids, one persistent launch per stage
# --------------------------------------------------------------------------
ENSEMBLE_ALG_BYTES_ZONE = 400   # 2-D ideal MHD: 5 x 8 B x (8 + 2)
REF_BINARY_2D = os.path.join(ROOT, "oracle", "_ref", "mhd2d_mc_lim_hlld_uct_hlld", "pluto")


def ensemble_config(args, table=None):
    from gpluto_dev_b200 import workloads
    shapes = workloads.ensemble_shapes(args.grids)
    cells = sum(a * b for (a, b), _ in shapes)
    c = {"workload": f"ensemble_{args.grids}x_2d_ideal_mhd",
         "grids": args.grids, "sides": "log-uniform 64..512, alternately square and 2:1",
         "cells_total": cells, "precision": "half FP64, half mixed (FP32 flux)",
         "scheme": "PLM-MC + HLLD + UCT_HLLD + RK2, CFL 0.4, gamma 5/3, per-grid dt",
         "ic": "2-D turbulence (random |k|<=4 modes), seed = grid index",
         "launch": "per RK stage: one persistent sweep kernel + one persistent EMF/finish "
                   "kernel over all grids; CUDA graph",
         "l2": "inputs larger than L2 (state of all grids ~15 GB), no flush",
         "parallelism": "replicas x1"}
    if table is not None:
        c["tile_table"] = table
    return c


def run_reference_grids(states, nsteps_timed, nwarm, binary, ndim=2):
    """The reference serial build on `states`, one concurrent process per
    grid.  Returns (Mzone-updates/s aggregate, mean s/step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    from gpluto_dev_b200 import ics
    import build_ref as br
    total = nwarm + nsteps_timed
    with tempfile.TemporaryDirectory() as tmp:
        procs = []
        for r, st in enumerate(states):
            d = os.path.join(tmp, f"p{r}")
            os.makedirs(d)
            nx, ny, nz = st.shape
            cfg = br.RefConfig(name="bench", physics="MHD", ndim=ndim, n=(nx, ny, nz),
                               limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                               first_dt=FIRST_DT)
            open(os.path.join(d, "pluto.ini"), "w").write(cfg.ini())
            icp = os.path.join(d, "ic.bin")
            ics.write_ic(icp, st)
            env = dict(os.environ, GPLUTO_FTZ_DAZ="0", GP_IC_FILE=icp,
                       GP_DUMP_STEP=str(total + 1), GP_DUMP_FILE=os.path.join(d, "out.dump"))
            procs.append((d, st, subprocess.Popen([binary, "-no-write", "-maxsteps", str(total + 1)],
                                                  cwd=d, env=env, stdout=subprocess.DEVNULL,
                                                  stderr=subprocess.DEVNULL)))
        rate, per = 0.0, []
        for d, st, p in procs:
            p.wait()
            w = br.read_dump(os.path.join(d, "out.dump")).wall
            sps = (w[nwarm + nsteps_timed] - w[nwarm]) / nsteps_timed
            per.append(sps)
            rate += st.ncells / sps
    return rate / 1e6, statistics.mean(per)


def ensemble_cpu_baseline(args, nproc):
    from gpluto_dev_b200 import workloads
    members = workloads.ensemble(args.grids, members=set(range(0, args.grids, max(1, args.grids // nproc))))
    members = members[:nproc]
    states = [m.state for m in members]
    if os.path.exists(REF_BINARY_2D):
        v, sps = run_reference_grids(states, 2, 1, REF_BINARY_2D)
        kind = "reference"
    else:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(len(states), mp_context=mp.get_context("spawn")) as ex:
            per = list(ex.map(_oracle_grid_worker, [(m.shape, m.seed) for m in members]))
        v = sum(st.ncells / t for st, t in zip(states, per)) / 1e6
        sps = statistics.mean(per)
        kind = "port"
    sample = (f"{len(states)} concurrent single-thread processes, each one ensemble member "
              f"(every {max(1, args.grids // nproc)}th grid, FP64), 2 timed RK2 steps after 1 "
              f"warm-up; Mzone-updates/s summed over processes")
    return {"value": v, "unit": METRIC, "cores": len(states), "kind": kind, "sample": sample}, sps


def _oracle_grid_worker(a):
    shape, seed = a
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from gpluto_dev_b200 import ics
    o = orc.Oracle(ics.mhd2d_turbulence(n=shape, seed=seed), limiter="mc", solver="hlld",
                   ct="uct_hlld")
    dt = FIRST_DT
    inv, _ = o.step(dt)
    dt = orc.lib().orc_next_dt(inv, 0.4, 1.1, dt)
    t0 = time.perf_counter()
    for _ in range(2):
        inv, _ = o.step(dt)
        dt = orc.lib().orc_next_dt(inv, 0.4, 1.1, dt)
    return (time.perf_counter() - t0) / 2


def ensemble_leg(args, ranks, steps, warmup, with_e2e=True, with_cpu=True, tune=True):
    """The batched ensemble (every rank its own set of grids): autotune on a
    sample, warm-up, `steps` timed steps of all grids; returns the fields of
    its JSON line."""
    import torch
    from gpluto_dev_b200 import autotune, replicas, workloads
    from gpluto_dev_b200 import batch as gb

    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier = ranks.barrier
    members = workloads.ensemble(args.grids, seed0=replicas.replica_seed(0, rank, args.grids))
    cells = sum(m.state.ncells for m in members)
    stream = torch.cuda.Stream()
    pool = sum(gb.slot_bytes(m.state, m.scheme) for m in members) + (64 << 20)

    # ---- autotune tile shapes per size bin on a sample (every 4th grid) ----
    trials = []
    if not tune:
        table = autotune.default_table()
    else:
        sample = members[::4]
        tb = gb.Batch(sum(gb.slot_bytes(m.state, m.scheme) for m in sample) + (64 << 20),
                      len(sample), stream=stream.cuda_stream)
        info = {tb.add(m.state, m.scheme, FIRST_DT, 10 ** 7): (2, m.state.ncells)
                for m in sample}
        table = autotune.tune(tb, info, steps=3, reps=2, log=trials)
        tb.close()
        del tb

    # ---- the run: all grids, warm-up then K timed steps -----------------
    b = gb.Batch(pool, len(members), stream=stream.cuda_stream)
    slots = [b.add(m.state, m.scheme, FIRST_DT, warmup + steps,
                   autotune.shape_for(table, 2, m.state.ncells)) for m in members]
    autotune.apply(b, table, {s: (2, m.state.ncells) for s, m in zip(slots, members)})
    b.advance(warmup)
    b.wait()
    clock = ClockSampler(local)
    barrier()
    clock.start()
    time.sleep(0.25)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    b.advance(steps)
    e1.record(stream)
    b.wait()
    clocks = clock.stop()
    barrier()
    t_ms = e0.elapsed_time(e1)
    t_ms = ranks.max_over_ranks(t_ms)
    err = 0
    done = []
    for s in slots:
        st = b.status(s)
        err |= st.err_bits
        done.append(st.steps_done)
    ctas = b.info()["ctas"]
    b.close()
    del b
    value = replicas.whole_job_rate(world, cells, steps, t_ms)
    peak, peak_kind = peaks()
    achieved = ENSEMBLE_ALG_BYTES_ZONE * cells * steps / (t_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "batch_sweep_kernel + batch_cell_kernel (all grids)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": None,
                "alg_bytes_per_zone_update": ENSEMBLE_ALG_BYTES_ZONE,
                "note": "step-level algorithmic bytes (2-D MHD state read+written once per "
                        "stage) over the whole-batch time"}

    # ---- end to end: admission from host arrays, K steps, download -------
    e2e = None
    if with_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b = gb.Batch(pool, len(members), stream=stream.cuda_stream)
        sl = [b.add(m.state, m.scheme, FIRST_DT, steps,
                    autotune.shape_for(table, 2, m.state.ncells)) for m in members]
        autotune.apply(b, table, {s: (2, m.state.ncells) for s, m in zip(sl, members)})
        b.advance(steps)
        b.wait()
        nout = 0
        for s in sl:
            V, U, Bs = b.download(s)
            nout += (V.size + U.size + sum(x.size for x in Bs)) * 8
        te = time.perf_counter() - t0
        b.close()
        nin = sum((m.state.V.size + sum(x.size for x in m.state.Bs)) * 8 for m in members)
        te = ranks.max_over_ranks(te)
        e2e = {"value": world * cells * steps / te / 1e6, "unit": METRIC,
               "h2d_bytes_per_step": nin / steps, "d2h_bytes_per_step": nout / steps,
               "steps": steps,
               "path": "gp_batch_add of every grid from host arrays, gp_batch_advance(K), "
                       "gp_batch_download of every grid; bytes amortised over K steps"}

    cpu = None
    if with_cpu and rank == 0 and world == 1:
        cpu, _ = ensemble_cpu_baseline(args, max(1, min(os.cpu_count() or 1, 16)))
    return {"value": value, "unit": METRIC, "steps": steps, "warmup": warmup,
            "ms_per_step": t_ms / steps, "config": ensemble_config(args, table),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": 4 * steps, "clocks": clocks, "ctas": ctas, "err_bits": err,
            "steps_done_min": min(done), "autotune_trials": len(trials)}


def impl_ensemble(args):
    import torch
    from gpluto_dev_b200 import replicas

    ranks = replicas.init("nccl")          # replicas: one grid (set) per GPU
    torch.cuda.set_device(ranks.local)
    leg = ensemble_leg(args, ranks, args.steps, args.warmup, with_e2e=not args.no_e2e,
                       with_cpu=not args.no_cpu, tune=not args.no_tune)
    world, rank = ranks.world, ranks.rank
    ranks.close()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "n_gpus": world, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic (seeded 2-D turbulence ensemble)", **leg}
    print(json.dumps(line), flush=True)
    return 0


def impl_reference_ensemble(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nproc = max(1, min(os.cpu_count() or 1, 64))
    cpu, sps = ensemble_cpu_baseline(args, nproc)
    line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": METRIC,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": ensemble_config(args), "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# special-relativistic MHD 192^3: both forms, and the mixed form's error
# --------------------------------------------------------------------------
RMHD_N = 192
RMHD_ALG_BYTES_ZONE = 696   # 440 + 4 x 64: the stored primitives read and written per stage
REF_BINARY_RMHD = os.path.join(ROOT, "oracle", "_ref", "rmhd3d_mc_lim_hlld_uct_hll", "pluto")


def rmhd_forms(n, steps, warmup, clock=None, profile=True):
    """The RMHD n^3 workload's FP64 and mixed forms, each timed over `steps`
    RK2 steps after `warmup` (CUDA events on the library's stream).  Returns
    (forms, state, solver factory, clocks sampled during the FP64 steps)."""
    import torch
    from gpluto_dev_b200 import api, ics
    st = ics.rmhd3d_turbulence(n=(n, n, n), seed=1)
    ncell = n ** 3

    def solver(precision):
        sch = api.Scheme(physics=api.RMHD, limiter="mc", riemann="hlld", ct_emf="uct_hll",
                         precision=precision, gamma=st.gamma, cfl=0.3)
        return api.Solver.from_state(st, sch)

    forms = {}
    clocks = None
    for prec, name in ((api.FP64, "fp64"), (api.MIXED, "mixed")):
        s = solver(prec)
        dt, _, _ = s.run(warmup, 1e-4, history=False)
        torch.cuda.synchronize()
        if name == "fp64" and clock is not None:
            clock.start()
            time.sleep(0.25)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, _, out = s.run(steps, dt, history=False)
        e1.record()
        torch.cuda.synchronize()
        if name == "fp64" and clock is not None:
            clocks = clock.stop()
        ms = e0.elapsed_time(e1) / steps
        forms[name] = {"value": ncell / ms / 1e3, "ms_per_step": ms, "err_bits": out.err_bits}
        if profile:
            prof, _ = s.profile(2, dt)
            forms[name]["kernels"] = [{"kernel": k, "stage": g, "ms": t} for k, g, t in prof]
        s.close()
        del s
        torch.cuda.empty_cache()
    forms["mixed"]["speedup_vs_fp64"] = forms["mixed"]["value"] / forms["fp64"]["value"]
    return forms, st, solver, clocks


def rmhd_leg(steps, warmup):
    """Short RMHD leg of the default line: the 192^3 workload's two forms."""
    forms, _, _, _ = rmhd_forms(RMHD_N, steps, warmup, profile=False)
    return {"value": forms["fp64"]["value"], "unit": METRIC, "steps": steps,
            "ms_per_step": forms["fp64"]["ms_per_step"], "err_bits": forms["fp64"]["err_bits"],
            "mixed": {k: forms["mixed"][k] for k in ("value", "ms_per_step", "speedup_vs_fp64",
                                                     "err_bits")},
            "workload": f"3d_rmhd_{RMHD_N}^3",
            "scheme": "PLM-MC + RMHD HLLD + UCT_HLL + RK2, CFL 0.3, gamma 4/3"}


def impl_rmhd(args):
    import torch
    from gpluto_dev_b200 import api, ics

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    n = args.n if args.n != N else RMHD_N
    ncell = n ** 3
    forms, st, solver, clocks = rmhd_forms(n, args.steps, args.warmup, ClockSampler(0))
    # error of the mixed form against FP64 after 100 steps on FP64's dt sequence
    a = solver(api.FP64)
    _, hist, _ = a.run(args.error_steps, 1e-4)
    Va, Ua, _ = a.download()
    a.close()
    del a
    torch.cuda.empty_cache()
    b = solver(api.MIXED)
    for dt in hist:
        b.AdvanceStep(float(dt))
    Vb, Ub, _ = b.download()
    b.close()
    l1 = [float(np.abs(Ub[v] - Ua[v]).sum() / np.abs(Ua[v]).sum()) for v in range(8)]
    linf = [float(np.abs(Ub[v] - Ua[v]).max() / np.abs(Ua[v]).max()) for v in range(8)]
    forms["mixed"]["error_vs_fp64"] = {"steps": args.error_steps, "l1_rel": l1, "linf_rel": linf,
                                       "variables": ["D", "mx", "my", "mz", "Bx", "By", "Bz",
                                                     "E-D"]}
    value = forms["fp64"]["value"]
    peak, peak_kind = peaks()
    achieved = RMHD_ALG_BYTES_ZONE * ncell / (forms["fp64"]["ms_per_step"] * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu and os.path.exists(REF_BINARY_RMHD):
        m = 32
        states = [ics.rmhd3d_turbulence(n=(m, m, m), seed=1 + r)
                  for r in range(max(1, min(os.cpu_count() or 1, 16)))]
        v, _ = run_reference_grids_rmhd(states, 2, 1)
        cpu = {"value": v, "unit": METRIC, "cores": len(states), "kind": "reference",
               "sample": f"{len(states)} concurrent single-thread processes, each a {m}^3 "
                         f"grid of the same RMHD scheme, 2 timed RK2 steps after 1 warm-up"}
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": forms["fp64"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 3-D RMHD turbulence)",
            "config": {"workload": f"3d_rmhd_{n}^3", "grid": [n, n, n],
                       "scheme": "PLM-MC + RMHD HLLD + UCT_HLL + RK2, CFL 0.3, gamma 4/3",
                       "ic": "rho = 1 + 0.5 f, p = 0.1, Lorentz factor log-uniform [1, 10] "
                             "along one seeded bulk direction, sigma = 1",
                       "l2": "inputs larger than L2, no flush", "parallelism": "replicas x1"},
            "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "alg_bytes_per_zone_update": RMHD_ALG_BYTES_ZONE},
            "forms": forms, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": args.steps * 11, "e2e": None}
    print(json.dumps(line), flush=True)
    return 0


def impl_reference_rmhd(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from gpluto_dev_b200 import ics
    if not os.path.exists(REF_BINARY_RMHD):
        print(json.dumps({"impl": "reference", "unavailable": "reference RMHD binary not built "
                          "(oracle/_ref/rmhd3d_mc_lim_hlld_uct_hll)"}))
        return 0
    m = 32
    nproc = max(1, min(os.cpu_count() or 1, 64))
    states = [ics.rmhd3d_turbulence(n=(m, m, m), seed=1 + r) for r in range(nproc)]
    v, _ = run_reference_grids_rmhd(states, 2, 1)
    cpu = {"value": v, "unit": METRIC, "cores": nproc, "kind": "reference",
           "sample": f"{nproc} concurrent single-thread processes, each a {m}^3 grid of the "
                     f"same RMHD scheme, 2 timed RK2 steps after 1 warm-up"}
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC,
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic",
                      "config": {"workload": f"3d_rmhd_{RMHD_N}^3"}, "cpu_baseline": cpu,
                      "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)
    return 0


def run_reference_grids_rmhd(states, nsteps_timed, nwarm):
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    from gpluto_dev_b200 import ics
    import build_ref as br
    total = nwarm + nsteps_timed
    with tempfile.TemporaryDirectory() as tmp:
        procs = []
        for r, st in enumerate(states):
            d = os.path.join(tmp, f"p{r}")
            os.makedirs(d)
            cfg = br.RefConfig(name="bench", physics="RMHD", ndim=3, n=st.shape,
                               limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLL", cfl=0.3,
                               first_dt=1e-4)
            open(os.path.join(d, "pluto.ini"), "w").write(cfg.ini())
            icp = os.path.join(d, "ic.bin")
            ics.write_ic(icp, st)
            env = dict(os.environ, GPLUTO_FTZ_DAZ="0", GP_IC_FILE=icp,
                       GP_DUMP_STEP=str(total + 1), GP_DUMP_FILE=os.path.join(d, "out.dump"))
            procs.append((d, st, subprocess.Popen([REF_BINARY_RMHD, "-no-write", "-maxsteps",
                                                   str(total + 1)], cwd=d, env=env,
                                                  stdout=subprocess.DEVNULL,
                                                  stderr=subprocess.DEVNULL)))
        rate = 0.0
        for d, st, p in procs:
            p.wait()
            w = br.read_dump(os.path.join(d, "out.dump")).wall
            rate += st.ncells / ((w[nwarm + nsteps_timed] - w[nwarm]) / nsteps_timed)
    return rate / 1e6, None


# --------------------------------------------------------------------------
# serving: Poisson arrivals, continuous batching, p50/p99 latency vs rate
# --------------------------------------------------------------------------
SERVE_RATES = (2.0, 4.0, 8.0, 16.0)
SERVE_DEFAULT_RATE = 8.0     # requests/s of the serving leg in the default line


def serve_leg(args, rates, nreq):
    """The serving loop on a Poisson stream of `nreq` requests at each rate
    in `rates` (requests/s); returns (sweep rows, tile table, clocks)."""
    import torch
    from gpluto_dev_b200 import autotune, serve, workloads
    from gpluto_dev_b200 import batch as gb

    base = workloads.requests(nreq, 1.0, seed=7)          # unit-rate arrival times
    states = [q.state() for q in base]                    # request payloads, built up front
    stream = torch.cuda.Stream()
    # tile shapes per size bin, tuned on a sample of the requests
    sample = list(range(0, nreq, max(1, nreq // 16)))
    tb = gb.Batch(sum(gb.slot_bytes(states[i], base[i].scheme()) for i in sample) + (64 << 20),
                  len(sample), stream=stream.cuda_stream)
    info = {tb.add(states[i], base[i].scheme(), 1e-4, 10 ** 7): (base[i].ndim, base[i].cells)
            for i in sample}
    table = autotune.tune(tb, info, steps=3, reps=2)
    tb.close()
    del tb
    sweep = []
    clock = ClockSampler(0)
    clock.start()
    for lam in rates:
        jobs = [serve.Job(q.rid, q.arrival / lam, st, q.scheme(), q.nsteps)
                for q, st in zip(base, states)]
        srv = serve.Server(pool_bytes=args.hbm_budget, max_slots=1024, chunk=args.chunk,
                           table=table, keep_results=True, stream=stream.cuda_stream)
        t0 = time.perf_counter()
        done = srv.serve(jobs, t0=t0)
        makespan = time.perf_counter() - t0
        row = serve.summary(done, srv.depth, makespan)
        srv.close()
        del srv
        row["lambda_per_s"] = lam
        row["steps_ok"] = all(j.status.steps_done == j.nsteps for j in done)
        row["err_bits"] = 0
        for j in done:
            row["err_bits"] |= j.status.err_bits
        sweep.append(row)
    clocks = clock.stop()
    work = sum(q.cells * q.nsteps for q in base)
    return sweep, table, clocks, work


def serve_config(args, nreq, rates, work, table):
    return {"workload": f"serve_poisson_{nreq}req", "requests": nreq,
            "rates_per_s": list(rates),
            "mix": "2-D/3-D ideal MHD (PLM-MC/HLLD/UCT_HLLD) or HD (PLM-MC/HLLC), "
                   "cells log-uniform 32^2..128^3, steps log-uniform 50..2000, FP64 or mixed",
            "hbm_budget_bytes": args.hbm_budget, "chunk_steps": args.chunk,
            "work_zone_updates": work, "tile_table": table,
            "launch": "per chunk: CUDA graph of chunk x RK2 steps, 2 persistent launches per "
                      "stage over all active requests"}


def impl_serve(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:          # replicas only: the serving sweep runs on one GPU
        return 0
    nreq = args.requests
    sweep, table, clocks, work = serve_leg(args, args.rates, nreq)
    # headline value: p99 latency at the highest rate of the sweep
    head = sweep[-1]
    line = {"metric": "p99 serve latency", "value": head["p99_s"], "unit": "s",
            "n_gpus": 1, "steps": None, "warmup": None, "ms_per_step": None,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32", "data": "synthetic (seeded serving stream)",
            "config": serve_config(args, nreq, args.rates, work, table),
            "throughput_Mzone_updates_per_s": head["Mzone_updates_per_s"],
            "sweep": sweep, "clocks": clocks,
            "e2e": {"value": head["Mzone_updates_per_s"], "unit": METRIC,
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "path": "request payloads admitted from host arrays, results downloaded to "
                            "host at completion; latency on the host clock"},
            "gpu_launches": None}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mhd3d_blast",
                    choices=["mhd3d_blast", "ensemble", "serve", "rmhd"])
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rates", type=float, nargs="+", default=list(SERVE_RATES))
    ap.add_argument("--chunk", type=int, default=25)
    ap.add_argument("--hbm-budget", type=int, default=150 * 10 ** 9)
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--grids", type=int, default=512)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--error-steps", type=int, default=100)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the short ensemble and serving legs of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps is None:
        args.steps = 200 if args.workload == "ensemble" else 100
    if args.workload == "ensemble":
        return impl_reference_ensemble(args) if args.impl == "reference" else impl_ensemble(args)
    if args.workload == "rmhd":
        if args.impl == "reference":
            return impl_reference_rmhd(args)
        return impl_rmhd(args)
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving "
                              "loop; its CPU rate per zone is the ensemble/blast reference arm"}))
            return 0
        return impl_serve(args)
    if args.impl == "reference":
        return impl_reference(args)
    return impl_ours(args)


if __name__ == "__main__":
    sys.exit(main())
