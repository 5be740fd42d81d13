#!/usr/bin/env python
"""Throughput benchmark: Kelvin-Helmholtz 4096^2, PLM + HLLC + RK2, FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one RK2 time step over the whole 4096^2 grid (the hot path of
Sim::Advance).  Prints one JSON line (rank 0).

ours (default):
  * value: zone-updates/s over exactly K device-resident steps, timed with
    CUDA events on the library's stream between a barrier + synchronize on
    both sides; max over ranks.  The K-step block is timed --repeats times
    (25 by default) and the median block is reported, with every block's
    time in `timed_blocks`; nvidia-smi samples the clocks every 50 ms across
    all blocks.  The state (4 x 4100^2 doubles, 538 MB per buffer) is larger
    than L2, so no flush is needed between steps.
  * e2e: the same metric through the reference-facing call with host
    buffers, at the reference's own cadence: its main loop calls
    Sim::Advance(dtoutput) once per output, dtoutput = 0.1 in its KH input,
    and the drop-in Advance uploads the state from pinned host memory
    (gk_upload_cons), runs the steps to the next output time (gk_advance) and
    downloads it (gk_download_planes).  Bytes per step are a call's bytes
    over its steps.  e2e_state_every_step is the same with the state in and
    out around every single step (gk_run_steps(1)), which PCIe bounds.  The
    z-momentum plane, zero in this 2D problem, is checked on the host and
    stays put, so four planes cross the bus each way (gk_io_bytes).
  * roofline: the fused stage kernel's algorithmic HBM bytes per launch
    (80 B per cell on average: stage 1 reads and writes 4 doubles, stage 2
    reads 8 and writes 4) over its average launch time, measured with CUDA
    events around each launch in an un-graphed pass of the same workload.
  * cpu_baseline: the reference itself (oracle/_ref/ref_fast_kh_baseline,
    built from the reference sources with its Makefile flags) on this host's
    cores, on a bounded number of steps of the same problem; rank 0, N=1.
  With N > 1 each rank runs an independent replica (weak scaling, no
  collective on the data path); torch.distributed is used only for the
  barrier and the max over ranks.

reference: the reference's OpenMP CPU path on the host cores, same metric;
  each step is one time step of KH at the largest size from {4096^2,
  2048^2, 1024^2} that keeps the whole run within about two minutes.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s"
UNIT = "zone-updates/s"
BYTES_PER_ZU_RK2 = 160  # 5 * V * 8 B with V = 4 (2D): algorithmic HBM bytes per zone-update
STAGE_BYTES_PER_CELL = 80  # per stage launch, averaged over the two RK2 stages
# FP64 add/mul/fma thread-instructions per zone-update of the fast-mode fused
# RK2 step (stage 1 + last stage), from the ncu capture in
# profiles/stage2d_tma_kh2048_ncu.md; the FP64 pipe issues 64 lanes per
# SM per clock on B200 (148 SMs)
FP64_OPS_PER_ZU_FAST = 283 + 310
FP64_LANES = 64 * 148


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per stage-kernel launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "stage2d_tma_kh4096_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def start(self, wait_s: float = 5.0):
        """Starts sampling every 50 ms and returns once the first sample is
        in (or after wait_s), so the timed region that follows is covered."""
        try:
            self.out = tempfile.NamedTemporaryFile(mode="w+", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.device)], stdout=self.out,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < wait_s and self.proc.poll() is None:
            if os.path.getsize(self.out.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"],
                    "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        with open(self.out.name) as f:
            text = f.read()
        self.out.close()
        try:
            os.unlink(self.out.name)
        except OSError:
            pass
        return self.summarise(text)

    @staticmethod
    def summarise(text: str):
        """Median SM clock, the highest max clock and the throttle reasons seen
        Active in nvidia-smi's CSV rows (FIELDS, no header, no units); rows
        that do not parse are skipped."""
        rows = [r.split(",") for r in text.strip().splitlines() if r.strip()]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def config_dict(n, mode, extra=None):
    d = {"workload": f"Kelvin-Helmholtz {n}x{n}, PLM (van Leer) + HLLC + RK2, CFL 0.4, periodic",
         "grid": [n, n], "integrator": "rk2", "reconstruction": "plm-vanleer", "riemann": "hllc",
         "arith_mode": mode, "l2": "state larger than L2 (538 MB per buffer); no flush needed",
         "parallelism": "replicas"}
    if extra:
        d.update(extra)
    return d


# --------------------------------------------------------------- reference
def run_reference_binary(exe, n, steps, threads, timeout=900):
    """Runs the reference build on KH n^2 for `steps` steps; returns the
    driver's JSON (per-step timestamps included)."""
    from gaukuk_b200 import problems
    p, _ = problems.kh(8)
    import dataclasses
    p = dataclasses.replace(p, nx=n, ny=n, stepmax=steps, tmax=2.0, dtoutput=2.0)
    with tempfile.TemporaryDirectory() as td:
        inf = os.path.join(td, "kh.in")
        with open(inf, "w") as f:
            f.write(p.to_in_text({"seed": 0, "amp": 0.01, "noise": 1e-3}))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        r = subprocess.run([exe, "-i", inf, "--step-times"], cwd=td, capture_output=True,
                           text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stderr[-500:]}")
        return json.loads(r.stderr.strip().splitlines()[-1])


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_rate(exe, n, warm, steps, threads):
    """zone-updates/s of the reference over steps warm+1 .. warm+steps."""
    d = run_reference_binary(exe, n, warm + steps, threads)
    st = d["step_stamps"]
    # stamps[i] is written at the end of step i+1
    t = st[warm + steps - 1] - st[warm - 1] if warm >= 1 else st[steps - 1]
    return n * n * steps / t, t, d


PORTABLE_FLAGS = ("reference Makefile flags (-O3 -ffast-math -funroll-loops, OpenMP) with "
                  "-march=x86-64-v3 in place of -march=native")
NATIVE_FLAGS = ("the reference Makefile's flags exactly (-O3 -march=native -ffast-math "
                "-funroll-loops, OpenMP; native = sapphirerapids, the benchmark hosts' CPU)")


def reference_exe(portable=False):
    """The reference build for this host and its flags: the reference
    Makefile's flags exactly (oracle/_ref/ref_native_kh_baseline, built for
    the benchmark hosts' CPU) when it runs here, else the portable build."""
    native = os.path.join(ROOT, "oracle", "_ref", "ref_native_kh_baseline")
    port = os.path.join(ROOT, "oracle", "_ref", "ref_fast_kh_baseline")
    if not portable and os.path.exists(native):
        try:
            run_reference_binary(native, 64, 2, 1, timeout=120)
            return native, NATIVE_FLAGS
        except Exception:
            pass
    return port, PORTABLE_FLAGS


def main_reference(args, rank, world):
    if rank != 0:
        return 0
    exe, flags = reference_exe()
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference build oracle/_ref missing (run build())"}))
        return 0
    threads = host_threads()
    # calibrate on 1024^2: seconds per zone-update on this host
    rate0, _, _ = cpu_rate(exe, 1024, 1, 3, threads)
    budget_s = 120.0
    n = 1024
    for cand in (4096, 2048, 1024):
        if cand * cand * (args.warmup + args.steps) / rate0 <= budget_s:
            n = cand
            break
    warm = max(1, args.warmup)
    rate, secs, _ = cpu_rate(exe, n, warm, args.steps, threads)
    cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
           "sample": f"KH {n}^2 RK2 PLM HLLC, steps {warm + 1}..{warm + args.steps} of one run, "
                     f"{flags}", "build": os.path.basename(exe)}
    out = dict(base)
    out.update({"value": rate, "ms_per_step": 1000.0 * secs / args.steps,
                "config": config_dict(args.n, "reference-cpu",
                                      {"reference_grid": [n, n], "parallelism": "openmp"}),
                "cpu_baseline": cpu,
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}})
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------- ours
def main_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from gaukuk_b200 import problems
    from gaukuk_b200.replicas import Replicas
    from gaukuk_b200.sim import Sim

    torch.cuda.set_device(local_rank)
    reps = Replicas("nccl", timeout_s=300, device_sync=torch.cuda.synchronize)
    barrier, max_over_ranks = reps.barrier, reps.max

    n = args.n
    if args.ncu_case and args.box3d:
        # a 3D case for profilers: periodic box with a smooth random state, RK2
        from gaukuk_b200.config import Params
        m = args.box3d
        p = Params(nx=m, ny=m, nz=m, bc=(1,) * 6, integrator=2, tmax=1.0, dtoutput=1.0)
        c = problems.random_smooth(p, seed=rank, with_vz=True)
    else:
        p, c = problems.kh(n, seed=rank)
    cells = p.nx * p.ny
    sim = Sim(p, c, mode=args.mode, device=local_rank)
    if args.ncu_case:
        # a short run for profilers: upload + `steps` steps, nothing else
        sim.run_steps(args.steps)
        if rank == 0:
            print(json.dumps({"ncu_case": True, "n": n, "box3d": args.box3d, "path": sim.path,
                              "steps": args.steps, "mode": args.mode,
                              "t": sim.get_time()}))
        sim.close()
        return 0
    steps_per_graph, launches_per_step = sim.graph_info()

    # warm-up
    sim.run_steps(args.warmup)
    step0 = sim.get_step()

    def timed(sim_, k):
        st = torch.cuda.ExternalStream(sim_.stream, device=torch.device("cuda", local_rank))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(st)
        sim_.enqueue_steps(k)
        ev1.record(st)
        ev1.synchronize()
        barrier()
        return ev0.elapsed_time(ev1)

    # `repeats` timed blocks of exactly K steps each, every block bracketed by
    # a barrier + synchronize; the line reports the median block (max over
    # ranks per block), and the clocks are sampled across all of them
    sampler = ClockSampler(local_rank)
    sampler.start()
    blocks = []
    for _ in range(max(1, args.repeats)):
        blocks.append(max_over_ranks(timed(sim, args.steps)))
    clocks = sampler.stop()
    took = sim.get_step() - step0
    if took != args.steps * len(blocks):
        raise RuntimeError(f"expected {args.steps * len(blocks)} steps, device ran {took}")
    ms_max = statistics.median(blocks)
    value = world * cells * args.steps / (ms_max / 1000.0)

    # the other arithmetic mode, same workload (reported, not the headline)
    other_mode = "parity" if args.mode == "fast" else "fast"
    sim2 = Sim(p, c, mode=other_mode, device=local_rank)
    sim2.run_steps(args.warmup)
    ms2 = statistics.median([max_over_ranks(timed(sim2, max(2, args.steps // 4)))
                             for _ in range(5)])
    other = {"arith_mode": other_mode,
             "value": world * cells * max(2, args.steps // 4) / (ms2 / 1000.0),
             "ms_per_step": ms2 / max(2, args.steps // 4)}
    sim2.close()

    # per-kernel profile (events around every launch, un-graphed)
    prof_steps = 4
    prof = sim.profile(prof_steps)
    total = sum(v[0] for v in prof.values())
    shares = {k: {"ms_total": v[0], "launches": v[1], "share": v[0] / total if total else None}
              for k, v in prof.items()}
    stage_ms, stage_n = prof.get("stage2d", (0.0, 0))
    avg_stage_s = (stage_ms / stage_n) / 1000.0 if stage_n else None
    peak, peak_kind = measured_peaks()
    roof = None
    if avg_stage_s:
        achieved = STAGE_BYTES_PER_CELL * cells / avg_stage_s / 1e9
        roof = {"bound": "hbm", "kernel": "gk_fast::k_stage2d" if args.mode == "fast"
                else "gk_parity::k_stage2d",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": STAGE_BYTES_PER_CELL * cells,
                "avg_launch_ms": avg_stage_s * 1000.0,
                "traffic": ncu_traffic(),
                "step_frac_of_hbm_roofline": (BYTES_PER_ZU_RK2 * value / world / 1e9) / peak}
    roof64 = None
    if args.mode == "fast":
        # the bound that binds: FP64 issue of the stage kernel (add/mul/fma only;
        # compares and min/max also use the pipe)
        mhz = (clocks or {}).get("sm_mhz")
        src = "the median SM clock sampled in the timed region"
        if not mhz:
            mhz, src = 1965.0, "the B200's maximum SM clock (no clock sample in the timed region)"
        ach = FP64_OPS_PER_ZU_FAST * value / world / 1e12
        pk = FP64_LANES * mhz * 1e6 / 1e12
        roof64 = {"bound": "fp64 issue", "achieved": ach, "peak": pk,
                  "unit": "T FP64 thread-instructions/s", "frac": ach / pk,
                  "ops_per_zone_update": FP64_OPS_PER_ZU_FAST,
                  "peak_source": "64 FP64 lanes x 148 SMs x " + src,
                  "ops_source": "ncu, profiles/stage2d_tma_kh2048_ncu.md"}

    # end to end through the C ABI with pinned host buffers
    e2e_steps = max(1, args.e2e_steps)
    host = torch.empty(p.shape, dtype=torch.float64, pin_memory=True).numpy()
    host[...] = c
    g = p.ng
    sim.upload(host)
    sim.run_steps(1)
    sim.download(host, planes_only=True)
    h2d, d2h = sim.io_bytes()  # what crossed the bus per step (the zero MTZ plane stays put)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.upload(host)
        sim.run_steps(1)
        sim.download(host, planes_only=True)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0)
    e2e_value = world * cells * e2e_steps / e2e_s
    assert np.isfinite(host[0, g, g:g + p.ny, g:g + p.nx]).all()

    # end to end at the reference's own cadence: its main loop calls
    # Sim::Advance(dtoutput) once per output (src/main.cpp:44-52), dtoutput
    # 0.1 in its KH input; the drop-in Advance uploads the state from pinned
    # host memory, runs the steps to the next output time and downloads it
    calls = max(1, args.e2e_calls)
    barrier()
    s0 = sim.get_step()
    t0 = time.perf_counter()
    for _ in range(calls):
        sim.upload(host)
        up_call, _ = sim.io_bytes()
        sim.advance(args.e2e_dtoutput)
        sim.download(host, planes_only=True)
    t1 = time.perf_counter()
    _, down_call = sim.io_bytes()
    adv_steps = sim.get_step() - s0
    adv_s = max_over_ranks(t1 - t0)
    adv_all = int(reps.sum(adv_steps))  # the ranks' problems differ, and so do their steps
    adv_value = cells * adv_all / adv_s
    assert np.isfinite(host[0, g, g:g + p.ny, g:g + p.nx]).all()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        exe, flags = reference_exe()
        if os.path.exists(exe):
            threads = host_threads()
            rate0, _, _ = cpu_rate(exe, 1024, 1, 3, threads)
            # bounded sample: about 10 s of CPU work on the full grid
            nsteps = int(max(3, min(40, 10.0 * rate0 / cells)))
            rate, secs, _ = cpu_rate(exe, n, 1, nsteps, threads)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"KH {n}^2, steps 2..{nsteps + 1} of one run ({secs:.1f} s), {flags}",
                   "build": os.path.basename(exe)}
            pexe, pflags = reference_exe(portable=True)
            if pexe != exe and os.path.exists(pexe):
                prate, psecs, _ = cpu_rate(pexe, n, 1, nsteps, threads)
                cpu["portable_build"] = {"value": prate, "sample": f"same steps ({psecs:.1f} s), "
                                                                    f"{pflags}"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                   "sample": "reference build absent"}

    if rank == 0:
        # per block: the begin kernel, then whole graphs of steps
        launches_block = launches_per_step * steps_per_graph * (-(-args.steps // steps_per_graph)) + 1
        launches = launches_block * len(blocks)
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded KH initial condition of the named shape)",
               "config": config_dict(n, args.mode, {"path": sim.path}),
               "e2e": {"value": adv_value, "unit": UNIT,
                       "h2d_bytes_per_step": up_call * calls / adv_steps,
                       "d2h_bytes_per_step": down_call * calls / adv_steps,
                       "steps_all_ranks": adv_all,
                       "cadence": f"one Sim::Advance(dtoutput={args.e2e_dtoutput}) per call, the "
                                  "reference's KH output interval: gk_upload_cons + gk_advance "
                                  "+ gk_download_planes from pinned host memory",
                       "calls": calls, "steps": adv_steps, "h2d_bytes_per_call": up_call,
                       "d2h_bytes_per_call": down_call,
                       "timing": "host wall clock around the C-ABI calls, max over ranks"},
               "e2e_state_every_step": {
                   "value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                   "cadence": "the state in and out around every single step (PCIe-bound)",
                   "timing": "host wall clock around the C-ABI calls, max over ranks"},
               "roofline": roof, "roofline_fp64": roof64, "cpu_baseline": cpu, "clocks": clocks,
               "gpu_launches": launches, "kernel_shares": shares, "other_mode": other,
               "timed_blocks": {"repeats": len(blocks), "steps_per_block": args.steps,
                                "ms_per_block": blocks, "reported": "median block",
                                "min_ms": min(blocks), "max_ms": max(blocks)}}
        print(json.dumps(out))
    sim.close()
    reps.close()
    return 0


def main_slabs(args, rank, world, local_rank):
    """One KH grid of n x (n * N) cells split into N y-slabs, one per GPU
    (weak scaling: n^2 cells per GPU), exchanging ghost rows through NCCL
    every RK stage and the CFL maximum every step (gaukuk_b200.slabs).
    value = zone-updates/s of the whole grid over K steps, timed with CUDA
    events on the library's stream between a barrier + synchronize, max over
    ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from gaukuk_b200 import problems
    from gaukuk_b200.slabs import DistSlabs

    torch.cuda.set_device(local_rank)
    if not dist.is_initialized():
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29531")
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=120))
    n = args.n
    p, c = problems.kh(n, ny=n * world, seed=0)
    s = DistSlabs(p, c, dist, mode=args.mode, device=local_rank)
    s.run_steps(args.warmup)
    torch.cuda.synchronize()
    blocks = []
    for _ in range(max(1, args.repeats)):
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        s.run_steps(args.steps)
        ev1.record()
        ev1.synchronize()
        ms = torch.tensor([ev0.elapsed_time(ev1)])
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        blocks.append(float(ms[0]))
    med = statistics.median(blocks)
    if rank == 0:
        print(json.dumps({"metric": METRIC + " (one grid in y-slabs)", "unit": UNIT,
                          "value": p.nx * p.ny * args.steps / (med / 1000.0), "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": med / args.steps,
                          "higher_is_better": True, "scaling": "weak", "dtype": "f64",
                          "config": {"workload": f"KH {p.nx}x{p.ny} in {world} y-slabs",
                                     "arith_mode": args.mode},
                          "timed_blocks": blocks,
                          "timing": "CUDA events around run_steps (the host waits for each "
                                    "step's NCCL calls to be enqueued), max over ranks"}))
    s.close()
    dist.destroy_process_group()
    return 0


def main_ncu_case(args, local_rank):
    """Short runs for profilers, nothing else:
    * ensemble: 16 KH instances (sizes drawn from 128^2, 256^2, 512^2) in one
      ensemble, `steps` steps (k_ens_stage, k_ens_bc);
    * learned: `steps` Adam steps of batch 65536 on 2^20 synthetic faces
      (k_mlp_grad, k_adam), then `steps` steps of KH 256^2 with the model
      installed (the generic path with k_flux_correct)."""
    import numpy as np
    import torch

    from gaukuk_b200 import problems
    from gaukuk_b200.sim import Sim
    torch.cuda.set_device(local_rank)
    if args.workload == "ensemble":
        from gaukuk_b200.ensemble import Ensemble
        inst = problems.kh_ensemble(16, seed=0)
        sims = [Sim(p, c, mode=args.mode, device=local_rank) for p, c, _ in inst]
        ens = Ensemble(sims)
        ens.run_steps(args.steps)
        ens.close()
        for s in sims:
            s.close()
    else:
        from gaukuk_b200 import learned
        rng = np.random.default_rng(0)
        X = rng.normal(size=(1 << 20, learned.NI)).astype(np.float32)
        Y = (0.1 * rng.normal(size=(1 << 20, 4))).astype(np.float32)
        blob = learned.init_model(X, Y, seed=0)
        tr = learned.Trainer(blob, X, Y, device=local_rank)
        tr.train(args.steps, batch=65536, lr=1e-3)
        blob = tr.model()
        tr.close()
        p, c = problems.kh(256)
        with Sim(p, c, mode="fast", device=local_rank) as s:
            learned.install(s, blob)
            s.run_steps(args.steps)
    torch.cuda.synchronize()
    print(json.dumps({"ncu_case": True, "workload": args.workload, "steps": args.steps}))
    return 0


def main_ensemble(args, rank, world, local_rank):
    """Pattern 2: 64 independent KH problems (sizes drawn from 128^2, 256^2,
    512^2) in one persistent launch per RK stage, to t = 1, against the same
    64 problems run one after another through the single-problem path."""
    import numpy as np
    import torch

    from gaukuk_b200 import autotune, problems
    from gaukuk_b200.ensemble import Ensemble
    from gaukuk_b200.sim import Sim

    torch.cuda.set_device(local_rank)
    n, tmax = args.ens_n, args.ens_tmax
    inst = problems.kh_ensemble(n, seed=rank, tmax=tmax)
    sims = [Sim(p, c, mode=args.mode, device=local_rank) for p, c, _ in inst]
    ens = Ensemble(sims)
    tuned = autotune.tune_ensemble(ens, steps=4, use_cache=False)
    for s, (p, c, _) in zip(sims, inst):  # back to t = 0
        s.set_time(0.0, 0)
        s.upload(c)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ens.run(tmax)
    torch.cuda.synchronize()
    t_ens = time.perf_counter() - t0
    zu = sum(p.nx * p.ny * len(s.dt_log()) for s, (p, _, _) in zip(sims, inst))
    finals = [s.download() for s in sims]
    # the same problems one after another, each through its own handle
    t_seq = 0.0
    same = True
    for (p, c, _), fin in zip(inst, finals):
        solo = Sim(p, c, mode=args.mode, device=local_rank)
        solo.run_steps(1)  # build its graph outside the timing
        solo.set_time(0.0, 0)
        solo.upload(c)
        torch.cuda.synchronize()
        a = time.perf_counter()
        solo.run(tmax, tmax)
        torch.cuda.synchronize()
        t_seq += time.perf_counter() - a
        same &= bool(np.array_equal(solo.download(), fin))
        solo.close()
    sizes = {}
    for _, _, d in inst:
        sizes[d["size"]] = sizes.get(d["size"], 0) + 1
    if rank == 0:
        print(json.dumps({
            "metric": "ensemble zone-updates/s", "unit": UNIT, "value": zu / t_ens,
            "workload": f"{n} independent KH problems to t={tmax}, sizes {sizes} (per size), "
                        f"density ratio U[1.5,4], half-width U[0.2,0.3], amplitude U[0.005,0.02]",
            "arith_mode": args.mode, "zone_updates": zu, "seconds": t_ens,
            "sequential": {"value": zu / t_seq, "seconds": t_seq},
            "speedup_vs_sequential": t_seq / t_ens, "identical_to_sequential": same,
            "tiling": tuned, "timing": "host wall clock between device synchronisations"}))
    ens.close()
    for s in sims:
        s.close()
    return 0


def main_configs(args, rank, world, local_rank):
    """The plain-method configurations run to their end times on one GPU:
    Sod 256 (t = 0.2, against the exact Riemann solution), KH 256^2 (t = 2,
    conservation), RT 1024x3072 (RK3 + gravity, t = 5, mirror symmetry), in
    both arithmetic modes, with the reference build (fast flags, OpenMP on
    the host cores) on the same inputs -- the whole run for Sod and KH 256^2,
    the first 200 steps for RT.  Timing: host wall clock around Sim.run with
    a device synchronise on both sides (each config is one long sequence of
    graph launches); the reference's is its driver's time inside Advance."""
    import numpy as np
    import torch

    from gaukuk_b200 import problems
    from gaukuk_b200.sim import Sim
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gk_oracle
    import riemann_exact as rx

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    threads = host_threads()
    out = []
    cases = [("sod256", problems.sod(256)), ("kh256", problems.kh(256)),
             ("rt1024x3072", problems.rt(1024, 3072))]
    for name, (p, c) in cases:
        cells = p.nx * p.ny * p.nz
        row = {"config": name, "grid": [p.nx, p.ny, p.nz], "integrator": p.integrator, "tmax": p.tmax}
        a0 = c[:, p.ng, p.ng:p.ng + p.ny, p.ng:p.ng + p.nx]
        for mode in ("fast", "parity"):
            with Sim(p, c, mode=mode) as s:
                s.run_steps(1)  # graph and first-touch outside the timing
                s.set_time(0.0, 0)
                s.upload(c)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                s.run(p.tmax, p.tmax)
                torch.cuda.synchronize()
                secs = time.perf_counter() - t0
                steps = s.get_step()
                fin = s.download()
            a = fin[:, p.ng, p.ng:p.ng + p.ny, p.ng:p.ng + p.nx]
            r = {"steps": steps, "seconds": secs, "zone_updates_per_s": cells * steps / secs}
            r["mass_drift"] = float(abs(a[0].sum() - a0[0].sum()) / a0[0].sum())
            if name.startswith("sod"):
                xl = np.arange(p.nx) / p.nx
                rho, _, _ = rx.cell_average(xl, xl + 1.0 / p.nx, p.tmax, 0.5, (1.0, 0.0, 1.0),
                                            (0.125, 0.0, 0.1))
                r["l1_rho_vs_exact"] = float(np.abs(a[0, 0] - rho).mean())
            elif name.startswith("kh"):
                r["energy_drift"] = float(abs(a[4].sum() - a0[4].sum()) / a0[4].sum())
            else:
                r["mirror_asymmetry_rho"] = float(np.abs(a[0] - a[0][:, ::-1]).max() / a[0].max())
            row[mode] = r
        full = not name.startswith("rt")
        try:
            _, dts, st = gk_oracle.run_reference(p, c, stepmax=None if full else 200, flavour="fast",
                                                 threads=threads, timeout=900)
            row["reference"] = {"steps": st["steps"], "seconds": st["advance_seconds"],
                                "zone_updates_per_s": cells * st["steps"] / st["advance_seconds"],
                                "cores": threads, "sample": "whole run" if full else "first 200 steps"}
        except Exception as e:  # the reference build is optional on the box
            row["reference"] = {"unavailable": str(e)[:200]}
        out.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    print(json.dumps({"workload": "configs", "metric": METRIC, "unit": UNIT, "dtype": "f64",
                      "data": "synthetic (seeded initial conditions of the named shapes)",
                      "runs": out}))
    return 0


def main_learned(args, rank, world, local_rank):
    """Pattern 4: data from 4x finer plain runs, training on the GPU with the
    project's BF16 kernels, evaluation on held-out seeds against plain coarse,
    plain 2x coarse and the 4x fine plain run (L1 density error, GPU time)."""
    import numpy as np
    import torch

    from gaukuk_b200 import learned

    torch.cuda.set_device(local_rank)
    log = (lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else None
    train_seeds = list(range(1000, 1000 + args.train_seeds))
    eval_seeds = list(range(5000, 5000 + args.eval_seeds))
    t0 = time.perf_counter()
    tv_min = learned.TV_GATE if args.tv_min is None else args.tv_min
    diss_frac = learned.DISS_FRAC if args.diss_frac is None else args.diss_frac
    X, Y = learned.generate(train_seeds, coarse=args.coarse, t_end=args.t_end,
                            snapshots=args.snapshots, frac=args.frac, tv_min=tv_min,
                            noise=args.noise, log=log)
    t_data = time.perf_counter() - t0
    hold = np.random.default_rng(7).random(len(X)) < 0.1
    Xv, Yv, X, Y = X[hold], Y[hold], X[~hold], Y[~hold]
    blob = learned.init_model(X, Y, seed=0)
    tr = learned.Trainer(blob, X, Y, device=local_rank)
    losses = [tr.train(1, batch=args.batch, lr=args.lr)]
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    chunk = max(1, args.train_steps // 10)
    done = 0
    while done < args.train_steps:
        k = min(chunk, args.train_steps - done)
        losses.append(tr.train(k, batch=args.batch, lr=args.lr, seed=done + 1))
        done += k
        if log:
            log(f"step {done}: loss {losses[-1]:.4g}")
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    model = tr.model()
    tr.close()
    fit = {"r2_train": learned.r2(model, X, Y), "r2_held_out": learned.r2(model, Xv, Yv)}
    if log:
        log(f"fit: {fit}")
    if args.model_out:
        os.makedirs(os.path.dirname(os.path.abspath(args.model_out)), exist_ok=True)
        np.save(args.model_out, model)
    ev = learned.evaluate(model, eval_seeds, coarse=args.coarse, t_end=args.t_end,
                          times=(0.25 * args.t_end, 0.5 * args.t_end, args.t_end),
                          tv_min=tv_min, diss_frac=diss_frac, log=log)
    sm = ev["summary"]
    c, c2 = "plain_%d" % args.coarse, "plain_%d" % (2 * args.coarse)
    lr_ = "learned_%d" % args.coarse
    if rank == 0:
        print(json.dumps({
            "metric": "L1 density error vs 4x fine plain FP64 run, at equal resolution",
            "workload": f"KH (ensemble parameter ranges, tanh shear layers of thickness "
                        f"{learned.KH_SMOOTH}), coarse {args.coarse}^2, t = {0.25 * args.t_end}, "
                        f"{0.5 * args.t_end} and {args.t_end}; {len(train_seeds)} training "
                        f"seeds (fine {4 * args.coarse}^2 restricted), {len(eval_seeds)} held-out",
            "train": {"samples": int(len(X)), "steps": args.train_steps, "batch": args.batch,
                      "lr": args.lr, "loss_first": losses[0], "loss_last": losses[-1],
                      "data_seconds": t_data, "train_seconds": t_train, "noise": args.noise,
                      **fit},
            "gate": {"tv_min": tv_min, "diss_frac": diss_frac, "shock_jump": 0.5, "pos_frac": 0.02},
            "summary": sm,
            "time_ratio_learned_over_plain2x": (sm[lr_]["mean_seconds"] / sm[c2]["mean_seconds"]
                                                if sm[lr_]["mean_seconds"] else None),
            "l1_ratio_learned_over_plain": [a / b for a, b in zip(sm[lr_]["mean_l1_at_%d" % args.coarse],
                                                                  sm[c]["mean_l1_at_%d" % args.coarse])],
            "l1_ratio_learned_over_plain2x": [a / b for a, b in zip(sm[lr_]["mean_l1_at_%d" % args.coarse],
                                                                    sm[c2]["mean_l1_at_%d" % args.coarse])],
            "learned_diverged": sm[lr_]["diverged"],
            "model": args.model_out}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=None)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--repeats", type=int, default=25,
                    help="timed blocks of --steps steps each; the median block is reported")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="fast", choices=["fast", "parity"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--e2e-dtoutput", type=float, default=0.1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="kh4096",
                    choices=["kh4096", "ensemble", "learned", "configs", "slabs"])
    ap.add_argument("--train-seeds", type=int, default=16)
    ap.add_argument("--eval-seeds", type=int, default=8)
    ap.add_argument("--coarse", type=int, default=256)
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--snapshots", type=int, default=12)
    ap.add_argument("--frac", type=float, default=0.25)
    ap.add_argument("--train-steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--model-out", default="")
    ap.add_argument("--noise", type=float, default=0.03, help="training-state block noise")
    ap.add_argument("--tv-min", type=float, default=None, help="smoothness gate (default: library's)")
    ap.add_argument("--diss-frac", type=float, default=None, help="dissipation clip (default: library's)")
    ap.add_argument("--ens-n", type=int, default=64)
    ap.add_argument("--ens-tmax", type=float, default=1.0)
    ap.add_argument("--ncu-case", action="store_true",
                    help="upload and run --steps steps only (for ncu captures)")
    ap.add_argument("--box3d", type=int, default=0,
                    help="with --ncu-case: a periodic N^3 box (the 3D stage) instead of KH")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.gpus is not None and world == 1 and args.gpus > 1:
        print(json.dumps({"error": "launch N>1 with torch.distributed.run"}))
        return 2
    if args.warmup < 3 and not args.ncu_case:
        args.warmup = 3
    if args.impl == "reference":
        return main_reference(args, rank, world)
    if args.ncu_case and args.workload in ("ensemble", "learned"):
        return main_ncu_case(args, local_rank)
    if args.workload == "ensemble":
        return main_ensemble(args, rank, world, local_rank)
    if args.workload == "learned":
        return main_learned(args, rank, world, local_rank)
    if args.workload == "slabs":
        return main_slabs(args, rank, world, local_rank)
    if args.workload == "configs":
        return main_configs(args, rank, world, local_rank)
    return main_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
