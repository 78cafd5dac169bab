"""Benchmark of the B200 PySPH particle-update path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam_break|drop|lattice3d|batched]

Default workload: the 2D dam break (320,000 fluid + 12,018 wall particles,
dx = 0.0025, summation density + Tait + momentum with Monaghan viscosity +
gravity, predictor-corrector with the CFL time step), FP32 pair sums with
Kahan compensation and FP64 state.  One bench step = one predictor-corrector
step (two rebins, two density+EOS passes, two force passes, two integrator
stages), replayed from a captured CUDA graph.  Between timed steps the L2 is
flushed by writing a 256 MiB buffer, outside the timed events.

The JSON line reports pair-interactions/s (value), steps/s, the plain FP64
GPU path on the same workload, the density error of the FP32C path against
FP64, the roofline of the dominant kernel, a CPU baseline (the oracle port on
this host) and an end-to-end figure through host buffers.

--impl reference times the reference algorithm's CPU implementation (the
C restatement in oracle/, OpenMP over all host cores) on a bounded sample of
the same workload.  Under torchrun (N > 1) every rank advances its own
independent replica (weak scaling) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("pair-interactions/s & steps/s, FP32-comp vs FP64 GPU at <=1e-5 rho "
          "error; bwd/fwd ratio")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dam_break",
                    choices=["dam_break", "dam_break_continuity", "drop", "lattice3d",
                             "batched"])
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the timed steps (no FP64 leg, e2e, per-kernel timing)")
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--pair-block", type=int, default=0)
    ap.add_argument("--stencil", type=int, default=0,
                    help="fix the cell size (support / R); default: autotuned")
    ap.add_argument("--pairs", default="auto", choices=["auto", "lists", "tiled"],
                    help="neighbour lists or shared-memory tiles; default: autotuned")
    ap.add_argument("--list-batch", type=int, default=0,
                    help="list entries the force pass loads ahead (2 or 4); default: autotuned")
    return ap.parse_args()


# ------------------------------------------------------------------ inputs
def workload(name):
    from pysph_b200 import workloads as W
    from pysph_b200.engine import continuity_scheme, fluid_scheme
    if name == "dam_break":
        arrays, types, params = W.dam_break()
        return dict(scenes=[(arrays, params)], scheme=fluid_scheme(2), dim=2, types=types,
                    desc="2D dam break, dx=0.0025, 320,000 fluid + 12,018 wall, CFL dt")
    if name == "dam_break_continuity":
        arrays, types, params = W.dam_break()
        return dict(scenes=[(arrays, params)], scheme=continuity_scheme(2, 0.5), dim=2,
                    desc="2D dam break, dx=0.0025, continuity equation + XSPH (eps 0.5), "
                         "CFL dt")
    if name == "drop":
        arrays, types, params = W.elliptical_drop(dx=0.025)
        return dict(scenes=[(arrays, dict(params, dt=1e-5))], scheme=fluid_scheme(1),
                    dim=2, types=types,
                    desc="2D elliptical drop, dx=0.025, 5,025 particles, dt=1e-5")
    if name == "lattice3d":
        arrays, types, params = W.lattice3d(n=128)
        return dict(scenes=[(arrays, dict(params, dt=1e-6))], scheme=fluid_scheme(1),
                    dim=3, desc="3D jittered 128^3 lattice (2,097,152 particles), h=1.2dx")
    if name == "batched":
        scenes = W.batched_drops(num_scenes=256, seed=0)
        return dict(scenes=[(a, p) for a, _, p in scenes],
                    scheme=fluid_scheme(1), dim=2,
                    desc="256 elliptical drops, N_s ~ U[1k,20k], dt_s = 1e-5 dx_s / 0.025")
    raise ValueError(name)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        # nvidia-smi numbers GPUs physically and ignores CUDA_VISIBLE_DEVICES:
        # name the device by its UUID so the samples are this GPU's
        self.index = gpu_id(dev)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=3.0):
        """Block until nvidia-smi has produced a sample (it needs ~0.2 s to
        start), so the samples cover the timed region that follows."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm), "gpu": self.index}


def gpu_id(dev):
    """nvidia-smi's -i argument for a torch device: its UUID (GPU-...), else
    the CUDA ordinal."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(getattr(dev, "index", dev) or 0)


# ------------------------------------------------------------------ helpers
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_over_ranks(v, world, op="max", device="cuda"):
    """Max or sum of a host scalar over the ranks (no-op on one rank); the
    only collective of the benchmark -- the replicas share no data."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(v, world):
    return reduce_over_ranks(v, world, "max")


def sum_over_ranks(v, world):
    return reduce_over_ranks(v, world, "sum")


def replica_result(ms_per_rank, pairs_per_rank, steps, world, device="cuda"):
    """Whole-job figures of independent replicas: the time is the slowest
    rank's, the work is every rank's."""
    ms = reduce_over_ranks(ms_per_rank, world, "max", device)
    pairs = reduce_over_ranks(pairs_per_rank, world, "sum", device)
    return {"ms": ms, "pairs": pairs, "value": pairs / (ms / 1e3),
            "steps_per_s": steps / (ms / 1e3)}


# DRAM bytes (read + write) per launch from `ncu --set full` on the bench's
# own workload (the dam break, FP32C, lists, 1 lane, 256-thread blocks,
# cells of half the reach, force list batches of 2; the force pass with the
# integrator stage fused into it): the mean of the two captured launches of
# each kernel (profiles/k_force_dam_break_fp32c.md,
# profiles/k_density_dam_break_fp32c.md)
NCU_TRAFFIC = {("dam_break", "fp32c", "lists", "force"): 0.5 * ((73.27e6 + 3.05e6) +
                                                                (63.03e6 + 4.72e6)),
               ("dam_break", "fp32c", "lists", "density"): 44.90e6 + 0.03e6,
               ("dam_break", "fp32c", "lists", "pc_stage"): 17.951e6 + 0.000256e6,
               # the 256 drops (block 128, the rest as above;
               # profiles/k_pairs_batched_fp32c.md)
               ("batched", "fp32c", "lists", "force"): 583.87e6 + 257.02e6,
               ("batched", "fp32c", "lists", "density"): 389.22e6 + 43.41e6}


# FP32 work of one launch from the same capture: flops = 2 FFMA + FADD +
# FMUL + 4 FFMA2 + 2 FADD2 + 2 FMUL2 (sm__sass_thread_inst_executed_op_*;
# no paired instructions were issued), and the fraction of cycles the
# schedulers issued (smsp__issue_active.avg.pct_of_peak_sustained_active)
NCU_FP32 = {("dam_break", "fp32c", "lists", "force"): {"flops": 396.3e6, "issue_active": 0.587},
            ("dam_break", "fp32c", "lists", "density"): {"flops": 225.6e6,
                                                         "issue_active": 0.663},
            ("batched", "fp32c", "lists", "force"): {"flops": 3507.2e6, "issue_active": 0.585},
            ("batched", "fp32c", "lists", "density"): {"flops": 1934.9e6,
                                                       "issue_active": 0.801}}


def fma_peaks(dev):
    """Measured FP32 and FP64 FMA rates (TFLOP/s) of this GPU: sphb_fma_probe
    on 8 full blocks per SM, the compute denominators of the pair passes'
    roofline."""
    import ctypes
    import torch
    from pysph_b200 import build as B
    L = ctypes.CDLL(B.PROBE_LIB)
    L.sphb_fma_probe.restype = ctypes.c_int
    L.sphb_fma_probe.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_void_p]
    props = torch.cuda.get_device_properties(dev)
    blocks = props.multi_processor_count * 8
    out = {}
    for name, fp64, dtype in (("fp32_tflops", 0, torch.float32), ("fp64_tflops", 1, torch.float64)):
        buf = torch.empty(blocks, dtype=dtype, device=dev)
        iters = 400 if fp64 else 1600
        stream = torch.cuda.current_stream(dev)
        def run():
            rc = L.sphb_fma_probe(fp64, buf.data_ptr(), blocks, iters, ctypes_stream(stream))
            if rc:
                raise RuntimeError(f"sphb_fma_probe failed ({rc})")
        run()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(5):
            run()
        b.record(stream)
        torch.cuda.synchronize()
        flops = 5.0 * blocks * 256 * iters * 256
        out[name] = flops / (a.elapsed_time(b) * 1e-3) / 1e12
    return out


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def algorithmic_bytes(dim, f32):
    """Bytes per particle each phase must move once, at the stored widths
    (neighbour re-reads and the neighbour lists, which are scratch, are not
    counted).  pc_stage includes the FP32 record refresh and the anchor
    read of the displacement check; bin is one full rebin."""
    if f32 and dim == 2:
        d = {"density": 16 + 4 + 4 + 16 + 16,           # geo, cell, tag; thermo r/w
             "force": 16 + 8 + 16 + 4 + 4 + 12,         # geo, vel, thermo, cell, tag; a, dt_fac
             # x,y,u,v r/w, x0..v0, tag, a; cell, geo.xy w, vel w, anchor r
             "pc_stage": 8 * 8 + 4 + 8 + 4 + 8 + 8 + 8,
             # hash x,y 16, key/slot w+r 16, perm w+r 8, key 4; gather
             # x,y,u,v,m,h,idx,tag 56 r + 56 w; cell 4, geo 16, vel 8,
             # anchor 8 w; copy back 56 r + 56 w
             "bin": 16 + 16 + 8 + 4 + 56 + 56 + 4 + 16 + 8 + 8 + 56 + 56}
    elif f32 and dim == 3:
        d = {"density": 16 + 4 + 4 + 4 + 16 + 16,
             "force": 16 + 4 + 16 + 16 + 4 + 4 + 16,
             "pc_stage": 12 * 8 + 4 + 12 + 4 + 8 + 16 + 16 + 16,
             "bin": 24 + 16 + 8 + 4 + 72 + 72 + 4 + 16 + 4 + 16 + 16 + 72 + 72}
    else:
        w = 8
        d = {"density": dim * w + 2 * w + 4 + 4 + 3 * w,
             "force": 2 * dim * w + 2 * w + 3 * w + 4 + 4 + (dim + 1) * w,
             "pc_stage": 4 * dim * w + 4 + dim * w + 4 + (8 if dim == 2 else 16),
             "bin": (dim * w + 16 + 8 + 4 + 2 * (2 * dim * w + 2 * w + 8) + 4
                     + (8 if dim == 2 else 16) + 2 * (2 * dim * w + 2 * w + 8))}
    return d


# ------------------------------------------------------------------ our arm
def launch_shape(wl, precision, args, dev, force_tune=False):
    """The engine's launch shape: fixed from the command line, else the
    autotuner's (both pair modes, every cell size / lanes / block / skin)."""
    if not force_tune and (args.lanes or args.pair_block or args.stencil or args.list_batch
                           or args.pairs != "auto"):
        pairs = "lists" if args.pairs == "auto" else args.pairs
        return dict(pairs=pairs, lanes=args.lanes or (4 if wl["dim"] == 3 else 1),
                    pair_block=args.pair_block or 128, stencil=args.stencil or 1,
                    list_batch=args.list_batch or 4, skin_margin=None), None
    from pysph_b200.autotune import autotune
    tune = autotune(wl["scenes"], wl["scheme"], wl["dim"], precision, device=dev)
    shape = {k: tune.get(k) for k in ("pairs", "lanes", "pair_block", "stencil", "list_batch",
                                      "skin_margin")}
    shape["pairs"] = shape["pairs"] or "lists"
    shape["list_batch"] = shape["list_batch"] or 4
    return shape, tune


def make_engine(wl, precision, shape, dev):
    from pysph_b200.engine import Engine
    return Engine(wl["scenes"], wl["scheme"], dim=wl["dim"], precision=precision,
                  stencil=shape["stencil"], lanes=shape["lanes"],
                  pair_block=shape["pair_block"], device=dev,
                  list_batch=shape["list_batch"], skin_margin=shape["skin_margin"],
                  pairs=shape["pairs"])


def capture_step(eng, stream):
    """One PC step captured in a CUDA graph (after a side-stream warm-up)."""
    import torch
    s = torch.cuda.Stream(eng.device)
    s.wait_stream(stream)
    with torch.cuda.stream(s):
        eng.pc_step()
    stream.wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        eng.pc_step()
    torch.cuda.synchronize()
    return g


def run_ours(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = workload(args.workload)
    shape, tune = launch_shape(wl, args.precision, args, dev)
    eng = make_engine(wl, args.precision, shape, dev)
    N = eng.N
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    # clocks are sampled from the warm-up through the end of the timed region
    clk = ClockSampler(dev).__enter__()
    # the warm-up advances the state: the timed steps are steps W+1 .. W+K of
    # the run from the workload's initial state
    for _ in range(max(args.warmup, 3)):
        eng.pc_step()
    torch.cuda.synchronize()
    eng.check_status()
    graph = None
    if not args.no_graph:
        graph = capture_step(eng, stream)
        graph.replay()
        torch.cuda.synchronize()
        eng.check_status()
    start_step = max(args.warmup, 3) + (2 if graph is not None else 0)

    def step():
        if graph is not None:
            graph.replay()
        else:
            eng.pc_step()

    # ---- timed region: K steps, L2 flushed between them
    eng.reset_pair_counts()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clk.wait_first()
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    ms = sum(starts[i].elapsed_time(ends[i]) for i in range(args.steps))
    eng.check_status()
    pairs_d, pairs_f = eng.pair_counts()
    rebins = eng.device_rebins()
    pairs = pairs_d + pairs_f
    job = replica_result(ms, pairs, args.steps, world)
    ms_max, value, steps_per_s = job["ms"], job["value"], job["steps_per_s"]

    if args.no_extras:
        out = {"metric": METRIC, "value": value, "unit": "pair-interactions/s",
               "n_gpus": world, "steps": args.steps, "ms_per_step": ms_max / args.steps,
               "steps_per_s": steps_per_s, "config": {"workload": args.workload,
                                                      "pairs": shape["pairs"]},
               "clocks": clk.summary()}
        del graph
        return out

    roof = roofline(eng, args.workload, args.precision, flush, stream,
                    rebins / (2.0 * args.steps))
    out = {"metric": METRIC, "value": value, "unit": "pair-interactions/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_max / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32+kahan pair sums, fp64 state" if eng.f32 else "fp64",
           "data": "synthetic",
           "config": {"workload": args.workload, "description": wl["desc"],
                      "particles": N, "precision": args.precision,
                      "pairs": shape["pairs"], "stencil": shape["stencil"],
                      "lanes": shape["lanes"], "pair_block": shape["pair_block"],
                      "list_batch": shape["list_batch"], "skin_margin": eng.skin_margin,
                      "cuda_graph": graph is not None,
                      "timed_steps": f"steps {start_step + 1}..{start_step + args.steps} of "
                                     "the run from the initial state",
                      "l2": "flushed (256 MiB write) between timed steps",
                      "parallelism": f"replicas x{world}"},
           "steps_per_s": steps_per_s,
           "rebins_per_stage": rebins / (2.0 * args.steps),
           "autotune": ({"chosen": {k: tune.get(k) for k in ("pairs", "stencil", "lanes",
                                                              "pair_block", "list_batch",
                                                              "skin_margin")},
                         "table": tune["table"]} if tune else None),
           "pairs_per_step": pairs / args.steps,
           "gpu_launches": launches_per_step(eng) * args.steps,
           "roofline": roof, "clocks": clk.summary()}
    del graph
    if rank == 0:
        if args.workload == "dam_break":
            out["full_run"] = full_run(wl, args.precision, shape, dev, stream, 2000)
        if args.precision == "fp32c":
            out["fp64_gpu"] = fp64_comparison(args, wl, shape, flush, stream, dev)
            out["fp64_gpu"]["fp32c_speedup_steps"] = steps_per_s / out["fp64_gpu"]["steps_per_s"]
        out["e2e"] = e2e_facade(wl, args, shape, dev, stream)
        out["e2e"]["engine_api"] = e2e_engine(eng, stream, dev, args)
        if args.precision == "fp32c":
            out["calc_by_calc"] = calc_by_calc(wl, args, shape, dev, stream)
        del eng
        torch.cuda.empty_cache()
        if args.workload == "dam_break":
            out["batched"] = batched_config(dev, flush, stream)
            out["adjoint"] = adjoint_measure(dev, stream)
            out["other_configs"] = other_configs(dev, flush, stream)
        if not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline(args, shape, dev)
    return out


def roofline(eng, workload_name, precision, flush, stream, rebins_per_stage):
    """Per-kernel times (each alone, L2 flushed) and the HBM roofline of the
    dominant kernel: its algorithmic bytes per particle times the particles
    of one launch, over its CUDA-event launch time, against the measured copy
    peak.  A stage's time weighs the kept-cells and rebinning variants by
    the rebin rate of the timed steps."""
    kern = kernel_times(eng, flush, stream)
    byts = algorithmic_bytes(eng.dim, eng.f32)
    rate = rebins_per_stage
    fused = "force_stage" in kern
    t_force = kern["force_stage"] if fused else kern["force"]
    per_stage = {"density": (1 - rate) * kern["density"] + rate * kern["density_record"],
                 "force": t_force,
                 "bin": rate * kern["rebin"] + (1 - rate) * kern.get("bin_kept", 0.0)}
    if not fused:
        per_stage["pc_stage"] = kern["pc_stage"]
    else:
        byts = dict(byts, force=byts["force"] + byts["pc_stage"])
    dominant = max(per_stage, key=lambda k: per_stage[k])
    per_launch = {"density": kern["density"], "force": t_force, "pc_stage": kern["pc_stage"],
                  "bin": kern["rebin"]}
    hbm, which = peaks()
    ach = byts[dominant] * eng.N / (per_launch[dominant] * 1e-3) / 1e9
    traffic = NCU_TRAFFIC.get((workload_name, precision, eng.pairs, dominant))
    roof = {"bound": "hbm", "kernel": dominant, "achieved": round(ach, 1),
            "peak": hbm, "peak_kind": which, "unit": "GB/s",
            "frac": round(ach / hbm, 4), "traffic": traffic,
            "traffic_note": ("dram__bytes_read.sum + dram__bytes_write.sum per launch, one ncu "
                             "capture of this workload and launch shape") if traffic else None,
            "per_kernel_ms": {k: round(v, 5) for k, v in kern.items()},
            "per_stage_ms": {k: round(v, 5) for k, v in per_stage.items()},
            "bytes_per_particle": byts}
    # the pair passes are bound by instruction issue: their FP32 flop rate
    # against the measured FMA peak, and the issue-active fraction ncu saw
    peaks_c = fma_peaks(eng.device)
    fp = NCU_FP32.get((workload_name, precision, eng.pairs, dominant))
    if fp:
        ach_c = fp["flops"] / (per_launch[dominant] * 1e-3) / 1e12
        roof["compute"] = {"bound": "fp32", "achieved": round(ach_c, 2),
                           "peak": round(peaks_c["fp32_tflops"], 2), "unit": "TFLOP/s",
                           "frac": round(ach_c / peaks_c["fp32_tflops"], 4),
                           "issue_active": fp["issue_active"],
                           "note": ("flops per launch from one ncu capture; peak from "
                                    "sphb_fma_probe on this GPU")}
    roof["fma_peaks_measured"] = {k: round(v, 2) for k, v in peaks_c.items()}
    return roof


def full_run(wl, precision, shape, dev, stream, steps):
    """The workload's whole run: `steps` PC steps from the initial state (a
    fresh engine), replayed from one captured graph in chunks timed with CUDA
    events (no L2 flush: the state, ~200 MB, exceeds the L2), with the
    device's rebin count over the run."""
    import torch
    eng = make_engine(wl, precision, shape, dev)
    eng.reset_pair_counts()
    eng.pc_step()                       # step 1 (eager)
    g = capture_step(eng, stream)       # steps 2 (warm-up) and 3 (capture)
    done = 3
    tot = 0.0
    chunk = 100
    while done < steps:
        n = min(chunk, steps - done)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            g.replay()
        b.record(stream)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
        done += n
    eng.check_status()
    st = eng.scene_state()[0]
    pd, pf = eng.pair_counts()
    rebins = eng.device_rebins()
    timed = steps - 3
    out = {"steps": steps, "timed_steps": timed, "ms_per_step": tot / timed,
           "steps_per_s": timed / (tot * 1e-3), "simulated_time_s": st.t,
           "pairs_per_step": (pd + pf) / steps,
           "rebins_per_stage": rebins / (2.0 * steps),
           "note": "steps 4..N timed (graph replays, L2 not flushed); rebins counted by the "
                   "device decisions over all N steps"}
    del g, eng
    torch.cuda.empty_cache()
    return out


def batched_config(dev, flush, stream, steps=500):
    """256 elliptical drops (N_s ~ U[1k, 20k]) advanced together, one launch
    per kernel over all scenes, under a captured CUDA graph: the autotuned
    shape, `steps` steps timed with CUDA events, per-kernel times and the
    roofline of the dominant kernel; the FP64 path on its own autotuned shape
    beside it."""
    import torch

    class A:
        pass
    args = A()
    args.lanes = args.pair_block = args.stencil = args.list_batch = 0
    args.pairs = "auto"
    wl = workload("batched")
    out = {"workload": wl["desc"]}
    for prec, nsteps in (("fp32c", steps), ("fp64", max(50, steps // 10))):
        shape, tune = launch_shape(wl, prec, args, dev)
        eng = make_engine(wl, prec, shape, dev)
        eng.pc_step()
        g = capture_step(eng, stream)
        eng.reset_pair_counts()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(nsteps):
            g.replay()
        b.record(stream)
        torch.cuda.synchronize()
        eng.check_status()
        ms = a.elapsed_time(b) / nsteps
        pd, pf = eng.pair_counts()
        rebins = eng.device_rebins()
        del g
        r = {"particles": eng.N, "scenes": eng.S, "steps": nsteps, "ms_per_step": ms,
             "steps_per_s": 1e3 / ms, "pair_interactions_per_s": (pd + pf) / nsteps / (ms / 1e3),
             "rebins_per_stage": rebins / (2.0 * nsteps),
             "shape": shape, "cuda_graph": True,
             "l2": "not flushed (the state, ~1.7 GB, exceeds the L2)"}
        if prec == "fp32c":
            r["roofline"] = roofline(eng, "batched", prec, flush, stream,
                                     r["rebins_per_stage"])
        out[prec] = r
        del eng
        torch.cuda.empty_cache()
    out["fp32c_speedup_steps"] = out["fp32c"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    return out


def other_configs(dev, flush, stream):
    """The other workloads, briefly: the dam break with the continuity
    equation and XSPH (the reference example's scheme), the elliptical drop
    (5,025) and the 3D 128^3 lattice (one evaluation), each FP32C and FP64."""
    import torch
    from pysph_b200.engine import Engine
    out = {}
    for name, steps in (("dam_break_continuity", 100), ("drop", 50)):
        wl = workload(name)
        for prec in ("fp32c", "fp64"):
            # launch shapes measured on B200 for these workloads
            shape = {"dam_break_continuity": dict(lanes=1, pair_block=256, stencil=1),
                     "drop": dict(lanes=1, pair_block=128, stencil=1)}[name]
            eng = Engine(wl["scenes"], wl["scheme"], dim=2, precision=prec, device=dev,
                         **shape)
            ms, pairs = timed_steps(eng, steps, flush, stream)
            out[f"{name}_{prec}"] = {"particles": eng.N, "scenes": eng.S,
                                     "ms_per_step": ms, "steps_per_s": 1e3 / ms,
                                     "pair_interactions_per_s": pairs / (ms / 1e3)}
            del eng
            torch.cuda.empty_cache()
    wl = workload("lattice3d")
    for prec in ("fp32c", "fp64"):
        # the launch shapes measured best for this lattice on B200: cells of
        # half the support, 1 lane per particle (FP32C) or 2 (FP64).  One
        # evaluation reuses no lists, so they carry no skin (the density pass
        # records them for the force pass of the same evaluation)
        eng = Engine(wl["scenes"], wl["scheme"], dim=3, precision=prec,
                     lanes=1 if prec == "fp32c" else 2, pair_block=128, stencil=2,
                     step_lists=False, device=dev)

        # one evaluation: rebin + SPHRho + SPHPressureGradient
        def one():
            eng.bin(0)
            eng.density(eos=False)
            eng.momentum(gravity=False, mode=1 | (16 if eng.list_cap else 0))
        for _ in range(3):
            one()
        eng.reset_pair_counts()
        tot = 0.0
        for _ in range(5):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one()
            b.record(stream)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        eng.check_status()
        pd, pf = eng.pair_counts()
        ms = tot / 5
        out[f"lattice3d_{prec}"] = {"particles": eng.N, "ms_per_evaluation": ms,
                                    "pair_interactions_per_s": (pd + pf) / 5 / (ms / 1e3)}
        del eng
        torch.cuda.empty_cache()
    return out


def timed_steps(eng, steps, flush, stream, graph=True):
    """ms per PC step of an engine (CUDA graph replay, L2 flushed between
    steps, events around each step) and pair-interactions per step."""
    import torch
    for _ in range(3):
        eng.pc_step()
    g = capture_step(eng, stream) if graph else None
    eng.reset_pair_counts()
    tot = 0.0
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if g is not None:
            g.replay()
        else:
            eng.pc_step()
        b.record(stream)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    eng.check_status()
    pd, pf = eng.pair_counts()
    del g
    return tot / steps, (pd + pf) / steps


def adjoint_measure(dev, stream):
    """Differentiable rollout: elliptical drop, 50k particles (dx = 0.0079),
    200 steps of dt = 2e-6, checkpoints every 20, FP32C forward, FP64
    adjoint; times forward and backward with CUDA events, after a warm-up
    pair that captures the rollout's graphs."""
    import torch
    from pysph_b200 import workloads as W
    from pysph_b200.adjoint import Rollout
    from pysph_b200.engine import fluid_scheme
    arrays, _, params = W.elliptical_drop(dx=0.0079)
    tarr, _, _ = W.elliptical_drop(dx=0.0079, vel_scale=110.0)
    a = arrays[0]
    n = len(a["x"])
    v0 = torch.tensor(np.stack([a["u"], a["v"]]), dtype=torch.float64, device=dev)
    vt = torch.tensor(np.stack([tarr[0]["u"], tarr[0]["v"]]), dtype=torch.float64, device=dev)
    xt = Rollout(tarr, params, fluid_scheme(1), 2, 2e-6, 200, precision="fp32c",
                 device=dev).forward({0: vt})[0][0]
    r = Rollout(arrays, params, fluid_scheme(1), 2, 2e-6, 200, checkpoint_every=20,
                precision="fp32c", device=dev)
    # warm: the first forward and backward run eagerly and capture the
    # step and segment graphs that the timed pairs replay
    xw = r.forward({0: v0})[0][0]
    r.backward({0: (2.0 * (xw - xt) / n, torch.zeros_like(xw))})
    fwds, bwds = [], []
    for _ in range(3):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        xf = r.forward({0: v0})[0][0]
        ev[1].record(stream)
        lam = {0: (2.0 * (xf - xt) / n, torch.zeros_like(xf))}
        g = r.backward(lam)
        ev[2].record(stream)
        torch.cuda.synchronize()
        fwds.append(ev[0].elapsed_time(ev[1]))
        bwds.append(ev[1].elapsed_time(ev[2]))
    fwd, bwd = statistics.median(fwds), statistics.median(bwds)
    # the adjoint kernels, each timed alone per launch at the final state
    # (CUDA events on the engine's stream, 20 launches each, L2 warm); the
    # backward runs them twice per step (once per stage)
    eng = r.adj
    r.set_state(r.get_state(r.fwd), eng)
    eng.density()
    S = r._scratch
    mom, rho = r.scheme.mom_dests, r.scheme.rho_dests

    def per_launch(fn, reps=20):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        fn()
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    kernels = {
        "force_vjp": per_launch(lambda: eng.call(
            "sphb_force_vjp", eng.cur, mom, S["lam_a"].data_ptr(), S["lam_x"].data_ptr(),
            S["lam_v"].data_ptr(), S["lam_rho"].data_ptr(), S["lam_p"].data_ptr(),
            S["lam_c"].data_ptr())),
        "eos_vjp": per_launch(lambda: eng.call(
            "sphb_eos_vjp", eng.cur, S["lam_rho"].data_ptr(), S["lam_p"].data_ptr(),
            S["lam_c"].data_ptr())),
        "density_vjp": per_launch(lambda: eng.call(
            "sphb_density_vjp", eng.cur, rho, S["lam_rho"].data_ptr(), S["lam_x"].data_ptr())),
        "density_fp64": per_launch(lambda: eng.density(reuse=True)),
    }
    eng.check_status()
    return {"workload": "elliptical drop 50k (dx=0.0079), 200 steps dt=2e-6, "
                        "checkpoints every 20, FP32C forward, FP64 adjoint",
            "particles": n, "fwd_ms": fwd, "bwd_ms": bwd, "bwd_fwd_ratio": bwd / fwd,
            "adjoint_kernel_ms": kernels,
            "runs": "median of 3 forward + backward pairs",
            "fwd_ms_runs": fwds, "bwd_ms_runs": bwds,
            "grad_norm": float(torch.linalg.norm(g[0][1]))}


def launches_per_step(eng):
    """Kernels launched per PC step (every launch counts, including the
    rebin launches that return at once when the device keeps the lists)."""
    # per bin: one cooperative k_rebin (decision, and every phase of a rebin)
    rebin = 1
    # per stage: density, force, and pc_stage unless the force pass runs it
    stage = 2 if eng.fuses_stage else 3
    # the step prologue: its own launch, or inside the first decision
    begin = 0 if eng.step_lists else 1
    return begin + 2 * rebin + 2 * stage + (2 if eng.tait_only_mask else 0)


def kernel_times(eng, flush, stream, reps=20):
    """Device time of each phase of the step, each timed alone with CUDA
    events around its own launches on the engine's stream and the L2
    flushed (256 MiB write) before every launch: the density pass of a stage
    that keeps its cells (lists: reading them; tiled: the same pass as every
    stage), the density pass after a rebin (lists: searching cells and
    recording them with the steps' skin), force, pc_stage, the force pass
    with the stage fused, a
    full rebin, and a kept-cells rebin decision (a captured graph of that bin
    call, whose kernels return at once)."""
    import torch
    from pysph_b200 import _native as nat

    def timed(fn, n=reps):
        tot = 0.0
        for _ in range(n):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / n

    mode_f = eng.force_mode | (nat.FORCE_USE_LIST if eng.list_cap else 0)
    rho = eng.scheme.rho_dests
    out = {}
    eng.bin(nat.BIN_MOVE_INITIAL)
    # recorded as the steps record them: with the skin when the lists are
    # kept across stages, so the list passes below walk lists of the steps'
    # length (on the dam break 8.18 M entries against 6.88 M without it)
    rec = nat.DENSITY_EOS | (nat.DENSITY_LIST_IF_VALID if eng.step_lists else 0)
    out["density_record"] = timed(lambda: eng.call("sphb_density", eng.cur, rho, rec))
    if eng.list_cap and eng.pairs == "lists":
        out["density"] = timed(lambda: eng.call(
            "sphb_density", eng.cur, rho, nat.DENSITY_EOS | nat.DENSITY_USE_LIST))
    else:
        out["density"] = out["density_record"]
    out["force"] = timed(lambda: eng.call("sphb_momentum", eng.cur, eng.scheme.mom_dests,
                                          1, mode_f))
    out["pc_stage"] = timed(lambda: eng.pc_stage(0))
    if eng.fuses_stage:
        # the force pass with the predictor stage in its epilogue (the
        # records it writes go to the second copy, which the rebin below
        # rewrites)
        mode_s = mode_f | nat.FORCE_STAGE(0) | nat.FORCE_NO_MAXIMA
        dests = eng.scheme.pair_dests if eng.scheme.continuity else eng.scheme.mom_dests
        out["force_stage"] = timed(lambda: eng.call("sphb_momentum", eng.cur, dests, 1, mode_s))
    out["rebin"] = timed(lambda: eng.bin(nat.BIN_MOVE_INITIAL))
    if eng.step_lists:
        # positions at the anchors: the decision keeps the cells every time
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(eng.device)
        s.wait_stream(stream)
        with torch.cuda.stream(s):
            eng.bin(nat.BIN_IF_NEEDED | nat.BIN_MOVE_INITIAL)
        stream.wait_stream(s)
        torch.cuda.synchronize()
        with torch.cuda.graph(g):
            eng.bin(nat.BIN_IF_NEEDED | nat.BIN_MOVE_INITIAL)
        torch.cuda.synchronize()
        n = 50
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            g.replay()
        b.record(stream)
        torch.cuda.synchronize()
        out["bin_kept"] = a.elapsed_time(b) / n
        assert eng.rebin_count() == 0
        del g
    out["step_begin"] = timed(eng.step_begin)
    eng.check_status()
    return out


def fp64_comparison(args, wl, shape32, flush, stream, dev):
    """The plain FP64 GPU path on the same workload, on its own autotuned
    launch shape (and, for comparison, on the FP32C shape), timed like the
    FP32C line: one captured step replayed, L2 flushed between steps."""
    import torch
    shape64, tune64 = launch_shape(wl, "fp64", args, dev, force_tune=True)
    k = max(10, args.steps // 4)
    e64 = make_engine(wl, "fp64", shape64, dev)
    for _ in range(max(args.warmup, 3)):
        e64.pc_step()
    ms, pairs = timed_steps(e64, k, flush, stream, graph=True)
    del e64
    # the FP32C shape on FP64 (lists only: the tiled passes are FP32C)
    same = dict(shape32, pairs="lists")
    e64b = make_engine(wl, "fp64", same, dev)
    for _ in range(max(args.warmup, 3)):
        e64b.pc_step()
    ms_b, _ = timed_steps(e64b, k, flush, stream, graph=True)
    del e64b
    torch.cuda.empty_cache()
    return {"steps_per_s": 1e3 / ms, "value": pairs / (ms / 1e3),
            "unit": "pair-interactions/s", "steps": k, "cuda_graph": True,
            "shape": shape64, "autotune_table": tune64["table"] if tune64 else None,
            "steps_per_s_on_fp32c_shape": 1e3 / ms_b, "fp32c_shape": same}


def e2e_engine(eng, stream, dev, args):
    """Through the engine API with host buffers driving the state: every
    step uploads the fluid's x, y, u, v from pinned host memory -- the values
    the previous step read back -- advances one PC step, and reads x, y, u,
    v, rho, p back into pinned host memory.  The step depends on the last
    read-back, so the copies cannot overlap the kernels."""
    import torch
    a = 0
    n = eng.user_n[a]
    names_in = ("x", "y", "u", "v")
    names_out = ("x", "y", "u", "v", "rho", "p")
    host = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in names_out}
    for k in names_out:
        host[k].copy_(eng.get(a, k).cpu())
    f64 = dict(dtype=torch.float64, device=dev)
    dev_in = {k: torch.empty(n, **f64) for k in names_in}
    dev_out = {k: torch.empty(n, **f64) for k in names_out}

    def device_step():
        for k in names_in:
            eng.exchange_in(a, k, dev_in[k])
        eng.invalidate_box()
        eng.pc_step()
        for k in names_out:
            eng.exchange_out(a, k, out=dev_out[k])

    for k in names_in:
        dev_in[k].copy_(host[k])
    device_step()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        device_step()
    torch.cuda.synchronize()
    k_steps = max(10, args.steps // 4)
    eng.reset_pair_counts()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(k_steps):
        for k in names_in:
            dev_in[k].copy_(host[k], non_blocking=True)
        g.replay()
        for k in names_out:
            host[k].copy_(dev_out[k], non_blocking=True)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    pd, pf = eng.pair_counts()
    rebins = eng.device_rebins()
    eng.check_status()
    del g
    return {"value": (pd + pf) / (ms / 1e3), "unit": "pair-interactions/s",
            "steps_per_s": k_steps / (ms / 1e3), "steps": k_steps,
            "rebins_per_stage": rebins / (2.0 * k_steps),
            "h2d_bytes_per_step": 8 * n * len(names_in),
            "d2h_bytes_per_step": 8 * n * len(names_out),
            "note": "each step uploads the state the previous step read back (in stream "
                    "order), one CUDA graph for the device part"}


def dam_break_solver(wl, args, shape):
    """The dam break through the reference-facing API: its ParticleArrays,
    Particles, the Solver's operations (SPHRho, TaitEquation,
    MomentumEquation, GravityForce, PositionStepping) and a
    PredictorCorrectorIntegrator, set up; returns (solver, fluid array,
    particles, params)."""
    from pysph_b200.base import api as base
    from pysph_b200.solver import api as solver
    from pysph_b200.sph import api as sph
    from pysph_b200.base.particle_types import ParticleType
    arrays, p = wl["scenes"][0]
    prec = "single" if args.precision == "fp32c" else "double"
    f = base.get_particle_array(name="fluid", type=ParticleType.Fluid, cl_precision=prec,
                                **{k: v for k, v in arrays[0].items()})
    w = base.get_particle_array(name="wall", type=ParticleType.Solid, cl_precision=prec,
                                **{k: v for k, v in arrays[1].items()})
    particles = base.Particles([f, w])
    particles.engine_options = {k: v for k, v in shape.items() if v is not None}
    Fluid, Solid = ParticleType.Fluid, ParticleType.Solid
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid, Solid],
                                        from_types=[Fluid, Solid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=p["c0"], ro=p["rho0"]),
                                        on_types=[Fluid, Solid], updates=["p", "cs"],
                                        id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=p["alpha"], beta=p["beta"]), on_types=[Fluid],
        from_types=[Fluid, Solid], updates=["u", "v"], id="mom"))
    s.add_operation(solver.SPHIntegration(sph.GravityForce.withargs(gy=p["gravity"][1]),
                                          on_types=[Fluid], updates=["u", "v"], id="grav"))
    s.add_operation_step([Fluid])
    s.set_time_step(p["dt_initial"])
    s.setup(particles)
    return s, f, particles, p


def calc_by_calc(wl, args, shape, dev, stream):
    """The integrator's general path on the dam break, for a calc list it
    does not fuse: every SPHCalc one engine pass (the same kernels, one
    operation at a time, each density and force pass searching the cells),
    the stage arithmetic in torch elementwise ops, at a fixed dt of 1e-5
    (below the CFL step, ~1.5e-5; the workload's dt_initial of 1e-4 is only
    the CFL rule's first guess).  Device-resident, CUDA events around 10
    steps after 3."""
    import torch
    if args.workload != "dam_break":
        return None
    s, f, particles, p = dam_break_solver(wl, args, shape)
    integ = s.integrator
    integ.plan = None
    for _ in range(3):
        integ.integrate(1e-5)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    k = 10
    t0.record(stream)
    for _ in range(k):
        integ.integrate(1e-5)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / k
    particles.session().engine.check_status()
    particles.session().detach()
    del s, integ, particles, f
    torch.cuda.empty_cache()
    return {"ms_per_step": ms, "steps_per_s": 1e3 / ms, "steps": k,
            "note": "Integrator.eval / step calc by calc (plan None): one engine pass per "
                    "SPHCalc, torch elementwise stepping; fixed dt 1e-5"}


def e2e_facade(wl, args, shape, dev, stream):
    """Through the reference-facing API with host (numpy) arrays: the dam
    break's Solver (dam_break_solver) and
    PredictorCorrectorIntegrator.integrate with the device CFL rule.  Every
    step sets the fluid's x, y, u, v from numpy arrays (the values the last
    step read back), integrates, and reads x, y, u, v, rho, p back into
    numpy arrays."""
    import torch
    if args.workload != "dam_break":
        return {"value": None, "note": "the facade run is the dam break's"}
    s, f, particles, p = dam_break_solver(wl, args, shape)
    integ = s.integrator
    assert integ.plan is not None, "the dam break's scheme runs fused on the engine"
    sess = integ._fused_session()
    sess.engine.update_params(cfl=p["cfl"], c0=p["c0"], dt_initial=p["dt_initial"])
    integ.plan.params = sess.engine.params[0]
    names_out = ("x", "y", "u", "v", "rho", "p")
    # the caller's host arrays: numpy views of pinned host memory, allocated
    # once, as a host driving the GPU every step would keep them
    pinned = {k: torch.empty(f.get_number_of_particles(), dtype=torch.float64).pin_memory()
              for k in names_out}
    host = {k: pinned[k].numpy() for k in names_out}
    for k in names_out:
        pinned[k].copy_(f.get(k))

    def step():
        f.set(x=host["x"], y=host["y"], u=host["u"], v=host["v"])
        integ.integrate(0.0, device_dt=True)
        # into the numpy arrays' memory: the six properties read in one get,
        # the six read-backs queued on the stream, then one wait before the
        # host touches them
        for k, t in zip(names_out, f.get(*names_out)):
            pinned[k].copy_(t, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    for _ in range(3):
        step()
    k_steps = max(10, args.steps // 4)
    eng = particles.session().engine
    eng.reset_pair_counts()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(k_steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    pd, pf = eng.pair_counts()
    rebins = eng.device_rebins()
    eng.check_status()
    n = f.get_number_of_particles()
    out = {"value": (pd + pf) / (ms / 1e3), "unit": "pair-interactions/s",
           "steps_per_s": k_steps / (ms / 1e3), "steps": k_steps,
           "rebins_per_stage": rebins / (2.0 * k_steps),
           "h2d_bytes_per_step": 8 * n * 4, "d2h_bytes_per_step": 8 * n * len(names_out),
           "api": "ParticleArray.set(numpy) -> PredictorCorrectorIntegrator.integrate "
                  "(device CFL dt) -> ParticleArray.get(x, y, u, v, rho, p) -> numpy, every "
                  "step; the numpy "
                  "arrays live in pinned host memory allocated once, the read-backs "
                  "queued together and waited for once per step",
           "rebins": "device-decided after each host write of the positions (kept while "
                     "every particle stays within half the list skin of its last rebin)",
           "shape": particles.engine_options}
    particles.session().detach()
    del s, integ, particles, f
    torch.cuda.empty_cache()
    return out


def oracle_systems(name, threads):
    """The workload's scenes as oracle systems (CPU legs only)."""
    from oracle import OracleArray, OracleSystem
    wl = workload(name)
    sc = wl["scheme"]
    systems = []
    for arrays, p in wl["scenes"]:
        oarrs = [OracleArray(f"a{i}", **{k: np.array(v, np.float64, copy=True)
                                         for k, v in a.items()})
                 for i, a in enumerate(arrays)]
        systems.append((OracleSystem(
            oarrs, dim=wl["dim"], rho_src=sc.rho_src, tait_on=sc.tait_on,
            mom_src=sc.mom_src, step_on=sc.step_on, c0=p["c0"], rho0=p["rho0"],
            gamma=p.get("gamma", 7.0), alpha=p["alpha"], beta=p["beta"],
            eta=p.get("eta", 0.1), gravity=tuple(p.get("gravity", (0, 0, 0))),
            nthreads=threads), p))
    return wl, systems


def oracle_step(osys, p):
    if p.get("cfl", 0) > 0:
        dt = osys.cfl_time_step(p["cfl"], p["c0"], p["dt_initial"])
    else:
        dt = p.get("dt", 1e-5)
    osys.pc_step(dt)


def oracle_run(name, steps, warmup, threads, max_scenes=None):
    """Time `steps` PC steps of the oracle port after `warmup` steps."""
    wl, systems = oracle_systems(name, threads)
    if max_scenes:
        systems = systems[:max_scenes]
    for _ in range(warmup):
        for osys, p in systems:
            oracle_step(osys, p)
    p0 = sum(o.pairs for o, _ in systems)
    t0 = time.perf_counter()
    for _ in range(steps):
        for osys, p in systems:
            oracle_step(osys, p)
    dt = time.perf_counter() - t0
    pairs = sum(o.pairs for o, _ in systems) - p0
    n = sum(sum(a.n for a in o.arrays) for o, _ in systems)
    return {"value": pairs / dt, "ms_per_step": 1e3 * dt / steps,
            "steps_per_s": steps / dt, "particles": n, "desc": wl["desc"]}


# timed steps of the reference's own Cython path per sample (one host
# thread: ~5 s per dam-break step on a current Xeon core)
REF_STEPS = {"dam_break": 2, "drop": 20}
REF_STEPS_MAX = {"dam_break": 8, "drop": 200}


def reference_cython(name, steps, warmup):
    """The reference's own FP64 Cython path (built from its sources into
    oracle/_ref by oracle/build_reference.py) on one host thread, through its
    own API, over `steps` steps after `warmup`; its pair count comes from the
    oracle port over the same steps (the same states, bit for bit).  None
    when the build is absent or the workload has no driver there."""
    from oracle import reference as ref
    if name not in REF_STEPS or not ref.available():
        return None
    wl = workload(name)
    arrays, p = wl["scenes"][0]
    r = ref.time_steps(arrays, wl["types"], p, wl["dim"], steps, warmup)
    o = oracle_run(name, steps, warmup, threads=os.cpu_count() or 1)
    pairs = o["value"] * o["ms_per_step"] * steps / 1e3
    return {"value": pairs / r["seconds"], "ms_per_step": 1e3 * r["seconds"] / steps,
            "steps_per_s": r["steps_per_s"], "steps": steps, "desc": wl["desc"]}


def cpu_baseline(args, shape=None, dev=None):
    """The CPU path on a bounded sample of the workload (about 10-30 s of CPU
    work): the reference's own Cython path when it is built (kind
    "reference", one thread: it has no threads), with the oracle port (C,
    1 thread) beside it; the port alone otherwise.  On the dam break the
    same leg also checks the bench's FP32C engine and the FP64 GPU path
    against the FP64 oracle (parity_vs_oracle)."""
    steps = {"dam_break": 16, "drop": 100, "lattice3d": 1, "batched": 2,
             "dam_break_continuity": 16}[args.workload]
    scenes = 16 if args.workload == "batched" else None
    r = oracle_run(args.workload, steps, 1, threads=1, max_scenes=scenes)
    sample = f"{steps} PC steps of {r['desc']}"
    if scenes:
        sample += f" (first {scenes} scenes)"
    port = {"value": r["value"], "unit": "pair-interactions/s", "cores": 1,
            "kind": "port", "sample": sample, "steps_per_s": r["steps_per_s"]}
    out = dict(port, cpu=cpu_model())
    ref = reference_cython(args.workload, REF_STEPS.get(args.workload, 0), 1)
    if ref is not None:
        out = {"value": ref["value"], "unit": "pair-interactions/s", "cores": 1,
               "kind": "reference",
               "sample": f"{ref['steps']} PC steps (after 1) of {ref['desc']} through the "
                         "reference's own Cython path",
               "steps_per_s": ref["steps_per_s"], "cpu": cpu_model(), "port": port}
    if args.workload == "dam_break" and shape is not None:
        out["parity_vs_oracle"] = parity_vs_oracle(shape, dev)
    return out


def parity_vs_oracle(shape, dev):
    """Per-quantity errors of the GPU engines against the FP64 oracle on the
    2D dam break (332,018 particles): the first evaluation (rho, p of fluid
    and walls; the fluid's accelerations, with gravity, and dt_fac) and two
    predictor-corrector steps with the CFL time step (dt, positions in
    particle spacings, velocities relative to the largest, densities).  The
    FP32C engine runs the bench's launch shape."""
    import torch
    threads = os.cpu_count() or 1
    out = {}
    for prec in ("fp32c", "fp64"):
        wl = workload("dam_break")
        arrays, p = wl["scenes"][0]
        sh = dict(shape) if prec == "fp32c" else dict(shape, pairs="lists")
        eng = make_engine(wl, prec, sh, dev)
        _, systems = oracle_systems("dam_break", threads)
        osys = systems[0][0]
        osys.update()
        osys.eval()
        eng.eval_stage()
        eng.check_status()
        B = p["c0"] ** 2 * p["rho0"] / p["gamma"]
        r = {}
        for a in range(2):
            O = osys.arrays[a]
            r[f"rho{a}_max_rel"] = float(np.max(np.abs(eng.get(a, "rho").cpu().numpy() - O.rho)
                                                / np.abs(O.rho)))
            r[f"p{a}_max_abs_over_B"] = float(np.max(np.abs(eng.get(a, "p").cpu().numpy() - O.p))
                                              / B)
        O = osys.arrays[0]
        scale = max(np.max(np.abs(O.au)), np.max(np.abs(O.av)))
        for n, ref in (("au", O.au), ("av", O.av)):
            r[f"{n}_max_abs_over_max"] = float(np.max(np.abs(eng.get(0, n).cpu().numpy() - ref))
                                               / scale)
        # (at rest every dt_fac is 0: the absolute error then)
        r["dt_fac_max_abs_over_max"] = float(
            np.max(np.abs(eng.get(0, "dt_fac").cpu().numpy() - O.dt_fac))
            / (np.max(O.dt_fac) or 1.0))
        del eng
        eng = make_engine(wl, prec, sh, dev)
        _, systems = oracle_systems("dam_break", threads)
        osys, po = systems[0]
        dts = []
        for _ in range(2):
            dt = osys.cfl_time_step(po["cfl"], po["c0"], po["dt_initial"])
            osys.pc_step(dt)
            eng.pc_step()
            dts.append(abs(eng.scene_state()[0].dt - dt) / dt)
        eng.check_status()
        O = osys.arrays[0]
        r["step2_dt_max_rel"] = max(dts)
        for n in ("x", "y"):
            r[f"step2_{n}_max_abs_over_dx"] = float(
                np.max(np.abs(eng.get(0, n).cpu().numpy() - getattr(O, n))) / 0.0025)
        vs = max(np.max(np.abs(O.u)), np.max(np.abs(O.v)))
        for n in ("u", "v"):
            r[f"step2_{n}_max_abs_over_max"] = float(
                np.max(np.abs(eng.get(0, n).cpu().numpy() - getattr(O, n))) / vs)
        for a in range(2):
            Oa = osys.arrays[a]
            r[f"step2_rho{a}_max_rel"] = float(
                np.max(np.abs(eng.get(a, "rho").cpu().numpy() - Oa.rho) / np.abs(Oa.rho)))
        out[prec] = r
        del eng
        torch.cuda.empty_cache()
    out["oracle"] = "oracle/sph_oracle.c (FP64), all host threads"
    return out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ------------------------------------------------------------ reference arm
def run_reference(args, rank, world):
    """The reference's CPU implementation of the path on this host: its own
    Cython build (oracle/_ref) where it is built and drives the workload,
    on its one thread, over a bounded number of steps; else the oracle port
    on every host core."""
    if rank != 0:
        return None
    ncores = os.cpu_count() or 1
    ref = None
    if args.workload in REF_STEPS:
        steps = max(1, min(args.steps, REF_STEPS_MAX[args.workload]))
        ref = reference_cython(args.workload, steps, min(args.warmup, 1))
    if ref is not None:
        cores, kind = 1, "reference"
        sample = (f"{ref['steps']} PC steps (after {min(args.warmup, 1)}) of {ref['desc']} "
                  "through the reference's own Cython path (one thread: it has no threads)")
        res = {"value": ref["value"], "ms_per_step": ref["ms_per_step"], "sample": sample}
    else:
        scenes = 32 if args.workload == "batched" else None
        r = oracle_run(args.workload, args.steps, args.warmup, threads=ncores,
                       max_scenes=scenes)
        sample = f"{args.steps} PC steps of {r['desc']} (the oracle port)"
        if scenes:
            sample += f" (first {scenes} scenes)"
        cores, kind = ncores, "port"
        res = {"value": r["value"], "ms_per_step": r["ms_per_step"], "sample": sample}
    out = {"metric": METRIC, "impl": "reference", "value": res["value"],
           "unit": "pair-interactions/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp64", "data": "synthetic",
           "config": {"workload": args.workload, "sample": res["sample"]},
           "cpu_baseline": {"value": res["value"], "unit": "pair-interactions/s",
                            "cores": cores, "kind": kind, "sample": res["sample"]},
           "e2e": {"value": res["value"], "unit": "pair-interactions/s",
                   "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return out


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if rank == 0:
            print(json.dumps(out))
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    out = run_ours(args, rank, world, local)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
