"""Benchmark of the staggered-grid elastic timestep loop on B200.

A "step" is one full time step (velocity + stress update, source, receivers)
of one model.  Default workload: the random-medium cube, 344^3 interior +
20-cell split PML (384^3 computed cells, 394^3 GRID), dt 1 ms, 64x64
receivers recording vx, vy, vz, FP32.  Metric: Gcell-updates/s (computed
cells x steps / device seconds), whole job over all ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sgfd|reference]

With N > 1 (torchrun) every rank advances its own independent replica of the
model on its own GPU (no exchange step), so scaling is weak.  `--slabs N`
instead cuts the one model into z-slabs that trade 5-plane halos every half
step: N slabs on one GPU, or one slab per rank under torchrun (NCCL
send/recv; total work fixed, strong scaling).  `--impl reference` times the reference algorithm's CPU
implementation (this project's oracle port, all host threads) on rank 0 and
also reports the reference's own GPU program (compiled from its sources under
oracle/_ref/) timed on this GPU.
"""
from __future__ import annotations

import argparse
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
sys.path.insert(0, os.path.join(ROOT, "staggered-grid_b200"))

# Algorithmic bytes per computed cell and kernel launch (FP32): every field
# value read or written once per kernel.  velocity: interior reads 6 stresses
# + 3 velocities + buoyancy and writes 3 velocities; PML reads 6 stresses + 9
# velocity splits + buoyancy and writes 9 splits + 3 velocities.  stress:
# interior reads 3 velocities + 6 stresses + lambda + mu, writes 6 stresses;
# PML reads 3 velocities + 15 stress splits + lambda + mu, writes 15 splits +
# 6 stresses.  Sum per step: 120 B interior, 276 B PML.
BYTES = {"velocity": (52, 112), "stress": (68, 164)}
# DRAM traffic / algorithmic bytes per kernel, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on the 216^3 + 20 PML cube of the same kernels (REF); the
# 394^3 workload is too large for a multi-metric capture, so its traffic is
# reported as its algorithmic bytes times this ratio.
TRAFFIC_RATIO = {"velocity": 1.19, "stress": 1.32}
TRAFFIC_SOURCE = ("ncu dram bytes / algorithmic bytes of the z-march kernels (REF rounding) on the 216^3 + 20 PML "
                  "cube, times this launch's algorithmic bytes")
# 16-bit storage: fields and splits 2 B, medium 4 B (per step 66 B interior, 144 B PML).
BYTES16 = {"velocity": (28, 58), "stress": (38, 86)}
STORAGE = {"f32": 0, "bf16": 1, "f16": 2}
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["sgfd", "reference"], default="sgfd")
    p.add_argument("--workload", choices=["random344", "random472", "random216", "interior512", "interior256",
                                               "plain100", "reference_main", "batch32", "learned256", "combined32"],
                   default="random344")
    p.add_argument("--no-autotune", action="store_true", help="batch32: keep the default launch shapes")
    p.add_argument("--batch-mode", choices=["persistent", "graph"], default="graph",
                   help="batch32: graph replays with one branch per model (faster here), or one persistent launch per run")
    p.add_argument("--kernel", choices=["auto", "simple", "zmarch"], default="auto")
    p.add_argument("--tile", choices=["default", "32x8", "32x16", "64x8"], default="default",
                   help="z-marching tile shape (default: the library's choice)")
    p.add_argument("--zchunk", type=int, default=0, help="z-marching planes per chunk (0: automatic)")
    p.add_argument("--arith", choices=["ref", "fast"], default="ref",
                   help="ref: the reference's rounding (the drop-in's); fast: pre-divided coefficients")
    p.add_argument("--storage", choices=["f32", "bf16", "f16"], default="f32",
                   help="wavefield storage; 16-bit also reports errors on a 128^3 crop")
    p.add_argument("--no-accuracy", action="store_true", help="skip the accuracy leg against the FP64 oracle")
    p.add_argument("--no-large", action="store_true", help="random344: skip the 472^3 + 20 (512^3 computed) line")
    p.add_argument("--no-other-arith", action="store_true", help="skip timing the other rounding mode")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-steps", type=int, default=6, help="steps of the CPU sample")
    p.add_argument("--slabs", type=int, default=0,
                   help="one model cut into z-slabs with halo exchange: this many slabs on one GPU, or with "
                        "N > 1 one slab per rank (NCCL send/recv between neighbours)")
    return p.parse_args()


def build_workload(name):
    import sgfd.workloads as wl
    if name == "random344":
        return wl.random_cube(n_interior=344, pml=20, nt=2000)
    if name == "random472":
        return wl.random_cube(n_interior=472, pml=20, nt=3000, dt=0.0008, std=0.08, corr_m=80.0, seed=4,
                              src_computed=(256, 256, 40))
    if name == "random216":            # a smaller cube of the same kind, for ncu captures
        return wl.random_cube(n_interior=216, pml=20, nt=2000, src_computed=(128, 128, 40))
    # no PML (zero frame): the interior-cell rate alone, 512^3 and, for ncu captures, 256^3 computed
    if name == "interior512":
        return wl.random_cube(n_interior=512, pml=0, nt=2000, src_computed=(256, 256, 40))
    if name == "interior256":
        return wl.random_cube(n_interior=256, pml=0, nt=2000, src_computed=(128, 128, 40))
    if name == "plain100":
        return wl.plain_cube(n_interior=100, pml=20, nt=500)
    return wl.reference_case(nt=1500)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = (bus_id or "").lower()
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once sampling runs (its first line is out)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.05)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [l.split(", ") for l in self.lines if l.count(",") >= 8]
        if self.bus_id:
            mine = [r for r in rows if r[0].lower()[-7:] == self.bus_id[-7:]]
            rows = mine or rows
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    """Largest value over the ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells_per_rank: int, steps: int, ms_max: float, world: int) -> float:
    """Whole-job Gcell-updates/s: every rank advances its own replica."""
    return world * cells_per_rank * steps / (ms_max / 1e3) / 1e9


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_rate(w, steps: int, warm: int = 1):
    """Time the oracle port (FP32, flush-to-zero on, all host threads) on the full
    workload grid for `steps` steps after `warm` untimed steps.  Returns
    (Gcell/s, threads, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    threads = oracle_py.set_threads(os.cpu_count() or 1)
    o = oracle_py.Oracle(w.cfg, fp64=False, ftz=True)
    o.set_medium(w.b, w.lam, w.mu)
    o.set_source(*w.src)
    o.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
    wav = w.wavelet.astype(np.float64)
    o.run(wav, 0, warm)
    t0 = time.perf_counter()
    o.run(wav, warm, steps)
    dt = time.perf_counter() - t0
    o.close()
    return w.computed_cells() * steps / dt / 1e9, threads, dt


def run_reference_arm(args, w, world, rank):
    """CPU implementation of the reference algorithm on rank 0 (+ the reference's
    own GPU program, if built)."""
    if rank != 0:
        return
    steps = max(1, min(args.steps, args.cpu_steps))
    rate, threads, secs = cpu_oracle_rate(w, steps, warm=min(args.warmup, 1))
    line = {
        "impl": "reference", "metric": "Gcell-updates/s", "value": rate, "unit": "Gcell/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": min(args.warmup, 1),
        "ms_per_step": secs / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "grid": [w.cfg["nx"], w.cfg["ny"], w.cfg["nz"]], "pml": w.cfg["pml"],
                   "computed_cells": w.computed_cells()},
        "cpu_baseline": {"value": rate, "unit": "Gcell/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full time steps of the {w.name} grid after 1 untimed step; "
                                   f"C++ oracle restating the reference kernels, FP32, OpenMP {threads} threads, "
                                   f"flush-to-zero on (the reference's own CPU program implements another PML "
                                   f"and does not build unmodified)"},
        "e2e": {"value": rate, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "ref_opt")
    if os.path.exists(ref_bin):
        line["gpu_reference"] = reference_gpu_program(ref_bin, w, steps=min(max(args.steps, 20), 200))
    cpml = cpu_reference_program()
    if cpml:
        line["cpu_reference_program"] = cpml
    print(json.dumps(line), flush=True)


def cpu_reference_program(steps: int = 8):
    """The reference's own CPU program (3DCPUwithPML_3DArray_GridIncludePMLandOrder,
    its split-field PML everywhere in the PML, 3-D arrays), built from its
    sources by oracle/Makefile behind a timing harness, on its main.cpp's grid
    (101^3 interior + 10-cell PML), single thread as shipped, flush-to-zero
    off and on.  None if it was not built."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cpml_bench")
    if not os.path.exists(exe):
        return None
    out = {}
    with tempfile.TemporaryDirectory() as d:   # it writes its damping profiles to the working directory
        for ftz in (0, 1):
            r = subprocess.run([exe, "101", "10", str(steps), str(ftz)], cwd=d, capture_output=True, text=True,
                               timeout=600)
            if r.returncode != 0:
                return {"error": r.stderr[-300:]}
            tok = dict(t.split("=") for t in r.stdout.split() if t.startswith(("cells=", "steps=", "seconds=")))
            out["ftz_on" if ftz else "ftz_off"] = int(tok["cells"]) * int(tok["steps"]) / float(tok["seconds"]) / 1e9
    return {"value": out["ftz_off"], "unit": "Gcell/s", "cores": 1, "ftz_on": out["ftz_on"],
            "sample": f"{steps} steps of the reference CPU program's own case (101^3 interior + 10-cell PML, "
                      f"131^3 arrays) after 1 untimed step; its split fields cover the whole PML and its profile "
                      f"uses a constant velocity, so it does more work per PML cell than the GPU program"}


def write_case(path, w, nt):
    c = w.cfg
    with open(path, "wb") as f:
        hdr = np.array([0x43464753, 1, c["nx"], c["ny"], c["nz"], c["pml"], nt, *w.src, *w.src, 0], np.int32)
        f.write(hdr.tobytes())
        fl = np.array([c["dt"], c["dx"], c["dy"], c["dz"], 20.0, *c["coef"]], np.float32)
        f.write(fl.tobytes())
        for a in (w.b, w.lam, w.mu):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())


def reference_gpu_program(ref_bin, w, steps):
    """The reference's own single-GPU PML program (OPT/ElasticWaveEquation.cu),
    built unmodified from its sources, timed with CUDA events over `steps`
    calls of its propagate() on this workload's grid and medium."""
    with tempfile.TemporaryDirectory() as d:
        case, out = os.path.join(d, "case.bin"), os.path.join(d, "out.bin")
        write_case(case, w, steps)
        r = subprocess.run([ref_bin, case, out], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr[-300:]}
    tok = dict(t.split("=") for t in r.stdout.split()[1:])
    ms = float(tok["ms"])
    return {"value": w.computed_cells() * steps / (ms / 1e3) / 1e9, "unit": "Gcell/s", "steps": steps,
            "ms_per_step": ms / steps,
            "note": "reference OPT program (velocityUpdate/stressUpdate as shipped, 4 launches + device sync per "
                    "step), built for sm_100a from its own sources, CUDA events around its propagate() loop"}


def main():
    args = parse()
    if args.impl == "reference":
        # CPU arm: rank 0 alone runs it, no process group is needed
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            if args.workload in ("batch32", "combined32"):
                import sgfd.workloads as wl
                w = wl.layered_model(wl.batch_specs()[0])
                w.name = "batch32 (sample: model 0, %s)" % w.name
                run_reference_arm(args, w, 1, 0)
            else:
                run_reference_arm(args, build_workload(args.workload), 1, 0)
        return
    world, rank, local = dist_setup(args)
    if args.slabs:
        main_slabs(args, world, rank, local)
        return
    if args.workload in ("batch32", "combined32"):
        main_batch(args, world, rank, local)
        return
    if args.workload == "learned256":
        main_learned(args, world, rank, local)
        return
    w = build_workload(args.workload)
    import torch
    import sgfd
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    leg = timed_leg(w, args, local, world, args.arith, STORAGE[args.storage], K, W, e2e=not args.no_e2e)
    result = {
        "metric": "Gcell-updates/s", "value": leg["value"], "unit": "Gcell/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": leg["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.storage == "f32" else f"f32 arithmetic, {args.storage} storage", "data": "synthetic",
        "config": {"workload": w.name, "grid": [w.cfg["nx"], w.cfg["ny"], w.cfg["nz"]], "pml": w.cfg["pml"],
                   "computed_cells": w.computed_cells(), "interior_cells": leg["n_int"], "pml_cells": leg["n_pml"],
                   "receivers": len(w.rec_comp), "kernel": leg["kernel"], "tile": leg["tile"], "arith": args.arith,
                   "storage": args.storage, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (9 wavefields of %.0f MB each)"
                         % (w.cfg["nx"] * w.cfg["ny"] * w.cfg["nz"] * 4 / 1e6)},
        "roofline": leg["roofline"], "clocks": leg["clocks"], "gpu_launches": leg["launches"], "e2e": leg["e2e"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, secs = cpu_oracle_rate(w, args.cpu_steps)
        result["cpu_baseline"] = {
            "value": rate, "unit": "Gcell/s", "cores": threads, "kind": "port",
            "sample": f"{args.cpu_steps} full time steps of {w.name} ({secs:.1f} s) after 1 untimed step; "
                      f"C++ oracle of the reference kernels, FP32, flush-to-zero, OpenMP {threads} threads"}
        cpml = cpu_reference_program()
        if cpml:
            result["cpu_reference_program"] = cpml
    if rank == 0 and world == 1 and not args.no_accuracy:
        result["accuracy"] = accuracy_leg(w, args, local)
    # the other rounding mode on the same model, for comparison
    if not args.no_other_arith and args.storage == "f32":
        other = "fast" if args.arith == "ref" else "ref"
        o = timed_leg(w, args, local, world, other, STORAGE["f32"], K, W, e2e=False)
        result[f"arith_{other}"] = {k: o[k] for k in ("value", "ms_per_step", "clocks", "tile")} | {
            "kernel_ms": o["roofline"]["kernel_ms"], "frac": o["roofline"]["frac"]}
    # the 512^3-computed cube on which the FP32 roofline target is stated
    if args.workload == "random344" and not args.no_large:
        del w
        big = build_workload("random472")
        b = timed_leg(big, args, local, world, args.arith, STORAGE["f32"], K, W, e2e=False)
        result["random472"] = {
            "workload": big.name, "grid": [big.cfg["nx"], big.cfg["ny"], big.cfg["nz"]],
            "computed_cells": big.computed_cells(), "arith": args.arith, "value": b["value"], "unit": "Gcell/s",
            "ms_per_step": b["ms_per_step"], "steps": K, "warmup": W, "tile": b["tile"], "roofline": b["roofline"],
            "clocks": b["clocks"], "gpu_launches": b["launches"]}
        if rank == 0 and world == 1 and not args.no_accuracy:
            result["random472"]["accuracy"] = accuracy_leg(big, args, local)
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _part_launches(h, has_source: bool) -> int:
    """Kernel launches of one step of a slab run as inner and outer parts."""
    nzc = h.cfg.nz - 10
    cols, rows, zc = h.tile()
    if zc:                                # z-marching: chunk ranges [0, i0), [i0, i1), [i1, nchunks)
        nch = (nzc + zc - 1) // zc
        i0 = min(nch, (5 + zc - 1) // zc)
        i1 = max(i0, (nzc - 5) // zc)
        return 2 * sum(1 for a, b in ((0, i0), (i0, i1), (i1, nch)) if b > a)
    i0 = min(5, nzc)                      # simple kernels: plane ranges, plus source and receivers
    i1 = max(i0, nzc - 5)
    n = 2 * sum(1 for a, b in ((0, i0), (i0, i1), (i1, nzc)) if b > a)
    return n + (1 if has_source else 0) + (2 if h.nrec else 0)


def main_slabs(args, world, rank, local):
    """One model cut along z: args.slabs slabs on this GPU (world 1), or one
    slab per rank (world > 1; total work fixed, "strong" scaling).  Each step
    trades the 5 planes beside every cut twice (sgfd.slabs); timed with CUDA
    events on the stream all slab work runs on, max over ranks."""
    import torch
    import sgfd
    import sgfd.slabs as sl
    w = build_workload(args.workload)
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    nslabs = world if world > 1 else args.slabs
    arith = sgfd.ARITH_FAST if args.arith == "fast" else sgfd.ARITH_REF
    cfg = sgfd.default_config(**{**w.cfg, "device": local, "arith": arith})
    cuts = sl.plan_cuts(cfg.nz, nslabs, src_z=w.src[2])
    nt = max(w.nt, W + K + 4)
    wav = np.resize(w.wavelet, nt).astype(np.float32)
    if world > 1:
        m = sl.DistributedSlab(cfg, cuts, rank, world, local)
        handles = [m.s]
    else:
        m = sl.SlabModel(cfg, cuts)
        handles = m.slabs
    m.set_medium(w.b, w.lam, w.mu)
    m.set_source(*w.src)
    m.set_receivers(w.rec_xyz, w.rec_comp, nt)
    m.run(0, W, wav)
    torch.cuda.synchronize()
    n_int = sum(h.cell_counts()[0] for h in handles)
    n_pml = sum(h.cell_counts()[1] for h in handles)
    stream = m.stream                     # every slab's work runs on it
    clocks = ClockSampler(None)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.run(W, K, wav)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    cells = w.computed_cells()
    value = cells * K / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    # algorithmic bytes of this GPU's cells (all slabs on one GPU, this rank's slab otherwise)
    alg = (sum(v[0] for v in BYTES.values()) * n_int + sum(v[1] for v in BYTES.values()) * n_pml)
    halo = 2 * 2 * (nslabs - 1) * handles[0].halo_bytes()   # bytes crossing cuts per step, both directions
    result = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{w.name} in {nslabs} z-slabs", "grid": [cfg.nx, cfg.ny, cfg.nz],
                   "cuts": cuts, "computed_cells": cells, "arith": args.arith,
                   "parallelism": f"zslab{nslabs}" + ("" if world > 1 else " on one GPU"),
                   "halo_bytes_per_step": halo if world > 1 else 0,
                   "l2": "inputs larger than L2 (9 wavefields of %.0f MB each)" % (cfg.nx * cfg.ny * cfg.nz * 4 / 1e6)},
        "roofline": {"bound": "hbm", "kernel": "step (all slabs' kernels and halo copies)",
                     "achieved": alg / (ms / K / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg / (ms / K / 1e3) / 1e9 / peak,
                     "peak_source": peak_kind, "traffic": None},
        "clocks": clk,
        "gpu_launches": K * sum(_part_launches(h, (rank if world > 1 else k) == m.src_slab)
                                for k, h in enumerate(handles)),
        "e2e": None,
    }
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def timed_leg(w, args, local, world, arith_name, storage, K, W, e2e):
    """W untimed steps, then exactly K steps of w timed with CUDA events on the
    solver's stream (barrier and synchronize on both sides, max over ranks),
    nvidia-smi clocks sampled meanwhile; then the per-kernel launch times
    (roofline of the dominant kernel) and, with e2e, the end-to-end leg."""
    import torch
    import sgfd
    kernel = {"auto": sgfd.KERNEL_AUTO, "simple": sgfd.KERNEL_SIMPLE, "zmarch": sgfd.KERNEL_ZMARCH}[args.kernel]
    arith = sgfd.ARITH_FAST if arith_name == "fast" else sgfd.ARITH_REF
    cfg = sgfd.default_config(**{**w.cfg, "device": local, "kernel": kernel, "arith": arith, "storage": storage})
    nt = max(w.nt, W + K + 64)
    wav = np.resize(w.wavelet, nt).astype(np.float32)
    stream = torch.cuda.Stream()          # a real stream: events below see the solver's work
    torch.cuda.set_stream(stream)
    s = sgfd.Solver(cfg)
    s.set_stream(stream.cuda_stream)
    s.set_medium(w.b, w.lam, w.mu)
    s.set_source(*w.src)
    s.set_receivers(w.rec_xyz, w.rec_comp, nt)
    s.set_wavelet(wav)
    if s.kernel_name() == "zmarch" and (args.tile != "default" or args.zchunk):
        cols, rows = (int(v) for v in (args.tile if args.tile != "default" else "x".join(
            str(v) for v in s.tile()[:2])).split("x"))
        s.set_tile(cols, rows, args.zchunk)
    cells = w.computed_cells()
    n_int, n_pml = s.cell_counts()

    s.run(0, W)
    s.prepare_run()                       # graph captured and uploaded outside the timed region
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(local)
    try:
        bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except AttributeError:
        bus = None
    clocks = ClockSampler(bus)
    clocks.start()
    time.sleep(0.1)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.run(W, K)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = job_rate(cells, K, ms, world)

    # roofline of the dominant kernel (events around each kernel launch)
    P = max(3, min(K, 20))
    tv, ts = s.profile(W + K, P)
    per = {"velocity": tv / P, "stress": ts / P}
    dom = max(per, key=per.get)
    bpc = BYTES if storage == STORAGE["f32"] else BYTES16
    alg = bpc[dom][0] * n_int + bpc[dom][1] * n_pml
    peak, peak_kind = measured_peak()
    achieved = alg / (per[dom] / 1e3) / 1e9
    traffic = alg * TRAFFIC_RATIO[dom] if s.kernel_name() == "zmarch" and storage == STORAGE["f32"] else None
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
            "traffic_source": TRAFFIC_SOURCE if traffic else None,
            "alg_bytes_per_launch": alg, "avg_launch_ms": per[dom],
            "step_frac": (sum(v[0] for v in bpc.values()) * n_int + sum(v[1] for v in bpc.values()) * n_pml)
                         / (ms / K / 1e3) / 1e9 / peak,
            "kernel_ms": per}
    out = {"value": value, "ms_per_step": ms / K, "n_int": n_int, "n_pml": n_pml, "roofline": roof, "clocks": clk,
           "kernel": s.kernel_name(), "tile": "%dx%d, z chunk %d" % s.tile(), "launches": s.run_launches(K),
           "e2e": None}
    if e2e:
        out["e2e"] = end_to_end(s, w, K, world, stream, wav)
    s.close()
    torch.cuda.set_stream(torch.cuda.default_stream())
    return out


def accuracy_leg(w, args, local):
    """Relative L2 errors of this configuration's arithmetic against the FP64
    CPU oracle (exact arithmetic): traces and final vx / txx.  The CPU-sized
    plain cube runs in full; a large cube runs on the centre 128^3 crop of its
    medium for 300 steps.  16-bit storage also reports its error against the
    FP32 GPU path, and the FP32 path's own error against FP64."""
    import sgfd
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    import sgfd.workloads as wl
    cw = w if w.computed_cells() <= 150 ** 3 else wl.crop_workload(w)
    arith = sgfd.ARITH_FAST if args.arith == "fast" else sgfd.ARITH_REF

    def gpu(storage):
        s = sgfd.Solver(sgfd.default_config(**{**cw.cfg, "device": local, "arith": arith, "storage": storage}))
        s.set_medium(cw.b, cw.lam, cw.mu)
        s.set_source(*cw.src)
        s.set_receivers(cw.rec_xyz, cw.rec_comp, cw.nt)
        s.set_wavelet(cw.wavelet)
        s.run(0, cw.nt)
        out = (s.traces(), s.field(sgfd.VX), s.field(sgfd.TXX))
        s.close()
        return out

    oracle_py.set_threads(os.cpu_count() or 1)
    o = oracle_py.Oracle(cw.cfg, fp64=True)
    o.set_medium(cw.b, cw.lam, cw.mu)
    o.set_source(*cw.src)
    o.set_receivers(cw.rec_xyz, cw.rec_comp, cw.nt)
    o.run(cw.wavelet64, 0, cw.nt)
    ref64 = (o.traces(), o.field(sgfd.VX), o.field(sgfd.TXX))
    o.close()

    def rel(a, b):
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))

    names = ("traces", "vx", "txx")
    r32 = gpu(0)
    out = {"workload": cw.name, "steps": cw.nt, "arith": args.arith, "storage": args.storage,
           "vs_fp64": {n: rel(a, b) for n, a, b in zip(names, r32, ref64)}}
    if args.storage != "f32":
        r16 = gpu(STORAGE[args.storage])
        out["vs_fp64"] = {n: rel(a, b) for n, a, b in zip(names, r16, ref64)}
        out["vs_fp32"] = {n: rel(a, b) for n, a, b in zip(names, r16, r32)}
        out["fp32_vs_fp64"] = {n: rel(a, b) for n, a, b in zip(names, r32, ref64)}
    return out


def main_learned(args, world, rank, local):
    """The learned-boundary configuration: 256^3 interior with a 6-cell
    learned strip (268^3 computed cells, pml = 0, the trained network in the
    package) against the same interior with a 20-cell split-field PML (296^3
    computed), random medium (std 5 %, 50 m), Ricker 20 Hz at the centre.
    value: computed-cell updates per second of the strip model; the line
    also gives interior-cell updates per second of both, the quantity the two
    boundaries compete on."""
    import torch
    import sgfd
    import sgfd.learned as L
    import sgfd.workloads as wl
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    n_int, pml20 = 256, 20
    big = wl.random_cube(n_interior=n_int, pml=pml20, nt=W + K + 16, seed=5)
    params = L.load_params()
    out = {}
    for name, width, pml in (("learned_strip", L.WIDTH, 0), ("pml20", pml20, pml20)):
        n = n_int + 2 * width + 2 * wl.HALO
        off = pml20 - width
        cut = slice(off, off + n)
        mb, ml, mm = (np.ascontiguousarray(a[cut, cut, cut]) for a in (big.b, big.lam, big.mu))
        cfg = sgfd.default_config(**{**big.cfg, "nx": n, "ny": n, "nz": n, "pml": pml, "device": local,
                                     "arith": sgfd.ARITH_FAST if args.arith == "fast" else sgfd.ARITH_REF})
        s = sgfd.Solver(cfg)
        s.set_medium(mb, ml, mm)
        s.set_source(n // 2, n // 2, n // 2)
        s.set_wavelet(np.resize(big.wavelet, W + K + 16))
        if pml == 0:
            s.set_learned_strip(L.WIDTH, params)
        s.run(0, W)
        s.prepare_run()
        s.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        e0.record(st)
        s.run(W, K)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"ms_per_step": ms / K, "computed_cells": (n - 10) ** 3,
                     "gcell_per_s": (n - 10) ** 3 * K / ms / 1e6, "interior_gcell_per_s": n_int ** 3 * K / ms / 1e6,
                     "launches_per_step": s.launches_per_step()}
        s.close()
    ls = out["learned_strip"]
    refl = L.reflection(params, seed=999) if not args.no_accuracy else None
    result = {
        "metric": "Gcell-updates/s", "value": ls["gcell_per_s"], "unit": "Gcell/s", "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": ls["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "learned256", "interior": n_int, "strip_width": L.WIDTH, "pml_compared": pml20,
                   "arith": args.arith,
                   "computed_cells": ls["computed_cells"], "parallelism": "replicas1"},
        "comparison": out,
        "reflected_energy_over_peak": None if refl is None else
            {k: v["final_over_peak"] for k, v in refl.items()},
        "gpu_launches": ls["launches_per_step"] * K,
    }
    if rank == 0:
        print(json.dumps(result), flush=True)


def main_batch(args, world, rank, local):
    """The batched configuration: 32 layered models of uneven size (359 M
    computed cells in all), each with its own source and 128 receivers,
    advanced together by sgfd_batch_run: by default 16-step graphs with one
    branch per model and autotuned launch shapes (--batch-mode persistent: one
    persistent launch per run over all models' work items).  With N ranks the models are dealt out by computed cells (greedy,
    largest first); value = all ranks' cells x steps / slowest rank's time."""
    import dataclasses
    import torch
    import sgfd
    import sgfd.learned as L
    import sgfd.workloads as wl
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    combined = args.workload == "combined32"
    storage = args.storage if not (combined and args.storage == "f32") else "f16"
    mode = args.batch_mode if storage == "f32" else "graph"      # the persistent kernel is FP32-only
    arith = sgfd.ARITH_FAST if args.arith == "fast" else sgfd.ARITH_REF
    specs = wl.batch_specs()
    gate = None
    if combined:
        # the learned strip is used only where its gate (calibration against the
        # 20-cell PML) accepts it; otherwise every model keeps its PML
        gate = L.gate(L.load_params(), nt=400, device=local)
        if gate["boundary"] == "learned_strip":
            specs = [dataclasses.replace(sp, pml=0, n_interior=sp.n_interior + 2 * L.WIDTH,
                                         src=tuple(v - sp.pml + L.WIDTH for v in sp.src)) for sp in specs]
    cells_all = [sp.computed_cells() for sp in specs]
    mine = wl.balance(cells_all, world)[rank]
    models, media, tunings = [], [], []
    n_int = n_pml = 0
    for i in mine:
        w = wl.layered_model(specs[i])
        nt = max(w.nt, W + K + 16)
        wav = np.resize(w.wavelet, nt).astype(np.float32)
        s = sgfd.Solver(sgfd.default_config(**{**w.cfg, "device": local, "arith": arith,
                                               "storage": STORAGE[storage]}))
        s.set_medium(w.b, w.lam, w.mu)
        s.set_source(*w.src)
        s.set_receivers(w.rec_xyz, w.rec_comp, nt)
        s.set_wavelet(wav)
        if gate is not None and gate["boundary"] == "learned_strip":
            s.set_learned_strip(L.WIDTH, L.load_params())
        if not args.no_autotune and mode == "graph":
            t = s.autotune(3)
            tunings.append({"model": i, "kernel": "zmarch" if t.kernel == sgfd.KERNEL_ZMARCH else "simple",
                            "tile_rows": t.tile_rows, "zchunk": t.zchunk, "ms": round(t.ms_per_step, 4)})
        a, b = s.cell_counts()
        n_int += a
        n_pml += b
        models.append(s)
        media.append((w.b, w.lam, w.mu, len(w.rec_comp)))
    batch = sgfd.Batch(models)
    if mode == "persistent":
        batch.set_persistent(True)
    stream = torch.cuda.ExternalStream(batch.stream())
    batch.run(0, W)
    batch.synchronize()
    props = torch.cuda.get_device_properties(local)
    try:
        bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except AttributeError:
        bus = None
    clocks = ClockSampler(bus)
    clocks.start()
    time.sleep(0.1)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(W, K)
    e1.record(stream)
    e1.synchronize()
    batch.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    total_cells = sum(cells_all)
    value = total_cells * K / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    bpc = BYTES if storage == "f32" else BYTES16
    alg = (sum(v[0] for v in bpc.values()) * n_int + sum(v[1] for v in bpc.values()) * n_pml)   # this rank's bytes
    achieved = alg / (ms / K / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "batch step (all models' velocity + stress kernels, overlapped)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": None, "alg_bytes_per_launch": alg, "avg_launch_ms": ms / K}
    launches = batch.run_launches(K)

    # end to end: media upload from host arrays, K batched steps, all traces read back
    e2e = None
    if not args.no_e2e:
        for s in models:
            s.reset()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        for s, (b, lam, mu, _) in zip(models, media):
            s.set_medium(b, lam, mu)
        batch.run(0, K)
        batch.synchronize()
        for s in models:
            s.traces()
        secs = max_over_ranks(time.perf_counter() - t0, world)
        h2d = sum(3 * m[0].size * 4 for m in media) / K
        d2h = sum(m[3] * s.nt * 4 for m, s in zip(media, models)) / K
        e2e = {"value": total_cells * K / secs / 1e9, "unit": "Gcell/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": K,
               "note": "per model: sgfd_set_medium from host arrays; sgfd_batch_run of K steps; sgfd_get_traces "
                       "of every model; wall clock, max over ranks"}
    batch.close()
    for s in models:
        s.close()
    result = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if storage == "f32" else f"f32 arithmetic, {storage} storage", "data": "synthetic",
        "config": {"workload": args.workload, "models": len(specs), "computed_cells": total_cells, "storage": storage,
                   "models_this_rank": len(mine), "interior_cells_rank0": n_int, "pml_cells_rank0": n_pml,
                   "arith": args.arith, "parallelism": f"replicas{world} (models dealt by cells)",
                   "batch_mode": mode,
                   "autotune": tunings or "off",
                   "l2": "inputs larger than L2 (%.1f GB of wavefields)" % (sum(cells_all) * 36 / 1e9)},
        "roofline": roof, "clocks": clk, "gpu_launches": launches, "e2e": e2e,
    }
    if gate is not None:
        result["gate"] = {k: gate[k] for k in ("boundary", "faces_accept", "steps", "learned_final_over_peak",
                                               "pml_final_over_peak")}
    if rank == 0 and world == 1 and not args.no_accuracy:
        # the batch's smallest model alone, 300 steps, against the FP64 oracle
        k0 = min(range(len(specs)), key=lambda k: cells_all[k])
        sp = dataclasses.replace(specs[k0], nt=300)
        wa = wl.layered_model(sp)
        if gate is not None and gate["boundary"] == "learned_strip":
            result["accuracy"] = {"note": "a learned-strip model has no FP64 oracle counterpart"}
        else:
            args_acc = argparse.Namespace(**{**vars(args), "storage": storage})
            result["accuracy"] = accuracy_leg(wa, args_acc, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        w0 = wl.layered_model(specs[0])
        rate, threads, secs = cpu_oracle_rate(w0, args.cpu_steps)
        result["cpu_baseline"] = {
            "value": rate, "unit": "Gcell/s", "cores": threads, "kind": "port",
            "sample": f"{args.cpu_steps} time steps of batch model 0 ({w0.name}, {secs:.1f} s) after 1 untimed "
                      f"step; C++ oracle of the reference kernels, FP32, flush-to-zero, OpenMP {threads} threads"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def end_to_end(s, w, K, world, stream, wav):
    """The reference's run() pattern through the C ABI with host buffers
    (OPT/ElasticWaveEquation.cu:140-182): the medium uploaded from pinned host
    memory, one sgfd_step per step with the host-computed source value, and
    the receivers' samples of the K steps read back into pinned memory at the
    end (the reference's station output), all inside the timed region; wall
    clock, max over ranks."""
    import torch
    n = w.b.size
    pinned = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(3)]
    for t, a in zip(pinned, (w.b, w.lam, w.mu)):
        t.numpy()[:] = a.reshape(-1)
    nrec = len(w.rec_comp)
    out = torch.empty((K, nrec), dtype=torch.float32, pin_memory=True).numpy()
    s.reset()
    s.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    s.set_medium(*[t.numpy() for t in pinned])
    for it in range(K):
        s.step(it, float(wav[it]))
    s.trace_range(0, K, out)
    secs = time.perf_counter() - t0
    secs = max_over_ranks(secs, world)
    h2d = (3 * n * 4) / K + 4
    return {"value": world * w.computed_cells() * K / secs / 1e9, "unit": "Gcell/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": nrec * 4, "steps": K,
            "note": "medium upload (3 x GRID floats, pinned) + K x sgfd_step with the host source value + "
                    "sgfd_get_trace_range of the K steps' receiver samples (pinned), wall clock"}


if __name__ == "__main__":
    main()
