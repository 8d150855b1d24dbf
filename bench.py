"""Benchmark: FDTD cell-update throughput of the dispersive 256^3 workload on B200.

Workload (one "step" = one leapfrog time step over the whole grid): 256^3 cells
with 12-cell CPML, a radius-60 Lorentz sphere, a 40-cell Drude slab, an x-normal
plane wave through a TFSF box and 16-frequency running DFTs on two flux planes
and a closed six-face flux box; FP32 fields.  Inputs are synthetic (seeded
scene builders), resident in HBM before the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs one independent replica per GPU (launched by torch.distributed.run);
the job value is the sum of all ranks' cell updates over the max rank time.
``--impl reference`` times the reference algorithm's CPU restatement (the
oracle, FP32, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "witwin-maxwell_b200"
METRIC = "Gcell-updates/s"
WORKLOAD = "dispersive_256: 256^3 cells, 12-cell CPML, Lorentz sphere r=60 + Drude slab, TFSF plane wave, 16-freq DFT on 2 flux planes + closed flux box"


def load_package():
    import importlib.util

    name = "witwin_maxwell_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        exe = shutil.which("nvidia-smi")
        if exe is None:
            return
        self.proc = subprocess.Popen(
            [exe, f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200", "-i", str(self.gpu_index)],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm, sm_max, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                sm_max.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(sm_max) if sm_max else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_workload_run(wm, steps: int, warmup: int, threads: int, budget_s: float | None = None) -> dict:
    """The workload (full 256^3 grid) stepped by the oracle in FP32 on `threads`
    host threads: `warmup` untimed steps, then `steps` timed ones, or as many as
    fit in `budget_s` seconds when that is given (at least two)."""
    from oracle import oracle as orc

    orc.build()
    total = warmup + max(steps, 2) + (64 if budget_s else 2)
    cs = wm.compile_scene(wm.workloads.dispersive_256(), total)
    sim = orc.OracleSimulation(cs, "f32", threads=threads)
    for _ in range(warmup):
        sim.step_once()
    done = 0
    t0 = time.perf_counter()
    while True:
        sim.step_once()
        done += 1
        elapsed = time.perf_counter() - t0
        if budget_s is None and done >= steps:
            break
        if budget_s is not None and done >= 2 and (elapsed >= budget_s or done >= total - warmup - 2):
            break
    sim.close()
    return {"cells": int(cs.cells), "steps": done, "elapsed_s": elapsed, "value": cs.cells * done / elapsed / 1e9,
            "compiled": cs}


def cpu_baseline_entry(run: dict, threads: int, what: str) -> dict:
    return {
        "value": run["value"], "unit": METRIC, "cores": threads, "kind": "port",
        "cpu_model": cpu_model(), "host_threads": os.cpu_count(),
        "sample": f"{run['steps']} steps of the full 256^3 workload ({what}), FP32 C oracle (the reference's "
                  f"algorithm restated), {threads} threads, {run['elapsed_s']:.1f} s",
    }


def reference_gpu_bar(wm, cs, span: int = 8, reps: int = 5) -> dict:
    """The reference's own CUDA ops (built from its sources into oracle/_ref) on
    the same scene tensors, stepped in the reference's order with its own FP32
    observer kernels (monitors on), captured into CUDA graphs of `span` and
    2 * `span` steps; ms per step = (T(2 span) - T(span)) / span, the two-point
    slope of the median replay times (CUDA events)."""
    import torch

    from oracle import ref_gpu

    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref not built"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    sim = ref_gpu.RefGpuSimulation(cs, monitor_ops=True)
    sim.run(3)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    graphs = {}
    for n in (span, 2 * span):
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            sim.run(1)
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            sim.run(n)
        graphs[n] = g
    times = {}
    for n, g in graphs.items():
        g.replay()
        torch.cuda.synchronize()
        samples = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            g.replay()
            b.record()
            b.synchronize()
            samples.append(a.elapsed_time(b))
        times[n] = statistics.median(samples)
    ms = (times[2 * span] - times[span]) / span
    del graphs, sim
    torch.cuda.empty_cache()
    return {
        "ms_per_step": ms,
        "value": cs.cells / (ms * 1e-3) / 1e9,
        "unit": METRIC,
        "what": "the reference's CUDA ops compiled for sm_100 from its own sources, stepped in its order "
                "(stepping.py:1740-1815, 2295-2330) with its FP32 observer kernels per (region, frequency), "
                "CUDA-graph captured, two-point slope of graph replays",
        "graph_ms": {str(k): v for k, v in times.items()},
    }


def run_reference_arm(args, wm, world, rank):
    """The reference's algorithm on the host cores (the FP32 C oracle, all host
    threads) over the full workload, and beside it the reference's own CUDA ops
    from oracle/_ref on the GPU (graph-captured, monitors on)."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    run = cpu_workload_run(wm, args.steps, args.warmup, threads)
    value = run["value"]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": run["elapsed_s"] * 1e3 / run["steps"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": run["cells"]},
        "cpu_baseline": cpu_baseline_entry(run, threads, f"after {args.warmup} warm-up steps"),
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.reference_gpu:
        try:
            line["reference_gpu"] = reference_gpu_bar(wm, wm.compile_scene(wm.workloads.dispersive_256(), 64))
        except Exception as exc:  # reported beside the CPU value, never fatal
            line["reference_gpu"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    return line


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# step kernels of one step of the full 256^3 workload, from one ncu capture of
# this launch shape (kernel name -> bytes); the capture and its command are
# summarised in profiles/.  Reported as `traffic` only when the run used the
# same kernels and grid; null otherwise.
NCU_TRAFFIC = {
    "cells": 256 ** 3,
    "kernels": {"warp_step_kernel<1,1,1,4,0>": 1055.3e6, "ade_pass_kernel": 372.1e6},
    "launch": {"variant": 2, "chunk_planes": 13},
}


def measured_traffic(info, cells):
    rec = NCU_TRAFFIC
    if (info["variant"], info["chunk_planes"]) != (rec["launch"]["variant"], rec["launch"]["chunk_planes"]):
        return None
    if int(cells) != rec["cells"]:
        return None
    return int(sum(rec["kernels"].values()))


def run_b200_arm(args, wm, world, rank, local):
    import torch

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    total_steps = args.warmup + args.steps + 16
    sc = wm.workloads.dispersive_256(cells=args.cells)
    t_compile = time.perf_counter()
    cs = wm.compile_scene(sc, total_steps)
    t_compile = time.perf_counter() - t_compile
    solver = wm.solver.B200FDTD(cs, device=device, sample_block=args.sample_block).init_field()
    if args.autotune:
        solver.autotune()
    # warm-up steps (untimed), then the kernel-only timing used for the roofline
    solver.step_range(0, args.warmup)
    kernel_ms = solver.time_kernel(args.warmup, 8)
    solver.step_range(args.warmup, args.warmup + 2)
    info0 = solver.info()
    torch.cuda.synchronize(device)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    n0 = args.warmup + 2
    ms = solver.step_range(n0, n0 + args.steps)  # CUDA events on the engine stream, synchronized
    torch.cuda.synchronize(device)
    barrier(world)
    clock_info = clocks.stop()
    info1 = solver.info()
    launches = info1["launches"] - info0["launches"]
    elapsed_s = max_over_ranks(ms * 1e-3, world, device)
    cells = cs.cells
    value = cells * args.steps * world / elapsed_s / 1e9
    bytes_alg = wm.workloads.algorithmic_bytes(cs)
    peaks = measured_peaks()
    achieved = bytes_alg["step_kernel"] * cells / (kernel_ms * 1e-3) / 1e9
    result = {
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed_s * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD if args.cells == 256 else f"{WORKLOAD} (scaled to {args.cells}^3 cells)",
            "cells": int(cells),
            "nodes": list(cs.nodes),
            "frequencies": len(cs.frequencies),
            "monitor_points": int(solver.n_samples),
            "launch": {"variant": info1["variant"], "chunk_planes": info1["chunk_planes"], "grid": [info1["grid_x"], info1["grid_y"]], "block": info1["block"]},
            "sample_block": args.sample_block,
            "l2": "working set (~2.5 GB of fields, psi, ADE state, monitor buffers) far larger than the 126 MB L2; no flush needed",
            "parallelism": f"replicas x{world}",
        },
        "roofline": {
            "bound": "hbm",
            "kernel": ("step kernels: tile_step_kernel (+ warp_step_kernel on the CTAs that meet a CPML slab) "
                       "+ ade_pass_kernel (one step)") if info1["variant"] == 10 else
                      "step kernels: warp_step_kernel + ade_pass_kernel (one step)",
            "achieved": achieved,
            "peak": peaks["hbm_gbs"],
            "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"],
            "peak_source": peaks["source"],
            "bytes_per_cell_update": bytes_alg["step_kernel"],
            "kernel_ms": kernel_ms,
            "traffic": measured_traffic(info1, cells),
            "traffic_unit": "bytes per step, both kernels (dram__bytes_read.sum + dram__bytes_write.sum)",
        },
        "algorithmic_bytes_per_cell_update": {k: round(v, 3) for k, v in bytes_alg.items() if k != "cells"},
        # algorithmic bytes of the whole step (the per-step DFT read-modify-write
        # of every monitor point counted as the reference does it) over the timed
        # steps, which include every DFT flush of those steps; the engine moves
        # fewer bytes (the flush accumulates 32 steps per pass)
        "whole_step_alg_frac": bytes_alg["total"] * cells * args.steps * world / elapsed_s / 1e9 / peaks["hbm_gbs"],
        "clocks": clock_info,
        "gpu_launches": int(launches),
        "compile_s": t_compile,
    }
    solver.close()
    del solver
    torch.cuda.empty_cache()
    # ---------------- end to end through the public API, host buffers ----------------
    if args.e2e:
        result["e2e"] = run_e2e(args, wm, cs, device, world)
    if args.reduced:
        result["reduced_storage"] = run_reduced_bench(args, wm, cs, device, kernel_ms, elapsed_s * 1e3 / args.steps)
    if args.vacuum:
        result["vacuum_kernels"] = run_vacuum_kernels(wm, device)
    if args.batched:
        result["batched"] = run_batched_bench(wm, device)
    if args.grating:
        result["bloch_grating"] = run_grating_bench(wm, device)
    if args.adjoint:
        result["adjoint"] = run_adjoint_bench(wm, device)
    if rank == 0 and args.cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            run = cpu_workload_run(wm, 0, 2, threads, budget_s=12.0)
            result["cpu_baseline"] = cpu_baseline_entry(run, threads, "after 2 warm-up steps, about 12 s")
        except Exception as exc:  # the CPU baseline is reported, never fatal
            result["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "port",
                                      "sample": f"failed: {exc}"}
    return result


def _joint_rel_l2(got: dict, ref: dict) -> float:
    num = sum(float(np.linalg.norm(np.asarray(got[k], np.complex128).ravel() - np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    den = sum(float(np.linalg.norm(np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    return (num / den) ** 0.5 if den > 0 else 0.0


def run_reduced_bench(args, wm, cs, device, fp32_kernel_ms, fp32_step_ms):
    """FP16 / BF16 field storage (FP32 arithmetic): step-kernel time against FP32 on
    the workload, and each monitor's relative L2 against the FP32 engine after the
    workload's 2000 steps on its stable copy (the Drude slab stopped at the CPML:
    as specified the slab runs through the CPML and the field grows without bound
    after step ~800, which overflows FP16).  The FP32 engine itself is within 2e-6
    of the FP64 oracle on this workload scaled to 96^3 (tests/test_reference_gpu.py;
    tests/test_precision.py holds the FP64-oracle bars of the reduced forms)."""
    import torch

    steps = 2000  # the dispersive workload's step count
    cs_time = cs
    cs = wm.compile_scene(wm.workloads.dispersive_256(cells=args.cells, slab_through_pml=False), steps + 8)
    out = {"steps_compared": steps, "reference": "FP32 engine, same scene and steps",
           "error_scene": "dispersive_256 with the Drude slab stopped at the CPML (stable over 2000 steps)"}
    runs = {}
    for st in ("fp32", "fp16", "bf16"):
        solver = wm.solver.B200FDTD(cs_time, device=device, sample_block=args.sample_block, storage=st).init_field()
        solver.step_range(0, 4)
        k_ms = solver.time_kernel(4, 8) if st != "fp32" else fp32_kernel_ms
        solver.close()
        solver = wm.solver.B200FDTD(cs, device=device, sample_block=args.sample_block, storage=st).init_field()
        ms = solver.step_range(0, steps)
        runs[st] = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
        if st != "fp32":
            out[st] = {
                "kernel_ms": k_ms,
                "kernel_speedup_vs_fp32": fp32_kernel_ms / k_ms,
                "step_ms": ms / steps,
                "gcell_updates_per_s": cs.cells * steps / (ms * 1e-3) / 1e9,
                "scales": solver.storage_scales()[1],
            }
        else:
            out["fp32_step_ms"] = ms / steps
        solver.close()
        torch.cuda.empty_cache()
    norms = {m: sum(float(np.linalg.norm(v)) ** 2 for v in d.values()) ** 0.5 for m, d in runs["fp32"].items()}
    top = max(norms.values()) if norms else 0.0
    # monitors whose spectrum is below 1e-3 of the strongest carry no signal to compare
    live = [m for m in norms if norms[m] > 1e-3 * top]
    out["monitors_below_signal"] = sorted(set(norms) - set(live))
    for st in ("fp16", "bf16"):
        errs = {m: _joint_rel_l2(runs[st][m], runs["fp32"][m]) for m in live}
        out[st]["monitor_rel_l2_vs_fp32"] = {m: float(f"{e:.3e}") for m, e in errs.items()}
        out[st]["max_monitor_rel_l2_vs_fp32"] = max(errs.values())
        out[st]["algorithmic_bytes_per_cell_update"] = round(wm.workloads.algorithmic_bytes(cs, storage_bytes=2)["step_kernel"], 3)
    return out


def run_vacuum_kernels(wm, device, cells: int = 256):
    """The step kernels on a CPML-free scene (cells^3 vacuum, PEC faces, Ez
    dipole): the row-tile kernel (launch variant 10, the default of such
    engines) against the warp kernel (variant 2), device time of one launch
    (CUDA events over 10 back-to-back launches, best of 3), with the HBM
    fraction of the 48 B/cell field traffic."""
    import torch

    sc = wm.Scene(cells=(cells,) * 3, spacing=25e-9, pml_cells=0, boundary=(4,) * 6)
    sc.sources.append(wm.PointDipole((cells // 2,) * 3, "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    cs = wm.compile_scene(sc, 64)
    peak = measured_peaks()["hbm_gbs"]
    bytes_cell = wm.workloads.algorithmic_bytes(cs)["step_kernel"]
    out = {"workload": f"vacuum_{cells}: {cells}^3 cells, PEC faces, Ez dipole", "bytes_per_cell_update": bytes_cell}
    for variant in (10, 2):
        s = wm.solver.B200FDTD(cs, device=device).init_field()
        s.set_launch(variant, 1, 0)
        s.step_range(0, 8)
        ms = min(s.time_kernel(8, 10) for _ in range(3))
        info = s.info()
        s.close()
        torch.cuda.empty_cache()
        gbs = bytes_cell * cs.cells / (ms * 1e-3) / 1e9
        out[f"variant_{variant}"] = {"kernel_ms": ms, "chunk_planes": info["chunk_planes"], "achieved_gbs": gbs,
                                     "frac": gbs / peak}
    out["speedup_tile_over_warp"] = out["variant_2"]["kernel_ms"] / out["variant_10"]["kernel_ms"]
    return out


def run_batched_bench(wm, device, steps: int = 256):
    """32 independent anisotropic design scenes (cell counts per axis ~ U{64..192},
    seeded): the batch (one CUDA graph replay per 32-step block, scenes on their
    own streams, launch shapes from the per-size-class autotune) against the same
    scenes stepped one after another, device time."""
    import torch

    scenes = wm.workloads.batched_designs()
    compiled = [wm.compile_scene(sc, steps + 64) for sc in scenes]
    cells = sum(c.cells for c in compiled)
    solvers = [wm.solver.B200FDTD(c, device=device).init_field() for c in compiled]
    for sv in solvers:
        sv.step_range(0, 32)
    seq_ms = sum(sv.step_range(32, 32 + steps) for sv in solvers)
    for sv in solvers:
        sv.close()
    torch.cuda.empty_cache()
    solvers = [wm.solver.B200FDTD(c, device=device).init_field() for c in compiled]
    batch = wm.solver.B200Batch(solvers)
    t0 = time.perf_counter()
    batch.autotune()
    tune_s = time.perf_counter() - t0
    batch.step_range(0, 32)
    ms = batch.step_range(32, 32 + steps)
    info = batch.info()
    batch.close()
    for sv in solvers:
        sv.close()
    torch.cuda.empty_cache()
    return {
        "workload": "batched_designs: 32 scenes, cells per axis ~ U{64..192} (seed 1), 8-cell CPML, 4-8 diagonal "
                    "anisotropic eps boxes, Ez dipole, 8-frequency point monitor",
        "cells_total": int(cells),
        "steps": steps,
        "batched_ms": ms,
        "batched_gcell_updates_per_s": cells * steps / (ms * 1e-3) / 1e9,
        "sequential_ms": seq_ms,
        "sequential_gcell_updates_per_s": cells * steps / (seq_ms * 1e-3) / 1e9,
        "speedup": seq_ms / ms,
        "autotune_s": tune_s,
        "graph_launches": info["graph_launches"],
    }


def run_grating_bench(wm, device, steps: int = 64, warmup: int = 8):
    """The large Bloch grating (512x512x384 cells, Bloch x/y with k_x = 0.1 * 2 pi / L_x,
    16-cell CPML on z, Debye grating, 32-frequency diffraction plane): a complex field
    stepped as a pair of real engines coupled on the Bloch faces, device time of a
    bounded number of steps; a complex cell update counts once."""
    import torch

    t0 = time.perf_counter()
    cs = wm.compile_scene(wm.workloads.bloch_grating(), warmup + steps + 4)
    compile_s = time.perf_counter() - t0
    timed = {}
    for storage in ("fp32", "bf16"):
        solver = wm.solver.B200FDTD(cs, device=device, storage=storage).init_field()
        solver.step_range(0, warmup)
        timed[storage] = solver.step_range(warmup, warmup + steps)
        solver.close()
        del solver
        torch.cuda.empty_cache()
    ms = timed["fp32"]
    return {
        "workload": "bloch_grating: 512x512x384 cells, Bloch x/y (k_x = 0.1 * 2 pi / L_x), 16-cell CPML on z, "
                    "Debye grating layer (64-cell period, 50 % duty), pulsed Ex plane wave through a TFSF slab on z "
                    "(the reference's grating slab), 32-frequency diffraction plane",
        "cells": int(cs.cells),
        "steps": steps,
        "ms_per_step": ms / steps,
        "gcell_updates_per_s": cs.cells * steps / (ms * 1e-3) / 1e9,
        "channels": 2,
        "bf16_storage": {"ms_per_step": timed["bf16"] / steps,
                         "gcell_updates_per_s": cs.cells * steps / (timed["bf16"] * 1e-3) / 1e9},
        "compile_s": compile_s,
    }


def run_adjoint_bench(wm, device):
    """Forward + adjoint gradient of the 160x160x96 design workload (3000 steps)
    against a plain forward solve of the same scene, device time on the engine's
    stream.  Two history modes: "store" keeps the design-box E history of every
    step in HBM (2.4 GB here, no replay); "replay" keeps a full-state checkpoint
    every 100 steps and re-runs each segment during the backward pass, each
    replayed step restricted to the design block's domain of dependence
    ("replay_full_steps": whole replayed steps, for comparison; "replay_stride_50":
    a checkpoint every 50 steps)."""
    import torch

    steps, stride = 3000, 100
    modes = {"store": {"history": "store"}, "replay": {"history": "replay"},
             "replay_full_steps": {"history": "replay", "replay_region": False},
             "replay_stride_50": {"history": "replay", "stride": 50}}
    scene = wm.workloads.adjoint_160(steps)
    eps_r = scene.material_regions[0].eps_r
    out = {
        "workload": "adjoint_160: 160x160x96 cells, 10-cell CPML, 64x64x16 design block eps_r~U[1,12), "
                    "300 THz ramped CW, |E|^2 over a 16x16 patch",
        "steps": steps,
        "design_cells": int(np.prod(eps_r.shape)),
        "gradient_check": "tests/test_adjoint_golden.py: the reference's adjoint ops (golden, 1e-4); tests/test_adjoint.py: exact transpose and FP64 central differences on 16 seeded cells of the half-size layout",
    }
    cs = None
    grads = {}
    for mode, kw in modes.items():
        kw = dict(kw)
        st = kw.pop("stride", stride)
        problem = wm.adjoint.DesignProblem(scene, steps, stride=st, device=str(device), **kw)
        mons = problem.forward(eps_r)
        g = problem.backward({"patch": {c: 2.0 * v for c, v in mons["patch"].items()}})
        grads[mode] = g
        out[mode] = {"forward_ms": problem.timings["forward_ms"], "backward_ms": problem.timings["backward_ms"]}
        if kw["history"] == "replay":
            out[mode]["checkpoint_stride"] = st
        cs = problem.solver.compiled
        problem.close()
        torch.cuda.empty_cache()
    plain = wm.solver.B200FDTD(cs, device=device).init_field()
    plain_ms = plain.step_range(0, steps)
    plain.close()
    torch.cuda.empty_cache()
    out["forward_plain_ms"] = plain_ms
    for mode in modes:
        out[mode]["fwd_adj_over_fwd"] = (out[mode]["forward_ms"] + out[mode]["backward_ms"]) / plain_ms
    out["fwd_adj_over_fwd"] = out["store"]["fwd_adj_over_fwd"]
    den = float(np.abs(grads["replay"]).max())
    out["store_vs_replay_max_rel_diff"] = float(np.abs(grads["store"] - grads["replay"]).max() / den) if den else 0.0
    out["region_replay_equals_full_replay"] = bool(np.array_equal(grads["replay"], grads["replay_full_steps"]))
    return out


def run_xslab_arm(args, wm, world, rank, local):
    """Strong scaling of one dispersive workload split into x slabs over the ranks
    (``--decomp xslab``; witwin-maxwell_b200/distributed.py): every rank steps its
    slab with one ghost plane per cut and exchanges halo planes with its chain
    neighbours once per step (NCCL point-to-point).  Only the one-rank form runs
    on a single GPU; the exchange itself is tested on CPU ranks (gloo) and as
    ranks of one process on one GPU."""
    import torch

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    total = args.warmup + args.steps + 4
    cs = wm.compile_scene(wm.workloads.dispersive_256(cells=args.cells), total)
    run = wm.distributed.XSlabRun(cs, rank, world, device=device, sample_block=args.sample_block)
    for n in range(args.warmup):
        run.step(n)
    torch.cuda.synchronize(device)
    barrier(world)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for n in range(args.warmup, args.warmup + args.steps):
        run.step(n)
    ev[1].record()
    ev[1].synchronize()
    barrier(world)
    elapsed_s = max_over_ranks(ev[0].elapsed_time(ev[1]) * 1e-3, world, device)
    run.close()
    return {
        "metric": METRIC, "value": cs.cells * args.steps / elapsed_s / 1e9, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_s * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": int(cs.cells), "parallelism": f"x-slabs x{world}",
                   "slab_planes": [list(r) for r in wm.distributed.split_planes(cs.nodes[0], world)],
                   "l2": "working set far larger than the 126 MB L2; no flush needed"},
    }


def run_e2e(args, wm, cs, device, world):
    """Gcell-updates/s of Simulation-style solve from host buffers: upload the compiled
    scene tensors from host memory, run the steps, read the monitor spectra back."""
    import torch

    h2d = 0
    for arr in [*cs.inv_e, *cs.inv_h, *[x for v in cs.cpml.values() for x in v]]:
        h2d += arr.nbytes
    for n in cs.curl:
        if cs.curl[n] is not None:
            h2d += cs.curl[n].nbytes
    for p in cs.poles:
        h2d += p.drive.nbytes + p.inv_eps.nbytes
    for p in cs.patches:
        h2d += p.coeff.nbytes + p.signal.nbytes
    for lp in cs.line_patches:
        h2d += lp.coeff.nbytes + lp.sample_index.nbytes
    if cs.aux_line is not None:
        h2d += cs.aux_line.source.nbytes
    # the caller's inputs in pinned host memory (the large per-cell arrays; the
    # small ones stay numpy), made before the timed region
    cs_host = wm.solver.pin_scene(cs)
    # one untimed short solve first (module loading, allocator warm-up), as the
    # device-timed legs have their warm-up steps
    warm = wm.solver.B200FDTD(cs_host, device=device, sample_block=args.sample_block).init_field()
    warm.step_range(0, min(args.warmup, args.steps))
    warm.monitor_results(host=True)
    warm.close()
    torch.cuda.synchronize(device)
    barrier(world)
    t0 = time.perf_counter()
    solver = wm.solver.B200FDTD(cs_host, device=device, sample_block=args.sample_block).init_field()
    solver.step_range(0, args.steps)
    host = solver.monitor_results(host=True)
    torch.cuda.synchronize(device)
    elapsed = time.perf_counter() - t0
    barrier(world)
    elapsed = max_over_ranks(elapsed, world, device)
    d2h = sum(v.numel() * v.element_size() for d in host.values() for v in d.values())
    solver.close()
    return {
        "value": cs.cells * args.steps * world / elapsed / 1e9,
        "unit": METRIC,
        "h2d_bytes_per_step": int(round(h2d / args.steps)),
        "d2h_bytes_per_step": int(round(d2h / args.steps)),
        "h2d_bytes_per_solve": int(h2d),
        "d2h_bytes_per_solve": int(d2h),
        "what": f"one solve of {args.steps} steps through B200FDTD: scene upload from host memory (the per-cell "
                "coefficient and pole arrays pinned, wm.solver.pin_scene; the small ones numpy), engine build, "
                "stepping, spectra read-back into pinned host tensors (monitor_results(host=True)), after one "
                "untimed short solve; the per-step bytes are the solve's bytes over its steps",
        "wall_s": elapsed,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--sample-block", type=int, default=32)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-reduced", dest="reduced", action="store_false",
                    help="skip the FP16 / BF16 field-storage timing and error")
    ap.add_argument("--no-vacuum", dest="vacuum", action="store_false",
                    help="skip the row-tile against warp kernel timing on a 256^3 vacuum scene")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the 32-scene batched design workload")
    ap.add_argument("--no-grating", dest="grating", action="store_false",
                    help="skip the 512x512x384 Bloch grating timing")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the forward+adjoint timing of the 160x160x96 design workload")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="reference arm: skip the timing of the reference's own CUDA ops")
    ap.add_argument("--decomp", choices=("replicas", "xslab"), default="replicas",
                    help="N > 1: independent replicas (the default) or one workload split into x slabs")
    ap.add_argument("--cells", type=int, default=256,
                    help="cells per axis of the (scaled) workload; 256 is the benchmark, smaller sizes are for profiling")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    sys.path.insert(0, str(ROOT))
    wm = load_package()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            line = run_reference_arm(args, wm, world, rank)
        elif args.decomp == "xslab":
            line = run_xslab_arm(args, wm, world, rank, local)
        else:
            line = run_b200_arm(args, wm, world, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line))
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
