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


def cpu_reference_step_time(wm, cells: int, steps: int, threads: int) -> tuple[float, int]:
    """Seconds per step and cell count of the oracle (FP32) on a scaled-down copy
    (cells^3, same materials, sources and monitors scaled with the grid)."""
    from oracle import oracle as orc

    orc.build()
    cs = wm.compile_scene(wm.workloads.dispersive_256(cells=cells), steps + 2)
    sim = orc.OracleSimulation(cs, "f32", threads=threads)
    sim.step_once()  # warm
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step_once()
    dt = (time.perf_counter() - t0) / steps
    sim.close()
    return dt, cs.cells


def run_reference_arm(args, wm, world, rank):
    """CPU restatement of the reference path, all host threads, bounded sample per step."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    from oracle import oracle as orc

    orc.build()
    full_cells = 256 ** 3
    # size the per-step sample (a scaled copy of the workload) so the run stays within ~3 minutes
    probe_dt, probe_cells = cpu_reference_step_time(wm, 48, 2, threads)
    per_cell = probe_dt / probe_cells
    budget_cells = 150.0 / max(args.steps + args.warmup, 1) / per_cell
    n = int(max(32, min(256, round(budget_cells ** (1.0 / 3.0) / 8) * 8)))
    cs = wm.compile_scene(wm.workloads.dispersive_256(cells=n), args.steps + args.warmup + 2)
    sim = orc.OracleSimulation(cs, "f32", threads=threads)
    for _ in range(args.warmup):
        sim.step_once()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step_once()
    elapsed = time.perf_counter() - t0
    sim.close()
    value = cs.cells * args.steps / elapsed / 1e9
    sample = f"{args.steps} steps of the workload scaled to {n}^3 cells (same materials, sources, monitors, scaled geometry)"
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells_full": int(full_cells), "cells_sample": int(cs.cells)},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def measured_traffic(info, cells):
    """DRAM bytes of one step (the step kernel and the ADE pass after it) from
    the committed ncu capture (profiles/step_kernel_traffic.json), when it was
    taken on this launch shape and grid size; None otherwise."""
    path = ROOT / "profiles" / "step_kernel_traffic.json"
    if not path.exists():
        return None
    rec = json.loads(path.read_text())
    if (rec.get("variant"), rec.get("chunk_planes"), rec.get("cells")) != (info["variant"], info["chunk_planes"], int(cells)):
        return None
    if "kernels" not in rec:
        return None
    return int(sum(k["dram_bytes_read"] + k["dram_bytes_write"] for k in rec["kernels"]))


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
            "kernel": "step kernels: warp_step_kernel + ade_pass_kernel (one step)",
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
        "hbm_frac_whole_step": bytes_alg["total"] * cells * args.steps / (elapsed_s / world if world else elapsed_s) / 1e9 / peaks["hbm_gbs"],
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
    if args.batched:
        result["batched"] = run_batched_bench(wm, device)
    if args.grating:
        result["bloch_grating"] = run_grating_bench(wm, device)
    if args.adjoint:
        result["adjoint"] = run_adjoint_bench(wm, device)
    if rank == 0 and args.cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            step_dt, sample_cells = cpu_reference_step_time(wm, 96, 3, threads)
            cpu_value = sample_cells / step_dt / 1e9
            result["cpu_baseline"] = {
                "value": cpu_value, "unit": METRIC, "cores": threads, "kind": "port",
                "sample": "3 steps (after 1 warm-up) of the workload scaled to 96^3 cells, FP32 oracle, all host threads",
            }
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
    solver = wm.solver.B200FDTD(cs, device=device).init_field()
    solver.step_range(0, warmup)
    ms = solver.step_range(warmup, warmup + steps)
    solver.close()
    torch.cuda.empty_cache()
    return {
        "workload": "bloch_grating: 512x512x384 cells, Bloch x/y (k_x = 0.1 * 2 pi / L_x), 16-cell CPML on z, "
                    "Debye grating layer (64-cell period, 50 % duty), Ex plane source with the Bloch phase, "
                    "32-frequency diffraction plane",
        "cells": int(cs.cells),
        "steps": steps,
        "ms_per_step": ms / steps,
        "gcell_updates_per_s": cs.cells * steps / (ms * 1e-3) / 1e9,
        "channels": 2,
        "compile_s": compile_s,
    }


def run_adjoint_bench(wm, device):
    """Forward + adjoint gradient of the 160x160x96 design workload (3000 steps)
    against a plain forward solve of the same scene, device time on the engine's
    stream.  Two history modes: "store" keeps the design-box E history of every
    step in HBM (2.4 GB here, no replay); "replay" keeps a full-state checkpoint
    every 100 steps and re-runs each segment during the backward pass."""
    import torch

    steps, stride = 3000, 100
    scene = wm.workloads.adjoint_160(steps)
    eps_r = scene.material_regions[0].eps_r
    out = {
        "workload": "adjoint_160: 160x160x96 cells, 10-cell CPML, 64x64x16 design block eps_r~U[1,12), "
                    "300 THz ramped CW, |E|^2 over a 16x16 patch",
        "steps": steps,
        "design_cells": int(np.prod(eps_r.shape)),
        "gradient_check": "tests/test_adjoint.py: exact transpose (dot-product test) and central finite differences",
    }
    cs = None
    grads = {}
    for mode in ("store", "replay"):
        problem = wm.adjoint.DesignProblem(scene, steps, stride=stride, device=str(device), history=mode)
        mons = problem.forward(eps_r)
        g = problem.backward({"patch": {c: 2.0 * v for c, v in mons["patch"].items()}})
        grads[mode] = g
        out[mode] = {"forward_ms": problem.timings["forward_ms"], "backward_ms": problem.timings["backward_ms"]}
        if mode == "replay":
            out[mode]["checkpoint_stride"] = stride
        cs = problem.solver.compiled
        problem.close()
        torch.cuda.empty_cache()
    plain = wm.solver.B200FDTD(cs, device=device).init_field()
    plain_ms = plain.step_range(0, steps)
    plain.close()
    torch.cuda.empty_cache()
    out["forward_plain_ms"] = plain_ms
    for mode in ("store", "replay"):
        out[mode]["fwd_adj_over_fwd"] = (out[mode]["forward_ms"] + out[mode]["backward_ms"]) / plain_ms
    out["fwd_adj_over_fwd"] = out["store"]["fwd_adj_over_fwd"]
    den = float(np.abs(grads["replay"]).max())
    out["store_vs_replay_max_rel_diff"] = float(np.abs(grads["store"] - grads["replay"]).max() / den) if den else 0.0
    return out


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
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the 32-scene batched design workload")
    ap.add_argument("--no-grating", dest="grating", action="store_false",
                    help="skip the 512x512x384 Bloch grating timing")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the forward+adjoint timing of the 160x160x96 design workload")
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
