"""Reverse-time adjoint gradients of monitor objectives with respect to a
design region's permittivity, on the fused engine.

Restates the reference's differentiable run for this path
(witwin/maxwell/fdtd/adjoint/bridge.py:957-1409 loop, core.py:379-383 stride,
core.py:3527-3565 segment replay, checkpoint.py:365-568 checkpoints,
material_pullback.py:266 pullback):

1. forward: ``B200FDTD`` steps the scene and saves a full-state checkpoint
   (E, H, CPML psi) at the start of every ``stride``-step segment;
2. seeds: dL/d(monitor spectra) becomes dL/d(unscaled DFT accumulator);
3. reverse: segments from last to first: restore the checkpoint, replay the
   segment recording the design-box E history, run the adjoint steps
   backward (``fdtd_engine_adjoint_range``), which accumulates dL/deps of the
   Yee E components in the design boxes;
4. pullback: dL/deps(Yee) -> dL/deps_r of the design cells (the scene
   compiler averages node permittivities onto the components, eps = eps0 *
   (node_a + node_b) / 2).

``design_monitors`` wraps it as a ``torch.autograd.Function``: monitor
spectra are differentiable functions of the design permittivity.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib
from .scene import EPSILON_0, MaterialRegion, Scene, compile_scene, window_scales
from .solver import B200FDTD


def design_boxes(region: MaterialRegion, nodes) -> list[tuple[int, int, int, int, int, int] | None]:
    """Yee-index boxes of Ex, Ey, Ez whose permittivity depends on the design
    nodes [lo, hi): along a component's own axis a cell averages nodes i and
    i + 1, so the box starts one cell lower."""
    out = []
    for c in range(3):
        ext = [n - 1 if a == c else n for a, n in enumerate(nodes)]
        box = []
        for a in range(3):
            lo = region.lo[a] - (1 if a == c else 0)
            hi = region.hi[a]
            box += [max(lo, 0), min(hi, ext[a])]
        out.append(tuple(box))
    return out


def pullback(region: MaterialRegion, boxes, grads) -> np.ndarray:
    """dL/deps_r of the design cells from dL/deps of the Yee components."""
    shape = tuple(h - l for l, h in zip(region.lo, region.hi))
    out = np.zeros(shape, dtype=np.float64)
    for c, (box, g) in enumerate(zip(boxes, grads)):
        g = np.asarray(g, dtype=np.float64) * (0.5 * EPSILON_0)
        # node n of the design contributes to the cells n - e_c and n along axis c
        for shift in (0, 1):
            lo = [box[2 * a] for a in range(3)]
            # cell index = node index - shift (along axis c only)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            for a in range(3):
                node_lo = lo[a] + (shift if a == c else 0)
                node_hi = box[2 * a + 1] + (shift if a == c else 0)
                a0 = max(node_lo, region.lo[a])
                a1 = min(node_hi, region.hi[a])
                if a1 <= a0:
                    break
                src[a] = slice(a0 - node_lo, a1 - node_lo)
                dst[a] = slice(a0 - region.lo[a], a1 - region.lo[a])
            else:
                out[tuple(dst)] += g[tuple(src)]
    return out


class DesignProblem:
    """One scene with a design region; ``forward(eps_r)`` solves it,
    ``backward(grad)`` returns dL/deps_r for the spectra gradients ``grad``
    ({monitor: {component: complex array like forward's}}).

    ``history`` chooses how the reverse pass gets the design-box E history:
    "store" records all of it during the forward run (steps x design cells x 4
    bytes of HBM, no replay), "replay" keeps a full-state checkpoint every
    ``stride`` steps and re-runs each segment during the backward pass (the
    reference's scheme, for histories too large to keep), "auto" stores when
    the history fits in ``history_budget`` bytes.  ``replay_region`` (replay
    only): each replayed step updates only the domain of dependence of the
    design boxes (``fdtd_engine_set_replay_region``; the gradient is the full
    replay's bit for bit)."""

    def __init__(self, scene: Scene, steps: int, stride: int = 100, device: str = "cuda", history: str = "auto",
                 history_budget: int = 16 << 30, replay_region: bool = True):
        if not scene.material_regions:
            raise ValueError("the scene has no MaterialRegion to differentiate")
        if history not in ("auto", "store", "replay"):
            raise ValueError(f"history must be auto, store or replay, not {history!r}")
        self.scene = scene
        self.steps = int(steps)
        self.stride = max(1, min(int(stride), self.steps))
        self.device = device
        self.history = history
        self.history_budget = int(history_budget)
        self.replay_region = bool(replay_region)
        self.stored = False
        self.solver: B200FDTD | None = None
        self.boxes = None
        self.region = None
        self.timings: dict = {}  # device ms of the last forward (with checkpoints) and backward

    def _scene_with(self, eps_r: np.ndarray) -> Scene:
        region = self.scene.material_regions[0]
        new_region = MaterialRegion(region.lo, region.hi, np.asarray(eps_r, dtype=np.float64))
        return dataclasses.replace(self.scene, material_regions=[new_region] + list(self.scene.material_regions[1:]))

    def prepare(self, eps_r: np.ndarray) -> B200FDTD:
        """Compile the scene with ``eps_r``, create its engine with the adjoint
        state and (replay) the checkpoint slots; nothing is stepped yet."""
        if self.solver is not None:
            self.solver.close()
            self.solver = None
        scene = self._scene_with(eps_r)
        cs = compile_scene(scene, self.steps)
        self.region = cs.design
        solver = B200FDTD(cs, device=self.device).init_field()
        self.boxes = design_boxes(self.region, cs.nodes)
        flat = [v for box in self.boxes for v in box]
        cells = sum((b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]) for b in self.boxes)
        hist_bytes = 4 * cells * (self.steps + 1)
        self.stored = self.history == "store" or (self.history == "auto" and hist_bytes <= self.history_budget)
        lib, h = solver.lib, solver.handle
        segment = self.steps if self.stored else self.stride
        _lib.check(lib.fdtd_engine_adjoint_init(h, _lib.int_array(flat), segment), "adjoint_init")
        if not self.stored:
            n_slots = (self.steps + self.stride - 1) // self.stride
            _lib.check(lib.fdtd_engine_checkpoint_reserve(h, n_slots), "checkpoint_reserve")
            _lib.check(lib.fdtd_engine_set_replay_region(h, 1 if self.replay_region else 0), "set_replay_region")
        self.solver = solver
        return solver

    def forward(self, eps_r: np.ndarray) -> dict:
        solver = self.prepare(eps_r)
        lib, h = solver.lib, solver.handle
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(solver.stream)
        if self.stored:
            _lib.check(lib.fdtd_engine_step_range_recorded(h, 0, self.steps), "step_range_recorded")
            solver.steps_done = self.steps
        else:
            for s0 in range(0, self.steps, self.stride):
                solver.checkpoint_save(s0 // self.stride)
                solver.step_range(s0, min(s0 + self.stride, self.steps))
        ev[1].record(solver.stream)
        ev[1].synchronize()
        self.timings = {"forward_ms": ev[0].elapsed_time(ev[1])}
        return solver.monitor_results()

    def _seeds(self, grad: dict) -> tuple[torch.Tensor, torch.Tensor]:
        solver = self.solver
        cs = solver.compiled
        nf = len(cs.frequencies)
        g_re = torch.zeros((nf, solver.n_samples), device=solver.device)
        g_im = torch.zeros((nf, solver.n_samples), device=solver.device)
        scales = window_scales(cs.window, solver.steps_done, nf)
        for reg, base in zip(cs.regions, solver.region_base):
            g = grad.get(reg.monitor, {}).get(reg.component)
            if g is None:
                continue
            g = torch.as_tensor(g).to(device=solver.device, dtype=torch.complex64)
            b = reg.box
            count = (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4])
            fidx = [cs.frequencies.index(f) for f in cs.monitor_frequencies[reg.monitor]]
            flat = g.reshape(len(fidx), count)
            sc = torch.as_tensor(scales[fidx], dtype=torch.float32, device=solver.device)[:, None]
            g_re[fidx, base:base + count] += sc * flat.real
            g_im[fidx, base:base + count] += sc * flat.imag
        return g_re, g_im

    def backward(self, grad: dict) -> np.ndarray:
        solver = self.solver
        if solver is None:
            raise RuntimeError("backward before forward")
        lib, h = solver.lib, solver.handle
        g_re, g_im = self._seeds(grad)
        _lib.check(lib.fdtd_engine_adjoint_set_seed(h, _lib.ptr(g_re), _lib.ptr(g_im)), "adjoint_set_seed")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(solver.stream)
        if self.stored:
            _lib.check(lib.fdtd_engine_adjoint_range(h, self.steps, 0), "adjoint_range")
        else:
            # segment replays overlapped with the reverse steps of the segment after
            _lib.check(lib.fdtd_engine_backward_replay(h, self.steps, self.stride), "backward_replay")
        ev[1].record(solver.stream)
        ev[1].synchronize()
        self.timings["backward_ms"] = ev[0].elapsed_time(ev[1])
        grads = []
        for c, box in enumerate(self.boxes):
            shape = (box[1] - box[0], box[3] - box[2], box[5] - box[4])
            out = torch.empty(shape, device=solver.device)
            _lib.check(lib.fdtd_engine_adjoint_grad(h, c, _lib.ptr(out)), "adjoint_grad")
            grads.append(out.cpu().numpy())
        return pullback(self.region, self.boxes, grads)

    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None


class BatchDesignProblem:
    """Forward and adjoint gradients of many independent design scenes.

    The forward run steps every scene together through ``B200Batch`` (one CUDA
    graph per sample block, the scenes' kernels concurrent on their own
    streams), saving each scene's full-state checkpoint at the start of every
    ``stride``-step segment; ``backward`` then runs each scene's pipelined
    checkpoint replay and reverse steps (``fdtd_engine_backward_replay``).
    Gradients equal those of one ``DesignProblem`` per scene (the reference's
    per-simulation differentiable runs over its ensemble,
    witwin/maxwell/execution/ensemble.py:166 and fdtd/adjoint/bridge.py:1444)."""

    def __init__(self, scenes, steps: int, stride: int = 100, device: str = "cuda"):
        self.problems = [DesignProblem(sc, steps, stride=stride, device=device, history="replay") for sc in scenes]
        if not self.problems:
            raise ValueError("empty batch")
        self.steps = int(steps)
        self.stride = self.problems[0].stride
        self.batch = None
        self.timings: dict = {}

    def forward(self, eps_list) -> list[dict]:
        from .solver import B200Batch

        if len(eps_list) != len(self.problems):
            raise ValueError("one eps_r array per scene")
        self._close_batch()
        solvers = [p.prepare(e) for p, e in zip(self.problems, eps_list)]
        self.batch = B200Batch(solvers)
        stream = solvers[0].stream
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for s0 in range(0, self.steps, self.stride):
            for s in solvers:
                s.checkpoint_save(s0 // self.stride)
            self.batch.step_range(s0, min(s0 + self.stride, self.steps))
        ev[1].record(stream)
        ev[1].synchronize()
        self.timings = {"forward_ms": ev[0].elapsed_time(ev[1])}
        return [s.monitor_results() for s in solvers]

    def backward(self, grads) -> list[np.ndarray]:
        if self.batch is None:
            raise RuntimeError("backward before forward")
        stream = self.problems[0].solver.stream
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        out = [p.backward(g) for p, g in zip(self.problems, grads)]
        ev[1].record(stream)
        ev[1].synchronize()
        self.timings["backward_ms"] = ev[0].elapsed_time(ev[1])
        return out

    def _close_batch(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None

    def close(self):
        self._close_batch()
        for p in self.problems:
            p.close()


class _DesignFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps_r, problem, keys):
        mons = problem.forward(eps_r.detach().cpu().numpy())
        ctx.problem = problem
        ctx.keys = keys
        ctx.eps_shape = eps_r.shape
        ctx.eps_device = eps_r.device
        return tuple(mons[m][c].detach().clone() for m, c in keys)

    @staticmethod
    def backward(ctx, *grads):
        grad: dict = {}
        for (m, c), g in zip(ctx.keys, grads):
            if g is not None:
                grad.setdefault(m, {})[c] = g
        g_eps = ctx.problem.backward(grad)
        return torch.as_tensor(g_eps, dtype=torch.float32, device=ctx.eps_device).reshape(ctx.eps_shape), None, None


def design_monitors(eps_r: torch.Tensor, problem: DesignProblem, keys) -> dict:
    """Monitor spectra as differentiable functions of the design permittivity.

    ``keys`` lists the (monitor, component) pairs to return; the result maps
    monitor -> component -> complex tensor, as ``B200FDTD.monitor_results``."""
    keys = tuple((str(m), str(c)) for m, c in keys)
    outs = _DesignFunction.apply(eps_r, problem, keys)
    result: dict = {}
    for (m, c), t in zip(keys, outs):
        result.setdefault(m, {})[c] = t
    return result
