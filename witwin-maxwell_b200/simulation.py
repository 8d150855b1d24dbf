"""``Simulation.fdtd(scene, ...).run() -> Result``, the reference's public entry
(witwin/maxwell/simulation.py:512-661) restricted to the FDTD hot path."""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import torch

from .scene import Scene, compile_scene
from .solver import B200FDTD


@dataclass
class Result:
    monitors: dict
    stats: dict = field(default_factory=dict)

    def monitor(self, name: str) -> dict:
        """Monitor spectra: {"data": {component: complex tensor [F, ...]}, "frequencies": (...)}."""
        if name not in self.monitors:
            raise KeyError(f"unknown monitor {name!r}")
        return self.monitors[name]


class Simulation:
    def __init__(self, scene: Scene, time_steps: int, *, device=None, autotune: bool = False, sample_block: int = 32):
        self.scene = scene
        self.time_steps = int(time_steps)
        self.device = torch.device(device if device is not None else "cuda")
        self.autotune = bool(autotune)
        self.sample_block = int(sample_block)
        self.solver: B200FDTD | None = None

    @classmethod
    def fdtd(cls, scene: Scene, *, time_steps: int, device=None, autotune: bool = False, sample_block: int = 32):
        return cls(scene, time_steps, device=device, autotune=autotune, sample_block=sample_block)

    def prepare(self) -> B200FDTD:
        compiled = compile_scene(self.scene, self.time_steps)
        self.solver = B200FDTD(compiled, device=self.device, sample_block=self.sample_block).init_field()
        if self.autotune:
            self.solver.autotune()
        return self.solver

    def run(self) -> Result:
        if self.solver is None:
            self.prepare()
        solver = self.solver
        t0 = time.perf_counter()
        ms = solver.step_range(solver.steps_done, self.time_steps)
        raw = solver.monitor_results()
        torch.cuda.synchronize(self.device)
        elapsed = time.perf_counter() - t0
        freqs = solver.compiled.monitor_frequencies
        monitors = {name: {"data": data, "frequencies": freqs[name]} for name, data in raw.items()}
        cells = solver.compiled.cells
        stats = {
            "steps": self.time_steps,
            "device_ms": ms,
            "wall_s": elapsed,
            "ms_per_step": ms / max(self.time_steps, 1),
            "gcell_updates_per_s": cells * self.time_steps / (ms * 1e-3) / 1e9 if ms > 0 else 0.0,
        }
        return Result(monitors, stats)
