"""``Simulation.fdtd(scene, ...).run() -> Result``, the reference's public entry
(witwin/maxwell/simulation.py:512-547, :1522-1591) restricted to the FDTD hot
path: the run length from ``TimeConfig`` (an explicit step count, or the
automatic length of witwin/maxwell/fdtd/solver.py:108-131), the spectral window
of ``SpectralSampler`` with the reference's per-frequency start steps
(witwin/maxwell/fdtd/runtime/spectral.py:235-298), monitors without their own
frequencies sampled at the simulation's, and an optional full-field DFT of E.

Options of the reference that leave the hot path (plots, auto-shutoff,
excitations, multi-GPU configs, initial conditions, absorbers other than CPML)
raise NotImplementedError instead of being ignored."""
from __future__ import annotations

import dataclasses
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .scene import C_0, Scene, VolumeMonitor, compile_scene

_WINDOWS = ("none", "hanning", "ramp")


@dataclass
class TimeConfig:
    """Run length (witwin/maxwell/simulation.py:121-133): ``time_steps`` steps, or
    automatic (None): the transient (at least ``transient_cycles`` periods of the
    lowest frequency, 15 at least; five round trips across the domain; the
    source's settling time) plus ``steady_cycles`` periods."""

    time_steps: int | None = None
    steady_cycles: int = 20
    transient_cycles: int = 15

    @classmethod
    def auto(cls, steady_cycles: int = 20, transient_cycles: int = 15) -> "TimeConfig":
        return cls(time_steps=None, steady_cycles=steady_cycles, transient_cycles=transient_cycles)


@dataclass
class SpectralSampler:
    """Spectral window of the running DFTs (witwin/maxwell/simulation.py:136-143):
    "hanning" (the default), "ramp" or "none".  Pulsed sources force "none"."""

    window: str = "hanning"
    normalize_source: bool = False

    def __post_init__(self):
        self.window = str(getattr(self.window, "value", self.window)).lower()
        if self.window not in _WINDOWS:
            raise ValueError(f"unknown spectral window {self.window!r}; expected one of {_WINDOWS}")
        if self.normalize_source:
            raise NotImplementedError("source-normalised spectra are not supported")


def settling_time(source_time) -> float:
    """Time after which a source has settled (witwin/maxwell/sources.py:203-290):
    delay + 6 sigma_t for a Gaussian pulse, 0 for CW."""
    if getattr(source_time, "kind", "") == "gaussian_pulse":
        return float(source_time.resolved_delay) + 6.0 * float(source_time.sigma_t)
    return float(getattr(source_time, "settling_time", 0.0) or 0.0)


def physical_extent(scene: Scene) -> float:
    """Largest physical domain edge (the CPML cells are outside the reference's domain)."""
    lo, hi = scene.pml_lengths()
    return max((scene.cells[a] - lo[a] - hi[a]) * float(scene.spacing) for a in range(3))


def required_steps(frequency: float, dt: float, *, num_cycles: int = 20, transient_cycles: int = 15,
                   domain_size: float | None = None, source_time=None) -> int:
    """Automatic run length, witwin/maxwell/fdtd/solver.py:108-131."""
    period = 1.0 / frequency
    transient = max(transient_cycles, 15) * period
    if domain_size is not None:
        transient = max(transient, 2.0 * domain_size / C_0 * 5.0)
    if source_time is not None:
        transient = max(transient, settling_time(source_time))
    return int((transient + num_cycles * period) / dt)


def window_table(frequencies, dt: float, steps: int, window: str, *, pulsed: bool, domain_size: float) -> np.ndarray:
    """Window weight per (step, frequency) (spectral.py:235-298): with a pulsed
    source every frequency samples every step with weight 1; with CW sources
    frequency f starts after its transient int(max(15 / f, 10 L / c) / dt) and
    ends at the last step, weighted by a Hanning window or a 10 % raised-cosine
    ramp over that span ("none": weight 1 from step 0)."""
    if pulsed:
        window = "none"
    n = np.arange(steps, dtype=np.float64)
    out = np.zeros((steps, len(frequencies)), dtype=np.float64)
    domain = float(domain_size)
    for col, f in enumerate(frequencies):
        period = 1.0 / f
        start = 0 if window == "none" else int(max(15 * period, 2.0 * domain / C_0 * 5.0) / dt)
        active = (n >= start) & (n < steps)
        if window == "none":
            out[:, col] = active
            continue
        total = steps - start
        if total <= 0:
            continue
        pos = (n - start) / total
        if window == "hanning":
            w = 0.5 * (1.0 - np.cos(2.0 * np.pi * pos))
        else:  # ramp
            w = np.where(pos < 0.1, 0.5 * (1.0 - np.cos(np.pi * pos / 0.1)), 1.0)
        out[:, col] = np.where(active, w, 0.0)
    return out


def spectral_windows(scene: Scene, dt: float, steps: int, frequencies, window: str) -> np.ndarray:
    """window_table for a scene: pulsed if some source is not CW; L the largest
    physical domain edge."""
    pulsed = any(getattr(s.source_time, "kind", "cw") != "cw" for s in scene.sources)
    return window_table(frequencies, dt, steps, window, pulsed=pulsed, domain_size=physical_extent(scene))


@dataclass
class Result:
    monitors: dict
    stats: dict = field(default_factory=dict)

    def monitor(self, name: str, *, frequency: float | None = None, freq_index: int | None = None) -> dict:
        """Monitor spectra {"components": {component: complex tensor [F, ...]},
        "data": (the same dict), "frequencies": (...)}; ``frequency`` /
        ``freq_index`` select one frequency (the frequency axis is dropped)."""
        if name not in self.monitors:
            raise KeyError(f"unknown monitor {name!r}")
        payload = self.monitors[name]
        if frequency is None and freq_index is None:
            return payload
        freqs = list(payload["frequencies"])
        if freq_index is None:
            matches = [i for i, f in enumerate(freqs) if math.isclose(f, float(frequency), rel_tol=1e-9)]
            if not matches:
                raise KeyError(f"monitor {name!r} has no frequency {frequency}")
            freq_index = matches[0]
        comps = {c: v[freq_index] for c, v in payload["components"].items()}
        return {"components": comps, "data": comps, "frequencies": (freqs[freq_index],)}


class Simulation:
    def __init__(self, scene: Scene, *, frequencies=(), run_time: TimeConfig | None = None,
                 spectral_sampler: SpectralSampler | None = None, full_field_dft: bool = False,
                 cuda_graph: bool = True, time_steps: int | None = None, device=None, autotune: bool = False,
                 sample_block: int = 32):
        self.scene = scene
        self.frequencies = tuple(float(f) for f in frequencies)
        if time_steps is not None:
            run_time = TimeConfig(time_steps=int(time_steps))
        self.run_time = run_time or TimeConfig.auto()
        self.spectral_sampler = spectral_sampler or SpectralSampler()
        self.full_field_dft = bool(full_field_dft)
        self.cuda_graph = bool(cuda_graph)
        self.device = torch.device(device if device is not None else "cuda")
        self.autotune = bool(autotune)
        self.sample_block = int(sample_block)
        self.solver = None
        self.time_steps: int | None = None

    @classmethod
    def fdtd(cls, scene: Scene, *, frequencies=None, frequency=None, run_time: TimeConfig | None = None,
             absorber="cpml", spectral_sampler: SpectralSampler | None = None, cpml_config=None,
             enable_plot: bool = False, full_field_dft: bool = False, shutoff: float = 0.0,
             shutoff_check_interval: int = 100, cuda_graph: bool = True, excitations=None, parallel=None,
             initial_condition=None, time_steps: int | None = None, device=None, autotune: bool = False,
             sample_block: int = 32) -> "Simulation":
        """The reference's keywords (witwin/maxwell/simulation.py:512-547); the
        hot path's extras: ``time_steps`` (same as ``TimeConfig(time_steps=...)``),
        ``device``, ``autotune`` and the DFT ``sample_block``."""
        if str(getattr(absorber, "value", absorber)).lower() != "cpml":
            raise NotImplementedError("only the CPML absorber is on the B200 path")
        if cpml_config:
            raise NotImplementedError("custom CPML profiles are not supported (the reference's defaults are used)")
        for flag, what in ((enable_plot, "plots"), (shutoff, "auto-shutoff"), (excitations, "port excitations"),
                           (parallel, "multi-GPU configs (see witwin-maxwell_b200.distributed)"),
                           (initial_condition, "initial conditions")):
            if flag:
                raise NotImplementedError(f"{what} are not part of the B200 FDTD path")
        del shutoff_check_interval
        if frequencies is None:
            frequencies = () if frequency is None else (frequency,)
        elif frequency is not None:
            raise ValueError("pass frequencies or frequency, not both")
        return cls(scene, frequencies=tuple(np.atleast_1d(frequencies)), run_time=run_time,
                   spectral_sampler=spectral_sampler, full_field_dft=full_field_dft, cuda_graph=cuda_graph,
                   time_steps=time_steps, device=device, autotune=autotune, sample_block=sample_block)

    def _resolved_scene(self) -> Scene:
        """The scene with the simulation's frequencies on monitors that have none,
        plus the full-field DFT monitor when requested."""
        monitors = []
        for mon in self.scene.monitors:
            if not tuple(mon.frequencies):
                if not self.frequencies:
                    raise ValueError(f"monitor {mon.name!r} has no frequencies and the simulation sets none")
                mon = dataclasses.replace(mon, frequencies=self.frequencies)
            monitors.append(mon)
        if self.full_field_dft:
            if not self.frequencies:
                raise ValueError("full_field_dft needs the simulation's frequencies")
            monitors.append(VolumeMonitor("full_field", ("Ex", "Ey", "Ez"), self.frequencies))
        return dataclasses.replace(self.scene, monitors=monitors)

    def _steps(self, scene: Scene, dt: float) -> int:
        if self.run_time.time_steps is not None:
            return int(self.run_time.time_steps)
        freqs = list(self.frequencies) or [f for m in scene.monitors for f in m.frequencies]
        if not freqs:
            raise ValueError("automatic run length needs at least one frequency")
        timed = [s.source_time for s in scene.sources]
        source_time = max(timed, key=settling_time) if timed else None
        return required_steps(min(freqs), dt, num_cycles=self.run_time.steady_cycles,
                              transient_cycles=self.run_time.transient_cycles, domain_size=physical_extent(scene),
                              source_time=source_time)

    def prepare(self):
        from .solver import B200FDTD

        scene = self._resolved_scene()
        dt = scene.resolve_dt()
        self.time_steps = self._steps(scene, dt)
        compiled = compile_scene(scene, self.time_steps)
        if compiled.frequencies:
            compiled = dataclasses.replace(compiled, window=spectral_windows(
                scene, dt, self.time_steps, compiled.frequencies, self.spectral_sampler.window))
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
        monitors = {name: {"components": data, "data": data, "frequencies": freqs[name]} for name, data in raw.items()}
        cells = solver.compiled.cells
        stats = {
            "steps": self.time_steps,
            "device_ms": ms,
            "wall_s": elapsed,
            "ms_per_step": ms / max(self.time_steps, 1),
            "gcell_updates_per_s": cells * self.time_steps / (ms * 1e-3) / 1e9 if ms > 0 else 0.0,
        }
        return Result(monitors, stats)
