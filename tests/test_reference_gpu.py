"""GPU parity of the fused engine against the reference's own CUDA kernels.

The reference's torch ops are compiled from its sources by oracle/build_ref.py
into oracle/_ref/ and stepped op by op in the reference's order (oracle/ref_gpu.py)
on the same compiled scene tensors.  Tolerance: relative L2 <= 1e-5 over all
six field components together and over each monitor (both sides are FP32 on
the same GPU; they differ only in FMA contraction and summation order).

The last test is a speed bar: on the 256^3 dispersive workload the fused
engine (monitor DFT included) must advance a step at least twice as fast as
the reference's kernel sequence without any monitor work (eager, one launch
per op, timed with CUDA events).  It prints both.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import ref_gpu
from conftest import load_package
from test_engine_parity import FIELDS, TOL, _c1_scene, assert_monitors_close, joint_rel_l2

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref not built (python oracle/build_ref.py)"),
]


def _engine(cs, steps):
    wm = load_package()
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, steps)
    fields = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    mons = {name: {c: v.cpu().numpy() for c, v in comps.items()} for name, comps in solver.monitor_results().items()}
    solver.close()
    return fields, mons


def _compare(cs, steps):
    ref = ref_gpu.RefGpuSimulation(cs).run(steps)
    got_f, got_m = _engine(cs, steps)
    err = joint_rel_l2(got_f, ref.fields())
    assert err < TOL, err
    assert_monitors_close(got_m, ref.monitor_results())
    return err


def test_plain_small_matches_reference_kernels():
    """64^3 plain FP32 scene (CPML, eps box, dipole, plane + point monitors), 1000 steps."""
    wm = load_package()
    cs = wm.compile_scene(wm.workloads.plain_small(), 1000)
    _compare(cs, 1000)


def test_dispersive_tfsf_matches_reference_kernels():
    """Lorentz sphere, Drude slab, TFSF plane wave, flux planes and box; 96^3, 300 steps."""
    wm = load_package()
    cs = wm.compile_scene(wm.workloads.dispersive_256(cells=96, pml=8, n_freq=4), 300)
    _compare(cs, 300)


def test_dispersive_full_size_matches_reference_kernels():
    """The dispersive workload at its full 256^3 size (12-cell CPML, Lorentz
    sphere, Drude slab, TFSF plane wave, 16-frequency flux planes and box),
    400 steps (the pulse peak enters at step ~200), against the reference's
    kernels on the same tensors."""
    wm = load_package()
    cs = wm.compile_scene(wm.workloads.dispersive_256(), 400)
    assert cs.nodes == (257, 257, 257) and len(cs.frequencies) == 16
    _compare(cs, 400)


def test_reference_observer_ops_match_float64_accumulation():
    """The reference-timing mode of the checker (its own FP32 observer kernels
    per region and frequency) against the float64 accumulation the parity tests
    use, on the 40^3 scene: relative L2 <= 1e-5 per monitor."""
    wm = load_package()
    cs = wm.compile_scene(_c1_scene(wm, cells=40, pml=6), 120)
    a = ref_gpu.RefGpuSimulation(cs).run(120).monitor_results()
    b = ref_gpu.RefGpuSimulation(cs, monitor_ops=True).run(120).monitor_results()
    assert_monitors_close(b, a)


def test_small_scene_matches_reference_kernels():
    wm = load_package()
    cs = wm.compile_scene(_c1_scene(wm, cells=40, pml=6), 200)
    _compare(cs, 200)


def test_full_field_dft_matches_reference_kernels():
    """Full-field running DFT (VolumeMonitor over every cell of Ex, Ey, Ez and Hz)
    of a 32^3 CPML scene with a dielectric box and a Drude slab, 200 steps, 4
    frequencies: the engine's sample ring and batched flush against the
    reference's fields accumulated in float64."""
    wm = load_package()
    sc = _c1_scene(wm, cells=32, pml=6)
    sc.structures.append(wm.Structure(wm.Box((8, 0, 0), (12, 32, 32)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.monitors = [wm.VolumeMonitor("volume", ("Ex", "Ey", "Ez", "Hz"), (250e12, 280e12, 310e12, 350e12))]
    cs = wm.compile_scene(sc, 200)
    assert len(cs.regions) == 4 and cs.regions[0].box == (0, 32, 0, 33, 0, 33)
    _compare(cs, 200)


def test_engine_beats_reference_kernel_sequence():
    wm = load_package()
    steps = 10
    cs = wm.compile_scene(wm.workloads.dispersive_256(), 40)
    ref = ref_gpu.RefGpuSimulation(cs)
    ref.monitors = False  # the reference side does no monitor DFT at all; the engine does all of it
    ref.run(3)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ref.run(steps)
    b.record()
    b.synchronize()
    ref_ms = a.elapsed_time(b) / steps
    del ref
    torch.cuda.empty_cache()
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, 3)
    ms = solver.step_range(3, 3 + steps) / steps
    solver.close()
    print(f"\ndispersive_256: reference kernel sequence {ref_ms:.3f} ms/step, fused engine {ms:.3f} ms/step, "
          f"{ref_ms / ms:.1f}x")
    assert ms * 2.0 < ref_ms
