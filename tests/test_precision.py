"""Reduced field storage (FP16 / BF16 values, FP32 arithmetic) against the FP64 oracle.

The fields E and H are stored in 16 bits with per-component power-of-two
scales; every update is computed in FP32, the monitor DFT accumulates in FP32
with Kahan compensation from an FP64-reduced phase table.  Error measure: the
relative L2 of each monitor (all its components and frequencies together)
against the FP64 oracle of the same compiled scene.

Bars (written here, measured on B200):
  FP16 storage: <= 1e-3 per monitor on the plain 64^3 config (1000 steps) and
  on a dispersive TFSF scene (Lorentz sphere, Drude slab, flux planes and a
  closed flux box, 400 steps); measured 3.2e-4 and <= 8.3e-4.
  BF16 storage: <= 2e-2 per monitor (8-bit significand; measured 2.5e-3 and
  <= 9.3e-3), reported, not a parity form.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_package
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

FP16_TOL = 1e-3
BF16_TOL = 2e-2


def joint_rel_l2(got: dict, ref: dict) -> float:
    num = sum(float(np.linalg.norm(np.asarray(got[k], np.complex128).ravel() - np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    den = sum(float(np.linalg.norm(np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    return (num / den) ** 0.5


def _dispersive_tfsf_scene(wm):
    sc = wm.Scene(cells=(48, 40, 40), spacing=25e-9, pml_cells=8)
    sc.structures.append(wm.Structure(wm.Sphere((26, 20, 20), 8.0), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((12, 0, 0), (16, 40, 40)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (10, 10, 10), (38, 30, 30)))
    freqs = tuple(np.linspace(200e12, 400e12, 5))
    sc.monitors.append(wm.flux_monitor("flux_lo", 2, 14, freqs))
    sc.monitors.append(wm.flux_monitor("flux_hi", 2, 26, freqs))
    for face in wm.closed_box_monitor("box", (12, 12, 12), (36, 28, 28), freqs):
        sc.monitors.append(face)
    return sc


def _monitor_errors(wm, scene, steps, storage):
    cs = wm.compile_scene(scene, steps)
    ref = orc.OracleSimulation(cs, "f64").run(steps)
    refm = ref.monitor_results()
    solver = wm.solver.B200FDTD(cs, storage=storage).init_field()
    solver.step_range(0, steps)
    got = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    errs = {m: joint_rel_l2(got[m], refm[m]) for m in refm}
    solver.close()
    ref.close()
    return errs


@pytest.mark.parametrize("case", ["plain_small", "dispersive_tfsf"])
def test_fp16_storage_within_1e3_of_fp64(case):
    wm = load_package()
    if case == "plain_small":
        scene, steps = wm.workloads.plain_small(), 1000
    else:
        scene, steps = _dispersive_tfsf_scene(wm), 400
    errs = _monitor_errors(wm, scene, steps, "fp16")
    assert errs and max(errs.values()) <= FP16_TOL, errs


def test_bf16_storage_error_bound():
    wm = load_package()
    errs = _monitor_errors(wm, _dispersive_tfsf_scene(wm), 400, "bf16")
    assert errs and max(errs.values()) <= BF16_TOL, errs


def test_dispersive_workload_2000_steps_against_fp64():
    """The dispersive workload's layout at 96^3 (8-cell CPML, the Drude slab stopped
    at the CPML) over its 2000 steps: each monitor's relative L2 against the FP64
    oracle for FP32, FP16 and BF16 storage.  Bars: FP32 <= 1e-5 (the parity form),
    FP16 <= 5e-3, BF16 <= 5e-2; the measured values are printed."""
    wm = load_package()
    steps = 2000
    scene = wm.workloads.dispersive_256(cells=96, pml=8, slab_through_pml=False)
    cs = wm.compile_scene(scene, steps)
    ref = orc.OracleSimulation(cs, "f64").run(steps)
    refm = ref.monitor_results()
    ref.close()
    norms = {m: sum(float(np.linalg.norm(v)) ** 2 for v in d.values()) ** 0.5 for m, d in refm.items()}
    live = [m for m in refm if norms[m] > 1e-3 * max(norms.values())]
    report = {}
    for storage, bar in (("fp32", 1e-5), ("fp16", 5e-3), ("bf16", 5e-2)):
        solver = wm.solver.B200FDTD(cs, storage=storage).init_field()
        solver.step_range(0, steps)
        got = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
        solver.close()
        errs = {m: joint_rel_l2(got[m], refm[m]) for m in live}
        report[storage] = {m: float(f"{e:.3e}") for m, e in errs.items()}
        assert max(errs.values()) <= bar, (storage, errs)
    print("monitor rel. L2 vs FP64, dispersive layout 96^3, 2000 steps:", report)


def test_reduced_storage_state_round_trip_and_limits():
    """Packing a field into FP16 storage and reading it back rounds each value
    to FP16 relative precision (scales are exact powers of two); scales are
    estimated from the sources; launch variants other than 2 and the adjoint
    are refused."""
    wm = load_package()
    cs = wm.compile_scene(wm.workloads.plain_small(cells=32, pml=4), 10)
    solver = wm.solver.B200FDTD(cs, storage="fp16").init_field()
    kind, scales = solver.storage_scales()
    assert kind == "fp16"
    for s in scales:
        m, _ = np.frexp(s)
        assert m == 0.5
    assert scales[0] != 1.0  # estimated from the dipole's signal table
    g = torch.Generator().manual_seed(3)
    for name in ("Ex", "Hy"):
        ref = torch.randn(solver.field(name).shape, generator=g, dtype=torch.float32)
        ref = torch.sign(ref) * (1.0 + ref.abs()) * scales[0 if name[0] == "E" else 4] * 40.0  # FP16 normal range
        solver.set_field(name, ref.cuda())
        back = solver.field(name).cpu()
        rel = (back - ref).abs() / ref.abs().clamp_min(1e-30)
        assert float(rel.max()) <= 2.0 ** -11 * 1.0001
    with pytest.raises(wm._lib.FdtdError):
        solver.set_launch(5, 1, 0)
    solver.set_launch(2, 1, 8)
    solver.step_range(0, 5)
    with pytest.raises(wm._lib.FdtdError):
        wm._lib.check(solver.lib.fdtd_engine_adjoint_init(solver.handle, None, 4), "adjoint_init")
    solver.close()


def test_explicit_scales_must_be_powers_of_two():
    wm = load_package()
    cs = wm.compile_scene(wm.workloads.plain_small(cells=32, pml=4), 10)
    with pytest.raises(wm._lib.FdtdError):
        wm.solver.B200FDTD(cs, storage="fp16", storage_scales=[0.3] * 6).init_field()
    solver = wm.solver.B200FDTD(cs, storage="fp16", storage_scales=[0.25] * 3 + [2.0 ** -10] * 3).init_field()
    assert solver.storage_scales()[1] == [0.25] * 3 + [2.0 ** -10] * 3
    solver.close()
