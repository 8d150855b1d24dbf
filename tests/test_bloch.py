"""Periodic and Bloch-periodic faces of the fused engine.

The step kernel defers the E cells on a wrapped face and the wrap kernel
updates them from the whole new H (phase e^{ikL} across the wrap, the real and
imaginary channels coupled only there).  Checked against the reference's own
CUDA ops compiled from its sources (oracle/_ref, oracle/ref_gpu.py): the
standard / compressed-CPML ops with periodic boundary modes for periodic
scenes, and its complex Bloch E kernels for Bloch scenes.  Tolerance as the
other engine parity tests: joint relative L2 <= 1e-5 on fields and monitors.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import ref_gpu
from conftest import load_package
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
TOL = 1e-5
PERIODIC, BLOCH, PML, PEC = 2, 3, 1, 4


def joint(got: dict, ref: dict) -> float:
    num = sum(float(np.linalg.norm(np.asarray(got[k], np.complex128).ravel() - np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    den = sum(float(np.linalg.norm(np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    return (num / den) ** 0.5


def _periodic_scene(wm):
    sc = wm.Scene(cells=(28, 24, 32), spacing=25e-9, pml_cells=6, boundary=(PERIODIC, PERIODIC, PERIODIC, PERIODIC, PML, PML))
    sc.structures.append(wm.Structure(wm.Box((0, 0, 10), (28, 24, 14)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.structures.append(wm.Structure(wm.Box((6, 5, 18), (20, 16, 22)), wm.Medium(eps_r=3.0)))
    sc.sources.append(wm.PointDipole((3, 12, 16), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.sources.append(wm.PlaneSource(2, 24, "Ex", wm.GaussianPulse(300e12, 100e12)))
    freqs = (250e12, 300e12, 350e12)
    sc.monitors.append(wm.PlaneMonitor("plane", 2, 8, frequencies=freqs))
    sc.monitors.append(wm.PointMonitor("point", (0, 0, 20), frequencies=freqs))
    return sc


def _bloch_scene(wm, kx_frac=0.1, ky_frac=0.05):
    cells = (28, 24, 20)
    d = 25e-9
    k = (2 * np.pi / (cells[0] * d) * kx_frac, 2 * np.pi / (cells[1] * d) * ky_frac, 0.0)
    sc = wm.Scene(cells=cells, spacing=d, pml_cells=0, boundary=(BLOCH, BLOCH, BLOCH, BLOCH, PEC, PEC), bloch_k=k)
    sc.structures.append(wm.Structure(wm.Box((0, 0, 8), (28, 24, 11)), wm.Medium.debye(2.5, 3.5, 1e-14)))
    sc.sources.append(wm.PlaneSource(2, 14, "Ex", wm.GaussianPulse(300e12, 120e12)))
    sc.sources.append(wm.PointDipole((14, 12, 5), "Ey", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    freqs = (250e12, 300e12, 350e12)
    sc.monitors.append(wm.PlaneMonitor("plane", 2, 4, frequencies=freqs))
    sc.monitors.append(wm.PointMonitor("corner", (0, 0, 12), frequencies=freqs))
    return sc


def test_periodic_matches_reference_ops_and_oracle():
    wm = load_package()
    steps = 300
    cs = wm.compile_scene(_periodic_scene(wm), steps)
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, 150)
    solver.step_range(150, steps)
    fields = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    solver.close()
    ref = ref_gpu.RefGpuSimulation(cs).run(steps)
    assert joint(fields, ref.fields()) < TOL
    refm = ref.monitor_results()
    for m in refm:
        assert joint(mons[m], refm[m]) < TOL, m
    o64 = orc.OracleSimulation(cs, "f64").run(steps)
    o32 = orc.OracleSimulation(cs, "f32").run(steps)
    assert joint(fields, o64.fields) < 2.0 * joint(o32.fields, o64.fields) + 1e-7
    o64.close()
    o32.close()


@pytest.mark.parametrize("variant", [1, 3])
def test_periodic_launch_variants_agree(variant):
    wm = load_package()
    steps = 80
    cs = wm.compile_scene(_periodic_scene(wm), steps)
    out = []
    for v in (2, variant):
        solver = wm.solver.B200FDTD(cs).init_field()
        solver.set_launch(v, 1, 5)
        solver.step_range(0, steps)
        out.append({n: solver.field(n).cpu().numpy() for n in FIELDS})
        solver.close()
    for n in FIELDS:
        np.testing.assert_array_equal(out[0][n], out[1][n])


def test_bloch_matches_reference_bloch_kernels():
    wm = load_package()
    steps = 300
    cs = wm.compile_scene(_bloch_scene(wm), steps)
    assert cs.complex_fields
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, steps)
    got_re = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    got_im = {n: solver.field(n, imag=True).cpu().numpy() for n in FIELDS}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    solver.close()
    ref = ref_gpu.RefGpuBloch(cs).run(steps)
    ref_re, ref_im = ref.fields()
    got = {**{f"re_{n}": got_re[n] for n in FIELDS}, **{f"im_{n}": got_im[n] for n in FIELDS}}
    want = {**{f"re_{n}": ref_re[n] for n in FIELDS}, **{f"im_{n}": ref_im[n] for n in FIELDS}}
    assert joint(got, want) < TOL
    assert np.linalg.norm(got_im["Ex"]) > 1e-3 * np.linalg.norm(got_re["Ex"])  # the phase couples the channels
    refm = ref.monitor_results()
    for m in refm:
        assert joint(mons[m], refm[m]) < TOL, m


def test_bloch_grating_shape_with_z_cpml_matches_reference_kernels():
    """The large grating's boundary set on a small copy: Bloch x / y faces
    (k_x = 0.1 * 2 pi / L_x), 8-cell CPML on z only, the Debye grating layer
    and a phased current sheet in place of its TFSF slab (64 x 64 x 48 cells,
    4 frequencies, 300 steps), against the reference's Bloch-xy / standard-z E
    kernels followed by its z-CPML corrections of Ex and Ey on both channels."""
    wm = load_package()
    steps = 300
    sc = wm.workloads.bloch_grating(cells=(64, 64, 48), pml=8, n_freq=4)
    sc.sources[:] = [wm.PlaneSource(2, 48 - 8 - 5, "Ex", wm.GaussianPulse(300e12, 120e12))]
    cs = wm.compile_scene(sc, steps)
    assert cs.complex_fields and cs.pml_lo[2] == 8 and cs.pml_lo[0] == 0
    assert {p.kind for p in cs.poles} == {0}
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, steps)
    got_re = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    got_im = {n: solver.field(n, imag=True).cpu().numpy() for n in FIELDS}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    solver.close()
    ref = ref_gpu.RefGpuBloch(cs)
    assert ref.z_cpml
    ref.run(steps)
    ref_re, ref_im = ref.fields()
    got = {**{f"re_{n}": got_re[n] for n in FIELDS}, **{f"im_{n}": got_im[n] for n in FIELDS}}
    want = {**{f"re_{n}": ref_re[n] for n in FIELDS}, **{f"im_{n}": ref_im[n] for n in FIELDS}}
    assert np.linalg.norm(want["re_Ex"]) > 0 and np.linalg.norm(want["im_Ex"]) > 1e-3 * np.linalg.norm(want["re_Ex"])
    assert joint(got, want) < TOL
    refm = ref.monitor_results()
    for m in refm:
        assert joint(mons[m], refm[m]) < TOL, m


def test_bloch_at_zero_wavevector_is_periodic():
    """k = 0: the Bloch pair's real channel equals the periodic engine and the
    imaginary channel stays zero (a real source)."""
    wm = load_package()
    steps = 120
    sc = _bloch_scene(wm, 0.0, 0.0)
    cs_b = wm.compile_scene(sc, steps)
    sc.boundary = (PERIODIC, PERIODIC, PERIODIC, PERIODIC, PEC, PEC)
    cs_p = wm.compile_scene(sc, steps)
    b = wm.solver.B200FDTD(cs_b).init_field()
    p = wm.solver.B200FDTD(cs_p).init_field()
    b.step_range(0, steps)
    p.step_range(0, steps)
    for n in FIELDS:
        np.testing.assert_array_equal(b.field(n).cpu().numpy(), p.field(n).cpu().numpy())
        assert float(b.field(n, imag=True).abs().max()) == 0.0
    b.close()
    p.close()


def test_wrap_faces_refuse_other_variants_and_the_adjoint():
    wm = load_package()
    cs = wm.compile_scene(_periodic_scene(wm), 10)
    solver = wm.solver.B200FDTD(cs).init_field()
    with pytest.raises(wm._lib.FdtdError):
        solver.set_launch(5, 1, 0)
    with pytest.raises(wm._lib.FdtdError):
        wm._lib.check(solver.lib.fdtd_engine_adjoint_init(solver.handle, None, 4), "adjoint_init")
    solver.close()
