"""GPU parity of the fused step engine against the CPU oracle and the reference goldens.

Tolerance (relative L2): <= 1e-5 over all six field components together and
over each monitor (all its components together), against the FP32 oracle (same
arithmetic; the GPU contracts multiply-adds into FMAs and sums in another order)
and against the reference's own 60-step golden run; <= 1e-4 for each single
component, whose small cross-polarised components amplify round-off.
Against the FP64 oracle the engine must be as accurate as the FP32 oracle is
(within 2x of the FP32 oracle's own error).
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import load_package
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
TOL = 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / den) if den > 0 else float(np.linalg.norm(a.ravel()))


def joint_rel_l2(got: dict, ref: dict) -> float:
    num = sum(float(np.linalg.norm(np.asarray(got[k], np.complex128).ravel() - np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    den = sum(float(np.linalg.norm(np.asarray(ref[k], np.complex128).ravel())) ** 2 for k in ref)
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def assert_fields_close(got: dict, ref: dict, tol=TOL, comp_tol=1e-4):
    assert joint_rel_l2(got, ref) < tol
    for n in ref:
        assert rel_l2(got[n], ref[n]) < comp_tol, n


def assert_monitors_close(got: dict, ref: dict, tol=TOL, comp_tol=1e-4):
    for name, comps in ref.items():
        assert joint_rel_l2(got[name], comps) < tol, name
        for comp, r in comps.items():
            a = np.asarray(got[name][comp], np.complex128)
            b = np.asarray(r, np.complex128)
            err = float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
            # components far below the monitor's scale carry only round-off
            scale = max(float(np.linalg.norm(np.asarray(v, np.complex128).ravel())) for v in comps.values())
            if np.linalg.norm(b.ravel()) > 1e-3 * scale:
                assert err < comp_tol, (name, comp, err)


def _golden_module():
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    sys.modules["make_golden"] = mg
    spec.loader.exec_module(mg)
    return mg


def _run_engine(cs, steps, **kw):
    wm = load_package()
    solver = wm.solver.B200FDTD(cs, **kw).init_field()
    solver.step_range(0, steps)
    fields = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    return solver, fields, mons


def test_engine_matches_reference_golden_run():
    """Fused engine (FP32) vs the reference's Torch ops (FP64) on the golden scene."""
    wm = load_package()
    mg = _golden_module()
    gold = dict(np.load(GOLDEN / "steps.npz"))
    steps = int(gold["steps"])
    cs = wm.compile_scene(mg.golden_scene(), steps)
    solver, fields, mons = _run_engine(cs, steps)
    assert_fields_close(fields, {n: gold[f"field_{n}"] for n in FIELDS})
    scale = 2.0 / float(gold["window_sum"])
    ref_mons: dict = {}
    for i, reg in enumerate(cs.regions):
        data = (gold[f"dft_{i}_re"] + 1j * gold[f"dft_{i}_im"]) * scale
        ref_mons.setdefault(reg.monitor, {})[reg.component] = data
    assert_monitors_close(mons, ref_mons)
    solver.close()


def _c1_scene(wm, cells=64, pml=10):
    """64^3 cells, 10-cell CPML, eps 4 box, Ez dipole, z-plane + point monitors at 3 frequencies."""
    return wm.workloads.plain_small(cells=cells, pml=pml)


def test_engine_matches_oracle_small_plain_config():
    """Plain FP32 64^3 config (CPML, dielectric box, dipole, plane + point DFT), 1000 steps."""
    wm = load_package()
    steps = 1000
    cs = wm.compile_scene(_c1_scene(wm), steps)
    solver, fields, mons = _run_engine(cs, steps)
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    assert_fields_close(fields, ref32.fields)
    assert_monitors_close(mons, ref32.monitor_results())
    ref32.close()
    solver.close()


def test_engine_dispersive_tfsf_against_fp64_oracle():
    """Lorentz sphere + Drude slab + TFSF plane wave + flux planes, FP32 engine vs FP64 oracle."""
    wm = load_package()
    steps = 400
    sc = wm.Scene(cells=(48, 40, 40), spacing=25e-9, pml_cells=8)
    sc.structures.append(wm.Structure(wm.Sphere((26, 20, 20), 8.0), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((12, 0, 0), (16, 40, 40)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (10, 10, 10), (38, 30, 30)))
    freqs = tuple(np.linspace(200e12, 400e12, 5))
    sc.monitors.append(wm.flux_monitor("flux_lo", 2, 14, freqs))
    sc.monitors.append(wm.flux_monitor("flux_hi", 2, 26, freqs))
    for face in wm.closed_box_monitor("box", (12, 12, 12), (36, 28, 28), freqs):
        sc.monitors.append(face)
    cs = wm.compile_scene(sc, steps)
    solver, fields, mons = _run_engine(cs, steps)
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    ref64 = orc.OracleSimulation(cs, "f64").run(steps)
    assert_fields_close(fields, ref32.fields)
    # as accurate as an FP32 CPU run of the reference algorithm
    assert joint_rel_l2(fields, ref64.fields) < 2.0 * joint_rel_l2(ref32.fields, ref64.fields) + 1e-7
    for p_idx in range(len(cs.poles)):
        pol, cur = solver.pole_state(p_idx)
        b = cs.poles[p_idx].box
        sl = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
        assert rel_l2(cur.cpu().numpy(), ref32.poles[p_idx]["J"][sl]) < 1e-4
    assert_monitors_close(mons, ref32.monitor_results())
    ref32.close()
    ref64.close()
    solver.close()


def test_batched_design_scene_against_fp64_oracle():
    """One scene of the batched design workload as generated (seed 1): the
    smallest of the 32, diagonal anisotropic eps boxes (a different
    coefficient array per E component), 8-cell CPML, Ez dipole, 8-frequency
    point monitor; 600 steps of the FP32 engine against the FP32 and FP64
    oracles."""
    wm = load_package()
    steps = 600
    scenes = wm.workloads.batched_designs()
    sc = min(scenes, key=lambda s: int(np.prod(s.cells)))
    assert any(st.medium.eps_diag is not None and len(set(st.medium.eps_diag)) == 3 for st in sc.structures)
    cs = wm.compile_scene(sc, steps)
    curls = [cs.curl[n] for n in ("Ex", "Ey", "Ez")]
    assert all(c is not None for c in curls) and not np.array_equal(curls[0][:-1, :-1, :-1], curls[1][:-1, :-1, :-1])
    solver, fields, mons = _run_engine(cs, steps)
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    ref64 = orc.OracleSimulation(cs, "f64").run(steps)
    assert_fields_close(fields, ref32.fields)
    assert joint_rel_l2(fields, ref64.fields) < 2.0 * joint_rel_l2(ref32.fields, ref64.fields) + 1e-7
    assert_monitors_close(mons, ref32.monitor_results())
    m64 = ref64.monitor_results()
    for name in m64:
        assert joint_rel_l2(mons[name], m64[name]) < TOL, name
    ref32.close()
    ref64.close()
    solver.close()


@pytest.mark.parametrize(
    "tiles",
    [
        (1, 1, 8), (3, 1, 5), (2, 1, 64), (2, 1, 13), (4, 1, 8), (4, 1, 3), (4, 1, 41),
        (5, 1, 8), (5, 1, 13), (6, 1, 8), (6, 1, 41), (7, 1, 8), (7, 1, 3), (7, 1, 41), (8, 1, 13), (9, 1, 8),
        (9, 1, 41), (10, 1, 8), (10, 1, 3), (10, 1, 41), (10, 1, 1), (10, 1, 2),
    ],
)
def test_tile_shape_does_not_change_results(tiles):
    """Every chunk length and every launch variant of one kernel family gives
    bit-identical fields: the scalar warp kernels (register-prefetch budgets
    1-3, TMA-fed 4) among themselves, and the z-vectorised kernels (5-9, direct
    loads or cp.async ring) among themselves.  Across the two families the
    compiler may contract a different multiply-add pair, so the fields agree
    to 1e-6 of their peak instead."""
    wm = load_package()
    steps = 50
    cs = wm.compile_scene(_c1_scene(wm, cells=40, pml=6), steps)
    family = (lambda v: 5 <= v <= 9)
    base_variant = 7 if family(tiles[0]) else 2  # one member of the tile's family
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.set_launch(base_variant, 1, 32)
    solver.step_range(0, steps)
    base = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    solver.close()
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.set_launch(*tiles)
    assert solver.get_launch() == (tiles[0], 1, tiles[2])
    solver.step_range(0, steps)
    scale = max(float(np.abs(v).max()) for v in base.values())
    for n in FIELDS:
        got = solver.field(n).cpu().numpy()
        if tiles[0] == 10:
            # the row-tile kernel: same arithmetic, the compiler's own choice of
            # fused multiply-adds, so agreement to FP32 rounding of the field scale
            np.testing.assert_allclose(got, base[n], rtol=0, atol=1e-6 * scale)
        else:
            np.testing.assert_array_equal(got, base[n])
    solver.close()


def test_kernel_families_agree():
    """The scalar warp kernel, the z-vectorised ring kernel and the row-tile
    kernel give the same fields after 200 steps of a CPML + dielectric scene:
    relative L2 within 1e-5 per component (the engine's parity bar against the
    FP32 oracle)."""
    wm = load_package()
    steps = 200
    cs = wm.compile_scene(_c1_scene(wm, cells=40, pml=6), steps)
    out = []
    for variant in (2, 7, 10):
        solver = wm.solver.B200FDTD(cs).init_field()
        solver.set_launch(variant, 1, 0)
        solver.step_range(0, steps)
        out.append({n: solver.field(n).cpu().numpy() for n in FIELDS})
        solver.close()
    for other in out[1:]:
        for n in FIELDS:
            a, b = other[n].astype(np.float64), out[0][n].astype(np.float64)
            assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), n


def test_ade_pass_matches_poles_in_step_kernel():
    """Dispersive poles advanced in the ADE pass after the step kernel (the
    default) and inside the fused step kernel: a three-pole medium (Lorentz +
    Drude + Debye on every component, so nine poles share each plane and the
    pass runs more than one batch of four) beside a Lorentz sphere, a dipole
    source, 300 steps.  The two orders of the additive terms agree to FP32
    rounding (relative L2 within 1e-5 per field and per pole current), and the
    pass path matches the FP32 oracle."""
    wm = load_package()
    from importlib import import_module

    sc_mod = import_module(wm.__name__ + ".scene")
    steps = 300
    sc = wm.Scene(cells=(40, 36, 36), spacing=25e-9, pml_cells=6)
    multi = wm.Medium(eps_r=2.0, poles=(sc_mod.LorentzPole(1.5, 250e12, 20e12),
                                        sc_mod.DrudePole(1e15 / (2 * np.pi), 1e14 / (2 * np.pi)),
                                        sc_mod.DebyePole(1.0, 2e-15)))
    sc.structures.append(wm.Structure(wm.Box((10, 8, 9), (18, 27, 30)), multi))
    sc.structures.append(wm.Structure(wm.Sphere((27, 18, 18), 6.0), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.sources.append(wm.PointDipole((22, 18, 18), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    cs = wm.compile_scene(sc, steps)
    assert len(cs.poles) == 12
    out, cur = [], []
    for on in (True, False):
        solver = wm.solver.B200FDTD(cs).init_field()
        solver.set_ade_pass(on)
        solver.step_range(0, steps)
        out.append({n: solver.field(n).cpu().numpy() for n in FIELDS})
        cur.append([solver.pole_state(b)[1].cpu().numpy() for b in range(len(cs.poles))])
        solver.close()
    for n in FIELDS:
        assert rel_l2(out[0][n], out[1][n]) <= 1e-5, n
    for b in range(len(cs.poles)):
        assert rel_l2(cur[0][b], cur[1][b]) <= 1e-5, b
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    assert_fields_close(out[0], ref32.fields)
    ref32.close()


def test_pinned_scene_and_host_results_match():
    """An engine built from pin_scene's copy (coefficient and pole arrays in
    pinned memory, uploaded asynchronously) steps to bit-identical fields and
    spectra, and monitor_results(host=True) returns the same values on the host
    as the device tensors."""
    wm = load_package()
    steps = 120
    sc = wm.Scene(cells=(40, 36, 36), spacing=25e-9, pml_cells=6)
    sc.structures.append(wm.Structure(wm.Sphere((21, 18, 18), 6.0), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((8, 8, 8), (14, 28, 28)), wm.Medium(eps_r=3.0)))
    sc.sources.append(wm.PointDipole((26, 18, 18), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.monitors.append(wm.flux_monitor("flux", 2, 24, (250e12, 300e12)))
    cs = wm.compile_scene(sc, steps)
    ref = wm.solver.B200FDTD(cs).init_field()
    ref.step_range(0, steps)
    ref_fields = {n: ref.field(n).cpu().numpy() for n in FIELDS}
    ref_mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in ref.monitor_results().items()}
    ref.close()
    pinned = wm.solver.pin_scene(cs)
    assert all(v is None or v.is_pinned() for v in pinned.curl.values())
    assert all(p.drive.is_pinned() for p in pinned.poles)
    solver = wm.solver.B200FDTD(pinned).init_field()
    solver.step_range(0, steps)
    for n in FIELDS:
        np.testing.assert_array_equal(solver.field(n).cpu().numpy(), ref_fields[n], err_msg=n)
    host = solver.monitor_results(host=True)
    for name, comps in ref_mons.items():
        for comp, v in comps.items():
            assert host[name][comp].device.type == "cpu" and host[name][comp].is_pinned()
            np.testing.assert_array_equal(host[name][comp].numpy(), v, err_msg=f"{name} {comp}")
    solver.close()


def test_checkpoint_roundtrip_and_autotune_restore_state():
    wm = load_package()
    steps = 60
    cs = wm.compile_scene(_c1_scene(wm, cells=32, pml=6), steps)
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, 20)
    solver.checkpoint_save(0)
    solver.step_range(20, 40)
    after = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    solver.checkpoint_load(0)
    solver.autotune()  # times candidate tiles, then restores the saved state
    solver.step_range(20, 40)
    again = {n: solver.field(n).cpu().numpy() for n in FIELDS}
    for n in FIELDS:
        np.testing.assert_array_equal(again[n], after[n])
    solver.close()


def test_tfsf_total_field_stays_inside_box():
    """Plane wave in vacuum: the scattered-field region stays empty (leakage < 1e-3 of the TF field)."""
    wm = load_package()
    steps = 300
    sc = wm.Scene(cells=(48, 32, 32), spacing=25e-9, pml_cells=8)
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (12, 11, 11), (36, 21, 21)))
    cs = wm.compile_scene(sc, steps)
    _, fields, _ = _run_engine(cs, steps - 100)
    ez = fields["Ez"]
    inside = np.abs(ez[14:34, 13:19, 13:19]).max()
    outside = max(np.abs(ez[:, :9, :]).max(), np.abs(ez[:, 24:, :]).max(), np.abs(ez[:, :, :9]).max())
    assert inside > 0.1
    assert outside < 1e-3 * inside


def test_engine_rejects_bad_inputs():
    wm = load_package()
    lib = wm._lib.load()
    import ctypes

    desc = wm._lib.FdtdGridDesc()
    desc.nx = desc.ny = desc.nz = 2
    desc.dt = 1e-17
    handle = ctypes.c_void_p()
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == -1 and b"at least 3" in lib.fdtd_last_error()
    desc.nx = desc.ny = desc.nz = 10
    desc.boundary[0] = 5  # a PMC face with a CPML slab
    desc.pml_lo[0] = 2
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == -1 and b"PMC" in lib.fdtd_last_error()
    desc.pml_lo[0] = 0
    desc.boundary[2] = desc.boundary[3] = 2  # PMC beside periodic faces
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == -3
    desc.boundary[2] = desc.boundary[3] = 0
    desc.boundary[0] = 3  # a Bloch low face needs a Bloch high face
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == -1 and b"must match" in lib.fdtd_last_error()
    desc.boundary[4] = desc.boundary[5] = 2  # periodic z: not supported
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == -3
    desc.boundary[0] = 1
    desc.boundary[4] = desc.boundary[5] = 0
    rc = lib.fdtd_engine_create(ctypes.byref(desc), None, ctypes.byref(handle))
    assert rc == 0
    # stepping before finalize is a state error, not a crash
    assert lib.fdtd_engine_step_range(handle, 0, 1) == -4
    box = wm._lib.int_array([0, 20, 0, 1, 0, 1])
    dummy = torch.zeros(64, device="cuda")
    assert lib.fdtd_engine_add_patch(handle, 0, box, dummy.data_ptr(), dummy.data_ptr(), 1, 1.0) == -1
    assert lib.fdtd_engine_destroy(handle) == 0


def test_bounded_waits_report_timeout_and_leave_the_context_usable():
    """Failure detection without a GPU fault: the TMA-fed step kernel (variant
    4) waits on its mbarrier ring with a bounded number of polling rounds.
    With the bound at zero every pipeline wait runs out at once: the kernel
    records FDTD_ERR_TIMEOUT in the device status word and returns (its
    producer still waits for the copies it issued), and step_range reports
    the timeout.  With the default bound restored the same engine steps again
    without error, and a fresh engine still matches the register kernel
    bit for bit (the context is intact)."""
    wm = load_package()
    steps = 20
    cs = wm.compile_scene(_c1_scene(wm, cells=40, pml=6), steps + 4)
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.set_launch(4, 1, 0)
    solver.set_wait_limit(0)
    with pytest.raises(wm._lib.FdtdError) as err:
        solver.step_range(0, 2)
    assert "status -5" in str(err.value)
    solver.set_wait_limit(1 << 20)
    solver.step_range(2, 4)  # no timeout once the bound is back
    solver.close()
    fields = []
    for variant in (4, 2):
        solver = wm.solver.B200FDTD(cs).init_field()
        solver.set_launch(variant, 1, 0)
        solver.step_range(0, steps)
        fields.append({n: solver.field(n).cpu().numpy() for n in FIELDS})
        solver.close()
    for n in FIELDS:
        np.testing.assert_array_equal(fields[0][n], fields[1][n])


@pytest.mark.parametrize("faces", ["mixed", "closed"])
def test_pmc_faces_against_oracle(faces):
    """PMC faces in the fused engine (the tangential E on the face updated with
    the difference across it doubled, electric.cu:18-119) against the FP32 / FP64
    oracle: PMC beside CPML and PEC faces, and a closed PMC / PEC box with no
    CPML (the scalar warp kernel then replaces the row-tile default)."""
    wm = load_package()
    steps = 300
    pml, pec, pmc = wm.BOUNDARY_PML, wm.BOUNDARY_PEC, wm.BOUNDARY_PMC
    boundary = (pmc, pml, pmc, pmc, pec, pml) if faces == "mixed" else (pmc, pmc, pec, pmc, pmc, pec)
    sc = wm.Scene(cells=(30, 26, 24), spacing=25e-9, pml_cells=6, boundary=boundary)
    sc.structures.append(wm.Structure(wm.Box((8, 6, 6), (16, 14, 12)), wm.Medium(eps_r=3.0)))
    sc.structures.append(wm.Structure(wm.Sphere((18, 13, 12), 3.5), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.sources.append(wm.PointDipole((5, 4, 5), "Ey", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.sources.append(wm.PointDipole((12, 20, 3), "Ex", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    freqs = (250e12, 300e12)
    sc.monitors.append(wm.PlaneMonitor("x0", 0, 0, ("Ey", "Ez", "Hx"), freqs))
    sc.monitors.append(wm.PlaneMonitor("zmid", 2, 12, ("Ex", "Ey", "Hz"), freqs))
    cs = wm.compile_scene(sc, steps)
    solver, fields, mons = _run_engine(cs, steps)
    assert solver.info()["variant"] in (1, 2, 3)
    ref32 = orc.OracleSimulation(cs, "f32").run(steps)
    ref64 = orc.OracleSimulation(cs, "f64").run(steps)
    assert_fields_close(fields, ref32.fields)
    assert joint_rel_l2(fields, ref64.fields) < 2.0 * joint_rel_l2(ref32.fields, ref64.fields) + 1e-7
    assert_monitors_close(mons, ref32.monitor_results())
    # the tangential E on a PMC face is live (a PEC or CPML face would keep it zero)
    assert float(np.abs(fields["Ey"][0]).max()) > 1e-3 * float(np.abs(fields["Ey"]).max())
    ref32.close()
    ref64.close()
    solver.close()
