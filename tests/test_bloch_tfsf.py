"""CW plane wave through a TFSF slab on Bloch faces (the reference's grating-slab
provider, witwin/maxwell/fdtd/excitation/tfsf_state.py:202-279): the face terms
and the fold of the reference kernel's wrap copies on CPU (against a per-cell
restatement of add_bloch_source_patch_kernel, sources.cu:368-440), and on the
GPU the fused Bloch pair against the reference's own CUDA ops stepping the same
scene with the reference's own Bloch patch kernel (oracle/_ref, joint relative
L2 <= 1e-5), and the reference's confinement criterion (the scattered-field
region below the total-field maximum, tests/validation/physics/
test_bloch_broadband_vs_cw.py:173-213)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_package

BLOCH, PML = 3, 1
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _scene(wm, theta_deg=20.0, pol="s", steps_ramp=120, cells=(24, 20, 60)):
    th = math.radians(theta_deg)
    direction = (math.sin(th), 0.0, math.cos(th))
    polarization = (0.0, 1.0, 0.0) if pol == "s" else (math.cos(th), 0.0, -math.sin(th))
    sc = wm.Scene(cells=cells, spacing=25e-9, pml_cells=8, boundary=(BLOCH, BLOCH, BLOCH, BLOCH, PML, PML))
    dt = sc.resolve_dt()
    src = wm.PlaneWaveTFSF(direction, polarization, wm.CW(300e12, ramp_time=steps_ramp * dt), (0, 0, 20), (cells[0], cells[1], 40))
    sc.sources.append(src)
    k = wm.scene.tfsf_bloch_wavevector(sc, src)
    sc.bloch_k = (k[0], k[1], 0.0)
    sc.monitors.append(wm.PlaneMonitor("inside", 2, 30, ("Ex", "Ey", "Ez"), (300e12,)))
    sc.monitors.append(wm.PlaneMonitor("reflected", 2, 12, ("Ex", "Ey", "Ez"), (300e12,)))
    return sc


def _terms(wm, sc, cs, steps):
    curl = {n: cs.curl[n] if cs.curl[n] is not None else np.float32(cs.uniform[n][1]) for n in COMPONENTS}
    return wm.scene.grating_slab_terms(sc, sc.sources[0], curl, cs.dt, steps)


def _cw_delta(term, sig_c, sig_s):
    cp, sp = term.cos_patch.astype(np.float64), term.sin_patch.astype(np.float64)
    return (cp * sig_c + sp * sig_s) + 1j * (cp * sig_s - sp * sig_c)


def _kernel_restatement(wm, sc, term, delta_box):
    """Per-cell add_bloch_source_patch_kernel (sources.cu:368-440) for one term and
    its complex delta over the box: the field increment over the component's extent."""
    shape = wm.scene.component_shape(term.component, sc.nodes)
    out = np.zeros(shape, np.complex128)
    ph = wm.scene.bloch_patch_phases(sc, term.component)
    (ax_a, wrap_a, ca, sa), (ax_b, wrap_b, cb, sb) = ph
    b = term.box
    for i in range(b[1] - b[0]):
        for j in range(b[3] - b[2]):
            for k in range(b[5] - b[4]):
                delta = complex(delta_box[i, j, k])
                cell = [b[0] + i, b[2] + j, b[4] + k]
                out[tuple(cell)] += delta
                ca_, cb_ = cell[ax_a], cell[ax_b]
                bnd_a = wrap_a and (ca_ == 0 or ca_ + 1 >= shape[ax_a])
                bnd_b = wrap_b and (cb_ == 0 or cb_ + 1 >= shape[ax_b])
                rot_a = complex(ca, sa if ca_ == 0 else -sa)
                rot_b = complex(cb, sb if cb_ == 0 else -sb)
                pair_a = shape[ax_a] - 1 if ca_ == 0 else 0
                pair_b = shape[ax_b] - 1 if cb_ == 0 else 0
                if bnd_a:
                    t = list(cell)
                    t[ax_a] = pair_a
                    out[tuple(t)] += rot_a * delta
                if bnd_b:
                    t = list(cell)
                    t[ax_b] = pair_b
                    out[tuple(t)] += rot_b * delta
                if bnd_a and bnd_b:
                    t = list(cell)
                    t[ax_a], t[ax_b] = pair_a, pair_b
                    out[tuple(t)] += rot_a * rot_b * delta
    return out


def test_face_terms_and_checks():
    wm = load_package()
    sc = _scene(wm)
    cs = wm.compile_scene(sc, 40)
    assert cs.complex_fields and cs.aux_line is None
    by_channel = {0: [], 1: []}
    for p in cs.patches:
        by_channel[p.channel].append(p)
    assert len(by_channel[0]) == len(by_channel[1]) == 8  # Ey and Hx terms on both faces, s_c and s_s
    terms = _terms(wm, sc, cs, 40)
    assert [t.component for t in terms] == ["Ey", "Ey", "Hx", "Hx"]
    # at step n the unfolded term carries scale * e^{i (omega t + phase - omega delay)}
    t0 = terms[0]
    n = 25
    delta = (t0.cos_patch * t0.signal_cos[n] + t0.sin_patch * t0.signal_sin[n]
             + 1j * (t0.cos_patch * t0.signal_sin[n] - t0.sin_patch * t0.signal_cos[n]))
    np.testing.assert_allclose(np.abs(delta), np.hypot(t0.cos_patch, t0.sin_patch) * abs(t0.signal_cos[n] + 1j * t0.signal_sin[n]),
                               rtol=1e-5, atol=1e-12)
    # the transverse phase of the incident advances by -k_x d per cell (e^{-i k.r})
    phase = np.angle(t0.cos_patch + 1j * t0.sin_patch)[:, 0, 0]
    step = np.angle(np.exp(1j * np.diff(phase)))
    np.testing.assert_allclose(step, sc.bloch_k[0] * sc.spacing, rtol=1e-4)
    # the compiled per-channel patches equal the reference kernel's cell-by-cell
    # increments, wrap copies included, for every term at two signal values
    rng = np.random.default_rng(3)
    for x, t in enumerate(terms):
        comp_patches = [p for p in cs.patches if p.component == t.component and p.box == t.box]
        assert len(comp_patches) == 4
        for sig_c, sig_s in rng.normal(size=(2, 2)):
            want = _kernel_restatement(wm, sc, t, _cw_delta(t, sig_c, sig_s))
            got = np.zeros_like(want)
            b = t.box
            for p in comp_patches:
                sig = sig_c if np.array_equal(p.signal, t.signal_cos) else sig_s
                got[b[0]:b[1], b[2]:b[3], b[4]:b[5]] += (1 if p.channel == 0 else 1j) * p.coeff.astype(np.float64) * sig
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6 * np.abs(want).max())
    # a CW wave whose Bloch wavevector does not match it, an injection along a Bloch axis
    bad = _scene(wm)
    bad.bloch_k = (0.5 * bad.bloch_k[0], 0.0, 0.0)
    with pytest.raises(ValueError):
        wm.compile_scene(bad, 10)
    along_x = _scene(wm)
    along_x.sources[0] = wm.PlaneWaveTFSF((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), wm.GaussianPulse(300e12, 100e12),
                                          (4, 0, 0), (20, 20, 60))
    with pytest.raises(ValueError):
        wm.compile_scene(along_x, 10)
    # the reference's slab checks (tfsf_state.py:171-199): faces inside the non-CPML
    # region, in vacuum
    in_pml = _scene(wm)
    w = in_pml.sources[0]
    in_pml.sources[0] = wm.PlaneWaveTFSF(w.direction, w.polarization, w.source_time, (0, 0, 4), (24, 20, 40))
    with pytest.raises(ValueError):
        wm.compile_scene(in_pml, 10)
    dielectric_face = _scene(wm)
    dielectric_face.structures.append(wm.Structure(wm.Box((0, 0, 38), (24, 20, 44)), wm.Medium(2.0)))
    with pytest.raises(ValueError):
        wm.compile_scene(dielectric_face, 10)
    inside = _scene(wm)
    inside.structures.append(wm.Structure(wm.Box((0, 0, 26), (24, 20, 32)), wm.Medium(2.0)))
    wm.compile_scene(inside, 10)


@pytest.mark.gpu
@pytest.mark.parametrize("pol", ["s", "p"])
def test_bloch_tfsf_slab_matches_reference_ops(pol):
    from oracle import ref_gpu
    from test_bloch import FIELDS, TOL, joint

    if not ref_gpu.available():
        pytest.skip("oracle/_ref not built")
    wm = load_package()
    steps = 400
    sc = _scene(wm, pol=pol)
    cs = wm.compile_scene(sc, steps)
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, steps)
    got = {**{f"re_{n}": solver.field(n).cpu().numpy() for n in FIELDS},
           **{f"im_{n}": solver.field(n, imag=True).cpu().numpy() for n in FIELDS}}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    solver.close()
    phases = {c: [(w, co, si) for _a, w, co, si in wm.scene.bloch_patch_phases(sc, c)] for c in COMPONENTS}
    ref = ref_gpu.RefGpuBloch(cs, bloch_terms=_terms(wm, sc, cs, steps), term_phases=phases).run(steps)
    ref_re, ref_im = ref.fields()
    want = {**{f"re_{n}": ref_re[n] for n in FIELDS}, **{f"im_{n}": ref_im[n] for n in FIELDS}}
    err = joint(got, want)
    print(f"TFSF slab on Bloch faces ({pol}) vs the reference's ops: joint relative L2 {err:.2e}")
    assert err < TOL
    refm = ref.monitor_results()
    for m in refm:
        assert joint(mons[m], refm[m]) < TOL, m


@pytest.mark.gpu
@pytest.mark.parametrize("pol", ["s", "p"])
def test_bloch_tfsf_slab_confines_total_field(pol):
    wm = load_package()
    steps = 1200
    cs = wm.compile_scene(_scene(wm, pol=pol), steps)
    eng = wm.solver.B200FDTD(cs).init_field()
    eng.step_range(0, steps)
    e = {n: eng.field(n).cpu().numpy() + 1j * eng.field(n, imag=True).cpu().numpy() for n in ("Ex", "Ey", "Ez")}
    eng.close()
    assert all(np.isfinite(np.abs(v)).all() for v in e.values())
    inside = max(float(np.abs(v[:, :, 24:36]).max()) for v in e.values())
    outside = max(max(float(np.abs(v[:, :, 10:17]).max()), float(np.abs(v[:, :, 44:50]).max())) for v in e.values())
    print(f"TFSF slab on Bloch faces ({pol}): inside {inside:.3e}, outside {outside:.3e}, ratio {outside / inside:.2e}")
    assert inside > 0.1
    assert outside < inside


def _grating(wm):
    """The large grating's shape on a small copy: Bloch x / y (k_x = 0.1 * 2 pi / L_x),
    8-cell CPML on z, the Debye layer and the pulsed TFSF slab, 64 x 64 x 48 cells."""
    return wm.workloads.bloch_grating(cells=(64, 64, 48), pml=8, n_freq=4)


def test_pulsed_slab_terms_fold():
    from oracle.oracle import shifted_waveform

    wm = load_package()
    sc = _grating(wm)
    steps = 60
    cs = wm.compile_scene(sc, steps)
    assert cs.complex_fields and not cs.patches
    # Ex and Hy terms on both faces; the x copies of Hy carry the Bloch phase into
    # the imaginary channel, the y copies of Ex (k_y = 0) stay real
    assert sorted((p.component, p.channel) for p in cs.shifted) == [
        ("Ex", 0), ("Ex", 0), ("Hy", 0), ("Hy", 0), ("Hy", 1), ("Hy", 1)]
    terms = _terms(wm, sc, cs, steps)
    assert [t.component for t in terms] == ["Ex", "Ex", "Hy", "Hy"]
    for t in terms:
        for n in (7, 31):
            w = shifted_waveform(t.source_time, n * cs.dt + t.t_offset - t.delay.astype(np.float64))
            want = _kernel_restatement(wm, sc, t, t.scale.astype(np.float64) * w)
            got = np.zeros_like(want)
            for p in cs.shifted:
                if p.component != t.component or p.t_offset != t.t_offset:
                    continue
                b = p.box
                if not (b[4] == t.box[4] and b[5] == t.box[5]):
                    continue
                wp = shifted_waveform(p.source_time, n * cs.dt + p.t_offset - p.delay.astype(np.float64))
                got[b[0]:b[1], b[2]:b[3], b[4]:b[5]] += (1 if p.channel == 0 else 1j) * p.scale.astype(np.float64) * wp
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6 * max(np.abs(want).max(), 1e-30))


@pytest.mark.gpu
def test_grating_workload_slab_matches_reference_ops():
    """The pulsed TFSF slab of the grating workload (small copy, 300 steps) with
    the Debye layer and z CPML, against the reference's ops with its own Bloch
    patch kernel."""
    from oracle import ref_gpu
    from test_bloch import FIELDS, TOL, joint

    if not ref_gpu.available():
        pytest.skip("oracle/_ref not built")
    wm = load_package()
    steps = 300
    sc = _grating(wm)
    cs = wm.compile_scene(sc, steps)
    solver = wm.solver.B200FDTD(cs).init_field()
    solver.step_range(0, steps)
    got = {**{f"re_{n}": solver.field(n).cpu().numpy() for n in FIELDS},
           **{f"im_{n}": solver.field(n, imag=True).cpu().numpy() for n in FIELDS}}
    mons = {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in solver.monitor_results().items()}
    solver.close()
    phases = {c: [(w, co, si) for _a, w, co, si in wm.scene.bloch_patch_phases(sc, c)] for c in COMPONENTS}
    ref = ref_gpu.RefGpuBloch(cs, bloch_terms=_terms(wm, sc, cs, steps), term_phases=phases)
    assert ref.z_cpml
    ref.run(steps)
    ref_re, ref_im = ref.fields()
    want = {**{f"re_{n}": ref_re[n] for n in FIELDS}, **{f"im_{n}": ref_im[n] for n in FIELDS}}
    assert np.linalg.norm(want["re_Ex"]) > 0 and np.linalg.norm(want["im_Ex"]) > 1e-3 * np.linalg.norm(want["re_Ex"])
    err = joint(got, want)
    print(f"grating workload TFSF slab vs the reference's ops: joint relative L2 {err:.2e}")
    assert err < TOL
    refm = ref.monitor_results()
    for m in refm:
        assert joint(mons[m], refm[m]) < TOL, m


def test_auto_bloch_wavevector():
    """bloch_k = "auto" resolves to the CW plane wave's wavevector on the Bloch axes
    (witwin/maxwell/fdtd/boundary/bloch.py:60-78) and compiles the same patches."""
    wm = load_package()
    sc = _scene(wm)
    auto = _scene(wm)
    auto.bloch_k = "auto"
    assert wm.scene.resolve_bloch_wavevector(auto) == (sc.bloch_k[0], sc.bloch_k[1], 0.0)
    a, b = wm.compile_scene(auto, 20), wm.compile_scene(sc, 20)
    assert a.bloch_cos == b.bloch_cos and a.bloch_sin == b.bloch_sin
    for p, q in zip(a.patches, b.patches):
        np.testing.assert_array_equal(p.coeff, q.coeff)
    pulsed = _grating(wm)
    pulsed.bloch_k = "auto"
    with pytest.raises(ValueError):
        wm.compile_scene(pulsed, 10)


@pytest.mark.gpu
def test_grating_bf16_storage_tracks_fp32():
    """BF16 field storage on the Bloch pair (wrap faces included, Debye pole state
    in BF16): the grating copy's diffraction monitor within the BF16 bound of the
    FP32 pair; FP16 storage on Bloch faces is refused."""
    from test_precision import BF16_TOL, joint_rel_l2

    wm = load_package()
    steps = 300
    cs = wm.compile_scene(_grating(wm), steps)
    mons = {}
    for storage in ("fp32", "bf16"):
        solver = wm.solver.B200FDTD(cs, storage=storage).init_field()
        solver.step_range(0, steps)
        mons[storage] = {f"{m}_{c}": v.cpu().numpy() for m, d in solver.monitor_results().items() for c, v in d.items()}
        solver.close()
    err = joint_rel_l2(mons["bf16"], mons["fp32"])
    print(f"grating copy, BF16 storage on the Bloch pair: monitor joint relative L2 {err:.2e}")
    assert 0.0 < err <= BF16_TOL
    with pytest.raises(Exception):
        wm.solver.B200FDTD(cs, storage="fp16").init_field()
