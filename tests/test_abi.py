"""CPU checks of the drop-in boundary: the C ABI library loads, exports every
symbol include/fdtd_b200.h declares, and the Python binding covers them; the
scene compiler's host logic (CPML profiles, ADE templates, TFSF terms) holds
its invariants.  No kernel is launched here."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_package

HEADER = ROOT / "include" / "fdtd_b200.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"^\s*(?:const\s+char\*|int)\s+(fdtd_\w+)\s*\(", text, flags=re.M))


def test_library_exports_every_declared_symbol():
    wm = load_package()
    lib = wm._lib.load()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(wm._lib.EXPORTED_SYMBOLS) >= names, sorted(names - set(wm._lib.EXPORTED_SYMBOLS))
    assert lib.fdtd_version().startswith(b"fdtd_b200")


def test_backend_name_table_matches_reference_names():
    wm = load_package()
    from witwin_maxwell_b200 import backend

    for comp in ("Hx", "Hy", "Hz"):
        for suffix in ("Standard3D", "3D", "CpmlCompressed3D"):
            assert f"updateMagneticField{comp}{suffix}" in backend._KERNELS
    for comp in ("Ex", "Ey", "Ez"):
        for suffix in ("Standard3D", "Cpml3D", "CpmlCompressed3D"):
            assert f"updateElectricField{comp}{suffix}" in backend._KERNELS
    with pytest.raises(AttributeError):
        backend.NativeFDTDModule().notAKernel3D
    del wm


def test_cpml_profile_shape_and_grading():
    wm = load_package()
    sc = wm.Scene(cells=(32, 32, 32), spacing=25e-9, pml_cells=8)
    cs = wm.compile_scene(sc, 10)
    for a in range(3):
        b_e, c_e = cs.cpml["b_e"][a], cs.cpml["c_e"][a]
        assert b_e.shape == (33,) and cs.cpml["b_h"][a].shape == (32,)
        # outside the layer: b = 1, c = 0; inside: 0 < b < 1 and c < 0, growing with depth
        assert np.all(b_e[9:24] == 1.0) and np.all(c_e[9:24] == 0.0)
        assert np.all((b_e[:8] > 0) & (b_e[:8] < 1))
        assert np.all(np.diff(b_e[:9]) > 0)
        assert np.allclose(b_e, b_e[::-1])


def test_ade_templates_match_closed_form():
    wm = load_package()
    sc = wm.Scene(cells=(16, 16, 16), spacing=25e-9, pml_cells=4)
    sc.structures.append(wm.Structure(wm.Box((6, 6, 6), (10, 10, 10)), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    cs = wm.compile_scene(sc, 10)
    dt = cs.dt
    g = 2 * np.pi * 20e12
    w0 = 2 * np.pi * 250e12
    lor = [p for p in cs.poles if p.kind == 2]
    assert len(lor) == 3
    for p in lor:
        assert p.decay == pytest.approx((2 - g * dt) / (2 + g * dt))
        assert p.restoring == pytest.approx(2 * w0 * w0 * dt / (2 + g * dt))
        base = 2 * wm.scene.EPSILON_0 * 3.0 * w0 * w0 * dt / (2 + g * dt)
        assert float(p.drive.max()) == pytest.approx(base, rel=1e-6)
        # interior component cells carry eps_inf = 2
        assert float((1.0 / p.inv_eps).max()) == pytest.approx(2.0 * wm.scene.EPSILON_0, rel=1e-6)


def test_tfsf_terms_cover_the_box_faces():
    wm = load_package()
    sc = wm.Scene(cells=(32, 24, 24), spacing=25e-9, pml_cells=6)
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (8, 8, 8), (24, 16, 16)))
    cs = wm.compile_scene(sc, 20)
    comps = sorted((lp.component, lp.box[0], lp.box[2], lp.box[4]) for lp in cs.line_patches)
    # Ez polarisation, +x: H corrections read incident Ez (Hy on x faces, Hx on y faces),
    # E corrections read incident Hy (Ez on x faces, Ex on z faces).
    assert {c[0] for c in comps} == {"Hx", "Hy", "Ez", "Ex"}
    assert len(cs.line_patches) == 8
    src = cs.aux_line
    assert src.e_decay.size == 33 + 20
    assert src.source[0] == np.float32(wm.GaussianPulse(300e12, 100e12).evaluate(0.0))
