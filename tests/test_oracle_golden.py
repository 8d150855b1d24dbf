"""Pin the CPU oracle to the reference: every restated op and a 60-step run of a
small scene must reproduce the golden vectors that tests/golden/make_golden.py
recorded from the reference's frozen Torch kernels (float64)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import load_package
from oracle import oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden"
ATOL = 1e-12


@pytest.fixture(scope="module")
def ops():
    return dict(np.load(GOLDEN / "ops.npz"))


@pytest.fixture(scope="module")
def lib():
    orc.build()
    return orc.load("f64")


def _p(a):
    return orc._p(a)


H_SPEC = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey")}
E_SPEC = {"Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}
AX = {"x": 0, "y": 1, "z": 2}


@pytest.mark.parametrize("comp", ["Hx", "Hy", "Hz"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_magnetic_update_matches_reference(ops, lib, comp, mode):
    A, B, first, second = H_SPEC[comp]
    F = {n: ops[f"in_{n}"].copy() for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    H = F[comp]
    L = 2
    shape = H.shape
    if mode == 0:
        pa = pb = None
        slab = (0, 0, 0, 0, 0, 0)
        key = f"out_h_std_{comp}"
    elif mode == 1:
        pa, pb = ops[f"h_{comp}_psiA"].copy(), ops[f"h_{comp}_psiB"].copy()
        slab = (0, 0, 0, 0, 0, 0)
        key = f"out_h_dense_{comp}"
    else:
        pa, pb = ops[f"h_{comp}_cpsi0"].copy(), ops[f"h_{comp}_cpsi1"].copy()
        slab = (L, shape[AX[A]] - L, L, L, shape[AX[B]] - L, L)
        key = f"out_h_comp_{comp}"
    cp = lambda q, a: ops[f"cp_{q}_h_{a}"]  # noqa: E731
    lib.oracle_h_update(0, shape[0], "xyz".index(comp[1]), mode, *shape, _p(H), _p(F[first]), _p(F[second]),
                        _p(ops[f"h_{comp}_decay"]), _p(ops[f"h_{comp}_curl"]), _p(ops[f"inv_h_{A}"]), _p(ops[f"inv_h_{B}"]),
                        _p(pa), _p(pb), _p(cp("ik", A)), _p(cp("b", A)), _p(cp("c", A)), _p(cp("ik", B)), _p(cp("b", B)),
                        _p(cp("c", B)), *slab)
    np.testing.assert_allclose(H, ops[key], rtol=0, atol=ATOL)
    if mode == 1:
        np.testing.assert_allclose(pa, ops[f"{key}_psiA"], rtol=0, atol=ATOL)
        np.testing.assert_allclose(pb, ops[f"{key}_psiB"], rtol=0, atol=ATOL)
    if mode == 2:
        np.testing.assert_allclose(pa, ops[f"{key}_psi0"], rtol=0, atol=ATOL)
        np.testing.assert_allclose(pb, ops[f"{key}_psi1"], rtol=0, atol=ATOL)


@pytest.mark.parametrize("comp", ["Ex", "Ey", "Ez"])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("mname", ["pml", "pec", "mixed", "pmc"])
def test_electric_update_matches_reference(ops, lib, comp, mode, mname):
    A, B, first, second = E_SPEC[comp]
    F = {n: ops[f"in_{n}"].copy() for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    E = F[comp]
    shape = E.shape
    modes = [int(v) for v in ops[f"e_modes_{mname}"]]
    L = 2
    if mode == 0:
        pa = pb = None
        slab = (0, 0, 0, 0, 0, 0)
        key = f"out_e_std_{comp}_{mname}"
    elif mode == 1:
        pa, pb = ops[f"e_{comp}_{mname}_psiA"].copy(), ops[f"e_{comp}_{mname}_psiB"].copy()
        slab = (0, 0, 0, 0, 0, 0)
        key = f"out_e_dense_{comp}_{mname}"
    else:
        pa, pb = ops[f"e_{comp}_{mname}_cpsi0"].copy(), ops[f"e_{comp}_{mname}_cpsi1"].copy()
        slab = (L, shape[AX[A]] - L, L, L, shape[AX[B]] - L, L)
        key = f"out_e_comp_{comp}_{mname}"
    cp = lambda q, a: ops[f"cp_{q}_e_{a}"]  # noqa: E731
    lib.oracle_e_update(0, shape[0], "xyz".index(comp[1]), mode, *shape, _p(E), _p(F[first]), _p(F[second]),
                        _p(ops[f"e_{comp}_decay"]), _p(ops[f"e_{comp}_curl"]), _p(ops[f"inv_e_{A}"]), _p(ops[f"inv_e_{B}"]),
                        *modes, _p(pa), _p(pb), _p(cp("ik", A)), _p(cp("b", A)), _p(cp("c", A)), _p(cp("ik", B)),
                        _p(cp("b", B)), _p(cp("c", B)), *slab)
    np.testing.assert_allclose(E, ops[key], rtol=0, atol=ATOL)
    if mode == 1:
        np.testing.assert_allclose(pa, ops[f"{key}_psiA"], rtol=0, atol=ATOL)
        np.testing.assert_allclose(pb, ops[f"{key}_psiB"], rtol=0, atol=ATOL)
    if mode == 2:
        np.testing.assert_allclose(pa, ops[f"{key}_psi0"], rtol=0, atol=ATOL)
        np.testing.assert_allclose(pb, ops[f"{key}_psi1"], rtol=0, atol=ATOL)


def test_ade_ops_match_reference(ops, lib):
    e, drive, p0, j0, inv_eps = (ops[k] for k in ("ade_e", "ade_drive", "ade_p0", "ade_j0", "ade_inv_eps"))
    n = e.size
    P, J = p0.copy(), j0.copy()
    lib.oracle_debye(0, n, _p(e), _p(drive), 0.7, 0.3, _p(P), _p(J))
    np.testing.assert_allclose(P, ops["out_debye_p"], atol=ATOL)
    np.testing.assert_allclose(J, ops["out_debye_j"], atol=ATOL)
    J = j0.copy()
    lib.oracle_drude(0, n, _p(e), _p(drive), 0.8, _p(J))
    np.testing.assert_allclose(J, ops["out_drude_j"], atol=ATOL)
    P, J = p0.copy(), j0.copy()
    lib.oracle_lorentz(0, n, _p(e), _p(drive), 0.9, 0.05, 0.3, _p(P), _p(J))
    np.testing.assert_allclose(P, ops["out_lorentz_p"], atol=ATOL)
    np.testing.assert_allclose(J, ops["out_lorentz_j"], atol=ATOL)
    E = e.copy()
    lib.oracle_apply_polarization(0, n, _p(j0), _p(inv_eps), 0.3, _p(E))
    np.testing.assert_allclose(E, ops["out_apply_e"], atol=ATOL)


def test_patches_and_incident_line_match_reference(ops, lib):
    f = ops["patch_field"].copy()
    patch = ops["patch"]
    lib.oracle_add_patch(*f.shape, _p(f), *patch.shape, _p(patch), 3, -1, 2, 0.75)
    np.testing.assert_allclose(f, ops["out_patch"], atol=ATOL)
    f = ops["patch_field"].copy()
    coeff, inc, idx = ops["line_coeff"], ops["line_inc"], ops["line_idx"].astype(np.int64)
    lib.oracle_add_line_patch(*f.shape, _p(f), *coeff.shape, _p(coeff), _p(inc), _p(idx), 0, 1, 1, 1, -0.6)
    np.testing.assert_allclose(f, ops["out_line"], atol=ATOL)
    h, e = ops["aux_h"].copy(), ops["aux_e"].copy()
    lib.oracle_aux_magnetic(e.size, _p(h), _p(e), _p(ops["aux_hd"]), _p(ops["aux_hc"]))
    np.testing.assert_allclose(h, ops["out_aux_h"], atol=ATOL)
    lib.oracle_aux_electric(e.size, _p(e), _p(h), _p(ops["aux_ed"]), _p(ops["aux_ec"]), 3, 0.25)
    np.testing.assert_allclose(e, ops["out_aux_e"], atol=ATOL)


def test_observers_and_volume_dft_match_reference(ops, lib):
    fld = ops["obs_field"]
    re, im = ops["obs_re0"].copy(), ops["obs_im0"].copy()
    pi, pj, pk = (ops[k].astype(np.int32) for k in ("obs_pi", "obs_pj", "obs_pk"))
    lib.oracle_point_observers(fld.shape[1], fld.shape[2], _p(fld), 3, _p(pi), _p(pj), _p(pk), _p(re), _p(im), 0.3, -0.7)
    np.testing.assert_allclose(re, ops["out_points_re"], atol=ATOL)
    np.testing.assert_allclose(im, ops["out_points_im"], atol=ATOL)
    for axis in range(3):
        re, im = ops[f"obs_plane{axis}_re0"].copy(), ops[f"obs_plane{axis}_im0"].copy()
        lib.oracle_plane_observer(*fld.shape, _p(fld), axis, 1, _p(re), _p(im), 0.4, 0.2)
        np.testing.assert_allclose(re, ops[f"out_plane{axis}_re"], atol=ATOL)
        np.testing.assert_allclose(im, ops[f"out_plane{axis}_im"], atol=ATOL)
    wc, ws = ops["dft_wc"], ops["dft_ws"]
    for k in ("Ex", "Ey", "Ez"):
        v = ops[f"dft_{k.lower()}"]
        re = np.zeros((2,) + v.shape)
        im = np.zeros((2,) + v.shape)
        lib.oracle_dft_volume(0, v.size, v.size, 2, _p(v), _p(re), _p(im), _p(wc), _p(ws))
        np.testing.assert_allclose(re, ops[f"out_dft_{k}_re"], atol=ATOL)
        np.testing.assert_allclose(im, ops[f"out_dft_{k}_im"], atol=ATOL)


def _rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / den) if den > 0 else float(np.linalg.norm(a.ravel()))


def test_oracle_stepping_matches_reference_run():
    """60 steps through the oracle == 60 steps through the reference's Torch ops."""
    import importlib.util
    import sys

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    sys.modules["make_golden"] = mg
    spec.loader.exec_module(mg)
    wm = load_package()
    gold = dict(np.load(GOLDEN / "steps.npz"))
    cs = wm.compile_scene(mg.golden_scene(), int(gold["steps"]))
    # the scene compiler must still produce the inputs the goldens were made from
    assert float(np.abs(cs.curl["Ex"]).sum()) == pytest.approx(float(gold["check_curl_Ex"]), rel=1e-12)
    np.testing.assert_allclose([np.abs(p.drive).sum() for p in cs.poles], gold["check_poles"], rtol=1e-12)
    np.testing.assert_allclose([np.abs(p.coeff).sum() for p in cs.patches], gold["check_patch"], rtol=1e-12)
    np.testing.assert_allclose([np.abs(p.coeff).sum() for p in cs.line_patches], gold["check_lines"], rtol=1e-12)
    sim = orc.OracleSimulation(cs, "f64", threads=2).run(int(gold["steps"]))
    for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert np.abs(gold[f"field_{n}"]).max() > 0
        assert _rel_l2(sim.fields[n], gold[f"field_{n}"]) < 1e-12, n
    for i, (re, im) in enumerate(sim.acc):
        assert _rel_l2(re, gold[f"dft_{i}_re"]) < 1e-12
        assert _rel_l2(im, gold[f"dft_{i}_im"]) < 1e-12
    assert sim.window_sum == pytest.approx(float(gold["window_sum"]))
    sim.close()
