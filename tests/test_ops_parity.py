"""GPU parity of the per-op C ABI (through the NativeFDTDModule-compatible backend)
against the golden vectors recorded from the reference's Torch kernels.

Inputs are the golden float64 inputs cast to float32; tolerance rtol 1e-5,
atol 1e-6 (values are O(1)), the FP32 rounding of one op.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import load_package

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
RTOL, ATOL = 1e-5, 1e-6
AX = {"x": 0, "y": 1, "z": 2}


@pytest.fixture(scope="module")
def ops():
    return dict(np.load(GOLDEN / "ops.npz"))


@pytest.fixture(scope="module")
def mod():
    wm = load_package()
    return wm.backend.get_native_fdtd_module()


def g(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def close(t, ref):
    np.testing.assert_allclose(t.cpu().numpy(), ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("comp", ["Hx", "Hy", "Hz"])
@pytest.mark.parametrize("mode", ["std", "dense", "comp"])
def test_magnetic_ops(ops, mod, comp, mode):
    A, B, first, second = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey")}[comp]
    U, V = A.upper(), B.upper()
    H = g(ops[f"in_{comp}"])
    kw = {comp: H, first: g(ops[f"in_{first}"]), second: g(ops[f"in_{second}"]),
          f"{comp}Decay": g(ops[f"h_{comp}_decay"]), f"{comp}Curl": g(ops[f"h_{comp}_curl"]),
          f"invD{A}": g(ops[f"inv_h_{A}"]), f"invD{B}": g(ops[f"inv_h_{B}"])}
    if mode == "std":
        getattr(mod, f"updateMagneticField{comp}Standard3D")(**kw).launchRaw()
        close(H, ops[f"out_h_std_{comp}"])
        return
    prof = {f"InvKappa{comp}{U}": g(ops[f"cp_ik_h_{A}"]), f"By{comp}{U}": g(ops[f"cp_b_h_{A}"]),
            f"Cy{comp}{U}": g(ops[f"cp_c_h_{A}"]), f"InvKappa{comp}{V}": g(ops[f"cp_ik_h_{B}"]),
            f"By{comp}{V}": g(ops[f"cp_b_h_{B}"]), f"Cy{comp}{V}": g(ops[f"cp_c_h_{B}"])}
    if mode == "dense":
        pa, pb = g(ops[f"h_{comp}_psiA"]), g(ops[f"h_{comp}_psiB"])
        getattr(mod, f"updateMagneticField{comp}3D")(**kw, **prof, **{f"Psi{comp}{U}": pa, f"Psi{comp}{V}": pb}).launchRaw()
        close(H, ops[f"out_h_dense_{comp}"])
        close(pa, ops[f"out_h_dense_{comp}_psiA"])
        close(pb, ops[f"out_h_dense_{comp}_psiB"])
        return
    shape = ops[f"in_{comp}"].shape
    pa, pb = g(ops[f"h_{comp}_cpsi0"]), g(ops[f"h_{comp}_cpsi1"])
    L = 2
    getattr(mod, f"updateMagneticField{comp}CpmlCompressed3D")(
        **kw, **prof, **{f"Psi{comp}{U}": pa, f"Psi{comp}{V}": pb},
        **{f"psi{comp}{U}LowLength": L, f"psi{comp}{U}HighStart": shape[AX[A]] - L, f"psi{comp}{U}HighLength": L,
           f"psi{comp}{V}LowLength": L, f"psi{comp}{V}HighStart": shape[AX[B]] - L, f"psi{comp}{V}HighLength": L},
        uniformDecay=None, uniformCurl=None).launchRaw()
    close(H, ops[f"out_h_comp_{comp}"])
    close(pa, ops[f"out_h_comp_{comp}_psi0"])
    close(pb, ops[f"out_h_comp_{comp}_psi1"])


@pytest.mark.parametrize("comp", ["Ex", "Ey", "Ez"])
@pytest.mark.parametrize("mode", ["std", "dense", "comp"])
@pytest.mark.parametrize("mname", ["pml", "pec", "mixed", "pmc"])
def test_electric_ops(ops, mod, comp, mode, mname):
    A, B, first, second = {"Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}[comp]
    U, V = A.upper(), B.upper()
    modes = [int(v) for v in ops[f"e_modes_{mname}"]]
    E = g(ops[f"in_{comp}"])
    kw = {comp: E, first: g(ops[f"in_{first}"]), second: g(ops[f"in_{second}"]),
          f"{comp}Decay": g(ops[f"e_{comp}_decay"]), f"{comp}Curl": g(ops[f"e_{comp}_curl"]),
          f"invD{A}": g(ops[f"inv_e_{A}"]), f"invD{B}": g(ops[f"inv_e_{B}"]),
          f"{A}LowBoundaryMode": modes[0], f"{A}HighBoundaryMode": modes[1],
          f"{B}LowBoundaryMode": modes[2], f"{B}HighBoundaryMode": modes[3]}
    if mode == "std":
        getattr(mod, f"updateElectricField{comp}Standard3D")(**kw).launchRaw()
        close(E, ops[f"out_e_std_{comp}_{mname}"])
        return
    prof = {f"InvKappa{comp}{U}": g(ops[f"cp_ik_e_{A}"]), f"B{comp}{U}": g(ops[f"cp_b_e_{A}"]),
            f"C{comp}{U}": g(ops[f"cp_c_e_{A}"]), f"InvKappa{comp}{V}": g(ops[f"cp_ik_e_{B}"]),
            f"B{comp}{V}": g(ops[f"cp_b_e_{B}"]), f"C{comp}{V}": g(ops[f"cp_c_e_{B}"])}
    if mode == "dense":
        pa, pb = g(ops[f"e_{comp}_{mname}_psiA"]), g(ops[f"e_{comp}_{mname}_psiB"])
        getattr(mod, f"updateElectricField{comp}Cpml3D")(**kw, **prof, **{f"Psi{comp}{U}": pa, f"Psi{comp}{V}": pb}).launchRaw()
        close(E, ops[f"out_e_dense_{comp}_{mname}"])
        close(pa, ops[f"out_e_dense_{comp}_{mname}_psiA"])
        close(pb, ops[f"out_e_dense_{comp}_{mname}_psiB"])
        return
    shape = ops[f"in_{comp}"].shape
    pa, pb = g(ops[f"e_{comp}_{mname}_cpsi0"]), g(ops[f"e_{comp}_{mname}_cpsi1"])
    L = 2
    getattr(mod, f"updateElectricField{comp}CpmlCompressed3D")(
        **kw, **prof, **{f"Psi{comp}{U}": pa, f"Psi{comp}{V}": pb},
        **{f"psi{comp}{U}LowLength": L, f"psi{comp}{U}HighStart": shape[AX[A]] - L, f"psi{comp}{U}HighLength": L,
           f"psi{comp}{V}LowLength": L, f"psi{comp}{V}HighStart": shape[AX[B]] - L, f"psi{comp}{V}HighLength": L},
        uniformDecay=None, uniformCurl=None).launchRaw()
    close(E, ops[f"out_e_comp_{comp}_{mname}"])
    close(pa, ops[f"out_e_comp_{comp}_{mname}_psi0"])
    close(pb, ops[f"out_e_comp_{comp}_{mname}_psi1"])


def test_ade_ops(ops, mod):
    e, drive = g(ops["ade_e"]), g(ops["ade_drive"])
    P, J = g(ops["ade_p0"]), g(ops["ade_j0"])
    mod.updateDebyeCurrent3D(ElectricField=e, Polarization=P, PolarizationCurrent=J, DebyeDrive=drive, decay=0.7, dt=0.3).launchRaw()
    close(P, ops["out_debye_p"])
    np.testing.assert_allclose(J.cpu().numpy(), ops["out_debye_j"], rtol=1e-4, atol=1e-5)  # (P'-P)/dt cancels digits
    J = g(ops["ade_j0"])
    mod.updateDrudeCurrent3D(ElectricField=e, PolarizationCurrent=J, DrudeDrive=drive, decay=0.8).launchRaw()
    close(J, ops["out_drude_j"])
    P, J = g(ops["ade_p0"]), g(ops["ade_j0"])
    mod.updateLorentzCurrent3D(ElectricField=e, Polarization=P, PolarizationCurrent=J, LorentzDrive=drive, decay=0.9,
                               restoring=0.05, dt=0.3).launchRaw()
    close(P, ops["out_lorentz_p"])
    close(J, ops["out_lorentz_j"])
    E = g(ops["ade_e"])
    mod.applyPolarizationCurrent3D(ElectricField=E, PolarizationCurrent=g(ops["ade_j0"]),
                                   InvPermittivity=g(ops["ade_inv_eps"]), dt=0.3).launchRaw()
    close(E, ops["out_apply_e"])


def test_patch_line_aux_ops(ops, mod):
    f = g(ops["patch_field"])
    mod.addSourcePatch3D(field=f, sourcePatch=g(ops["patch"]), offsetI=3, offsetJ=-1, offsetK=2, signal=0.75).launchRaw()
    close(f, ops["out_patch"])
    f = g(ops["patch_field"])
    mod.addCwPhasedSourcePatch3D(field=f, sourcePatchCos=g(ops["cw_cos"]), sourcePatchSin=g(ops["cw_sin"]), offsetI=3,
                                 offsetJ=-1, offsetK=2, signalCos=0.6, signalSin=-0.3).launchRaw()
    close(f, ops["out_cw_patch"])
    for kind, gate in ((0, 0), (1, 0), (1, 1), (2, 1)):
        f = g(ops["patch_field"])
        mod.addTimeShiftedSourcePatch3D(field=f, sourcePatch=g(ops["patch"]), delayPatch=g(ops["shift_delay"]),
                                        activationDelayPatch=g(ops["shift_act"]), offsetI=3, offsetJ=-1, offsetK=2,
                                        timeKind=kind, time=1.1e-14, frequency=300e12, fwidth=100e12, amplitude=1.3,
                                        phase=0.2, delay=9.5e-15, causalGate=gate).launchRaw()
        close(f, ops[f"out_shift_{kind}_{gate}"])
    f = g(ops["patch_field"])
    mod.addScaledLineSourcePatch3D(field=f, coeffPatch=g(ops["line_coeff"]), incidentField=g(ops["line_inc"]),
                                   sampleIndices=g(ops["line_idx"], torch.int64), sampleAxisCode=0, offsetI=1,
                                   offsetJ=1, offsetK=1, scale=-0.6).launchRaw()
    close(f, ops["out_line"])
    h, e = g(ops["aux_h"]), g(ops["aux_e"])
    mod.updateAuxiliaryMagnetic1D(Magnetic=h, Electric=e, MagneticDecay=g(ops["aux_hd"]), MagneticCurl=g(ops["aux_hc"])).launchRaw()
    close(h, ops["out_aux_h"])
    mod.updateAuxiliaryElectric1D(Electric=e, Magnetic=h, ElectricDecay=g(ops["aux_ed"]), ElectricCurl=g(ops["aux_ec"]),
                                  sourceIndex=3, sourceValue=0.25).launchRaw()
    close(e, ops["out_aux_e"])


def test_observer_and_dft_ops(ops, mod):
    fld = g(ops["obs_field"])
    re, im = g(ops["obs_re0"]), g(ops["obs_im0"])
    mod.accumulatePointObservers3D(field=fld, pointI=g(ops["obs_pi"], torch.int32), pointJ=g(ops["obs_pj"], torch.int32),
                                   pointK=g(ops["obs_pk"], torch.int32), realAccum=re, imagAccum=im, weightedCos=0.3,
                                   weightedSin=-0.7).launchRaw()
    close(re, ops["out_points_re"])
    close(im, ops["out_points_im"])
    for axis in range(3):
        re, im = g(ops[f"obs_plane{axis}_re0"]), g(ops[f"obs_plane{axis}_im0"])
        mod.accumulatePlaneObserver3D(field=fld, planeRealAccum=re, planeImagAccum=im, axisCode=axis, planeIndex=1,
                                      weightedCos=0.4, weightedSin=0.2).launchRaw()
        close(re, ops[f"out_plane{axis}_re"])
        close(im, ops[f"out_plane{axis}_im"])
    acc = {k: (torch.zeros((2,) + ops[f"dft_{k.lower()}"].shape, device="cuda"),
               torch.zeros((2,) + ops[f"dft_{k.lower()}"].shape, device="cuda")) for k in ("Ex", "Ey", "Ez")}
    mod.accumulateRunningDftYee3DBatched(
        Ex=g(ops["dft_ex"]), Ey=g(ops["dft_ey"]), Ez=g(ops["dft_ez"]), ExRealAccum=acc["Ex"][0], ExImagAccum=acc["Ex"][1],
        EyRealAccum=acc["Ey"][0], EyImagAccum=acc["Ey"][1], EzRealAccum=acc["Ez"][0], EzImagAccum=acc["Ez"][1],
        weightedCos=g(ops["dft_wc"]), weightedSin=g(ops["dft_ws"])).launchRaw()
    for k in ("Ex", "Ey", "Ez"):
        close(acc[k][0], ops[f"out_dft_{k}_re"])
        close(acc[k][1], ops[f"out_dft_{k}_im"])


def test_backend_rejects_bad_arguments(mod):
    with pytest.raises(AttributeError):
        mod.updateMagneticFieldHwStandard3D
    h = torch.zeros((4, 3, 3), device="cuda", dtype=torch.float64)
    with pytest.raises(ValueError):
        mod.updateMagneticFieldHxStandard3D(Hx=h, Ey=h, Ez=h, HxDecay=h, HxCurl=h, invDy=h, invDz=h).launchRaw()


_BLOCH_E = {"Ex": ("Hy", "Hz", "Y", "Z"), "Ey": ("Hx", "Hz", "X", "Z"), "Ez": ("Hx", "Hy", "X", "Y")}


@pytest.mark.parametrize("comp,zmodes", [("Ex", None), ("Ey", None), ("Ez", None), ("Ex", (5, 2)), ("Ey", (0, 5))])
def test_bloch_electric_ops(ops, mod, comp, zmodes):
    first, second, a, b = _BLOCH_E[comp]
    phase = {ax: tuple(ops["bl_phase"][i]) for i, ax in enumerate("XYZ")}
    inv = {a: ops[f"inv_e_{a}"] for a in "xyz"}
    kw = {f"{comp}Real": g(ops[f"bl_{comp}_re"]), f"{comp}Imag": g(ops[f"bl_{comp}_im"]),
          f"{first}Real": g(ops[f"bl_{first}_re"]), f"{first}Imag": g(ops[f"bl_{first}_im"]),
          f"{second}Real": g(ops[f"bl_{second}_re"]), f"{second}Imag": g(ops[f"bl_{second}_im"]),
          f"{comp}Decay": g(ops[f"bl_{comp}_decay"]), f"{comp}Curl": g(ops[f"bl_{comp}_curl"]),
          f"phaseCos{a}": phase[a][0], f"phaseSin{a}": phase[a][1],
          f"invD{a.lower()}": g(inv[a.lower()]), f"invD{b.lower()}": g(inv[b.lower()])}
    if zmodes is None:
        kw[f"phaseCos{b}"], kw[f"phaseSin{b}"] = phase[b]
        name, key = f"updateElectricField{comp}Bloch3D", f"out_bl_{comp}"
    else:
        kw["zLowBoundaryMode"], kw["zHighBoundaryMode"] = zmodes
        name = "updateElectricFieldExBlochYStandardZ3D" if comp == "Ex" else "updateElectricFieldEyBlochXStandardZ3D"
        key = f"out_blz_{comp}"
    getattr(mod, name)(**kw).launchRaw()
    close(kw[f"{comp}Real"], ops[f"{key}_re"])
    close(kw[f"{comp}Imag"], ops[f"{key}_im"])


@pytest.mark.parametrize("comp", ["Ex", "Ey"])
def test_cpml_z_correction_ops(ops, mod, comp):
    h, off, t_ax, modes, full_t = (("Hy", (1, 0, 0), "Y", (1, 5), 6) if comp == "Ex" else
                                   ("Hx", (0, 1, 0), "X", (5, 4), 7))
    f, psi = g(ops[f"cz_{comp}_field"]), g(ops[f"cz_{comp}_psi"])
    getattr(mod, f"applyElectricField{comp}CpmlZCorrection3D")(
        **{comp: f, h: g(ops[f"cz_{comp}_h"]), f"{comp}Curl": g(ops[f"cz_{comp}_curl"]), f"Psi{comp}Z": psi,
           f"InvKappa{comp}Z": g(ops["cz_ik"]), f"B{comp}Z": g(ops["cz_b"]), f"C{comp}Z": g(ops["cz_c"]),
           "invDz": g(ops["inv_e_z"]), "offsetI": off[0], "offsetJ": off[1], "offsetK": off[2],
           f"{t_ax.lower()}LowBoundaryMode": modes[0], f"{t_ax.lower()}HighBoundaryMode": modes[1],
           f"fullSize{t_ax}": full_t, "fullSizeZ": int(ops["nodes"][2])}).launchRaw()
    close(f, ops[f"out_cz_{comp}"])
    close(psi, ops[f"out_cz_{comp}_psi"])


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_projection_ops(ops, mod, axis):
    f = g(ops["proj_re"])
    mod.projectPeriodicBoundary3D(field=f, axis=axis).launchRaw()
    close(f, ops[f"out_proj_per_{axis}"])
    fr, fi = g(ops["proj_re"]), g(ops["proj_im"])
    mod.projectBlochBoundary3D(fieldReal=fr, fieldImag=fi, axis=axis, phaseCos=0.6, phaseSin=0.8).launchRaw()
    close(fr, ops[f"out_proj_bl_{axis}_re"])
    close(fi, ops[f"out_proj_bl_{axis}_im"])
