"""NativeFDTDModule-compatible per-op surface backed by libfdtd_b200.so.

The reference dispatches every hot-path kernel through
``solver.fdtd_module.<camelCaseName>(**kwargs).launchRaw()``
(witwin/maxwell/fdtd/cuda/backend.py:73-115, name table :3583-).  This module
exposes the same names and keyword arguments for the forward hot-path ops, so a
reference solver can be re-pointed op by op (``solver.fdtd_module =
NativeFDTDModule()``).  Tensors must be float32 (index tensors int32/int64),
contiguous and on one CUDA device; every launch goes on torch's current stream
of that device, as in the reference (launch.h:14-20).  Unknown names raise
AttributeError, invalid arguments raise ValueError, as the reference does.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_AXIS = {"x": 0, "y": 1, "z": 2}
# component -> (a-axis, b-axis, first source, second source)
_H_SPEC = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey")}
_E_SPEC = {"Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}


def _check_tensor(t: torch.Tensor, name: str, dtype=torch.float32) -> None:
    if not isinstance(t, torch.Tensor):
        raise ValueError(f"{name} must be a tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _stream(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _uniform(value, tensor):
    """(pointer, scalar) for an optional uniform coefficient (common.cuh:16-44)."""
    if value is None:
        return _lib.ptr(tensor), 0.0
    return None, float(value)


def _magnetic(comp: str, mode: int):
    A, B, first, second = _H_SPEC[comp]
    U, V = A.upper(), B.upper()

    def run(**kw):
        field = kw[comp]
        for key in (comp, first, second, f"{comp}Decay", f"{comp}Curl"):
            _check_tensor(kw[key], key)
        nx, ny, nz = field.shape
        dec_p, dec_u = _uniform(kw.get("uniformDecay"), kw[f"{comp}Decay"])
        cur_p, cur_u = _uniform(kw.get("uniformCurl"), kw[f"{comp}Curl"])
        psi_a = psi_b = ika = ba = ca = ikb = bb = cb = None
        slab = None
        if mode:
            psi_a, psi_b = kw[f"Psi{comp}{U}"], kw[f"Psi{comp}{V}"]
            ika, ba, ca = kw[f"InvKappa{comp}{U}"], kw[f"By{comp}{U}"], kw[f"Cy{comp}{U}"]
            ikb, bb, cb = kw[f"InvKappa{comp}{V}"], kw[f"By{comp}{V}"], kw[f"Cy{comp}{V}"]
            for t, n in ((psi_a, "psi_a"), (psi_b, "psi_b")):
                _check_tensor(t, n)
        if mode == 2:
            slab = _lib.int_array([
                kw[f"psi{comp}{U}LowLength"], kw[f"psi{comp}{U}HighStart"], kw[f"psi{comp}{U}HighLength"],
                kw[f"psi{comp}{V}LowLength"], kw[f"psi{comp}{V}HighStart"], kw[f"psi{comp}{V}HighLength"],
            ])
        lib = _lib.load()
        _lib.check(lib.fdtd_op_update_magnetic(
            "xyz".index(comp[1]), mode, nx, ny, nz, _lib.ptr(field), _lib.ptr(kw[first]), _lib.ptr(kw[second]),
            dec_p, cur_p, dec_u, cur_u, _lib.ptr(kw[f"invD{A}"]), _lib.ptr(kw[f"invD{B}"]), _lib.ptr(psi_a),
            _lib.ptr(psi_b), _lib.ptr(ika), _lib.ptr(ba), _lib.ptr(ca), _lib.ptr(ikb), _lib.ptr(bb), _lib.ptr(cb),
            slab, _stream(field)), f"update magnetic {comp}")

    return run


def _electric(comp: str, mode: int):
    A, B, first, second = _E_SPEC[comp]
    U, V = A.upper(), B.upper()

    def run(**kw):
        field = kw[comp]
        for key in (comp, first, second, f"{comp}Decay", f"{comp}Curl"):
            _check_tensor(kw[key], key)
        nx, ny, nz = field.shape
        dec_p, dec_u = _uniform(kw.get("uniformDecay"), kw[f"{comp}Decay"])
        cur_p, cur_u = _uniform(kw.get("uniformCurl"), kw[f"{comp}Curl"])
        modes = _lib.int_array([kw[f"{A}LowBoundaryMode"], kw[f"{A}HighBoundaryMode"],
                                kw[f"{B}LowBoundaryMode"], kw[f"{B}HighBoundaryMode"]])
        psi_a = psi_b = ika = ba = ca = ikb = bb = cb = None
        slab = None
        if mode:
            psi_a, psi_b = kw[f"Psi{comp}{U}"], kw[f"Psi{comp}{V}"]
            ika, ba, ca = kw[f"InvKappa{comp}{U}"], kw[f"B{comp}{U}"], kw[f"C{comp}{U}"]
            ikb, bb, cb = kw[f"InvKappa{comp}{V}"], kw[f"B{comp}{V}"], kw[f"C{comp}{V}"]
        if mode == 2:
            slab = _lib.int_array([
                kw[f"psi{comp}{U}LowLength"], kw[f"psi{comp}{U}HighStart"], kw[f"psi{comp}{U}HighLength"],
                kw[f"psi{comp}{V}LowLength"], kw[f"psi{comp}{V}HighStart"], kw[f"psi{comp}{V}HighLength"],
            ])
        lib = _lib.load()
        _lib.check(lib.fdtd_op_update_electric(
            "xyz".index(comp[1]), mode, nx, ny, nz, _lib.ptr(field), _lib.ptr(kw[first]), _lib.ptr(kw[second]),
            dec_p, cur_p, dec_u, cur_u, _lib.ptr(kw[f"invD{A}"]), _lib.ptr(kw[f"invD{B}"]), modes, _lib.ptr(psi_a),
            _lib.ptr(psi_b), _lib.ptr(ika), _lib.ptr(ba), _lib.ptr(ca), _lib.ptr(ikb), _lib.ptr(bb), _lib.ptr(cb),
            slab, _stream(field)), f"update electric {comp}")

    return run


def _debye(*, ElectricField, Polarization, PolarizationCurrent, DebyeDrive, decay, dt):
    _lib.check(_lib.load().fdtd_op_update_debye(ElectricField.numel(), _lib.ptr(ElectricField), _lib.ptr(DebyeDrive),
                                                float(decay), float(dt), _lib.ptr(Polarization),
                                                _lib.ptr(PolarizationCurrent), _stream(ElectricField)), "debye")


def _drude(*, ElectricField, PolarizationCurrent, DrudeDrive, decay):
    _lib.check(_lib.load().fdtd_op_update_drude(ElectricField.numel(), _lib.ptr(ElectricField), _lib.ptr(DrudeDrive),
                                                float(decay), _lib.ptr(PolarizationCurrent), _stream(ElectricField)), "drude")


def _lorentz(*, ElectricField, Polarization, PolarizationCurrent, LorentzDrive, decay, restoring, dt):
    _lib.check(_lib.load().fdtd_op_update_lorentz(ElectricField.numel(), _lib.ptr(ElectricField), _lib.ptr(LorentzDrive),
                                                  float(decay), float(restoring), float(dt), _lib.ptr(Polarization),
                                                  _lib.ptr(PolarizationCurrent), _stream(ElectricField)), "lorentz")


def _apply_polarization(*, ElectricField, PolarizationCurrent, InvPermittivity, dt):
    _lib.check(_lib.load().fdtd_op_apply_polarization(ElectricField.numel(), _lib.ptr(PolarizationCurrent),
                                                      _lib.ptr(InvPermittivity), float(dt), _lib.ptr(ElectricField),
                                                      _stream(ElectricField)), "apply polarization")


def _full(t, like, n=None):
    """A coefficient or spacing argument as a contiguous float32 CUDA tensor: full
    E-shaped (or n-long) from a one-element tensor or a Python float."""
    shape = like.shape if n is None else (n,)
    if not isinstance(t, torch.Tensor):
        return torch.full(shape, float(t), device=like.device, dtype=torch.float32)
    if t.numel() == 1 and t.numel() != int(np.prod(shape)):
        return t.reshape(1).to(device=like.device, dtype=torch.float32).expand(*shape).contiguous()
    _check_tensor(t, "coefficient")
    return t


# (curl component of the first coefficient, of the second) per E component
_ANISO = {"Ex": ("Y", "Z"), "Ey": ("X", "Z"), "Ez": ("X", "Y")}


def _full_aniso(comp: str):
    """updateElectricField{Ex,Ey,Ez}FullAniso3D (witwin/maxwell/fdtd/cuda/backend.py,
    update_electric_e*_full_aniso; kernels/aniso.cu:26-580)."""
    c = "xyz".index(comp[1].lower())
    first, second = _ANISO[comp]

    def run(*, Hx, Hy, Hz, invDx, invDy, invDz, periodicX=0, periodicY=0, periodicZ=0, **kw):
        e = kw[comp]
        ca, cb = kw[f"Coeff{first}"], kw[f"Coeff{second}"]
        for name, t in ((comp, e), ("Hx", Hx), ("Hy", Hy), ("Hz", Hz), (f"Coeff{first}", ca), (f"Coeff{second}", cb)):
            _check_tensor(t, name)
        nodes = [Hx.shape[0], Hy.shape[1], Hz.shape[2]]
        inv = [_full(t, e, n) for t, n in zip((invDx, invDy, invDz), nodes)]
        _lib.check(_lib.load().fdtd_op_update_electric_full_aniso(
            c, *nodes, _lib.ptr(e), _lib.ptr(Hx), _lib.ptr(Hy), _lib.ptr(Hz), _lib.ptr(ca), _lib.ptr(cb),
            *(_lib.ptr(t) for t in inv), int(periodicX), int(periodicY), int(periodicZ), _stream(e)), "full aniso")

    return run


def _nl_shapes(ex, ey, ez):
    return (ctypes.c_int * 9)(*ex.shape, *ey.shape, *ez.shape)


def _kerr_curl(comp: str):
    """updateKerrElectricField{Ex,Ey,Ez}Curl3D (witwin/maxwell/fdtd/cuda/backend.py:2232-2275)."""
    c = "xyz".index(comp[1].lower())

    def run(*, DynamicCurl, Ex, Ey, Ez, LinearPermittivity, KerrChi3, dt, eps0, **kw):
        decay = kw[f"{comp}Decay"]
        for name, t in (("DynamicCurl", DynamicCurl), ("Ex", Ex), ("Ey", Ey), ("Ez", Ez),
                        ("LinearPermittivity", LinearPermittivity), (f"{comp}Decay", decay), ("KerrChi3", KerrChi3)):
            _check_tensor(t, name)
        _lib.check(_lib.load().fdtd_op_update_kerr_curl(
            c, _nl_shapes(Ex, Ey, Ez), _lib.ptr(Ex), _lib.ptr(Ey), _lib.ptr(Ez), _lib.ptr(LinearPermittivity),
            _lib.ptr(decay), _lib.ptr(KerrChi3), float(dt), float(eps0), _lib.ptr(DynamicCurl),
            _stream(DynamicCurl)), "kerr curl")

    return run


def _nonlinear_coefficients(*, DynamicDecay, DynamicCurl, Ex, Ey, Ez, LinearPermittivity, ExternalDecay, SigmaStatic,
                            Chi2, Chi3, TpaSigma, component, dt, eps0):
    """updateNonlinearElectricCoefficients3D (witwin/maxwell/fdtd/cuda/backend.py:2277-2309)."""
    if component not in ("Ex", "Ey", "Ez"):
        raise ValueError(f"unsupported nonlinear component {component!r}")
    tensors = (("DynamicDecay", DynamicDecay), ("DynamicCurl", DynamicCurl), ("Ex", Ex), ("Ey", Ey), ("Ez", Ez),
               ("LinearPermittivity", LinearPermittivity), ("ExternalDecay", ExternalDecay),
               ("SigmaStatic", SigmaStatic), ("Chi2", Chi2), ("Chi3", Chi3), ("TpaSigma", TpaSigma))
    for name, t in tensors:
        _check_tensor(t, name)
    _lib.check(_lib.load().fdtd_op_update_nonlinear_coefficients(
        "xyz".index(component[1].lower()), _nl_shapes(Ex, Ey, Ez), _lib.ptr(Ex), _lib.ptr(Ey), _lib.ptr(Ez),
        _lib.ptr(LinearPermittivity), _lib.ptr(ExternalDecay), _lib.ptr(SigmaStatic), _lib.ptr(Chi2), _lib.ptr(Chi3),
        _lib.ptr(TpaSigma), float(dt), float(eps0), _lib.ptr(DynamicDecay), _lib.ptr(DynamicCurl),
        _stream(DynamicCurl)), "nonlinear coefficients")


# (component, first H, second H, axis a, axis b) of the Bloch E kernels
_BLOCH_E = {"Ex": ("Hy", "Hz", "Y", "Z"), "Ey": ("Hx", "Hz", "X", "Z"), "Ez": ("Hx", "Hy", "X", "Y")}


def _electric_bloch(comp: str, z_standard: bool):
    first, second, a, b = _BLOCH_E[comp]

    def run(**kw):
        er, ei = kw[f"{comp}Real"], kw[f"{comp}Imag"]
        for key in (f"{comp}Real", f"{comp}Imag", f"{first}Real", f"{first}Imag", f"{second}Real", f"{second}Imag"):
            _check_tensor(kw[key], key)
        nx, ny, nz = er.shape
        sizes = {"X": nx, "Y": ny, "Z": nz}
        decay = _full(kw[f"{comp}Decay"], er)
        curl = _full(kw[f"{comp}Curl"], er)
        inv_a = _full(kw[f"invD{a.lower()}"], er, sizes[a])
        inv_b = _full(kw[f"invD{b.lower()}"], er, sizes[b])
        pcb = float(kw.get(f"phaseCos{b}", 1.0))
        psb = float(kw.get(f"phaseSin{b}", 0.0))
        _lib.check(_lib.load().fdtd_op_update_electric_bloch(
            "xyz".index(comp[1].lower()), 1 if z_standard else 0, nx, ny, nz, _lib.ptr(er), _lib.ptr(ei),
            _lib.ptr(kw[f"{first}Real"]), _lib.ptr(kw[f"{first}Imag"]), _lib.ptr(kw[f"{second}Real"]),
            _lib.ptr(kw[f"{second}Imag"]), _lib.ptr(decay), _lib.ptr(curl), float(kw[f"phaseCos{a}"]),
            float(kw[f"phaseSin{a}"]), pcb, psb, _lib.ptr(inv_a), _lib.ptr(inv_b),
            int(kw.get("zLowBoundaryMode", 0)), int(kw.get("zHighBoundaryMode", 0)), _stream(er)),
            f"update electric {comp} Bloch")

    return run


def _cpml_z_correction(comp: str):
    h, t = ("Hy", "Y") if comp == "Ex" else ("Hx", "X")

    def run(**kw):
        field = kw[comp]
        for key in (comp, h, f"{comp}Curl", f"Psi{comp}Z", f"InvKappa{comp}Z", f"B{comp}Z", f"C{comp}Z"):
            _check_tensor(kw[key], key)
        inv_dz = _full(kw["invDz"], field, int(kw["fullSizeZ"]))
        _lib.check(_lib.load().fdtd_op_apply_cpml_z_correction(
            0 if comp == "Ex" else 1, _lib.ptr(field), _lib.int_array(field.shape), _lib.ptr(kw[h]),
            _lib.int_array(kw[h].shape), _lib.ptr(kw[f"{comp}Curl"]), _lib.ptr(kw[f"Psi{comp}Z"]),
            _lib.ptr(kw[f"InvKappa{comp}Z"]), _lib.ptr(kw[f"B{comp}Z"]), _lib.ptr(kw[f"C{comp}Z"]), _lib.ptr(inv_dz),
            _lib.int_array([kw["offsetI"], kw["offsetJ"], kw["offsetK"]]), int(kw[f"{t.lower()}LowBoundaryMode"]),
            int(kw[f"{t.lower()}HighBoundaryMode"]), int(kw[f"fullSize{t}"]), int(kw["fullSizeZ"]), _stream(field)),
            f"{comp} CPML z correction")

    return run


def _project_periodic(*, field, axis):
    _check_tensor(field, "field")
    _lib.check(_lib.load().fdtd_op_project_periodic(_lib.ptr(field), _lib.int_array(field.shape), int(axis),
                                                   _stream(field)), "periodic projection")


def _project_bloch(*, fieldReal, fieldImag, axis, phaseCos, phaseSin):
    _check_tensor(fieldReal, "fieldReal")
    _check_tensor(fieldImag, "fieldImag")
    _lib.check(_lib.load().fdtd_op_project_bloch(_lib.ptr(fieldReal), _lib.ptr(fieldImag),
                                                _lib.int_array(fieldReal.shape), int(axis), float(phaseCos),
                                                float(phaseSin), _stream(fieldReal)), "Bloch projection")


def _add_source_patch(*, field, sourcePatch, offsetI, offsetJ, offsetK, signal):
    _check_tensor(field, "field")
    _check_tensor(sourcePatch, "sourcePatch")
    _lib.check(_lib.load().fdtd_op_add_source_patch(
        _lib.ptr(field), _lib.int_array(field.shape), _lib.ptr(sourcePatch), _lib.int_array(sourcePatch.shape),
        _lib.int_array([offsetI, offsetJ, offsetK]), float(signal), _stream(field)), "add source patch")


def _add_cw_patch(*, field, sourcePatchCos, sourcePatchSin, offsetI, offsetJ, offsetK, signalCos, signalSin):
    _check_tensor(field, "field")
    _check_tensor(sourcePatchCos, "sourcePatchCos")
    _check_tensor(sourcePatchSin, "sourcePatchSin")
    _lib.check(_lib.load().fdtd_op_add_cw_patch(
        _lib.ptr(field), _lib.int_array(field.shape), _lib.ptr(sourcePatchCos), _lib.ptr(sourcePatchSin),
        _lib.int_array(sourcePatchCos.shape), _lib.int_array([offsetI, offsetJ, offsetK]), float(signalCos),
        float(signalSin), _stream(field)), "add CW-phased patch")


def _add_shifted_patch(*, field, sourcePatch, delayPatch, activationDelayPatch, offsetI, offsetJ, offsetK, timeKind,
                       time, frequency, fwidth, amplitude, phase, delay, causalGate):
    _check_tensor(field, "field")
    _check_tensor(sourcePatch, "sourcePatch")
    _check_tensor(delayPatch, "delayPatch")
    if int(timeKind) not in (0, 1, 2):
        raise ValueError("timeKind must be 0 (CW), 1 (Gaussian pulse) or 2 (Ricker)")
    gate = int(causalGate) != 0
    if gate:
        _check_tensor(activationDelayPatch, "activationDelayPatch")
    _lib.check(_lib.load().fdtd_op_add_shifted_patch(
        _lib.ptr(field), _lib.int_array(field.shape), _lib.ptr(sourcePatch), _lib.ptr(delayPatch),
        _lib.ptr(activationDelayPatch) if gate else None, 1 if gate else 0, _lib.int_array(sourcePatch.shape),
        _lib.int_array([offsetI, offsetJ, offsetK]), int(timeKind), float(time), float(frequency), float(fwidth),
        float(amplitude), float(phase), float(delay), _stream(field)), "add time-shifted patch")


def _add_line_patch(*, field, coeffPatch, incidentField, sampleIndices, sampleAxisCode, offsetI, offsetJ, offsetK, scale):
    _check_tensor(field, "field")
    idx = sampleIndices.to(dtype=torch.int64).contiguous()
    _lib.check(_lib.load().fdtd_op_add_line_patch(
        _lib.ptr(field), _lib.int_array(field.shape), _lib.ptr(coeffPatch), _lib.int_array(coeffPatch.shape),
        _lib.int_array([offsetI, offsetJ, offsetK]), _lib.ptr(incidentField), _lib.ptr(idx), int(sampleAxisCode),
        float(scale), _stream(field)), "add line patch")


def _aux_magnetic(*, Magnetic, Electric, MagneticDecay, MagneticCurl):
    _lib.check(_lib.load().fdtd_op_aux_magnetic(Electric.numel(), _lib.ptr(Magnetic), _lib.ptr(Electric),
                                                _lib.ptr(MagneticDecay), _lib.ptr(MagneticCurl), _stream(Magnetic)), "aux H")


def _aux_electric(*, Electric, Magnetic, ElectricDecay, ElectricCurl, sourceIndex, sourceValue):
    _lib.check(_lib.load().fdtd_op_aux_electric(Electric.numel(), _lib.ptr(Electric), _lib.ptr(Magnetic),
                                                _lib.ptr(ElectricDecay), _lib.ptr(ElectricCurl), int(sourceIndex),
                                                float(sourceValue), _stream(Electric)), "aux E")


def _point_observers(*, field, pointI, pointJ, pointK, realAccum, imagAccum, weightedCos, weightedSin):
    pi, pj, pk = (t.to(dtype=torch.int32).contiguous() for t in (pointI, pointJ, pointK))
    _lib.check(_lib.load().fdtd_op_point_observers(
        _lib.ptr(field), _lib.int_array(field.shape), int(pi.numel()), _lib.ptr(pi), _lib.ptr(pj), _lib.ptr(pk),
        _lib.ptr(realAccum), _lib.ptr(imagAccum), float(weightedCos), float(weightedSin), _stream(field)), "point observers")


def _plane_observer(*, field, planeRealAccum, planeImagAccum, axisCode, planeIndex, weightedCos, weightedSin):
    _lib.check(_lib.load().fdtd_op_plane_observer(
        _lib.ptr(field), _lib.int_array(field.shape), int(axisCode), int(planeIndex), _lib.ptr(planeRealAccum),
        _lib.ptr(planeImagAccum), float(weightedCos), float(weightedSin), _stream(field)), "plane observer")


def _dft_batched(*, Ex, Ey, Ez, ExRealAccum, ExImagAccum, EyRealAccum, EyImagAccum, EzRealAccum, EzImagAccum,
                 weightedCos, weightedSin):
    lib = _lib.load()
    nf = int(weightedCos.numel())
    for f, re, im in ((Ex, ExRealAccum, ExImagAccum), (Ey, EyRealAccum, EyImagAccum), (Ez, EzRealAccum, EzImagAccum)):
        _lib.check(lib.fdtd_op_dft_volume(f.numel(), nf, _lib.ptr(f), _lib.ptr(re), _lib.ptr(im), _lib.ptr(weightedCos),
                                          _lib.ptr(weightedSin), _stream(f)), "running DFT")


def _clamp_face(*, field, axis, side):
    _lib.check(_lib.load().fdtd_op_clamp_face(_lib.ptr(field), _lib.int_array(field.shape), int(axis), int(side),
                                              _stream(field)), "clamp face")


_KERNELS = {}
for _c in ("Hx", "Hy", "Hz"):
    _KERNELS[f"updateMagneticField{_c}Standard3D"] = _magnetic(_c, 0)
    _KERNELS[f"updateMagneticField{_c}3D"] = _magnetic(_c, 1)
    _KERNELS[f"updateMagneticField{_c}CpmlCompressed3D"] = _magnetic(_c, 2)
for _c in ("Ex", "Ey", "Ez"):
    _KERNELS[f"updateElectricField{_c}Standard3D"] = _electric(_c, 0)
    _KERNELS[f"updateElectricField{_c}Cpml3D"] = _electric(_c, 1)
    _KERNELS[f"updateElectricField{_c}CpmlCompressed3D"] = _electric(_c, 2)
for _c in ("Ex", "Ey", "Ez"):
    _KERNELS[f"updateElectricField{_c}Bloch3D"] = _electric_bloch(_c, False)
_KERNELS["updateElectricFieldExBlochYStandardZ3D"] = _electric_bloch("Ex", True)
_KERNELS["updateElectricFieldEyBlochXStandardZ3D"] = _electric_bloch("Ey", True)
_KERNELS.update({
    "applyElectricFieldExCpmlZCorrection3D": _cpml_z_correction("Ex"),
    "applyElectricFieldEyCpmlZCorrection3D": _cpml_z_correction("Ey"),
    "projectPeriodicBoundary3D": _project_periodic,
    "projectBlochBoundary3D": _project_bloch,
    "updateDebyeCurrent3D": _debye,
    "updateDrudeCurrent3D": _drude,
    "updateLorentzCurrent3D": _lorentz,
    "applyPolarizationCurrent3D": _apply_polarization,
    "updateElectricFieldExFullAniso3D": _full_aniso("Ex"),
    "updateElectricFieldEyFullAniso3D": _full_aniso("Ey"),
    "updateElectricFieldEzFullAniso3D": _full_aniso("Ez"),
    "updateKerrElectricFieldExCurl3D": _kerr_curl("Ex"),
    "updateKerrElectricFieldEyCurl3D": _kerr_curl("Ey"),
    "updateKerrElectricFieldEzCurl3D": _kerr_curl("Ez"),
    "updateNonlinearElectricCoefficients3D": _nonlinear_coefficients,
    "addSourcePatch3D": _add_source_patch,
    "addCwPhasedSourcePatch3D": _add_cw_patch,
    "addTimeShiftedSourcePatch3D": _add_shifted_patch,
    "addScaledLineSourcePatch3D": _add_line_patch,
    "updateAuxiliaryMagnetic1D": _aux_magnetic,
    "updateAuxiliaryElectric1D": _aux_electric,
    "accumulatePointObservers3D": _point_observers,
    "accumulatePlaneObserver3D": _plane_observer,
    "accumulateRunningDftYee3DBatched": _dft_batched,
    "clampFieldFace3D": _clamp_face,
})


class _Launch:
    __slots__ = ("kernel", "kwargs")

    def __init__(self, kernel, kwargs):
        self.kernel = kernel
        self.kwargs = kwargs

    def launchRaw(self):  # noqa: N802 - the reference's kernel-module API
        # Strided views are made contiguous and written back, as the reference
        # does for its in-place kernels (backend.py:54-70).
        write_back = []
        kwargs = dict(self.kwargs)
        for key, value in kwargs.items():
            if isinstance(value, torch.Tensor) and not value.is_contiguous():
                contiguous = value.contiguous()
                kwargs[key] = contiguous
                write_back.append((value, contiguous))
        self.kernel(**kwargs)
        for original, contiguous in write_back:
            original.copy_(contiguous)


class NativeFDTDModule:
    """``fdtd_module`` drop-in: ``module.<name>(**kwargs).launchRaw()``."""

    def __getattr__(self, name: str):
        kernel = _KERNELS.get(name)
        if kernel is None:
            raise AttributeError(f"B200 FDTD backend does not implement kernel {name!r}.")

        def bind(**kwargs):
            return _Launch(kernel, kwargs)

        bind.__name__ = name
        object.__setattr__(self, name, bind)
        return bind


def get_native_fdtd_module() -> NativeFDTDModule:
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 FDTD backend requires a CUDA device")
    _lib.load()
    return NativeFDTDModule()
