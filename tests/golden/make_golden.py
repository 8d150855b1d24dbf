"""Generate the golden vectors that pin the CPU oracle to the reference.

Run from the repository root in a container where the reference checkout is
available (it is not needed anywhere else):

    python tests/golden/make_golden.py [--reference CHECKOUT]

(the checkout defaults to WITWIN_MAXWELL_REFERENCE or the build container's
copy, as oracle/build_ref.py resolves it)

It imports the reference's frozen Torch implementation of the FDTD kernels
(tests/fdtd/cuda/torch_reference.py, "a snapshot of the pre-CUDA-only backend
Torch code path") with a minimal stand-in for its one package import
(witwin.maxwell.fdtd.boundary.common, loaded from the reference file itself),
and records, in float64:

  ops.npz    seeded inputs and outputs of every hot-path op the oracle restates
             (H/E updates in all boundary/CPML modes, ADE, source and TFSF line
             patches, the 1-D incident line, observers, batched volume DFT);
  steps.npz  a 60-step run of a small scene (CPML, dielectric box, Lorentz and
             Drude poles, point dipole, TFSF plane wave, plane/point monitors)
             driven through the reference ops in the order of
             witwin/maxwell/fdtd/runtime/stepping.py:1740-1815, 2289-2345,
             with the observer DFT of witwin/maxwell/fdtd/observers.py:577-659.
"""
from __future__ import annotations

import argparse
import importlib.util
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REFERENCE: Path | None = None  # the reference checkout (set by main)


def load_reference(ref_root: Path):
    for name in ("witwin", "witwin.maxwell", "witwin.maxwell.fdtd", "witwin.maxwell.fdtd.boundary"):
        mod = types.ModuleType(name)
        mod.__path__ = []
        sys.modules[name] = mod
    common_path = ref_root / "witwin/maxwell/fdtd/boundary/common.py"
    spec = importlib.util.spec_from_file_location("witwin.maxwell.fdtd.boundary.common", common_path)
    common = importlib.util.module_from_spec(spec)
    sys.modules["witwin.maxwell.fdtd.boundary.common"] = common
    spec.loader.exec_module(common)
    tr_path = ref_root / "tests/fdtd/cuda/torch_reference.py"
    spec = importlib.util.spec_from_file_location("torch_reference", tr_path)
    tr = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tr)
    tr._require_cuda_tensors = lambda *a, **k: None  # CPU tensors are fine for the Torch reference
    return tr


def t(a):
    return torch.as_tensor(np.array(a, dtype=np.float64))


def shapes(nodes):
    nx, ny, nz = nodes
    return {
        "Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
        "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz),
    }


def op_vectors(tr, rng) -> dict:
    K = tr._KERNELS
    out = {}
    nodes = (7, 6, 5)
    S = shapes(nodes)
    F = {n: rng.standard_normal(s) for n, s in S.items()}
    inv = {a: rng.uniform(0.5, 2.0, n) for a, n in zip("xyz", nodes)}
    invh = {a: rng.uniform(0.5, 2.0, n - 1) for a, n in zip("xyz", nodes)}
    out["nodes"] = np.array(nodes)
    for n, v in F.items():
        out[f"in_{n}"] = v
    for a in "xyz":
        out[f"inv_e_{a}"] = inv[a]
        out[f"inv_h_{a}"] = invh[a]
    # CPML profiles on each axis
    prof = {}
    for a, n in zip("xyz", nodes):
        for kind, length in (("e", n), ("h", n - 1)):
            for q in ("b", "c", "ik"):
                arr = rng.uniform(0.1, 0.9, length)
                prof[(q, kind, a)] = arr
                out[f"cp_{q}_{kind}_{a}"] = arr
    L = 2
    spec_h = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey")}
    for n, (A, B, first, second) in spec_h.items():
        shape = S[n]
        decay = rng.uniform(0.9, 1.0, shape)
        curl = rng.uniform(0.1, 0.5, shape)
        out[f"h_{n}_decay"] = decay
        out[f"h_{n}_curl"] = curl
        # standard
        H = t(F[n])
        kw = {n: H, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
              f"invD{A}": t(invh[A]), f"invD{B}": t(invh[B])}
        K[f"updateMagneticField{n}Standard3D"](**kw)
        out[f"out_h_std_{n}"] = H.numpy()
        # dense CPML
        H = t(F[n])
        psiA = rng.standard_normal(shape) * 0.1
        psiB = rng.standard_normal(shape) * 0.1
        out[f"h_{n}_psiA"] = psiA
        out[f"h_{n}_psiB"] = psiB
        pa, pb = t(psiA), t(psiB)
        U, V = A.upper(), B.upper()
        kw = {n: H, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
              f"Psi{n}{U}": pa, f"Psi{n}{V}": pb,
              f"InvKappa{n}{U}": t(prof[("ik", "h", A)]), f"By{n}{U}": t(prof[("b", "h", A)]), f"Cy{n}{U}": t(prof[("c", "h", A)]),
              f"InvKappa{n}{V}": t(prof[("ik", "h", B)]), f"By{n}{V}": t(prof[("b", "h", B)]), f"Cy{n}{V}": t(prof[("c", "h", B)]),
              f"invD{A}": t(invh[A]), f"invD{B}": t(invh[B])}
        K[f"updateMagneticField{n}3D"](**kw)
        out[f"out_h_dense_{n}"] = H.numpy()
        out[f"out_h_dense_{n}_psiA"] = pa.numpy()
        out[f"out_h_dense_{n}_psiB"] = pb.numpy()
        # compressed CPML (L low + L high on both axes)
        H = t(F[n])
        ax = {"x": 0, "y": 1, "z": 2}
        cps = []
        for which, axname in ((0, A), (1, B)):
            size = shape[ax[axname]]
            cshape = list(shape)
            cshape[ax[axname]] = 2 * L
            c = rng.standard_normal(cshape) * 0.1
            out[f"h_{n}_cpsi{which}"] = c
            cps.append((t(c), L, size - L, L))
        kw = {n: H, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
              f"Psi{n}{U}": cps[0][0], f"Psi{n}{V}": cps[1][0],
              f"InvKappa{n}{U}": t(prof[("ik", "h", A)]), f"By{n}{U}": t(prof[("b", "h", A)]), f"Cy{n}{U}": t(prof[("c", "h", A)]),
              f"InvKappa{n}{V}": t(prof[("ik", "h", B)]), f"By{n}{V}": t(prof[("b", "h", B)]), f"Cy{n}{V}": t(prof[("c", "h", B)]),
              f"invD{A}": t(invh[A]), f"invD{B}": t(invh[B]),
              f"psi{n}{U}LowLength": cps[0][1], f"psi{n}{U}HighStart": cps[0][2], f"psi{n}{U}HighLength": cps[0][3],
              f"psi{n}{V}LowLength": cps[1][1], f"psi{n}{V}HighStart": cps[1][2], f"psi{n}{V}HighLength": cps[1][3],
              "uniformDecay": None, "uniformCurl": None}
        K[f"updateMagneticField{n}CpmlCompressed3D"](**kw)
        out[f"out_h_comp_{n}"] = H.numpy()
        out[f"out_h_comp_{n}_psi0"] = cps[0][0].numpy()
        out[f"out_h_comp_{n}_psi1"] = cps[1][0].numpy()
    # E updates
    spec_e = {"Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}
    mode_sets = {
        "pml": (1, 1, 1, 1),
        "pec": (4, 4, 4, 4),
        "mixed": (2, 2, 5, 4),   # periodic on a, PMC low / PEC high on b
        "pmc": (5, 5, 0, 1),
    }
    for n, (A, B, first, second) in spec_e.items():
        shape = S[n]
        decay = rng.uniform(0.9, 1.0, shape)
        curl = rng.uniform(0.1, 0.5, shape)
        out[f"e_{n}_decay"] = decay
        out[f"e_{n}_curl"] = curl
        U, V = A.upper(), B.upper()
        ax = {"x": 0, "y": 1, "z": 2}
        for mname, modes in mode_sets.items():
            out[f"e_modes_{mname}"] = np.array(modes)
            names = {f"{A}LowBoundaryMode": modes[0], f"{A}HighBoundaryMode": modes[1],
                     f"{B}LowBoundaryMode": modes[2], f"{B}HighBoundaryMode": modes[3]}
            E = t(F[n])
            kw = {n: E, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
                  f"invD{A}": t(inv[A]), f"invD{B}": t(inv[B]), **names}
            K[f"updateElectricField{n}Standard3D"](**kw)
            out[f"out_e_std_{n}_{mname}"] = E.numpy()
            # dense CPML
            E = t(F[n])
            psiA = rng.standard_normal(shape) * 0.1
            psiB = rng.standard_normal(shape) * 0.1
            out[f"e_{n}_{mname}_psiA"] = psiA
            out[f"e_{n}_{mname}_psiB"] = psiB
            pa, pb = t(psiA), t(psiB)
            kw = {n: E, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
                  f"Psi{n}{U}": pa, f"Psi{n}{V}": pb,
                  f"InvKappa{n}{U}": t(prof[("ik", "e", A)]), f"B{n}{U}": t(prof[("b", "e", A)]), f"C{n}{U}": t(prof[("c", "e", A)]),
                  f"InvKappa{n}{V}": t(prof[("ik", "e", B)]), f"B{n}{V}": t(prof[("b", "e", B)]), f"C{n}{V}": t(prof[("c", "e", B)]),
                  f"invD{A}": t(inv[A]), f"invD{B}": t(inv[B]), **names}
            K[f"updateElectricField{n}Cpml3D"](**kw)
            out[f"out_e_dense_{n}_{mname}"] = E.numpy()
            out[f"out_e_dense_{n}_{mname}_psiA"] = pa.numpy()
            out[f"out_e_dense_{n}_{mname}_psiB"] = pb.numpy()
            # compressed CPML
            E = t(F[n])
            cps = []
            for which, axname in ((0, A), (1, B)):
                size = shape[ax[axname]]
                cshape = list(shape)
                cshape[ax[axname]] = 2 * L
                c = rng.standard_normal(cshape) * 0.1
                out[f"e_{n}_{mname}_cpsi{which}"] = c
                cps.append((t(c), L, size - L, L))
            kw = {n: E, first: t(F[first]), second: t(F[second]), f"{n}Decay": t(decay), f"{n}Curl": t(curl),
                  f"Psi{n}{U}": cps[0][0], f"Psi{n}{V}": cps[1][0],
                  f"InvKappa{n}{U}": t(prof[("ik", "e", A)]), f"B{n}{U}": t(prof[("b", "e", A)]), f"C{n}{U}": t(prof[("c", "e", A)]),
                  f"InvKappa{n}{V}": t(prof[("ik", "e", B)]), f"B{n}{V}": t(prof[("b", "e", B)]), f"C{n}{V}": t(prof[("c", "e", B)]),
                  f"invD{A}": t(inv[A]), f"invD{B}": t(inv[B]), **names,
                  f"psi{n}{U}LowLength": cps[0][1], f"psi{n}{U}HighStart": cps[0][2], f"psi{n}{U}HighLength": cps[0][3],
                  f"psi{n}{V}LowLength": cps[1][1], f"psi{n}{V}HighStart": cps[1][2], f"psi{n}{V}HighLength": cps[1][3],
                  "uniformDecay": None, "uniformCurl": None}
            K[f"updateElectricField{n}CpmlCompressed3D"](**kw)
            out[f"out_e_comp_{n}_{mname}"] = E.numpy()
            out[f"out_e_comp_{n}_{mname}_psi0"] = cps[0][0].numpy()
            out[f"out_e_comp_{n}_{mname}_psi1"] = cps[1][0].numpy()
    # ADE
    e = rng.standard_normal(40)
    drive = rng.uniform(0.0, 1.0, 40)
    p0 = rng.standard_normal(40)
    j0 = rng.standard_normal(40)
    inv_eps = rng.uniform(0.2, 1.0, 40)
    out.update(ade_e=e, ade_drive=drive, ade_p0=p0, ade_j0=j0, ade_inv_eps=inv_eps)
    P, J = t(p0), t(j0)
    K["updateDebyeCurrent3D"](ElectricField=t(e), Polarization=P, PolarizationCurrent=J, DebyeDrive=t(drive), decay=0.7, dt=0.3)
    out["out_debye_p"], out["out_debye_j"] = P.numpy(), J.numpy()
    J = t(j0)
    K["updateDrudeCurrent3D"](ElectricField=t(e), PolarizationCurrent=J, DrudeDrive=t(drive), decay=0.8)
    out["out_drude_j"] = J.numpy()
    P, J = t(p0), t(j0)
    K["updateLorentzCurrent3D"](ElectricField=t(e), Polarization=P, PolarizationCurrent=J, LorentzDrive=t(drive), decay=0.9,
                                restoring=0.05, dt=0.3)
    out["out_lorentz_p"], out["out_lorentz_j"] = P.numpy(), J.numpy()
    E = t(e)
    K["applyPolarizationCurrent3D"](ElectricField=E, PolarizationCurrent=t(j0), InvPermittivity=t(inv_eps), dt=0.3)
    out["out_apply_e"] = E.numpy()
    # source patch partially outside the field
    fld = rng.standard_normal((5, 4, 6))
    patch = rng.standard_normal((3, 3, 3))
    out.update(patch_field=fld, patch=patch)
    f = t(fld)
    K["addSourcePatch3D"](field=f, sourcePatch=t(patch), offsetI=3, offsetJ=-1, offsetK=2, signal=0.75)
    out["out_patch"] = f.numpy()
    # TFSF line patch (sample axis 0)
    coeff = rng.standard_normal((3, 2, 4))
    inc = rng.standard_normal(12)
    idx = np.array([2, 5, 7], dtype=np.int64)
    out.update(line_coeff=coeff, line_inc=inc, line_idx=idx)
    f = t(fld)
    K["addScaledLineSourcePatch3D"](field=f, coeffPatch=t(coeff), incidentField=t(inc), sampleIndices=torch.as_tensor(idx),
                                    sampleAxisCode=0, offsetI=1, offsetJ=1, offsetK=1, scale=-0.6)
    out["out_line"] = f.numpy()
    # 1-D incident line
    ae = rng.standard_normal(10)
    ah = rng.standard_normal(9)
    aed, aec = rng.uniform(0.9, 1, 10), rng.uniform(0.1, 0.5, 10)
    ahd, ahc = rng.uniform(0.9, 1, 9), rng.uniform(0.1, 0.5, 9)
    out.update(aux_e=ae, aux_h=ah, aux_ed=aed, aux_ec=aec, aux_hd=ahd, aux_hc=ahc)
    H = t(ah)
    K["updateAuxiliaryMagnetic1D"](Magnetic=H, Electric=t(ae), MagneticDecay=t(ahd), MagneticCurl=t(ahc))
    out["out_aux_h"] = H.numpy()
    E = t(ae)
    K["updateAuxiliaryElectric1D"](Electric=E, Magnetic=H, ElectricDecay=t(aed), ElectricCurl=t(aec), sourceIndex=3,
                                   sourceValue=0.25)
    out["out_aux_e"] = E.numpy()
    # observers
    fld = rng.standard_normal((5, 4, 6))
    re0, im0 = rng.standard_normal(3), rng.standard_normal(3)
    pi, pj, pk = np.array([0, 2, 4]), np.array([1, 3, 0]), np.array([5, 2, 1])
    out.update(obs_field=fld, obs_re0=re0, obs_im0=im0, obs_pi=pi, obs_pj=pj, obs_pk=pk)
    re, im = t(re0), t(im0)
    K["accumulatePointObservers3D"](field=t(fld), pointI=torch.as_tensor(pi), pointJ=torch.as_tensor(pj),
                                    pointK=torch.as_tensor(pk), realAccum=re, imagAccum=im, weightedCos=0.3, weightedSin=-0.7)
    out["out_points_re"], out["out_points_im"] = re.numpy(), im.numpy()
    for axis in range(3):
        pshape = [s for a, s in enumerate(fld.shape) if a != axis]
        r0 = rng.standard_normal(pshape)
        i0 = rng.standard_normal(pshape)
        out[f"obs_plane{axis}_re0"], out[f"obs_plane{axis}_im0"] = r0, i0
        re, im = t(r0), t(i0)
        K["accumulatePlaneObserver3D"](field=t(fld), planeRealAccum=re, planeImagAccum=im, axisCode=axis, planeIndex=1,
                                       weightedCos=0.4, weightedSin=0.2)
        out[f"out_plane{axis}_re"], out[f"out_plane{axis}_im"] = re.numpy(), im.numpy()
    # batched volume DFT
    ex, ey, ez = (rng.standard_normal(s) for s in ((3, 4, 5), (4, 3, 5), (4, 4, 4)))
    wc, ws = rng.standard_normal(2), rng.standard_normal(2)
    out.update(dft_ex=ex, dft_ey=ey, dft_ez=ez, dft_wc=wc, dft_ws=ws)
    acc = {k: t(np.zeros((2,) + v.shape)) for k, v in (("Ex", ex), ("Ey", ey), ("Ez", ez))}
    acc_i = {k: t(np.zeros((2,) + v.shape)) for k, v in (("Ex", ex), ("Ey", ey), ("Ez", ez))}
    K["accumulateRunningDftYee3DBatched"](Ex=t(ex), Ey=t(ey), Ez=t(ez), ExRealAccum=acc["Ex"], ExImagAccum=acc_i["Ex"],
                                          EyRealAccum=acc["Ey"], EyImagAccum=acc_i["Ey"], EzRealAccum=acc["Ez"],
                                          EzImagAccum=acc_i["Ez"], weightedCos=t(wc), weightedSin=t(ws))
    for k in ("Ex", "Ey", "Ez"):
        out[f"out_dft_{k}_re"], out[f"out_dft_{k}_im"] = acc[k].numpy(), acc_i[k].numpy()
    # CW-phased and time-shifted patches (sources.cu:156-221), partially outside
    fld, patch = out["patch_field"], out["patch"]
    pc, ps = rng.standard_normal((3, 3, 3)), rng.standard_normal((3, 3, 3))
    out.update(cw_cos=pc, cw_sin=ps)
    f = t(fld)
    K["addCwPhasedSourcePatch3D"](field=f, sourcePatchCos=t(pc), sourcePatchSin=t(ps), offsetI=3, offsetJ=-1,
                                  offsetK=2, signalCos=0.6, signalSin=-0.3)
    out["out_cw_patch"] = f.numpy()
    delay = rng.uniform(0.0, 2e-15, (3, 3, 3))
    act = rng.uniform(0.0, 2e-14, (3, 3, 3))
    out.update(shift_delay=delay, shift_act=act)
    for kind, gate in ((0, 0), (1, 0), (1, 1), (2, 1)):
        f = t(fld)
        K["addTimeShiftedSourcePatch3D"](field=f, sourcePatch=t(patch), delayPatch=t(delay),
                                         activationDelayPatch=t(act), offsetI=3, offsetJ=-1, offsetK=2, timeKind=kind,
                                         time=1.1e-14, frequency=300e12, fwidth=100e12, amplitude=1.3, phase=0.2,
                                         delay=9.5e-15, causalGate=gate)
        out[f"out_shift_{kind}_{gate}"] = f.numpy()
    # complex E updates on Bloch faces (electric.cu:356-453, 1164-1528)
    cplx = {n: (rng.standard_normal(sh), rng.standard_normal(sh)) for n, sh in S.items()}
    for n, (re_, im_) in cplx.items():
        out[f"bl_{n}_re"], out[f"bl_{n}_im"] = re_, im_
    phase = {a: (float(np.cos(0.3 + 0.5 * i)), float(np.sin(0.3 + 0.5 * i))) for i, a in enumerate("XYZ")}
    bl_coef = {n: (rng.uniform(0.5, 1.0, S[n]), rng.uniform(0.1, 0.5, S[n])) for n in ("Ex", "Ey", "Ez")}
    for n, (dcy, crl) in bl_coef.items():
        out[f"bl_{n}_decay"], out[f"bl_{n}_curl"] = dcy, crl
    spec = {"Ex": ("Hy", "Hz", "Y", "Z"), "Ey": ("Hx", "Hz", "X", "Z"), "Ez": ("Hx", "Hy", "X", "Y")}
    variants = [(n, None) for n in ("Ex", "Ey", "Ez")] + [("Ex", (5, 2)), ("Ey", (0, 5))]
    for comp, zmodes in variants:
        first, second, a, b = spec[comp]
        kw = {f"{comp}Real": t(cplx[comp][0]), f"{comp}Imag": t(cplx[comp][1]),
              f"{first}Real": t(cplx[first][0]), f"{first}Imag": t(cplx[first][1]),
              f"{second}Real": t(cplx[second][0]), f"{second}Imag": t(cplx[second][1]),
              f"{comp}Decay": t(bl_coef[comp][0]), f"{comp}Curl": t(bl_coef[comp][1]),
              f"phaseCos{a}": phase[a][0], f"phaseSin{a}": phase[a][1],
              f"invD{a.lower()}": t(inv[a.lower()]), f"invD{b.lower()}": t(inv[b.lower()])}
        if zmodes is None:
            kw[f"phaseCos{b}"], kw[f"phaseSin{b}"] = phase[b]
            name = f"updateElectricField{comp}Bloch3D"
            key = f"out_bl_{comp}"
        else:
            kw["zLowBoundaryMode"], kw["zHighBoundaryMode"] = zmodes
            name = "updateElectricFieldExBlochYStandardZ3D" if comp == "Ex" else "updateElectricFieldEyBlochXStandardZ3D"
            key = f"out_blz_{comp}"
        K[name](**kw)
        out[f"{key}_re"], out[f"{key}_im"] = kw[f"{comp}Real"].numpy(), kw[f"{comp}Imag"].numpy()
    out["bl_phase"] = np.array([phase[a] for a in "XYZ"])
    # z-CPML corrections of Ex / Ey over a region (Bloch-x/y + CPML-z scenes)
    nzf = nodes[2]
    prof = {k: rng.uniform(0.2, 1.0, nzf) for k in ("ik", "b", "c")}
    out.update(cz_ik=prof["ik"], cz_b=prof["b"], cz_c=prof["c"])
    for comp, h, off, region, t_ax, modes in (("Ex", "Hy", (1, 0, 0), (4, 6, 5), "Y", (1, 5)),
                                               ("Ey", "Hx", (0, 1, 0), (7, 3, 5), "X", (5, 4))):
        fld = rng.standard_normal(region)
        crl = rng.uniform(0.1, 0.5, region)
        psi = rng.standard_normal(region)
        hh = rng.standard_normal(S[h])
        out.update({f"cz_{comp}_field": fld, f"cz_{comp}_curl": crl, f"cz_{comp}_psi": psi, f"cz_{comp}_h": hh})
        f, pz = t(fld), t(psi)
        K[f"applyElectricField{comp}CpmlZCorrection3D"](
            **{comp: f, h: t(hh), f"{comp}Curl": t(crl), f"Psi{comp}Z": pz, f"InvKappa{comp}Z": t(prof["ik"]),
               f"B{comp}Z": t(prof["b"]), f"C{comp}Z": t(prof["c"]), "invDz": t(inv["z"]), "offsetI": off[0],
               "offsetJ": off[1], "offsetK": off[2], f"{t_ax.lower()}LowBoundaryMode": modes[0],
               f"{t_ax.lower()}HighBoundaryMode": modes[1], f"fullSize{t_ax}": S[comp][0 if t_ax == "X" else 1],
               "fullSizeZ": nzf})
        out[f"out_cz_{comp}"], out[f"out_cz_{comp}_psi"] = f.numpy(), pz.numpy()
    # periodic and Bloch face projections (projection.cu:43-125)
    pf = rng.standard_normal((5, 4, 6))
    pim = rng.standard_normal((5, 4, 6))
    out.update(proj_re=pf, proj_im=pim)
    for axis in range(3):
        f = t(pf)
        K["projectPeriodicBoundary3D"](field=f, axis=axis)
        out[f"out_proj_per_{axis}"] = f.numpy()
        fr, fi = t(pf), t(pim)
        K["projectBlochBoundary3D"](fieldReal=fr, fieldImag=fi, axis=axis, phaseCos=0.6, phaseSin=0.8)
        out[f"out_proj_bl_{axis}_re"], out[f"out_proj_bl_{axis}_im"] = fr.numpy(), fi.numpy()
    # instantaneous nonlinear coefficients: the Kerr curl ops of torch_reference
    # (updateKerrElectricField{Ex,Ey,Ez}Curl3D) and the general chi2 / chi3 / TPA
    # formula of the reference's own test (tests/materials/nonlinear/
    # test_fdtd_nonlinear.py, _reference_nonlinear_coefficients), on fields large
    # enough that every channel matters; a few cells drive eps_eff below its
    # floor and the TPA conductivity below zero
    nonlinear_vectors(tr, rng, out)
    return out


def _reference_test_functions(names):
    """The named top-level functions of the reference's nonlinear test module,
    executed without the module's package imports."""
    import ast

    path = REFERENCE / "tests/materials/nonlinear/test_fdtd_nonlinear.py"
    tree = ast.parse(path.read_text())
    body = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in names]
    ns = {"torch": torch}
    exec(compile(ast.Module(body=body, type_ignores=[]), str(path), "exec"), ns)
    return [ns[n] for n in names]


def nonlinear_vectors(tr, rng, out):
    nodes = (7, 6, 5)
    S = shapes(nodes)
    eps0, dt = 8.8541878128e-12, 4.8e-17
    fields = {c: rng.standard_normal(S[c]) * 30.0 for c in ("Ex", "Ey", "Ez")}
    out.update(nl_dt=np.array(dt), nl_eps0=np.array(eps0), nl_Ex=fields["Ex"], nl_Ey=fields["Ey"], nl_Ez=fields["Ez"])
    (general,) = _reference_test_functions(["_clamped_gather", "_collocate_reference",
                                            "_reference_nonlinear_coefficients"])[2:]
    solver = types.SimpleNamespace(Ex=t(fields["Ex"]), Ey=t(fields["Ey"]), Ez=t(fields["Ez"]), eps0=eps0, dt=dt)
    for comp in ("Ex", "Ey", "Ez"):
        sh = S[comp]
        eps = eps0 * rng.uniform(1.0, 4.0, sh)
        dec = rng.uniform(0.5, 1.0, sh)
        ext = rng.uniform(0.5, 1.0, sh)
        sig = rng.uniform(0.0, 1.0e6, sh)
        chi2 = rng.uniform(-0.01, 0.01, sh)
        chi3 = rng.uniform(0.0, 2.0e-3, sh)
        tpa = rng.uniform(-2.0e2, 1.0e4, sh)
        chi3.flat[::7] = -1.0  # eps_eff below the floor
        chi2.flat[3::11] = -2.0
        vals = dict(eps=eps, dec=dec, ext=ext, sig=sig, chi2=chi2, chi3=chi3, tpa=tpa)
        for k, v in vals.items():
            out[f"nl_{comp}_{k}"] = v
        dyn = torch.zeros(sh)
        tr.__dict__[f"_update_kerr_{comp.lower()}"](
            DynamicCurl=dyn, Ex=solver.Ex, Ey=solver.Ey, Ez=solver.Ez, LinearPermittivity=t(eps),
            **{f"{comp}Decay": t(dec)}, KerrChi3=t(chi3), dt=dt, eps0=eps0)
        out[f"out_kerr_{comp}"] = dyn.numpy()
        low = comp.lower()
        setattr(solver, f"eps_{comp}", t(eps))
        setattr(solver, f"c{low}_decay_external", t(ext))
        setattr(solver, f"sigma_e_{comp}", t(sig))
        setattr(solver, f"nonlinear_chi2_{comp}", t(chi2))
        setattr(solver, f"kerr_chi3_{comp}", t(chi3))
        setattr(solver, f"tpa_sigma_{comp}", t(tpa))
    for comp in ("Ex", "Ey", "Ez"):
        d, c = general(solver, comp)
        out[f"out_nl_{comp}_decay"], out[f"out_nl_{comp}_curl"] = d.numpy(), c.numpy()


def _package():
    sys.path.insert(0, str(ROOT / "tests"))
    import conftest  # noqa: F401  (registers the package under its import name)

    return conftest.load_package()


def golden_scene():
    """The small scene of steps.npz (node-index geometry, 16 cells, 4-cell CPML)."""
    wm = _package()

    d = 25e-9
    sc = wm.Scene(cells=(16, 14, 12), spacing=d, pml_cells=4)
    sc.structures.append(wm.Structure(wm.Box((6, 5, 5), (10, 9, 8)), wm.Medium(eps_r=3.0)))
    sc.structures.append(wm.Structure(wm.Sphere((9, 7, 6), 2.2), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((4, 0, 0), (6, 14, 12)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.sources.append(wm.PointDipole((11, 7, 6), "Ez", wm.GaussianPulse(300e12, 100e12), width=25e-9))
    sc.sources.append(wm.PlaneWaveTFSF((1, 0, 0), (0, 0, 1), wm.GaussianPulse(300e12, 100e12), (5, 5, 5), (12, 10, 8)))
    freqs = (250e12, 300e12)
    sc.monitors.append(wm.PlaneMonitor("plane", 2, 8, frequencies=freqs))
    sc.monitors.append(wm.PointMonitor("point", (12, 7, 6), frequencies=freqs))
    return sc


GOLDEN_STEPS = 60


def step_vectors(tr) -> dict:
    """Drive the reference ops in stepping order over the golden scene."""
    wm = _package()

    sc = golden_scene()
    cs = wm.compile_scene(sc, GOLDEN_STEPS)
    K = tr._KERNELS
    S = shapes(cs.nodes)
    F = {n: torch.zeros(s, dtype=torch.float64) for n, s in S.items()}
    coef = {}
    for n in S:
        du, cu = cs.uniform[n]
        coef[n] = (
            torch.full(S[n], du, dtype=torch.float64) if cs.decay[n] is None else t(cs.decay[n]),
            torch.full(S[n], cu, dtype=torch.float64) if cs.curl[n] is None else t(cs.curl[n]),
        )
    cp = {k: [t(a) for a in v] for k, v in cs.cpml.items()}
    inv_e = [t(a) for a in cs.inv_e]
    inv_h = [t(a) for a in cs.inv_h]
    ax = {"x": 0, "y": 1, "z": 2}
    psi = {}
    slabs = {}
    specs = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey"),
             "Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}
    for n, (A, B, _, _) in specs.items():
        for which, a in ((0, A), (1, B)):
            size = S[n][ax[a]]
            low = min(cs.pml_lo[ax[a]], size)
            high = min(cs.pml_hi[ax[a]], size - low)
            shp = list(S[n])
            shp[ax[a]] = low + high
            psi[(n, which)] = torch.zeros(shp, dtype=torch.float64)
            slabs[(n, which)] = (low, size - high, high)
    poles = []
    for p in cs.poles:
        b = p.box
        sl = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
        drive = torch.zeros(S[p.component], dtype=torch.float64)
        drive[sl] = t(p.drive)
        inv_eps = t((1.0 / cs.eps[p.component]).astype(np.float32))
        inv_eps[sl] = t(p.inv_eps)
        poles.append(dict(p=p, drive=drive, inv_eps=inv_eps, P=torch.zeros_like(drive), J=torch.zeros_like(drive)))
    aux = cs.aux_line
    aux_e = torch.zeros(aux.e_decay.size, dtype=torch.float64)
    aux_h = torch.zeros(aux.e_decay.size - 1, dtype=torch.float64)
    freqs = np.asarray(cs.frequencies)
    omega = 2 * np.pi * freqs
    pc, ps = np.ones(freqs.size), np.zeros(freqs.size)
    sc_, ss_ = np.cos(omega * cs.dt), np.sin(omega * cs.dt)
    hc_, hs_ = np.cos(-0.5 * omega * cs.dt), np.sin(-0.5 * omega * cs.dt)
    acc = []
    for reg in cs.regions:
        b = reg.box
        shp = (freqs.size, b[1] - b[0], b[3] - b[2], b[5] - b[4])
        acc.append([torch.zeros(shp, dtype=torch.float64), torch.zeros(shp, dtype=torch.float64)])
    window_sum = 0.0

    def line_terms(magnetic):
        sample = aux_e if magnetic else aux_h
        for lp in cs.line_patches:
            if (lp.component[0] == "H") != magnetic:
                continue
            K["addScaledLineSourcePatch3D"](field=F[lp.component], coeffPatch=t(lp.coeff), incidentField=sample,
                                            sampleIndices=torch.as_tensor(lp.sample_index.astype(np.int64)),
                                            sampleAxisCode=lp.sample_axis, offsetI=lp.box[0], offsetJ=lp.box[2],
                                            offsetK=lp.box[4], scale=lp.scale)

    for n in range(GOLDEN_STEPS):
        for h in ("Hx", "Hy", "Hz"):
            A, B, first, second = specs[h]
            U, V = A.upper(), B.upper()
            (s0, s1) = slabs[(h, 0)], slabs[(h, 1)]
            K[f"updateMagneticField{h}CpmlCompressed3D"](**{
                h: F[h], first: F[first], second: F[second], f"{h}Decay": coef[h][0], f"{h}Curl": coef[h][1],
                f"Psi{h}{U}": psi[(h, 0)], f"Psi{h}{V}": psi[(h, 1)],
                f"InvKappa{h}{U}": cp["ik_h"][ax[A]], f"By{h}{U}": cp["b_h"][ax[A]], f"Cy{h}{U}": cp["c_h"][ax[A]],
                f"InvKappa{h}{V}": cp["ik_h"][ax[B]], f"By{h}{V}": cp["b_h"][ax[B]], f"Cy{h}{V}": cp["c_h"][ax[B]],
                f"invD{A}": inv_h[ax[A]], f"invD{B}": inv_h[ax[B]],
                f"psi{h}{U}LowLength": s0[0], f"psi{h}{U}HighStart": s0[1], f"psi{h}{U}HighLength": s0[2],
                f"psi{h}{V}LowLength": s1[0], f"psi{h}{V}HighStart": s1[1], f"psi{h}{V}HighLength": s1[2],
                "uniformDecay": None, "uniformCurl": None})
        line_terms(True)
        K["updateAuxiliaryMagnetic1D"](Magnetic=aux_h, Electric=aux_e, MagneticDecay=t(aux.h_decay), MagneticCurl=t(aux.h_curl))
        for pl in poles:
            p = pl["p"]
            e = F[p.component]
            if p.kind == 0:
                K["updateDebyeCurrent3D"](ElectricField=e, Polarization=pl["P"], PolarizationCurrent=pl["J"],
                                          DebyeDrive=pl["drive"], decay=p.decay, dt=cs.dt)
            elif p.kind == 1:
                K["updateDrudeCurrent3D"](ElectricField=e, PolarizationCurrent=pl["J"], DrudeDrive=pl["drive"], decay=p.decay)
            else:
                K["updateLorentzCurrent3D"](ElectricField=e, Polarization=pl["P"], PolarizationCurrent=pl["J"],
                                            LorentzDrive=pl["drive"], decay=p.decay, restoring=p.restoring, dt=cs.dt)
        bnd = cs.boundary
        for e_name in ("Ex", "Ey", "Ez"):
            A, B, first, second = specs[e_name]
            U, V = A.upper(), B.upper()
            (s0, s1) = slabs[(e_name, 0)], slabs[(e_name, 1)]
            K[f"updateElectricField{e_name}CpmlCompressed3D"](**{
                e_name: F[e_name], first: F[first], second: F[second], f"{e_name}Decay": coef[e_name][0],
                f"{e_name}Curl": coef[e_name][1], f"Psi{e_name}{U}": psi[(e_name, 0)], f"Psi{e_name}{V}": psi[(e_name, 1)],
                f"InvKappa{e_name}{U}": cp["ik_e"][ax[A]], f"B{e_name}{U}": cp["b_e"][ax[A]], f"C{e_name}{U}": cp["c_e"][ax[A]],
                f"InvKappa{e_name}{V}": cp["ik_e"][ax[B]], f"B{e_name}{V}": cp["b_e"][ax[B]], f"C{e_name}{V}": cp["c_e"][ax[B]],
                f"invD{A}": inv_e[ax[A]], f"invD{B}": inv_e[ax[B]],
                f"{A}LowBoundaryMode": bnd[2 * ax[A]], f"{A}HighBoundaryMode": bnd[2 * ax[A] + 1],
                f"{B}LowBoundaryMode": bnd[2 * ax[B]], f"{B}HighBoundaryMode": bnd[2 * ax[B] + 1],
                f"psi{e_name}{U}LowLength": s0[0], f"psi{e_name}{U}HighStart": s0[1], f"psi{e_name}{U}HighLength": s0[2],
                f"psi{e_name}{V}LowLength": s1[0], f"psi{e_name}{V}HighStart": s1[1], f"psi{e_name}{V}HighLength": s1[2],
                "uniformDecay": None, "uniformCurl": None})
        line_terms(False)
        K["updateAuxiliaryElectric1D"](Electric=aux_e, Magnetic=aux_h, ElectricDecay=t(aux.e_decay), ElectricCurl=t(aux.e_curl),
                                       sourceIndex=aux.source_index, sourceValue=float(aux.source[n]))
        for patch in cs.patches:
            K["addSourcePatch3D"](field=F[patch.component], sourcePatch=t(patch.coeff), offsetI=patch.box[0],
                                  offsetJ=patch.box[2], offsetK=patch.box[4], signal=float(patch.signal[n]))
        for pl in poles:
            K["applyPolarizationCurrent3D"](ElectricField=F[pl["p"].component], PolarizationCurrent=pl["J"],
                                            InvPermittivity=pl["inv_eps"], dt=cs.dt)
        w = float(cs.window[n])
        wc, ws = w * pc, w * ps
        hcv, hsv = wc * hc_ - ws * hs_, ws * hc_ + wc * hs_
        for reg, (re, im) in zip(cs.regions, acc):
            b = reg.box
            v = F[reg.component][b[0]:b[1], b[2]:b[3], b[4]:b[5]]
            cc, ss = (wc, ws) if reg.component[0] == "E" else (hcv, hsv)
            for f in range(freqs.size):
                re[f] += v * float(cc[f])
                im[f] += v * float(ss[f])
        window_sum += w
        pc, ps = pc * sc_ - ps * ss_, ps * sc_ + pc * ss_
    out = {"steps": np.array(GOLDEN_STEPS), "window_sum": np.array(window_sum)}
    for n in S:
        out[f"field_{n}"] = F[n].numpy()
    for i, (reg, (re, im)) in enumerate(zip(cs.regions, acc)):
        out[f"dft_{i}_re"] = re.numpy()
        out[f"dft_{i}_im"] = im.numpy()
    # checksums of the compiled inputs, to detect a drifted scene compiler
    out["check_curl_Ex"] = np.array(float(np.abs(cs.curl["Ex"]).sum()))
    out["check_poles"] = np.array([float(np.abs(p.drive).sum()) for p in cs.poles])
    out["check_patch"] = np.array([float(np.abs(p.coeff).sum()) for p in cs.patches])
    out["check_lines"] = np.array([float(np.abs(lp.coeff).sum()) for lp in cs.line_patches])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    args = ap.parse_args()
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle.build_ref import reference_checkout

    ref = reference_checkout(args.reference)
    if ref is None:
        sys.exit("no reference checkout: pass --reference or set WITWIN_MAXWELL_REFERENCE")
    torch.set_default_dtype(torch.float64)
    global REFERENCE
    REFERENCE = Path(ref)
    tr = load_reference(ref)
    rng = np.random.default_rng(20261203)
    np.savez_compressed(HERE / "ops.npz", **op_vectors(tr, rng))
    np.savez_compressed(HERE / "steps.npz", **step_vectors(tr))
    print("wrote", HERE / "ops.npz", HERE / "steps.npz")


if __name__ == "__main__":
    main()
