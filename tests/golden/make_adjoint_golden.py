"""Generate adjoint.npz: the reference's own adjoint gradient of a small design
scene, the golden vector that pins the engine's reverse-time adjoint.

Run from the repository root in a container where the reference checkout is
available (it is not needed anywhere else):

    python tests/golden/make_adjoint_golden.py [--reference CHECKOUT]

It imports the reference's frozen Torch implementation of the FDTD kernels
(tests/fdtd/cuda/torch_reference.py, loaded as make_golden.py loads it), which
holds the forward ops and the reverse (adjoint) ops under the names the
native runtime launches, and drives them in float64:

forward, in the reference's step order (stepping.py:1740-1815, 2295-2330)
with dense CPML psi (the layout the reverse ops read): H update with CPML,
ADE advance from E^n, E update with CPML, soft source patches, ADE
subtraction.  Per step it keeps what the reverse step consumes: the mid-step
H (core.py _forward_magnetic_fields), the pre-step E psi, and every pole's
post-advance current (core.py _advance_dispersive_state).

objective: L = sum over the probe's six components of |X|^2 at 300 THz, X the
probe's DFT scaled by 2 / sum(window) with the E / H phases of
observers.py:577-659 (H retarded by omega dt / 2).  Its seed enters the
adjoint of step n's output through seedInjectPoint3D, the reference's seed op
(adjoint.cu seed_inject_point; the seed values are dL/dfield of each sample).

reverse, from the last step to the first, in the order of the reference's
native dispersive runner over its CPML core (fdtd/adjoint/native.py:2104-2290
over :608-725, phases :381-568; allocate_cpml_reverse_context,
reverse_common.py:149-208):
  1. the mid-step H adjoint starts as the post-step H adjoint;
  2. per E component reverseElectricComponentE?Cpml3D, then the two
     accumulateBackwardDiffAdjoint folds of its curl(H) derivative adjoints
     into the mid-step H adjoint;
  3. per H component reverseMagneticComponentH?Cpml3D, then the two
     accumulateForwardDiffAdjoint folds into the pre-step E adjoint;
  4. per pole reverseDispersiveCorrection3D (the 1/eps coupling and its eps
     gradient), then reverseDebye/Drude/LorentzCurrent3D;
  5. the source-term eps gradient of _accumulate_source_term_gradients
     (core.py:778-881): the dipole patch coefficient carries dt / eps, so each
     patch cell gets - lambda_E(post) * coeff * signal[n] / eps (the patch of a
     one-cell-wide dipole reaches the design region).
The per-step eps gradients of Ex, Ey, Ez are summed over the run.

Output (float64): the gradients over the design boxes of the three E
components (dL/d eps, absolute permittivity, the engine's
fdtd_engine_adjoint_grad convention), the spectra, L, the design eps_r and
checksums of the compiled inputs.  The scene: 12 x 10 x 10 cells, 2-cell CPML,
a 3 x 3 x 3 design region (eps_r ~ U[1, 4), seed 5), Drude, Lorentz and Debye
media outside it, an Ez dipole with a 10-step ramped CW at 300 THz, 48 steps.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

from make_golden import _package, load_reference, shapes, t  # noqa: E402

ADJ_STEPS = 48
FREQ = 300e12
PROBE = (3, 5, 5)
DESIGN_LO, DESIGN_HI = (4, 3, 3), (7, 6, 6)
SPEC = {"Hx": ("y", "z", "Ey", "Ez"), "Hy": ("x", "z", "Ex", "Ez"), "Hz": ("x", "y", "Ex", "Ey"),
        "Ex": ("y", "z", "Hy", "Hz"), "Ey": ("x", "z", "Hx", "Hz"), "Ez": ("x", "y", "Hx", "Hy")}
AX = {"x": 0, "y": 1, "z": 2}
# pos / neg CPML axes of each component's reverse op (native.py:411-568): the
# first term of the curl is the positive one
POS_NEG = {"Ex": ("y", "z"), "Ey": ("z", "x"), "Ez": ("x", "y"),
           "Hx": ("y", "z"), "Hy": ("z", "x"), "Hz": ("x", "y")}


def design_eps():
    rng = np.random.default_rng(5)
    return 1.0 + 3.0 * rng.random(tuple(h - l for l, h in zip(DESIGN_LO, DESIGN_HI)))


def adjoint_scene(eps_r=None):
    """The design scene (node-index geometry); eps_r defaults to design_eps()."""
    wm = _package()
    sc = wm.Scene(cells=(12, 10, 10), spacing=25e-9, pml_cells=2)
    sc.structures.append(wm.Structure(wm.Box((8, 1, 1), (9, 9, 9)), wm.Medium.drude(2e15 / (2 * np.pi), 1e14 / (2 * np.pi))))
    sc.structures.append(wm.Structure(wm.Sphere((5, 8, 8), 1.2), wm.Medium.lorentz(2.0, 3.0, 250e12, 20e12)))
    sc.structures.append(wm.Structure(wm.Box((1, 7, 1), (3, 9, 4)), wm.Medium.debye(2.5, 3.5, 1e-14)))
    sc.material_regions.append(wm.MaterialRegion(DESIGN_LO, DESIGN_HI, design_eps() if eps_r is None else eps_r))
    dt = sc.resolve_dt()
    sc.sources.append(wm.PointDipole((9, 5, 5), "Ez", wm.scene.ramped_cw(FREQ, 10, dt, ADJ_STEPS), width=25e-9))
    sc.monitors.append(wm.PointMonitor("probe", PROBE, frequencies=(FREQ,)))
    return sc


def run(tr) -> dict:
    wm = _package()
    cs = wm.compile_scene(adjoint_scene(), ADJ_STEPS)
    K = tr._KERNELS
    S = shapes(cs.nodes)
    N = ADJ_STEPS
    dt = float(cs.dt)
    F = {n: torch.zeros(s, dtype=torch.float64) for n, s in S.items()}
    decay, curl = {}, {}
    for n in S:
        du, cu = cs.uniform[n]
        decay[n] = torch.full(S[n], du, dtype=torch.float64) if cs.decay[n] is None else t(cs.decay[n])
        curl[n] = torch.full(S[n], cu, dtype=torch.float64) if cs.curl[n] is None else t(cs.curl[n])
    eps = {n: t(cs.eps[n]) for n in ("Ex", "Ey", "Ez")}
    cp = {k: [t(a) for a in v] for k, v in cs.cpml.items()}
    inv_e = [t(a) for a in cs.inv_e]
    inv_h = [t(a) for a in cs.inv_h]
    bnd = cs.boundary
    psi = {(n, a): torch.zeros(S[n], dtype=torch.float64) for n, (A, B, _, _) in SPEC.items() for a in (A, B)}
    poles = []
    for p in cs.poles:
        b = p.box
        sl = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
        drive = torch.zeros(S[p.component], dtype=torch.float64)
        drive[sl] = t(p.drive)
        inv_eps = 1.0 / eps[p.component].clone()
        inv_eps[sl] = t(p.inv_eps)
        poles.append(dict(p=p, drive=drive, inv_eps=inv_eps, P=torch.zeros_like(drive), J=torch.zeros_like(drive)))
    omega = 2.0 * np.pi * FREQ
    h_mid, psi_pre, j_post, samples = [], [], [], []

    def prof(kind, a):
        return {q: cp[f"{q}_{kind}"][AX[a]] for q in ("b", "c", "ik")}

    for n in range(N):
        for h in ("Hx", "Hy", "Hz"):
            A, B, first, second = SPEC[h]
            U, V = A.upper(), B.upper()
            pa, pb = prof("h", A), prof("h", B)
            K[f"updateMagneticField{h}3D"](**{
                h: F[h], first: F[first], second: F[second], f"{h}Decay": decay[h], f"{h}Curl": curl[h],
                f"Psi{h}{U}": psi[(h, A)], f"Psi{h}{V}": psi[(h, B)],
                f"InvKappa{h}{U}": pa["ik"], f"By{h}{U}": pa["b"], f"Cy{h}{U}": pa["c"],
                f"InvKappa{h}{V}": pb["ik"], f"By{h}{V}": pb["b"], f"Cy{h}{V}": pb["c"],
                f"invD{A}": inv_h[AX[A]], f"invD{B}": inv_h[AX[B]]})
        h_mid.append({h: F[h].clone() for h in ("Hx", "Hy", "Hz")})
        psi_pre.append({k: v.clone() for k, v in psi.items() if k[0][0] == "E"})
        for pl in poles:
            p = pl["p"]
            e = F[p.component]
            if p.kind == 0:
                K["updateDebyeCurrent3D"](ElectricField=e, Polarization=pl["P"], PolarizationCurrent=pl["J"],
                                          DebyeDrive=pl["drive"], decay=p.decay, dt=dt)
            elif p.kind == 1:
                K["updateDrudeCurrent3D"](ElectricField=e, PolarizationCurrent=pl["J"], DrudeDrive=pl["drive"], decay=p.decay)
            else:
                K["updateLorentzCurrent3D"](ElectricField=e, Polarization=pl["P"], PolarizationCurrent=pl["J"],
                                            LorentzDrive=pl["drive"], decay=p.decay, restoring=p.restoring, dt=dt)
        j_post.append([pl["J"].clone() for pl in poles])
        for e_name in ("Ex", "Ey", "Ez"):
            A, B, first, second = SPEC[e_name]
            U, V = A.upper(), B.upper()
            pa, pb = prof("e", A), prof("e", B)
            K[f"updateElectricField{e_name}Cpml3D"](**{
                e_name: F[e_name], first: F[first], second: F[second], f"{e_name}Decay": decay[e_name],
                f"{e_name}Curl": curl[e_name], f"Psi{e_name}{U}": psi[(e_name, A)], f"Psi{e_name}{V}": psi[(e_name, B)],
                f"InvKappa{e_name}{U}": pa["ik"], f"B{e_name}{U}": pa["b"], f"C{e_name}{U}": pa["c"],
                f"InvKappa{e_name}{V}": pb["ik"], f"B{e_name}{V}": pb["b"], f"C{e_name}{V}": pb["c"],
                f"invD{A}": inv_e[AX[A]], f"invD{B}": inv_e[AX[B]],
                f"{A}LowBoundaryMode": bnd[2 * AX[A]], f"{A}HighBoundaryMode": bnd[2 * AX[A] + 1],
                f"{B}LowBoundaryMode": bnd[2 * AX[B]], f"{B}HighBoundaryMode": bnd[2 * AX[B] + 1]})
        for patch in cs.patches:
            K["addSourcePatch3D"](field=F[patch.component], sourcePatch=t(patch.coeff), offsetI=patch.box[0],
                                  offsetJ=patch.box[2], offsetK=patch.box[4], signal=float(patch.signal[n]))
        for pl in poles:
            K["applyPolarizationCurrent3D"](ElectricField=F[pl["p"].component], PolarizationCurrent=pl["J"],
                                            InvPermittivity=pl["inv_eps"], dt=dt)
        samples.append({c: float(F[c][PROBE]) for c in S})

    # objective and its seeds
    window = np.asarray(cs.window[:N], dtype=np.float64)
    scale = 2.0 / window.sum()
    steps = np.arange(N, dtype=np.float64)
    phase_e = omega * steps * dt
    phase_h = phase_e - 0.5 * omega * dt
    X = {}
    for c in S:
        ph = phase_e if c[0] == "E" else phase_h
        v = np.array([s[c] for s in samples])
        X[c] = scale * np.sum(window * v * (np.cos(ph) + 1j * np.sin(ph)))
    loss = float(sum(abs(x) ** 2 for x in X.values()))
    pi, pj, pk = (torch.tensor([v], dtype=torch.int64) for v in PROBE)

    def seed(c, n, lam):
        ph = phase_e if c[0] == "E" else phase_h
        g = 2.0 * X[c]  # dL/dRe X + i dL/dIm X
        cos_pack = torch.tensor((scale * window * np.cos(ph))[None, :])
        sin_pack = torch.tensor((scale * window * np.sin(ph))[None, :])
        K["seedInjectPoint3D"](AdjField=lam, GradReal=torch.tensor([[g.real]]), GradImag=torch.tensor([[g.imag]]),
                               PointI=pi, PointJ=pj, PointK=pk, CosPack=cos_pack, SinPack=sin_pack, step=n)

    lam = {n: torch.zeros(s, dtype=torch.float64) for n, s in S.items()}
    lam_psi = {k: torch.zeros_like(v) for k, v in psi.items()}
    lam_pole = [{"P": torch.zeros_like(pl["P"]), "J": torch.zeros_like(pl["J"])} for pl in poles]
    grad = {n: torch.zeros(S[n], dtype=torch.float64) for n in ("Ex", "Ey", "Ez")}
    for n in range(N - 1, -1, -1):
        for c in S:
            seed(c, n, lam[c])
        hm = h_mid[n]
        adj_h_mid = {h: lam[h].clone() for h in ("Hx", "Hy", "Hz")}
        pre = {}
        step_grad = {}
        for e_name in ("Ex", "Ey", "Ez"):
            A, B, first, second = SPEC[e_name]
            pos, neg = POS_NEG[e_name]
            pre[e_name] = torch.zeros(S[e_name], dtype=torch.float64)
            step_grad[e_name] = torch.zeros(S[e_name], dtype=torch.float64)
            pre[(e_name, pos)] = torch.zeros(S[e_name], dtype=torch.float64)
            pre[(e_name, neg)] = torch.zeros(S[e_name], dtype=torch.float64)
            d_pos = torch.zeros(S[e_name], dtype=torch.float64)
            d_neg = torch.zeros(S[e_name], dtype=torch.float64)
            pp, pn = prof("e", pos), prof("e", neg)
            # the H component differentiated along the pos / neg axis
            h_pos = {"Ex": "Hz", "Ey": "Hx", "Ez": "Hy"}[e_name]
            h_neg = {"Ex": "Hy", "Ey": "Hz", "Ez": "Hx"}[e_name]
            kw = {f"Adj{e_name}Prev": pre[e_name], f"GradEps{e_name}": step_grad[e_name],
                  "AdjPsiPosPrev": pre[(e_name, pos)], "AdjPsiNegPrev": pre[(e_name, neg)],
                  "AdjDPos": d_pos, "AdjDNeg": d_neg, f"Adj{e_name}Post": lam[e_name],
                  "AdjPsiPosPost": lam_psi[(e_name, pos)], "AdjPsiNegPost": lam_psi[(e_name, neg)],
                  f"{e_name}Decay": decay[e_name], f"{e_name}Curl": curl[e_name], f"Eps{e_name}": eps[e_name],
                  "PsiPos": psi_pre[n][(e_name, pos)], "PsiNeg": psi_pre[n][(e_name, neg)],
                  "BPos": pp["b"], "CPos": pp["c"], "InvKappaPos": pp["ik"],
                  "BNeg": pn["b"], "CNeg": pn["c"], "InvKappaNeg": pn["ik"],
                  f"{first}Mid": hm[first], f"{second}Mid": hm[second],
                  f"invD{A}": inv_e[AX[A]], f"invD{B}": inv_e[AX[B]],
                  f"{A}LowBoundaryMode": bnd[2 * AX[A]], f"{A}HighBoundaryMode": bnd[2 * AX[A] + 1],
                  f"{B}LowBoundaryMode": bnd[2 * AX[B]], f"{B}HighBoundaryMode": bnd[2 * AX[B] + 1]}
            K[f"reverseElectricComponent{e_name}Cpml3D"](**kw)
            P_, N_ = pos.upper(), neg.upper()
            K[f"accumulateBackwardDiffAdjoint{P_}3D"](FieldGrad=adj_h_mid[h_pos], DiffGrad=d_pos,
                                                     **{f"invD{pos}": inv_e[AX[pos]]})
            K[f"accumulateBackwardDiffAdjoint{N_}3D"](FieldGrad=adj_h_mid[h_neg], DiffGrad=d_neg,
                                                     **{f"invD{neg}": inv_e[AX[neg]]})
        for h in ("Hx", "Hy", "Hz"):
            pos, neg = POS_NEG[h]
            pre[h] = torch.zeros(S[h], dtype=torch.float64)
            pre[(h, pos)] = torch.zeros(S[h], dtype=torch.float64)
            pre[(h, neg)] = torch.zeros(S[h], dtype=torch.float64)
            d_pos = torch.zeros(S[h], dtype=torch.float64)
            d_neg = torch.zeros(S[h], dtype=torch.float64)
            pp, pn = prof("h", pos), prof("h", neg)
            K[f"reverseMagneticComponent{h}Cpml3D"](**{
                f"Adj{h}Prev": pre[h], "AdjPsiPosPrev": pre[(h, pos)], "AdjPsiNegPrev": pre[(h, neg)],
                "AdjDPos": d_pos, "AdjDNeg": d_neg, f"Adj{h}Post": adj_h_mid[h],
                "AdjPsiPosPost": lam_psi[(h, pos)], "AdjPsiNegPost": lam_psi[(h, neg)],
                f"{h}Decay": decay[h], f"{h}Curl": curl[h],
                "BPos": pp["b"], "CPos": pp["c"], "InvKappaPos": pp["ik"],
                "BNeg": pn["b"], "CNeg": pn["c"], "InvKappaNeg": pn["ik"]})
            # the E component differentiated along pos / neg by this H update
            e_pos = {"Hx": "Ez", "Hy": "Ex", "Hz": "Ey"}[h]
            e_neg = {"Hx": "Ey", "Hy": "Ez", "Hz": "Ex"}[h]
            P_, N_ = pos.upper(), neg.upper()
            K[f"accumulateForwardDiffAdjoint{P_}3D"](FieldGrad=pre[e_pos], DiffGrad=d_pos,
                                                    **{f"invD{pos}": inv_h[AX[pos]]})
            K[f"accumulateForwardDiffAdjoint{N_}3D"](FieldGrad=pre[e_neg], DiffGrad=d_neg,
                                                    **{f"invD{neg}": inv_h[AX[neg]]})
        new_pole = []
        for pl, lp, jp in zip(poles, lam_pole, j_post[n]):
            p = pl["p"]
            c = p.component
            corrected = torch.zeros_like(lp["J"])
            K["reverseDispersiveCorrection3D"](AdjCurrentCorrected=corrected, GradEps=step_grad[c],
                                               AdjCurrentPost=lp["J"], AdjElectricPost=lam[c], Current=jp,
                                               Eps=eps[c], dt=dt)
            np_ = {"P": torch.zeros_like(lp["P"]), "J": torch.zeros_like(lp["J"])}
            if p.kind == 0:
                K["reverseDebyeCurrent3D"](AdjElectricPrev=pre[c], AdjPolarizationPrev=np_["P"],
                                           AdjPolarizationPost=lp["P"], AdjCurrentPost=corrected,
                                           DebyeDrive=pl["drive"], decay=p.decay, dt=dt)
            elif p.kind == 1:
                K["reverseDrudeCurrent3D"](AdjElectricPrev=pre[c], AdjCurrentPrev=np_["J"], AdjCurrentPost=corrected,
                                           DrudeDrive=pl["drive"], decay=p.decay)
            else:
                K["reverseLorentzCurrent3D"](AdjElectricPrev=pre[c], AdjPolarizationPrev=np_["P"],
                                             AdjCurrentPrev=np_["J"], AdjPolarizationPost=lp["P"],
                                             AdjCurrentPost=corrected, LorentzDrive=pl["drive"], decay=p.decay,
                                             restoring=p.restoring, dt=dt)
            new_pole.append(np_)
        # source-term eps gradient (core.py:778-881): a soft source adds
        # payload = coeff * signal[n] with coeff ~ dt / eps, so its cells get
        # - lambda_post * payload / eps
        for patch in cs.patches:
            c = patch.component
            if c not in step_grad:
                continue
            b = patch.box
            sl = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
            payload = t(patch.coeff) * float(patch.signal[n])
            step_grad[c][sl] -= lam[c][sl] * payload / eps[c][sl]
        for e_name in ("Ex", "Ey", "Ez"):
            grad[e_name] += step_grad[e_name]
        lam = {c: pre[c] for c in S}
        lam_psi = {k: pre[k] for k in lam_psi}
        lam_pole = new_pole
        print(f"reverse step {n}", flush=True)

    region = cs.design
    out = {"steps": np.array(N), "loss": np.array(loss), "eps_r": region.eps_r,
           "design_lo": np.array(DESIGN_LO), "design_hi": np.array(DESIGN_HI)}
    for c in S:
        out[f"X_{c}"] = np.array(X[c])
    sys.path.insert(0, str(ROOT))
    wm_adj = wm.adjoint
    boxes = wm_adj.design_boxes(region, cs.nodes)
    for c, (name, box) in enumerate(zip(("Ex", "Ey", "Ez"), boxes)):
        b = box
        out[f"box_{name}"] = np.array(b)
        out[f"grad_{name}"] = grad[name][b[0]:b[1], b[2]:b[3], b[4]:b[5]].numpy()
    out["check_curl_Ex"] = np.array(float(np.abs(cs.curl["Ex"]).sum()))
    out["check_poles"] = np.array([float(np.abs(p.drive).sum()) for p in cs.poles])
    out["check_patch"] = np.array([float(np.abs(p.coeff).sum()) for p in cs.patches])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    args = ap.parse_args()
    from oracle.build_ref import reference_checkout

    ref = reference_checkout(args.reference)
    if ref is None:
        sys.exit("no reference checkout: pass --reference or set WITWIN_MAXWELL_REFERENCE")
    torch.set_default_dtype(torch.float64)
    tr = load_reference(ref)
    out = run(tr)
    np.savez_compressed(HERE / "adjoint.npz", **out)
    print("wrote", HERE / "adjoint.npz", "loss", float(out["loss"]))


if __name__ == "__main__":
    main()
