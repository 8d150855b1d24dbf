"""The reference's own CUDA FDTD ops, stepped in the reference's order (checker).

Loads the library that ``oracle/build_ref.py`` compiles from the reference's
sources into ``oracle/_ref/`` and drives its torch ops
(``torch.ops.witwin_maxwell_fdtd_cuda.*``, schemas at
witwin/maxwell/fdtd/cuda/extension.cpp:2059-2196) over the tensors of one
compiled scene, one op per launch, in the order of
witwin/maxwell/fdtd/runtime/stepping.py:1740-1815 and :2295-2330: H update,
TFSF magnetic corrections, aux H, ADE advance, E update, TFSF electric
corrections, aux E, soft sources, ADE subtraction, PEC clamp.  The monitor
DFT is accumulated in float64 from the stepped fields (phase recurrence as
observers.py:577-659), or -- with ``monitor_ops=True``, for timing the
reference -- by the reference's own FP32 observer kernels, one
accumulate_plane_observer launch per (plane region, frequency) and one
accumulate_point_observers launch per (point group, frequency), with the
weights evaluated on the host per step as accumulate_observers does
(observers.py:577-659).

Test and measurement infrastructure: only tests/ and bench.py's reference
arm import this module.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
REF_LIB = ROOT / "oracle" / "_ref" / "witwin_maxwell_fdtd_cuda.so"
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_H_SPEC = {"Hx": (1, 2, "Ey", "Ez"), "Hy": (0, 2, "Ex", "Ez"), "Hz": (0, 1, "Ex", "Ey")}
_E_SPEC = {"Ex": (1, 2, "Hy", "Hz"), "Ey": (0, 2, "Hx", "Hz"), "Ez": (0, 1, "Hx", "Hy")}
_loaded = False


def available() -> bool:
    return REF_LIB.exists()


def ops():
    global _loaded
    if not _loaded:
        torch.ops.load_library(str(REF_LIB))
        _loaded = True
    return torch.ops.witwin_maxwell_fdtd_cuda


def _shape(name, nodes):
    nx, ny, nz = nodes
    return {
        "Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
        "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz),
    }[name]


class RefGpuSimulation:
    def __init__(self, compiled, device: str = "cuda", channel: int = 0, monitor_ops: bool = False):
        self.cs = cs = compiled
        self.op = ops()
        dev = torch.device(device)
        self.dev = dev

        def t(a, dtype=torch.float32):
            return torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dtype).contiguous()

        nodes = cs.nodes
        self.F = {n: torch.zeros(_shape(n, nodes), device=dev) for n in COMPONENTS}
        self.decay, self.curl = {}, {}
        for n in COMPONENTS:
            du, cu = cs.uniform[n]
            shape = _shape(n, nodes)
            self.decay[n] = torch.full(shape, du, device=dev) if cs.decay[n] is None else t(cs.decay[n])
            self.curl[n] = torch.full(shape, cu, device=dev) if cs.curl[n] is None else t(cs.curl[n])
        self.inv_e = [t(a) for a in cs.inv_e]
        self.inv_h = [t(a) for a in cs.inv_h]
        self.cp = {k: [t(a) for a in v] for k, v in cs.cpml.items()}
        self.cpml = any(cs.pml_lo) or any(cs.pml_hi)
        self.psi, self.slab = {}, {}
        for n in COMPONENTS:
            spec = _H_SPEC.get(n) or _E_SPEC[n]
            shape = _shape(n, nodes)
            for which, axis in enumerate(spec[:2]):
                size = shape[axis]
                low = min(cs.pml_lo[axis], size)
                high = min(cs.pml_hi[axis], max(size - low, 0))
                cshape = list(shape)
                cshape[axis] = low + high
                self.psi[(n, which)] = torch.zeros(cshape, device=dev)
                self.slab[(n, which)] = (low, size - high, high)
        self.poles = []
        for pole in cs.poles:
            shape = _shape(pole.component, nodes)
            b = pole.box
            drive = np.zeros(shape, np.float32)
            drive[b[0]:b[1], b[2]:b[3], b[4]:b[5]] = pole.drive
            inv_eps = (1.0 / cs.eps[pole.component]).astype(np.float32)
            inv_eps[b[0]:b[1], b[2]:b[3], b[4]:b[5]] = pole.inv_eps
            self.poles.append({
                "comp": pole.component, "kind": pole.kind, "decay": float(pole.decay),
                "restoring": float(pole.restoring), "drive": t(drive), "inv_eps": t(inv_eps),
                "P": torch.zeros(shape, device=dev), "J": torch.zeros(shape, device=dev),
            })
        self.patches = [(p.component, p.box, t(p.coeff), np.asarray(p.signal, np.float32)) for p in cs.patches
                        if getattr(p, "channel", 0) == channel]
        self.aux = None
        if cs.aux_line is not None:
            a = cs.aux_line
            ne = a.e_decay.size
            self.aux = {
                "e": torch.zeros(ne, device=dev), "h": torch.zeros(ne - 1, device=dev),
                "ed": t(a.e_decay), "ec": t(a.e_curl), "hd": t(a.h_decay), "hc": t(a.h_curl),
                "src": int(a.source_index), "signal": np.asarray(a.source, np.float32),
            }
        self.lines = [(lp.component, lp.box, t(lp.coeff), lp.sample_kind, int(lp.sample_axis),
                       t(lp.sample_index, torch.int32), float(lp.scale)) for lp in cs.line_patches]
        self.freqs = np.asarray(cs.frequencies, dtype=np.float64)
        nf = self.freqs.size
        self.acc = []
        for reg in cs.regions:
            b = reg.box
            shape = (nf, b[1] - b[0], b[3] - b[2], b[5] - b[4])
            self.acc.append([torch.zeros(shape, dtype=torch.float64, device=dev),
                             torch.zeros(shape, dtype=torch.float64, device=dev)])
        omega = 2.0 * np.pi * self.freqs
        self.step_c, self.step_s = np.cos(omega * cs.dt), np.sin(omega * cs.dt)
        self.hoff_c, self.hoff_s = np.cos(-0.5 * omega * cs.dt), np.sin(-0.5 * omega * cs.dt)
        self.pc, self.ps = np.ones(nf), np.zeros(nf)
        self.window_sum = 0.0
        self.step = 0
        self.monitors = True
        self.monitor_ops = bool(monitor_ops)
        self.ops_groups = self._observer_groups(nf) if self.monitor_ops else []

    def _observer_groups(self, nf):
        """The reference's observer launch groups: a region one cell thick along
        an axis is a plane observer over the component's whole plane
        (observers.cu accumulate_plane_observer); every other region's cells
        form a point group of that component (accumulate_point_observers).
        FP32 accumulators, one per frequency."""
        groups = []
        nodes = self.cs.nodes
        for r, reg in enumerate(self.cs.regions):
            b = reg.box
            ext = _shape(reg.component, nodes)
            sizes = [b[1] - b[0], b[3] - b[2], b[5] - b[4]]
            axis = next((a for a in (2, 0, 1) if sizes[a] == 1), None)
            if axis is not None and sizes.count(1) < 3:
                plane = [ext[a] for a in range(3) if a != axis]
                acc = [torch.zeros((nf, *plane), device=self.dev) for _ in range(2)]
                groups.append(("plane", r, reg.component, axis, b[2 * axis], acc))
            else:
                ii, jj, kk = np.meshgrid(np.arange(b[0], b[1]), np.arange(b[2], b[3]), np.arange(b[4], b[5]),
                                         indexing="ij")
                idx = [torch.as_tensor(v.ravel().astype(np.int64), device=self.dev) for v in (ii, jj, kk)]
                acc = [torch.zeros((nf, idx[0].numel()), device=self.dev) for _ in range(2)]
                groups.append(("points", r, reg.component, idx, None, acc))
        return groups

    # ------------------------------------------------------------------ ops
    def _update_h(self):
        F, cp = self.F, self.cp
        for n, (A, B, first, second) in _H_SPEC.items():
            fn = f"update_magnetic_h{n[1]}"
            if self.cpml:
                sa, sb = self.slab[(n, 0)], self.slab[(n, 1)]
                getattr(self.op, fn + "_cpml_compressed")(
                    F[n], F[first], F[second], self.decay[n], self.curl[n], self.psi[(n, 0)], self.psi[(n, 1)],
                    cp["ik_h"][A], cp["b_h"][A], cp["c_h"][A], cp["ik_h"][B], cp["b_h"][B], cp["c_h"][B],
                    self.inv_h[A], self.inv_h[B], sa[0], sa[1], sa[2], sb[0], sb[1], sb[2], None, None)
            else:
                getattr(self.op, fn + "_standard")(F[n], F[first], F[second], self.decay[n], self.curl[n],
                                                   self.inv_h[A], self.inv_h[B], None, None)

    def _update_e(self):
        F, cp, bnd = self.F, self.cp, self.cs.boundary
        for n, (A, B, first, second) in _E_SPEC.items():
            fn = f"update_electric_e{n[1]}"
            modes = (bnd[2 * A], bnd[2 * A + 1], bnd[2 * B], bnd[2 * B + 1])
            if self.cpml:
                sa, sb = self.slab[(n, 0)], self.slab[(n, 1)]
                getattr(self.op, fn + "_cpml_compressed")(
                    F[n], F[first], F[second], self.decay[n], self.curl[n], self.psi[(n, 0)], self.psi[(n, 1)],
                    cp["ik_e"][A], cp["b_e"][A], cp["c_e"][A], cp["ik_e"][B], cp["b_e"][B], cp["c_e"][B],
                    self.inv_e[A], self.inv_e[B], *modes, sa[0], sa[1], sa[2], sb[0], sb[1], sb[2], None, None)
            else:
                getattr(self.op, fn + "_standard")(F[n], F[first], F[second], self.decay[n], self.curl[n],
                                                   self.inv_e[A], self.inv_e[B], *modes, None, None)

    def _advance_ade(self):
        dt = float(self.cs.dt)
        for p in self.poles:
            e = self.F[p["comp"]]
            if p["kind"] == 0:
                self.op.update_debye_current(e, p["P"], p["J"], p["drive"], p["decay"], dt)
            elif p["kind"] == 1:
                self.op.update_drude_current(e, p["J"], p["drive"], p["decay"])
            else:
                self.op.update_lorentz_current(e, p["P"], p["J"], p["drive"], p["decay"], p["restoring"], dt)

    def _apply_ade(self):
        dt = float(self.cs.dt)
        for p in self.poles:
            self.op.apply_polarization_current(self.F[p["comp"]], p["J"], p["inv_eps"], dt)

    def _line_corrections(self, magnetic: bool):
        incident = self.aux["e"] if magnetic else self.aux["h"]
        for comp, box, coeff, _kind, axis, idx, scale in self.lines:
            if (comp[0] == "H") != magnetic:
                continue
            self.op.add_scaled_line_source_patch(self.F[comp], coeff, incident, idx, axis, box[0], box[2], box[4],
                                                 scale)

    def _clamp_pec(self):
        bnd = self.cs.boundary
        for n, (A, B, _, _) in _E_SPEC.items():
            for axis in (A, B):
                for side in (0, 1):
                    if bnd[2 * axis + side] == 4:
                        self.op.clamp_field_face(self.F[n], axis, side)

    def _accumulate(self, n):
        cs = self.cs
        if self.freqs.size == 0 or not cs.regions:
            return
        w = float(cs.window[n])
        wc, ws = w * self.pc, w * self.ps
        hc = wc * self.hoff_c - ws * self.hoff_s
        hs = ws * self.hoff_c + wc * self.hoff_s
        if self.monitor_ops:
            for kind, _r, comp, where, index, (re, im) in self.ops_groups:
                cc, ss = (wc, ws) if comp[0] == "E" else (hc, hs)
                for f in range(self.freqs.size):
                    if kind == "plane":
                        self.op.accumulate_plane_observer(self.F[comp], re[f], im[f], int(where), int(index),
                                                          float(cc[f]), float(ss[f]))
                    else:
                        self.op.accumulate_point_observers(self.F[comp], where[0], where[1], where[2], re[f], im[f],
                                                           float(cc[f]), float(ss[f]))
            self.window_sum += w
            self.pc, self.ps = (self.pc * self.step_c - self.ps * self.step_s,
                                self.ps * self.step_c + self.pc * self.step_s)
            return
        for reg, (re, im) in zip(cs.regions, self.acc):
            b = reg.box
            v = self.F[reg.component][b[0]:b[1], b[2]:b[3], b[4]:b[5]].double()
            cc, ss = (wc, ws) if reg.component[0] == "E" else (hc, hs)
            re += torch.as_tensor(cc, device=self.dev).view(-1, 1, 1, 1) * v
            im += torch.as_tensor(ss, device=self.dev).view(-1, 1, 1, 1) * v
        self.window_sum += w
        self.pc, self.ps = (self.pc * self.step_c - self.ps * self.step_s,
                            self.ps * self.step_c + self.pc * self.step_s)

    def _add_patches(self, n: int, magnetic: bool):
        """Soft patches of one phase: H components right after the H update
        (witwin/maxwell/fdtd/runtime/stepping.py:1773-1777), E components after
        the E update (:2296-2308)."""
        for comp, box, coeff, signal in self.patches:
            if (comp[0] == "H") == magnetic:
                self.op.add_source_patch(self.F[comp], coeff, box[0], box[2], box[4], float(signal[n]))

    def step_once(self):
        n = self.step
        self._update_h()
        self._add_patches(n, magnetic=True)
        if self.aux is not None:
            self._line_corrections(True)
            self.op.update_auxiliary_magnetic(self.aux["h"], self.aux["e"], self.aux["hd"], self.aux["hc"])
        self._advance_ade()
        self._update_e()
        if self.aux is not None:
            self._line_corrections(False)
            self.op.update_auxiliary_electric(self.aux["e"], self.aux["h"], self.aux["ed"], self.aux["ec"],
                                              self.aux["src"], float(self.aux["signal"][n]))
        self._add_patches(n, magnetic=False)
        self._apply_ade()
        if self.aux is None:
            self._clamp_pec()
        if self.monitors:
            self._accumulate(n)
        self.step += 1

    def run(self, steps: int):
        for _ in range(int(steps)):
            self.step_once()
        return self

    def fields(self) -> dict:
        return {n: v.cpu().numpy() for n, v in self.F.items()}

    def monitor_results(self) -> dict:
        cs = self.cs
        scale = 2.0 / self.window_sum if self.window_sum > 0 else 0.0
        out: dict = {}
        if self.monitor_ops:
            for kind, r, comp, where, index, (re, im) in self.ops_groups:
                reg = cs.regions[r]
                b = reg.box
                shape = (b[1] - b[0], b[3] - b[2], b[5] - b[4])
                if kind == "plane":
                    sl = [slice(b[2 * a], b[2 * a + 1]) for a in range(3) if a != where]
                    data = (re[(slice(None), *sl)].double() + 1j * im[(slice(None), *sl)].double()).cpu().numpy()
                else:
                    data = (re.double() + 1j * im.double()).cpu().numpy()
                fidx = [cs.frequencies.index(f) for f in cs.monitor_frequencies[reg.monitor]]
                out.setdefault(reg.monitor, {})[comp] = data[fidx].reshape((len(fidx),) + shape) * scale
            return out
        for reg, (re, im) in zip(cs.regions, self.acc):
            fidx = [cs.frequencies.index(f) for f in cs.monitor_frequencies[reg.monitor]]
            data = (re[fidx].cpu().numpy() + 1j * im[fidx].cpu().numpy()) * scale
            out.setdefault(reg.monitor, {})[reg.component] = data
        return out


class RefGpuBloch:
    """A complex field on x / y Bloch faces with PEC, NONE or CPML z faces,
    stepped with the reference's own ops: per channel the H updates (standard,
    or compressed CPML with slabs on z only), ADE, source patches and PEC
    clamps of RefGpuSimulation, and for E the reference's complex Bloch kernels
    update_electric_ex_bloch_y_standard_z, update_electric_ey_bloch_x_standard_z
    and update_electric_ez_bloch (electric.cu:356-453, 1164-1229), as
    stepping.py:1118-1173 and 1790 order them; with CPML on z the Ex / Ey
    stretch is folded in afterwards by apply_electric_e{x,y}_cpml_z_correction
    over each z slab of each channel (update_electric_fields_bloch_cpml,
    stepping.py:1373-1387 and 1236-1277; the ops take contiguous copies of the
    slab views and write them back, as the reference's launcher does,
    cuda/backend.py:54-70).  Monitors are the complex DFT A + iB of the two
    channels' spectra."""

    def __init__(self, compiled, device: str = "cuda", bloch_terms=None, term_phases=None):
        """``bloch_terms``: Bloch face terms injected through the reference's own
        add_source_patch_bloch in place of the compiled patches: a CW term
        (component, box, cos_patch, sin_patch, signal_cos, signal_sin) as its real
        and imaginary values in two launches (cuda/backend.py:1817-1854), a pulsed
        term (scale, delay, t_offset, source_time) as the real values scale * w(n dt
        + t_offset - delay) (excitation/temporal.py:229-247, 395-405);
        ``term_phases[component]``: the two tangential (wrap, cos kL, sin kL)."""
        cs = compiled
        if cs.cpml and (any(cs.pml_lo[:2]) or any(cs.pml_hi[:2])):
            raise ValueError("the Bloch checker covers CPML on z only")
        self.cs = cs
        self.re = RefGpuSimulation(cs, device, channel=0)
        self.im = RefGpuSimulation(cs, device, channel=1)
        self.op = self.re.op
        self.z_cpml = bool(cs.cpml and (cs.pml_lo[2] or cs.pml_hi[2]))
        self.terms = None
        if bloch_terms is not None:
            self.re.patches, self.im.patches = [], []
            self.terms = [(t, term_phases[t.component]) for t in bloch_terms]

    def _bloch_terms(self, n: int, magnetic: bool):
        if not self.terms:
            return
        from oracle.oracle import shifted_waveform

        R, I = self.re.F, self.im.F
        dev = self.re.dev
        for t, ph in self.terms:
            comp, box = t.component, t.box
            if (comp[0] == "H") != magnetic:
                continue
            names = ("Hx", "Hy", "Hz") if magnetic else ("Ex", "Ey", "Ez")
            triplet = [f for nm in names for f in (R[nm], I[nm])]
            (wa, ca, sa), (wb, cb, sb) = ph
            if t.cos_patch is None:
                w = shifted_waveform(t.source_time, n * self.cs.dt + t.t_offset - t.delay.astype(np.float64))
                launches = ((torch.as_tensor((t.scale * w).astype(np.float32), device=dev), 1.0, 0.0),)
            else:
                cp, sp = torch.as_tensor(t.cos_patch, device=dev), torch.as_tensor(t.sin_patch, device=dev)
                c, s = float(t.signal_cos[n]), float(t.signal_sin[n])
                launches = ((cp * c + sp * s, 1.0, 0.0), (cp * s - sp * c, 0.0, 1.0))
            for values, sr, si in launches:
                self.op.add_source_patch_bloch(*triplet, values.contiguous(), box[0], box[2], box[4], sr, si,
                                               "xyz".index(comp[1]), float(ca), float(sa), float(cb), float(sb),
                                               int(wa), int(wb))

    def _z_cpml_corrections(self, sim):
        bnd = self.cs.boundary
        cp, F = sim.cp, sim.F
        for comp, h, op, modes, tangent in (("Ex", "Hy", self.op.apply_electric_ex_cpml_z_correction, (bnd[2], bnd[3]), 1),
                                            ("Ey", "Hx", self.op.apply_electric_ey_cpml_z_correction, (bnd[0], bnd[1]), 0)):
            low, hstart, high = sim.slab[(comp, 1)]
            psi = sim.psi[(comp, 1)]
            for local, start, length in ((0, 0, low), (low, hstart, high)):
                if length <= 0:
                    continue
                view = F[comp].narrow(2, start, length)
                pview = psi.narrow(2, local, length)
                field, psi_c = view.contiguous(), pview.contiguous()
                curl = sim.curl[comp].narrow(2, start, length).contiguous()
                op(field, F[h], curl, psi_c, cp["ik_e"][2], cp["b_e"][2], cp["c_e"][2], sim.inv_e[2], 0, 0, start,
                   int(modes[0]), int(modes[1]), int(F[comp].shape[tangent]), int(F[comp].shape[2]))
                view.copy_(field)
                pview.copy_(psi_c)

    def _update_e(self):
        cs, R, I = self.cs, self.re.F, self.im.F
        c, s = cs.bloch_cos, cs.bloch_sin
        inv = self.re.inv_e
        zl, zh = cs.boundary[4], cs.boundary[5]
        self.op.update_electric_ex_bloch_y_standard_z(
            R["Ex"], I["Ex"], R["Hy"], I["Hy"], R["Hz"], I["Hz"], self.re.decay["Ex"], self.re.curl["Ex"],
            float(c[1]), float(s[1]), inv[1], inv[2], zl, zh)
        self.op.update_electric_ey_bloch_x_standard_z(
            R["Ey"], I["Ey"], R["Hx"], I["Hx"], R["Hz"], I["Hz"], self.re.decay["Ey"], self.re.curl["Ey"],
            float(c[0]), float(s[0]), inv[0], inv[2], zl, zh)
        self.op.update_electric_ez_bloch(
            R["Ez"], I["Ez"], R["Hx"], I["Hx"], R["Hy"], I["Hy"], self.re.decay["Ez"], self.re.curl["Ez"],
            float(c[0]), float(s[0]), float(c[1]), float(s[1]), inv[0], inv[1])
        if self.z_cpml:
            self._z_cpml_corrections(self.re)
            self._z_cpml_corrections(self.im)

    def step_once(self):
        re, im = self.re, self.im
        n = re.step
        re._update_h()
        im._update_h()
        re._add_patches(n, magnetic=True)
        im._add_patches(n, magnetic=True)
        self._bloch_terms(n, magnetic=True)
        re._advance_ade()
        im._advance_ade()
        self._update_e()
        re._add_patches(n, magnetic=False)
        im._add_patches(n, magnetic=False)
        self._bloch_terms(n, magnetic=False)
        for sim in (re, im):
            sim._apply_ade()
            sim._clamp_pec()
            sim._accumulate(n)
            sim.step += 1

    def run(self, steps: int):
        for _ in range(int(steps)):
            self.step_once()
        return self

    def fields(self) -> tuple[dict, dict]:
        return self.re.fields(), self.im.fields()

    def monitor_results(self) -> dict:
        a, b = self.re.monitor_results(), self.im.monitor_results()
        return {m: {c: a[m][c] + 1j * b[m][c] for c in a[m]} for m in a}
