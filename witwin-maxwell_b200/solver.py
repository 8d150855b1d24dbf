"""The fused-engine FDTD solver: a drop-in for the reference's ``FDTD`` step path.

``B200FDTD`` binds one compiled scene (``scene.compile_scene``) to the
``fdtd_engine_*`` C ABI, advances it with one fused sm_100a kernel per time step
and returns monitor spectra in the reference's conventions: running DFT with
phase exp(+i w n dt), H samples retarded by half a step, scaled by
2 / sum(window) (witwin/maxwell/fdtd/observers.py:236-241, spectral.py:165-232).

It replaces the reference's per-step Python loop (witwin/maxwell/fdtd/runtime/
stepping.py:2289-2345), whose kernel sequence per step is H update, TFSF H
correction, ADE advance, E update, TFSF E correction, soft sources, ADE
subtraction, PEC clamp, observers.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .scene import COMP_INDEX, CompiledScene, GaussianPulse, component_shape, window_scales


def _require_cuda(device: torch.device) -> None:
    if device.type != "cuda" or not torch.cuda.is_available():
        raise RuntimeError("B200FDTD requires a CUDA device; there is no CPU path")


# Field storage kinds of the engine (fdtd_engine_set_storage): FP32 is the exact
# path; FP16 / BF16 store E and H in 16 bits with per-component power-of-two
# scales (arithmetic stays FP32; ADE pole state is FP32 with FP16 fields and
# BF16 with BF16 fields).
STORAGE_KINDS = {"fp32": 0, "fp16": 1, "bf16": 2}


def pin_scene(cs):
    """A copy of a compiled scene whose large per-cell arrays (the decay / curl
    coefficient arrays and the pole drive / 1/eps boxes) are CPU tensors in
    pinned memory, so that building an engine from it uploads them
    asynchronously at full PCIe / C2C speed.  The small arrays stay numpy."""
    import dataclasses

    def pin(a):
        return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).pin_memory()

    return dataclasses.replace(
        cs,
        decay={k: pin(v) for k, v in cs.decay.items()},
        curl={k: pin(v) for k, v in cs.curl.items()},
        poles=[dataclasses.replace(p, drive=pin(p.drive), inv_eps=pin(p.inv_eps)) for p in cs.poles],
    )


class B200FDTD:
    def __init__(
        self,
        compiled: CompiledScene,
        *,
        device: str | torch.device | None = None,
        sample_block: int = 32,
        tile_rows: int = 0,
        chunk_planes: int = 0,
        storage: str = "fp32",
        storage_scales=None,
    ):
        if storage not in STORAGE_KINDS:
            raise ValueError(f"storage must be one of {sorted(STORAGE_KINDS)}")
        self.storage = storage
        self.storage_scales_arg = None if storage_scales is None else [float(x) for x in storage_scales]
        self.compiled = compiled
        self.device = torch.device(device if device is not None else "cuda")
        _require_cuda(self.device)
        self.lib = _lib.load()
        self.sample_block = int(sample_block)
        self.tile_rows = int(tile_rows)
        self.chunk_planes = int(chunk_planes)
        self.handle = None
        self.handle_imag = None  # imaginary-part engine of a Bloch scene
        self.pair = None  # fdtd_bloch pair coupling the two on the Bloch faces
        self.region_base: list[int] = []
        self.n_samples = 0
        self.pole_ids: list[int] = []
        self.steps_done = 0
        self._keep: list = []

    # ------------------------------------------------------------------ setup
    def _dev(self, array, dtype=torch.float32) -> torch.Tensor:
        if isinstance(array, torch.Tensor):
            # a CPU tensor (pinned by pin_scene) uploads asynchronously on the
            # engine's stream, which every later use of it is ordered behind
            t = array.to(device=self.device, dtype=dtype, non_blocking=True).contiguous()
        else:
            t = torch.as_tensor(np.ascontiguousarray(array)).to(device=self.device, dtype=dtype).contiguous()
        self._keep.append(t)
        return t

    def init_field(self) -> "B200FDTD":
        cs = self.compiled
        with torch.cuda.device(self.device):
            self.stream = torch.cuda.current_stream(self.device)
        self.handle = self._build_engine(0)
        self.handle_imag = None
        self.pair = None
        if cs.complex_fields:
            # Bloch faces: the imaginary part is a second engine, coupled to the
            # first on the wrap faces by fdtd_bloch_step_range
            self.handle_imag = self._build_engine(1)
            pc = (ctypes.c_float * 3)(*cs.bloch_cos)
            ps = (ctypes.c_float * 3)(*cs.bloch_sin)
            pair = ctypes.c_void_p()
            _lib.check(self.lib.fdtd_bloch_create(self.handle, self.handle_imag, pc, ps, ctypes.byref(pair)),
                       "fdtd_bloch_create")
            self.pair = pair
        return self

    def _build_engine(self, channel: int):
        """Create and finalize one engine for this scene: channel 0 holds the
        field (the real part on a Bloch scene), channel 1 the imaginary part."""
        cs = self.compiled
        lib = self.lib
        with torch.cuda.device(self.device):
            stream = self.stream
            desc = _lib.FdtdGridDesc()
            desc.nx, desc.ny, desc.nz = (int(n) for n in cs.nodes)
            desc.dt = float(cs.dt)
            for f in range(6):
                desc.boundary[f] = int(cs.boundary[f])
            for a in range(3):
                desc.pml_lo[a] = int(cs.pml_lo[a])
                desc.pml_hi[a] = int(cs.pml_hi[a])
            desc.sample_block = self.sample_block
            desc.tile_rows = self.tile_rows
            desc.chunk_planes = self.chunk_planes
            handle = ctypes.c_void_p()
            _lib.check(lib.fdtd_engine_create(ctypes.byref(desc), ctypes.c_void_p(stream.cuda_stream), ctypes.byref(handle)),
                       "fdtd_engine_create")
            h = handle
            if self.storage != "fp32" or self.storage_scales_arg is not None:
                sc = None
                if self.storage_scales_arg is not None:
                    if len(self.storage_scales_arg) != 6:
                        raise ValueError("storage_scales needs six values (Ex, Ey, Ez, Hx, Hy, Hz)")
                    sc = (ctypes.c_float * 6)(*self.storage_scales_arg)
                _lib.check(lib.fdtd_engine_set_storage(h, STORAGE_KINDS[self.storage], sc), "set_storage")
            for a in range(3):
                _lib.check(lib.fdtd_engine_set_spacing(h, a, _lib.ptr(self._dev(cs.inv_e[a])), _lib.ptr(self._dev(cs.inv_h[a]))),
                           "set_spacing")
                cp = cs.cpml
                _lib.check(
                    lib.fdtd_engine_set_cpml(
                        h, a, *(_lib.ptr(self._dev(cp[key][a])) for key in ("b_e", "c_e", "ik_e", "b_h", "c_h", "ik_h"))
                    ),
                    "set_cpml",
                )
            for name, idx in COMP_INDEX.items():
                dec_u, curl_u = cs.uniform[name]
                dec = None if cs.decay[name] is None else self._dev(cs.decay[name])
                cur = None if cs.curl[name] is None else self._dev(cs.curl[name])
                _lib.check(
                    lib.fdtd_engine_set_coefficients(
                        h, idx, _lib.ptr(dec), float(dec_u if dec_u is not None else 0.0), _lib.ptr(cur),
                        float(curl_u if curl_u is not None else 0.0),
                    ),
                    "set_coefficients",
                )
            nl = getattr(cs, "nonlinear", None)
            if nl is not None:
                # the nonlinear cells' parameters (materials.py:1664-1770); the
                # coefficient arrays above hold the formula with the channels at rest
                for name in ("Ex", "Ey", "Ez"):
                    m = nl.active(name)
                    ijk = np.ascontiguousarray(np.argwhere(m), dtype=np.int32)
                    ch = nl.channels[name]
                    prm = np.ascontiguousarray(np.stack(
                        [cs.eps[name][m], ch["decay"][m], ch["sigma"][m], ch["chi2"][m], ch["chi3"][m], ch["tpa"][m]],
                        axis=1), dtype=np.float32)
                    _lib.check(
                        lib.fdtd_engine_set_nonlinear(h, COMP_INDEX[name], int(len(ijk)), ctypes.c_void_p(ijk.ctypes.data),
                                                      ctypes.c_void_p(prm.ctypes.data), int(nl.general),
                                                      float(np.float32(nl.eps0))),
                        "set_nonlinear",
                    )
            for name, (box, ca, cb) in (getattr(cs, "aniso", None) or {}).items():
                _lib.check(
                    lib.fdtd_engine_set_full_aniso(h, COMP_INDEX[name], _lib.int_array(box), _lib.ptr(self._dev(ca)),
                                                   _lib.ptr(self._dev(cb))),
                    "set_full_aniso",
                )
            self.pole_ids = []
            for pole in cs.poles:
                pid = ctypes.c_int()
                _lib.check(
                    lib.fdtd_engine_add_pole(
                        h, COMP_INDEX[pole.component], pole.kind, _lib.int_array(pole.box), _lib.ptr(self._dev(pole.drive)),
                        _lib.ptr(self._dev(pole.inv_eps)), float(pole.decay), float(pole.restoring), ctypes.byref(pid),
                    ),
                    "add_pole",
                )
                self.pole_ids.append(pid.value)
            for patch in cs.patches:
                if getattr(patch, "channel", 0) != channel:
                    continue
                sig = self._dev(patch.signal)
                _lib.check(
                    lib.fdtd_engine_add_patch(
                        h, COMP_INDEX[patch.component], _lib.int_array(patch.box), _lib.ptr(self._dev(patch.coeff)),
                        _lib.ptr(sig), int(sig.numel()), 1.0,
                    ),
                    "add_patch",
                )
            for sp in (sp for sp in getattr(cs, "shifted", []) if getattr(sp, "channel", 0) == channel):
                st = sp.source_time
                pulse = isinstance(st, GaussianPulse)
                _lib.check(
                    lib.fdtd_engine_add_shifted_patch(
                        h, COMP_INDEX[sp.component], _lib.int_array(sp.box), _lib.ptr(self._dev(sp.scale)),
                        _lib.ptr(self._dev(sp.delay)), float(sp.t_offset), 1 if pulse else 0, float(st.frequency),
                        float(st.fwidth) if pulse else 0.0, float(st.amplitude), float(st.phase),
                        float(st.resolved_delay) if pulse else 0.0, int(cs.time_steps),
                    ),
                    "add_shifted_patch",
                )
            if cs.aux_line is not None and channel == 0:
                aux = cs.aux_line
                line = ctypes.c_int()
                src = self._dev(aux.source)
                _lib.check(
                    lib.fdtd_engine_add_aux_line(
                        h, int(aux.e_decay.size), _lib.ptr(self._dev(aux.e_decay)), _lib.ptr(self._dev(aux.e_curl)),
                        _lib.ptr(self._dev(aux.h_decay)), _lib.ptr(self._dev(aux.h_curl)), int(aux.source_index),
                        _lib.ptr(src), int(src.numel()), ctypes.byref(line),
                    ),
                    "add_aux_line",
                )
                for lp in cs.line_patches:
                    _lib.check(
                        lib.fdtd_engine_add_line_patch(
                            h, COMP_INDEX[lp.component], _lib.int_array(lp.box), _lib.ptr(self._dev(lp.coeff)),
                            line.value, int(lp.sample_kind), _lib.ptr(self._dev(lp.sample_index, torch.int32)),
                            int(lp.sample_axis), float(lp.scale),
                        ),
                        "add_line_patch",
                    )
            self.region_base = []
            for reg in cs.regions:
                base = ctypes.c_int64()
                _lib.check(
                    lib.fdtd_engine_add_sample_region(h, COMP_INDEX[reg.component], _lib.int_array(reg.box), ctypes.byref(base)),
                    "add_sample_region",
                )
                self.region_base.append(base.value)
            self.n_samples = sum(
                (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]) for b in (r.box for r in cs.regions)
            )
            if cs.regions and cs.frequencies:
                omega = (ctypes.c_double * len(cs.frequencies))(*[2.0 * np.pi * f for f in cs.frequencies])
                window = np.ascontiguousarray(cs.window, dtype=np.float64)
                # one weight per step, or per (step, frequency)
                setter = lib.fdtd_engine_set_dft_windows if window.ndim == 2 else lib.fdtd_engine_set_dft
                _lib.check(
                    setter(
                        h, len(cs.frequencies), omega, int(window.shape[0]),
                        window.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                    ),
                    "set_dft",
                )
            _lib.check(lib.fdtd_engine_finalize(h), "finalize")
            torch.cuda.synchronize(self.device)
            self._keep.clear()
        return h

    # --------------------------------------------------------------- stepping
    def step_range(self, n0: int, n1: int) -> float:
        """Advance steps [n0, n1); returns the device time in ms (CUDA events)."""
        ms = ctypes.c_float()
        if getattr(self, "pair", None) is not None:
            _lib.check(self.lib.fdtd_bloch_step_range(self.pair, int(n0), int(n1)), "fdtd_bloch_step_range")
            _lib.check(self.lib.fdtd_bloch_last_ms(self.pair, ctypes.byref(ms)), "fdtd_bloch_last_ms")
        else:
            _lib.check(self.lib.fdtd_engine_step_range(self.handle, int(n0), int(n1)), "step_range")
            _lib.check(self.lib.fdtd_engine_last_ms(self.handle, ctypes.byref(ms)), "last_ms")
        self.steps_done = max(self.steps_done, int(n1))
        return float(ms.value)

    def time_kernel(self, n: int, reps: int) -> float:
        """Average ms of one fused step kernel (advances the fields, records no samples)."""
        ms = ctypes.c_float()
        _lib.check(self.lib.fdtd_engine_time_kernel(self.handle, int(n), int(reps), ctypes.byref(ms)), "time_kernel")
        return float(ms.value)

    def autotune(self) -> tuple[int, int]:
        ty, cx = ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.fdtd_engine_autotune(self.handle, ctypes.byref(ty), ctypes.byref(cx)), "autotune")
        return ty.value, cx.value

    def set_launch(self, variant: int, tile_rows: int = 0, chunk_planes: int = 0) -> None:
        _lib.check(self.lib.fdtd_engine_set_launch(self.handle, int(variant), int(tile_rows), int(chunk_planes)), "set_launch")

    def set_prefetch(self, planes: int) -> None:
        """L2 prefetch distance of the scalar step kernels in x planes (0 disables)."""
        _lib.check(self.lib.fdtd_engine_set_prefetch(self.handle, int(planes)), "set_prefetch")

    def set_wait_limit(self, rounds: int) -> None:
        """Polling rounds of a bounded pipeline wait in the step kernels before it
        reports FDTD_ERR_TIMEOUT (failure detection; 0 makes every wait run out)."""
        _lib.check(self.lib.fdtd_engine_set_wait_limit(self.handle, int(rounds)), "set_wait_limit")

    def set_ade_pass(self, on: bool) -> None:
        """Advance the dispersive poles in a pass after the step kernel (True) or inside it."""
        _lib.check(self.lib.fdtd_engine_set_ade_pass(self.handle, 1 if on else 0), "set_ade_pass")

    def storage_scales(self) -> tuple[str, list[float]]:
        """The engine's field storage kind and per-component scales (Ex..Hz)."""
        kind = ctypes.c_int()
        sc = (ctypes.c_float * 6)()
        _lib.check(self.lib.fdtd_engine_get_storage(self.handle, ctypes.byref(kind), sc), "get_storage")
        name = {v: k for k, v in STORAGE_KINDS.items()}[kind.value]
        return name, [float(x) for x in sc]

    def get_launch(self) -> tuple[int, int, int]:
        v, ty, cx = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.fdtd_engine_get_launch(self.handle, ctypes.byref(v), ctypes.byref(ty), ctypes.byref(cx)), "get_launch")
        return v.value, ty.value, cx.value

    def info(self) -> dict:
        vals = [ctypes.c_int() for _ in range(5)]
        launches = ctypes.c_int64()
        _lib.check(self.lib.fdtd_engine_info(self.handle, *[ctypes.byref(v) for v in vals], ctypes.byref(launches)), "info")
        keys = ("tile_rows", "chunk_planes", "grid_x", "grid_y", "block")
        out = {k: v.value for k, v in zip(keys, vals)}
        out["launches"] = launches.value
        out["variant"] = self.get_launch()[0]
        return out

    def solve(self, time_steps: int | None = None) -> dict:
        steps = self.compiled.time_steps if time_steps is None else int(time_steps)
        if self.handle is None:
            self.init_field()
        self.step_range(self.steps_done, steps)
        return self.monitor_results()

    def checkpoint_save(self, slot: int) -> None:
        _lib.check(self.lib.fdtd_engine_checkpoint_save(self.handle, int(slot)), "checkpoint_save")

    def checkpoint_load(self, slot: int) -> None:
        _lib.check(self.lib.fdtd_engine_checkpoint_load(self.handle, int(slot)), "checkpoint_load")

    # ---------------------------------------------------------------- outputs
    def field(self, name: str, imag: bool = False) -> torch.Tensor:
        """A field component in its Yee shape (the imaginary part of a Bloch field with imag=True)."""
        shape = component_shape(name, self.compiled.nodes)
        out = torch.empty(shape, device=self.device, dtype=torch.float32)
        h = self.handle_imag if imag else self.handle
        if h is None:
            raise ValueError("the scene has no imaginary field channel")
        _lib.check(self.lib.fdtd_engine_unpack_field(h, COMP_INDEX[name], _lib.ptr(out)), "unpack_field")
        return out

    def set_field(self, name: str, value: torch.Tensor) -> None:
        value = value.to(device=self.device, dtype=torch.float32).contiguous()
        _lib.check(self.lib.fdtd_engine_pack_field(self.handle, COMP_INDEX[name], _lib.ptr(value)), "pack_field")
        torch.cuda.synchronize(self.device)

    def pole_state(self, index: int) -> tuple[torch.Tensor, torch.Tensor]:
        pole = self.compiled.poles[index]
        b = pole.box
        shape = (b[1] - b[0], b[3] - b[2], b[5] - b[4])
        pol = torch.empty(shape, device=self.device)
        cur = torch.empty(shape, device=self.device)
        _lib.check(self.lib.fdtd_engine_pole_state(self.handle, self.pole_ids[index], _lib.ptr(pol), _lib.ptr(cur)), "pole_state")
        return pol, cur

    def raw_dft(self, imag: bool = False) -> tuple[torch.Tensor, torch.Tensor]:
        """Unscaled DFT accumulators of one field channel, [freq][slot]."""
        nf = len(self.compiled.frequencies)
        re = torch.empty((nf, self.n_samples), device=self.device)
        im = torch.empty((nf, self.n_samples), device=self.device)
        h = self.handle_imag if imag else self.handle
        _lib.check(self.lib.fdtd_engine_read_dft(h, _lib.ptr(re), _lib.ptr(im)), "read_dft")
        return re, im

    def monitor_results(self, host: bool = False) -> dict:
        """{monitor: {component: complex64 tensor [F, *box shape]}} scaled by 2/sum(window).
        host=True returns CPU tensors in pinned memory (torch's caching host
        allocator), copied asynchronously on the engine stream and synchronized
        once: several times faster than .cpu() on each device tensor."""
        cs = self.compiled
        if not cs.regions or not cs.frequencies:
            return {}
        re, im = self.raw_dft()
        if getattr(self, "handle_imag", None) is not None:
            # complex field F = A + iB: DFT(F) = DFT(A) + i DFT(B)
            re_b, im_b = self.raw_dft(imag=True)
            re, im = re - im_b, im + re_b
        scales = torch.as_tensor(window_scales(cs.window, self.steps_done, len(cs.frequencies)),
                                 dtype=torch.float32, device=self.device)
        out: dict = {}
        for reg, base in zip(cs.regions, self.region_base):
            b = reg.box
            shape = (b[1] - b[0], b[3] - b[2], b[5] - b[4])
            count = shape[0] * shape[1] * shape[2]
            fidx = [cs.frequencies.index(f) for f in cs.monitor_frequencies[reg.monitor]]
            data = torch.complex(re[fidx, base:base + count], im[fidx, base:base + count]) * scales[fidx, None]
            out.setdefault(reg.monitor, {})[reg.component] = data.reshape((len(fidx),) + shape)
        if host:
            staged: dict = {}
            for name, comps in out.items():
                staged[name] = {}
                for comp, v in comps.items():
                    hv = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                    hv.copy_(v, non_blocking=True)
                    staged[name][comp] = hv
            torch.cuda.current_stream(self.device).synchronize()
            return staged
        return out

    def close(self) -> None:
        if getattr(self, "pair", None) is not None:
            self.lib.fdtd_bloch_destroy(self.pair)
            self.pair = None
        if getattr(self, "handle_imag", None) is not None:
            self.lib.fdtd_engine_destroy(self.handle_imag)
            self.handle_imag = None
        if self.handle is not None:
            self.lib.fdtd_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200Batch:
    """Independent scenes stepped together (fdtd_batch_*): each block of
    ``sample_block`` steps of every scene is one CUDA graph replay in which the
    scenes' kernels run concurrently on their own streams.  Results equal the
    solvers stepped one by one.  The solvers must share the device and the
    stream they were initialised on; while the batch exists, step them through it."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        if not self.solvers:
            raise ValueError("empty batch")
        for s in self.solvers:
            if s.handle is None:
                s.init_field()
        self.lib = _lib.load()
        self.handle = None
        handles = (ctypes.c_void_p * len(self.solvers))(*[s.handle.value for s in self.solvers])
        stream = self.solvers[0].stream
        out = ctypes.c_void_p()
        _lib.check(self.lib.fdtd_batch_create(handles, len(self.solvers), ctypes.c_void_p(stream.cuda_stream), ctypes.byref(out)),
                   "fdtd_batch_create")
        self.handle = out
        self.steps_done = 0

    def autotune(self) -> None:
        _lib.check(self.lib.fdtd_batch_autotune(self.handle), "fdtd_batch_autotune")

    def step_range(self, n0: int, n1: int) -> float:
        """Advance every scene over [n0, n1); returns the device time in ms."""
        _lib.check(self.lib.fdtd_batch_step_range(self.handle, int(n0), int(n1)), "fdtd_batch_step_range")
        self.steps_done = max(self.steps_done, int(n1))
        for s in self.solvers:
            s.steps_done = max(s.steps_done, int(n1))
        ms = ctypes.c_float()
        _lib.check(self.lib.fdtd_batch_last_ms(self.handle, ctypes.byref(ms)), "fdtd_batch_last_ms")
        return float(ms.value)

    def info(self) -> dict:
        n, m, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        _lib.check(self.lib.fdtd_batch_info(self.handle, ctypes.byref(n), ctypes.byref(m), ctypes.byref(g)), "fdtd_batch_info")
        return {"scenes": n.value, "block_steps": m.value, "graph_launches": g.value}

    def close(self) -> None:
        if self.handle is not None:
            self.lib.fdtd_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
