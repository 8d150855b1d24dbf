"""x-slab decomposition of one scene over the ranks of a process group.

The reference shards a simulation into x slabs with one-plane halos exchanged by
``torch.distributed.batch_isend_irecv`` between chain neighbours
(witwin/maxwell/fdtd/distributed/nccl_transport.py:14-24): the electric halo
(first owned Ey/Ez node plane to the left neighbour's high ghost) after the E
update and the magnetic halo (last owned Hy/Hz cell plane to the right
neighbour's low ghost) after the H update, each rank's kernels bounded to its
slab (fdtd/cuda/extension.cpp:2066-2068).

The fused engine updates H and E in one launch, so there is no point between
the half-steps at which to exchange.  Each rank instead steps its owned planes
plus one ghost plane on each cut side, and the halos are exchanged once per
step:

* leftwards: the first owned node plane's Ey, Ez (E^{n+1}) to the left
  neighbour's high ghost node plane, which its next H update reads (the
  reference's electric halo);
* rightwards: every component of the last owned plane (E^{n+1}, H^{n+1/2}) to
  the right neighbour's low ghost plane, from which the neighbour recomputes
  the ghost H that its first owned E update reads (the reference's magnetic
  halo, with the E that the recompute needs).

What a rank computes on a ghost plane but does not receive is never read by an
owned cell: the low ghost's CPML psi and ADE state advance from exchanged fields
only (y / z slab terms use in-plane differences), and the x slabs lie wholly in
the end ranks.  Owned cells therefore get exactly the single-domain arithmetic.
Monitors sample owned cells only; rank 0 assembles the spectra.

The same code drives the GPU engine (one process per GPU, NCCL) and the CPU
oracle (gloo), so the decomposition is tested without a second GPU.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .scene import BOUNDARY_BLOCH, BOUNDARY_NONE, BOUNDARY_PERIODIC, COMPONENTS, CompiledRegion, CompiledScene

# components that are half a cell along x (N - 1 entries): Ex, Hy, Hz
_HALF_X = {"Ex": True, "Ey": False, "Ez": False, "Hx": False, "Hy": True, "Hz": True}
# halo payloads (see the module docstring)
LEFT_COMPONENTS = ("Ey", "Ez")
RIGHT_COMPONENTS = COMPONENTS


def split_planes(nx: int, world: int) -> list[tuple[int, int]]:
    """Owned node-plane ranges [x0, x1) of ``world`` ranks over ``nx`` node planes,
    as even as possible (the first ranks take one more)."""
    if world < 1 or nx < 2 * world:
        raise ValueError("need at least two node planes per rank")
    base, extra = divmod(nx, world)
    out, x = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((x, x + n))
        x += n
    return out


def local_range(nx: int, x0: int, x1: int) -> tuple[int, int]:
    """Node planes a rank steps: its owned planes plus one ghost plane per cut."""
    return max(x0 - 1, 0), min(x1 + 1, nx)


def _comp_x_extent(name: str, n: int) -> int:
    return n - 1 if _HALF_X[name] else n


def _clip_box(box, lo: int, hi: int):
    """x-clip of a component box to [lo, hi) (component indices); None when empty."""
    a, b = max(box[0], lo), min(box[1], hi)
    if a >= b:
        return None
    return (a, b) + tuple(box[2:])


def _slice_box_array(arr: np.ndarray, box, clipped) -> np.ndarray:
    return np.ascontiguousarray(arr[clipped[0] - box[0]:clipped[1] - box[0]])


def slice_scene(cs: CompiledScene, x0: int, x1: int) -> tuple[CompiledScene, list]:
    """The compiled scene of the rank owning node planes [x0, x1): its local grid of
    node planes ``local_range`` (ghosts included), every x-dependent tensor cut to
    it, sources and poles clipped, monitors clipped to the owned cells.  Returns
    the local scene and, per local monitor region, (global region index, x offset
    of the local box inside the global region box)."""
    if cs.complex_fields or cs.boundary[0] in (BOUNDARY_PERIODIC, BOUNDARY_BLOCH):
        raise ValueError("x-slab decomposition needs non-periodic x faces")
    if cs.design is not None:
        raise ValueError("the adjoint is not decomposed: build the design problem on one GPU")
    nx = cs.nodes[0]
    lx0, lx1 = local_range(nx, x0, x1)
    nl = lx1 - lx0
    lo_slab, hi_slab = cs.pml_lo[0], cs.pml_hi[0]
    first, last = lx0 == 0, lx1 == nx
    # the x slabs must lie wholly in the end ranks' owned planes: a rank's ghost
    # planes (and their H cells) stay clear of them
    if not first and x0 - 1 < lo_slab:
        raise ValueError("a cut falls inside the low x CPML slab")
    if not last and x1 > nx - 2 - hi_slab:
        raise ValueError("a cut falls inside the high x CPML slab")

    def cut(name: str, arr):
        if arr is None or np.ndim(arr) == 0:
            return arr
        return np.ascontiguousarray(arr[lx0:lx0 + _comp_x_extent(name, nl)])

    boundary = list(cs.boundary)
    if not first:
        boundary[0] = BOUNDARY_NONE
    if not last:
        boundary[1] = BOUNDARY_NONE
    pml_lo, pml_hi = list(cs.pml_lo), list(cs.pml_hi)
    pml_lo[0] = lo_slab if first else 0
    pml_hi[0] = hi_slab if last else 0
    cpml = {k: list(v) for k, v in cs.cpml.items()}
    for k in ("b_e", "c_e", "ik_e"):
        cpml[k][0] = np.ascontiguousarray(cs.cpml[k][0][lx0:lx1])
    for k in ("b_h", "c_h", "ik_h"):
        cpml[k][0] = np.ascontiguousarray(cs.cpml[k][0][lx0:lx1 - 1])
    inv_e = list(cs.inv_e)
    inv_h = list(cs.inv_h)
    inv_e[0] = np.ascontiguousarray(cs.inv_e[0][lx0:lx1])
    inv_h[0] = np.ascontiguousarray(cs.inv_h[0][lx0:lx1 - 1])

    def local_box(name, box):
        """Clip to the local grid and shift to local indices."""
        c = _clip_box(box, lx0, lx0 + _comp_x_extent(name, nl))
        if c is None:
            return None, None
        return c, (c[0] - lx0, c[1] - lx0) + tuple(c[2:])

    poles = []
    for p in cs.poles:
        c, lb = local_box(p.component, p.box)
        if c is None:
            continue
        poles.append(dataclasses.replace(p, box=lb, drive=_slice_box_array(p.drive, p.box, c),
                                         inv_eps=_slice_box_array(p.inv_eps, p.box, c)))
    patches = []
    for p in cs.patches:
        c, lb = local_box(p.component, p.box)
        if c is not None:
            patches.append(dataclasses.replace(p, box=lb, coeff=_slice_box_array(p.coeff, p.box, c)))
    shifted = []
    for p in cs.shifted:
        c, lb = local_box(p.component, p.box)
        if c is not None:
            shifted.append(dataclasses.replace(p, box=lb, scale=_slice_box_array(p.scale, p.box, c),
                                               delay=_slice_box_array(p.delay, p.box, c)))
    line_patches = []
    for lp in cs.line_patches:
        c, lb = local_box(lp.component, lp.box)
        if c is None:
            continue
        idx = lp.sample_index
        if lp.sample_axis == 0:
            idx = np.ascontiguousarray(idx[c[0] - lp.box[0]:c[1] - lp.box[0]])
        line_patches.append(dataclasses.replace(lp, box=lb, coeff=_slice_box_array(lp.coeff, lp.box, c),
                                                sample_index=idx))
    regions, placement = [], []
    for g, reg in enumerate(cs.regions):
        own_hi = min(x1, _comp_x_extent(reg.component, nx))
        c = _clip_box(reg.box, x0, own_hi)
        if c is None:
            continue
        regions.append(CompiledRegion(reg.monitor, reg.component, (c[0] - lx0, c[1] - lx0) + tuple(c[2:])))
        placement.append((g, c[0] - reg.box[0]))
    nonlinear = cs.nonlinear
    if nonlinear is not None:
        # the collocation of a cell next to a cut reads the ghost plane, which
        # the exchange fills: owned cells see the single-domain values
        nonlinear = dataclasses.replace(
            nonlinear, channels={n: {k: cut(n, v) for k, v in ch.items()} for n, ch in nonlinear.channels.items()})
    local = dataclasses.replace(
        cs, nodes=(nl, cs.nodes[1], cs.nodes[2]), boundary=tuple(boundary), pml_lo=pml_lo, pml_hi=pml_hi,
        inv_e=inv_e, inv_h=inv_h, cpml=cpml,
        eps={n: cut(n, a) for n, a in cs.eps.items()},
        decay={n: cut(n, a) for n, a in cs.decay.items()},
        curl={n: cut(n, a) for n, a in cs.curl.items()},
        poles=poles, patches=patches, line_patches=line_patches, regions=regions, shifted=shifted,
        nonlinear=nonlinear,
    )
    return local, placement


class _EngineStepper:
    """One rank's slab on the fused engine (FP32 storage)."""

    def __init__(self, local: CompiledScene, device, **solver_kw):
        from . import _lib
        from .solver import B200FDTD

        self._lib = _lib
        self.solver = B200FDTD(local, device=device, **solver_kw).init_field()
        _lib.check(self.solver.lib.fdtd_engine_set_range_flush(self.solver.handle, 0), "set_range_flush")
        nodes = local.nodes
        self.shape = {n: (nodes[1] - (1 if n in ("Ey", "Hx", "Hz") else 0),
                          nodes[2] - (1 if n in ("Ez", "Hx", "Hy") else 0)) for n in COMPONENTS}
        self.device = self.solver.device

    def buffer(self, name):
        return torch.empty(self.shape[name], device=self.device, dtype=torch.float32)

    def get(self, name, i, out):
        c = COMPONENTS.index(name)
        self._lib.check(self.solver.lib.fdtd_engine_get_plane(self.solver.handle, c, int(i), self._lib.ptr(out)),
                        "get_plane")

    def put(self, name, i, src):
        c = COMPONENTS.index(name)
        self._lib.check(self.solver.lib.fdtd_engine_set_plane(self.solver.handle, c, int(i), self._lib.ptr(src)),
                        "set_plane")

    def step(self, n):
        self.solver.step_range(n, n + 1)

    def sync(self):
        torch.cuda.current_stream(self.device).synchronize()

    def finish(self):
        self._lib.check(self.solver.lib.fdtd_engine_flush(self.solver.handle), "flush")

    def fields(self):
        return {n: self.solver.field(n).cpu().numpy() for n in COMPONENTS}

    def monitors(self):
        return {k: {c: v.cpu().numpy() for c, v in d.items()} for k, d in self.solver.monitor_results().items()}

    def close(self):
        self.solver.close()


class _OracleStepper:
    """One rank's slab on a CPU stepper with the oracle's interface (``fields``,
    ``step_once``, ``monitor_results``): the decomposition's CPU test double."""

    def __init__(self, sim):
        self.sim = sim
        self.device = torch.device("cpu")

    def buffer(self, name):
        f = self.sim.fields[name]
        return torch.empty(f.shape[1:], dtype=torch.float64 if f.dtype == np.float64 else torch.float32)

    def get(self, name, i, out):
        out.copy_(torch.from_numpy(np.ascontiguousarray(self.sim.fields[name][i])))

    def put(self, name, i, src):
        self.sim.fields[name][i] = src.numpy()

    def step(self, n):
        self.sim.step_once()

    def sync(self):
        pass

    def finish(self):
        pass

    def fields(self):
        return {n: np.array(v) for n, v in self.sim.fields.items()}

    def monitors(self):
        return self.sim.monitor_results()

    def close(self):
        self.sim.close()


class XSlabRun:
    """One rank of an x-slab decomposed run of the compiled scene ``cs``.

    ``stepper``: "engine" (the fused engine on ``device``, the default) or a
    callable taking the local compiled scene and returning an object with the
    CPU oracle's interface (used by the tests).  ``exchange`` moves the halo
    planes; by default it is torch.distributed point-to-point over ``group``
    (NCCL with the engine, gloo on the CPU)."""

    def __init__(self, cs: CompiledScene, rank: int, world: int, stepper="engine", device=None, group=None,
                 exchange=None, **solver_kw):
        self.cs = cs
        self.rank, self.world, self.group = rank, world, group
        self.x0, self.x1 = split_planes(cs.nodes[0], world)[rank]
        self.lx0, self.lx1 = local_range(cs.nodes[0], self.x0, self.x1)
        self.local, self.placement = slice_scene(cs, self.x0, self.x1)
        if stepper == "engine":
            self.stepper = _EngineStepper(self.local, device, **solver_kw)
        else:
            self.stepper = _OracleStepper(stepper(self.local))
        self.exchange = exchange or self._p2p
        st = self.stepper
        self.send_left = {n: st.buffer(n) for n in LEFT_COMPONENTS} if rank > 0 else {}
        self.recv_left = {n: st.buffer(n) for n in RIGHT_COMPONENTS} if rank > 0 else {}
        self.send_right = {n: st.buffer(n) for n in RIGHT_COMPONENTS} if rank < world - 1 else {}
        self.recv_right = {n: st.buffer(n) for n in LEFT_COMPONENTS} if rank < world - 1 else {}
        self.steps_done = 0

    # local plane indices of the halo planes
    @property
    def first_owned(self) -> int:
        return self.x0 - self.lx0

    @property
    def last_owned(self) -> int:
        return self.x1 - 1 - self.lx0

    def _p2p(self, run: "XSlabRun") -> None:
        import torch.distributed as dist

        ops = []
        if run.rank > 0:
            for n in LEFT_COMPONENTS:
                ops.append(dist.P2POp(dist.isend, run.send_left[n], run.rank - 1, run.group))
            for n in RIGHT_COMPONENTS:
                ops.append(dist.P2POp(dist.irecv, run.recv_left[n], run.rank - 1, run.group))
        if run.rank < run.world - 1:
            for n in RIGHT_COMPONENTS:
                ops.append(dist.P2POp(dist.isend, run.send_right[n], run.rank + 1, run.group))
            for n in LEFT_COMPONENTS:
                ops.append(dist.P2POp(dist.irecv, run.recv_right[n], run.rank + 1, run.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def pack(self) -> None:
        """Copy this step's outgoing halo planes into the send buffers."""
        st = self.stepper
        for n, b in self.send_left.items():
            st.get(n, self.first_owned, b)
        for n, b in self.send_right.items():
            st.get(n, self.last_owned, b)
        st.sync()

    def unpack(self) -> None:
        """Write the received halo planes into the ghost planes."""
        st = self.stepper
        for n, b in self.recv_left.items():
            st.put(n, 0, b)
        for n, b in self.recv_right.items():
            st.put(n, self.lx1 - 1 - self.lx0, b)

    def step(self, n: int) -> None:
        self.stepper.step(n)
        self.pack()
        self.exchange(self)
        self.unpack()
        self.steps_done = n + 1

    def run(self, n0: int, n1: int) -> None:
        for n in range(n0, n1):
            self.step(n)
        self.stepper.finish()

    def owned_fields(self) -> dict:
        """This rank's owned x range of every component (global x offset, array)."""
        out = {}
        for n, f in self.stepper.fields().items():
            hi = min(self.x1, _comp_x_extent(n, self.cs.nodes[0]))
            out[n] = (self.x0, f[self.first_owned:hi - self.lx0])
        return out

    def local_monitors(self) -> list:
        """(global region index, x offset, spectrum [F, box]) per local region."""
        mons = self.stepper.monitors()
        out = []
        for reg, (g, off) in zip(self.local.regions, self.placement):
            out.append((g, off, np.asarray(mons[reg.monitor][reg.component])))
        return out

    def close(self):
        self.stepper.close()


def assemble_fields(cs: CompiledScene, parts: list) -> dict:
    """Global fields from every rank's ``owned_fields``."""
    out = {}
    for rank_parts in parts:
        for n, (x0, arr) in rank_parts.items():
            if n not in out:
                shape = (_comp_x_extent(n, cs.nodes[0]),) + arr.shape[1:]
                out[n] = np.zeros(shape, dtype=arr.dtype)
            out[n][x0:x0 + arr.shape[0]] = arr
    return out


def assemble_monitors(cs: CompiledScene, parts: list) -> dict:
    """Global spectra {monitor: {component: [F, box]}} from every rank's ``local_monitors``."""
    out: dict = {}
    for rank_parts in parts:
        for g, off, data in rank_parts:
            reg = cs.regions[g]
            b = reg.box
            shape = (data.shape[0], b[1] - b[0], b[3] - b[2], b[5] - b[4])
            dest = out.setdefault(reg.monitor, {})
            if reg.component not in dest:
                dest[reg.component] = np.zeros(shape, dtype=np.complex128)
            dest[reg.component][:, off:off + data.shape[1]] = data
    return out


def step_in_process(runs: list, n: int) -> None:
    """Advance the ranks of one process (``runs`` in rank order, e.g. slabs of one
    device) by step n, exchanging their halo planes by direct copies."""
    for r in runs:
        r.stepper.step(n)
    for r in runs:
        r.pack()
    for left, right in zip(runs[:-1], runs[1:]):
        for name in RIGHT_COMPONENTS:
            right.recv_left[name].copy_(left.send_right[name])
        for name in LEFT_COMPONENTS:
            left.recv_right[name].copy_(right.send_left[name])
    for r in runs:
        r.unpack()
        r.steps_done = n + 1
