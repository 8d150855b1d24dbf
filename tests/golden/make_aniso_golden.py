"""Generate aniso.npz: the reference's own off-diagonal anisotropic coupling
ops (update_electric_e{x,y,z}_full_aniso, witwin/maxwell/fdtd/cuda/kernels/
aniso.cu:373-580, compiled from the reference's sources into oracle/_ref by
oracle/build_ref.py) on seeded random fields and coefficients, the golden
vectors that pin the oracle's restatement (oracle.full_aniso_correction).

Needs a CUDA device and oracle/_ref (the reference's ops run on the GPU):

    python tests/golden/make_aniso_golden.py [OUTPUT]

Cases: a 9 x 8 x 7 node grid, non-uniform inverse spacings, coefficients with
zeros, each component with every periodic-flag combination of two patterns
(none; x and z periodic) so that wrapped and skipped stencils both occur.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import ref_gpu  # noqa: E402


def run() -> dict:
    op = ref_gpu.ops()
    rng = np.random.default_rng(20261205)
    nodes = (9, 8, 7)
    nx, ny, nz = nodes
    shapes = {"Ex": (nx - 1, ny, nz), "Ey": (nx, ny - 1, nz), "Ez": (nx, ny, nz - 1),
              "Hx": (nx, ny - 1, nz - 1), "Hy": (nx - 1, ny, nz - 1), "Hz": (nx - 1, ny - 1, nz)}
    out = {"nodes": np.array(nodes)}
    for name in ("Hx", "Hy", "Hz"):
        out[name] = rng.standard_normal(shapes[name]).astype(np.float32)
    for a, n in zip("xyz", nodes):
        out[f"inv_d{a}"] = rng.uniform(0.5, 2.0, n).astype(np.float32)
    dev = torch.device("cuda")

    def t(x):
        return torch.tensor(x, device=dev)

    h = [t(out[n]) for n in ("Hx", "Hy", "Hz")]
    inv = [t(out[f"inv_d{a}"]) for a in "xyz"]
    fns = {"Ex": op.update_electric_ex_full_aniso, "Ey": op.update_electric_ey_full_aniso,
           "Ez": op.update_electric_ez_full_aniso}
    for name in ("Ex", "Ey", "Ez"):
        e0 = rng.standard_normal(shapes[name]).astype(np.float32)
        ca = rng.standard_normal(shapes[name]).astype(np.float32)
        cb = rng.standard_normal(shapes[name]).astype(np.float32)
        ca.flat[::5] = 0.0
        cb.flat[::7] = 0.0
        out.update({f"{name}_e0": e0, f"{name}_ca": ca, f"{name}_cb": cb})
        for tag, per in (("open", (0, 0, 0)), ("perxz", (1, 0, 1))):
            e = t(e0)
            fns[name](e, *h, t(ca), t(cb), *inv, *per)
            out[f"{name}_{tag}"] = e.cpu().numpy()
    torch.cuda.synchronize()
    return out


def main():
    target = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "aniso.npz"
    np.savez_compressed(target, **run())
    print("wrote", target)


if __name__ == "__main__":
    main()
