"""Generate the golden fixtures in this directory from oracle/af_emulation.py.

The fixtures hold the state of the reference drivers' array programs (restated literally in numpy,
see af_emulation.py) after a few iterations at small sizes.  The reference itself needs ArrayFire,
which is not available, so these vectors come from the emulation; they pin both the C oracle and the
CUDA engine to the reference's array semantics.  Run from the repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import af_emulation as E  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # name: (callable, kwargs)
    "d2q9_lid_16x12": (E.d2q9_lid, dict(nx=16, ny=12, u_lid=0.1, omega=1 / 0.884, steps=200)),
    "d2q9_channel_60x24": (E.d2q9_channel, dict(nx=60, ny=24, u_max=0.1, omega=1 / (3 * (0.1 * 2 * 3 / 20) + 0.5),
                                                ox=13, oy=12, r=3, steps=100)),
    "d3q27_bgk_lid_8x9x10": (E.d3q27_bgk_lid, dict(nx=8, ny=9, nz=10, u_lid=0.1, omega=1.3, steps=40)),
    "d3q27_mrt_lid_8": (E.d3q27_mrt_lid, dict(n=8, u_lid=0.1, steps=40)),
}


def main():
    for name, (fn, kw) in CASES.items():
        arrays = {}
        for tag, dt in (("f64", np.float64), ("f32", np.float32)):
            out = fn(dtype=dt, **kw)
            F, rho = out[0], out[1]
            arrays[f"F_{tag}"] = np.asarray(F, dtype=dt).ravel(order="F")
            arrays[f"rho_{tag}"] = np.asarray(rho, dtype=dt).ravel(order="F")
            for k, comp in zip("xyz", out[2:]):
                arrays[f"u{k}_{tag}"] = np.asarray(comp, dtype=dt).ravel(order="F")
        meta = {k: v for k, v in kw.items()}
        np.savez_compressed(OUT / f"{name}.npz", meta=np.array(repr(meta)), **arrays)
        print(name, {k: v.shape for k, v in arrays.items() if k.endswith("f64")})


if __name__ == "__main__":
    main()
