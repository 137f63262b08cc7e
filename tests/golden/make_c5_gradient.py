"""FP64 reference gradient of the cell-shape loss (the adjoint workload).

TEST INFRASTRUCTURE.  Runs the FP64 CPU oracle (the restated reference step)
on the single-cell duct (64 x 32 x 32, one subdivision-3 cell, tau = 1):

  * target: final vertex positions after NSTEPS steps with Gs = 7e-4,
    g = 1.2e-6 (C = 100);
  * loss L = mean over vertices of |X - target|^2 (minimum image in the
    periodic x and z) after NSTEPS steps at Gs = 5e-4, C = 100, g = 1e-6;
  * dL/dGs, dL/dC, dL/dg by central differences with relative steps 1e-3 and
    1e-4 (their agreement shows the differences are converged).

Writes tests/golden/c5_fp64_gradient.npz (target positions, loss, gradients).
About 2 minutes on 8 cores:

    python tests/golden/make_c5_gradient.py
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from preprocess_src_b200 import configs  # noqa: E402

NSTEPS = 2000
BASE = dict(Gs=5e-4, C=100.0, g=1e-6)
TARGET = dict(Gs=7e-4, C=100.0, g=1.2e-6)
OUT = Path(__file__).resolve().parent / "c5_fp64_gradient.npz"


def final_positions(theta: dict, nsteps: int = NSTEPS) -> np.ndarray:
    case = configs.single_cell_duct(Gs=theta["Gs"], C=theta["C"], g=theta["g"])
    o = oracle.Oracle(case)
    o.step(nsteps)
    return np.stack([o["x"].copy(), o["y"].copy(), o["z"].copy()])


def shape_loss(x: np.ndarray, target: np.ndarray, LX: float, LZ: float) -> float:
    d = x - target
    d[0] -= LX * np.round(d[0] / LX)
    d[2] -= LZ * np.round(d[2] / LZ)
    return float((d * d).sum(axis=0).mean())


def main():
    p = configs.single_cell_duct().params
    LX, LZ = p["LX"], p["LZ"]
    t0 = time.time()
    target = final_positions(TARGET)
    x0 = final_positions(BASE)
    L0 = shape_loss(x0, target, LX, LZ)
    grads = {}
    for hrel in (1e-3, 1e-4):
        g = []
        for k in ("Gs", "C", "g"):
            h = hrel * BASE[k]
            up, dn = dict(BASE), dict(BASE)
            up[k] += h
            dn[k] -= h
            g.append((shape_loss(final_positions(up), target, LX, LZ)
                      - shape_loss(final_positions(dn), target, LX, LZ)) / (2 * h))
        grads[hrel] = np.array(g)
        print(f"h = {hrel:g}: dL/d(Gs, C, g) = {g}", flush=True)
    np.savez(OUT, nsteps=NSTEPS, base=np.array([BASE["Gs"], BASE["C"], BASE["g"]]),
             target_params=np.array([TARGET["Gs"], TARGET["C"], TARGET["g"]]), target=target,
             final=x0, loss=L0, grad_h1e3=grads[1e-3], grad_h1e4=grads[1e-4])
    print(f"loss {L0:.9e}; wrote {OUT} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
