"""Mixed-precision study on the single-cell duct (64 x 32 x 32, one cell).

TEST INFRASTRUCTURE (runs the FP64 oracle as the reference).  Runs the FP64
oracle, the GPU path with FP32 populations and the GPU path with FP16
(f - w) populations from the same initial state for N steps and reports, at
checkpoints:
  - relative L2 error of the velocity field (COMP nodes) against FP64,
  - per-cell volume and area drift (relative to V0, A0) and their difference
    from the FP64 run,
  - Taylor deformation D = (L - B) / (L + B) of the cell (L, B from the
    largest / smallest eigenvalue of the vertex gyration tensor) and its error,
  - vertex position error (max, relative to the cell radius).

    python tests/precision_study.py [steps] [every] [out.json]
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Oracle  # noqa: E402
from preprocess_src_b200 import configs  # noqa: E402
from preprocess_src_b200.step import Simulation  # noqa: E402


def taylor(x, y, z):
    p = np.stack([x, y, z], axis=1)
    p = p - p.mean(axis=0)
    ev = np.linalg.eigvalsh(p.T @ p / len(p))
    L, B = np.sqrt(ev[-1]), np.sqrt(ev[0])
    return float((L - B) / (L + B))


def area_volume(x, y, z, tri):
    p = np.stack([x, y, z], axis=1)
    a, b, c = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
    n = np.cross(b - a, c - a)
    return float(0.5 * np.linalg.norm(n, axis=1).sum()), float(np.einsum("ij,ij->i", (a + b + c) / 3.0, n).sum() / 6.0)


def run(steps=10000, every=1000, out=None):
    case = configs.single_cell_duct()
    m = case.bc == configs.COMP
    o = Oracle(case)
    sims = {"f32": Simulation(case, storage=0), "f16": Simulation(case, storage=1)}
    A0, V0 = area_volume(case.xr[0::3], case.xr[1::3], case.xr[2::3], case.tri)
    rows = []
    done = 0
    t_oracle = 0.0
    while done < steps:
        k = min(every, steps - done)
        t0 = time.perf_counter()
        o.step(k)
        t_oracle += time.perf_counter() - t0
        for s in sims.values():
            s.step(k)
        done += k
        uref = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
        zref = o["z"]
        Aref, Vref = area_volume(o["x"], o["y"], zref, case.tri)
        Dref = taylor(o["x"], o["y"], zref)
        row = {"step": done, "fp64": {"volume_drift": Vref / V0 - 1, "area_drift": Aref / A0 - 1, "taylor_D": Dref}}
        for name, s in sims.items():
            lat = s.export_lattice(fn=False)
            cel = s.export_cells()
            u = np.concatenate([lat["un"][m], lat["vn"][m], lat["wn"][m]])
            A, V = area_volume(cel["x"], cel["y"], cel["z"], case.tri)
            D = taylor(cel["x"], cel["y"], cel["z"])
            dz = cel["z"] - zref
            dz -= case.params["LZ"] * np.round(dz / case.params["LZ"])
            dpos = np.sqrt((cel["x"] - o["x"]) ** 2 + (cel["y"] - o["y"]) ** 2 + dz ** 2).max()
            row[name] = {"u_rel_l2": float(np.linalg.norm(u - uref) / np.linalg.norm(uref)),
                         "volume_drift": V / V0 - 1, "area_drift": A / A0 - 1,
                         "volume_vs_fp64": V / Vref - 1, "area_vs_fp64": A / Aref - 1,
                         "taylor_D": D, "taylor_D_err": D - Dref, "max_pos_err_over_R": float(dpos / 7.82),
                         "flags": s.status()[0]}
        rows.append(row)
        print(json.dumps(row), flush=True)
    res = {"case": case.name, "steps": steps, "oracle_s": round(t_oracle, 2), "rows": rows}
    if out:
        Path(out).write_text(json.dumps(res, indent=1))
    return res


if __name__ == "__main__":
    a = sys.argv[1:]
    run(int(a[0]) if a else 10000, int(a[1]) if len(a) > 1 else 1000, a[2] if len(a) > 2 else None)
