"""Golden vectors from the reference's own kernels.

TEST INFRASTRUCTURE.  The reference ships no tests or fixtures, so the FP64
oracle is pinned against outputs of the reference's own step modules
(lbm.cu, ibm.cu, stress.cu, matrix_solver.cu, volume_correction.cu, init2.cu),
compiled unmodified from the reference sources with the project-written
oracle/ref_harness (def.h stand-in, helper shims, driver).

    python tests/golden/make_golden.py build [CASE...]          # here: nvcc, needs the reference sources
    python tests/golden/make_golden.py run OUTDIR [CASE...]     # on a GPU: writes OUTDIR/<case>.npz
    python tests/golden/make_golden.py time-dense       # on a GPU: reference step timing, dense suspension

g4 runs the volume fraction (front tracking every K = 10 steps, THINC/WLIC
every step) with viscosity ratio LAMBDA1 = 5: fronttrack.cu and thincwlic.cu
join the compiled modules.

The reference takes lengths and physical constants as compile-time macros, so
each case gets its own library (oracle/_ref/librefstep_<case>.so).  Inputs are
regenerated from the case definitions below (seeded mesh placement), so a
fixture stores only outputs: macroscopic fields on COMP nodes and the cell
state after selected steps.
"""
from __future__ import annotations

import ctypes as C
import json
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from preprocess_src_b200 import configs  # noqa: E402

REF_DIR = ROOT / "oracle" / "_ref"
SNAPSHOTS = (1, 30)


def golden_cases():
    """name -> Case.  Parameters must match the -D flags from ref_defs().

    Element counts are multiples of 256: the reference's calc_tension grid is
    (cells * elements) / 256 with no tail guard (stress.cu:604-610), so other
    sizes leave elements without tension in the reference.  g2's first cell
    starts hanging past zmin, which exercises the BUFF-plane bound of the
    spread, the periodic wrap of ibm_st2 and the unwrap of the volume
    correction."""
    return {
        "g1_duct24x20x20_1c": configs.duct_case("g1_duct24x20x20_1c", 24, 20, 20,
                                                centers_duct=[(12.3, 9.6, 9.4)], subdiv=3, radius=5.5,
                                                seed=21, g=4e-5, Gs=2e-3, residual=1e-12),
        "g2_duct32x20x20_2c_wrap": configs.duct_case("g2_duct32x20x20_2c_wrap", 32, 20, 20,
                                                     centers_duct=[(2.5, 9.6, 9.4), (18.0, 9.3, 9.7)],
                                                     subdiv=3, radius=5.0, seed=22, g=4e-5, Gs=2e-3,
                                                     residual=1e-12),
        "g3_duct24x20x20_1c_bend": configs.duct_case("g3_duct24x20x20_1c_bend", 24, 20, 20,
                                                     centers_duct=[(12.3, 9.6, 9.4)], subdiv=3, radius=5.5,
                                                     seed=23, g=4e-5, Gs=2e-3, br=0.02, residual=1e-12),
        "g4_duct24x20x20_1c_vof": configs.duct_case("g4_duct24x20x20_1c_vof", 24, 20, 20,
                                                    centers_duct=[(12.3, 9.6, 9.4)], subdiv=3, radius=5.5,
                                                    seed=24, g=4e-5, Gs=2e-3, residual=1e-12, itrmax=20000,
                                                    lambda1=5.0, vof_k=10, vof_residual=1e-12,
                                                    vof_itrmax=20000),
    }


def snapshots(case):
    """Steps after which a fixture holds the state: with VOF (front tracking
    every K = 10 steps) also one five steps after a solve."""
    return (1, 25, 30) if case.params["vof_k"] > 0 else SNAPSHOTS


def dense_case():
    return configs.dense_suspension(residual=1e-12)


def ref_defs(case) -> str:
    p = case.params
    df = (2.0 * p["tau"] - 1.0) / 6.0
    return (f"-DREF_LX={p['LX']!r} -DREF_LY={float(p['ny'] - 4)!r} -DREF_LZ={p['LZ']!r} -DREF_P={p['P']!r} "
            f"-DREF_B={p['B']!r} -DREF_C={p['C']!r} -DREF_DF={df!r} -DREF_RESIDUAL={p['residual']!r} "
            f"-DREF_ITRMAX={p['itrmax']} -DREF_BR={p['br']!r} -DREF_LAMBDA1={p['lambda1']!r} "
            f"-DREF_K={p['vof_k'] if p['vof_k'] > 0 else 1000000000}")


def build(names=()):
    for name, case in list(golden_cases().items()) + [("dense", dense_case())]:
        if names and name not in names:
            continue
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REFTAG={name}",
                        f"REFDEFS={ref_defs(case)}"], check=True)
        print("built", REF_DIR / f"librefstep_{name}.so")


class Ref:
    """The reference's step modules on the GPU, through oracle/ref_harness/ref_driver.cu."""

    def __init__(self, name, case):
        self.L = C.CDLL(str(REF_DIR / f"librefstep_{name}.so"))
        self.case = case
        bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        tri = np.ascontiguousarray(case.tri, dtype=np.int32).reshape(-1)
        xr = np.ascontiguousarray(case.xr, dtype=np.float64)
        rc = self.L.ref_setup(case.nx, case.ny, case.nz, bc.ctypes.data_as(C.c_void_p), case.ncell, case.vertex,
                              case.element, tri.ctypes.data_as(C.c_void_p), xr.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(f"ref_setup failed: {rc}")
        if case.params["vof_k"] > 0 and self.L.ref_vof_init():
            raise RuntimeError("reference vof_init failed")

    def vf(self):
        out = np.empty(self.case.n)
        self.L.ref_get_vf(out.ctypes.data_as(C.c_void_p))
        return out

    def step(self, n):
        rc = self.L.ref_step(int(n))
        if rc:
            raise RuntimeError(f"reference step failed with error({rc})")

    def lattice(self):
        n = self.case.n
        out = {k: np.empty(n) for k in ("dn", "un", "vn", "wn")}
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        self.L.ref_get_lattice(None, p(out["dn"]), p(out["un"]), p(out["vn"]), p(out["wn"]), None, None, None)
        return out

    def cells(self):
        case = self.case
        nv, nc = case.ncell * case.vertex, case.ncell
        keys = ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz", "xd", "gx", "volume0", "nd")
        sizes = (nv,) * 9 + (3 * nv, 3 * nc, nc, 4 * case.ncell * case.element)
        out = {k: np.empty(s) for k, s in zip(keys, sizes)}
        self.L.ref_get_cells(*[out[k].ctypes.data_as(C.c_void_p) for k in keys])
        return out


def run(outdir, names=()):
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    for name, case in golden_cases().items():
        if names and name not in names:
            continue
        ref = Ref(name, case)
        m = case.bc == configs.COMP
        data = {}
        c0 = ref.cells()
        data["setup_nd"], data["setup_volume0"], data["setup_gx"] = c0["nd"], c0["volume0"], c0["gx"]
        vof = case.params["vof_k"] > 0
        if vof:
            data["setup_vf"] = ref.vf()[m]
        done = 0
        for s in snapshots(case):
            ref.step(s - done)
            done = s
            lat, cel = ref.lattice(), ref.cells()
            if vof:
                data[f"s{s}_vf"] = ref.vf()[m]
            for k in ("dn", "un", "vn", "wn"):
                data[f"s{s}_{k}"] = lat[k][m]
            for k in ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz", "gx"):
                data[f"s{s}_{k}"] = cel[k]
        np.savez_compressed(outdir / f"{name}.npz", **data)
        print("wrote", outdir / f"{name}.npz")


def time_dense(steps=3):
    case = dense_case()
    ref = Ref("dense", case)
    ref.step(1)
    ms = np.zeros(5)
    t0 = time.perf_counter()
    ref.L.ref_time_steps(int(steps), ms.ctypes.data_as(C.c_void_p))
    wall = time.perf_counter() - t0
    fluid = case.fluid_nodes()
    per = ms / steps
    res = {"workload": case.name, "steps": steps, "ms_per_step_by_module": dict(zip(
        ("stress", "ibm_st1", "lbm_d3q19", "ibm_st2", "volume_correction"), per.round(3).tolist())),
        "ms_per_step": round(float(per.sum()), 3), "mlups": round(fluid / (per.sum() * 1e-3) / 1e6, 3),
        "lbm_module_mlups": round(fluid / (per[2] * 1e-3) / 1e6, 1), "wall_s": round(wall, 2)}
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else "build"
    if cmd == "build":
        build(sys.argv[2:])
    elif cmd == "run":
        run(sys.argv[2] if len(sys.argv) > 2 else ROOT / "gpurun_out" / "golden", sys.argv[3:])
    elif cmd == "time-dense":
        time_dense(int(sys.argv[2]) if len(sys.argv) > 2 else 3)
    else:
        raise SystemExit(__doc__)
