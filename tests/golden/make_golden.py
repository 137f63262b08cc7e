"""Golden vectors from the reference's own kernels.

TEST INFRASTRUCTURE.  The reference ships no tests or fixtures, so the FP64
oracle is pinned against outputs of the reference's own step modules
(lbm.cu, ibm.cu, stress.cu, matrix_solver.cu, volume_correction.cu, init2.cu),
compiled unmodified from the reference sources with the project-written
oracle/ref_harness (def.h stand-in, helper shims, driver).

    python tests/golden/make_golden.py build [CASE...]          # here: nvcc, needs the reference sources
    python tests/golden/make_golden.py run OUTDIR [CASE...]     # on a GPU: writes OUTDIR/<case>.npz
    python tests/golden/make_golden.py run-dense OUTDIR         # on a GPU: OUTDIR/c2_dense_suspension.npz
    python tests/golden/make_golden.py run-files OUTDIR         # on a GPU: files of the reference's output_data
    python tests/golden/make_golden.py time-dense       # on a GPU: reference step timing, dense suspension

OUTDIR defaults to tests/golden, where the committed fixtures live.

The dense-suspension fixture (256 x 128 x 128, 200 cells) keeps a seeded
sample of its nodes and vertices (dense_sample), the per-plane sums of the
velocity over COMP nodes and the per-cell centroids after DENSE_SNAPSHOTS
steps: the full fields would not fit a repository.

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
        # shear flow (CapsuleSHEARFLOW), both walls moving: one cell across the
        # periodic x boundary, one inside
        "g5_shear24x20x24_2c": configs.shear_case("g5_shear24x20x24_2c", 24, 20, 24,
                                                  centers=[(11.2, 0.4, -3.1), (-2.0, -0.6, 6.3)], sr=4e-3,
                                                  walls=0, subdiv=3, radius=5.0, seed=25, Gs=2e-3,
                                                  residual=1e-12),
        # shear flow with the top wall moving only (topwall)
        "g6_shear20x16x20_1c_top": configs.shear_case("g6_shear20x16x20_1c_top", 20, 16, 20,
                                                      centers=[(0.3, -0.4, 0.6)], sr=5e-3, walls=1, subdiv=3,
                                                      radius=4.5, seed=26, Gs=2e-3, residual=1e-12),
        # one red cell and one white cell (N_W = 1, GSw / GS = 2.5, BRw = 0.02) on
        # the same mesh; fixtures hold the red cells' arrays followed by the
        # white cells' (the layout of the two-cell case)
        "g7_duct32x20x20_1r1w": _with_wbc(configs.duct_case("g7_duct32x20x20_1r1w", 32, 20, 20,
                                                            centers_duct=[(8.2, 9.6, 9.4), (23.9, 9.3, 9.7)],
                                                            subdiv=3, radius=5.0, seed=27, g=4e-5, Gs=2e-3,
                                                            residual=1e-12), nred=1, rgs=2.5, br=0.02),
        # sub-cycling: the membrane and the spread every M steps, the advection
        # with the velocity averaged over them, RUNGE_KUTTA 2 and 1
        "g9_duct24x20x20_1c_m2rk2": configs.duct_case("g9_duct24x20x20_1c_m2rk2", 24, 20, 20,
                                                      centers_duct=[(12.3, 9.6, 9.4)], subdiv=3, radius=5.5,
                                                      seed=29, g=4e-5, Gs=2e-3, residual=1e-12, M=2, rk_order=2),
        "g10_duct24x20x20_1c_m3rk1": configs.duct_case("g10_duct24x20x20_1c_m3rk1", 24, 20, 20,
                                                       centers_duct=[(12.3, 9.6, 9.4)], subdiv=3, radius=5.5,
                                                       seed=30, g=4e-5, Gs=2e-3, residual=1e-12, M=3, rk_order=1),
    }


def _with_wbc(case, nred, rgs, br):
    """case with its cells after the first nred as white cells (GSw / GS = rgs,
    BRw = br): case.meta["wbc"] = (nred, rgs, br)."""
    case.meta["wbc"] = (nred, float(rgs), float(br))
    return case


def wbc_split(case):
    """(red case, white case, rgs, br) of a golden case with white cells, else None."""
    if "wbc" not in case.meta:
        return None
    nred, rgs, br = case.meta["wbc"]
    red, white = configs.split_cells(case, nred)
    return red, white, rgs, br


def cell_coefficients(case):
    """Per-cell (rgs, br) lists of the two-cell oracle run of a white-cell case."""
    nred, rgs, br = case.meta["wbc"]
    nw = case.ncell - nred
    return [1.0] * nred + [rgs] * nw, [case.params["br"]] * nred + [br] * nw


def snapshots(case):
    """Steps after which a fixture holds the state: with VOF (front tracking
    every K = 10 steps) also one five steps after a solve; with M > 1 every
    place in the first cycle."""
    if case.params["vof_k"] > 0:
        return (1, 25, 30)
    if case.params["M"] > 1:
        return tuple(range(1, case.params["M"] + 1)) + (30,)
    return SNAPSHOTS


def dense_case():
    return configs.dense_suspension(residual=1e-12)


DENSE_SNAPSHOTS = (2, 30)


def dense_sample(case, nodes=16384, verts=8192, seed=77):
    """Seeded sample of COMP node indices and vertex indices of the dense
    suspension, sorted (the same on every machine: numpy's PCG64)."""
    rng = np.random.default_rng(seed)
    comp = np.flatnonzero(case.bc == configs.COMP)
    n = np.sort(rng.choice(comp, size=nodes, replace=False))
    v = np.sort(rng.choice(case.ncell * case.vertex, size=verts, replace=False))
    return n, v


def ref_defs(case) -> str:
    p = case.params
    df = (2.0 * p["tau"] - 1.0) / 6.0
    d = (f"-DREF_LX={p['LX']!r} -DREF_LY={float(p['ny'] - 4)!r} -DREF_LZ={p['LZ']!r} -DREF_P={p['P']!r} "
         f"-DREF_B={p['B']!r} -DREF_C={p['C']!r} -DREF_DF={df!r} -DREF_RESIDUAL={p['residual']!r} "
         f"-DREF_ITRMAX={p['itrmax']} -DREF_BR={p['br']!r} -DREF_LAMBDA1={p['lambda1']!r} "
         f"-DREF_K={p['vof_k'] if p['vof_k'] > 0 else 1000000000} -DREF_FLOWSTART={p['flowstart']}")
    if p["flow"] == 1:   # CapsuleSHEARFLOW
        d += f" -DREF_SHEAR -DREF_SR={p['sr']!r}" + (" -DREF_TOPWALL" if p["walls"] == 1 else "")
    if "wbc" in case.meta:
        nred, rgs, br = case.meta["wbc"]
        d += f" -DREF_NW={case.ncell - nred} -DREF_GSW={rgs!r} -DREF_BRW={br!r}"
    if p["M"] != 1 or p["rk_order"] != 4:
        d += f" -DREF_M={p['M']} -DREF_RK={p['rk_order']}"
    return d


def file_cases():
    """Cases whose fixture holds the files the reference's own output_data
    (etc.cu:449-790) wrote: two red cells in a 16 x 12 x 12 duct, after
    FILE_STEPS steps, fnum = FILE_FNUM.  Red cells only: with N_W > 0 the
    reference's output_data does not compile (etc.cu:863-866 redeclare tv and
    leave a declaration list without its ';')."""
    return {"g8_duct16x12x12_files": configs.duct_case("g8_duct16x12x12_files", 16, 12, 12,
                                                       centers_duct=[(4.2, 5.6, 5.4), (12.1, 5.3, 5.7)],
                                                       subdiv=3, radius=3.2, seed=28, g=4e-5, Gs=2e-3,
                                                       residual=1e-12)}


FILE_STEPS, FILE_FNUM = 4, 50
FILE_NAMES = ("restart.bin", f"prof{FILE_FNUM:04d}.bin", f"cell/cell{FILE_FNUM:04d}.bin", f"center{FILE_FNUM:04d}.dat")


def bench_cases():
    """The workloads bench.py's reference arm times with the reference's own
    kernels: the dense suspension and the single-cell duct (tag -> Case)."""
    return {"dense": dense_case(), "single": configs.single_cell_duct(residual=1e-12)}


def build(names=(), if_present=False):
    """Reference-kernel libraries of the golden and bench cases; if_present:
    skip quietly when the reference sources are absent (the recipe checks)."""
    files = file_cases()
    for name, case in list(golden_cases().items()) + list(bench_cases().items()) + list(files.items()):
        if names and name not in names:
            continue
        target = "ref-if-present" if if_present else "ref"
        extra = ["REFETC=1"] if name in files else []
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), target, f"REFTAG={name}",
                        f"REFDEFS={ref_defs(case)}", *extra], check=True)
        if (REF_DIR / f"librefstep_{name}.so").exists():
            print("built", REF_DIR / f"librefstep_{name}.so")


class Ref:
    """The reference's step modules on the GPU, through oracle/ref_harness/ref_driver.cu."""

    def __init__(self, name, case):
        self.L = C.CDLL(str(REF_DIR / f"librefstep_{name}.so"))
        self.case = case
        split = wbc_split(case)
        self.red, self.white = (split[0], split[1]) if split else (case, None)
        red = self.red
        bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        tri = np.ascontiguousarray(red.tri, dtype=np.int32).reshape(-1)
        xr = np.ascontiguousarray(red.xr, dtype=np.float64)
        rc = self.L.ref_setup(case.nx, case.ny, case.nz, bc.ctypes.data_as(C.c_void_p), red.ncell, red.vertex,
                              red.element, tri.ctypes.data_as(C.c_void_p), xr.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(f"ref_setup failed: {rc}")
        if self.white is not None:
            w = self.white
            triw = np.ascontiguousarray(w.tri, dtype=np.int32).reshape(-1)
            xrw = np.ascontiguousarray(w.xr, dtype=np.float64)
            rc = self.L.ref_setup_wbc(w.ncell, w.vertex, w.element, triw.ctypes.data_as(C.c_void_p),
                                      xrw.ctypes.data_as(C.c_void_p))
            if rc:
                raise RuntimeError(f"ref_setup_wbc failed: {rc}")
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
        """dn/un/vn/wn, and with M > 1 also dm/um/vm/wm: the sums of the cycle
        (velocity averaged after its last step)."""
        n = self.case.n
        out = {k: np.empty(n) for k in ("dn", "un", "vn", "wn")}
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        self.L.ref_get_lattice(None, p(out["dn"]), p(out["un"]), p(out["vn"]), p(out["wn"]), None, None, None)
        if self.case.params["M"] > 1:
            out.update({k: np.empty(n) for k in ("dm", "um", "vm", "wm")})
            self.L.ref_get_lattice_m(p(out["dm"]), p(out["um"]), p(out["vm"]), p(out["wm"]))
        return out

    def _population(self, pop, getter):
        nv, nc = pop.ncell * pop.vertex, pop.ncell
        keys = ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz", "xd", "gx", "volume0", "nd")
        sizes = (nv,) * 9 + (3 * nv, 3 * nc, nc, 4 * pop.ncell * pop.element)
        out = {k: np.empty(s) for k, s in zip(keys, sizes)}
        getter(*[out[k].ctypes.data_as(C.c_void_p) for k in keys])
        return out

    def cells(self):
        """Cell arrays of the case: the red cells', followed by the white cells'
        when there are any."""
        out = self._population(self.red, self.L.ref_get_cells)
        if self.white is not None:
            w = self._population(self.white, self.L.ref_get_wbc)
            out = {k: np.concatenate([out[k], w[k]]) for k in out}
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
            for k in ("dn", "un", "vn", "wn", "dm", "um", "vm", "wm"):
                if k in lat:
                    data[f"s{s}_{k}"] = lat[k][m]
            for k in ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz", "gx"):
                data[f"s{s}_{k}"] = cel[k]
        np.savez_compressed(outdir / f"{name}.npz", **data)
        print("wrote", outdir / f"{name}.npz")


def run_dense(outdir):
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    case = dense_case()
    ref = Ref("dense", case)
    m = case.bc == configs.COMP
    nodes, verts = dense_sample(case)
    data = {"snapshots": np.array(DENSE_SNAPSHOTS)}
    done = 0
    for s in DENSE_SNAPSHOTS:
        t0 = time.perf_counter()
        ref.step(s - done)
        done = s
        lat, cel = ref.lattice(), ref.cells()
        for k in ("dn", "un", "vn", "wn"):
            data[f"s{s}_{k}"] = lat[k][nodes]
        data[f"s{s}_plane_u"] = np.stack([np.where(m, lat[k], 0.0).reshape(case.nz, -1).sum(axis=1)
                                          for k in ("un", "vn", "wn")])
        for k in ("x", "y", "z"):
            data[f"s{s}_{k}"] = cel[k][verts]
        data[f"s{s}_gx"] = cel["gx"]
        print(f"dense: step {s} in {time.perf_counter() - t0:.1f} s", flush=True)
    np.savez_compressed(outdir / "c2_dense_suspension.npz", **data)
    print("wrote", outdir / "c2_dense_suspension.npz")


def run_files(outdir):
    """Run each file case FILE_STEPS steps with the reference's kernels, let its
    output_data write the files and keep their bytes (uint8 arrays) and the
    text of center%04d.dat in OUTDIR/<case>.npz."""
    import os
    import tempfile
    outdir = Path(outdir).resolve()
    outdir.mkdir(parents=True, exist_ok=True)
    for name, case in file_cases().items():
        ref = Ref(name, case)
        ref.step(FILE_STEPS)
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as tmp:
            (Path(tmp) / "result" / "cell").mkdir(parents=True)
            os.chdir(tmp)
            try:
                rc = ref.L.ref_write_files(FILE_FNUM)
            finally:
                os.chdir(cwd)
            if rc:
                raise RuntimeError(f"reference output_data failed: {rc}")
            data = {f"file_{k}": np.frombuffer((Path(tmp) / "result" / k).read_bytes(), dtype=np.uint8)
                    for k in FILE_NAMES}
        data["steps"], data["fnum"] = np.array(FILE_STEPS), np.array(FILE_FNUM)
        np.savez_compressed(outdir / f"{name}.npz", **data)
        print("wrote", outdir / f"{name}.npz", {k: v.size for k, v in data.items()})


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
        run(sys.argv[2] if len(sys.argv) > 2 else ROOT / "tests" / "golden", sys.argv[3:])
    elif cmd == "run-files":
        run_files(sys.argv[2] if len(sys.argv) > 2 else ROOT / "tests" / "golden")
    elif cmd == "run-dense":
        run_dense(sys.argv[2] if len(sys.argv) > 2 else ROOT / "tests" / "golden")
    elif cmd == "time-dense":
        time_dense(int(sys.argv[2]) if len(sys.argv) > 2 else 3)
    else:
        raise SystemExit(__doc__)
