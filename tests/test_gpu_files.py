"""The reference's restart and output files (rbc_write_restart & co.) against
the numpy restatement of their layouts (oracle/ref_files.py) and against the
FP64 oracle's state.

  * a restart written and read back resumes the same trajectory;
  * every field of restart.bin, cell%04d.bin and prof%04d.bin sits where the
    reference's writer puts it, with the values the library exports;
  * a restart written from the oracle's FP64 state (a file as the reference
    would write it) resumes on the GPU with the step's parity tolerances;
  * the output-interval averages fem->qi and fem->tp match the oracle's
    per-step load and principal tensions averaged as stress.cu does.
"""
import numpy as np
import pytest

from oracle import ref_files as RF
from tests.test_gpu_parity import comp, parity_case, rel_l2

pytestmark = pytest.mark.gpu


def _dims(case):
    return case.n, case.ncell, case.vertex, case.element


def test_restart_round_trip_resumes_the_same_steps(native_lib, tmp_path):
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    with Simulation(case) as a, Simulation(case) as b:
        a.set_output_interval(4)
        b.set_output_interval(4)
        a.step(7)
        a.write_restart(tmp_path / "restart.bin", fnum=3)
        a.write_center_file(tmp_path / "center.dat")
        assert b.read_restart(tmp_path / "restart.bin") == 3
        b.read_center_file(tmp_path / "center.dat")
        assert b.iter == a.iter == 7
        # the reference restarts with fem->xd = cel->x (etc.cu:248-255): give a the same
        ca = a.export_cells()
        a.import_cells(xd=np.stack([ca["x"], ca["y"], ca["z"]], axis=1).reshape(-1), gx=b.export_cells()["gx"])
        a.step(5)
        b.step(5)
        ea, eb = a.export_cells(), b.export_cells()
        for k in ("x", "y", "z", "xd"):
            np.testing.assert_allclose(eb[k], ea[k], rtol=0, atol=1e-9)
        la, lb = a.export_lattice(fn=False), b.export_lattice(fn=False)
        m = comp(case)
        assert rel_l2(lb["wn"][m], la["wn"][m]) <= 1e-7
        a.write_cell_file(tmp_path / "a.bin")
        b.write_cell_file(tmp_path / "b.bin")
        fa, fb = RF.read_cell_file(tmp_path / "a.bin"), RF.read_cell_file(tmp_path / "b.bin")
        np.testing.assert_allclose(fb["tp"], fa["tp"], rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(fb["qi"], fa["qi"], rtol=1e-4, atol=1e-6 * np.abs(fa["qi"]).max())


def test_file_layouts_match_the_reference_writer(native_lib, tmp_path):
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    n, N, V, E = _dims(case)
    with Simulation(case) as sim:
        sim.step(5)   # odd: non-COMP populations are 0 in the reference's fn buffer
        sim.write_restart(tmp_path / "restart.bin", fnum=1)
        sim.write_cell_file(tmp_path / "cell0001.bin")
        sim.write_prof_file(tmp_path / "prof0001.bin")
        sim.write_center_file(tmp_path / "center.dat")
        lat = sim.export_lattice()
        cel = sim.export_cells()
    r = RF.read_restart(tmp_path / "restart.bin", n, N, V, E)
    assert int(r["iter"][0]) == 5 and int(r["fnum"][0]) == 1
    m = comp(case)
    mq = np.repeat(m, 19)
    np.testing.assert_array_equal(r["fn"][mq], lat["fn"][mq])
    assert not r["fn"][~mq].any()
    for k, e in (("dm", "dn"), ("um", "un"), ("vm", "vn"), ("wm", "wn")):
        np.testing.assert_array_equal(r[k], lat[e])
    assert not r["vf"].any() and not r["vf2"].any() and not r["rx"].any()
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_array_equal(r[k], cel[k])
    assert not r["qi"].any() and not r["tp"].any()   # no output interval set
    c = RF.read_cell_file(tmp_path / "cell0001.bin")
    assert (int(c["N"][0]), int(c["V"][0]), int(c["E"][0])) == (N, V, E)
    for k in ("x", "y", "z", "u", "v", "w"):
        np.testing.assert_array_equal(c[k], cel[k])
    np.testing.assert_array_equal(c["ele"], case.ele_global())
    p = RF.read_prof_file(tmp_path / "prof0001.bin", n)
    assert int(p["iter"][0]) == 5
    np.testing.assert_array_equal(p["bc"], case.bc)
    np.testing.assert_array_equal(p["wm"], lat["wn"])
    np.testing.assert_allclose(RF.read_center(tmp_path / "center.dat"), cel["gx"], rtol=1e-6)


def test_restart_written_from_the_oracle_resumes_on_the_gpu(native_lib, oracle_mod, tmp_path):
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    n, N, V, E = _dims(case)
    o = oracle_mod.Oracle(case)
    o.step(20)
    fields = dict(iter=o.iter, fnum=2, fn=o.fn, dm=o["dm"], um=o["um"], vm=o["vm"], wm=o["wm"],
                  x=o["x"], y=o["y"], z=o["z"], u=o["u"], v=o["v"], w=o["w"])
    RF.write_restart(tmp_path / "restart.bin", n, N, V, E, fields)
    RF.write_center(tmp_path / "center.dat", o["gx"])
    # the reference's restart continues with fem->xd = cel->x and the centroids at %e precision
    o["xd"][:] = np.stack([o["x"], o["y"], o["z"]], axis=1).reshape(-1)
    o["gx"][:] = RF.read_center(tmp_path / "center.dat")
    with Simulation(case) as sim:
        assert sim.read_restart(tmp_path / "restart.bin") == 2
        sim.read_center_file(tmp_path / "center.dat")
        assert sim.iter == o.iter
        o.step(3)
        sim.step(3)
        c = sim.export_cells()
        scale = np.abs(o["x"]).max()
        for k in ("x", "y", "z"):
            assert np.abs(c[k] - o[k]).max() <= 1e-5 * scale, k
        lat = sim.export_lattice(fn=False)
        m = comp(case)
        uref = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
        assert rel_l2(np.concatenate([lat["un"][m], lat["vn"][m], lat["wn"][m]]), uref) <= 1e-5


def test_output_averages_match_the_oracle(native_lib, oracle_mod, tmp_path):
    """FILEOUTPUT = 4 over 6 steps: the averages hold steps 5 and 6 (reset in
    step 5, (5 - 1) % 4 == 0), each weighted 1/4.  Both quantities scale with
    the membrane strain, which six steps from rest leaves near 1e-4, while the
    GPU's and the oracle's positions differ by ~1e-9 after those steps (FP32
    lattice): 1e-4 relative bounds that, and a wrong reset or weight would be
    off by O(1)."""
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    n, N, V, E = _dims(case)
    F, steps = 4, 6
    p = case.params
    o = oracle_mod.Oracle(case)
    ele = case.ele_global()
    tp = np.zeros(N * E * 2)
    qi = np.zeros(N * V * 3)
    for _ in range(steps):
        o.iter += 1
        t = RF.principal_tensions(o["xd"], o["nd"], ele, E, p["C"], p["LX"], p["LZ"])
        o.stress()
        q = o["qd"][:3 * N * V]
        if (o.iter - 1) % F == 0:
            tp[:] = 0.0
            qi[:] = 0.0
        tp += t / F
        qi += q / F
        o.ibm_st1(); o.lbm_d3q19(); o.ibm_st2(); o.volume_correction()
    with Simulation(case, membrane_fp64=1) as sim:
        sim.set_output_interval(F)
        sim.step(steps)
        sim.write_cell_file(tmp_path / "cell.bin")
    c = RF.read_cell_file(tmp_path / "cell.bin")
    print(f"tp rel L2 {rel_l2(c['tp'], tp):.3e}  qi rel L2 {rel_l2(c['qi'], qi):.3e}")
    assert rel_l2(c["tp"], tp) <= 1e-4
    assert rel_l2(c["qi"], qi) <= 1e-4


def test_reads_and_writes_the_reference_writers_files(native_lib, tmp_path):
    """restart.bin, cell%04d.bin, prof%04d.bin and center%04d.dat written by the
    reference's own output_data (etc.cu:449-790) after four steps of its own
    kernels: rbc_read_restart takes the state from the reference's restart.bin,
    and the library's writers then write the same layouts with the same values
    (FP64 positions, averages, centroids and connectivity exact; populations
    and velocities as the FP32 step stores them)."""
    from preprocess_src_b200.step import Simulation
    from tests.test_ref_files_host import _file_golden
    cases = _file_golden()
    if not cases:
        pytest.skip("no output-file fixture")
    for name, case, g, names in cases:
        n, N, V, E = case.n, case.ncell, case.vertex, case.element
        fnum = int(g["fnum"])
        ref = {}
        for k in names:
            p = tmp_path / ("ref_" + k.replace("/", "_"))
            p.write_bytes(g[f"file_{k}"].tobytes())
            ref[k] = p
        with Simulation(case) as sim:
            sim.set_output_interval(1000000)
            assert sim.read_restart(ref["restart.bin"]) == fnum
            assert sim.iter == int(g["steps"])
            sim.read_center_file(ref[f"center{fnum:04d}.dat"])
            sim.write_restart(tmp_path / "restart.bin", fnum=fnum)
            sim.write_cell_file(tmp_path / "cell.bin")
            sim.write_prof_file(tmp_path / "prof.bin")
            sim.write_center_file(tmp_path / "center.dat")
        a = RF.read_restart(ref["restart.bin"], n, N, V, E)
        b = RF.read_restart(tmp_path / "restart.bin", n, N, V, E)
        assert (tmp_path / "restart.bin").stat().st_size == ref["restart.bin"].stat().st_size
        for k in ("iter", "fnum", "x", "y", "z", "qi", "tp", "rx", "ry", "rz"):
            np.testing.assert_array_equal(b[k], a[k], err_msg=k)
        m = np.repeat(case.bc == 0, 19)
        assert np.abs(b["fn"][m] - a["fn"][m]).max() <= 1e-9   # FP32 (f - w): ~1e-10 here
        for k in ("dm", "um", "vm", "wm", "u", "v", "w"):
            scale = max(np.abs(a[k]).max(), 1e-30)
            assert np.abs(b[k] - a[k]).max() <= 1e-6 * scale, k
        ca, cb = RF.read_cell_file(ref[f"cell/cell{fnum:04d}.bin"]), RF.read_cell_file(tmp_path / "cell.bin")
        for k in ("N", "V", "E", "x", "y", "z", "qi", "tp", "ele"):
            np.testing.assert_array_equal(cb[k], ca[k], err_msg=k)
        for k in ("u", "v", "w"):
            assert np.abs(cb[k] - ca[k]).max() <= 1e-6 * np.abs(ca[k]).max(), k
        pa, pb = RF.read_prof_file(ref[f"prof{fnum:04d}.bin"], n), RF.read_prof_file(tmp_path / "prof.bin", n)
        np.testing.assert_array_equal(pb["iter"], pa["iter"])
        np.testing.assert_array_equal(pb["bc"], pa["bc"])
        mc = case.bc == 0
        for k in ("dm", "um", "vm", "wm"):
            assert np.abs(pb[k][mc] - pa[k][mc]).max() <= 1e-6 * max(np.abs(pa[k][mc]).max(), 1e-30), k
        assert (tmp_path / "center.dat").read_text() == ref[f"center{fnum:04d}.dat"].read_text()
