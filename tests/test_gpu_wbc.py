"""White cells: a second cell population (rbc_add_wbc & co.; wbc_init
init3.cu, stress.cu:620-655, ibm.cu:334-360 and 670-690,
volume_correction.cu:260-340) against the FP64 oracle.

  * red cells {c0, c1} step exactly as red {c0} + white {c1} with the red
    cells' coefficients: the populations share the lattice and nothing else;
  * red {c0} + white {c1} with their own rgs and BR follow the oracle run with
    per-cell coefficients;
  * a white population of spheres on its own mesh (and no red cells) follows
    the oracle run of the same cells;
  * the restart, cell and center files carry the white cells' blocks where the
    reference's writer puts them, and a restart written from the oracle's
    state resumes on the GPU.
"""
import dataclasses

import numpy as np
import pytest

from oracle import ref_files as RF
from preprocess_src_b200 import configs
from tests.test_gpu_parity import comp, parity_case, rel_l2

pytestmark = pytest.mark.gpu


def _xyz(c, sl=slice(None)):
    return np.concatenate([c["x"][sl], c["y"][sl], c["z"][sl]])


def _u(lat, m):
    return np.concatenate([lat["un"][m], lat["vn"][m], lat["wn"][m]])


def test_split_population_equals_one_population(native_lib):
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    V = case.vertex
    with Simulation(case) as a, Simulation(red) as b:
        b.add_wbc(white)
        assert b.wbc_dims() == (1, V, case.element)
        n0 = b.launches
        a.step(6)
        b.step(6)
        assert b.launches - n0 == 6 * 11   # step_begin, lbm, force reset, and 4 kernels per population
        ca, cr, cw = a.export_cells(), b.export_cells(), b.export_wbc()
        scale = np.abs(_xyz(ca)).max()
        assert np.abs(_xyz(cr) - _xyz(ca, slice(0, V))).max() <= 1e-9 * scale
        assert np.abs(_xyz(cw) - _xyz(ca, slice(V, 2 * V))).max() <= 1e-9 * scale
        np.testing.assert_allclose(cw["gx"], ca["gx"][3:], rtol=0, atol=1e-9 * scale)
        m = comp(case)
        assert rel_l2(_u(b.export_lattice(fn=False), m), _u(a.export_lattice(fn=False), m)) <= 1e-6
        ma, mw = a.cell_metrics(), b.wbc_metrics()
        np.testing.assert_allclose(mw["volume"], ma["volume"][1:], rtol=1e-12)
        np.testing.assert_allclose(mw["area"], ma["area"][1:], rtol=1e-12)
        assert b.status()[0] & 3 == 0


def test_mixed_populations_match_oracle(oracle_mod, native_lib):
    """Red cell rgs = 1, BR = 0; white cell rgs = 2.5 (GSw / GS), BR = 0.02."""
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    o = oracle_mod.Oracle(case, cell_rgs=[1.0, 2.5], cell_br=[0.0, 0.02])
    m = comp(case)
    V = case.vertex
    with Simulation(red) as s:
        s.add_wbc(white, rgs=2.5, br=0.02)
        for nsteps in (1, 4, 10):
            o.step(nsteps)
            s.step(nsteps)
            ref = np.concatenate([o["x"], o["y"], o["z"]]).reshape(3, -1)
            cr, cw = s.export_cells(), s.export_wbc()
            scale = np.abs(ref).max()
            perr = max(np.abs(_xyz(cr).reshape(3, -1) - ref[:, :V]).max(),
                       np.abs(_xyz(cw).reshape(3, -1) - ref[:, V:]).max())
            uerr = rel_l2(_u(s.export_lattice(fn=False), m), _u(o.a, m))
            print(f"iter {o.iter}: u rel L2 {uerr:.3e}  max|dx| {perr:.3e}")
            assert uerr <= 1e-5 * o.iter and perr <= 1e-5 * scale
        assert s.iter == o.iter
        np.testing.assert_allclose(s.wbc_metrics()["volume"], o.volumes()[0][1:], rtol=1e-6)


def test_white_spheres_on_their_own_mesh_match_oracle(oracle_mod, native_lib):
    """No red cells; two icosphere white cells (162 vertices, 320 triangles),
    one across the periodic end of the duct, rgs = 3."""
    from preprocess_src_b200.step import Simulation
    base = configs.duct_case("wbc_only_40x24x24", 40, 24, 24, g=4e-5, Gs=2e-3)
    spheres = configs.sphere_cells(base, [(0.4, -0.6, 3.0), (-0.8, 0.7, 18.2)], subdiv=2, radius=4.5, seed=3)
    assert spheres.vertex == 162 and spheres.element == 320
    o = oracle_mod.Oracle(dataclasses.replace(spheres, params=dict(spheres.params, rgs=3.0)))
    m = comp(base)
    with Simulation(base) as s:
        s.add_wbc(spheres, rgs=3.0)
        for nsteps in (1, 5):
            o.step(nsteps)
            s.step(nsteps)
            cw = s.export_wbc()
            ref = np.concatenate([o["x"], o["y"], o["z"]])
            perr = np.abs(_xyz(cw) - ref).max()
            uerr = rel_l2(_u(s.export_lattice(fn=False), m), _u(o.a, m))
            print(f"iter {o.iter}: u rel L2 {uerr:.3e}  max|dx| {perr:.3e}")
            assert uerr <= 1e-5 * o.iter and perr <= 1e-5 * np.abs(ref).max()
        assert s.status()[0] & 3 == 0


def test_white_cell_files(native_lib, tmp_path):
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    n, V, E = case.n, case.vertex, case.element
    with Simulation(red) as a, Simulation(red) as b:
        for s in (a, b):
            s.add_wbc(white, rgs=2.0)
            s.set_output_interval(3)
        a.step(5)
        a.write_restart(tmp_path / "restart.bin", fnum=4)
        a.write_cell_file(tmp_path / "cell.bin")
        a.write_center_file(tmp_path / "center.dat")
        cr, cw = a.export_cells(), a.export_wbc()
        r = RF.read_restart(tmp_path / "restart.bin", n, 1, V, E, 1, V, E)
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_array_equal(r[k], cr[k])
            np.testing.assert_array_equal(r[k + "_w"], cw[k])
        assert r["qi_w"].any() and r["tp_w"].any() and not r["rx_w"].any()
        c = RF.read_cell_file(tmp_path / "cell.bin", blocks=2)
        assert (int(c["N_w"][0]), int(c["V_w"][0]), int(c["E_w"][0])) == (1, V, E)
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_array_equal(c[k + "_w"], cw[k])
        np.testing.assert_array_equal(c["ele_w"], white.ele_global())
        np.testing.assert_array_equal(c["tp_w"], r["tp_w"])
        lines = (tmp_path / "center.dat").read_text().splitlines()
        assert [ln.split()[0] for ln in lines] == ["0", "0"]
        np.testing.assert_allclose(RF.read_center(tmp_path / "center.dat"), np.concatenate([cr["gx"], cw["gx"]]),
                                   rtol=1e-6)
        assert b.read_restart(tmp_path / "restart.bin") == 4
        b.read_center_file(tmp_path / "center.dat")
        # the reference restarts with fem->xd = cel->x and the centroids at %e precision
        for exp, imp in ((a.export_cells, a.import_cells), (a.export_wbc, a.import_wbc)):
            e = exp()
            imp(xd=np.stack([e["x"], e["y"], e["z"]], axis=1).reshape(-1))
        a.import_cells(gx=b.export_cells()["gx"])
        a.import_wbc(gx=b.export_wbc()["gx"])
        a.step(4)
        b.step(4)
        for ea, eb in ((a.export_cells(), b.export_cells()), (a.export_wbc(), b.export_wbc())):
            for k in ("x", "y", "z"):
                np.testing.assert_allclose(eb[k], ea[k], rtol=0, atol=1e-9)
        a.write_cell_file(tmp_path / "a.bin")
        b.write_cell_file(tmp_path / "b.bin")
        fa, fb = RF.read_cell_file(tmp_path / "a.bin", 2), RF.read_cell_file(tmp_path / "b.bin", 2)
        np.testing.assert_allclose(fb["tp_w"], fa["tp_w"], rtol=1e-6, atol=1e-12)


def test_restart_from_the_oracle_with_white_cells(oracle_mod, native_lib, tmp_path):
    """A restart.bin with a red and a white block, written from the oracle's
    per-cell-coefficient state, resumes on the GPU."""
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    n, V, E = case.n, case.vertex, case.element
    o = oracle_mod.Oracle(case, cell_rgs=[1.0, 2.5])
    o.step(15)
    f = dict(iter=o.iter, fnum=1, fn=o.fn, dm=o["dm"], um=o["um"], vm=o["vm"], wm=o["wm"])
    for k in ("x", "y", "z", "u", "v", "w"):
        f[k], f[k + "_w"] = o[k][:V], o[k][V:]
    RF.write_restart(tmp_path / "restart.bin", n, 1, V, E, f, 1, V, E)
    RF.write_center(tmp_path / "center.dat", o["gx"])
    o["xd"][:] = np.stack([o["x"], o["y"], o["z"]], axis=1).reshape(-1)
    o["gx"][:] = RF.read_center(tmp_path / "center.dat")
    with Simulation(red) as s:
        s.add_wbc(white, rgs=2.5)
        assert s.read_restart(tmp_path / "restart.bin") == 1
        s.read_center_file(tmp_path / "center.dat")
        o.step(3)
        s.step(3)
        ref = np.concatenate([o["x"], o["y"], o["z"]]).reshape(3, -1)
        got = np.concatenate([_xyz(s.export_cells()).reshape(3, -1), _xyz(s.export_wbc()).reshape(3, -1)], axis=1)
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
        m = comp(case)
        assert rel_l2(_u(s.export_lattice(fn=False), m), _u(o.a, m)) <= 1e-5


def test_add_wbc_argument_checks(native_lib):
    from preprocess_src_b200 import _native as N
    from preprocess_src_b200.step import Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    with Simulation(red) as s:
        with pytest.raises(N.RbcError):
            s.add_wbc(white, rgs=0.0)
        assert s.wbc_dims() == (0, 0, 0)
        with pytest.raises(N.RbcError):   # no white cells yet
            N.check(N.lib().rbc_export_ref_wbc(s._h, *([None] * 11)), s._h)
        s.add_wbc(white)
        with pytest.raises(N.RbcError):
            s.add_wbc(white)
        s.step(2)
        assert s.status()[0] & 3 == 0


def test_white_cells_in_a_batch_and_out_of_the_adjoint(native_lib):
    """A simulation with white cells steps in a batch as it does alone; the
    adjoint refuses it (one population only)."""
    from preprocess_src_b200 import _native as N
    from preprocess_src_b200.step import Batch, Simulation
    case = parity_case()
    red, white = configs.split_cells(case, 1)
    with Simulation(red) as a, Simulation(red) as b:
        for s in (a, b):
            s.add_wbc(white, rgs=2.0)
        batch = Batch([a])
        batch.step(3)
        b.step(3)
        batch.synchronize()
        for ea, eb in ((a.export_cells(), b.export_cells()), (a.export_wbc(), b.export_wbc())):
            for k in ("x", "y", "z"):
                np.testing.assert_allclose(ea[k], eb[k], rtol=0, atol=1e-12, err_msg=k)
        batch.close()
        with pytest.raises(N.RbcError):
            a.adjoint_record(2, 1)
