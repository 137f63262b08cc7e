"""Shear-flow mode (CapsuleSHEARFLOW: x and z periodic, y walls moving along z)
on the GPU against the FP64 oracle and the exact Couette profile.

Tolerances as in test_gpu_parity.py (FP32 lattice and IB arithmetic, FP64
positions): velocity relative L2 <= 1e-5 per step, vertex positions
max |dx| <= 1e-5 max|x|."""
import numpy as np
import pytest

from preprocess_src_b200 import configs
from tests.test_gpu_parity import comp, rel_l2

pytestmark = pytest.mark.gpu


def _vel(lat, m):
    return np.concatenate([lat["un"][m], lat["vn"][m], lat["wn"][m]])


@pytest.mark.parametrize("walls", [0, 1])
def test_couette_profile(native_lib, walls):
    from preprocess_src_b200.step import Simulation
    case = configs.shear_case("couette_8x16x8", 8, 16, 8, sr=1e-3, walls=walls, flowstart=1)
    with Simulation(case) as sim:
        sim.step(4000)
        lat = sim.export_lattice(fn=False)
    nx, ny, nz = case.nx, case.ny, case.nz
    w = lat["wn"].reshape(nz, ny, nx)[2:nz - 2, 2:ny - 2, 2:nx - 2]
    LY = ny - 4
    y = -LY / 2 - 1.5 + np.arange(2, ny - 2)
    exact = 1e-3 * (y if walls == 0 else y + LY / 2)
    err = np.abs(w - exact[None, :, None]).max() / np.abs(exact).max()
    print(f"walls {walls}: Couette max rel err {err:.2e}")
    assert err <= 1e-5


def _shear_cells():
    # one cell across the periodic x boundary, one inside; sr large enough to deform them in a few steps
    return configs.shear_case("shear_24x20x24_2c", 24, 20, 24, centers=[(11.2, 0.4, -3.1), (-2.0, -0.6, 6.3)],
                              sr=4e-3, walls=0, subdiv=3, radius=5.0, seed=5, Gs=2e-3)


def test_shear_steps_match_oracle(native_lib, oracle_mod):
    from preprocess_src_b200.step import Simulation
    case = _shear_cells()
    o = oracle_mod.Oracle(case)
    m = comp(case)
    with Simulation(case) as sim:
        done = 0
        for n in (1, 5, 20):
            o.step(n - done)
            sim.step(n - done)
            done = n
            lat = sim.export_lattice(fn=False)
            uref = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
            uerr = rel_l2(_vel(lat, m), uref)
            c = sim.export_cells()
            scale = np.abs(o["x"]).max()
            dx = max(np.abs(c[k] - o[k]).max() for k in ("x", "y", "z"))
            print(f"after {n} steps: u rel L2 {uerr:.3e}  max|dx| {dx:.3e}")
            assert uerr <= 1e-5 * max(1, n / 5)
            assert dx <= 1e-5 * scale
        assert sim.status()[0] == 0


def test_shear_state_imported_mid_run_continues_as_the_oracle(native_lib, oracle_mod):
    """The reference-layout state of a running shear flow (moving-wall terms in
    the wall-link populations) imported into a fresh handle continues as the
    oracle does."""
    from preprocess_src_b200.step import Simulation
    case = _shear_cells()
    o = oracle_mod.Oracle(case)
    o.step(15)
    with Simulation(case) as sim:
        sim.iter = o.iter
        sim.import_lattice(o.fn)
        sim.import_cells(x=o["x"], y=o["y"], z=o["z"], xd=o["xd"], nd=o["nd"], volume0=o["volume0"], gx=o["gx"])
        out = sim.export_lattice()
        mq = np.repeat(comp(case), 19)
        assert np.abs(out["fn"][mq] - o.fn[mq]).max() <= 1e-8   # the import/export pair is exact to FP32
        o.step(3)
        sim.step(3)
        lat = sim.export_lattice(fn=False)
        m = comp(case)
        uref = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
        assert rel_l2(_vel(lat, m), uref) <= 1e-5
        c = sim.export_cells()
        assert max(np.abs(c[k] - o[k]).max() for k in ("x", "y", "z")) <= 1e-5 * np.abs(o["x"]).max()


def test_shear_restart_files_round_trip(native_lib, tmp_path):
    from preprocess_src_b200.step import Simulation
    case = _shear_cells()
    with Simulation(case) as a, Simulation(case) as b:
        a.step(4)
        a.write_restart(tmp_path / "restart.bin", fnum=1)
        a.write_center_file(tmp_path / "center.dat")
        b.read_restart(tmp_path / "restart.bin")
        b.read_center_file(tmp_path / "center.dat")
        ca = a.export_cells()
        a.import_cells(xd=np.stack([ca["x"], ca["y"], ca["z"]], axis=1).reshape(-1), gx=b.export_cells()["gx"])
        a.step(3)
        b.step(3)
        ea, eb = a.export_cells(), b.export_cells()
        for k in ("x", "y", "z"):
            np.testing.assert_allclose(eb[k], ea[k], rtol=0, atol=1e-9)


def test_adjoint_rejects_the_shear_mode(native_lib):
    from preprocess_src_b200.step import Simulation
    with Simulation(configs.shear_case("s", 8, 8, 8, sr=1e-3)) as sim:
        with pytest.raises(RuntimeError, match="channel mode"):
            sim.adjoint_record(2, 1)
