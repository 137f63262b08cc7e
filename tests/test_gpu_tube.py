"""Circular tube with the interpolated bounce-back of lbm_cylinder.cu on the GPU
against the FP64 oracle (same restated reference algorithm) and the
Poiseuille profile.  Tolerances as in test_gpu_parity.py."""
import numpy as np
import pytest

from preprocess_src_b200 import configs
from tests.test_gpu_parity import comp, rel_l2

pytestmark = pytest.mark.gpu


def test_tube_poiseuille_matches_the_oracle(native_lib, oracle_mod):
    from preprocess_src_b200.step import Simulation
    R, g = 7.3, 1e-5
    case = configs.tube_case("tube", 6, R, interp=True, g=g)
    o = oracle_mod.Oracle(case)
    o.step(6000)
    with Simulation(case) as sim:
        sim.step(6000)
        lat = sim.export_lattice()
    m = comp(case)
    err = rel_l2(lat["wn"][m], o["wn"][m])
    nx, ny, nz = case.nx, case.ny, case.nz
    x = np.arange(nx) - (nx - 1) / 2.0
    y = np.arange(ny) - (ny - 1) / 2.0
    r2 = np.broadcast_to((x[None, :] ** 2 + y[:, None] ** 2)[None], (nz, ny, nx)).reshape(-1)
    exact = g / (4 * (1.0 / 6.0)) * (R * R - r2)
    perr = rel_l2(lat["wn"][m], exact[m])
    print(f"tube: GPU vs oracle rel L2 {err:.2e}, vs Poiseuille {perr:.3e}")
    assert err <= 1e-4 and perr <= 0.015
    mq = np.repeat(m, 19)
    assert np.abs(lat["fn"][mq] - o.fn[mq]).max() <= 1e-7


def test_tube_with_a_cell_matches_the_oracle(native_lib, oracle_mod):
    from preprocess_src_b200.step import Simulation
    case = configs.tube_case("tube_cell", 32, 9.0, interp=True, g=4e-5, Gs=2e-3, centers=[(0.4, -0.3, 1.0)],
                             subdiv=3, radius=5.0, seed=9)
    o = oracle_mod.Oracle(case)
    o.step(30)
    with Simulation(case) as sim:
        sim.iter = o.iter
        sim.import_lattice(o.fn)
        sim.import_cells(x=o["x"], y=o["y"], z=o["z"], xd=o["xd"], nd=o["nd"], volume0=o["volume0"], gx=o["gx"])
        m = comp(case)
        for n in (1, 5):
            o.step(n if n == 1 else n - 1)
            sim.step(n if n == 1 else n - 1)
            lat = sim.export_lattice(fn=False)
            uref = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
            uerr = rel_l2(np.concatenate([lat["un"][m], lat["vn"][m], lat["wn"][m]]), uref)
            c = sim.export_cells()
            dx = max(np.abs(c[k] - o[k]).max() for k in ("x", "y", "z"))
            print(f"tube + cell, +{n} steps: u rel L2 {uerr:.3e}  max|dx| {dx:.3e}")
            assert uerr <= 1e-5 and dx <= 1e-5 * np.abs(o["x"]).max()
