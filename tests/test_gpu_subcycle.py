"""Sub-cycling (M > 1) and the lower-order advection (RUNGE_KUTTA 1 and 2)
against the FP64 oracle, through the C ABI.

main.cu:78-106 runs the membrane pass and the spread at the first of every M
lattice steps and the advection and the volume correction at the last; the
force spread at the first acts in all M collide-streams, and the advection
moves the vertices by the velocity averaged over the M steps (lbm.cu:1097-1126,
1435-1460) times M dt.  Both sides start from the same developed state at a
cycle boundary and compare after every step of two cycles, so each place in a
cycle (first, middle, last) is checked.  The exported density and velocity of a
sub-cycled step are the sums of its cycle (ltc->dmD / umD), which the oracle
holds as dm / um.
"""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def sub_case(M, rk):
    return configs.duct_case(f"sub_40x24x24_m{M}rk{rk}", 40, 24, 24,
                             centers_duct=[(0.6, 12.2, 11.7), (21.0, 11.6, 12.4)],
                             subdiv=3, radius=6.0, seed=11, g=4e-5, Gs=2e-3, M=M, rk_order=rk)


@pytest.fixture(scope="module")
def developed(oracle_mod, native_lib):
    """A developed flow with deformed cells (40 plain steps of the oracle)."""
    o = oracle_mod.Oracle(sub_case(1, 4))
    o.step(40)
    return o


def start(oracle_mod, o, M, rk, iter0=42):
    """The oracle of the sub-cycled case from the developed state, and the
    GPU simulation loaded from it; iter0 is a multiple of M (a cycle boundary,
    where the velocity sums restart)."""
    from preprocess_src_b200.step import Simulation
    case = sub_case(M, rk)
    c = oracle_mod.Oracle(case, init_fluid=False)
    for k in ("dn", "un", "vn", "wn", "dm", "um", "vm", "wm", "fx", "fy", "fz", "x", "y", "z", "u", "v", "w",
              "cfx", "cfy", "cfz", "xd", "nd", "volume0", "gx"):
        c.a[k][:] = o.a[k]
    c.fn[:] = o.fn
    c.iter = iter0
    sim = Simulation(case)
    sim.import_lattice(c.fn)
    sim.import_cells(x=c["x"], y=c["y"], z=c["z"], xd=c["xd"], nd=c["nd"], volume0=c["volume0"], gx=c["gx"])
    sim.iter = iter0
    return case, c, sim


@pytest.mark.parametrize("M,rk", [(2, 2), (3, 1), (2, 4)])
def test_subcycled_steps_match_oracle(developed, oracle_mod, M, rk):
    case, c, sim = start(oracle_mod, developed, M, rk)
    m = case.bc == configs.COMP
    x0 = np.concatenate([c["x"], c["y"], c["z"]])
    xlast = None   # the GPU's positions after the last step of the previous cycle
    for s in range(1, 2 * M + 1):
        c.step(1)
        sim.step(1)
        out = sim.export_lattice(fn=False)
        got = sim.export_cells()
        uref = np.concatenate([c["um"][m], c["vm"][m], c["wm"][m]])
        umine = np.concatenate([out["un"][m], out["vn"][m], out["wn"][m]])
        uerr = rel_l2(umine, uref)
        derr = np.abs(out["dn"][m] - c["dm"][m]).max()
        ref = np.concatenate([c["x"], c["y"], c["z"]])
        mine = np.concatenate([got["x"], got["y"], got["z"]])
        perr = np.abs(mine - ref).max()
        moved = np.abs(ref - x0).max()
        print(f"M={M} RK{rk} step {s}: u rel L2 {uerr:.3e}  max|d rho| {derr:.3e}  max|dx| {perr:.3e}"
              f"  (moved {moved:.2e})")
        assert uerr <= 8e-7 * s
        assert derr <= 6e-7 * s
        assert perr <= 1e-9 * s * s
        if s % M and xlast is not None:   # inside a cycle the cells stay where the last cycle left them
            assert np.array_equal(mine, xlast)
        if s % M == 0:
            xlast = mine
    assert sim.iter == c.iter
    assert np.abs(np.concatenate([c["x"], c["y"], c["z"]]) - x0).max() > 0   # the cells did move
    sim.close()


def test_calls_ending_inside_a_cycle_equal_one_call(developed, oracle_mod):
    """rbc_step(h, 1) five times against rbc_step(h, 5) with M = 3: the force
    of a cycle survives the end of a call, bit for bit."""
    _, _, a = start(oracle_mod, developed, 3, 2)
    _, _, b = start(oracle_mod, developed, 3, 2)
    a.step(5)
    for _ in range(5):
        b.step(1)
    ea, eb = a.export_lattice(fn=True), b.export_lattice(fn=True)
    for k in ("fn", "dn", "un", "vn", "wn"):
        np.testing.assert_array_equal(ea[k], eb[k], err_msg=k)
    ca, cb = a.export_cells(), b.export_cells()
    for k in ("x", "y", "z", "xd", "fx", "fy", "fz"):
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    a.close(); b.close()


def test_stage_calls_equal_subcycled_steps(developed, oracle_mod):
    """One cycle of M = 2 through the stage entry points as main.cu:78-106
    calls them (rbc_stress and rbc_ibm_st1 at the first step, rbc_ibm_st2 and
    rbc_volume_correction at the last) against rbc_step(h, 2)."""
    _, _, a = start(oracle_mod, developed, 2, 4)
    _, _, b = start(oracle_mod, developed, 2, 4)
    a.step(2)
    b.iter = b.iter + 1
    b.stress(); b.ibm_st1(); b.lbm_d3q19()
    b.iter = b.iter + 1
    b.lbm_d3q19(); b.ibm_st2(); b.volume_correction()
    ea, eb = a.export_lattice(fn=True), b.export_lattice(fn=True)
    for k in ("fn", "dn", "un", "vn", "wn"):
        np.testing.assert_array_equal(ea[k], eb[k], err_msg=k)
    ca, cb = a.export_cells(), b.export_cells()
    for k in ("x", "y", "z", "xd"):
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    a.close(); b.close()


def test_subcycled_simulations_do_not_batch(native_lib):
    from preprocess_src_b200 import _native as N
    from preprocess_src_b200.step import Batch, Simulation
    sims = [Simulation(sub_case(2, 4))]
    with pytest.raises(N.RbcError) as e:
        Batch(sims)
    assert e.value.code == N.RBC_ERR_UNSUPPORTED
    sims[0].close()
