"""Host side of the adjoint workload: the FP64 reference-gradient fixture and
the loss used by the autograd wrapper (no GPU)."""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "c5_fp64_gradient.npz"


def test_c5_fixture_central_differences_are_converged():
    fx = np.load(GOLD)
    np.testing.assert_allclose(fx["grad_h1e3"], fx["grad_h1e4"], rtol=1e-6)
    assert int(fx["nsteps"]) == 2000
    np.testing.assert_array_equal(fx["base"], [5e-4, 100.0, 1e-6])
    np.testing.assert_array_equal(fx["target_params"], [7e-4, 100.0, 1.2e-6])


def test_c5_fixture_final_shape_is_reproduced_by_the_oracle(oracle_mod):
    """The fixture's final positions at the base parameters come from the
    oracle: one 2000-step FP64 run reproduces them."""
    import sys
    sys.path.insert(0, str(GOLD.parent))
    from make_c5_gradient import BASE, final_positions, shape_loss
    from preprocess_src_b200 import configs
    fx = np.load(GOLD)
    x = final_positions(BASE)
    np.testing.assert_allclose(x, fx["final"], rtol=0, atol=1e-10)
    p = configs.single_cell_duct().params
    assert abs(shape_loss(x, fx["target"], p["LX"], p["LZ"]) - float(fx["loss"])) <= 1e-12


def test_shape_loss_takes_the_minimum_image():
    torch = pytest.importorskip("torch")
    from preprocess_src_b200.adjoint import shape_loss
    t = torch.zeros(3, 4, dtype=torch.float64)
    x = t.clone()
    x[0, 0] = 60.0 - 0.5   # across the periodic x boundary of LX = 60: distance 0.5
    x[2, 1] = -0.25 + 64.0  # across z (LZ = 64): distance 0.25
    x[1, 2] = 0.5           # y is not periodic
    L = shape_loss(x, t, 60.0, 64.0)
    assert abs(float(L) - (0.25 + 0.0625 + 0.25) / 4) < 1e-15


def _plan(units, snaps):
    import ctypes as C

    from preprocess_src_b200 import _native as N
    L = N.lib()
    n = C.c_int(0)
    assert L.rbc_adjoint_binomial_plan(units, snaps, None, None, 0, C.byref(n)) == N.RBC_OK
    ops = (C.c_int * n.value)()
    args = (C.c_int * n.value)()
    assert L.rbc_adjoint_binomial_plan(units, snaps, ops, args, n.value, C.byref(n)) == N.RBC_OK
    assert L.rbc_adjoint_binomial_plan(units, snaps, ops, args, n.value - 1, C.byref(n)) == N.RBC_ERR_ARG
    return list(zip(ops, args))


def _binomial(s, r):
    from math import comb
    return comb(s + r + 1, s + 1)


@pytest.mark.parametrize("units,snaps", [(1, 4), (2, 0), (7, 0), (20, 1), (20, 3), (2000, 16), (2000, 5),
                                         (255, 6), (100, 200)])
def test_binomial_schedule_reverses_every_unit_once(native_lib, units, snaps):
    """Simulate the schedule of rbc_adjoint_record_binomial: every unit is
    recorded from its own state and reversed right after, in order from the
    last to the first; a restore reads a slot that holds a state; at most
    snaps + 1 slots are used; no unit is advanced more than r times, r the
    least with C(snaps + r + 1, snaps + 1) >= units."""
    plan = _plan(units, snaps)
    s_eff = min(snaps, units - 1)
    r = 0
    while _binomial(s_eff, r) < units:
        r += 1
    pos, slots, reversed_, advanced = None, {}, [], [0] * units
    last_recorded = None
    for op, arg in plan:
        if op == 1:      # keep the current state in slot arg
            if pos is None:
                pos = 0
            assert 0 <= arg <= s_eff
            slots[arg] = pos
        elif op == 2:    # restore
            assert arg in slots
            pos = slots[arg]
        elif op == 0:    # advance
            assert arg >= 1 and pos + arg < units
            for t in range(pos, pos + arg):
                advanced[t] += 1
            pos += arg
        elif op == 3:    # record unit arg from the state at arg
            assert pos == arg and last_recorded is None
            last_recorded = arg
            pos = arg + 1
        else:            # reverse the unit just recorded
            assert arg == last_recorded
            reversed_.append(arg)
            last_recorded = None
    assert reversed_ == list(range(units - 1, -1, -1))
    assert max(advanced) <= r, (max(advanced), r)
