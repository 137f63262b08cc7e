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
