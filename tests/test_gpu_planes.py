"""The collide-stream kernel with several z planes per thread against one
plane per thread.

  * A z-periodic duct driven by a uniform body force from rest stays
    z-invariant under FP32 storage, so every plane of a long duct (two planes
    per thread) must equal, bit for bit, the planes of an 8-plane duct of the
    same cross-section (one plane per thread there): a wrong plane index, a
    skipped or repeated plane, or a wrong periodic neighbour plane breaks the
    equality.
  * On one lattice, every launch shape (1, 2, 4, 8 planes per thread, set by
    rbc_set_launch_shape) gives the same fields bit for bit, with FP32 and with
    FP16 storage (whose stochastic rounding draws its bits from the node index
    and the step, not from the thread).
"""
import numpy as np
import pytest

from preprocess_src_b200 import _native as N
from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def test_planes_per_thread_match_one_plane_per_thread(native_lib):
    from preprocess_src_b200.step import Simulation
    big = configs.duct_case("planes_130x128x128", 130, 128, 128, g=1e-4, storage=0)
    small = configs.duct_case("planes_8x128x128", 8, 128, 128, g=1e-4, storage=0)
    # internal nodes over planes per thread stay at or above 2^19 threads
    assert big.nx * big.ny * (big.nz - 4) >= (1 << 19) * 2
    with Simulation(big) as a, Simulation(small) as b:
        a.step(7)
        b.step(7)
        la, lb = a.export_lattice(fn=False), b.export_lattice(fn=False)
        for k in ("un", "vn", "wn", "dn"):
            fa = la[k].reshape(big.nz, big.ny, big.nx)[2:-2]
            fb = lb[k].reshape(small.nz, small.ny, small.nx)[2]
            assert np.array_equal(fa, np.broadcast_to(fb, fa.shape)), k
        assert np.abs(la["wn"]).max() > 1e-5   # the drive has moved the fluid


@pytest.mark.parametrize("storage", [0, 1])
def test_launch_shapes_give_identical_fields(native_lib, storage):
    """A suspension (cells, so IB forces reach the collision) on 66 planes: an
    odd plane count per thread leaves some threads fewer planes."""
    from preprocess_src_b200.step import Simulation
    case = configs.suspension_case("shapes_66x40x40", 66, 40, 40, 3, subdiv=2, radius=4.0, seed=9,
                                   g=4e-5, Gs=2e-3, storage=storage)
    ref = None
    for planes in (1, 2, 4, 8, 0):
        with Simulation(case) as s:
            s.set_launch_shape(N.RBC_SHAPE_LBM_PLANES, planes)
            assert s.launch_shape(N.RBC_SHAPE_LBM_PLANES) == planes
            s.step(3)
            s.set_launch_shape(N.RBC_SHAPE_LBM_PLANES, 1 if planes != 1 else 2)   # graphs rebuilt mid-run
            s.step(3)
            out = s.export_lattice(fn=True)
            cel = s.export_cells()
        if ref is None:
            ref = (out, cel)
            continue
        for k in ("fn", "dn", "un", "vn", "wn"):
            np.testing.assert_array_equal(out[k], ref[0][k], err_msg=f"{planes} {k}")
        for k in ("x", "y", "z"):
            np.testing.assert_array_equal(cel[k], ref[1][k], err_msg=f"{planes} {k}")


def test_launch_shape_refusals(native_lib):
    from preprocess_src_b200.step import Simulation
    with Simulation(configs.small_duct()) as s:
        for bad in (3, 16, -1):
            with pytest.raises(Exception):
                s.set_launch_shape(N.RBC_SHAPE_LBM_PLANES, bad)
        with pytest.raises(Exception):
            s.set_launch_shape(99, 1)
        assert s.launch_shape(N.RBC_SHAPE_LBM_PLANES) == 0
