"""The collide-stream kernel on lattices large enough for several z planes per
thread (two with FP32 storage, four with FP16 at >= 2^19 threads) against one
plane per thread.

A z-periodic duct driven by a uniform body force from rest stays z-invariant,
so every plane of a long duct must equal, bit for bit, the planes of an
8-plane duct of the same cross-section (one plane per thread there): a wrong
plane index, a skipped or repeated plane, or a wrong periodic neighbour plane
breaks the equality.
"""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", [0, 1])
def test_planes_per_thread_match_one_plane_per_thread(native_lib, storage):
    from preprocess_src_b200.step import Simulation
    big = configs.duct_case("planes_130x128x128", 130, 128, 128, g=1e-4, storage=storage)
    small = configs.duct_case("planes_8x128x128", 8, 128, 128, g=1e-4, storage=storage)
    # internal nodes over planes per thread stay at or above 2^19 threads
    assert big.nx * big.ny * (big.nz - 4) >= (1 << 19) * (4 if storage else 2)
    with Simulation(big) as a, Simulation(small) as b:
        a.step(7)
        b.step(7)
        la, lb = a.export_lattice(fn=False), b.export_lattice(fn=False)
        for k in ("un", "vn", "wn", "dn"):
            fa = la[k].reshape(big.nz, big.ny, big.nx)[2:-2]
            fb = lb[k].reshape(small.nz, small.ny, small.nx)[2]
            assert np.array_equal(fa, np.broadcast_to(fb, fa.shape)), k
        assert np.abs(la["wn"]).max() > 1e-5   # the drive has moved the fluid
