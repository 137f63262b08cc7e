"""The reference-layout lattice import (rbc_import_ref_lattice) on a duct long
enough that its copy pipeline reuses every slot of its ring: 201 planes of
64 x 48 nodes are 6 chunks of at most 35 planes (16 MiB each) through 4 slots,
the last chunk partial.  Import followed by export returns the populations of
every COMP node (the two conversions are inverse pulls), with FP32 and FP16
population storage; the same lattice stepped once from the import matches the
FP64 oracle stepped from the same populations."""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def long_duct(storage=0):
    return configs.duct_case("import_ring_201x64x48", 201, 64, 48, g=4e-5, storage=storage)


def random_lattice(case, seed):
    rng = np.random.default_rng(seed)
    fn = np.tile(W, case.n) + rng.uniform(-1e-3, 1e-3, case.n * 19)
    return fn


@pytest.mark.parametrize("storage,tol", [(0, 1e-9), (1, 1e-6)])
def test_import_export_roundtrip_long_duct(native_lib, storage, tol):
    from preprocess_src_b200.step import Simulation
    case = long_duct(storage)
    assert case.params["nz"] - 4 == 201
    fn = random_lattice(case, 5)
    sim = Simulation(case)
    sim.import_lattice(fn)
    out = sim.export_lattice(fn=True, macro=False)["fn"]
    m = np.repeat(case.bc == configs.COMP, 19)
    err = np.abs(out[m] - fn[m]).max()
    print(f"storage {storage}: max |d fn| {err:.3e}")
    assert err <= tol, err
    # a second import into the same handle (the ring and its events reused)
    fn2 = random_lattice(case, 6)
    sim.import_lattice(fn2)
    out2 = sim.export_lattice(fn=True, macro=False)["fn"]
    assert np.abs(out2[m] - fn2[m]).max() <= tol
    sim.close()


def test_step_after_long_import_matches_oracle(native_lib, oracle_mod):
    from preprocess_src_b200.step import Simulation
    case = long_duct()
    fn = random_lattice(case, 7)
    o = oracle_mod.Oracle(case)
    o.fn[:] = fn
    o.step(1)
    sim = Simulation(case)
    sim.import_lattice(fn)
    sim.step(1)
    got = sim.export_lattice(fn=True, macro=True)
    m = case.bc == configs.COMP
    err_f = np.abs(got["fn"][np.repeat(m, 19)] - o.fn[np.repeat(m, 19)]).max()
    err_u = np.abs(got["wn"][m] - o["wn"][m]).max()
    print(f"one step from the import: max |d fn| {err_f:.3e}, max |d w| {err_u:.3e}")
    assert err_f <= 5e-9 and err_u <= 1e-8, (err_f, err_u)   # measured 8.4e-10, 1.5e-9
    sim.close()
