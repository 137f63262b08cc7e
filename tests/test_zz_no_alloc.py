"""The allocation-free metrics entry point against the handle-based one.

rbc_cell_metrics_noalloc serves callers that cannot allocate device memory
(a framework that owns the device memory pool, a loop that must not call the
allocator): it reads positions the caller already holds on the device and uses
a static device array as its only scratch.  Its volumes, areas and centroids
must equal rbc_cell_metrics' for the same cells, on repeated calls (the
scratch keeps the previous call's contents).  This file is collected last so a
failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from preprocess_src_b200 import _native as N
from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def _call(X, tri, case, out):
    L = N.lib()
    p = case.params
    return L.rbc_cell_metrics_noalloc(X.data_ptr(), case.ncell, case.vertex, case.element, tri.data_ptr(),
                                      p["LZ"], p["zmin"], p["zmax"], 0, None,
                                      out["volume"].ctypes.data_as(N._DP), out["area"].ctypes.data_as(N._DP),
                                      out["centroid"].ctypes.data_as(N._DP))


def test_noalloc_metrics_match_handle_metrics(native_lib):
    import torch

    from preprocess_src_b200.step import Simulation
    # two cells, the first hanging across the periodic end so the z unwrap matters
    case = configs.duct_case("noalloc_32x20x20_2c", 32, 20, 20, centers_duct=[(0.5, 9.6, 9.4), (16.0, 9.3, 9.7)],
                             subdiv=3, radius=5.0, seed=7, g=4e-5, Gs=2e-3)
    sim = Simulation(case, device=0)
    sim.step(6)
    ref = sim.cell_metrics()
    cells = sim.export_cells()
    # device buffers owned by the caller (allocated here by the test, not by the call)
    X = torch.tensor(np.concatenate([cells["x"], cells["y"], cells["z"]]), dtype=torch.float64, device="cuda:0")
    tri = torch.tensor(case.tri.reshape(-1), dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    for call in range(2):
        out = {"volume": np.full(case.ncell, np.nan), "area": np.full(case.ncell, np.nan),
               "centroid": np.full(3 * case.ncell, np.nan)}
        rc = _call(X, tri, case, out)
        assert rc == N.RBC_OK, N.lib().rbc_last_error(None)
        assert np.allclose(out["volume"], ref["volume"], rtol=1e-12, atol=0), (call, out["volume"], ref["volume"])
        assert np.allclose(out["area"], ref["area"], rtol=1e-12, atol=0), call
        assert np.abs(out["centroid"] - ref["centroid"]).max() <= 1e-10, call
    sim.close()


def test_noalloc_rejects_oversize(native_lib):
    import torch
    case = configs.small_duct()
    X = torch.zeros(3 * case.vertex, dtype=torch.float64, device="cuda:0")
    tri = torch.tensor(case.tri.reshape(-1), dtype=torch.int32, device="cuda:0")
    big = N.RBC_NOALLOC_MAX_CELLS + 1
    out = {"volume": np.zeros(big), "area": np.zeros(big), "centroid": np.zeros(3 * big)}
    p = case.params
    rc = N.lib().rbc_cell_metrics_noalloc(X.data_ptr(), big, case.vertex, case.element, tri.data_ptr(), p["LZ"],
                                          p["zmin"], p["zmax"], 0, None, out["volume"].ctypes.data_as(N._DP),
                                          out["area"].ctypes.data_as(N._DP), out["centroid"].ctypes.data_as(N._DP))
    assert rc == N.RBC_ERR_ARG
    assert str(N.RBC_NOALLOC_MAX_CELLS) in N.lib().rbc_last_error(None).decode()
