"""The allocation-free metrics entry point against the handle-based one.

rbc_cell_metrics_noalloc serves callers that cannot allocate device memory
(a framework that owns the device memory pool, a loop that must not call the
allocator): it reads positions the caller already holds on the device and uses
a static device array as its only scratch.  Its volumes, areas and centroids
must equal rbc_cell_metrics' for the same cells, on repeated calls (the
scratch keeps the previous call's contents), on the calling thread's current
device and on a caller's stream, and in the shear mode with a cell across the
periodic x boundary.  This file is collected last so a failure here comes
after every other test has run.
"""
import numpy as np
import pytest

from preprocess_src_b200 import _native as N
from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def _xargs(case):
    """(LX, xmin, xmax): periodic x only in the shear mode."""
    p = case.params
    return (p["LX"], p["xmin"], p["xmax"]) if p["flow"] == 1 else (0.0, 0.0, 0.0)


def _call(X, tri, case, out, device=0, stream=None, ncell=None, vertex=None, LZ=None):
    L = N.lib()
    p = case.params
    return L.rbc_cell_metrics_noalloc(X.data_ptr(), case.ncell if ncell is None else ncell,
                                      case.vertex if vertex is None else vertex, case.element, tri.data_ptr(),
                                      *_xargs(case), p["LZ"] if LZ is None else LZ, p["zmin"], p["zmax"],
                                      device, stream,
                                      out["volume"].ctypes.data_as(N._DP), out["area"].ctypes.data_as(N._DP),
                                      out["centroid"].ctypes.data_as(N._DP))


def _empty(n):
    return {"volume": np.full(n, np.nan), "area": np.full(n, np.nan), "centroid": np.full(3 * n, np.nan)}


def _device_state(case, steps):
    import torch

    from preprocess_src_b200.step import Simulation
    sim = Simulation(case, device=0)
    sim.step(steps)
    ref = sim.cell_metrics()
    cells = sim.export_cells()
    sim.close()
    # device buffers owned by the caller (allocated here by the test, not by the call)
    X = torch.tensor(np.concatenate([cells["x"], cells["y"], cells["z"]]), dtype=torch.float64, device="cuda:0")
    tri = torch.tensor(case.tri.reshape(-1), dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    return ref, cells, X, tri


def _check(out, ref, what):
    assert np.allclose(out["volume"], ref["volume"], rtol=1e-12, atol=0), (what, out["volume"], ref["volume"])
    assert np.allclose(out["area"], ref["area"], rtol=1e-12, atol=0), what
    assert np.abs(out["centroid"] - ref["centroid"]).max() <= 1e-10, what


def test_noalloc_metrics_match_handle_metrics(native_lib):
    import torch
    # two cells, the first hanging across the periodic end so the z unwrap matters
    case = configs.duct_case("noalloc_32x20x20_2c", 32, 20, 20, centers_duct=[(0.5, 9.6, 9.4), (16.0, 9.3, 9.7)],
                             subdiv=3, radius=5.0, seed=7, g=4e-5, Gs=2e-3)
    ref, _, X, tri = _device_state(case, 6)
    for call in range(2):
        out = _empty(case.ncell)
        rc = _call(X, tri, case, out)
        assert rc == N.RBC_OK, N.lib().rbc_last_error(None)
        _check(out, ref, f"call {call}")
    # the calling thread's current device (-1) and a stream of the caller's
    torch.cuda.set_device(0)
    out = _empty(case.ncell)
    assert _call(X, tri, case, out, device=-1) == N.RBC_OK, N.lib().rbc_last_error(None)
    _check(out, ref, "device -1")
    s = torch.cuda.Stream(device=0)
    out = _empty(case.ncell)
    assert _call(X, tri, case, out, stream=s.cuda_stream) == N.RBC_OK, N.lib().rbc_last_error(None)
    _check(out, ref, "caller stream")
    assert torch.cuda.current_device() == 0


def test_noalloc_shear_cell_across_x_boundary(native_lib):
    """Shear mode (x periodic): a cell straddling x = xmin/xmax must be unwrapped
    along x as the handle's volume correction does (volume_correction.cu:319-325)."""
    case = configs.shear_case("noalloc_shear_24x20x24", 24, 20, 24, centers=[(11.2, 0.4, -3.1), (-2.0, -0.6, 6.3)],
                              sr=4e-3, walls=0, subdiv=3, radius=5.0, seed=5, Gs=2e-3)
    ref, cells, X, tri = _device_state(case, 4)
    LX = case.params["LX"]
    x0 = cells["x"][:case.vertex]
    assert np.ptp(x0) > LX / 2, "the first cell must lie across the x boundary"
    for call in range(2):
        out = _empty(case.ncell)
        rc = _call(X, tri, case, out)
        assert rc == N.RBC_OK, N.lib().rbc_last_error(None)
        _check(out, ref, f"shear call {call}")


def test_noalloc_rejects_bad_arguments(native_lib):
    import torch
    case = configs.small_duct()
    X = torch.zeros(3 * case.vertex, dtype=torch.float64, device="cuda:0")
    tri = torch.tensor(case.tri.reshape(-1), dtype=torch.int32, device="cuda:0")
    big = N.RBC_NOALLOC_MAX_CELLS + 1
    out = _empty(big)
    assert _call(X, tri, case, out, ncell=big) == N.RBC_ERR_ARG
    assert str(N.RBC_NOALLOC_MAX_CELLS) in N.lib().rbc_last_error(None).decode()
    out = _empty(1)
    assert _call(X, tri, case, out, vertex=N.RBC_NOALLOC_MAX_VERTEX + 1) == N.RBC_ERR_ARG
    assert "vertex" in N.lib().rbc_last_error(None).decode()
    assert _call(X, tri, case, out, LZ=0.0) == N.RBC_ERR_ARG
    assert "LZ" in N.lib().rbc_last_error(None).decode()


def test_noalloc_reports_out_of_range_connectivity(native_lib):
    """A triangle entry outside 0..vertex-1 is skipped (no out-of-range read)
    and the call returns RBC_ERR_ARG; the next call with valid input succeeds."""
    import torch
    case = configs.small_duct()
    ref, _, X, tri_ok = _device_state(case, 2)
    bad = case.tri.reshape(-1).copy()
    bad[7] = case.vertex + 3
    tri_bad = torch.tensor(bad, dtype=torch.int32, device="cuda:0")
    out = _empty(case.ncell)
    assert _call(X, tri_bad, case, out) == N.RBC_ERR_ARG
    assert "outside" in N.lib().rbc_last_error(None).decode()
    out = _empty(case.ncell)
    assert _call(X, tri_ok, case, out) == N.RBC_OK, N.lib().rbc_last_error(None)
    _check(out, ref, "after a refused call")
