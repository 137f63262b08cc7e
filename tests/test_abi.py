"""The C ABI library without a GPU: it loads, exports every declared entry
point, and validates arguments before touching a device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from preprocess_src_b200 import _native as N
from preprocess_src_b200 import configs

HEADER = Path(__file__).resolve().parents[1] / "include" / "rbc_step.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(rbc_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding():
    assert declared_functions() == sorted(N.EXPORTED)


def test_library_exports_every_declared_symbol(native_lib):
    for name in declared_functions():
        assert hasattr(native_lib, name), name


def _create(case, **over):
    p = dict(case.params)
    p.update(over)
    ps = N.params_struct(p)
    tri = np.ascontiguousarray(case.tri, dtype=np.int32).reshape(-1)
    xr = np.ascontiguousarray(case.xr, dtype=np.float64)
    m = N.RbcMesh(case.ncell, case.vertex, case.element, tri.ctypes.data_as(N._IP), xr.ctypes.data_as(N._DP))
    bc = np.ascontiguousarray(case.bc, dtype=np.int32)
    h = N._H()
    rc = N.lib().rbc_create(C.byref(ps), C.byref(m), bc.ctypes.data_as(N._IP), C.byref(h))
    msg = N.lib().rbc_last_error(None).decode()
    if rc == 0:
        N.lib().rbc_destroy(h)
    return rc, msg


def _cuda_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_rejects_unsupported_options(native_lib):
    case = configs.small_duct()
    assert _create(case, M=0)[0] == N.RBC_ERR_ARG
    assert _create(case, rk_order=3)[0] == N.RBC_ERR_ARG
    # the reference's RUNGE_KUTTA 1 / 2 branches drop dx and dt (ibm.cu:522-562)
    rc, msg = _create(case, rk_order=2, dx=0.5)
    assert rc == N.RBC_ERR_UNSUPPORTED and "dx = dt = 1" in msg
    assert _create(case, M=2, vof_k=10)[0] == N.RBC_ERR_UNSUPPORTED
    assert _create(case, br=float("inf"))[0] == N.RBC_ERR_ARG
    assert _create(case, tau=0.5)[0] == N.RBC_ERR_ARG
    assert _create(case, storage=7)[0] == N.RBC_ERR_ARG
    assert _create(case, bend_spont=2)[0] == N.RBC_ERR_ARG


def test_rejects_bad_bc(native_lib):
    case = configs.small_duct()
    bc = case.bc.copy().reshape(case.nz, case.ny, case.nx)
    bc[5, 5, 5] = configs.WALL          # an obstacle in one plane only: not z-invariant
    case.bc = bc.reshape(-1)
    rc, msg = _create(case)
    assert rc == N.RBC_ERR_UNSUPPORTED and "COMP plane" in msg
    case2 = configs.small_duct()
    bc2 = case2.bc.copy().reshape(case2.nz, case2.ny, case2.nx)
    bc2[0, 5, 5] = configs.COMP          # BUFF plane must hold BUFF over fluid
    case2.bc = bc2.reshape(-1)
    assert _create(case2)[0] == N.RBC_ERR_ARG


def test_rejects_broken_mesh(native_lib):
    case = configs.small_duct()
    case.tri = case.tri[:-1].copy()      # open surface
    case.element -= 1
    assert _create(case)[0] == N.RBC_ERR_TOPOLOGY


@pytest.mark.skipif(_cuda_present(), reason="checks the no-device path")
def test_no_device_is_reported(native_lib):
    rc, msg = _create(configs.small_duct())
    assert rc == N.RBC_ERR_NO_DEVICE, (rc, msg)


def test_simulation_fails_loudly_without_device(native_lib):
    if _cuda_present():
        pytest.skip("GPU present")
    from preprocess_src_b200.step import Simulation
    with pytest.raises(N.RbcError):
        Simulation(configs.small_duct())
