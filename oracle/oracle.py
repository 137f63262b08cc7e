"""ctypes binding of the FP64 CPU oracle (oracle/rbc_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker.  Used by tests/, by
``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg, never by the
product library.  ``Oracle`` holds the reference-layout state in numpy arrays
and steps it with the restated reference algorithm.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "librbc_oracle.so"

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


class OrcParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("dt", C.c_double),
                ("tau", C.c_double), ("Cr", C.c_double), ("P", C.c_double), ("B", C.c_double),
                ("flowstart", C.c_int), ("freq", C.c_double), ("C", C.c_double), ("rgs", C.c_double),
                ("law", C.c_int), ("residual", C.c_double), ("itrmax", C.c_int), ("LX", C.c_double),
                ("LZ", C.c_double), ("xmin", C.c_double), ("xmax", C.c_double), ("zmin", C.c_double),
                ("zmax", C.c_double), ("ncell", C.c_int), ("vertex", C.c_int), ("element", C.c_int),
                ("mn", C.c_int), ("br", C.c_double), ("flow", C.c_int), ("sr", C.c_double), ("walls", C.c_int),
                ("tube_r", C.c_double), ("lambda1", C.c_double), ("vof_k", C.c_int),
                ("vof_residual", C.c_double), ("vof_itrmax", C.c_int), ("M", C.c_int), ("rk_order", C.c_int)]


_STATE_D = ["fn", "fm", "dn", "un", "vn", "wn", "dm", "um", "vm", "wm", "fx", "fy", "fz"]
_STATE_CELL_D = ["x", "y", "z", "u", "v", "w", "cfx", "cfy", "cfz", "xd", "nd", "t", "rg", "qd"]


class OrcState(C.Structure):
    _fields_ = ([(k, _DP) for k in _STATE_D] + [("bc", _IP)] + [(k, _DP) for k in _STATE_CELL_D]
                + [("ele", _IP), ("nln", _IP), ("ln", _IP), ("lo", _IP), ("nle", _IP), ("le", _IP),
                   ("volume0", _DP), ("gx", _DP), ("iter", C.c_int), ("bicg_iters", C.c_int), ("ec", _IP),
                   ("crg", _DP), ("cbr", _DP), ("c0", _DP), ("s0", _DP), ("vf", _DP), ("vof_iters", C.c_int)])


_lib = None


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < max((HERE / f).stat().st_mtime for f in ("rbc_oracle.c", "rbc_oracle.h")):
        subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(build()))
        for name in ("orc_fem_init", "orc_stress", "orc_calc_load", "orc_volume_correction", "orc_step",
                     "orc_front_tracking"):
            getattr(L, name).restype = C.c_int
        for name in ("orc_flu_init", "orc_volume_init", "orc_ibm_st1", "orc_lbm_d3q19", "orc_ibm_st2",
                     "orc_calc_tension", "orc_q2f", "orc_bend", "orc_bend_reference", "orc_thinc_wlic"):
            getattr(L, name).restype = None
        L.orc_num_threads.restype = C.c_int
        L.orc_calc_volume.restype = None
        _lib = L
    return _lib


def expand2pow2(n: int) -> int:
    """etc.cu:425-446"""
    cnt = 0
    while n > 1:
        if n % 2 == 1:
            n += 1
        n //= 2
        cnt += 1
    return 2 ** cnt


class Oracle:
    """Reference-layout FP64 state of one case, stepped on the CPU."""

    def __init__(self, case, init_fluid=True, cell_rgs=None, cell_br=None, bend_spont=None):
        """cell_rgs, cell_br: optional [ncell] per-cell tension normalisation and
        bending modulus (cells of a second population on the same mesh).
        bend_spont (default: case.params["bend_spont"]): bending about the
        spontaneous angles of the initial shape instead of 0."""
        self.case = case
        p = case.params
        self.N, self.V, self.E = case.ncell, case.vertex, case.element
        nv, ne = max(self.N * self.V, 1), max(self.N * self.E, 1)
        self.mn = expand2pow2(3 * self.V) if self.N else 256
        self.p = OrcParams(nx=p["nx"], ny=p["ny"], nz=p["nz"], dx=p["dx"], dt=p["dt"], tau=p["tau"], Cr=p["Cr"],
                           P=p["P"], B=p["B"], flowstart=p["flowstart"], freq=p["freq"], C=p["C"], rgs=p["rgs"],
                           law=p["law"], residual=p["residual"], itrmax=p["itrmax"], LX=p["LX"], LZ=p["LZ"],
                           xmin=p["xmin"], xmax=p["xmax"], zmin=p["zmin"], zmax=p["zmax"], ncell=self.N,
                           vertex=self.V, element=self.E, mn=self.mn, br=float(p.get("br", 0.0)),
                           flow=int(p.get("flow", 0)), sr=float(p.get("sr", 0.0)), walls=int(p.get("walls", 0)),
                           tube_r=float(p.get("tube_r", 0.0)), lambda1=float(p.get("lambda1", 1.0)),
                           vof_k=int(p.get("vof_k", 0)), vof_residual=float(p.get("vof_residual", 1e-10)),
                           vof_itrmax=int(p.get("vof_itrmax", 20000)), M=int(p.get("M", 1)),
                           rk_order=int(p.get("rk_order", 4)))
        n = case.n
        self.a = {}
        for k in _STATE_D:
            self.a[k] = np.zeros(n * 19 if k in ("fn", "fm") else n)
        self.a["bc"] = np.ascontiguousarray(case.bc, dtype=np.int32)
        sizes = dict(x=nv, y=nv, z=nv, u=nv, v=nv, w=nv, cfx=nv, cfy=nv, cfz=nv, xd=3 * nv, nd=4 * ne, t=4 * ne,
                     rg=ne, qd=max(self.N, 1) * self.mn)
        for k, s in sizes.items():
            self.a[k] = np.zeros(s)
        self.a["ele"] = case.ele_global() if self.N else np.zeros(3, np.int32)
        for k, s in dict(nln=nv, ln=7 * nv, lo=7 * nv, nle=nv, le=6 * nv).items():
            self.a[k] = np.zeros(s, dtype=np.int32)
        self.a["ec"] = np.zeros(3 * ne, dtype=np.int32)
        self.a["volume0"] = np.zeros(max(self.N, 1))
        self.a["gx"] = np.zeros(3 * max(self.N, 1))
        self.a["vf"] = np.zeros(n)
        for k, v in (("crg", cell_rgs), ("cbr", cell_br)):
            if v is not None:
                self.a[k] = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
                if self.a[k].size != self.N:
                    raise ValueError(f"{k}: one value per cell")
        self.s = OrcState()
        for k, arr in self.a.items():
            setattr(self.s, k, arr.ctypes.data_as(_IP if arr.dtype == np.int32 else _DP))
        self.s.iter = 0
        L = lib()
        if init_fluid:
            L.orc_flu_init(C.byref(self.p), C.byref(self.s))
        if self.N:
            xr = np.asarray(case.xr, dtype=np.float64)
            self.a["xd"][:] = xr
            self.a["x"][:] = xr[0::3]
            self.a["y"][:] = xr[1::3]
            self.a["z"][:] = xr[2::3]
            rc = L.orc_fem_init(C.byref(self.p), C.byref(self.s))
            if rc != 0:
                raise RuntimeError(f"oracle fem_init failed with error({rc})")
            L.orc_volume_init(C.byref(self.p), C.byref(self.s))
            if bend_spont is None:
                bend_spont = bool(p.get("bend_spont", 0))
            if bend_spont:
                self.a["c0"] = np.zeros(3 * ne)
                self.a["s0"] = np.zeros(3 * ne)
                self.s.c0 = self.a["c0"].ctypes.data_as(_DP)
                self.s.s0 = self.a["s0"].ctypes.data_as(_DP)
                L.orc_bend_reference(C.byref(self.p), C.byref(self.s))
            if self.p.vof_k > 0 and init_fluid:   # vof_init (init1.cu:1094-1120, main.cu:56)
                if L.orc_front_tracking(C.byref(self.p), C.byref(self.s)) < 0:
                    raise RuntimeError("oracle front tracking did not converge")

    # the population buffers swap like ltc->fnD / ltc->fmD (lbm.cu:1575)
    @property
    def fn(self) -> np.ndarray:
        a, b = self.a["fn"], self.a["fm"]
        return a if C.cast(self.s.fn, C.c_void_p).value == a.ctypes.data else b

    @property
    def fm(self) -> np.ndarray:
        a, b = self.a["fn"], self.a["fm"]
        return b if C.cast(self.s.fn, C.c_void_p).value == a.ctypes.data else a

    def __getitem__(self, k):
        if k == "fn":
            return self.fn
        return self.a[k]

    @property
    def iter(self) -> int:
        return self.s.iter

    @iter.setter
    def iter(self, v: int):
        self.s.iter = int(v)

    def _c(self, name):
        return getattr(lib(), name)(C.byref(self.p), C.byref(self.s))

    def stress(self) -> int:
        return self._c("orc_stress")

    def ibm_st1(self):
        self._c("orc_ibm_st1")

    def lbm_d3q19(self):
        self._c("orc_lbm_d3q19")

    def ibm_st2(self):
        self._c("orc_ibm_st2")

    def volume_correction(self) -> int:
        return self._c("orc_volume_correction")

    def calc_tension(self):
        self._c("orc_calc_tension")

    def thinc_wlic(self):
        self._c("orc_thinc_wlic")

    def front_tracking(self) -> int:
        return self._c("orc_front_tracking")

    def step(self, n: int = 1) -> int:
        rc = lib().orc_step(C.byref(self.p), C.byref(self.s), int(n))
        if rc != 0:
            raise RuntimeError(f"oracle step failed with code {rc}")
        return rc

    def volumes(self):
        vol, area = np.zeros(self.N), np.zeros(self.N)
        lib().orc_calc_volume(C.byref(self.p), C.byref(self.s), vol.ctypes.data_as(_DP), area.ctypes.data_as(_DP))
        return vol, area

    def set_fn(self, fn):
        self.fn[:] = fn


def num_threads() -> int:
    return lib().orc_num_threads()
