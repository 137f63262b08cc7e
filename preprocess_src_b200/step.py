"""Python mirror of the reference's step modules over the C ABI.

``Simulation`` owns one device handle.  Its methods carry the names of the
reference entry points they replace and run in the same order inside
``step()`` (main.cu:73-110 with M = 1):

    stress()            stress.cu:580       membrane FEM nodal forces
    ibm_st1()           ibm.cu:299          spread forces to the lattice
    lbm_d3q19()         lbm.cu:1463         collide + stream
    ibm_st2()           ibm.cu:642          interpolate + RK4 advect
    thinc_wlic()        thincwlic.cu:316    advect the volume fraction (vof_k > 0)
    front_tracking()    fronttrack.cu:628   volume fraction from the cells (every vof_k steps)
    volume_correction() volume_correction.cu:453

State moves in and out in the reference's layouts (``import_*``/``export_*``).
All compute runs in the CUDA library; nothing here computes physics.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .configs import Case


def _dp(a):
    return None if a is None else a.ctypes.data_as(N._DP)


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class Simulation:
    def __init__(self, case: Case, **overrides):
        L = N.lib()
        self.case = case
        params = dict(case.params)
        params.update(overrides)
        self.params = params
        self._p = N.params_struct(params)
        self._bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        self._tri = np.ascontiguousarray(case.tri, dtype=np.int32).reshape(-1)
        self._xr = np.ascontiguousarray(case.xr, dtype=np.float64)
        m = None
        if case.ncell > 0:
            m = N.RbcMesh(case.ncell, case.vertex, case.element, self._tri.ctypes.data_as(N._IP),
                          self._xr.ctypes.data_as(N._DP))
        h = N._H()
        N.check(L.rbc_create(C.byref(self._p), C.byref(m) if m is not None else None,
                             self._bc.ctypes.data_as(N._IP), C.byref(h)))
        self._h = h
        self.n = case.n
        self.nv = case.ncell * case.vertex
        self.ne = case.ncell * case.element

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            N.lib().rbc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        N.check(getattr(N.lib(), name)(self._h, *args), self._h)

    # -- the step (reference entry-point names) -----------------------------
    def stress(self):
        self._call("rbc_stress")

    def ibm_st1(self):
        self._call("rbc_ibm_st1")

    def lbm_d3q19(self):
        self._call("rbc_lbm_d3q19")

    def ibm_st2(self):
        self._call("rbc_ibm_st2")

    def volume_correction(self) -> int:
        it = C.c_int(0)
        self._call("rbc_volume_correction", C.byref(it))
        return it.value

    def thinc_wlic(self):
        self._call("rbc_thinc_wlic")

    def front_tracking(self) -> int:
        """Solver sweeps of the red cells' solve (-1: not converged)."""
        it = C.c_int(0)
        self._call("rbc_front_tracking", C.byref(it))
        return it.value

    def step(self, nsteps: int = 1):
        self._call("rbc_step", int(nsteps))

    @property
    def iter(self) -> int:
        v = C.c_int(0)
        self._call("rbc_get_iter", C.byref(v))
        return v.value

    @iter.setter
    def iter(self, value: int):
        self._call("rbc_set_iter", int(value))

    # -- state in / out ------------------------------------------------------
    def import_lattice(self, fn):
        self._call("rbc_import_ref_lattice", _dp(_f64(fn, self.n * 19)))

    def export_lattice(self, fn=True, macro=True) -> dict:
        out = {}
        if fn:
            out["fn"] = np.empty(self.n * 19)
        if macro:
            for k in ("dn", "un", "vn", "wn"):
                out[k] = np.empty(self.n)
        self._call("rbc_export_ref_lattice", _dp(out.get("fn")), _dp(out.get("dn")), _dp(out.get("un")),
                   _dp(out.get("vn")), _dp(out.get("wn")))
        return out

    def export_vof(self) -> tuple[np.ndarray, np.ndarray]:
        """ltc->vf, ltc->vf2 in the reference layout."""
        vf, vf2 = np.empty(self.n), np.empty(self.n)
        self._call("rbc_export_ref_vof", _dp(vf), _dp(vf2))
        return vf, vf2

    def import_vof(self, vf=None, vf2=None):
        args = [None if a is None else _f64(a, self.n) for a in (vf, vf2)]
        self._call("rbc_import_ref_vof", *map(_dp, args))

    def export_force(self) -> dict:
        out = {k: np.empty(self.n) for k in ("fx", "fy", "fz")}
        self._call("rbc_export_ref_force", _dp(out["fx"]), _dp(out["fy"]), _dp(out["fz"]))
        return out

    def import_cells(self, x=None, y=None, z=None, xd=None, nd=None, volume0=None, gx=None):
        nv, ne, nc = self.nv, self.ne, self.case.ncell
        args = [None if a is None else _f64(a, n)
                for a, n in ((x, nv), (y, nv), (z, nv), (xd, 3 * nv), (nd, 4 * ne), (volume0, nc), (gx, 3 * nc))]
        self._keep = args
        self._call("rbc_import_ref_cells", *map(_dp, args))

    def import_vertex_force(self, fx, fy, fz):
        nv = self.nv
        args = [_f64(fx, nv), _f64(fy, nv), _f64(fz, nv)]
        self._call("rbc_import_ref_vertex_force", *map(_dp, args))

    def export_cells(self) -> dict:
        nv, nc = self.nv, self.case.ncell
        keys = ("x", "y", "z", "xd", "u", "v", "w", "fx", "fy", "fz", "gx")
        sizes = (nv, nv, nv, 3 * nv, nv, nv, nv, nv, nv, nv, 3 * nc)
        out = {k: np.empty(s) for k, s in zip(keys, sizes)}
        self._call("rbc_export_ref_cells", *[_dp(out[k]) for k in keys])
        return out

    # -- white cells (init3.cu) --------------------------------------------------
    def add_wbc(self, wbc: Case, rgs: float = 1.0, br: float = 0.0):
        """A second cell population (cel->*_w): wbc's mesh (tri, xr, ncell,
        vertex, element; its lattice is ignored), tension normalisation rgs =
        GSw / GS and bending modulus br = BRw."""
        self._tri_w = np.ascontiguousarray(wbc.tri, dtype=np.int32).reshape(-1)
        self._xr_w = np.ascontiguousarray(wbc.xr, dtype=np.float64)
        m = N.RbcMesh(wbc.ncell, wbc.vertex, wbc.element, self._tri_w.ctypes.data_as(N._IP),
                      self._xr_w.ctypes.data_as(N._DP))
        self._call("rbc_add_wbc", C.byref(m), C.c_double(rgs), C.c_double(br))
        self.wbc = wbc
        self.nv_w = wbc.ncell * wbc.vertex
        self.ne_w = wbc.ncell * wbc.element

    def wbc_dims(self) -> tuple[int, int, int]:
        n, v, e = C.c_int(0), C.c_int(0), C.c_int(0)
        self._call("rbc_wbc_dims", C.byref(n), C.byref(v), C.byref(e))
        return n.value, v.value, e.value

    def import_wbc(self, x=None, y=None, z=None, xd=None, nd=None, volume0=None, gx=None):
        nv, ne, nc = self.nv_w, self.ne_w, self.wbc.ncell
        args = [None if a is None else _f64(a, n)
                for a, n in ((x, nv), (y, nv), (z, nv), (xd, 3 * nv), (nd, 4 * ne), (volume0, nc), (gx, 3 * nc))]
        self._keep = args
        self._call("rbc_import_ref_wbc", *map(_dp, args))

    def export_wbc(self) -> dict:
        nv, nc = self.nv_w, self.wbc.ncell
        keys = ("x", "y", "z", "xd", "u", "v", "w", "fx", "fy", "fz", "gx")
        sizes = (nv, nv, nv, 3 * nv, nv, nv, nv, nv, nv, nv, 3 * nc)
        out = {k: np.empty(s) for k, s in zip(keys, sizes)}
        self._call("rbc_export_ref_wbc", *[_dp(out[k]) for k in keys])
        return out

    def wbc_metrics(self) -> dict:
        nc = self.wbc.ncell
        out = {"volume": np.empty(nc), "area": np.empty(nc), "centroid": np.empty(3 * nc)}
        self._call("rbc_wbc_metrics", _dp(out["volume"]), _dp(out["area"]), _dp(out["centroid"]))
        return out

    # -- files in the reference's formats (etc.cu) -------------------------------
    def set_output_interval(self, fileoutput: int):
        """FILEOUTPUT: average fem->qi and fem->tp over intervals of this many steps."""
        self._call("rbc_set_output_interval", int(fileoutput))

    def write_restart(self, path, fnum: int = 0):
        self._call("rbc_write_restart", str(path).encode(), int(fnum))

    def read_restart(self, path) -> int:
        """Returns the file's fnum."""
        f = C.c_int(0)
        self._call("rbc_read_restart", str(path).encode(), C.byref(f))
        return f.value

    def write_cell_file(self, path):
        self._call("rbc_write_cell_file", str(path).encode())

    def write_prof_file(self, path):
        self._call("rbc_write_prof_file", str(path).encode())

    def write_center_file(self, path):
        self._call("rbc_write_center_file", str(path).encode())

    def read_center_file(self, path):
        self._call("rbc_read_center_file", str(path).encode())

    # -- adjoint ----------------------------------------------------------------
    def set_coefficients(self, P=None, B=None, C_=None):
        """Replace the drive P, IB-force B and area-dilation C coefficients."""
        P = self.params["P"] if P is None else float(P)
        B = self.params["B"] if B is None else float(B)
        C_ = self.params["C"] if C_ is None else float(C_)
        self._call("rbc_set_coefficients", C.c_double(P), C.c_double(B), C.c_double(C_))
        self.params.update(P=P, B=B, C=C_)

    def adjoint_record(self, nsteps: int, ckpt_every: int = 100):
        """Run nsteps steps keeping a checkpoint every ckpt_every steps."""
        self._call("rbc_adjoint_record", int(nsteps), int(ckpt_every))

    def adjoint_record_binomial(self, nsteps: int, unit: int = 1, snapshots: int = 16):
        """Run nsteps steps for a reverse sweep under binomial checkpointing:
        units of `unit` steps, `snapshots` snapshot slots beside the initial
        state."""
        self._call("rbc_adjoint_record_binomial", int(nsteps), int(unit), int(snapshots))

    def adjoint_schedule(self) -> dict:
        """The recorded run's schedule: units, steps per unit, snapshot slots
        (the initial state's included) and units advanced without recording in
        one backward sweep (binomial schedule; 0 for the fixed interval)."""
        u, k, sn, adv = C.c_int(0), C.c_int(0), C.c_int(0), C.c_longlong(0)
        self._call("rbc_adjoint_schedule", C.byref(u), C.byref(k), C.byref(sn), C.byref(adv))
        return {"units": u.value, "unit_steps": k.value, "snapshots": sn.value, "advanced_units": adv.value}

    def adjoint_backward(self, xbar, ybar, zbar, want_x0: bool = False) -> dict:
        """Reverse sweep of the recorded run from dL/d(final cel->x, y, z).
        Returns grad (dL/dP, dL/dB, dL/dC), flags, ms and, with want_x0,
        dx0 [3, nv] = dL/d(initial positions)."""
        nv = self.nv
        seeds = [_f64(a, nv) for a in (xbar, ybar, zbar)]
        grad = np.zeros(3)
        x0 = np.zeros((3, nv)) if want_x0 else None
        flags = C.c_int(0)
        ms = C.c_float(0.0)
        outs = [_dp(x0[k]) for k in range(3)] if want_x0 else [None, None, None]
        self._call("rbc_adjoint_backward", *[_dp(s) for s in seeds], _dp(grad), *outs, C.byref(flags), C.byref(ms))
        r = dict(grad=grad, flags=flags.value, ms=ms.value)
        if want_x0:
            r["dx0"] = x0
        return r

    # -- launch shapes (speed only; results do not depend on them) -------------
    def set_launch_shape(self, what: int, value: int):
        self._call("rbc_set_launch_shape", int(what), int(value))

    def launch_shape(self, what: int) -> int:
        v = C.c_int(0)
        self._call("rbc_get_launch_shape", int(what), C.byref(v))
        return v.value

    # -- diagnostics ----------------------------------------------------------
    def status(self) -> tuple[int, int]:
        f, v = C.c_int(0), C.c_int(0)
        self._call("rbc_get_status", C.byref(f), C.byref(v))
        return f.value, v.value

    def cell_metrics(self) -> dict:
        nc = self.case.ncell
        out = {"volume": np.empty(nc), "area": np.empty(nc), "centroid": np.empty(3 * nc)}
        self._call("rbc_cell_metrics", _dp(out["volume"]), _dp(out["area"]), _dp(out["centroid"]))
        return out

    def cell_metrics_async(self, out: np.ndarray) -> None:
        """Enqueue the copies of the metrics into out (5 * ncell float64:
        volume, area, centroid x, y, z); valid after synchronize()."""
        assert out.dtype == np.float64 and out.size >= 5 * self.case.ncell and out.flags["C_CONTIGUOUS"]
        self._call("rbc_cell_metrics_async", _dp(out))

    def profile_steps(self, nsteps: int) -> dict:
        """Run nsteps with a CUDA event around each kernel; returns the summed
        device milliseconds per kernel."""
        ms = np.zeros(N.RBC_NUM_KERNELS)
        self._call("rbc_profile_steps", int(nsteps), _dp(ms))
        return dict(zip(N.RBC_KERNEL_NAMES, ms.tolist()))

    @property
    def stream(self) -> int:
        v = C.c_void_p()
        self._call("rbc_get_stream", C.byref(v))
        return v.value or 0

    def synchronize(self):
        self._call("rbc_synchronize")

    @property
    def launches(self) -> int:
        v = C.c_longlong(0)
        self._call("rbc_launch_count", C.byref(v))
        return v.value


class Batch:
    """Independent simulations stepped together (rbc_batch_*): every batch step
    is one CUDA graph launch -- in the fused form seven launches, one per stage,
    each over the blocks of all simulations; otherwise the simulations' whole
    steps as child graphs.  The simulations stay usable on their own between
    batch steps."""

    def __init__(self, sims):
        self.sims = list(sims)   # the handles must outlive the batch
        arr = (N._H * len(self.sims))(*[s._h.value for s in self.sims])
        b = N._H()
        code = N.lib().rbc_batch_create(arr, len(self.sims), C.byref(b))
        if code != N.RBC_OK:
            msg = N.lib().rbc_batch_last_error(None)
            raise N.RbcError(code, msg.decode() if msg else "")
        self._b = b

    def _call(self, name, *args):
        code = getattr(N.lib(), name)(self._b, *args)
        if code != N.RBC_OK:
            msg = N.lib().rbc_batch_last_error(self._b)
            raise N.RbcError(code, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_b", None):
            N.lib().rbc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps: int = 1):
        self._call("rbc_batch_step", int(nsteps))

    def synchronize(self):
        self._call("rbc_batch_synchronize")

    @property
    def stream(self) -> int:
        v = C.c_void_p()
        self._call("rbc_batch_get_stream", C.byref(v))
        return v.value or 0

    @property
    def chain(self) -> int:
        v = C.c_int(0)
        self._call("rbc_batch_get_chain", C.byref(v))
        return v.value

    @chain.setter
    def chain(self, value: int):
        self._call("rbc_batch_set_chain", int(value))

    def autotune(self, steps_per_trial: int = 3) -> int:
        """Picks the fastest launch shapes (fused form) or chain length (child
        graphs); the timed steps advance every simulation.  Returns the chain."""
        v = C.c_int(0)
        self._call("rbc_batch_autotune", int(steps_per_trial), C.byref(v))
        return v.value

    @property
    def fused(self) -> bool:
        """Whether the next step uses the fused form."""
        v = C.c_int(0)
        self._call("rbc_batch_get_form", C.byref(v), None)
        return bool(v.value)

    def obstacle(self) -> str:
        """Why the simulations cannot run in the fused form ("" if they can)."""
        v, msg = C.c_int(0), C.c_char_p()
        self._call("rbc_batch_get_form", C.byref(v), C.byref(msg))
        return (msg.value or b"").decode()

    def set_form(self, fused: bool):
        self._call("rbc_batch_set_form", 1 if fused else 0)

    @property
    def shape(self) -> tuple[int, int, int]:
        """(collide-stream threads per block, z planes per thread, membrane
        vertices per thread) of the fused form; 0 = automatic."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        self._call("rbc_batch_get_shape", C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def set_shape(self, lbm_threads: int = 256, lbm_planes: int = 0, membrane_vpt: int = 0):
        self._call("rbc_batch_set_shape", int(lbm_threads), int(lbm_planes), int(membrane_vpt))

    @property
    def launches(self) -> int:
        v = C.c_longlong(0)
        self._call("rbc_batch_launch_count", C.byref(v))
        return v.value

