"""The FP64 oracle against golden vectors from the reference's own kernels.

Fixtures in tests/golden/*.npz were produced by tests/golden/make_golden.py,
which runs the reference's step modules (compiled unmodified from the
reference sources with oracle/ref_harness) on a GPU from the inputs that
golden_cases() regenerates here.  FP64 against FP64: the only differences are
summation order (tree reductions, thrust) and the BiCGSTAB stopping point.
"""
from pathlib import Path

import numpy as np
import pytest

from tests.golden.make_golden import cell_coefficients, golden_cases, snapshots
from preprocess_src_b200 import configs

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fixtures():
    return [(name, case) for name, case in golden_cases().items() if (GOLDEN / f"{name}.npz").exists()]


@pytest.mark.parametrize("name,case", fixtures() or [pytest.param(None, None, marks=pytest.mark.skip("no fixtures"))])
def test_oracle_matches_reference_kernels(name, case, oracle_mod):
    g = np.load(GOLDEN / f"{name}.npz")
    if "wbc" in case.meta:   # red and white cells: one oracle run with per-cell coefficients
        rgs, br = cell_coefficients(case)
        o = oracle_mod.Oracle(case, cell_rgs=rgs, cell_br=br)
    else:
        o = oracle_mod.Oracle(case)
    assert np.abs(o["nd"] - g["setup_nd"]).max() <= 1e-12 * np.abs(g["setup_nd"]).max()
    assert np.allclose(o["volume0"], g["setup_volume0"], rtol=1e-13)
    assert np.allclose(o["gx"], g["setup_gx"], rtol=0, atol=1e-12)
    m = case.bc == configs.COMP
    vof = case.params["vof_k"] > 0
    # with the volume fraction, THINC/WLIC rounds through the float expf/coshf
    # (thincwlic.cu:193-198), whose last bit differs between glibc and CUDA:
    # ~1e-8 per node and step in vf, and through omega in the flow
    utol = 1e-7 if vof else 1e-9
    loose = 1e3 if vof else 1.0   # the same through the flow into the cells
    if vof:
        print(f"setup vf max|d| {np.abs(o['vf'][m] - g['setup_vf']).max():.2e}")
        assert np.abs(o["vf"][m] - g["setup_vf"]).max() <= 1e-9
    done = 0
    for s in snapshots(case):
        o.step(s - done)
        done = s
        u = np.concatenate([o["un"][m], o["vn"][m], o["wn"][m]])
        uref = np.concatenate([g[f"s{s}_un"], g[f"s{s}_vn"], g[f"s{s}_wn"]])
        if vof:
            print(f"step {s}: vf max|d| {np.abs(o['vf'][m] - g[f's{s}_vf']).max():.2e}  u rel {rel(u, uref):.2e}")
            assert np.abs(o["vf"][m] - g[f"s{s}_vf"]).max() <= 1e-6
        assert rel(u, uref) <= utol, (s, rel(u, uref))
        assert np.abs(o["dn"][m] - g[f"s{s}_dn"]).max() <= 1e-12 * loose
        if f"s{s}_um" in g:   # sub-cycled: the sums of the cycle (averaged velocity at its end)
            um = np.concatenate([o["um"][m], o["vm"][m], o["wm"][m]])
            umref = np.concatenate([g[f"s{s}_um"], g[f"s{s}_vm"], g[f"s{s}_wm"]])
            assert rel(um, umref) <= utol, (s, rel(um, umref))
            assert np.abs(o["dm"][m] - g[f"s{s}_dm"]).max() <= 1e-12 * case.params["M"]
        x = np.concatenate([o[k] for k in ("x", "y", "z")])
        xref = np.concatenate([g[f"s{s}_{k}"] for k in ("x", "y", "z")])
        assert np.abs(x - xref).max() <= 1e-12 * loose * np.abs(xref).max(), (s, np.abs(x - xref).max())
        assert np.abs(o["u"] - g[f"s{s}_u"]).max() <= 1e-12 * loose
        # at step 1 the cells are still at their stress-free shape and the
        # forces are round-off (~1e-13), hence the absolute floor
        f = np.concatenate([o[k] for k in ("cfx", "cfy", "cfz")])
        fref = np.concatenate([g[f"s{s}_{k}"] for k in ("fx", "fy", "fz")])
        assert np.abs(f - fref).max() <= 1e-8 * loose * np.abs(fref).max() + 1e-12, (s, np.abs(f - fref).max())
        assert np.abs(o["gx"] - g[f"s{s}_gx"]).max() <= 1e-10 * loose
