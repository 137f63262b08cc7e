"""Batches of independent simulations (rbc_batch_*) against the same
simulations stepped one by one.

Four capillaries of config 4 (uneven lengths, their own Gs and g) run as one
batch; every simulation must end where it ends when stepped alone.  A
simulation stepped on its own between batch steps changes its population
buffer parity, which the batch must notice.  Tolerances are those of the
graph-vs-stage test in test_gpu_parity.py (the spread's global FP32 atomics
may add in a different order)."""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def _cases():
    return configs.capillary_batch(4, seed=7, lengths=(48, 64))


def _same(a, b):
    m = a.case.bc == configs.COMP
    ea, eb = a.export_lattice(fn=False), b.export_lattice(fn=False)
    assert np.abs(ea["wn"][m] - eb["wn"][m]).max() <= 1e-9
    assert np.abs(ea["un"][m] - eb["un"][m]).max() <= 1e-9
    ca, cb = a.export_cells(), b.export_cells()
    for k in ("x", "y", "z", "xd"):
        assert np.abs(ca[k] - cb[k]).max() <= 1e-10, k
    assert a.iter == b.iter


def test_batch_equals_individual_steps(native_lib):
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases()
    assert len({c.name.split("_")[1] for c in cases}) > 1, "lengths should differ"
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    batch.step(3)
    for s in b:
        s.step(3)
    for x, y in zip(a, b):
        _same(x, y)
    # one simulation stepped alone flips its buffer parity; the batch rebuilds its graphs
    a[1].step(1)
    b[1].step(1)
    batch.step(2)
    for s in b:
        s.step(2)
    for x, y in zip(a, b):
        _same(x, y)
        assert x.status() == y.status()
    batch.close()


def test_batch_autotune_advances_and_keeps_results(native_lib):
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases()
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    it0 = a[0].iter
    chain = batch.autotune(1)
    assert chain in (1, 2, 4) and batch.chain == chain
    steps = a[0].iter - it0
    assert steps >= 2 and all(s.iter == a[0].iter for s in a)
    for s in b:
        s.step(steps)
    for x, y in zip(a, b):
        _same(x, y)
    batch.close()
