"""Batches of independent simulations (rbc_batch_*) against the same
simulations stepped one by one.

Four capillaries of config 4 (uneven lengths, their own Gs and g) run as one
batch, in the fused form (one launch per stage over the blocks of all four)
and as child graphs; every simulation must end where it ends when stepped
alone, bit for bit (the kernels and the order of every sum are the same, and
the spread's lattice sums are integers).  A simulation stepped on its own
between batch steps changes its population buffer parity, which the batch
must notice.  The autotuner's launch shapes do not change the results."""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu


def _cases(**kw):
    return configs.capillary_batch(4, seed=7, lengths=(48, 64), **kw)


def _same(a, b):
    ea, eb = a.export_lattice(fn=True), b.export_lattice(fn=True)
    for k in ("fn", "dn", "un", "vn", "wn"):
        np.testing.assert_array_equal(ea[k], eb[k], err_msg=k)
    ca, cb = a.export_cells(), b.export_cells()
    for k in ("x", "y", "z", "xd", "fx", "fy", "fz"):
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert a.iter == b.iter
    assert a.cell_metrics()["volume"].tolist() == b.cell_metrics()["volume"].tolist()


@pytest.mark.parametrize("fused", [True, False])
def test_batch_equals_individual_steps(native_lib, fused):
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases()
    assert len({c.name.split("_")[1] for c in cases}) > 1, "lengths should differ"
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    batch.set_form(fused)
    assert batch.fused == fused and batch.obstacle() == ""
    n0 = batch.launches
    batch.step(3)
    for s in b:
        s.step(3)
    if fused:
        assert batch.launches - n0 == 3 * 7   # step begin, clear, membrane, spread, collide-stream, advect, volume
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


def test_fused_batch_with_fp16_storage(native_lib):
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases(storage=1)
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    assert batch.fused
    batch.step(4)
    for s in b:
        s.step(4)
    for x, y in zip(a, b):
        _same(x, y)
    batch.close()


def test_batch_autotune_advances_and_keeps_results(native_lib):
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases()
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    it0 = a[0].iter
    batch.autotune(1)
    tpb, planes, vpt = batch.shape
    assert tpb in (128, 256) and planes in (1, 2, 4) and vpt >= 1
    steps = a[0].iter - it0
    assert steps >= 2 and all(s.iter == a[0].iter for s in a)
    for s in b:
        s.step(steps)
    for x, y in zip(a, b):
        _same(x, y)
    # the child-graph form tunes its chain length
    batch.set_form(False)
    it0 = a[0].iter
    chain = batch.autotune(1)
    assert chain in (1, 2, 4) and batch.chain == chain
    for s in b:
        s.step(a[0].iter - it0)
    for x, y in zip(a, b):
        _same(x, y)
    batch.close()


def test_batch_falls_back_to_child_graphs(native_lib):
    """A simulation with bending (a stage the fused step leaves out) makes the
    batch use child graphs; it still equals the simulations stepped alone."""
    import dataclasses
    from preprocess_src_b200.step import Batch, Simulation
    cases = _cases()
    cases[2] = dataclasses.replace(cases[2], params=dict(cases[2].params, br=0.02))
    a = [Simulation(c) for c in cases]
    b = [Simulation(c) for c in cases]
    batch = Batch(a)
    assert not batch.fused and "bending" in batch.obstacle()
    batch.step(3)
    for s in b:
        s.step(3)
    for x, y in zip(a, b):
        _same(x, y)
    batch.close()
