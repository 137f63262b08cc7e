"""Adjoint of the step (rbc_adjoint_record / rbc_adjoint_backward) against
central finite differences of the forward step on the GPU.

The case is a small duct with one subdivision-2 cell whose initial shape is
stretched by 3 % along x and shrunk by the same factor along y (volume kept,
so the correction starts converged) to give the membrane forces something to
act on from the first step.  L = sum r . X_final with a fixed random r is
linear in the final positions, so the differences measure only the step's
own nonlinearity.  The forward computes in FP32, so each difference step is
chosen large enough that FP32 round-off of the perturbed runs stays below
the tolerance and small enough that the truncation error of central
differences does too: relative 1e-2 for the coefficients over one or two
steps (where the response is small and nearly linear), 1e-3 over 24 steps,
and 1e-3 lattice units for the positions."""
import numpy as np
import pytest

from preprocess_src_b200 import configs

pytestmark = pytest.mark.gpu

REL_TOL = 2e-3   # adjoint vs central differences, relative to the derivative


def _case():
    return configs.small_duct(subdiv=2, radius=5.0, flow=32, width=20, g=2e-5, Gs=5e-3)


def _stretched(case):
    x = case.xr.reshape(-1, 3).T.copy()   # [3, nv]
    c = x.mean(axis=1, keepdims=True)
    s = np.array([1.03, 1.0 / 1.03, 1.0])[:, None]
    return c + s * (x - c)


class _Run:
    def __init__(self, sim, x0, nsteps, ckpt):
        from preprocess_src_b200.adjoint import InitialState
        self.sim, self.x0, self.nsteps, self.ckpt = sim, x0, nsteps, ckpt
        self.init = InitialState(sim)
        self.theta0 = dict(P=sim.params["P"], B=sim.params["B"], C_=sim.params["C"])
        rng = np.random.default_rng(11)
        self.r = rng.standard_normal((3, sim.nv))

    def loss(self, x0=None, **coef):
        th = dict(self.theta0)
        th.update(coef)
        self.sim.set_coefficients(**th)
        self.init.restore(self.sim, self.x0 if x0 is None else x0)
        self.sim.step(self.nsteps)
        c = self.sim.export_cells()
        return float((self.r * np.stack([c["x"], c["y"], c["z"]])).sum())

    def adjoint(self, want_x0=False):
        self.sim.set_coefficients(**self.theta0)
        self.init.restore(self.sim, self.x0)
        self.sim.adjoint_record(self.nsteps, self.ckpt)
        return self.sim.adjoint_backward(self.r[0], self.r[1], self.r[2], want_x0=want_x0)


@pytest.mark.parametrize("nsteps,ckpt", [(1, 1), (2, 1), (24, 7)])
def test_parameter_gradients_match_central_differences(native_lib, nsteps, ckpt):
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        run = _Run(sim, _stretched(case), nsteps, ckpt)
        adj = run.adjoint()
        assert adj["flags"] == 0
        got = dict(zip(("P", "B", "C_"), adj["grad"]))
        for k, v0 in run.theta0.items():
            h = (1e-2 if nsteps <= 2 else 1e-3) * abs(v0)
            fd = (run.loss(**{k: v0 + h}) - run.loss(**{k: v0 - h})) / (2 * h)
            print(f"nsteps={nsteps} d/d{k}: adjoint {got[k]:.9e}  central {fd:.9e}  rel {abs(got[k] - fd) / abs(fd):.2e}")
            assert abs(got[k] - fd) <= REL_TOL * abs(fd), (k, got[k], fd)


@pytest.mark.parametrize("nsteps,ckpt", [(1, 1), (2, 1), (24, 7)])
def test_initial_position_gradient_matches_directional_difference(native_lib, nsteps, ckpt):
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        x0 = _stretched(case)
        run = _Run(sim, x0, nsteps, ckpt)
        adj = run.adjoint(want_x0=True)
        rng = np.random.default_rng(5)
        d = rng.standard_normal(x0.shape)
        eps = 1e-3
        fd = (run.loss(x0=x0 + eps * d) - run.loss(x0=x0 - eps * d)) / (2 * eps)
        got = float((adj["dx0"] * d).sum())
        print(f"nsteps={nsteps} dL/dx0 . d: adjoint {got:.9e}  central {fd:.9e}  rel {abs(got - fd) / abs(fd):.2e}")
        assert abs(got - fd) <= REL_TOL * abs(fd)


def test_checkpoint_interval_does_not_change_the_gradient(native_lib):
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        run = _Run(sim, _stretched(case), 12, 1)
        g = {}
        for ckpt in (1, 5, 12):
            run.ckpt = ckpt
            g[ckpt] = run.adjoint(want_x0=True)
        # equal up to the order of the forward's FP32 atomics (about 1e-6 relative)
        for ckpt in (5, 12):
            np.testing.assert_allclose(g[ckpt]["grad"], g[1]["grad"], rtol=2e-5)
            np.testing.assert_allclose(g[ckpt]["dx0"], g[1]["dx0"], rtol=0, atol=2e-5 * np.abs(g[1]["dx0"]).max())


def test_backward_leaves_the_end_state_and_repeats(native_lib):
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        run = _Run(sim, _stretched(case), 10, 4)
        a1 = run.adjoint()
        end = sim.export_cells()
        it = sim.iter
        a2 = sim.adjoint_backward(run.r[0], run.r[1], run.r[2])
        after = sim.export_cells()
        assert sim.iter == it
        for k in ("x", "y", "z", "xd"):
            np.testing.assert_array_equal(after[k], end[k])
        np.testing.assert_allclose(a2["grad"], a1["grad"], rtol=2e-5)   # FP32 atomics order
        assert a1["ms"] > 0.0


def test_shape_run_autograd_matches_the_c_abi(native_lib):
    import torch
    from preprocess_src_b200.adjoint import InitialState, ShapeRun, shape_loss
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        p = sim.params
        init = InitialState(sim)
        theta = torch.tensor([2 * p["B"], p["C"], 2 * p["P"]], dtype=torch.float64, requires_grad=True)
        with torch.no_grad():
            target = ShapeRun.apply(theta * torch.tensor([1.4, 1.0, 1.2], dtype=torch.float64), None, sim, init, 8, 3)
        x = ShapeRun.apply(theta, None, sim, init, 8, 3)
        L = shape_loss(x, target, p["LX"], p["LZ"])
        L.backward()
        seed = (2.0 / sim.nv) * (x.detach() - target).numpy()
        r = sim.adjoint_backward(seed[0], seed[1], seed[2])
        dP, dB, dC = r["grad"]
        np.testing.assert_allclose(theta.grad.numpy(), [dB / 2, dC, dP / 2], rtol=2e-5)   # FP32 atomics order
        assert float(L.detach()) > 0.0


def test_adjoint_rejects_unsupported_and_out_of_order(native_lib):
    from preprocess_src_b200 import _native as N
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case, storage=1) as sim:
        with pytest.raises(RuntimeError, match="FP32"):
            sim.adjoint_record(2, 1)
    with Simulation(case) as sim:
        with pytest.raises(RuntimeError, match="before rbc_adjoint_record"):
            sim.adjoint_backward(np.zeros(sim.nv), np.zeros(sim.nv), np.zeros(sim.nv))
    assert N.RBC_ERR_UNSUPPORTED == 3


def test_c5_shape_gradient_against_differences_and_fp64_reference(native_lib):
    """The adjoint workload: single-cell duct, 2000 steps, checkpoints every
    100 steps, L = mean |X - target|^2 with the target shape of a run at
    Gs = 7e-4, g = 1.2e-6; gradient with respect to (Gs, C, g) at (5e-4, 100,
    1e-6) against central differences of the FP32 forward (relative step
    1e-3) and against central differences of the FP64 oracle (fixture made by
    tests/golden/make_c5_gradient.py, same target positions).  The FP64
    differences are converged (steps 1e-3 and 1e-4 agree to 3e-7), and the
    adjoint must match them to 1e-4.  Differences of the FP32 forward carry
    its round-off (about 1e-3 of the derivative at this step size), so they
    are held to 3e-3."""
    import time
    from pathlib import Path

    import torch
    from preprocess_src_b200.adjoint import InitialState, ShapeRun, shape_loss
    from preprocess_src_b200.step import Simulation
    fx = np.load(Path(__file__).resolve().parent / "golden" / "c5_fp64_gradient.npz")
    nsteps = int(fx["nsteps"])
    case = configs.single_cell_duct()
    with Simulation(case) as sim:
        p = sim.params
        init = InitialState(sim)
        target = torch.from_numpy(fx["target"])

        def loss_at(th):
            with torch.no_grad():
                x = ShapeRun.apply(torch.tensor(th, dtype=torch.float64), None, sim, init, nsteps, 100)
            return float(shape_loss(x, target, p["LX"], p["LZ"]))

        theta = torch.tensor(fx["base"], dtype=torch.float64, requires_grad=True)
        t0 = time.perf_counter()
        x = ShapeRun.apply(theta, None, sim, init, nsteps, 100)
        t1 = time.perf_counter()
        L = shape_loss(x, target, p["LX"], p["LZ"])
        L.backward()
        t2 = time.perf_counter()
        assert abs(float(L.detach()) - float(fx["loss"])) <= 1e-3 * float(fx["loss"])
        adj = theta.grad.numpy()
        fd = np.zeros(3)
        for k in range(3):
            up, dn = fx["base"].copy(), fx["base"].copy()
            h = 1e-3 * abs(fx["base"][k])
            up[k] += h
            dn[k] -= h
            fd[k] = (loss_at(up) - loss_at(dn)) / (2 * h)
        ref = fx["grad_h1e3"]
        print(f"\nloss {float(L.detach()):.9e} (FP64 oracle {float(fx['loss']):.9e}); record {t1 - t0:.3f} s, backward {t2 - t1:.3f} s")
        for k, name in enumerate(("Gs", "C", "g")):
            print(f"dL/d{name}: adjoint {adj[k]:.9e}  FP32 central {fd[k]:.9e} (rel {abs(adj[k] - fd[k]) / abs(fd[k]):.2e})"
                  f"  FP64 oracle central {ref[k]:.9e} (rel {abs(adj[k] - ref[k]) / abs(ref[k]):.2e})"
                  f"  oracle h=1e-4 {fx['grad_h1e4'][k]:.9e}")
        np.testing.assert_allclose(adj, ref, rtol=1e-4)
        np.testing.assert_allclose(adj, fd, rtol=3e-3)


@pytest.mark.parametrize("unit,snaps", [(1, 3), (1, 0), (4, 2), (5, 1)])
def test_binomial_checkpointing_equals_fixed_interval(native_lib, unit, snaps):
    """rbc_adjoint_record_binomial (units of `unit` steps, `snaps` slots)
    against a checkpoint every step: the same recomputed states (the forward
    is bitwise repeatable), so the gradients agree up to the order of the
    reverse sweep's FP32 atomics."""
    from preprocess_src_b200.step import Simulation
    case = _case()
    with Simulation(case) as sim:
        run = _Run(sim, _stretched(case), 23, 1)
        ref = run.adjoint(want_x0=True)
        sim.set_coefficients(**run.theta0)
        run.init.restore(sim, run.x0)
        sim.adjoint_record_binomial(23, unit, snaps)
        end = sim.export_cells()
        sch = sim.adjoint_schedule()
        got = sim.adjoint_backward(run.r[0], run.r[1], run.r[2], want_x0=True)
        after = sim.export_cells()
        print(f"unit {unit} snaps {snaps}: {sch}, grad {got['grad']} vs {ref['grad']}")
        assert sch["units"] == -(-23 // unit) and sch["snapshots"] == min(snaps, sch["units"] - 1) + 1
        np.testing.assert_allclose(got["grad"], ref["grad"], rtol=2e-5)
        np.testing.assert_allclose(got["dx0"], ref["dx0"], rtol=0, atol=2e-5 * np.abs(ref["dx0"]).max())
        for k in ("x", "y", "z", "xd"):   # the handle is left at the end of the run
            np.testing.assert_array_equal(after[k], end[k])


def test_binomial_checkpointing_on_the_dense_suspension(native_lib):
    """The adjoint at the dense suspension's size (256 x 128 x 128, 200 cells):
    binomial checkpointing with units of one step and two snapshot slots
    (memory independent of the run length) against a checkpoint every 12
    steps (a store of 24 steps, 11.5 GB), over 12 steps."""
    from preprocess_src_b200.step import Simulation
    case = configs.dense_suspension()
    nsteps = 12
    with Simulation(case) as sim:
        run = _Run(sim, None, nsteps, nsteps)
        ref = run.adjoint()
        sim.set_coefficients(**run.theta0)
        run.init.restore(sim)
        sim.adjoint_record_binomial(nsteps, 1, 2)
        got = sim.adjoint_backward(run.r[0], run.r[1], run.r[2])
        print(f"dense: binomial {got['grad']} ({got['ms']:.1f} ms) vs fixed {ref['grad']} ({ref['ms']:.1f} ms)")
        scale = np.abs(ref["grad"]).max()
        assert scale > 0
        np.testing.assert_allclose(got["grad"], ref["grad"], rtol=0, atol=2e-5 * scale)
        assert got["flags"] == 0
