#!/usr/bin/env python
"""Benchmark of the coupled fluid-membrane step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dense|single] [--storage f32|f16]

Workload (default): the 256 x 128 x 128 duct with 200 subdivision-4 red cells
(4,064,256 fluid nodes, 512,400 vertices).  A step is one full coupled step
(membrane forces, spreading, collide-stream, RK4 advection, volume correction).

value   device-timed MLUPS (fluid-node updates per second) of K steps with the
        state resident in HBM, CUDA events on the library's stream, barrier and
        synchronize on both sides, max over ranks.  The lattice (0.65 GB) is
        larger than L2, so no flush is needed between steps.
e2e     the same metric through the public C ABI with host buffers: import of
        the reference-layout FP64 state from pinned memory, K steps each
        followed by a device->host copy of the per-cell volume/area/centroid
        (the host reads each step's copy while the next step runs), and a final
        export of the vertex positions, all inside the timed region.
roofline  the collide-stream kernel's algorithmic bytes (180 B/LU in FP32,
        104 B/LU in FP16) over its average launch time, from CUDA events around
        each kernel in profiled steps on the same stream, against the measured
        HBM copy bandwidth.
With N > 1 each rank runs an independent replica (weak scaling): the step has no
cross-rank exchange, so no collective is on the data path.
--impl reference times the FP64 CPU oracle (the reference has no CPU
implementation of the step) on the host cores, rank 0 only.
"""
import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS + membrane vertices/s at stated FP64 error; FP16/batched vs plain FP32, 1 B200"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dense", choices=["dense", "single", "capillaries", "adjoint", "vof"],
                    help="dense: config 2 (the headline); single: config 1; capillaries: config 4 "
                         "(512 uneven capillaries as one batch vs one after another); vof: the dense suspension "
                         "with the cells' volume fraction tracked (front tracking every --vof-k steps) and "
                         "viscosity ratio LAMBDA1 = 5")
    ap.add_argument("--vof-k", type=int, default=100, help="front-tracking interval K (vof workload)")
    ap.add_argument("--br", type=float, default=0.0, help="bending modulus BR (dense and single workloads)")
    ap.add_argument("--capillaries", type=int, default=512, help="number of capillaries (capillaries workload)")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16"])
    ap.add_argument("--adjoint-steps", type=int, default=2000, help="steps of the recorded run (adjoint workload)")
    ap.add_argument("--ckpt", type=int, default=100, help="checkpoint interval (adjoint workload)")
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def make_case(workload, seed_offset=0, storage="f32", vof_k=100, br=0.0):
    from preprocess_src_b200 import configs
    st = 1 if storage == "f16" else 0
    if workload == "single":
        return configs.single_cell_duct(seed=1 + seed_offset, storage=st, br=br)
    if workload == "vof":
        return configs.dense_suspension(seed=2 + seed_offset, storage=st, lambda1=5.0, vof_k=vof_k,
                                        vof_residual=1e-10)
    return configs.dense_suspension(seed=2 + seed_offset, storage=st, br=br)


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(workload, storage):
    """Per-launch DRAM bytes of the collide-stream kernel from the committed
    ncu summary (line 'traffic_bytes_per_launch[<workload>/<storage>]: N')."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"traffic_bytes_per_launch\[{workload}/{storage}\]:\s*([0-9.eE+]+)", f.read_text())
        if m:
            return float(m.group(1))
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(case, budget_s, warm=1, keep=None):
    """FP64 CPU oracle on the same workload: whole steps until the budget.
    keep: a list that receives the oracle (for the FP64 error of the step)."""
    from oracle.oracle import Oracle, num_threads
    o = Oracle(case)
    o.step(warm)
    t0 = time.perf_counter()
    n = 0
    while True:
        o.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    if keep is not None:
        keep.append(o)
    fl = case.fluid_nodes()
    return {"value": fl * n / el / 1e6, "unit": "MLUPS", "cores": num_threads(), "kind": "port",
            "sample": f"{n} full FP64 oracle steps of {case.name} after {warm} warm-up step(s), {el:.1f} s"}


def fp64_error(case, o, dev):
    """The error the metric is stated at: a fresh simulation of the workload
    stepped as many steps as the FP64 oracle o (pinned to the reference's own
    kernels), from the same initial state, against it."""
    import numpy as np
    from preprocess_src_b200 import configs
    from preprocess_src_b200.step import Simulation
    sim = Simulation(case, device=dev)
    sim.step(o.iter)
    lat = sim.export_lattice(fn=False)
    cel = sim.export_cells()
    sim.close()
    m = case.bc == configs.COMP
    u = np.concatenate([lat[k][m] for k in ("un", "vn", "wn")])
    uref = np.concatenate([o[k][m] for k in ("un", "vn", "wn")])
    x = np.concatenate([cel[k] for k in ("x", "y", "z")])
    xref = np.concatenate([o[k] for k in ("x", "y", "z")])
    return {"steps": int(o.iter), "velocity_rel_l2": float(np.linalg.norm(u - uref) / np.linalg.norm(uref)),
            "density_max_abs": float(np.abs(lat["dn"][m] - o["dn"][m]).max()),
            "position_max_abs": float(np.abs(x - xref).max()),
            "against": "the FP64 CPU oracle (pinned to the reference's kernels by the golden tests), "
                       "same initial state, same number of steps"}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from preprocess_src_b200.step import Simulation

    case = make_case(args.workload, seed_offset=rank, storage=args.storage, vof_k=args.vof_k, br=args.br)
    dev = local
    sim = Simulation(case, device=dev)
    fluid, nv = case.fluid_nodes(), case.ncell * case.vertex
    stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", dev))
    torch.cuda.set_device(dev)

    sim.step(args.warmup)
    sim.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    l0 = sim.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        time.sleep(0.3)
        ev0.record(stream)
        sim.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = sim.launches - l0
    ms_max = allreduce_max(ms, world)
    flags, vcmax = sim.status()

    # per-kernel device times (profiled steps, events around each kernel)
    kern = sim.profile_steps(args.profile_steps)
    if args.workload != "vof":
        kern.pop("vof", None)   # no volume fraction: its slot holds only the gap between two events
    lbm_ms = kern["lbm_collide_stream"] / args.profile_steps
    bytes_lu = 104 if args.storage == "f16" else 180
    achieved = bytes_lu * fluid / (lbm_ms * 1e-3) / 1e9
    peak, peak_kind = measured_hbm()
    traffic = ncu_traffic(args.workload, args.storage)

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, case, dev, world)

    result = None
    if rank == 0:
        value = world * fluid * args.steps / (ms_max * 1e-3) / 1e6
        step_total = sum(kern.values()) / args.profile_steps
        result = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
            "config": {"workload": case.name, "lattice_duct": f"{case.meta['flow']}x{case.meta['Ly']}x{case.meta['Lz']}",
                       "fluid_nodes": fluid, "cells": case.ncell, "vertices_per_cell": case.vertex,
                       "population_storage": args.storage, "positions": "f64", "volume_correction": "f64",
                       "l2": "inputs larger than L2 (populations 2 x %.2f GB), no flush" % (19 * (4 if args.storage == 'f32' else 2) * case.nx * case.ny * (case.nz - 4) / 1e9),
                       "parallelism": f"replicas x{world}" if world > 1 else "single"},
            "vertices_per_s": round(world * nv * args.steps / (ms_max * 1e-3), 1),
            "gpu_launches": launches,
            "kernel_ms_per_step": {k: round(v / args.profile_steps, 5) for k, v in kern.items()},
            "kernel_sum_ms_per_step": round(step_total, 5),
            "roofline": {"bound": "hbm", "kernel": "lbm_collide_stream", "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "bytes_per_lu": bytes_lu, "lus_per_launch": fluid,
                         "traffic": traffic},
            "status_flags": flags, "vc_iters_max": vcmax,
            "clocks": clk.summary(),
        }
        if args.workload == "vof":
            result["config"].update(lambda1=case.params["lambda1"], vof_k=case.params["vof_k"],
                                    vof_residual=case.params["vof_residual"])
        if args.br:
            result["config"]["bending_br"] = args.br
        if e2e:
            result["e2e"] = e2e
        if world == 1 and not args.no_cpu and args.workload != "vof":
            keep = []
            result["cpu_baseline"] = cpu_sample(case, args.cpu_seconds, keep=keep)
            result["fp64_error"] = fp64_error(case, keep[0], dev)
    sim.close()
    return result


def run_capillaries(args, world, rank, local):
    """Config 4: independent capillaries of uneven length stepped as one batch
    (one CUDA graph launch per step of seven fused launches, one per stage over
    all capillaries, launch shapes from the autotuner) against the same
    capillaries stepped one after another.  value = aggregate MLUPS of
    the batch; the sequential arm is the sum of each capillary's own
    event-timed steps."""
    import torch

    from preprocess_src_b200 import configs
    from preprocess_src_b200.step import Batch, Simulation

    dev = local
    torch.cuda.set_device(dev)
    cases = configs.capillary_batch(args.capillaries, seed=4 + 1000 * rank)
    sims = [Simulation(c, device=dev) for c in cases]
    fluid = sum(c.fluid_nodes() for c in cases)
    batch = Batch(sims)
    chain = batch.autotune(2)
    fused, shape = batch.fused, batch.shape
    batch.step(args.warmup)
    batch.synchronize()
    bstream = torch.cuda.ExternalStream(batch.stream, device=torch.device("cuda", dev))
    barrier(world)
    l0 = batch.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        time.sleep(0.3)
        ev0.record(bstream)
        batch.step(args.steps)
        ev1.record(bstream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = batch.launches - l0
    ms_max = allreduce_max(ms, world)
    flags = [s.status()[0] for s in sims]
    # the same capillaries one after another, each timed on its own stream
    seq_ms = 0.0
    for s in sims:
        st = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", dev))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.step(args.steps)
        b.record(st)
        b.synchronize()
        seq_ms += a.elapsed_time(b)
    batch.close()
    for s in sims:
        s.close()
    if rank != 0:
        return None
    value = world * fluid * args.steps / (ms_max * 1e-3) / 1e6
    seq = fluid * args.steps / (seq_ms * 1e-3) / 1e6
    return {"metric": "aggregate MLUPS, %d uneven capillaries in one batch (config 4)" % len(cases),
            "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "capillary_batch_%d_32x32xL" % len(cases), "capillaries": len(cases),
                       "fluid_nodes": fluid, "lengths": "uniform {48, 64, ..., 128}", "cells_per_capillary": 1,
                       "vertices_per_cell": cases[0].vertex,
                       "form": "fused: one launch per stage over all capillaries" if fused else
                               "child graphs (chain %d)" % chain,
                       "autotuned_shape": {"lbm_threads": shape[0], "lbm_planes": shape[1],
                                           "membrane_vertices_per_thread": shape[2]} if fused else None,
                       "l2": "inputs larger than L2 (populations %.2f GB), no flush" % (2 * 19 * 4 * sum(c.nx * c.ny * (c.nz - 4) for c in cases) / 1e9)},
            "sequential": {"value": round(seq, 2), "unit": "MLUPS", "ms_per_step": round(seq_ms / args.steps, 4),
                           "how": "each capillary stepped alone (rbc_step, CUDA graphs), one after another"},
            "speedup_vs_sequential": round(value / seq, 2),
            "gpu_launches": launches, "status_flags_nonzero": int(sum(1 for f in flags if f & 3)),
            "clocks": clk.summary()}


def run_adjoint(args, world, rank, local):
    """Config 5: gradient of the cell-shape loss through --adjoint-steps steps
    of the single-cell duct with a checkpoint every --ckpt steps.  Times, with
    CUDA events on the library's stream: plain forward steps (rbc_step), the
    recorded forward (rbc_adjoint_record) and the reverse sweep
    (rbc_adjoint_backward, which recomputes each segment once).  value = device
    milliseconds per step of the reverse sweep."""
    import numpy as np
    import torch

    from preprocess_src_b200 import configs
    from preprocess_src_b200.adjoint import InitialState
    from preprocess_src_b200.step import Simulation

    dev = local
    torch.cuda.set_device(dev)
    n = args.adjoint_steps
    case = configs.single_cell_duct()
    sim = Simulation(case, device=dev)
    init = InitialState(sim)
    st = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", dev))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    sim.step(args.warmup)
    init.restore(sim)
    # untimed: allocates the checkpoints and stores, captures the segment graphs
    sim.adjoint_record(n, args.ckpt)
    sim.adjoint_backward(np.zeros(sim.nv), np.zeros(sim.nv), np.zeros(sim.nv))
    init.restore(sim)
    barrier(world)
    with ClockSampler(dev) as clk:
        time.sleep(0.3)
        ev[0].record(st)
        sim.step(n)
        ev[1].record(st)
        ev[1].synchronize()
        init.restore(sim)
        ev[2].record(st)
        sim.adjoint_record(n, args.ckpt)
        ev[3].record(st)
        ev[3].synchronize()
        c = sim.export_cells()
        # seed: gradient of the mean squared distance to the initial shape
        x0 = np.stack([init.x, init.y, init.z])
        seed = (2.0 / sim.nv) * (np.stack([c["x"], c["y"], c["z"]]) - x0)
        r = sim.adjoint_backward(seed[0], seed[1], seed[2])
    fwd_ms, rec_ms, bwd_ms = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), r["ms"]
    bwd_max = allreduce_max(bwd_ms, world)
    sim.close()
    if rank != 0:
        return None
    fluid = case.fluid_nodes()
    return {"metric": "adjoint ms per step, single-cell duct (config 5)", "value": round(bwd_max / n, 4),
            "unit": "ms/step", "n_gpus": world, "steps": n, "warmup": args.warmup,
            "ms_per_step": round(bwd_max / n, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": case.name, "fluid_nodes": fluid, "vertices": sim.nv, "ckpt_every": args.ckpt,
                       "l2": "lattice and checkpoints below L2 size: steady-state timing of a small case"},
            "forward_ms_per_step": round(fwd_ms / n, 4), "record_ms_per_step": round(rec_ms / n, 4),
            "backward_over_forward": round(bwd_ms / fwd_ms, 2),
            "grad": {"dL/dP": r["grad"][0], "dL/dB": r["grad"][1], "dL/dC": r["grad"][2]},
            "adjoint_flags": r["flags"], "clocks": clk.summary()}


def run_e2e(args, case, dev, world):
    """Public-API run with host buffers (pinned), copies inside the timed region."""
    import numpy as np
    import torch

    from preprocess_src_b200.step import Simulation

    n, nv, ne, nc = case.n, case.ncell * case.vertex, case.ncell * case.element, case.ncell

    def pinned(count):
        return torch.empty(count, dtype=torch.float64, pin_memory=True).numpy()

    # reference-layout initial state: rest equilibrium and the initial cells
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    fn = pinned(n * 19)
    fn.reshape(n, 19)[:] = w
    xr = np.asarray(case.xr).reshape(-1, 3)
    x, y, z, xd = pinned(nv), pinned(nv), pinned(nv), pinned(3 * nv)
    x[:], y[:], z[:] = xr[:, 0], xr[:, 1], xr[:, 2]
    xd[:] = case.xr
    nd = pinned(4 * ne)
    sim = Simulation(case, device=dev)
    # reference metric as fem_init computes it (the import replaces the handle's own)
    a, b, c = xr[case.ele_global()[0::3]], xr[case.ele_global()[1::3]], xr[case.ele_global()[2::3]]
    v1, v2 = b - a, c - a
    l1, l2, i12 = (v1 * v1).sum(1), (v2 * v2).sum(1), (v1 * v2).sum(1)
    dv = l1 * l2 - i12 * i12
    nd.reshape(-1, 4)[:] = np.stack([l2 / dv, -i12 / dv, -i12 / dv, l1 / dv], axis=1)
    met = sim.cell_metrics()
    vol0, gx = pinned(nc), pinned(3 * nc)
    vol0[:], gx[:] = met["volume"], met["centroid"]
    # each step's metrics land in one of two pinned buffers; the host reads step k - 1's while
    # step k runs
    ring = [pinned(5 * nc), pinned(5 * nc)]
    ox, oy, oz = pinned(nv), pinned(nv), pinned(nv)
    stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", dev))
    import ctypes as C

    from preprocess_src_b200 import _native as N
    L, h = N.lib(), sim._h
    dp = lambda arr: arr.ctypes.data_as(N._DP)  # noqa: E731
    sim.step(2)     # build the step graphs outside the timed region
    sim.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    N.check(L.rbc_import_ref_lattice(h, dp(fn)), h)
    N.check(L.rbc_import_ref_cells(h, dp(x), dp(y), dp(z), dp(xd), dp(nd), dp(vol0), dp(gx)), h)
    N.check(L.rbc_set_iter(h, 0), h)
    ready = [torch.cuda.Event(), torch.cuda.Event()]
    vol_seen = 0.0
    for k in range(args.steps):
        N.check(L.rbc_step(h, 1), h)
        N.check(L.rbc_cell_metrics_async(h, dp(ring[k % 2])), h)
        ready[k % 2].record(stream)
        if k > 0:
            ready[(k - 1) % 2].synchronize()
            vol_seen += float(ring[(k - 1) % 2][:nc].sum())
    ready[(args.steps - 1) % 2].synchronize()
    vol_seen += float(ring[(args.steps - 1) % 2][:nc].sum())
    N.check(L.rbc_export_ref_cells(h, dp(ox), dp(oy), dp(oz), None, None, None, None, None, None, None, None), h)
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - t0
    ms = allreduce_max(ev0.elapsed_time(ev1), world)
    fluid = case.fluid_nodes()
    h2d = (fn.nbytes + x.nbytes * 3 + xd.nbytes + nd.nbytes + vol0.nbytes + gx.nbytes) / args.steps
    d2h = ring[0].nbytes + (ox.nbytes * 3) / args.steps
    sim.close()
    return {"value": round(world * fluid * args.steps / (ms * 1e-3) / 1e6, 2), "unit": "MLUPS",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "wall_s": round(wall, 4),
            "path": "rbc_import_ref_lattice + rbc_import_ref_cells + K x (rbc_step(1) + rbc_cell_metrics_async, the host reading each step's metrics one step behind) + "
                    "rbc_export_ref_cells, pinned host buffers"}


def run_reference_capillaries(args):
    """The FP64 oracle on the config-4 capillaries, one after another, for a
    bounded sample (about 60 s): aggregate MLUPS over the capillaries run."""
    from preprocess_src_b200 import configs
    from oracle.oracle import Oracle, num_threads
    cases = configs.capillary_batch(args.capillaries, seed=4)
    steps = max(1, min(args.steps, 20))
    done_nodes, el, ncap = 0, 0.0, 0
    for c in cases:
        o = Oracle(c)
        o.step(1)
        t0 = time.perf_counter()
        o.step(steps)
        el += time.perf_counter() - t0
        done_nodes += c.fluid_nodes() * steps
        ncap += 1
        if el > 60.0:
            break
    value = done_nodes / el / 1e6
    sample = f"{steps} FP64 oracle steps of each of the first {ncap} of {len(cases)} capillaries, one after another ({el:.1f} s)"
    return {"metric": "aggregate MLUPS, %d uneven capillaries in one batch (config 4)" % len(cases), "impl": "reference",
            "value": round(value, 4), "unit": "MLUPS", "n_gpus": 1, "steps": steps, "warmup": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "capillary_batch_%d_32x32xL" % len(cases)},
            "cpu_baseline": {"value": round(value, 4), "unit": "MLUPS", "cores": num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_kernels_b200(args, tag, case):
    """The reference's own CUDA step modules (lbm.cu, ibm.cu, stress.cu,
    matrix_solver.cu, volume_correction.cu compiled from the reference sources
    for sm_100a by oracle/Makefile, lengths and constants as -D macros) on this
    GPU: main.cu:73-110's step order, each module timed by CUDA events (the
    reference synchronises the device after every module).  None when the
    library was not built (no reference sources where the package was built)
    or there is no GPU."""
    import ctypes as C

    import numpy as np
    lib = ROOT / "oracle" / "_ref" / f"librefstep_{tag}.so"
    if not lib.exists():
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    L = C.CDLL(str(lib))
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    bc = np.ascontiguousarray(case.bc, dtype=np.int32)
    tri = np.ascontiguousarray(case.tri, dtype=np.int32).reshape(-1)
    xr = np.ascontiguousarray(case.xr, dtype=np.float64)
    t0 = time.perf_counter()
    if L.ref_setup(case.nx, case.ny, case.nz, p(bc), case.ncell, case.vertex, case.element, p(tri), p(xr)):
        return {"unavailable": "the reference's setup reported an error"}
    setup_s = time.perf_counter() - t0
    if L.ref_step(1):
        return {"unavailable": "the reference's step reported an error"}
    steps = max(1, min(args.steps, 3 if tag == "dense" else 50))
    ms = np.zeros(5)
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        rc = L.ref_time_steps(steps, p(ms))
    if rc:
        return {"unavailable": "the reference's step reported an error"}
    per = ms / steps
    fluid = case.fluid_nodes()
    return {"value": round(fluid / (per.sum() * 1e-3) / 1e6, 3), "unit": "MLUPS", "steps": steps, "warmup": 1,
            "ms_per_step": round(float(per.sum()), 3),
            "ms_per_step_by_module": dict(zip(("stress", "ibm_st1", "lbm_d3q19", "ibm_st2", "volume_correction"),
                                              [round(float(v), 3) for v in per])),
            "lbm_module_mlups": round(fluid / (per[2] * 1e-3) / 1e6, 1), "setup_s": round(setup_s, 2),
            "dtype": "f64", "residual": case.params["residual"],
            "how": "the reference's own kernels compiled unmodified for sm_100a with a project-written def.h "
                   "(oracle/ref_harness), CUDA events around each module, FP64 throughout",
            "clocks": clk.summary()}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    if args.workload == "capillaries":
        return run_reference_capillaries(args)
    if args.workload == "vof":
        return {"impl": "reference", "unavailable": "the CPU oracle's setup front tracking (red-black SOR on the "
                "4.1M-node lattice) alone exceeds the reference arm's few-minute budget"}
    case = make_case(args.workload)
    from oracle.oracle import Oracle, num_threads
    o = Oracle(case)
    budget = 150.0
    t_start = time.perf_counter()
    o.step(max(1, min(args.warmup, 2)))
    warm_s = time.perf_counter() - t_start
    per = warm_s / max(1, min(args.warmup, 2))
    steps = max(1, min(args.steps, int(budget / max(per, 1e-9))))
    t0 = time.perf_counter()
    o.step(steps)
    el = time.perf_counter() - t0
    fluid = case.fluid_nodes()
    value = fluid * steps / el / 1e6
    sample = (f"{steps} full FP64 oracle steps of {case.name} ({el:.1f} s, capped by a {budget:.0f} s budget); "
              "the reference implements the step only as CUDA kernels, so its CPU arm is the oracle port")
    res = {"metric": METRIC, "impl": "reference", "value": round(value, 4), "unit": "MLUPS", "n_gpus": world,
            "steps": steps, "warmup": min(args.warmup, 2), "ms_per_step": round(el / steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": case.name, "fluid_nodes": fluid, "cells": case.ncell,
                       "vertices_per_cell": case.vertex},
            "vertices_per_s": round(case.ncell * case.vertex * steps / el, 1),
            "cpu_baseline": {"value": round(value, 4), "unit": "MLUPS", "cores": num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # beside the CPU value: the reference's own CUDA kernels on this GPU
    if args.workload in ("dense", "single") and not args.br:
        from tests.golden.make_golden import bench_cases
        rk = reference_kernels_b200(args, args.workload, bench_cases()[args.workload])
        if rk is not None:
            res["reference_kernels_b200"] = rk
    return res


def main():
    args = parse()
    if args.impl == "reference":
        world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
        res = run_reference(args, world, rank)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    world, rank, local = dist_setup(args)
    runner = {"capillaries": run_capillaries, "adjoint": run_adjoint}.get(args.workload, run_ours)
    res = runner(args, world, rank, local)
    if res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
