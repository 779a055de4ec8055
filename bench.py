#!/usr/bin/env python
"""Benchmark of the relaxation loop: node-iterations per second.

Workload (default): 256^3 volume, six nested noisy ellipsoidal shells (semi-axes
60..120 voxels, 4-octave seeded noise of amplitude 6 voxels), h in [1.5, 6]
voxels graded by the distance to the nearest interface, ~1M seeded nodes, 500
FP32 FIRE iterations (dptol 0: no early stop), the reference's Verlet rebuild
trigger. One step = one whole relaxation from the seeds (first list build +
500 iterations), inputs resident in HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
  python bench.py --workload batch64   (the batched form against sequential runs)
  python bench.py --workload adjoint   (the unroll's backward against its forward)
  python bench.py --workload seed_tpm182   (seeding on the device against seed_cpu)
  python bench.py --workload grid_shells256   (the grid build on the device against build_grid_cpu)

--workload batch64: 64 independent volumes of seeded sizes 32^3..160^3 with
2..18 nested-shell labels (~4M nodes in all), 200 FIRE iterations each. One
step relaxes all of them in one session whose iteration loop is a CUDA graph
(the tiles picked by the autotuner); the line adds the time of the same 64
relaxations run one after another, each in its own session with plain
launches, and the ratio of the two.

N > 1 runs under torchrun, one process per GPU: a single volume does not
shard, so each rank relaxes its own replica (weak scaling, no collective on the
data path); the step time is the max over ranks (all_reduce MAX over NCCL).
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "relax node-iters/s at 1M nodes"
UNIT = "node-iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="shells256")
    ap.add_argument("--iters", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ref-iters", type=int, default=10, help="iterations per reference-arm / CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload(name, seed=0):
    from trussnet_b200 import synth
    if name == "shells256":
        g, nd = synth.shells(seed=seed)
        prm = synth.params_for("shells256")
        desc = ("shells256: 256^3, 6 nested noisy ellipsoidal shells (semi-axes 60-120 vox, noise amp 6 vox, "
                "4 octaves), h in [1.5,6] vox graded by interface distance, FIRE, reference Verlet trigger")
    elif name == "sphere64":
        g, nd = synth.sphere(seed=seed)
        prm = synth.params_for("sphere64")
        desc = "sphere64: 64^3 sphere r=24, h=2, 2-voxel lattice + jitter, dt=0.2"
    elif name == "tpm182":
        g, nd = synth.tpm(seed=seed)
        prm = synth.params_for("tpm182")
        desc = "tpm182: 182x218x182 argmax of 6 smoothed noise fields (sigma 4), h=1.3"
    else:
        raise SystemExit(f"unknown workload {name}")
    return g, nd, prm, desc


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload_name: str):
    """dram bytes per launch of `kernel` from the committed ncu summary
    (profiles/<kernel>_<workload>.txt, line 'traffic_bytes_per_launch: X')."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload_name}.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def cpu_baseline(g, nd, prm, iters):
    """The reference's relax_cpu (oracle/_ref, the compiled reference) on a bounded
    sample: the same grid and seeds, `iters` iterations."""
    from oracle.ref import RefLib, available
    from trussnet_b200.types import RelaxParams
    p = RelaxParams(**{**prm.__dict__, "max_iters": iters})
    if not available():
        return None
    lib = RefLib()
    a = nd.copy()
    t0 = time.perf_counter()
    lib.relax_cpu(g, p, a)
    dt = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    if os.environ.get("OMP_NUM_THREADS"):
        cores = int(os.environ["OMP_NUM_THREADS"])
    else:
        cap = int(os.environ.get("V2M_OMP_MAX_THREADS", "64"))
        cores = min(cores, cap) if cap > 0 else cores
    return {"value": nd.size() * iters / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"relax_cpu on the same grid and seeds, {iters} iterations (first list build included), "
                      f"{dt:.2f} s", "_nodes": a, "_seeds": nd, "_params": p}


def parity_check(g, cb, local):
    """The bench's own output check: relax_cl (the CUDA path, through the C ABI)
    on the CPU baseline's sample -- the same grid, seeds and iterations -- compared
    bit for bit (positions, types, partners) with the reference's relax_cpu result,
    or, where the parameters use an extension of the loop that the reference lacks,
    with the plain-C restatement's."""
    from trussnet_b200 import relax_cl
    ref = cb.pop("_nodes")
    p = cb.pop("_params")
    seeds = cb.pop("_seeds")
    against = "relax_cpu (oracle/_ref, the compiled reference)"
    if p.rebuild_policy != 0 or p.h_mode != 0 or p.rebuild_div != 0:
        # an extension of the loop the reference does not have: checked against the
        # plain-C restatement, which implements it (the reference sample is timing only)
        from oracle.oracle import Oracle
        ref = seeds.copy()
        Oracle("f32").relax(g, p, ref)
        against = "the plain-C FP32 restatement (oracle/v2m_oracle.c): the parameters use an extension"
    dev = seeds.copy()
    st = relax_cl(g, p, dev, device=local)
    same = {"P": bool(np.array_equal(dev.P.view(np.uint32), ref.P.view(np.uint32))),
            "typ": bool(np.array_equal(dev.typ, ref.typ)), "part": bool(np.array_equal(dev.part, ref.part))}
    return {"against": against, "iterations": p.max_iters,
            "nodes": int(ref.size()), "list_builds": st.rebuilds, "bit_exact": all(same.values()), **same}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_seed_reference(args):
    """The reference arm of seed_tpm182: seed_cpu on the host cores, W + K whole
    seedings of the same grid."""
    from oracle.ref import RefLib, available
    from trussnet_b200 import synth
    from trussnet_b200.types import RelaxParams
    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libv2m_ref.so is not built"}))
        return
    g, _ = synth.tpm()
    g.grade = synth.size_grades(g.h, g.hmin, g.hmax)
    prm = RelaxParams()
    lib = RefLib()
    for _ in range(args.warmup):
        lib.seed(g, prm)
    ts = []
    n = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        n = lib.seed(g, prm).size()
        ts.append(time.perf_counter() - t0)
    dt = statistics.mean(ts)
    cores = os.cpu_count() or 1
    cap = int(os.environ.get("V2M_OMP_MAX_THREADS", "64"))
    cores = min(cores, cap) if cap > 0 else cores
    v = n / dt
    print(json.dumps({"metric": "seeding seeds/s", "value": v, "unit": "seeds/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "impl": "reference",
                      "config": {"workload": "seed_tpm182: the tpm182 grid, nseed 8, jseed 0.8, corners on",
                                 "nodes": n},
                      "cpu_baseline": {"value": v, "unit": "seeds/s", "cores": cores, "kind": "reference",
                                       "sample": f"seed_cpu, whole seedings of the grid, {dt:.2f} s each"},
                      "e2e": {"value": v, "unit": "seeds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_grid_reference(args):
    """The reference arm of grid_shells256: build_grid_cpu on the host cores,
    W + K whole builds of the same labels."""
    from oracle.ref import RefLib, available
    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libv2m_ref.so is not built"}))
        return
    L, gp = grid_workload()
    lib = RefLib()
    for _ in range(args.warmup):
        lib.build_grid_p(L, prm=gp)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        lib.build_grid_p(L, prm=gp)
        ts.append(time.perf_counter() - t0)
    dt = statistics.mean(ts)
    v = L.size / dt
    print(json.dumps({"metric": "grid build voxels/s", "value": v, "unit": "voxels/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "impl": "reference", "config": {"workload": "grid_shells256", "voxels": int(L.size)},
                      "cpu_baseline": {"value": v, "unit": "voxels/s", "cores": _cores(), "kind": "reference",
                                       "sample": f"build_grid_cpu, whole builds, {dt:.2f} s each"},
                      "e2e": {"value": v, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    if args.workload == "seed_tpm182":
        run_seed_reference(args)
        return
    if args.workload == "grid_shells256":
        run_grid_reference(args)
        return
    if args.workload in ("batch64", "adjoint"):
        why = {"batch64": "the reference relaxes one volume per call; its arm is the default workload's",
               "adjoint": "the reference has no adjoint of the relaxation"}[args.workload]
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    g, nd, prm, desc = workload(args.workload)
    from oracle.ref import available
    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libv2m_ref.so is not built"}))
        return
    for _ in range(args.warmup):
        cpu_baseline(g, nd, prm, args.ref_iters)
    vals = []
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(g, nd, prm, args.ref_iters)
        vals.append(cb["value"])
    v = statistics.mean(vals)
    ms = nd.size() * args.ref_iters / v * 1e3
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "nodes": nd.size(), "iters_per_step": args.ref_iters,
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "reference",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_PINNED = []   # the torch tensors that own the pinned pages of pinned_copy's arrays


def pinned_copy(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory."""
    import torch
    t = torch.empty(a.shape, dtype={np.dtype(np.float32): torch.float32, np.dtype(np.uint16): torch.int16,
                                    np.dtype(np.int32): torch.int32, np.dtype(np.uint8): torch.uint8}[a.dtype],
                    pin_memory=True)
    _PINNED.append(t)
    out = t.numpy().view(a.dtype)
    out[...] = a
    return out


def run_batch(args):
    """The batched form (64 volumes, one graph-captured session) against the same
    relaxations run one volume at a time with plain launches; device time by CUDA
    events on each session's stream. Under torchrun (N > 1) the volumes are
    sharded over the ranks by node count (shard.assign_volumes: no collective
    while the loops run), each rank relaxing its share in one session on its
    GPU; the step time is the max over ranks and the end-to-end leg goes
    through shard.relax_batch_distributed (every rank ends with every volume)."""
    import torch
    from trussnet_b200 import Session, synth
    from trussnet_b200.shard import assign_volumes
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    vols = synth.batch()
    prm = synth.params_for("batch64")
    if args.iters:
        prm.max_iters = args.iters
    iters = prm.max_iters
    grids = [g for g, _ in vols]
    nodes = [nd for _, nd in vols]
    prms = [prm] * len(vols)
    n = sum(nd.size() for nd in nodes)
    mine = assign_volumes([nd.size() for nd in nodes], world)[rank]

    def barrier():
        torch.cuda.synchronize(local)
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    sess = Session([grids[v] for v in mine], [prm] * len(mine), [nodes[v] for v in mine], device=local)
    tune = sess.autotune()
    sess.timed_runs(args.warmup, graph=True)
    sess.clear_counters()
    barrier()
    clk = ClockSampler(local)
    clk.start()
    ms = sess.timed_runs(args.steps, graph=True)
    clocks = clk.stop()
    barrier()
    cnt = sess.counters()
    sess.close()
    step_ms = max_over_ranks(ms / args.steps)
    seq_ms = None
    seq_sync_ms = None
    e2e = {}
    from trussnet_b200 import relax_cl, relax_cl_batch
    if world == 1:
        # the same relaxations, one volume at a time, plain launches (each session warmed once):
        # the loop's control on the device, the host reading it every 25 iterations; and the
        # same with the reference relax_cl's blocking read-back every iteration
        seq_ms = 0.0
        seq_sync_ms = 0.0
        for g, nd in vols:
            with Session(g, prm, nd, device=local) as s1:
                s1.timed_runs(1, graph=False)
                seq_ms += s1.timed_runs(1, graph=False)
                os.environ["V2M_CUDA_HOST_CHECK"] = "1"
                try:
                    seq_sync_ms += s1.timed_runs(1, graph=False)
                finally:
                    del os.environ["V2M_CUDA_HOST_CHECK"]
        torch.cuda.synchronize(local)
        # end to end through the C ABI: one batch call against one relax_cl call per
        # volume (host buffers, every upload, set-up and read-back inside), same results
        for k in range(2):   # the first pass warms the module and the allocator
            outs_b = [nd.copy() for nd in nodes]
            t0 = time.perf_counter()
            relax_cl_batch(grids, prms, outs_b, device=local)
            tb = time.perf_counter() - t0
            outs_s = [nd.copy() for nd in nodes]
            t0 = time.perf_counter()
            for g, o in zip(grids, outs_s):
                relax_cl(g, prm, o, device=local)
            ts_ = time.perf_counter() - t0
            e2e = {"batch_call_s": tb, "sequential_calls_s": ts_, "speedup": ts_ / tb}
        e2e["identical"] = all(np.array_equal(a.P.view(np.uint32), b.P.view(np.uint32)) and
                               np.array_equal(a.typ, b.typ) for a, b in zip(outs_b, outs_s))
    else:
        from trussnet_b200.shard import relax_batch_distributed
        for k in range(2):
            outs_b = [nd.copy() for nd in nodes]
            barrier()
            t0 = time.perf_counter()
            relax_batch_distributed(grids, prms, outs_b, device=local)
            torch.cuda.synchronize(local)
            tb = max_over_ranks(time.perf_counter() - t0)
            e2e = {"batch_call_s": tb}
    if rank == 0:
        line = {"metric": "batched relax node-iters/s, 64 volumes", "value": n * iters / (step_ms / 1e3),
                "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batch64: 64 volumes 32^3..160^3, 2..18 nested-shell labels, h in [1.55, 6.2] "
                                       "vox, 200 FIRE iterations, dptol 0", "volumes": len(vols), "nodes": n,
                           "min_nodes": min(nd.size() for nd in nodes), "max_nodes": max(nd.size() for nd in nodes),
                           "iters_per_step": iters, "autotune": tune.strip().splitlines()[-1] if tune else None,
                           "parallelism": (f"volumes sharded over {world} ranks by node count (LPT), no collective "
                                           f"in the loop" if world > 1 else "one session")},
                "sequential_plain_ms": seq_ms, "batched_speedup": (seq_ms / step_ms) if seq_ms else None,
                "sequential_plain_readback_every_iteration_ms": seq_sync_ms if world == 1 else None,
                "batched_speedup_vs_readback_every_iteration": (seq_sync_ms / step_ms) if world == 1 else None,
                "e2e": {"value": n * iters / e2e["batch_call_s"], "unit": UNIT,
                        "h2d_bytes_per_step": int(sum(g.nbytes() for g in grids) + sum(nd.nbytes() for nd in nodes)),
                        "d2h_bytes_per_step": int(sum(nd.P.nbytes + nd.typ.nbytes + nd.part.nbytes for nd in nodes)),
                        **{k: v for k, v in e2e.items()}},
                "clocks": clocks, "gpu_launches": int(cnt["launches"])}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def adjoint_leg(local, steps=3, warmup=3):
    """The differentiable unroll: K = 50 Jacobi steps on a 128^3 4-label nested
    ellipsoid volume (~150k nodes) with a 64^3 sizing grid, checkpoint every 10
    steps; device time (CUDA events) of the forward pass and of the backward pass
    (gradients w.r.t. the nodes and the grid, the loss's gradient included)."""
    import torch
    from trussnet_b200 import Session, synth
    from trussnet_b200.adjoint import Unroll
    from trussnet_b200.types import RelaxParams
    g, nd, G, cs = synth.ellipsoids_adjoint()
    with Session(g, RelaxParams(max_iters=1), nd, device=local) as s:
        s.rebuild()
        nbr, nnb = s.read("nbr"), s.read("nnb")
    K, ckpt = 50, 10
    u = Unroll(nbr, nnb, nd.typ, G.shape[::-1], cs, 1.2, 1.0, 0.2, K, ckpt, device=local)
    x0 = torch.tensor(nd.P, device=f"cuda:{local}")
    Gt = torch.tensor(G, device=f"cuda:{local}")
    f = b = 0.0
    for k in range(warmup + steps):
        xK = u.forward(x0, Gt)
        gxK, _ = u.loss_backward(xK, Gt)
        u.backward(Gt, gxK)
        if k >= warmup:
            tf, tb = u.timing()
            f += tf
            b += tb
    u.close()
    return {"workload": "ellipsoids_adjoint: 128^3, 4 nested labels, 64^3 sizing grid in [1.5,4], K=50, "
                        "checkpoint every 10", "nodes": nd.size(), "K": K, "ckpt": ckpt,
            "forward_us_per_step": f / steps / K * 1e3, "backward_us_per_step": b / steps / K * 1e3,
            "backward_over_forward": b / f}


def run_adjoint(args):
    world, rank, local = dist_setup(args)
    if rank != 0:
        return
    a = adjoint_leg(local, args.steps, args.warmup)
    line = {"metric": "adjoint/fwd ratio", "value": a["backward_over_forward"], "unit": "x", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["backward_us_per_step"] * a["K"] / 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": a}
    print(json.dumps(line), flush=True)


def run_seed(args):
    """Seeding of the tpm182 grid (182x218x182, argmax of six smoothed noise
    fields: interfaces, junction lines and 4-label corners everywhere; h = 1.3)
    with the reference's default parameters (8 seed levels, junction-line seeds,
    corners):
    seeds per second through seed_cl, a whole call from host arrays (grid upload,
    corner tables, the seeding stages, the copy back), against the reference's
    seed_cpu on the same grid, whose result it must equal bit for bit."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return
    import torch
    from trussnet_b200 import seed_cl, synth
    from trussnet_b200.types import RelaxParams
    torch.cuda.set_device(local)
    g, _ = synth.tpm()
    g.grade = synth.size_grades(g.h, g.hmin, g.hmax)
    prm = RelaxParams()
    for _ in range(args.warmup):
        nd, p3 = seed_cl(g, prm, device=local)
    ts = []
    clk = ClockSampler(local)
    clk.start()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        nd, p3 = seed_cl(g, prm, device=local)
        ts.append(time.perf_counter() - t0)
    clocks = clk.stop()
    dt = statistics.mean(ts)
    n = nd.size()
    h2d = g.nbytes() + g.grade.nbytes
    d2h = n * (12 + 2 + 1 + 4 + 2)
    cb, same = None, None
    if not args.no_cpu_baseline:
        from oracle.ref import RefLib, available
        if available():
            lib = RefLib()
            t0 = time.perf_counter()
            rnd = lib.seed(g, prm)
            tc = time.perf_counter() - t0
            same = bool(rnd.size() == n and all(np.array_equal(getattr(rnd, a), getattr(nd, a))
                                                for a in ("P", "lab", "typ", "part")) and np.array_equal(rnd.part3, p3))
            cores = os.cpu_count() or 1
            cap = int(os.environ.get("V2M_OMP_MAX_THREADS", "64"))
            cores = min(cores, cap) if cap > 0 else cores
            cb = {"value": rnd.size() / tc, "unit": "seeds/s", "cores": cores, "kind": "reference",
                  "sample": f"seed_cpu on the same grid, one whole seeding, {tc:.2f} s"}
    line = {"metric": "seeding seeds/s", "value": n / dt, "unit": "seeds/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "seed_tpm182: the tpm182 grid (182x218x182, argmax of 6 smoothed noise fields, "
                                   "h = 1.3), nseed 8, jseed 0.8, corners on", "nodes": n,
                       "types": np.bincount(nd.typ, minlength=4).tolist(), "timed": "whole seed_cl calls from host "
                       "arrays (upload, corner tables, seeding, copy back)"},
            "e2e": {"value": n / dt, "unit": "seeds/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "cpu_baseline": cb, "results_identical": same, "clocks": clocks}
    print(json.dumps(line), flush=True)


def grid_workload():
    """The shells256 label volume (256^3, six noisy shells) and grid parameters
    giving its h range: hbase 4, hmin 1.5, hmax 6 voxels."""
    from trussnet_b200 import GridParams, synth
    g, _ = synth.shells(seed=0)
    return g.L, GridParams(hbase=4.0, hmin=1.5, hmax=6.0)


def run_grid(args):
    """The grid build on the device (grid_cl: labels from host memory in, the
    grid's arrays to host memory out, the whole call timed) against the
    reference's build_grid_cpu on the same labels and parameters; results
    compared bit for bit."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return
    import torch
    from trussnet_b200 import grid_cl
    torch.cuda.set_device(local)
    L, gp = grid_workload()
    nv = L.size
    for _ in range(args.warmup):
        gd = grid_cl(L, (1.0, 1.0, 1.0), gp, device=local)
    clk = ClockSampler(local)
    clk.start()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        gd = grid_cl(L, (1.0, 1.0, 1.0), gp, device=local)
        ts.append(time.perf_counter() - t0)
    clocks = clk.stop()
    dt = statistics.mean(ts)
    cb, same = None, None
    if not args.no_cpu_baseline:
        from oracle.ref import RefLib, available
        if available():
            t0 = time.perf_counter()
            gr = RefLib().build_grid_p(L, prm=gp)
            tc = time.perf_counter() - t0
            same = all(np.array_equal(getattr(gd, a), getattr(gr, a)) for a in
                       ("bl_cnt", "bl_lab", "bl_slot", "phi", "h", "grade"))
            cb = {"value": nv / tc, "unit": "voxels/s", "cores": _cores(), "kind": "reference",
                  "sample": f"build_grid_cpu on the same labels and parameters, one whole build, {tc:.2f} s"}
    line = {"metric": "grid build voxels/s", "value": nv / dt, "unit": "voxels/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "grid_shells256: the shells256 label volume (256^3, six noisy shells), "
                                   "hbase 4, hmin 1.5, hmax 6 voxels, the reference's other GridParams defaults",
                       "voxels": int(nv), "slots": int(gd.phi.size // 512),
                       "timed": "whole grid_cl calls from host labels to host grid arrays"},
            "e2e": {"value": nv / dt, "unit": "voxels/s", "h2d_bytes_per_step": int(L.nbytes),
                    "d2h_bytes_per_step": int(gd.nbytes() + gd.grade.nbytes - L.nbytes)},
            "cpu_baseline": cb, "results_identical": same, "clocks": clocks}
    print(json.dumps(line), flush=True)


def _cores():
    cores = os.cpu_count() or 1
    cap = int(os.environ.get("V2M_OMP_MAX_THREADS", "64"))
    return min(cores, cap) if cap > 0 else cores


def run_cuda(args):
    import torch
    world, rank, local = dist_setup(args)
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from trussnet_b200 import Session, relax_cl
    from trussnet_b200.types import Grid, Nodes
    g, nd, prm, desc = workload(args.workload)
    if args.iters:
        prm.max_iters = args.iters
    iters = prm.max_iters
    n = nd.size()
    sess = Session(g, prm, nd, device=local)
    sess.timed_runs(args.warmup, graph=True)
    sess.clear_counters()

    def barrier():
        torch.cuda.synchronize(local)
        if world > 1:
            torch.distributed.barrier()

    barrier()
    clk = ClockSampler(local)
    clk.start()
    ms = sess.timed_runs(args.steps, graph=True, time_force=True)
    clocks = clk.stop()
    barrier()
    cnt = sess.counters()
    step_ms = ms / args.steps
    if world > 1:
        t = torch.tensor([step_ms], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_ms = float(t.item())
    value = world * n * iters / (step_ms / 1e3)
    # force kernel roofline: algorithmic bytes per launch / mean event-timed launch
    nnb = sess.read("nnb").astype(np.int64)
    force_bytes = 37 * n + 4 * int(nnb.sum())
    force_avg_ms = cnt["force_ms"] / max(1, cnt["force_launches"])
    peak, peak_kind = peaks()
    achieved = force_bytes / (force_avg_ms / 1e3) / 1e9 if force_avg_ms > 0 else None
    roofline = {"kernel": "k_force", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
                "traffic": profiled_traffic("k_force", args.workload),
                "bytes_per_launch": force_bytes, "mean_nnb": float(nnb.mean()) if n else 0.0,
                "force_ms_per_launch": force_avg_ms, "force_share_of_step": cnt["force_ms"] / ms if ms else None}
    st = sess.stats()
    # where an iteration's time goes: one more run from the seeds, its first 100
    # iterations profiled stage by stage (plain launches, outside the timed region)
    sess.reset()
    sess.rebuild()
    nprof = min(100, iters)
    stages = sess.profile_stages(nprof)
    trapped, interior = sess.queue_sizes()
    sess.close()
    # the move's roofline: algorithmic bytes per iteration -- every node's 91 B
    # (read P 12, F 16, V 12, typ 1, lab 2, part 4, h 4; write P 12, V 12, h 4,
    # |dp|/h 4, power 4) and, per trapped node, one brick record (48 B) and two
    # labels' eight corner values (64 B) -- over the move stage's time per iteration
    move_ms = stages["move"] / nprof if nprof else 0.0
    move_bytes = 91 * n + 112 * trapped
    move_achieved = move_bytes / (move_ms / 1e3) / 1e9 if move_ms > 0 else None
    # (traffic: the ncu dram bytes of one iteration's k_move_int + k_move_main)
    mtr = [profiled_traffic(k, args.workload) for k in ("k_move_int", "k_move_main")]
    move_roofline = {"kernel": "k_move_pre + k_move_int + k_move_main", "bound": "hbm", "achieved": move_achieved,
                     "peak": peak, "unit": "GB/s", "frac": move_achieved / peak if move_achieved else None,
                     "peak_source": peak_kind, "bytes_per_iteration": move_bytes, "ms_per_iteration": move_ms,
                     "queued_trapped": trapped, "queued_interior": interior,
                     "traffic": sum(mtr) if all(t is not None for t in mtr) else None}
    # end to end through the public call (tn::relax_cl's C ABI) with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        e2e = e2e_leg(args, g, nd, prm, n, iters, world, local, barrier)
    cb = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(g, nd, prm, args.ref_iters)
        if cb is not None:
            parity = parity_check(g, cb, local)
    adj = adjoint_leg(local) if rank == 0 and world == 1 and args.e2e_steps > 0 else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": desc, "nodes": n, "iters_per_step": iters, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (grid %.0f MB + nodes %.0f MB per replica)" %
                                 (g.nbytes() / 1e6, nd.nbytes() / 1e6),
                           "rebuilds_per_step": st.rebuilds, "final_types": [st.n_interior, st.n_interface,
                                                                             st.n_junction, st.n_corner]},
                "clocks": clocks, "e2e": e2e, "gpu_launches": int(cnt["launches"]), "roofline": roofline,
                "move_roofline": move_roofline,
                "stage_ms_first100": stages, "cpu_baseline": cb, "parity": parity, "adjoint": adj}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def e2e_leg(args, g, nd, prm, n, iters, world, local, barrier):
    """The same metric through relax_cl (the C ABI's v2m_relax_cuda) from pinned
    host buffers: every step uploads the grid and the seeds, relaxes, and reads
    the nodes back."""
    import torch
    from trussnet_b200 import relax_cl
    from trussnet_b200.types import Grid, Nodes
    gp = Grid(nx=g.nx, ny=g.ny, nz=g.nz, vs=g.vs, L=pinned_copy(g.L), bl_cnt=pinned_copy(g.bl_cnt),
              bl_lab=pinned_copy(g.bl_lab), bl_slot=pinned_copy(g.bl_slot), phi=pinned_copy(g.phi),
              h=pinned_copy(g.h), hmin=g.hmin, hmax=g.hmax)
    npin = Nodes(P=pinned_copy(nd.P), lab=pinned_copy(nd.lab), typ=pinned_copy(nd.typ), part=pinned_copy(nd.part))
    e2e_times = []
    for k in range(args.e2e_steps + 1):
        npin.P[...] = nd.P
        npin.typ[...] = nd.typ
        npin.part[...] = nd.part
        barrier()
        t0 = time.perf_counter()
        relax_cl(gp, prm, npin, device=local)
        torch.cuda.synchronize(local)
        t1 = time.perf_counter()
        if k > 0:   # the first call loads the module and warms the allocator
            e2e_times.append(t1 - t0)
    e2e_s = statistics.mean(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = g.nbytes() + nd.nbytes()
    d2h = nd.P.nbytes + nd.typ.nbytes + nd.part.nbytes
    return {"value": world * n * iters / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "s_per_step": e2e_s}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch64":
        run_batch(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "seed_tpm182":
        run_seed(args)
    elif args.workload == "grid_shells256":
        run_grid(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
