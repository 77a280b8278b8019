#!/usr/bin/env python
"""Benchmark of the SignedDistances hot path on B200: SDF grid nodes/s.

Headline (`value`): the learned-radius form of the signed distance field of the workload mesh on
its grid.  One step = build the acceleration data from the device-resident mesh
(sdfgpu_set_mesh_device: triangle records + LBVH), train the radius network on a coarse exact
distance grid of that mesh (sdfgpu_train_radius: the coarse grid's distances and every training
step are inside the step), then distances with the learned radius, signs and sdf = dist .* sign for
every node (sdfgpu_sdf_device, SDFGPU_MODE_LEARNED).  The reference builds its KD-trees and BVH
inside every call too (evalDistancesOnTriMesh, raycast_sign_detection).  Beside it, with the same
step structure: the plain unbounded search (SDFGPU_MODE_UNBOUNDED, no network) and the
reference-rule truncated distance (SDFGPU_MODE_REF_RULE, the reference's own semantics).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload blobs256|torus128|icosphere|gyroid320]
    python bench.py --workload batch256 [--streams S]   # uneven batch of 256 meshes (sdfgpu_sdf_batch)
    python bench.py --impl reference ...   # the reference algorithm on the host cores

Both arms read the same binary STL of the workload (written once by a child process, see
workloads.ensure_stl) and build the same grid; their `config` objects are identical.  The
reference arm loads numpy and the oracle only.

Multi-GPU (torchrun, one rank per GPU): every rank computes its own copy of the workload (weak
scaling, no data-path collective); value = nodes of all ranks / max-over-ranks device time.
`--split zslab` instead splits one grid into z-slabs (sdfgpu_sdf_slab_device), one per rank, and
gathers the slabs on rank 0 with NCCL (strong scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "stl2sdf.jl_b200"))
sys.path.insert(0, ROOT)

METRIC = "SDF grid nodes/s on 1 B200: learned-radius vs plain GPU vs CPU ref, sign exact"
L2_NOTE = "a 256 MB device write between timed steps flushes the 126 MB L2 (the mesh records and fields exceed it too)"
TRAIN = dict(coarse_n=24, steps=50, batch=2048, lr=5e-3, seed=0)  # the learned form's per-mesh training


def common_config(name, X, IEN, g):
    """The workload's `config` object, the same in both arms."""
    import workloads

    return {"workload": name, "description": f"{workloads.description(name)}: {int(IEN.shape[0])} tris",
            "ngp": int(g["ngp"]), "nel": int(IEN.shape[0]), "nnp": int(X.shape[0]),
            "N": [int(v) for v in g["N"]], "h": float(g["h"]), "l2": L2_NOTE}


def load_gpu(name: str, device: int):
    """(X, IEN, grid) of a workload through the product's own import (GPU vertex deduplication) and grid
    setup."""
    import numpy as np

    import workloads
    from stl2sdf import DataImport, _native

    V, T = DataImport.read_binary_stl(workloads.ensure_stl(name))
    X, IEN = DataImport.process_stl_mesh(V, T, device=device)
    kind, v = workloads.grid_args(name)
    if kind == "nmax":
        o, amax, N, h, ngp = _native.grid_setup(X.min(0), X.max(0), v, 3)
    else:
        o, amax, N, h, ngp = _native.grid_from_cell_size(X, v)
    return X, IEN, dict(origin=np.asarray(o), N=np.asarray(N), h=float(h), ngp=int(ngp))


def load_reference(name: str):
    """(X, IEN, grid) of a workload with numpy and the oracle only: binary STL records, the oracle's
    restatement of process_stl_mesh (ImportStlData.jl:198-309) and of Grid (Grid.jl:9-32)."""
    import numpy as np

    import oracle
    import workloads
    from oracle import stl_dedupe

    path = workloads.ensure_stl(name)
    rec_t = np.dtype([("n", "<f4", (3,)), ("v", "<f4", (3, 3)), ("attr", "<u2")])
    with open(path, "rb") as f:
        f.read(80)
        n = int(np.frombuffer(f.read(4), "<u4")[0])
        rec = np.frombuffer(f.read(n * 50), rec_t, count=n)
    V = rec["v"].reshape(-1, 3).astype(np.float64)
    T = np.arange(1, 3 * n + 1, dtype=np.int64).reshape(n, 3)
    X, IEN = stl_dedupe.exact(V, T)
    if stl_dedupe.near_pairs(X):
        X, IEN = stl_dedupe.sequential(V, T)
    kind, v = workloads.grid_args(name)
    g = oracle.grid(X.min(0), X.max(0), v, 3) if kind == "nmax" else oracle.grid_from_cell_size(X, v)
    return X, IEN, dict(origin=g["origin"], N=g["N"], h=float(g["h"]), ngp=int(g["ngp"]))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._proc = None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                           "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        import statistics

        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def reference_sample(X, IEN, g, nodes, nthreads):
    """The reference algorithm (the oracle's FP64 restatement, reference rule) on a node sample."""
    import oracle

    oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=0, nodes=nodes, nthreads=nthreads)
    oracle.signs(X, IEN, g["origin"], g["h"], g["N"], nodes=nodes, nthreads=nthreads)


def cpu_baseline(X, IEN, g, budget_s=12.0, seed=42):
    """The oracle (C++ FP64 restatement of the reference, all host threads) on a seeded node
    sample of the workload grid, doubled until it takes >= budget_s or covers the grid."""
    import numpy as np

    import oracle

    nthreads = oracle.max_threads()
    k = 1 << 14
    rng = np.random.default_rng(seed)
    while True:
        nodes = np.sort(rng.choice(g["ngp"], size=min(k, g["ngp"]), replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        reference_sample(X, IEN, g, nodes, nthreads)
        dt = time.perf_counter() - t0
        if dt >= budget_s or nodes.shape[0] >= g["ngp"] or k >= (1 << 24):
            break
        k *= 2
    return {"value": nodes.shape[0] / dt, "unit": "nodes/s", "cores": nthreads, "kind": "port",
            "sample": f"{nodes.shape[0]} seeded (seed {seed}) uniform grid nodes of the workload, reference-rule "
                      f"distance + sign, {dt:.1f} s"}


def run_reference(args, rank, world):
    """--impl reference: the reference algorithm (the oracle's restatement) on the host cores, rank 0
    only; every step is a seeded node sample of the workload grid sized so the run lasts ~90 s."""
    if rank != 0:
        return 0
    import numpy as np

    import oracle

    X, IEN, g = load_reference(args.workload)
    nthreads = oracle.max_threads()
    sample = min(g["ngp"], args.ref_sample)
    rng = np.random.default_rng(7)
    times = []
    for step in range(args.warmup + args.steps):
        nodes = np.sort(rng.choice(g["ngp"], size=sample, replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        reference_sample(X, IEN, g, nodes, nthreads)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
        if step == 0:  # size the per-step sample so the whole run takes about 90 s
            per_step = 90.0 / (args.warmup + args.steps)
            sample = int(min(sample, max(256, sample / dt * per_step)))
    total = sum(times)
    value = sample * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": common_config(args.workload, X, IEN, g),
        "step": f"reference-rule distance + sign of {sample} seeded grid nodes (oracle, {nthreads} threads)",
        "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": nthreads, "kind": "port",
                         "sample": f"{sample} seeded grid nodes per step, reference-rule distance + sign"},
        "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def make_batch(name: str):
    """Meshes and grids of an uneven batch: batch256 = 256 meshes, seed 3 (icospheres L2-6 and
    8-32-blob marching-cubes meshes, 32..160 nodes on each grid's long axis); batchN = the first N."""
    from stl2sdf import DataImport, _native
    from workloads import synthetic

    count = int(name[len("batch"):] or 256)
    items = []
    for r in synthetic.uneven_batch(count, seed=3):
        X, IEN = DataImport.roundtrip_float32(*synthetic.batch_mesh(r))
        o, _, N, h, ngp = _native.grid_setup(X.min(0), X.max(0), r["K"] - 7, 3)
        items.append((X, IEN, o, h, N))
    desc = (f"{count} meshes, seed 3: even entries icospheres L2-6 (320-81920 tris), odd entries marching cubes of "
            f"8-32 Gaussian blobs at 32-320 cells (log-uniform); K nodes on each grid's long axis, K in [32, 160]")
    return items, desc


def run_batch(args, rank, world, local):
    """Uneven batch through sdfgpu_sdf_batch (host meshes in, host fields out), the meshes dealt to
    ranks by LPT.  Timed by the host clock around the call (the batch spans several streams and
    host threads), max over ranks."""
    import numpy as np
    import torch

    from stl2sdf import _native, sharding

    items, desc = make_batch(args.workload)
    ngps = [int(np.prod(np.asarray(m[4]) + 1)) for m in items]
    plan = sharding.lpt_assign([sharding.mesh_work(n, m[1].shape[0]) for n, m in zip(ngps, items)], world)

    held = []  # the page-locked tensors behind the numpy views, alive for the whole run

    def pinned(a):  # a numpy view of page-locked host memory holding a copy of a
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        held.append(t)
        return t.numpy()

    # inputs and outputs in page-locked host memory, as the single-mesh end-to-end arm uses
    mine = [(pinned(items[i][0]), pinned(items[i][1])) + tuple(items[i][2:]) for i in plan[rank]]
    outs = [pinned(np.empty(ngps[i])) for i in plan[rank]]
    ctx = _native.Context(local)
    dist_on = world > 1
    if dist_on:
        import torch.distributed as tdist

    def timed(k, **kw):
        if dist_on:
            tdist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        launches = 0
        for _ in range(k):
            ctx.sdf_batch(mine, out=outs, **kw)
            launches += ctx.stats()["launches"] + ctx.stats()["mesh_launches"]
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if dist_on:
            tt = torch.tensor([dt], dtype=torch.float64, device=f"cuda:{local}")
            tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
            dt = float(tt.item())
        return dt, launches

    t_tune = time.perf_counter()
    ctx.sdf_batch(mine, out=outs, streams=args.streams, autotune=True)  # first call: autotuning + allocation
    t_tune = time.perf_counter() - t_tune
    for _ in range(args.warmup - 1):
        ctx.sdf_batch(mine, out=outs, streams=args.streams, autotune=True)
    with ClockSampler(local) as clk:
        dt, launches = timed(args.steps, streams=args.streams, autotune=True)
    st = ctx.stats()
    one, _ = timed(1, streams=1, autotune=False)  # same batch, one stream, default tile
    # the same batch with the folds of all meshes in one persistent launch inside a CUDA graph
    ctx.sdf_batch(mine, out=outs, streams=args.streams, autotune=True, persistent=True)  # buffers
    pers, _ = timed(max(1, min(args.steps, 3)), streams=args.streams, autotune=True, persistent=True)
    # the same batch in the learned-radius form: every mesh trains its own network inside the call
    from stl2sdf import _native as _nat

    ctx.sdf_batch(mine, out=outs, streams=args.streams, autotune=True, mode=_nat.MODE_LEARNED)  # tuning, buffers
    lrn, _ = timed(1, streams=args.streams, autotune=True, mode=_nat.MODE_LEARNED)
    lst = ctx.stats()
    # ... and with every mesh's search in one persistent launch (two with the radius) in a CUDA graph
    ctx.sdf_batch(mine, out=outs, streams=args.streams, autotune=True, mode=_nat.MODE_LEARNED, persistent=True)
    lrp, _ = timed(1, streams=args.streams, autotune=True, mode=_nat.MODE_LEARNED, persistent=True)
    lpst = ctx.stats()
    total = sum(ngps)
    value = total * args.steps / dt
    line = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "meshes": len(items), "ngp": total,
                   "nel": int(sum(m[1].shape[0] for m in items)), "mode": "ref-rule", "streams": args.streams,
                   "l2": "inputs larger than L2 (sum of all fields)", "host_buffers": "page-locked",
                   "step": "sdfgpu_sdf_batch over every mesh: upload, LBVH, distance, sign, combine, fields to host",
                   "timing": "host clock around the call, barrier + device sync on both sides"},
        "e2e": {"value": value, "unit": "nodes/s",
                "h2d_bytes_per_step": int(sum(m[0].nbytes + m[1].nbytes for m in mine)),
                "d2h_bytes_per_step": int(8 * sum(ngps[i] for i in plan[rank]))},
        "gpu_launches": int(launches),
        "single_stream_default_tile": {"value": total / one, "s": one},
        "persistent_graph_form": {"value": total * max(1, min(args.steps, 3)) / pers,
                                  "note": "sdfgpu_sdf_batch_ex(persistent=1): every fold in one persistent launch, "
                                          "captured with the epilogues in one CUDA graph"},
        "learned_radius_form": {"value": total / lrn, "s": lrn, "train_ms_summed": lst["ms_train"],
                                "certified_fraction": lst["certified_nodes"] / max(1, lst["ngp"]),
                                "fallback_rate": lst["unbounded_fallbacks"] / max(1, lst["ngp"]),
                                "note": "SDFGPU_MODE_LEARNED: unbounded distances, one radius network trained per "
                                        "mesh inside the call (training time included)"},
        "learned_radius_persistent_form": {"value": total / lrp, "s": lrp, "train_ms_summed": lpst["ms_train"],
                                           "search_ms": lpst["ms_distance"],
                                           "certified_fraction": lpst["certified_nodes"] / max(1, lpst["ngp"]),
                                           "fallback_rate": lpst["unbounded_fallbacks"] / max(1, lpst["ngp"]),
                                           "note": "SDFGPU_MODE_LEARNED, sdfgpu_sdf_batch_ex(persistent=1): networks "
                                                   "trained while the items are prepared, every mesh's search in one "
                                                   "persistent launch inside a CUDA graph"},
        "first_call_s": t_tune,
        "stages_ms_summed": {k: st[k] for k in ("ms_mesh", "ms_tiles", "ms_fold", "ms_rows", "ms_parity", "ms_vote")},
        "counters_summed": {k: st[k] for k in ("tile_pairs", "fp64_evals", "row_hits", "undecided_nodes", "extra_rays",
                                                "winding_nodes", "knn_fallback_nodes", "launches", "mesh_launches")},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        nthreads = oracle.max_threads()
        rng = np.random.default_rng(42)
        picks = list(range(0, len(items), max(1, len(items) // 32)))
        t0, nodes_done = time.perf_counter(), 0
        for i in picks:
            X, IEN, o, h, N = items[i]
            nodes = np.sort(rng.choice(ngps[i], size=min(256, ngps[i]), replace=False)).astype(np.int64)
            oracle.distances(X, IEN, o, h, N, mode=0, nodes=nodes, nthreads=nthreads)
            oracle.signs(X, IEN, o, h, N, nodes=nodes, nthreads=nthreads)
            nodes_done += nodes.shape[0]
        cdt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": nodes_done / cdt, "unit": "nodes/s", "cores": nthreads, "kind": "port",
                                "sample": f"256 seeded nodes of each of {len(picks)} meshes (every "
                                          f"{max(1, len(items) // 32)}th), distance+sign, {cdt:.1f} s"}
    if dist_on:
        tdist.barrier()
        tdist.destroy_process_group()
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


class Arm:
    """One form of the SDF step (mode + whether the radius network is trained inside the step) on a
    resident mesh, timed with CUDA events on the context stream, L2 flushed between steps."""

    def __init__(self, ctx, stream, dX, dIEN, nnp, nel, g, out, flush, mode, train):
        self.ctx, self.stream, self.dX, self.dIEN, self.nnp, self.nel = ctx, stream, dX, dIEN, nnp, nel
        self.g, self.out, self.flush, self.mode, self.train = g, out, flush, mode, train
        self.launches = 0
        self.fold_ms = []
        self.train_ms = []

    def step(self):
        c, g = self.ctx, self.g
        c.set_mesh_device(self.dX.data_ptr(), self.nnp, self.dIEN.data_ptr(), self.nel)
        n = c.stats()["mesh_launches"]
        if self.train:
            c.train_radius(**TRAIN)
            st = c.stats()
            n += st["train_launches"]
            self.train_ms.append(st["ms_train"])
        c.sdf_device(g["origin"], g["h"], g["N"], self.out.data_ptr(), mode=self.mode)
        st = c.stats()
        self.fold_ms.append(st["ms_fold"])
        self.launches += n + st["launches"]

    def run(self, steps, warmup, dist_on=False, clock=None):
        import torch

        for _ in range(warmup):
            self.step()
            with torch.cuda.stream(self.stream):
                self.flush.fill_(1)
        torch.cuda.synchronize()
        self.launches, self.fold_ms, self.train_ms = 0, [], []
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        if dist_on:
            import torch.distributed as tdist

            tdist.barrier()
        torch.cuda.synchronize()
        if clock is not None:
            clock.__enter__()
        for s in range(steps):
            starts[s].record(self.stream)
            self.step()
            ends[s].record(self.stream)
            with torch.cuda.stream(self.stream):
                self.flush.fill_(s & 0xFF)
        torch.cuda.synchronize()
        if clock is not None:
            clock.__exit__()
        if dist_on:
            tdist.barrier()
        return sum(a.elapsed_time(b) for a, b in zip(starts, ends))


def e2e_run(ctx, X, IEN, g, mode, train, steps):
    """The same step through the C ABI with page-locked host buffers: H2D of X and IEN, training
    (learned form), every stage and the D2H of the sdf inside the timed region."""
    import ctypes

    import numpy as np
    import torch

    from stl2sdf import _native

    hX = torch.from_numpy(np.ascontiguousarray(X)).pin_memory()
    hIEN = torch.from_numpy(np.ascontiguousarray(IEN)).pin_memory()
    hout = torch.empty(g["ngp"], dtype=torch.float64).pin_memory()
    L = _native.lib()
    o = np.ascontiguousarray(g["origin"], np.float64)
    N = np.ascontiguousarray(g["N"], np.int64)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int64)
    loss = ctypes.c_float()

    def one():
        rc = L.sdfgpu_set_mesh(ctx.handle, ctypes.cast(hX.data_ptr(), dp), X.shape[0], ctypes.cast(hIEN.data_ptr(), ip),
                               IEN.shape[0])
        if not rc and train:
            rc = L.sdfgpu_train_radius(ctx.handle, TRAIN["coarse_n"], TRAIN["steps"], TRAIN["batch"], TRAIN["lr"],
                                       TRAIN["seed"], ctypes.byref(loss))
        rc = rc or L.sdfgpu_sdf(ctx.handle, o.ctypes.data_as(dp), g["h"], N.ctypes.data_as(ip), mode, 6, 30, 0.6, 1,
                                ctypes.cast(hout.data_ptr(), dp), None, None, None)
        if rc:
            raise _native.SdfGpuError(rc, L.sdfgpu_last_error(ctx.handle).decode())

    for _ in range(2):
        one()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    es.record(stream)
    for _ in range(steps):
        one()
    ee.record(stream)
    torch.cuda.synchronize()
    return es.elapsed_time(ee), hout, int(X.nbytes + IEN.nbytes), int(g["ngp"] * 8)


def distance_variants(ctx, X, IEN, g, reps=3, work=None, peak_tflops=None):
    """Distance-stage throughput (device time of sdfgpu_distances, mesh resident) of the reference
    rule (clamped), the true minimum clamped to h, the plain unbounded search and the learned-radius
    search (bit-identical to plain), with the network's training time and certified fraction."""
    ctx.set_mesh(X, IEN)
    out = {}

    def run(mode, learned=False):
        ms = []
        for _ in range(reps + 1):
            ctx.distances(g["origin"], g["h"], g["N"], mode, learned=learned)
            ms.append(ctx.stats()["ms_distance"])
        ms = sorted(ms[1:])[len(ms[1:]) // 2]
        st = ctx.stats()
        return {"nodes_per_s": g["ngp"] / (ms / 1e3), "ms": ms, "bvh_visits_per_node": st["bvh_visits"] / g["ngp"],
                "fp64_steps_per_node": st["fp64_evals"] / g["ngp"]}

    out["ref_rule"] = run(0)
    out["exact_h_bounded"] = run(1)
    out["plain_unbounded"] = run(2)
    ctx.train_radius(**TRAIN)
    st = ctx.stats()
    train_ms = st["ms_train"]
    out["learned_unbounded"] = run(2, learned=True)
    st = ctx.stats()
    out["learned_unbounded"].update({"certified_fraction": st["certified_nodes"] / g["ngp"],
                                     "fallback_nodes": st["unbounded_fallbacks"],
                                     "fallback_rate": st["unbounded_fallbacks"] / g["ngp"], "train_ms": train_ms,
                                     "train_loss": st["radius_loss"], "train": dict(TRAIN)})
    # the same search with every radius infinite: what the network's bound adds
    ctx.set_radius_margin(float("inf"), 0.0)
    out["learned_search_without_network"] = run(2, learned=True)
    ctx.set_radius_margin()
    lu = out["learned_unbounded"]
    lu["ms_with_training"] = lu["ms"] + train_ms
    out["learned_vs_plain_unbounded"] = out["plain_unbounded"]["ms"] / lu["ms"]
    out["network_gain"] = out["learned_search_without_network"]["ms"] / lu["ms"]
    out["learned_with_training_vs_plain_unbounded"] = out["plain_unbounded"]["ms"] / lu["ms_with_training"]
    if work is not None and peak_tflops:
        # FP32 roofline of the distance stage alone: F_pt |D*| per node (clamped forms) or F_pt |D*_u|
        # (unbounded forms), against the measured FP32 peak
        for k, w in (("ref_rule", work["mean_W_dist_flop"]), ("exact_h_bounded", work["mean_W_dist_flop"]),
                     ("plain_unbounded", work["mean_W_dist_unbounded_flop"]),
                     ("learned_unbounded", work["mean_W_dist_unbounded_flop"])):
            bound = peak_tflops * 1e12 / w
            out[k]["roofline_fp32"] = {"mean_W_flop_per_node": w, "roofline_nodes_per_s": bound,
                                       "frac": out[k]["nodes_per_s"] / bound}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 20 for blobs256/gyroid320, 100 for the small grids, 3 for batches)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sdfgpu", choices=["sdfgpu", "reference"])
    ap.add_argument("--workload", default="blobs256")
    ap.add_argument("--split", default="copies", choices=["copies", "zslab"],
                    help="multi-GPU: a copy of the workload per rank (weak) or z-slabs of one grid (strong)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--variant-steps", type=int, default=3, help="timed steps of the plain and ref-rule SDF forms")
    ap.add_argument("--ref-sample", type=int, default=1 << 14)
    ap.add_argument("--streams", type=int, default=8, help="batch workloads: worker streams")
    ap.add_argument("--once", action="store_true",
                    help="run one untimed learned-form step (set_mesh, train_radius, sdf) and exit: the "
                         "kernel sequence a profiler captures")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.steps is None:
        args.steps = 3 if args.workload.startswith("batch") else (20 if args.workload in ("blobs256", "gyroid320") else 100)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch

    from stl2sdf import _native

    torch.cuda.set_device(local)
    dist_on = world > 1
    if dist_on:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.workload.startswith("batch"):
        return run_batch(args, rank, world, local)
    if args.once:
        X, IEN, g = load_gpu(args.workload, local)
        ctx = _native.Context(local)
        ctx.set_mesh(X, IEN)
        ctx.train_radius(**TRAIN)
        ctx.sdf(g["origin"], g["h"], g["N"], mode=_native.MODE_LEARNED)
        print(json.dumps({"once": args.workload, "ms_distance": ctx.stats()["ms_distance"]}), flush=True)
        ctx.close()
        return 0
    if args.split == "zslab" and dist_on:
        return run_zslab(args, rank, world, local)
    X, IEN, g = load_gpu(args.workload, local)
    ngp = g["ngp"]
    ctx = _native.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{local}")
    dev = torch.device(f"cuda:{local}")
    dX = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
    dIEN = torch.from_numpy(np.ascontiguousarray(IEN)).to(dev)
    out = torch.empty(ngp, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    # the project's autotuner picks the reference-rule tile and the unbounded search's warp brick for
    # this mesh and grid (untimed, once)
    ctx.set_mesh(X, IEN)
    tile, _ = ctx.autotune(g["origin"], g["h"], g["N"], mode=0)
    brick, _ = ctx.autotune(g["origin"], g["h"], g["N"], mode=2)
    torch.cuda.synchronize()

    def arm(mode, train):
        return Arm(ctx, stream, dX, dIEN, X.shape[0], IEN.shape[0], g, out, flush, mode, train)

    learned = arm(_native.MODE_LEARNED, True)
    clk = ClockSampler(local)
    t_wall = time.perf_counter()
    dev_ms = learned.run(args.steps, args.warmup, dist_on, clock=clk)
    wall = time.perf_counter() - t_wall
    if dist_on:
        tt = torch.tensor([dev_ms], dtype=torch.float64, device=dev)
        tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
        dev_ms = float(tt.item())
    value = ngp * args.steps * world / (dev_ms / 1e3)
    stats = ctx.stats()
    sdf_learned = out.cpu().numpy()

    e2e_steps = max(3, min(args.steps, 10))
    e2e_ms, hout, h2d, d2h = e2e_run(ctx, X, IEN, g, _native.MODE_LEARNED, True, e2e_steps)
    if dist_on:
        tt = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e_value = ngp * e2e_steps * world / (e2e_ms / 1e3)
    assert np.array_equal(hout.numpy(), sdf_learned), "e2e and device-resident results differ"

    forms = {}
    if not args.no_variants:
        for name, mode in (("plain_unbounded", _native.MODE_UNBOUNDED), ("ref_rule", _native.MODE_REF_RULE)):
            a = arm(mode, False)
            ms = a.run(args.variant_steps, 1, dist_on)
            f = {"value": ngp * args.variant_steps * world / (ms / 1e3), "ms_per_step": ms / args.variant_steps,
                 "steps": args.variant_steps, "gpu_launches": a.launches}
            if name == "plain_unbounded":
                f["sdf_equal_to_learned"] = bool(np.array_equal(out.cpu().numpy(), sdf_learned))
            if name == "ref_rule":
                ems, _, _, _ = e2e_run(ctx, X, IEN, g, mode, False, e2e_steps)
                f["e2e"] = ngp * e2e_steps * world / (ems / 1e3)
                f["fold_ms"] = sum(a.fold_ms) / max(1, len(a.fold_ms))
            forms[name] = f
        forms["learned_vs_plain_unbounded_sdf"] = value / forms["plain_unbounded"]["value"]

    # HBM roofline of the dominant kernel (k_unbounded, the packet search bounded by the learned
    # radius): algorithmic bytes per launch = the radius read and the distance written per node
    # (4 + 8 B) + the triangle data read once (FP32 vertices 48 B, FP64 record 352 B) + the LBVH read
    # once (64 B node and 128 B of oriented child boxes per inner node).
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    search_ms = sum(learned.fold_ms) / len(learned.fold_ms)
    alg_bytes = 12 * ngp + 400 * IEN.shape[0] + 192 * (IEN.shape[0] - 1)
    achieved = alg_bytes / (search_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(args.workload, {}).get("k_unbounded")

    # FP32 roofline of the same kernel (the path's real bound: CUDA-core arithmetic): the oracle's
    # work model gives the algorithmic FP32 FLOPs per node of the unbounded nearest search, F_pt |D*_u|
    # (profiles/roofline.json, made by oracle/work_model.py); the peak is measured here.
    import workloads

    roof32 = None
    rpath = os.path.join(ROOT, "profiles", "roofline.json")
    wm = json.load(open(rpath)).get(args.workload) if os.path.exists(rpath) else None
    p32 = workloads.measure_fp32_peak(local)
    if wm:
        w = wm["mean_W_dist_unbounded_flop"]
        bound = p32 * 1e12 / w
        ach = ngp / (search_ms / 1e3)
        roof32 = {"bound": "fp32", "kernel": "k_unbounded", "mean_W_flop_per_node": w, "F_pt": wm["F_pt"],
                  "work_sample": wm["sample"], "peak": p32, "unit": "TFLOP/s", "peak_source": "measured (FMA probe)",
                  "achieved": ach * w / 1e12, "roofline_nodes_per_s": bound, "frac": ach / bound,
                  "step_frac": value / world / (p32 * 1e12 / wm["mean_W_flop"]) if wm.get("mean_W_flop") else None}

    cfg = common_config(args.workload, X, IEN, g)
    line = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "step": ("set_mesh_device (triangle records + LBVH) + train_radius (coarse exact grid + "
                 f"{TRAIN['steps']} Adam steps) + sdf_device(SDFGPU_MODE_LEARNED: learned-radius distance, sign, combine)"),
        "tuning": {"tile": [int(v) for v in tile], "brick": [int(v) for v in brick], "train": dict(TRAIN)},
        "e2e": {"value": e2e_value, "unit": "nodes/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "gpu_launches": int(learned.launches),
        "roofline": {"bound": "hbm", "kernel": "k_unbounded", "achieved": achieved, "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": int(alg_bytes), "ms_per_launch": search_ms},
        "roofline_fp32": roof32,
        "train_ms_per_step": sum(learned.train_ms) / max(1, len(learned.train_ms)),
        "stages_ms": {k: stats[k] for k in ("ms_mesh", "ms_fold", "ms_rows", "ms_parity", "ms_vote", "ms_distance",
                                             "ms_sign")},
        "counters": {k: stats[k] for k in ("fp64_evals", "certified_nodes", "unbounded_fallbacks", "bvh_visits",
                                            "row_hits", "undecided_nodes", "extra_rays", "winding_nodes")},
        "fallback_rate": stats["unbounded_fallbacks"] / ngp,
        "sdf_forms": forms,
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    if not args.no_variants:
        line["distance_variants"] = distance_variants(ctx, X, IEN, g, work=wm, peak_tflops=p32)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(X, IEN, g)
    if dist_on:
        tdist.barrier()
        tdist.destroy_process_group()
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_zslab(args, rank, world, local):
    """--split zslab: one grid of the workload cut into z-slabs (stl2sdf.sharding.zslab_bounds), rank r
    computing slab r with sdfgpu_sdf_slab_device (reference-rule sdf) and rank 0 gathering the slabs
    over NCCL into the full field.  Value = nodes of the grid / max-over-ranks device time of
    (compute + gather)."""
    import numpy as np
    import torch
    import torch.distributed as tdist

    from stl2sdf import _native, sharding

    X, IEN, g = load_gpu(args.workload, local)
    dev = torch.device(f"cuda:{local}")
    ctx = _native.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    bounds = [sharding.zslab_bounds(int(g["N"][2]) + 1, world, r) for r in range(world)]
    if any(b is None for b in bounds):
        raise SystemExit("zslab: more ranks than z layers")
    k0, k1 = bounds[rank]
    layer = int((g["N"][0] + 1) * (g["N"][1] + 1))
    cap = max(b1 - b0 + 1 for b0, b1 in bounds) * layer
    mine = torch.zeros(cap, dtype=torch.float64, device=dev)
    parts = [torch.empty(cap, dtype=torch.float64, device=dev) for _ in range(world)] if rank == 0 else None
    ctx.set_mesh(X, IEN)

    def step():
        ctx.sdf_slab_device(g["origin"], g["h"], g["N"], k0, k1, mine.data_ptr(), mode=_native.MODE_REF_RULE)
        torch.cuda.current_stream(dev).wait_stream(stream)
        tdist.gather(mine, parts, dst=0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    tdist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(torch.cuda.current_stream(dev))
    torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    tdist.all_reduce(ms, op=tdist.ReduceOp.MAX)
    ms = float(ms.item())
    if rank == 0:
        full = torch.cat([parts[r][: (b1 - b0 + 1) * layer] for r, (b0, b1) in enumerate(bounds)]).cpu().numpy()
        assert full.shape[0] == g["ngp"]
        line = {"metric": METRIC, "value": g["ngp"] * args.steps / (ms / 1e3), "unit": "nodes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": common_config(args.workload, X, IEN, g),
                "step": "reference-rule sdf of one z-slab per rank (sdfgpu_sdf_slab_device) + NCCL gather to rank 0",
                "slabs": [list(b) for b in bounds]}
    tdist.barrier()
    tdist.destroy_process_group()
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
