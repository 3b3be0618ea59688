#!/usr/bin/env python
"""Build + closest-hit trace throughput on B200 (one JSON line on rank 0).

A step is one pass of the hot path over one batch of synthetic input: build a
BVH over the mesh, then trace every ray of the batch. The default workload is
the 4,194,304-triangle clustered scene with 16,777,216 incoherent rays
(1024 Gaussian clusters, sigma 0.02, vertex offsets +-0.005; origins uniform in
the scene box, directions uniform on the sphere; 60-bit Morton codes).

value      build throughput, Mtris/s, inputs resident in HBM (CUDA events);
           trace_mrays_s gives the closest-hit throughput of the same steps.
           The context is autotuned once during warm-up (hp_autotune: sort CTA
           size, tracer CTAs per SM and stack depth, ray Morton order; none of
           them changes a result); trace_untuned_mrays_s is the same trace
           with the default choices.
e2e        the same metrics through the C ABI with pinned host buffers: the
           H2D copy of the mesh plus the build (and a read-back of the node
           counts), then hp_trace_host over the host ray and result buffers
           (every ray uploaded and every hit record downloaded, in chunks whose
           copies overlap the traces of their neighbours).
roofline   the radix-sort phase of the build (HBM-bound): the algorithmic bytes of
           an 8-bit LSD sort, n * P * 2 * (K + 4) (P = ceil(bits / 8) passes), over the
           summed CUDA-event durations of its kernels (for 60-bit keys three
           LSD passes and the segment sort);
           roofline.phases gives every HBM-bound build phase with its
           algorithmic bytes (scene box + boxes + Morton, the sort), and
           large.roofline_phases_lbvh the same plus the refit climb on the
           33,554,432-triangle LBVH.
Multi-GPU: one process per GPU (torchrun). Default (--parallel rays): one
scene, its rays split contiguously across the ranks; every rank builds the
BVH from the same input (no collective on the data path), or with
--bvh-broadcast 1 rank 0 builds it and broadcasts nodes, Woop rows and
triangle indices over NCCL; value = triangles of the one scene over the max
build time, trace_mrays_s = all rays over the max trace time (strong scaling).
--parallel replicas: every rank builds and traces a scene of its own (weak
scaling). Times are the max over ranks.

--impl reference times the CPU restatement of the same algorithms (the
reference has no CPU path of its own) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mtris/s build + Mrays/s closest-hit; batched & fwd+bwd vs plain, same B200"
SEED = 0xC0FFEE

CONFIGS = {
    "ploc4m": dict(workload="clustered 4,194,304 tris (1024 clusters), 16,777,216 sphere rays, 60-bit",
                   mesh="clustered", n=4194304, rays=16777216, bits=60, method="ploc", config_id=1),
    "lbvh64k": dict(workload="uniform 65,536 tris, 1,048,576 targeted rays, 30-bit", mesh="uniform",
                    n=65536, rays=1048576, bits=30, method="lbvh", config_id=0),
    # the headline scene built as an LBVH (for profiling the refit climb)
    "lbvh4m": dict(workload="clustered 4,194,304 tris (1024 clusters), 16,777,216 sphere rays, 60-bit, LBVH",
                   mesh="clustered", n=4194304, rays=16777216, bits=60, method="lbvh", config_id=1),
}
DEFAULT_CONFIG = "ploc4m"


def make_inputs(cfg, rank, library_free=False):
    """The workload's mesh and rays (rank > 0: another scene of the same size,
    for replicas). library_free: the oracle's copy of the generators, so that
    the CPU arm never loads the GPU library (same bytes)."""
    if library_free:
        import oracle
        gen = oracle.gen
    else:
        import hippie_b200 as hp
        gen = hp.gen
    seed = SEED + cfg["config_id"] + 1000 * rank
    if cfg["mesh"] == "uniform":
        v, t = gen.uniform_mesh(seed, cfg["n"], 0.01)
        rays = gen.rays_targeted(seed + 1, cfg["rays"], -0.5, 1.5)
    else:
        v, t = gen.clustered_mesh(seed, cfg["n"], 1024, 0.02, 0.005)
        box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
        rays = gen.rays_sphere(seed + 1, cfg["rays"], box)
    return v, t, rays


def build_params(cfg):
    import hippie_b200 as hp
    kw = dict(method=cfg["method"], morton_bits=cfg["bits"])
    if cfg["method"] == "ploc":
        kw.update(ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0)
    return hp.BuildParams(**kw)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), line.strip()))

    def window(self, t0, t1):
        self.t0, self.t1 = t0, t1

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for ts, line in self.samples:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append((ts, parts))
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        inside = [r for r in rows if self.t0 is not None and self.t0 - 0.05 <= r[0] <= self.t1 + 0.05]
        use = inside or rows
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(p[1]) for _, p in use if num(p[1]) is not None]
        mx = [num(p[2]) for _, p in use if num(p[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, p in use for i in range(4) if p[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(use), "in_window": bool(inside)}


def peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def committed_traffic(name):
    """DRAM bytes per launch of a kernel from a committed ncu summary, if present."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(name)
        except ValueError:
            return None
    return None


def profile_phases(ctx, fn):
    """Run fn() with the context's phase events on; {phase: [ms per occurrence]}."""
    import ctypes as C
    import torch
    from hippie_b200 import _lib
    lib = _lib.load()
    lib.hp_profile_reset(ctx.h)
    lib.hp_profile_enable(ctx.h, 1)
    fn()
    torch.cuda.synchronize()
    out = {}
    for i in range(1, lib.hp_profile_count(ctx.h)):
        nm = C.create_string_buffer(64)
        ms = C.c_float()
        lib.hp_profile_get(ctx.h, i, nm, 64, C.byref(ms))
        out.setdefault(nm.value.decode(), []).append(ms.value)
    lib.hp_profile_enable(ctx.h, 0)
    lib.hp_profile_reset(ctx.h)
    return out


def phase_rooflines(n, bits, phases, peak):
    """HBM fractions of the build phases with their algorithmic bytes
    (K = key bytes, AABB = 24 B):
      scene box + boxes + Morton  36 n + n (12 idx + 36 verts + K + 4)
      radix sort                  n * P * 2 * (K + 4), P = ceil(bits / 8)
      refit (LBVH climb)          24 (2n-2) + 24 (n-1) + 8 (n-1) + 4 (2n-1) + 8 (n-1)
    over the phases' CUDA-event times. The refit is the two climb kernels
    (CTA-local nodes in shared memory, then the nodes that cross CTA ranges);
    its collapse-cost and state writes are not in the formula."""
    kb = 4 if bits <= 32 else 8
    passes = (bits + 7) // 8
    rows = []

    def add(name, nbytes, ms, extra=None):
        if ms <= 0:
            return
        a = nbytes / (ms * 1e-3) / 1e9
        r = {"phase": name, "bytes": int(nbytes), "ms": round(ms, 5), "achieved_gbs": round(a, 1),
             "frac": round(a / peak, 4)}
        if extra:
            r.update(extra)
        rows.append(r)

    if "boxes" in phases and "morton" in phases:
        add("scene box + boxes + Morton", 36 * n + n * (12 + 36 + kb + 4),
            sum(phases["boxes"]) + sum(phases["morton"]))
    if "sort_pass" in phases:
        seg = sum(phases.get("sort_segments", []))
        name = (f"radix sort ({len(phases['sort_pass'])} passes + segment sort)" if seg > 0 else
                f"radix sort ({len(phases['sort_pass'])} passes)")
        add(name, n * passes * 2 * (kb + 4), sum(phases["sort_pass"]) + seg,
            {"per_pass_ms": round(float(np.mean(phases["sort_pass"])), 5), "segments_ms": round(seg, 5)})
    if "climb" in phases:
        refit = 24 * (2 * n - 2) + 24 * (n - 1) + 8 * (n - 1) + 4 * (2 * n - 1) + 8 * (n - 1)
        local = sum(phases.get("climb_local", []))
        add("refit (LBVH climb)", refit, local + sum(phases["climb"]),
            {"local_ms": round(local, 5), "frontier_ms": round(sum(phases["climb"]), 5)})
    return rows


def oracle_build(cfg, v, t):
    """The CPU restatement of the workload's builder (LBVH or PLOC, same parameters)."""
    import oracle
    if cfg["method"] == "ploc":
        return oracle.build_ploc(v, t, bits=cfg["bits"], radius=16, max_radius=256)
    return oracle.build_lbvh(v, t, bits=cfg["bits"])


def cpu_sample(cfg, v, t, budget_s):
    """Largest prefix of the mesh whose oracle build fits about budget_s seconds."""
    n = cfg["n"]
    m = min(n, 131072)
    t0 = time.perf_counter()
    oracle_build(cfg, v, np.ascontiguousarray(t[:m]))
    dt = time.perf_counter() - t0
    return int(min(n, max(m, m * budget_s / max(dt, 1e-4))))


def cpu_baseline(cfg, v, t, rays, budget_s=20.0):
    """Time the CPU restatement (oracle) on a bounded sample of the workload."""
    import oracle
    oracle.load()
    cores = os.cpu_count() or 1
    m = cpu_sample(cfg, v, t, 0.4 * budget_s)
    tt = np.ascontiguousarray(t[:m])
    t0 = time.perf_counter()
    r = oracle_build(cfg, v, tt)
    b_s = time.perf_counter() - t0
    k = min(rays.shape[0], 1 << 18)
    t0 = time.perf_counter()
    oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays[:k])
    tr_s = time.perf_counter() - t0
    return {"value": m / b_s / 1e6, "unit": "Mtris/s", "cores": cores, "kind": "port",
            "sample": f"{cfg['method'].upper()} build of the first {m} triangles; trace of {k} rays on that BVH",
            "trace_mrays_s": k / tr_s / 1e6}


def reference_kernels(cfg, V, T, R, v, reps=3):
    """The reference's own CUDA kernels (oracle/_ref, built from its sources) on the
    same device inputs: summed kernel time of the build and the tracer's rate.
    Reported beside the product's numbers; None where the harness was not built."""
    import oracle.ref_harness as rh
    if not rh.available():
        return None
    import torch
    box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    kw = dict(method=cfg["method"], bits=cfg["bits"])
    if cfg["method"] == "ploc":
        kw.update(radius=16, max_radius=256)
    builds = [rh.build(V, T, box, **kw) for _ in range(reps)]
    b = builds[-1]
    nodes = torch.from_numpy(b["nodes"]).cuda()
    woop = torch.from_numpy(b["woop"]).cuda()
    tri = torch.from_numpy(b["tri_idx"]).cuda()
    secs = [rh.trace(nodes, woop, tri, R)[1] for _ in range(reps)]
    n, nr = T.shape[0], R.shape[0]
    bs = float(np.median([x["seconds"] for x in builds]))
    return {"build_ms": 1e3 * bs, "mtris_s": n / bs / 1e6, "trace_mrays_s": nr / float(np.median(secs)) / 1e6,
            "note": "reference kernels compiled from its sources for sm_100a; CUB radix sort in place of its "
                    "own sort; times are sums of per-kernel CUDA events as the reference reports them"}


def _events(torch, k):
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]


def extra_batched(ctx, steps=3, num_meshes=2048, seed=SEED + 2, rank=0, world=1):
    """Batched build + trace of 2048 meshes (log-uniform 256..262,144 triangles,
    the uniform generator; 4 rays per triangle, origins uniform in [-0.5,1.5]^3,
    directions uniform on the sphere) against the same meshes and rays built and
    traced one mesh at a time through the plain path: as host-loop launches, and
    with those per-mesh launches captured into one CUDA graph. The launch
    choices are autotuned on the batch first and used by both. Under torchrun
    the meshes are split across ranks by LPT (no data-path collective) and the
    times are the max over ranks."""
    import torch
    import hippie_b200 as hp
    from hippie_b200.shard import lpt_partition, mesh_work
    rng = np.random.default_rng(seed)
    all_sizes = np.round(np.exp(rng.uniform(np.log(256), np.log(262144), num_meshes))).astype(np.int64)
    mine = lpt_partition(mesh_work(all_sizes, 4 * all_sizes), world)[rank]
    sizes = all_sizes[mine]
    num_meshes = len(mine)
    box = np.array([-0.5, -0.5, -0.5, 1.5, 1.5, 1.5], np.float32)
    meshes, counts = [], []
    for j, m in enumerate(mine):
        v, t = hp.gen.uniform_mesh(seed + 17 * int(m), int(sizes[j]), 0.01)
        meshes.append((torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()))
        counts.append(4 * int(sizes[j]))
    R_total = int(sum(counts))
    R = torch.empty((max(R_total, 1), 8), dtype=torch.float32, device="cuda")
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    for j, m in enumerate(mine):
        R[off[j]:off[j + 1]] = torch.from_numpy(hp.gen.rays_sphere(seed + 17 * int(m) + 5, counts[j], box)).cuda()
    p = hp.BuildParams(method="lbvh", morton_bits=30)
    res_plain = torch.zeros((R_total, 4), dtype=torch.int32, device="cuda")
    res_batch = torch.zeros((R_total, 4), dtype=torch.int32, device="cuda")
    bvhs = [hp.BVH(ctx) for _ in range(num_meshes)]
    views = [(R[off[m]:off[m + 1]], res_plain[off[m]:off[m + 1]]) for m in range(num_meshes)]

    def plain():
        for m in range(num_meshes):
            ctx.build(meshes[m][0], meshes[m][1], p, bvh=bvhs[m])
            ctx.trace(bvhs[m], views[m][0], results=views[m][1])

    s = torch.cuda.Stream()
    batch = hp.Batch(ctx, meshes, counts, p)
    with torch.cuda.stream(s):
        plain()  # allocates every per-mesh BVH once
        batch.build_trace(R, results=res_batch)
        torch.cuda.synchronize()
        ctx.check()
        # Autotuned launch choices for this batch (result-neutral): the sort CTA
        # size, the tracer's CTAs per SM and shared-stack depth, timed on the
        # batched build + trace itself (direct launches: a CUDA graph keeps the
        # launch choices it was captured with); the per-mesh baseline below
        # uses the same choices. Ray-order tracing is not a batch option.
        cand = [dict(sort_block=sb, trace_stack=st, trace_ctas_per_sm=ct, trace_sorted=0)
                for sb in (512, 256) for st in (8, 16, 32) for ct in (0, 6, 4)]
        times = []
        for c in cand:
            ctx.set_tune(**c)
            batch.build_trace(R, results=res_batch, graph=False)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            batch.build_trace(R, results=res_batch, graph=False)
            e1.record(s)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        tuned = cand[int(np.argmin(times))]
        ctx.set_tune(**tuned)
        batch.close()  # a fresh batch captures its graph with the tuned choices
        batch = hp.Batch(ctx, meshes, counts, p)
        batch.build_trace(R, results=res_batch)
        torch.cuda.synchronize()
        ctx.check()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            plain()
        ev_loop, ev_graph, ev_batch = _events(torch, steps), _events(torch, steps), _events(torch, steps)
        for k in range(steps):
            ev_loop[k][0].record(s)
            plain()
            ev_loop[k][1].record(s)
        for k in range(steps):
            ev_graph[k][0].record(s)
            g.replay()
            ev_graph[k][1].record(s)
        for k in range(steps):
            ev_batch[k][0].record(s)
            batch.build_trace(R, results=res_batch)
            ev_batch[k][1].record(s)
        # build and trace separately, for the split
        batch.build()
        eb = _events(torch, 2)
        eb[0][0].record(s)
        batch.build()
        eb[0][1].record(s)
        eb[1][0].record(s)
        batch.trace(R, results=res_batch)
        eb[1][1].record(s)
    torch.cuda.synchronize()
    ctx.check()
    same = bool(torch.equal(res_plain, res_batch))
    t = torch.tensor([float(np.median([a.elapsed_time(b) for a, b in ev_loop])),
                      float(np.median([a.elapsed_time(b) for a, b in ev_graph])),
                      float(np.median([a.elapsed_time(b) for a, b in ev_batch])),
                      eb[0][0].elapsed_time(eb[0][1]), eb[1][0].elapsed_time(eb[1][1]),
                      0.0 if same else 1.0], device="cuda")
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_loop, t_graph, t_batch, t_build, t_trace, bad = t.tolist()
    tris, rays = int(all_sizes.sum()), int(4 * all_sizes.sum())
    out = {"workload": f"{len(all_sizes)} meshes, {tris} triangles (log-uniform 256..262144), "
                       f"{rays} sphere rays", "triangles": tris, "rays": rays,
           "plain_host_loop_ms": t_loop, "plain_graph_ms": t_graph, "batched_ms": t_batch,
           "speedup_vs_plain_host_loop": t_loop / t_batch, "speedup_vs_plain_graph": t_graph / t_batch,
           "batched_build_ms": t_build, "batched_trace_ms": t_trace,
           "batched_mtris_s": tris / t_batch / 1e3, "batched_mrays_s": rays / t_batch / 1e3,
           "results_identical": bad == 0.0, "sharding": f"LPT over {world} rank(s), max over ranks",
           "autotuned": {"choice": tuned, "candidates": len(cand),
                         "applied": "batched and per-mesh runs use the chosen launch choices"}}
    del g
    batch.close()
    ctx.reset_tune()
    return out


def extra_differentiable(ctx, steps=10, seed=SEED + 3):
    """Heightfield of 512 x 1024 vertices (1,045,506 triangles, 16 sinusoids),
    4,194,304 downward rays on a jittered 2048 x 2048 grid, loss weights
    w ~ N(0,1): forward trace, adjoint into vertex gradients, refit after a
    vertex step. Ratio (forward + adjoint) / forward on CUDA events."""
    import torch
    import hippie_b200 as hp
    v, t = hp.gen.heightfield(seed, 512, 1024, 1.0, 2.0, 16)
    rays = hp.gen.rays_grid_down(seed + 1, 2048, 2048, 1.0, 2.0, 1.0)
    w = np.random.default_rng(seed + 2).standard_normal((rays.shape[0], 3)).astype(np.float32)
    V, T, R, W = (torch.from_numpy(x).cuda() for x in (v, t, rays, w))
    p = hp.BuildParams(method="lbvh", morton_bits=60)
    bvh = ctx.build(V, T, p)
    res = torch.zeros((R.shape[0], 4), dtype=torch.int32, device="cuda")
    grad = torch.zeros_like(V)
    s = torch.cuda.current_stream()
    for _ in range(3):
        ctx.trace(bvh, R, results=res)
        grad.zero_()
        ctx.adjoint(V, T, R, res, W, dl_dverts=grad)
        ctx.refit(bvh, V, T)
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(steps)]
    for k in range(steps):
        ev[k][0].record(s)
        ctx.trace(bvh, R, results=res)
        ev[k][1].record(s)
        grad.zero_()
        ev[k][2].record(s)
        ctx.adjoint(V, T, R, res, W, dl_dverts=grad)
        ev[k][3].record(s)
        ctx.refit(bvh, V, T)
        ev[k][4].record(s)
    torch.cuda.synchronize()
    ctx.check()
    fwd = float(np.median([e[0].elapsed_time(e[1]) for e in ev]))
    adj = float(np.median([e[2].elapsed_time(e[3]) for e in ev]))
    ref = float(np.median([e[3].elapsed_time(e[4]) for e in ev]))
    return {"workload": "heightfield 512x1024 (1,045,506 triangles), 4,194,304 downward rays",
            "forward_ms": fwd, "adjoint_ms": adj, "refit_ms": ref, "fwd_plus_adjoint_over_fwd": (fwd + adj) / fwd,
            "hits": int((res[:, 0] >= 0).sum())}


def extra_large(ctx, steps=3, seed=SEED + 4):
    """33,554,432 triangles (16,777,216 from the uniform generator interleaved with
    16,777,216 from the clustered one), LBVH 60-bit then ATR (treelet 9, 2
    iterations); 64 Mi rays: 32 Mi pinhole primaries on an 8192 x 4096 grid
    (camera at (0.5, 0.5, -1.5) looking at the unit box, 45 degree field of view,
    pixel-table order) and 32 Mi rays from origins uniform in the scene box with
    directions uniform on the sphere, traced plain and in ray Morton order."""
    import torch
    import hippie_b200 as hp
    half = 1 << 24
    v1, t1 = hp.gen.uniform_mesh(seed, half, 0.01)
    v2, t2 = hp.gen.clustered_mesh(seed + 1, half, 1024, 0.02, 0.005)
    tris = np.empty((2 * half, 3), np.int32)
    tris[0::2] = t1
    tris[1::2] = t2 + v1.shape[0]
    verts = np.concatenate([v1, v2])
    del v1, v2, t1, t2
    V, T = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    box = np.concatenate([verts.min(0), verts.max(0)]).astype(np.float32)
    del verts, tris
    n = 2 * half
    w, h = 8192, 4096
    pos = np.array([0.5, 0.5, -1.5], np.float32)
    m = hp.camera_screen_to_world(pos, [0.0, 0.0, 1.0], 45.0, w, h, 0.01, 100.0)
    table = torch.from_numpy(hp.pixel_table(w, h)).cuda()
    prim = ctx.primary_rays(pos, m, w, h, index_to_pixel=table)
    sec = torch.from_numpy(hp.gen.rays_sphere(seed + 2, w * h, box)).cuda()
    res = torch.zeros((w * h, 4), dtype=torch.int32, device="cuda")
    p_atr = hp.BuildParams(method="atr", morton_bits=60, atr_treelet=9, atr_iterations=2)
    p_lbvh = hp.BuildParams(method="lbvh", morton_bits=60)
    lb = ctx.build(V, T, p_lbvh)
    at = ctx.build(V, T, p_atr)
    s = torch.cuda.current_stream()
    ctx.trace(at, prim, results=res)
    ctx.trace_sorted(at, sec, results=res)
    torch.cuda.synchronize()
    ctx.check()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(7)] for _ in range(steps)]
    for k in range(steps):
        e = ev[k]
        e[0].record(s)
        ctx.build(V, T, p_lbvh, bvh=lb)
        e[1].record(s)
        ctx.build(V, T, p_atr, bvh=at)
        e[2].record(s)
        ctx.primary_rays(pos, m, w, h, index_to_pixel=table, out=prim)
        e[3].record(s)
        ctx.trace(at, prim, results=res)
        e[4].record(s)
        ctx.trace(at, sec, results=res)
        e[5].record(s)
        ctx.trace_sorted(at, sec, results=res)
        e[6].record(s)
    torch.cuda.synchronize()
    ctx.check()

    def med(a, b):
        return float(np.median([e[a].elapsed_time(e[b]) for e in ev]))

    t_lbvh, t_atr, t_gen, t_prim, t_sec, t_sort = (med(0, 1), med(1, 2), med(2, 3), med(3, 4), med(4, 5),
                                                   med(5, 6))
    # Build-phase roofline fractions of the LBVH (boxes + Morton, sort, refit
    # climb) from per-phase CUDA events of one more build; the ATR stage's
    # treelet kernels are instruction-bound and reported by time only.
    peak, peak_kind = peak_hbm()
    ph = profile_phases(ctx, lambda: ctx.build(V, T, p_lbvh, bvh=lb))
    ph_atr = profile_phases(ctx, lambda: ctx.build(V, T, p_atr, bvh=at))
    # Traversal is latency- and L2-bound: its HBM fraction counts only the
    # ray and result bytes it must move (32 B in, 16 B out per ray).
    io = 48 * w * h
    trace_roof = {"bound": "latency / L2 (BVH of 33.5 M triangles, about 1.3 GB, exceeds the 126 MB L2)",
                  "io_bytes_per_trace": io,
                  "primary_io_frac": io / (t_prim * 1e-3) / 1e9 / peak,
                  "secondary_io_frac": io / (t_sec * 1e-3) / 1e9 / peak,
                  "secondary_sorted_io_frac": io / (t_sort * 1e-3) / 1e9 / peak}
    return {"workload": "33,554,432 tris (uniform + clustered, interleaved), LBVH 60-bit + ATR treelet 9 x 2; "
                        "32Mi pinhole primaries (8192x4096) + 32Mi sphere rays",
            "roofline_phases_lbvh": phase_rooflines(n, 60, ph, peak), "peak_gbs": peak, "peak_kind": peak_kind,
            "atr_phases_ms": {k: round(sum(x), 4) for k, x in ph_atr.items()},
            "trace_roofline": trace_roof,
            "lbvh_build_ms": t_lbvh, "atr_build_ms": t_atr, "atr_mtris_s": n / t_atr / 1e3,
            "lbvh_mtris_s": n / t_lbvh / 1e3, "sah_cost_lbvh": lb.cost(), "sah_cost_atr": at.cost(),
            "primary_gen_ms": t_gen, "primary_trace_mrays_s": w * h / t_prim / 1e3,
            "secondary_trace_mrays_s": w * h / t_sec / 1e3,
            "secondary_sorted_trace_mrays_s": w * h / t_sort / 1e3,
            "rays_total": 2 * w * h}


def extra_wide(ctx, cfg, V, T, R, RES, steps=3):
    """The headline scene in the Quad and Oct layouts (Bvh.layout quad / oct):
    build time, SAH cost, leaf statistics and trace rate of the same rays, with
    the hits checked against the binary layout's."""
    import torch
    import hippie_b200 as hp
    s = torch.cuda.current_stream()
    n, nr = T.shape[0], R.shape[0]
    kw = dict(method=cfg["method"], morton_bits=cfg["bits"])
    if cfg["method"] == "ploc":
        kw.update(ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0)
    base = ctx.build(V, T, hp.BuildParams(**kw))
    ctx.trace(base, R, results=RES)
    torch.cuda.synchronize()
    want = RES[:, :2].clone()
    out = {"workload": cfg["workload"] + ", same rays"}
    for name, layout in (("quad", 4), ("oct", 8)):
        p = hp.BuildParams(layout=layout, **kw)
        bvh = ctx.build(V, T, p)
        ctx.trace(bvh, R, results=RES)
        torch.cuda.synchronize()
        same = bool(torch.equal(RES[:, :2], want))
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        for k in range(steps):
            ev[k][0].record(s)
            ctx.build(V, T, p, bvh=bvh)
            ev[k][1].record(s)
            ctx.trace(bvh, R, results=RES)
            ev[k][2].record(s)
        torch.cuda.synchronize()
        ctx.check()
        tb = float(np.median([e[0].elapsed_time(e[1]) for e in ev]))
        tt = float(np.median([e[1].elapsed_time(e[2]) for e in ev]))
        st = bvh.stats()
        out[name] = {"build_ms": tb, "build_mtris_s": n / tb / 1e3, "trace_ms": tt,
                     "trace_mrays_s": nr / tt / 1e3, "sah_cost": st["sah_cost"],
                     "avg_leaf_size": st["avg_leaf_size"], "nodes": st["num_interior"] + st["num_leaf"],
                     "hits_equal_binary": same}
        del bvh
    out["binary_sah_cost"] = base.cost()
    del base
    return out


def extra_methods(ctx, cfg, V, T, R, RES, steps=3):
    """The headline scene built by the other builders of the path (Bvh.method lbvh,
    hlbvh, atr, tr; 60-bit keys, the reference's defaults): build time, SAH cost
    and trace rate of the same rays, with the hits checked against the headline
    build's."""
    import torch
    import hippie_b200 as hp
    s = torch.cuda.current_stream()
    n, nr = T.shape[0], R.shape[0]
    kw = dict(method=cfg["method"], morton_bits=cfg["bits"])
    if cfg["method"] == "ploc":
        kw.update(ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0)
    base = ctx.build(V, T, hp.BuildParams(**kw))
    ctx.trace(base, R, results=RES)
    torch.cuda.synchronize()
    want = RES[:, :2].clone()
    out = {"workload": cfg["workload"] + ", same rays", "headline_sah_cost": base.cost()}
    del base
    for method in ("lbvh", "hlbvh", "atr", "tr"):
        p = hp.BuildParams(method=method, morton_bits=60)
        bvh = ctx.build(V, T, p)
        ctx.trace(bvh, R, results=RES)
        torch.cuda.synchronize()
        same = bool(torch.equal(RES[:, :2], want))
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        for k in range(steps):
            ev[k][0].record(s)
            ctx.build(V, T, p, bvh=bvh)
            ev[k][1].record(s)
            ctx.trace(bvh, R, results=RES)
            ev[k][2].record(s)
        torch.cuda.synchronize()
        ctx.check()
        tb = float(np.median([e[0].elapsed_time(e[1]) for e in ev]))
        tt = float(np.median([e[1].elapsed_time(e[2]) for e in ev]))
        out[method] = {"build_ms": tb, "build_mtris_s": n / tb / 1e3, "trace_ms": tt,
                       "trace_mrays_s": nr / tt / 1e3, "sah_cost": bvh.cost(), "hits_equal_headline": same}
        del bvh
    return out


def run_reference(args, cfg, rank):
    """CPU restatement of the path (the oracle), timed on the host cores, rank 0
    only. Each step builds and traces the whole workload when the run fits
    about 150 s of CPU time (calibrated on 131,072 triangles and rays), else
    the same fraction of the triangles and of the rays."""
    if rank != 0:
        return 0
    import oracle
    v, t, rays = make_inputs(cfg, 0, library_free=True)
    oracle.load()
    steps, warmup = args.steps, args.warmup
    c = min(t.shape[0], 131072)
    t0 = time.perf_counter()
    r = oracle_build(cfg, v, np.ascontiguousarray(t[:c]))
    t1 = time.perf_counter()
    oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays[:c])
    t2 = time.perf_counter()
    full = (t1 - t0) * t.shape[0] / c + (t2 - t1) * rays.shape[0] / c
    frac = min(1.0, 150.0 / max(1, steps + warmup) / max(full, 1e-6))
    m = max(c, int(t.shape[0] * frac)) if frac < 1.0 else t.shape[0]
    k = max(c, int(rays.shape[0] * frac)) if frac < 1.0 else rays.shape[0]
    tm = np.ascontiguousarray(t[:m])
    bt, tt = [], []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        r = oracle_build(cfg, v, tm)
        t1 = time.perf_counter()
        oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays[:k])
        t2 = time.perf_counter()
        if i >= warmup:
            bt.append(t1 - t0)
            tt.append(t2 - t1)
    b = float(np.mean(bt))
    tr = float(np.mean(tt))
    val = m / b / 1e6
    cores = os.cpu_count() or 1
    whole = m == t.shape[0] and k == rays.shape[0]
    sample = ("the whole workload every step" if whole else
              f"first {m} of {t.shape[0]} triangles built, first {k} of {rays.shape[0]} rays traced per step")
    line = {"metric": METRIC, "value": val, "unit": "Mtris/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * (b + tr), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "method": cfg["method"], "triangles": m, "rays": k},
            "trace_mrays_s": k / tr / 1e6,
            "cpu_baseline": {"value": val, "unit": "Mtris/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": "Mtris/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--once", action="store_true",
                    help="one build and one trace, then print the phase times (for profiler runs)")
    ap.add_argument("--tune", type=int, default=1, help="run the autotuner and report its trace rate")
    ap.add_argument("--extras", type=int, default=1,
                    help="also measure the batched (2048 meshes) and differentiable (heightfield) workloads")
    ap.add_argument("--rays", type=int, default=0, help="override the workload's ray count (profiling)")
    ap.add_argument("--parallel", default="rays", choices=["rays", "replicas"],
                    help="N > 1: 'rays' splits one scene's rays across the ranks (every rank holds the BVH); "
                         "'replicas' gives every rank a scene of its own")
    ap.add_argument("--bvh-broadcast", type=int, default=0,
                    help="rays mode: rank 0 builds and broadcasts the BVH over NCCL (default: every rank builds)")
    ap.add_argument("--reference-kernels", type=int, default=1,
                    help="also time the reference's own CUDA kernels where they were built (1 GPU)")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    cfg = dict(CONFIGS[args.config])
    if args.rays:
        cfg["rays"] = args.rays
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, cfg, rank)

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    import hippie_b200 as hp
    from hippie_b200 import _lib
    from hippie_b200.shard import broadcast_bvh_arrays, ray_ranges
    lib = _lib.load()
    ctx = hp.Context(local)
    # rays: one scene, its rays split contiguously across ranks, the BVH on every
    # rank (built there, or built on rank 0 and broadcast); replicas: every rank
    # builds and traces a scene of its own.
    mode = args.parallel if world > 1 else "rays"
    bcast = mode == "rays" and world > 1 and bool(args.bvh_broadcast)
    v, t, rays = make_inputs(cfg, rank if mode == "replicas" else 0)
    n, nr_all = t.shape[0], rays.shape[0]
    lo, hi = ray_ranges(nr_all, world)[rank] if mode == "rays" else (0, nr_all)
    nr = hi - lo                                     # this rank's rays
    job_tris = world * n if mode == "replicas" else n
    job_rays = world * nr_all if mode == "replicas" else nr_all
    Vh = torch.from_numpy(v).pin_memory()
    Th = torch.from_numpy(t).pin_memory()
    Rh = torch.from_numpy(np.ascontiguousarray(rays[lo:hi])).pin_memory()
    del rays
    V, T, R = Vh.cuda(), Th.cuda(), Rh.cuda()
    RES = torch.empty((nr, 4), dtype=torch.int32, device="cuda")
    RESh = torch.empty((nr, 4), dtype=torch.int32).pin_memory()
    params = build_params(cfg)
    bvh = hp.BVH.reserve(ctx, n) if bcast and rank != 0 else hp.BVH(ctx)

    def build_step():
        """One build of the scene on this rank, or, with the broadcast, on rank 0
        followed by an NCCL broadcast of its arrays into every rank's BVH."""
        if not bcast:
            ctx.build(V, T, params, bvh=bvh)
            return
        info = None
        if rank == 0:
            ctx.build(V, T, params, bvh=bvh)
            bvh.sync()
            info = bvh.info()
        got = broadcast_bvh_arrays(bvh.arrays(), info)
        if rank != 0:
            bvh.set_info(got["num_interior"], got["num_leaf"], got["scene_box"], got["morton_scale"])

    build_step()
    stream = torch.cuda.current_stream()
    if args.once:
        ctx.trace(bvh, R, results=RES)
        bvh.sync()
        ctx.check()
        print(json.dumps({"once": cfg["workload"], "rays": nr, "interior": bvh.c.num_interior,
                          "leaves": bvh.c.num_leaf}), flush=True)
        del bvh
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return 0

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(*xs):
        if world == 1:
            return list(xs)
        tt = torch.tensor(list(xs), device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return tt.tolist()

    for _ in range(args.warmup):
        build_step()
        ctx.trace(bvh, R, results=RES)
    torch.cuda.synchronize()
    ctx.check()
    # Tune once, as a user would before running: the result-neutral launch
    # choices (sort CTA size, tracer CTAs per SM and stack depth, ray Morton
    # order) are timed on these inputs and applied; the PLOC radius stays the
    # workload's (the tuner's pick is only reported).
    choice, tune_s = None, 0.0
    if args.tune:
        t0 = time.perf_counter()
        choice = ctx.autotune(V, T, R, params, ploc_radius=True)
        tune_s = time.perf_counter() - t0
        build_step()
        ctx.trace(bvh, R, results=RES)
        torch.cuda.synchronize()
        ctx.check()

    # ---- timed region: inputs resident in HBM (mesh 200 MB + rays 512 MB, larger than L2) ----
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.hp_launch_count()
    w0 = time.time()
    for k in range(args.steps):
        ev[k][0].record(stream)
        build_step()
        ev[k][1].record(stream)
        ctx.trace(bvh, R, results=RES)
        ev[k][2].record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    barrier()
    launches = lib.hp_launch_count() - launches0
    clocks.window(w0, w1)
    time.sleep(0.1)
    clocks.stop()
    ctx.check()
    build_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    trace_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    step_ms = float(ev[0][0].elapsed_time(ev[-1][2])) / args.steps
    build_ms, trace_ms, step_ms = max_over_ranks(build_ms, trace_ms, step_ms)

    # ---- the same rays traced in ray Morton order (keys + sort + trace, HipTracer::traceSort) ----
    for _ in range(2):
        ctx.trace_sorted(bvh, R, results=RES)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for k in range(args.steps):
        evs[k][0].record(stream)
        ctx.trace_sorted(bvh, R, results=RES)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    ctx.check()
    sorted_ms, = max_over_ranks(float(np.mean([e[0].elapsed_time(e[1]) for e in evs])))

    # ---- the same trace with the default launch choices (no tuning, input order) ----
    tuned_set = ctx.get_tune()
    ctx.reset_tune()
    ctx.trace(bvh, R, results=RES)
    evp = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    for k in range(args.steps):
        evp[k][0].record(stream)
        ctx.trace(bvh, R, results=RES)
        evp[k][1].record(stream)
    torch.cuda.synchronize()
    ctx.check()
    plain_ms, = max_over_ranks(float(np.mean([e[0].elapsed_time(e[1]) for e in evp])))
    ctx.set_tune(**{k: tuned_set[k] for k in ("sort_block", "trace_ctas_per_sm", "trace_stack", "trace_sorted")})
    tuned = None if choice is None else {
        "choice": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in choice.items()},
        "tuning_s": tune_s, "applied": "timed steps and e2e use the tuned launch choices"}

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e_b, e2e_t = [], []
    for k in range(max(3, args.steps // 2)):
        torch.cuda.synchronize()
        barrier()
        a = time.perf_counter()
        V.copy_(Vh, non_blocking=True)
        T.copy_(Th, non_blocking=True)
        build_step()
        bvh.sync()
        b = time.perf_counter()
        ctx.trace_host(bvh, Rh, results=RESh)  # hp_trace_host: chunked uploads / traces / downloads overlap
        torch.cuda.synchronize()
        c = time.perf_counter()
        e2e_b.append(b - a)
        e2e_t.append(c - b)
    e2e_b_s, e2e_t_s = max_over_ranks(float(np.median(e2e_b)), float(np.median(e2e_t)))

    # ---- per-phase CUDA events of one more build: sort-pass roofline and the phase fractions ----
    phases_l = profile_phases(ctx, build_step)
    phases = {k: sum(x) for k, x in phases_l.items()}
    passes = phases_l.get("sort_pass", [])
    seg_ms = sum(phases_l.get("sort_segments", []))
    kb = 4 if cfg["bits"] <= 32 else 8
    lsd_passes = (cfg["bits"] + 7) // 8
    sort_bytes = n * lsd_passes * 2 * (kb + 4)   # n * P * 2 * (K + 4): an 8-bit LSD sort's bytes
    sort_ms = sum(passes) + seg_ms
    pass_ms = float(np.mean(passes)) if passes else float("nan")
    achieved = sort_bytes / (sort_ms * 1e-3) / 1e9
    peak, peak_kind = peak_hbm()
    traffic = committed_traffic("sort_phase")
    parallelism = (f"replicas x{world}" if mode == "replicas" else
                   f"rays x{world}, BVH " + ("broadcast from rank 0 (NCCL)" if bcast else "built on every rank"))

    line = {
        "metric": METRIC, "value": job_tris / (build_ms * 1e-3) / 1e6, "unit": "Mtris/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak" if mode == "replicas" else "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "method": cfg["method"], "triangles": n, "rays": nr_all,
                   "morton_bits": cfg["bits"], "parallelism": parallelism,
                   "l2": "inputs larger than L2 (mesh 200 MB, rays 512 MB)"},
        "trace_mrays_s": job_rays / (trace_ms * 1e-3) / 1e6,
        "trace_sorted_mrays_s": job_rays / (sorted_ms * 1e-3) / 1e6,
        "trace_untuned_mrays_s": job_rays / (plain_ms * 1e-3) / 1e6,
        "autotuned": tuned,
        "build_ms": build_ms, "trace_ms": trace_ms,
        "phases_ms": {k: round(x, 4) for k, x in phases.items()},
        "e2e": {"value": job_tris / e2e_b_s / 1e6, "unit": "Mtris/s",
                "trace_mrays_s": job_rays / e2e_t_s / 1e6,
                "h2d_bytes_per_step": int(world * (v.nbytes + t.nbytes) + job_rays * 32),
                "d2h_bytes_per_step": int(job_rays * 16 + 8 * world)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm",
                     "kernel": (f"radix sort phase: {len(passes)} LSD passes (k_onesweep)" +
                                (" + segment sort (k_seg_sort, k_seg_big)" if seg_ms > 0 else "")),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": sort_bytes,
                     "algorithmic_bytes": f"n * {lsd_passes} * 2 * ({kb} + 4): the 8-bit LSD sort's key and value "
                                          "reads and writes, n = triangles",
                     "launch_ms": sort_ms, "per_pass_ms": pass_ms, "segments_ms": seg_ms,
                     "phases": phase_rooflines(n, cfg["bits"], phases_l, peak)},
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, v, t, Rh.numpy())
    if rank == 0 and world == 1 and args.reference_kernels:
        line["reference_kernels_gpu"] = reference_kernels(cfg, V, T, R, v)
    ctx.reset_tune()  # the other workloads run with the default launch choices
    if args.extras:
        if world == 1:
            line["wide"] = extra_wide(ctx, cfg, V, T, R, RES)
            line["methods"] = extra_methods(ctx, cfg, V, T, R, RES)
        del V, T, R, RES
        torch.cuda.empty_cache()
        line["batched"] = extra_batched(ctx, rank=rank, world=world)
        if world == 1:
            torch.cuda.empty_cache()
            line["differentiable"] = extra_differentiable(ctx)
            torch.cuda.empty_cache()
            line["large"] = extra_large(ctx)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del bvh
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
