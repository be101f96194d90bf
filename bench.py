#!/usr/bin/env python
"""S(Q)+g(r) frames/s on the N=1,000,188 three-species frame (one step = one frame).

Workload (default ``c3``): FCC 63^3 cells at density 0.8 (L=107.73), species 50:30:20,
Gaussian displacements 0.1 a plus 2% re-placed atoms, seeded synthetic frames.
g_ab(r): deltar=0.01, rcrdf=8 (cell lists).  S_ab(Q): qmax=10, qmin=3, bsc=(1,0.8,0.5);
k-set ``full+axes`` (every lattice vector of every complete shell below qmin, as +-k pairs,
plus the axis vectors of the shells above), method ``split`` (tcgen05 split-BF16) and, for
comparison, ``plain`` (FP32 direct sum).

Contract: ``python bench.py --gpus N --steps K --warmup W``; under torchrun each rank runs an
independent replica on its own frames (weak scaling, no data-path collective); rank 0 prints
one JSON line.  ``--impl reference`` times the CPU restatement of the reference algorithm on
the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "S(Q)+g(r) frames/s at N=1M vs plain FP32 kernel (1e-5 rel err); p50/p99 ms"

WORKLOADS = {
    "c3": dict(spec="c3", deltar=0.01, rcrdf=8.0, qmax=10.0, qmin=3.0, bsc=(1.0, 0.8, 0.5), kset="full+axes"),
    "c2": dict(spec="c2", deltar=0.01, rcrdf=10.0, qmax=15.0, qmin=5.0, bsc=(1.0, 0.6), kset="full+sampled"),
    "c1": dict(spec="c1", deltar=0.02, rcrdf=1e9, qmax=20.0, qmin=None, bsc=(1.0,), kset="full"),
    "c4": dict(spec="c4", deltar=0.02, rcrdf=6.0, qmax=8.0, qmin=2.0, bsc=(1.0, 1.0), kset="full+axes"),
}


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` on
    `workload`, from the committed ncu summary profiles/<kernel>_<workload>.md, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--method", default="split", choices=["split", "plain"])
    ap.add_argument("--kset", default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-FP32 comparison pass")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--serving", type=int, default=2000, help="requests in the serving run (0: skip)")
    ap.add_argument("--row", default="main", choices=["main", "charges", "dyn", "extras", "fused"],
                    help="main: the g(r)+S(Q) frame rate; charges: the same frames with per-atom charges "
                         "(g_qq, S_qq); dyn: F(Q,t)/Fs(Q,t)/MSD over time origins; extras: number "
                         "fluctuations, a two-dimensional frame and the slab analysis")
    return ap.parse_args()


def make_frames(wl, count, start):
    from trj_analysis_b200 import frames
    spec = frames.WORKLOADS[wl["spec"]]()
    return spec, [spec.frame(start + i) for i in range(count)]


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, rank, world, local_rank):
    import torch
    from trj_analysis_b200 import _lib, analysis, engine, refsem
    from trj_analysis_b200.analysis import Config, Session

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = dict(WORKLOADS[args.workload])
    if args.kset:
        wl["kset"] = args.kset
    nsp = len(wl["bsc"])
    W, K = args.warmup, args.steps
    spec, fr = make_frames(wl, W + K, start=1000 * rank)
    n = fr[0].n
    box = fr[0].box
    ctx = engine.Context(local_rank)
    stream = torch.cuda.current_stream()

    # device-resident inputs: raw coordinates and species of every step's frame
    d_xyz = [torch.from_numpy(f.xyz).to(dev) for f in fr]
    d_sp = [torch.from_numpy((f.types - 1).astype(np.int32)).to(dev) for f in fr]
    packed = torch.empty((n, 4), dtype=torch.float32, device=dev)
    counts = torch.zeros(nsp, dtype=torch.int64, device=dev)
    rdf = engine.RdfPlan(ctx, nsp, wl["deltar"], wl["rcrdf"], box, n)
    hist = rdf.new_hist()
    edge = torch.zeros(4, dtype=torch.int64, device=dev)
    ks = refsem.make_kset(wl["kset"], box, wl["qmax"], wl["qmin"], seed=0)
    sp_counts = np.bincount(fr[0].types - 1, minlength=nsp)
    sq = engine.SqPlan(ctx, nsp, ks, sp_counts)
    out = sq.new_out()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    method = args.method
    if method == "split" and sq.n_tiles == 0:
        method = "plain"

    def step(i, m):
        engine.pack_frame(ctx, d_xyz[i], d_sp[i], nsp, box, packed, counts)
        rdf.accumulate(packed, n, box, hist, edge)
        sq.accumulate(packed, n, box, out, engine.METHODS[m])

    def timed(m, steps, warm):
        for i in range(warm):
            step(i % len(fr), m)
            flush.zero_()
        ctx.check()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches0 = ctx.lib.trj_ctx_launches(ctx.h)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.lib.trj_ctx_set_timing(ctx.h, 1)
        kms = {"rdf": [], "sq": []}
        per = []
        ev0.record(stream)
        for i in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step((warm + i) % len(fr), m)
            b.record(stream)
            flush.zero_()
            per.append((a, b))
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        launches = ctx.lib.trj_ctx_launches(ctx.h) - launches0
        ctx.lib.trj_ctx_set_timing(ctx.h, 0)
        step_ms = [a.elapsed_time(b) for a, b in per]
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        ctx.check()
        return ms, step_ms, launches

    # kernel durations: one instrumented pass per kernel (events on the launch stream)
    def kernel_ms(m, reps):
        ctx.lib.trj_ctx_set_timing(ctx.h, 1)
        r_ms, s_ms = [], []
        import ctypes
        for i in range(reps):
            step(i % len(fr), m)
            v = ctypes.c_float()
            _lib.check(ctx.lib.trj_rdf_kernel_ms(rdf.h, ctypes.byref(v)), ctx.h)
            r_ms.append(v.value)
            _lib.check(ctx.lib.trj_sq_kernel_ms(sq.h, ctypes.byref(v)), ctx.h)
            s_ms.append(v.value)
            flush.zero_()
        ctx.lib.trj_ctx_set_timing(ctx.h, 0)
        return statistics.mean(r_ms), statistics.mean(s_ms)

    with ClockSampler(local_rank) as clk:
        total_ms, step_ms, launches = timed(method, K, W)
    clocks = clk.summary()
    value = world * K / (total_ms / 1000.0)
    rdf_ms, sq_ms = kernel_ms(method, max(3, min(K, 5)))

    plain = None
    if not args.no_plain and method == "split":
        pk = max(3, K // 3)
        p_ms, p_step, _ = timed("plain", pk, 1)
        _, plain_sq_ms = kernel_ms("plain", 2)
        plain = {"value": world * pk / (p_ms / 1000.0), "unit": "frames/s", "steps": pk,
                 "sq_kernel_ms": plain_sq_ms, "ms_per_step": p_ms / pk}

    # e2e through the public API: host frames -> Session (pinned copy, H2D, pack, g(r), S(Q)),
    # then a device->host read of the accumulated results every step.
    e2e = None
    if not args.no_e2e:
        cfg = Config(nsp=nsp, sp_types_selected=list(range(1, nsp + 1)), deltar=wl["deltar"], rcrdf=wl["rcrdf"],
                     qmax=wl["qmax"], qmin=wl["qmin"], bsc=wl["bsc"], kset=wl["kset"], method=method)
        sess = Session(cfg, ctx=ctx, n_max=n)
        for i in range(W):
            sess.add_frame(fr[i])
            sess.hist.cpu(), sess.sq_out.cpu()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        # Every step copies its frame in from pinned host memory and its results (counts and S sums) out
        # to pinned host memory.  The result copy of step i is waited for after step i+1 has been
        # submitted, so the host preparation of a frame overlaps the device work of the previous one.
        res_pin = [(torch.empty(sess.hist.shape, dtype=sess.hist.dtype, pin_memory=True),
                    torch.empty(sess.sq_out.shape, dtype=sess.sq_out.dtype, pin_memory=True)) for _ in range(2)]
        lat = []
        pending = None
        t0 = time.perf_counter()
        for i in range(K):
            ts = time.perf_counter()
            sess.add_frame(fr[W + i])
            h, s = res_pin[i % 2]
            h.copy_(sess.hist, non_blocking=True)
            s.copy_(sess.sq_out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            if pending is not None:
                pending[0].synchronize()
                lat.append((time.perf_counter() - pending[1]) * 1000.0)
            pending = (ev, ts)
        pending[0].synchronize()
        lat.append((time.perf_counter() - pending[1]) * 1000.0)
        torch.cuda.synchronize()
        e_ms = (time.perf_counter() - t0) * 1000.0
        if world > 1:
            t = torch.tensor([e_ms], dtype=torch.float64, device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(t.item())
        sess.ctx.check()
        e2e = {"value": world * K / (e_ms / 1000.0), "unit": "frames/s",
               "h2d_bytes_per_step": int(n * 12 + n * 4), "d2h_bytes_per_step": int(h.numel() * 8 + s.numel() * 8),
               "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}
        sess.rdf.close()
        sess.sq.close()

    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    # roofline of the dominant kernel
    n_dense = sq.n_dense
    if method == "split" and sq_ms >= rdf_ms:
        flops = 8.0 * n * n_dense
        # the kernel runs ~10 ms inside a ~20 ms step, not a seconds-long loop: the burst peak applies
        peak = peaks.get("bf16_tflops", 1590.0)
        achieved = flops / (sq_ms / 1000.0) / 1e12
        roof = {"kernel": "sq_tc (tcgen05 split-BF16)", "bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": profile_traffic("sq_tc_kernel", args.workload),
                "peak_source": "measured burst (MEASURED_PEAKS.json bf16_tflops)" if peaks else "fallback 1.59 PFLOP/s",
                "algorithmic": f"8*N*n_kvec = 8*{n}*{n_dense} flops per launch"}
    elif sq_ms >= rdf_ms:
        bytes_ = 16.0 * n * sq.kset.nvec / 1024.0
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = (n * sq.kset.nvec) / (sq_ms / 1000.0) / 1e12
        roof = {"kernel": "sq_plain (FP32 direct sum)", "bound": "hbm", "achieved": 16.0 * n / (sq_ms / 1e3) / 1e9,
                "peak": peak, "unit": "GB/s", "frac": 16.0 * n / (sq_ms / 1e3) / 1e9 / peak, "traffic": None,
                "terms_per_s": achieved * 1e12}
    else:
        nit = nsp * (nsp + 1) // 2
        alg = 16.0 * n + 8.0 * nit * rdf.lsmax
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = alg / (rdf_ms / 1000.0) / 1e9
        roof = {"kernel": "rdf_pairs (cell list)", "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": profile_traffic("rdf_pairs_kernel", args.workload),
                "algorithmic": f"16*N + 8*nit*lsmax = {alg:.0f} bytes per launch"}
    roof["kernels_ms"] = {"rdf_pairs": rdf_ms, "sq_main": sq_ms}
    # The pair kernel's own bound is SM-side (shared-memory atomics and instruction issue), not HBM:
    # one frame's edge counters give the in-range pairs (one shared u32 atomic each) and the pairs tested.
    hist1 = rdf.new_hist()
    edge1 = torch.zeros(4, dtype=torch.int64, device=dev)
    engine.pack_frame(ctx, d_xyz[0], d_sp[0], nsp, box, packed, counts)
    rdf.accumulate(packed, n, box, hist1, edge1)
    e1 = edge1.cpu().numpy()
    atomics_peak = 2.7e12  # u32 shared atomics/s on B200 (random bins), measured with a microbenchmark
    roof_pairs = {"kernel": "rdf_pairs (cell list)", "bound": "issue / shared atomics",
                  "in_range_pairs": int(e1[2]), "tested_pairs": int(e1[3]),
                  "achieved_atomics_per_s": float(e1[2]) / (rdf_ms / 1e3),
                  "atomics_peak_per_s": atomics_peak, "frac": float(e1[2]) / (rdf_ms / 1e3) / atomics_peak,
                  "tested_pairs_per_s": float(e1[3]) / (rdf_ms / 1e3), "ms": rdf_ms}

    result = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+bf16x3" if method == "split" else "f32", "data": "synthetic (seeded FCC frames)",
        "config": {"workload": f"{args.workload}: N={n} nsp={nsp} L={float(box[0]):.3f}, g(r) deltar={wl['deltar']} "
                               f"rcrdf={wl['rcrdf']}, S(Q) qmax={wl['qmax']} qmin={wl['qmin']} kset={wl['kset']}",
                   "method": method, "n_kvec": int(sq.kset.nvec), "n_kvec_tensor": int(n_dense),
                   "rdf_cells": list(rdf.cells), "parallelism": f"replicas x{world}",
                   "plan_scratch_bytes": {"rdf": int(rdf.scratch_bytes), "sq": int(sq.scratch_bytes)},
                   "device_bytes_in_use": int(torch.cuda.memory_allocated(dev)),
                   "l2": "256 MB buffer written between steps (inside the timed region)",
                   "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99))},
        "clocks": clocks, "gpu_launches": int(launches), "roofline": roof, "roofline_pairs": roof_pairs, "e2e": e2e,
    }
    if plain is not None:
        result["plain_fp32"] = plain
        result["speedup_split_vs_plain"] = value / plain["value"]
    return result, (spec, fr, wl, ks)


# ---------------------------------------------------------------------------
# serving: continuous batching vs offline vs the plain per-request path
# ---------------------------------------------------------------------------

def run_serving(n_req, seed=5):
    import copy
    from trj_analysis_b200.serve import Server, serving_workload, summarize
    reqs = serving_workload(n_req, seed=seed)

    def timed(srv, rq, realtime):
        t0 = time.perf_counter()
        res = srv.run(rq, realtime=realtime)
        return summarize(res, time.perf_counter() - t0)

    warm = reqs[: max(8, n_req // 10)]
    srv = Server(slots=8)
    timed(srv, [copy.copy(r) for r in warm], False)  # tunes the buckets, warms caches
    c0 = (srv.fused_requests, srv.fused_frames, srv.fuse_turns)
    offline = timed(srv, [copy.copy(r) for r in reqs], False)
    fused_stats = {"fused_requests": srv.fused_requests - c0[0], "fused_frames": srv.fused_frames - c0[1],
                   "fused_turns": srv.fuse_turns - c0[2], "fuse_max_atoms": srv.fuse_max_atoms,
                   "batch_device_bytes": srv.batch.device_bytes if srv.batch is not None else 0,
                   "note": "offline run: requests packed into fused launches, their frames, and the fused "
                           "launches (each one table copy + five kernels, replayed from a CUDA graph)"}

    def poisson(load, seed_):
        rng = np.random.default_rng(seed_)
        rate = load * offline["requests_per_s"]
        t, out = 0.0, []
        for r in reqs:
            t += rng.exponential(1.0 / rate)
            q = copy.copy(r)
            q.arrival = t
            out.append(q)
        return out

    online = timed(srv, poisson(0.8, seed + 1), True)
    # arrivals faster than the offline rate: the queue never empties, so the frames/s is what the loop
    # sustains at saturation, with queueing in the latencies
    saturated = timed(srv, poisson(1.25, seed + 2), True)
    # the same loop without fused launches (every request in a slot), for comparison
    unfused_srv = Server(slots=8, fuse_max_atoms=0)
    timed(unfused_srv, [copy.copy(r) for r in warm], False)
    unfused = timed(unfused_srv, [copy.copy(r) for r in reqs], False)
    base_srv = Server(slots=1, use_graphs=False, method="plain", fuse_max_atoms=0)
    baseline = timed(base_srv, [copy.copy(r) for r in reqs], False)
    return {"workload": f"{n_req} requests, N log-uniform [1e3, 2e5], 1-3 species, cubic or 1:1:2, 1-8 frames, "
                        "deltar 0.02, rcrdf min(L/2, 8), S(Q) reference k-set qmax 12 qmin 3; Poisson arrivals at "
                        "80% (online) and 125% (saturated) of the offline request rate",
            "offline": offline, "online": online, "saturated": saturated, "offline_unfused": unfused,
            "per_request_plain_path": baseline, "fused": fused_stats,
            "offline_vs_unfused": offline["frames_per_s"] / unfused["frames_per_s"],
            "online_vs_offline_throughput": online["frames_per_s"] / offline["frames_per_s"],
            "saturated_vs_offline_throughput": saturated["frames_per_s"] / offline["frames_per_s"],
            "offline_vs_plain_path": offline["frames_per_s"] / baseline["frames_per_s"],
            "latency_note": "offline latencies count from time 0 (every request queued at once); online ones from "
                            "each request's arrival",
            "peak_hbm_in_use_bytes": srv.peak_in_use, "admission_waits": srv.admission_waits}


# ---------------------------------------------------------------------------
# CPU restatement (reference algorithm on host cores)
# ---------------------------------------------------------------------------

def cpu_frame_estimate(wl, fr0, ks, seconds, part=0):
    """Times a bounded sample of one frame on the host cores and scales it to the whole frame.

    g(r): the oracle's linked-cell port (FP32 binning of rdf_sh, pairs j > i) over a run of home atoms
    from the middle of the frame, grown until it takes about half the budget.  S(Q): the reference's
    FP32-phase direct sum (sqfnD) over a stratified sample of the k-vectors: every s-th vector of every
    shell (at least one per shell), starting at offset ``part`` mod s, so that successive calls with
    part = 0, 1, 2, ... time disjoint slices.  Returns (seconds per frame, details)."""
    from oracle import orc
    from trj_analysis_b200 import refsem
    nsp = len(wl["bsc"])
    pos, sp, off = orc.layout(fr0.xyz, fr0.types - 1, fr0.box, nsp)
    p = refsem.rdf_params(nsp, wl["deltar"], wl["rcrdf"], fr0.box)
    n = pos.shape[0]
    m = 2000
    while True:
        i0 = n // 2 - m // 2
        t = time.perf_counter()
        h, e = orc.rdf_counts_range(pos, sp, fr0.box, p.side2, p.deltar, p.lsmax, nsp, i0, i0 + m)
        dt = time.perf_counter() - t
        if dt > seconds / 16 or m >= n:
            break
        m = min(n, m * 4)
    t_rdf = dt * n / m
    pairs = int(h.sum())
    # stratified S(Q) sample: per shell, vectors part, part + s, part + 2s, ... of that shell
    order = np.argsort(ks.bins, kind="stable")
    starts = np.searchsorted(ks.bins[order], np.arange(ks.nbins + 1))

    def sample(stride):
        idx = []
        for b in range(ks.nbins):
            v = order[starts[b]:starts[b + 1]]
            if v.size:
                k = part % stride
                idx.append(v[k::stride] if k < v.size else v[-1:])
        return np.concatenate(idx) if idx else np.zeros(0, np.int64)

    # calibrate on a small slice, then time the slice sized for about 3/4 of the budget
    stride = max(1, ks.nvec // 64)
    idx = sample(stride)
    t = time.perf_counter()
    orc.rho_ref32(pos, off, fr0.box, ks.vectors[idx[:64]])
    per_vec = (time.perf_counter() - t) / min(64, idx.size)
    stride = int(min(ks.nvec, max(1, ks.nvec * per_vec / (0.75 * seconds))))
    idx = sample(stride)
    t = time.perf_counter()
    orc.rho_ref32(pos, off, fr0.box, ks.vectors[idx])
    dt2 = time.perf_counter() - t
    t_sq = dt2 * ks.nvec / idx.size
    cores = orc.lib().orc_num_threads()
    detail = {
        "extrapolated": True,
        "sample_seconds": dt + dt2,
        "sample": (f"g(r): {m} home atoms of {n} (linked cells, pairs j>i); S(Q): {idx.size} of {ks.nvec} k-vectors "
                   f"(every {stride}th of each shell, offset {part % stride}) x {n} atoms; scaled to one frame"),
        "rdf_home_fraction": m / n, "sq_vector_fraction": idx.size / ks.nvec, "sq_stride": stride,
        "rdf_pairs_per_s": pairs / dt, "sq_terms_per_s": idx.size * n / dt2, "cores": cores,
    }
    return t_rdf + t_sq, detail


IMPLEMENTATION = ("CPU restatement of the reference algorithm (oracle/, C + OpenMP on all host threads): g(r) by the "
                  "oracle's linked-cell port with rdf_sh's FP32 binning (a cell list, not rdf_sh's O(N^2) all-pairs "
                  "loop), S(Q) by the FP32-phase direct sum of sqfnD; each step times a bounded sample and scales it "
                  "to one frame")


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from trj_analysis_b200 import refsem
    wl = dict(WORKLOADS[args.workload])
    if args.kset:
        wl["kset"] = args.kset
    spec, fr = make_frames(wl, 1, 0)
    ks = refsem.make_kset(wl["kset"], fr[0].box, wl["qmax"], wl["qmin"], seed=0)
    per_step = max(2.0, 100.0 / max(1, args.steps + min(args.warmup, 1)))
    for _ in range(min(args.warmup, 1)):
        cpu_frame_estimate(wl, fr[0], ks, per_step / 2)
    times, walls, fracs = [], [], []
    d = None
    for i in range(args.steps):
        w0 = time.perf_counter()
        t, d = cpu_frame_estimate(wl, fr[0], ks, per_step, part=i)
        walls.append(time.perf_counter() - w0)
        times.append(t)
        fracs.append(d["sq_vector_fraction"])
    v = 1.0 / statistics.mean(times)
    covered = min(1.0, sum(fracs)) if d and d["sq_stride"] > 1 else 1.0
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded FCC frames)", "extrapolated": True,
            "frame_ms_extrapolated": 1000.0 * statistics.mean(times),
            "config": {"workload": f"{args.workload}: N={fr[0].n}, kset={wl['kset']}", "implementation": IMPLEMENTATION,
                       "note": "ms_per_step is the measured wall time of one step's sample; value is frames/s "
                               "scaled from the samples (frame_ms_extrapolated per frame)",
                       "sq_vectors_covered_over_steps": covered},
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": d["cores"], "kind": "port",
                             "sample": d["sample"], "extrapolated": True,
                             "sample_seconds": statistics.mean([x for x in walls]),
                             "rdf_pairs_per_s": d["rdf_pairs_per_s"], "sq_terms_per_s": d["sq_terms_per_s"]},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
# secondary rows: charge-weighted columns, time correlations
# ---------------------------------------------------------------------------

def _events(fn, reps, flush):
    import torch
    out = []
    for i in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn(i)
        b.record()
        if flush is not None:
            flush.zero_()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return out


def run_charges(args):
    """The benchmark frame with per-atom charges (species charges 1, -0.8, 0.5 plus a 0.05 spread):
    pack with charges, g(r) with g_qq, S(Q) with S_qq, against the same frames without charges."""
    import ctypes
    import torch
    from trj_analysis_b200 import _lib, engine, frames, refsem
    wl = dict(WORKLOADS[args.workload])
    spec = frames.WORKLOADS[wl["spec"]]()
    spec.charges = (1.0, -0.8, 0.5, 0.3)[:len(wl["bsc"])]
    spec.charge_jitter = 0.05
    fr = [spec.frame(i) for i in range(3)]
    n, box, nsp = fr[0].n, fr[0].box, len(wl["bsc"])
    ctx = engine.Context(0)
    dev = ctx.torch_device
    d = [(torch.from_numpy(f.xyz).to(dev), torch.from_numpy((f.types - 1).astype(np.int32)).to(dev),
          torch.from_numpy(f.charges).to(dev)) for f in fr]
    packed = torch.empty((n, 4), dtype=torch.float32, device=dev)
    qpacked = torch.empty((n,), dtype=torch.float32, device=dev)
    counts = torch.zeros(nsp, dtype=torch.int64, device=dev)
    rdf = engine.RdfPlan(ctx, nsp, wl["deltar"], wl["rcrdf"], box, n)
    hist, gqq = rdf.new_hist(), rdf.new_gqq()
    ks = refsem.make_kset(wl["kset"], box, wl["qmax"], wl["qmin"], seed=0)
    cnt = np.bincount(fr[0].types - 1, minlength=nsp)
    sq, sqc = engine.SqPlan(ctx, nsp, ks, cnt), engine.SqPlan(ctx, nsp, ks, cnt, charged=True)
    out, outc = sq.new_out(), sqc.new_out()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    M = engine.METHODS[args.method]
    res = {}
    for charged in (False, True):
        def step(i, charged=charged):
            x, spc, q = d[i % 3]
            engine.pack_frame(ctx, x, spc, nsp, box, packed, counts, charges=q if charged else None,
                              qpacked=qpacked)
            if charged:
                rdf.accumulate(packed, n, box, hist, qpacked=qpacked, gqq=gqq)
                sqc.accumulate(packed, n, box, outc, M, qpacked=qpacked)
            else:
                rdf.accumulate(packed, n, box, hist)
                sq.accumulate(packed, n, box, out, M)
        _events(step, args.warmup, flush)
        ctx.check()
        ctx.lib.trj_ctx_set_timing(ctx.h, 1)
        r_ms, s_ms = [], []

        def timed(i, step=step, charged=charged):
            step(i)
            v = ctypes.c_float()
            _lib.check(ctx.lib.trj_rdf_kernel_ms(rdf.h, ctypes.byref(v)), ctx.h)
            r_ms.append(v.value)
            _lib.check(ctx.lib.trj_sq_kernel_ms((sqc if charged else sq).h, ctypes.byref(v)), ctx.h)
            s_ms.append(v.value)
        ms = _events(timed, args.steps, flush)
        ctx.lib.trj_ctx_set_timing(ctx.h, 0)
        ctx.check()
        res["charged" if charged else "uncharged"] = {
            "frame_ms": statistics.median(ms), "pair_kernel_ms": statistics.median(r_ms),
            "sq_kernel_ms": statistics.median(s_ms)}
    c = res["charged"]
    return {"metric": "g(r)+g_qq+S(Q)+S_qq frames/s, per-atom charges", "value": 1000.0 / c["frame_ms"],
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": c["frame_ms"], "higher_is_better": True, "dtype": "f32/f64",
            "data": "synthetic", "config": {"workload": args.workload + "+charges", "n_atoms": n,
                                              "method": args.method, "l2": "flushed between steps"},
            "detail": res}


def run_dyn(args):
    """F(Q,t), Fs(Q,t) and the MSD over time origins: N = 62,500 (the binary c2 shape), a random walk
    of 0.2 per axis per frame, 30 frames, 10 buffers one frame apart, shells qw = 1, 2, 4, 7."""
    import ctypes
    import torch
    from trj_analysis_b200 import _lib, dynamics, engine, frames
    spec = frames.FCCSpec(cells=(25, 25, 25), sigma=0.1, fractions=(0.8, 0.2), seed=2)
    nconf, nbuf = 30, 10
    frs = list(frames.random_walk_frames(spec, nconf, 0.2))
    n, box = frs[0].n, frs[0].box
    ctx = engine.Context(0)
    stage = engine.FrameStage(ctx, n, 2)
    dyn = dynamics.Dynamics(ctx, 2, n, nconf, dynamics.DynConfig(nbuffer=nbuf, jump=1, qw=(1.0, 2.0, 4.0, 7.0)),
                            box, np.array([1.0, 0.6], np.float32))
    ctx.lib.trj_ctx_set_timing(ctx.h, 1)
    ms, kms, terms = [], [], []
    for iconf in range(1, nconf + 1):
        f = frs[iconf - 1]
        nn = stage.upload_and_pack(f.xyz, f.types - 1, box)
        lags, origins = dyn.sched.schedule(iconf, f.time)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dyn.plan.accumulate(stage.packed, nn, box, lags, origins)
        b.record()
        done = dyn.sched.finish_frame(iconf)
        if done.any():
            dyn.plan.flush(done, dyn.fkt, dyn.fskt, dyn.r2t)
        torch.cuda.synchronize()
        v = ctypes.c_float()
        _lib.check(ctx.lib.trj_dyn_kernel_ms(dyn.plan.h, ctypes.byref(v)), ctx.h)
        if iconf > nbuf:  # every buffer active
            ms.append(a.elapsed_time(b))
            kms.append(v.value)
            terms.append(int((lags >= 0).sum()) * n * dyn.sqw.nvec)
    ctx.check()
    self_tps = float(np.median(np.array(terms) / (np.array(kms) * 1e-3)))
    return {"metric": "F(Q,t)+Fs(Q,t)+MSD frames/s (10 time origins)", "value": 1000.0 / statistics.median(ms),
            "unit": "frames/s", "n_gpus": 1, "steps": len(ms), "warmup": nbuf, "ms_per_step": statistics.median(ms),
            "higher_is_better": True, "dtype": "f32 terms, f64 sums", "data": "synthetic",
            "config": {"workload": "random walk N=62500, 30 frames, nbuffer 10, qw 1/2/4/7",
                       "n_atoms": n, "nvec": dyn.sqw.nvec},
            "self_kernel": {"ms": statistics.median(kms), "terms_per_s": self_tps,
                            "terms_per_clk_per_sm": self_tps / (ctx.sm_count * 1.9e9)}}


def run_fused(args):
    """One fused turn: frame 0 of 64 small serving requests (N log-uniform in [1e3, 16384], 1-3 species,
    cubic or 1:1:2 boxes, deltar 0.02, rcrdf min(L/2, 8), reference k-set qmax 12 qmin 3) through
    one batch launch replayed from a CUDA graph, against the same 64 frames through the per-request
    calls (layout, g(r), plain S(Q): the path each request takes alone).  Both time device work only
    (inputs already staged / resident), CUDA events on the launching stream, L2 flushed between steps."""
    import torch
    from trj_analysis_b200 import engine, refsem
    from trj_analysis_b200.serve import serving_workload
    reqs = serving_workload(64, seed=3, n_lo=1e3, n_hi=16384)
    dev = torch.device("cuda", 0)
    ctx = engine.Context(0)
    batch = engine.Batch(ctx, 64, 1 << 20)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    st = []
    for r in reqs:
        fr0 = r.frames[0]
        sel = sorted(set(int(t) for t in np.unique(fr0.types)))[: r.nsp]
        sp = refsem.species_by_first_appearance(fr0.types, sel)[0].astype(np.int32)
        ks = refsem.make_kset(r.kset, fr0.box, r.qmax, r.qmin)
        counts = np.bincount(sp, minlength=r.nsp)
        with torch.cuda.stream(stream):
            rdf = engine.RdfPlan(ctx, r.nsp, r.deltar, r.rcrdf, fr0.box, r.n)
            sq = engine.SqPlan(ctx, r.nsp, ks, counts)
            hist, out = rdf.new_hist(), sq.new_out()
            xyz = torch.from_numpy(np.ascontiguousarray(fr0.xyz, np.float32)).to(dev)
            spd = torch.from_numpy(sp).to(dev)
            packed = torch.empty((r.n, 4), dtype=torch.float32, device=dev)
            cnt = torch.zeros(16, dtype=torch.int64, device=dev)
        st.append(dict(r=r, sp=sp, ks=ks, rdf=rdf, sq=sq, hist=hist, out=out, xyz=xyz, spd=spd, packed=packed,
                       cnt=cnt))
    torch.cuda.synchronize()
    for b in (0, 1):  # both staging buffers hold the same turn
        batch.begin(b)
        off = 0
        for e in st:
            r = e["r"]
            batch.stage(b, off, r.frames[0].xyz, e["sp"])
            batch.add(b, e["rdf"], e["sq"], off, r.n, r.frames[0].box, e["hist"], e["out"])
            off += r.n
    graphs = []
    with torch.cuda.stream(stream):
        for b in (0, 1):
            g = torch.cuda.CUDAGraph()
            g.capture_begin()
            batch.launch(b, stream)
            g.capture_end()
            graphs.append(g)
    launches0 = ctx.lib.trj_ctx_launches(ctx.h)

    def fused_step(i):
        graphs[i & 1].replay()

    def unfused_step(i):
        for e in st:
            r, box = e["r"], e["r"].frames[0].box
            engine.pack_frame(ctx, e["xyz"], e["spd"], r.nsp, box, e["packed"], e["cnt"], stream=stream)
            e["rdf"].accumulate(e["packed"], r.n, box, e["hist"], stream=stream)
            e["sq"].accumulate(e["packed"], r.n, box, e["out"], engine.METHODS["plain"], stream=stream)

    def timed(step, k0, k):
        ts = []
        for i in range(k0 + k):
            with torch.cuda.stream(stream):
                flush.fill_(i & 255)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                step(i)
                b.record(stream)
            b.synchronize()
            if i >= k0:
                ts.append(a.elapsed_time(b))
        return ts

    l0 = ctx.lib.trj_ctx_launches(ctx.h)
    unf = timed(unfused_step, args.warmup, args.steps)
    unfused_launches = (ctx.lib.trj_ctx_launches(ctx.h) - l0) / (args.warmup + args.steps)
    fus = timed(fused_step, args.warmup, args.steps)
    ctx.check()
    n = np.array([e["r"].n for e in st], np.float64)
    nvec = np.array([e["ks"].nvec for e in st], np.float64)
    pairs = float((n * (n - 1) / 2).sum())
    terms = float((n * nvec).sum())
    f_ms, u_ms = statistics.median(fus), statistics.median(unf)
    return {"metric": "fused turn: frame 0 of 64 small requests (g(r) + plain S(Q))", "value": 64.0 / (f_ms * 1e-3),
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": f_ms,
            "higher_is_better": True, "dtype": "f32 terms, f64 sums", "data": "synthetic",
            "config": {"workload": "64 serving requests, N log-uniform [1e3, 16384]", "atoms": int(n.sum()),
                       "kvec": int(nvec.sum()), "l2": "256 MB buffer written between steps"},
            "fused": {"ms": f_ms, "launches": 5, "copies": 1, "pair_tests_per_s": pairs / (f_ms * 1e-3),
                      "sq_terms_per_s": terms / (f_ms * 1e-3)},
            "per_request": {"ms": u_ms, "launches": unfused_launches, "frames_per_s": 64.0 / (u_ms * 1e-3)},
            "fused_vs_per_request": u_ms / f_ms, "launches_before_timing": int(launches0)}


def run_extras(args):
    """Timings of the remaining analyses on the benchmark frame's scale:
    s2n: trj_rdf_s2n with 4096 sample points after the c3 frame's pair pass;
    2d: a two-dimensional frame of 1,000,000 atoms (square lattice with noise, 2 species) through the 2D
        pair plan (deltar 0.01, rcrdf 8) and the 2D reference vector set (qmax 10, qmin 3, direct sum);
    slab: the c3 frame in three z slices (g_xy and S_xy, host-orchestrated per slice)."""
    import torch
    from trj_analysis_b200 import analysis, engine, frames, refsem
    out = {}
    wl = WORKLOADS["c3"]
    spec = frames.c3_spec()
    fr = spec.frame(0)
    n, box = fr.n, fr.box
    ctx = engine.Context(0)
    stage = engine.FrameStage(ctx, n, 3)
    nn = stage.upload_and_pack(fr.xyz, fr.types - 1, box)
    rdf = engine.RdfPlan(ctx, 3, wl["deltar"], wl["rcrdf"], box, n)
    hist = rdf.new_hist()
    gi, g2i = rdf.new_s2n()
    rdf.accumulate(stage.packed, nn, box, hist)
    ms = _events(lambda i: rdf.s2n(4096, gi, g2i), args.warmup + args.steps, None)[args.warmup:]
    out["s2n"] = {"points": 4096, "ms": statistics.median(ms), "workload": "c3 frame, 13^3 cells"}
    ctx.check()
    # two-dimensional frame
    rng = np.random.default_rng(7)
    side = 1000
    a = 1.1
    gx, gy = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
    xy = np.stack([gx.ravel(), gy.ravel()], axis=1) * a + rng.normal(0, 0.12 * a, size=(side * side, 2))
    xyz = np.concatenate([xy, np.zeros((side * side, 1))], axis=1).astype(np.float32)
    types = rng.permutation(np.repeat(np.array([1, 2], np.int32), [side * side // 2, side * side // 2]))
    f2 = frames.Frame(xyz=xyz, types=types, box=np.array([side * a, side * a, 1.0], np.float32))
    out["2d"] = {"n_atoms": side * side}
    for method in ("split", "plain"):  # split: the planar tile form on the tensor cores
        cfg = analysis.Config(nsp=2, ndim=2, sp_types_selected=(1, 2), deltar=0.01, rcrdf=8.0, qmax=10.0, qmin=3.0,
                              method=method, kset="ref")
        sess = analysis.Session(cfg, ctx=ctx)
        sess.add_frame(f2)
        torch.cuda.synchronize()
        ms = _events(lambda i: (sess.RDFcomp(), sess.SQcalc()), args.warmup + args.steps, None)[args.warmup:]
        out["2d"]["n_kvec"] = int(sess.kset.nvec)
        out["2d"][method] = {"frame_ms": statistics.median(ms), "frames_per_s": 1000.0 / statistics.median(ms)}
        sess.ctx.check()
        sess.close()
    # slab analysis of the c3 frame in three slices
    zmax = float(box[2])
    cfg = analysis.Config(nsp=3, sp_types_selected=(1, 2, 3), deltar=wl["deltar"], rcrdf=wl["rcrdf"], qmax=6.0,
                          qmin=3.0, slab=analysis.SlabConfig(zslice=(0.25 * zmax, 0.5 * zmax, 0.75 * zmax),
                                                             zgrid=0.1 * zmax))
    sess = analysis.Session(cfg, ctx=ctx)
    sess.add_frame(fr)
    t = []
    for i in range(max(2, args.steps // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sess.add_frame(fr)
        torch.cuda.synchronize()
        t.append((time.perf_counter() - t0) * 1000.0)
    out["slab"] = {"slices": 3, "frame_ms_wall": statistics.median(t), "workload": "c3 frame, 3 slices of 0.1 L"}
    sess.close()
    ctx.check()
    return {"metric": "secondary analyses: s2n, 2D frame, slabs", "unit": "ms", "n_gpus": 1, "data": "synthetic",
            "detail": out}


def main():
    args = parse()
    if args.row != "main":
        res = {"charges": run_charges, "dyn": run_dyn, "extras": run_extras, "fused": run_fused}[args.row](args)
        print(json.dumps(res), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    res, (spec, fr, wl, ks) = run_ours(args, rank, world, local_rank)
    if rank == 0 and args.serving > 0:
        res["serving"] = run_serving(args.serving)
    if rank == 0 and not args.no_cpu:
        t, d = cpu_frame_estimate(wl, fr[0], ks, args.cpu_seconds)
        res["cpu_baseline"] = {"value": 1.0 / t, "unit": "frames/s", "cores": d["cores"], "kind": "port",
                               "sample": d["sample"], "extrapolated": True, "sample_seconds": d["sample_seconds"],
                               "rdf_pairs_per_s": d["rdf_pairs_per_s"], "sq_terms_per_s": d["sq_terms_per_s"],
                               "implementation": IMPLEMENTATION}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
