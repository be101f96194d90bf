"""Continuous-batching request loop for g(r) / S(Q) analysis requests on one GPU.

A request is a short trajectory (1..F frames of one system) with its own g(r) and S(Q)
parameters.  The loop:

* admits queued requests when a slot (CUDA stream + pinned staging) is free and the
  request's device footprint fits the HBM budget still unused by running requests;
* creates the request's plans with the library's device memory drawn from PyTorch's
  caching allocator (``trj_ctx_set_allocator``), so plan set-up and tear-down never
  synchronise the device while other requests run;
* enqueues one frame per running request per turn (host->device copy, layout, g(r),
  S(Q)) on that request's stream, so frames of different requests overlap on the GPU;
  requests with several frames replay a CUDA graph of the per-frame launch sequence
  after the first frame (double-buffered pinned input);
* on the last frame reads the accumulated counts and sums back, normalises them on the
  host, stamps the latency and frees the slot for the next request;
* packs small requests (at most ``fuse_max_atoms`` atoms, reference bins within the batch's shared
  histogram) into one fused launch per turn instead of slots: one frame of each packed request goes
  through a single table copy and five kernels (layout, all-pairs histogram, direct sum, shell
  reduction) over all of them (``engine.Batch``), replayed from a CUDA graph captured once per staging
  buffer; their S(Q) is the direct sum, bit-identical to the per-request plain method;
* ``cancel(rid)`` (from any thread) drops a request that is still waiting, or stops a running one
  after the frames already on its stream: once they have finished its plans, slot and HBM budget
  are released and it yields no result (its id is listed in ``cancelled``).

The S(Q) method and the tensor-core tile width of each (size, species) bucket are picked by an
autotuner that times the candidates once on the bucket's first request.
Results do not depend on what else runs: pair counts are integers and the S(Q) sums use a
fixed reduction order, so a request gives bit-identical output alone and in a mix.
"""
from __future__ import annotations

import collections
import ctypes
import dataclasses
import json
import math
import os
import threading
import time
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import engine, refsem
from .analysis import normalise_rdf, normalise_sq
from .frames import FCCSpec, Frame

ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)


class TorchAllocator:
    """Library device allocations served by PyTorch's caching allocator on the current stream."""

    def __init__(self, device: torch.device):
        self.device = device
        self.live: Dict[int, torch.Tensor] = {}
        self.bytes_live = 0
        self._lock = threading.Lock()
        self._alloc = ALLOC_FN(self._alloc_cb)
        self._free = FREE_FN(self._free_cb)

    def _alloc_cb(self, nbytes, user):
        try:
            t = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=self.device)
        except RuntimeError:
            return None
        with self._lock:
            self.live[t.data_ptr()] = t
            self.bytes_live += t.numel()
        return t.data_ptr()

    def _free_cb(self, ptr, user):
        with self._lock:
            t = self.live.pop(int(ptr), None)
            if t is not None:
                self.bytes_live -= t.numel()

    def install(self, ctx: engine.Context) -> None:
        engine.check(ctx.lib.trj_ctx_set_allocator(ctx.h, ctypes.cast(self._alloc, ctypes.c_void_p),
                                                   ctypes.cast(self._free, ctypes.c_void_p), None),
                     ctx.h, "trj_ctx_set_allocator")


@dataclasses.dataclass
class Request:
    rid: int
    frames: Sequence[Frame]
    nsp: int
    deltar: float = 0.02
    rcrdf: float = 8.0
    qmax: float = 12.0
    qmin: float = 3.0
    bsc: Optional[Sequence[float]] = None
    kset: str = "ref"
    method: Optional[str] = None       # None: autotuner decides
    arrival: float = 0.0               # seconds after the start of the run

    @property
    def n(self) -> int:
        return self.frames[0].n


@dataclasses.dataclass
class Result:
    rid: int
    hist: np.ndarray                   # uint64 [nit][lsmax]
    sq_sums: np.ndarray                # float64 [nbins][nit]
    rdf: Dict[str, np.ndarray]
    sq: Dict[str, np.ndarray]
    method: str
    arrival: float
    done: float
    nframes: int = 1

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class Autotuner:
    """Chooses, per (k-set mode, log2 N, species) bucket, the S(Q) method and the widest tensor-core tile
    (output columns per tile: narrow tiles make more, smaller work items for small frames; wide ones issue
    fewer tensor-core instructions per vector) by timing every candidate once on the bucket's first
    request.  The table is kept (and saved to `path`, when given) with the measured times."""

    CANDIDATES = (("split", 224), ("split", 160), ("split", 96), ("plain", 0))

    def __init__(self, path: Optional[str] = None):
        self.path = path
        self.table: Dict[str, dict] = {}
        if path and os.path.exists(path):
            self.table = json.load(open(path))

    @staticmethod
    def key(n: int, nsp: int, kset: str) -> str:
        return f"{kset}:{int(math.log2(max(n, 1)))}:{nsp}"

    def lookup(self, n: int, nsp: int, kset: str):
        """(method, tile columns) of the bucket, or None before it is tuned."""
        e = self.table.get(self.key(n, nsp, kset))
        return None if e is None else (e["method"], int(e["cols"]))

    def tune(self, ctx: engine.Context, ks: refsem.KSet, counts, packed: torch.Tensor, n: int, box, stream):
        """Times every candidate on the laid-out frame `packed` (2 accumulations after a warm one);
        returns (method, tile columns, {candidate: ms})."""
        nsp = len(counts)
        times = {}
        for method, cols in self.CANDIDATES:
            ctx.set_sq_tile_cols(cols)
            try:
                with torch.cuda.stream(stream):
                    plan = engine.SqPlan(ctx, nsp, ks, counts)
            finally:
                ctx.set_sq_tile_cols(0)
            if method == "split" and plan.n_tiles == 0:
                plan.close()
                continue
            with torch.cuda.stream(stream):
                out = plan.new_out()
                plan.accumulate(packed, n, box, out, engine.METHODS[method], stream=stream)  # warm
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                for _ in range(2):
                    plan.accumulate(packed, n, box, out, engine.METHODS[method], stream=stream)
                b.record(stream)
            b.synchronize()
            times[f"{method}:{cols}"] = a.elapsed_time(b) / 2.0
            plan.close()
        best = min(times, key=times.get)
        method, cols = best.split(":")
        return method, int(cols), times

    def record(self, n: int, nsp: int, kset: str, method: str, cols: int, times=None) -> None:
        self.table[self.key(n, nsp, kset)] = {"method": method, "cols": int(cols), "ms": times or {}}
        if self.path:
            with open(self.path, "w") as f:
                json.dump(self.table, f, indent=1)


class _Slot:
    def __init__(self, ctx: engine.Context, n_max: int):
        self.stream = torch.cuda.Stream(device=ctx.torch_device)
        dev = ctx.torch_device
        self.n_max = n_max
        self.h_xyz = [torch.empty((n_max, 3), dtype=torch.float32, pin_memory=True) for _ in range(2)]
        self.h_sp = [torch.empty((n_max,), dtype=torch.int32, pin_memory=True) for _ in range(2)]
        self.h_ev = [None, None]       # event after the copy out of each pinned buffer
        with torch.cuda.stream(self.stream):
            self.d_xyz = torch.empty((n_max, 3), dtype=torch.float32, device=dev)
            self.d_sp = torch.empty((n_max,), dtype=torch.int32, device=dev)
            self.packed = torch.empty((n_max, 4), dtype=torch.float32, device=dev)
            self.counts = torch.zeros((16,), dtype=torch.int64, device=dev)
        self.req: Optional[Request] = None


class _Job:
    """A request bound to a slot: plans, outputs and progress."""

    def __init__(self, req: Request, slot: _Slot):
        self.req, self.slot = req, slot
        self.next_frame = 0
        self.graphs = [None, None]
        self.done_event = None
        self.footprint = 0
        self.cancelled = False
        self.fused = False


class Server:
    def __init__(self, device: int = 0, slots: int = 8, hbm_budget: Optional[int] = None, n_max: int = 1 << 18,
                 use_graphs: bool = True, autotuner: Optional[Autotuner] = None, method: Optional[str] = None,
                 fuse_max_atoms: int = 16384, fuse_items: int = 64, fuse_atoms: int = 1 << 20,
                 fuse_hist_words: int = 4096):
        self.ctx = engine.Context(device)
        self.alloc = TorchAllocator(self.ctx.torch_device)
        self.alloc.install(self.ctx)
        free, total = torch.cuda.mem_get_info(self.ctx.torch_device)
        self.hbm_budget = int(hbm_budget if hbm_budget is not None else 0.6 * free)
        self.slots = [_Slot(self.ctx, n_max) for _ in range(slots)]
        self.n_max = n_max
        self.use_graphs = use_graphs
        self.tuner = autotuner or Autotuner()
        self.method = method
        self.in_use = 0
        self.peak_in_use = 0
        self.admission_waits = 0
        self.cancelled: List[int] = []
        self._cancel: set = set()
        self._cancel_lock = threading.Lock()
        # fused launches of small requests
        self.fuse_max_atoms = int(fuse_max_atoms)
        self.fuse_items, self.fuse_atoms, self.fuse_hist_words = int(fuse_items), int(fuse_atoms), int(fuse_hist_words)
        self.batch: Optional[engine.Batch] = None
        self.fuse_stream = None
        self.fuse_graphs = [None, None]
        self.fuse_turns = 0
        self._fuse_cache: Dict[tuple, bool] = {}
        self.fused_requests = 0
        self.fused_frames = 0
        if self.fuse_max_atoms > 0:
            self.batch = engine.Batch(self.ctx, self.fuse_items, self.fuse_atoms, self.fuse_hist_words)
            self.fuse_stream = torch.cuda.Stream(device=self.ctx.torch_device)

    def cancel(self, rid: int) -> None:
        """Requests cancellation of request `rid` (thread-safe; takes effect at the loop's next turn)."""
        with self._cancel_lock:
            self._cancel.add(int(rid))

    def _apply_cancels(self, pending, queue, jobs) -> None:
        with self._cancel_lock:
            want = set(self._cancel)
        if not want:
            return
        done = set()
        for dq in (pending, queue):
            keep = [r for r in dq if r.rid not in want]
            for r in dq:
                if r.rid in want:
                    self.cancelled.append(r.rid)
                    done.add(r.rid)
            dq.clear()
            dq.extend(keep)
        for job in jobs:
            if job.req.rid in want and not job.cancelled:
                # no further frames; the release waits for the frames already on the stream
                job.cancelled = True
                job.next_frame = len(job.req.frames)
                job.done_event = torch.cuda.Event()
                job.done_event.record(self.fuse_stream if job.fused else job.slot.stream)
                done.add(job.req.rid)
        with self._cancel_lock:
            self._cancel -= done

    def _release(self, job: _Job) -> None:
        job.graphs = [None, None]
        job.rdf.close()
        job.sq.close()
        self.in_use -= job.footprint
        if job.slot is not None:
            job.slot.req = None

    # ---- footprint / admission ---------------------------------------------------------
    def footprint(self, req: Request, ks: refsem.KSet, method: str) -> int:
        n, nsp, nv = req.n, req.nsp, ks.nvec
        rdf = 64 * n + 3 * 4 * 4096
        sq = 16 * n + 16 * nsp * nv * 9 + 16 * nsp * nv + 24 * nv
        if method == "split":
            sq += 2 * (2 * 64) * 2 * (n + 32 * nsp) + 2 * 8 * 128 * (n + 32 * nsp) + 8 * nsp * nv * 4
        return int(rdf + sq)

    # ---- fused launches -------------------------------------------------------------------
    def _fusable(self, req: Request) -> bool:
        key = (req.rid, id(req))
        hit = self._fuse_cache.get(key)
        if hit is not None:
            return hit
        ok = (self.batch is not None and req.n <= min(self.fuse_max_atoms, self.fuse_atoms)
              and (req.method or self.method or "plain") == "plain")
        if ok:
            p = refsem.rdf_params(req.nsp, req.deltar, req.rcrdf, req.frames[0].box)
            ok = req.nsp * (req.nsp + 1) // 2 * p.lsmax <= self.fuse_hist_words
        self._fuse_cache[key] = ok
        return ok

    def _start_fused(self, req: Request, fused: List[_Job]) -> Optional[_Job]:
        if len(fused) >= self.fuse_items or sum(j.req.n for j in fused) + req.n > self.fuse_atoms:
            return None
        fr0 = req.frames[0]
        sel = sorted(set(int(t) for t in np.unique(fr0.types)))[: req.nsp]
        sp, wtypes, perm = refsem.species_by_first_appearance(fr0.types, sel)
        bsc = list(req.bsc) if req.bsc is not None else [1.0] * req.nsp
        ks = refsem.make_kset(req.kset, fr0.box, req.qmax, req.qmin)
        counts = np.bincount(sp[sp >= 0], minlength=req.nsp)
        fp = self.footprint(req, ks, "plain") - 64 * req.n  # no cell arrays
        if self.in_use + fp > self.hbm_budget and self.in_use > 0:
            self.admission_waits += 1
            return None
        job = _Job(req, None)
        job.fused = True
        job.species = sp.astype(np.int32)
        job.bsc = np.array([bsc[perm[s]] for s in range(req.nsp)], np.float32)
        job.ntype = counts
        job.ks = ks
        with torch.cuda.stream(self.fuse_stream):
            # the pair plan gives the batch its cutoff, bins and species; its cell arrays stay unused
            job.rdf = engine.RdfPlan(self.ctx, req.nsp, req.deltar, req.rcrdf, fr0.box, 0)
            job.sq = engine.SqPlan(self.ctx, req.nsp, ks, counts)
            job.hist = job.rdf.new_hist()
            job.out = job.sq.new_out()
        job.method = "plain"
        job.cols = 0
        job.tune = False
        job.footprint = fp
        self.in_use += fp
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        self.fused_requests += 1
        return job

    def _fused_turn(self, fused: List[_Job]) -> bool:
        """One frame of every packed request with frames left, through one fused launch."""
        active = [j for j in fused if j.next_frame < len(j.req.frames)]
        if not active:
            return False
        b, s = self.batch, self.fuse_stream
        buf = self.fuse_turns & 1
        b.begin(buf)  # waits until this buffer's previous launch has run
        off = 0
        for job in active:
            fr = job.req.frames[job.next_frame]
            n = job.req.n
            b.stage(buf, off, fr.xyz, job.species)
            b.add(buf, job.rdf, job.sq, off, n, fr.box, job.hist, job.out)
            off += n
            job.next_frame += 1
        with torch.cuda.stream(s):
            if self.use_graphs:
                if self.fuse_graphs[buf] is None:
                    g = torch.cuda.CUDAGraph()
                    g.capture_begin(capture_error_mode="relaxed")
                    try:
                        b.launch(buf, s)
                    finally:
                        g.capture_end()
                    self.fuse_graphs[buf] = g
                self.fuse_graphs[buf].replay()
            else:
                b.launch(buf, s)
            b.mark(buf, s)
            for job in active:
                if job.next_frame == len(job.req.frames):
                    job.h_hist = job.hist.to("cpu", non_blocking=True)
                    job.h_out = job.out.to("cpu", non_blocking=True)
                    job.done_event = torch.cuda.Event()
                    job.done_event.record(s)
        self.fuse_turns += 1
        self.fused_frames += len(active)
        return True

    # ---- request life cycle -------------------------------------------------------------
    def _start(self, req: Request, slot: _Slot) -> Optional[_Job]:
        fr0 = req.frames[0]
        sel = sorted(set(int(t) for t in np.unique(fr0.types)))[: req.nsp]
        sp, wtypes, perm = refsem.species_by_first_appearance(fr0.types, sel)
        bsc = list(req.bsc) if req.bsc is not None else [1.0] * req.nsp
        ks = refsem.make_kset(req.kset, fr0.box, req.qmax, req.qmin)
        counts = np.bincount(sp[sp >= 0], minlength=req.nsp)
        tuned = self.tuner.lookup(req.n, req.nsp, req.kset)
        method = req.method or self.method or (tuned[0] if tuned else "split")
        cols = tuned[1] if (tuned and req.method is None and self.method is None) else 0
        fp = self.footprint(req, ks, method)
        if self.in_use + fp > self.hbm_budget and self.in_use > 0:
            self.admission_waits += 1
            return None
        job = _Job(req, slot)
        job.species = sp
        job.bsc = np.array([bsc[perm[s]] for s in range(req.nsp)], np.float32)
        job.ntype = counts
        job.ks = ks
        with torch.cuda.stream(slot.stream):
            job.rdf = engine.RdfPlan(self.ctx, req.nsp, req.deltar, req.rcrdf, fr0.box, max(req.n, 2))
            self.ctx.set_sq_tile_cols(cols)
            try:
                job.sq = engine.SqPlan(self.ctx, req.nsp, ks, counts)
            finally:
                self.ctx.set_sq_tile_cols(0)
            job.hist = job.rdf.new_hist()
            job.out = job.sq.new_out()
        job.method = method
        job.cols = cols
        job.tune = req.method is None and self.method is None and tuned is None
        job.footprint = fp
        self.in_use += fp
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        slot.req = req
        return job

    def _frame_work(self, job: _Job, buf: int) -> None:
        """H2D copy of pinned buffer `buf`, layout, g(r) and S(Q) of one frame on the job's stream."""
        s, req, n = job.slot, job.req, job.req.n
        box = req.frames[0].box
        s.d_xyz[:n].copy_(s.h_xyz[buf][:n], non_blocking=True)
        s.d_sp[:n].copy_(s.h_sp[buf][:n], non_blocking=True)
        engine.pack_frame(self.ctx, s.d_xyz[:n], s.d_sp[:n], req.nsp, box, s.packed, s.counts, stream=s.stream)
        job.rdf.accumulate(s.packed, n, box, job.hist, stream=s.stream)
        job.sq.accumulate(s.packed, n, box, job.out, engine.METHODS[job.method], stream=s.stream)

    def _enqueue_frame(self, job: _Job) -> None:
        s, req = job.slot, job.req
        k = job.next_frame
        buf = k & 1
        if s.h_ev[buf] is not None:
            s.h_ev[buf].synchronize()  # the pinned buffer still feeds an earlier copy
        fr = req.frames[k]
        n = req.n
        s.h_xyz[buf][:n].numpy()[:] = fr.xyz
        s.h_sp[buf][:n].numpy()[:] = job.species  # frames of a request share atom order and types
        with torch.cuda.stream(s.stream):
            if k == 0 and job.tune:
                # first frame of a new bucket: lay it out, time both S(Q) paths, keep the faster
                s.d_xyz[:n].copy_(s.h_xyz[buf][:n], non_blocking=True)
                s.d_sp[:n].copy_(s.h_sp[buf][:n], non_blocking=True)
                engine.pack_frame(self.ctx, s.d_xyz[:n], s.d_sp[:n], req.nsp, fr.box, s.packed, s.counts,
                                  stream=s.stream)
                job.method, cols, times = self.tuner.tune(self.ctx, job.ks, job.ntype, s.packed, n, fr.box, s.stream)
                self.tuner.record(req.n, req.nsp, req.kset, job.method, cols, times)
                if cols != job.cols:  # the job's plan takes the tuned tile width
                    job.sq.close()
                    self.ctx.set_sq_tile_cols(cols)
                    try:
                        job.sq = engine.SqPlan(self.ctx, req.nsp, job.ks, job.ntype)
                    finally:
                        self.ctx.set_sq_tile_cols(0)
                    job.cols = cols
            graphed = self.use_graphs and len(req.frames) >= 4
            if graphed and k >= 1 and job.graphs[buf] is None:
                # capture this frame's launch sequence (no device synchronisation: other requests keep
                # running on their streams); later frames using the same pinned buffer replay it
                g = torch.cuda.CUDAGraph()
                g.capture_begin(capture_error_mode="relaxed")
                try:
                    self._frame_work(job, buf)
                finally:
                    g.capture_end()
                job.graphs[buf] = g
            if graphed and job.graphs[buf] is not None:
                job.graphs[buf].replay()
            else:
                self._frame_work(job, buf)
            ev = torch.cuda.Event()
            ev.record(s.stream)
            s.h_ev[buf] = ev
        job.next_frame += 1
        if job.next_frame == len(req.frames):
            with torch.cuda.stream(s.stream):
                job.h_hist = job.hist.to("cpu", non_blocking=True)
                job.h_out = job.out.to("cpu", non_blocking=True)
                job.done_event = torch.cuda.Event()
                job.done_event.record(s.stream)

    def _finish(self, job: _Job, t0: float) -> Result:
        req = job.req
        hist = job.h_hist.numpy().astype(np.uint64)
        out = job.h_out.numpy()
        nconf = len(req.frames)
        rdf = normalise_rdf(hist, req.nsp, job.rdf.lsmax, req.deltar, refsem.volume(req.frames[0].box),
                            job.ntype, nconf)
        sq = normalise_sq(out, job.ks, job.ntype, job.bsc, nconf)
        res = Result(rid=req.rid, hist=hist, sq_sums=out, rdf=rdf, sq=sq, method=job.method, arrival=req.arrival,
                     done=time.perf_counter() - t0, nframes=nconf)
        self._release(job)
        return res

    # ---- the loop ---------------------------------------------------------------------
    def run(self, requests: Sequence[Request], realtime: bool = True, on_turn=None) -> List[Result]:
        """Serves `requests` (arrival times in seconds from now when realtime, else all at once).
        ``on_turn(server, turn)``, if given, is called at the start of every turn of the loop."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue: collections.deque = collections.deque()
        jobs: List[_Job] = []
        results: List[Result] = []
        t0 = time.perf_counter()
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        turn = 0
        while pending or queue or jobs:
            if on_turn is not None:
                on_turn(self, turn)
            turn += 1
            self._apply_cancels(pending, queue, jobs)
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.popleft())
            # admission in arrival order within each class: small requests join the fused launch,
            # others take a free slot, while the HBM budget allows; a request that cannot start
            # blocks the later ones of its own class only
            blocked = set()
            kept = collections.deque()
            while queue:
                req = queue.popleft()
                if req.n > self.n_max:
                    raise ValueError(f"request {req.rid}: {req.n} atoms exceed the server's n_max {self.n_max}")
                fuse = self._fusable(req)
                job = None
                if fuse not in blocked:
                    if fuse:
                        job = self._start_fused(req, [j for j in jobs if j.fused])
                    else:
                        slot = next((sl for sl in self.slots if sl.req is None), None)
                        job = self._start(req, slot) if slot is not None else None
                if job is None:
                    blocked.add(fuse)
                    kept.append(req)
                    if len(blocked) == 2:
                        kept.extend(queue)
                        queue.clear()
                else:
                    jobs.append(job)
            queue.extend(kept)
            # one frame per running request per turn: the packed requests in one fused launch
            progressed = self._fused_turn([j for j in jobs if j.fused])
            for job in jobs:
                if not job.fused and job.next_frame < len(job.req.frames):
                    self._enqueue_frame(job)
                    progressed = True
            # completions
            still = []
            for job in jobs:
                if job.done_event is not None and job.done_event.query():
                    if job.cancelled:
                        self._release(job)
                        self.cancelled.append(job.req.rid)
                    else:
                        results.append(self._finish(job, t0))
                else:
                    still.append(job)
            jobs = still
            if not progressed:
                if jobs:
                    jobs[0].done_event.synchronize() if jobs[0].done_event is not None else None
                elif pending and not queue:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - (time.perf_counter() - t0))))
        self.ctx.check()
        self._fuse_cache.clear()
        return results


def summarize(results: Sequence[Result], wall: float) -> Dict[str, float]:
    lat = np.array([r.latency for r in results]) * 1000.0
    frames = sum(r.nframes for r in results)
    return {"requests": len(results), "frames": frames, "wall_s": wall, "requests_per_s": len(results) / wall,
            "frames_per_s": frames / wall, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean())}


def serving_workload(n_requests: int, seed: int = 0, n_lo: float = 1e3, n_hi: float = 2e5) -> List[Request]:
    """Requests with N log-uniform in [n_lo, n_hi] (FCC-derived, density log-uniform in [0.5, 1],
    sigma 0.1), 1-3 species with random fractions, cubic or 1:1:2 boxes, 1-8 frames,
    deltar 0.02, rcrdf = min(L/2, 8), S(Q) qmax 12 with the reference k-set below qmin 3."""
    rng = np.random.default_rng([seed, 0x5e7])
    reqs = []
    for i in range(n_requests):
        n_target = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        rho = math.exp(rng.uniform(math.log(0.5), math.log(1.0)))
        slab = rng.random() < 0.5
        if slab:
            c = max(1, round((n_target / 8.0) ** (1 / 3)))
            cells = (c, c, 2 * c)
        else:
            c = max(1, round((n_target / 4.0) ** (1 / 3)))
            cells = (c, c, c)
        nsp = int(rng.integers(1, 4))
        fr = tuple(rng.dirichlet(np.ones(nsp)) * 0.9 + 0.1 / nsp)
        spec = FCCSpec(cells=cells, density=rho, sigma=0.1, fractions=fr, seed=int(rng.integers(1 << 30)))
        nfr = int(rng.integers(1, 9))
        frames = [spec.frame(k) for k in range(nfr)]
        L = float(np.min(spec.box))
        reqs.append(Request(rid=i, frames=frames, nsp=nsp, deltar=0.02, rcrdf=min(L / 2, 8.0), qmax=12.0, qmin=3.0))
    return reqs
