"""One trajectory over several ranks: frames are dealt round-robin, each rank accumulates its own
g(r) counts and S(Q) sums, and one all-reduce merges them.

The reference analyses a trajectory on one GPU, frame after frame (trj_analysis.f90:211,217 call
RDFcomp and SQcalc per frame); its accumulators are sums over frames (histomix_d, sqf_d/sqfp_d), so
splitting the frames over ranks and summing the per-rank accumulators gives the same totals.
Counts are uint64 and merge exactly; the FP64 S sums merge in the backend's reduction order.

Works with any torch.distributed backend: ``nccl`` for device tensors on GPU ranks, ``gloo`` for
host tensors.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Optional, Sequence, TypeVar

import torch
import torch.distributed as dist

T = TypeVar("T")


def frames_of_rank(nframes: int, rank: int, world: int) -> List[int]:
    """Frame indices rank `rank` of `world` analyses: rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return list(range(rank, nframes, world))


def shard(frames: Sequence[T], rank: int, world: int) -> List[T]:
    """The frames of one rank, in trajectory order."""
    return [frames[i] for i in frames_of_rank(len(frames), rank, world)]


def merge(hist: Optional[torch.Tensor] = None, sq_sums: Optional[torch.Tensor] = None,
          nframes: Optional[int] = None, group=None) -> Dict[str, object]:
    """Sum the per-rank accumulators in place over `group` (the default group when None).

    hist:     uint64 [nit][lsmax] pair counts (the layout trj_rdf_accumulate writes).
    sq_sums:  float64 [nbins][nit] S sums (the layout trj_sq_accumulate writes).
    nframes:  frames this rank analysed; the returned total is Nconf for the normalisation.
    Every rank must call this with the same tensors' shapes (a collective).
    """
    out: Dict[str, object] = {}
    if hist is not None:
        if hist.dtype not in (torch.uint64, torch.int64):
            raise TypeError("hist must be a 64-bit integer tensor")
        view = hist.view(torch.int64)  # counts < 2^63: the same bits either way
        dist.all_reduce(view, op=dist.ReduceOp.SUM, group=group)
        out["hist"] = hist
    if sq_sums is not None:
        if sq_sums.dtype != torch.float64:
            raise TypeError("sq_sums must be float64")
        dist.all_reduce(sq_sums, op=dist.ReduceOp.SUM, group=group)
        out["sq_sums"] = sq_sums
    if nframes is not None:
        dev = hist.device if hist is not None else (sq_sums.device if sq_sums is not None else torch.device("cpu"))
        t = torch.tensor([int(nframes)], dtype=torch.int64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out["nframes"] = int(t.item())
    return out


def run_sharded(session, frames: Iterable, rank: int, world: int, group=None) -> Dict[str, object]:
    """Analyse this rank's frames with an `analysis.Session`, then merge over the group.

    Afterwards the session's device accumulators (counts, edge statistics, S sums, g_qq and s2n sums) and its frame
    count hold the whole trajectory on every rank, so its printrdf/printSQ give the one-GPU result.
    Needs at least one frame per rank (the plans are sized from a rank's first frame).  Time
    correlations need consecutive frames on one rank and are not sharded.
    """
    frames = list(frames)
    if len(frames) < world:
        raise ValueError(f"{len(frames)} frames for {world} ranks: every rank needs a frame")
    mine = shard(frames, rank, world)
    for fr in mine:
        session.add_frame(fr)
    session.ctx.check()
    out = merge(session.hist, session.sq_out, nframes=len(mine), group=group)
    if session.edge is not None:
        dist.all_reduce(session.edge, op=dist.ReduceOp.SUM, group=group)
    gqq = getattr(session, "gqq", None)
    if gqq is not None:  # charge-product histogram over avq2: a per-frame sum like the counts
        dist.all_reduce(gqq, op=dist.ReduceOp.SUM, group=group)
    for t in (getattr(session, "gi", None), getattr(session, "g2i", None)):  # s2n sums over frames
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    session.nconf = int(out["nframes"])
    return out
