"""Multi-rank path on the CPU: two gloo ranks share a trajectory round-robin, each accumulates
its frames (oracle counts and FP64 S sums standing in for the device accumulators), and
replicas.merge / replicas.run_sharded must give every rank the one-process totals."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

NFRAMES = 5
NSP = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _trajectory():
    from trj_analysis_b200 import frames
    spec = frames.FCCSpec(cells=(4, 4, 4), fractions=(0.6, 0.4), replace_frac=0.05, seed=17)
    return spec, [spec.frame(i) for i in range(NFRAMES)]


def _frame_sums(fr, kset, p):
    from oracle import orc
    pos, sp, off = orc.layout(fr.xyz, fr.types - 1, fr.box, NSP)
    hist, _ = orc.rdf_counts(pos, sp, fr.box, p.side2, p.deltar, p.lsmax, NSP, cells=True)
    rho = orc.rho_fp64(pos, off, fr.box, kset.vectors)
    s = orc.bin_sums(rho, kset.bins, kset.weights, kset.nbins)
    return hist.astype(np.int64), s


def _setup():
    from trj_analysis_b200 import refsem
    spec, frs = _trajectory()
    p = refsem.rdf_params(NSP, 0.05, 1e9, frs[0].box)
    kset = refsem.make_kset("full", frs[0].box, 4.0)
    return frs, kset, p


class _FakeCtx:
    def check(self, stream=None):
        pass


class _HostSession:
    """The accumulate surface of analysis.Session, on the host (oracle sums)."""

    def __init__(self, kset, p):
        self.kset, self.p = kset, p
        self.ctx = _FakeCtx()
        self.hist = torch.zeros((NSP * (NSP + 1) // 2, p.lsmax), dtype=torch.int64)
        self.sq_out = torch.zeros((kset.nbins, NSP * (NSP + 1) // 2), dtype=torch.float64)
        self.edge = torch.zeros(4, dtype=torch.int64)
        self.nconf = 0

    def add_frame(self, fr):
        h, s = _frame_sums(fr, self.kset, self.p)
        self.hist += torch.from_numpy(h)
        self.sq_out += torch.from_numpy(s)
        self.edge[2] += int(h.sum())
        self.nconf += 1


def _worker(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from trj_analysis_b200 import replicas
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        frs, kset, p = _setup()
        # merge() on explicit accumulators
        hist = torch.zeros((NSP * (NSP + 1) // 2, p.lsmax), dtype=torch.int64)
        sq = torch.zeros((kset.nbins, NSP * (NSP + 1) // 2), dtype=torch.float64)
        mine = replicas.frames_of_rank(NFRAMES, rank, world)
        for i in mine:
            h, s = _frame_sums(frs[i], kset, p)
            hist += torch.from_numpy(h)
            sq += torch.from_numpy(s)
        out = replicas.merge(hist, sq, nframes=len(mine))
        # run_sharded() on a session-shaped object
        sess = _HostSession(kset, p)
        replicas.run_sharded(sess, frs, rank, world)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), hist=out["hist"].numpy(), sq=out["sq_sums"].numpy(),
                 nframes=out["nframes"], s_hist=sess.hist.numpy(), s_sq=sess.sq_out.numpy(),
                 s_nconf=sess.nconf, s_counted=int(sess.edge[2]))
    finally:
        dist.destroy_process_group()


def test_frames_of_rank_partition():
    from trj_analysis_b200 import replicas
    for world in (1, 2, 3, 4):
        got = sorted(i for r in range(world) for i in replicas.frames_of_rank(10, r, world))
        assert got == list(range(10))
    assert replicas.frames_of_rank(5, 1, 2) == [1, 3]
    with pytest.raises(ValueError):
        replicas.frames_of_rank(5, 2, 2)


def test_two_gloo_ranks_merge_to_one_process_totals(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    frs, kset, p = _setup()
    ref_h = np.zeros((NSP * (NSP + 1) // 2, p.lsmax), np.int64)
    ref_s = np.zeros((kset.nbins, NSP * (NSP + 1) // 2))
    for fr in frs:
        h, s = _frame_sums(fr, kset, p)
        ref_h += h
        ref_s += s
    assert ref_h.sum() > 0
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["hist"], ref_h)              # integer counts merge exactly
        assert np.allclose(d["sq"], ref_s, rtol=1e-12, atol=1e-9)
        assert int(d["nframes"]) == NFRAMES
        assert np.array_equal(d["s_hist"], ref_h)
        assert np.allclose(d["s_sq"], ref_s, rtol=1e-12, atol=1e-9)
        assert int(d["s_nconf"]) == NFRAMES
        assert int(d["s_counted"]) == int(ref_h.sum())
