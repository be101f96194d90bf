"""Fused launches over several small requests (trj_batch_*): the counts and S(Q) sums of every request
are those of its own single-request calls bit for bit (pair counts also against the oracle's all-pairs
sweep), alone or in any mix, eager or replayed from a CUDA graph."""
import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import _lib, engine, refsem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return engine.Context(0)


@pytest.fixture(scope="module")
def requests():
    from trj_analysis_b200.serve import serving_workload
    reqs = serving_workload(10, seed=11, n_lo=200, n_hi=9000)
    return reqs


class _State:
    """Plans and accumulators of one request."""

    def __init__(self, ctx, req, n_max=None):
        fr0 = req.frames[0]
        sel = sorted(set(int(t) for t in np.unique(fr0.types)))[: req.nsp]
        self.sp = refsem.species_by_first_appearance(fr0.types, sel)[0].astype(np.int32)
        self.ks = refsem.make_kset(req.kset, fr0.box, req.qmax, req.qmin)
        self.counts = np.bincount(self.sp[self.sp >= 0], minlength=req.nsp)
        self.rdf = engine.RdfPlan(ctx, req.nsp, req.deltar, req.rcrdf, fr0.box, req.n if n_max is None else n_max)
        self.sq = engine.SqPlan(ctx, req.nsp, self.ks, self.counts)
        self.hist = self.rdf.new_hist()
        self.out = self.sq.new_out()
        self.edge = torch.zeros(8, dtype=torch.int64, device=ctx.torch_device)

    def close(self):
        self.rdf.close()
        self.sq.close()


def _single(ctx, req):
    st = _State(ctx, req)
    n = req.n
    packed = torch.empty((n, 4), dtype=torch.float32, device=ctx.torch_device)
    cnt = torch.zeros(16, dtype=torch.int64, device=ctx.torch_device)
    sp = torch.from_numpy(st.sp).to(ctx.torch_device)
    for fr in req.frames:
        xyz = torch.from_numpy(np.ascontiguousarray(fr.xyz, np.float32)).to(ctx.torch_device)
        engine.pack_frame(ctx, xyz, sp, req.nsp, fr.box, packed, cnt)
        st.rdf.accumulate(packed, n, fr.box, st.hist, edge=st.edge)
        st.sq.accumulate(packed, n, fr.box, st.out, engine.METHODS["plain"])
    torch.cuda.synchronize()
    ctx.check()
    res = st.hist.cpu().numpy(), st.out.cpu().numpy(), st.edge.cpu().numpy()
    st.close()
    return res


def _batched(ctx, reqs, graph=False, order=None):
    """All frames of `reqs` through one batch, one frame of each request per turn."""
    batch = engine.Batch(ctx, max_items=16, max_atoms=1 << 17)
    states = {r.rid: _State(ctx, r, n_max=0) for r in reqs}
    stream = torch.cuda.Stream(device=ctx.torch_device)
    graphs = [None, None]
    seq = reqs if order is None else [reqs[i] for i in order]
    for t in range(max(len(r.frames) for r in reqs)):
        buf = t & 1
        batch.begin(buf)
        off = 0
        for r in seq:
            if t < len(r.frames):
                st = states[r.rid]
                fr = r.frames[t]
                batch.stage(buf, off, fr.xyz, st.sp)
                batch.add(buf, st.rdf, st.sq, off, r.n, fr.box, st.hist, st.out, edge=st.edge)
                off += r.n
        with torch.cuda.stream(stream):
            if graph:
                if graphs[buf] is None:
                    g = torch.cuda.CUDAGraph()
                    g.capture_begin()
                    batch.launch(buf, stream)
                    g.capture_end()
                    graphs[buf] = g
                graphs[buf].replay()
            else:
                batch.launch(buf, stream)
        batch.mark(buf, stream)
    stream.synchronize()
    ctx.check()
    res = {r.rid: (st.hist.cpu().numpy(), st.out.cpu().numpy(), st.edge.cpu().numpy())
           for r, st in ((r, states[r.rid]) for r in reqs)}
    graphs = None
    for st in states.values():
        st.close()
    batch.close()
    return res


def test_batch_matches_single_request_calls(ctx, requests):
    mixed = _batched(ctx, requests)
    for r in requests:
        h, o, e = _single(ctx, r)
        bh, bo, be = mixed[r.rid]
        assert np.array_equal(h, bh), f"request {r.rid} (n={r.n}): pair counts differ"
        assert np.array_equal(o, bo), f"request {r.rid} (n={r.n}): S(Q) sums differ"
        # ulp and fma edge counters and the counted pairs agree; the tested-pair count differs by route
        assert np.array_equal(e[:3], be[:3])


def test_batch_counts_match_oracle_all_pairs(ctx, requests):
    res = _batched(ctx, requests[:4])
    for r in requests[:4]:
        st_sp = res[r.rid]
        sel = sorted(set(int(t) for t in np.unique(r.frames[0].types)))[: r.nsp]
        sp = refsem.species_by_first_appearance(r.frames[0].types, sel)[0]
        p = refsem.rdf_params(r.nsp, r.deltar, r.rcrdf, r.frames[0].box)
        H = 0
        for fr in r.frames:
            pos, sps, off = orc.layout(fr.xyz, sp, fr.box, r.nsp)
            h, _ = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, r.nsp, cells=False)
            H = H + h
        assert np.array_equal(st_sp[0].astype(np.uint64), H)


def test_batch_sq_against_fp64(ctx, requests):
    r = max(requests[:5], key=lambda q: q.n)
    res = _batched(ctx, [r])
    sel = sorted(set(int(t) for t in np.unique(r.frames[0].types)))[: r.nsp]
    sp = refsem.species_by_first_appearance(r.frames[0].types, sel)[0]
    ks = refsem.make_kset(r.kset, r.frames[0].box, r.qmax, r.qmin)
    ref = 0
    for fr in r.frames:
        pos, _, off = orc.layout(fr.xyz, sp, fr.box, r.nsp)
        rho = orc.rho_fp64(pos, off, fr.box, ks.vectors)
        ref = ref + orc.bin_sums(rho, ks.bins, ks.weights, ks.nbins)
    got = res[r.rid][1]
    # per shell and species pair, relative to sqrt(S_aa S_bb): the direct sum's bar
    rows = refsem.pair_rows(r.nsp)
    diag = {a: rows.index((a, a)) for a in range(r.nsp)}
    used = np.bincount(ks.bins, minlength=ks.nbins) > 0
    for k, (a, b) in enumerate(rows):
        scale = np.sqrt(np.abs(ref[:, diag[a]] * ref[:, diag[b]]))[used]
        err = np.abs(got[:, k] - ref[:, k])[used] / scale
        assert err.max() < 1e-5, (a, b, err.max())


def test_batch_alone_equals_in_mix_and_order_free(ctx, requests):
    mixed = _batched(ctx, requests, order=list(reversed(range(len(requests)))))
    for r in requests[:3]:
        alone = _batched(ctx, [r])
        for x, y in zip(alone[r.rid], mixed[r.rid]):
            assert np.array_equal(x, y)


def test_batch_graph_replay_matches_eager(ctx, requests):
    eager = _batched(ctx, requests)
    replay = _batched(ctx, requests, graph=True)
    for r in requests:
        for x, y in zip(eager[r.rid], replay[r.rid]):
            assert np.array_equal(x, y)


def test_batch_refuses_plans_it_cannot_run(ctx, requests):
    r = requests[0]
    batch = engine.Batch(ctx, max_items=2, max_atoms=1 << 17, hist_words=64)
    st = _State(ctx, r, n_max=0)
    batch.begin(0)
    with pytest.raises(_lib.TrjError, match="UNSUPPORTED"):  # nit * lsmax > 64 words
        batch.add(0, st.rdf, st.sq, 0, r.n, r.frames[0].box, st.hist, st.out)
    batch2 = engine.Batch(ctx, max_items=1, max_atoms=r.n)
    batch2.begin(0)
    batch2.add(0, st.rdf, st.sq, 0, r.n, r.frames[0].box, st.hist, st.out)
    with pytest.raises(_lib.TrjError, match="CAPACITY"):
        batch2.add(0, st.rdf, st.sq, 0, r.n, r.frames[0].box, st.hist, st.out)
    st.close()
    batch.close()
    batch2.close()


def test_batch_species_count_mismatch_is_reported(ctx, requests):
    """A frame whose species counts differ from the S(Q) plan's is flagged on the host (no write lands
    outside the frame's own range)."""
    r = next(q for q in requests if q.nsp >= 2)
    batch = engine.Batch(ctx, max_items=2, max_atoms=1 << 15)
    st = _State(ctx, r, n_max=0)
    sp = st.sp.copy()
    sp[sp == 1] = 0  # species 1's atoms relabelled: counts no longer match the plan
    batch.begin(0)
    batch.stage(0, 0, r.frames[0].xyz, sp)
    batch.add(0, st.rdf, st.sq, 0, r.n, r.frames[0].box, st.hist, st.out)
    batch.launch(0)
    with pytest.raises(_lib.TrjError):
        ctx.check()
    ctx.check()  # the status word is cleared once reported
    st.close()
    batch.close()


def test_batch_partial_items_and_tiny_frames(ctx, requests):
    """Items with only a pair plan (atoms keep their order), only an S(Q) plan, and frames of one and
    two atoms: each equals its single-request calls."""
    from trj_analysis_b200.frames import Frame
    r = next(q for q in requests if q.nsp >= 2)
    st_full = _State(ctx, r, n_max=0)
    st_g = _State(ctx, r, n_max=0)
    st_s = _State(ctx, r, n_max=0)
    fr = r.frames[0]
    tiny = []
    for n in (1, 2):
        t = Frame(xyz=np.ascontiguousarray(fr.xyz[:n]), types=np.ones(n, np.int32), box=fr.box)
        q = type(r)(rid=1000 + n, frames=[t], nsp=1, deltar=r.deltar, rcrdf=r.rcrdf, qmax=r.qmax, qmin=r.qmin)
        tiny.append((q, _State(ctx, q, n_max=0)))
    batch = engine.Batch(ctx, max_items=8, max_atoms=1 << 16)
    batch.begin(0)
    off = 0
    for st, rdf, sq in ((st_g, st_g.rdf, None), (st_s, None, st_s.sq), (st_full, st_full.rdf, st_full.sq)):
        batch.stage(0, off, fr.xyz, st.sp)
        batch.add(0, rdf, sq, off, r.n, fr.box, st.hist if rdf else None, st.out if sq else None)
        off += r.n
    for q, st in tiny:
        batch.stage(0, off, q.frames[0].xyz, np.zeros(q.n, np.int32))
        batch.add(0, st.rdf, st.sq, off, q.n, fr.box, st.hist, st.out)
        off += q.n
    batch.launch(0)
    torch.cuda.synchronize()
    ctx.check()
    h, o, _ = _single(ctx, type(r)(rid=r.rid, frames=[fr], nsp=r.nsp, deltar=r.deltar, rcrdf=r.rcrdf,
                                   qmax=r.qmax, qmin=r.qmin))
    assert np.array_equal(st_g.hist.cpu().numpy(), h)
    assert np.array_equal(st_s.out.cpu().numpy(), o)
    assert np.array_equal(st_full.hist.cpu().numpy(), h) and np.array_equal(st_full.out.cpu().numpy(), o)
    assert not st_s.hist.any() and not st_g.out.any()
    for q, st in tiny:
        th, to, _ = _single(ctx, q)
        assert np.array_equal(st.hist.cpu().numpy(), th) and np.array_equal(st.out.cpu().numpy(), to)
        if q.n == 1:
            assert not st.hist.any()
        st.close()
    for st in (st_full, st_g, st_s):
        st.close()
    batch.close()
