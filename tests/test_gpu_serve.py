"""The request loop: isolation (same bits alone and in a mix), admission, graphs, parity."""
import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import refsem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    from trj_analysis_b200.serve import serving_workload
    reqs = serving_workload(12, seed=7, n_lo=500, n_hi=6000)
    return reqs


def _run(reqs, **kw):
    from trj_analysis_b200.serve import Server
    srv = Server(slots=kw.pop("slots", 6), n_max=1 << 14, **kw)
    res = srv.run(reqs, realtime=False)
    return srv, {r.rid: r for r in res}


def test_results_identical_alone_and_in_mix(workload):
    _, mixed = _run(workload, method="split")
    assert len(mixed) == len(workload)
    for req in workload[:6]:
        _, alone = _run([req], slots=1, method="split")
        a, b = alone[req.rid], mixed[req.rid]
        assert np.array_equal(a.hist, b.hist)
        assert np.array_equal(a.sq_sums, b.sq_sums)


def test_graph_replay_matches_eager(workload):
    multi = [r for r in workload if len(r.frames) >= 4][:3]
    assert multi
    _, g = _run(multi, method="plain", use_graphs=True)
    _, e = _run(multi, method="plain", use_graphs=False)
    for r in multi:
        assert np.array_equal(g[r.rid].hist, e[r.rid].hist)
        assert np.array_equal(g[r.rid].sq_sums, e[r.rid].sq_sums)


def test_admission_under_small_budget(workload):
    srv, res = _run(workload, hbm_budget=1)
    assert len(res) == len(workload)
    assert srv.admission_waits > 0


def test_served_counts_match_oracle(workload):
    _, res = _run(workload[:4], method="split")
    for req in workload[:4]:
        H = 0
        sel = sorted(set(int(t) for t in np.unique(req.frames[0].types)))[: req.nsp]
        sp = refsem.species_by_first_appearance(req.frames[0].types, sel)[0]
        p = refsem.rdf_params(req.nsp, req.deltar, req.rcrdf, req.frames[0].box)
        for fr in req.frames:
            pos, sps, off = orc.layout(fr.xyz, sp, fr.box, req.nsp)
            h, _ = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, req.nsp, cells=True)
            H = H + h
        assert np.array_equal(res[req.rid].hist, H)


def test_cancel_running_and_queued_requests(workload):
    """A request cancelled while it runs stops after the frames already on its stream and releases its
    slot and budget; one cancelled while queued never starts; the others are unchanged."""
    from trj_analysis_b200.serve import Server
    reqs = sorted(workload, key=lambda r: -len(r.frames))[:6]
    assert len(reqs[0].frames) >= 4
    running, queued = reqs[0].rid, reqs[-1].rid

    def hook(srv, turn):
        if turn == 1:
            srv.cancel(running)
            srv.cancel(queued)

    srv = Server(slots=2, n_max=1 << 14, method="split")
    res = {r.rid: r for r in srv.run(reqs, realtime=False, on_turn=hook)}
    assert sorted(srv.cancelled) == sorted([running, queued])
    assert set(res) == {r.rid for r in reqs} - {running, queued}
    assert srv.in_use == 0 and all(s.req is None for s in srv.slots)
    for req in reqs:
        if req.rid in res:
            _, alone = _run([req], slots=1, method="split")
            assert np.array_equal(alone[req.rid].hist, res[req.rid].hist)
            assert np.array_equal(alone[req.rid].sq_sums, res[req.rid].sq_sums)


def test_autotuner_picks_method_and_tile_width(workload):
    from trj_analysis_b200.serve import Autotuner, Server
    tuner = Autotuner()
    srv = Server(slots=2, n_max=1 << 14, autotuner=tuner, fuse_max_atoms=0)
    res = srv.run(workload[:3], realtime=False)
    assert len(res) == 3 and tuner.table
    for e in tuner.table.values():
        assert (e["method"], e["cols"]) in Autotuner.CANDIDATES and e["ms"]


def test_fused_requests_match_the_per_request_plain_path(workload):
    """Small requests packed into fused launches give the bits of the per-request plain method, in a mix
    with requests that take slots (split method: those above the fused size)."""
    fused_srv, fused = _run(workload, fuse_max_atoms=3000)
    assert 0 < fused_srv.fused_requests < len(workload) and fused_srv.fuse_turns > 0
    _, slots = _run(workload, fuse_max_atoms=0, method="plain")
    for req in workload:
        a, b = fused[req.rid], slots[req.rid]
        assert np.array_equal(a.hist, b.hist)
        if req.n <= 3000:
            assert a.method == "plain"
            assert np.array_equal(a.sq_sums, b.sq_sums)


def test_fused_alone_equals_in_mix_and_cancel(workload):
    """A packed request gives the same bits alone and among others; one cancelled while packed leaves the
    others unchanged and releases its budget."""
    from trj_analysis_b200.serve import Server
    reqs = sorted(workload, key=lambda r: -len(r.frames))[:6]
    victim = reqs[0].rid
    assert len(reqs[0].frames) >= 3

    def hook(srv, turn):
        if turn == 1:
            srv.cancel(victim)

    srv = Server(slots=2, n_max=1 << 14)
    res = {r.rid: r for r in srv.run(reqs, realtime=False, on_turn=hook)}
    assert srv.cancelled == [victim] and victim not in res
    assert srv.in_use == 0 and srv.fused_requests == len(reqs)
    for req in reqs[1:4]:
        _, alone = _run([req], slots=1)
        assert np.array_equal(alone[req.rid].hist, res[req.rid].hist)
        assert np.array_equal(alone[req.rid].sq_sums, res[req.rid].sq_sums)
