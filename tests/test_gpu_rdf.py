"""g_ab(r) on the GPU against the CPU oracle: bit-exact pair counts and edge statistics."""
import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import frames, refsem
from trj_analysis_b200._lib import TrjError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trj_analysis_b200 import engine
    c = engine.Context(0)
    yield c
    c.close()


def gpu_counts(ctx, fr, nsp, deltar, rcrdf, species=None, nframes_same=1):
    from trj_analysis_b200 import engine
    sp = (fr.types - 1) if species is None else species
    stage = engine.FrameStage(ctx, max(fr.n, 1), nsp)
    rdf = engine.RdfPlan(ctx, nsp, deltar, rcrdf, fr.box, max(fr.n, 1))
    hist = rdf.new_hist()
    edge = torch.zeros(4, dtype=torch.int64, device="cuda")
    for _ in range(nframes_same):
        n = stage.upload_and_pack(fr.xyz, sp, fr.box)
        rdf.accumulate(stage.packed, n, fr.box, hist, edge)
    ctx.check()
    out = hist.cpu().numpy().astype(np.uint64), edge.cpu().numpy().astype(np.uint64), rdf
    rdf.close()
    return out


def oracle_counts(fr, nsp, deltar, rcrdf, species=None, cells=False):
    sp = (fr.types - 1) if species is None else species
    pos, sps, off = orc.layout(fr.xyz, sp, fr.box, nsp)
    p = refsem.rdf_params(nsp, deltar, rcrdf, fr.box)
    return orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, nsp, cells=cells), p


CASES = [
    # (name, spec, deltar, rcrdf, oracle uses cells)
    ("allpairs_1sp", frames.FCCSpec(cells=(5, 5, 5), sigma=0.12, seed=1), 0.02, 1e9, False),
    ("allpairs_3sp", frames.FCCSpec(cells=(6, 6, 6), sigma=0.1, fractions=(0.5, 0.3, 0.2), replace_frac=0.02,
                                    seed=2), 0.01, 1e9, False),
    ("cells_3sp", frames.FCCSpec(cells=(10, 10, 10), sigma=0.1, fractions=(0.5, 0.3, 0.2), replace_frac=0.02,
                                 seed=3), 0.01, 2.5, True),
    ("cells_noncubic", frames.FCCSpec(cells=(8, 9, 20), sigma=0.1, fractions=(0.5, 0.5), seed=4), 0.02, 3.0, True),
    ("cells_mixed_axes", frames.FCCSpec(cells=(3, 12, 12), sigma=0.1, fractions=(0.7, 0.3), seed=5), 0.02, 2.4,
     True),
    ("cells_3_per_axis", frames.FCCSpec(cells=(7, 7, 7), sigma=0.1, seed=6), 0.02, 3.9, True),
    # 5 cells per axis (no minimum image inside the box) with ~562 atoms per cell: two home rounds of
    # 512 and self tasks whose neighbours span two staged chunks, with the box cull active.
    ("cells_fast_rounds", frames.FCCSpec(cells=(26, 26, 26), density=1.0, sigma=0.1, fractions=(0.5, 0.5),
                                         seed=9), 0.02, 8.2, True),
]


@pytest.mark.parametrize("name,spec,deltar,rcrdf,cells", CASES, ids=[c[0] for c in CASES])
def test_rdf_counts_bit_exact(ctx, name, spec, deltar, rcrdf, cells):
    fr = spec.frame(0)
    nsp = len(spec.fractions)
    (h_o, e_o), p = oracle_counts(fr, nsp, deltar, rcrdf, cells=cells)
    h_g, e_g, plan = gpu_counts(ctx, fr, nsp, deltar, rcrdf)
    assert plan.lsmax == p.lsmax
    assert np.array_equal(h_g, h_o)
    assert int(e_g[2]) == int(e_o[2]) == int(h_o.sum())
    assert int(e_g[0]) == int(e_o[0])
    assert int(e_g[1]) == int(e_o[1])


def test_rdf_binary_precision_config_one_frame(ctx):
    """N=62,500 binary 80:20, deltar=0.01, rcrdf=10 (4 cells per axis)."""
    spec = frames.c2_spec()
    fr = spec.frame(0)
    (h_o, e_o), p = oracle_counts(fr, 2, 0.01, 10.0, cells=True)
    h_g, e_g, plan = gpu_counts(ctx, fr, 2, 0.01, 10.0)
    assert plan.cells == (4, 4, 4)
    assert np.array_equal(h_g, h_o)
    assert np.array_equal(e_g[:3], e_o)


def test_rdf_accumulates_over_frames(ctx):
    spec = frames.FCCSpec(cells=(6, 6, 6), sigma=0.1, fractions=(0.5, 0.5), seed=8)
    fr = spec.frame(2)
    (h_o, _), _ = oracle_counts(fr, 2, 0.02, 2.0, cells=True)
    h_g, _, _ = gpu_counts(ctx, fr, 2, 0.02, 2.0, nframes_same=3)
    assert np.array_equal(h_g, 3 * h_o)


def test_rdf_unfolded_and_negative_coordinates(ctx):
    spec = frames.FCCSpec(cells=(6, 6, 6), sigma=0.1, seed=9)
    fr = spec.frame(0)
    rng = np.random.default_rng(0)
    shift = rng.integers(-3, 4, size=fr.xyz.shape).astype(np.float32) * fr.box
    fr2 = frames.Frame(xyz=(fr.xyz + shift).astype(np.float32), types=fr.types, box=fr.box)
    (h_o, e_o), _ = oracle_counts(fr2, 1, 0.02, 2.5, cells=True)
    h_g, e_g, _ = gpu_counts(ctx, fr2, 1, 0.02, 2.5)
    assert np.array_equal(h_g, h_o)
    assert np.array_equal(e_g[:3], e_o)


def test_rdf_duplicates_and_tiny_frames(ctx):
    box = np.array([10.0, 10.0, 10.0], np.float32)
    xyz = np.array([[1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [1.5, 1.0, 1.0], [9.9, 1.0, 1.0]], np.float32)
    fr = frames.Frame(xyz=xyz, types=np.ones(4, np.int32), box=box)
    (h_o, e_o), _ = oracle_counts(fr, 1, 0.1, 4.0)
    h_g, e_g, _ = gpu_counts(ctx, fr, 1, 0.1, 4.0)
    assert np.array_equal(h_g, h_o)
    one = frames.Frame(xyz=xyz[:1], types=np.ones(1, np.int32), box=box)
    h1, e1, _ = gpu_counts(ctx, one, 1, 0.1, 4.0)
    assert h1.sum() == 0


def test_rdf_nan_positions_raise_data_error(ctx):
    from trj_analysis_b200 import engine
    spec = frames.FCCSpec(cells=(3, 3, 3), seed=10)
    fr = spec.frame(0)
    xyz = fr.xyz.copy()
    xyz[5, 1] = np.nan
    stage = engine.FrameStage(ctx, fr.n, 1)
    stage.upload_and_pack(xyz, fr.types - 1, fr.box)
    with pytest.raises(TrjError) as ei:
        ctx.check()
    assert ei.value.code == -5
    ctx.check()  # status cleared after the report


def test_rdf_capacity_error(ctx):
    from trj_analysis_b200 import engine
    spec = frames.FCCSpec(cells=(3, 3, 3), seed=10)
    fr = spec.frame(0)
    rdf = engine.RdfPlan(ctx, 1, 0.1, 2.0, fr.box, 10)
    hist = rdf.new_hist()
    packed = torch.zeros((fr.n, 4), device="cuda")
    with pytest.raises(TrjError) as ei:
        rdf.accumulate(packed, fr.n, fr.box, hist)
    assert ei.value.code == -4
    rdf.close()


def test_pack_matches_oracle_layout(ctx):
    from trj_analysis_b200 import engine
    spec = frames.FCCSpec(cells=(9, 9, 9), sigma=0.2, fractions=(0.2, 0.5, 0.3), replace_frac=0.1, seed=12)
    fr = spec.frame(0)
    xyz = fr.xyz.copy()
    xyz[::7] -= fr.box  # negative coordinates stay negative after the fold
    stage = engine.FrameStage(ctx, fr.n, 3)
    n = stage.upload_and_pack(xyz, fr.types - 1, fr.box)
    ctx.check()
    pos, sp, off = orc.layout(xyz, fr.types - 1, fr.box, 3)
    got = stage.packed[:n].cpu().numpy()
    assert np.array_equal(got[:, :3], pos)
    assert np.array_equal(got[:, 3].view(np.int32), sp)
    assert np.array_equal(stage.counts.cpu().numpy(), np.diff(off))


@pytest.mark.parametrize("cells,nrandom", [((8, 8, 8), 64), ((3, 3, 3), 9), ((10, 10, 4), 33)])
def test_s2n_matches_oracle(cells, nrandom):
    """Number fluctuations: exact int64 sums against the oracle at the GPU's own sample points; the points
    are the same every frame and lie in the box."""
    import torch
    from oracle import orc
    from trj_analysis_b200 import engine, frames, refsem
    ctx = engine.Context(0)
    spec = frames.FCCSpec(cells=cells, sigma=0.1, fractions=(0.5, 0.5), seed=7)
    frs = [spec.frame(i) for i in range(2)]
    box = frs[0].box
    stage = engine.FrameStage(ctx, frs[0].n, 2)
    plan = engine.RdfPlan(ctx, 2, 0.05, 0.0, box, frs[0].n)
    hist = plan.new_hist()
    gi, g2i = plan.new_s2n()
    want_gi = np.zeros(plan.lsmax + 1, np.int64)
    want_g2i = np.zeros(plan.lsmax + 1, np.int64)
    pts_seen = []
    for fr in frs:
        n = stage.upload_and_pack(fr.xyz, fr.types - 1, box)
        plan.accumulate(stage.packed, n, box, hist)
        pts = torch.zeros(3 * nrandom, dtype=torch.float32, device=ctx.torch_device)
        plan.s2n(nrandom, gi, g2i, points=pts)
        p = pts.cpu().numpy().reshape(-1, 3)
        pts_seen.append(p)
        pos, sp, off = orc.layout(fr.xyz, fr.types - 1, box, 2)
        a, b = orc.s2n_counts(pos, box, plan.side2, 0.05, plan.lsmax, p)
        want_gi += a
        want_g2i += b
    ctx.check()
    np.testing.assert_array_equal(pts_seen[0], pts_seen[1])
    assert np.all(pts_seen[0] > 0) and np.all(pts_seen[0] <= box)
    assert len(np.unique(pts_seen[0][:, 0])) == nrandom
    np.testing.assert_array_equal(gi.cpu().numpy(), want_gi)
    np.testing.assert_array_equal(g2i.cpu().numpy(), want_g2i)
    assert want_gi[-1] > 0
    plan.close()
    ctx.close()


def test_session_writes_s2n(tmp_path):
    from trj_analysis_b200 import analysis
    spec = frames.FCCSpec(cells=(6, 6, 6), sigma=0.1, seed=8)
    cfg = analysis.Config(nsp=1, sp_types_selected=(1,), run_sq=False, deltar=0.05, nrandom=24)
    s = analysis.Session(cfg).run(list(spec.frames(3)))
    files = s.printrdf(str(tmp_path))
    assert files[-1].endswith("s2n.dat")
    res = s.rdf_results()
    assert res["s2n"].shape == res["r"].shape and np.all(np.isfinite(res["s2n"]))
    assert np.all(res["s2n"] >= -1e-9)  # a variance
    s.close()
