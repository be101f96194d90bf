"""Charge-weighted g_qq(r) and S_qq(Q) on the GPU against the oracle, through the C ABI.

g_qq: the counts of the charged call equal the oracle's (bit-exact, and equal to the uncharged
call's); the FP64 charge-product sums over avq2 agree with the oracle's FP64 sums to
1e-12 * (max |q|^2 * pairs in the bin) / avq2 (only the summation order differs).
S_qq: the charge density rho_q(k) is checked per vector like a species density, with the atom count
replaced by sum |q_j| (plain: 2e-6, split: 3e-5 per unit weight), and the shell sums of all
(nsp+1)(nsp+2)/2 rows with the 1e-5 shell tolerance of the species rows.
"""
import math

import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import analysis, frames, refsem
from trj_analysis_b200.refsem import F32

pytestmark = pytest.mark.gpu

REL_SHELL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from trj_analysis_b200 import engine
    c = engine.Context(0)
    yield c
    c.close()


CASES = {
    # small box: fewer than 3 cells per axis -> the all-pairs form of the pair kernel
    "1sp_allpairs": frames.FCCSpec(cells=(3, 3, 3), sigma=0.12, seed=31, charges=(1.0,), charge_jitter=0.3),
    "3sp_cells": frames.FCCSpec(cells=(9, 9, 9), sigma=0.1, fractions=(0.5, 0.3, 0.2), replace_frac=0.02, seed=32,
                                charges=(1.0, -0.8476, 0.4238), charge_jitter=0.05),
    "2sp_species_constant": frames.FCCSpec(cells=(8, 8, 12), sigma=0.1, fractions=(0.5, 0.5), seed=33,
                                           charges=(1.0, -1.0)),
}


def _rdf_setup(fr):
    rc = float(F32(min(fr.box) / F32(2)))
    deltar = 0.02
    lsmax = int(math.floor(float(F32(rc / deltar)) + 0.5)) + 1
    return rc, deltar, lsmax


@pytest.mark.parametrize("name", list(CASES))
def test_pack_carries_charges_in_packed_order(ctx, name):
    from trj_analysis_b200 import engine
    spec = CASES[name]
    fr = spec.frame(0)
    nsp = len(spec.fractions)
    stage = engine.FrameStage(ctx, fr.n, nsp, charged=True)
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box, charges=fr.charges)
    plain = engine.FrameStage(ctx, fr.n, nsp)
    plain.upload_and_pack(fr.xyz, fr.types - 1, fr.box)
    ctx.check()
    pos, sp, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp, charges=fr.charges)
    np.testing.assert_array_equal(stage.qpacked[:n].cpu().numpy(), qs)
    np.testing.assert_array_equal(stage.packed[:n].cpu().numpy(), plain.packed[:n].cpu().numpy())


@pytest.mark.parametrize("name", list(CASES))
def test_rdf_charged_matches_oracle(ctx, name):
    from trj_analysis_b200 import engine
    spec = CASES[name]
    nsp = len(spec.fractions)
    fr0 = spec.frame(0)
    rc, deltar, lsmax = _rdf_setup(fr0)
    stage = engine.FrameStage(ctx, fr0.n, nsp, charged=True)
    plan = engine.RdfPlan(ctx, nsp, deltar, rc, fr0.box, fr0.n)
    assert plan.lsmax == lsmax
    hist, gqq = plan.new_hist(), plan.new_gqq()
    edge = torch.zeros(4, dtype=torch.int64, device=ctx.torch_device)
    hist_plain = plan.new_hist()
    want_h = np.zeros((plan.nit, lsmax), np.uint64)
    want_q = np.zeros(lsmax)
    scale = np.zeros(lsmax)
    for f in range(2):
        fr = spec.frame(f)
        q = fr.charges.copy()
        q[::7] *= np.float32(-1.5)  # charges that change between frames
        n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box, charges=q)
        plan.accumulate(stage.packed, n, fr.box, hist, edge, qpacked=stage.qpacked, gqq=gqq)
        plan.accumulate(stage.packed, n, fr.box, hist_plain)
        pos, sp, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp, charges=q)
        h, _, g = orc.rdf_charged(pos, sp, qs, fr.box, plan.side2, deltar, lsmax, nsp)
        a2 = orc.avq2(qs)
        want_h += h
        want_q += g / a2
        scale += float(np.abs(qs).max()) ** 2 * h.sum(axis=0).astype(np.float64) / a2
    ctx.check()
    got_h = hist.cpu().numpy().astype(np.uint64)
    np.testing.assert_array_equal(got_h, want_h)
    np.testing.assert_array_equal(hist_plain.cpu().numpy().astype(np.uint64), want_h)
    got_q = gqq.cpu().numpy()
    assert np.all(np.abs(got_q - want_q) <= 1e-12 * scale + 1e-12), np.abs(got_q - want_q).max()
    assert np.any(want_q != 0)


def test_rdf_charged_zero_charges_give_non_finite(ctx):
    """avq2 = 0: the reference's gqq_d/avq2 is 0/0; the same IEEE result here."""
    from trj_analysis_b200 import engine
    spec = CASES["3sp_cells"]
    fr = spec.frame(0)
    rc, deltar, lsmax = _rdf_setup(fr)
    stage = engine.FrameStage(ctx, fr.n, 3, charged=True)
    plan = engine.RdfPlan(ctx, 3, deltar, rc, fr.box, fr.n)
    hist, gqq = plan.new_hist(), plan.new_gqq()
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box, charges=np.zeros(fr.n, np.float32))
    plan.accumulate(stage.packed, n, fr.box, hist, qpacked=stage.qpacked, gqq=gqq)
    ctx.check()
    assert np.all(np.isnan(gqq.cpu().numpy()))


def _sq_gpu(ctx, fr, nsp, ks, method):
    from trj_analysis_b200 import engine
    stage = engine.FrameStage(ctx, fr.n, nsp, charged=True)
    counts = np.bincount(fr.types - 1, minlength=nsp)
    plan = engine.SqPlan(ctx, nsp, ks, counts, charged=True)
    out = plan.new_out()
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box, charges=fr.charges)
    plan.accumulate(stage.packed, n, fr.box, out, engine.METHODS[method], qpacked=stage.qpacked)
    rho = plan.rho().cpu().numpy()
    ctx.check()
    res = out.cpu().numpy()
    plan.close()
    return rho, res


def _shell_check(res, ref, ndens):
    rows = refsem.pair_rows(ndens)
    diag = {a: ref[:, refsem.pair_row(a, a, ndens)] for a in range(ndens)}
    scale = np.stack([np.sqrt(np.abs(diag[a] * diag[b])) for a, b in rows], axis=1)
    live = scale > 0
    rel = np.abs(res - ref)[live] / scale[live]
    assert rel.max(initial=0) <= REL_SHELL, rel.max()


SQ_CASES = [("3sp_cells", "ref", 7.0, 3.0), ("2sp_species_constant", "full+axes", 6.0, 2.0),
            ("1sp_allpairs", "full", 5.0, None)]


@pytest.mark.parametrize("method", ["plain", "split"])
@pytest.mark.parametrize("case", SQ_CASES, ids=[c[0] for c in SQ_CASES])
def test_sq_charged_matches_oracle(ctx, case, method):
    name, mode, qmax, qmin = case
    spec = CASES[name]
    fr = spec.frame(0)
    nsp = len(spec.fractions)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin, seed=5, per_shell=30)
    rho_g, res = _sq_gpu(ctx, fr, nsp, ks, method)
    assert rho_g.shape == (nsp + 1, ks.nvec)
    pos, sp, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp, charges=fr.charges)
    rho_o = np.concatenate([orc.rho_fp64(pos, off, fr.box, ks.vectors),
                            orc.rho_charge_fp64(pos, qs, fr.box, ks.vectors)[None, :]])
    per = 2e-6 if method == "plain" else 3e-5
    for a in range(nsp + 1):
        weight = (off[a + 1] - off[a]) if a < nsp else float(np.abs(qs.astype(np.float64)).sum())
        err = np.abs(rho_g[a] - rho_o[a]).max()
        assert err <= per * weight + (1e-6 if method == "plain" else 1e-5), (a, err, weight)
    ref = orc.bin_sums(rho_o, ks.bins, ks.weights, ks.nbins)
    _shell_check(res, ref, nsp + 1)


def test_sq_plans_refuse_the_other_call(ctx):
    from trj_analysis_b200 import _lib, engine
    spec = CASES["3sp_cells"]
    fr = spec.frame(0)
    ks = refsem.make_kset("ref", fr.box, 5.0, 2.0)
    counts = np.bincount(fr.types - 1, minlength=3)
    stage = engine.FrameStage(ctx, fr.n, 3, charged=True)
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box, charges=fr.charges)
    charged = engine.SqPlan(ctx, 3, ks, counts, charged=True)
    plain = engine.SqPlan(ctx, 3, ks, counts)
    out_c, out_p = charged.new_out(), plain.new_out()
    box = _lib.box3(fr.box)
    rc = ctx.lib.trj_sq_accumulate(charged.h, engine._ptr(stage.packed), n, box, _lib.TRJ_SQ_PLAIN_FP32,
                                   engine._ptr(out_c), engine._stream(None))
    assert rc == _lib.TRJ_ERR_INVALID
    rc = ctx.lib.trj_sq_accumulate_charged(plain.h, engine._ptr(stage.packed), engine._ptr(stage.qpacked), n, box,
                                           _lib.TRJ_SQ_PLAIN_FP32, engine._ptr(out_p), engine._stream(None))
    assert rc == _lib.TRJ_ERR_INVALID
    ctx.check()
    charged.close()
    plain.close()


def test_session_with_charges_writes_g_qq_and_s_qq(ctx, tmp_path):
    spec = CASES["3sp_cells"]
    frs = list(spec.frames(2))
    cfg = analysis.Config(nsp=3, sp_types_selected=(1, 2, 3), deltar=0.02, qmax=6.0, qmin=2.0, method="split")
    s = analysis.Session(cfg, ctx=ctx).run(frs)
    assert s.ex_qc
    files = s.printrdf(str(tmp_path)) + s.printSQ(str(tmp_path))
    g = open(files[0]).read().splitlines()
    assert "g_qq(r)" in g[0]
    sq = open(files[1]).read().splitlines()
    assert "S_qq(Q)" in sq[0]
    # g_qq against the oracle's charge-product sums, normalised as printrdf does
    res = s.rdf_results()
    lsmax = s.rdf.lsmax
    want = np.zeros(lsmax)
    for fr in frs:
        pos, sp, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, 3, charges=fr.charges)
        _, _, gq = orc.rdf_charged(pos, sp, qs, fr.box, s.rdf.side2, cfg.deltar, lsmax, 3)
        want += gq / orc.avq2(qs)
    ref = analysis.normalise_rdf(s.rdf_transfer(), 3, lsmax, cfg.deltar, s.volumen, s.ntype, 2, gqq=want)
    np.testing.assert_allclose(res["g_qq"], ref["g_qq"], rtol=1e-9, atol=1e-9)
    # S_qq shell sums against the oracle
    sq_res = s.sq_results()
    ks = s.kset
    tot = np.zeros(ks.nbins)
    for fr in frs:
        pos, sp, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, 3, charges=fr.charges)
        rq = orc.rho_charge_fp64(pos, qs, fr.box, ks.vectors)
        np.add.at(tot, ks.bins, ks.weights * np.abs(rq) ** 2)
    nq = ks.nq.astype(np.float64)
    sl = slice(1, ks.nqmax + 1)
    live = nq[sl] > 0
    want_sqq = (tot / orc.avq2(s.charges) / (s.ntype.sum() * 2 * np.where(nq > 0, nq, 1.0)))[sl]
    got = sq_res["s_qq"]
    rel = np.abs(got[live] - want_sqq[live]) / np.abs(want_sqq[live])
    assert rel.max() <= REL_SHELL, rel.max()
    s.close()


def test_species_charge_mode_matches_atom_mode(ctx):
    """Species-constant charges: the derived g_qq/S_qq equal those of the charge-weighted kernels."""
    spec = CASES["2sp_species_constant"]
    frs = list(spec.frames(2))
    res = {}
    for mode in ("atom", "species"):
        cfg = analysis.Config(nsp=2, sp_types_selected=(1, 2), deltar=0.02, qmax=6.0, qmin=2.0, method="plain",
                              charge_mode=mode)
        s = analysis.Session(cfg, ctx=ctx).run(frs)
        res[mode] = (s.rdf_results(), s.sq_results(), s.device_charges)
        s.close()
    assert res["atom"][2] and not res["species"][2]
    np.testing.assert_allclose(res["species"][0]["g_qq"], res["atom"][0]["g_qq"], rtol=1e-10, atol=1e-10)
    a, b = res["atom"][1]["s_qq"], res["species"][1]["s_qq"]
    live = np.isfinite(a)
    assert np.all(np.abs(a[live] - b[live]) <= REL_SHELL * np.abs(a[live]) + 1e-9)


def test_species_charge_mode_rejects_per_atom_charges(ctx):
    spec = CASES["3sp_cells"]
    cfg = analysis.Config(nsp=3, sp_types_selected=(1, 2, 3), charge_mode="species")
    s = analysis.Session(cfg, ctx=ctx)
    with pytest.raises(ValueError, match="different charges"):
        s.add_frame(spec.frame(0))
    s.close()
