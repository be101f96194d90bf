"""S_ab(Q) on the GPU against the FP64 oracle.

Tolerances: per vector, |rho_gpu - rho_fp64| <= 2e-6 * n_atoms_of_species + 1e-6
(each term carries <= ~5e-7 absolute phase/sine error); per shell and species pair,
|sum_gpu - sum_fp64| <= 1e-5 * sqrt(sum_aa * sum_bb) -- the relative error of S_aa for
the self rows, and for the cross rows relative to their Cauchy-Schwarz bound (a cross
sum can cancel to ~0, where a ratio to itself means nothing).
"""
import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import frames, refsem

pytestmark = pytest.mark.gpu

REL_SHELL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from trj_analysis_b200 import engine
    c = engine.Context(0)
    yield c
    c.close()


def run_gpu(ctx, fr, nsp, ks, method, nframes=1):
    from trj_analysis_b200 import engine
    stage = engine.FrameStage(ctx, fr.n, nsp)
    counts = np.bincount(fr.types - 1, minlength=nsp)
    plan = engine.SqPlan(ctx, nsp, ks, counts)
    out = plan.new_out()
    for _ in range(nframes):
        n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box)
        plan.accumulate(stage.packed, n, fr.box, out, engine.METHODS[method])
    rho = plan.rho().cpu().numpy()
    ctx.check()
    res = out.cpu().numpy()
    plan.close()
    return rho, res


def oracle_rho(fr, nsp, ks):
    pos, sp, off = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp)
    return orc.rho_fp64(pos, off, fr.box, ks.vectors), off


def shell_scale(ref, nsp):
    rows = refsem.pair_rows(nsp)
    diag = {a: ref[:, refsem.pair_row(a, a, nsp)] for a in range(nsp)}
    return np.stack([np.sqrt(np.abs(diag[a] * diag[b])) for a, b in rows], axis=1)


def check_shells(res, ref, nsp):
    scale = shell_scale(ref, nsp)
    live = scale > 0
    rel = np.abs(res - ref)[live] / scale[live]
    assert rel.max(initial=0) <= REL_SHELL, rel.max()
    assert np.all(res[~live] == 0)


SPECS = {
    "1sp_full": (frames.FCCSpec(cells=(5, 5, 5), sigma=0.12, seed=1), "full", 6.0, None),
    "3sp_ref": (frames.FCCSpec(cells=(6, 6, 6), sigma=0.1, fractions=(0.5, 0.3, 0.2), replace_frac=0.02, seed=2),
                "ref", 8.0, 3.0),
    "2sp_axes_noncubic": (frames.FCCSpec(cells=(6, 6, 12), sigma=0.1, fractions=(0.5, 0.5), seed=3), "full+axes",
                          6.0, 2.0),
    "2sp_sampled": (frames.FCCSpec(cells=(8, 8, 8), sigma=0.1, fractions=(0.8, 0.2), seed=4), "full+sampled", 7.0,
                    2.5),
}


@pytest.mark.parametrize("name", list(SPECS))
def test_sq_plain_matches_fp64_oracle(ctx, name):
    spec, mode, qmax, qmin = SPECS[name]
    fr = spec.frame(0)
    nsp = len(spec.fractions)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin, seed=5, per_shell=30)
    rho_g, res = run_gpu(ctx, fr, nsp, ks, "plain")
    rho_o, off = oracle_rho(fr, nsp, ks)
    for a in range(nsp):
        na = off[a + 1] - off[a]
        assert np.abs(rho_g[a] - rho_o[a]).max() <= 2e-6 * na + 1e-6
    ref = orc.bin_sums(rho_o, ks.bins, ks.weights, ks.nbins)
    check_shells(res, ref, nsp)


def test_sq_accumulates_over_frames(ctx):
    spec, mode, qmax, qmin = SPECS["3sp_ref"]
    fr = spec.frame(1)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin)
    _, r1 = run_gpu(ctx, fr, 3, ks, "plain", nframes=1)
    _, r3 = run_gpu(ctx, fr, 3, ks, "plain", nframes=3)
    assert np.allclose(r3, 3 * r1, rtol=1e-12, atol=0)


def test_sq_deterministic(ctx):
    spec, mode, qmax, qmin = SPECS["1sp_full"]
    fr = spec.frame(0)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin)
    _, a = run_gpu(ctx, fr, 1, ks, "plain")
    _, b = run_gpu(ctx, fr, 1, ks, "plain")
    assert np.array_equal(a, b)


# ---- tensor-core split-BF16 path ------------------------------------------------

SPLIT_CASES = {
    "tiny_1sp_full": (frames.FCCSpec(cells=(3, 3, 3), sigma=0.1, seed=21), "full", 3.0, None),
    "1sp_full": SPECS["1sp_full"],
    "3sp_ref": SPECS["3sp_ref"],
    "2sp_axes_noncubic": SPECS["2sp_axes_noncubic"],
    "2sp_sampled": SPECS["2sp_sampled"],
}


@pytest.mark.parametrize("name", list(SPLIT_CASES))
def test_sq_split_matches_fp64_oracle(ctx, name):
    spec, mode, qmax, qmin = SPLIT_CASES[name]
    fr = spec.frame(0)
    nsp = len(spec.fractions)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin, seed=5, per_shell=30)
    assert ks.dense.any()
    rho_g, res = run_gpu(ctx, fr, nsp, ks, "split")
    rho_o, off = oracle_rho(fr, nsp, ks)
    for a in range(nsp):
        na = off[a + 1] - off[a]
        err = np.abs(rho_g[a] - rho_o[a])
        # per vector: BF16 hi+lo keeps ~16 significant bits per factor (<= 2^-16 relative, worst case)
        assert err.max() <= 3e-5 * na + 1e-5, (a, err.max(), na)
    ref = orc.bin_sums(rho_o, ks.bins, ks.weights, ks.nbins)
    check_shells(res, ref, nsp)


def test_sq_split_agrees_with_plain(ctx):
    spec, mode, qmax, qmin = SPECS["3sp_ref"]
    fr = spec.frame(0)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin)
    _, a = run_gpu(ctx, fr, 3, ks, "plain")
    _, b = run_gpu(ctx, fr, 3, ks, "split")
    check_shells(b, a, 3)


def test_sq_split_deterministic(ctx):
    spec, mode, qmax, qmin = SPECS["1sp_full"]
    fr = spec.frame(0)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin)
    _, a = run_gpu(ctx, fr, 1, ks, "split")
    _, b = run_gpu(ctx, fr, 1, ks, "split")
    assert np.array_equal(a, b)


def test_sq_tile_width_knob(ctx):
    """Narrower tensor-core tiles (more, smaller work items) give the same shell sums: every output
    element sums the same atoms in the same order whatever the tile's width."""
    from trj_analysis_b200._lib import TrjError
    spec, mode, qmax, qmin = SPECS["3sp_ref"]
    fr = spec.frame(0)
    ks = refsem.make_kset(mode, fr.box, qmax, qmin)
    _, a = run_gpu(ctx, fr, 3, ks, "split")
    ctx.set_sq_tile_cols(96)
    try:
        _, b = run_gpu(ctx, fr, 3, ks, "split")
    finally:
        ctx.set_sq_tile_cols(0)
    check_shells(b, a, 3)
    assert np.allclose(a, b, rtol=1e-12, atol=0)
    with pytest.raises(TrjError):
        ctx.set_sq_tile_cols(100)
