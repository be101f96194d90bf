"""Split-BF16 tensor-core S(Q) at full scale: N = 1,000,188 (three species), every lattice vector
below qmin = 3 plus axis vectors to qmax = 10 (270k k-vectors, as the benchmark), against the
exact FP64 oracle on selected shells.

Bar (per selected shell and species pair): |sum_gpu - sum_fp64| <= 1e-5 * sqrt(sum_aa * sum_bb),
the relative error of S_aa on the self rows and of the Cauchy-Schwarz scale on the cross rows.
The oracle evaluates only the vectors of the selected shells (tens of thousands of k-vectors x
1e6 atoms in FP64 on the host cores).
"""
import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import frames, refsem

pytestmark = pytest.mark.gpu

SHELLS = [1, 2, 3, 5, 8, 13, 21, 34]


@pytest.fixture(scope="module")
def c3():
    spec = frames.c3_spec()
    fr = spec.frame(0)
    ks = refsem.make_kset("full+axes", fr.box, 10.0, 3.0)
    pos, sp, off = orc.layout(fr.xyz, fr.types - 1, fr.box, 3)
    sel = np.isin(ks.bins, SHELLS)
    rho_o = orc.rho_fp64(pos, off, fr.box, ks.vectors[sel])
    return fr, ks, sel, rho_o


def _gpu_rho(fr, ks, method, flush=None, pairs=True):
    from trj_analysis_b200 import engine
    ctx = engine.Context(0)
    stage = engine.FrameStage(ctx, fr.n, 3)
    plan = engine.SqPlan(ctx, 3, ks, np.bincount(fr.types - 1, minlength=3))
    if flush:
        plan.set_flush(flush)
    plan.set_pairs(pairs)
    out = plan.new_out()
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box)
    plan.accumulate(stage.packed, n, fr.box, out, engine.METHODS[method])
    rho = plan.rho().cpu().numpy()
    ctx.check()
    plan.close()
    ctx.close()
    return rho


def _shell_errors(rho_g, rho_o, ks, sel):
    bins, w = ks.bins[sel], ks.weights[sel]
    nb = ks.nbins
    ref = orc.bin_sums(rho_o, bins, w, nb)
    got = orc.bin_sums(rho_g, bins, w, nb)
    rows = refsem.pair_rows(3)
    diag = {a: ref[:, refsem.pair_row(a, a, 3)] for a in range(3)}
    scale = np.stack([np.sqrt(np.abs(diag[a] * diag[b])) for a, b in rows], axis=1)
    live = scale > 0
    return (np.abs(got - ref)[live] / scale[live]).max()


@pytest.mark.parametrize("flush,pairs", [(None, True), (None, False), (128, True)])
def test_split_bf16_full_scale_within_1e5_per_shell(c3, flush, pairs):
    fr, ks, sel, rho_o = c3
    rho_g = _gpu_rho(fr, ks, "split", flush, pairs)[:, sel]
    err = _shell_errors(rho_g, rho_o, ks, sel)
    print(f"flush={flush} pairs={pairs}: max per-shell error {err:.3e}")
    assert err <= 1e-5


def test_plain_fp32_full_scale_within_1e5_per_shell(c3):
    fr, ks, sel, rho_o = c3
    rho_g = _gpu_rho(fr, ks, "plain")[:, sel]
    err = _shell_errors(rho_g, rho_o, ks, sel)
    print(f"plain: max per-shell error {err:.3e}")
    assert err <= 1e-5
