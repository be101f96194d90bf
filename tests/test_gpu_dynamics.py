"""F(Q,t), Fs(Q,t) and the MSD on the GPU (trj_dyn_accumulate / trj_dyn_flush through the Session)
against the loop-for-loop oracle of rtcorr/FqtnD/rtcal.

Tolerances: per term the GPU's cosine and sine of an exactly reduced angle are within 4e-7 of the FP64
values (fast-math error of __sincosf on [-pi, pi) plus the 2^-32 fixed-point phase), so
* Fs (normalised by N count_org nw): 1e-6 absolute;
* F: each rho is within 4e-7 N per vector, so a product term within 4e-7 N (|rho0| + |rho_t|) + O(N^2 1e-13);
  the oracle returns the sum of |rho0| + |rho_t| normalised like F (fkt_scale): tolerance 1e-6 N fkt_scale;
* C_r(t): the per-atom FP32 arithmetic is the oracle's, only the FP64 summation order differs: 1e-12.
"""
import numpy as np
import pytest

from oracle import orc, orc_dyn
from trj_analysis_b200 import analysis, dynamics, frames, refsem
from trj_analysis_b200.refsem import F32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trj_analysis_b200 import engine
    c = engine.Context(0)
    yield c
    c.close()


CASES = {
    "1sp_default_tlimit": (frames.FCCSpec(cells=(6, 6, 6), sigma=0.08, seed=41), 16, 0.25,
                           dynamics.DynConfig(nbuffer=3, jump=2, qw=(1.2, 2.5, 4.0))),
    "2sp_tlimit_bsc": (frames.FCCSpec(cells=(7, 7, 8), sigma=0.08, fractions=(0.6, 0.4), seed=42), 20, 0.4,
                       dynamics.DynConfig(nbuffer=4, jump=1, tlimit=2.0, tmax=3.0, qw=(0.9, 2.0), tstep=0.5)),
    "3sp_many_buffers": (frames.FCCSpec(cells=(5, 5, 5), sigma=0.1, fractions=(0.5, 0.3, 0.2), seed=43), 30, 0.15,
                         dynamics.DynConfig(nbuffer=9, jump=2, tlimit=5.0, qw=(1.5, 3.0, 5.0, 6.5))),
}


def _oracle(frs, nsp, cfg, bsc):
    box = frs[0].box
    sp = frs[0].types - 1
    packed = [orc.layout(f.xyz, sp, box, nsp)[0] for f in frs]
    sps = orc.layout(frs[0].xyz, sp, box, nsp)[1]
    dq = refsem.sq_init_params(box, max(cfg.qw), max(cfg.qw)).dq
    s = refsem.sqw_kset(box, cfg.qw, dq)
    times = [F32(F32(f.time) * F32(cfg.tstep)) for f in frs]
    return orc_dyn.dynamics(packed, sps, box, bsc, s.vectors, s.bins, len(cfg.qw), s.nw, cfg.nbuffer, cfg.jump,
                            cfg.tlimit, times)


@pytest.mark.parametrize("name", list(CASES))
def test_dynamics_matches_oracle(ctx, name, tmp_path):
    spec, nconf, step, dcfg = CASES[name]
    nsp = len(spec.fractions)
    frs = list(frames.random_walk_frames(spec, nconf, step))
    bsc = (1.0, 0.7, 0.4)[:nsp]
    cfg = analysis.Config(nsp=nsp, sp_types_selected=tuple(range(1, nsp + 1)), run_rdf=False, run_sq=False,
                          run_sqw=True, dyn=dcfg, bsc=bsc)
    s = analysis.Session(cfg, ctx=ctx, nconf_total=nconf).run(frs)
    got = s.dyn.results()
    want = _oracle(frs, nsp, dcfg, bsc)
    assert got["count_org"] == want["count_org"] > 0
    assert got["itlimit"] == want["itlimit"]
    np.testing.assert_array_equal(got["t"], want["t"])
    np.testing.assert_allclose(got["r2t"], want["r2t"], rtol=1e-12, atol=1e-12)
    assert np.nanmax(np.abs(got["fskt"] - want["fskt"])) <= 1e-6
    n = frs[0].n
    tol = 1e-6 * n * want["fkt_scale"] + 1e-9
    diff = np.abs(got["fkt"] - want["fkt"])
    live = np.isfinite(want["fkt"])
    assert np.all(diff[live] <= tol[live]), (diff[live] / tol[live]).max()
    files = s.print_rtcor(str(tmp_path))
    assert [f.split("/")[-1] for f in files] == ["dyn.dat", "fkt.dat", "fskt.dat", "sqw.dat"]
    s.close()


def test_dynamics_deterministic(ctx):
    spec, nconf, step, dcfg = CASES["1sp_default_tlimit"]
    frs = list(frames.random_walk_frames(spec, nconf, step))
    out = []
    for _ in range(2):
        cfg = analysis.Config(nsp=1, sp_types_selected=(1,), run_rdf=False, run_sq=False, run_sqw=True, dyn=dcfg)
        s = analysis.Session(cfg, ctx=ctx, nconf_total=nconf).run(frs)
        r = s.dyn.results()
        out.append((r["fkt"], r["fskt"], r["r2t"]))
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b, equal_nan=True)


def test_dyn_accumulate_rejects_bad_schedules(ctx):
    from trj_analysis_b200 import _lib, engine
    spec = frames.FCCSpec(cells=(3, 3, 3), seed=5)
    fr = spec.frame(0)
    stage = engine.FrameStage(ctx, fr.n, 1)
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box)
    s = refsem.sqw_kset(fr.box, (2.0,), refsem.sq_init_params(fr.box, 2, 2).dq)
    plan = engine.DynPlan(ctx, 1, n, 2, 10, s, (1.0,))
    with pytest.raises(_lib.TrjError):
        plan.accumulate(stage.packed, n, fr.box, np.array([10, -1]), np.array([0, 0]))  # lag >= ndyn
    with pytest.raises(_lib.TrjError):
        plan.accumulate(stage.packed, n, fr.box, np.array([3, -1]), np.array([1, 0]))   # origin at lag 3
    with pytest.raises(_lib.TrjError):
        plan.accumulate(stage.packed, n - 1, fr.box, np.array([0, -1]), np.array([1, 0]))  # wrong atom count
    plan.accumulate(stage.packed, n, fr.box, np.array([0, -1]), np.array([1, 0]))
    ctx.check()
    plan.close()
