"""Two-dimensional frames on the GPU (Session with ndim = 2): pair counts, number fluctuations and
the direct-sum S(Q) against the oracle on the same z = 0 layout.  Counts and s2n sums are exact;
rho within the direct-sum tolerance 2e-6 * N_a + 1e-6 per vector."""
import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import analysis, frames, refsem

pytestmark = pytest.mark.gpu


def _frames_2d(nx, ny, a, nframes, seed):
    rng = np.random.default_rng(seed)
    gx, gy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    base = np.stack([gx.ravel(), gy.ravel()], axis=1).astype(np.float64) * a
    n = base.shape[0]
    types = rng.permutation(np.repeat(np.array([1, 2], np.int32), [n - n // 3, n // 3]))
    box = np.array([nx * a, ny * a, 7.0], np.float32)
    out = []
    for f in range(nframes):
        xy = base + rng.normal(0, 0.15 * a, size=base.shape)
        z = rng.uniform(0, 7.0, size=(n, 1))  # discarded for ndim = 2
        out.append(frames.Frame(xyz=np.concatenate([xy, z], axis=1).astype(np.float32), types=types, box=box.copy()))
    return out


@pytest.mark.parametrize("method", ["plain", "split"])  # split: the planar tile form on the tensor cores
def test_session_2d_matches_oracle(method):
    frs = _frames_2d(60, 48, 1.1, 2, seed=12)
    cfg = analysis.Config(nsp=2, ndim=2, sp_types_selected=(1, 2), deltar=0.05, rcrdf=6.0, qmax=6.0, qmin=2.5,
                          method=method, kset="ref", nrandom=20)
    s = analysis.Session(cfg)
    hist_want = None
    gi_w = g2i_w = None
    for fr in frs:
        s.add_frame(fr)
        xyz = fr.xyz.copy()
        xyz[:, 2] = 0
        box = np.array([fr.box[0], fr.box[1], 1.0], np.float32)
        pos, sp, off = orc.layout(xyz, fr.types - 1, box, 2)
        h, _ = orc.rdf_counts(pos, sp, box, s.rdf.side2, cfg.deltar, s.rdf.lsmax, 2, cells=True)
        hist_want = h if hist_want is None else hist_want + h
        pts = torch.zeros(3 * cfg.nrandom, dtype=torch.float32, device=s.ctx.torch_device)
        gi1, g2i1 = s.rdf.new_s2n()
        s.rdf.s2n(cfg.nrandom, gi1, g2i1, points=pts)
        p = pts.cpu().numpy().reshape(-1, 3)
        assert np.all(p[:, 2] == 0)
        a, b = orc.s2n_counts(pos, box, s.rdf.side2, cfg.deltar, s.rdf.lsmax, p)
        gi_w = a if gi_w is None else gi_w + a
        g2i_w = b if g2i_w is None else g2i_w + b
        rho = s.sq.rho().cpu().numpy()
        v = s.kset.vectors.astype(np.int64)
        if method == "split":  # planar tile form (nx, ny mod 8, ny div 8) -> in-plane (nx, ny, 0)
            assert s.sq.n_tiles > 0
            v = np.stack([v[:, 0], v[:, 1] + 8 * v[:, 2], 0 * v[:, 2]], axis=1)
        rho_o = orc.rho_fp64(pos, off, box, v.astype(np.int32))
        per, floor = (2e-6, 1e-6) if method == "plain" else (3e-5, 1e-5)
        for k in range(2):
            assert np.abs(rho[k] - rho_o[k]).max() <= per * (off[k + 1] - off[k]) + floor
    s.ctx.check()
    np.testing.assert_array_equal(s.rdf_transfer(), hist_want)
    np.testing.assert_array_equal(s.gi.cpu().numpy(), gi_w)
    np.testing.assert_array_equal(s.g2i.cpu().numpy(), g2i_w)
    assert s.volumen == float(np.float32(np.float32(frs[0].box[0]) * np.float32(frs[0].box[1])))
    res = s.rdf_results()
    # 2D normalisation: g(r) -> 1 at large r for a disordered lattice
    assert abs(res["gtot"][-20:].mean() - 1.0) < 0.05
    sq = s.sq_results()
    assert np.all(sq["nq"] > 0)
    s.close()
