"""Slab (twoDstruc_3D) g_xy(r) and S_xy(Q) on the GPU against a numpy restatement of rdfxy
(rdf.cuf:672-738) and sqf3xy/sqf2xy (sq.cuf:594-771) with the per-frame normalisations of RDFcomp
(rdf.cuf:284-299).  Slice histograms are exact integer counts, so g_xy agrees to FP64 rounding;
S_xy uses FP64 phases in the oracle and the direct-sum tolerance (1e-5 of each shell sum)."""
import numpy as np
import pytest

from trj_analysis_b200 import analysis, frames, refsem
from trj_analysis_b200.refsem import F32

pytestmark = pytest.mark.gpu


def _roundf(x):
    x = np.asarray(x, np.float64)
    return np.trunc(x + np.copysign(0.5, x)).astype(F32)


def _oracle(frs, nsp, cfg):
    zs, zg = cfg.slab.zslice, cfg.slab.zgrid
    box = frs[0].box
    p3 = refsem.rdf_params(nsp, cfg.deltar, cfg.rcrdf, box)
    lsmax = p3.lsmax
    ns = len(zs)
    hist_xy = np.zeros((nsp, nsp, ns, lsmax))
    ks = refsem.slab_kset(box, cfg.qmax, cfg.qmin)
    sqf = np.zeros((ks.nbins, ns))
    sqfp = np.zeros((ks.nbins, nsp, ns))
    bsc = np.asarray(cfg.bsc, np.float64)
    L = np.asarray(box, F32)
    for fr in frs:
        sp = fr.types - 1
        order = np.argsort(sp, kind="stable")
        sp = sp[order]
        xyz = fr.xyz[order]
        pos = refsem.fold(xyz, box)
        sl = refsem.slab_of(xyz[:, 2], zs, zg)
        n = sp.shape[0]
        countp = np.zeros((nsp, ns), np.int64)
        for i in range(n - 1):  # rdfxy: i = 1..N-1
            if sl[i] >= 0:
                countp[sp[i], sl[i]] += 1
        i, j = np.triu_indices(n, 1)
        same = (sl[i] >= 0) & (sl[i] == sl[j])
        i, j = i[same], j[same]
        d = (pos[j, :2] - pos[i, :2]).astype(F32)
        d = (d - (L[:2] * _roundf((d / L[:2]).astype(F32))).astype(F32)).astype(F32)
        rr2 = ((d[:, 0] * d[:, 0]).astype(F32) + (d[:, 1] * d[:, 1]).astype(F32)).astype(F32)
        ok = rr2 < F32(p3.side2)
        ind = (np.floor((np.sqrt(rr2[ok]).astype(F32) / F32(cfg.deltar)).astype(F32)) + 1).astype(np.int64)
        ii, jj = i[ok], j[ok]
        good = (ind >= 1) & (ind <= lsmax)
        h = np.zeros((nsp, nsp, ns, lsmax))
        a = np.minimum(sp[ii][good], sp[jj][good])
        b = np.maximum(sp[ii][good], sp[jj][good])
        np.add.at(h, (a, b, sl[ii][good], ind[good] - 1), 1)
        for x in range(nsp):
            for y in range(x, nsp):
                for s in range(ns):
                    if countp[x, s] > 0 and countp[y, s] > 0:
                        hist_xy[x, y, s] += h[x, y, s] / (countp[x, s] * countp[y, s])
        # S_xy with FP64 phases
        sfrac = pos[:, :2].astype(np.float64) / L[:2].astype(np.float64)
        ph = 2 * np.pi * (ks.vectors[:, :2].astype(np.float64) @ sfrac.T)
        e = np.exp(1j * ph)
        for s in range(ns):
            cnt = 0
            tot = np.zeros(ks.nvec, complex)
            for x in range(nsp):
                m = (sl == s) & (sp == x)
                c = int(m.sum())
                cnt += c
                r = e[:, m].sum(axis=1)
                tot += bsc[x] * r
                if c > 0:
                    np.add.at(sqfp[:, x, s], ks.bins, np.abs(r) ** 2 / c)
            if cnt > 0:
                np.add.at(sqf[:, s], ks.bins, np.abs(tot) ** 2 / cnt)
    return hist_xy, sqf, sqfp, ks


@pytest.mark.parametrize("qmax,qmin", [(8.0, 6.6), (5.0, 2.5)])  # sqf3xy + sqf2xy; sqf2xy only
def test_slab_matches_oracle(tmp_path, qmax, qmin):
    spec = frames.FCCSpec(cells=(9, 9, 12), sigma=0.1, fractions=(0.6, 0.4), seed=21)
    frs = list(spec.frames(2))
    zmax = float(frs[0].box[2])
    cfg = analysis.Config(nsp=2, sp_types_selected=(1, 2), deltar=0.05, rcrdf=4.0, qmax=qmax, qmin=qmin,
                          bsc=(1.0, 0.5), slab=analysis.SlabConfig(zslice=(0.2 * zmax, 0.5 * zmax, 0.75 * zmax),
                                                                   zgrid=0.12 * zmax))
    s = analysis.Session(cfg).run(frs)
    hist_xy, sqf, sqfp, ks = _oracle(frs, 2, cfg)
    st = s.slab
    np.testing.assert_allclose(st.hist_xy, hist_xy, rtol=1e-13, atol=0)
    assert hist_xy.sum() > 0
    scale = np.maximum(np.abs(sqf), 1e-12)
    assert np.all(np.abs(st.sqf_xy - sqf) <= 1e-5 * scale + 1e-9)
    assert np.all(np.abs(st.sqf_pxy - sqfp) <= 1e-5 * np.maximum(np.abs(sqfp), 1e-12) + 1e-9)
    files = s.print_slabs(str(tmp_path))
    names = sorted(f.split("/")[-1] for f in files)
    assert names == ["gxy_1-1.dat", "gxy_1-2.dat", "gxy_2-2.dat", "sqpxy_1-1.dat", "sqpxy_2-2.dat", "sqxy.dat"]
    res = s.slab_results()
    assert res["g_xy"].shape[1:] == (2, 2, 3)
    s.close()
