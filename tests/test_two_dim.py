"""Two-dimensional frames (ndim = 2) on the host: the oracle's pair counts of z = 0 frames against a
plain restatement of rdf2_sh (rdf.cuf:617-670), and sq_init's 2D n(Q) and k-set (sq.cuf:157-192,
313-325; sqfnD with dim = 2, 523-591; sqfact2, 456-521) against loop transcriptions."""
import math

import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import analysis, refsem
from trj_analysis_b200.refsem import F32


def _roundf(x):
    x = np.asarray(x, np.float64)
    return np.trunc(x + np.copysign(0.5, x)).astype(F32)


def rdf2_numpy(pos2, sp, box2, side2, deltar, lsmax, nsp):
    """rdf2_sh: xd, yd minimum image, rr2 = xd*xd + yd*yd, bin nint(sqrt(rr2)/deltar), FP32; bins 1..lsmax."""
    n = pos2.shape[0]
    i, j = np.triu_indices(n, 1)
    L = np.asarray(box2, F32)
    d = (pos2[j] - pos2[i]).astype(F32)
    d = (d - (L * _roundf((d / L).astype(F32))).astype(F32)).astype(F32)
    rr2 = ((d[:, 0] * d[:, 0]).astype(F32) + (d[:, 1] * d[:, 1]).astype(F32)).astype(F32)
    ok = rr2 < F32(side2)
    ind = _roundf((np.sqrt(rr2[ok]).astype(F32) / F32(deltar)).astype(F32)).astype(np.int64)
    good = (ind >= 1) & (ind <= lsmax)
    ii, jj, ind = i[ok][good], j[ok][good], ind[good]
    hist = np.zeros((nsp * (nsp + 1) // 2, lsmax), np.uint64)
    rows = np.array([refsem.pair_row(int(a), int(b), nsp) for a, b in zip(sp[ii], sp[jj])], np.int64)
    np.add.at(hist, (rows, ind - 1), 1)
    return hist


@pytest.mark.parametrize("cells", [False, True])
def test_oracle_2d_counts_match_rdf2(cells):
    rng = np.random.default_rng(3)
    n, nsp = 700, 2
    box2 = np.array([13.0, 11.5], np.float32)
    xy = (rng.uniform(-0.2, 1.2, size=(n, 2)) * box2).astype(np.float32)
    sp = rng.integers(0, nsp, size=n).astype(np.int32)
    xyz = np.zeros((n, 3), np.float32)
    xyz[:, :2] = xy
    box = np.array([box2[0], box2[1], 1.0], np.float32)
    p = refsem.rdf_params(nsp, 0.05, 0.0, box, ndim=2)
    pos, sps, off = orc.layout(xyz, sp, box, nsp)
    assert np.all(pos[:, 2] == 0)
    h, _ = orc.rdf_counts(pos, sps, box, p.side2, p.deltar, p.lsmax, nsp, cells=cells)
    np.testing.assert_array_equal(h, rdf2_numpy(pos[:, :2], sps, box2, p.side2, p.deltar, p.lsmax, nsp))
    assert p.side2 == float(F32(F32(5.75) * F32(5.75)))  # half of min(Lx, Ly), not of the unit z edge


def _nq2_loops(si):
    nq = [0] * (si.nqmax + 1)
    indm = 0
    for i in range(si.lmax[0] + 1):
        for j in range(si.lmax[1] + 1):
            if i + j == 0:
                continue
            rr = F32(math.sqrt(float(F32(F32(F32(i) * si.fk[0]) ** 2 + F32(F32(j) * si.fk[1]) ** 2))))
            if rr < F32(si.qmin_eff):
                ind = refsem.nint(F32(rr / F32(si.dq)))
                indm = max(indm, ind)
                if ind <= si.nqmax:
                    nq[ind] += 1
    for i in range(indm + 1, si.nqmax + 1):
        nq[i] = 2
    return np.array(nq)


@pytest.mark.parametrize("box,qmax,qmin", [((40.0, 40.0), 10.0, 4.0), ((31.0, 45.0), 8.0, 5.0),
                                           ((20.0, 20.0), 6.0, 0.5)])
def test_sq_init_2d(box, qmax, qmin):
    b = np.array([box[0], box[1], 1.0], np.float32)
    si = refsem.sq_init_params(b, qmax, qmin, ndim=2)
    fk = [F32(refsem.TWOPI32 / F32(L)) for L in box]
    assert si.dq == float(F32(min(fk)))
    lm = [refsem.nint(F32(F32(qmin) / fk[d])) for d in range(2)]
    lm = [l - 16 + l % 16 if l % 16 else l for l in lm]
    if min(lm) == 0:
        assert si.nqmin == 1 and si.lmax == (1, 1, 1)
    else:
        assert si.lmax[:2] == tuple(lm) and si.nqmin == min(lm)
    ks = refsem.make_kset("ref", b, qmax, qmin, ndim=2)
    assert np.all(ks.vectors[:, 2] == 0)
    pt = refsem.planar_tiles(ks, 8)
    v = ks.vectors.astype(np.int64)
    np.testing.assert_array_equal(pt.vectors[:, 1] + 8 * pt.vectors[:, 2], v[:, 1])
    np.testing.assert_array_equal(pt.vectors[:, 0], v[:, 0])
    assert np.all((pt.vectors[:, 1] >= 0) & (pt.vectors[:, 1] < 8))
    if si.nqmin > 1:
        np.testing.assert_array_equal(ks.nq, _nq2_loops(si))
        # sqfnD, dim = 2: every (kx, ky) of the launch grid with 0 < q2 <= qmin^2, q2 = fma(kf2, kf2, kf1*kf1)
        want = set()
        for kx in range((si.lmax[0] // 16 + 1) * 16):
            for ky in range((si.lmax[1] // 16 + 1) * 16):
                kf1, kf2 = F32(F32(kx) * si.fk[0]), F32(F32(ky) * si.fk[1])
                q2 = F32(np.float64(kf2) * np.float64(kf2) + np.float64(F32(kf1 * kf1)))
                if 0 < q2 <= F32(F32(si.qmin_eff) * F32(si.qmin_eff)):
                    ind = int(np.floor(F32(F32(math.sqrt(float(q2))) / F32(si.dq)) + F32(0.501)))
                    if ind <= si.nqmax:
                        want.add((kx, ky, ind))
        dense_part = {(int(v[0]), int(v[1]), int(b_)) for v, b_ in zip(ks.vectors[:len(want)], ks.bins[:len(want)])}
        assert dense_part == want
    else:
        np.testing.assert_array_equal(ks.nq[1:], 2)
    # sqfact2: (k, 0) and (0, k) for k = minPts..nqmax, binned at k
    axes = ks.vectors[-2 * (si.nqmax - (si.nqmin + 1 if si.nqmin > 1 else 1) + 1):]
    assert np.all((axes[:, 0] == 0) | (axes[:, 1] == 0))


def test_shell_areas_2d():
    dv, ri = analysis.shell_volumes(6, 0.1, ndim=2)
    np.testing.assert_allclose(dv, np.pi * ((ri + 0.05) ** 2 - (ri - 0.05) ** 2), rtol=1e-7)
    assert refsem.volume([3.0, 4.0, 100.0], ndim=2) == 12.0


@pytest.mark.parametrize("qmax,qmin", [(8.0, 4.0), (9.0, 3.5), (5.0, 0.4)])
def test_slab_kset_matches_loops(qmax, qmin):
    box = np.array([30.0, 26.0, 60.0], np.float32)
    ks = refsem.slab_kset(box, qmax, qmin)
    si = refsem.sq_init_params(box, qmax, qmin, ndim=2)
    want = []
    for kx in range((si.lmax[0] // 16 + 1) * 16):
        for ky in range((si.lmax[1] // 16 + 1) * 16):
            kf1, kf2 = F32(F32(kx) * si.fk[0]), F32(F32(ky) * si.fk[1])
            q2 = F32(np.float64(kf2) * np.float64(kf2) + np.float64(F32(kf1 * kf1)))
            if si.nqmin > 1 and 0 < q2 <= F32(F32(si.qmin_eff) * F32(si.qmin_eff)):
                ind = refsem.nint(F32(F32(math.sqrt(float(q2))) / F32(si.dq)))  # sqf3xy: nint(q/dq)
                if ind <= si.nqmax:
                    want.append((kx, ky, 0, ind))
    for k in range(max(1, si.nqmin + 1), si.nqmax + 1):
        want.append((k, 0, 0, k))
    for k in range(max(1, si.nqmin + 1), si.nqmax + 1):
        want.append((0, k, 0, k))
    got = [tuple(int(x) for x in v) + (int(b),) for v, b in zip(ks.vectors, ks.bins)]
    assert got == want
    np.testing.assert_array_equal(ks.nq, refsem.reference_nq(si, 2))


def test_slab_of_matches_minloc():
    rng = np.random.default_rng(1)
    z = rng.uniform(-2, 12, size=500).astype(np.float32)
    zs = [1.0, 4.0, 4.0, 8.5]
    got = refsem.slab_of(z, zs, 1.5)
    for k in range(z.shape[0]):
        d = [abs(F32(F32(c) - z[k])) for c in zs]
        m = int(np.argmin(d))  # first minimum
        assert got[k] == (m if d[m] <= F32(F32(1.5) / F32(2.0)) else -1)
