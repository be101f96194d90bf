"""The CPU oracle against independent restatements (numpy) on small cases."""
import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import frames, refsem
from trj_analysis_b200.refsem import F32


def _numpy_rdf(pos, sp, box, side2, deltar, lsmax, nsp):
    """Vectorised restatement of rdf_sh's arithmetic (no FMA: numpy float32 ops)."""
    n = pos.shape[0]
    nit = nsp * (nsp + 1) // 2
    hist = np.zeros((nit, lsmax), np.uint64)
    L = np.asarray(box, F32)
    for i in range(n - 1):
        d = (pos[i + 1:] - pos[i]).astype(F32)
        q = (d / L).astype(F32)
        nn = np.sign(q) * np.floor(np.abs(q.astype(np.float64)) + 0.5)
        d = (d - (L * nn.astype(F32)).astype(F32)).astype(F32)
        sq = (d * d).astype(F32)
        rr2 = ((sq[:, 0] + sq[:, 1]).astype(F32) + sq[:, 2]).astype(F32)
        m = rr2 < F32(side2)
        rr = np.sqrt(rr2[m]).astype(F32)
        ind = refsem.nint((rr / F32(deltar)).astype(F32))
        ok = (ind >= 1) & (ind <= lsmax)
        js = np.nonzero(m)[0][ok] + i + 1
        rows = [refsem.pair_row(sp[i], sp[j], nsp) for j in js]
        np.add.at(hist, (np.array(rows, dtype=np.int64), ind[ok] - 1), 1)
    return hist


def test_oracle_rdf_matches_numpy_restatement():
    spec = frames.FCCSpec(cells=(4, 4, 4), density=0.8, sigma=0.15, fractions=(0.6, 0.4), seed=7)
    fr = spec.frame(0)
    sp = fr.types - 1
    pos, sps, off = orc.layout(fr.xyz, sp, fr.box, 2)
    p = refsem.rdf_params(2, 0.05, 100.0, fr.box)
    h_c, e = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 2)
    h_n = _numpy_rdf(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 2)
    assert np.array_equal(h_c, h_n)
    assert int(e[2]) == int(h_c.sum())


def test_oracle_cells_equal_allpairs():
    spec = frames.FCCSpec(cells=(8, 8, 8), density=0.8, sigma=0.1, fractions=(0.5, 0.3, 0.2),
                          replace_frac=0.05, seed=3)
    fr = spec.frame(1)
    pos, sps, off = orc.layout(fr.xyz, fr.types - 1, fr.box, 3)
    p = refsem.rdf_params(3, 0.01, 3.0, fr.box)
    h_a, e_a = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 3)
    h_c, e_c = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 3, cells=True)
    assert np.array_equal(h_a, h_c)
    assert np.array_equal(e_a, e_c)


def test_pair_count_conservation_at_half_box():
    """With rcrdf = L/2 and tiny deltar every pair inside the sphere is counted once."""
    spec = frames.FCCSpec(cells=(3, 3, 3), density=0.8, sigma=0.1, seed=11)
    fr = spec.frame(0)
    pos, sps, off = orc.layout(fr.xyz, fr.types - 1, fr.box, 1)
    p = refsem.rdf_params(1, 0.001, 1e9, fr.box)
    h, e = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 1)
    # brute-force count of min-image pairs with rr2 < side2 and bin >= 1
    n = pos.shape[0]
    assert int(h.sum()) <= n * (n - 1) // 2
    assert int(h.sum()) == int(e[2])


def test_rho_fp64_matches_direct_numpy():
    rng = np.random.default_rng(0)
    box = np.array([7.5, 8.0, 9.25], F32)
    pos = (rng.random((50, 3)) * box).astype(F32)
    off = np.array([0, 30, 50])
    vec = rng.integers(-6, 7, size=(40, 3)).astype(np.int32)
    rho = orc.rho_fp64(pos, off, box, vec)
    s = pos.astype(np.float64) / box.astype(np.float64)
    ph = 2 * np.pi * (s @ vec.T.astype(np.float64))
    ref = np.stack([np.exp(1j * ph[0:30]).sum(0), np.exp(1j * ph[30:50]).sum(0)])
    assert np.allclose(rho, ref, rtol=0, atol=1e-11)


def test_rho_ref32_close_to_fp64_for_small_arguments():
    rng = np.random.default_rng(1)
    box = np.array([10.0, 10.0, 10.0], F32)
    pos = (rng.random((64, 3)) * box).astype(F32)
    off = np.array([0, 64])
    vec = rng.integers(0, 4, size=(16, 3)).astype(np.int32)
    a = orc.rho_fp64(pos, off, box, vec)
    b = orc.rho_ref32(pos, off, box, vec)
    assert np.max(np.abs(a - b)) < 1e-3


def test_layout_fold_semantics():
    box = np.array([10.0, 10.0, 10.0], F32)
    xyz = np.array([[-0.5, 10.5, 25.0], [9.999, -13.0, 0.0]], F32)
    pos, sp, off = orc.layout(xyz, np.array([1, 0], np.int32), box, 2)
    # species 0 first (stable), truncation keeps negatives negative
    assert np.allclose(pos[0], [9.999, -3.0, 0.0], atol=1e-5)
    assert np.allclose(pos[1], [-0.5, 0.5, 5.0], atol=1e-5)
    assert list(off) == [0, 1, 2]
    assert np.array_equal(refsem.fold(xyz, box)[0], pos[1])
