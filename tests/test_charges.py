"""Charge-weighted g_qq(r) and S_qq(Q) on the host: the oracle's charge arithmetic against a
plain numpy restatement of the reference's ex_qc branch, identities that hold when every atom of a
species carries the same charge, the charge columns of the output files, and the charge variable
of the trajectory readers.

Reference: rdf.cuf:469-472 (gqq_d(ind) += qci*qcj for every counted pair), rdf.cuf:272-273
(avq2 = sum(q^2)/N; gqq += gqq_d/avq2), sq.cuf:569-588 (sum_j q_j cos/sin of the phase, sqfq_d +=
|.|^2), sq.cuf:143-145, log.f90:502-504 and 386/393 (normalisations and columns).
"""
import math

import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import analysis, frames, refsem, writers
from trj_analysis_b200.refsem import F32


def _roundf(x):
    """C roundf on float32 values (half away from zero), exact through float64."""
    x = np.asarray(x, np.float64)
    return np.trunc(x + np.copysign(0.5, x)).astype(np.float32)


def pairs_numpy(pos, sp, q, box, side2, deltar, lsmax, nsp):
    """All unordered pairs with the reference's FP32 arithmetic (rdf.cuf:451-472), vectorised."""
    n = pos.shape[0]
    i, j = np.triu_indices(n, 1)
    L = np.asarray(box, F32)
    d = (pos[j] - pos[i]).astype(F32)
    nimg = _roundf((d / L).astype(F32))
    d = (d - (L * nimg).astype(F32)).astype(F32)
    sq = (d * d).astype(F32)
    rr2 = ((sq[:, 0] + sq[:, 1]).astype(F32) + sq[:, 2]).astype(F32)
    ok = rr2 < F32(side2)
    rr = np.sqrt(rr2[ok]).astype(F32)
    ind = _roundf((rr / F32(deltar)).astype(F32)).astype(np.int64)
    good = (ind >= 1) & (ind <= lsmax)
    ii, jj, ind = i[ok][good], j[ok][good], ind[good]
    hist = np.zeros((nsp * (nsp + 1) // 2, lsmax), np.uint64)
    rows = np.array([refsem.pair_row(int(a), int(b), nsp) for a, b in zip(sp[ii], sp[jj])], np.int64)
    np.add.at(hist, (rows, ind - 1), 1)
    gqq = np.zeros(lsmax)
    np.add.at(gqq, ind - 1, q[ii].astype(np.float64) * q[jj].astype(np.float64))
    return hist, gqq


def small_charged_frame(seed=0, n=300, nsp=2):
    rng = np.random.default_rng(seed)
    box = np.array([7.1, 7.9, 8.3], np.float32)
    xyz = (rng.uniform(-0.3, 1.3, size=(n, 3)) * box).astype(np.float32)
    sp = rng.integers(0, nsp, size=n).astype(np.int32)
    q = rng.normal(0.0, 0.8, size=n).astype(np.float32)
    return xyz, sp, q, box


@pytest.mark.parametrize("cells", [False, True])
def test_oracle_charge_histogram_matches_numpy_restatement(cells):
    xyz, sp, q, box = small_charged_frame()
    nsp = 2
    pos, sps, off, qs = orc.layout(xyz, sp, box, nsp, charges=q)
    rc = float(F32(min(box) / F32(2)))
    side2, deltar = float(F32(rc * rc)), 0.05
    lsmax = int(math.floor(rc / deltar + 0.5)) + 1
    hist, edge, gqq = orc.rdf_charged(pos, sps, qs, box, side2, deltar, lsmax, nsp, cells=cells)
    hist_np, gqq_np = pairs_numpy(pos, sps, qs, box, side2, deltar, lsmax, nsp)
    np.testing.assert_array_equal(hist, hist_np)
    scale = np.abs(qs).max() ** 2 * np.maximum(hist.sum(axis=0), 1)
    assert np.all(np.abs(gqq - gqq_np) <= 1e-13 * scale)
    # the charge mode does not change the counts
    h2, e2 = orc.rdf_counts(pos, sps, box, side2, deltar, lsmax, nsp, cells=cells)
    np.testing.assert_array_equal(hist, h2)
    np.testing.assert_array_equal(edge, e2)


def test_species_constant_charges_reduce_to_species_rows():
    """q_j = q_a for every atom of species a: gqq = sum_{a<=b} q_a q_b H_ab, rho_q = sum_a q_a rho_a."""
    spec = frames.FCCSpec(cells=(5, 5, 5), sigma=0.1, fractions=(0.5, 0.3, 0.2), seed=7,
                          charges=(1.0, -0.8476, 0.4238))
    fr = spec.frame(0)
    nsp = 3
    pos, sps, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp, charges=fr.charges)
    rc = float(F32(min(fr.box) / F32(2)))
    lsmax = int(math.floor(rc / 0.05 + 0.5)) + 1
    hist, _, gqq = orc.rdf_charged(pos, sps, qs, fr.box, float(F32(rc * rc)), 0.05, lsmax, nsp)
    qa = np.asarray(spec.charges, np.float32).astype(np.float64)
    want = np.zeros(lsmax)
    for a, b in refsem.pair_rows(nsp):
        want += qa[a] * qa[b] * hist[refsem.pair_row(a, b, nsp)].astype(np.float64)
    np.testing.assert_allclose(gqq, want, rtol=1e-12, atol=1e-9)
    ks = refsem.make_kset("full", fr.box, 4.0, None)
    rho = orc.rho_fp64(pos, off, fr.box, ks.vectors)
    rho_q = orc.rho_charge_fp64(pos, qs, fr.box, ks.vectors)
    np.testing.assert_allclose(rho_q, (qa[:, None] * rho).sum(axis=0), rtol=0, atol=1e-9)


def test_rho_charge_matches_direct_sum():
    xyz, sp, q, box = small_charged_frame(seed=3, n=120)
    pos, sps, off, qs = orc.layout(xyz, sp, box, 2, charges=q)
    vecs = np.array([[1, 0, 0], [0, 2, -1], [3, -1, 2], [-2, 2, 5]], np.int32)
    s = pos.astype(np.float64) / np.asarray(box, np.float32).astype(np.float64)
    want = (qs.astype(np.float64)[None, :] * np.exp(2j * np.pi * (vecs @ s.T))).sum(axis=1)
    np.testing.assert_allclose(orc.rho_charge_fp64(pos, qs, box, vecs), want, rtol=0, atol=1e-10)


def test_avq2_is_fp32_of_fp64_mean():
    q = np.array([0.4238, 0.4238, -0.8476, 1.0], np.float32)
    want = np.float32(np.sum(q.astype(np.float64) ** 2) / 4)
    assert orc.avq2(q) == float(want)


def test_g_qq_normalisation_and_columns(tmp_path):
    lsmax, nsp, nconf = 8, 2, 3
    hist = np.arange(3 * lsmax, dtype=np.uint64).reshape(3, lsmax)
    gqq = np.linspace(-2.0, 5.0, lsmax)
    ntype = np.array([30, 20])
    res = analysis.normalise_rdf(hist, nsp, lsmax, 0.1, 1000.0, ntype, nconf, gqq=gqq)
    dv, _ = analysis.shell_volumes(lsmax, 0.1)
    np.testing.assert_allclose(res["g_qq"], 2 * 1000.0 * gqq[:lsmax - 2] / (50 ** 2 * dv[:lsmax - 2] * nconf))
    files = writers.write_gmixsim(str(tmp_path), res["r"], res["g"], nsp, g_qq=res["g_qq"])
    lines = open(files[0]).read().splitlines()
    assert lines[0] == "#       r        " + " " * 9 + "g_qq(r)" + " " * 9 + "g_11(r)" + " " * 9 + "g_12(r)" + \
        " " * 9 + "g_22(r)"
    row = lines[1]
    assert len(row) == 16 * 5
    assert row[16:32] == writers.fmt_f(res["g_qq"][0], 16, 6)
    assert row[32:48] == writers.fmt_f(res["g"][0, 0, 0], 16, 6)


def test_g_qq_many_species_goes_to_first_file(tmp_path):
    nsp, nrow = 7, 3
    g = np.ones((nrow, nsp, nsp))
    files = writers.write_gmixsim(str(tmp_path), np.arange(nrow, dtype=np.float32), g, nsp,
                                  g_qq=np.full(nrow, 0.5))
    first = open(files[0]).read().splitlines()
    assert "g_qq(r)" in first[0]
    assert first[1][16:32] == writers.fmt_f(0.5, 16, 5)
    assert all("g_qq" not in open(f).read() for f in files[1:])


def test_s_qq_normalisation_and_columns(tmp_path):
    nsp = 2
    ks = refsem.make_kset("ref", np.array([10.0, 10.0, 10.0], np.float32), 4.0, 2.0)
    ndens = nsp + 1
    rng = np.random.default_rng(0)
    out = rng.uniform(1.0, 2.0, size=(ks.nbins, ndens * (ndens + 1) // 2))
    ntype = np.array([600, 400])
    avq2 = 0.75
    res = analysis.normalise_sq(out, ks, ntype, np.ones(nsp, np.float32), 2, avq2=avq2)
    sp_rows, cross, qq = analysis.split_charged_rows(out, nsp)
    plain = analysis.normalise_sq(sp_rows, ks, ntype, np.ones(nsp, np.float32), 2)
    np.testing.assert_array_equal(res["s_nn"], plain["s_nn"])
    nq = ks.nq.astype(np.float64)
    sl = slice(1, ks.nqmax + 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        want = (qq / avq2 / (1000 * 2 * np.where(nq > 0, nq, np.nan)))[sl]
    np.testing.assert_allclose(res["s_qq"], want)
    files = writers.write_sq(str(tmp_path), res["q"], res["s_nn"], res["nq"], res["s_self"], res.get("binary"),
                             s_qq=res["s_qq"])
    lines = open(files[0]).read().splitlines()
    assert lines[0] == writers.SQ_HEADER_BINARY_QQ
    live = [i for i in range(len(res["q"])) if res["nq"][i] > 0]
    i = live[0]
    row = lines[1 + i]
    assert len(row) == 7 * 15 + 12
    assert row[30:45] == writers.fmt_f(res["s_qq"][i], 15, 7)


def test_split_charged_rows_layout():
    nsp = 3
    ndens = 4
    out = np.arange(2 * ndens * (ndens + 1) // 2, dtype=np.float64).reshape(2, -1)
    sp, cross, qq = analysis.split_charged_rows(out, nsp)
    for r, (a, b) in enumerate(refsem.pair_rows(nsp)):
        np.testing.assert_array_equal(sp[:, r], out[:, refsem.pair_row(a, b, ndens)])
    for a in range(nsp):
        np.testing.assert_array_equal(cross[:, a], out[:, refsem.pair_row(a, 3, ndens)])
    np.testing.assert_array_equal(qq, out[:, -1])


@pytest.mark.parametrize("fmt", ["nc", "npz"])
def test_trajectory_charges_round_trip(tmp_path, fmt):
    spec = frames.FCCSpec(cells=(3, 3, 3), fractions=(0.5, 0.5), seed=2, charges=(1.0, -1.0), charge_jitter=0.1)
    frs = list(spec.frames(2))
    assert frs[0].charges.dtype == np.float32
    assert not np.all(frs[0].charges == np.float32(1.0)) and np.all(np.abs(frs[0].charges) < 2)
    path = str(tmp_path / f"t.{fmt}")
    (frames.write_netcdf_trajectory if fmt == "nc" else frames.write_npz_trajectory)(path, frs)
    back = list(frames.open_trajectory(path))
    for a, b in zip(frs, back):
        np.testing.assert_array_equal(a.charges, b.charges)
        np.testing.assert_array_equal(a.xyz, b.xyz)


def test_uncharged_trajectory_has_no_charges(tmp_path):
    frs = list(frames.FCCSpec(cells=(2, 2, 2), seed=1).frames(1))
    assert frs[0].charges is None
    path = str(tmp_path / "t.nc")
    frames.write_netcdf_trajectory(path, frs)
    assert next(iter(frames.open_trajectory(path))).charges is None


def test_species_charge_derivations_match_charge_density():
    """Charge-layout rows derived from the species rows equal those of the charge density itself."""
    spec = frames.FCCSpec(cells=(4, 4, 4), sigma=0.1, fractions=(0.5, 0.3, 0.2), seed=9,
                          charges=(1.0, -0.8476, 0.4238))
    fr = spec.frame(0)
    nsp = 3
    pos, sps, off, qs = orc.layout(fr.xyz, fr.types - 1, fr.box, nsp, charges=fr.charges)
    ks = refsem.make_kset("full+axes", fr.box, 5.0, 2.0)
    rho = orc.rho_fp64(pos, off, fr.box, ks.vectors)
    rho_all = np.concatenate([rho, orc.rho_charge_fp64(pos, qs, fr.box, ks.vectors)[None, :]])
    want = orc.bin_sums(rho_all, ks.bins, ks.weights, ks.nbins)
    got = analysis.species_charged_rows(orc.bin_sums(rho, ks.bins, ks.weights, ks.nbins),
                                        np.asarray(spec.charges, np.float32), nsp)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-6)
    rc = float(F32(min(fr.box) / F32(2)))
    lsmax = int(math.floor(rc / 0.05 + 0.5)) + 1
    hist, _, gqq = orc.rdf_charged(pos, sps, qs, fr.box, float(F32(rc * rc)), 0.05, lsmax, nsp)
    np.testing.assert_allclose(analysis.species_gqq(hist, np.asarray(spec.charges, np.float32), nsp), gqq,
                               rtol=1e-12, atol=1e-9)
