"""Host logic that needs no GPU: C-ABI exports, species numbering, k-sets, normalisation, writers."""
import ctypes
import os
import re

import numpy as np
import pytest

from trj_analysis_b200 import frames, refsem, writers
from trj_analysis_b200.refsem import F32

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "trj_sm100.h")).read()
    return sorted(set(re.findall(r"TRJ_API\s+[\w\s\*]+?\b(trj_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from trj_analysis_b200 import _lib
    lib = _lib.load()
    syms = _declared_symbols()
    assert len(syms) >= 16
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_lib.SIGNATURES)
    assert lib.trj_abi_version() == 1


def test_ctx_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from trj_analysis_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.trj_ctx_create(0, ctypes.byref(h)) != 0
    assert not h.value


def test_null_and_invalid_arguments_return_status():
    from trj_analysis_b200 import _lib
    lib = _lib.load()
    assert lib.trj_ctx_create(0, None) == _lib.TRJ_ERR_INVALID
    assert lib.trj_rdf_plan_create(None, 1, 0.1, 1.0, None, 10, None) == _lib.TRJ_ERR_INVALID
    assert lib.trj_sq_plan_destroy(None) == 0
    assert lib.trj_ctx_last_error(None) == b"null context"


def test_species_numbered_by_first_appearance():
    types = np.array([3, 3, 1, 2, 1, 3, 2], np.int32)
    sp, wtypes, perm = refsem.species_by_first_appearance(types, [1, 2, 3])
    assert wtypes == [3, 1, 2]
    assert list(sp) == [0, 0, 1, 2, 1, 0, 2]
    assert perm == [2, 0, 1]
    sp2, wt2, _ = refsem.species_by_first_appearance(types, [1, 3])
    assert wt2 == [3, 1] and list(sp2) == [0, 0, 1, -1, 1, 0, -1]


def test_rdf_params_clip_and_lsmax():
    p = refsem.rdf_params(1, 0.02, 1e6, [17.0998, 17.0998, 17.0998])
    assert abs(p.rcrdf - 8.5499) < 1e-4
    assert p.lsmax == refsem.nint(F32(F32(p.rcrdf) / F32(0.02))) + 1 == 428
    p2 = refsem.rdf_params(3, 0.01, 8.0, [107.73] * 3)
    assert p2.lsmax == 801 and p2.side2 == float(F32(8.0) * F32(8.0))
    p3 = refsem.rdf_params(2, 0.02, 6.0, [107.72, 107.72, 430.89])
    assert p3.lsmax == 301


def test_nint_half_away_from_zero():
    assert refsem.nint(F32(0.5)) == 1 and refsem.nint(F32(-0.5)) == -1
    assert refsem.nint(F32(2.5)) == 3 and refsem.nint(F32(0.49999997)) == 0


@pytest.mark.parametrize("mode", ["full", "full+axes", "full+sampled", "ref"])
def test_kset_structure(mode):
    box = np.array([12.0, 12.0, 13.5], F32)
    ks = refsem.make_kset(mode, box, qmax=4.0, qmin=2.5, seed=3, per_shell=20)
    assert ks.vectors.shape == (ks.nvec, 3) and ks.bins.shape == (ks.nvec,)
    assert ks.bins.min() >= 1 and ks.bins.max() <= ks.nqmax
    assert not np.any(np.all(ks.vectors == 0, axis=1))
    if mode.startswith("full"):
        tot = np.zeros(ks.nqmax + 1)
        np.add.at(tot, ks.bins, ks.weights)
        assert np.array_equal(tot.astype(np.int64), ks.nq)
        # no vector and its negative both present among the +-paired (weight 2) vectors
        w2 = ks.vectors[ks.weights == 2]
        s = {tuple(v) for v in w2}
        assert not any(tuple(-v) in s for v in w2)


def test_full_kset_covers_sphere():
    box = np.array([10.0, 10.0, 10.0], F32)
    ks = refsem.make_kset("full", box, qmax=3.0)
    fk = 2 * np.pi / 10.0
    m = 6
    g = np.stack(np.meshgrid(*[np.arange(-m, m + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    q = np.sqrt(((g * fk) ** 2).sum(1))
    b = np.floor(q / float(ks.dq) + 0.5)
    expect = np.bincount(b[(b >= 1) & (b <= ks.nqmax)].astype(int), minlength=ks.nqmax + 1)
    assert np.array_equal(expect, ks.nq)


def test_reference_kset_axis_quirk_noncubic():
    box = np.array([20.0, 20.0, 40.0], F32)
    ks = refsem.reference_kset(box, qmax=3.0, qmin=1.0)
    axes = ks.vectors[ks.dense == 0]
    # axis vectors are binned at k whatever their |q| (sq.cuf:413-449)
    for v, b in zip(axes, ks.bins[ks.dense == 0]):
        assert int(np.abs(v).max()) == int(b)


def test_writers_fortran_format():
    assert writers.fmt_f(0.123456, 16, 5) == "         0.12346"
    assert writers.fmt_f(1e20, 15, 7) == "*" * 15
    assert writers.fmt_f(0.015625, 16, 5) == "         0.01563"
    assert writers.fmt_i(145, 12) == "         145"


def test_normalise_rdf_ideal_gas_limit():
    from trj_analysis_b200.analysis import normalise_rdf, shell_volumes
    lsmax, dr, V, N = 50, 0.1, 1000.0, 1000
    dv, ri = shell_volumes(lsmax, dr)
    # ideal counts for one species: N(N-1)/2 * dV/V
    h = np.round(N * N / 2 * dv / V).astype(np.uint64)[None, :]
    res = normalise_rdf(h, 1, lsmax, dr, V, np.array([N]), 1)
    assert np.allclose(res["g"][5:, 0, 0], 1.0, rtol=2e-3)


def test_synthetic_frames_shape_and_determinism():
    s = frames.c3_spec()
    assert s.n == 1000188 and abs(float(s.box[0]) - 107.728) < 1e-2
    small = frames.FCCSpec(cells=(5, 5, 5), fractions=(0.5, 0.3, 0.2), replace_frac=0.02, seed=9)
    a, b = small.frame(0), small.frame(0)
    assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.types, b.types)
    c = small.frame(1)
    assert np.array_equal(a.types, c.types) and not np.array_equal(a.xyz, c.xyz)
    counts = np.bincount(a.types)[1:]
    assert list(counts) == [250, 150, 100]
    assert frames.c4_spec().n == 4000000


def test_namelist_reader():
    from trj_analysis_b200 import namelist
    text = """&INPUT
  trj_input_file='run.nc'   ! a comment
  nsp=2
  ncfs_from_to=1000 1 1000
  rdf_sq_cl_dyn_sqw_conf_ord=T T F F F  F T
  rcl=1.5
/
&INPUT_SP
  sp_types_selected=3 1
  mat=1.0 2.0
/
&INPUT_RDF
  deltar=0.25
  rcrdf=15.0
/
&INPUT_SQ
  qmax=25.0
  qmin=6.4
  bsc=1.0 0.6d0
/
"""
    g = namelist.parse(text)
    assert g["INPUT"]["trj_input_file"] == "run.nc" and g["INPUT"]["nsp"] == 2
    assert g["INPUT"]["rdf_sq_cl_dyn_sqw_conf_ord"] == [True, True, False, False, False, False, True]
    cfg = namelist.config_from_namelist(g)
    assert cfg.sp_types_selected == [3, 1] and cfg.deltar == 0.25 and cfg.rcrdf == 15.0
    assert cfg.qmax == 25.0 and cfg.qmin == 6.4 and cfg.bsc == [1.0, 0.6]
    assert namelist.parse("&A x=3*0 /\n")["A"]["x"] == [0, 0, 0]


def test_netcdf_roundtrip(tmp_path):
    spec = frames.FCCSpec(cells=(3, 3, 3), fractions=(0.5, 0.5), seed=5)
    frs = [spec.frame(i) for i in range(3)]
    p = str(tmp_path / "t.nc")
    frames.write_netcdf_trajectory(p, frs)
    got = list(frames.open_trajectory(p))
    assert len(got) == 3
    for a, b in zip(got, frs):
        assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.types, b.types)
        assert np.array_equal(a.box, b.box)


def test_netcdf4_file_refused_with_conversion_hint(tmp_path):
    """A NETCDF4 (HDF5) trajectory, the format of tools/lammpstrj_to_netcdf.py:28, needs netCDF4;
    without it the reader names the conversion to the classic 64-bit-offset format."""
    p = tmp_path / "t4.nc"
    p.write_bytes(frames.NetCDFTrajectory.HDF5_SIGNATURE + bytes(64))
    try:
        import netCDF4  # noqa: F401
        pytest.skip("netCDF4 is installed: the file would be read by it")
    except ImportError:
        pass
    with pytest.raises(ValueError, match="nccopy -k 64-bit-offset"):
        frames.open_trajectory(str(p))


def test_linear_kset_counts():
    box = np.array([20.0, 20.0, 20.0], F32)
    ks = refsem.linear_kset(box, 2 * np.pi / 20.0, 2.0, 10)
    fk = 2 * np.pi / 20.0
    m = 8
    g = np.stack(np.meshgrid(*[np.arange(-m, m + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    q = np.sqrt(((g * fk) ** 2).sum(1))
    sel = (q >= fk) & (q < 2.0)
    assert ks.nq.sum() == sel.sum()


def test_s2n_normalisation_and_file(tmp_path):
    from trj_analysis_b200 import analysis
    lsmax, nconf, nrandom = 8, 3, 4
    gi = np.arange(lsmax + 1, dtype=np.int64) * 12
    g2i = gi * gi // 10 + 7
    s = analysis.normalise_s2n(gi, g2i, nconf, nrandom, lsmax)
    m = nconf * nrandom
    np.testing.assert_allclose(s, g2i[1:lsmax - 1] / m - (gi[1:lsmax - 1] / m) ** 2)
    r = np.arange(1, lsmax - 1, dtype=np.float32) * np.float32(0.1)
    p = writers.write_s2n(str(tmp_path), r, s)
    lines = open(p).read().splitlines()
    assert lines[0] == "#       r                s2n"
    assert lines[1] == writers.fmt_f(r[0], 16, 5) + writers.fmt_f(s[0], 16, 5)
    assert len(lines) == 1 + lsmax - 2


def test_oracle_s2n_counts_small_case():
    """Two atoms around one point: cumulative counts from the bins nint(r/deltar)."""
    from oracle import orc
    box = np.array([10.0, 10.0, 10.0], np.float32)
    pos = np.array([[1.0, 1.0, 1.0], [1.0, 1.0, 1.55], [9.9, 1.0, 1.0]], np.float32)
    gi, g2i = orc.s2n_counts(pos, box, 4.0, 0.1, 25, np.array([[1.0, 1.0, 1.0]], np.float32))
    # distances 0 (bin 0); 1.0 - 1.55 = -0.54999995 in FP32, /0.1 = 5.4999995 -> bin 5; 1.1000004 through
    # the boundary -> bin 11
    want = np.zeros(26, np.int64)
    want[0:] += 1
    want[5:] += 1
    want[11:] += 1
    np.testing.assert_array_equal(gi, want)
    np.testing.assert_array_equal(g2i, want * want)
