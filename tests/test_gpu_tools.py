"""The command-line tools end to end (classic NetCDF in, reference-format files out)."""
import math
import os

import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import frames, refsem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def traj(tmp_path_factory):
    d = tmp_path_factory.mktemp("traj")
    spec = frames.FCCSpec(cells=(7, 7, 7), sigma=0.1, fractions=(0.7, 0.3), seed=31)
    frs = [spec.frame(i) for i in range(2)]
    path = str(d / "run.nc")
    frames.write_netcdf_trajectory(path, frs)
    return d, path, frs


def test_netcdf_roundtrip(traj):
    d, path, frs = traj
    got = list(frames.open_trajectory(path))
    assert len(got) == 2
    assert np.array_equal(got[1].xyz, frs[1].xyz) and np.array_equal(got[1].types, frs[1].types)


def test_fast_grfreud_matches_oracle(traj, monkeypatch):
    from trj_analysis_b200.tools import fast_grfreud_netcdf as tool
    d, path, frs = traj
    monkeypatch.chdir(d)
    assert tool.main([path, "--r-max", "5.0", "--bins", "100"]) == 0
    data = np.loadtxt(d / "gr.dat")
    head = open(d / "gr.dat").readline()
    assert head.startswith("# r g(r)")
    # oracle: floor bins of width 0.05 on [0, 5)
    H = 0
    for fr in frs:
        sp, wt = refsem.species_by_first_appearance(fr.types, sorted(set(fr.types)))[:2]
        pos, sps, off = orc.layout(fr.xyz, sp, fr.box, 2)
        h, _ = orc.rdf_counts(pos, sps, fr.box, float(np.float32(5.0) * np.float32(5.0)),
                              float(np.float32(5.0) / np.float32(100)), 100, 2, cells=True, floor_bins=True)
        H = H + h.astype(np.float64)
    n = frs[0].n
    V = refsem.volume(frs[0].box)
    edges = np.arange(101) * (5.0 / 100)
    dv = 4 * math.pi / 3 * (edges[1:] ** 3 - edges[:-1] ** 3)
    g = 2 * H.sum(0) / (2 * n * (n / V) * dv)
    assert np.allclose(data[:, 1], g, rtol=1e-12, atol=0)
    assert data.shape[1] == 2 + 3


def test_fast_sq_freud_matches_oracle(traj, monkeypatch):
    from trj_analysis_b200.tools import fast_sq_freud_netcdf as tool
    d, path, frs = traj
    monkeypatch.chdir(d)
    assert tool.main([path, "--k-max", "3.0", "--bins", "12"]) == 0
    data = np.loadtxt(d / "Sq.dat")
    kmin = 2 * math.pi / float(np.max(frs[0].box))
    ks = refsem.linear_kset(frs[0].box, kmin, 3.0, 12)
    tot = np.zeros(12)
    for fr in frs:
        sp = refsem.species_by_first_appearance(fr.types, sorted(set(fr.types)))[0]
        pos, sps, off = orc.layout(fr.xyz, sp, fr.box, 2)
        rho = orc.rho_fp64(pos, off, fr.box, ks.vectors)
        s = rho[0] + rho[1]
        np.add.at(tot, ks.bins, ks.weights * np.abs(s) ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        S = tot / (frs[0].n * ks.nq * 2)
    live = ks.nq > 0
    assert np.allclose(data[live, 1], S[live], rtol=1e-5)
    assert np.all(np.isnan(data[~live, 1]))


def test_trj_analysis_reference_outputs(traj, monkeypatch):
    from trj_analysis_b200.tools import trj_analysis as tool
    d, path, frs = traj
    nml = d / "input.nml"
    nml.write_text("&INPUT\n trj_input_file='run.nc'\n nsp=2\n ncfs_from_to=2 1 2\n"
                   " rdf_sq_cl_dyn_sqw_conf_ord=T T F F F F F\n/\n&INPUT_SP\n sp_types_selected=1 2\n/\n"
                   "&INPUT_RDF\n deltar=0.05\n rcrdf=5.0\n/\n&INPUT_SQ\n qmax=4.0\n qmin=2.0\n/\n")
    monkeypatch.chdir(d)
    assert tool.main([str(nml), "0", "--kset", "ref"]) == 0
    g = open(d / "gmixsim.dat").read().splitlines()
    p = refsem.rdf_params(2, 0.05, 5.0, frs[0].box)
    assert len(g) - 1 == p.lsmax - 2
    assert g[0] == "#       r                 g_11(r)         g_12(r)         g_22(r)"
    sq = open(d / "sq.dat").read().splitlines()
    ks = refsem.reference_kset(frs[0].box, 4.0, 2.0)
    assert [int(r.split()[-1]) for r in sq[1:]] == list(ks.nq[1:])
    assert sq[0].startswith("#           Q        S_NN(Q)")  # binary with bsc = 1
    # g_11 column against the oracle counts normalised as printrdf does
    H = 0
    for fr in frs:
        sp = refsem.species_by_first_appearance(fr.types, [1, 2])[0]
        pos, sps, off = orc.layout(fr.xyz, sp, fr.box, 2)
        h, _ = orc.rdf_counts(pos, sps, fr.box, p.side2, p.deltar, p.lsmax, 2, cells=True)
        H = H + h.astype(np.float64)
    sp0, wt, _ = refsem.species_by_first_appearance(frs[0].types, [1, 2])
    nt = np.bincount(sp0, minlength=2)
    from trj_analysis_b200.analysis import normalise_rdf
    ref = normalise_rdf(H.astype(np.uint64), 2, p.lsmax, 0.05, refsem.volume(frs[0].box), nt, 2)
    got = np.array([[float(x) for x in r.split()] for r in g[1:]])
    assert np.allclose(got[:, 1], ref["g"][:, 0, 0], atol=6e-6)


def test_trj_analysis_dynamics_charges_s2n(tmp_path, monkeypatch):
    """The namelist driver with time correlations (/INPUT_DYN/, /INPUT_SQW/), number fluctuations
    (nrandom) and a trajectory that carries charges and times: every output file of the reference."""
    from trj_analysis_b200.tools import trj_analysis as tool
    spec = frames.FCCSpec(cells=(5, 5, 5), sigma=0.1, fractions=(0.5, 0.5), seed=44, charges=(1.0, -1.0))
    frs = []
    for f in frames.random_walk_frames(spec, 12, 0.1):
        f.time = f.time + 1.0  # no step 0 (the reference skips it)
        frs.append(f)
    frames.write_netcdf_trajectory(str(tmp_path / "run.nc"), frs)
    nml = tmp_path / "input.nml"
    nml.write_text("&INPUT\n trj_input_file='run.nc'\n nsp=2\n ncfs_from_to=12 1 12\n"
                   " rdf_sq_cl_dyn_sqw_conf_ord=T T F T T F F\n/\n&INPUT_SP\n sp_types_selected=1 2\n/\n"
                   "&INPUT_RDF\n deltar=0.05\n rcrdf=3.0\n nrandom=8\n/\n&INPUT_SQ\n qmax=4.0\n qmin=2.0\n/\n"
                   "&INPUT_DYN\n nbuffer=2\n tmax=3.0\n/\n&INPUT_SQW\n qw=1.5 3.0\n/\n")
    monkeypatch.chdir(tmp_path)
    assert tool.main([str(nml), "0"]) == 0
    g = open(tmp_path / "gmixsim.dat").read().splitlines()
    assert "g_qq(r)" in g[0]
    assert open(tmp_path / "sq.dat").readline().startswith("#           Q        S_NN(Q)          S_qq(Q)")
    assert open(tmp_path / "s2n.dat").readline().strip().endswith("s2n")
    fkt = open(tmp_path / "fkt.dat").read().splitlines()
    assert fkt[0] == "#  t(ps)         F(1.5000,t)    F(3.0000,t)"
    assert len(fkt) - 1 == 11  # itlimit = Nconf - (nbuffer-1)*jump
    row = [float(x) for x in fkt[1].split()]
    assert row[0] == 0.0 and all(np.isfinite(row))
    fs = [float(x) for x in open(tmp_path / "fskt.dat").read().splitlines()[1].split()]
    assert abs(fs[1] - 1.0) < 1e-5 and abs(fs[2] - 1.0) < 1e-5  # Fs(Q, 0) = 1
    dyn = open(tmp_path / "dyn.dat").read().splitlines()
    assert dyn[0] == "#  t(ps)         C_r(t)" and float(dyn[1].split()[1]) == 0.0 and float(dyn[3].split()[1]) > 0
    assert len(open(tmp_path / "sqw.dat").read().splitlines()) == 1 + 11
