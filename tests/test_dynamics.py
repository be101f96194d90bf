"""Host side of F(Q,t)/Fs(Q,t)/MSD: the time-origin bookkeeping of rtcorr, the S(Q,w) vector set,
the fftw1d transform and the output files, against independent restatements.

Reference: src/modules/dynamics.cuf:157-276 (rtcorr), 278-393 (print_rtcor), src/modules/sq.cuf:239-297
(vectors of the qw shells), src/core/fftwlib.f90:50-119 (fftw1d, fftw1, window).
"""
import math

import numpy as np
import pytest

from oracle import orc, orc_dyn
from trj_analysis_b200 import dynamics, frames, refsem, writers
from trj_analysis_b200.refsem import F32


def _schedule_loops(nconf, nbuffer, jump, tlimit, times):
    """rtcorr's bookkeeping as plain loops: per frame, the (buffer, lag, origin) triples accumulated
    and the buffers finished."""
    ndyn = nconf - (nbuffer - 1) * jump
    origin = [i * jump + 1 for i in range(nbuffer)]
    itlimit = nconf
    out = []
    for iconf in range(1, nconf + 1):
        if iconf == 2:
            dt = F32(F32(times[1]) - F32(times[0]))
            itlimit = nconf - (nbuffer - 1) * jump if tlimit < 0 else refsem.nint(F32(F32(tlimit) / dt))
        acc = []
        for i in range(nbuffer):
            indx = iconf - origin[i] + 1
            if iconf >= origin[i] and 1 <= indx <= ndyn:
                acc.append((i, indx - 1, iconf == origin[i]))
        done = []
        for i in range(nbuffer):
            if iconf - origin[i] == itlimit:
                origin[i] = iconf + 1
                done.append(i)
        out.append((acc, done))
    return out


@pytest.mark.parametrize("nconf,nbuffer,jump,tlimit", [(20, 3, 2, -1.0), (30, 4, 3, 6.0), (12, 2, 1, -1.0),
                                                        (25, 5, 1, 3.0)])
def test_origin_schedule_matches_loops(nconf, nbuffer, jump, tlimit):
    cfg = dynamics.DynConfig(nbuffer=nbuffer, jump=jump, tlimit=tlimit, qw=(1.0,))
    sc = dynamics.OriginSchedule(nconf, cfg)
    times = [0.5 * k for k in range(nconf)]
    want = _schedule_loops(nconf, nbuffer, jump, tlimit, [F32(t) for t in times])
    for iconf in range(1, nconf + 1):
        lags, origins = sc.schedule(iconf, times[iconf - 1])
        acc = [(i, int(lags[i]), bool(origins[i])) for i in range(nbuffer) if lags[i] >= 0]
        done = list(np.flatnonzero(sc.finish_frame(iconf)))
        assert (acc, done) == want[iconf - 1], iconf
    assert sc.count_org == sum(len(d) for _, d in want)


def test_origin_schedule_errors():
    with pytest.raises(ValueError, match="too short"):
        dynamics.OriginSchedule(12, dynamics.DynConfig(nbuffer=4, jump=1))
    sc = dynamics.OriginSchedule(20, dynamics.DynConfig(nbuffer=2, tlimit=100.0))
    sc.schedule(1, 0.0)
    with pytest.raises(ValueError, match="tlimit"):
        sc.schedule(2, 1.0)


def _sqw_loops(box, qw, dq):
    """sq_init's storing loop (sq.cuf:269-295) with FqtnD's shell search (dynamics.cuf:464-471)."""
    box = np.asarray(box, F32)
    fk = [F32(refsem.TWOPI32 / L) for L in box]
    qw = [F32(q) for q in qw]
    half = F32(F32(dq) / F32(2))
    qmm = max(qw)
    lim = [refsem.nint(F32(qmm / fk[d])) for d in range(3)]
    vecs, bins, nw = [], [], [0] * len(qw)
    for i in range(lim[0] + 1):
        for j in range(lim[1] + 1):
            for k in range(lim[2] + 1):
                if i + j + k == 0:
                    continue
                s2 = F32(F32(F32(F32(i) * fk[0]) ** 2 + F32(F32(j) * fk[1]) ** 2) + F32(F32(k) * fk[2]) ** 2)
                rr = F32(math.sqrt(float(s2)))
                for l, q in enumerate(qw):
                    if F32(q - half) < rr < F32(q + half):
                        nw[l] += 1
                        q8 = math.sqrt(float(s2))
                        for m, q2 in enumerate(qw):
                            if float(F32(q2 - half)) < q8 < float(F32(q2 + half)):
                                vecs.append((i, j, k))
                                bins.append(m)
                                break
                        break
    return np.array(vecs, np.int32).reshape(-1, 3), np.array(bins, np.int32), np.array(nw)


@pytest.mark.parametrize("box,qw", [((20.0, 20.0, 20.0), (1.0, 2.0, 3.5)), ((11.3, 14.7, 9.1), (0.9, 2.2, 2.5)),
                                    ((30.0, 30.0, 60.0), (4.0,))])
def test_sqw_kset_matches_loops(box, qw):
    dq = refsem.sq_init_params(box, 5.0, 2.0).dq
    s = refsem.sqw_kset(box, qw, dq)
    v, b, nw = _sqw_loops(box, qw, dq)
    np.testing.assert_array_equal(s.vectors, v)
    np.testing.assert_array_equal(s.bins, b)
    np.testing.assert_array_equal(s.nw, nw)
    assert np.all(s.vectors >= 0) and not np.any(np.all(s.vectors == 0, axis=1))


@pytest.mark.parametrize("nin,tmax", [(40, 12.0), (100, 0.0), (130, 30.0), (17, -5.0)])
def test_fftw1d_matches_cosine_sums(nin, tmax):
    rng = np.random.default_rng(nin)
    f = np.exp(-np.arange(nin) / 9.0).astype(F32) + F32(0.01) * rng.normal(size=nin).astype(F32)
    dt = F32(0.05)
    fout, w, tm = dynamics.fftw1d(f, dt, tmax)
    nu = int(math.log(nin) / math.log(2.0) + 0.54)
    n = 2 ** (nu + 1)
    tm_want = F32(n * dt) if abs(tmax) < 1e-6 else F32(tmax)
    assert tm == tm_want
    tx = (np.arange(n).astype(F32) * dt).astype(F32)
    win = (F32(0.5) * (F32(1) - np.tanh((tx - tm_want).astype(F32)).astype(F32))).astype(F32).astype(np.float64)
    g = np.zeros(n)
    g[:nin] = f.astype(np.float64)
    g = g * win
    g[0] *= 0.5
    m = np.arange(n)
    for i in range(nin):
        if i == 0:
            want = float(dt) * g.sum()
        elif i < n // 2:
            want = float(dt) * np.sum(g * np.cos(2 * np.pi * i * m / n))
        else:  # rows past n/2 are the raw transform (fftw1 scales 2..n/2 only)
            want = np.sum(g * np.cos(2 * np.pi * i * m / n))
        assert abs(float(fout[i]) - want) <= 1e-6 * (1 + abs(want)), (i, fout[i], want)
    np.testing.assert_allclose(w, (np.arange(nin) * 2 * np.pi / (n * float(dt))), rtol=1e-6)


def test_oracle_dynamics_limits():
    """Lag 0: Fs = 1 and C_r = 0 exactly; F(k, 0) equals the bsc-weighted S(k) of the origin frames."""
    spec = frames.FCCSpec(cells=(3, 3, 3), sigma=0.1, fractions=(0.5, 0.5), seed=4)
    frs = list(frames.random_walk_frames(spec, 12, 0.3))
    box = frs[0].box
    sp = frs[0].types - 1
    packed = [orc.layout(f.xyz, sp, box, 2)[0] for f in frs]
    sps = orc.layout(frs[0].xyz, sp, box, 2)[1]
    dq = refsem.sq_init_params(box, 4, 1).dq
    s = refsem.sqw_kset(box, (1.5, 3.0), dq)
    res = orc_dyn.dynamics(packed, sps, box, (1.0, 0.5), s.vectors, s.bins, 2, s.nw, 2, 1, -1.0,
                           [F32(f.time) for f in frs])
    assert res["count_org"] >= 1
    np.testing.assert_allclose(res["fskt"][0], 1.0, rtol=1e-12)
    assert res["r2t"][0] == 0.0
    assert np.all(res["r2t"][1:res["itlimit"]] > 0)
    assert np.all(np.diff(res["t"]) > 0)


def test_dynamics_files(tmp_path):
    nd, nq = 12, 10
    res = {"t": np.arange(nd, dtype=F32) * F32(0.1), "r2t": np.linspace(0, 1, nd), "fkt": np.ones((nd, nq)),
           "fskt": np.ones((nd, nq)) * 0.5, "sqw": np.zeros((nd, nq), F32), "ssqw": np.zeros((nd, nq), F32),
           "w": np.arange(nd, dtype=F32), "itlimit": 9, "qw": np.arange(1, nq + 1, dtype=F32) * F32(0.5),
           "count_org": 2}
    files = writers.write_dynamics(str(tmp_path), res, "lj")
    dyn = open(files[0]).read().splitlines()
    assert dyn[0] == "#  t(tau)         C_r(t)"
    assert len(dyn) == 1 + 9
    assert dyn[2] == writers.fmt_f(F32(0.1), 10, 3) + writers.fmt_f(res["r2t"][1], 15, 5)
    fkt = open(files[1]).read().splitlines()
    assert fkt[0] == "#  t(tau)         " + "    ".join(f"F({q:6.4f},t)" for q in res["qw"][:8])
    assert fkt[1] == "    ".join(f"F({q:6.4f},t)" for q in res["qw"][8:])
    # 1 + 10 values per row: f10.3 + 8 f15.5, then reversion to f10.3, f15.5
    assert fkt[2] == writers.fmt_f(0.0, 10, 3) + writers.fmt_f(1.0, 15, 5) * 8
    assert fkt[3] == writers.fmt_f(1.0, 10, 3) + writers.fmt_f(1.0, 15, 5)
    sqw = open(files[3]).read().splitlines()
    assert sqw[0].startswith("#  w(1/tau)     S(0.5000,w)    Ss(0.5000,w)    S(1.0000,w)")
    files = writers.write_dynamics(str(tmp_path), res, "real")
    assert open(files[0]).read().startswith("#  t(ps)         C_r(t)")
    assert open(files[3]).read().startswith("#  w(THz)       w(meV)     S(0.5000,w)")
    assert writers.fmt_f(10.0, 6, 4) == "******"  # f6.4 overflow, as Fortran prints it


# ---- known answers from the reference's shipped dynamics outputs (tests/golden/dynamics.json) ----

import json
import os

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "dynamics.json")))


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_row_counts(name):
    """dyn.dat / fkt.dat hold itlimit rows: Nconf - (nbuffer-1)*jump with the default tlimit."""
    g = GOLDEN[name]
    nconf = g["ncfs_from_to"][0]
    cfg = dynamics.DynConfig(nbuffer=g["nbuffer"], jump=g["jump"], tlimit=g["tlimit"], tmax=g["tmax"], qw=(1.0,))
    sc = dynamics.OriginSchedule(nconf, cfg)
    sc.schedule(1, 0.0)
    sc.schedule(2, 0.005)
    assert sc.itlimit == g["dyn_rows"]
    if "fkt" in g:
        assert len(g["fkt"]) == len(g["fskt"]) == len(g["sqw"]) == g["dyn_rows"] == sc.ndyn


def test_golden_headers_and_time_column(tmp_path):
    g = GOLDEN["salr"]
    nd = g["dyn_rows"]
    t = (np.arange(nd).astype(F32) * F32(0.005)).astype(F32)
    res = {"t": t, "r2t": np.zeros(nd), "fkt": np.zeros((nd, 1)), "fskt": np.zeros((nd, 1)),
           "sqw": np.zeros((nd, 1), F32), "ssqw": np.zeros((nd, 1), F32), "w": np.zeros(nd, F32),
           "itlimit": nd, "qw": np.asarray(g["qw"], F32), "count_org": 1}
    files = writers.write_dynamics(str(tmp_path), res, units="real")
    got = [open(f).read().splitlines() for f in files]
    assert g["dyn_header"].startswith(got[0][0])  # the reference adds C_v(t) when the trajectory has velocities
    assert got[1][0] == g["fkt_header"]
    assert got[2][0] == g["fskt_header"]
    assert got[3][0] == g["sqw_header"]
    assert [ln[:10].strip() for ln in got[1][1:]] == g["dyn_t"]


@pytest.mark.parametrize("col,key", [(2, "fkt"), (3, "fskt")])
def test_golden_transform(col, key):
    """sqw.dat is fftw1d of fkt.dat / fskt.dat (print_rtcor, dynamics.cuf:306-313) with tmax = 2.0 from
    /INPUT_DYN/ and dt = t(2) - t(1).  The frame times are FP32 products nstep*tstep; their difference,
    printed as 0.005, is an FP32 difference of two times between 8 and 16 ps, i.e. a multiple of 2^-20:
    5243 * 2^-20 = 0.0050001144 (5242 or 5244 * 2^-20 miss by 1e-2).  With it the restated transform of
    the printed F(t) reproduces the printed S(w) to the rounding of the five printed decimals."""
    g = GOLDEN["salr"]
    f = np.array([float(r[0]) for r in g[key]], np.float32)
    dt = F32(5243 * 2.0 ** -20)
    s, w, _ = dynamics.fftw1d(f, dt, F32(g["tmax"]))
    want = np.array([float(r[col]) for r in g["sqw"]])
    err = np.max(np.abs(s.astype(np.float64) - want))
    assert err <= 1e-5, err
    s2, _, _ = dynamics.fftw1d(f, dt, F32(g["tmax"] - 0.01))  # the window position matters at this level
    assert np.max(np.abs(s2.astype(np.float64) - want)) > 100 * err
    twopi = F32(F32(2) * F32(3.141592653589793))
    thz = [writers.fmt_f(F32(x / twopi), 10, 3).strip() for x in w]
    mev = [writers.fmt_f(F32(F32(F32(4.135) * x) / twopi), 10, 3).strip() for x in w]
    assert thz == [r[0] for r in g["sqw"]]
    assert mev == [r[1] for r in g["sqw"]]
