"""Known-answer checks of the oracle and the host-side k-set/bin logic against the
reference's shipped example outputs (tests/golden/examples.json).

Pinned columns: n(Q) (sq.dat last column) and Q = i*dq (first column) of
examples/3D/{LJmix, meam-dyn, salr}, and the r grid / row count of gmixsim.dat.
The boxes are cubic; L is recovered as the FP32 value whose 2*pi/L reproduces
every printed Q.  salr's sq.dat was written by an older version that printed
only the first 51 Q values on the i*dq grid; its n(Q) column matches on all rows.
"""
import json
import os

import numpy as np
import pytest

from oracle import orc
from trj_analysis_b200 import refsem
from trj_analysis_b200.refsem import F32

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "examples.json")))


def recover_box(qcol, rows=None):
    rows = len(qcol) if rows is None else rows
    guess = F32(float(qcol[0]))
    base = int(np.frombuffer(np.array([guess], F32).tobytes(), np.uint32)[0])
    for off in range(-4000, 4000):
        dq = np.frombuffer(np.array([base + off], np.uint32).tobytes(), F32)[0]
        if all(f"{F32(F32(i + 1) * dq):.7f}" == qcol[i] for i in range(rows)):
            L = F32(refsem.TWOPI32 / dq)
            for c in (L, np.nextafter(L, F32(np.inf)), np.nextafter(L, F32(0))):
                if F32(refsem.TWOPI32 / c) == dq:
                    return F32(c)
    raise AssertionError("no FP32 box reproduces the Q column")


CASES = [("LJmix", None), ("meam-dyn", None), ("salr", 51)]


@pytest.mark.parametrize("name,qrows", CASES)
def test_nq_column_matches_reference(name, qrows):
    ex = GOLD[name]
    L = recover_box(ex["sq_q"], qrows)
    ks = refsem.reference_kset([L, L, L], ex["qmax"], ex["qmin"])
    gold = np.array(ex["sq_nq"])
    got = ks.nq[1:1 + gold.size]
    assert np.array_equal(got, gold)


@pytest.mark.parametrize("name,qrows", CASES)
def test_q_column_matches_reference(name, qrows):
    ex = GOLD[name]
    L = recover_box(ex["sq_q"], qrows)
    ks = refsem.reference_kset([L, L, L], ex["qmax"], ex["qmin"])
    q = ks.q_column()
    rows = len(ex["sq_q"]) if qrows is None else qrows
    assert [f"{v:.7f}" for v in q[:rows]] == ex["sq_q"][:rows]
    if name == "LJmix":
        # meam-dyn's file stops one row short of nint(qmax/dq) (an older writer).
        assert ks.nqmax == len(ex["sq_q"])


def test_nq_loops_restatement_agrees():
    ex = GOLD["LJmix"]
    L = recover_box(ex["sq_q"])
    loops = orc.nq_loops(float(L), ex["qmax"], ex["qmin"])
    ks = refsem.reference_kset([L, L, L], ex["qmax"], ex["qmin"])
    assert list(ks.nq) == loops


@pytest.mark.parametrize("name,qrows", CASES)
def test_gmix_grid_matches_reference(name, qrows):
    ex = GOLD[name]
    L = recover_box(ex["sq_q"], qrows)
    p = refsem.rdf_params(ex["nsp"], ex["deltar"], ex["rcrdf"], [L, L, L])
    rows = p.lsmax - 2
    assert rows == len(ex["gmix_r"])
    r = [f"{F32(F32(i) * F32(ex['deltar'])):.5f}" for i in range(1, rows + 1)]
    assert r == ex["gmix_r"]


def test_headers_match_reference():
    from trj_analysis_b200 import writers
    assert GOLD["LJmix"]["sq_header"] == writers.SQ_HEADER_BINARY
    assert GOLD["salr"]["sq_header"] == writers.SQ_HEADER
    assert writers.sqmix_header(2)[0] == GOLD["LJmix"]["sqmix_header"]
    assert writers.sqmix_header(1)[0] == GOLD["salr"]["sqmix_header"]
    labels = [f"g_{j + 1}{k + 1}(r)" for j in range(2) for k in range(j, 2)]
    assert writers._group_header("#       r        " + " " * 9, labels, 16, " " * 9)[0] == GOLD["LJmix"]["gmix_header"]


def test_meam_dyn_needs_fp32_geometry():
    """The FP64 evaluation of rr < qmin would give a different last full shell (2922 vs 2928)."""
    ex = GOLD["meam-dyn"]
    L = recover_box(ex["sq_q"])
    ks = refsem.reference_kset([L, L, L], ex["qmax"], ex["qmin"])
    assert 2928 in list(ks.nq)


def test_two_dimensional_example_columns():
    """examples/2D/salr (ndim = 2): sq_init's 2D n(Q) (x and y only, lmax aligned to 16, loops over
    0..lmax inclusive) reproduces every printed n(Q); the box is square, recovered from the Q column.
    Like salr's 3D file, this sq.dat comes from an older writer: past the fully sampled region
    (rows 1..nqmin+1 = 149) it printed every third Q of the axis region, all with n(Q) = 2."""
    ex = GOLD["2D/salr"]
    assert ex["ndim"] == 2
    L = recover_box(ex["sq_q"], 50)
    ks = refsem.reference_kset([L, L, F32(1.0)], ex["qmax"], ex["qmin"], ndim=2)
    gold = np.array(ex["sq_nq"])
    assert np.array_equal(ks.nq[1:1 + gold.size], gold)
    assert ks.nqmin + 1 == 149
    assert [f"{v:.7f}" for v in ks.q_column()[:149]] == ex["sq_q"][:149]
    p = refsem.rdf_params(ex["nsp"], ex["deltar"], ex["rcrdf"], [L, L, F32(1.0)], ndim=2)
    assert p.lsmax - 2 == len(ex["gmix_r"])
    assert [f"{F32(F32(i) * F32(ex['deltar'])):.5f}" for i in range(1, p.lsmax - 1)] == ex["gmix_r"]


@pytest.mark.parametrize("name,charged", [("Conf", False), ("RTIL+H20_rigid", True)])
def test_seven_species_files_and_charge_columns(name, charged, tmp_path):
    """nsp = 7 writes one gmixsim<k>.dat per species; with charges (RTIL+H20_rigid) the first file has
    g_qq(r) after r and sq.dat has S_qq(Q) after S_NN(Q) (log.f90:353-362, 456-458, 565-567)."""
    from trj_analysis_b200 import writers
    ex = GOLD[name]
    nrow = len(ex["gmix1_r"])
    r = np.array([F32(F32(i) * F32(ex["deltar"])) for i in range(1, nrow + 1)], np.float32)
    g = np.zeros((nrow, 7, 7))
    files = writers.write_gmixsim(str(tmp_path), r, g, 7, g_qq=np.zeros(nrow) if charged else None)
    lines = open(files[0]).read().splitlines()
    assert lines[0] == ex["gmix1_header"]
    assert len(lines[1].split()) == ex["gmix1_ncols"]
    assert [ln.split()[0] for ln in lines[1:]] == ex["gmix1_r"]
    head = writers.SQ_HEADER_QQ if charged else writers.SQ_HEADER
    assert head == ex["sq_header"]
