"""Python side of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module,
and only as the checker (or the timed CPU baseline).  It restates the
reference's algorithm for the g_ab(r) / S_ab(Q) path on the CPU:

* layout (select_ncdfinput, src/core/netcdf.f90:582-692): FP32 fold
  r - L*int(r/L) and a stable species-contiguous order;
* pair counts (rdf_sh, src/modules/rdf.cuf:451-475) in oracle.c, all-pairs or
  linked cells, with the reference's FP32 operation order and NINT;
* rho_a(k) exactly in FP64 (oracle.c, orc_rho_fp64), and the charge density
  rho_q(k) = sum q_j exp(i k.r_j) (orc_rho_fp64_w; sq.cuf:569-573);
* the charge-product histogram of counted pairs (orc_rdf_charged; rdf.cuf:469-472)
  and avq2 = sum(q^2)/N (rdf.cuf:272);
* the reference's FP32-phase S(Q) arithmetic (sqfnD, src/modules/sq.cuf:537-581)
  for the timed CPU baseline (orc_rho_ref32);
* a pure-Python loop restatement of sq_init's n(Q) count (sq.cuf:328-342) for
  small cross-checks of the product's vectorised version.

Pinning: the n(Q) counts, Q columns and g(r) row grids of the reference's example
outputs (tests/golden/examples.json, made by tests/golden/make_golden.py) are
reproduced by the k-set/bin logic; pair counts and rho values are pinned to the
restated arithmetic only (the reference's trajectories are not shipped).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
F32 = np.float32

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.c")):
            build()
        L = ctypes.CDLL(LIB)
        vp, i64, f32, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_int
        for name in ("orc_rdf_allpairs", "orc_rdf_cells"):
            fn = getattr(L, name)
            fn.restype = None
            fn.argtypes = [vp, vp, i64, vp, f32, f32, i32, i32, vp, vp]
        L.orc_rdf_cells_range.restype = None
        L.orc_rdf_cells_range.argtypes = [vp, vp, i64, vp, f32, f32, i32, i32, vp, vp, i64, i64]
        for name in ("orc_rho_fp64", "orc_rho_ref32"):
            fn = getattr(L, name)
            fn.restype = None
            fn.argtypes = [vp, i64, vp, i32, vp, i64, vp, vp]
        L.orc_rdf_charged.restype = None
        L.orc_rdf_charged.argtypes = [vp, vp, vp, i64, vp, f32, f32, i32, i32, vp, vp, vp, i32]
        L.orc_rho_fp64_w.restype = None
        L.orc_rho_fp64_w.argtypes = [vp, vp, i64, vp, i32, vp, i64, vp, vp]
        L.orc_num_threads.restype = i32
        L.orc_set_binning.restype = None
        L.orc_set_binning.argtypes = [i32]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def layout(xyz: np.ndarray, species: np.ndarray, box, nsp: int, charges=None):
    """Fold + stable species-contiguous order; returns (pos N x 3 FP32, species N, offsets nsp+1),
    and the charges in the same order as a fourth item when given (netcdf.f90:656-658)."""
    xyz = np.asarray(xyz, F32)
    box32 = np.asarray(box, F32)
    q = (xyz / box32).astype(F32)
    folded = (xyz - (box32 * np.trunc(q)).astype(F32)).astype(F32)
    order = np.argsort(species, kind="stable")
    sp = np.asarray(species, np.int32)[order]
    off = np.zeros(nsp + 1, np.int64)
    off[1:] = np.cumsum(np.bincount(sp, minlength=nsp))
    res = (np.ascontiguousarray(folded[order]), np.ascontiguousarray(sp), off)
    if charges is not None:
        res = res + (np.ascontiguousarray(np.asarray(charges, F32)[order]),)
    return res


def rdf_counts(pos: np.ndarray, species: np.ndarray, box, side2: float, deltar: float, lsmax: int, nsp: int,
               cells: bool = False, floor_bins: bool = False):
    """uint64 [nit][lsmax] pair counts and (edge_ulp, edge_fma, counted) of one frame.
    floor_bins: bin floor(r/deltar)+1 instead of the reference's nint(r/deltar)."""
    pos = np.ascontiguousarray(pos, F32)
    sp = np.ascontiguousarray(species, np.int32)
    nit = nsp * (nsp + 1) // 2
    hist = np.zeros((nit, lsmax), np.uint64)
    edge = np.zeros(3, np.uint64)
    b = np.asarray(box, F32)
    fn = lib().orc_rdf_cells if cells else lib().orc_rdf_allpairs
    lib().orc_set_binning(1 if floor_bins else 0)
    try:
        fn(_p(pos), _p(sp), pos.shape[0], _p(b), float(F32(side2)), float(F32(deltar)), int(lsmax), int(nsp),
           _p(hist), _p(edge))
    finally:
        lib().orc_set_binning(0)
    return hist, edge


def rdf_charged(pos, species, charges, box, side2, deltar, lsmax, nsp, cells: bool = True):
    """Counts, edge statistics and the FP64 charge-product sums per bin (q_i q_j of counted pairs,
    not divided by avq2) of one frame."""
    pos = np.ascontiguousarray(pos, F32)
    sp = np.ascontiguousarray(species, np.int32)
    q = np.ascontiguousarray(charges, F32)
    hist = np.zeros((nsp * (nsp + 1) // 2, lsmax), np.uint64)
    edge = np.zeros(3, np.uint64)
    gqq = np.zeros(lsmax, np.float64)
    b = np.asarray(box, F32)
    lib().orc_set_binning(0)
    lib().orc_rdf_charged(_p(pos), _p(sp), _p(q), pos.shape[0], _p(b), float(F32(side2)), float(F32(deltar)),
                          int(lsmax), int(nsp), _p(hist), _p(edge), _p(gqq), 1 if cells else 0)
    return hist, edge, gqq


def avq2(charges) -> float:
    """sum(q^2)/N in FP64, rounded to FP32 as the reference's avq2 (rdf.cuf:272, sq.cuf:144)."""
    q = np.asarray(charges, F32).astype(np.float64)
    return float(F32(np.sum(q * q) / q.shape[0]))


def rho_charge_fp64(pos: np.ndarray, charges: np.ndarray, box, vectors: np.ndarray) -> np.ndarray:
    """Exact charge density rho_q(k) = sum_j q_j exp(i k.r_j): (nvec,) complex128."""
    pos = np.ascontiguousarray(pos, F32)
    q = np.ascontiguousarray(charges, F32)
    off = np.array([0, pos.shape[0]], np.int64)
    v = np.ascontiguousarray(vectors, np.int32)
    out = np.zeros((1, v.shape[0], 2), np.float64)
    b = np.asarray(box, F32)
    lib().orc_rho_fp64_w(_p(pos), _p(q), pos.shape[0], _p(off), 1, _p(b), v.shape[0], _p(v), _p(out))
    return out[0, :, 0] + 1j * out[0, :, 1]


def s2n_counts(pos: np.ndarray, box, side2: float, deltar: float, lsmax: int, points: np.ndarray):
    """s2D3_sh (rdf.cuf:489-553) for given sample points: per point, atoms with FP32 minimum-image
    distance r (difference point - atom, (x^2 + y^2) + z^2), r^2 < side2, binned at nint(r/deltar) and
    made cumulative (gi_s(ind:lsmax) += 1); returns the int64 sums over points of N_k and N_k^2."""
    pos = np.ascontiguousarray(pos, F32)
    L = np.asarray(box, F32)
    gi = np.zeros(lsmax + 1, np.int64)
    g2i = np.zeros(lsmax + 1, np.int64)

    def roundf(x):
        x = np.asarray(x, np.float64)
        return np.trunc(x + np.copysign(0.5, x)).astype(F32)

    for p in np.asarray(points, F32).reshape(-1, 3):
        d = (p[None, :] - pos).astype(F32)
        d = (d - (L * roundf((d / L).astype(F32))).astype(F32)).astype(F32)
        sq = (d * d).astype(F32)
        rr2 = ((sq[:, 0] + sq[:, 1]).astype(F32) + sq[:, 2]).astype(F32)
        ok = rr2 < F32(side2)
        ind = roundf((np.sqrt(rr2[ok]).astype(F32) / F32(deltar)).astype(F32)).astype(np.int64)
        h = np.bincount(ind[(ind >= 0) & (ind <= lsmax)], minlength=lsmax + 1)[:lsmax + 1]
        nk = np.cumsum(h).astype(np.int64)
        gi += nk
        g2i += nk * nk
    return gi, g2i


def rdf_counts_range(pos, species, box, side2, deltar, lsmax, nsp, i0, i1):
    """Linked-cell counts of pairs (i, j>i) with home atom i in [i0, i1)."""
    pos = np.ascontiguousarray(pos, F32)
    sp = np.ascontiguousarray(species, np.int32)
    hist = np.zeros((nsp * (nsp + 1) // 2, lsmax), np.uint64)
    edge = np.zeros(3, np.uint64)
    b = np.asarray(box, F32)
    lib().orc_rdf_cells_range(_p(pos), _p(sp), pos.shape[0], _p(b), float(F32(side2)), float(F32(deltar)),
                              int(lsmax), int(nsp), _p(hist), _p(edge), int(i0), int(i1))
    return hist, edge


def rho_fp64(pos: np.ndarray, offsets: np.ndarray, box, vectors: np.ndarray) -> np.ndarray:
    """Exact rho_a(k): (nsp, nvec) complex128."""
    pos = np.ascontiguousarray(pos, F32)
    off = np.ascontiguousarray(offsets, np.int64)
    v = np.ascontiguousarray(vectors, np.int32)
    nsp = off.shape[0] - 1
    out = np.zeros((nsp, v.shape[0], 2), np.float64)
    b = np.asarray(box, F32)
    lib().orc_rho_fp64(_p(pos), pos.shape[0], _p(off), nsp, _p(b), v.shape[0], _p(v), _p(out))
    return out[..., 0] + 1j * out[..., 1]


def rho_ref32(pos: np.ndarray, offsets: np.ndarray, box, vectors: np.ndarray) -> np.ndarray:
    """The reference's FP32-phase arithmetic (CPU baseline): (nsp, nvec) complex128."""
    pos = np.ascontiguousarray(pos, F32)
    off = np.ascontiguousarray(offsets, np.int64)
    v = np.ascontiguousarray(vectors, np.int32)
    nsp = off.shape[0] - 1
    out = np.zeros((nsp, v.shape[0], 2), np.float64)
    b = np.asarray(box, F32)
    lib().orc_rho_ref32(_p(pos), pos.shape[0], _p(off), nsp, _p(b), v.shape[0], _p(v), _p(out))
    return out[..., 0] + 1j * out[..., 1]


def bin_sums(rho: np.ndarray, bins: np.ndarray, weights: np.ndarray, nbins: int) -> np.ndarray:
    """[nbins][nit] sums of w Re(rho_a conj(rho_b)) in ind_ij row order."""
    nsp = rho.shape[0]
    rows = [(a, b) for a in range(nsp) for b in range(a, nsp)]
    out = np.zeros((nbins, len(rows)))
    for r, (a, b) in enumerate(rows):
        val = weights * (rho[a] * np.conj(rho[b])).real
        np.add.at(out[:, r], bins, val)
    return out


def nq_loops(L: float, qmax: float, qmin: float) -> list:
    """n(Q) of sq_init for a cubic box, as plain loops over FP32 scalars (sq.cuf:159-193, 328-342)."""
    f = F32
    pi = f(3.1415926535898)
    fk = f(f(f(2.0) * pi) / f(L))
    dq = fk
    nqmax = _nint(f(f(qmax) / dq))
    l = _nint(f(f(qmin) / fk))
    if l % 4 != 0:
        l = l - 4 + l % 4
    qm = f(fk * f(l))
    nq = [0] * (nqmax + 1)
    if l <= 1:
        return [0] + [3] * nqmax
    indm = 0
    for i in range(l):
        a = f(f(f(i) * fk) * f(f(i) * fk))
        for j in range(l):
            b = f(f(f(j) * fk) * f(f(j) * fk))
            ab = f(a + b)
            for k in range(l):
                if i + j + k == 0:
                    continue
                c = f(f(f(k) * fk) * f(f(k) * fk))
                rr = f(math.sqrt(float(f(ab + c))))
                if rr < qm:
                    ind = _nint(f(rr / dq))
                    indm = max(indm, ind)
                    if ind <= nqmax:
                        nq[ind] += 1
    for i in range(indm + 1, nqmax + 1):
        nq[i] = 3
    return nq


def _nint(x) -> int:
    x = float(x)
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))
