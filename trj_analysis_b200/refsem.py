"""Host-side parameter semantics of the reference, restated with FP32 arithmetic.

Everything here is O(1) or O(k-vectors) set-up work that the reference does on
the host: the rcrdf clip and bin count of the g(r) path, the species numbering
by first appearance, and ``sq_init``'s k-set.  Values that the reference keeps
in ``real(myprec)`` (FP32, src/core/precision.f90:22) are computed here with
numpy float32 scalars, one rounding per operation, in the order the Fortran
states them.  Fortran NINT rounds half away from zero.
"""
from __future__ import annotations

import dataclasses
from typing import Optional, Sequence

import numpy as np

F32 = np.float32
# pi is a real(myprec) parameter (src/core/common.cuf:43): the FP32 value of 3.1415926535898.
PI32 = F32(3.1415926535898)
TWOPI32 = F32(F32(2.0) * PI32)


def nint(x):
    """Fortran NINT: nearest integer, halves away from zero (exact for FP32 input)."""
    a = np.asarray(x, dtype=np.float64)
    r = np.sign(a) * np.floor(np.abs(a) + 0.5)
    if np.ndim(r) == 0:
        return int(r)
    return r.astype(np.int64)


def pair_row(a: int, b: int, nsp: int) -> int:
    """0-based row of species pair (a, b): ind_ij (src/modules/rdf.cuf:741-753) minus one."""
    if a > b:
        a, b = b, a
    return a * (nsp - 1) - a * (a - 1) // 2 + b


def pair_rows(nsp: int):
    """[(a, b)] for rows 0..nit-1 in ind_ij order (a <= b, a-major)."""
    return [(a, b) for a in range(nsp) for b in range(a, nsp)]


# ---------------------------------------------------------------------------
# Species numbering and the fold (select_ncdfinput, src/core/netcdf.f90:472-509, 582-692)
# ---------------------------------------------------------------------------

def species_by_first_appearance(types: np.ndarray, selected: Sequence[int]):
    """Species index (0-based) of each atom, numbered by first appearance of its type.

    Mirrors read_nc_cfg (src/core/netcdf.f90:472-491): the selected LAMMPS types are
    numbered in the order they first occur in the atom array.  Returns
    (species per atom, -1 for unselected; ordered list of type ids; permutation p such
    that parameters given per ``selected`` entry map to species s via p[s]).
    """
    types = np.asarray(types)
    sel = [int(t) for t in selected]
    _, first = np.unique(types, return_index=True)
    order = types[np.sort(first)]
    wtypes = [int(t) for t in order if int(t) in sel]
    lut = {t: s for s, t in enumerate(wtypes)}
    sp = np.array([lut.get(int(t), -1) for t in np.unique(types)], dtype=np.int32)
    uniq = np.unique(types)
    species = sp[np.searchsorted(uniq, types)]
    perm = [sel.index(t) for t in wtypes]
    return species.astype(np.int32), wtypes, perm


def fold(xyz: np.ndarray, box: np.ndarray) -> np.ndarray:
    """r = r - L*int(r/L) in FP32 (netcdf.f90:681); negatives stay negative."""
    xyz = np.asarray(xyz, F32)
    box = np.asarray(box, F32)
    q = (xyz / box).astype(F32)
    return (xyz - (box * np.trunc(q)).astype(F32)).astype(F32)


def volume(box, ndim: int = 3) -> float:
    """volumen = product of the first ndim box edges in FP32 (netcdf.f90:618-622)."""
    v = F32(1.0)
    for L in np.asarray(box, F32)[:ndim]:
        v = F32(v * L)
    return float(v)


# ---------------------------------------------------------------------------
# g(r) parameters (RDF_init, src/modules/rdf.cuf:51-66, with netcdf.f90:610-617)
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class RdfParams:
    nsp: int
    deltar: float      # FP32 value
    rcrdf: float       # FP32 value after the clip
    side2: float       # FP32 value
    lsmax: int

    @property
    def nit(self) -> int:
        return self.nsp * (self.nsp + 1) // 2


def rdf_params(nsp: int, deltar: float, rcrdf: float, box, ndim: int = 3) -> RdfParams:
    box = np.asarray(box, F32)
    side = F32(box[:ndim].min())  # minval(sidel(1:ndim)) (netcdf.f90:610)
    half = F32(side / F32(2.0))
    rc = F32(min(F32(rcrdf), half))
    dr = F32(deltar)
    if rc > 0:
        side2 = F32(rc * rc)
        lsmax = nint(F32(rc / dr)) + 1
    else:
        side2 = F32(half * half)
        lsmax = nint(F32(half / dr)) + 1
    return RdfParams(nsp=nsp, deltar=float(dr), rcrdf=float(rc), side2=float(side2), lsmax=int(lsmax))


# ---------------------------------------------------------------------------
# S(Q) k-sets
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class KSet:
    """Integer lattice vectors n (k = 2 pi n / L), their bins, weights and denominators."""
    mode: str
    dq: float                      # FP32 shell width (minval(2 pi / L))
    nqmax: int
    vectors: np.ndarray            # (nvec, 3) int32
    bins: np.ndarray               # (nvec,) int32 in 0..nqmax
    weights: np.ndarray            # (nvec,) float64 multiplicity
    dense: np.ndarray              # (nvec,) uint8, 1 = compact region (tensor tiles)
    nq: np.ndarray                 # (nqmax+1,) int64 denominators per bin
    qmin_eff: float = 0.0
    lmax: tuple = (0, 0, 0)
    nqmin: int = 0

    @property
    def nvec(self) -> int:
        return int(self.vectors.shape[0])

    @property
    def nbins(self) -> int:
        return self.nqmax + 1

    def q_column(self) -> np.ndarray:
        """Q of rows i = 1..nqmax as the reference prints it: i*dq in FP32 (log.f90:364-405)."""
        return np.array([F32(F32(i) * F32(self.dq)) for i in range(1, self.nqmax + 1)], dtype=F32)


@dataclasses.dataclass
class SqInit:
    """The scalars sq_init derives (src/modules/sq.cuf:150-193)."""
    fk: np.ndarray        # (3,) FP32 2*pi/L
    dq: float
    nqmax: int
    lmax: tuple
    nqmin: int
    qmin_eff: float


def sq_init_params(box, qmax: float, qmin: float, ndim: int = 3) -> SqInit:
    """dq, nqmax, lmax per axis (with the 4-alignment quirk), nqmin and the reduced qmin.

    qedge is read uninitialised at sq.cuf:165-166; the shipped example outputs are
    consistent with qedge = qmin (no reduction), which is what is used here.
    ndim = 2 (sq.cuf:157-158, 185-192): dq and qmin from x and y only, lmax aligned to 16, lmaxz = 0.
    """
    box = np.asarray(box, F32)
    fk = np.array([F32(TWOPI32 / L) for L in box], dtype=F32)
    if ndim == 2:
        dq = F32(min(fk[0], fk[1]))
        nqmax = nint(F32(F32(qmax) / dq))
        lmax = [nint(F32(F32(qmin) / fk[d])) for d in range(2)]
        for d in range(2):
            if lmax[d] % 16 != 0:
                lmax[d] = lmax[d] - 16 + lmax[d] % 16        # sq.cuf:186-187
        nqmin = min(lmax)
        qmin_eff = min(F32(fk[d] * F32(lmax[d])) for d in range(2))  # sq.cuf:191
        lmax = lmax + [0]
        if nqmin == 0:
            nqmin = 1
            lmax = [1, 1, 1]
        return SqInit(fk=fk, dq=float(dq), nqmax=int(nqmax), lmax=tuple(int(l) for l in lmax),
                      nqmin=int(nqmin), qmin_eff=float(qmin_eff))
    dq = F32(fk.min())
    nqmax = nint(F32(F32(qmax) / dq))
    lmax = [nint(F32(F32(qmin) / fk[d])) for d in range(3)]
    ndg = 4
    for d in range(3):
        if lmax[d] % ndg != 0:
            lmax[d] = lmax[d] - ndg + lmax[d] % ndg          # sq.cuf:176-178
    nqmin = min(lmax)
    qmin_eff = min(F32(fk[d] * F32(lmax[d])) for d in range(3))  # sq.cuf:193
    if nqmin == 0:
        nqmin = 1
        lmax = [1, 1, 1]
    return SqInit(fk=fk, dq=float(dq), nqmax=int(nqmax), lmax=tuple(int(l) for l in lmax),
                  nqmin=int(nqmin), qmin_eff=float(qmin_eff))


def reference_nq(si: SqInit, ndim: int = 3) -> np.ndarray:
    """n(Q) denominators exactly as sq_init counts them (sq.cuf:303-342), FP32 geometry.
    In 2D the loops run over 0..lmax inclusive (sq.cuf:313-325) and the default is 2."""
    nq = np.zeros(si.nqmax + 1, dtype=np.int64)
    if si.nqmin <= 1:
        nq[1:] = 2 if ndim == 2 else 3
        return nq
    fk = si.fk
    if ndim == 2:
        i = np.arange(si.lmax[0] + 1, dtype=np.int64)[:, None]
        j = np.arange(si.lmax[1] + 1, dtype=np.int64)[None, :]
        a = (i.astype(F32) * fk[0]).astype(F32)
        b = (j.astype(F32) * fk[1]).astype(F32)
        rr = np.sqrt(((a * a).astype(F32) + (b * b).astype(F32)).astype(F32)).astype(F32)
        mask = ((i + j) != 0) & (rr < F32(si.qmin_eff))
        ind = nint((rr[mask] / F32(si.dq)).astype(F32))
        indm = int(ind.max()) if ind.size else 0
        ok = ind <= si.nqmax
        np.add.at(nq, ind[ok], 1)
        nq[indm + 1:] = 2
        return nq
    lx, ly, lz = si.lmax
    i = np.arange(lx, dtype=np.int64)[:, None, None]
    j = np.arange(ly, dtype=np.int64)[None, :, None]
    k = np.arange(lz, dtype=np.int64)[None, None, :]
    a = (i.astype(F32) * fk[0]).astype(F32)
    b = (j.astype(F32) * fk[1]).astype(F32)
    c = (k.astype(F32) * fk[2]).astype(F32)
    s = ((a * a).astype(F32) + (b * b).astype(F32)).astype(F32)
    s = (s + (c * c).astype(F32)).astype(F32)
    rr = np.sqrt(s).astype(F32)
    mask = ((i + j + k) != 0) & (rr < F32(si.qmin_eff))
    ind = nint((rr[mask] / F32(si.dq)).astype(F32))
    indm = int(ind.max()) if ind.size else 0
    ok = ind <= si.nqmax
    np.add.at(nq, ind[ok], 1)
    nq[indm + 1:] = 3
    return nq


def _fma32(a, b, c):
    """FP32 fused multiply-add (single rounding), via an exact FP64 product."""
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(F32)


def reference_kset(box, qmax: float, qmin: float, ndim: int = 3) -> KSet:
    """The vectors the reference's kernels sum, with their bins (reference mode).

    sqfnD (sq.cuf:523-591): every (kx,ky,kz) >= 0 of the launch grid with
    0 < q2 <= qmin^2, q2 = kf1^2 + kf2^2 + kf3^2 in FP32 as the GPU contracts it
    (fma(kf3,kf3, fma(kf2,kf2, kf1*kf1))), bin int(sqrt(q2)/dq + 0.501).
    sqfact (sq.cuf:372-454): (k,0,0), (0,k,0), (0,0,k) for k from nqmin+1 (or 1) to nqmax,
    each binned at k.  Denominators: reference_nq.
    """
    si = sq_init_params(box, qmax, qmin, ndim)
    vecs, bins = [], []
    if si.nqmin > 1:
        fk = si.fk
        if ndim == 2:  # launch grid (lmax/16+1) x 16 per axis, one z thread (sq.cuf:183-189)
            ext = [(si.lmax[0] // 16 + 1) * 16, (si.lmax[1] // 16 + 1) * 16, 1]
        else:
            ext = [(l // 4 + 1) * 4 for l in si.lmax]  # launch grid (lmax/4+1) blocks of 4
        kx = np.arange(ext[0])[:, None, None]
        ky = np.arange(ext[1])[None, :, None]
        kz = np.arange(ext[2])[None, None, :]
        kf1 = (kx.astype(F32) * fk[0]).astype(F32)
        kf2 = (ky.astype(F32) * fk[1]).astype(F32)
        kf3 = (kz.astype(F32) * fk[2]).astype(F32)
        q2 = _fma32(kf3, kf3, _fma32(kf2, kf2, (kf1 * kf1).astype(F32)))
        qmin2 = F32(F32(si.qmin_eff) * F32(si.qmin_eff))
        mask = (q2 > 0) & (q2.astype(np.float64) <= np.float64(qmin2))
        idx = np.nonzero(mask)
        q = np.sqrt(q2[idx].astype(np.float64)).astype(F32)
        ind = np.floor((q / F32(si.dq)).astype(F32) + F32(0.501)).astype(np.int64)
        keep = ind <= si.nqmax
        v = np.stack([idx[0][keep], idx[1][keep], idx[2][keep]], axis=1)
        vecs.append(v)
        bins.append(ind[keep])
        min_pts = si.nqmin + 1
    else:
        min_pts = 1
    ks = np.arange(min_pts, si.nqmax + 1, dtype=np.int64)
    if ks.size:
        z = np.zeros_like(ks)
        for ax in range(ndim):  # sqfact2 in 2D: (k,0) and (0,k) (sq.cuf:456-521)
            cols = [z, z, z]
            cols[ax] = ks
            vecs.append(np.stack(cols, axis=1))
            bins.append(ks)
    nd = vecs[0].shape[0] if si.nqmin > 1 else 0
    V = np.concatenate(vecs).astype(np.int32) if vecs else np.zeros((0, 3), np.int32)
    B = np.concatenate(bins).astype(np.int32) if bins else np.zeros(0, np.int32)
    dense = np.zeros(V.shape[0], np.uint8)
    dense[:nd] = 1  # 2D: tensor tiles only in the planar tile form (planar_tiles)
    return KSet(mode="ref", dq=si.dq, nqmax=si.nqmax, vectors=V, bins=B,
                weights=np.ones(V.shape[0]), dense=dense, nq=reference_nq(si, ndim),
                qmin_eff=si.qmin_eff, lmax=si.lmax, nqmin=si.nqmin)


def _half_space(v: np.ndarray) -> np.ndarray:
    """True for the representative of each +-n pair: nz>0, or nz=0 & ny>0, or nz=ny=0 & nx>0."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    return (z > 0) | ((z == 0) & ((y > 0) | ((y == 0) & (x > 0))))


def _sphere(box, qcut: float, strict: bool) -> np.ndarray:
    """All nonzero lattice n with |q| (FP64) < or <= qcut."""
    fk = 2.0 * np.pi / np.asarray(box, np.float64)
    m = [int(np.floor(qcut / fk[d])) + 1 for d in range(3)]
    out = []
    ys = np.arange(-m[1], m[1] + 1)
    zs = np.arange(-m[2], m[2] + 1)
    Y, Z = np.meshgrid(ys, zs, indexing="ij")
    Y = Y.ravel()
    Z = Z.ravel()
    yz2 = (Y * fk[1]) ** 2 + (Z * fk[2]) ** 2
    for x in range(-m[0], m[0] + 1):
        q2 = (x * fk[0]) ** 2 + yz2
        sel = (q2 < qcut * qcut) if strict else (q2 <= qcut * qcut)
        sel &= ~((x == 0) & (Y == 0) & (Z == 0))
        if sel.any():
            out.append(np.stack([np.full(sel.sum(), x), Y[sel], Z[sel]], axis=1))
    return np.concatenate(out).astype(np.int32) if out else np.zeros((0, 3), np.int32)


def _bin_of(v: np.ndarray, box, dq: float) -> np.ndarray:
    fk = 2.0 * np.pi / np.asarray(box, np.float64)
    q = np.sqrt(((v * fk[None, :]) ** 2).sum(axis=1))
    return np.floor(q / dq + 0.5).astype(np.int64)


def full_kset(box, qmax: float, qmin: Optional[float] = None, above: str = "axes",
              per_shell: int = 200, seed: int = 0) -> KSet:
    """Corrected-mode k-sets with FP64 geometry and exact denominators.

    Complete shells: every lattice vector of every bin b with (b+0.5)*dq <= qmin
    (qmin=None or qmin >= qmax: all bins up to nqmax), evaluated as +-n pairs (weight 2).
    Bins above: ``axes`` = +-(k,0,0), +-(0,k,0), +-(0,0,k) vectors of the bin;
    ``sampled`` = ``per_shell`` lattice vectors drawn uniformly without replacement
    from the bin's shell (seeded), weight 1; ``none`` = no vectors.
    nq[b] = sum of weights in bin b.
    """
    box = np.asarray(box, F32)
    si = sq_init_params(box, qmax, qmax if qmin is None else qmin)
    dq = si.dq
    nqmax = si.nqmax
    qcut_full = qmax if qmin is None else min(qmin, qmax)
    bfull = int(np.floor(qcut_full / dq - 0.5)) if qmin is not None and qmin < qmax else nqmax
    bfull = max(0, min(bfull, nqmax))
    vecs, bins, w, dense = [], [], [], []
    if bfull >= 1:
        sph = _sphere(box, (bfull + 0.5) * dq, strict=True)
        b = _bin_of(sph, box, dq)
        keep = (b >= 1) & (b <= bfull) & _half_space(sph)
        vecs.append(sph[keep])
        bins.append(b[keep])
        w.append(np.full(int(keep.sum()), 2.0))
        dense.append(np.ones(int(keep.sum()), np.uint8))
    if bfull < nqmax and above != "none":
        if above == "axes":
            fk = 2.0 * np.pi / np.asarray(box, np.float64)
            for ax in range(3):
                kmax = int(np.floor((nqmax + 0.5) * dq / fk[ax])) + 1
                ks = np.arange(1, kmax + 1)
                v = np.zeros((ks.size, 3), np.int32)
                v[:, ax] = ks
                b = _bin_of(v, box, dq)
                keep = (b > bfull) & (b <= nqmax)
                vecs.append(v[keep])
                bins.append(b[keep])
                w.append(np.full(int(keep.sum()), 2.0))
                dense.append(np.zeros(int(keep.sum()), np.uint8))
        elif above == "sampled":
            rng = np.random.default_rng([seed, 0x5c])
            shells = _shell_points(box, dq, bfull + 1, nqmax)
            for b in range(bfull + 1, nqmax + 1):
                pts = shells.get(b)
                if pts is None or pts.shape[0] == 0:
                    continue
                k = min(per_shell, pts.shape[0])
                pick = np.sort(rng.choice(pts.shape[0], size=k, replace=False))
                vecs.append(pts[pick])
                bins.append(np.full(k, b))
                w.append(np.ones(k))
                dense.append(np.zeros(k, np.uint8))
        else:
            raise ValueError(f"unknown above-qmin sampling {above!r}")
    V = np.concatenate(vecs).astype(np.int32) if vecs else np.zeros((0, 3), np.int32)
    B = np.concatenate(bins).astype(np.int32) if bins else np.zeros(0, np.int32)
    W = np.concatenate(w) if w else np.zeros(0)
    D = np.concatenate(dense) if dense else np.zeros(0, np.uint8)
    nq = np.zeros(nqmax + 1, np.int64)
    np.add.at(nq, B, W.astype(np.int64))
    mode = "full" if bfull >= nqmax else f"full+{above}"
    return KSet(mode=mode, dq=dq, nqmax=nqmax, vectors=V, bins=B, weights=W, dense=D, nq=nq,
                qmin_eff=float(qcut_full), lmax=si.lmax, nqmin=bfull)


def _shell_points(box, dq: float, b0: int, b1: int) -> dict:
    """Lattice points of bins b0..b1 (full sphere), keyed by bin."""
    fk = 2.0 * np.pi / np.asarray(box, np.float64)
    qhi = (b1 + 0.5) * dq
    qlo = (b0 - 0.5) * dq
    m = [int(np.floor(qhi / fk[d])) + 1 for d in range(3)]
    ys = np.arange(-m[1], m[1] + 1)
    zs = np.arange(-m[2], m[2] + 1)
    Y, Z = np.meshgrid(ys, zs, indexing="ij")
    Y = Y.ravel().astype(np.int32)
    Z = Z.ravel().astype(np.int32)
    yz2 = (Y * fk[1]) ** 2 + (Z * fk[2]) ** 2
    chunks = {}
    for x in range(-m[0], m[0] + 1):
        q2 = (x * fk[0]) ** 2 + yz2
        sel = (q2 >= (qlo * 0.999) ** 2) & (q2 < (qhi * 1.001) ** 2)
        if not sel.any():
            continue
        v = np.stack([np.full(int(sel.sum()), x, np.int32), Y[sel], Z[sel]], axis=1)
        b = _bin_of(v, box, dq)
        ok = (b >= b0) & (b <= b1)
        for bb in np.unique(b[ok]):
            chunks.setdefault(int(bb), []).append(v[ok & (b == bb)])
    return {k: np.concatenate(v) for k, v in chunks.items()}


def make_kset(mode: str, box, qmax: float, qmin: Optional[float] = None, seed: int = 0,
              per_shell: int = 200, ndim: int = 3) -> KSet:
    """Named k-set modes: ``ref`` (reference octant + axes, reference n(Q)),
    ``full`` (every vector up to qmax), ``full+axes`` and ``full+sampled``
    (complete shells below qmin, axis or random lattice vectors per shell above).
    Two-dimensional frames (ndim = 2) take ``ref`` only."""
    if ndim == 2:
        if mode != "ref":
            raise ValueError(f"k-set mode {mode!r}: two-dimensional frames support 'ref' only")
        return reference_kset(box, qmax, qmax if qmin is None else qmin, ndim=2)
    if mode == "ref":
        return reference_kset(box, qmax, qmax if qmin is None else qmin)
    if mode == "full":
        return full_kset(box, qmax, None)
    if mode == "full+axes":
        return full_kset(box, qmax, qmin, above="axes")
    if mode == "full+sampled":
        return full_kset(box, qmax, qmin, above="sampled", per_shell=per_shell, seed=seed)
    raise ValueError(f"unknown k-set mode {mode!r}")


def linear_kset(box, k_min: float, k_max: float, nbins: int) -> KSet:
    """Every lattice vector with k_min <= |k| < k_max in nbins linear bins of (k_max-k_min)/nbins.

    The binning of the freud StaticStructureFactorDirect used by the reference's
    tools/fast_sq_freud_netcdf.py (bins=60, k_min=2 pi / max(L), k_max=0.5).  Vectors are
    evaluated as +-k pairs (weight 2); nq[b] = number of vectors in bin b.  ``dq`` holds the
    bin width and the bin centres are k_min + (b + 1/2) dq.
    """
    box = np.asarray(box, F32)
    sph = _sphere(box, k_max, strict=True)
    fk = 2.0 * np.pi / np.asarray(box, np.float64)
    q = np.sqrt(((sph * fk[None, :]) ** 2).sum(axis=1))
    keep = (q >= k_min) & _half_space(sph)
    v = sph[keep]
    dk = (k_max - k_min) / nbins
    b = np.floor((q[keep] - k_min) / dk).astype(np.int64)
    b = np.clip(b, 0, nbins - 1)
    w = np.full(v.shape[0], 2.0)
    nq = np.zeros(nbins, np.int64)
    np.add.at(nq, b, 2)
    return KSet(mode="linear", dq=float(dk), nqmax=nbins - 1, vectors=v.astype(np.int32), bins=b.astype(np.int32),
                weights=w, dense=np.zeros(v.shape[0], np.uint8), nq=nq, qmin_eff=float(k_min))


# ---------------------------------------------------------------------------
# S(Q, w) vectors (sq_init, src/modules/sq.cuf:239-297; FqtnD, src/modules/dynamics.cuf:444-471)
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class SqwSet:
    """Lattice vectors of the qw shells, the shell each one is accumulated into, and nw per shell."""
    qw: np.ndarray        # (nqw,) FP32 shell centres
    dq: float             # FP32 shell width
    vectors: np.ndarray   # (nvec, 3) int32, octant i, j, k >= 0
    bins: np.ndarray      # (nvec,) int32 shell index 0..nqw-1 (FqtnD's search)
    nw: np.ndarray        # (nqw,) int64 vectors per shell (sq_init's count)

    @property
    def nvec(self) -> int:
        return int(self.vectors.shape[0])


def _first_shell(q: np.ndarray, qw: np.ndarray, half: np.float32) -> np.ndarray:
    """Per element, the first l with qw(l) - dq/2 < q < qw(l) + dq/2 (bounds in FP32, q compared in
    its own precision), or -1."""
    out = np.full(q.shape, -1, np.int64)
    for l in range(qw.size - 1, -1, -1):  # last to first: the first match wins
        lo, hi = F32(qw[l] - half), F32(qw[l] + half)
        hit = (q > q.dtype.type(lo)) & (q < q.dtype.type(hi))
        out[hit] = l
    return out


def sqw_kset(box, qw: Sequence[float], dq: float, ndim: int = 3) -> SqwSet:
    """The S(Q, w) vector set: lattice vectors with 0 <= i <= nint(qmax/fk_x) (and likewise for j,
    k), not all zero, whose |k| lies inside a shell qw(l) +- dq/2.  nw counts them per shell with
    sq_init's FP32 |k| = sqrt((i fk_x)^2 + (j fk_y)^2 + (k fk_z)^2); the shell a vector is added to
    is FqtnD's: the same FP32 sum of squares, square root in FP64.  The storing loop of sq_init is
    the one followed (its counting loop takes k = 0 only and allocates too few rows for 3D)."""
    box = np.asarray(box, F32)
    qw32 = np.asarray(qw, F32)
    if qw32.size == 0:
        raise ValueError("qw: no shells")
    dq32 = F32(dq)
    half = F32(dq32 / F32(2))
    fk = np.array([F32(TWOPI32 / L) for L in box], dtype=F32)
    qmm = F32(qw32.max())
    lim = [nint(F32(qmm / fk[d])) for d in range(3)]
    if ndim == 2:
        lim[2] = 0  # kmaxz = 0 (sq.cuf:273-277)
    i, j, k = np.meshgrid(np.arange(lim[0] + 1), np.arange(lim[1] + 1), np.arange(lim[2] + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    keep = (i + j + k) != 0
    i, j, k = i[keep], j[keep], k[keep]
    a = (i.astype(F32) * fk[0]).astype(F32)
    b = (j.astype(F32) * fk[1]).astype(F32)
    c = (k.astype(F32) * fk[2]).astype(F32)
    s2 = (((a * a).astype(F32) + (b * b).astype(F32)).astype(F32) + (c * c).astype(F32)).astype(F32)
    l_init = _first_shell(np.sqrt(s2).astype(F32), qw32, half)
    nw = np.bincount(l_init[l_init >= 0], minlength=qw32.size).astype(np.int64)
    l_fqt = _first_shell(np.sqrt(s2.astype(np.float64)), qw32, half)
    # FqtnD finding no shell for a stored vector would write past its arrays; such vectors are dropped
    sel = (l_init >= 0) & (l_fqt >= 0)
    v = np.stack([i[sel], j[sel], k[sel]], axis=1).astype(np.int32)
    return SqwSet(qw=qw32, dq=float(dq32), vectors=v, bins=l_fqt[sel].astype(np.int32), nw=nw)


def slab_kset(box, qmax: float, qmin: float) -> KSet:
    """The vectors of the slab S(Q) (twoDstruc_3D; SQcalc, sq.cuf:73-85): sq_init's 2D geometry
    (dq, lmax, nqmin, n(Q) as for ndim = 2).  sqf3xy (sq.cuf:594-674): every (kx, ky, 0) of the
    launch grid with 0 < q2 <= qmin^2, q2 = kf1^2 + kf2^2 as the GPU contracts it, bin nint(q/dq)
    (not sqfnD's int(q/dq + 0.501)); sqf2xy (676-771): (k, 0, 0) and (0, k, 0) for k from nqmin + 1
    to nqmax, binned at k.  With nqmin <= 1 only sqf2xy runs, still from nqmin + 1 (sq.cuf:113-116): k = 1 is
    skipped when nqmin = 1; the 16-alignment of lmax can make nqmin negative, and then k starts at 1."""
    si = sq_init_params(box, qmax, qmin, 2)
    vecs, bins = [], []
    if si.nqmin > 1:
        fk = si.fk
        ext = [(si.lmax[0] // 16 + 1) * 16, (si.lmax[1] // 16 + 1) * 16]
        kx = np.arange(ext[0])[:, None]
        ky = np.arange(ext[1])[None, :]
        kf1 = (kx.astype(F32) * fk[0]).astype(F32)
        kf2 = (ky.astype(F32) * fk[1]).astype(F32)
        q2 = _fma32(kf2, kf2, (kf1 * kf1).astype(F32))
        qmin2 = F32(F32(si.qmin_eff) * F32(si.qmin_eff))
        mask = (q2 > 0) & (q2.astype(np.float64) <= np.float64(qmin2))
        idx = np.nonzero(mask)
        q = np.sqrt(q2[idx].astype(np.float64)).astype(F32)
        ind = nint((q / F32(si.dq)).astype(F32))
        ind = np.atleast_1d(ind)
        keep = ind <= si.nqmax
        vecs.append(np.stack([idx[0][keep], idx[1][keep], np.zeros(int(keep.sum()), np.int64)], axis=1))
        bins.append(ind[keep])
    # sqf2xy's k starts at 1 (its thread index) or at minPts = nqmin + 1, whichever is larger
    ks = np.arange(max(1, si.nqmin + 1), si.nqmax + 1, dtype=np.int64)
    if ks.size:
        z = np.zeros_like(ks)
        vecs.append(np.stack([ks, z, z], axis=1))
        vecs.append(np.stack([z, ks, z], axis=1))
        bins += [ks, ks]
    V = np.concatenate(vecs).astype(np.int32) if vecs else np.zeros((0, 3), np.int32)
    B = np.concatenate(bins).astype(np.int32) if bins else np.zeros(0, np.int32)
    return KSet(mode="slab", dq=si.dq, nqmax=si.nqmax, vectors=V, bins=B, weights=np.ones(V.shape[0]),
                dense=np.zeros(V.shape[0], np.uint8), nq=reference_nq(si, 2), qmin_eff=si.qmin_eff,
                lmax=si.lmax, nqmin=si.nqmin)


def slab_of(z: np.ndarray, zslice: Sequence[float], zgrid: float) -> np.ndarray:
    """Slice of each z (0-based), -1 outside: the first slice centre nearest to z (minloc of
    |zslice - z|), kept if |zslice - z| <= zgrid/2, in FP32 (rdf.cuf:694-699, sq.cuf:633-635)."""
    z = np.asarray(z, F32)
    zs = np.asarray(zslice, F32)
    d = np.abs((zs[None, :] - z[:, None]).astype(F32))
    s = np.argmin(d, axis=1)  # first minimum, as minloc
    ok = d[np.arange(z.shape[0]), s] <= F32(F32(zgrid) / F32(2.0))
    return np.where(ok, s, -1).astype(np.int64)


def planar_tiles(ks: KSet, mul: int = 8) -> KSet:
    """The vectors of a two-dimensional k-set in the planar tile form: (nx, ny, 0) becomes
    (nx, ny mod mul, ny div mul), to be evaluated with the third phase taken as mul times the second
    (trj_sq_plan_set_z_from_y), which gives it exactly the phase of (nx, ny).  Tensor tiles of 16 nx x
    8 ny rows then fill with in-plane vectors (ny mod 8 over the rows, ny div 8 over the columns).
    Bins, weights and n(Q) are unchanged."""
    v = ks.vectors.astype(np.int64)
    if np.any(v[:, 2] != 0) or np.any(v[:, 1] < 0):
        raise ValueError("planar tile form: vectors must be (nx, ny >= 0, 0)")
    t = np.stack([v[:, 0], v[:, 1] % mul, v[:, 1] // mul], axis=1).astype(np.int32)
    return dataclasses.replace(ks, vectors=t)
