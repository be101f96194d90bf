"""CPU restatement of the reference's multiple-origin time correlations.  TEST INFRASTRUCTURE ONLY.

Only tests/ import this module, as the checker.  It transcribes, loop for loop:
* rtcorr's bookkeeping (src/modules/dynamics.cuf:157-276): buffer origins (i-1)*jump+1, itlimit set
  at the second frame, origin shift and accumulation of a buffer when iconf - origin = itlimit;
* FqtnD (dynamics.cuf:421-507): for every buffer past its origin, both densities are recomputed from
  the stored origin positions and the current ones, rho = sum_a bsc_a sum_j e^{i k.r_j}, and
  F += Re(rho(t0) conj(rho(t))), Fs += sum_j cos(k.(r_j(t) - r_j(t0))), per qw shell;
* rtcal (dynamics.cuf:510-547): per buffer, coordinates unwrapped toward the current frame
  (rt = r + L nint((rt - r)/L), FP32) and sum_j |rt_j - r0_j|^2 / N;
* the normalisation of print_rtcor (dynamics.cuf:286-315).
Phases are exact in FP64 (k.r = 2 pi n.s with s = x/L reduced mod 1), the reference's are FP32; the
MSD keeps the reference's FP32 per-atom arithmetic with FP64 sums.  Lag rows past ndyn are not
accumulated.  Besides the results, ``fkt_scale`` bounds the magnitude behind each coherent entry:
the sum over its terms of |rho(t0)| + |rho(t)|, normalised like F.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32


def _roundf(x):
    x = np.asarray(x, np.float64)
    return np.trunc(x + np.copysign(0.5, x)).astype(F32)


def _nint(x) -> int:
    x = float(x)
    return int(np.floor(x + 0.5)) if x >= 0 else -int(np.floor(-x + 0.5))


def _phases(pos, box, vectors):
    s = pos.astype(np.float64) / np.asarray(box, F32).astype(np.float64)
    s = s - np.floor(s)
    t = vectors.astype(np.float64) @ s.T          # (nvec, n)
    return 2.0 * np.pi * (t - np.round(t))


def dynamics(frames, species, box, bsc, vectors, bins, nbins, nw, nbuffer, jump, tlimit, times):
    """frames: list of (n, 3) FP32 folded positions in packed order; species: (n,) 0-based;
    times: per frame (FP32).  Returns the print_rtcor arrays (before the transform)."""
    nconf = len(frames)
    n = frames[0].shape[0]
    ndyn = nconf - (nbuffer - 1) * jump
    L = np.asarray(box, F32)
    w = np.asarray(bsc, np.float64)[species]
    t = np.zeros(ndyn, F32)
    origin = np.zeros(nbuffer, np.int64)
    itlimit = nconf
    tlimit = F32(tlimit)
    fkt_b = np.zeros((nbuffer, ndyn, nbins))
    fskt_b = np.zeros((nbuffer, ndyn, nbins))
    scl_b = np.zeros((nbuffer, ndyn, nbins))
    r2t_b = np.zeros((nbuffer, ndyn))
    fkt = np.zeros((ndyn, nbins))
    fskt = np.zeros((ndyn, nbins))
    scl = np.zeros((ndyn, nbins))
    r2t = np.zeros(ndyn)
    r0 = [None] * nbuffer
    rt = [None] * nbuffer
    count_org = 0
    for iconf in range(1, nconf + 1):
        pos = frames[iconf - 1]
        if iconf <= ndyn:
            t[iconf - 1] = times[iconf - 1]
        if iconf == 1:
            for i in range(nbuffer):
                origin[i] = i * jump + 1
            itlimit = nconf
        elif iconf == 2:
            dt = F32(t[1] - t[0])
            if tlimit < 0:
                itlimit = nconf - (nbuffer - 1) * jump
                tlimit = F32(F32(itlimit) * dt)
            else:
                itlimit = _nint(F32(tlimit / dt))
        for i in range(nbuffer):
            if iconf == origin[i]:
                r0[i] = pos.copy()
        ph_t = _phases(pos, box, vectors)
        for i in range(nbuffer):
            iorg = origin[i]
            indx = iconf - iorg + 1
            if iconf == iorg:
                rt[i] = pos.copy()
            if iconf >= iorg and indx <= ndyn:
                m = _roundf(((rt[i] - pos).astype(F32) / L).astype(F32))
                rt[i] = (pos + (L * m).astype(F32)).astype(F32)
                d = (rt[i] - r0[i]).astype(F32)
                d2 = (((d[:, 0] * d[:, 0]).astype(F32) + (d[:, 1] * d[:, 1]).astype(F32)).astype(F32)
                      + (d[:, 2] * d[:, 2]).astype(F32)).astype(F32)
                r2t_b[i, indx - 1] += d2.astype(np.float64).sum() / n
            if iconf >= iorg and 1 <= indx <= ndyn:
                ph0 = _phases(r0[i], box, vectors)
                rho0 = (w[None, :] * np.exp(1j * ph0)).sum(axis=1)
                rhot = (w[None, :] * np.exp(1j * ph_t)).sum(axis=1)
                coh = (rho0 * np.conj(rhot)).real
                slf = np.cos(ph_t - ph0).sum(axis=1)
                np.add.at(fkt_b[i, indx - 1], bins, coh)
                np.add.at(fskt_b[i, indx - 1], bins, slf)
                np.add.at(scl_b[i, indx - 1], bins, np.abs(rho0) + np.abs(rhot))
        for i in range(nbuffer):
            if iconf - origin[i] == itlimit:
                origin[i] = iconf + 1
                r2t += r2t_b[i]
                fkt += fkt_b[i]
                fskt += fskt_b[i]
                scl += scl_b[i]
                r2t_b[i] = 0
                fkt_b[i] = 0
                fskt_b[i] = 0
                scl_b[i] = 0
                count_org += 1
    with np.errstate(divide="ignore", invalid="ignore"):
        den = n * count_org * np.asarray(nw, np.float64)
        return {"t": (t - t[0]).astype(F32), "r2t": r2t / count_org, "fkt": fkt / den, "fskt": fskt / den,
                "fkt_scale": scl / den, "itlimit": itlimit, "count_org": count_org, "ndyn": ndyn}
