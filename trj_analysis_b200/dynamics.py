"""Time correlations over multiple origins: F(Q,t), Fs(Q,t), the mean-squared displacement C_r(t)
and their spectra S(Q,w), Ss(Q,w).

Mirrors the reference's mod_dyn (src/modules/dynamics.cuf): ``dyn_init`` (88-135) sizes the buffers,
``rtcorr`` (157-276) is called once per frame and keeps the bookkeeping of the time origins, and
``print_rtcor`` (278-393) normalises, transforms (``fftw1d``, src/core/fftwlib.f90:50-120) and writes
``dyn.dat``, ``fkt.dat``, ``fskt.dat`` and ``sqw.dat``.  The per-frame sums run in libtrj_sm100.so
(``trj_dyn_accumulate``); the origin bookkeeping, the normalisation and the transform are host work,
as in the reference.

Bookkeeping (rtcorr): buffer i starts at frame (i-1)*jump + 1; frame iconf adds lag row
iconf - origin(i) to every buffer whose origin has been reached; when iconf - origin(i) = itlimit the
buffer is added to the totals, cleared, and restarts at iconf + 1 (count_org counts these).  itlimit
is set at the second frame: ndyn = Nconf - (nbuffer-1)*jump when tlimit < 0, else nint(tlimit/dt).
Lag rows beyond ndyn are not accumulated (FqtnD writes them into the next buffer's first row).

Velocity and stress correlations (C_v(t), Z(w), viscosity) need velocities and stresses in the
trajectory and are not part of this build.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import refsem, writers
from .refsem import F32


@dataclasses.dataclass
class DynConfig:
    """/INPUT_DYN/ and /INPUT_SQW/ (src/io/input.f90:73-74) plus the time step of the frames."""
    nbuffer: int = 2
    jump: int = 1
    tlimit: float = -1.0
    tmax: float = -1.0
    qw: Sequence[float] = (1.0,)
    tstep: float = 1.0       # t = time * tstep (frames without a time: t = (iconf-1) * tstep)


def fftw1d(fin: np.ndarray, dtin: float, tmax: float):
    """fftw1d (fftwlib.f90:50-86) with fftw1 (88-112) and window (114-119), forward transform:
    zero-pad to n = 2^(nu+1), nu = int(log(nin)/log(2) + 0.54); multiply by the window
    0.5 (1 - tanh(t - tmax)); halve the first point; DFT with sign -1; scale the first point by dt and
    points 2..n/2 by dt/2 after adding their mirror n-i+2.  Returns (fout, w, tmax) with fout the real
    part of the first nin points, w(i) = (i-1) 2 pi/(n dt), and tmax replaced by n dt when it was 0."""
    fin = np.asarray(fin, F32)
    nin = fin.shape[0]
    nu = int(F32(F32(np.log(F32(nin))) / F32(np.log(F32(2.0)))) + F32(0.540))
    n = 2 ** (nu + 1)
    dt = F32(dtin)
    pi = F32(3.141592653589793)
    dq = F32(F32(F32(2) * pi) / F32(F32(n) * dt))
    inp = np.zeros(n, np.complex128)
    inp[:nin] = fin.astype(np.float64)
    tx = (np.arange(n, dtype=np.float64).astype(F32) * dt).astype(F32)
    tmax = F32(tmax)
    if abs(float(tmax)) < 1.0e-6:
        tmax = F32(F32(n) * dt)
    alpha = F32(1.0)
    win = (F32(0.5) * (F32(1) - np.tanh((alpha * (tx - tmax).astype(F32)).astype(F32)).astype(F32))).astype(F32)
    inp = inp * win.astype(np.float64)
    dfact = float(dt)
    inp[0] = 0.5 * inp[0]
    out = np.fft.fft(inp)
    out[0] = out[0] * dfact
    i = np.arange(1, n // 2)
    out[i] = (out[i] + out[n - i]) * dfact / 2
    w = (np.arange(nin, dtype=np.float64).astype(F32) * dq).astype(F32)
    return out[:nin].real.astype(F32), w, tmax


class OriginSchedule:
    """The host bookkeeping of rtcorr (dynamics.cuf:164-186, 239-269) for nbuffer time origins."""

    def __init__(self, nconf: int, cfg: DynConfig):
        if cfg.nbuffer > 1000:
            raise ValueError("nbuffer > 1000")  # nbmax (dynamics.cuf:71, 92-95)
        self.cfg = cfg
        self.nconf = int(nconf)
        self.ndyn = self.nconf - (cfg.nbuffer - 1) * cfg.jump
        if self.ndyn < 10:
            raise ValueError("length of dynamics too short: reduce the number of buffers")  # dynamics.cuf:99-102
        self.t = np.zeros(self.ndyn, np.float32)
        self.origin = np.zeros(cfg.nbuffer, np.int64)
        self.itlimit = self.nconf
        self.tlimit = F32(cfg.tlimit)
        self.tmax = F32(cfg.tmax)
        self.count_org = 0

    def frame_time(self, iconf: int, time: Optional[float]) -> np.float32:
        base = F32(iconf - 1) if time is None else F32(time)
        return F32(base * F32(self.cfg.tstep))

    def schedule(self, iconf: int, time: Optional[float] = None):
        """Before the kernels: times, origins, itlimit; returns (lag per buffer, -1 = none; origin flags)."""
        cfg = self.cfg
        if iconf <= self.ndyn:
            self.t[iconf - 1] = self.frame_time(iconf, time)
        if iconf == 1:
            self.origin[:] = np.arange(cfg.nbuffer) * cfg.jump + 1
            self.itlimit = self.nconf
        elif iconf == 2:
            dt = F32(self.t[1] - self.t[0])
            if self.tlimit < 0:
                self.itlimit = self.nconf - (cfg.nbuffer - 1) * cfg.jump
                self.tlimit = F32(F32(self.itlimit) * dt)
            else:
                self.itlimit = refsem.nint(F32(self.tlimit / dt))
            if self.itlimit > self.nconf:
                raise ValueError("tlimit longer than the trajectory")  # dynamics.cuf:179-182
            if self.tmax < 0:
                self.tmax = self.tlimit
        indx = iconf - self.origin + 1
        active = (iconf >= self.origin) & (indx >= 1) & (indx <= self.ndyn)
        lags = np.where(active, indx - 1, -1).astype(np.int32)
        origins = (active & (iconf == self.origin)).astype(np.uint8)
        return lags, origins

    def finish_frame(self, iconf: int) -> np.ndarray:
        """After the kernels: buffers whose time window is full restart at the next frame; returns them."""
        done = (iconf - self.origin) == self.itlimit
        self.origin[done] = iconf + 1
        self.count_org += int(done.sum())
        return done.astype(np.uint8)


class Dynamics:
    """Per-trajectory state of the F(Q,t)/Fs(Q,t)/MSD analysis on one device."""

    def __init__(self, ctx, nsp: int, n: int, nconf: int, cfg: DynConfig, box, bsc, dq: Optional[float] = None,
                 ndim: int = 3):
        from . import engine
        if cfg.nbuffer < 2:
            cfg = dataclasses.replace(cfg, nbuffer=2)  # input.f90:162-165
        self.cfg = cfg
        self.sched = OriginSchedule(nconf, cfg)
        self.ndyn = self.sched.ndyn
        if len(cfg.qw) == 0:  # C_r(t) only (run_dyn without run_sqw)
            self.sqw = refsem.SqwSet(qw=np.zeros(0, np.float32), dq=0.0, vectors=np.zeros((0, 3), np.int32),
                                     bins=np.zeros(0, np.int32), nw=np.zeros(0, np.int64))
        else:
            if dq is None:
                dq = refsem.sq_init_params(box, max(cfg.qw), max(cfg.qw), ndim).dq
            self.sqw = refsem.sqw_kset(box, cfg.qw, dq, ndim)
        self.n = int(n)
        self.plan = engine.DynPlan(ctx, nsp, n, cfg.nbuffer, self.ndyn, self.sqw, bsc)
        self.fkt, self.fskt, self.r2t = self.plan.new_totals()

    def rtcorr(self, iconf: int, packed, n: int, box, time: Optional[float] = None, stream=None) -> None:
        lags, origins = self.sched.schedule(iconf, time)
        self.plan.accumulate(packed, n, box, lags, origins, stream=stream)
        done = self.sched.finish_frame(iconf)
        if done.any():
            self.plan.flush(done, self.fkt, self.fskt, self.r2t, stream=stream)

    def results(self) -> Dict[str, np.ndarray]:
        """print_rtcor's arrays (dynamics.cuf:278-315): t from 0, C_r = r2t/count_org,
        F = fkt/(N count_org nw), Fs likewise, and their transforms."""
        sc = self.sched
        nq_ = self.sqw.qw.size
        t = (sc.t - sc.t[0]).astype(F32)
        with np.errstate(divide="ignore", invalid="ignore"):
            r2t = self.r2t.cpu().numpy() / sc.count_org
            den = self.n * sc.count_org * self.sqw.nw.astype(np.float64)
            fkt = self.fkt.cpu().numpy()[:, :nq_] / den[None, :]
            fskt = self.fskt.cpu().numpy()[:, :nq_] / den[None, :]
        dt = F32(t[1] - t[0]) if t.shape[0] > 1 else F32(1)
        nq = self.sqw.qw.size
        sqw = np.zeros((self.ndyn, nq), F32)
        ssqw = np.zeros((self.ndyn, nq), F32)
        tmax = sc.tmax
        w = np.zeros(self.ndyn, F32)
        for i in range(nq):  # fkt/fskt are single precision in the reference (dynamics.cuf:77)
            sqw[:, i], w, tmax = fftw1d(fkt[:, i].astype(F32), dt, tmax)
            ssqw[:, i], w, tmax = fftw1d(fskt[:, i].astype(F32), dt, tmax)
        return {"t": t, "r2t": r2t, "fkt": fkt, "fskt": fskt, "sqw": sqw, "ssqw": ssqw, "w": w,
                "itlimit": sc.itlimit, "count_org": sc.count_org, "qw": self.sqw.qw, "nw": self.sqw.nw}

    def print_rtcor(self, outdir: str = ".", units: str = "lj") -> List[str]:
        return writers.write_dynamics(outdir, self.results(), units)

    def close(self) -> None:
        self.plan.close()
