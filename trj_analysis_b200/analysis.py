"""Reference-facing operators for the g_ab(r) / S_ab(Q) path.

The reference drives this path through Fortran subroutines that share module
globals: ``RDF_init`` / ``RDFcomp`` / ``printrdf`` (src/modules/rdf.cuf:51,184;
src/core/log.f90:414) and ``sq_init`` / ``SQcalc`` / ``sq_transfer_gpu_cpu`` /
``printSQ`` (src/modules/sq.cuf:150,58,128; src/core/log.f90:317), called from
the frame loop of src/main/trj_analysis.f90:173-242 after ``select_ncdfinput``
(src/core/netcdf.f90:582).  :class:`Session` holds that state explicitly and
keeps the routine names; the arithmetic runs in libtrj_sm100.so.

Differences from the reference, by design:
* pair counts are exact uint64 (the reference sums FP32 copies of per-block int32
  histograms on the host, rdf.cuf:301-310, which loses exactness above 2^24);
* S(Q) sums are FP64 with a fixed reduction order (the reference adds FP32 atomics,
  sq.cuf:447,449,584);
* normalisations (printrdf, printSQ) are evaluated in FP64;
* histograms and S(Q) sums stay on the device across frames; nothing is copied
  back per frame.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np
import torch

from . import engine, refsem, writers
from .dynamics import DynConfig, Dynamics
from .frames import Frame
from .refsem import F32


@dataclasses.dataclass
class SlabConfig:
    """/INPUT_CONF/ zslice, zgrid (input.f90:72): slice centres along z and their width.  With a slab
    configuration and g(r) or S(Q) requested, the analysis is the reference's twoDstruc_3D one
    (input.f90:171-191): per-slice g_xy(r) and S_xy(Q) in the xy plane.  z is taken as the trajectory
    stores it (the confined direction is not folded)."""
    zslice: Sequence[float] = (0.0,)
    zgrid: float = 1.0


@dataclasses.dataclass
class Config:
    """The /INPUT/, /INPUT_SP/, /INPUT_RDF/ and /INPUT_SQ/ keys this path uses (input.f90:64-75)."""
    nsp: int = 1
    ndim: int = 3                  # 2: the z coordinate of the frames is discarded (netcdf.f90:649-651)
    sp_types_selected: Sequence[int] = (1,)
    run_rdf: bool = True
    run_sq: bool = True
    deltar: float = 0.02
    rcrdf: float = 0.0             # <= 0: half the smallest box edge
    nrandom: int = 0               # /INPUT_RDF/ nrandom: random points for the number fluctuations s2n(r)
    qmax: float = 10.0
    qmin: float = 3.0
    bsc: Optional[Sequence[float]] = None   # per sp_types_selected entry; default 1.0
    kset: str = "ref"              # ref | full | full+axes | full+sampled
    method: str = "split"          # split (tcgen05 split-BF16) | plain (FP32 direct sum)
    per_shell: int = 200
    seed: int = 0
    units: str = "lj"
    # Frames with charges: "atom" runs the charge-weighted kernels (any per-atom charges, as the
    # reference's ex_qc path); "species" requires every atom of a species to carry the same charge in
    # every frame and derives g_qq and S_qq from the species rows, with no extra device work.
    charge_mode: str = "atom"
    slab: Optional[SlabConfig] = None
    # F(Q,t), Fs(Q,t), MSD over multiple time origins (rtcorr; needs the trajectory's frame count)
    run_sqw: bool = False
    dyn: Optional["DynConfig"] = None

    def bsc_list(self) -> List[float]:
        return list(self.bsc) if self.bsc is not None else [1.0] * self.nsp


class Session:
    """Per-trajectory state of the g(r)/S(Q) path on one device."""

    def __init__(self, cfg: Config, device: int = 0, n_max: Optional[int] = None,
                 ctx: Optional[engine.Context] = None, stream: Optional[torch.cuda.Stream] = None,
                 nconf_total: Optional[int] = None):
        self.cfg = cfg
        self.nconf_total = nconf_total  # Nconf of the trajectory (dyn_init sizes its buffers from it)
        self.dyn = None
        self.ctx = ctx if ctx is not None else engine.Context(device)
        self.stream = stream
        self.n_max = n_max
        self.nconf = 0
        self.first = True
        self.species_lut = None
        self.ntype = None
        self.box = None
        self.volumen = None
        self.bsc_sp = None
        self.stage = None
        self.rdf = None
        self.sq = None
        self.hist = None
        self.edge = None
        self.sq_out = None
        self.kset = None
        self.n = 0
        self.ex_qc = None      # frames carry charges (set by the first frame, netcdf.f90:404-408)
        self.gqq = None        # FP64 [lsmax] charge-product histogram over avq2, summed over frames
        self.gi = self.g2i = None  # uint64 [lsmax+1] number-fluctuation sums (nrandom > 0)
        self.slab = None           # per-slice accumulators (SlabState) in the twoDstruc_3D analysis
        self._lut_dev = None       # type -> species table on the device (frames with only selected types)
        self._ntype_stale = False  # species counts of the last frame are on the device only
        self.charges = None    # charges of the last frame (FP32, selected atoms)
        self.species_q = None  # charge of each species (charge_mode "species")

    # ---- layout (select_ncdfinput) ------------------------------------------------
    def _species_of(self, types: np.ndarray) -> np.ndarray:
        if self.species_lut is None:
            sp, wtypes, perm = refsem.species_by_first_appearance(types, self.cfg.sp_types_selected)
            if len(wtypes) != self.cfg.nsp:
                raise ValueError(f"selected types {list(self.cfg.sp_types_selected)} not all in the frame "
                                 f"(found {wtypes})")
            lut = np.full(int(max(types.max(), max(self.cfg.sp_types_selected))) + 2, -1, np.int32)
            for s, t in enumerate(wtypes):
                lut[t] = s
            self.species_lut = lut
            b = self.cfg.bsc_list()
            self.bsc_sp = np.array([b[perm[s]] for s in range(self.cfg.nsp)], np.float32)
            self.wtypes = wtypes
        t = np.asarray(types)
        if t.max() >= self.species_lut.shape[0] or t.min() < 0:
            raise ValueError("frame holds a type id outside the first frame's range")
        return self.species_lut[t]

    def _fast_layout(self, frame: Frame) -> bool:
        """Frames after the first whose atoms are all of selected types (as the first frame's were) go to
        the device with their raw type column; the type-to-species table is applied there
        (trj_frame_pack_types), and a type that is not selected is reported by the device as bad data."""
        if self.first or self._lut_dev is None or self.cfg.ndim != 3 or frame.charges is not None or self.ex_qc:
            return False
        box = np.asarray(frame.box, np.float32)
        self.box = box
        self.volumen = refsem.volume(box)
        self.n = self.stage.upload_and_pack_types(frame.xyz, frame.types, box, self._lut_dev, stream=self.stream)
        self._ntype_stale = True
        return True

    def _refresh_ntype(self) -> None:
        if self._ntype_stale:
            self.ntype = self.stage.counts[:self.cfg.nsp].cpu().numpy().astype(np.int64)
            self._ntype_stale = False

    def select_ncdfinput(self, frame: Frame) -> None:
        """Species numbering, host->device copy, fold and species-contiguous order."""
        if self._fast_layout(frame):
            return
        species = self._species_of(frame.types)
        keep = species >= 0
        xyz = frame.xyz if keep.all() else frame.xyz[keep]
        species = species if keep.all() else species[keep]
        box = np.asarray(frame.box, np.float32)
        if self.cfg.ndim == 2:
            # two-dimensional frames: z discarded (netcdf.f90:649-651); packed with z = 0 in a unit z box
            xyz = np.array(xyz, np.float32, copy=True)
            xyz[:, 2] = 0.0
            box = np.array([box[0], box[1], 1.0], np.float32)
        elif self.cfg.ndim != 3:
            raise ValueError(f"ndim={self.cfg.ndim}: 2 or 3")
        if self.ex_qc is None:
            self.ex_qc = frame.charges is not None
        if self.ex_qc != (frame.charges is not None):
            raise ValueError("frames with and without charges in one trajectory")
        charges = None
        if self.ex_qc:
            q = np.asarray(frame.charges, np.float32)
            charges = q if keep.all() else q[keep]
            self.charges = charges
            if self.cfg.charge_mode == "species":
                self._check_species_charges(charges, species)
                charges = None  # nothing charge-weighted runs on the device
            elif self.cfg.charge_mode != "atom":
                raise ValueError(f"charge_mode {self.cfg.charge_mode!r}: 'atom' or 'species'")
        if self.stage is None:
            n_max = self.n_max or xyz.shape[0]
            self.stage = engine.FrameStage(self.ctx, n_max, self.cfg.nsp, charged=self.device_charges)
        self.box = box
        self.volumen = refsem.volume(self.box, self.cfg.ndim)
        self.ntype = np.bincount(species, minlength=self.cfg.nsp).astype(np.int64)
        self._ntype_stale = False
        self.n = self.stage.upload_and_pack(xyz, species, self.box, stream=self.stream, charges=charges)
        if self.first and keep.all() and self.cfg.ndim == 3 and not self.ex_qc and self.species_lut.size <= (1 << 20):
            self._lut_dev = torch.from_numpy(self.species_lut.astype(np.int32)).to(self.ctx.torch_device)

    @property
    def device_charges(self) -> bool:
        """The charge-weighted kernels run (frames with charges, charge_mode 'atom')."""
        return bool(self.ex_qc) and self.cfg.charge_mode == "atom"

    def _check_species_charges(self, q: np.ndarray, species: np.ndarray) -> None:
        """Every atom of a species carries the species' charge, the same in every frame, and the species
        counts do not change (so avq2 = sum_a N_a q_a^2 / N is the same in every frame)."""
        nsp = self.cfg.nsp
        vals, first = np.unique(species, return_index=True)
        qa = np.zeros(nsp, np.float32)
        qa[vals] = q[first]
        if not np.array_equal(q, qa[species]):
            raise ValueError("charge_mode 'species': atoms of one species carry different charges "
                             "(use charge_mode 'atom')")
        counts = np.bincount(species, minlength=nsp)
        if self.species_q is None:
            self.species_q, self._species_q_counts = qa, counts
        elif not (np.array_equal(qa, self.species_q) and np.array_equal(counts, self._species_q_counts)):
            raise ValueError("charge_mode 'species': species charges or counts change between frames "
                             "(use charge_mode 'atom')")

    # ---- g(r) -----------------------------------------------------------------------
    def RDF_init(self) -> None:
        c = self.cfg
        self.rdf = engine.RdfPlan(self.ctx, c.nsp, c.deltar, c.rcrdf, self.box, self.stage.n_max, ndim=c.ndim)
        self.hist = self.rdf.new_hist()
        self.edge = torch.zeros(4, dtype=torch.int64, device=self.ctx.torch_device)
        if self.device_charges:
            self.gqq = self.rdf.new_gqq()
        if self.cfg.nrandom > 0:
            self.gi, self.g2i = self.rdf.new_s2n()

    def RDFcomp(self) -> None:
        dq = self.device_charges
        self.rdf.accumulate(self.stage.packed, self.n, self.box, self.hist, self.edge, stream=self.stream,
                            qpacked=self.stage.qpacked if dq else None, gqq=self.gqq)
        if self.cfg.nrandom > 0 and self.n >= 2:  # s2D3_sh after rdf_sh (rdf.cuf:243-245)
            self.rdf.s2n(self.cfg.nrandom, self.gi, self.g2i, stream=self.stream)

    # ---- S(Q) -----------------------------------------------------------------------
    def sq_init(self) -> None:
        c = self.cfg
        self.kset = refsem.make_kset(c.kset, self.box, c.qmax, c.qmin, seed=c.seed, per_shell=c.per_shell, ndim=c.ndim)
        planar = c.ndim == 2 and c.method in ("split", "split_bf16x3")
        if planar:  # in-plane vectors as (nx, ny mod 8, ny div 8) so that they fill tensor tiles
            self.kset = refsem.planar_tiles(self.kset, 8)
        elif c.ndim == 2:
            self.kset = dataclasses.replace(self.kset, dense=np.zeros_like(self.kset.dense))
        self.sq = engine.SqPlan(self.ctx, c.nsp, self.kset, self.ntype, charged=self.device_charges)
        if planar:
            self.sq.set_z_from_y(8)
        self.sq_out = self.sq.new_out()

    def SQcalc(self) -> None:
        self.sq.accumulate(self.stage.packed, self.n, self.box, self.sq_out, engine.METHODS[self.cfg.method],
                           stream=self.stream, qpacked=self.stage.qpacked if self.device_charges else None)

    # ---- frame loop (trj_analysis.f90:173-242) ---------------------------------------
    def add_frame(self, frame: Frame) -> None:
        if self.cfg.slab is not None:
            self._add_slab_frame(frame)
            return
        self.select_ncdfinput(frame)
        if self.first:
            if self.cfg.run_rdf:
                self.RDF_init()
            if self.cfg.run_sq:
                self.sq_init()
            self.first = False
        if self.cfg.run_rdf:
            self.RDFcomp()
        if self.cfg.run_sq:
            self.SQcalc()
        if self.cfg.run_sqw:
            self.rtcorr(frame)
        self.nconf += 1

    # ---- slabs (twoDstruc_3D: rdfxy, sqf3xy/sqf2xy) -----------------------------------------
    def _add_slab_frame(self, frame: Frame) -> None:
        c = self.cfg
        if c.ndim != 3:
            raise ValueError("slab analysis needs three-dimensional frames (input.f90:172-175)")
        if c.charge_mode != "atom" or frame.charges is not None:
            raise ValueError("slab analysis with charges (gqqxy, sqfqxy) is not part of this build")
        species = self._species_of(frame.types)
        keep = species >= 0
        xyz = np.asarray(frame.xyz if keep.all() else frame.xyz[keep], np.float32)
        species = species if keep.all() else species[keep]
        self.box = np.asarray(frame.box, np.float32)
        self.volumen = refsem.volume(self.box)
        self.ntype = np.bincount(species, minlength=c.nsp).astype(np.int64)
        order = np.argsort(species, kind="stable")  # select_ncdfinput's species-contiguous order
        sp = species[order].astype(np.int32)
        z = xyz[order, 2]
        xy = refsem.fold(xyz[order], self.box)
        xy[:, 2] = 0.0
        if self.slab is None:
            self.slab = SlabState(self, xyz.shape[0])
        self.slab.frame(xy, sp, z, self.box)
        self.nconf += 1

    def slab_results(self) -> Dict[str, np.ndarray]:
        return self.slab.results(self.nconf)

    def print_slabs(self, outdir: str = ".") -> List[str]:
        res = self.slab_results()
        files = []
        if "g_xy" in res:
            files += writers.write_gxy(outdir, res["r"], res["g_xy"], self.cfg.nsp, self.cfg.slab.zslice)
        if "s_xy" in res:
            files += writers.write_sqxy(outdir, res["q"], res["s_xy"], res["s_pxy"], self.cfg.slab.zslice)
        return files

    # ---- F(Q,t), Fs(Q,t), MSD (dyn_init / rtcorr) -----------------------------------------
    def dyn_init(self) -> None:
        if self.nconf_total is None:
            raise ValueError("run_sqw needs nconf_total (the trajectory's number of frames)")
        self.dyn = Dynamics(self.ctx, self.cfg.nsp, self.n, self.nconf_total, self.cfg.dyn or DynConfig(),
                            self.box, self.bsc_sp, ndim=self.cfg.ndim)

    def rtcorr(self, frame: Frame) -> None:
        if self.dyn is None:
            self.dyn_init()
        self.dyn.rtcorr(self.nconf + 1, self.stage.packed, self.n, self.box, time=frame.time, stream=self.stream)

    def print_rtcor(self, outdir: str = ".") -> List[str]:
        return self.dyn.print_rtcor(outdir, units=self.cfg.units)

    def run(self, frames: Iterable[Frame], check_every: int = 0) -> "Session":
        for k, f in enumerate(frames):
            self.add_frame(f)
            if check_every and (k + 1) % check_every == 0:
                self.ctx.check(self.stream)
        self.ctx.check(self.stream)
        return self

    # ---- results ----------------------------------------------------------------------
    def rdf_transfer(self) -> np.ndarray:
        """uint64 [nit][lsmax] pair counts summed over frames."""
        return self.hist.cpu().numpy().astype(np.uint64)

    def edge_stats(self) -> Dict[str, int]:
        e = self.edge.cpu().numpy()
        return {"edge_ulp": int(e[0]), "edge_fma": int(e[1]), "counted": int(e[2]), "tested": int(e[3])}

    def sq_transfer_gpu_cpu(self) -> np.ndarray:
        """FP64 [nbins][nit] sums of w Re(rho_a conj(rho_b)) (with charges: over the species and the
        charge density, nit = (nsp+1)(nsp+2)/2)."""
        return self.sq_out.cpu().numpy()

    def gqq_transfer(self) -> Optional[np.ndarray]:
        """FP64 [lsmax] sum over frames of the charge-product histogram over avq2 (None without charges)."""
        if self.gqq is not None:
            return self.gqq.cpu().numpy()
        if self.ex_qc and self.species_q is not None:
            return species_gqq(self.rdf_transfer(), self.species_q, self.cfg.nsp) / self.avq2()
        return None

    def sq_charged_sums(self) -> np.ndarray:
        """S sums in the charged row layout: from the device (charge_mode 'atom') or derived from the
        species rows (charge_mode 'species')."""
        out = self.sq_transfer_gpu_cpu()
        if self.device_charges:
            return out
        return species_charged_rows(out, self.species_q, self.cfg.nsp)

    def avq2(self) -> float:
        """sum(q^2)/N of the last frame, rounded to FP32 as the reference's variable (sq.cuf:144)."""
        q = self.charges.astype(np.float64)
        return float(F32(np.sum(q * q) / q.shape[0]))

    def rdf_results(self) -> Dict[str, np.ndarray]:
        self._refresh_ntype()
        res = normalise_rdf(self.rdf_transfer(), self.cfg.nsp, self.rdf.lsmax, self.cfg.deltar, self.volumen,
                            self.ntype, self.nconf, gqq=self.gqq_transfer(), ndim=self.cfg.ndim)
        if self.gi is not None:
            res["s2n"] = normalise_s2n(self.gi.cpu().numpy(), self.g2i.cpu().numpy(), self.nconf, self.cfg.nrandom,
                                       self.rdf.lsmax)
        return res

    def sq_results(self) -> Dict[str, np.ndarray]:
        self._refresh_ntype()
        if not self.ex_qc:
            return normalise_sq(self.sq_transfer_gpu_cpu(), self.kset, self.ntype, self.bsc_sp, self.nconf)
        return normalise_sq(self.sq_charged_sums(), self.kset, self.ntype, self.bsc_sp, self.nconf,
                            avq2=self.avq2())

    def printrdf(self, outdir: str = ".") -> List[str]:
        res = self.rdf_results()
        files = writers.write_gmixsim(outdir, res["r"], res["g"], self.cfg.nsp, g_qq=res.get("g_qq"))
        if "s2n" in res:
            files.append(writers.write_s2n(outdir, res["r"], res["s2n"]))
        return files

    def printSQ(self, outdir: str = ".") -> List[str]:
        res = self.sq_results()
        return writers.write_sq(outdir, res["q"], res["s_nn"], res["nq"], res["s_self"], res.get("binary"),
                                s_qq=res.get("s_qq"))

    def suggested_rcl(self) -> float:
        """First minimum of the total g(r) after its first peak (rdf.cuf:313-352, 755-822)."""
        self._refresh_ntype()
        return first_minimum(self.rdf_transfer(), self.rdf.lsmax, self.cfg.deltar, self.volumen,
                             int(self.ntype.sum()), ndim=self.cfg.ndim)

    def close(self) -> None:
        if self.slab is not None:
            self.slab.close()
        for obj in (self.sq, self.rdf, self.dyn):
            if obj is not None:
                obj.close()


class SlabState:
    """Per-slice g_xy(r) and S_xy(Q) of the reference's twoDstruc_3D analysis.

    g_xy (RDFcomp with rdfxy, rdf.cuf:218-232, 284-299, 672-738): pairs of atoms in the same slice,
    xy minimum-image distance, bins int(r/deltar)+1; per frame the slice histogram of species pair
    (k, j) is divided by countp(k, s) countp(j, s), the atoms of each species in the slice counted
    over atoms 1..N-1 (rdfxy's home loop stops one short, so the last atom is never counted).  Each
    slice runs as a two-dimensional pair plan over the slice's atoms with the 3D cutoff.
    S_xy (SQcalc with sqf3xy/sqf2xy, sq.cuf:73-85, 594-771): per frame and vector, the density of every
    species in every slice (trj_sq_rho_groups); S_pxy(bin, a, s) += |rho_as|^2 / countsp(s, a) and
    S_xy(bin, s) += |sum_a bsc_a rho_as|^2 / count(s), counting every atom of the slice.
    Normalisations of printrdf / printSQ (log.f90:337-376, 424-436, 516-523, 546-554)."""

    def __init__(self, sess: "Session", n_max: int):
        c = sess.cfg
        self.sess = sess
        self.nsp = c.nsp
        self.zslice = np.asarray(c.slab.zslice, np.float32)
        self.zgrid = np.float32(c.slab.zgrid)
        self.nslice = int(self.zslice.size)
        box = sess.box
        self.stage = engine.FrameStage(sess.ctx, n_max, c.nsp)
        self.rdf = None
        if c.run_rdf:
            p3 = refsem.rdf_params(c.nsp, c.deltar, c.rcrdf, box)  # the 3D clip of select_ncdfinput
            box2 = np.array([box[0], box[1], 1.0], np.float32)
            self.rdf = engine.RdfPlan(sess.ctx, c.nsp, c.deltar, p3.rcrdf, box2, n_max, ndim=2)
            self.rdf.set_binning(True)
            self.lsmax = self.rdf.lsmax
            self.hist_xy = np.zeros((c.nsp, c.nsp, self.nslice, self.lsmax))
            self.h_dev = self.rdf.new_hist()
        self.sq = None
        if c.run_sq:
            self.kset = refsem.slab_kset(box, c.qmax, c.qmin)
            self.sq = engine.SqPlan(sess.ctx, c.nsp, self.kset, np.array([n_max] + [0] * (c.nsp - 1)))
            self.sqf_xy = np.zeros((self.kset.nbins, self.nslice))
            self.sqf_pxy = np.zeros((self.kset.nbins, c.nsp, self.nslice))
            self.bsc = np.asarray(sess.bsc_sp, np.float64)

    def frame(self, xy: np.ndarray, sp: np.ndarray, z: np.ndarray, box) -> None:
        sl = refsem.slab_of(z, self.zslice, self.zgrid)
        nsp, ns = self.nsp, self.nslice
        if self.rdf is not None:
            counted = sl >= 0
            counted[-1] = False  # rdfxy counts atoms 1..N-1
            countp = np.zeros((nsp, ns), np.int64)
            np.add.at(countp, (sp[counted], sl[counted]), 1)
            box2 = np.array([box[0], box[1], 1.0], np.float32)
            for s in range(ns):
                sel = sl == s
                m = int(sel.sum())
                if m < 2:
                    continue
                self.h_dev.zero_()
                n = self.stage.upload_and_pack(xy[sel], sp[sel], box2)
                self.rdf.accumulate(self.stage.packed, n, box2, self.h_dev)
                h = self.h_dev.cpu().numpy().astype(np.float64)
                for a in range(nsp):
                    for b in range(a, nsp):
                        if countp[a, s] > 0 and countp[b, s] > 0:
                            self.hist_xy[a, b, s] += h[refsem.pair_row(a, b, nsp)] / (countp[a, s] * countp[b, s])
        if self.sq is not None:
            inc = sl >= 0
            grp = sp[inc].astype(np.int64) * ns + sl[inc]
            order = np.argsort(grp, kind="stable")
            cnt = np.bincount(grp, minlength=nsp * ns)
            off = np.zeros(nsp * ns + 1, np.int64)
            off[1:] = np.cumsum(cnt)
            pos = np.zeros((int(inc.sum()), 4), np.float32)
            pos[:, :2] = xy[inc][order, :2]
            dev = torch.from_numpy(pos).to(self.sess.ctx.torch_device)
            rho = self.sq.rho_groups(dev, pos.shape[0], box, off).cpu().numpy().reshape(nsp, ns, -1)
            countsp = cnt.reshape(nsp, ns)
            count = countsp.sum(axis=0)
            bins = self.kset.bins
            for s in range(ns):
                for a in range(nsp):
                    if countsp[a, s] > 0:
                        np.add.at(self.sqf_pxy[:, a, s], bins, np.abs(rho[a, s]) ** 2 / countsp[a, s])
                if count[s] > 0:
                    tot = (self.bsc[:, None] * rho[:, s, :]).sum(axis=0)
                    np.add.at(self.sqf_xy[:, s], bins, np.abs(tot) ** 2 / count[s])

    def results(self, nconf: int) -> Dict[str, np.ndarray]:
        out: Dict[str, np.ndarray] = {}
        sess = self.sess
        if self.rdf is not None:
            dr = float(F32(sess.cfg.deltar))
            nrow = max(self.lsmax - 2, 0)
            ri = np.array([float(F32(F32(i) * F32(sess.cfg.deltar))) for i in range(1, nrow + 1)])
            zg = float(self.zgrid)
            dv = math.pi * ((ri + dr / 2) ** 2 - (ri - dr / 2) ** 2) * zg   # log.f90:478-480
            fac = sess.volumen * (zg / float(sess.box[2]))
            g = np.zeros((nrow, self.nsp, self.nsp, self.nslice))
            for a in range(self.nsp):
                for b in range(a, self.nsp):
                    v = (2.0 if a == b else 1.0) * fac * self.hist_xy[a, b, :, :nrow].T / (dv[:, None] * nconf)
                    g[:, a, b] = v
                    g[:, b, a] = v
            out["r"] = ri.astype(np.float32)
            out["g_xy"] = g
        if self.sq is not None:
            nq = self.kset.nq.astype(np.float64)
            sl = slice(1, self.kset.nqmax + 1)
            with np.errstate(divide="ignore", invalid="ignore"):
                den = np.where(nq > 0, nq, np.nan)[:, None] * nconf
                out["q"] = self.kset.q_column()
                out["s_xy"] = (self.sqf_xy / den)[sl]
                out["s_pxy"] = (self.sqf_pxy / den[:, :, None])[sl]
            out["nq"] = self.kset.nq[sl]
        return out

    def close(self) -> None:
        for obj in (self.rdf, self.sq):
            if obj is not None:
                obj.close()


def shell_volumes(lsmax: int, deltar: float, ndim: int = 3) -> np.ndarray:
    """4 pi/3 ((r+dr/2)^3 - (r-dr/2)^3), in 2D pi ((r+dr/2)^2 - (r-dr/2)^2), for r = i*dr,
    i = 1..lsmax (log.f90:475-487)."""
    dr = float(F32(deltar))
    ri = np.array([float(F32(F32(i) * F32(deltar))) for i in range(1, lsmax + 1)])
    if ndim == 2:
        return math.pi * ((ri + dr / 2) ** 2 - (ri - dr / 2) ** 2), ri
    return 4.0 * math.pi * ((ri + dr / 2) ** 3 - (ri - dr / 2) ** 3) / 3.0, ri


def normalise_rdf(hist: np.ndarray, nsp: int, lsmax: int, deltar: float, volumen: float, ntype: np.ndarray,
                  nconf: int, gqq: Optional[np.ndarray] = None, ndim: int = 3) -> Dict[str, np.ndarray]:
    """printrdf's g_jl(r_i) = (j/l+1) V H_jl(i) / (dV_i N_l N_j Nconf) for i = 1..lsmax-2 (FP64), and with
    charges g_qq(r_i) = 2 V gqq(i) / (N^2 dV_i Nconf) (log.f90:502-504)."""
    dv, ri = shell_volumes(lsmax, deltar, ndim)
    nrow = max(lsmax - 2, 0)
    g = np.zeros((nrow, nsp, nsp))
    h = hist.astype(np.float64)
    for j in range(nsp):
        for l in range(j, nsp):
            row = refsem.pair_row(j, l, nsp)
            fac = 2.0 if j == l else 1.0
            v = fac * volumen * h[row, :nrow] / (dv[:nrow] * float(ntype[l]) * float(ntype[j]) * nconf)
            g[:, j, l] = v
            g[:, l, j] = v
    # total g(r) with the 2V/(dV N^2) normalisation of RDFcomp (rdf.cuf:313-341), per frame
    n = float(np.sum(ntype))
    gtot = 2.0 * volumen * h[:, :nrow].sum(axis=0) / (dv[:nrow] * n * n * nconf)
    res = {"r": ri[:nrow].astype(np.float32), "g": g, "gtot": gtot}
    if gqq is not None:
        res["g_qq"] = 2.0 * volumen * np.asarray(gqq, np.float64)[:nrow] / (n * n * dv[:nrow] * nconf)
    return res


def normalise_s2n(gi: np.ndarray, g2i: np.ndarray, nconf: int, nrandom: int, lsmax: int) -> np.ndarray:
    """s2n(r_i) = g2i(i)/(Nconf nrandom) - (gi(i)/(Nconf nrandom))^2 for i = 1..lsmax-2 (log.f90:532), FP64."""
    m = float(nconf * nrandom)
    g = gi.astype(np.float64)[1:lsmax - 1]
    g2 = g2i.astype(np.float64)[1:lsmax - 1]
    return g2 / m - (g / m) ** 2


def first_minimum(hist: np.ndarray, lsmax: int, deltar: float, volumen: float, natms: int, ndim: int = 3) -> float:
    dv, _ = shell_volumes(lsmax, deltar, ndim)
    g = np.zeros(lsmax + 1)
    g[1:] = 2.0 * volumen * hist.astype(np.float64).sum(axis=0) / (dv * natms * natms)
    nrdf = lsmax
    imax = 1
    for i in range(2, nrdf):
        if g[i] > 0.1 and g[i] > g[i - 1] and g[i] > g[i + 1]:
            imax = i
            break
    if imax == 1:
        imax = int(np.argmax(g[1:nrdf + 1])) + 1
    imin = imax + 1
    for i in range(imax + 1, nrdf):
        if g[i] < g[i - 1] and g[i] < g[i + 1]:
            imin = i
            break
    if 0 < imin < nrdf:
        x1, x2, x3 = deltar * (imin - 1), deltar * imin, deltar * (imin + 1)
        y1, y2, y3 = g[imin - 1], g[imin], g[imin + 1]
        den = y1 - 2.0 * y2 + y3
        return x2 + 0.5 * (y1 - y3) / den * (x3 - x1) / 2.0 if abs(den) > 1e-12 else x2
    return deltar * imin


def species_gqq(hist: np.ndarray, qa: np.ndarray, nsp: int) -> np.ndarray:
    """Charge-product sums per bin when species a carries charge q_a: sum_{a<=b} q_a q_b H_ab (FP64),
    the sum rdf.cuf:469-472 forms pair by pair."""
    q = np.asarray(qa, np.float32).astype(np.float64)
    out = np.zeros(hist.shape[1])
    for a, b in refsem.pair_rows(nsp):
        out += q[a] * q[b] * hist[refsem.pair_row(a, b, nsp)].astype(np.float64)
    return out


def species_charged_rows(out: np.ndarray, qa: np.ndarray, nsp: int) -> np.ndarray:
    """Charged-layout S sums from the species rows when species a carries charge q_a:
    rho_q = sum_a q_a rho_a, so Re(rho_a rho_q*) = sum_b q_b Re(rho_a rho_b*) and
    |rho_q|^2 = sum_{a,b} q_a q_b Re(rho_a rho_b*)."""
    q = np.asarray(qa, np.float32).astype(np.float64)
    ndens = nsp + 1
    res = np.zeros((out.shape[0], ndens * (ndens + 1) // 2))

    def sp(a, b):
        return out[:, refsem.pair_row(a, b, nsp)]

    for a, b in refsem.pair_rows(nsp):
        res[:, refsem.pair_row(a, b, ndens)] = sp(a, b)
    for a in range(nsp):
        res[:, refsem.pair_row(a, nsp, ndens)] = sum(q[b] * sp(a, b) for b in range(nsp))
    res[:, refsem.pair_row(nsp, nsp, ndens)] = sum(q[a] * q[b] * sp(a, b) for a in range(nsp) for b in range(nsp))
    return res


def split_charged_rows(out: np.ndarray, nsp: int):
    """Rows of a charged S(Q) output ((nsp+1)(nsp+2)/2 rows over the species and the charge density
    nsp): the species-pair rows in the uncharged layout, the cross rows (a, q) and the (q, q) row."""
    ndens = nsp + 1
    sp = np.stack([out[:, refsem.pair_row(a, c, ndens)] for a, c in refsem.pair_rows(nsp)], axis=1)
    cross = np.stack([out[:, refsem.pair_row(a, nsp, ndens)] for a in range(nsp)], axis=1)
    return sp, cross, out[:, refsem.pair_row(nsp, nsp, ndens)]


def normalise_sq(out: np.ndarray, kset: refsem.KSet, ntype: np.ndarray, bsc: np.ndarray,
                 nconf: int, avq2: Optional[float] = None) -> Dict[str, np.ndarray]:
    """printSQ (log.f90:317-412) in FP64: S_NN = sqf/(baver^2 N Nconf nq), S_aa = sqfp_a/(N_a Nconf nq),
    and for two species with bsc = 1 the Bhatia-Thornton S_cc and the partials s11, s22, s12.
    Also returns every species-pair S_ab = sum Re(rho_a rho_b*)/(sqrt(N_a N_b) Nconf nq).
    With avq2 (charged output layout): S_qq = sqfq/(N Nconf nq), sqfq = sum |rho_q|^2 / avq2
    (sq.cuf:143-145, log.f90:386,393)."""
    nsp = ntype.shape[0]
    sqfq = None
    if avq2 is not None:
        out, _, qq = split_charged_rows(out, nsp)
        sqfq = qq / avq2
    n = float(ntype.sum())
    b = np.asarray(bsc, np.float64)
    rows = refsem.pair_rows(nsp)
    sqf = np.zeros(out.shape[0])
    for r, (a, c) in enumerate(rows):
        sqf += (1.0 if a == c else 2.0) * b[a] * b[c] * out[:, r]
    baver = float((ntype * b).sum() / n)
    sqf = sqf / baver ** 2
    nq = kset.nq.astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        den = np.where(nq > 0, nq, np.nan)
        s_nn = sqf / (n * nconf * den)
        s_self = np.stack([out[:, refsem.pair_row(a, a, nsp)] / (ntype[a] * nconf * den) for a in range(nsp)],
                          axis=1)
        s_pair = np.stack([out[:, r] / (math.sqrt(ntype[a] * ntype[c]) * nconf * den) for r, (a, c) in
                           enumerate(rows)], axis=1)
    sl = slice(1, kset.nqmax + 1)
    res = {"q": kset.q_column(), "s_nn": s_nn[sl], "nq": kset.nq[sl], "s_self": s_self[sl], "s_pair": s_pair[sl],
           "sqf": sqf[sl]}
    if sqfq is not None:
        with np.errstate(divide="ignore", invalid="ignore"):
            res["s_qq"] = (sqfq / (n * nconf * den))[sl]
    if nsp == 2 and np.all(np.abs(b - 1.0) <= 1e-4):
        x1, x2 = ntype[0] / n, ntype[1] / n
        s11 = x1 * s_self[sl, 0]
        s22 = x2 * s_self[sl, 1]
        s12 = 0.5 * (s_nn[sl] - s11 - s22)
        scc = x2 ** 2 * s11 + x1 ** 2 * s22 - 2 * x1 * x2 * s12
        res["binary"] = {"scc": scc, "s11": s11, "s22": s22, "s12": s12}
    return res
