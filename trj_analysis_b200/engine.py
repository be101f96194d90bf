"""Device layer: contexts, plans and frame buffers over the C ABI.

PyTorch supplies device memory and streams only; every kernel that touches the
data is in libtrj_sm100.so.  Pointers are passed as integers from
``tensor.data_ptr()`` and streams as ``torch.cuda.Stream.cuda_stream``.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import box3, check
from .refsem import KSet

vp = ctypes.c_void_p


def _ptr(t: Optional[torch.Tensor]):
    return vp(t.data_ptr()) if t is not None else vp(0)


def _stream(stream: Optional[torch.cuda.Stream]):
    s = stream if stream is not None else torch.cuda.current_stream()
    return vp(s.cuda_stream)


class Context:
    """One device's library context (status word, pack scratch)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("trj_analysis_b200 needs a CUDA device (sm_100); no CPU path exists")
        self.device = int(device)
        self.torch_device = torch.device("cuda", self.device)
        h = vp()
        rc = self.lib.trj_ctx_create(self.device, ctypes.byref(h))
        if rc != _lib.TRJ_OK:
            raise _lib.TrjError(rc, f"trj_ctx_create(device={device}) failed (an sm_100 device is required)")
        self.h = h
        self.sm_count = self.lib.trj_ctx_sm_count(h)

    def check(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Synchronises ``stream`` and raises on device-side status (bad data, timeouts)."""
        check(self.lib.trj_ctx_check(self.h, _stream(stream)), self.h, "device status")

    def set_sq_tile_cols(self, cols: int) -> None:
        """Widest tensor-core S(Q) tile of plans created from now on (0: default 224)."""
        check(self.lib.trj_ctx_set_sq_tile_cols(self.h, int(cols)), self.h, "trj_ctx_set_sq_tile_cols")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.trj_ctx_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


def pack_frame(ctx: Context, xyz: torch.Tensor, species: torch.Tensor, nsp: int, box,
               packed: torch.Tensor, counts: torch.Tensor, stream=None, charges: Optional[torch.Tensor] = None,
               qpacked: Optional[torch.Tensor] = None) -> None:
    """Device layout step (fold + stable species-contiguous order); charges, when given, are written
    to ``qpacked`` in the packed order."""
    n = int(xyz.shape[0])
    assert xyz.dtype == torch.float32 and xyz.is_contiguous() and xyz.is_cuda
    assert species.dtype == torch.int32 and species.is_contiguous()
    assert packed.dtype == torch.float32 and packed.shape[0] >= n and packed.shape[1] == 4
    assert counts.dtype == torch.int64 and counts.numel() >= nsp
    if charges is None:
        rc = ctx.lib.trj_frame_pack(ctx.h, _ptr(xyz), _ptr(species), n, nsp, box3(box), _ptr(packed),
                                    _ptr(counts), _stream(stream))
        check(rc, ctx.h, "trj_frame_pack")
        return
    assert charges.dtype == torch.float32 and charges.is_contiguous() and charges.numel() >= n
    assert qpacked is not None and qpacked.dtype == torch.float32 and qpacked.numel() >= n
    rc = ctx.lib.trj_frame_pack_charges(ctx.h, _ptr(xyz), _ptr(species), _ptr(charges), n, nsp, box3(box),
                                        _ptr(packed), _ptr(qpacked), _ptr(counts), _stream(stream))
    check(rc, ctx.h, "trj_frame_pack_charges")


class RdfPlan:
    """g_ab(r) plan.  Reference bins (nint(r/deltar), rcrdf clipped to half the box) by default;
    ``floor_bins=nbins`` gives nbins bins [k dr, (k+1) dr) on [0, rcrdf) instead."""

    def __init__(self, ctx: Context, nsp: int, deltar: float, rcrdf: float, box, n_max: int,
                 floor_bins: Optional[int] = None, ndim: int = 3):
        self.ctx = ctx
        h = vp()
        if ndim == 2:
            rc = ctx.lib.trj_rdf_plan_create_2d(ctx.h, nsp, float(deltar), float(rcrdf), box3(box), int(n_max),
                                                ctypes.byref(h))
        elif floor_bins:
            rc = ctx.lib.trj_rdf_plan_create_floor(ctx.h, nsp, float(rcrdf), int(floor_bins), box3(box), int(n_max),
                                                   ctypes.byref(h))
        else:
            rc = ctx.lib.trj_rdf_plan_create(ctx.h, nsp, float(deltar), float(rcrdf), box3(box), int(n_max),
                                             ctypes.byref(h))
        check(rc, ctx.h, "trj_rdf_plan_create")
        self.h = h
        self.nsp = nsp
        self.refresh_info()

    def refresh_info(self) -> None:
        lsmax, nit = ctypes.c_int(), ctypes.c_int()
        cells = (ctypes.c_int * 3)()
        rc_eff, side2 = ctypes.c_float(), ctypes.c_float()
        sb = ctypes.c_int64()
        check(self.ctx.lib.trj_rdf_plan_info(self.h, ctypes.byref(lsmax), ctypes.byref(nit), cells,
                                             ctypes.byref(rc_eff), ctypes.byref(side2), ctypes.byref(sb)),
              self.ctx.h, "trj_rdf_plan_info")
        self.lsmax, self.nit = lsmax.value, nit.value
        self.cells = tuple(cells)
        self.rcrdf, self.side2 = rc_eff.value, side2.value
        self.scratch_bytes = sb.value

    def new_hist(self) -> torch.Tensor:
        return torch.zeros((self.nit, self.lsmax), dtype=torch.int64, device=self.ctx.torch_device)

    def new_gqq(self) -> torch.Tensor:
        """FP64 [lsmax] accumulator of the charge-product histogram divided by avq2 per frame."""
        return torch.zeros((self.lsmax,), dtype=torch.float64, device=self.ctx.torch_device)

    def accumulate(self, packed: torch.Tensor, n: int, box, hist: torch.Tensor,
                   edge: Optional[torch.Tensor] = None, stream=None, qpacked: Optional[torch.Tensor] = None,
                   gqq: Optional[torch.Tensor] = None) -> None:
        """Adds the frame's pair counts to ``hist``; with ``qpacked`` (charges in packed order) and
        ``gqq`` also the charge-product histogram over avq2."""
        assert hist.dtype == torch.int64 and hist.shape == (self.nit, self.lsmax)
        if qpacked is None and gqq is None:
            rc = self.ctx.lib.trj_rdf_accumulate(self.h, _ptr(packed), int(n), box3(box), _ptr(hist), _ptr(edge),
                                                 _stream(stream))
            check(rc, self.ctx.h, "trj_rdf_accumulate")
            return
        assert qpacked is not None and gqq is not None
        assert qpacked.dtype == torch.float32 and gqq.dtype == torch.float64 and gqq.shape == (self.lsmax,)
        rc = self.ctx.lib.trj_rdf_accumulate_charged(self.h, _ptr(packed), _ptr(qpacked), int(n), box3(box),
                                                     _ptr(hist), _ptr(edge), _ptr(gqq), _stream(stream))
        check(rc, self.ctx.h, "trj_rdf_accumulate_charged")

    def set_binning(self, floor_bins: bool) -> None:
        """Bins nint(r/deltar) (False) or int(r/deltar)+1 (True, the slab g(r))."""
        check(self.ctx.lib.trj_rdf_plan_set_binning(self.h, 1 if floor_bins else 0), self.ctx.h,
              "trj_rdf_plan_set_binning")

    def set_wait(self, clocks: int = 0, stall_test: bool = False) -> None:
        """Limit (SM clocks, 0 = default) of the pair kernel's waits for staged chunks; stall_test makes
        every launch run out of it once (see trj_rdf_plan_set_wait)."""
        check(self.ctx.lib.trj_rdf_plan_set_wait(self.h, int(clocks), 1 if stall_test else 0), self.ctx.h,
              "trj_rdf_plan_set_wait")

    def new_s2n(self):
        """(gi, g2i): uint64 [lsmax+1] sums of N_k and N_k^2 over sample points and frames."""
        dev = self.ctx.torch_device
        return (torch.zeros((self.lsmax + 1,), dtype=torch.int64, device=dev),
                torch.zeros((self.lsmax + 1,), dtype=torch.int64, device=dev))

    def s2n(self, nrandom: int, gi: torch.Tensor, g2i: torch.Tensor, points: Optional[torch.Tensor] = None,
            stream=None) -> None:
        """Number fluctuations around nrandom fixed random points for the frame last accumulated."""
        assert gi.dtype == g2i.dtype == torch.int64 and gi.numel() == g2i.numel() == self.lsmax + 1
        if points is not None:
            assert points.dtype == torch.float32 and points.numel() >= 3 * nrandom
        rc = self.ctx.lib.trj_rdf_s2n(self.h, int(nrandom), _ptr(gi), _ptr(g2i), _ptr(points), _stream(stream))
        check(rc, self.ctx.h, "trj_rdf_s2n")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.ctx.lib.trj_rdf_plan_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class SqPlan:
    """S(Q) plan.  ``charged=True`` adds the charge density as species ``nsp``: the output then has
    (nsp+1)(nsp+2)/2 rows (last row: sums of w |rho_q|^2) and accumulate takes the packed charges."""

    def __init__(self, ctx: Context, nsp: int, kset: KSet, species_counts, charged: bool = False):
        self.ctx = ctx
        self.nsp = nsp
        self.charged = bool(charged)
        self.kset = kset
        counts = np.ascontiguousarray(np.asarray(species_counts, dtype=np.int64))
        assert counts.shape == (nsp,)
        self._vec = np.ascontiguousarray(kset.vectors.astype(np.int32))
        self._bin = np.ascontiguousarray(kset.bins.astype(np.int32))
        self._w = np.ascontiguousarray(kset.weights.astype(np.float64))
        self._dense = np.ascontiguousarray(kset.dense.astype(np.uint8))
        h = vp()
        create = ctx.lib.trj_sq_plan_create_charged if self.charged else ctx.lib.trj_sq_plan_create
        rc = create(
            ctx.h, nsp, int(kset.nvec), self._vec.ctypes.data_as(vp), self._bin.ctypes.data_as(vp),
            self._w.ctypes.data_as(vp), self._dense.ctypes.data_as(vp), int(kset.nbins),
            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(h))
        check(rc, ctx.h, "trj_sq_plan_create")
        self.h = h
        self.ndens = nsp + 1 if self.charged else nsp  # densities: species (+ charge)
        self.nit = self.ndens * (self.ndens + 1) // 2
        self.n_total = int(counts.sum())
        nd, nt, ts, sb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(ctx.lib.trj_sq_plan_info(h, ctypes.byref(nd), ctypes.byref(nt), ctypes.byref(ts), ctypes.byref(sb)),
              ctx.h, "trj_sq_plan_info")
        self.n_dense, self.n_tiles, self.tile_slots, self.scratch_bytes = nd.value, nt.value, ts.value, sb.value

    def new_out(self) -> torch.Tensor:
        return torch.zeros((self.kset.nbins, self.nit), dtype=torch.float64, device=self.ctx.torch_device)

    def set_flush(self, atoms: int) -> None:
        """Atoms the tensor cores accumulate in one FP32 run before it is added into the running sum."""
        check(self.ctx.lib.trj_sq_plan_set_flush(self.h, int(atoms)), self.ctx.h, "trj_sq_plan_set_flush")

    def set_z_from_y(self, mul: int) -> None:
        """Planar tile form: third phase = mul * second phase (exact); vectors (nx, ny % mul, ny // mul)."""
        check(self.ctx.lib.trj_sq_plan_set_z_from_y(self.h, int(mul)), self.ctx.h, "trj_sq_plan_set_z_from_y")

    def set_pairs(self, enable: bool) -> None:
        """Tensor-core tiles in CTA pairs (one M = 256 contraction per two tiles) or one per CTA."""
        check(self.ctx.lib.trj_sq_plan_set_pairs(self.h, 1 if enable else 0), self.ctx.h, "trj_sq_plan_set_pairs")

    def accumulate(self, packed: torch.Tensor, n: int, box, out: torch.Tensor, method: int, stream=None,
                   qpacked: Optional[torch.Tensor] = None) -> None:
        assert out.dtype == torch.float64 and out.shape == (self.kset.nbins, self.nit)
        if self.charged:
            if qpacked is None:
                raise ValueError("charged S(Q) plan: pass the packed charges")
            assert qpacked.dtype == torch.float32 and qpacked.numel() >= n
            rc = self.ctx.lib.trj_sq_accumulate_charged(self.h, _ptr(packed), _ptr(qpacked), int(n), box3(box),
                                                        int(method), _ptr(out), _stream(stream))
            check(rc, self.ctx.h, "trj_sq_accumulate_charged")
            return
        rc = self.ctx.lib.trj_sq_accumulate(self.h, _ptr(packed), int(n), box3(box), int(method), _ptr(out),
                                            _stream(stream))
        check(rc, self.ctx.h, "trj_sq_accumulate")

    def rho_groups(self, packed: torch.Tensor, n: int, box, group_off: np.ndarray, stream=None) -> torch.Tensor:
        """rho_g(k) over contiguous atom groups of ``packed`` (offsets ``group_off``, ngroups+1):
        (ngroups, nvec) complex128 in the caller's vector order."""
        off = np.ascontiguousarray(np.asarray(group_off, np.int64))
        ng = off.shape[0] - 1
        t = torch.empty((ng, self.kset.nvec, 2), dtype=torch.float64, device=self.ctx.torch_device)
        rc = self.ctx.lib.trj_sq_rho_groups(self.h, _ptr(packed), int(n), box3(box), ng, off.ctypes.data_as(vp),
                                            _ptr(t), _stream(stream))
        check(rc, self.ctx.h, "trj_sq_rho_groups")
        return torch.view_as_complex(t)

    def rho(self, stream=None) -> torch.Tensor:
        """rho_a(k) of the last accumulate, (ndens, nvec) complex128, caller vector order (charged plans:
        the charge density last)."""
        t = torch.empty((self.ndens, self.kset.nvec, 2), dtype=torch.float64, device=self.ctx.torch_device)
        check(self.ctx.lib.trj_sq_rho(self.h, _ptr(t), _stream(stream)), self.ctx.h, "trj_sq_rho")
        return torch.view_as_complex(t)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.ctx.lib.trj_sq_plan_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Fused launches over one frame of each of several small requests per turn (``trj_batch_*``).

    Per turn: ``begin(buf)``; for every request ``stage(buf, off, xyz, species)`` and
    ``add(buf, rdf, sq, off, n, box, hist, out)``; then ``launch(buf, stream)`` (or a CUDA graph of
    it, captured once per buffer).  Buffer ``buf`` may be refilled only after its previous launch
    has run (``wait(buf)``)."""

    def __init__(self, ctx: Context, max_items: int = 64, max_atoms: int = 1 << 20, hist_words: int = 4096):
        self.ctx = ctx
        h = vp()
        check(ctx.lib.trj_batch_create(ctx.h, int(max_items), int(max_atoms), int(hist_words), ctypes.byref(h)),
              ctx.h, "trj_batch_create")
        self.h = h
        self.max_items, self.max_atoms, self.hist_words = int(max_items), int(max_atoms), int(hist_words)
        self.xyz, self.species, self.events = [], [], [None, None]
        for b in range(2):
            px, ps = vp(), vp()
            check(ctx.lib.trj_batch_staging(h, b, ctypes.byref(px), ctypes.byref(ps)), ctx.h, "trj_batch_staging")
            fx = ctypes.cast(px, ctypes.POINTER(ctypes.c_float))
            fs = ctypes.cast(ps, ctypes.POINTER(ctypes.c_int32))
            self.xyz.append(np.ctypeslib.as_array(fx, shape=(self.max_atoms, 3)))
            self.species.append(np.ctypeslib.as_array(fs, shape=(self.max_atoms,)))
        dbytes = ctypes.c_int64()
        check(ctx.lib.trj_batch_info(h, 0, None, None, ctypes.byref(dbytes)), ctx.h, "trj_batch_info")
        self.device_bytes = dbytes.value

    def wait(self, buf: int) -> None:
        """Blocks until the last launch from staging buffer ``buf`` has run."""
        if self.events[buf] is not None:
            self.events[buf].synchronize()

    def begin(self, buf: int) -> None:
        self.wait(buf)
        check(self.ctx.lib.trj_batch_begin(self.h, int(buf)), self.ctx.h, "trj_batch_begin")

    def stage(self, buf: int, off: int, xyz: np.ndarray, species: np.ndarray) -> None:
        n = xyz.shape[0]
        self.xyz[buf][off:off + n] = xyz
        self.species[buf][off:off + n] = species

    def add(self, buf: int, rdf: Optional["RdfPlan"], sq: Optional["SqPlan"], off: int, n: int, box,
            hist: Optional[torch.Tensor], out: Optional[torch.Tensor], edge: Optional[torch.Tensor] = None) -> None:
        if rdf is not None:
            assert hist is not None and hist.dtype == torch.int64 and hist.shape == (rdf.nit, rdf.lsmax)
        if sq is not None:
            assert out is not None and out.dtype == torch.float64 and out.shape == (sq.kset.nbins, sq.nit)
        rc = self.ctx.lib.trj_batch_add(self.h, int(buf), rdf.h if rdf is not None else vp(0),
                                        sq.h if sq is not None else vp(0), int(off), int(n), box3(box),
                                        _ptr(hist), _ptr(edge), _ptr(out))
        check(rc, self.ctx.h, "trj_batch_add")

    def info(self, buf: int):
        """(items, [layout units, pair tiles, direct-sum blocks, shell bins]) of the buffer's turn."""
        ni = ctypes.c_int()
        units = (ctypes.c_int64 * 4)()
        check(self.ctx.lib.trj_batch_info(self.h, int(buf), ctypes.byref(ni), units, None), self.ctx.h,
              "trj_batch_info")
        return ni.value, list(units)

    def launch(self, buf: int, stream=None) -> None:
        check(self.ctx.lib.trj_batch_launch(self.h, int(buf), _stream(stream)), self.ctx.h, "trj_batch_launch")

    def mark(self, buf: int, stream=None) -> None:
        """Records the end of buffer ``buf``'s launch on ``stream`` (what ``wait``/``begin`` wait for)."""
        ev = torch.cuda.Event()
        ev.record(stream if stream is not None else torch.cuda.current_stream())
        self.events[buf] = ev

    def kernel_ms(self) -> float:
        ms = ctypes.c_float()
        check(self.ctx.lib.trj_batch_kernel_ms(self.h, ctypes.byref(ms)), self.ctx.h, "trj_batch_kernel_ms")
        return ms.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.xyz, self.species = [], []
            self.ctx.lib.trj_batch_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class DynPlan:
    """Multiple-origin time correlations (F(Q,t), Fs(Q,t), MSD) over the vectors of an SqwSet."""

    def __init__(self, ctx: Context, nsp: int, n: int, nbuffer: int, ndyn: int, sqw, bsc):
        self.ctx = ctx
        self.nsp, self.n, self.nbuffer, self.ndyn = nsp, int(n), int(nbuffer), int(ndyn)
        self.nbins = max(1, int(sqw.qw.size))  # one unused bin when only C_r(t) is wanted
        self._vec = np.ascontiguousarray(sqw.vectors.astype(np.int32))
        self._bin = np.ascontiguousarray(sqw.bins.astype(np.int32))
        self._bsc = np.ascontiguousarray(np.asarray(bsc, np.float32))
        assert self._bsc.shape == (nsp,)
        h = vp()
        rc = ctx.lib.trj_dyn_plan_create(ctx.h, nsp, self.n, self.nbuffer, self.ndyn, int(self._vec.shape[0]),
                                         self._vec.ctypes.data_as(vp), self._bin.ctypes.data_as(vp), self.nbins,
                                         self._bsc.ctypes.data_as(vp), ctypes.byref(h))
        check(rc, ctx.h, "trj_dyn_plan_create")
        self.h = h
        sb = ctypes.c_int64()
        check(ctx.lib.trj_dyn_plan_info(h, ctypes.byref(sb)), ctx.h, "trj_dyn_plan_info")
        self.scratch_bytes = sb.value

    def new_totals(self):
        """(fkt [ndyn][nbins], fskt [ndyn][nbins], r2t [ndyn]) FP64 device accumulators."""
        dev = self.ctx.torch_device
        return (torch.zeros((self.ndyn, self.nbins), dtype=torch.float64, device=dev),
                torch.zeros((self.ndyn, self.nbins), dtype=torch.float64, device=dev),
                torch.zeros((self.ndyn,), dtype=torch.float64, device=dev))

    def accumulate(self, packed: torch.Tensor, n: int, box, lags: np.ndarray, origins: np.ndarray,
                   stream=None) -> None:
        lag = np.ascontiguousarray(np.asarray(lags, np.int32))
        org = np.ascontiguousarray(np.asarray(origins, np.uint8))
        assert lag.shape == (self.nbuffer,) and org.shape == (self.nbuffer,)
        rc = self.ctx.lib.trj_dyn_accumulate(self.h, _ptr(packed), int(n), box3(box), lag.ctypes.data_as(vp),
                                             org.ctypes.data_as(vp), _stream(stream))
        check(rc, self.ctx.h, "trj_dyn_accumulate")

    def flush(self, done: np.ndarray, fkt: torch.Tensor, fskt: torch.Tensor, r2t: torch.Tensor, stream=None) -> None:
        d = np.ascontiguousarray(np.asarray(done, np.uint8))
        assert d.shape == (self.nbuffer,)
        assert fkt.dtype == fskt.dtype == r2t.dtype == torch.float64
        rc = self.ctx.lib.trj_dyn_flush(self.h, d.ctypes.data_as(vp), _ptr(fkt), _ptr(fskt), _ptr(r2t),
                                        _stream(stream))
        check(rc, self.ctx.h, "trj_dyn_flush")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.ctx.lib.trj_dyn_plan_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


METHODS = {"plain": _lib.TRJ_SQ_PLAIN_FP32, "split": _lib.TRJ_SQ_SPLIT_BF16X3,
           "plain_fp32": _lib.TRJ_SQ_PLAIN_FP32, "split_bf16x3": _lib.TRJ_SQ_SPLIT_BF16X3}


class FrameStage:
    """Pinned host staging + device buffers for frames of up to ``n_max`` atoms."""

    def __init__(self, ctx: Context, n_max: int, nsp: int, charged: bool = False):
        dev = ctx.torch_device
        self.ctx = ctx
        self.n_max = n_max
        self.nsp = nsp
        self.charged = bool(charged)
        if self.charged:
            self.h_q = torch.empty((n_max,), dtype=torch.float32, pin_memory=True)
            self.d_q = torch.empty((n_max,), dtype=torch.float32, device=dev)
            self.qpacked = torch.empty((n_max,), dtype=torch.float32, device=dev)
        else:
            self.h_q = self.d_q = self.qpacked = None
        self.h_xyz = torch.empty((n_max, 3), dtype=torch.float32, pin_memory=True)
        self.h_sp = torch.empty((n_max,), dtype=torch.int32, pin_memory=True)
        self.d_xyz = torch.empty((n_max, 3), dtype=torch.float32, device=dev)
        self.d_sp = torch.empty((n_max,), dtype=torch.int32, device=dev)
        self.packed = torch.empty((n_max, 4), dtype=torch.float32, device=dev)
        self.counts = torch.zeros((max(nsp, 1),), dtype=torch.int64, device=dev)
        self._copied = None  # event after the last host->device copy out of the pinned buffers

    def upload_and_pack_types(self, xyz: np.ndarray, types: np.ndarray, box, lut: torch.Tensor, stream=None) -> int:
        """Copies the raw coordinates and type ids and lays the frame out with the type-to-species
        table ``lut`` (device int32) applied on the device (trj_frame_pack_types)."""
        n = int(xyz.shape[0])
        if n > self.n_max:
            raise _lib.TrjError(_lib.TRJ_ERR_CAPACITY, f"frame of {n} atoms exceeds stage size {self.n_max}")
        if self.charged:
            raise ValueError("frame charges: use upload_and_pack")
        if self._copied is not None:
            self._copied.synchronize()  # pinned buffers may still feed the previous copy
        self.h_xyz[:n].numpy()[:] = xyz
        self.h_sp[:n].numpy()[:] = types
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            self.d_xyz[:n].copy_(self.h_xyz[:n], non_blocking=True)
            self.d_sp[:n].copy_(self.h_sp[:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
            self._copied = ev
        assert lut.dtype == torch.int32 and lut.is_cuda
        rc = self.ctx.lib.trj_frame_pack_types(self.ctx.h, _ptr(self.d_xyz), _ptr(self.d_sp), _ptr(lut),
                                               int(lut.numel()), n, self.nsp, box3(box), _ptr(self.packed),
                                               _ptr(self.counts), _stream(s))
        check(rc, self.ctx.h, "trj_frame_pack_types")
        return n

    def upload_and_pack(self, xyz: np.ndarray, species: np.ndarray, box, stream=None,
                        charges: Optional[np.ndarray] = None) -> int:
        n = int(xyz.shape[0])
        if n > self.n_max:
            raise _lib.TrjError(_lib.TRJ_ERR_CAPACITY, f"frame of {n} atoms exceeds stage size {self.n_max}")
        if self.charged != (charges is not None):
            raise ValueError("frame charges: the stage was made " + ("with" if self.charged else "without") +
                             " charges")
        if self._copied is not None:
            self._copied.synchronize()  # pinned buffers may still feed the previous copy
        self.h_xyz[:n].numpy()[:] = xyz
        self.h_sp[:n].numpy()[:] = species
        if self.charged:
            self.h_q[:n].numpy()[:] = charges
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            self.d_xyz[:n].copy_(self.h_xyz[:n], non_blocking=True)
            self.d_sp[:n].copy_(self.h_sp[:n], non_blocking=True)
            if self.charged:
                self.d_q[:n].copy_(self.h_q[:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
            self._copied = ev
        pack_frame(self.ctx, self.d_xyz[:n], self.d_sp[:n], self.nsp, box, self.packed, self.counts, stream=s,
                   charges=self.d_q[:n] if self.charged else None, qpacked=self.qpacked)
        return n
