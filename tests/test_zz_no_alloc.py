"""trj_frame_pack_static: the frame layout step without any device allocation.

Some callers may not let a library allocate device memory: their device memory is
owned by another allocator (a framework's caching allocator or a pre-sized arena), or
their frame loop cannot take the implicit synchronisation of cudaMalloc.  For them
trj_frame_pack_static keeps its per-block scratch in a fixed 1 MiB array inside the
library (ceil(n/1024) * nsp <= 87381).  This file checks, through the C ABI, that it
lays out frames exactly as trj_frame_pack does on two calls in a row with different
frames (so nothing left in the shared array from the first call leaks into the
second), and that an oversized frame is refused.  It is collected last so that a
failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest
import torch

from trj_analysis_b200 import _lib, frames

pytestmark = pytest.mark.gpu

vp = ctypes.c_void_p


def _pack(lib, fn, ctx, xyz, sp, nsp, box, packed, counts):
    rc = getattr(lib, fn)(ctx, vp(xyz.data_ptr()), vp(sp.data_ptr()), xyz.shape[0], nsp, _lib.box3(box),
                          vp(packed.data_ptr()), vp(counts.data_ptr()), vp(torch.cuda.current_stream().cuda_stream))
    return rc


@pytest.fixture(scope="module")
def ctx():
    lib = _lib.load()
    h = vp()
    assert lib.trj_ctx_create(0, ctypes.byref(h)) == 0
    yield lib, h
    lib.trj_ctx_destroy(h)


def _frame(seed, cells, fractions):
    fr = frames.FCCSpec(cells=cells, sigma=0.2, fractions=fractions, replace_frac=0.05, seed=seed).frame(seed)
    xyz = fr.xyz.copy()
    xyz[::5] -= fr.box  # negative coordinates exercise the fold
    return fr, torch.from_numpy(xyz).cuda(), torch.from_numpy((fr.types - 1).astype(np.int32)).cuda()


def test_static_pack_matches_allocating_pack_twice(ctx):
    lib, h = ctx
    for seed, cells, fractions in [(1, (12, 12, 12), (0.5, 0.3, 0.2)), (2, (9, 10, 11), (0.25, 0.75))]:
        fr, xyz, sp = _frame(seed, cells, fractions)
        nsp = len(fractions)
        ref_p = torch.full((fr.n, 4), -7.0, device="cuda")
        ref_c = torch.zeros(nsp, dtype=torch.int64, device="cuda")
        got_p = torch.full((fr.n, 4), 3.0, device="cuda")
        got_c = torch.full((nsp,), 99, dtype=torch.int64, device="cuda")
        assert _pack(lib, "trj_frame_pack", h, xyz, sp, nsp, fr.box, ref_p, ref_c) == 0
        assert _pack(lib, "trj_frame_pack_static", h, xyz, sp, nsp, fr.box, got_p, got_c) == 0
        assert lib.trj_ctx_check(h, vp(torch.cuda.current_stream().cuda_stream)) == 0
        assert torch.equal(got_c, ref_c)
        assert torch.equal(got_p.view(torch.int32), ref_p.view(torch.int32))  # bit-exact, species bits included


def test_static_pack_rejects_oversized_frame(ctx):
    lib, h = ctx
    xyz = torch.zeros((4, 3), device="cuda")
    sp = torch.zeros(4, dtype=torch.int32, device="cuda")
    packed = torch.zeros((4, 4), device="cuda")
    counts = torch.zeros(16, dtype=torch.int64, device="cuda")
    n_too_big = (87381 // 16 + 1) * 1024  # ceil(n/1024) * 16 = 87392 > 87381
    rc = lib.trj_frame_pack_static(h, vp(xyz.data_ptr()), vp(sp.data_ptr()), n_too_big, 16, _lib.box3([1, 1, 1]),
                                   vp(packed.data_ptr()), vp(counts.data_ptr()), vp(0))
    assert rc == _lib.TRJ_ERR_CAPACITY
    assert b"fixed array" in lib.trj_ctx_last_error(h)


def test_static_pack_at_the_exact_limit(ctx):
    """ceil(n/1024) * nsp == 87381 (nsp 9, n = 9709 * 1024) is the largest frame the fixed array takes:
    it is laid out exactly as trj_frame_pack does; one atom more is refused before any launch."""
    lib, h = ctx
    nsp, n = 9, 9709 * 1024
    assert -(-n // 1024) * nsp == 87381
    g = torch.Generator(device="cuda").manual_seed(5)
    box = np.array([300.0, 310.0, 320.0], np.float32)
    xyz = (torch.rand((n, 3), device="cuda", generator=g) * 1.2 - 0.1) * torch.from_numpy(box).cuda()
    sp = torch.randint(0, nsp, (n,), device="cuda", dtype=torch.int32, generator=g)
    ref_p = torch.full((n, 4), -7.0, device="cuda")
    ref_c = torch.zeros(nsp, dtype=torch.int64, device="cuda")
    got_p = torch.full((n, 4), 3.0, device="cuda")
    got_c = torch.full((nsp,), 99, dtype=torch.int64, device="cuda")
    assert _pack(lib, "trj_frame_pack", h, xyz, sp, nsp, box, ref_p, ref_c) == 0
    assert _pack(lib, "trj_frame_pack_static", h, xyz, sp, nsp, box, got_p, got_c) == 0
    assert lib.trj_ctx_check(h, vp(torch.cuda.current_stream().cuda_stream)) == 0
    assert torch.equal(got_c, ref_c) and int(got_c.sum()) == n
    assert torch.equal(got_p.view(torch.int32), ref_p.view(torch.int32))
    del xyz, sp, ref_p, got_p
    small = torch.zeros((4, 4), device="cuda")
    rc = lib.trj_frame_pack_static(h, vp(small.data_ptr()), vp(small.data_ptr()), n + 1, nsp, _lib.box3(box),
                                   vp(small.data_ptr()), vp(got_c.data_ptr()), vp(0))
    assert rc == _lib.TRJ_ERR_CAPACITY


def test_static_pack_empty_frame_zeroes_counts(ctx):
    lib, h = ctx
    counts = torch.full((3,), 99, dtype=torch.int64, device="cuda")
    packed = torch.zeros((1, 4), device="cuda")
    rc = lib.trj_frame_pack_static(h, vp(0), vp(0), 0, 3, _lib.box3([5, 5, 5]), vp(packed.data_ptr()),
                                   vp(counts.data_ptr()), vp(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    assert lib.trj_ctx_check(h, vp(torch.cuda.current_stream().cuda_stream)) == 0
    assert counts.cpu().tolist() == [0, 0, 0]
