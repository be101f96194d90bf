"""Failure handling without a fault: a device wait that runs out.

The reference prints the CUDA error and stops (rdf.cuf:241-242).  Here every device wait is
bounded: when one runs out, the kernel sets TRJ_DEV_TIMEOUT, lets its copies in flight land and
returns, and trj_ctx_check reports TRJ_ERR_TIMEOUT.  The pair kernel's stall test makes each warp's
first wait target a barrier that nothing arrives on, with a limit of about 10 ms, so the timeout path
runs on every launch; afterwards the same context and plan count a frame bit-exact.
"""
import numpy as np
import pytest
import torch

from oracle import orc
from trj_analysis_b200 import _lib, frames, refsem
from trj_analysis_b200._lib import TrjError

pytestmark = pytest.mark.gpu


def test_pair_kernel_wait_timeout_then_recovery():
    from trj_analysis_b200 import engine
    ctx = engine.Context(0)
    spec = frames.FCCSpec(cells=(10, 10, 10), sigma=0.1, fractions=(0.5, 0.5), seed=13)
    fr = spec.frame(0)
    stage = engine.FrameStage(ctx, fr.n, 2)
    n = stage.upload_and_pack(fr.xyz, fr.types - 1, fr.box)
    rdf = engine.RdfPlan(ctx, 2, 0.02, 2.5, fr.box, fr.n)
    with pytest.raises(TrjError):
        rdf.set_wait(10, False)  # below the accepted range
    rdf.set_wait(20_000_000, stall_test=True)
    hist = rdf.new_hist()
    rdf.accumulate(stage.packed, n, fr.box, hist)
    with pytest.raises(TrjError) as ei:
        ctx.check()
    assert ei.value.code == _lib.TRJ_ERR_TIMEOUT
    ctx.check()  # the status was cleared by the report
    # the same plan, back to the default limit: the next frame is counted exactly
    rdf.set_wait(0, False)
    hist = rdf.new_hist()
    edge = torch.zeros(4, dtype=torch.int64, device=ctx.torch_device)
    rdf.accumulate(stage.packed, n, fr.box, hist, edge)
    ctx.check()
    pos, sp, _ = orc.layout(fr.xyz, fr.types - 1, fr.box, 2)
    p = refsem.rdf_params(2, 0.02, 2.5, fr.box)
    h_o, e_o = orc.rdf_counts(pos, sp, fr.box, p.side2, p.deltar, p.lsmax, 2, cells=True)
    assert np.array_equal(hist.cpu().numpy().astype(np.uint64), h_o)
    assert np.array_equal(edge.cpu().numpy()[:3].astype(np.uint64), e_o)
    rdf.close()
    ctx.close()
