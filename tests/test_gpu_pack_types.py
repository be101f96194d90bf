"""The layout step with the type-to-species table on the device (trj_frame_pack_types) against the
host-numbered layout (trj_frame_pack): identical packed frames and counts; a type outside the table
or not selected is reported as bad data."""
import numpy as np
import pytest
import torch

from trj_analysis_b200 import analysis, frames

pytestmark = pytest.mark.gpu


def test_pack_types_equals_host_numbering():
    from trj_analysis_b200 import _lib, engine
    ctx = engine.Context(0)
    spec = frames.FCCSpec(cells=(7, 7, 7), fractions=(0.5, 0.3, 0.2), seed=9)
    fr = spec.frame(0)
    # selected types 3, 1, 2 -> species by first appearance of a selected type
    sess = analysis.Session(analysis.Config(nsp=3, sp_types_selected=(3, 1, 2)), ctx=ctx)
    species = sess._species_of(fr.types)
    lut = torch.from_numpy(sess.species_lut.astype(np.int32)).to(ctx.torch_device)
    a = engine.FrameStage(ctx, fr.n, 3)
    b = engine.FrameStage(ctx, fr.n, 3)
    a.upload_and_pack(fr.xyz, species, fr.box)
    b.upload_and_pack_types(fr.xyz, fr.types, fr.box, lut)
    ctx.check()
    assert torch.equal(a.packed, b.packed)
    assert torch.equal(a.counts, b.counts)
    bad = fr.types.copy()
    bad[17] = 9  # outside the table
    b.upload_and_pack_types(fr.xyz, bad, fr.box, lut)
    with pytest.raises(_lib.TrjError, match="TRJ_ERR_DATA"):
        ctx.check()
    ctx.close()


def test_session_fast_layout_matches_first_frame_path():
    """A trajectory analysed frame by frame gives the same counts whether frames 2.. take the device
    type table or the host numbering."""
    spec = frames.FCCSpec(cells=(8, 8, 8), sigma=0.1, fractions=(0.6, 0.4), seed=10)
    frs = list(spec.frames(3))
    cfg = analysis.Config(nsp=2, sp_types_selected=(1, 2), run_sq=False, deltar=0.05)
    s1 = analysis.Session(cfg).run(frs)
    assert s1._lut_dev is not None
    s2 = analysis.Session(cfg)
    s2._fast_layout = lambda frame: False  # host numbering for every frame
    s2.run(frs)
    np.testing.assert_array_equal(s1.rdf_transfer(), s2.rdf_transfer())
    np.testing.assert_array_equal(s1.ntype, s2.ntype)
    s1.close()
    s2.close()
