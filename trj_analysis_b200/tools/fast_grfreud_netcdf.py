"""g(r) of a trajectory: the call shape and output of the reference's tools/fast_grfreud_netcdf.py.

    python fast_grfreud_netcdf.py traj.nc        -> gr.dat  ('# r g(r)' + one row per bin)

Like the reference script: 200 bins on [0, r_max) with r_max = 150, every atom a
point and a query point (i != j), accumulated over all frames.  Differences: the pair
histogram comes from the B200 kernel (exact integer counts); r_max is clipped below
half the smallest box edge (the reference's 150 exceeds L/2 for ordinary boxes, which
its RDF cannot use) and the clip is reported; columns g_ab(r) of every species pair
(types numbered by first appearance) follow the two reference columns.
g(r_i) = 2 H_i / (frames * N * (N / V) * dV_i), dV_i = 4 pi/3 (r_{i+1}^3 - r_i^3).
Accepts classic NetCDF (AMBER convention: coordinates, cell_lengths, optional type) or .npz.
"""
from __future__ import annotations

import argparse
import math
import sys

import numpy as np

if __package__ in (None, ""):
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

from trj_analysis_b200.tools._common import species_of  # noqa: E402

BINS = 200
R_MAX = 150.0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("trajfile")
    ap.add_argument("--bins", type=int, default=BINS)
    ap.add_argument("--r-max", type=float, default=R_MAX)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default="gr.dat")
    a = ap.parse_args(argv)

    import torch
    from trj_analysis_b200 import engine, frames as fmod, refsem

    traj = fmod.open_trajectory(a.trajfile)
    ctx = engine.Context(a.device)
    rdf = hist = stage = None
    nframes, natoms, vol_sum = 0, 0, 0.0
    r_max = a.r_max
    for k, fr in enumerate(traj):
        sp, wtypes = species_of(fr.types)
        nsp = len(wtypes)
        if rdf is None:
            half = float(np.min(fr.box)) / 2.0
            if r_max >= half:
                r_max = float(np.nextafter(np.float32(half), np.float32(0)))
                print(f" r_max {a.r_max} >= L/2; clipped to {r_max:.6f}")
            stage = engine.FrameStage(ctx, fr.n, nsp)
            rdf = engine.RdfPlan(ctx, nsp, r_max / a.bins, r_max, fr.box, fr.n, floor_bins=a.bins)
            hist = rdf.new_hist()
            counts = np.bincount(sp, minlength=nsp)
        print(" Processing frame ", k)
        n = stage.upload_and_pack(fr.xyz, sp, fr.box)
        rdf.accumulate(stage.packed, n, fr.box, hist)
        nframes += 1
        natoms = n
        vol_sum += refsem.volume(fr.box)
        if k % 10 == 0:
            print("processed frame", k)
    ctx.check()
    H = hist.cpu().numpy().astype(np.float64)
    dr = r_max / a.bins
    edges = np.arange(a.bins + 1) * dr
    dv = 4.0 * math.pi / 3.0 * (edges[1:] ** 3 - edges[:-1] ** 3)
    vol = vol_sum / nframes
    r = 0.5 * (edges[1:] + edges[:-1])
    g_tot = 2.0 * H.sum(axis=0) / (nframes * natoms * (natoms / vol) * dv)
    cols, names = [r, g_tot], ["r", "g(r)"]
    if nsp > 1:
        for x in range(nsp):
            for y in range(x, nsp):
                row = refsem.pair_row(x, y, nsp)
                fac = 2.0 if x == y else 1.0
                cols.append(fac * H[row] / (nframes * counts[x] * (counts[y] / vol) * dv))
                names.append(f"g_{x + 1}{y + 1}(r)")
    np.savetxt(a.out, np.column_stack(cols), header=" ".join(names))
    print("Finished. Frames processed:", nframes)
    return 0


if __name__ == "__main__":
    sys.exit(main())
