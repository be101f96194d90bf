"""S(k) of a trajectory: the call shape and output of the reference's tools/fast_sq_freud_netcdf.py.

    python fast_sq_freud_netcdf.py traj.nc       -> Sq.dat  ('# k S(k)' + one row per bin)

Like the reference script: 60 linear bins on [k_min, k_max] with k_min = 2 pi / max(L)
and k_max = 0.5, every lattice vector of the (first frame's) box in that range, accumulated
over all frames; S(k) = sum |rho(k)|^2 / (N * vectors * frames) per bin at the bin centre.
Columns S_aa(k) = sum |rho_a(k)|^2 / (N_a * vectors * frames) of every species (types
numbered by first appearance) follow the two reference columns.  Bins without a lattice
vector print nan.  The sums run in the B200 library (FP32 direct sum with exact phase
reduction for these short vector lists).
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

BINS = 60
K_MAX = 0.5


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("trajfile")
    ap.add_argument("--bins", type=int, default=BINS)
    ap.add_argument("--k-max", type=float, default=K_MAX)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--method", default="plain", choices=["plain", "split"])
    ap.add_argument("--out", default="Sq.dat")
    a = ap.parse_args(argv)

    from trj_analysis_b200 import engine, frames as fmod, refsem

    traj = fmod.open_trajectory(a.trajfile)
    ctx = engine.Context(a.device)
    plan = out = stage = ks = None
    nframes = 0
    for k, fr in enumerate(traj):
        sp, wtypes = species_of(fr.types)
        nsp = len(wtypes)
        if plan is None:
            k_min = 2.0 * math.pi / float(np.max(fr.box))
            ks = refsem.linear_kset(fr.box, k_min, a.k_max, a.bins)
            counts = np.bincount(sp, minlength=nsp)
            stage = engine.FrameStage(ctx, fr.n, nsp)
            plan = engine.SqPlan(ctx, nsp, ks, counts)
            out = plan.new_out()
        n = stage.upload_and_pack(fr.xyz, sp, fr.box)
        plan.accumulate(stage.packed, n, fr.box, out, engine.METHODS[a.method])
        nframes += 1
        if k % 10 == 0:
            print("processed frame", k)
    ctx.check()
    res = out.cpu().numpy()
    nq = ks.nq.astype(np.float64)
    n_tot = float(counts.sum())
    total = np.zeros(ks.nbins)
    for r, (x, y) in enumerate(refsem.pair_rows(nsp)):
        total += (1.0 if x == y else 2.0) * res[:, r]
    with np.errstate(divide="ignore", invalid="ignore"):
        den = np.where(nq > 0, nq, np.nan) * nframes
        S = total / (n_tot * den)
        centers = k_min + (np.arange(ks.nbins) + 0.5) * ks.dq
        cols, names = [centers, S], ["k", "S(k)"]
        if nsp > 1:
            for x in range(nsp):
                cols.append(res[:, refsem.pair_row(x, x, nsp)] / (counts[x] * den))
                names.append(f"S_{x + 1}{x + 1}(k)")
    np.savetxt(a.out, np.column_stack(cols), header=" ".join(names))
    print("Finished. Frames processed:", nframes)
    return 0


if __name__ == "__main__":
    sys.exit(main())
