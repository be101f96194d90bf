"""The g(r)/S(Q) part of the reference program's run: python trj_analysis.py input.nml [GPU id].

Reads the namelist groups /INPUT/ (nsp, trj_input_file, ncfs_from_to, the rdf and S(Q)
switches), /INPUT_SP/ (sp_types_selected), /INPUT_RDF/ (deltar, rcrdf) and /INPUT_SQ/
(qmax, qmin, bsc) as src/io/input.f90 does, runs every selected frame through the B200
kernels and writes gmixsim.dat (printrdf) and sq.dat / sqmix.dat (printSQ) in the current
directory, in the reference's formats.  The trajectory is a classic NetCDF file (AMBER
convention) or .npz; frames ncfs_from_to = (count, first, stride) as the reference reads them.
"""
from __future__ import annotations

import argparse
import sys

if __package__ in (None, ""):
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("input_nml")
    ap.add_argument("gpu", nargs="?", type=int, default=0)
    ap.add_argument("--kset", default="ref", help="ref (reference octant + axes) | full | full+axes | full+sampled")
    ap.add_argument("--method", default="split", choices=["split", "plain"])
    ap.add_argument("--outdir", default=".")
    a = ap.parse_args(argv)

    import itertools

    from trj_analysis_b200 import analysis, frames as fmod, namelist

    groups = namelist.read(a.input_nml)
    cfg = namelist.config_from_namelist(groups)
    cfg.kset = a.kset
    cfg.method = a.method
    inp = groups.get("INPUT", {})
    traj = fmod.open_trajectory(str(inp.get("trj_input_file", "run.nc")))
    ncfs = inp.get("ncfs_from_to", [0, 1, 1])
    ncfs = list(ncfs) if isinstance(ncfs, list) else [ncfs]
    ncfs = (ncfs + [0, 1, 1])[:3]
    count, first, stride = int(ncfs[0]), max(1, int(ncfs[1])), max(1, int(ncfs[2]))
    frames_iter = itertools.islice(iter(traj), first - 1, None, stride)
    if count > 0:
        frames_iter = itertools.islice(frames_iter, count)
    sess = analysis.Session(cfg, device=a.gpu)
    sess.run(frames_iter)
    files = []
    if cfg.run_rdf:
        files += sess.printrdf(a.outdir)
        print(f" *** Suggested rcl (NN and/or connectivity distance): {sess.suggested_rcl():10.4f}")
    if cfg.run_sq:
        files += sess.printSQ(a.outdir)
    print(f" ** {sess.nconf} configurations analysed; wrote {', '.join(files)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
