"""The g(r)/S(Q)/dynamics part of the reference program's run: python trj_analysis.py input.nml [GPU id].

Reads the namelist groups /INPUT/ (ndim, nsp, nslice, trj_input_file, ncfs_from_to, the module
switches), /INPUT_SP/ (sp_types_selected), /INPUT_RDF/ (deltar, rcrdf, nrandom), /INPUT_SQ/
(qmax, qmin, bsc), /INPUT_CONF/ (zslice, zgrid), /INPUT_DYN/ and /INPUT_SQW/ as src/io/input.f90
does, runs the selected frames through the B200 kernels and writes, in the reference's formats,
gmixsim.dat (+ s2n.dat), sq.dat / sqmix.dat, the slab files gxy_*.dat / sqxy.dat / sqpxy_*.dat,
and dyn.dat / fkt.dat / fskt.dat / sqw.dat.  The trajectory is a classic NetCDF file (AMBER
convention, with charges q and times when present) or .npz; ncfs_from_to = (count, from, to) as the
reference reads it (trj_analysis.f90:173-198).
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

    from trj_analysis_b200 import analysis, frames as fmod, namelist

    groups = namelist.read(a.input_nml)
    cfg = namelist.config_from_namelist(groups)
    cfg.kset = a.kset
    cfg.method = a.method
    inp = groups.get("INPUT", {})
    traj = fmod.open_trajectory(str(inp.get("trj_input_file", "run.nc")))
    ncfs = inp.get("ncfs_from_to", [0, 0, 0])
    ncfs = list(ncfs) if isinstance(ncfs, list) else [ncfs]
    probe = traj.frame(max(0, int((ncfs + [0, 1])[1]) - 1)) if len(traj) else None
    first_zero = probe is not None and probe.time is not None and probe.time == 0
    order = namelist.frame_schedule(ncfs, len(traj), first_zero)
    if cfg.dyn is not None:
        cfg.dyn.tstep = fmod.tstep_of(traj)
        cfg.units = "lj" if traj.time_units == "lj" else "ps"

    def frames_iter():
        for f in order:
            fr = traj.frame(f)
            if fr.time is not None and fr.time == 0:  # step 0 is read but not analysed (trj_analysis.f90:196-198)
                continue
            yield fr

    count = int((ncfs + [0])[0]) or len(traj)
    sess = analysis.Session(cfg, device=a.gpu, nconf_total=min(count, len(traj)))  # Nconf (util.f90:128-145)
    sess.run(frames_iter())
    files = []
    if cfg.slab is not None:
        files += sess.print_slabs(a.outdir)
    else:
        if cfg.run_rdf:
            files += sess.printrdf(a.outdir)
            print(f" *** Suggested rcl (NN and/or connectivity distance): {sess.suggested_rcl():10.4f}")
        if cfg.run_sq:
            files += sess.printSQ(a.outdir)
    if cfg.run_sqw and sess.dyn is not None:
        files += sess.print_rtcor(a.outdir)
    print(f" ** {sess.nconf} configurations analysed; wrote {', '.join(files)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
