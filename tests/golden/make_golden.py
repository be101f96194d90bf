"""Extracts known-answer vectors from the reference's shipped example outputs.

Run in a checkout that has the reference project next to it:

    python tests/golden/make_golden.py /path/to/trj_analysis

It reads ``examples/3D/<name>/{input.nml, sq.dat, sqmix.dat, gmixsim.dat}`` and
writes ``tests/golden/examples.json`` (and, from the dynamics outputs of two examples,
``tests/golden/dynamics.json``): per example, the /INPUT_RDF/ and
/INPUT_SQ/ parameters, nsp, the header lines, the Q column (as printed), the
n(Q) column, and the r column / row count of gmixsim.dat.  The g and S values
themselves are not kept: the trajectories that produced them are not shipped,
so they cannot be regenerated.  Only the columns that depend on the box and
the input parameters alone are kept.
"""
from __future__ import annotations

import json
import os
import re
import sys

EXAMPLES = ["LJmix", "salr", "meam-dyn", "Conf", "RTIL+H20_rigid"]


def _nml_value(text: str, group: str, key: str):
    m = re.search(r"&%s(.*?)\n\s*/" % group, text, re.S | re.I)
    if not m:
        return None
    body = m.group(1)
    m2 = re.search(r"^\s*%s\s*=\s*([^!\n]*)" % key, body, re.M | re.I)
    if not m2:
        return None
    return m2.group(1).strip()


def main(ref_root: str) -> None:
    out = {}
    for name in EXAMPLES + ["2D/salr"]:
        d = os.path.join(ref_root, "examples", name if "/" in name else os.path.join("3D", name))
        nml = open(os.path.join(d, "input.nml")).read()
        ex = {
            "ndim": int(_nml_value(nml, "INPUT", "ndim")),
            "nsp": int(_nml_value(nml, "INPUT", "nsp")),
            "deltar": float(_nml_value(nml, "INPUT_RDF", "deltar")),
            "rcrdf": float(_nml_value(nml, "INPUT_RDF", "rcrdf").split("!")[0]),
            "qmax": float(_nml_value(nml, "INPUT_SQ", "qmax")),
            "qmin": float(_nml_value(nml, "INPUT_SQ", "qmin")),
        }
        sq = open(os.path.join(d, "sq.dat")).read().splitlines()
        ex["sq_header"] = sq[0]
        rows = [r.split() for r in sq[1:] if r.strip()]
        ex["sq_q"] = [r[0] for r in rows]
        ex["sq_nq"] = [int(r[-1]) for r in rows]
        mix = open(os.path.join(d, "sqmix.dat")).read().splitlines()
        ex["sqmix_header"] = mix[0]
        gpath = os.path.join(d, "gmixsim.dat")
        if os.path.exists(gpath):
            g = open(gpath).read().splitlines()
            ex["gmix_header"] = g[0]
            ex["gmix_r"] = [r.split()[0] for r in g[1:] if r.strip()]
        g1path = os.path.join(d, "gmixsim1.dat")  # nsp > 6: one file per species
        if os.path.exists(g1path):
            g = open(g1path).read().splitlines()
            ex["gmix1_header"] = g[0]
            ex["gmix1_r"] = [r.split()[0] for r in g[1:] if r.strip()]
            ex["gmix1_ncols"] = len(g[1].split())
        out[name] = ex
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "examples.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)
    dynamics(ref_root)


def _table(path):
    lines = open(path).read().splitlines()
    return lines[0], [r.split() for r in lines[1:] if r.strip()]


def dynamics(ref_root: str) -> None:
    """Known answers of the time-correlation outputs: for examples/3D/salr (F(Q,t), Fs(Q,t) and their
    transforms) and examples/3D/meam-dyn (row count of dyn.dat), the /INPUT/ frame range and
    /INPUT_DYN/, /INPUT_SQW/ keys, the header lines, and the printed columns.  fkt.dat and fskt.dat
    are the inputs of the transform that wrote sqw.dat, so the transform can be checked against them;
    C_r(t) and C_v(t) depend on the unshipped trajectory and are not kept."""
    out = {}
    for name in ["salr", "meam-dyn"]:
        d = os.path.join(ref_root, "examples", "3D", name)
        nml = open(os.path.join(d, "input.nml")).read()
        frm = [int(x) for x in _nml_value(nml, "INPUT", "ncfs_from_to").split()]

        def num(group, key, default):
            v = _nml_value(nml, group, key)
            return float(v.split("!")[0]) if v is not None else default
        ex = {"ncfs_from_to": frm, "nbuffer": int(num("INPUT_DYN", "nbuffer", 2)),
              "jump": int(num("INPUT_DYN", "jump", 1)), "tlimit": num("INPUT_DYN", "tlimit", -1.0),
              "tmax": num("INPUT_DYN", "tmax", -1.0)}
        head, rows = _table(os.path.join(d, "dyn.dat"))
        ex["dyn_header"] = head
        ex["dyn_rows"] = len(rows)
        ex["dyn_t"] = [r[0] for r in rows]
        if os.path.exists(os.path.join(d, "fkt.dat")):
            ex["qw"] = [float(x) for x in _nml_value(nml, "INPUT_SQW", "qw").split("!")[0].split()]
            for key in ("fkt", "fskt"):
                head, rows = _table(os.path.join(d, key + ".dat"))
                ex[key + "_header"] = head
                ex[key] = [r[1:] for r in rows]
            head, rows = _table(os.path.join(d, "sqw.dat"))
            ex["sqw_header"] = head
            ex["sqw"] = rows
        out[name] = ex
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dynamics.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TRJ_REFERENCE", "."))
