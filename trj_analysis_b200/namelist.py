"""Reader for the Fortran namelist input of the reference (src/io/input.f90:64-75).

Only what the g(r)/S(Q) path needs is interpreted (see ``config_from_namelist``); the
parser itself accepts any group: ``&NAME key=value ... /`` with integers, reals (also
``d`` exponents), quoted strings, logicals (T, F, .true., .false.), space- or
comma-separated arrays, repeat counts (``3*0``) and ``!`` comments.
"""
from __future__ import annotations

import re
from typing import Dict, List, Union

Value = Union[int, float, str, bool, List]


def _atom(tok: str):
    t = tok.strip()
    if not t:
        return None
    if t[0] in "'\"":
        return t[1:-1] if len(t) >= 2 and t[-1] == t[0] else t[1:]
    lo = t.lower()
    if lo in ("t", ".true.", "true", ".t."):
        return True
    if lo in ("f", ".false.", "false", ".f."):
        return False
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(lo.replace("d", "e"))
    except ValueError:
        return t


def _values(text: str) -> List:
    toks = re.findall(r"'[^']*'|\"[^\"]*\"|[^\s,]+", text)
    out: List = []
    for tok in toks:
        m = re.fullmatch(r"(\d+)\*(.+)", tok)
        if m and tok[0] not in "'\"":
            out.extend([_atom(m.group(2))] * int(m.group(1)))
        else:
            out.append(_atom(tok))
    return out


def parse(text: str) -> Dict[str, Dict[str, Value]]:
    # strip comments outside quotes
    lines = []
    for line in text.splitlines():
        buf, q = [], None
        for ch in line:
            if q:
                buf.append(ch)
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                buf.append(ch)
            elif ch == "!":
                break
            else:
                buf.append(ch)
        lines.append("".join(buf))
    body = "\n".join(lines)
    groups: Dict[str, Dict[str, Value]] = {}
    for m in re.finditer(r"&(\w+)(.*?)(?:^\s*/|/\s*$)", body, re.S | re.M):
        name = m.group(1).upper()
        content = m.group(2)
        parts = re.split(r"(\b[A-Za-z_]\w*(?:\(\s*\d+\s*\))?)\s*=", content)
        g: Dict[str, Value] = {}
        for k in range(1, len(parts) - 1, 2):
            key = parts[k].strip().lower()
            vals = _values(parts[k + 1])
            g[key] = vals[0] if len(vals) == 1 else vals
        groups[name] = g
    return groups


def read(path: str) -> Dict[str, Dict[str, Value]]:
    with open(path) as f:
        return parse(f.read())


def _list(v) -> List:
    return list(v) if isinstance(v, list) else [v]


def config_from_namelist(groups: Dict[str, Dict[str, Value]]):
    """Config of the g(r)/S(Q) path from /INPUT/, /INPUT_SP/, /INPUT_RDF/, /INPUT_SQ/ (input.f90:78-217)."""
    from .analysis import Config, SlabConfig
    from .dynamics import DynConfig
    inp = groups.get("INPUT", {})
    sp = groups.get("INPUT_SP", {})
    rdf = groups.get("INPUT_RDF", {})
    sq = groups.get("INPUT_SQ", {})
    nsp = int(inp.get("nsp", 1))
    flags = [bool(x) for x in _list(inp.get("rdf_sq_cl_dyn_sqw_conf_ord", [True, True]))]
    flags += [False] * (7 - len(flags))
    sel = [int(x) for x in _list(sp.get("sp_types_selected", list(range(1, nsp + 1))))]
    if len(sel) < nsp:  # unset entries default to 0 in the reference; number the rest by type id
        sel = sel + [t for t in range(1, 64) if t not in sel][: nsp - len(sel)]
    bsc = sq.get("bsc")
    bsc = [float(x) for x in _list(bsc)] if bsc is not None else [1.0] * nsp
    bsc = (bsc + [1.0] * nsp)[:nsp]
    cfg = Config(nsp=nsp, sp_types_selected=sel[:nsp], run_rdf=flags[0], run_sq=flags[1],
                 deltar=float(rdf.get("deltar", 0.02)), rcrdf=float(rdf.get("rcrdf", 0.0)),
                 qmax=float(sq.get("qmax", -1.0)), qmin=float(sq.get("qmin", 0.0)), bsc=bsc, kset="ref",
                 ndim=int(inp.get("ndim", 3)), nrandom=int(rdf.get("nrandom", 0)))
    # /INPUT_CONF/ with the confinement switch and g(r) or S(Q): the slab analysis (input.f90:171-191)
    if flags[5] and (flags[0] or flags[1]):
        conf = groups.get("INPUT_CONF", {})
        nslice = int(inp.get("nslice", 1))
        zs = [float(x) for x in _list(conf.get("zslice", [0.0]))][:max(1, nslice)]
        cfg.slab = SlabConfig(zslice=tuple(zs), zgrid=float(conf.get("zgrid", 1.0)))
    # /INPUT_DYN/, /INPUT_SQW/: time correlations (flags 4 and 5, util.f90:175-180)
    if flags[3] or flags[4]:
        dyn = groups.get("INPUT_DYN", {})
        sqw = groups.get("INPUT_SQW", {})
        qw = [float(x) for x in _list(sqw.get("qw", []))] if flags[4] else []
        cfg.run_sqw = True
        cfg.dyn = DynConfig(nbuffer=int(dyn.get("nbuffer", 2)), jump=int(dyn.get("jump", 1)),
                            tlimit=float(dyn.get("tlimit", -1.0)), tmax=float(dyn.get("tmax", -1.0)),
                            qw=tuple(qw))
    return cfg


def frame_schedule(ncfs_from_to, nframes: int, first_step_is_zero: bool = False) -> List[int]:
    """0-based trajectory frames the reference reads for ncfs_from_to = (count, from, to)
    (trj_analysis.f90:173-183 with reset_confs, util.f90:128-145): count = 0 means every frame;
    ``to`` is increased by one; frame i (1..count) is from + (i-1)*(to-from)/count in integer
    arithmetic, one later when the ``from`` frame is step 0 and from = 1; reading stops at the end
    of the file."""
    v = (list(ncfs_from_to) + [0, 0, 0])[:3]
    count, frm, to = int(v[0]), int(v[1]), int(v[2])
    if count == 0:
        count, frm, to = nframes, 1, nframes
    to += 1
    shift = 1 if (first_step_is_zero and frm == 1) else 0
    out = []
    for i in range(1, count + 1):
        ncstart = frm + (i - 1) * (to - frm) // count + shift
        if ncstart < 1 or ncstart > nframes:
            break
        out.append(ncstart - 1)
    return out
