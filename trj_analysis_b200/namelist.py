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
    from .analysis import Config
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
    return Config(nsp=nsp, sp_types_selected=sel[:nsp], run_rdf=flags[0], run_sq=flags[1],
                  deltar=float(rdf.get("deltar", 0.02)), rcrdf=float(rdf.get("rcrdf", 0.0)),
                  qmax=float(sq.get("qmax", -1.0)), qmin=float(sq.get("qmin", 0.0)), bsc=bsc, kset="ref")
