"""Output files in the reference's formats.

printrdf  -> gmixsim.dat (src/core/log.f90:414-596): header
             '#       r        ',9x,16('g_',2i1,'(r)',9x:), rows '(16f16.5)'
             (nsp > 6: one file gmixsim<k>.dat per species k, full rows g_k1..g_knsp).
             With charges a g_qq(r) column follows r (log.f90:456-458, 559-560: rows
             '(16f16.6)'; nsp > 6: in gmixsim1.dat only, rows '(16f16.5)', 565-567).
printSQ   -> sq.dat  (log.f90:317-412): '(2f15.7,i12)' or, for 2 species with all
             bsc = 1, '(6f15.7,i12)' with S_NN, S_cc, S_11, S_22, S_12, n(Q);
             with charges S_qq(Q) follows S_NN ('(3f15.7,i12)' / '(7f15.7,i12)',
             log.f90:353-362, 385-394); sqmix.dat '(15f16.7)' with S_aa per species.
freud-style tools -> gr.dat / Sq.dat as numpy.savetxt writes them ('%.18e', header
             '# r g(r)' / '# k S(k)'); species-resolved columns are appended.

Fortran fixed-point edit descriptors are emulated: values are rounded half away
from zero from their exact binary value; a record holds at most the repeat count
of items and continues on the next line (format reversion); a value wider than the
field prints as asterisks; an i1 field of a value >= 10 prints '*'.
"""
from __future__ import annotations

import decimal
from typing import Iterable, List, Optional, Sequence

import numpy as np


def fmt_f(value: float, width: int, decimals: int) -> str:
    d = decimal.Decimal(float(value)).quantize(decimal.Decimal(1).scaleb(-decimals),
                                               rounding=decimal.ROUND_HALF_UP)
    s = f"{d:.{decimals}f}"
    if s.startswith("-") and d == 0:
        s = s  # keep the sign, as formatted Fortran output does for tiny negatives
    if len(s) > width:
        return "*" * width
    return s.rjust(width)


def fmt_i(value: int, width: int) -> str:
    s = str(int(value))
    return "*" * width if len(s) > width else s.rjust(width)


def _records(values: Sequence[float], per_line: int, width: int, decimals: int) -> List[str]:
    lines = []
    for k in range(0, len(values), per_line):
        lines.append("".join(fmt_f(v, width, decimals) for v in values[k:k + per_line]))
    return lines or [""]


def _i1(v: int) -> str:
    return str(v) if 0 <= v <= 9 else "*"


def _group_header(prefix: str, labels: Sequence[str], per_line: int, sep: str) -> List[str]:
    """Header with a repeated group ('label', sep) and reversion after per_line groups."""
    lines = []
    for k in range(0, len(labels), per_line):
        chunk = labels[k:k + per_line]
        body = sep.join(chunk)
        lines.append((prefix if k == 0 else "") + body)
    return lines or [prefix.rstrip()]


def write_gmixsim(path_dir: str, r: np.ndarray, g: np.ndarray, nsp: int,
                  g_qq: Optional[np.ndarray] = None) -> List[str]:
    """g: (nrows, nsp, nsp) symmetric partial g_ab(r); g_qq: (nrows,) charge-charge g(r) or None.
    Returns the files written."""
    import os
    files = []
    qhead = "#       r        " + " " * 9 + ("g_qq(r)" + " " * 9 if g_qq is not None else "")
    if nsp <= 6:
        labels = [f"g_{_i1(j + 1)}{_i1(k + 1)}(r)" for j in range(nsp) for k in range(j, nsp)]
        head = _group_header(qhead, labels, 16, " " * 9)
        rows = []
        for i in range(r.shape[0]):
            vals = [r[i]] + ([g_qq[i]] if g_qq is not None else []) + \
                [g[i, j, k] for j in range(nsp) for k in range(j, nsp)]
            rows.extend(_records(vals, 16, 16, 6 if g_qq is not None else 5))
        p = os.path.join(path_dir, "gmixsim.dat")
        with open(p, "w") as f:
            f.write("\n".join(head + rows) + "\n")
        files.append(p)
    else:
        for k in range(nsp):
            labels = [f"g_{_i1(k + 1)}{_i1(j + 1)}(r)" for j in range(nsp)]
            withq = g_qq is not None and k == 0
            head = _group_header(qhead if withq else "#       r        " + " " * 9, labels, 16, " " * 9)
            rows = []
            for i in range(r.shape[0]):
                vals = [r[i]] + ([g_qq[i]] if withq else []) + [g[i, k, j] for j in range(nsp)]
                rows.extend(_records(vals, 16, 16, 5))
            p = os.path.join(path_dir, f"gmixsim{k + 1}.dat")
            with open(p, "w") as f:
                f.write("\n".join(head + rows) + "\n")
            files.append(p)
    return files


SQ_HEADER_BINARY = ("#           Q        S_NN(Q)          S_cc(Q)       S_11(Q)        S_22(Q)"
                    "           S_12(Q)         n(Q)")
SQ_HEADER = "#           Q       S_NN(Q)          n(Q)"
SQ_HEADER_BINARY_QQ = ("#           Q        S_NN(Q)          S_qq(Q)          S_cc(Q)       S_11(Q)        S_22(Q)"
                       "           S_12(Q)         n(Q)")
SQ_HEADER_QQ = "#           Q       S_NN(Q)          S_qq(Q)          n(Q)"


def sqmix_header(nsp: int) -> List[str]:
    labels = [f"S_{_i1(j + 1)}{_i1(j + 1)}(Q)" for j in range(nsp)]
    return _group_header("#       Q" + " " * 14, labels, 15, " " * 9)


def write_sq(path_dir: str, q: np.ndarray, s_nn: np.ndarray, nq: np.ndarray, s_self: np.ndarray,
             binary: dict = None, s_qq: Optional[np.ndarray] = None) -> List[str]:
    """q, s_nn, nq: rows 1..nqmax; s_self: (nrows, nsp); binary: scc, s11, s22, s12 arrays;
    s_qq: charge-charge S(Q) rows or None."""
    import os
    if s_qq is not None:
        lines = [SQ_HEADER_BINARY_QQ if binary is not None else SQ_HEADER_QQ]
    else:
        lines = [SQ_HEADER_BINARY if binary is not None else SQ_HEADER]
    for i in range(q.shape[0]):
        qq = [s_qq[i]] if s_qq is not None else []
        if binary is not None:
            vals = [q[i], s_nn[i]] + qq + [binary["scc"][i], binary["s11"][i], binary["s22"][i], binary["s12"][i]]
        else:
            vals = [q[i], s_nn[i]] + qq
        lines.append("".join(fmt_f(v, 15, 7) for v in vals) + fmt_i(nq[i], 12))
    p1 = os.path.join(path_dir, "sq.dat")
    with open(p1, "w") as f:
        f.write("\n".join(lines) + "\n")
    nsp = s_self.shape[1]
    mix = sqmix_header(nsp)
    for i in range(q.shape[0]):
        mix.extend(_records([q[i]] + list(s_self[i]), 15, 16, 7))
    p2 = os.path.join(path_dir, "sqmix.dat")
    with open(p2, "w") as f:
        f.write("\n".join(mix) + "\n")
    return [p1, p2]


def savetxt_columns(path: str, columns: Iterable[np.ndarray], header: str) -> None:
    np.savetxt(path, np.column_stack(list(columns)), header=header)


def format_record(values: Sequence[float], descs: Sequence[tuple]) -> List[str]:
    """Values written with the F edit descriptors ``descs`` [(width, decimals), ...]; when the list
    outlasts the format, a new record starts at the format's beginning (reversion to the whole
    format, which has no inner parentheses)."""
    lines, cur, k = [], "", 0
    for v in values:
        if k == len(descs):
            lines.append(cur)
            cur, k = "", 0
        w, d = descs[k]
        cur += fmt_f(v, w, d)
        k += 1
    lines.append(cur)
    return lines


ROW_T8 = [(10, 3)] + [(15, 5)] * 8            # '(f10.3,8f15.5)'
ROW_2T8 = [(10, 3), (10, 3)] + [(15, 5)] * 8  # '(2f10.3,8f15.5)'


def write_dynamics(path_dir: str, res: dict, units: str = "lj") -> List[str]:
    """print_rtcor (src/modules/dynamics.cuf:278-393) without velocities or stresses:
    dyn.dat   '#',2x,'t(tau)',9x,'C_r(t)'                  rows (f10.3,8f15.5) t, C_r, i <= itlimit
    fkt.dat   '#',2x,'t(tau)',9x,8('F(',f6.4,',t)',4x:)    rows (f10.3,8f15.5) t, F(q_1..q_nqw, t)
    fskt.dat  the same with 'Fs('
    sqw.dat   '#',2x,'w(1/tau)',5x,8('S(',f6.4,',w)    Ss(',f6.4,',w)',4x:)
              rows (f10.3,8f15.5) w/2pi, S(q_1,w), Ss(q_1,w), ... for every lag row;
    other units: 't(ps)', and sqw.dat '#',2x,'w(THz)',7x,'w(meV)',5x,... rows (2f10.3,8f15.5)
    with w/2pi and 4.135 w/2pi."""
    import os
    lj = units == "lj"
    tl = "t(tau)" if lj else "t(ps)"
    t, qw = res["t"], res["qw"]
    ndyn = t.shape[0]
    rows_t = [i for i in range(ndyn) if i + 1 <= res["itlimit"]]
    files = []

    def emit(name, lines):
        p = os.path.join(path_dir, name)
        with open(p, "w") as f:
            f.write("\n".join(lines) + "\n")
        files.append(p)

    emit("dyn.dat", ["#  " + tl + " " * 9 + "C_r(t)"] +
         [ln for i in rows_t for ln in format_record([t[i], res["r2t"][i]], ROW_T8)])
    if len(qw) == 0:  # run_dyn without run_sqw: C_r(t) only
        return files
    for name, key, lab in (("fkt.dat", "fkt", "F("), ("fskt.dat", "fskt", "Fs(")):
        head = _group_header("#  " + tl + " " * 9, [f"{lab}{fmt_f(q, 6, 4)},t)" for q in qw], 8, " " * 4)
        emit(name, head + [ln for i in rows_t for ln in format_record([t[i]] + list(res[key][i]), ROW_T8)])
    pi = np.float32(3.141592653589793)
    twopi = np.float32(np.float32(2) * pi)
    labels = [f"S({fmt_f(q, 6, 4)},w)    Ss({fmt_f(q, 6, 4)},w)" for q in qw]
    if lj:
        head = _group_header("#  w(1/tau)" + " " * 5, labels, 8, " " * 4)
    else:
        head = _group_header("#  w(THz)" + " " * 7 + "w(meV)" + " " * 5, labels, 8, " " * 4)
    lines = []
    for i in range(ndyn):
        f = np.float32(res["w"][i] / twopi)
        vals = [v for j in range(len(qw)) for v in (res["sqw"][i, j], res["ssqw"][i, j])]
        if lj:
            lines.extend(format_record([f] + vals, ROW_T8))
        else:
            lines.extend(format_record([f, np.float32(np.float32(4.135) * res["w"][i] / twopi)] + vals, ROW_2T8))
    emit("sqw.dat", head + lines)
    return files


def write_s2n(path_dir: str, r: np.ndarray, s2n: np.ndarray) -> str:
    """s2n.dat of printrdf (log.f90:449, 482, 532): header '#       r',16x,'s2n', rows '(18f16.5)' r, s2n."""
    import os
    lines = ["#       r" + " " * 16 + "s2n"]
    for i in range(r.shape[0]):
        lines.extend(_records([r[i], s2n[i]], 18, 16, 5))
    p = os.path.join(path_dir, "s2n.dat")
    with open(p, "w") as f:
        f.write("\n".join(lines) + "\n")
    return p


def write_gxy(path_dir: str, r: np.ndarray, g: np.ndarray, nsp: int, zslice: Sequence[float]) -> List[str]:
    """printrdf for slabs (log.f90:424-432, 546-554): gxy_<i>-<j>.dat for i <= j, header
    '#     r        ',3x,16('g_xy(r,',f7.2,')',3x:), rows '(15f16.7)' r, g_xy(r, slice 1..nslice)."""
    import os
    files = []
    labels = [f"g_xy(r,{fmt_f(z, 7, 2)})" for z in zslice]
    for i in range(nsp):
        for j in range(i, nsp):
            lines = _group_header("#     r        " + " " * 3, labels, 16, " " * 3)
            for k in range(r.shape[0]):
                lines.extend(_records([r[k]] + list(g[k, i, j]), 15, 16, 7))
            p = os.path.join(path_dir, f"gxy_{_i1(i + 1)}-{_i1(j + 1)}.dat")
            with open(p, "w") as f:
                f.write("\n".join(lines) + "\n")
            files.append(p)
    return files


def write_sqxy(path_dir: str, q: np.ndarray, s_xy: np.ndarray, s_pxy: np.ndarray, zslice: Sequence[float]) -> List[str]:
    """printSQ for slabs (log.f90:337-349, 364-376): sqxy.dat and sqpxy_<j>-<j>.dat, header
    '#     Q        ',3x,16('S_xy(Q,',f7.2,')',3x:), rows '(15f16.7)' Q, S(Q, slice 1..nslice)."""
    import os
    labels = [f"S_xy(Q,{fmt_f(z, 7, 2)})" for z in zslice]
    files = []

    def emit(name, rows):
        lines = _group_header("#     Q        " + " " * 3, labels, 16, " " * 3)
        for k in range(q.shape[0]):
            lines.extend(_records([q[k]] + list(rows[k]), 15, 16, 7))
        p = os.path.join(path_dir, name)
        with open(p, "w") as f:
            f.write("\n".join(lines) + "\n")
        files.append(p)

    emit("sqxy.dat", s_xy)
    for j in range(s_pxy.shape[1]):
        emit(f"sqpxy_{_i1(j + 1)}-{_i1(j + 1)}.dat", s_pxy[:, j, :])
    return files
