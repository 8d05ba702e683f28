"""Text interchange formats of a CDT.

* The reference's own CDT text file (``saveCDT`` / ``readCDT``,
  GPU_Refine/mesh.cpp:402-532): the point, triangle and segment counts on
  three lines, then one line per point ``x y``, per triangle ``a b c``, per
  triangle its neighbours ``n0 n1 n2`` and per segment ``a b``; zero-based
  indices.  The reference prints coordinates with ``%lf`` (six decimals);
  :func:`write_reference_cdt` does the same by default (``exact=False``) and
  can write every coordinate exactly instead (17 significant digits), which
  the same reader reads back bit for bit.
* Triangle's ``.node`` / ``.ele`` / ``.neigh`` / ``.poly`` files (its
  published file formats): a header line, then one numbered line per item;
  ``#`` starts a comment.  Written zero-based (as Triangle's ``z`` switch);
  the readers accept either numbering by looking at the first index.
"""
from __future__ import annotations

import numpy as np

from .cdtio import CDT


def _lines(path):
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if line:
                yield line.split()


# --- the reference's CDT text file ------------------------------------------

def write_reference_cdt(path, cdt: CDT, exact: bool = False) -> None:
    fmt = "{:.17g} {:.17g}\n" if exact else "{:f} {:f}\n"
    with open(path, "w") as f:
        f.write(f"{cdt.numberofpoints}\n{cdt.numberoftriangles}\n{cdt.numberofsegments}\n")
        f.writelines(fmt.format(x, y) for x, y in cdt.pointlist)
        f.writelines(f"{a} {b} {c}\n" for a, b, c in cdt.trianglelist)
        f.writelines(f"{a} {b} {c}\n" for a, b, c in cdt.neighborlist)
        f.writelines(f"{a} {b}\n" for a, b in cdt.segmentlist)


def read_reference_cdt(path) -> CDT:
    with open(path) as f:
        rows = [line.split() for line in f if line.strip()]
    try:
        n, t, s = int(rows[0][0]), int(rows[1][0]), int(rows[2][0])
        body = rows[3:3 + n + 2 * t + s]
        if len(body) != n + 2 * t + s:
            raise ValueError("truncated")
        pts = np.array([[float(r[0]), float(r[1])] for r in body[:n]], np.float64).reshape(n, 2)
        tri = np.array([[int(v) for v in r[:3]] for r in body[n:n + t]], np.int32).reshape(t, 3)
        nbr = np.array([[int(v) for v in r[:3]] for r in body[n + t:n + 2 * t]], np.int32).reshape(t, 3)
        seg = np.array([[int(v) for v in r[:2]] for r in body[n + 2 * t:]], np.int32).reshape(s, 2)
    except (IndexError, ValueError) as e:
        raise ValueError(f"{path}: not a CDT text file ({e})") from None
    return CDT(pts, tri, nbr, seg)


# --- Triangle's file formats ------------------------------------------------

def write_node(path, points) -> None:
    pts = np.asarray(points, np.float64).reshape(-1, 2)
    with open(path, "w") as f:
        f.write(f"{pts.shape[0]} 2 0 0\n")
        f.writelines(f"{i} {x:.17g} {y:.17g}\n" for i, (x, y) in enumerate(pts))


def read_node(path):
    """Points of a .node file, and the first index (0 or 1)."""
    it = _lines(path)
    head = next(it)
    n, dim = int(head[0]), int(head[1])
    if dim != 2:
        raise ValueError(f"{path}: dimension {dim}")
    rows = [next(it) for _ in range(n)]
    first = int(rows[0][0]) if n else 0
    pts = np.array([[float(r[1]), float(r[2])] for r in rows], np.float64).reshape(n, 2)
    return pts, first


def _write_table(path, head, rows):
    with open(path, "w") as f:
        f.write(head + "\n")
        f.writelines(f"{i} " + " ".join(str(int(v)) for v in r) + "\n" for i, r in enumerate(rows))


def _read_table(path, ncols, base):
    it = _lines(path)
    head = next(it)
    n = int(head[0])
    rows = [next(it) for _ in range(n)]
    a = np.array([[int(v) for v in r[1:1 + ncols]] for r in rows], np.int64).reshape(n, ncols)
    return np.where(a >= 0, a - base, -1).astype(np.int32), head


def write_triangle_files(stem, cdt: CDT) -> None:
    """stem.node, stem.ele, stem.neigh and stem.poly (segments, no holes)."""
    write_node(stem + ".node", cdt.pointlist)
    _write_table(stem + ".ele", f"{cdt.numberoftriangles} 3 0", cdt.trianglelist)
    _write_table(stem + ".neigh", f"{cdt.numberoftriangles} 3", cdt.neighborlist)
    with open(stem + ".poly", "w") as f:
        f.write("0 2 0 0\n")  # the vertices are in the .node file
        f.write(f"{cdt.numberofsegments} 0\n")
        f.writelines(f"{i} {a} {b}\n" for i, (a, b) in enumerate(cdt.segmentlist))
        f.write("0\n")  # no holes


def read_triangle_files(stem) -> CDT:
    pts, base = read_node(stem + ".node")
    tri, _ = _read_table(stem + ".ele", 3, base)
    nbr, _ = _read_table(stem + ".neigh", 3, base)
    it = _lines(stem + ".poly")
    head = next(it)
    for _ in range(int(head[0])):  # vertices listed in the .poly itself are skipped
        next(it)
    ns = int(next(it)[0])
    seg = np.array([[int(r[1]) - base, int(r[2]) - base] for r in (next(it) for _ in range(ns))],
                   np.int32).reshape(ns, 2)
    return CDT(pts, tri, nbr, seg)
