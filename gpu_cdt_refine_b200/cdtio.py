"""CDT container and the binary "GQMCDT1" file format.

A :class:`CDT` holds the fields of Triangle's ``triangulateio`` that the
refiner reads and writes (GPU_Refine/triangle.h:253-284): ``pointlist``
(float64, N x 2), ``trianglelist`` (int32, T x 3, counterclockwise),
``neighborlist`` (int32, T x 3, neighbour j opposite vertex j, -1 on the
boundary) and ``segmentlist`` (int32, S x 2).

File layout (little endian): 8-byte magic ``GQMCDT1\\0``; int32 N, T, S,
has_neighbors; float64 points[2N]; int32 triangles[3T]; int32 neighbors[3T]
when has_neighbors; int32 segments[2S].
"""
from __future__ import annotations

import dataclasses

import numpy as np

MAGIC = b"GQMCDT1\x00"


@dataclasses.dataclass
class CDT:
    pointlist: np.ndarray
    trianglelist: np.ndarray
    neighborlist: np.ndarray
    segmentlist: np.ndarray

    @classmethod
    def wrap(cls, pointlist, trianglelist, neighborlist, segmentlist):
        """A CDT over arrays that already have the right dtypes and shapes
        (n x 2 float64, n x 3 int32, n x 3 int32, n x 2 int32): no checks, no copies."""
        c = cls.__new__(cls)
        c.pointlist, c.trianglelist, c.neighborlist, c.segmentlist = pointlist, trianglelist, neighborlist, segmentlist
        return c

    def __post_init__(self):
        self.pointlist = np.ascontiguousarray(self.pointlist, dtype=np.float64).reshape(-1, 2)
        self.trianglelist = np.ascontiguousarray(self.trianglelist, dtype=np.int32).reshape(-1, 3)
        self.neighborlist = np.ascontiguousarray(self.neighborlist, dtype=np.int32).reshape(-1, 3)
        self.segmentlist = np.ascontiguousarray(self.segmentlist, dtype=np.int32).reshape(-1, 2)

    @property
    def numberofpoints(self) -> int:
        return int(self.pointlist.shape[0])

    @property
    def numberoftriangles(self) -> int:
        return int(self.trianglelist.shape[0])

    @property
    def numberofsegments(self) -> int:
        return int(self.segmentlist.shape[0])

    def nbytes(self) -> int:
        return (self.pointlist.nbytes + self.trianglelist.nbytes + self.neighborlist.nbytes
                + self.segmentlist.nbytes)


def write_cdt(path, cdt: CDT) -> None:
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.array([cdt.numberofpoints, cdt.numberoftriangles, cdt.numberofsegments, 1],
                         dtype="<i4").tobytes())
        f.write(cdt.pointlist.astype("<f8").tobytes())
        f.write(cdt.trianglelist.astype("<i4").tobytes())
        f.write(cdt.neighborlist.astype("<i4").tobytes())
        f.write(cdt.segmentlist.astype("<i4").tobytes())


def read_cdt(path) -> CDT:
    with open(path, "rb") as f:
        if f.read(8)[:7] != MAGIC[:7]:
            raise ValueError(f"{path}: not a GQMCDT1 file")
        n, t, s, hn = np.frombuffer(f.read(16), dtype="<i4")
        pts = np.frombuffer(f.read(16 * n), dtype="<f8").reshape(n, 2)
        tri = np.frombuffer(f.read(12 * t), dtype="<i4").reshape(t, 3)
        nbr = (np.frombuffer(f.read(12 * t), dtype="<i4").reshape(t, 3) if hn
               else np.full((t, 3), -1, np.int32))
        seg = np.frombuffer(f.read(8 * s), dtype="<i4").reshape(s, 2)
    return CDT(pts.copy(), tri.copy(), nbr.copy(), seg.copy())


def canonical(cdt: CDT):
    """Order-independent form of a mesh for comparisons.

    Returns (points, triangles, segments) where points are sorted
    lexicographically by (x, y) bit pattern order of values, and triangles and
    segments are expressed in the sorted point numbering, rotated so the
    smallest index comes first (triangles keep their orientation), and sorted.
    Two meshes with the same vertex coordinates, triangles and segments have
    identical canonical forms whatever their numbering.
    """
    pts = cdt.pointlist
    order = np.lexsort((pts[:, 1], pts[:, 0]))
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    tri = rank[cdt.trianglelist]
    k = np.argmin(tri, axis=1)
    rows = np.arange(tri.shape[0])
    tri = np.stack([tri[rows, k], tri[rows, (k + 1) % 3], tri[rows, (k + 2) % 3]], axis=1)
    tri = tri[np.lexsort((tri[:, 2], tri[:, 1], tri[:, 0]))]
    seg = np.sort(rank[cdt.segmentlist], axis=1)
    seg = seg[np.lexsort((seg[:, 1], seg[:, 0]))]
    return pts[order], tri, seg


def same_mesh(a: CDT, b: CDT) -> bool:
    pa, ta, sa = canonical(a)
    pb, tb, sb = canonical(b)
    return (pa.shape == pb.shape and np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
            and np.array_equal(ta, tb) and np.array_equal(sa, sb))
