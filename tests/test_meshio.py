"""Text interchange formats (gpu_cdt_refine_b200/meshio.py): the reference's
saveCDT layout (GPU_Refine/mesh.cpp:402-421) and Triangle's files."""
import numpy as np

from gpu_cdt_refine_b200 import inputs, meshio
from gpu_cdt_refine_b200.cdtio import CDT


def _cdt():
    return inputs.plain_small(seed=401, n=500, nseg=20)


def test_reference_text_layout(tmp_path):
    c = CDT(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]), np.array([[0, 1, 2], [1, 3, 2]]),
            np.array([[1, -1, -1], [-1, 0, -1]]), np.array([[0, 1], [1, 3], [3, 2], [2, 0]]))
    p = tmp_path / "c.txt"
    meshio.write_reference_cdt(p, c)
    lines = p.read_text().splitlines()
    # counts on three lines, points printed as %lf, then triangles, neighbours, segments
    assert lines[:3] == ["4", "2", "4"]
    assert lines[3:5] == ["0.000000 0.000000", "1.000000 0.000000"]
    assert lines[7:9] == ["0 1 2", "1 3 2"] and lines[9:11] == ["1 -1 -1", "-1 0 -1"]
    assert lines[11:] == ["0 1", "1 3", "3 2", "2 0"]


def test_reference_text_round_trip(tmp_path):
    c = _cdt()
    p = tmp_path / "c.txt"
    meshio.write_reference_cdt(p, c, exact=True)
    d = meshio.read_reference_cdt(p)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(c, f), getattr(d, f)), f
    meshio.write_reference_cdt(p, c)  # six decimals, as the reference prints
    d = meshio.read_reference_cdt(p)
    assert np.max(np.abs(d.pointlist - c.pointlist)) <= 5e-7
    assert np.array_equal(d.trianglelist, c.trianglelist)


def test_triangle_files_round_trip(tmp_path):
    c = _cdt()
    stem = str(tmp_path / "m")
    meshio.write_triangle_files(stem, c)
    d = meshio.read_triangle_files(stem)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(c, f), getattr(d, f)), f
    # one-based files (Triangle without the z switch) read to the same mesh
    for ext in (".node", ".ele", ".neigh"):
        rows = open(stem + ext).read().splitlines()
        out = [rows[0]] + [" ".join([str(int(r.split()[0]) + 1)] +
                                    [str(int(v) + 1) if (ext != ".node" and int(v) >= 0) else v
                                     for v in r.split()[1:]]) for r in rows[1:]]
        open(stem + ext, "w").write("\n".join(out) + "\n")
    prow = open(stem + ".poly").read().splitlines()
    seg = [" ".join(str(int(v) + 1) for v in r.split()) for r in prow[2:2 + c.numberofsegments]]
    open(stem + ".poly", "w").write("\n".join(prow[:2] + seg + prow[2 + c.numberofsegments:]) + "\n")
    e = meshio.read_triangle_files(stem)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(c, f), getattr(e, f)), f
