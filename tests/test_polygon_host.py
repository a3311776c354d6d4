"""Polygon meshes on the host (no device): the DCEL quantities of polygon soups against the
reference's soupToDCEL (committed fixtures, and the reference library where it is built), and the
file readers keeping polygon faces exactly as the reference's parser does."""
import numpy as np
import pytest

import oracle
from ebgeometry_b200 import EbgError, TriMeshSDF, polygon_normals, read_polygon_soup, read_soup
from ebgeometry_b200 import workloads as W

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle library not built on this host")


@pytest.mark.parametrize("name", ["prism", "quad", "mixed"])
def test_normals_match_fixture(golden, name):
    g = golden("polygons.npz")
    fn, c, vn, en = polygon_normals(g[f"{name}_v"], (g[f"{name}_off"], g[f"{name}_idx"]))
    assert np.array_equal(fn, g[f"{name}_face_n"])
    assert np.array_equal(c, g[f"{name}_centroid"])
    assert np.array_equal(vn, g[f"{name}_vert_n"])
    assert np.array_equal(en, g[f"{name}_edge_n"])


@needs_ref
@pytest.mark.parametrize("mesh", ["quad16", "mixed12", "prism5", "prism12", "icosphere"])
def test_normals_match_reference(mesh):
    if mesh == "icosphere":
        v, f = W.displaced_icosphere(3, 4)
        faces = (np.arange(f.shape[0] + 1, dtype=np.int64) * 3, f.ravel())
    else:
        v, faces = {"quad16": lambda: W.displaced_quad_sphere(16, 2), "mixed12": lambda: W.mixed_polygon_sphere(12, 8),
                    "prism5": lambda: W.polygon_prism(5), "prism12": lambda: W.polygon_prism(12, 0.3, 2.0)}[mesh]()
    ours = polygon_normals(v, faces)
    ref = oracle.ref().polymesh(v, faces[0], faces[1]).polygon_normals()
    for a, b in zip(ours, ref):
        assert np.array_equal(a, b), mesh


def test_polygon_errors():
    v, (off, idx) = W.polygon_prism(6)
    with pytest.raises(EbgError):
        polygon_normals(v, [[0, 1]])  # fewer than three vertices
    flat = v.copy()
    flat[:, 2] = 0.0  # the prism collapses onto its base: side quads span no plane
    with pytest.raises(EbgError):
        polygon_normals(flat, (off, idx))
    with pytest.raises(EbgError):
        polygon_normals(v, [[0, 1, 99]])


def fmt(x):
    return repr(float(x))


def write_obj(path, v, faces):
    with open(path, "w") as fh:
        for p in v:
            fh.write(f"v {fmt(p[0])} {fmt(p[1])} {fmt(p[2])}\n")
        for f in faces:
            fh.write("f " + " ".join(str(int(i) + 1) for i in f) + "\n")


def write_ply(path, v, faces, binary):
    import struct
    with open(path, "wb") as fh:
        fmt_ = "binary_little_endian" if binary else "ascii"
        fh.write(f"ply\nformat {fmt_} 1.0\nelement vertex {len(v)}\nproperty double x\nproperty double y\n"
                 f"property double z\nelement face {len(faces)}\nproperty list uchar int vertex_indices\n"
                 "end_header\n".encode())
        for p in v:
            fh.write(struct.pack("<3d", *p) if binary else f"{fmt(p[0])} {fmt(p[1])} {fmt(p[2])}\n".encode())
        for f in faces:
            if binary:
                fh.write(struct.pack("<B", len(f)) + struct.pack(f"<{len(f)}i", *[int(i) for i in f]))
            else:
                fh.write((f"{len(f)} " + " ".join(str(int(i)) for i in f) + "\n").encode())


def write_vtk(path, v, faces):
    with open(path, "w") as fh:
        fh.write(f"# vtk DataFile Version 3.0\npolygons\nASCII\nDATASET POLYDATA\nPOINTS {len(v)} double\n")
        for p in v:
            fh.write(f"{fmt(p[0])} {fmt(p[1])} {fmt(p[2])}\n")
        fh.write(f"POLYGONS {len(faces)} {sum(len(f) + 1 for f in faces)}\n")
        for f in faces:
            fh.write(f"{len(f)} " + " ".join(str(int(i)) for i in f) + "\n")


def face_lists(off, idx):
    return [list(idx[off[k]:off[k + 1]]) for k in range(off.size - 1)]


WRITERS = {"obj": write_obj, "ply": lambda p, v, f: write_ply(p, v, f, False),
           "bin.ply": lambda p, v, f: write_ply(p, v, f, True), "vtk": write_vtk}


@needs_ref
@pytest.mark.parametrize("ext", sorted(WRITERS))
@pytest.mark.parametrize("mesh", ["quad", "mixed", "prism"])
def test_polygon_reader_matches_reference_parser(tmp_path, ext, mesh):
    v, (off, idx) = {"quad": lambda: W.displaced_quad_sphere(3, 1), "mixed": lambda: W.mixed_polygon_sphere(4, 2),
                     "prism": lambda: W.polygon_prism(9)}[mesh]()
    path = str(tmp_path / f"m.{ext}")
    WRITERS[ext](path, v, face_lists(off, idx))
    ours = read_polygon_soup(path)
    ref = oracle.ref().read_polysoup(path)
    assert np.array_equal(ours[0], ref[0])
    assert np.array_equal(ours[1], ref[1])
    assert np.array_equal(ours[2], ref[2].astype(np.int32))


def test_polygon_files_are_not_triangle_meshes(tmp_path):
    v, (off, idx) = W.polygon_prism(6)
    path = str(tmp_path / "prism.obj")
    write_obj(path, v, face_lists(off, idx))
    with pytest.raises(EbgError):
        read_soup(path)
    with pytest.raises(EbgError):
        TriMeshSDF.from_file(path)
    pv, poff, pidx = read_polygon_soup(path)
    assert poff.size - 1 == off.size - 1 and pidx.size == idx.size
