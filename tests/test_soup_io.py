"""Mesh files: the host readers (ebg_soup_read) against the reference's own parser
(Parser::readIntoDCEL through the oracle) on the same files, written here in every supported
format and variant.  Vertices (after merging) and triangles must be identical."""
import struct

import numpy as np
import pytest

import oracle
from ebgeometry_b200 import EbgError, read_soup
from ebgeometry_b200 import workloads as W

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle library not built on this host")


@pytest.fixture(scope="module")
def mesh():
    v, f = W.displaced_icosphere(2, 7)
    return v, f.astype(np.int64)


def fmt(x):
    return repr(float(x))


def write_stl_ascii(path, v, f):
    with open(path, "w") as fh:
        fh.write("solid test\n")
        for t in f:
            n = np.cross(v[t[1]] - v[t[0]], v[t[2]] - v[t[0]])
            fh.write(f"  facet normal {fmt(n[0])} {fmt(n[1])} {fmt(n[2])}\n    outer loop\n")
            for i in t:
                fh.write(f"      vertex {fmt(v[i][0])} {fmt(v[i][1])} {fmt(v[i][2])}\n")
            fh.write("    endloop\n  endfacet\n")
        fh.write("endsolid test\n")
        # a second solid: the reference reads the first one only
        fh.write("solid other\n  facet normal 0 0 1\n    outer loop\n      vertex 9 9 9\n      vertex 9 9 10\n"
                 "      vertex 9 10 9\n    endloop\n  endfacet\nendsolid other\n")


def write_stl_binary(path, v, f):
    with open(path, "wb") as fh:
        fh.write(b"binary header".ljust(80, b" "))
        fh.write(struct.pack("<I", len(f) + 2))
        for k, t in enumerate(f):
            fh.write(struct.pack("<3f", 0, 0, 0))
            for i in t:
                fh.write(struct.pack("<3f", *v[i]))
            fh.write(struct.pack("<H", 3))
        # two triangles with a larger attribute id: the reference keeps the smallest id's group
        for _ in range(2):
            fh.write(struct.pack("<3f", 0, 0, 0) + struct.pack("<9f", 5, 5, 5, 5, 5, 6, 5, 6, 5) + struct.pack("<H", 9))


def write_obj(path, v, f, negative=False):
    with open(path, "w") as fh:
        fh.write("# test\no sphere\n")
        for p in v:
            fh.write(f"v {fmt(p[0])} {fmt(p[1])} {fmt(p[2])}\n")
        fh.write("vt 0 0\nvn 0 0 1\n")
        for t in f:
            if negative:
                fh.write("f " + " ".join(str(int(i) - len(v)) for i in t) + "\n")
            else:
                fh.write(f"f {t[0] + 1}/1/1 {t[1] + 1}//1 {t[2] + 1}\n")
        fh.write("f 1 2\n")  # a line, dropped


def write_ply(path, v, f, mode):
    with open(path, "wb") as fh:
        fh.write(f"ply\nformat {mode} 1.0\ncomment test\nelement vertex {len(v)}\nproperty double x\n"
                 f"property double y\nproperty double z\nproperty uchar red\nelement face {len(f)}\n"
                 "property list uchar int vertex_indices\nend_header\n".encode())
        if mode == "ascii":
            for p in v:
                fh.write(f"{fmt(p[0])} {fmt(p[1])} {fmt(p[2])} 7\n".encode())
            for t in f:
                fh.write(f"3 {t[0]} {t[1]} {t[2]}\n".encode())
        else:
            e = "<" if mode == "binary_little_endian" else ">"
            for p in v:
                fh.write(struct.pack(e + "3dB", p[0], p[1], p[2], 7))
            for t in f:
                fh.write(struct.pack(e + "B3i", 3, *t))


def write_vtk(path, v, f, offsets=False):
    with open(path, "w") as fh:
        fh.write("# vtk DataFile Version 3.0\ntest\nASCII\nDATASET POLYDATA\n")
        fh.write(f"POINTS {len(v)} double\n")
        for p in v:
            fh.write(f"{fmt(p[0])} {fmt(p[1])} {fmt(p[2])}\n")
        if offsets:
            fh.write(f"POLYGONS {len(f) + 1} {3 * len(f)}\nOFFSETS vtktypeint64\n")
            fh.write(" ".join(str(3 * i) for i in range(len(f) + 1)) + "\n")
            fh.write("CONNECTIVITY vtktypeint64\n" + " ".join(str(int(i)) for i in f.ravel()) + "\n")
        else:
            fh.write(f"POLYGONS {len(f)} {4 * len(f)}\n")
            for t in f:
                fh.write(f"3 {t[0]} {t[1]} {t[2]}\n")


CASES = {
    "ascii.stl": lambda p, v, f: write_stl_ascii(p, v, f),
    "binary.stl": lambda p, v, f: write_stl_binary(p, v, f),
    "plain.obj": lambda p, v, f: write_obj(p, v, f),
    "negative.obj": lambda p, v, f: write_obj(p, v, f, negative=True),
    "ascii.ply": lambda p, v, f: write_ply(p, v, f, "ascii"),
    "le.ply": lambda p, v, f: write_ply(p, v, f, "binary_little_endian"),
    "be.ply": lambda p, v, f: write_ply(p, v, f, "binary_big_endian"),
    "lists.vtk": lambda p, v, f: write_vtk(p, v, f),
    "offsets.vtk": lambda p, v, f: write_vtk(p, v, f, offsets=True),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_matches_reference_parser(tmp_path, mesh, name):
    v, f = mesh
    path = str(tmp_path / name)
    CASES[name](path, v, f)
    ours_v, ours_f = read_soup(path)
    ref_v, ref_f = oracle.ref().read_soup(path)
    assert np.array_equal(ours_v, ref_v), name
    assert np.array_equal(ours_f, ref_f.astype(np.int32)), name


def test_merged_soup_is_the_mesh(tmp_path, mesh):
    """Merging the STL's per-facet vertex copies gives back the icosphere's vertices, sorted."""
    v, f = mesh
    path = str(tmp_path / "m.stl")
    write_stl_binary(path, v, f)
    ours_v, ours_f = read_soup(path)
    v32 = v.astype(np.float32).astype(np.float64)
    assert ours_v.shape == v.shape and ours_f.shape == f.shape
    assert np.array_equal(ours_v[ours_f], v32[f])
    key = np.lexsort((ours_v[:, 2], ours_v[:, 1], ours_v[:, 0]))
    assert np.array_equal(key, np.arange(len(ours_v)))


def test_reader_errors(tmp_path):
    with pytest.raises(EbgError):
        read_soup(str(tmp_path / "missing.obj"))
    bad = tmp_path / "quad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(EbgError):
        read_soup(str(bad))  # quads: triangle meshes only
    other = tmp_path / "mesh.xyz"
    other.write_text("0 0 0\n")
    with pytest.raises(EbgError):
        read_soup(str(other))
