"""Wavefront OBJ meshes: both front ends' loaders against the reference's own parser, UseNormals, WriteWavefront.

* The reference's parser (src/core/utils/WavefrontMeshLoader.hpp, compiled here by oracle/ref_build.py into
  ``oracle/_ref/ref_obj_dump``) reads the reference's five mesh files (data/mesh) and an OBJ text with polygons,
  texture and normal indices, upper-case tags, comments, tabs and CRLF line ends; deme_b200.scene.read_wavefront and
  deme::DEMMeshConnected::LoadWavefrontMesh (tests/cpp/obj_dump.cpp) must give the same vertices and normals bit for
  bit and the same facet vertex and normal indices.
* UseNormals: the facets' nodes as initialisation places them, bit-identical between the front ends, and every
  facet's right-hand normal then on the side of its first corner's normal.
* WriteWavefront of a mesh with normals and one without: byte-identical text from both front ends, which the
  reference's parser reads back to the same facets and normal indices and to the vertices at 6 significant digits.
* Merge, negative indices (counted back from the last record, where the reference would leave an index outside the
  mesh) and records the reference skips.
Compiling and running the C++ side needs no GPU.
"""
import os
import subprocess

import numpy as np
import pytest

from _util import ROOT
from deme_b200 import solver
from deme_b200.scene import MeshObj, SceneBuilder, facet_nodes, read_wavefront, write_wavefront

f32 = np.float32
CUDA_INC = "/usr/local/cuda/include"

EDGE_OBJ = (
    "# polygons, texture and normal indices, tags in upper case\r\n"
    "mtllib none.mtl\r\n"
    "o part\n"
    "v 0 0 0\n"
    "v 1.0 0 0\n"
    "V 1 1 0.1\n"
    "v\t0\t1\t-0.2\n"
    "v 0.5 0.5 1e-1\n"
    "v 0.333333333333333333 0.1 2.5e+0\n"
    "vt 0 0\nvt 1 0\nvt 1 1\n"
    "vn 0 0 1\nVN 0 0 -1\nvn 0.6 0.8 0\n"
    "f 1/1/1 2/2/1 3/3/1 4/1/1\n"          # a quad with texture and normal indices
    "F 1//2 5//2 2//2\n"                   # upper-case tag, normals only
    "f 2 3 5 6 4\n"                        # a pentagon without normals
    "g group\n"
    "s off\n"
    "f 6//3 5//3 3//3\n"
)


def _ref_obj_dump():
    from oracle import ref_build
    if not ref_build.obj_loader_available():
        pytest.skip("the reference's sources are not mounted")
    return ref_build


@pytest.fixture(scope="module")
def cpp_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("objcpp")
    exe = str(d / "obj_dump")
    libdir = os.path.dirname(solver.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
                           CUDA_INC, os.path.join(ROOT, "tests", "cpp", "obj_dump.cpp"), "-o", exe, "-L", libdir,
                           "-ldeme_b200", f"-Wl,-rpath,{libdir}"])
    return exe


def _read_mesh(raw, off):
    nv, nf, nn, nfn = np.frombuffer(raw, np.int32, 4, off)
    off += 16
    out = {}
    for key, n, dt in (("vertices", nv, f32), ("faces", nf, np.int32), ("normals", nn, f32),
                       ("face_normals", nfn, np.int32)):
        a = np.frombuffer(raw, dt, 3 * int(n), off).reshape(-1, 3)
        off += a.nbytes
        out[key] = a
    return out, off


def cpp_load(exe, path, tmp_path, written=None):
    out = tmp_path / "cpp.bin"
    subprocess.check_call([exe, str(path), str(out)] + ([str(written)] if written else []))
    raw = out.read_bytes()
    mesh, off = _read_mesh(raw, 0)
    oriented = int(np.frombuffer(raw, np.int32, 1, off)[0])
    off += 4
    if oriented:
        nf = len(mesh["faces"])
        mesh["oriented"] = np.frombuffer(raw, f32, 9 * nf, off).reshape(-1, 9)
        off += 36 * nf
    mesh["merged"], _ = _read_mesh(raw, off)
    return mesh


def ref_load(path, tmp_path):
    rb = _ref_obj_dump()
    exe = rb.build_obj_dump()
    out = tmp_path / "ref.bin"
    subprocess.check_call([exe, str(path), str(out)])
    return rb.read_obj_dump(str(out))


def _same(a, b, what):
    for k in ("vertices", "faces", "normals", "face_normals"):
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape, (what, k, x.shape, y.shape)
        if x.dtype.kind == "f":
            assert x.astype(f32).tobytes() == y.astype(f32).tobytes(), (what, k)
        else:
            np.testing.assert_array_equal(x.astype(np.int64), y.astype(np.int64), err_msg=f"{what} {k}")


def _mesh_files():
    from oracle import ref_build
    if not os.path.isdir(ref_build.MESH_DIR):
        return []
    return sorted(os.path.join(ref_build.MESH_DIR, f) for f in os.listdir(ref_build.MESH_DIR) if f.endswith(".obj"))


@pytest.mark.parametrize("path", _mesh_files() or [pytest.param(None, marks=pytest.mark.skip("no reference"))],
                         ids=lambda p: os.path.basename(p) if p else "none")
def test_reference_mesh_files_load_as_the_reference_reads_them(path, cpp_exe, tmp_path):
    ref = ref_load(path, tmp_path)
    assert len(ref["faces"]) > 100
    _same(read_wavefront(path), ref, "python")
    cpp = cpp_load(cpp_exe, path, tmp_path)
    _same(cpp, ref, "c++")


def test_polygons_tags_comments_and_line_ends(cpp_exe, tmp_path):
    p = tmp_path / "edge.obj"
    p.write_bytes(EDGE_OBJ.encode())
    py = read_wavefront(str(p))
    # quad -> 2 fans, triangle, pentagon -> 3 fans, triangle
    assert len(py["faces"]) == 7 and len(py["vertices"]) == 6 and len(py["normals"]) == 3
    np.testing.assert_array_equal(py["faces"][:3], [[0, 1, 2], [0, 2, 3], [0, 4, 1]])
    # normal triples only for the facets whose corners carry them (the pentagon's three carry none)
    np.testing.assert_array_equal(py["face_normals"], [[0, 0, 0], [0, 0, 0], [1, 1, 1], [2, 2, 2]])
    assert py["vertices"][5, 0] == f32(float("0.333333333333333333"))
    _same(cpp_load(cpp_exe, p, tmp_path), py, "c++")
    if _mesh_files():
        _same(py, ref_load(p, tmp_path), "reference")


def test_negative_indices_and_skipped_records(cpp_exe, tmp_path):
    """Negative indices count back from the last record read; a vertex record with fewer than three coordinates
    and a facet with fewer than three corners are skipped, as the reference skips them; a vertex with a fourth
    number or a trailing comment is read (the reference drops such a record)."""
    p = tmp_path / "neg.obj"
    p.write_text("v 0 0 0\nv 1 0 0 1.0\nv 2\nv 0 1 0 # apex\nvn 0 0 1\nf -3//-1 -2//-1 -1//-1\nf 1 2\nv 0 0 1\n"
                 "f 1 2 -1\n")
    py = read_wavefront(str(p))
    np.testing.assert_array_equal(py["vertices"], [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    np.testing.assert_array_equal(py["faces"], [[0, 1, 2], [0, 1, 3]])
    np.testing.assert_array_equal(py["face_normals"], [[0, 0, 0]])
    _same(cpp_load(cpp_exe, p, tmp_path), py, "c++")


def _box_obj(tmp_path):
    """A unit cube with outward face normals whose every other triangle is wound inwards."""
    v = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float64)
    quads = {(-1, 0, 0): (0, 1, 3, 2), (1, 0, 0): (4, 5, 7, 6), (0, -1, 0): (0, 1, 5, 4), (0, 1, 0): (2, 3, 7, 6),
             (0, 0, -1): (0, 2, 6, 4), (0, 0, 1): (1, 3, 7, 5)}
    lines = [f"v {x:g} {y:g} {z:g}" for x, y, z in v] + [f"vn {x} {y} {z}" for x, y, z in quads]
    k = 0
    for ni, (n, (a, b, c, d)) in enumerate(quads.items()):
        for t in ((a, b, c), (a, c, d)):
            outward = np.dot(np.cross(v[t[1]] - v[t[0]], v[t[2]] - v[t[0]]), n) > 0
            if outward == (k % 2 == 1):
                t = (t[0], t[2], t[1])
            lines.append("f " + " ".join(f"{i + 1}//{ni + 1}" for i in t))
            k += 1
    p = tmp_path / "box.obj"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


def test_use_normals_orders_facets_alike(cpp_exe, tmp_path):
    flipped = {}
    for path in [_box_obj(tmp_path)] + _mesh_files():
        r = read_wavefront(path)
        py = facet_nodes(r["vertices"], r["faces"], r["normals"], r["face_normals"])
        cpp = cpp_load(cpp_exe, path, tmp_path)
        assert py.tobytes() == cpp["oriented"].tobytes(), path
        t = py.reshape(-1, 3, 3).astype(np.float64)
        n = r["normals"][r["face_normals"][:, 0]].astype(np.float64)
        c = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
        d = np.einsum("ij,ij->i", c, n)
        assert np.all(d >= -1e-6 * np.linalg.norm(c, axis=1) * np.linalg.norm(n, axis=1)), path
        flipped[os.path.basename(path)] = int(np.sum(np.any(py != facet_nodes(r["vertices"], r["faces"]), axis=1)))
    assert flipped["box.obj"] == 6, flipped


def test_write_wavefront_agrees_and_reads_back(cpp_exe, tmp_path):
    files = _mesh_files()
    src = files[1] if files else None
    if src is None:
        src = tmp_path / "edge.obj"
        src.write_bytes(EDGE_OBJ.encode())
    cpp_written = tmp_path / "cpp_out.obj"
    cpp = cpp_load(cpp_exe, src, tmp_path, cpp_written)
    r = read_wavefront(str(src))
    m = MeshObj(r["vertices"], r["faces"], 0, r["normals"], r["face_normals"])
    bare = MeshObj(r["vertices"], r["faces"], 1)
    py_written = tmp_path / "py_out.obj"
    write_wavefront(str(py_written), [m, bare])
    assert py_written.read_bytes() == cpp_written.read_bytes()
    back = read_wavefront(str(py_written))
    nv, nf = len(r["vertices"]), len(r["faces"])
    np.testing.assert_array_equal(back["faces"], np.concatenate([r["faces"], r["faces"] + nv]))
    np.testing.assert_array_equal(back["face_normals"], r["face_normals"])
    for half in (back["vertices"][:nv], back["vertices"][nv:]):
        np.testing.assert_allclose(half, r["vertices"], rtol=5e-6, atol=1e-30)
    if files:
        _same(back, ref_load(py_written, tmp_path), "reference reads the written file")
    # Merge of the mesh with itself: nodes, normals and facets offset into one mesh
    mm = MeshObj.Merge([m, m])
    _same({"vertices": mm.vertices, "faces": mm.faces, "normals": mm.normals, "face_normals": mm.face_normals},
          cpp["merged"], "merge")
    assert mm.GetNumTriangles() == 2 * nf


def test_use_normals_reaches_the_scene(tmp_path):
    """A mesh body with UseNormals places its facets' nodes in the flattened scene as facet_nodes orders them."""
    p = tmp_path / "edge.obj"
    p.write_bytes(EDGE_OBJ.encode())
    lines = [ln for ln in EDGE_OBJ.replace("\r\n", "\n").split("\n") if not ln.lower().startswith("f 2 3 5")]
    p2 = tmp_path / "tri.obj"
    p2.write_text("\n".join(lines) + "\n")
    s = SceneBuilder()
    s.InstructBoxDomainDimension(4, 4, 4)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    t = s.LoadSphereType(1e-3, 0.05, mat)
    s.AddClumps([t], np.array([[0, 0, 1.5]], f32))
    m = s.AddWavefrontMeshObject(str(p2), mat)
    m.UseNormals()
    s.SetInitTimeStep(1e-5)
    built = s.Initialize()
    r = read_wavefront(str(p2))
    want = facet_nodes(r["vertices"], r["faces"], r["normals"], r["face_normals"])
    got = np.concatenate([built.arrays[k].reshape(-1, 3) for k in ("tri_node1", "tri_node2", "tri_node3")], 1)
    np.testing.assert_array_equal(got, want)
    assert np.any(want != facet_nodes(r["vertices"], r["faces"]))
