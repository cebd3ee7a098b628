"""The oracle's sphere--mesh contacts (oracle/deme_oracle.c), pinned on the CPU without the CUDA path.

The reference declares the sphere--mesh contact type but has no detection for it, so there is no reference output to
pin this part of the oracle to.  Instead:

* geometry: for seeded sphere centres around one facet (over its interior, beside its edges and corners, above and
  below it), the contact exists exactly when an independent closest-point computation (projection onto the facet's
  plane, else the nearest of its three edges) puts the centre within the radius, and its force equals the force of
  an analytical plane through that closest point, facing the centre (the plane's conventions are the mesh's): 1e-5
  relative;
* order: a sphere touching an analytical plane and several facets lists the plane first, then the facets by id;
* the Wavefront OBJ reader splits polygons into fans, takes negative indices from the end and ignores texture and
  normal indices;
* flattening: mesh owners follow the external objects, facets carry owner, material and owner-frame nodes.
"""
import numpy as np
import pytest

from _util import oracle, capi
from deme_b200.scene import SceneBuilder, load_wavefront

R = 2e-3
TRI = np.array([[0.0, 0.0, 0.0], [0.02, 0.0, 0.0], [0.004, 0.015, 0.0]])


def _closest_independent(p, tri):
    a, b, c = tri
    n = np.cross(b - a, c - a)
    n /= np.linalg.norm(n)
    q = p - np.dot(p - a, n) * n
    # barycentric coordinates of the projection
    m = np.array([b - a, c - a]).T
    uv, *_ = np.linalg.lstsq(m, q - a, rcond=None)
    if uv[0] >= 0 and uv[1] >= 0 and uv.sum() <= 1:
        return q
    best = None
    for s0, s1 in ((a, b), (b, c), (c, a)):
        d = s1 - s0
        t = np.clip(np.dot(p - s0, d) / np.dot(d, d), 0.0, 1.0)
        x = s0 + t * d
        if best is None or np.linalg.norm(p - x) < np.linalg.norm(p - best):
            best = x
    return best


def _scene(centre, mesh=None, plane=None, floor=None):
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    ms = s.LoadMaterial({"E": 1e8, "nu": 0.3, "CoR": 0.5, "mu": 0.0, "Crr": 0.0})
    mw = s.LoadMaterial({"E": 2e8, "nu": 0.25, "CoR": 0.4, "mu": 0.0, "Crr": 0.0})
    t = s.LoadSphereType(1e-4, R, ms)
    s.AddClumps([t], np.asarray(centre, np.float32).reshape(1, 3))
    if floor is not None:
        s.AddBCPlane(*floor, mw)
    if plane is not None:
        s.AddBCPlane(plane[0], plane[1], mw)
    if mesh is not None:
        s.AddWavefrontMeshObject(mesh, mw)
    s.SetInitTimeStep(1e-5)
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)
    s.SetInitBinSize(4 * R)
    return s.Initialize()


def _forces(built):
    o = oracle(built, threads=1)
    o.detect_contacts()
    o.compute_forces()
    c, f = o.contacts(), o.contact_forces()
    o.close()
    return c, f


def test_facet_contact_geometry_matches_independent_closest_point():
    rng = np.random.default_rng(7)
    v = TRI.astype(np.float32)
    tri = v.astype(np.float64)
    n_contact = n_edge = 0
    for _ in range(24):
        # centres over and around the facet, above and below it, some out of reach
        p = np.array([rng.uniform(-0.004, 0.024), rng.uniform(-0.004, 0.019), rng.uniform(-1.3, 1.3) * R])
        p = p.astype(np.float32).astype(np.float64)
        built = _scene(p, mesh=(v, np.array([[0, 1, 2]])))
        c, f = _forces(built)
        q = _closest_independent(p, tri)
        gap = np.linalg.norm(p - q)
        has = np.any(c["type"] == capi.SPHERE_MESH_CONTACT)
        if abs(gap - R) < 1e-9:
            continue  # at the reach within rounding: either answer is right
        assert has == (gap < R), (p, gap)
        if not has:
            continue
        n_contact += 1
        n = (p - q) / gap
        on_face = abs(abs(np.dot(n, [0, 0, 1])) - 1) < 1e-9
        n_edge += not on_face
        cp, fp = _forces(_scene(p, plane=(q, n)))
        assert np.any(cp["type"] == capi.SPHERE_PLANE_CONTACT)
        a, b = f["force"][0].astype(np.float64), fp["force"][0].astype(np.float64)
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max(), (p, a, b)
        np.testing.assert_allclose(f["cpA"][0], fp["cpA"][0], rtol=0, atol=1e-5 * R)
    assert n_contact >= 6 and n_edge >= 2, (n_contact, n_edge)


def test_segment_order_plane_then_facets_by_id():
    # a sphere in the corner of a floor plane and three facets (two of them touching it)
    p = np.array([0.001, 0.001, 0.0015])
    v = np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0],          # facet 0 at z = 0: touches
                  [0, 0, 0], [0, 0.01, 0], [0, 0, 0.01],          # facet 1 at x = 0: touches
                  [0.05, 0.05, 0], [0.06, 0.05, 0], [0.05, 0.06, 0]], np.float32)  # facet 2: far
    built = _scene(p, mesh=(v, np.arange(9).reshape(3, 3)), floor=((0, 0, 0.0005), (0, 0, 1)))
    c, _ = _forces(built)
    assert list(c["type"]) == [capi.SPHERE_PLANE_CONTACT, capi.SPHERE_MESH_CONTACT, capi.SPHERE_MESH_CONTACT]
    assert list(c["idB"]) == [0, 0, 1]


def test_wavefront_reader(tmp_path):
    f = tmp_path / "quad.obj"
    f.write_text("# a quad and a triangle\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
                 "f 1/1/1 2/1/1 3/1/1 4/1/1\nf -1 -3 -2\n")
    v, faces = load_wavefront(str(f))
    assert v.shape == (4, 3) and v.dtype == np.float32
    np.testing.assert_array_equal(faces, [[0, 1, 2], [0, 2, 3], [3, 1, 2]])
    s = SceneBuilder()
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    obj = s.AddWavefrontMeshObject(str(f), m)
    assert obj.GetNumTriangles() == 3
    with pytest.raises(ValueError, match="must have length 3"):
        obj.SetMaterial([m, m])


def test_mesh_owners_follow_the_external_objects_when_flattened():
    """Owners: clumps, external objects, then mesh objects (kT.cpp:603-625); facets carry their owner, per-facet
    material and their nodes in the owner frame (after Translate / Scale); the owner its pose, mass and moments."""
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    m0 = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    m1 = s.LoadMaterial({"E": 2e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    t = s.LoadSphereType(1e-4, R, m0)
    s.AddClumps([t] * 3, np.zeros((3, 3), np.float32) + np.arange(3, dtype=np.float32)[:, None] * 0.01)
    s.AddBCPlane((0, 0, -0.05), (0, 0, 1), m0)
    a = s.AddWavefrontMeshObject((TRI.astype(np.float32), np.array([[0, 1, 2]])), m1)
    a.Translate((0.001, 0.0, 0.0))
    a.Scale(2.0)
    b = s.AddWavefrontMeshObject((TRI.astype(np.float32), np.array([[0, 1, 2], [2, 1, 0]])))
    b.SetMaterial([m0, m1])
    b.SetInitPos((0.01, 0.02, 0.03))
    b.SetInitQuat((0.8, 0.0, 0.6, 0.0))
    b.SetMass(3.0)
    b.SetMOI((1.0, 2.0, 3.0))
    b.SetFamily(7)
    built = s.Initialize()
    arr = built.arrays
    assert built.counts["o"] == 3 + 1 + 2 and built.counts["t"] == 3
    np.testing.assert_array_equal(arr["tri_owner"], [4, 5, 5])
    np.testing.assert_array_equal(arr["tri_material"], [1, 0, 1])
    np.testing.assert_array_equal(arr["tri_node1"][0], (TRI[0].astype(np.float32) + np.float32([0.001, 0, 0])) * 2)
    np.testing.assert_array_equal(arr["tri_node1"][2], TRI[2].astype(np.float32))
    assert arr["family"][5] == 7 and arr["mass"][5] == np.float32(3.0) and arr["mmiZZ"][5] == np.float32(3.0)
    np.testing.assert_array_equal([arr[k][5] for k in ("oriQw", "oriQx", "oriQy", "oriQz")],
                                  np.float32([0.8, 0.0, 0.6, 0.0]))
    pos = built.decode_positions(built.initial_state(), kernel_literals=False) + built.info["lbf"]
    assert np.abs(pos[5] - [0.01, 0.02, 0.03]).max() < 1e-7
    assert arr["family"][4] == capi.RESERVED_FAMILY
    # a mesh without a material is refused at Initialize, as the reference refuses it
    s2 = SceneBuilder()
    s2.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s2.AddWavefrontMeshObject((TRI.astype(np.float32), np.array([[0, 1, 2]])))
    with pytest.raises(ValueError, match="does not have associated material"):
        s2.Initialize()


def test_zero_area_facets_are_refused():
    """A facet whose nodes are collinear has no closest-point region test that is defined everywhere; Initialize
    refuses it (the C ABI does too), naming the facet."""
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    v = np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0], [0.02, 0, 0]], np.float32)
    s.AddWavefrontMeshObject((v, np.array([[0, 1, 2], [0, 1, 3]])), m)
    with pytest.raises(ValueError, match="mesh facet 1 has zero area"):
        s.Initialize()


def test_mesh_mass_properties_rotation_and_writer(tmp_path):
    """ComputeMassProperties on a unit cube (volume 1, centroid at its centre, moments 1/6) and an icosphere (the
    sphere's 4/3 pi R^3 and 2/5 m R^2 within its faceting, 0.3 %); Rotate turns a mesh without changing its volume;
    WriteWavefront then LoadWavefrontMesh gives the meshes back."""
    import math
    from deme_b200 import workloads
    from deme_b200.scene import MeshObj, write_wavefront
    V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.float32)
    F = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4], [1, 2, 6], [1, 6, 5],
                  [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]])
    cube = MeshObj(V, F, 0)
    m, c, inertia = cube.ComputeMassProperties()
    assert abs(m - 1.0) < 1e-12 and np.abs(c - 0.5).max() < 1e-12 and np.abs(inertia - 1 / 6).max() < 1e-12
    v, f = workloads.icosphere(0.1, 4)
    ball = MeshObj(v, f, 1)
    m, c, inertia = ball.ComputeMassProperties()
    assert abs(m / (4 / 3 * math.pi * 1e-3) - 1) < 3e-3 and np.abs(c).max() < 1e-9
    assert np.abs(inertia / (0.4 * m * 0.01) - 1).max() < 3e-3
    cube.Rotate((math.cos(0.3), math.sin(0.3), 0.0, 0.0))
    m2, c2, _ = cube.ComputeMassProperties()
    assert abs(m2 - 1.0) < 1e-6 and abs(c2[0] - 0.5) < 1e-6
    write_wavefront(str(tmp_path / "two.obj"), [cube, ball])
    vv, ff = load_wavefront(str(tmp_path / "two.obj"))
    assert len(vv) == 8 + len(v) and len(ff) == 12 + len(f)
    np.testing.assert_array_equal(ff[12:], f + 8)
    assert np.abs(vv[8:] - v).max() <= 1e-6
