"""Host-side scene assembly with the reference DEMSolver's setup semantics.

``SceneBuilder`` keeps the method names of ``deme::DEMSolver`` (src/DEM/API.h:44-443) for scene assembly and
reproduces what ``Initialize`` computes on the host before any kernel runs (src/DEM/APIPublic.cpp:659-693):

* the voxel bit split and length unit (figureOutNV, src/DEM/APIPrivate.cpp:222-333),
* the world origin and optional bounding box (APIPrivate.cpp:647-687),
* owner ordering: clumps in batch order, then external objects, then mesh objects (src/DEM/dT.cpp:522-640,
  src/DEM/kT.cpp:603-625),
* initial position encoding of ``xyz - LBF`` (hostPositionToVoxelID, src/DEM/HostSideHelpers.hpp:328-350),
* bin size and bin counts (decideBinSize, APIPrivate.cpp:335-369),
* expand factor (transferSimParams, APIPrivate.cpp:730-758),
* family masks and merged prescriptions (figureOutFamilyMasks, APIPrivate.cpp:574-645; the reserved family 255
  is made fixed in validateUserInputs, APIPrivate.cpp:906),
* the two JIT literals ``_l_`` / ``_voxelSize_`` that the kernels see (17-decimal std::fixed text,
  APIPrivate.cpp:1358-1359).

Everything is vectorised with numpy so million-clump scenes assemble in seconds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi

f32 = np.float32


def _kernel_literal(x: float) -> float:
    """Value of a double printed with std::fixed precision 17 and parsed back (to_string_with_precision)."""
    return float("%.17f" % x)


def _normalize_f32(v) -> np.ndarray:
    """helper_math normalize on the host: v * (1 / sqrtf(dot(v, v))) in float."""
    v = np.asarray(v, dtype=f32)
    d = f32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    inv = f32(f32(1.0) / f32(np.sqrt(d)))
    return (v * inv).astype(f32)


@dataclass
class Material:
    load_order: int
    props: dict


@dataclass
class ClumpTemplate:
    mark: int
    mass: float
    moi: tuple
    radii: np.ndarray
    rel_pos: np.ndarray
    materials: list
    name: str = ""  # DEMClumpTemplate::m_name; "%04d" of the load count unless assigned (APIPublic.cpp:337-341)

    def AssignName(self, some_name: str):
        self.name = some_name


class ClumpBatch:
    """DEMClumpBatch (src/DEM/Structs.h:450-559)."""

    def __init__(self, types: np.ndarray, xyz: np.ndarray):
        n = len(types)
        self.types = np.asarray(types, dtype=np.int64)
        self.xyz = np.ascontiguousarray(xyz, dtype=f32).reshape(n, 3)
        self.vel = np.zeros((n, 3), f32)
        self.ang_vel = np.zeros((n, 3), f32)
        self.oriQ = np.zeros((n, 4), f32)  # (w, x, y, z)
        self.oriQ[:, 0] = 1
        self.families = np.zeros(n, np.uint32)
        self.family_is_specified = False
        self.analytical_objects = None  # packed scenes: the external objects these clumps may touch
        self.scene_box = None  # packed scenes: (lower, upper) corner of this batch's own search grid

    def SetSceneBox(self, lower, upper):
        """Packed independent scenes (no reference counterpart): this batch is a scene of its own whose spheres stay
        inside the box [lower, upper] (user coordinates); it gets a contact-search grid of its own, with cells
        sized by its own spheres.  Either every batch of a scene builder has a box or none has."""
        self.scene_box = (np.asarray(lower, np.float64), np.asarray(upper, np.float64))

    def SetAnalyticalObjects(self, objs):
        """Packed independent scenes (no reference counterpart): the spheres of this batch meet only the analytical
        components of ``objs`` (consecutively loaded external objects), not the walls of other scenes."""
        objs = list(objs)
        orders = [o.load_order for o in objs]
        if orders != list(range(orders[0], orders[0] + len(orders))):
            raise ValueError("the external objects of one batch must have been added consecutively")
        self.analytical_objects = objs

    def GetNumClumps(self) -> int:
        return len(self.types)

    def SetVel(self, v):
        self.vel[:] = np.asarray(v, f32).reshape(-1, 3)

    def SetAngVel(self, w):
        self.ang_vel[:] = np.asarray(w, f32).reshape(-1, 3)

    def SetOriQ(self, q):
        """Quaternions as (w, x, y, z) rows."""
        self.oriQ[:] = np.asarray(q, f32).reshape(-1, 4)

    def SetFamilies(self, fams):
        fams = np.asarray(fams, np.int64)
        if np.any(fams > 255) or np.any(fams < 0):
            raise ValueError("family numbers must be in [0, 255]")
        self.families[:] = fams
        self.family_is_specified = True

    def SetFamily(self, fam: int):
        self.SetFamilies(np.full(self.GetNumClumps(), fam))


class ExternObj:
    """DEMExternObj (src/DEM/BdrsAndObjs.h:95-170), plus cylinder and cone components."""

    def __init__(self, load_order: int):
        self.load_order = load_order
        self.family_code = capi.RESERVED_FAMILY
        self.init_pos = np.zeros(3, f32)
        self.mass = f32(1e15)
        self.moi = np.full(3, f32(1e15))
        self.components = []  # (type, material, pos, rot, s1, s2, s3, normal)

    def SetFamily(self, code: int):
        if code > 255 or code < 0:
            raise ValueError(f"family number {code} is larger than the max allowance 255")
        self.family_code = code

    def SetMass(self, m):
        self.mass = f32(m)

    def SetMOI(self, moi):
        self.moi = np.asarray(moi, f32)

    def AddPlane(self, pos, normal, material: Material):
        self.components.append((capi.ANAL_PLANE, material, np.asarray(pos, f32), _normalize_f32(normal), 0.0, 0.0,
                                0.0, 0))

    def AddPlate(self, pos, normal, xdim: float, ydim: float, material: Material):
        """DEMExternObj::AddPlate (src/DEM/BdrsAndObjs.h:152-170): kept as a component with its half sizes, and, as
        in the reference (DEMHelperKernels.cu:385-387, 439-441), it meets no sphere."""
        self.components.append((capi.ANAL_PLATE, material, np.asarray(pos, f32), _normalize_f32(normal),
                                float(f32(xdim) / 2.0), float(f32(ydim) / 2.0), 0.0, 0))

    def AddCylinder(self, point, axis, radius: float, material: Material, normal_outward: bool = False):
        """Infinite cylinder through ``point`` along ``axis``.  Spheres live inside unless normal_outward."""
        self.components.append((capi.ANAL_CYLINDER, material, np.asarray(point, f32), _normalize_f32(axis),
                                float(radius), 0.0, 0.0, 1 if normal_outward else 0))

    def AddCone(self, apex, axis, half_angle: float, u_min: float, u_max: float, material: Material,
                normal_outward: bool = False):
        """Cone with apex ``apex`` opening along ``axis``; the wall exists for axial distance [u_min, u_max]."""
        self.components.append((capi.ANAL_CONE, material, np.asarray(apex, f32), _normalize_f32(axis),
                                float(half_angle), float(u_min), float(u_max), 1 if normal_outward else 0))


def write_wavefront(path: str, meshes) -> None:
    """DEMMeshConnected::WriteWavefront (src/DEM/MeshUtils.cpp:119-165): every mesh's vertices, then the normals of
    the meshes that have them, then the faces with indices offset into one object (``f a//n b//n c//n`` for a mesh
    with normals); numbers printed as C++'s default stream prints a float (6 significant digits)."""
    with open(path, "w") as fh:
        for m in meshes:
            for v in m.vertices:
                fh.write("v " + " ".join(f"{float(x):g}" for x in v) + "\n")
        for m in meshes:
            for v in m.normals:
                fh.write("vn " + " ".join(f"{float(x):g}" for x in v) + "\n")
        off, noff = 1, 1
        for m in meshes:
            if len(m.normals):
                if len(m.face_normals) != len(m.faces):
                    raise ValueError("a mesh with normals needs one normal triple per facet")
                for f, n in zip(m.faces, m.face_normals):
                    fh.write("f " + " ".join(f"{int(i) + off}//{int(j) + noff}" for i, j in zip(f, n)) + "\n")
            else:
                for f in m.faces:
                    fh.write("f " + " ".join(str(int(i) + off) for i in f) + "\n")
            off += len(m.vertices)
            noff += len(m.normals)


def mesh_mass_properties(vertices, faces):
    """Volume (the mass at unit density), centroid and the principal-axis-aligned moments of inertia about the
    centroid of the solid a closed, outward-wound triangle mesh bounds, by the divergence theorem over each facet
    (Eberly's polyhedral mass properties).  In float64."""
    t = np.asarray(vertices, np.float64)[np.asarray(faces, np.int64)]
    p0, p1, p2 = t[:, 0], t[:, 1], t[:, 2]
    d = np.cross(p1 - p0, p2 - p0)

    def sub(w0, w1, w2):
        t0 = w0 + w1
        f1 = t0 + w2
        t1 = w0 * w0
        t2 = t1 + w1 * t0
        f2 = t2 + w2 * f1
        f3 = w0 * t1 + w1 * t2 + w2 * f2
        return f1, f2, f3, f2 + w0 * (f1 + w0), f2 + w1 * (f1 + w1), f2 + w2 * (f1 + w2)

    fx = sub(p0[:, 0], p1[:, 0], p2[:, 0])
    fy = sub(p0[:, 1], p1[:, 1], p2[:, 1])
    fz = sub(p0[:, 2], p1[:, 2], p2[:, 2])
    mass = np.sum(d[:, 0] * fx[0]) / 6.0
    cx = np.sum(d[:, 0] * fx[1]) / 24.0 / mass
    cy = np.sum(d[:, 1] * fy[1]) / 24.0 / mass
    cz = np.sum(d[:, 2] * fz[1]) / 24.0 / mass
    xx = np.sum(d[:, 0] * fx[2]) / 60.0
    yy = np.sum(d[:, 1] * fy[2]) / 60.0
    zz = np.sum(d[:, 2] * fz[2]) / 60.0
    inertia = np.array([yy + zz - mass * (cy * cy + cz * cz), zz + xx - mass * (cz * cz + cx * cx),
                        xx + yy - mass * (cx * cx + cy * cy)])
    return float(mass), np.array([cx, cy, cz]), inertia


def read_clump_components(path: str, x_id="x", y_id="y", z_id="z", r_id="r"):
    """DEMClumpTemplate::ReadComponentFromFile (src/DEM/Structs.h:419-437): radii and relative positions from a CSV
    file with a header row naming the columns (any order among others; a missing column or an empty cell reads 0),
    the numbers formed as the reference's CSV reader forms them (io.csv_floats)."""
    with open(path) as fh:
        # the reader's default comment policy: a line starting with '#', and a blank line, are skipped
        lines = [ln for ln in fh.read().splitlines() if ln.strip(" \t") and not ln.startswith("#")]
    if not lines:
        return np.zeros(0, f32), np.zeros((0, 3), f32)
    from .io import csv_floats
    head = [c.strip() for c in lines[0].split(",")]
    cols = [head.index(k) if k in head else -1 for k in (x_id, y_id, z_id, r_id)]
    cells = []
    for ln in lines[1:]:
        row = ln.split(",")
        cells.extend(row[c] if 0 <= c < len(row) else "" for c in cols)
    a = csv_floats(cells).reshape(-1, 4)
    return a[:, 3].copy(), a[:, :3].copy()


def read_wavefront(path: str) -> dict:
    """The records of a Wavefront OBJ file as the reference's parser reads them (OBJ::ParseLine,
    src/core/utils/WavefrontMeshLoader.hpp:578-647, behind DEMMeshConnected::LoadWavefrontMesh,
    src/DEM/MeshUtils.cpp:44-112): ``v`` and ``vn`` records with three coordinates (a float rounded from the decimal
    value), ``f`` records of three or more corners split into fans about the first corner, tags in any letter case.
    Returns the vertices (n x 3), the facets' vertex indices (m x 3), the normals and the facets' normal indices
    (the corners' ``a//n`` or ``a/t/n`` normal indices, three at a time).  Where the reference misreads a record,
    this reads it as the OBJ format defines it: a negative index counts back from the last record read (the
    reference subtracts one from it, leaving an index outside the mesh), and a vertex or normal record with more
    numbers (a weight, a colour) or a trailing ``#`` comment is kept with its first three (the reference drops it,
    shifting every later index)."""
    verts, norms, faces, flat_n = [], [], [], []
    with open(path) as fh:
        for line in fh:
            tok = line.split("#", 1)[0].split()
            if not tok:
                continue
            tag = tok[0].lower()
            if tag in ("v", "vn"):
                if len(tok) >= 4:
                    (verts if tag == "v" else norms).append([float(x) for x in tok[1:4]])
            elif tag == "f" and len(tok) >= 4:
                vi, ni = [], []
                for t in tok[1:]:
                    parts = t.split("/")
                    i = int(parts[0])
                    vi.append(i - 1 if i > 0 else len(verts) + i)
                    if len(parts) >= 3 and parts[2]:
                        k = int(parts[2])
                        ni.append(k - 1 if k > 0 else len(norms) + k)
                    else:
                        ni.append(None)
                for j in range(1, len(vi) - 1):
                    faces.append([vi[0], vi[j], vi[j + 1]])
                    flat_n.extend(ni[c] for c in (0, j, j + 1) if ni[c] is not None)
    nf = len(flat_n) // 3
    return {"vertices": np.asarray(verts, f32).reshape(-1, 3), "faces": np.asarray(faces, np.int64).reshape(-1, 3),
            "normals": np.asarray(norms, f32).reshape(-1, 3),
            "face_normals": np.asarray(flat_n[:3 * nf], np.int64).reshape(-1, 3)}


def load_wavefront(path: str) -> tuple[np.ndarray, np.ndarray]:
    """Vertices (n x 3) and triangles (m x 3 vertex indices) of a Wavefront OBJ file (read_wavefront)."""
    r = read_wavefront(path)
    return r["vertices"], r["faces"]


def facet_nodes(vertices, faces, normals=None, face_normals=None) -> np.ndarray:
    """Each facet's three nodes (m x 9, float32).  Given the file's normals, a facet whose right-hand normal
    cross(p2 - p1, p3 - p1) points away from the normal of its first corner has nodes 2 and 3 swapped
    (DEMMeshConnected::UseNormals, applied at initialisation: src/DEM/APIPrivate.cpp:545-560), the products
    in float as the reference's float3 arithmetic forms them."""
    t = np.asarray(vertices, f32)[np.asarray(faces, np.int64)]
    if normals is not None:
        if len(face_normals) < len(t):
            raise ValueError("UseNormals needs a normal index for every facet")
        n = np.asarray(normals, f32)[np.asarray(face_normals, np.int64)[:len(t), 0]]
        ab, ac = t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]
        cx = ab[:, 1] * ac[:, 2] - ab[:, 2] * ac[:, 1]
        cy = ab[:, 2] * ac[:, 0] - ab[:, 0] * ac[:, 2]
        cz = ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0]
        flip = (cx * n[:, 0] + cy * n[:, 1]) + cz * n[:, 2] < 0
        t = t.copy()
        t[flip, 1], t[flip, 2] = t[flip, 2], t[flip, 1].copy()
    return t.reshape(-1, 9)


class MeshObj:
    """DEMMeshConnected (src/DEM/BdrsAndObjs.h:173-300): a body represented by triangle facets, given in its own
    frame.  Defaults as the reference's: the fixed family, mass 1, principal moments 1, at the origin."""

    def __init__(self, vertices, faces, load_order: int, normals=None, face_normals=None):
        self.vertices = np.asarray(vertices, f32).reshape(-1, 3).copy()
        self.faces = np.asarray(faces, np.int64).reshape(-1, 3)
        if self.faces.size and (self.faces.min() < 0 or self.faces.max() >= len(self.vertices)):
            raise ValueError("mesh face index out of range")
        # the file's normals and each facet's corner normal indices (kept for UseNormals and WriteWavefront)
        self.normals = np.zeros((0, 3), f32) if normals is None else np.asarray(normals, f32).reshape(-1, 3).copy()
        self.face_normals = np.zeros((0, 3), np.int64) if face_normals is None else \
            np.asarray(face_normals, np.int64).reshape(-1, 3)
        if self.face_normals.size and (self.face_normals.min() < 0 or self.face_normals.max() >= len(self.normals)):
            raise ValueError("mesh normal index out of range")
        self.use_normals = False
        self.load_order = load_order
        self.family_code = capi.RESERVED_FAMILY
        self.mass = f32(1.0)
        self.moi = np.ones(3, f32)
        self.init_pos = np.zeros(3, f32)
        self.init_oriQ = np.array([1, 0, 0, 0], f32)  # (w, x, y, z)
        self.init_vel = np.zeros(3, f32)
        self.init_angvel = np.zeros(3, f32)
        self.materials = None

    def GetNumTriangles(self) -> int:
        return len(self.faces)

    def GetTriangle(self, i: int) -> np.ndarray:
        return self.vertices[self.faces[i]]

    def Clear(self):
        self.vertices = np.zeros((0, 3), f32)
        self.faces = np.zeros((0, 3), np.int64)
        self.normals = np.zeros((0, 3), f32)
        self.face_normals = np.zeros((0, 3), np.int64)
        self.materials = None

    def UseNormals(self, use: bool = True):
        """At initialisation, order each facet's nodes so that their right-hand normal agrees with the file's
        normal at its first corner (facet_nodes)."""
        self.use_normals = bool(use)

    def facet_nodes(self) -> np.ndarray:
        """The facets' nodes in the mesh's own frame as initialisation places them (m x 9)."""
        if self.use_normals:
            return facet_nodes(self.vertices, self.faces, self.normals, self.face_normals)
        return facet_nodes(self.vertices, self.faces)

    def SetFamily(self, code: int):
        if code > 255 or code < 0:
            raise ValueError(f"family number {code} is larger than the max allowance 255")
        self.family_code = code

    def SetMass(self, m):
        self.mass = f32(m)

    def SetMOI(self, moi):
        self.moi = np.asarray(moi, f32).reshape(3)

    def SetMaterial(self, mat):
        """One material for every facet, or a list with one per facet."""
        if isinstance(mat, Material):
            mat = [mat] * self.GetNumTriangles()
        if len(mat) != self.GetNumTriangles():
            raise ValueError(f"SetMaterial input argument must have length {self.GetNumTriangles()} (not "
                             f"{len(mat)}), same as the number of triangle facets in the mesh.")
        self.materials = list(mat)

    def SetInitPos(self, pos):
        self.init_pos = np.asarray(pos, f32).reshape(3)

    def SetInitQuat(self, q):
        """(w, x, y, z)."""
        self.init_oriQ = np.asarray(q, f32).reshape(4)

    def SetInitVel(self, v):
        self.init_vel = np.asarray(v, f32).reshape(3)

    def SetInitAngVel(self, w):
        self.init_angvel = np.asarray(w, f32).reshape(3)

    def Translate(self, d):
        """Moves the nodes in the mesh's own frame (DEMMeshConnected::Translate)."""
        self.vertices += np.asarray(d, f32).reshape(1, 3)

    def Scale(self, s):
        """Scales the nodes (one factor, or one per axis); the normals keep their direction on the scaled
        surface."""
        s = np.asarray(s, f32)
        self.vertices *= s
        if len(self.normals):
            n = self.normals.astype(np.float64) / np.broadcast_to(s, (3,)).astype(np.float64)
            self.normals = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(f32)

    def Rotate(self, q):
        """Rotates the nodes in the mesh's own frame by the unit quaternion q = (w, x, y, z)."""
        w, x, y, z = (float(c) for c in np.asarray(q, np.float64).reshape(4))
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        self.vertices = (self.vertices.astype(np.float64) @ R.T).astype(f32)
        self.normals = (self.normals.astype(np.float64) @ R.T).astype(f32)

    def ComputeMassProperties(self):
        """(mass at unit density, centroid, moments of inertia about the centroid) of the closed, outward-wound mesh
        (DEMMeshConnected::ComputeMassProperties, declared in src/DEM/BdrsAndObjs.h:291; see
        mesh_mass_properties)."""
        return mesh_mass_properties(self.vertices, self.faces)

    @staticmethod
    def WriteWavefront(path: str, meshes):
        write_wavefront(path, meshes)

    @staticmethod
    def Merge(meshes) -> "MeshObj":
        """One mesh of the given meshes' nodes, normals and facets (declared in src/DEM/BdrsAndObjs.h:250); the
        first mesh's body properties, no materials."""
        vo = np.cumsum([0] + [len(m.vertices) for m in meshes])
        no = np.cumsum([0] + [len(m.normals) for m in meshes])
        cat = (lambda xs, shape, dt: np.concatenate(xs) if xs else np.zeros(shape, dt))
        out = MeshObj(cat([m.vertices for m in meshes], (0, 3), f32),
                      cat([m.faces + vo[i] for i, m in enumerate(meshes)], (0, 3), np.int64), 0,
                      cat([m.normals for m in meshes], (0, 3), f32),
                      cat([m.face_normals + no[i] for i, m in enumerate(meshes)], (0, 3), np.int64))
        if meshes:
            out.mass, out.moi, out.family_code = meshes[0].mass, meshes[0].moi.copy(), meshes[0].family_code
        return out


@dataclass
class _Prescription:
    family: int
    linPos: list = field(default_factory=lambda: ["none"] * 3)
    linVel: list = field(default_factory=lambda: ["none"] * 3)
    rotVel: list = field(default_factory=lambda: ["none"] * 3)
    linVelPrescribed: bool = False
    rotVelPrescribed: bool = False
    linPosPrescribed: bool = False
    rotPosPrescribed: bool = False


def _const(expr: str):
    """The value of a prescription string that is a plain number, else None: an expression (of the time t, as the
    reference accepts), compiled at run time into the integration kernel by deme_set_prescribed_motion."""
    try:
        return float(expr)
    except ValueError:
        return None


class BuiltScene:
    """Output of SceneBuilder.Initialize: parameter struct plus flattened arrays."""

    def __init__(self, params: capi.SimParams, arrays: dict, counts: dict, prescriptions, info: dict):
        self.params = params
        self.arrays = arrays
        self.counts = counts
        self.prescriptions = prescriptions
        self.info = info

    @property
    def n_spheres(self):
        return self.counts["s"]

    @property
    def n_owners(self):
        return self.counts["o"]

    def scene_struct(self):
        return capi.make_scene_struct(self.arrays, self.counts, self.prescriptions)

    def initial_state(self) -> dict:
        a = self.arrays
        st = {k: np.ascontiguousarray(a[k]).copy() for k in
              ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz", "vX", "vY", "vZ", "omgX", "omgY",
               "omgZ", "family")}
        return st

    def decode_positions(self, state: dict, kernel_literals: bool = True) -> np.ndarray:
        """Owner positions (relative to LBF) decoded like voxelIDToPosition."""
        p = self.params
        vs = p.voxel_size_kernel if kernel_literals else p.voxel_size
        l = p.l_kernel if kernel_literals else p.l
        v = state["voxel"].astype(np.uint64)
        mx = np.uint64((1 << p.nvXp2) - 1)
        my = np.uint64((1 << p.nvYp2) - 1)
        vx = v & mx
        vy = (v >> np.uint64(p.nvXp2)) & my
        vz = v >> np.uint64(p.nvXp2 + p.nvYp2)
        X = vx.astype(np.float64) * vs + state["locX"].astype(np.float64) * l
        Y = vy.astype(np.float64) * vs + state["locY"].astype(np.float64) * l
        Z = vz.astype(np.float64) * vs + state["locZ"].astype(np.float64) * l
        return np.stack([X, Y, Z], axis=1)


class SceneBuilder:
    """Scene assembly with the reference DEMSolver's method names (src/DEM/API.h)."""

    def __init__(self):
        self.materials: list[Material] = []
        self.templates: list[ClumpTemplate] = []
        self.batches: list[ClumpBatch] = []
        self.extern: list[ExternObj] = []
        self.meshes: list[MeshObj] = []
        self.box = None
        self.dir_exact = None
        self.origin = "explicit"
        self.lbf = np.zeros(3, f32)
        self.bounding_bc = "none"
        self.bounding_mat = None
        self.G = np.zeros(3, f32)
        self.ts = -1.0
        self.bin_size = None
        self.expand_factor = 0.0
        self.expand_fixed = False
        self.max_vel = -1.0
        self.safety = 1.0
        self.update_freq = 0
        self.integrator = capi.EXTENDED_TAYLOR
        self.no_contact_pairs = []
        self.prescriptions: list[_Prescription] = []
        self.n_wildcards = 4
        self.explicit_nv = None

    # ---- world ----
    def InstructBoxDomainDimension(self, x, y, z, dir_exact=None):
        self.box = np.array([x, y, z], f32)
        self.dir_exact = dir_exact

    def InstructBoxDomainNumVoxel(self, x, y, z, len_unit=1e-10):
        """The voxel bit split and length unit given directly (APIPublic.cpp:94-114); the domain is the voxel
        world."""
        if int(x) + int(y) + int(z) != 64:
            raise ValueError("Please give voxel numbers (as powers of 2) along each direction such that they add up "
                             "to 64.")
        self.explicit_nv = (int(x), int(y), int(z), float(np.float32(len_unit)))

    def SetCoordSysOrigin(self, where):
        if isinstance(where, str):
            self.origin = where
        else:
            self.lbf = np.asarray(where, f32)
            self.origin = "explicit"

    def InstructBoxDomainBoundingBC(self, inst: str, mat: Material):
        self.bounding_bc = inst
        self.bounding_mat = mat

    def SetGravitationalAcceleration(self, g):
        self.G = np.asarray(g, f32)

    def SetInitTimeStep(self, ts):
        self.ts = float(ts)

    def SetInitBinSize(self, b):
        self.bin_size = float(b)

    def SetCDUpdateFreq(self, f):
        self.update_freq = int(f)

    def SetExpandFactor(self, beta, fix=True):
        self.expand_factor = float(np.float32(beta))
        self.expand_fixed = fix

    def SetMaxVelocity(self, v):
        self.max_vel = float(np.float32(v))

    def SetExpandSafetyParam(self, s):
        self.safety = float(np.float32(s))

    def SetIntegrator(self, intg):
        self.integrator = intg

    def UseFrictionlessHertzianModel(self):
        """The frictionless Hertzian model (the reference's FrictionlessHertzianForceModel.cu): the normal spring and
        damper only, no rolling resistance, no tangential force and so no contact wildcards (history)."""
        self.n_wildcards = 0

    def UseFrictionalHertzianModel(self):
        """The full Hertz--Mindlin model (the default): four contact wildcards (tangential displacement, time)."""
        self.n_wildcards = 4

    # ---- materials / templates / clumps ----
    def LoadMaterial(self, props: dict) -> Material:
        m = Material(len(self.materials), {k: float(np.float32(v)) for k, v in props.items()})
        self.materials.append(m)
        return m

    def LoadClumpType(self, mass, moi, radii, rel_pos, materials=None) -> ClumpTemplate:
        """Components as arrays (radii, rel_pos, materials), or from a CSV file: LoadClumpType(mass, moi, path,
        materials) (API.h:175-184; the file's header names the columns x, y, z and r, read as
        DEMClumpTemplate::ReadComponentFromFile reads them)."""
        if isinstance(radii, str):
            radii, rel_pos, materials = (*read_clump_components(radii), rel_pos)
        radii = np.asarray(radii, f32).reshape(-1)
        rel_pos = np.asarray(rel_pos, f32).reshape(-1, 3)
        if not isinstance(materials, (list, tuple)):
            materials = [materials] * len(radii)
        t = ClumpTemplate(len(self.templates), float(np.float32(mass)), tuple(np.asarray(moi, f32)), radii, rel_pos,
                          list(materials), "%04d" % len(self.templates))
        self.templates.append(t)
        return t

    def LoadSphereType(self, mass, radius, material) -> ClumpTemplate:
        moi = 0.4 * mass * radius * radius
        return self.LoadClumpType(mass, (moi, moi, moi), [radius], [[0, 0, 0]], material)

    def AddClumps(self, types, xyz) -> ClumpBatch:
        xyz = np.asarray(xyz, f32).reshape(-1, 3)
        if isinstance(types, ClumpTemplate):
            types = np.full(len(xyz), types.mark)
        elif isinstance(types, (list, tuple)) and len(types) and isinstance(types[0], ClumpTemplate):
            types = np.array([t.mark for t in types])
        b = ClumpBatch(np.asarray(types), xyz)
        self.batches.append(b)
        return b

    def AddExternalObject(self) -> ExternObj:
        o = ExternObj(len(self.extern))
        self.extern.append(o)
        return o

    def AddWavefrontMeshObject(self, mesh, material: Material | None = None, load_normals: bool = True) -> MeshObj:
        """A mesh-represented body: a Wavefront OBJ path (its normals kept unless load_normals is False), or
        (vertices, faces) arrays (AddWavefrontMeshObject, src/DEM/API.h:231-238)."""
        if isinstance(mesh, MeshObj):
            m = mesh
            m.load_order = len(self.meshes)
        elif isinstance(mesh, str):
            r = read_wavefront(mesh)
            m = MeshObj(r["vertices"], r["faces"], len(self.meshes), *((r["normals"], r["face_normals"])
                                                                       if load_normals else ()))
        else:
            v, f = mesh
            m = MeshObj(v, f, len(self.meshes))
        if material is not None:
            m.SetMaterial(material)
        self.meshes.append(m)
        return m

    def AddBCPlane(self, pos, normal, material) -> ExternObj:
        o = self.AddExternalObject()
        o.AddPlane(pos, normal, material)
        return o

    # ---- families ----
    def DisableContactBetweenFamilies(self, a, b):
        lo, hi = min(a, b), max(a, b)
        if (1 + hi) * hi // 2 + lo >= 255 * 256 // 2:
            raise IndexError("family mask entry out of range (the reference's mask table holds 32640 entries)")
        self.no_contact_pairs.append((a, b))

    def SetFamilyFixed(self, fam):
        p = _Prescription(fam, linPos=["none"] * 3, linVel=["0"] * 3, rotVel=["0"] * 3, linVelPrescribed=True,
                          rotVelPrescribed=True, linPosPrescribed=True, rotPosPrescribed=True)
        self.prescriptions.append(p)

    def SetFamilyPrescribedLinVel(self, fam, vx, vy, vz, dictate=True):
        self.prescriptions.append(_Prescription(fam, linVel=[vx, vy, vz], linVelPrescribed=dictate,
                                                rotVelPrescribed=dictate))

    def SetFamilyPrescribedAngVel(self, fam, wx, wy, wz, dictate=True):
        self.prescriptions.append(_Prescription(fam, rotVel=[wx, wy, wz], linVelPrescribed=dictate,
                                                rotVelPrescribed=dictate))

    def SetFamilyPrescribedPosition(self, fam, x, y, z):
        self.prescriptions.append(_Prescription(fam, linPos=[x, y, z], linPosPrescribed=True, rotPosPrescribed=True))

    # ---- Initialize ----
    def _figure_out_nv(self):
        """figureOutNV, src/DEM/APIPrivate.cpp:222-333 (NONE exact direction)."""
        XYZ = [f32(v) for v in self.box]
        rank = [0, 1, 2]
        for i in range(2):
            for j in range(i + 1, 3):
                if XYZ[i] > XYZ[j]:
                    XYZ[i], XYZ[j] = XYZ[j], XYZ[i]
                    rank[i], rank[j] = rank[j], rank[i]
        size321 = list(XYZ)
        more = [0, 0]
        while XYZ[0] < XYZ[1]:
            if math.sqrt(2.0) * float(XYZ[0]) > float(XYZ[1]):
                break
            more[0] += 1
            XYZ[0] = f32(float(XYZ[0]) * 2.0)
        while XYZ[1] < XYZ[2]:
            if math.sqrt(2.0) * float(XYZ[1]) > float(XYZ[2]):
                break
            more[1] += 1
            XYZ[1] = f32(float(XYZ[1]) * 2.0)
        base = (64 - more[0] - more[1]) // 3
        left = (64 - more[0] - more[1]) % 3
        b3 = base
        b2 = b3 + more[0]
        b1 = b2 + more[1]
        while left > 0:
            if b3 < b2:
                b3 += 1
            elif b2 < b1:
                b2 += 1
            else:
                b1 += 1
            left -= 1
        bits = [b3, b2, b1]
        if sum(bits) > 64:
            # The reference's split (APIPrivate.cpp:267-281) subtracts the second-place extra bits once but gives
            # them to both larger axes, so it overshoots 64 bits whenever that extra is non-zero; the top bits of
            # the voxel id then wrap and positions jump.  Refuse such domains instead of corrupting positions.
            raise ValueError(f"domain {list(map(float, self.box))} needs {sum(bits)} voxel bits (> 64) under the "
                             "reference's bit split; use a domain whose two smaller sides are within a factor sqrt(2)")
        if self.dir_exact is not None:
            raise NotImplementedError("exact-direction world sizing")
        ls = [float(size321[i]) / 2.0**16 / 2.0**bits[i] for i in range(3)]
        l = float(f32(max(ls[0], max(ls[1], ls[2]))))
        nv = [0, 0, 0]
        for i in range(3):
            nv[rank[i]] = bits[i]
        return nv, l

    def Initialize(self) -> BuiltScene:
        if self.box is None and self.explicit_nv is None:
            raise ValueError("InstructBoxDomainDimension must be called before Initialize")
        if self.explicit_nv is not None:
            nv, l = list(self.explicit_nv[:3]), self.explicit_nv[3]
            voxel = float(1 << 16) * l
            self.box = np.array([voxel * (1 << n) for n in nv], f32)
        else:
            nv, l = self._figure_out_nv()
        voxel_size = float(1 << 16) * l
        if self.origin == "center":
            self.lbf = (-self.box / f32(2.0)).astype(f32)
        elif self.origin != "explicit":
            raise ValueError("Unrecognized location of system origin.")
        lbf = self.lbf
        if self.bounding_bc != "none":
            b = self.AddExternalObject()
            X, Y, Z = lbf
            bx, by, bz = self.box
            m = self.bounding_mat
            b.AddPlane([X + bx / 2.0, Y + by / 2.0, Z], [0, 0, 1], m)
            if self.bounding_bc != "only_bottom":
                b.AddPlane([X, Y + by / 2.0, Z + bz / 2.0], [1, 0, 0], m)
                b.AddPlane([X + bx, Y + by / 2.0, Z + bz / 2.0], [-1, 0, 0], m)
                b.AddPlane([X + bx / 2.0, Y, Z + bz / 2.0], [0, 1, 0], m)
                b.AddPlane([X + bx / 2.0, Y + by, Z + bz / 2.0], [0, -1, 0], m)
                if self.bounding_bc != "top_open":
                    b.AddPlane([X + bx / 2.0, Y + by / 2.0, Z + bz], [0, 0, -1], m)
        # validateUserInputs: family 255 is fixed
        self.SetFamilyFixed(capi.RESERVED_FAMILY)

        # ---- owners: clumps ----
        nT = len(self.templates)
        tmpl_nc = np.array([len(t.radii) for t in self.templates], np.int64)
        tmpl_off = np.zeros(nT + 1, np.int64)
        tmpl_off[1:] = np.cumsum(tmpl_nc)
        all_r = np.concatenate([t.radii for t in self.templates]) if nT else np.zeros(0, f32)
        all_p = np.concatenate([t.rel_pos for t in self.templates]) if nT else np.zeros((0, 3), f32)
        all_m = np.concatenate([[m.load_order for m in t.materials] for t in self.templates]).astype(np.uint16) \
            if nT else np.zeros(0, np.uint16)
        t_mass = np.array([t.mass for t in self.templates], f32)
        t_moi = np.array([t.moi for t in self.templates], f32).reshape(-1, 3)
        if self.batches:
            types = np.concatenate([b.types for b in self.batches])
            xyz = np.concatenate([b.xyz for b in self.batches])
            vel = np.concatenate([b.vel for b in self.batches])
            angv = np.concatenate([b.ang_vel for b in self.batches])
            oriq = np.concatenate([b.oriQ for b in self.batches])
            fams = np.concatenate([b.families for b in self.batches])
        else:
            types = np.zeros(0, np.int64)
            xyz = vel = angv = np.zeros((0, 3), f32)
            oriq = np.zeros((0, 4), f32)
            fams = np.zeros(0, np.uint32)
        nClumps = len(types)
        nExt = len(self.extern)
        nMesh = len(self.meshes)
        for m in self.meshes:
            if m.materials is None:
                raise ValueError("A meshed object is loaded but does not have associated material. Please assign "
                                 "material to meshes via SetMaterial.")
        nO = nClumps + nExt + nMesh
        ncomp = tmpl_nc[types] if nClumps else np.zeros(0, np.int64)
        nS = int(ncomp.sum())
        # sphere arrays
        sph_owner = np.repeat(np.arange(nClumps, dtype=np.uint32), ncomp)
        first = np.zeros(nClumps + 1, np.int64)
        first[1:] = np.cumsum(ncomp)
        local = np.arange(nS, dtype=np.int64) - np.repeat(first[:-1], ncomp)
        gidx = np.repeat(tmpl_off[types], ncomp) + local
        radius = all_r[gidx].astype(f32)
        rel = all_p[gidx].astype(f32)
        smat_w = all_m[gidx].astype(np.uint16)
        # owner positions relative to LBF in float (input_xyz - LBF, src/DEM/dT.cpp:539)
        ext_xyz = np.array([o.init_pos for o in self.extern] + [m.init_pos for m in self.meshes], f32).reshape(-1, 3)
        pos_f = np.concatenate([xyz, ext_xyz]).astype(f32) - lbf.astype(f32)
        vox, lx, ly, lz = self.host_position_to_voxel(pos_f.astype(np.float64), nv, voxel_size, float(l))
        oriQw = np.ones(nO, f32)
        oriQx = np.zeros(nO, f32)
        oriQy = np.zeros(nO, f32)
        oriQz = np.zeros(nO, f32)
        oriQw[:nClumps], oriQx[:nClumps], oriQy[:nClumps], oriQz[:nClumps] = oriq.T
        vX = np.zeros(nO, f32)
        vY = np.zeros(nO, f32)
        vZ = np.zeros(nO, f32)
        vX[:nClumps], vY[:nClumps], vZ[:nClumps] = vel.T
        wX = np.zeros(nO, f32)
        wY = np.zeros(nO, f32)
        wZ = np.zeros(nO, f32)
        wX[:nClumps], wY[:nClumps], wZ[:nClumps] = angv.T
        m0 = nClumps + nExt  # mesh owners follow the external objects (src/DEM/kT.cpp:603-625)
        for i, m in enumerate(self.meshes):
            oriQw[m0 + i], oriQx[m0 + i], oriQy[m0 + i], oriQz[m0 + i] = m.init_oriQ
            vX[m0 + i], vY[m0 + i], vZ[m0 + i] = m.init_vel
            wX[m0 + i], wY[m0 + i], wZ[m0 + i] = m.init_angvel
        family = np.concatenate([fams, [o.family_code for o in self.extern],
                                 [m.family_code for m in self.meshes]]).astype(np.uint8)
        mass = np.concatenate([t_mass[types], [o.mass for o in self.extern], [m.mass for m in self.meshes]]).astype(f32)
        moi = np.concatenate([t_moi[types], np.array([o.moi for o in self.extern], f32).reshape(-1, 3),
                              np.array([m.moi for m in self.meshes], f32).reshape(-1, 3)]).astype(f32)
        # ---- mesh facets ----
        tri = [m.facet_nodes() for m in self.meshes]
        tri = np.concatenate(tri).astype(f32) if tri else np.zeros((0, 9), f32)
        nTri = len(tri)
        tri_owner = np.concatenate([np.full(m.GetNumTriangles(), m0 + i, np.uint32) for i, m in enumerate(self.meshes)]) \
            if nMesh else np.zeros(0, np.uint32)
        tri_material = np.array([mt.load_order for m in self.meshes for mt in m.materials], np.uint16)
        if nTri:
            t64 = tri.astype(np.float64)
            area2 = np.sum(np.cross(t64[:, 3:6] - t64[:, 0:3], t64[:, 6:9] - t64[:, 0:3]) ** 2, axis=1)
            bad = np.nonzero(~(area2 > 0.0))[0]
            if len(bad):
                raise ValueError(f"mesh facet {int(bad[0])} has zero area (or non-finite nodes); "
                                 f"{len(bad)} such facets in all")

        # ---- analytical components ----
        comps = []
        for oi, o in enumerate(self.extern):
            for (tp, mat, pos, rot, s1, s2, s3, nrm) in o.components:
                comps.append((tp, nClumps + oi, nrm, mat.load_order, pos, rot, s1, s2, s3, o.mass))
        nA = len(comps)
        restricted = any(b.analytical_objects is not None for b in self.batches)
        if nA > 255 and not restricted:
            raise ValueError("at most 255 analytical components (objID_t is uint8)")
        owner_anal = None
        if restricted:
            comp_start = np.zeros(nExt + 1, np.int64)
            comp_start[1:] = np.cumsum([len(o.components) for o in self.extern])
            first = np.zeros(nO, np.uint32)
            count = np.zeros(nO, np.uint32)
            o0 = 0
            for b in self.batches:
                nb_ = b.GetNumClumps()
                if b.analytical_objects is None:
                    f_, c_ = 0, nA
                else:
                    lo = b.analytical_objects[0].load_order
                    hi = b.analytical_objects[-1].load_order + 1
                    f_, c_ = int(comp_start[lo]), int(comp_start[hi] - comp_start[lo])
                if c_ > 255:
                    raise ValueError("a batch may meet at most 255 analytical components")
                first[o0:o0 + nb_] = f_
                count[o0:o0 + nb_] = c_
                o0 += nb_
            owner_anal = (first, count)
        anal = {
            "anal_type": np.array([c[0] for c in comps], np.uint8),
            "anal_owner": np.array([c[1] for c in comps], np.uint32),
            "anal_normal": np.array([c[2] for c in comps], np.uint8),
            "anal_material": np.array([c[3] for c in comps], np.uint16),
            "anal_relX": np.array([c[4][0] for c in comps], f32),
            "anal_relY": np.array([c[4][1] for c in comps], f32),
            "anal_relZ": np.array([c[4][2] for c in comps], f32),
            "anal_rotX": np.array([c[5][0] for c in comps], f32),
            "anal_rotY": np.array([c[5][1] for c in comps], f32),
            "anal_rotZ": np.array([c[5][2] for c in comps], f32),
            "anal_size1": np.array([c[6] for c in comps], f32),
            "anal_size2": np.array([c[7] for c in comps], f32),
            "anal_size3": np.array([c[8] for c in comps], f32),
            "anal_mass": np.array([c[9] for c in comps], f32),
        }
        # ---- materials ----
        nM = len(self.materials)

        def matarr(key):
            return np.array([m.props.get(key, 0.0) for m in self.materials], f32)

        # ---- family masks ----
        masks = np.zeros(capi.NUM_FAMILY_MASK, np.uint8)
        for a, b in self.no_contact_pairs:
            lo, hi = min(a, b), max(a, b)
            masks[(1 + hi) * hi // 2 + lo] = 1
        presc = self._merge_prescriptions()

        # ---- bins ----
        rmin = float(np.min(radius)) if nS else float("inf")
        for t in self.templates:
            rmin = min(rmin, float(np.min(t.radii)))
        if self.bin_size is not None:
            bin_size = self.bin_size
        else:
            if not rmin > 1e-12:
                raise ValueError("spheres with zero radius and no bin size given")
            bin_size = 2.0 * float(f32(rmin))
        nb = [int(voxel_size * float(1 << nv[i]) / bin_size) + 1 for i in range(3)]
        if nb[0] * nb[1] * nb[2] > 0xFFFFFFFF:
            raise ValueError("too many bins for binID_t; enlarge the bin size")
        # ---- expand factor ----
        beta = self.expand_factor
        if not self.expand_fixed:
            beta = float(f32(self.max_vel * self.ts * self.update_freq * self.safety))

        p = capi.SimParams()
        p.nvXp2, p.nvYp2, p.nvZp2 = nv
        p.nbX, p.nbY, p.nbZ = nb
        p.l = float(l)
        p.voxel_size = voxel_size
        p.l_kernel = _kernel_literal(float(l))
        p.voxel_size_kernel = _kernel_literal(voxel_size)
        p.bin_size = bin_size
        p.lbf[:] = [float(v) for v in lbf]
        p.G[:] = [float(v) for v in self.G]
        p.h = float(f32(self.ts))
        p.beta = float(f32(beta))
        p.integrator = self.integrator
        p.cd_update_freq = self.update_freq
        p.n_contact_wildcards = self.n_wildcards
        p.domain[:] = [float(v) for v in self.box]

        wide = len(self.materials) > 256
        ext_arrays = {}
        if wide:
            ext_arrays["sphere_material_wide"] = smat_w
            ext_arrays["anal_material_wide"] = anal["anal_material"].astype(np.uint16)
        anal["anal_material"] = (anal["anal_material"] & 0xFF).astype(np.uint8)
        if owner_anal is not None:
            ext_arrays["owner_anal_first"], ext_arrays["owner_anal_count"] = owner_anal
        boxed = [b.scene_box is not None for b in self.batches]
        if any(boxed):
            if not all(boxed):
                raise ValueError("SetSceneBox: either every clump batch has a scene box or none has")
            owner_scene = np.zeros(nO, np.uint32)
            boxes = np.zeros((len(self.batches), 6), f32)
            o0 = 0
            for i, b in enumerate(self.batches):
                owner_scene[o0:o0 + b.GetNumClumps()] = i
                o0 += b.GetNumClumps()
                boxes[i, :3] = b.scene_box[0] - lbf
                boxes[i, 3:] = b.scene_box[1] - lbf
            ext_arrays["owner_scene"] = owner_scene
            ext_arrays["scene_box"] = boxes.ravel()
        arrays = dict(voxel=vox, locX=lx, locY=ly, locZ=lz, oriQw=oriQw, oriQx=oriQx, oriQy=oriQy, oriQz=oriQz,
                      vX=vX, vY=vY, vZ=vZ, omgX=wX, omgY=wY, omgZ=wZ, family=family, mass=mass,
                      mmiXX=np.ascontiguousarray(moi[:, 0]), mmiYY=np.ascontiguousarray(moi[:, 1]),
                      mmiZZ=np.ascontiguousarray(moi[:, 2]), sphere_owner=sph_owner, relX=np.ascontiguousarray(rel[:, 0]),
                      relY=np.ascontiguousarray(rel[:, 1]), relZ=np.ascontiguousarray(rel[:, 2]), radius=radius,
                      sphere_material=(smat_w & 0xFF).astype(np.uint8), mat_E=matarr("E"), mat_nu=matarr("nu"), mat_CoR=matarr("CoR"),
                      mat_mu=matarr("mu"), mat_Crr=matarr("Crr"), family_masks=masks, **anal, **ext_arrays)
        if nTri:
            arrays.update(tri_owner=tri_owner, tri_node1=np.ascontiguousarray(tri[:, 0:3]),
                          tri_node2=np.ascontiguousarray(tri[:, 3:6]), tri_node3=np.ascontiguousarray(tri[:, 6:9]),
                          tri_material=tri_material)
        counts = dict(o=nO, s=nS, a=nA, m=nM, t=nTri)
        info = dict(n_clumps=nClumps, n_ext=nExt, n_meshes=nMesh, n_templates=nT, rmin=rmin, bin_size=bin_size, nb=nb, nv=nv, l=l,
                    beta=beta, lbf=lbf.copy(), box=self.box.copy(), merged_prescriptions=self.merged_prescriptions,
                    motion_expressions=self.motion_expressions,
                    owner_template=np.asarray(types, np.int64) if nClumps else np.zeros(0, np.int64),
                    template_names=[t.name for t in self.templates])
        return BuiltScene(p, arrays, counts, presc, info)

    @staticmethod
    def host_position_to_voxel(pos: np.ndarray, nv, voxel_size: float, l: float):
        """hostPositionToVoxelID, src/DEM/HostSideHelpers.hpp:328-350, with saturating conversions."""
        q = pos / voxel_size
        q = np.where(q > 0, q, 0.0)
        n = np.floor(q).astype(np.uint64)
        sub = (pos - n.astype(np.float64) * voxel_size) / l
        sub = np.clip(np.where(sub > 0, sub, 0.0), 0, 65535)
        s = np.floor(sub).astype(np.uint16)
        vid = n[:, 0] + (n[:, 1] << np.uint64(nv[0])) + (n[:, 2] << np.uint64(nv[0] + nv[1]))
        return (vid.astype(np.uint64), np.ascontiguousarray(s[:, 0]), np.ascontiguousarray(s[:, 1]),
                np.ascontiguousarray(s[:, 2]))

    def _merge_prescriptions(self):
        arr = (capi.FamilyPrescription * capi.NUM_FAMILIES)()
        merged: dict[int, _Prescription] = {}
        for pr in self.prescriptions:
            m = merged.setdefault(pr.family, _Prescription(pr.family))
            for k in range(3):
                if pr.linPos[k] != "none":
                    m.linPos[k] = pr.linPos[k]
                if pr.linVel[k] != "none":
                    m.linVel[k] = pr.linVel[k]
                if pr.rotVel[k] != "none":
                    m.rotVel[k] = pr.rotVel[k]
            m.linVelPrescribed |= pr.linVelPrescribed
            m.rotVelPrescribed |= pr.rotVelPrescribed
            m.linPosPrescribed |= pr.linPosPrescribed
            m.rotPosPrescribed |= pr.rotPosPrescribed
        self.merged_prescriptions = merged
        self.motion_expressions = []
        for fam, m in merged.items():
            strings = [x for x in m.linVel + m.rotVel + m.linPos if x != "none"]
            if any(_const(x) is None for x in strings):
                # the whole family goes to the compiled kernel; its table entry stays unused
                self.motion_expressions.append(dict(
                    family=fam, lin_vel=list(m.linVel), ang_vel=list(m.rotVel), lin_pos=list(m.linPos),
                    lin_vel_prescribed=m.linVelPrescribed, rot_vel_prescribed=m.rotVelPrescribed,
                    lin_pos_prescribed=m.linPosPrescribed, rot_pos_prescribed=m.rotPosPrescribed))
                continue
            e = arr[fam]
            e.used = 1
            e.lin_vel_prescribed = int(m.linVelPrescribed)
            e.rot_vel_prescribed = int(m.rotVelPrescribed)
            e.lin_pos_prescribed = int(m.linPosPrescribed)
            e.rot_pos_prescribed = int(m.rotPosPrescribed)
            for k in range(3):
                if m.linVel[k] != "none":
                    e.has_vel[k] = 1
                    e.vel[k] = float(f32(_const(m.linVel[k])))
                if m.rotVel[k] != "none":
                    e.has_omg[k] = 1
                    e.omg[k] = float(f32(_const(m.rotVel[k])))
                if m.linPos[k] != "none":
                    e.has_pos[k] = 1
                    e.pos[k] = _const(m.linPos[k])
        return arr
