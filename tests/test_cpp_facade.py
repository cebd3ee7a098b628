"""The C++ DEMSolver facade (include/deme_solver.hpp) flattens a scene exactly as the Python SceneBuilder does.

tests/cpp/facade_dump.cpp builds a scene with every kind of input (sphere and clump templates with mixed
materials, two clump batches with orientations, velocities and families, bounding planes, an extra plane, a
cylinder and a cone on one family-10 object, fixed and prescribed families, a family mask, contact margin and CD
frequency, a Wavefront mesh body with per-facet materials) through the C++ API, and writes the flat arrays Initialize
would upload.  The same scene is built here
with SceneBuilder; every array and the parameter and prescription structs must agree bit for bit.  Compiling and
running the C++ side needs no GPU.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from _util import ROOT, capi
from deme_b200 import solver
from deme_b200.scene import SceneBuilder

f32 = np.float32
CUDA_INC = "/usr/local/cuda/include"


def scene_inputs(seed=5):
    rng = np.random.default_rng(seed)
    n1, n2 = 57, 23
    types = rng.integers(0, 3, n1).astype(np.int32)
    xyz1 = rng.uniform(-0.1, 0.1, (n1, 3)).astype(f32)
    q = rng.normal(size=(n1, 4))
    q1 = (q / np.linalg.norm(q, axis=1)[:, None]).astype(f32)
    v1 = rng.normal(0, 0.3, (n1, 3)).astype(f32)
    w1 = rng.normal(0, 3.0, (n1, 3)).astype(f32)
    fam1 = rng.integers(0, 6, n1).astype(np.int32)
    xyz2 = rng.uniform(-0.1, 0.1, (n2, 3)).astype(f32)
    return types, xyz1, q1, v1, w1, fam1, xyz2


# the mesh body of the scene (tests/cpp/facade_dump.cpp writes the same text)
MESH_OBJ = ("v 0 0 0\nv 0.02 0 0\nv 0.02 0.02 0\nv 0 0.02 0\nv 0.01 0.01 0.015\n"
            "f 1 2 3 4\nf 1/1 2/1 5/1\nf -4 -3 -1\nf 3 4 5\nf 4 1 5\n")


# the third clump template's components (tests/cpp/facade_dump.cpp writes the same text)
CLUMP_CSV = "r,note,x,y,z\n0.004,top,0,0,0.0025\n0.004,bottom,0,0,-0.0025\n"


def _clump_from_file(s, mat):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "clump.csv")
        with open(path, "w") as fh:
            fh.write(CLUMP_CSV)
        return s.LoadClumpType(1.8e-3, (8e-8, 9e-8, 9e-8), path, mat)


def python_scene(types, xyz1, q1, v1, w1, fam1, xyz2, extra=None, numvoxel=False):
    """The scene of tests/cpp/facade_dump.cpp; `extra` = (positions, velocity) of sphere clumps of a third batch;
    `numvoxel`: the voxel split given by InstructBoxDomainNumVoxel instead of the domain's dimensions."""
    s = SceneBuilder()
    if numvoxel:
        s.InstructBoxDomainNumVoxel(21, 21, 22, 4e-12)
    else:
        s.InstructBoxDomainDimension(0.3, 0.3, 0.45)
    s.SetCoordSysOrigin("center")
    m0 = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.0})
    m1 = s.LoadMaterial({"E": 5e7, "nu": 0.25, "CoR": 0.3, "mu": 0.4, "Crr": 0.02})
    s.InstructBoxDomainBoundingBC("top_open", m0)
    mass_s, r_s = float(f32(1.361e-3)), float(f32(5e-3))
    T = [s.LoadSphereType(mass_s, r_s, m0),
         s.LoadClumpType(2.5e-3, (1e-7, 1.2e-7, 1.5e-7), [4e-3, 5e-3, 4.5e-3],
                         [[3e-3, 0, 0], [-1.5e-3, 2.6e-3, 0], [-1.5e-3, -2.6e-3, 0]], [m0, m1, m0]),
         _clump_from_file(s, m1)]
    b1 = s.AddClumps([T[t] for t in types], xyz1)
    b1.SetOriQ(q1)
    b1.SetVel(v1)
    b1.SetAngVel(w1)
    b1.SetFamilies(fam1)
    b2 = s.AddClumps(T[2], xyz2)
    b2.SetFamily(3)
    if extra is not None:
        b3 = s.AddClumps(T[0], np.asarray(extra[0], f32))
        b3.SetVel(np.tile(np.asarray(extra[1], f32), (len(extra[0]), 1)))
    s.AddBCPlane((0, 0, -0.1), (0.1, 0, 1), m1)
    wall = s.AddExternalObject()
    wall.AddCylinder((0, 0, 0), (0, 0, 1), 0.12, m0)
    wall.AddPlate((0, 0.05, -0.15), (0, 0, 1), 0.04, 0.03, m0)
    wall.AddCone((0, 0, -0.2), (0, 0, 1), float(f32(0.5235988)), 0.03, 0.15, m1)
    wall.SetFamily(10)
    with tempfile.TemporaryDirectory() as d:
        obj = os.path.join(d, "mesh.obj")
        with open(obj, "w") as fh:
            fh.write(MESH_OBJ)
        mesh = s.AddWavefrontMeshObject(obj, m0)
    mesh.SetMaterial([m0, m1, m0, m1, m0, m1])
    mesh.SetInitPos((0.02, 0.08, -0.06))
    mesh.SetInitQuat((0.8, 0.0, 0.6, 0.0))
    mesh.SetMass(2.5)
    mesh.SetMOI((1e-3, 2e-3, 3e-3))
    mesh.SetFamily(3)
    s.SetFamilyFixed(3)
    s.SetFamilyPrescribedAngVel(10, "0", "2.0943951", "0")
    s.SetFamilyPrescribedLinVel(4, "0.1", "none", "0")
    s.SetFamilyPrescribedLinVel(5, "0", "0", "0.2 * sin(3000.0 * t)")
    s.DisableContactBetweenFamilies(3, 10)
    s.SetInitTimeStep(1e-5)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(5)
    s.SetExpandFactor(1e-4)
    return s.Initialize()


def read_dump(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        n = int(np.frombuffer(data, np.uint32, 1, i)[0])
        i += 4
        name = data[i:i + n].decode()
        i += n
        nb = int(np.frombuffer(data, np.uint64, 1, i)[0])
        i += 8
        out[name] = data[i:i + nb]
        i += nb
    return out


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INC, "vector_types.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    solver.load_product_library()  # the facade links the product library
    d = tmp_path_factory.mktemp("facade")
    exe = build_exe(d)
    inputs = scene_inputs()
    inp = write_inputs(d, inputs)
    subprocess.check_call([exe, str(inp), str(d / "out.bin")])
    cpp = read_dump(d / "out.bin")
    cpp["_dir"] = str(d)
    return cpp, python_scene(*inputs)


def write_inputs(d, inputs):
    inp = d / "inputs.bin"
    with open(inp, "wb") as f:
        for a in inputs:
            a = np.ascontiguousarray(a)
            f.write(np.uint64(a.size).tobytes())
            f.write(a.tobytes())
    return inp


def test_csv_output_agrees_byte_for_byte(dump, tmp_path):
    from deme_b200 import io
    cpp, built = dump
    st = built.initial_state()
    every = io.ABSV | io.VEL | io.FAMILY
    io.write_sphere_file(str(tmp_path / "s.csv"), built, st, every, families_no_output=(3,))
    io.write_clump_file(str(tmp_path / "c.csv"), built, st, every)
    assert (tmp_path / "s.csv").read_bytes() == cpp["csv_spheres"]
    assert (tmp_path / "c.csv").read_bytes() == cpp["csv_clumps"]
    i = np.arange(9, dtype=np.float32)
    forces = {"force": (np.float32(0.5) * (i + 1) - np.float32(1.25)).reshape(3, 3),
              "torque_only_force": (np.float32(0.01) * (i * i)).reshape(3, 3),
              "cpA": (np.float32(1e-3) * (i % 3 + 1) * np.where(i % 2 == 1, -1, 1).astype(np.float32)).reshape(3, 3)}
    contacts = {"idA": np.array([0, 1, 2], np.uint32), "idB": np.array([1, 3, 0], np.uint32),
                "type": np.array([1, 1, 3], np.uint8)}
    io.write_contact_file(str(tmp_path / "k.csv"), built, st, contacts, forces,
                          io.FORCE | io.POINT | io.NORMAL | io.TORQUE_ONLY_FORCE)
    assert (tmp_path / "k.csv").read_bytes() == cpp["csv_contacts"]
    # the clump file reads back as template name -> positions (ReadClumpXyzFromCsv)
    xyz = io.read_clump_xyz_from_csv(str(tmp_path / "c.csv"))
    assert sum(len(v) for v in xyz.values()) == built.info["n_clumps"]
    assert set(xyz) <= set(built.info["template_names"])


def test_flat_arrays_agree_bit_for_bit(dump):
    cpp, built = dump
    names = [k for k in cpp if k not in ("params", "prescriptions", "motion", "mesh_props", "inspect")
             and not k.startswith("csv_") and not k.startswith("_")]
    assert len(names) == 50
    for k in names:
        py = np.ascontiguousarray(built.arrays[k])
        assert cpp[k] == py.tobytes(), f"array {k} differs"


def build_exe(d):
    exe = str(d / "facade_dump")
    libdir = os.path.dirname(solver.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
                           CUDA_INC, os.path.join(ROOT, "tests", "cpp", "facade_dump.cpp"), "-o", exe, "-L", libdir,
                           "-ldeme_b200", f"-Wl,-rpath,{libdir}"])
    return exe


def test_explicit_voxel_split_agrees(tmp_path):
    """InstructBoxDomainNumVoxel: the same parameters and owner encoding from both front ends."""
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INC, "vector_types.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    solver.load_product_library()
    exe = build_exe(tmp_path)
    inputs = scene_inputs()
    inp = write_inputs(tmp_path, inputs)
    subprocess.check_call([exe, str(inp), str(tmp_path / "out.bin"), "nv"])
    cpp = read_dump(tmp_path / "out.bin")
    built = python_scene(*inputs, numvoxel=True)
    assert cpp["params"] == bytes(built.params)
    p = capi.SimParams.from_buffer_copy(cpp["params"])
    assert (p.nvXp2, p.nvYp2, p.nvZp2) == (21, 21, 22)
    for k in ("voxel", "locX", "locY", "locZ", "anal_relX", "anal_relZ"):
        assert cpp[k] == np.ascontiguousarray(built.arrays[k]).tobytes(), k
    with pytest.raises(ValueError, match="add up to 64"):
        SceneBuilder().InstructBoxDomainNumVoxel(20, 21, 22)


def test_mesh_utilities_agree(dump, tmp_path):
    """DEMMeshConnected's Rotate, ComputeMassProperties and WriteWavefront from both front ends: the rotated copy's
    mass properties within 1e-6, the written file's numbers within 1e-6 and its faces equal."""
    from deme_b200.scene import MeshObj, load_wavefront, write_wavefront
    cpp, _ = dump
    obj = tmp_path / "mesh.obj"
    obj.write_text(MESH_OBJ)
    m = MeshObj(*load_wavefront(str(obj)), 0)
    copy = MeshObj(m.vertices, m.faces, 1)
    copy.Rotate((0.8, 0.0, 0.6, 0.0))
    mass, c, inertia = copy.ComputeMassProperties()
    props = np.frombuffer(cpp["mesh_props"], f32).astype(np.float64)
    want = np.concatenate([[mass], c, inertia])
    assert np.abs(props - want).max() <= 1e-6 * np.abs(want).max(), (props, want)
    write_wavefront(str(tmp_path / "py.obj"), [m, copy])
    v_py, f_py = load_wavefront(str(tmp_path / "py.obj"))
    v_cpp, f_cpp = load_wavefront(cpp["_dir"] + "/out.bin.out.obj")
    np.testing.assert_array_equal(f_py, f_cpp)
    assert np.abs(v_py - v_cpp).max() <= 1e-6


def test_inspectors_agree(dump):
    """The inspectors' reductions (CreateInspector: clump_max_z, clump_min_z, clump_max_absv, clump_volume) on the
    initial state, from the façade's inspect_quantity and statistics.inspect, bit for bit."""
    from deme_b200 import statistics
    cpp, built = dump
    st = built.initial_state()
    got = np.frombuffer(cpp["inspect"], f32)
    want = [statistics.inspect(built, st, q, template_volume=[1.0, 2.0, 3.0])
            for q in ("clump_max_z", "clump_min_z", "clump_max_absv", "clump_volume")]
    np.testing.assert_array_equal(got, np.asarray(want, f32))
    assert got[0] > got[1] and got[2] > 0 and got[3] > 0


def test_params_and_prescriptions_agree(dump):
    cpp, built = dump
    assert cpp["params"] == bytes(built.params)
    assert cpp["prescriptions"] == bytes(built.prescriptions)
    p = capi.SimParams.from_buffer_copy(cpp["params"])
    assert p.cd_update_freq == 5 and abs(p.beta - 1e-4) < 1e-9 and (p.nvXp2, p.nvYp2, p.nvZp2) == (21, 21, 22)


def test_expression_families_agree(dump):
    """A family whose prescription is an expression goes to deme_set_prescribed_motion from both front ends."""
    cpp, built = dump
    lines = [ln.split("|") for ln in cpp["motion"].decode().splitlines()]
    py = []
    for m in built.info["motion_expressions"]:
        py.append([str(m["family"])] + [str(int(bool(m[k]))) for k in ("lin_vel_prescribed", "rot_vel_prescribed",
                                                                        "lin_pos_prescribed", "rot_pos_prescribed")]
                  + list(m["lin_vel"]) + list(m["ang_vel"]) + list(m["lin_pos"]))
    assert lines == py
    assert lines and lines[0][0] == "5" and lines[0][7] == "0.2 * sin(3000.0 * t)"
    assert built.prescriptions[5].used == 0


@pytest.mark.gpu
def test_cpp_facade_steps_like_the_python_solver(tmp_path):
    """Initialize + DoStepDynamics through the C++ facade and through the Python Solver on the same scene: the same
    contact count, kinetic energy within 1e-5, owner positions within 1e-7 m after 3 steps (owner accumulators sum
    with float atomics, so the last bits may differ between runs)."""
    solver.load_product_library()
    exe = build_exe(tmp_path)
    inputs = scene_inputs()
    inp = write_inputs(tmp_path, inputs)
    subprocess.check_call([exe, str(inp), str(tmp_path / "out.bin"), "3"])
    cpp = read_dump(tmp_path / "out.bin")
    built = python_scene(*inputs)
    g = solver.Solver(built)
    g.step(3)
    st = g.state()
    pos = built.decode_positions(st, kernel_literals=False) + np.asarray(built.params.lbf, np.float64)
    cpos = np.frombuffer(cpp["run_pos"], f32).reshape(-1, 3).astype(np.float64)
    assert np.abs(cpos - pos).max() <= 1e-7, np.abs(cpos - pos).max()
    assert int(np.frombuffer(cpp["run_ncontacts"], np.uint32)[0]) == g.num_contacts()
    ke = float(np.frombuffer(cpp["run_ke"], np.float64)[0])
    assert abs(ke - g.kinetic_energy()) <= 1e-5 * abs(g.kinetic_energy())


@pytest.mark.gpu
def test_cpp_facade_owner_setters_getters_and_update_clumps(tmp_path):
    """SetOwnerPosition / SetOwnerVelocity / SetOwnerAngVel / SetOwnerOriQ, GetOwnerAcc / GetOwnerAngAcc and
    UpdateClumps through the C++ facade (src/DEM/API.h:194-214, 392), against the Python Solver doing the same
    through deme_upload_state / deme_download_state:
    * the accelerations read owner by owner equal the whole-state download (float-sum-order bound);
    * each setter reads back what was set (the position to within the sub-voxel step) and the next step moves the
      owners as the Python run with the same state edits does;
    * UpdateClumps keeps every owner's state, the contact count and the time, puts the external objects after the
      old clumps in the reference's owner numbering and the new clumps after them, and the run continues as a fresh
      handle with the carried-over state, contacts and time does."""
    solver.load_product_library()
    exe = build_exe(tmp_path)
    inputs = scene_inputs()
    inp = write_inputs(tmp_path, inputs)
    subprocess.check_call([exe, str(inp), str(tmp_path / "out.bin"), "3", "ops"])
    cpp = read_dump(tmp_path / "out.bin")
    built = python_scene(*inputs)
    lbf = np.asarray(built.params.lbf, np.float64)
    nO = built.counts["o"]
    g = solver.Solver(built)
    g.step(3)
    st = g.state()
    # accelerations of the last step
    acc = np.stack([st["aX"], st["aY"], st["aZ"]], 1).astype(np.float64)
    aacc = np.stack([st["alphaX"], st["alphaY"], st["alphaZ"]], 1).astype(np.float64)
    cacc = np.frombuffer(cpp["ops_acc"], f32).reshape(-1, 3).astype(np.float64)
    caacc = np.frombuffer(cpp["ops_angacc"], f32).reshape(-1, 3).astype(np.float64)
    assert cacc.shape == (nO, 3)
    assert np.abs(cacc - acc).max() <= 1e-4 * max(np.abs(acc).max(), 1e-6)
    assert np.abs(caacc - aacc).max() <= 1e-4 * max(np.abs(aacc).max(), 1e-6)
    # setters read back
    p0, v1, w2 = np.array([0.01, -0.02, 0.05], f32), np.array([0.3, -0.1, 0.2], f32), np.array([5, -3, 1], f32)
    q3 = np.array([0.8, 0.0, 0.6, 0.0], f32)  # (w, x, y, z)
    rb = np.frombuffer(cpp["ops_readback"], f32).reshape(3, 3)
    rq = np.frombuffer(cpp["ops_readback_q"], f32)
    assert np.abs(rb[0].astype(np.float64) - p0).max() <= 2 * built.params.l + 1e-7
    np.testing.assert_array_equal(rb[1], v1)
    np.testing.assert_array_equal(rb[2], w2)
    np.testing.assert_array_equal(rq, [q3[1], q3[2], q3[3], q3[0]])  # float4 (x, y, z, w)
    # the same edits through the whole-state upload, then one step
    p = built.params
    rel = (p0 - np.asarray(p.lbf, f32)).astype(np.float64)[None, :]
    vox, sx, sy, sz = SceneBuilder.host_position_to_voxel(rel, (p.nvXp2, p.nvYp2, p.nvZp2), p.voxel_size, p.l)
    st["voxel"][0], st["locX"][0], st["locY"][0], st["locZ"][0] = vox[0], sx[0], sy[0], sz[0]
    st["vX"][1], st["vY"][1], st["vZ"][1] = v1
    st["omgX"][2], st["omgY"][2], st["omgZ"][2] = w2
    st["oriQw"][3], st["oriQx"][3], st["oriQy"][3], st["oriQz"][3] = q3
    g.set_state(st)
    g.step(1)
    st = g.state()
    pos = built.decode_positions(st, kernel_literals=False) + lbf
    cpos = np.frombuffer(cpp["ops_pos"], f32).reshape(-1, 3).astype(np.float64)
    assert np.abs(cpos - pos).max() <= 1e-7, np.abs(cpos - pos).max()
    # trackers (DEMTracker): the second batch starts at owner len(types), the cylinder-and-cone object is the second
    # external object
    tid = np.frombuffer(cpp["trk_id"], np.uint32)
    assert list(tid) == [len(inputs[0]), built.info["n_clumps"] + 1]
    trk = np.frombuffer(cpp["trk"], f32).reshape(3, 3)
    cvel = np.frombuffer(cpp["ops_vel"], f32).reshape(-1, 3)
    np.testing.assert_array_equal(trk[0], np.frombuffer(cpp["ops_pos"], f32).reshape(-1, 3)[tid[0]])
    np.testing.assert_array_equal(trk[1], cvel[tid[0] + 1])
    np.testing.assert_array_equal(trk[2], np.frombuffer(cpp["ops_pos"], f32).reshape(-1, 3)[tid[1]])
    # UpdateClumps: nothing moves, the counts and the time carry over, owners are numbered as the reference does
    nC = built.info["n_clumps"]
    nExt = nO - nC
    upos = np.frombuffer(cpp["upd_pos"], f32).reshape(-1, 3).astype(np.float64)
    assert upos.shape == (nO + 3, 3)
    np.testing.assert_array_equal(upos[:nO], cpos)
    p3 = np.array([[-0.05, 0.05, 0.15], [0.05, 0.05, 0.15], [0.0, -0.05, 0.15]], f32)
    assert np.abs(upos[nO:] - p3).max() <= 2 * built.params.l + 1e-7
    uvel = np.frombuffer(cpp["upd_vel"], f32).reshape(-1, 3)
    np.testing.assert_array_equal(uvel[nO:], np.tile(np.array([0, 0, -0.5], f32), (3, 1)))
    ncs = np.frombuffer(cpp["upd_ncontacts"], np.uint32)
    ts = np.frombuffer(cpp["upd_time"], np.float64)
    assert ncs[0] == ncs[1] == g.num_contacts() and ts[0] == ts[1]
    # the carried-over run: the same scene with the third batch, the old owners' state (external objects behind the
    # new clumps in the handle), the old contacts and the time
    built3 = python_scene(*inputs, extra=(p3, (0.0, 0.0, -0.5)))
    assert built3.counts["o"] == nO + 3 and built3.info["n_clumps"] == nC + 3
    g3 = solver.Solver(built3)
    s3 = g3.state()
    for k in s3:
        if k.startswith("a"):
            continue
        s3[k][:nC] = st[k][:nC]
        s3[k][nC + 3:] = st[k][nC:]
    g3.set_state(s3)
    c = g.contacts()
    g3.set_contacts({k: c[k] for k in ("idA", "idB", "type", "wildcards")})
    g3.set_time(*g.time())
    g3.step(3)
    pos3 = built3.decode_positions(g3.state(), kernel_literals=False) + lbf
    ref_order = np.concatenate([pos3[:nC], pos3[nC + 3:], pos3[nC:nC + 3]])  # the reference's owner numbering
    after = np.frombuffer(cpp["upd_pos_after"], f32).reshape(-1, 3).astype(np.float64)
    assert np.abs(after - ref_order).max() <= 1e-7, np.abs(after - ref_order).max()
    assert (after[nO:, 2] < upos[nO:, 2]).all()  # the new spheres fall
    assert nExt > 0
