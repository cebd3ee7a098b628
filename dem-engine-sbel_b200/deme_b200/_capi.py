"""ctypes mirror of include/deme_b200.h.

The same struct layouts are used by three shared libraries that export the same entry points under
different prefixes: the CUDA product library (``deme_``), the C oracle (``orc_``) and the reference kernels
compiled for the CPU (``ref_``).  Only the product library is loaded by the solver classes; the other two are
loaded by tests and by bench.py's CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

DEME_OK = 0
STATUS_NAMES = {
    0: "DEME_OK",
    1: "DEME_ERR_INVALID",
    2: "DEME_ERR_CUDA",
    3: "DEME_ERR_OOM",
    4: "DEME_ERR_OVERFLOW",
    5: "DEME_ERR_NVRTC",
    6: "DEME_ERR_TIMEOUT",
    7: "DEME_ERR_STATE",
    8: "DEME_ERR_NO_DEVICE",
    9: "DEME_ERR_TOO_LARGE",
}

NOT_A_CONTACT = 0
SPHERE_SPHERE_CONTACT = 1
SPHERE_MESH_CONTACT = 2
SPHERE_PLANE_CONTACT = 3
SPHERE_CYLINDER_CONTACT = 5
SPHERE_CONE_CONTACT = 6
ANAL_PLANE, ANAL_PLATE, ANAL_CYLINDER, ANAL_CONE = 0, 1, 2, 3
FORWARD_EULER, CENTERED_DIFFERENCE, EXTENDED_TAYLOR = 0, 1, 2
NULL_MAPPING_PARTNER = 0xC0000000  # value of the reference's expression (src/DEM/Defines.h:80-81)
NUM_FAMILY_MASK = 32896
NUM_FAMILIES = 256
RESERVED_FAMILY = 255

_P = C.c_void_p


class SimParams(C.Structure):
    _fields_ = [
        ("nvXp2", C.c_uint8),
        ("nvYp2", C.c_uint8),
        ("nvZp2", C.c_uint8),
        ("pad0", C.c_uint8),
        ("nbX", C.c_uint32),
        ("nbY", C.c_uint32),
        ("nbZ", C.c_uint32),
        ("l", C.c_double),
        ("voxel_size", C.c_double),
        ("l_kernel", C.c_double),
        ("voxel_size_kernel", C.c_double),
        ("bin_size", C.c_double),
        ("lbf", C.c_float * 3),
        ("G", C.c_float * 3),
        ("h", C.c_float),
        ("beta", C.c_float),
        ("integrator", C.c_int32),
        ("cd_update_freq", C.c_int32),
        ("n_contact_wildcards", C.c_int32),
        ("pad1", C.c_int32),
        ("domain", C.c_float * 3),
        ("pad2", C.c_float),
    ]


class FamilyPrescription(C.Structure):
    _fields_ = [
        ("used", C.c_uint8),
        ("lin_vel_prescribed", C.c_uint8),
        ("rot_vel_prescribed", C.c_uint8),
        ("lin_pos_prescribed", C.c_uint8),
        ("rot_pos_prescribed", C.c_uint8),
        ("has_vel", C.c_uint8 * 3),
        ("has_omg", C.c_uint8 * 3),
        ("has_pos", C.c_uint8 * 3),
        ("pad", C.c_uint8 * 4),
        ("vel", C.c_float * 3),
        ("omg", C.c_float * 3),
        ("pos", C.c_double * 3),
    ]


class MotionExpressions(C.Structure):
    """deme_motion_expressions: one family's prescribed motion as C expression strings (NULL = free)."""
    _fields_ = [
        ("family", C.c_int32),
        ("lin_vel_prescribed", C.c_uint8),
        ("rot_vel_prescribed", C.c_uint8),
        ("lin_pos_prescribed", C.c_uint8),
        ("rot_pos_prescribed", C.c_uint8),
        ("lin_vel", C.c_char_p * 3),
        ("ang_vel", C.c_char_p * 3),
        ("lin_pos", C.c_char_p * 3),
    ]


SCENE_ARRAYS = [
    # (field, dtype, count key)
    ("voxel", np.uint64, "o"),
    ("locX", np.uint16, "o"),
    ("locY", np.uint16, "o"),
    ("locZ", np.uint16, "o"),
    ("oriQw", np.float32, "o"),
    ("oriQx", np.float32, "o"),
    ("oriQy", np.float32, "o"),
    ("oriQz", np.float32, "o"),
    ("vX", np.float32, "o"),
    ("vY", np.float32, "o"),
    ("vZ", np.float32, "o"),
    ("omgX", np.float32, "o"),
    ("omgY", np.float32, "o"),
    ("omgZ", np.float32, "o"),
    ("family", np.uint8, "o"),
    ("mass", np.float32, "o"),
    ("mmiXX", np.float32, "o"),
    ("mmiYY", np.float32, "o"),
    ("mmiZZ", np.float32, "o"),
    ("sphere_owner", np.uint32, "s"),
    ("relX", np.float32, "s"),
    ("relY", np.float32, "s"),
    ("relZ", np.float32, "s"),
    ("radius", np.float32, "s"),
    ("sphere_material", np.uint8, "s"),
    ("anal_type", np.uint8, "a"),
    ("anal_owner", np.uint32, "a"),
    ("anal_normal", np.uint8, "a"),
    ("anal_material", np.uint8, "a"),
    ("anal_relX", np.float32, "a"),
    ("anal_relY", np.float32, "a"),
    ("anal_relZ", np.float32, "a"),
    ("anal_rotX", np.float32, "a"),
    ("anal_rotY", np.float32, "a"),
    ("anal_rotZ", np.float32, "a"),
    ("anal_size1", np.float32, "a"),
    ("anal_size2", np.float32, "a"),
    ("anal_size3", np.float32, "a"),
    ("anal_mass", np.float32, "a"),
    ("mat_E", np.float32, "m"),
    ("mat_nu", np.float32, "m"),
    ("mat_CoR", np.float32, "m"),
    ("mat_mu", np.float32, "m"),
    ("mat_Crr", np.float32, "m"),
    ("family_masks", np.uint8, "mask"),
]


# optional arrays (packed multi-scene runs); absent keys leave the pointer NULL
SCENE_EXTENSIONS = [
    ("sphere_material_wide", np.uint16, "s"),
    ("anal_material_wide", np.uint16, "a"),
    ("owner_anal_first", np.uint32, "o"),
    ("owner_anal_count", np.uint32, "o"),
    ("owner_scene", np.uint32, "o"),
    ("scene_box", np.float32, None),  # 6 per scene
]


# mesh facets (n_tris of each; the nodes as n_tris x 3 floats)
SCENE_TRIS = [
    ("tri_owner", np.uint32),
    ("tri_node1", np.float32),
    ("tri_node2", np.float32),
    ("tri_node3", np.float32),
    ("tri_material", np.uint16),
]


class Scene(C.Structure):
    _fields_ = [("n_owners", C.c_uint32), ("n_spheres", C.c_uint32), ("n_anal", C.c_uint32),
                ("n_materials", C.c_uint32)] + [(name, _P) for name, _, _ in SCENE_ARRAYS] + [
                    ("prescriptions", _P)] + [(name, _P) for name, _, _ in SCENE_EXTENSIONS] + [
                    ("n_tris", C.c_uint32)] + [(name, _P) for name, _ in SCENE_TRIS]


STATE_FIELDS = [
    ("voxel", np.uint64),
    ("locX", np.uint16),
    ("locY", np.uint16),
    ("locZ", np.uint16),
    ("oriQw", np.float32),
    ("oriQx", np.float32),
    ("oriQy", np.float32),
    ("oriQz", np.float32),
    ("vX", np.float32),
    ("vY", np.float32),
    ("vZ", np.float32),
    ("omgX", np.float32),
    ("omgY", np.float32),
    ("omgZ", np.float32),
    ("aX", np.float32),
    ("aY", np.float32),
    ("aZ", np.float32),
    ("alphaX", np.float32),
    ("alphaY", np.float32),
    ("alphaZ", np.float32),
    ("family", np.uint8),
]


class State(C.Structure):
    _fields_ = [(name, _P) for name, _ in STATE_FIELDS]


class Contacts(C.Structure):
    _fields_ = [
        ("capacity", C.c_uint32),
        ("n_contacts", C.c_uint32),
        ("idA", _P),
        ("idB", _P),
        ("type", _P),
        ("mapping", _P),
        ("wildcards", _P),
    ]


class ContactForces(C.Structure):
    _fields_ = [
        ("capacity", C.c_uint32),
        ("n_contacts", C.c_uint32),
        ("force", _P),
        ("torque_only_force", _P),
        ("cpA", _P),
        ("cpB", _P),
    ]


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed through the C ABI must be contiguous"
    return a.ctypes.data


def make_scene_struct(arrays: dict, counts: dict, prescriptions) -> tuple[Scene, list]:
    """Build a Scene struct pointing into ``arrays`` (kept alive by the returned list)."""
    keep = []
    s = Scene()
    s.n_owners = counts["o"]
    s.n_spheres = counts["s"]
    s.n_anal = counts["a"]
    s.n_materials = counts["m"]
    for name, dt, key in SCENE_ARRAYS:
        a = np.ascontiguousarray(arrays[name], dtype=dt)
        n = NUM_FAMILY_MASK if key == "mask" else counts[key]
        if a.shape[0] != n:
            raise ValueError(f"scene array {name} has {a.shape[0]} entries, expected {n}")
        keep.append(a)
        setattr(s, name, ptr(a) if n > 0 else None)
    keep.append(prescriptions)
    s.prescriptions = C.addressof(prescriptions)
    for name, dt, key in SCENE_EXTENSIONS:
        if arrays.get(name) is None:
            continue
        a = np.ascontiguousarray(arrays[name], dtype=dt)
        if key is not None and a.shape[0] != counts[key]:
            raise ValueError(f"scene array {name} has {a.shape[0]} entries, expected {counts[key]}")
        keep.append(a)
        setattr(s, name, ptr(a) if a.size > 0 else None)
    s.n_tris = counts.get("t", 0)
    for name, dt in SCENE_TRIS:
        if not s.n_tris:
            break
        a = np.ascontiguousarray(arrays[name], dtype=dt)
        if a.shape[0] != s.n_tris:
            raise ValueError(f"scene array {name} has {a.shape[0]} entries, expected {s.n_tris}")
        keep.append(a)
        setattr(s, name, ptr(a))
    return s, keep


def state_struct(arrays: dict) -> tuple[State, list]:
    st = State()
    keep = []
    for name, dt in STATE_FIELDS:
        a = arrays.get(name)
        if a is not None:
            assert a.dtype == dt and a.flags["C_CONTIGUOUS"], name
            keep.append(a)
            setattr(st, name, ptr(a))
    return st, keep


class Tuning(C.Structure):
    """deme_tuning: the search shape deme_autotune chose."""
    _fields_ = [("shape", C.c_int32), ("find_warps", C.c_int32), ("find_slots", C.c_int32),
                ("cell_factor", C.c_float), ("ms_per_step", C.c_float), ("ms_per_step_default", C.c_float),
                ("trials", C.c_int32), ("find_persistent", C.c_int32), ("force_shape", C.c_int32),
                ("force_threads", C.c_int32), ("exact_threads", C.c_int32), ("integrate_threads", C.c_int32)]


def bind(lib: C.CDLL, prefix: str):
    """Declare the argument/return types of the shared entry points under ``prefix``."""
    VP = C.c_void_p
    sig = {
        "create": (VP, [C.POINTER(SimParams), C.POINTER(Scene)]),
        "destroy": (None, [VP]),
        "detect_contacts": (C.c_int32, [VP]),
        "compute_forces": (C.c_int32, [VP]),
        "integrate": (C.c_int32, [VP]),
        "step": (C.c_int32, [VP, C.c_int32]),
        "download_state": (C.c_int32, [VP, C.POINTER(State)]),
        "upload_state": (C.c_int32, [VP, C.POINTER(State)]),
        "download_contacts": (C.c_int32, [VP, C.POINTER(Contacts)]),
        "upload_contacts": (C.c_int32, [VP, C.POINTER(Contacts)]),
        "download_contact_forces": (C.c_int32, [VP, C.POINTER(ContactForces)]),
        "bin_assignment": (C.c_int32, [VP, VP, VP, C.c_uint32, VP, VP, C.POINTER(C.c_uint32)]),
        "set_threads": (C.c_int32, [C.c_int32]),
        "num_contacts": (C.c_uint32, [VP]),
        "kinetic_energy": (C.c_double, [VP]),
        "time": (C.c_double, [VP]),
        "max_spheres_in_bin": (C.c_int32, [VP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


def load_library(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path, mode=C.RTLD_LOCAL)
