"""Shared test helpers: library loading, canonical contact order and comparisons.

The oracle (oracle/) is only ever used here as the checker.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dem-engine-sbel_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

from deme_b200 import capi, HandleSolver, Solver, workloads  # noqa: E402

ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "libdeme_oracle.so")


def oracle_lib():
    if not os.path.exists(ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    try:
        return capi.load_library(ORACLE_LIB)
    except OSError:
        # prebuilt with an OpenMP runtime this machine lacks: rebuild without it
        subprocess.check_call(["make", "-s", "-B", "-C", os.path.join(ROOT, "oracle")])
        return capi.load_library(ORACLE_LIB)


def oracle(built, threads=4):
    return HandleSolver(oracle_lib(), "orc_", built, threads=threads)


def reference_available() -> bool:
    from oracle import ref_build
    return ref_build.available()


def reference(built, threads=4):
    from oracle import ref_build
    lib = ref_build.build(built)
    return HandleSolver(capi.load_library(lib), "ref_", built, threads=threads)


def canonical_order(c: dict) -> np.ndarray:
    """Permutation putting a contact list in (idA, group, idB) order, groups sphere--analytical, sphere--mesh,
    sphere--sphere."""
    t = c["type"].astype(np.int64)
    grp = np.where(t == capi.SPHERE_SPHERE_CONTACT, 2, np.where(t == capi.SPHERE_MESH_CONTACT, 1, 0))
    return np.lexsort((c["idB"].astype(np.int64), grp, c["idA"].astype(np.int64)))


def canonical(c: dict) -> dict:
    p = canonical_order(c)
    out = {k: (v[..., p] if k == "wildcards" else v[p]) for k, v in c.items() if k != "mapping"}
    out["perm"] = p
    return out


def partner_keys(c: dict, prev: dict) -> np.ndarray:
    """For each contact, the (idA, idB, type) key of its history partner in ``prev`` (-1 when new)."""
    keys = np.full((len(c["idA"]), 3), -1, np.int64)
    m = c["mapping"]
    ok = m != capi.NULL_MAPPING_PARTNER
    mi = m[ok].astype(np.int64)
    keys[ok, 0] = prev["idA"][mi]
    keys[ok, 1] = prev["idB"][mi]
    keys[ok, 2] = prev["type"][mi]
    return keys


def contact_key(c: dict) -> np.ndarray:
    return np.stack([c["idA"].astype(np.int64), c["idB"].astype(np.int64), c["type"].astype(np.int64)], 1)


def rel_err(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b) / (np.abs(b) + floor)) if a.size else 0.0


def positions(built, st):
    return built.decode_positions(st)


GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
GOLDEN = ["clumps_planes", "spheres_families", "settle_small"]


class _Built:
    """A BuiltScene rebuilt from a golden fixture."""

    def __init__(self, rec):
        from deme_b200.scene import BuiltScene
        p = capi.SimParams()
        for name, _ in capi.SimParams._fields_:
            v = rec["param_" + name]
            if v.ndim:
                getattr(p, name)[:] = list(v)
            else:
                setattr(p, name, v.item())
        presc = (capi.FamilyPrescription * capi.NUM_FAMILIES).from_buffer_copy(rec["presc"].tobytes())
        arrays = {k[len("scene_"):]: rec[k] for k in rec.files if k.startswith("scene_")}
        o, s, a, m = (int(x) for x in rec["counts"])
        self.inner = BuiltScene(p, arrays, dict(o=o, s=s, a=a, m=m), presc, {})

    def __getattr__(self, k):
        return getattr(self.inner, k)


def load_golden(name):
    rec = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    return _Built(rec).inner, rec


def shaker_motion(t32) -> dict:
    """The shaker box's prescribed motions (workloads.shaker_box) evaluated at the float time ``t32`` the way the
    compiled expressions evaluate them (t promoted to double, the result stored in the component's type), as
    constant prescriptions per family, for the oracle, which integrates from a constant table."""
    import math
    t = float(np.float32(t32))
    out = {}
    p = capi.FamilyPrescription()
    p.used, p.lin_vel_prescribed, p.rot_vel_prescribed = 1, 1, 1
    p.has_vel[:] = [1, 1, 1]
    vz = 0.5 * math.sin(2000.0 * math.pi * (t - 1e-4)) if t > 1e-4 else 0.0
    p.vel[:] = [0.0, 0.0, float(np.float32(vz))]
    out[1] = p
    p = capi.FamilyPrescription()
    p.used, p.lin_pos_prescribed, p.rot_pos_prescribed = 1, 1, 1
    p.has_pos[:] = [1, 0, 0]
    p.pos[:] = [0.03 + 2.0 * t, 0.0, 0.0]
    out[2] = p
    p = capi.FamilyPrescription()
    p.used = 1
    p.has_omg[:] = [1, 1, 1]
    wz = 4000.0 * t if t < 2e-4 else 0.8 - 1000.0 * (t - 2e-4)
    p.omg[:] = [0.0, 0.0, float(np.float32(wz))]
    out[3] = p
    return out


def set_oracle_motion(orc, table: dict):
    """Loads constant prescriptions into an oracle (orc_set_family_prescription)."""
    import ctypes as C
    fn = orc.lib.orc_set_family_prescription
    fn.argtypes = [C.c_void_p, C.c_int32, C.POINTER(capi.FamilyPrescription)]
    for fam, p in table.items():
        assert fn(orc.h, int(fam), C.byref(p)) == capi.DEME_OK
