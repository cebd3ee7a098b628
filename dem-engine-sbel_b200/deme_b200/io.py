"""CSV output and input in DEM-Engine's formats.

* write_sphere_file: every sphere component (DEMDynamicThread::writeSpheresAsCsv, src/DEM/dT.cpp:896-969);
* write_clump_file: every clump owner with its quaternion and template name (writeClumpsAsCsv, dT.cpp:973-1051);
* write_contact_file: every contact with owner ids, type name and the chosen quantities (writeContactsAsCsv,
  dT.cpp:1053-1180);
* read_clump_xyz_from_csv / read_clump_quat_from_csv: template name -> positions / quaternions from a clump file
  (DEMSolver::ReadClumpXyzFromCsv / ReadClumpQuatFromCsv, src/DEM/API.h:326-371).

Values are formed in float as the reference's host code forms them (hostVoxelIDToPosition<float> plus the domain's
lower corner, hostApplyOriQToVector3<float>; src/DEM/HostSideHelpers.hpp:308-324, 384-394) and printed the way a
default std::ostream prints a float (6 significant digits, shortest of fixed and scientific).

One deliberate difference: the reference rotates a contact's local point with the quaternion of the owner whose
index equals the contact's index (``oriQw.at(i)`` in writeContactsAsCsv), which is not the contact's owner; here
the point is rotated with owner A's quaternion.
"""
from __future__ import annotations

import csv

import numpy as np

f32 = np.float32

# OUTPUT_CONTENT and CNT_OUTPUT_CONTENT bits (src/DEM/Defines.h:118-143)
XYZ, QUAT, ABSV, VEL, ANG_VEL, ACC, ANG_ACC, FAMILY, MAT = 0, 1, 2, 4, 8, 16, 32, 64, 128
OWNERS, FORCE, POINT, COMPONENT, NORMAL, TORQUE_ONLY_FORCE = 0, 1, 2, 4, 8, 16
DEFAULT_CONTENT = QUAT | ABSV
DEFAULT_CONTACT_CONTENT = FORCE | POINT
CONTACT_TYPE_NAME = {0: "fake", 1: "SS", 2: "SM", 3: "SA", 4: "SA", 5: "SA", 6: "SA"}


def fmt(v) -> str:
    """A float as a default std::ostream prints it."""
    return format(float(v), ".6g")


def _owner_com(built, state) -> np.ndarray:
    """Owner centres in float: voxel index times voxel size plus sub-voxel position times l, plus the lower corner."""
    p = built.params
    v = state["voxel"].astype(np.uint64)
    mx = np.uint64((1 << p.nvXp2) - 1)
    my = np.uint64((1 << p.nvYp2) - 1)
    ids = (v & mx, (v >> np.uint64(p.nvXp2)) & my, v >> np.uint64(p.nvXp2 + p.nvYp2))
    vs, l = f32(p.voxel_size), f32(p.l)
    out = []
    for a, (vid, sub) in enumerate(zip(ids, (state["locX"], state["locY"], state["locZ"]))):
        x = vid.astype(f32) * vs + sub.astype(f32) * l
        out.append(x + f32(p.lbf[a]))
    return np.stack(out, 1).astype(f32)


def _rotate(x, y, z, qw, qx, qy, qz):
    """hostApplyOriQToVector3<float, float>, evaluated in float32 in the reference's order."""
    two, one = f32(2.0), f32(1.0)
    X = (two * (qw * qw + qx * qx) - one) * x + (two * (qx * qy - qw * qz)) * y + (two * (qx * qz + qw * qy)) * z
    Y = (two * (qx * qy + qw * qz)) * x + (two * (qw * qw + qy * qy) - one) * y + (two * (qy * qz - qw * qx)) * z
    Z = (two * (qx * qz - qw * qy)) * x + (two * (qy * qz + qw * qx)) * y + (two * (qw * qw + qz * qz) - one) * z
    return X.astype(f32), Y.astype(f32), Z.astype(f32)


def _quat(state, idx):
    return tuple(np.asarray(state[k], f32)[idx] for k in ("oriQw", "oriQx", "oriQy", "oriQz"))


def _speed(vx, vy, vz):
    return np.sqrt((vx * vx + vy * vy + vz * vz).astype(f32)).astype(f32)


def write_sphere_file(path: str, built, state, content: int = DEFAULT_CONTENT, families_no_output=()) -> None:
    a = built.arrays
    owner = np.asarray(a["sphere_owner"], np.int64)
    com = _owner_com(built, state)[owner]
    rx, ry, rz = (np.asarray(a[k], f32) for k in ("relX", "relY", "relZ"))
    rx, ry, rz = _rotate(rx, ry, rz, *_quat(state, owner))
    pos = np.stack([com[:, 0] + rx, com[:, 1] + ry, com[:, 2] + rz], 1).astype(f32)
    r = np.asarray(a["radius"], f32)
    fam = np.asarray(state["family"])[owner]
    v = [np.asarray(state[k], f32)[owner] for k in ("vX", "vY", "vZ")]
    head = "X,Y,Z,r" + (",absv" if content & ABSV else "") + (",v_x,v_y,v_z" if content & VEL else "") + \
        (",family" if content & FAMILY else "")
    skip = set(int(f) for f in families_no_output)
    speed = _speed(*v)
    lines = [head]
    for i in range(len(r)):
        if int(fam[i]) in skip:
            continue
        row = [fmt(pos[i, 0]), fmt(pos[i, 1]), fmt(pos[i, 2]), fmt(r[i])]
        if content & ABSV:
            row.append(fmt(speed[i]))
        if content & VEL:
            row += [fmt(v[0][i]), fmt(v[1][i]), fmt(v[2][i])]
        if content & FAMILY:
            row.append(str(int(fam[i])))
        lines.append(",".join(row))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_clump_file(path: str, built, state, content: int = DEFAULT_CONTENT, families_no_output=()) -> None:
    n = int(built.info["n_clumps"])
    com = _owner_com(built, state)[:n]
    q = [np.asarray(state[k], f32)[:n] for k in ("oriQw", "oriQx", "oriQy", "oriQz")]
    names = built.info.get("template_names", [])
    tmpl = np.asarray(built.info.get("owner_template", np.zeros(n, np.int64)))
    fam = np.asarray(state["family"])[:n]
    v = [np.asarray(state[k], f32)[:n] for k in ("vX", "vY", "vZ")]
    speed = _speed(*v)
    head = "X,Y,Z,Qw,Qx,Qy,Qz,clump_type" + (",absv" if content & ABSV else "") + \
        (",v_x,v_y,v_z" if content & VEL else "") + (",family" if content & FAMILY else "")
    skip = set(int(f) for f in families_no_output)
    lines = [head]
    for i in range(n):
        if int(fam[i]) in skip:
            continue
        t = int(tmpl[i])
        row = [fmt(com[i, 0]), fmt(com[i, 1]), fmt(com[i, 2]), fmt(q[0][i]), fmt(q[1][i]), fmt(q[2][i]), fmt(q[3][i]),
               names[t] if t < len(names) else "%04d" % t]
        if content & ABSV:
            row.append(fmt(speed[i]))
        if content & VEL:
            row += [fmt(v[0][i]), fmt(v[1][i]), fmt(v[2][i])]
        if content & FAMILY:
            row.append(str(int(fam[i])))
        lines.append(",".join(row))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_contact_file(path: str, built, state, contacts: dict, forces: dict | None,
                       content: int = DEFAULT_CONTACT_CONTENT) -> None:
    """``contacts`` as the solvers' contacts() returns them; ``forces`` as contact_forces() returns them (needed for
    FORCE, POINT, NORMAL and TORQUE_ONLY_FORCE)."""
    a = built.arrays
    owner = np.asarray(a["sphere_owner"], np.int64)
    anal_owner = np.asarray(a["anal_owner"], np.int64) if len(a["anal_owner"]) else np.zeros(1, np.int64)
    idA = np.asarray(contacts["idA"], np.int64)
    idB = np.asarray(contacts["idB"], np.int64)
    tp = np.asarray(contacts["type"])
    oA = owner[idA]
    ss = tp == 1
    oB = np.where(ss, owner[np.where(ss, idB, 0)], anal_owner[np.where(ss, 0, idB)])
    need = content & (FORCE | POINT | NORMAL | TORQUE_ONLY_FORCE)
    if need and forces is None:
        raise ValueError("per-contact forces are needed for this content (keep_contact_forces before stepping)")
    head = "A,B,contact_type" + (",f_x,f_y,f_z" if content & FORCE else "") + (",X,Y,Z" if content & POINT else "") + \
        (",n_x,n_y,n_z" if content & NORMAL else "") + (",tof_x,tof_y,tof_z" if content & TORQUE_ONLY_FORCE else "")
    lines = [head]
    if len(idA):
        com = _owner_com(built, state)[oA]
        qA = _quat(state, oA)
        if need:
            F = np.asarray(forces["force"], f32)
            T = np.asarray(forces["torque_only_force"], f32)
            cp = np.asarray(forces["cpA"], f32)
            px, py, pz = _rotate(cp[:, 0], cp[:, 1], cp[:, 2], *qA)
            px, py, pz = (com[:, 0] + px).astype(f32), (com[:, 1] + py).astype(f32), (com[:, 2] + pz).astype(f32)
            rx, ry, rz = (np.asarray(a[k], f32)[idA] for k in ("relX", "relY", "relZ"))
            rx, ry, rz = _rotate(rx, ry, rz, *qA)
            nx = (px - (com[:, 0] + rx)).astype(f32)
            ny = (py - (com[:, 1] + ry)).astype(f32)
            nz = (pz - (com[:, 2] + rz)).astype(f32)
            inv = (f32(1.0) / np.sqrt((nx * nx + ny * ny + nz * nz).astype(f32))).astype(f32)
            nx, ny, nz = (nx * inv).astype(f32), (ny * inv).astype(f32), (nz * inv).astype(f32)
        for i in range(len(idA)):
            if int(tp[i]) == 0:
                continue
            row = [str(int(oA[i])), str(int(oB[i])), CONTACT_TYPE_NAME.get(int(tp[i]), "SA")]
            if content & FORCE:
                row += [fmt(F[i, 0]), fmt(F[i, 1]), fmt(F[i, 2])]
            if content & POINT:
                row += [fmt(px[i]), fmt(py[i]), fmt(pz[i])]
            if content & NORMAL:
                row += [fmt(nx[i]), fmt(ny[i]), fmt(nz[i])]
            if content & TORQUE_ONLY_FORCE:
                row += [fmt(T[i, 0]), fmt(T[i, 1]), fmt(T[i, 2])]
            lines.append(",".join(row))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def csv_floats(cells) -> np.ndarray:
    """float32 values of CSV cells as the reference's CSV reader forms them (io::detail::parse_float<float>,
    src/core/utils/csv.hpp:936-997, the reader behind DEMClumpTemplate::ReadComponentFromFile and
    ReadClumpXyzFromCsv / ReadClumpQuatFromCsv).  That reader is not correctly rounded: it accumulates the integer
    digits in float (x = x * 10 + d), each fraction digit as d * p with p divided by 10 per digit in float, and applies
    an exponent by repeated squaring of 10 or 0.1 in float, so its values can differ from the nearest float by a few
    units in the last place; this forms them with the same float32 operations in the same order, for a whole column
    at once.  Cells are trimmed of spaces and tabs; an empty cell is 0.  One deliberate difference: an exponent
    written with '+' is read (the reference rejects it).  Anything else that is not a number raises ValueError."""
    cells = [str(c).strip(" \t") for c in cells]
    n = len(cells)
    if n == 0:
        return np.zeros(0, f32)
    w = max(1, max(len(c) for c in cells))
    try:
        b = np.frombuffer("".join(c.ljust(w, "\0") for c in cells).encode("ascii"), np.uint8).reshape(n, w)
    except UnicodeEncodeError:
        raise ValueError("a CSV number cell holds a character that is not ASCII") from None
    x = np.zeros(n, f32)
    pos = np.ones(n, f32)
    neg = b[:, 0] == ord("-")
    phase = np.zeros(n, np.int8)  # 0 integer digits, 1 fraction digits, 2 exponent sign, 3 exponent digits, 4 done
    e = np.zeros(n, np.int64)
    e_neg = np.zeros(n, bool)
    bad = np.zeros(n, bool)
    ten = f32(10)
    for j in range(w):
        c = b[:, j]
        if j == 0:
            c = np.where((c == ord("-")) | (c == ord("+")), np.uint8(0xFF), c)  # a leading sign: nothing more here
        skip = c == 0xFF
        digit = (c >= ord("0")) & (c <= ord("9"))
        d = (c.astype(np.int64) - ord("0"))
        end = c == 0
        m = (phase == 0) & digit
        x[m] = x[m] * ten
        x[m] = x[m] + d[m].astype(f32)
        m = (phase == 1) & digit
        pos[m] = pos[m] / ten
        x[m] = x[m] + d[m].astype(f32) * pos[m]
        m = (phase >= 2) & (phase <= 3) & digit
        e[m] = np.minimum(e[m] * 10 + d[m], 1 << 20)
        dot = (phase == 0) & ((c == ord(".")) | (c == ord(",")))
        expo = (phase <= 1) & ((c == ord("e")) | (c == ord("E")))
        esign = (phase == 2) & ((c == ord("-")) | (c == ord("+")))
        e_neg |= esign & (c == ord("-"))
        bad |= ~(skip | digit | end | dot | expo | esign) & (phase < 4)
        phase = np.where(dot, 1, np.where(expo, 2, np.where(esign | ((phase == 2) & digit), 3, phase))).astype(np.int8)
        phase[end] = 4
    if bad.any():
        raise ValueError(f"not a number in a CSV cell: {cells[int(np.argmax(bad))]!r}")
    base = np.where(e_neg, f32(0.1), ten).astype(f32)
    active = e != 0
    while active.any():
        step = active & (e != 1)
        even = step & (e % 2 == 0)
        odd = step & (e % 2 == 1)
        base[even] = base[even] * base[even]
        e[even] >>= 1
        x[odd] = x[odd] * base[odd]
        e[odd] -= 1
        fin = active & (e == 1)
        x[fin] = x[fin] * base[fin]
        active &= ~fin
    x[neg] = -x[neg]
    return x


def _read_columns(path: str, headers):
    with open(path, newline="") as f:
        rows = [r for r in csv.reader(f) if r and any(c.strip() for c in r)]
    head = [h.strip() for h in rows[0]]
    idx = [head.index(h) for h in headers]
    return [[r[i].strip() for i in idx] for r in rows[1:]]


def read_clump_xyz_from_csv(path: str, clump_header="clump_type", x_header="X", y_header="Y", z_header="Z") -> dict:
    """Template name -> (n, 3) float32 positions, in file order."""
    return _by_name(_read_columns(path, (clump_header, x_header, y_header, z_header)), 3)


def read_clump_quat_from_csv(path: str, clump_header="clump_type", qw_header="Qw", qx_header="Qx", qy_header="Qy",
                             qz_header="Qz") -> dict:
    """Template name -> (n, 4) float32 quaternions (w, x, y, z), in file order."""
    return _by_name(_read_columns(path, (clump_header, qw_header, qx_header, qy_header, qz_header)), 4)


def _by_name(rows, k: int) -> dict:
    """Rows of (name, k numbers) -> name -> (n, k) float32 in file order, the numbers read by csv_floats."""
    if not rows:
        return {}
    vals = csv_floats([r[i] for r in rows for i in range(1, k + 1)]).reshape(-1, k)
    names = [r[0] for r in rows]
    out: dict = {}
    for i, name in enumerate(names):
        out.setdefault(name, []).append(i)
    return {name: vals[idx] for name, idx in out.items()}
