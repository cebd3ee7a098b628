"""FP64 evaluation of one DEM step on a given state and contact list: the reference's contact model and
integration with every quantity in float64.

TEST INFRASTRUCTURE ONLY: the yardstick the CUDA path's per-contact forces and one-step state updates are measured
against (tests/), never part of the product.

It restates, in double precision throughout, what the reference computes in its float/double mix:

* sphere centres: owner position (voxel + sub-voxel, ``voxelIDToPosition``, src/kernel/DEMHelperKernels.cu:93-110)
  plus the owner's orientation applied to the relative position (``applyOriQToVector3``, :137-148);
* contact geometry of ``calculateContactForces`` (src/kernel/DEMCalcForceKernels.cu:14-179): sphere--sphere
  overlap with the contact point formed from B's side (``checkSpheresOverlap``, DEMHelperKernels.cu:233-264),
  sphere--plane with the halved overlap (``checkSphereEntityOverlap``, :394-445), and the cylinder and cone walls of
  this build (same conventions as the plane);
* the frictional Hertz--Mindlin model (src/kernel/DEMCustomizablePolicies/FullHertzianForceModel.cu) with
  ``matProxy2ContactParam`` (DEMHelperKernels.cu:316-339), tangential history and rolling resistance;
* force collection onto owners (src/kernel/DEMCollectForceKernels.cu:68-120);
* Extended Taylor integration with constant family prescriptions (src/kernel/DEMIntegrationKernels.cu:46-179), the
  position left unquantised (no sub-voxel rounding) and the quaternion not renormalised, as the reference leaves it.
"""
from __future__ import annotations

import numpy as np

TINY = 1e-12
HUGE = 1e15
C5 = 1.825741858350554  # 2 sqrt(5/6)
PI = 3.1415926535897932385
SPHERE_SPHERE = 1
ANAL_PLANE, ANAL_CYLINDER = 0, 2


def rot(q, v):
    """applyOriQToVector3 in float64: q = (w, x, y, z) rows, v rows."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    ox, oy, oz = v[:, 0], v[:, 1], v[:, 2]
    X = (2 * (w * w + x * x) - 1) * ox + 2 * (x * y - w * z) * oy + 2 * (x * z + w * y) * oz
    Y = 2 * (x * y + w * z) * ox + (2 * (w * w + y * y) - 1) * oy + 2 * (y * z - w * x) * oz
    Z = 2 * (x * z - w * y) * ox + 2 * (y * z + w * x) * oy + (2 * (w * w + z * z) - 1) * oz
    return np.stack([X, Y, Z], 1)


def rot_t(q, v):
    """The inverse rotation (conjugate quaternion)."""
    return rot(q * np.array([1.0, -1.0, -1.0, -1.0]), v)


def owner_state(built, st):
    """Owner positions (relative to the lower corner, kernel literals), quaternions, velocities, angular
    velocities (owner frame), masses and principal moments, all float64."""
    pos = built.decode_positions(st)
    q = np.stack([st[k] for k in ("oriQw", "oriQx", "oriQy", "oriQz")], 1).astype(np.float64)
    v = np.stack([st[k] for k in ("vX", "vY", "vZ")], 1).astype(np.float64)
    w = np.stack([st[k] for k in ("omgX", "omgY", "omgZ")], 1).astype(np.float64)
    a = built.arrays
    m = a["mass"].astype(np.float64)
    I = np.stack([a["mmiXX"], a["mmiYY"], a["mmiZZ"]], 1).astype(np.float64)
    return pos, q, v, w, m, I


def rot_f32(q, v):
    """applyOriQToVector3<float, float> as the CUDA path evaluates it: every operation rounded to float32 in the
    same order (no contraction), the result widened to float64."""
    f = np.float32
    w, x, y, z = (q[:, k].astype(f) for k in range(4))
    ox, oy, oz = (v[:, k].astype(f) for k in range(3))
    two, one = f(2.0), f(1.0)
    X = (two * (w * w + x * x) - one) * ox + (two * (x * y - w * z)) * oy + (two * (x * z + w * y)) * oz
    Y = (two * (x * y + w * z)) * ox + (two * (w * w + y * y) - one) * oy + (two * (y * z - w * x)) * oz
    Z = (two * (x * z - w * y)) * ox + (two * (y * z + w * x)) * oy + (two * (w * w + z * z) - one) * oz
    return np.stack([X, Y, Z], 1).astype(np.float64)


def _rotate(q, v, f32, q_anchor):
    if not f32:
        return rot(q, v)
    if q_anchor is None:
        return rot_f32(q, v)
    # float32 at the anchor, plus the float64 change from it: equal to the float32 rotation at the anchor, and
    # differentiable there with the exact derivative
    return rot_f32(q_anchor, v) + (rot(q, v) - rot(q_anchor, v))


def sphere_centres(built, pos, q, f32=False, q_anchor=None):
    """Sphere centres: owner position plus the rotated offset (rotated in float32 as the CUDA path rotates it when
    ``f32``; with ``q_anchor``, float32 at the anchor quaternions plus the float64 change from them)."""
    a = built.arrays
    o = a["sphere_owner"].astype(np.int64)
    rel = np.stack([a["relX"], a["relY"], a["relZ"]], 1).astype(np.float64)
    return pos[o] + _rotate(q[o], rel, f32, None if q_anchor is None else q_anchor[o])


def placed_analytical(built, pos, q, f32=False, q_anchor=None):
    """Analytical components in the world frame: reference point, direction (plane normal / axis) and the shape
    numbers (cylinder radius; cone sin, cos of the half angle and its axial range).  ``f32``: the reference point's
    offset and the direction rotated in float32 as the CUDA path places them."""
    a = built.arrays
    nA = built.counts["a"]
    if nA == 0:
        return None
    o = a["anal_owner"].astype(np.int64)
    rel = np.stack([a["anal_relX"], a["anal_relY"], a["anal_relZ"]], 1).astype(np.float64)
    d = np.stack([a["anal_rotX"], a["anal_rotY"], a["anal_rotZ"]], 1).astype(np.float64)
    half = a["anal_size1"].astype(np.float64)
    qa = None if q_anchor is None else q_anchor[o]
    return dict(p=pos[o] + _rotate(q[o], rel, f32, qa), d=_rotate(q[o], d, f32, qa), owner=o,
                type=a["anal_type"].astype(np.int64),
                normal=a["anal_normal"].astype(np.int64), size1=a["anal_size1"].astype(np.float64),
                c1=np.sin(half), c2=np.cos(half), umin=a["anal_size2"].astype(np.float64),
                umax=a["anal_size3"].astype(np.float64), mat=a["anal_material"].astype(np.int64),
                mass=a["anal_mass"].astype(np.float64))


def _analytical_geometry(an, k, X, rA):
    """Contact point, unit normal (wall -> sphere) and overlap depth of spheres X (rows) with components k."""
    typ = an["type"][k]
    P, d = an["p"][k], an["d"][k]
    gap = np.zeros(len(k))
    nrm = np.zeros((len(k), 3))
    valid = np.ones(len(k), bool)
    pl = typ == ANAL_PLANE
    if pl.any():
        gap[pl] = np.einsum("ij,ij->i", X[pl] - P[pl], d[pl])
        nrm[pl] = d[pl]
    cu = ~pl
    if cu.any():
        v = X[cu] - P[cu]
        ax = d[cu]
        t = np.einsum("ij,ij->i", v, ax)
        wv = v - t[:, None] * ax
        rho = np.linalg.norm(wv, axis=1)
        ok = rho > 0
        u = wv / np.where(ok, rho, 1.0)[:, None]
        isc = an["type"][k][cu] == ANAL_CYLINDER
        out = an["normal"][k][cu] == 1
        g = np.where(isc, np.where(out, rho - an["size1"][k][cu], an["size1"][k][cu] - rho), 0.0)
        n_ = np.where((isc & out)[:, None], u, -u)
        # cone
        c1, c2 = an["c1"][k][cu], an["c2"][k][cu]
        gc = t * c1 - rho * c2
        gv = c1[:, None] * ax - c2[:, None] * u
        g = np.where(isc, g, np.where(out, -gc, gc))
        n_ = np.where(isc[:, None], n_, np.where(out[:, None], -gv, gv))
        # the cone wall exists over its axial range only
        uc = (t * c2 + rho * c1) * c2
        ok &= isc | ((uc >= an["umin"][k][cu]) & (uc <= an["umax"][k][cu]))
        gap[cu] = g
        nrm[cu] = n_
        valid[cu] = ok
    od = (rA - gap) / 2.0
    cp = X - nrm * (gap + od)[:, None]
    return cp, nrm, np.where(valid, od, -1.0)


def step(built, st, contacts, h=None):
    """One step of the reference's dynamics in float64 on state ``st`` (a downloaded deme_state) and the contact
    list ``contacts`` (idA, idB, type and the four history wildcards at the step's start).

    Returns per-contact force, torque-only force and local contact points (zero where the contact does not touch),
    the updated history, the owners' accelerations, and the state after integration (positions relative to the
    lower corner, velocities, owner-frame angular velocities, quaternions)."""
    pos, q, v, w, _, _ = owner_state(built, st)
    S = dict(pos=pos, q=q, v=v, w=w, family=st["family"].astype(np.int64))
    return step_state(built, S, contacts, h=h)


def step_state(built, S, contacts, hist=None, h=None, mats=None, f32=False, q_anchor=None):
    """``step`` on a float64 state S (pos, q, v, w in the owner frame, family) with the incoming history ``hist``
    (rows of 4; default: the list's wildcards) and, optionally, material arrays ``mats`` (E, nu, CoR, mu, Crr)
    replacing the scene's.  ``f32``: sphere offsets and wall placements rotated in float32 as the CUDA path does
    (the rest in float64), so that the contact geometry is evaluated where the CUDA path evaluates it; with
    ``q_anchor`` (owner quaternions), float32 at the anchor plus the float64 change from it, which keeps that
    geometry differentiable in the quaternions."""
    p = built.params
    a = built.arrays
    h = float(p.h) if h is None else float(h)
    pos, q, v, w = S["pos"], S["q"], S["v"], S["w"]
    m = a["mass"].astype(np.float64)
    I = np.stack([a["mmiXX"], a["mmiYY"], a["mmiZZ"]], 1).astype(np.float64)
    Xs = sphere_centres(built, pos, q, f32, q_anchor)
    an = placed_analytical(built, pos, q, f32, q_anchor)
    o_s = a["sphere_owner"].astype(np.int64)
    rad = a["radius"].astype(np.float64)
    mat_s = (a["sphere_material_wide"] if "sphere_material_wide" in a else a["sphere_material"]).astype(np.int64)
    if mats is None:
        E, nu, CoR, mu, Crr = (a[k].astype(np.float64) for k in ("mat_E", "mat_nu", "mat_CoR", "mat_mu", "mat_Crr"))
    else:
        E, nu, CoR, mu, Crr = (np.asarray(mats[k], np.float64) for k in ("E", "nu", "CoR", "mu", "Crr"))
    A = contacts["idA"].astype(np.int64)
    Bid = contacts["idB"].astype(np.int64)
    typ = contacts["type"].astype(np.int64)
    if hist is None:
        hist = contacts["wildcards"].astype(np.float64).T.copy() if contacts["wildcards"].size else np.zeros((len(A), 4))
    nC = len(A)
    ss = typ == SPHERE_SPHERE
    oA = o_s[A]
    oB = np.where(ss, o_s[np.where(ss, Bid, 0)], an["owner"][np.where(ss, 0, Bid)] if an is not None else 0)
    XA = Xs[A]
    rA = rad[A]
    # geometry
    cp = np.zeros((nC, 3))
    nrm = np.zeros((nC, 3))
    depth = np.zeros(nC)
    rB = np.full(nC, HUGE)
    mB = np.zeros(nC)
    matB = np.zeros(nC, np.int64)
    if ss.any():
        XB = Xs[Bid[ss]]
        r_b = rad[Bid[ss]]
        dv = XA[ss] - XB
        d = np.linalg.norm(dv, axis=1)
        n_ = dv / d[:, None]
        dep = rA[ss] + r_b - d
        cp[ss] = XB + (r_b - dep / 2.0)[:, None] * n_
        nrm[ss] = n_
        depth[ss] = np.where(d <= rA[ss] + r_b, dep, -1.0)
        rB[ss] = r_b
        mB[ss] = m[oB[ss]]
        matB[ss] = mat_s[Bid[ss]]
    an_c = ~ss
    if an_c.any():
        k = Bid[an_c]
        cpa, na, od = _analytical_geometry(an, k, XA[an_c], rA[an_c])
        cp[an_c], nrm[an_c] = cpa, na
        depth[an_c] = np.where(od >= 0, od, -1.0)
        mB[an_c] = an["mass"][k]
        matB[an_c] = an["mat"][k]
    act = depth >= 0
    cpA = rot_t(q[oA], cp - pos[oA])
    cpB = rot_t(q[oB], cp - pos[oB])
    mA = m[oA]
    # material pair (matProxy2ContactParam)
    ma, mb = mat_s[A], matB
    Es = 1.0 / ((1 - nu[ma] ** 2) / E[ma] + (1 - nu[mb] ** 2) / E[mb])
    Gs = 1.0 / (2 * (2 - nu[ma]) * (1 + nu[ma]) / E[ma] + 2 * (2 - nu[mb]) * (1 + nu[mb]) / E[mb])
    cor = np.minimum(CoR[ma], CoR[mb])
    mu_c = np.maximum(mu[ma], mu[mb])
    crr = np.maximum(Crr[ma], Crr[mb])
    loge = np.where(cor < TINY, np.log(TINY), np.log(np.maximum(cor, 1e-300)))
    beta = loge / np.sqrt(loge * loge + PI * PI)
    # Hertz-Mindlin (FullHertzianForceModel.cu) in float64
    rAv = rot(q[oA], np.cross(w[oA], cpA))
    rBv = rot(q[oB], np.cross(w[oB], cpB))
    vrel = (v[oA] + rAv) - (v[oB] + rBv)
    proj = np.einsum("ij,ij->i", vrel, nrm)
    vt = vrel - proj[:, None] * nrm
    dt = hist[:, :3] + h * vt
    dt = dt - np.einsum("ij,ij->i", dt, nrm)[:, None] * nrm
    dtime = hist[:, 3] + h
    meff = mA * mB / (mA + mB)
    Rs = rA * rB / (rA + rB)
    dep = np.maximum(depth, 0.0)
    sqrt_Rd = np.sqrt(dep * Rs)
    Sn = 2 * Es * sqrt_Rd
    kn = 2.0 / 3.0 * Sn
    gn = C5 * beta * np.sqrt(Sn * meff)
    F = ((kn * dep + gn * proj)[:, None]) * nrm
    fmag = np.linalg.norm(F, axis=1)
    TOF = np.zeros((nC, 3))
    R_eff = np.sqrt(Rs)
    kn_s = 4.0 / 3.0 * Es * np.sqrt(R_eff)
    gn_s = -2 * np.sqrt(5.0 / 3.0 * meff * Es) * beta * R_eff ** 0.25
    dc = gn_s / (2 * np.sqrt(kn_s * meff))
    with np.errstate(invalid="ignore", divide="ignore"):
        t_coll = PI * np.sqrt(meff / (kn_s * (1 - dc * dc)))
    add_rr = (crr > 0) & ~((dc < 1) & (dtime <= t_coll))
    vr = rBv - rAv
    vmag = np.linalg.norm(vr, axis=1)
    rr = add_rr & (vmag > TINY)
    TOF[rr] = vr[rr] / vmag[rr, None] * (crr[rr] * fmag[rr])[:, None]
    kt = 8 * Gs * sqrt_Rd
    gt = -C5 * beta * np.sqrt(meff * kt)
    tf = -kt[:, None] * dt - gt[:, None] * vt
    ft = np.linalg.norm(tf, axis=1)
    fr = mu_c > 0
    ftmax = fmag * mu_c
    cap = fr & (ft > TINY) & (ft > ftmax)
    with np.errstate(invalid="ignore", divide="ignore"):
        ratio = np.where(cap, ftmax / np.where(ft > 0, ft, 1.0), 1.0)
    tf = tf * ratio[:, None]
    with np.errstate(invalid="ignore", divide="ignore"):
        dt = np.where(cap[:, None], (tf + gt[:, None] * vt) / np.where(kt > 0, -kt, 1.0)[:, None], dt)
    tf = np.where((fr & (ft > TINY))[:, None], tf, 0.0)
    F = F + tf
    # contacts that do not touch carry nothing and lose their history
    F[~act] = 0.0
    TOF[~act] = 0.0
    cpA[~act] = 0.0
    cpB[~act] = 0.0
    hout = np.concatenate([dt, dtime[:, None]], 1)
    hout[~act] = 0.0
    # collection (forceToAcc / forceToAngAcc)
    nO = built.counts["o"]
    acc = np.zeros((nO, 3))
    alpha = np.zeros((nO, 3))
    U = F + TOF
    np.add.at(acc, oA[act], F[act] / mA[act, None])
    np.add.at(alpha, oA[act], np.cross(cpA[act], rot_t(q[oA[act]], U[act])) / I[oA[act]])
    np.add.at(acc, oB[act], -F[act] / m[oB[act], None])
    np.add.at(alpha, oB[act], np.cross(cpB[act], rot_t(q[oB[act]], -U[act])) / I[oB[act]])
    # Extended Taylor integration with the constant family prescriptions
    G = np.asarray(p.G[:], np.float64)
    fam = S["family"]
    vn, wn = v.copy(), w.copy()
    u_lin = (acc + G) * h
    u_rot = alpha * h
    lin_p = np.zeros(nO, bool)
    rot_p = np.zeros(nO, bool)
    lin_pos = np.zeros(nO, bool)
    rot_pos = np.zeros(nO, bool)
    for f in np.unique(fam):
        pr = built.prescriptions[int(f)]
        if not pr.used:
            continue
        sel = fam == f
        for c in range(3):
            if pr.has_vel[c]:
                vn[sel, c] = float(np.float32(pr.vel[c]))
            if pr.has_omg[c]:
                wn[sel, c] = float(np.float32(pr.omg[c]))
        lin_p[sel] = bool(pr.lin_vel_prescribed)
        rot_p[sel] = bool(pr.rot_vel_prescribed)
        lin_pos[sel] = bool(pr.lin_pos_prescribed)
        rot_pos[sel] = bool(pr.rot_pos_prescribed)
        if any(pr.has_pos[c] for c in range(3)):
            raise NotImplementedError("prescribed positions are outside this model")
    vn = np.where(lin_p[:, None], vn, vn + u_lin)
    wn = np.where(rot_p[:, None], wn, wn + u_rot)
    vmid = np.where(lin_p[:, None], v, v + u_lin * 0.5)
    wmid = np.where(rot_p[:, None], w, w + u_rot * 0.5)
    pos_n = np.where(lin_pos[:, None], pos, pos + vmid * h)
    ln = np.linalg.norm(wmid, axis=1)
    th = 0.5 * h * ln
    with np.errstate(invalid="ignore", divide="ignore"):
        sfac = np.where(ln > 0, np.sin(th) / np.where(ln > 0, ln, 1.0), 0.0)
    dq = np.concatenate([np.where(ln > 0, np.cos(th), 1.0)[:, None], wmid * sfac[:, None]], 1)
    a1, b1, c1, d1 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    a2, b2, c2, d2 = dq[:, 0], dq[:, 1], dq[:, 2], dq[:, 3]
    qn = np.stack([a1 * a2 - b1 * b2 - c1 * c2 - d1 * d2, a1 * b2 + b1 * a2 + c1 * d2 - d1 * c2,
                   a1 * c2 - b1 * d2 + c1 * a2 + d1 * b2, a1 * d2 + b1 * c2 - c1 * b2 + d1 * a2], 1)
    qn = np.where(rot_pos[:, None], q, qn)
    return dict(force=F, torque_only_force=TOF, cpA=cpA, cpB=cpB, active=act, hist=hout, acc=acc, alpha=alpha,
                pos=pos_n, vel=vn, angvel=wn, quat=qn, pos0=pos)


def _keys(c):
    ss = c["type"].astype(np.int64) == SPHERE_SPHERE
    return (c["idA"].astype(np.int64) << 33) | (ss.astype(np.int64) << 32) | c["idB"].astype(np.int64)


def rollout_fixed(built, S0, lists, mats=None, f32=False, q_anchor=None):
    """Steps of ``step_state`` over the contact lists a run found (one list per step, each with idA, idB, type;
    the first also with the incoming history wildcards), the lists held fixed: each step's incoming history is the
    previous step's updated history of the contact with the same (idA, idB, type), 0 for a new contact -- the
    reference's history map (src/kernel/DEMHistoryMappingKernels.cu).  ``f32`` and ``q_anchor`` (the first step's
    only) as in ``step_state``.  Returns the final state (pos, q, v, w, family) and the per-step results."""
    S = dict(S0)
    prev_keys = prev_hist = None
    out = []
    for s, c in enumerate(lists):
        if s == 0:
            hist = c["wildcards"].astype(np.float64).T.copy() if c["wildcards"].size else np.zeros((len(c["idA"]), 4))
        else:
            k = _keys(c)
            order = np.argsort(prev_keys, kind="stable")
            hist = np.zeros((len(k), 4))
            if len(order):
                at = np.minimum(np.searchsorted(prev_keys[order], k), len(order) - 1)
                hit = prev_keys[order][at] == k
                hist[hit] = prev_hist[order[at[hit]]]
        r = step_state(built, S, c, hist=hist, mats=mats, f32=f32, q_anchor=q_anchor if s == 0 else None)
        S = dict(pos=r["pos"], q=r["quat"], v=r["vel"], w=r["angvel"], family=S["family"])
        prev_keys, prev_hist = _keys(c), r["hist"]
        out.append(r)
    return S, out

