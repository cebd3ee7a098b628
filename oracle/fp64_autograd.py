"""FP64 host adjoint of the DEM step for clumps and analytical walls: the model of ``oracle.fp64_model.step_state``
restated in torch (float64, on the CPU) and differentiated by torch's reverse mode.

TEST INFRASTRUCTURE ONLY: the reference the CUDA adjoint (deme_adjoint_backward) is checked against in tests/,
never part of the product.

``step`` evaluates one step of the reference's dynamics -- contact geometry of ``calculateContactForces``
(src/kernel/DEMCalcForceKernels.cu:14-179), the frictional Hertz--Mindlin model
(src/kernel/DEMCustomizablePolicies/FullHertzianForceModel.cu) with ``matProxy2ContactParam``
(src/kernel/DEMHelperKernels.cu:316-339), force collection (src/kernel/DEMCollectForceKernels.cu:68-120) and
Extended Taylor integration (src/kernel/DEMIntegrationKernels.cu:46-179) -- exactly as ``fp64_model.step_state``
does, with sphere offsets and wall placements rotated in float32 at the step's recorded quaternions plus the
float64 change from them (``fp64_model._rotate``), so that the geometry is the CUDA path's at the recorded state.
``adjoint`` chains the steps' reverse mode along a recorded trajectory: at every step the recorded state and
incoming contact histories, the contact list held fixed, the incoming-history gradient passed to the previous
step's contact with the same (idA, idB, type) -- the reverse of the history map
(src/kernel/DEMHistoryMappingKernels.cu).  That is the CUDA adjoint's own construction, so the two evaluate the
same derivatives at the same points; only the arithmetic (FP64 throughout here) differs.
"""
from __future__ import annotations

import numpy as np
import torch

from oracle import fp64_model as M

f64 = torch.float64


def _t(x):
    return torch.as_tensor(np.asarray(x), dtype=f64)


def rot(q, v):
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    ox, oy, oz = v[:, 0], v[:, 1], v[:, 2]
    X = (2 * (w * w + x * x) - 1) * ox + 2 * (x * y - w * z) * oy + 2 * (x * z + w * y) * oz
    Y = 2 * (x * y + w * z) * ox + (2 * (w * w + y * y) - 1) * oy + 2 * (y * z - w * x) * oz
    Z = 2 * (x * z - w * y) * ox + 2 * (y * z + w * x) * oy + (2 * (w * w + z * z) - 1) * oz
    return torch.stack([X, Y, Z], 1)


def rot_t(q, v):
    return rot(q * _t([1.0, -1.0, -1.0, -1.0]), v)


def _norm(x, safe):
    """Row norms; rows where ``safe`` is False get the norm of (1, 0, 0), so that no gradient meets sqrt(0)."""
    y = torch.where(safe[:, None], x, _t([1.0, 0.0, 0.0]).expand_as(x))
    return torch.sqrt((y * y).sum(1))


def free_owners(built, family):
    """Owners integrated from their forces: clumps of families without a prescription."""
    used = np.array([bool(built.prescriptions[int(f)].used) for f in family])
    nC = int(built.arrays["sphere_owner"].max()) + 1
    return (np.arange(built.counts["o"]) < nC) & ~used


def step(built, S_rec, contacts, pos, q, v, w, hist, mats):
    """One step from the differentiable state (pos, q, v, w: owners x 3 / 4, owner-frame angular velocity), incoming
    histories ``hist`` (contacts x 4) and materials ``mats`` (torch tensors E, nu, CoR, mu, Crr), at the recorded
    state ``S_rec`` (numpy; anchors the float32 rotations, places the walls and gives the families).  Returns the
    step-end state of the free owners (pos, q, v, w; driven owners keep their inputs) and the updated histories."""
    a = built.arrays
    h = float(built.params.h)
    m = _t(a["mass"])
    I = _t(np.stack([a["mmiXX"], a["mmiYY"], a["mmiZZ"]], 1))
    qr = S_rec["q"]
    o_np = a["sphere_owner"].astype(np.int64)
    o_s = torch.as_tensor(o_np)
    rel_np = np.stack([a["relX"], a["relY"], a["relZ"]], 1).astype(np.float64)
    rel = _t(rel_np)
    off_rec = _t(M.rot_f32(qr[o_np], rel_np))
    Xs = pos[o_s] + off_rec + rot(q[o_s], rel) - rot(_t(qr)[o_s], rel)
    an = M.placed_analytical(built, S_rec["pos"], qr, True)
    rad = _t(a["radius"])
    mat_s = torch.as_tensor((a["sphere_material_wide"] if "sphere_material_wide" in a else
                             a["sphere_material"]).astype(np.int64))
    E, nu, CoR, mu, Crr = (mats[k] for k in ("E", "nu", "CoR", "mu", "Crr"))
    A_np = contacts["idA"].astype(np.int64)
    B_np = contacts["idB"].astype(np.int64)
    ss_np = contacts["type"].astype(np.int64) == M.SPHERE_SPHERE
    A, Bid, ss = torch.as_tensor(A_np), torch.as_tensor(B_np), torch.as_tensor(ss_np)
    nC = len(A_np)
    Bs = torch.where(ss, Bid, torch.zeros_like(Bid))
    oA = o_s[A]
    if an is not None:
        k_np = np.where(ss_np, 0, B_np)
        an_owner = torch.as_tensor(an["owner"][k_np])
    else:
        k_np = np.zeros(nC, np.int64)
        an_owner = torch.zeros(nC, dtype=torch.int64)
    oB = torch.where(ss, o_s[Bs], an_owner)
    XA, rA = Xs[A], rad[A]
    # sphere pairs (checkSpheresOverlap form)
    XB, r_b = Xs[Bs], rad[Bs]
    dv = XA - XB
    d = _norm(dv, ss)
    n_ss = dv / d[:, None]
    dep_ss = rA + r_b - d
    cp_ss = XB + (r_b - dep_ss / 2.0)[:, None] * n_ss
    # walls (checkSphereEntityOverlap form; cylinder and cone with the plane's conventions)
    wall = ~ss
    if an is not None:
        P, dd = _t(an["p"][k_np]), _t(an["d"][k_np])
        tw = torch.as_tensor(an["type"][k_np])
        outw = torch.as_tensor(an["normal"][k_np] == 1)
        size1, c1, c2 = _t(an["size1"][k_np]), _t(an["c1"][k_np]), _t(an["c2"][k_np])
        umin, umax = _t(an["umin"][k_np]), _t(an["umax"][k_np])
        mB_w, mat_w = _t(an["mass"][k_np]), torch.as_tensor(an["mat"][k_np])
    else:
        P = dd = torch.zeros((nC, 3), dtype=f64)
        tw = torch.zeros(nC, dtype=torch.int64)
        outw = torch.zeros(nC, dtype=torch.bool)
        size1 = c1 = c2 = umin = umax = mB_w = torch.zeros(nC, dtype=f64)
        mat_w = torch.zeros(nC, dtype=torch.int64)
    pl = tw == M.ANAL_PLANE
    vv = XA - P
    t = (vv * dd).sum(1)
    wv = vv - t[:, None] * dd
    curved = wall & ~pl
    rho_np_ok = curved.clone()
    rho = _norm(wv, rho_np_ok)
    valid = ~curved | (rho > 0)
    u = wv / rho[:, None]
    isc = tw == M.ANAL_CYLINDER
    gap_cy = torch.where(outw, rho - size1, size1 - rho)
    n_cy = torch.where(outw[:, None], u, -u)
    gc = t * c1 - rho * c2
    gvv = c1[:, None] * dd - c2[:, None] * u
    gap_co = torch.where(outw, -gc, gc)
    n_co = torch.where(outw[:, None], -gvv, gvv)
    uc = (t * c2 + rho * c1) * c2
    valid = valid & (~(curved & ~isc) | ((uc >= umin) & (uc <= umax)))
    gap = torch.where(pl, t, torch.where(isc, gap_cy, gap_co))
    n_w = torch.where(pl[:, None], dd, torch.where(isc[:, None], n_cy, n_co))
    od = (rA - gap) / 2.0
    cp_w = XA - n_w * (gap + od)[:, None]
    nrm = torch.where(ss[:, None], n_ss, n_w)
    cp = torch.where(ss[:, None], cp_ss, cp_w)
    depth = torch.where(ss, dep_ss, od)
    act = torch.where(ss, d <= rA + r_b, valid & (od >= 0))
    rB = torch.where(ss, r_b, torch.full_like(r_b, M.HUGE))
    mB = torch.where(ss, m[oB], mB_w)
    matB = torch.where(ss, mat_s[Bs], mat_w)
    mA = m[oA]
    dep = torch.where(act, depth, torch.ones_like(depth))  # a positive stand-in where the contact is open
    # material pair (matProxy2ContactParam)
    ma, mb = mat_s[A], matB
    Es = 1.0 / ((1 - nu[ma] ** 2) / E[ma] + (1 - nu[mb] ** 2) / E[mb])
    Gs = 1.0 / (2 * (2 - nu[ma]) * (1 + nu[ma]) / E[ma] + 2 * (2 - nu[mb]) * (1 + nu[mb]) / E[mb])
    cor = torch.minimum(CoR[ma], CoR[mb])
    mu_c = torch.maximum(mu[ma], mu[mb])
    crr = torch.maximum(Crr[ma], Crr[mb])
    loge = torch.log(torch.clamp(cor, min=M.TINY))
    beta = loge / torch.sqrt(loge * loge + M.PI * M.PI)
    # Hertz-Mindlin, rotational velocities formed through the owner frames as the reference forms them
    cpA = rot_t(q[oA], cp - pos[oA])
    cpB = rot_t(q[oB], cp - pos[oB])
    WA = rot(q[oA], torch.cross(w[oA], cpA, dim=1))
    WB = rot(q[oB], torch.cross(w[oB], cpB, dim=1))
    vrel = (v[oA] + WA) - (v[oB] + WB)
    proj = (vrel * nrm).sum(1)
    vt = vrel - proj[:, None] * nrm
    dt = hist[:, :3] + h * vt
    dt = dt - (dt * nrm).sum(1)[:, None] * nrm
    dtime = hist[:, 3] + h
    meff = mA * mB / (mA + mB)
    Rs = rA * rB / (rA + rB)
    sqrt_Rd = torch.sqrt(dep * Rs)
    Sn = 2 * Es * sqrt_Rd
    kn = 2.0 / 3.0 * Sn
    gn = M.C5 * beta * torch.sqrt(Sn * meff)
    fnm = kn * dep + gn * proj
    Fn = fnm[:, None] * nrm
    fmag = torch.abs(fnm) * torch.sqrt((nrm * nrm).sum(1))  # the length of the normal force vector
    R_eff = torch.sqrt(Rs)
    kn_s = 4.0 / 3.0 * Es * torch.sqrt(R_eff)
    gn_s = -2 * torch.sqrt(5.0 / 3.0 * meff * Es) * beta * R_eff ** 0.25
    dc = gn_s / (2 * torch.sqrt(kn_s * meff))
    dc_ok = dc < 1
    t_coll = M.PI * torch.sqrt(meff / (kn_s * torch.where(dc_ok, 1 - dc * dc, torch.ones_like(dc))))
    add_rr = (crr > 0) & ~(dc_ok & (dtime <= t_coll))
    vr = WB - WA
    vsq = (vr * vr).sum(1)
    rr = add_rr & (vsq > M.TINY * M.TINY)
    vmag = _norm(vr, rr)
    TOF = torch.where(rr[:, None], vr / vmag[:, None] * (crr * fmag)[:, None], torch.zeros_like(vr))
    kt = 8 * Gs * sqrt_Rd
    gt = -M.C5 * beta * torch.sqrt(meff * kt)
    tf = -kt[:, None] * dt - gt[:, None] * vt
    tsq = (tf * tf).sum(1)
    big = (mu_c > 0) & (tsq > M.TINY * M.TINY)
    ft = _norm(tf, big)
    cap = big & (ft > fmag * mu_c)
    ratio = torch.where(cap, fmag * mu_c / ft, torch.ones_like(ft))
    tfc = tf * ratio[:, None]
    dt = torch.where(cap[:, None], (tfc + gt[:, None] * vt) / (-kt)[:, None], dt)
    tfc = torch.where(big[:, None], tfc, torch.zeros_like(tfc))
    Fc = torch.where(act[:, None], Fn + tfc, torch.zeros_like(Fn))
    TOF = torch.where(act[:, None], TOF, torch.zeros_like(TOF))
    hout = torch.where(act[:, None], torch.cat([dt, dtime[:, None]], 1), torch.zeros((nC, 4), dtype=f64))
    # collection (forceToAcc / forceToAngAcc)
    nO = built.counts["o"]
    U = Fc + TOF
    acc = torch.zeros((nO, 3), dtype=f64).index_add(0, oA, Fc / mA[:, None]).index_add(0, oB, -Fc / m[oB][:, None])
    alpha = torch.zeros((nO, 3), dtype=f64).index_add(0, oA, torch.cross(cpA, rot_t(q[oA], U), dim=1) / I[oA])
    alpha = alpha.index_add(0, oB, torch.cross(cpB, rot_t(q[oB], -U), dim=1) / I[oB])
    # Extended Taylor integration of the free owners
    free = torch.as_tensor(free_owners(built, S_rec["family"]))[:, None]
    G = _t(np.asarray(built.params.G[:], np.float64))
    u_lin = (acc + G) * h
    u_rot = alpha * h
    vn = torch.where(free, v + u_lin, v)
    wn = torch.where(free, w + u_rot, w)
    pos_n = torch.where(free, pos + (v + u_lin * 0.5) * h, pos)
    wmid = w + u_rot * 0.5
    msq = (wmid * wmid).sum(1)
    spin = msq > 0
    ln = _norm(wmid, spin)
    th = 0.5 * h * ln
    # sin(h |w| / 2) / |w|, whose limit h / 2 at w = 0 carries the derivative there
    sfac = torch.where(spin, torch.sin(th) / ln, torch.full_like(ln, 0.5 * h))
    dq = torch.cat([torch.where(spin, torch.cos(th), torch.ones_like(th))[:, None], wmid * sfac[:, None]], 1)
    a1, b1, c1_, d1 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    a2, b2, c2_, d2 = dq[:, 0], dq[:, 1], dq[:, 2], dq[:, 3]
    qn = torch.stack([a1 * a2 - b1 * b2 - c1_ * c2_ - d1 * d2, a1 * b2 + b1 * a2 + c1_ * d2 - d1 * c2_,
                      a1 * c2_ - b1 * d2 + c1_ * a2 + d1 * b2, a1 * d2 + b1 * c2_ - c1_ * b2 + d1 * a2], 1)
    qn = torch.where(free, qn, q)
    return (pos_n, qn, vn, wn), hout


def adjoint(built, states, lists, seeds, mats):
    """Reverse mode along a recorded run: ``states`` the T + 1 recorded states (dicts pos, q, v, w, family; float64
    numpy), ``lists`` the T recorded contact lists (idA, idB, type, incoming history wildcards), ``seeds`` the loss
    gradients at the final state in the interface's variables (position, velocity, world angular velocity,
    quaternion at fixed world angular velocity; owners x 3 / 4), ``mats`` the materials (numpy float64 arrays).
    Returns the gradients at the first state in the same variables and the material gradients (n_materials x 4:
    E, CoR, mu, Crr)."""
    T = len(lists)
    mt = {k: _t(v).requires_grad_(True) for k, v in mats.items()}
    # seeds: w_world = R(q) w at the final state
    SF = states[T]
    qf = _t(SF["q"]).requires_grad_(True)
    wf = _t(SF["w"]).requires_grad_(True)
    gW = _t(seeds[2])
    (rot(qf, wf) * gW).sum().backward()
    lam = [_t(seeds[0]), _t(seeds[3]) + qf.grad, _t(seeds[1]), wf.grad.clone()]  # pos, q, v, w
    lamH = None
    gm = torch.zeros((len(mats["E"]), 4), dtype=f64)
    free = torch.as_tensor(free_owners(built, states[0]["family"]))[:, None]
    for s in range(T - 1, -1, -1):
        S = states[s]
        c = lists[s]
        xs = [_t(S[k]).requires_grad_(True) for k in ("pos", "q", "v", "w")]
        nC = len(c["idA"])
        H = _t(c["wildcards"].T.copy() if c["wildcards"].size else np.zeros((nC, 4))).requires_grad_(True)
        (pn, qn, vn, wn), hout = step(built, S, c, xs[0], xs[1], xs[2], xs[3], H, mt)
        outs = [pn, qn, vn, wn]
        gouts = list(lam)
        if lamH is not None and nC:
            outs.append(hout)
            gouts.append(lamH)
        ins = xs + [H] + [mt[k] for k in ("E", "CoR", "mu", "Crr")]
        g = torch.autograd.grad(outs, ins, grad_outputs=gouts, allow_unused=True)
        lam = [torch.where(free, gi, torch.zeros_like(gi)) if gi is not None else torch.zeros_like(xs[j])
               for j, gi in enumerate(g[:4])]
        for j in range(4):
            if g[5 + j] is not None:
                gm[:, j] += g[5 + j]
        # incoming-history gradient to the previous list's contact with the same (idA, idB, type)
        lamH = None
        if s > 0 and nC and g[4] is not None:
            prev = lists[s - 1]
            kp, kc = M._keys(prev), M._keys(c)
            order = np.argsort(kp, kind="stable")
            lamH = torch.zeros((len(kp), 4), dtype=f64)
            if len(order):
                at = np.minimum(np.searchsorted(kp[order], kc), len(order) - 1)
                hit = kp[order][at] == kc
                lamH[torch.as_tensor(order[at[hit]])] = g[4][torch.as_tensor(hit)]
    # results: w = R(q)^T w_world at the first state
    S0 = states[0]
    q0 = _t(S0["q"]).requires_grad_(True)
    wW0 = rot(_t(S0["q"]), _t(S0["w"]))
    lq, lw = lam[1], lam[3]
    (rot_t(q0, wW0) * lw).sum().backward()
    d_quat = lq + q0.grad
    d_angvel = rot(_t(S0["q"]), lw)
    mask = free.numpy()
    out = dict(d_pos0=lam[0].numpy() * mask, d_vel0=lam[2].numpy() * mask, d_angvel0=d_angvel.numpy() * mask,
               d_quat0=d_quat.numpy() * mask, d_material=gm.numpy())
    return out
