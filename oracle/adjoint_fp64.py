"""FP64 forward model and FP64 host adjoint of a DEM step for sphere scenes with plane walls.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA adjoint (tests/), never part of the product.

The model is the per-step dynamics of the built-in frictional Hertz-Mindlin contact
(src/kernel/DEMCustomizablePolicies/FullHertzianForceModel.cu, src/kernel/DEMCalcForceKernels.cu:14-179: overlap,
contact point from B's side, lever arms, normal spring-dashpot, rolling resistance after the collision time,
tangential spring with Coulomb cap and history), force collection onto owners
(src/kernel/DEMCollectForceKernels.cu:68-120) and Extended Taylor integration
(src/kernel/DEMIntegrationKernels.cu:46-179), all in float64, for single-sphere owners whose angular velocity is
kept in the world frame (for an isotropic sphere the orientation does not enter the contact law).  Contacts are
the overlapping pairs of each step; a pair keeps its tangential history while it stays in contact (the history
map of src/kernel/DEMHistoryMappingKernels.cu) and restarts from zero otherwise.

``rollout`` runs the forward pass and keeps every step; ``adjoint`` runs the reverse pass over it and returns the
gradients of a loss with respect to the initial state and to the material parameters (E, CoR, mu, Crr).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.spatial import cKDTree

C5 = 1.825741858350554   # 2 sqrt(5/6), src/DEM/Defines.h
PI2 = 9.869604401089358
TINY = 1e-12
HUGE_R = 1e15
# Floors in the derivatives at the model's non-smooth points (the same values as the CUDA adjoint): the rolling
# torque's direction (relative rolling speed, m/s), the damping's overlap^(1/4) (overlap relative to R*) and the
# Coulomb cap's 1/|Ft| (N).  The forward model is unchanged; where a floor binds, the derivative is that of the
# smoothed law, because the exact one (unbounded at zero rolling speed or zero overlap) measures sensitivity only
# in a neighbourhood far smaller than any parameter change of interest.
REG = {"delta_rel": 1e-4, "roll_speed": 1e-4, "ft": 1e-6}


@dataclass
class SphereScene:
    r: np.ndarray          # (n,) radii
    m: np.ndarray          # (n,) masses
    inertia: np.ndarray    # (n,) isotropic moments of inertia
    mat: np.ndarray        # (n,) material index
    planes: list           # [(point (3,), unit normal (3,), material, owner position (3,))]
    E: np.ndarray          # per material
    nu: np.ndarray
    CoR: np.ndarray
    mu: np.ndarray
    Crr: np.ndarray
    h: float
    g: np.ndarray          # gravity (3,)
    plane_mass: float = 1e15


@dataclass
class Step:
    x: np.ndarray
    v: np.ndarray
    w: np.ndarray
    ss: np.ndarray          # (C, 2) sphere pairs A < B
    sp: np.ndarray          # (P, 2) (sphere, plane index)
    hist_ss: np.ndarray     # (C, 4) history at step start (delta_tan xyz, delta_time)
    hist_sp: np.ndarray
    prev_ss: np.ndarray     # index of each pair in the previous step's list, -1 when new
    prev_sp: np.ndarray
    extra: dict = field(default_factory=dict)


def mat_pair(sc: SphereScene, ma, mb):
    """matProxy2ContactParam in float64, with the index of the material that sets CoR (min), mu and Crr (max)."""
    invE = (1 - sc.nu[ma] ** 2) / sc.E[ma] + (1 - sc.nu[mb] ** 2) / sc.E[mb]
    Es = 1.0 / invE
    invG = 2 * (2 - sc.nu[ma]) * (1 + sc.nu[ma]) / sc.E[ma] + 2 * (2 - sc.nu[mb]) * (1 + sc.nu[mb]) / sc.E[mb]
    Gs = 1.0 / invG
    cor_src = np.where(sc.CoR[ma] < sc.CoR[mb], ma, mb)
    mu_src = np.where(sc.mu[ma] > sc.mu[mb], ma, mb)
    crr_src = np.where(sc.Crr[ma] > sc.Crr[mb], ma, mb)
    return Es, Gs, sc.CoR[cor_src], sc.mu[mu_src], sc.Crr[crr_src], cor_src, mu_src, crr_src


def beta_of(e):
    le = np.log(np.maximum(e, TINY))
    return le / np.sqrt(le * le + PI2)


def dbeta_de(e):
    le = np.log(np.maximum(e, TINY))
    return (1.0 / np.maximum(e, TINY)) * PI2 / (le * le + PI2) ** 1.5


def _cross(a, b):
    return np.cross(a, b)


def _dot(a, b):
    return np.einsum("ij,ij->i", a, b)


def contact_law(geo, vA, vB, wA, wB, hist, Es, Gs, be, mu, crr, meff, Rs, h, keep=False):
    """One contact set.  geo: dict with n (C,3), delta (C,), rAv, rBv (C,3).  Returns f, t, hist_out (and the
    intermediates when ``keep``)."""
    n, delta, rAv, rBv = geo["n"], geo["delta"], geo["rAv"], geo["rBv"]
    WA = _cross(wA, rAv)
    WB = _cross(wB, rBv)
    vr = vA + WA - vB - WB
    p = _dot(vr, n)
    vt = vr - p[:, None] * n
    dt1 = hist[:, :3] + h * vt
    q = _dot(dt1, n)
    dt2 = dt1 - q[:, None] * n
    tau2 = hist[:, 3] + h
    s = np.sqrt(delta * Rs)
    Sn = 2 * Es * s
    kn = (2.0 / 3.0) * Sn
    gn = C5 * be * np.sqrt(Sn * meff)
    fnm = kn * delta + gn * p
    fn = fnm[:, None] * n
    A = np.abs(fnm)
    # rolling resistance after the collision time
    Reff = np.sqrt(Rs)
    kns = (4.0 / 3.0) * Es * np.sqrt(Reff)
    gns = -2 * np.sqrt((5.0 / 3.0) * meff * Es) * be * Reff ** 0.25
    dc = gns / (2 * np.sqrt(kns * meff))
    with np.errstate(invalid="ignore", divide="ignore"):
        tcoll = np.where(dc < 1.0, np.pi * np.sqrt(meff / (kns * (1 - dc * dc))), -np.inf)
    vroll = WB - WA
    L = np.linalg.norm(vroll, axis=1)
    roll = (crr > 0) & (tau2 > tcoll) & (L > TINY)
    e = np.where(roll[:, None], vroll / np.where(L > 0, L, 1)[:, None], 0.0)
    t = np.where(roll[:, None], (crr * A)[:, None] * e, 0.0)
    # tangential with Coulomb cap
    kt = 8 * Gs * s
    gt = -C5 * be * np.sqrt(meff * kt)
    Ft = -kt[:, None] * dt2 - gt[:, None] * vt
    ft = np.linalg.norm(Ft, axis=1)
    fric = mu > 0
    big = fric & (ft > TINY)
    cap = big & (ft > A * mu)
    rr = np.where(cap, A * mu / np.where(ft > 0, ft, 1), 1.0)
    Ftp = np.where(big[:, None], rr[:, None] * Ft, 0.0)
    dt3 = np.where(cap[:, None], (Ftp + gt[:, None] * vt) / (-kt)[:, None], dt2)
    f = fn + Ftp
    hist_out = np.concatenate([dt3, tau2[:, None]], axis=1)
    if keep:
        return f, t, hist_out, dict(WA=WA, WB=WB, vr=vr, p=p, vt=vt, dt1=dt1, q=q, dt2=dt2, s=s, Sn=Sn, kn=kn, gn=gn,
                                    fnm=fnm, A=A, roll=roll, e=e, L=L, kt=kt, gt=gt, Ft=Ft, ft=ft, big=big, cap=cap,
                                    rr=rr, Ftp=Ftp)
    return f, t, hist_out


def geometry_ss(x, r, A, B):
    d = x[A] - x[B]
    D = np.linalg.norm(d, axis=1)
    n = d / D[:, None]
    delta = r[A] + r[B] - D
    a_ = r[A] - delta / 2
    b_ = r[B] - delta / 2
    return dict(d=d, D=D, n=n, delta=delta, a_=a_, b_=b_, rAv=-a_[:, None] * n, rBv=b_[:, None] * n)


def geometry_sp(x, r, A, planes, P):
    pp = np.array([planes[k][0] for k in P]).reshape(-1, 3)
    nn = np.array([planes[k][1] for k in P]).reshape(-1, 3)
    bo = np.array([planes[k][3] for k in P]).reshape(-1, 3)
    dist = _dot(x[A] - pp, nn)
    delta = (r[A] - dist) / 2
    cp = x[A] - nn * (dist + delta)[:, None]
    return dict(n=nn, dist=dist, delta=delta, rAv=cp - x[A], rBv=cp - bo)


def detect(sc: SphereScene, x):
    """Overlapping sphere pairs (A < B) and sphere-plane contacts, sorted by (A, B) / (A, plane)."""
    n = len(sc.r)
    tree = cKDTree(x)
    pairs = np.array(sorted(tree.query_pairs(2 * float(sc.r.max()))), dtype=np.int64).reshape(-1, 2)
    if len(pairs):
        d = np.linalg.norm(x[pairs[:, 0]] - x[pairs[:, 1]], axis=1)
        pairs = pairs[d <= sc.r[pairs[:, 0]] + sc.r[pairs[:, 1]]]
    sp = []
    for k, (pt, nr, _, _) in enumerate(sc.planes):
        dist = (x - pt) @ nr
        idx = np.nonzero((sc.r - dist) / 2 >= 0)[0]
        sp += [(i, k) for i in idx]
    sp = np.array(sorted(sp), dtype=np.int64).reshape(-1, 2)
    return pairs, sp


def _match(keys, prev_keys):
    if len(prev_keys) == 0 or len(keys) == 0:
        return np.full(len(keys), -1, np.int64)
    order = np.argsort(prev_keys)
    pos = np.searchsorted(prev_keys[order], keys)
    pos = np.minimum(pos, len(prev_keys) - 1)
    hit = prev_keys[order][pos] == keys
    return np.where(hit, order[pos], -1)


def forces(sc: SphereScene, x, v, w, ss, sp, hss, hsp, keep=False):
    """Per-owner force and torque (world frame) and the updated histories."""
    n = len(sc.r)
    F = np.zeros((n, 3))
    T = np.zeros((n, 3))
    out = {}
    if len(ss):
        A, B = ss[:, 0], ss[:, 1]
        geo = geometry_ss(x, sc.r, A, B)
        Es, Gs, cor, mu, crr, cs, ms, rs = mat_pair(sc, sc.mat[A], sc.mat[B])
        meff = sc.m[A] * sc.m[B] / (sc.m[A] + sc.m[B])
        Rs = sc.r[A] * sc.r[B] / (sc.r[A] + sc.r[B])
        res = contact_law(geo, v[A], v[B], w[A], w[B], hss, Es, Gs, beta_of(cor), mu, crr, meff, Rs, sc.h, keep)
        f, t, hout = res[:3]
        u = f + t
        np.add.at(F, A, f)
        np.add.at(F, B, -f)
        np.add.at(T, A, _cross(geo["rAv"], u))
        np.add.at(T, B, -_cross(geo["rBv"], u))
        out["ss"] = (hout, geo, res[3] if keep else None, (Es, Gs, cor, mu, crr, cs, ms, rs, meff, Rs), f, t)
    if len(sp):
        A, P = sp[:, 0], sp[:, 1]
        geo = geometry_sp(x, sc.r, A, sc.planes, P)
        pm = np.array([sc.planes[k][2] for k in P], np.int64)
        Es, Gs, cor, mu, crr, cs, ms, rs = mat_pair(sc, sc.mat[A], pm)
        meff = sc.m[A] * sc.plane_mass / (sc.m[A] + sc.plane_mass)
        Rs = sc.r[A] * HUGE_R / (sc.r[A] + HUGE_R)
        zero = np.zeros((len(A), 3))
        res = contact_law(geo, v[A], zero, w[A], zero, hsp, Es, Gs, beta_of(cor), mu, crr, meff, Rs, sc.h, keep)
        f, t, hout = res[:3]
        np.add.at(F, A, f)
        np.add.at(T, A, _cross(geo["rAv"], f + t))
        out["sp"] = (hout, geo, res[3] if keep else None, (Es, Gs, cor, mu, crr, cs, ms, rs, meff, Rs), f, t)
    return F, T, out


def rollout(sc: SphereScene, x0, v0, w0, n_steps: int, free=None, init=None):
    """Forward pass; returns the final (x, v, w) and the list of steps (state, contacts and histories at each
    step start).  ``free`` masks the spheres that integrate (all by default).  ``init`` = (ss, sp, hist_ss,
    hist_sp) is the contact list of the step before the window with its updated histories, so that a window cut
    from a longer run keeps the contact histories it starts with."""
    x, v, w = x0.astype(np.float64).copy(), v0.astype(np.float64).copy(), w0.astype(np.float64).copy()
    n = len(sc.r)
    free = np.ones(n, bool) if free is None else free
    steps = []
    prev_ss = np.zeros((0, 2), np.int64)
    prev_sp = np.zeros((0, 2), np.int64)
    hout_ss = np.zeros((0, 4))
    hout_sp = np.zeros((0, 4))
    if init is not None:
        prev_ss, prev_sp = np.asarray(init[0], np.int64).reshape(-1, 2), np.asarray(init[1], np.int64).reshape(-1, 2)
        hout_ss, hout_sp = np.asarray(init[2], np.float64).reshape(-1, 4), np.asarray(init[3], np.float64).reshape(-1, 4)
    for _ in range(n_steps):
        ss, sp = detect(sc, x)
        mss = _match(ss[:, 0] * (n + 1) + ss[:, 1], prev_ss[:, 0] * (n + 1) + prev_ss[:, 1])
        msp = _match(sp[:, 0] * 4096 + sp[:, 1], prev_sp[:, 0] * 4096 + prev_sp[:, 1])
        hss = np.zeros((len(ss), 4))
        hss[mss >= 0] = hout_ss[mss[mss >= 0]]
        hsp = np.zeros((len(sp), 4))
        hsp[msp >= 0] = hout_sp[msp[msp >= 0]]
        steps.append(Step(x.copy(), v.copy(), w.copy(), ss, sp, hss, hsp, mss, msp))
        F, T, out = forces(sc, x, v, w, ss, sp, hss, hsp)
        hout_ss = out["ss"][0] if "ss" in out else np.zeros((0, 4))
        hout_sp = out["sp"][0] if "sp" in out else np.zeros((0, 4))
        a = F / sc.m[:, None] + sc.g
        al = T / sc.inertia[:, None]
        h = sc.h
        xn = x + h * (v + a * (h / 2))
        vn = v + a * h
        wn = w + al * h
        x = np.where(free[:, None], xn, x)
        v = np.where(free[:, None], vn, v)
        w = np.where(free[:, None], wn, w)
        prev_ss, prev_sp = ss, sp
    return (x, v, w), steps


def contact_law_vjp(geo, I, vA, vB, wA, wB, hist, Es, Gs, be, mu, crr, meff, Rs, h, g_f, g_t, g_hout):
    """Reverse pass of contact_law.  I holds its intermediates.  Returns the gradients with respect to the inputs
    (dict) given the gradients of f, t and hist_out."""
    n, delta, rAv, rBv = geo["n"], geo["delta"], geo["rAv"], geo["rBv"]
    C = len(delta)
    z3 = lambda: np.zeros((C, 3))  # noqa: E731
    g_dt3, g_tau2 = g_hout[:, :3], g_hout[:, 3]
    g_fn = g_f.copy()
    g_Ftp = g_f.copy()
    g_dt2, g_vt, g_n, g_WA, g_WB = z3(), z3(), z3(), z3(), z3()
    g_kt = np.zeros(C)
    g_gt = np.zeros(C)
    g_A = np.zeros(C)
    g_mu = np.zeros(C)
    # tangential
    cap, big = I["cap"], I["big"]
    kt, gt, vt, Ft, ft, A, Ftp = I["kt"], I["gt"], I["vt"], I["Ft"], I["ft"], I["A"], I["Ftp"]
    X = Ftp + gt[:, None] * vt
    kt_safe = np.where(kt != 0, kt, 1.0)
    g_Ftp_c = g_Ftp - np.where(cap[:, None], g_dt3 / kt_safe[:, None], 0.0)
    g_gt += np.where(cap, -_dot(g_dt3, vt) / kt_safe, 0.0)
    g_vt += np.where(cap[:, None], -gt[:, None] * g_dt3 / kt_safe[:, None], 0.0)
    g_kt += np.where(cap, _dot(g_dt3, X) / kt_safe ** 2, 0.0)
    g_dt2 += np.where(cap[:, None], 0.0, g_dt3)
    ft_safe = np.where(ft > 0, np.maximum(ft, REG["ft"]), 1.0)
    rr = I["rr"]
    g_Ft = np.where(big[:, None], rr[:, None] * g_Ftp_c, 0.0)
    g_rr = np.where(cap, _dot(g_Ftp_c, Ft), 0.0)
    g_A += np.where(cap, g_rr * mu / ft_safe, 0.0)
    g_mu += np.where(cap, g_rr * A / ft_safe, 0.0)
    g_ft = np.where(cap, -g_rr * A * mu / ft_safe ** 2, 0.0)
    g_Ft += np.where(cap[:, None], g_ft[:, None] * Ft / ft_safe[:, None], 0.0)
    # Ft = -kt dt2 - gt vt
    g_kt += -_dot(g_Ft, I["dt2"])
    g_dt2 += -kt[:, None] * g_Ft
    g_gt += -_dot(g_Ft, vt)
    g_vt += -gt[:, None] * g_Ft
    # gt = -C5 be sqrt(meff kt); kt = 8 Gs s
    smk = np.sqrt(meff * kt)
    s_d = np.maximum(I["s"], Rs * np.sqrt(REG["delta_rel"]))  # s = sqrt(delta Rs) floored in derivatives
    smk_d = np.sqrt(meff * 8 * Gs * s_d)
    g_be = g_gt * (-C5 * smk)
    g_kt += g_gt * (-C5 * be * meff / (2 * np.where(smk_d > 0, smk_d, 1.0)))
    g_Gs = 8 * I["s"] * g_kt
    g_s = 8 * Gs * g_kt
    # rolling: t = crr A e
    roll, e, L = I["roll"], I["e"], I["L"]
    ge = _dot(g_t, e)
    g_crr = np.where(roll, A * ge, 0.0)
    g_A += np.where(roll, crr * ge, 0.0)
    g_e = (crr * A)[:, None] * g_t
    L_safe = np.where(L > 0, np.maximum(L, REG["roll_speed"]), 1.0)
    g_vroll = np.where(roll[:, None], (g_e - _dot(g_e, e)[:, None] * e) / L_safe[:, None], 0.0)
    g_WB += g_vroll
    g_WA -= g_vroll
    # |fnm|, fn = fnm n
    fnm = I["fnm"]
    g_fnm = g_A * np.sign(fnm) + _dot(g_fn, n)
    g_n += fnm[:, None] * g_fn
    # fnm = kn delta + gn p
    kn, gn, p = I["kn"], I["gn"], I["p"]
    g_kn = g_fnm * delta
    g_delta = g_fnm * kn
    g_gn = g_fnm * p
    g_p = g_fnm * gn
    Sn = I["Sn"]
    ssm = np.sqrt(Sn * meff)
    ssm_d = np.sqrt(2 * Es * s_d * meff)
    g_be += g_gn * C5 * ssm
    g_Sn = g_gn * C5 * be * meff / (2 * np.where(ssm_d > 0, ssm_d, 1.0)) + (2.0 / 3.0) * g_kn
    g_Es = 2 * I["s"] * g_Sn
    g_s += 2 * Es * g_Sn
    s = I["s"]
    g_delta += g_s * Rs / (2 * np.where(s_d > 0, s_d, 1.0))
    # history
    g_tau = g_tau2
    q, dt1 = I["q"], I["dt1"]
    g_dt1 = g_dt2.copy()
    g_q = -_dot(g_dt2, n)
    g_n += -q[:, None] * g_dt2
    g_dt1 += g_q[:, None] * n
    g_n += g_q[:, None] * dt1
    g_dtan = g_dt1
    g_vt += h * g_dt1
    # vt = vr - p n ; p = vr . n
    vr = I["vr"]
    g_vr = g_vt.copy()
    g_p += -_dot(g_vt, n)
    g_n += -p[:, None] * g_vt
    g_vr += g_p[:, None] * n
    g_n += g_p[:, None] * vr
    # vr = vA + WA - vB - WB
    g_WA += g_vr
    g_WB -= g_vr
    g_wA = _cross(rAv, g_WA)
    g_rAv = _cross(g_WA, wA)
    g_wB = _cross(rBv, g_WB)
    g_rBv = _cross(g_WB, wB)
    return dict(vA=g_vr, vB=-g_vr, wA=g_wA, wB=g_wB, hist=np.concatenate([g_dtan, g_tau[:, None]], 1), rAv=g_rAv,
                rBv=g_rBv, n=g_n, delta=g_delta, Es=g_Es, Gs=g_Gs, be=g_be, mu=g_mu, crr=g_crr)


def geometry_ss_vjp(geo, g_n, g_delta, g_rAv, g_rBv):
    """Gradient of the sphere-pair geometry with respect to d = xA - xB."""
    n, D, a_, b_ = geo["n"], geo["D"], geo["a_"], geo["b_"]
    g_a = -_dot(g_rAv, n)
    g_b = _dot(g_rBv, n)
    g_n = g_n - a_[:, None] * g_rAv + b_[:, None] * g_rBv
    g_delta = g_delta - g_a / 2 - g_b / 2
    g_D = -g_delta
    g_d = (g_n - _dot(g_n, n)[:, None] * n) / D[:, None] + g_D[:, None] * n
    return g_d


def geometry_sp_vjp(geo, g_delta, g_rAv):
    """Gradient of the sphere-plane geometry with respect to xA (the plane is fixed; rBv only enters torques on
    the plane's owner, which does not move)."""
    n = geo["n"]
    # delta = (r - dist) / 2, rAv = -n (dist + delta) = -n (r + dist) / 2
    g_dist = -g_delta / 2 - _dot(g_rAv, n) / 2
    return g_dist[:, None] * n


def adjoint(sc: SphereScene, steps, gx, gv, gw, free=None):
    """Reverse pass over ``steps`` (from rollout) for the loss gradient (gx, gv, gw) at the final state.  Returns
    dL/dx0, dL/dv0, dL/dw0 and per-material dL/d(E, CoR, mu, Crr) as a (n_materials, 4) array."""
    n = len(sc.r)
    free = np.ones(n, bool) if free is None else free
    h = sc.h
    lx, lv, lw = gx.astype(np.float64).copy(), gv.astype(np.float64).copy(), gw.astype(np.float64).copy()
    gmat = np.zeros((len(sc.E), 4))
    g_hout_next_ss = None
    g_hout_next_sp = None
    for k in range(len(steps) - 1, -1, -1):
        st = steps[k]
        # integration: x' = x + h v + h^2/2 a, v' = v + h a, w' = w + h alpha
        fm = free[:, None]
        la = np.where(fm, (h * h / 2) * lx + h * lv, 0.0)
        lal = np.where(fm, h * lw, 0.0)
        lF = la / sc.m[:, None]
        lT = lal / sc.inertia[:, None]
        nlx = np.where(fm, lx, 0.0)
        nlv = np.where(fm, lv + h * lx, 0.0)
        nlw = np.where(fm, lw, 0.0)
        F, T, out = forces(sc, st.x, st.v, st.w, st.ss, st.sp, st.hist_ss, st.hist_sp, keep=True)
        g_hin_ss = np.zeros((len(st.ss), 4))
        g_hin_sp = np.zeros((len(st.sp), 4))
        for kind in ("ss", "sp"):
            if kind not in out:
                continue
            hout, geo, I, (Es, Gs, cor, mu, crr, cs, ms, rs, meff, Rs), f, t = out[kind]
            pairs = st.ss if kind == "ss" else st.sp
            A = pairs[:, 0]
            B = pairs[:, 1] if kind == "ss" else None
            u = f + t
            gtA = lT[A]
            g_u = _cross(gtA, geo["rAv"])
            g_rAv_t = _cross(u, gtA)
            g_f = lF[A].copy()
            if kind == "ss":
                gtB = lT[B]
                g_u -= _cross(gtB, geo["rBv"])
                g_rBv_t = -_cross(u, gtB)
                g_f -= lF[B]
            else:
                g_rBv_t = np.zeros_like(g_rAv_t)
            g_f = g_f + g_u
            g_t = g_u
            gnext = g_hout_next_ss if kind == "ss" else g_hout_next_sp
            g_hout = gnext if gnext is not None else np.zeros((len(A), 4))
            hin = st.hist_ss if kind == "ss" else st.hist_sp
            zero = np.zeros((len(A), 3))
            vB = st.v[B] if kind == "ss" else zero
            wB = st.w[B] if kind == "ss" else zero
            gr = contact_law_vjp(geo, I, st.v[A], vB, st.w[A], wB, hin, Es, Gs, beta_of(cor), mu, crr, meff, Rs, h,
                                 g_f, g_t, g_hout)
            g_rAv = gr["rAv"] + g_rAv_t
            g_rBv = gr["rBv"] + g_rBv_t
            np.add.at(nlv, A, gr["vA"])
            np.add.at(nlw, A, gr["wA"])
            if kind == "ss":
                np.add.at(nlv, B, gr["vB"])
                np.add.at(nlw, B, gr["wB"])
                g_d = geometry_ss_vjp(geo, gr["n"], gr["delta"], g_rAv, g_rBv)
                np.add.at(nlx, A, g_d)
                np.add.at(nlx, B, -g_d)
                g_hin_ss = gr["hist"]
                ma, mb = sc.mat[A], sc.mat[B]
            else:
                np.add.at(nlx, A, geometry_sp_vjp(geo, gr["delta"], g_rAv))
                g_hin_sp = gr["hist"]
                ma, mb = sc.mat[A], np.array([sc.planes[j][2] for j in pairs[:, 1]], np.int64)
            # material parameters
            EA, EB = sc.E[ma], sc.E[mb]
            dEs_dEA = Es ** 2 * (1 - sc.nu[ma] ** 2) / EA ** 2
            dEs_dEB = Es ** 2 * (1 - sc.nu[mb] ** 2) / EB ** 2
            dGs_dEA = Gs ** 2 * 2 * (2 - sc.nu[ma]) * (1 + sc.nu[ma]) / EA ** 2
            dGs_dEB = Gs ** 2 * 2 * (2 - sc.nu[mb]) * (1 + sc.nu[mb]) / EB ** 2
            np.add.at(gmat[:, 0], ma, gr["Es"] * dEs_dEA + gr["Gs"] * dGs_dEA)
            np.add.at(gmat[:, 0], mb, gr["Es"] * dEs_dEB + gr["Gs"] * dGs_dEB)
            np.add.at(gmat[:, 1], cs, gr["be"] * dbeta_de(cor))
            np.add.at(gmat[:, 2], ms, gr["mu"])
            np.add.at(gmat[:, 3], rs, gr["crr"])
        # history flows to the previous step's updated histories through the map
        if k > 0:
            prev = steps[k - 1]
            g_hout_next_ss = np.zeros((len(prev.ss), 4))
            g_hout_next_sp = np.zeros((len(prev.sp), 4))
            m_ = st.prev_ss >= 0
            g_hout_next_ss[st.prev_ss[m_]] = g_hin_ss[m_]
            m_ = st.prev_sp >= 0
            g_hout_next_sp[st.prev_sp[m_]] = g_hin_sp[m_]
        lx, lv, lw = nlx, nlv, nlw
    return lx, lv, lw, gmat


def from_built(built, state=None):
    """SphereScene + initial (x, v, w) of a single-sphere scene with plane walls (positions relative to the
    domain's lower corner, as the kernels hold them)."""
    a = built.arrays
    st = built.initial_state() if state is None else state
    nO = built.counts["o"]
    owner = a["sphere_owner"].astype(np.int64)
    n = len(owner)
    assert np.all(owner == np.arange(n)), "one sphere per owner"
    pos = built.decode_positions(st)
    planes = []
    for k in range(built.counts["a"]):
        assert int(a["anal_type"][k]) == 0, "planes only"
        o = int(a["anal_owner"][k])
        bo = pos[o]
        pt = bo + np.array([a["anal_relX"][k], a["anal_relY"][k], a["anal_relZ"][k]], np.float64)
        nr = np.array([a["anal_rotX"][k], a["anal_rotY"][k], a["anal_rotZ"][k]], np.float64)
        planes.append((pt, nr, int(a["anal_material"][k]), bo))
    sc = SphereScene(r=a["radius"].astype(np.float64), m=a["mass"][:n].astype(np.float64),
                     inertia=a["mmiXX"][:n].astype(np.float64), mat=a["sphere_material"].astype(np.int64),
                     planes=planes, E=a["mat_E"].astype(np.float64), nu=a["mat_nu"].astype(np.float64),
                     CoR=a["mat_CoR"].astype(np.float64), mu=a["mat_mu"].astype(np.float64),
                     Crr=a["mat_Crr"].astype(np.float64), h=float(built.params.h),
                     g=np.array(built.params.G[:], np.float64),
                     plane_mass=float(a["mass"][n]) if nO > n else 1e15)
    x0 = pos[:n]
    v0 = np.stack([st["vX"], st["vY"], st["vZ"]], 1)[:n].astype(np.float64)
    w0 = np.stack([st["omgX"], st["omgY"], st["omgZ"]], 1)[:n].astype(np.float64)
    return sc, x0, v0, w0
