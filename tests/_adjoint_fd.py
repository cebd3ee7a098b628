"""Central differences of the FP64 forward with the contact lists held fixed, for checking the CUDA adjoint on
clumps and analytical walls.

A run records, step by step, the contact list its detection found (idA, idB, type; the first step's list with its
incoming histories).  ``oracle.fp64_model.rollout_fixed`` steps the FP64 model over those lists, mapping the
histories from step to step as the reference's history map does.  The loss is linear in the final state:
sum of wx . position + wv . velocity + ww . world angular velocity + wq . quaternion over the owners, so its
gradient with respect to the final state is the weights themselves (the adjoint's seed).  Perturbations of the
initial state follow the adjoint's interface: the world angular velocity is R(q) w, and a quaternion perturbation
holds the world angular velocity fixed (w = R(q)^T w_world).
"""
from __future__ import annotations

import numpy as np

from oracle import fp64_model as M

FIELDS = ("E", "CoR", "mu", "Crr")


def record_lists(sol, T, built=None):
    """T steps of a solver, detection, forces and integration separately, keeping each step's contact list (and,
    given ``built``, the T + 1 states the steps start from and end at, as float64 owner states)."""
    lists, states = [], []
    for _ in range(T):
        if built is not None:
            states.append(initial_state(built, sol.state()))
        sol.detect_contacts()
        c = sol.contacts()
        lists.append({k: np.array(c[k], copy=True) for k in ("idA", "idB", "type", "wildcards")})
        sol.compute_forces()
        sol.integrate()
    if built is None:
        return lists
    states.append(initial_state(built, sol.state()))
    return lists, states


def initial_state(built, st):
    pos, q, v, w, _, _ = M.owner_state(built, st)
    return dict(pos=pos, q=q, v=v, w=w, family=st["family"].astype(np.int64))


def materials(built):
    a = built.arrays
    return {k: a["mat_" + k].astype(np.float64).copy() for k in ("E", "nu", "CoR", "mu", "Crr")}


def weights(nO, free, seed=11, scales=(1.0, 1e-2, 1e-4, 1e-2)):
    """Random loss weights on the free owners (position, velocity, world angular velocity, quaternion)."""
    rng = np.random.default_rng(seed)
    out = []
    for width, sc in zip((3, 3, 3, 4), scales):
        w = np.zeros((nO, width))
        w[free] = rng.normal(size=(int(np.count_nonzero(free)), width)) * sc
        out.append(w)
    return out


def loss(built, S0, lists, wts, mats=None, f32=False, q_anchor=None):
    S, _ = M.rollout_fixed(built, S0, lists, mats=mats, f32=f32, q_anchor=q_anchor)
    wx, wv, ww, wq = wts
    return float(np.sum(wx * S["pos"]) + np.sum(wv * S["v"]) + np.sum(ww * M.rot(S["q"], S["w"])) +
                 np.sum(wq * S["q"]))


def fd_materials(built, S0, lists, wts, rel=1e-6, base=None, f32=False):
    """dL/d(E, CoR, mu, Crr) of every material by central differences at relative step ``rel`` (around the scene's
    materials, or ``base``).  ``f32``: the FP64 forward places spheres and walls as the CUDA path does."""
    anchor = S0["q"] if f32 else None
    base = materials(built) if base is None else base
    nM = len(base["E"])
    out = np.zeros((nM, 4))
    for m in range(nM):
        for j, f in enumerate(FIELDS):
            b = base[f][m]
            if b == 0.0:
                continue
            vals = []
            for sg in (1.0, -1.0):
                mats = {k: v.copy() for k, v in base.items()}
                mats[f][m] = b * (1.0 + sg * rel)
                vals.append(loss(built, S0, lists, wts, mats, f32, anchor))
            out[m, j] = (vals[0] - vals[1]) / (2.0 * rel * b)
    return out


def fd_state(built, S0, lists, wts, owners, eps=(1e-9, 1e-7, 1e-5, 1e-8), mats=None, f32=False):
    """dL/d(position, velocity, world angular velocity, quaternion) of the given owners by central differences
    with steps ``eps`` (m, m/s, rad/s, 1) for the four groups.  ``f32``: the first step places spheres and walls in
    float32 at the initial quaternions plus the float64 change from them (M.step_state's ``q_anchor``), so the
    geometry is the CUDA path's and still differentiable in the quaternions."""
    anchor = S0["q"] if f32 else None
    wW0 = M.rot(S0["q"], S0["w"])
    res = {k: np.zeros((len(owners), n)) for k, n in (("pos", 3), ("vel", 3), ("angvel", 3), ("quat", 4))}
    for i, o in enumerate(owners):
        for key, n, e in (("pos", 3, eps[0]), ("vel", 3, eps[1]), ("angvel", 3, eps[2]), ("quat", 4, eps[3])):
            for j in range(n):
                vals = []
                for sg in (1.0, -1.0):
                    S = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in S0.items()}
                    if key == "pos":
                        S["pos"][o, j] += sg * e
                    elif key == "vel":
                        S["v"][o, j] += sg * e
                    elif key == "angvel":
                        ww = wW0[o].copy()
                        ww[j] += sg * e
                        S["w"][o] = M.rot_t(S["q"][o:o + 1], ww[None])[0]
                    else:
                        S["q"][o, j] += sg * e
                        S["w"][o] = M.rot_t(S["q"][o:o + 1], wW0[o:o + 1])[0]
                    vals.append(loss(built, S, lists, wts, mats, f32, anchor))
                res[key][i, j] = (vals[0] - vals[1]) / (2.0 * e)
    return res
