"""Adjoint of the DEM step through the C ABI (deme_adjoint_record / deme_adjoint_backward / deme_set_material), and a
torch.autograd.Function that makes a window of steps differentiable with respect to the material parameters.

Scope (enforced by the library): clumps (or single spheres) of free families or of families whose linear and
rotational motion are both prescribed, analytical walls (planes, cylinders, cones) of prescribed families, the
built-in Hertz-Mindlin model, Extended Taylor integration, contact detection every step.  Angular velocities are
in the world frame; quaternion gradients (w, x, y, z) hold the world angular velocity fixed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi


class AdjointSeed(C.Structure):
    _fields_ = [("d_pos", C.c_void_p), ("d_vel", C.c_void_p), ("d_angvel", C.c_void_p), ("d_quat", C.c_void_p)]


class AdjointGrads(C.Structure):
    _fields_ = [("d_pos0", C.c_void_p), ("d_vel0", C.c_void_p), ("d_angvel0", C.c_void_p), ("d_material", C.c_void_p),
                ("d_quat0", C.c_void_p)]


def _bind(lib):
    lib.deme_adjoint_record.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    lib.deme_adjoint_record.restype = C.c_int32
    lib.deme_adjoint_backward.argtypes = [C.c_void_p, C.POINTER(AdjointSeed), C.POINTER(AdjointGrads)]
    lib.deme_adjoint_backward.restype = C.c_int32
    lib.deme_set_material.argtypes = [C.c_void_p, C.c_uint32] + [C.c_float] * 5
    lib.deme_set_material.restype = C.c_int32


def set_material(solver, m: int, E: float, nu: float, CoR: float, mu: float, Crr: float):
    _bind(solver.lib)
    solver._check(solver.lib.deme_set_material(solver.h, m, E, nu, CoR, mu, Crr), "set_material")


def record(solver, n_steps: int, checkpoint_every: int):
    """Runs n_steps from the current state, keeping a checkpoint every checkpoint_every steps."""
    _bind(solver.lib)
    solver._check(solver.lib.deme_adjoint_record(solver.h, n_steps, checkpoint_every), "adjoint_record")


def backward(solver, d_pos=None, d_vel=None, d_angvel=None, d_quat=None) -> dict:
    """Gradients of a loss with respect to the window's initial state (world-frame angular velocity; quaternion
    (w, x, y, z) at fixed world angular velocity) and to the materials' (E, CoR, mu, Crr), given its gradient with
    respect to the final state (arrays n_owners x 3, quaternions n_owners x 4)."""
    _bind(solver.lib)
    nO = solver.nO
    nM = solver.built.counts["m"]
    keep = []

    def arr(a, w=3):
        if a is None:
            return None
        a = np.ascontiguousarray(a, np.float64).reshape(nO, w)
        keep.append(a)
        return a.ctypes.data

    seed = AdjointSeed(arr(d_pos), arr(d_vel), arr(d_angvel), arr(d_quat, 4))
    out = {k: np.zeros((nO, 3)) for k in ("d_pos0", "d_vel0", "d_angvel0")}
    out["d_quat0"] = np.zeros((nO, 4))
    out["d_material"] = np.zeros((max(nM, 1), 4))
    g = AdjointGrads(out["d_pos0"].ctypes.data, out["d_vel0"].ctypes.data, out["d_angvel0"].ctypes.data,
                     out["d_material"].ctypes.data, out["d_quat0"].ctypes.data)
    solver._check(solver.lib.deme_adjoint_backward(solver.h, C.byref(seed), C.byref(g)), "adjoint_backward")
    out["d_material"] = out["d_material"][:nM]
    return out


def world_angular_velocity(state: dict) -> np.ndarray:
    """Owner angular velocities rotated from the owner frame to the world frame."""
    w = np.stack([state["omgX"], state["omgY"], state["omgZ"]], 1).astype(np.float64)
    q = np.stack([state["oriQw"], state["oriQx"], state["oriQy"], state["oriQz"]], 1).astype(np.float64)
    u = q[:, 1:]
    t = 2 * np.cross(u, w)
    return w + q[:, :1] * t + np.cross(u, t)


def quaternions(state: dict) -> np.ndarray:
    """Owner quaternions (w, x, y, z) as float64 rows."""
    return np.stack([state["oriQw"], state["oriQx"], state["oriQy"], state["oriQz"]], 1).astype(np.float64)


def final_state(solver):
    st = solver.state()
    pos = solver.built.decode_positions(st, kernel_literals=False)
    vel = np.stack([st["vX"], st["vY"], st["vZ"]], 1).astype(np.float64)
    return pos, vel, world_angular_velocity(st)


def make_rollout_function():
    """torch.autograd.Function: (material parameters (n_materials, 4) = E, CoR, mu, Crr) -> final positions and
    velocities of a window of steps from the solver's current state.  Poisson ratios stay as loaded."""
    import torch

    class DEMRollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, solver, initial_state, nu, n_steps, checkpoint_every):
            p = params.detach().cpu().numpy().astype(np.float64)
            solver.set_state(initial_state)
            for m in range(p.shape[0]):
                set_material(solver, m, float(p[m, 0]), float(nu[m]), float(p[m, 1]), float(p[m, 2]), float(p[m, 3]))
            record(solver, n_steps, checkpoint_every)
            pos, vel, _ = final_state(solver)
            ctx.solver = solver
            return (torch.from_numpy(pos).to(params.device, torch.float64),
                    torch.from_numpy(vel).to(params.device, torch.float64))

        @staticmethod
        def backward(ctx, g_pos, g_vel):
            out = backward(ctx.solver, None if g_pos is None else g_pos.detach().cpu().numpy(),
                           None if g_vel is None else g_vel.detach().cpu().numpy())
            g = torch.from_numpy(out["d_material"]).to(g_pos.device if g_pos is not None else "cpu", torch.float64)
            return g, None, None, None, None, None

    return DEMRollout


def set_floors(solver, overlap_rel: float, roll_speed: float, tangential_force: float):
    """Floors in the derivatives at the contact law's non-smooth points (zeros: exact derivative)."""
    solver.lib.deme_adjoint_set_floors.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
    solver.lib.deme_adjoint_set_floors.restype = C.c_int32
    solver._check(solver.lib.deme_adjoint_set_floors(solver.h, overlap_rel, roll_speed, tangential_force),
                  "adjoint_set_floors")
