"""Bulk statistics of a granular state, for comparing long runs whose individual trajectories diverge (contact
chaos makes two correct solvers part ways after a few hundred steps while the bulk behaviour agrees).

* kinetic energy: translational plus rotational (principal moments in the owner frame, the frame the angular
  velocity is stored in, as the reference's integrator uses it: src/kernel/DEMIntegrationKernels.cu);
* packing fraction: sphere volume inside a horizontal slab of a box, counting the part of each sphere that lies in
  the slab (spherical caps);
* heap angle: slope of the free surface of a heap, from the highest sphere tops in rings around its axis.

All take a state dict as the solvers' ``state()`` returns it and the built scene it belongs to; coordinates are the
world frame of the scene builder.
"""
from __future__ import annotations

import math

import numpy as np


def world_positions(built, state) -> np.ndarray:
    """Owner positions in the world frame (decoded from voxel and sub-voxel position, plus the domain's lower
    corner)."""
    return built.decode_positions(state, kernel_literals=False) + np.asarray(list(built.params.lbf), np.float64)


def _owner_sphere_radius(built) -> np.ndarray:
    """Radius of each single-sphere owner (owners with one sphere centred on them)."""
    a = built.arrays
    owner = np.asarray(a["sphere_owner"], np.int64)
    r = np.zeros(built.counts["o"])
    r[owner] = np.asarray(a["radius"], np.float64)
    return r


def kinetic_energy(built, state) -> float:
    """Translational plus rotational kinetic energy of the clump owners (analytical owners carry no mass here)."""
    a = built.arrays
    n = int(built.info.get("n_clumps", built.counts["o"]))
    m = np.asarray(a["mass"], np.float64)[:n]
    v = np.stack([state["vX"], state["vY"], state["vZ"]], 1).astype(np.float64)[:n]
    w = np.stack([state["omgX"], state["omgY"], state["omgZ"]], 1).astype(np.float64)[:n]
    moi = np.stack([a["mmiXX"], a["mmiYY"], a["mmiZZ"]], 1).astype(np.float64)[:n]
    return float(0.5 * np.sum(m * np.sum(v * v, 1)) + 0.5 * np.sum(moi * w * w))


def _cap_volume(r: np.ndarray, h: np.ndarray) -> np.ndarray:
    """Volume of the part of a sphere of radius r below a plane at height h above its lowest point (0 <= h <= 2r)."""
    h = np.clip(h, 0.0, 2.0 * r)
    return math.pi * h * h * (3.0 * r - h) / 3.0


def packing_fraction(built, state, xy_lo, xy_hi, z_lo: float, z_hi: float) -> float:
    """Solid fraction of the box [xy_lo, xy_hi] x [z_lo, z_hi] (spheres cut by the horizontal faces count in part;
    the vertical faces are taken to be walls that no sphere crosses)."""
    pos = world_positions(built, state)
    r = _owner_sphere_radius(built)[:len(pos)]
    inside = ((pos[:, 0] >= xy_lo[0]) & (pos[:, 0] <= xy_hi[0]) & (pos[:, 1] >= xy_lo[1]) & (pos[:, 1] <= xy_hi[1])
              & (r > 0))
    z, rr = pos[inside, 2], r[inside]
    below_hi = _cap_volume(rr, z_hi - (z - rr))
    below_lo = _cap_volume(rr, z_lo - (z - rr))
    vol = np.sum(below_hi - below_lo)
    return float(vol / ((xy_hi[0] - xy_lo[0]) * (xy_hi[1] - xy_lo[1]) * (z_hi - z_lo)))


def bed_height(built, state, z_floor: float, quantile: float = 0.95) -> float:
    """Height above the floor below which ``quantile`` of the sphere tops lie."""
    pos = world_positions(built, state)
    r = _owner_sphere_radius(built)[:len(pos)]
    ok = r > 0
    return float(np.quantile(pos[ok, 2] + r[ok] - z_floor, quantile))


def heap_profile(built, state, axis_xy, z_floor: float, ring: float, n_rings: int = 40):
    """Free-surface height of a heap: for rings of width ``ring`` around the axis, the 90th percentile of the sphere
    tops in the ring (rings holding fewer than 8 spheres are left out).  Returns (ring centres, heights)."""
    pos = world_positions(built, state)
    r = _owner_sphere_radius(built)[:len(pos)]
    ok = r > 0
    rho = np.hypot(pos[ok, 0] - axis_xy[0], pos[ok, 1] - axis_xy[1])
    top = pos[ok, 2] + r[ok] - z_floor
    k = np.floor(rho / ring).astype(np.int64)
    xs, hs = [], []
    for i in range(n_rings):
        sel = k == i
        if sel.sum() >= 8:
            xs.append((i + 0.5) * ring)
            hs.append(float(np.quantile(top[sel], 0.9)))
    return np.asarray(xs), np.asarray(hs)


def heap_angle(built, state, axis_xy, z_floor: float, ring: float) -> float:
    """Angle of repose in degrees: least-squares slope of the free surface between 20 % and 80 % of the heap's
    height (the flat summit and the thin toe excluded)."""
    xs, hs = heap_profile(built, state, axis_xy, z_floor, ring)
    if len(xs) < 3:
        return float("nan")
    top = hs.max()
    sel = (hs <= 0.8 * top) & (hs >= 0.2 * top)
    if sel.sum() < 3:
        sel = np.ones_like(hs, bool)
    slope = np.polyfit(xs[sel], hs[sel], 1)[0]
    return float(math.degrees(math.atan(-slope)))


def _rotate_f32(q, r):
    """hostApplyOriQToVector3<float> (src/DEM/HostSideHelpers.hpp:384-394) in float32, operation by operation."""
    f = np.float32
    w, x, y, z = (np.asarray(c, f) for c in q)
    rx, ry, rz = (np.asarray(c, f) for c in r)
    two, one = f(2.0), f(1.0)
    X = (two * (w * w + x * x) - one) * rx + (two * (x * y - w * z)) * ry + (two * (x * z + w * y)) * rz
    Y = (two * (x * y + w * z)) * rx + (two * (w * w + y * y) - one) * ry + (two * (y * z - w * x)) * rz
    Z = (two * (x * z - w * y)) * rx + (two * (y * z + w * x)) * ry + (two * (w * w + z * z) - one) * rz
    return X, Y, Z


def inspect(built, state, quantity: str = "clump_max_z", template_volume=None) -> float:
    """The reference's inspectors over the whole domain (DEMInspector, src/DEM/AuxClasses.cpp:14-106;
    inspectSphereProperty, src/kernel/DEMSphereQueryKernels.cu:9-50):

    * "clump_max_z" / "clump_min_z": the largest sphere top / smallest sphere bottom, Z +- r, the sphere centre
      formed as the kernel forms it (owner position in float64 from the voxel code and the kernel literals, the
      relative position rotated in float32, the lower corner added, rounded to float32);
    * "clump_max_absv": the largest speed of a sphere centre, |v + R (omega x relPos)| in float32;
    * "clump_volume": the sum of the clumps' template volumes (``template_volume[i]`` for template i; 0 if not
      given).
    The C++ façade's inspect_quantity computes the same, bit for bit."""
    a = built.arrays
    f = np.float32
    if quantity == "clump_volume":
        tv = np.asarray(template_volume if template_volume is not None else [], f)
        marks = np.asarray(built.info["owner_template"], np.int64)
        vals = np.where(marks < len(tv), tv[np.minimum(marks, max(len(tv) - 1, 0))] if len(tv) else f(0), f(0))
        out = f(0)
        for v in np.asarray(vals, f):  # in owner order, as the façade sums
            out = f(out + v)
        return float(out)
    if quantity not in ("clump_max_z", "clump_min_z", "clump_max_absv"):
        raise ValueError(f"{quantity} is not a known query type.")
    own = np.asarray(a["sphere_owner"], np.int64)
    q = [np.asarray(state[k], f)[own] for k in ("oriQw", "oriQx", "oriQy", "oriQz")]
    rel = [np.asarray(a[k], f) for k in ("relX", "relY", "relZ")]
    rad = np.asarray(a["radius"], f)
    if quantity == "clump_max_absv":
        wx, wy, wz = (np.asarray(state[k], f)[own] for k in ("omgX", "omgY", "omgZ"))
        rx, ry, rz = rel
        X, Y, Z = _rotate_f32(q, (wy * rz - wz * ry, wz * rx - wx * rz, wx * ry - wy * rx))
        vx, vy, vz = (np.asarray(state[k], f)[own] for k in ("vX", "vY", "vZ"))
        sx, sy, sz = X + vx, Y + vy, Z + vz
        return float(np.max(np.sqrt(sx * sx + sy * sy + sz * sz)))
    _, _, dz = _rotate_f32(q, rel)
    oz = built.decode_positions(state, kernel_literals=True)[own, 2]
    Zs = (oz + dz.astype(np.float64) + float(f(built.params.lbf[2]))).astype(f)
    return float(np.max(Zs + rad) if quantity == "clump_max_z" else np.min(Zs - rad))
