"""Seeded synthetic scenes for the benchmark configurations and the parity tests.

Scene sizes and materials follow the benchmark configurations of this project (settling box, rotating drum,
hopper, column collapse).  Geometry that does not fit as literally specified is resized as recorded in the
``info`` of each scene (the design notes give the reasoning).  Generators use numpy's PCG64 with an explicit
seed, so every scene is reproducible bit for bit.
"""
from __future__ import annotations

import math

import numpy as np

from .scene import SceneBuilder

f32 = np.float32


def sphere_mass(r: float, rho: float) -> float:
    return 4.0 / 3.0 * math.pi * r**3 * rho


def random_quaternions(rng, n):
    """Uniform random unit quaternions (Shoemake), rows (w, x, y, z)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    return q[:, [3, 0, 1, 2]].astype(f32)


def settling_box(n: int = 10000, r: float = 5e-3, rho: float = 2600.0, box=(0.2, 0.2, 0.4), spacing: float = 2.2,
                 jitter: float = 0.1, seed: int = 1, dt: float = 1e-5, per_layer: int | None = None,
                 vel_scale: float = 0.0, ang_scale: float = 0.0):
    """Settling box: monodisperse spheres on a jittered cubic lattice inside a box of 6 planes.

    A lattice of spacing 2.2 r holds 18 x 18 sites per layer in a 0.2 m box; 10,000 spheres then need 31 layers
    (0.34 m), so the lattice is filled from the floor up instead of only the lower half.
    """
    rng = np.random.default_rng(seed)
    s = SceneBuilder()
    s.InstructBoxDomainDimension(*box)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.0})
    s.InstructBoxDomainBoundingBC("all", mat)
    m = sphere_mass(r, rho)
    t = s.LoadSphereType(m, r, mat)
    a = spacing * r
    nx = int(box[0] // a) if per_layer is None else per_layer
    ny = int(box[1] // a) if per_layer is None else per_layer
    nz = int(math.ceil(n / (nx * ny)))
    lbf = -np.asarray(box) / 2
    x0 = lbf[0] + (box[0] - nx * a) / 2 + a / 2
    y0 = lbf[1] + (box[1] - ny * a) / 2 + a / 2
    z0 = lbf[2] + a / 2
    idx = np.arange(n)
    pos = np.stack([x0 + (idx % nx) * a, y0 + ((idx // nx) % ny) * a, z0 + (idx // (nx * ny)) * a], axis=1)
    pos += rng.uniform(-jitter * r, jitter * r, size=pos.shape)
    b = s.AddClumps(t, pos.astype(f32))
    if vel_scale:
        b.SetVel(rng.normal(0, vel_scale, size=(n, 3)).astype(f32))
    if ang_scale:
        b.SetAngVel(rng.normal(0, ang_scale, size=(n, 3)).astype(f32))
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetInitBinSize(2.0 * r)
    built = s.Initialize()
    built.info.update(workload="settling_box", n_layers=nz, per_layer=(nx, ny), seed=seed)
    return built


PISTON_VZ = "(t > 1e-4) ? 0.5 * sin(2000.0 * deme::PI * (t - 1e-4)) : 0.0"
SLIDER_X = "0.03 + 2.0 * t"
SPINNER_WZ = "(t < 2e-4) ? 4000.0 * t : 0.8 - 1000.0 * (t - 2e-4)"


def shaker_box(n: int = 500, r: float = 5e-3, rho: float = 2600.0, box=(0.08, 0.08, 0.12), spacing: float = 2.05,
               jitter: float = 0.05, seed: int = 24, dt: float = 1e-5, piston_vz: str = PISTON_VZ,
               slider_x: str = SLIDER_X, spinner_wz: str = SPINNER_WZ):
    """Spheres on a jittered lattice in a box of 6 planes, with three families moved by time expressions (the
    reference's prescribed-motion strings, compiled into the integration kernel at run time):

    * family 1, the lattice's bottom layer: vertical velocity ``piston_vz`` (dictated; the rotation is held);
    * family 2, one sphere of the second layer: X (from the domain's lower corner) follows ``slider_x``, Y and Z
      stay free of prescription but are not integrated (a prescribed position holds the whole pose);
    * family 3, the third layer: angular velocity about z follows ``spinner_wz`` (not dictated: it is added to
      the integrated motion, as the reference does for dictate = false).
    """
    rng = np.random.default_rng(seed)
    s = SceneBuilder()
    s.InstructBoxDomainDimension(*box)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.01})
    s.InstructBoxDomainBoundingBC("all", mat)
    t = s.LoadSphereType(sphere_mass(r, rho), r, mat)
    a = spacing * r
    nx, ny = int(box[0] // a), int(box[1] // a)
    lbf = -np.asarray(box) / 2
    x0 = lbf[0] + (box[0] - nx * a) / 2 + a / 2
    y0 = lbf[1] + (box[1] - ny * a) / 2 + a / 2
    z0 = lbf[2] + a / 2 + 0.2 * r
    idx = np.arange(n)
    layer = idx // (nx * ny)
    pos = np.stack([x0 + (idx % nx) * a, y0 + ((idx // nx) % ny) * a, z0 + layer * a], axis=1)
    pos += rng.uniform(-jitter * r, jitter * r, size=pos.shape)
    fam = np.zeros(n, np.int64)
    fam[layer == 0] = 1
    fam[(layer == 1) & (idx == nx * ny + (nx * ny) // 2)] = 2
    fam[layer == 2] = 3
    b = s.AddClumps(t, pos.astype(f32))
    b.SetVel(rng.normal(0, 0.05, size=(n, 3)).astype(f32))
    b.SetFamilies(fam)
    s.SetFamilyPrescribedLinVel(1, "0", "0", piston_vz)
    s.SetFamilyPrescribedPosition(2, slider_x, "none", "none")
    s.SetFamilyPrescribedAngVel(3, "0", "0", spinner_wz, dictate=False)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetInitBinSize(2.0 * r)
    built = s.Initialize()
    built.info.update(workload="shaker_box", seed=seed)
    return built


def triangle_template(rng, r_nom: float, rho: float, n_mc: int = 20000):
    """Three-sphere triangular clump: radii U[0.8, 1.2] r_nom, centres 0.6 r from the clump centroid.

    Mass, centre of mass and principal moments are integrated by Monte Carlo over the union of the spheres;
    relative positions are re-centred on the centre of mass, and the clump frame is taken as principal
    (the in-plane symmetric layout makes the products of inertia small; they are dropped).
    """
    radii = rng.uniform(0.8, 1.2, 3) * r_nom
    ang = np.array([0.0, 2 * np.pi / 3, 4 * np.pi / 3])
    centers = np.stack([0.6 * radii * np.cos(ang), 0.6 * radii * np.sin(ang), np.zeros(3)], axis=1)
    lo = (centers - radii[:, None]).min(0)
    hi = (centers + radii[:, None]).max(0)
    pts = lo + (hi - lo) * rng.random((n_mc, 3))
    inside = np.zeros(n_mc, bool)
    for c, r in zip(centers, radii):
        inside |= ((pts - c) ** 2).sum(1) <= r * r
    vol = np.prod(hi - lo) * inside.mean()
    p = pts[inside]
    com = p.mean(0)
    d = p - com
    mass = rho * vol
    I = mass * np.array([(d[:, 1] ** 2 + d[:, 2] ** 2).mean(), (d[:, 0] ** 2 + d[:, 2] ** 2).mean(),
                         (d[:, 0] ** 2 + d[:, 1] ** 2).mean()])
    return radii.astype(f32), (centers - com).astype(f32), float(mass), I.astype(f32), float(vol)


def drum(n_clumps: int = 1_000_000, r_nom: float = 2e-3, rho: float = 2500.0, n_templates: int = 64,
         fill: float = 0.30, packing: float = 0.6, rpm: float = 20.0, dt: float = 5e-6, seed: int = 2,
         shell: bool = False, spacing: float = 1.02, wall_clearance: float = 1.05, mesh: bool = False):
    """Rotating drum of three-sphere clumps (analytical cylinder + two end planes, prescribed rotation).

    One million clumps of about 8e-8 m^3 do not fit a 30 % fill of an R = 0.25 m, L = 0.3 m drum, so the drum is
    scaled (same L / R ratio) until the clumps at ``packing`` bulk density fill ``fill`` of its volume.
    Clumps start on a loose lattice in the lower part of the drum with random orientations.  ``spacing`` is the
    lattice pitch over the clump's bounding diameter: above 1 no two clumps touch; below 1 neighbouring clumps
    interpenetrate, which gives a dense bed without settling (used to size CPU samples).  Lattice sites stay
    ``wall_clearance`` clump reaches inside the walls; below 1 the outer clumps start in contact with them.

    ``shell=True`` builds the variant the reference can express, which has only planes and plates as analytical
    components. The cylinder becomes a shell of fixed spheres of radius ``r_nom``, centred one radius outside R on
    a square lattice of pitch 1.9 ``r_nom``, so that no bed sphere fits through. The shell does not rotate. The two
    end planes and the shell form one fixed family with contacts inside it disabled.

    ``mesh=True`` makes the cylinder a mesh body turning with the end planes: a prism of flat facets whose planes
    touch the radius-R circle (so the lattice start is the same), enough of them around that a facet's sagitta is
    at most 0.05 ``r_nom``, split along the axis into near-square quads of two triangles, mass 1e15 as the
    analytical walls'.
    """
    rng = np.random.default_rng(seed)
    tmpl = [triangle_template(rng, r_nom, rho) for _ in range(n_templates)]
    vol_clump = float(np.mean([t[4] for t in tmpl]))
    bulk = n_clumps * vol_clump / packing
    # drum volume V = pi R^2 L with L = 1.2 R
    R = (bulk / fill / (math.pi * 1.2)) ** (1.0 / 3.0)
    L = 1.2 * R
    s = SceneBuilder()
    margin = 4 * r_nom
    # cubic domain, as in the reference's drum demo: the reference's voxel bit split overshoots 64 bits when the
    # two smaller sides differ by more than sqrt(2)
    side = 2 * R + 2 * margin
    box = (side, side, side)
    s.InstructBoxDomainDimension(*box)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 5e7, "nu": 0.3, "CoR": 0.3, "mu": 0.4, "Crr": 0.02})
    ts = [s.LoadClumpType(t[2], t[3], t[0], t[1], mat) for t in tmpl]
    # Clump centres on a hexagonal close-packed lattice of non-overlapping bounding spheres (the reference's drum
    # demo likewise starts from a grid sampler with spacing above the clump size), filled from the bottom of the
    # drum; the bed settles under gravity before measurements (bench.py).
    reach = float(max(np.max(np.linalg.norm(t[1], axis=1) + t[0]) for t in tmpl))
    a = 2.0 * reach * spacing
    dy, dz = a * math.sqrt(3.0) / 2.0, a * math.sqrt(2.0 / 3.0)
    nx, ny, nz = int(2 * R / a) + 2, int(L / dy) + 2, int(2 * R / dz) + 2
    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    px = -R + I * a + np.where((J + K) % 2 == 0, 0.0, a / 2)
    py = -L / 2 + J * dy + np.where(K % 2 == 0, 0.0, dy / 3)
    pz = -R + K * dz
    P = np.stack([px.ravel(), py.ravel(), pz.ravel()], axis=1)
    c = reach * wall_clearance
    inside = (P[:, 0] ** 2 + P[:, 2] ** 2 <= (R - c) ** 2) & (np.abs(P[:, 1]) <= L / 2 - c)
    P = P[inside]
    P = P[np.argsort(P[:, 2], kind="stable")]
    if len(P) < n_clumps:
        raise ValueError(f"lattice holds {len(P)} clumps, {n_clumps} requested")
    P = P[:n_clumps]
    types = rng.integers(0, n_templates, n_clumps)
    b = s.AddClumps(types, P.astype(f32))
    b.SetOriQ(random_quaternions(rng, n_clumps))
    drum_fam = 10
    if shell:
        pitch = 1.9 * r_nom
        Rc = R + r_nom
        n_ring = int(2 * math.pi * Rc / pitch)
        n_axial = int(L / pitch) + 1
        th = 2 * math.pi * np.arange(n_ring) / n_ring
        ys = -L / 2 + (np.arange(n_axial) + 0.5) * (L / n_axial)
        TH, Y = np.meshgrid(th, ys, indexing="ij")
        S = np.stack([Rc * np.cos(TH).ravel(), Y.ravel(), Rc * np.sin(TH).ravel()], 1)
        shell_t = s.LoadSphereType(sphere_mass(r_nom, rho), r_nom, mat)
        sb = s.AddClumps([shell_t] * len(S), S.astype(f32))
        sb.SetFamily(drum_fam)
        d = s.AddExternalObject()
        d.AddPlane((0, -L / 2, 0), (0, 1, 0), mat)
        d.AddPlane((0, L / 2, 0), (0, -1, 0), mat)
        d.SetFamily(drum_fam)
        s.SetFamilyFixed(drum_fam)
        s.DisableContactBetweenFamilies(drum_fam, drum_fam)
        s.SetInitTimeStep(dt)
        s.SetGravitationalAcceleration((0, 0, -9.81))
        built = s.Initialize()
        built.info.update(workload="drum_shell", R=R, L=L, n_templates=n_templates, seed=seed, vol_clump=vol_clump,
                          n_clumps=n_clumps, n_shell=len(S), lattice_spacing=a, clump_reach=reach)
        return built
    d = s.AddExternalObject()
    n_tris = 0
    if mesh:
        n_around = max(64, int(math.ceil(math.pi / math.sqrt(2 * 0.05 * r_nom / R))))
        Rv = R / math.cos(math.pi / n_around)  # vertices outside R: the facets' planes touch the circle
        n_axial = max(1, int(math.ceil(L / (2 * math.pi * Rv / n_around))))
        th = 2 * math.pi * np.arange(n_around + 1) / n_around
        ys = -L / 2 + L * np.arange(n_axial + 1) / n_axial
        tris = []
        for i in range(n_around):
            for j in range(n_axial):
                p = [(Rv * math.cos(th[a]), ys[b], Rv * math.sin(th[a])) for a, b in
                     ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1))]
                tris += [(p[0], p[1], p[2]), (p[0], p[2], p[3])]
        v, fc = _mesh_arrays(tris)
        cyl = s.AddWavefrontMeshObject((v, fc), mat)
        cyl.SetMass(1e15)
        cyl.SetMOI((1e15, 1e15, 1e15))
        cyl.SetFamily(drum_fam)
        n_tris = len(fc)
    else:
        d.AddCylinder((0, 0, 0), (0, 1, 0), R, mat)
    d.AddPlane((0, -L / 2, 0), (0, 1, 0), mat)
    d.AddPlane((0, L / 2, 0), (0, -1, 0), mat)
    d.SetFamily(drum_fam)
    omega = rpm * 2 * math.pi / 60.0
    s.SetFamilyPrescribedLinVel(drum_fam, "0", "0", "0")
    s.SetFamilyPrescribedAngVel(drum_fam, "0", repr(float(f32(omega))), "0")
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    built = s.Initialize()
    built.info.update(workload="drum_mesh" if mesh else "drum", R=R, L=L, n_templates=n_templates, omega=omega,
                      seed=seed, vol_clump=vol_clump, n_clumps=n_clumps, lattice_spacing=a, clump_reach=reach,
                      n_tris=n_tris)
    return built


def packed_clumps(n_clumps: int = 600, r: float = 4e-3, spacing: float = 1.55, seed: int = 3, three: bool = True,
                  vel_scale: float = 0.05, ang_scale: float = 5.0, dt: float = 1e-5, beta: float = 0.0,
                  families: bool = False):
    """Small dense scene for parity tests: overlapping clumps with random poses, velocities and spin, in a box of
    planes, so that one step exercises every branch of the force model."""
    rng = np.random.default_rng(seed)
    s = SceneBuilder()
    side = (n_clumps ** (1 / 3) + 1) * spacing * 2 * r
    s.InstructBoxDomainDimension(side, side, side)
    s.SetCoordSysOrigin("center")
    mA = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.05})
    mB = s.LoadMaterial({"E": 5e7, "nu": 0.25, "CoR": 0.3, "mu": 0.4, "Crr": 0.0})
    s.InstructBoxDomainBoundingBC("all", mB)
    tmpls = []
    for k in range(4):
        if three:
            radii = rng.uniform(0.8, 1.2, 3) * r
            ang = np.array([0, 2 * np.pi / 3, 4 * np.pi / 3]) + k
            rel = np.stack([0.6 * radii * np.cos(ang), 0.6 * radii * np.sin(ang), np.zeros(3)], 1)
            m = sphere_mass(r, 2500) * 2.4
            tmpls.append(s.LoadClumpType(m, (m * r * r * 0.5, m * r * r * 0.55, m * r * r * 0.6), radii, rel,
                                         [mA, mB, mA]))
        else:
            rr = r * (0.9 + 0.05 * k)
            tmpls.append(s.LoadSphereType(sphere_mass(rr, 2500), rr, [mA, mB][k % 2]))
    n_side = int(math.ceil(n_clumps ** (1 / 3)))
    a = spacing * 2 * r * (1.0 if three else 0.62)
    g = np.arange(n_side) * a
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)[:n_clumps]
    P = P - P.mean(0) + rng.uniform(-0.15 * r, 0.15 * r, size=P.shape)
    types = rng.integers(0, 4, n_clumps)
    b = s.AddClumps(types, P.astype(f32))
    b.SetOriQ(random_quaternions(rng, n_clumps))
    b.SetVel(rng.normal(0, vel_scale, (n_clumps, 3)).astype(f32))
    b.SetAngVel(rng.normal(0, ang_scale, (n_clumps, 3)).astype(f32))
    if families:
        fam = rng.integers(0, 3, n_clumps)
        b.SetFamilies(fam)
        s.DisableContactBetweenFamilies(1, 2)
        s.SetFamilyPrescribedLinVel(2, "0", "0", "-0.01")
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    if beta:
        s.SetExpandFactor(beta)
    built = s.Initialize()
    built.info.update(workload="packed_clumps", seed=seed)
    return built


# Family the hopper's outlet gate (family 2) moves to when it opens: fixed, and with no contact with the spheres
# (family 0), as the reference's scripts open a gate with ChangeFamily + DisableContactBetweenFamilies.
GATE_OPEN_FAMILY = 3


def _hopper_radii(n, r_median, sigma, r_clip, n_classes, rng):
    r = np.clip(rng.lognormal(math.log(r_median), sigma, n), r_clip[0], r_clip[1])
    edges = np.quantile(r, np.linspace(0, 1, n_classes + 1))
    cls = np.clip(np.searchsorted(edges, r, side="right") - 1, 0, n_classes - 1)
    r_cls = np.array([r[cls == c].mean() if np.any(cls == c) else edges[c] for c in range(n_classes)])
    return r_cls[cls], r_cls, cls


def _hopper_top(n, a, r_max, tan_t, cos_t, u_out, wall_clearance):
    """Height of the cone that holds n lattice sites of pitch a above the outlet, and the sites."""
    dy, dz = a * math.sqrt(3.0) / 2.0, a * math.sqrt(2.0 / 3.0)
    u_top = u_out + 10 * a
    while True:
        R_top = u_top * tan_t
        nx, ny, nz = int(2 * R_top / a) + 2, int(2 * R_top / dy) + 2, int((u_top - u_out) / dz) + 2
        K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        px = -R_top + I * a + np.where((J + K) % 2 == 0, 0.0, a / 2)
        py = -R_top + J * dy + np.where(K % 2 == 0, 0.0, dy / 3)
        pz = u_out + r_max + K * dz
        P = np.stack([px.ravel(), py.ravel(), pz.ravel()], axis=1)
        rho_ = np.hypot(P[:, 0], P[:, 1])
        clear = wall_clearance * r_max / cos_t
        ok = (rho_ <= P[:, 2] * tan_t - clear) & (P[:, 2] <= u_top - r_max)
        if ok.sum() >= n:
            return u_top, P[ok]
        u_top *= 1.15


def hopper(n: int = 4_000_000, r_median: float = 1.5e-3, sigma: float = 0.25, r_clip=(0.75e-3, 3e-3),
           rho: float = 2500.0, half_angle_deg: float = 30.0, outlet: float = 0.04, n_classes: int = 64,
           seed: int = 4, dt: float = 2e-6, cd_freq: int = 5, margin: float | None = None, closed: bool = True,
           wall_clearance: float = 1.02, packing_seed_jitter: float = 0.9, mesh: bool = False):
    """Conical hopper of log-normal polydisperse spheres (analytical cone + outlet gate + catch floor).

    Radii are log-normal (median ``r_median``, ``sigma``) clipped to ``r_clip`` and grouped into ``n_classes``
    sphere types (one template per class, as a reference scene would load them).  Spheres start on a
    hexagonal lattice of pitch 2 r_max filling the cone from the outlet up, each displaced randomly inside its own
    lattice cell (no overlaps): a seeded random packing that needs no insertion loop.  The hopper height follows
    from n.  The gate (family 2) closes the outlet while ``closed``; changing its family to ``GATE_OPEN_FAMILY``
    (deme_change_family / ChangeFamily) opens it.  The floor 0.1 m below catches discharge.
    Contact detection runs every ``cd_freq`` steps with the contact margin ``margin`` (default 0.1 r_median).
    ``wall_clearance`` below 1 starts the outer spheres pressed into the walls (used by parity tests).
    ``mesh=True`` makes the cone a fixed mesh body: a pyramid frustum of flat facets whose planes touch the cone
    along their middle lines, enough of them around that a facet's sagitta at the top is at most 0.05 ``r_median``,
    split along the slant into near-square quads of two triangles.
    """
    rng = np.random.default_rng(seed)
    th = math.radians(half_angle_deg)
    tan_t, cos_t = math.tan(th), math.cos(th)
    r, r_cls, cls = _hopper_radii(n, r_median, sigma, r_clip, n_classes, rng)
    r_max = float(r.max())
    a = 2.0 * r_max * 1.01
    u_out = (outlet / 2) / tan_t  # axial distance from the apex to the outlet
    u_top, P = _hopper_top(n, a, r_max, tan_t, cos_t, u_out, wall_clearance)
    P = P[np.argsort(P[:, 2], kind="stable")][:n]
    # random displacement inside each lattice cell, bounded so that no two spheres overlap
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    d *= (rng.random(n) * packing_seed_jitter * np.maximum(a / 2 - r, 0.0))[:, None]
    P = P + d
    z_floor = -0.1
    s = SceneBuilder()
    side = 2 * (u_top * tan_t) + 8 * r_max
    height = u_top - z_floor + 8 * r_max
    box = max(side, height)
    s.InstructBoxDomainDimension(box, box, box)
    # place the apex so that the floor sits 4 r_max above the domain's bottom face
    s.SetCoordSysOrigin("center")
    shift = -box / 2 + 4 * r_max - z_floor
    mat = s.LoadMaterial({"E": 1e8, "nu": 0.3, "CoR": 0.4, "mu": 0.5, "Crr": 0.0})
    types = [s.LoadSphereType(sphere_mass(float(rc), rho), float(rc), mat) for rc in r_cls]
    pos = P + np.array([0.0, 0.0, shift])
    b = s.AddClumps([types[c] for c in cls], pos.astype(f32))
    b.SetFamily(0)
    if mesh:
        r_top = u_top * tan_t
        n_around = max(64, int(math.ceil(math.pi / math.sqrt(2 * 0.05 * r_median / r_top))))
        kv = 1.0 / math.cos(math.pi / n_around)  # vertices outside the cone: the facets' planes touch it
        slant = (u_top - u_out) / cos_t
        n_axial = max(1, int(math.ceil(slant / (2 * math.pi * kv * 0.5 * (u_out + u_top) * tan_t / n_around))))
        ph = 2 * math.pi * np.arange(n_around + 1) / n_around
        us = u_out + (u_top - u_out) * np.arange(n_axial + 1) / n_axial
        tris = []
        for i in range(n_around):
            for j in range(n_axial):
                p = [(kv * us[b] * tan_t * math.cos(ph[a]), kv * us[b] * tan_t * math.sin(ph[a]), shift + us[b])
                     for a, b in ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1))]
                tris += [(p[0], p[1], p[2]), (p[0], p[2], p[3])]
        v, fc = _mesh_arrays(tris)
        cone = s.AddWavefrontMeshObject((v, fc), mat)
        cone.SetMass(1e15)
        cone.SetMOI((1e15, 1e15, 1e15))
        cone.SetFamily(1)
    else:
        wall = s.AddExternalObject()
        wall.AddCone((0.0, 0.0, shift), (0.0, 0.0, 1.0), th, u_out, u_top, mat)
        wall.SetFamily(1)
    floor = s.AddBCPlane((0.0, 0.0, shift + z_floor), (0.0, 0.0, 1.0), mat)
    floor.SetFamily(1)
    if closed:
        gate = s.AddBCPlane((0.0, 0.0, shift + u_out), (0.0, 0.0, 1.0), mat)
        gate.SetFamily(2)
        s.SetFamilyFixed(2)
        s.SetFamilyFixed(GATE_OPEN_FAMILY)
        s.DisableContactBetweenFamilies(0, GATE_OPEN_FAMILY)
    s.SetFamilyFixed(1)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(cd_freq)
    s.SetExpandFactor(0.1 * r_median if margin is None else margin)
    s.SetInitBinSize(2.0 * float(r.min()))
    built = s.Initialize()
    built.info.update(workload="hopper", n=n, u_out=u_out, u_top=u_top, R_top=u_top * tan_t, r_max=r_max,
                      lattice_spacing=a, seed=seed, n_classes=n_classes, apex_z=shift,
                      volume=math.pi * tan_t ** 2 * (u_top ** 3 - u_out ** 3) / 3.0)
    return built


def hopper_wedge(n: int = 4_000_000, r_median: float = 1.5e-3, sigma: float = 0.25, r_clip=(0.75e-3, 3e-3),
                 rho: float = 2500.0, half_angle_deg: float = 30.0, outlet: float = 0.04, n_classes: int = 64,
                 seed: int = 4, dt: float = 2e-6, cd_freq: int = 5, margin: float | None = None,
                 packing_seed_jitter: float = 0.9):
    """The hopper as the reference can express it, with planes only: a wedge (V-shaped trough) whose two walls lean
    ``half_angle_deg`` from the vertical, closed by two end planes, with an outlet slot ``outlet`` wide under a gate
    plane and a catch floor 0.1 m below.  Its length makes its volume between the outlet and the top equal to the
    conical hopper's for the same n; the same log-normal spheres start on the same kind of lattice.  Used to time
    the reference's own kernels on the polydisperse hopper workload, since the cone has no counterpart there."""
    rng = np.random.default_rng(seed)
    th = math.radians(half_angle_deg)
    tan_t, cos_t = math.tan(th), math.cos(th)
    r, r_cls, cls = _hopper_radii(n, r_median, sigma, r_clip, n_classes, rng)
    r_max = float(r.max())
    a = 2.0 * r_max * 1.01
    u_out = (outlet / 2) / tan_t
    u_top, _ = _hopper_top(n, a, r_max, tan_t, cos_t, u_out, 1.02)
    volume = math.pi * tan_t ** 2 * (u_top ** 3 - u_out ** 3) / 3.0
    L = volume / (tan_t * (u_top ** 2 - u_out ** 2))  # trough cross-section between outlet and top, times L
    dy, dz = a * math.sqrt(3.0) / 2.0, a * math.sqrt(2.0 / 3.0)
    while True:
        X_top = u_top * tan_t
        nx, ny, nz = int(2 * X_top / a) + 2, int(L / dy) + 2, int((u_top - u_out) / dz) + 2
        K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        px = -X_top + I * a + np.where((J + K) % 2 == 0, 0.0, a / 2)
        py = -L / 2 + r_max * 1.02 + J * dy + np.where(K % 2 == 0, 0.0, dy / 3)
        pz = u_out + r_max + K * dz
        P = np.stack([px.ravel(), py.ravel(), pz.ravel()], axis=1)
        clear = 1.02 * r_max / cos_t
        ok = ((np.abs(P[:, 0]) <= P[:, 2] * tan_t - clear) & (P[:, 2] <= u_top - r_max)
              & (np.abs(P[:, 1]) <= L / 2 - 1.02 * r_max))
        if ok.sum() >= n:
            break
        L *= 1.05
    P = P[ok]
    P = P[np.argsort(P[:, 2], kind="stable")][:n]
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    d *= (rng.random(n) * packing_seed_jitter * np.maximum(a / 2 - r, 0.0))[:, None]
    P = P + d
    z_floor = -0.1
    s = SceneBuilder()
    side = max(2 * u_top * tan_t, L) + 8 * r_max
    height = u_top - z_floor + 8 * r_max
    box = max(side, height)
    s.InstructBoxDomainDimension(box, box, box)
    s.SetCoordSysOrigin("center")
    shift = -box / 2 + 4 * r_max - z_floor
    mat = s.LoadMaterial({"E": 1e8, "nu": 0.3, "CoR": 0.4, "mu": 0.5, "Crr": 0.0})
    types = [s.LoadSphereType(sphere_mass(float(rc), rho), float(rc), mat) for rc in r_cls]
    b = s.AddClumps([types[c] for c in cls], (P + np.array([0.0, 0.0, shift])).astype(f32))
    b.SetFamily(0)
    walls = s.AddExternalObject()
    apex = (0.0, 0.0, shift)
    walls.AddPlane(apex, (cos_t, 0.0, math.sin(th)), mat)   # x >= -z tan(theta)
    walls.AddPlane(apex, (-cos_t, 0.0, math.sin(th)), mat)  # x <= z tan(theta)
    walls.AddPlane((0.0, -L / 2, shift), (0.0, 1.0, 0.0), mat)
    walls.AddPlane((0.0, L / 2, shift), (0.0, -1.0, 0.0), mat)
    walls.AddPlane((0.0, 0.0, shift + z_floor), (0.0, 0.0, 1.0), mat)
    walls.SetFamily(1)
    gate = s.AddBCPlane((0.0, 0.0, shift + u_out), (0.0, 0.0, 1.0), mat)
    gate.SetFamily(2)
    s.SetFamilyFixed(1)
    s.SetFamilyFixed(2)
    s.SetFamilyFixed(GATE_OPEN_FAMILY)
    s.DisableContactBetweenFamilies(0, GATE_OPEN_FAMILY)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(cd_freq)
    s.SetExpandFactor(0.1 * r_median if margin is None else margin)
    s.SetInitBinSize(2.0 * float(r.min()))
    built = s.Initialize()
    built.info.update(workload="hopper_wedge", n=n, u_out=u_out, u_top=u_top, L=L, r_max=r_max, lattice_spacing=a,
                      seed=seed, n_classes=n_classes, apex_z=shift,
                      volume=L * tan_t * (u_top ** 2 - u_out ** 2), cone_volume=volume)
    return built


def sphere_pile(n: int = 60, seed: int = 3, h: float = 2e-5, spread: float = 5.2e-3, noise: float = 4e-4,
                vel_scale: float = 0.05, spin_scale: float = 20.0, lift: float = 2.2e-3, mesh_floor: bool = False,
                frictionless: bool = False):
    """Loose pile of single spheres (radii U[2, 3] mm, two materials) pressed onto a floor plane with random
    velocities and spins: every contact branch of the Hertz-Mindlin model is active within a few dozen steps.
    Used by the adjoint tests.  ``mesh_floor``: the floor is a mesh body of two facets 0.19 m wide in the same
    plane instead of an analytical plane.  ``frictionless``: the frictionless Hertzian model
    (UseFrictionlessHertzianModel) instead of the full one."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(2e-3, 3e-3, n).astype(f32)
    rho = 2500.0
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    m0 = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.01})
    m1 = s.LoadMaterial({"E": 5e7, "nu": 0.25, "CoR": 0.4, "mu": 0.5, "Crr": 0.03})
    side = int(np.ceil(n ** (1 / 3)))
    idx = np.arange(n)
    z0 = -0.05
    x = np.stack([(idx % side) * spread, ((idx // side) % side) * spread, z0 + (idx // side // side) * spread + lift],
                 1)
    x += rng.normal(0, noise, x.shape)
    types = [s.LoadSphereType(float(f32(sphere_mass(float(ri), rho))), float(ri), m0 if i % 2 == 0 else m1)
             for i, ri in enumerate(r)]
    b = s.AddClumps(types, x.astype(f32))
    b.SetVel(rng.normal(0, vel_scale, (n, 3)).astype(f32))
    b.SetAngVel(rng.normal(0, spin_scale, (n, 3)).astype(f32))
    if mesh_floor:
        w = 0.095
        v = np.array([[-w, -w, z0], [w, -w, z0], [w, w, z0], [-w, w, z0]], f32)
        floor = s.AddWavefrontMeshObject((v, np.array([[0, 1, 2], [0, 2, 3]])), m1)
        floor.SetMass(1e15)  # as an analytical owner's (the mass enters the contacts' effective mass)
    else:
        s.AddBCPlane((0, 0, z0), (0, 0, 1), m1)
    s.SetInitTimeStep(h)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)  # contacts are exactly the overlapping pairs (the unset default would shrink them)
    if frictionless:
        s.UseFrictionlessHertzianModel()
    built = s.Initialize()
    built.info.update(workload="sphere_pile", n=n, seed=seed, mesh_floor=mesh_floor, frictionless=frictionless)
    return built


def column_collapse(n: int = 20000, r_range=(2e-3, 3e-3), rho: float = 2500.0, n_classes: int = 32, seed: int = 6,
                    dt: float = 1e-5, aspect: float = 3.0, domain_widths: float = 4.0, mu: float = 0.5,
                    Crr: float = 0.02):
    """Column collapse for the adjoint: n single spheres (radii uniform in r_range, grouped into n_classes sphere
    types) on a jittered square lattice of pitch 2 r_max (no overlaps) forming a column height:width = aspect over
    a floor plane, released from rest.  20,000 spheres of 2-3 mm do not fit the stated 0.05 x 0.05 x 0.15 m column,
    so the cross-section is widened (recorded in ``info``).  Contact margin 0, contact detection every step.  The
    cubic domain spans ``domain_widths`` column widths (or 1.3 column heights); a run long enough for the heap to
    spread needs more than the default 4, since spheres that leave the domain are lost."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(r_range[0], r_range[1], n)
    edges = np.linspace(r_range[0], r_range[1], n_classes + 1)
    cls = np.clip(np.searchsorted(edges, r, side="right") - 1, 0, n_classes - 1)
    r_cls = 0.5 * (edges[:-1] + edges[1:])
    r_max = float(r_cls.max())
    a = 2.0 * r_max * 1.01
    per_side = int(math.ceil((n / aspect) ** (1.0 / 3.0)))
    layers = int(math.ceil(n / (per_side * per_side)))
    idx = np.arange(n)
    w = per_side * a
    P = np.stack([(idx % per_side) * a - w / 2 + a / 2, ((idx // per_side) % per_side) * a - w / 2 + a / 2,
                  (idx // (per_side * per_side)) * a + r_max * 1.01], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    d *= (rng.random(n) * 0.9 * np.maximum(a / 2 - r_cls[cls], 0.0))[:, None]
    P += d
    height = layers * a
    s = SceneBuilder()
    box = max(domain_widths * w, 1.3 * height) + 0.05
    s.InstructBoxDomainDimension(box, box, box)
    s.SetCoordSysOrigin("center")
    z_floor = -box / 2 + 0.02
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": mu, "Crr": Crr})
    types = [s.LoadSphereType(float(f32(sphere_mass(float(rc), rho))), float(rc), mat) for rc in r_cls]
    s.AddClumps([types[c] for c in cls], (P + np.array([0.0, 0.0, z_floor])).astype(f32))
    s.AddBCPlane((0, 0, z_floor), (0, 0, 1), mat)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)
    built = s.Initialize()
    built.info.update(workload="column_collapse", n=n, width=w, height=height, layers=layers, per_side=per_side,
                      lattice_spacing=a, z_floor=z_floor, seed=seed)
    return built


def collapse_loss(pos: np.ndarray, axis_xy, z0: float):
    """Column-collapse loss on final positions (n x 3): mean squared horizontal runout from the column axis
    (axis_xy) plus a heap-angle proxy, the mean height above the floor z0 over the RMS runout.  Returns the loss and
    its gradient with respect to pos."""
    dx = pos[:, 0] - axis_xy[0]
    dy = pos[:, 1] - axis_xy[1]
    dz = pos[:, 2] - z0
    n = len(pos)
    R2 = np.mean(dx * dx + dy * dy)
    Rrms = math.sqrt(R2)
    H = np.mean(dz)
    loss = R2 + H / Rrms
    g = np.zeros_like(pos)
    dR2 = np.stack([2 * dx / n, 2 * dy / n, np.zeros(n)], 1)
    g += dR2 * (1.0 - 0.5 * H / (Rrms ** 3))
    g[:, 2] += 1.0 / (n * Rrms)
    return float(loss), g


def batch_scene_specs(n_scenes: int = 512, seed: int = 5, n_range=(500, 20000), r_range=(2e-3, 5e-3),
                      side_range=(0.05, 0.2), mu_range=(0.2, 0.8), cor_range=(0.2, 0.8), packing: float = 0.5):
    """Per-scene parameters of the batched calibration sweep: sphere count log-uniform in n_range, radius uniform
    in r_range, box side uniform in side_range (enlarged where the spheres would exceed packing), friction and
    restitution uniform in their ranges."""
    rng = np.random.default_rng(seed)
    N = np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), n_scenes)).astype(np.int64)
    r = rng.uniform(*r_range, n_scenes)
    side = rng.uniform(*side_range, n_scenes)
    need = (N * (4.0 / 3.0) * np.pi * r ** 3 / packing) ** (1.0 / 3.0)
    side = np.maximum(side, need)
    return [dict(n=int(N[i]), r=float(r[i]), side=float(side[i]), mu=float(rng.uniform(*mu_range)),
                 CoR=float(rng.uniform(*cor_range)), seed=int(seed * 100003 + i)) for i in range(n_scenes)]


def _settling_positions(spec, lbf):
    """Jittered cubic lattice (pitch 2.2 r, jitter 0.1 r) filling the scene's square box from the floor up."""
    rng = np.random.default_rng(spec["seed"])
    r, n, side = spec["r"], spec["n"], spec["side"]
    a = spec.get("pitch", 2.2) * r
    per = max(int(side // a), 1)
    idx = np.arange(n)
    pos = np.stack([lbf[0] + (side - per * a) / 2 + a / 2 + (idx % per) * a,
                    lbf[1] + (side - per * a) / 2 + a / 2 + ((idx // per) % per) * a,
                    lbf[2] + spec.get("lift", 1.1) * r + (idx // (per * per)) * a], 1)
    pos += rng.uniform(-0.1 * r, 0.1 * r, pos.shape)
    height = (int(np.ceil(n / (per * per))) + 1) * a
    return pos, height


def _add_settling_scene(s, spec, lbf, rho=2500.0):
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": spec["CoR"], "mu": spec["mu"], "Crr": 0.0})
    t = s.LoadSphereType(float(f32(sphere_mass(spec["r"], rho))), spec["r"], mat)
    pos, height = _settling_positions(spec, lbf)
    b = s.AddClumps(t, pos.astype(f32))
    box = s.AddExternalObject()
    side = spec["side"]
    X, Y, Z = lbf
    H = max(height, side)
    box.AddPlane((X + side / 2, Y + side / 2, Z), (0, 0, 1), mat)
    box.AddPlane((X, Y + side / 2, Z + H / 2), (1, 0, 0), mat)
    box.AddPlane((X + side, Y + side / 2, Z + H / 2), (-1, 0, 0), mat)
    box.AddPlane((X + side / 2, Y, Z + H / 2), (0, 1, 0), mat)
    box.AddPlane((X + side / 2, Y + side, Z + H / 2), (0, -1, 0), mat)
    box.AddPlane((X + side / 2, Y + side / 2, Z + H), (0, 0, -1), mat)
    return b, box, H


def batched_settling(specs, dt: float = 1e-5):
    """The scenes of ``specs`` packed into one: each in its own slot of a cubic grid of slots, with its own walls
    (six planes) and material; each scene's spheres meet only its own walls.  Scenes never interact (slots are
    separated by more than a contact reach).  ``info['scenes']`` maps each scene to its sphere range."""
    heights = [max(_settling_positions(sp, (0.0, 0.0, 0.0))[1], sp["side"]) for sp in specs]
    slot = max(max(sp["side"] for sp in specs), max(heights)) + 4 * max(sp["r"] for sp in specs) + 0.01
    per = int(np.ceil(len(specs) ** (1.0 / 3.0)))
    s = SceneBuilder()
    world = per * slot + 0.02
    s.InstructBoxDomainDimension(world, world, world)
    s.SetCoordSysOrigin("explicit")  # lower corner at the origin
    ranges = []
    first = 0
    for i, sp in enumerate(specs):
        lbf = (0.01 + (i % per) * slot, 0.01 + ((i // per) % per) * slot, 0.01 + (i // (per * per)) * slot)
        b, box, H = _add_settling_scene(s, sp, lbf)
        b.SetAnalyticalObjects([box])
        b.SetSceneBox(lbf, (lbf[0] + sp["side"], lbf[1] + sp["side"], lbf[2] + H))
        ranges.append((first, sp["n"]))
        first += sp["n"]
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetInitBinSize(2.0 * max(sp["r"] for sp in specs))
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)
    built = s.Initialize()
    built.info.update(workload="batched_settling", n_scenes=len(specs), scenes=ranges, slot=slot, slots_per_axis=per,
                      world=world, bin_size=2.0 * max(sp["r"] for sp in specs))
    return built


def single_settling(spec, dt: float = 1e-5, packed=None, index: int = 0):
    """One scene of ``specs`` alone (for the sequential baseline and parity against the packed run).

    With ``packed`` (a ``batched_settling`` scene) and the scene's ``index`` in it, the scene is built alone in the
    packed run's domain, slot and bin size, so that its positions encode on the same voxel grid and its search uses
    the same cells: the two runs then differ only in the order of float sums."""
    s = SceneBuilder()
    if packed is None:
        pos, height = _settling_positions(spec, (0.0, 0.0, 0.0))
        H = max(height, spec["side"])
        dom = max(spec["side"], H) + 0.02
        s.InstructBoxDomainDimension(dom, dom, dom)
        lbf = (0.01, 0.01, 0.01)
        bin_size = 2.0 * spec["r"]
    else:
        info = packed.info
        per, slot = info["slots_per_axis"], info["slot"]
        s.InstructBoxDomainDimension(info["world"], info["world"], info["world"])
        lbf = (0.01 + (index % per) * slot, 0.01 + ((index // per) % per) * slot, 0.01 + (index // (per * per)) * slot)
        bin_size = info["bin_size"]
    s.SetCoordSysOrigin("explicit")
    _add_settling_scene(s, spec, lbf)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetInitBinSize(bin_size)
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)
    return s.Initialize()


def icosphere(radius: float, subdivisions: int = 2):
    """Triangulated sphere: an icosahedron whose faces are split in four ``subdivisions`` times, vertices pushed
    onto the sphere.  Returns (vertices, faces), outward winding."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / math.sqrt(1 + t * t) for p in v]
    for _ in range(subdivisions):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return (np.array(verts) * radius).astype(f32), np.array(f, np.int64)


def _grid_quad(p0, p1, p2, p3, n: int):
    """The quad p0 p1 p2 p3 (in order around it) as 2 n^2 triangles on an n x n grid."""
    p0, p1, p2, p3 = (np.asarray(p, np.float64) for p in (p0, p1, p2, p3))
    tris = []
    for i in range(n):
        for j in range(n):
            def at(u, v):
                return (1 - v) * ((1 - u) * p0 + u * p1) + v * ((1 - u) * p3 + u * p2)
            a, b = at(i / n, j / n), at((i + 1) / n, j / n)
            c, d = at((i + 1) / n, (j + 1) / n), at(i / n, (j + 1) / n)
            tris += [(a, b, c), (a, c, d)]
    return tris


def _mesh_arrays(tris):
    v = np.array(tris, np.float64).reshape(-1, 3).astype(f32)
    return v, np.arange(len(v), dtype=np.int64).reshape(-1, 3)


def mesh_funnel(n: int = 2000, r: float = 2e-3, rho: float = 2500.0, seed: int = 11, wall_clearance: float = 0.8,
                tilt_deg: float = 20.0, grid: int = 4, dt: float = 2e-6, cd_freq: int = 1, margin: float = 0.0,
                mu: float = 0.4, crr: float = 0.02):
    """Spheres (radii U[0.8, 1] r) in a square funnel made of triangle facets: four walls leaning ``tilt_deg`` out
    from the vertical and a floor, each face a ``grid`` x ``grid`` grid of quads split into two triangles (a fixed
    mesh body, family 1).  Spheres start on a jittered cubic lattice; ``wall_clearance`` below 1 starts the outer
    ones pressed into the walls and the floor, so sphere--mesh contacts on facet interiors, edges and corners exist
    from the first step."""
    rng = np.random.default_rng(seed)
    th = math.radians(tilt_deg)
    w0 = 10 * r * max(1.0, (n / 1000.0) ** (1 / 3))  # floor half-width
    pitch = 2.02 * r
    # lattice in the funnel: distance to every wall plane and the floor at least clearance x radius
    H = 4 * w0
    g = np.arange(-w0 - H * math.tan(th), w0 + H * math.tan(th) + pitch, pitch)
    zs = np.arange(0.0, H, pitch)
    X, Y, Z = np.meshgrid(g, g, zs, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    P = P[np.lexsort((P[:, 0], P[:, 1], P[:, 2]))]
    rad = rng.uniform(0.8 * r, r, len(P))
    c, s_ = math.cos(th), math.sin(th)
    # inward normals of the walls x = +-(w0 + z tan th), y likewise: (-+c, 0, s)
    dmin = P[:, 2]
    for ax in (0, 1):
        for sg in (1.0, -1.0):
            d = (w0 - sg * P[:, ax]) * c + P[:, 2] * s_
            dmin = np.minimum(dmin, d)
    keep = dmin >= wall_clearance * rad
    P, rad = P[keep][:n], rad[keep][:n]
    if len(P) < n:
        raise ValueError("funnel too small for n")
    P = P + rng.uniform(-0.005 * r, 0.005 * r, P.shape)
    zt = float(P[:, 2].max()) + 4 * r
    wt = w0 + zt * math.tan(th)
    tris = _grid_quad((-w0, -w0, 0), (w0, -w0, 0), (w0, w0, 0), (-w0, w0, 0), grid)
    for (a0, a1, b0, b1) in (((-w0, -w0), (w0, -w0), (-wt, -wt), (wt, -wt)), ((w0, -w0), (w0, w0), (wt, -wt), (wt, wt)),
                             ((w0, w0), (-w0, w0), (wt, wt), (-wt, wt)), ((-w0, w0), (-w0, -w0), (-wt, wt), (-wt, -wt))):
        tris += _grid_quad((*a0, 0), (*a1, 0), (*b1, zt), (*b0, zt), grid)
    s = SceneBuilder()
    box = 2 * wt + 8 * r
    s.InstructBoxDomainDimension(box, box, box)
    s.SetCoordSysOrigin("center")
    shift = np.array([0.0, 0.0, -zt / 2])
    m_s = s.LoadMaterial({"E": 1e8, "nu": 0.3, "CoR": 0.4, "mu": mu, "Crr": crr})
    m_w = s.LoadMaterial({"E": 2e8, "nu": 0.25, "CoR": 0.5, "mu": mu, "Crr": crr})
    types = [s.LoadSphereType(sphere_mass(float(ri), rho), float(ri), m_s) for ri in rad.astype(f32)]
    b = s.AddClumps(types, (P + shift).astype(f32))
    b.SetFamily(0)
    v, f = _mesh_arrays(tris)
    mesh = s.AddWavefrontMeshObject((v, f), m_w)
    mesh.SetInitPos(shift)
    mesh.SetFamily(1)
    s.SetFamilyFixed(1)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(cd_freq)
    s.SetExpandFactor(margin)
    s.SetInitBinSize(2.0 * float(f32(rad.min())))
    built = s.Initialize()
    built.info.update(workload="mesh_funnel", n=n, seed=seed, n_tris=len(f))
    return built


def mesh_ball_drop(n: int = 2000, r: float = 2e-3, rho: float = 2600.0, ball_radius: float = 0.02,
                   subdivisions: int = 3, ball_rho: float = 7000.0, speed: float = 1.0, seed: int = 12,
                   dt: float = 2e-6, cd_freq: int = 1, margin: float = 0.0, press: float = 0.2, layers: int = 4,
                   packed: bool = False, ball: bool = True):
    """A mesh ball (icosphere of ``ball_radius``, a free body) driven into a bed of spheres (radii U[0.8, 1] r on a
    jittered lattice of about ``layers`` layers in a box of analytical planes), as in the reference's BallDrop demo
    where the projectile is a Wavefront mesh.  The ball starts moving down at ``speed``, pressed ``press`` x r into
    the bed's top layer.  ``packed``: spheres of radius r on a simple cubic lattice of pitch 1.998 r, each pressed
    into its six neighbours (about three contacts per sphere from the first step).  ``ball`` False leaves the ball
    out (the same bed without a mesh body)."""
    rng = np.random.default_rng(seed)
    pitch = 1.998 * r if packed else 2.02 * r
    side = max(int(math.ceil(2.5 * ball_radius / pitch)), int(math.ceil(math.sqrt(n / layers))))
    layers = int(math.ceil(n / side ** 2))
    idx = np.arange(n)
    P = np.stack([(idx % side) * pitch, (idx // side % side) * pitch, (idx // side // side) * pitch], 1)
    P -= np.array([(side - 1) * pitch / 2, (side - 1) * pitch / 2, 0.0])
    if packed:
        rad = np.full(n, r)
    else:
        P += rng.uniform(-0.005 * r, 0.005 * r, P.shape)
        rad = rng.uniform(0.8 * r, r, n)
    half = side * pitch / 2 + r
    top = float((layers - 1) * pitch)
    s = SceneBuilder()
    box = max(2 * half, top + 4 * ball_radius) + 8 * r
    s.InstructBoxDomainDimension(box, box, box)
    s.SetCoordSysOrigin("center")
    z0 = -box / 2 + 2 * r
    m_s = s.LoadMaterial({"E": 1e8, "nu": 0.3, "CoR": 0.3, "mu": 0.4, "Crr": 0.01})
    m_b = s.LoadMaterial({"E": 5e8, "nu": 0.3, "CoR": 0.3, "mu": 0.3, "Crr": 0.0})
    # one sphere type per distinct radius (a packed bed has one)
    r_u, r_idx = np.unique(rad.astype(f32), return_inverse=True)
    tmpl = [s.LoadSphereType(sphere_mass(float(ri), rho), float(ri), m_s) for ri in r_u]
    b = s.AddClumps([tmpl[k] for k in r_idx], (P + np.array([0.0, 0.0, z0 + r])).astype(f32))
    b.SetFamily(0)
    for ax, sg in ((0, 1), (0, -1), (1, 1), (1, -1)):
        pos = np.zeros(3)
        pos[ax] = -sg * half
        nrm = np.zeros(3)
        nrm[ax] = sg
        s.AddBCPlane(pos, nrm, m_s).SetFamily(2)
    s.AddBCPlane((0, 0, z0), (0, 0, 1), m_s).SetFamily(2)
    s.SetFamilyFixed(2)
    # the ball's lowest facet sits `press` x r below the top layer's tops
    v, f = icosphere(ball_radius, subdivisions)
    if ball:
        zc = z0 + r + top + r + float(-v[:, 2].min()) - press * r
        mesh = s.AddWavefrontMeshObject((v, f), m_b)
        mesh.SetInitPos((0.0, 0.0, zc))
        mb = sphere_mass(ball_radius, ball_rho)
        mesh.SetMass(mb)
        mesh.SetMOI([0.4 * mb * ball_radius ** 2] * 3)
        mesh.SetInitVel((0.0, 0.0, -speed))
        mesh.SetFamily(0)
    s.SetInitTimeStep(dt)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    s.SetCDUpdateFreq(cd_freq)
    s.SetExpandFactor(margin)
    s.SetInitBinSize(2.0 * float(f32(rad.min())))
    built = s.Initialize()
    built.info.update(workload="mesh_ball_drop", n=n, seed=seed, n_tris=len(f) if ball else 0)
    return built
