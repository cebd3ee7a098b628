// device_common.cuh -- shared device helpers of the B200 DEM hot path.
//
// The arithmetic restates the reference's device helpers operation by operation (paths relative to the
// reference's src/): voxel <-> position codec (kernel/DEMHelperKernels.cu:66-135), quaternion rotation (:137-148),
// sphere-sphere and sphere-entity overlap tests (:195-264, :356-445) and the bin id of a point (:266-273).
// The library is compiled with --fmad=false so every multiply and add rounds on its own, like the CPU oracle,
// and float-to-integer conversions are written as explicit saturating helpers (PTX cvt semantics).
#pragma once
#ifndef __CUDACC_RTC__
#include <cstdint>
#include <cuda_runtime.h>
#endif

#include "../../include/deme_b200.h"

namespace deme_b200 {

constexpr double kTinyFloat = 1e-12;
constexpr double kHugeFloat = 1e15;
// src/DEM/Defines.h:30-35
constexpr double kTwoOverThree = 0.666666666666667;
constexpr double kFourOverThree = 1.333333333333333;
constexpr double kFiveOverThree = 1.666666666666667;
constexpr double kTwoTimesSqrtFiveOverSix = 1.825741858350554;
constexpr double kPi = 3.1415926535897932385;
constexpr double kPiSquared = 9.869604401089358;

// The search grid of one scene: cubic cells of edge 1 / inv_cell from the origin (ox, oy, oz), in positions
// relative to the domain's lower corner; cells [base, base + gx gy gz) of the cell arrays, row-major in x.  Positions
// outside the grid fall into its boundary cells (cell_of clamps), which keeps every search complete.
struct SearchGrid {
    double ox, oy, oz;
    double inv_cell;
    uint32_t gx, gy, gz, base;
    float r_max_cd;  // largest CD radius (radius + beta) of the scene's spheres
    uint32_t pad[3];
};

// Owner state lives in HBM as packed structure-of-arrays so that one owner is read with a few wide loads:
//   pos   : uint64 voxel id + ushort4 (locX, locY, locZ, family)
//   quat  : float4 (w, x, y, z)
//   vel   : float4 (vx, vy, vz, mass)
//   omg   : float4 (wx, wy, wz, 0)
//   moi   : float4 (Ixx, Iyy, Izz, 0)
// Spheres: float4 (relX, relY, relZ, radius), uint32 owner, uint8 material.
struct SimConsts {
    uint32_t nvXp2, nvYp2;
    double l_kernel, voxel_kernel;
    double bin_size;
    uint32_t nbX, nbY, nbZ;
    float beta;
    float h;
    float G[3];
    int integrator;
    uint32_t n_spheres, n_owners, n_anal;
    uint32_t n_tris;  // mesh facets (sphere--mesh contacts); 0: none
    // contact-detection search grids: one per scene (several only when independent scenes are packed into one
    // run), each a block of cells in the cell arrays; ownerScene maps an owner to its scene (null: one scene, whose
    // grid is also held here by value, grid0, so that a plain run reads it from the kernel parameters)
    const SearchGrid* grids;
    const uint32_t* ownerScene;
    SearchGrid grid0;
    float r_max_cd;      // largest CD radius (radius + beta) of all spheres
    float prefilter_abs; // absolute slack of the float pre-filter
    // the cell-order float4 records carry the sphere id in their low q_shift bits and, above them, an upper bound
    // of the CD radius in units of q_scale (see k_gather_sorted)
    uint32_t q_shift, id_mask;
    float q_scale;
    uint32_t* err;       // device error block (4 words), see index_ok
};

// Per-family prescription (constant-valued form of the reference's jitified strings).
struct Prescription {
    uint8_t used, lin_vel, rot_vel, lin_pos, rot_pos;
    uint8_t has_vel[3], has_omg[3], has_pos[3];
    float vel[3];
    float omg[3];
    double pos[3];
};

// Analytical component, placed in the world for the current state (owner pose applied).
struct AnalPlaced {
    double x, y, z;        // component reference point (double)
    float dx, dy, dz;      // rotated direction (plane normal / axis)
    uint32_t owner;
    uint8_t type, normal;
    uint16_t material;
    float mass;
    double size1, c1, c2, umin, umax;  // cylinder radius / cone (sin, cos, axial range)
};

// Mesh facet (triangle) placed in the world for the current state: vertices = owner position (double) + the owner
// frame vertex rotated in float (as the analytical components are placed).
struct TriPlaced {
    double ax, ay, az, bx, by, bz, cx, cy, cz;
    uint32_t owner;
    uint16_t material;
    uint16_t pad;
    float mass;  // the owner's mass
};

// ---------------- saturating conversions (cvt.rzi semantics, NaN -> 0) ----------------
__host__ __device__ __forceinline__ uint32_t sat_u32(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967296.0) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

// Search-grid cell coordinate of x (clamped to the grid).  Monotone in x, which is all the search relies on.
__device__ __forceinline__ uint32_t cell_of(double x, double inv_cell, uint32_t g) {
    return min(sat_u32(x * inv_cell), g - 1u);
}
__host__ __device__ __forceinline__ uint64_t sat_u64(double x) {
    if (!(x > 0.0)) return 0ull;
    if (x >= 18446744073709551616.0) return ~0ull;
    return (uint64_t)x;
}
__host__ __device__ __forceinline__ uint16_t sat_u16(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 65536.0) return 65535u;
    return (uint16_t)x;
}

// ---------------- position codec ----------------
// voxelIDToPosition (DEMHelperKernels.cu:93-110)
__device__ __forceinline__ void voxel_to_pos(const SimConsts& k, uint64_t id, uint32_t sx, uint32_t sy, uint32_t sz,
                                             double& X, double& Y, double& Z) {
    uint64_t vx = id & ((1ull << k.nvXp2) - 1ull);
    uint64_t vy = (id >> k.nvXp2) & ((1ull << k.nvYp2) - 1ull);
    uint64_t vz = id >> (k.nvXp2 + k.nvYp2);
    X = __dadd_rn(__dmul_rn((double)vx, k.voxel_kernel), __dmul_rn((double)sx, k.l_kernel));
    Y = __dadd_rn(__dmul_rn((double)vy, k.voxel_kernel), __dmul_rn((double)sy, k.l_kernel));
    Z = __dadd_rn(__dmul_rn((double)vz, k.voxel_kernel), __dmul_rn((double)sz, k.l_kernel));
}
// positionToVoxelID (DEMHelperKernels.cu:113-135)
__device__ __forceinline__ void pos_to_voxel(const SimConsts& k, double X, double Y, double Z, uint64_t& id,
                                             uint16_t& sx, uint16_t& sy, uint16_t& sz) {
    const double vs = k.voxel_kernel, l = k.l_kernel;
    uint64_t nx = sat_u64(X / vs), ny = sat_u64(Y / vs), nz = sat_u64(Z / vs);
    sx = sat_u16((X - __dmul_rn((double)nx, vs)) / l);
    sy = sat_u16((Y - __dmul_rn((double)ny, vs)) / l);
    sz = sat_u16((Z - __dmul_rn((double)nz, vs)) / l);
    id = nx + (ny << k.nvXp2) + (nz << (k.nvXp2 + k.nvYp2));
}

// applyOriQToVector3<float, float> (DEMHelperKernels.cu:137-148)
__device__ __forceinline__ void rot_f(float& X, float& Y, float& Z, float w, float x, float y, float z) {
    const float ox = X, oy = Y, oz = Z;
    X = (2.0f * (w * w + x * x) - 1.0f) * ox + (2.0f * (x * y - w * z)) * oy + (2.0f * (x * z + w * y)) * oz;
    Y = (2.0f * (x * y + w * z)) * ox + (2.0f * (w * w + y * y) - 1.0f) * oy + (2.0f * (y * z - w * x)) * oz;
    Z = (2.0f * (x * z - w * y)) * ox + (2.0f * (y * z + w * x)) * oy + (2.0f * (w * w + z * z) - 1.0f) * oz;
}

// The matrix of applyOriQToVector3<float, float> for one quaternion: its nine coefficients formed exactly as rot_f
// forms them, so rot_apply equals rot_f bit for bit.  Rotating by the conjugate quaternion (the inverse rotation,
// which the reference writes as applyOriQToVector3 with -x, -y, -z) gives the transposed coefficients exactly --
// negating a component is exact, and a - (-b) rounds as a + b -- so rot_apply_t equals rot_f of the conjugate bit
// for bit.  One matrix thus serves every rotation by a body's orientation in a kernel.
struct RotF {
    float m00, m01, m02, m10, m11, m12, m20, m21, m22;
};
__device__ __forceinline__ RotF rot_matrix(float w, float x, float y, float z) {
    RotF r;
    r.m00 = 2.0f * (w * w + x * x) - 1.0f;
    r.m01 = 2.0f * (x * y - w * z);
    r.m02 = 2.0f * (x * z + w * y);
    r.m10 = 2.0f * (x * y + w * z);
    r.m11 = 2.0f * (w * w + y * y) - 1.0f;
    r.m12 = 2.0f * (y * z - w * x);
    r.m20 = 2.0f * (x * z - w * y);
    r.m21 = 2.0f * (y * z + w * x);
    r.m22 = 2.0f * (w * w + z * z) - 1.0f;
    return r;
}
__device__ __forceinline__ void rot_apply(const RotF& r, float& X, float& Y, float& Z) {
    const float ox = X, oy = Y, oz = Z;
    X = r.m00 * ox + r.m01 * oy + r.m02 * oz;
    Y = r.m10 * ox + r.m11 * oy + r.m12 * oz;
    Z = r.m20 * ox + r.m21 * oy + r.m22 * oz;
}
__device__ __forceinline__ void rot_apply_t(const RotF& r, float& X, float& Y, float& Z) {
    const float ox = X, oy = Y, oz = Z;
    X = r.m00 * ox + r.m10 * oy + r.m20 * oz;
    Y = r.m01 * ox + r.m11 * oy + r.m21 * oz;
    Z = r.m02 * ox + r.m12 * oy + r.m22 * oz;
}

// Rotational velocity of a body's contact point in the global frame, as the reference's force model forms it:
// cross(omega, local contact point) in the body frame, then the body's orientation applied
// (FullHertzianForceModel.cu), every operation rounded on its own.
__device__ __forceinline__ float3 rot_cp_velocity(const RotF& r, float3 w, float3 cp) {
    float x = w.y * cp.z - w.z * cp.y, y = w.z * cp.x - w.x * cp.z, z = w.x * cp.y - w.y * cp.x;
    rot_apply(r, x, y, z);
    return make_float3(x, y, z);
}

// locateMaskPair (DEMHelperKernels.cu:51-56)
__device__ __forceinline__ uint32_t mask_index(uint32_t i, uint32_t j) {
    if (i > j) {
        uint32_t t = i;
        i = j;
        j = t;
    }
    return (1u + j) * j / 2u + i;
}

// normalizeVector3<float> (DEMHelperKernels.cu:156-166)
__device__ __forceinline__ void normalize_f(float& x, float& y, float& z) {
    const float m = sqrtf(x * x + y * y + z * z);
    x /= m;
    y /= m;
    z /= m;
}

// Bin index range covered by a sphere along one axis (DEMBinSphereKernels.cu:52-64, 163-175).
__device__ __forceinline__ void bin_range(double p, double rD, double bs, uint32_t& lo, uint32_t& hi) {
    const double b = p / bs, span = rD / bs;
    lo = sat_u32(b - span);
    hi = sat_u32(b + span);
}

// Signed gap and wall normal of the cylinder / cone components (no reference counterpart; same conventions as the
// reference plane).  Returns false where the normal is undefined or the cone wall does not exist.
__device__ __forceinline__ bool curved_gap(const AnalPlaced& a, double xA, double yA, double zA, double& gap,
                                           double& nx, double& ny, double& nz) {
    const double ax = (double)a.dx, ay = (double)a.dy, az = (double)a.dz;
    const double vx = xA - a.x, vy = yA - a.y, vz = zA - a.z;
    const double t = vx * ax + vy * ay + vz * az;
    const double wx = vx - t * ax, wy = vy - t * ay, wz = vz - t * az;
    const double rho = sqrt(wx * wx + wy * wy + wz * wz);
    if (!(rho > 0.0)) return false;
    const double ux = wx / rho, uy = wy / rho, uz = wz / rho;
    if (a.type == DEME_ANAL_CYLINDER) {
        if (a.normal) {
            gap = rho - a.size1;
            nx = ux;
            ny = uy;
            nz = uz;
        } else {
            gap = a.size1 - rho;
            nx = -ux;
            ny = -uy;
            nz = -uz;
        }
        return true;
    }
    const double s = t * a.c2 + rho * a.c1;
    const double uc = s * a.c2;
    if (uc < a.umin || uc > a.umax) return false;
    const double g = t * a.c1 - rho * a.c2;
    const double gx = a.c1 * ax - a.c2 * ux, gy = a.c1 * ay - a.c2 * uy, gz = a.c1 * az - a.c2 * uz;
    if (a.normal) {
        gap = -g;
        nx = -gx;
        ny = -gy;
        nz = -gz;
    } else {
        gap = g;
        nx = gx;
        ny = gy;
        nz = gz;
    }
    return true;
}

// checkSphereEntityOverlap, contact-detection form (DEMHelperKernels.cu:356-391)
__device__ __forceinline__ int anal_overlap_cd(const AnalPlaced& a, double xA, double yA, double zA, double radA,
                                               float beta4) {
    if (a.type == DEME_ANAL_PLANE) {
        const double px = xA - a.x, py = yA - a.y, pz = zA - a.z;
        const double dist = px * (double)a.dx + py * (double)a.dy + pz * (double)a.dz;
        if (dist > radA + (double)beta4) return DEME_NOT_A_CONTACT;
        return DEME_SPHERE_PLANE_CONTACT;
    }
    if (a.type == DEME_ANAL_CYLINDER || a.type == DEME_ANAL_CONE) {
        double gap, nx, ny, nz;
        if (!curved_gap(a, xA, yA, zA, gap, nx, ny, nz)) return DEME_NOT_A_CONTACT;
        if (gap > radA + (double)beta4) return DEME_NOT_A_CONTACT;
        return a.type == DEME_ANAL_CYLINDER ? DEME_SPHERE_CYLINDER_CONTACT : DEME_SPHERE_CONE_CONTACT;
    }
    return DEME_NOT_A_CONTACT;
}

// checkSphereEntityOverlap, dynamics form with contact point and normal (DEMHelperKernels.cu:394-445)
__device__ __forceinline__ int anal_overlap_dt(const AnalPlaced& a, double xA, double yA, double zA, double radA,
                                               double& CPX, double& CPY, double& CPZ, float& nX, float& nY, float& nZ,
                                               double& depth) {
    if (a.type == DEME_ANAL_PLANE) {
        const double px = xA - a.x, py = yA - a.y, pz = zA - a.z;
        const double ddx = (double)a.dx, ddy = (double)a.dy, ddz = (double)a.dz;
        const double dist = px * ddx + py * ddy + pz * ddz;
        const double od = (radA + 0.0 - dist) / 2.0;
        if (od < 0.0) return DEME_NOT_A_CONTACT;
        depth = od;
        CPX = xA - ddx * (dist + od);
        CPY = yA - ddy * (dist + od);
        CPZ = zA - ddz * (dist + od);
        nX = (float)ddx;
        nY = (float)ddy;
        nZ = (float)ddz;
        return DEME_SPHERE_PLANE_CONTACT;
    }
    if (a.type == DEME_ANAL_CYLINDER || a.type == DEME_ANAL_CONE) {
        double gap, nx, ny, nz;
        if (!curved_gap(a, xA, yA, zA, gap, nx, ny, nz)) return DEME_NOT_A_CONTACT;
        const double od = (radA + 0.0 - gap) / 2.0;
        if (od < 0.0) return DEME_NOT_A_CONTACT;
        depth = od;
        CPX = xA - nx * (gap + od);
        CPY = yA - ny * (gap + od);
        CPZ = zA - nz * (gap + od);
        nX = (float)nx;
        nY = (float)ny;
        nZ = (float)nz;
        return a.type == DEME_ANAL_CYLINDER ? DEME_SPHERE_CYLINDER_CONTACT : DEME_SPHERE_CONE_CONTACT;
    }
    return DEME_NOT_A_CONTACT;
}

// Group of a contact type inside one sphere's segment of the contact list: sphere--analytical (0), sphere--mesh (1),
// sphere--sphere (2).  Segments are sorted by (group, idB).
__host__ __device__ __forceinline__ uint32_t contact_group(uint32_t type) {
    return type == DEME_SPHERE_SPHERE_CONTACT ? 2u : (type == DEME_SPHERE_MESH_CONTACT ? 1u : 0u);
}

// Sphere--mesh contact geometry (no reference counterpart: the reference declares the sphere--mesh contact type but
// has no detection for it).  The point of the triangle closest to the sphere centre p, by the region tests of
// Ericson's closest-point-on-triangle algorithm (Real-Time Collision Detection, 5.1.5), in double: the triangle is
// two-sided, and each triangle a sphere overlaps is one contact.  Contact-detection form: the distance to that point
// at most the reach.  Dynamics form, with the plane's conventions (anal_overlap_dt): gap = the distance,
// half the overlap as the depth, the normal from the closest point to the centre (float, normalised in float as the
// sphere pair's), the contact point p - n (gap + depth), the contact-detection reach the expanded radius plus the
// margin beta (as for an analytical component).  A centre exactly on the triangle takes the face normal
// a->b x a->c.
__device__ __forceinline__ void tri_closest(const TriPlaced& t, double px, double py, double pz, double& qx, double& qy,
                                            double& qz) {
    const double abx = t.bx - t.ax, aby = t.by - t.ay, abz = t.bz - t.az;
    const double acx = t.cx - t.ax, acy = t.cy - t.ay, acz = t.cz - t.az;
    const double apx = px - t.ax, apy = py - t.ay, apz = pz - t.az;
    const double d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= 0.0 && d2 <= 0.0) {
        qx = t.ax, qy = t.ay, qz = t.az;
        return;
    }
    const double bpx = px - t.bx, bpy = py - t.by, bpz = pz - t.bz;
    const double d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= 0.0 && d4 <= d3) {
        qx = t.bx, qy = t.by, qz = t.bz;
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        qx = t.ax + v * abx, qy = t.ay + v * aby, qz = t.az + v * abz;
        return;
    }
    const double cpx = px - t.cx, cpy = py - t.cy, cpz = pz - t.cz;
    const double d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= 0.0 && d5 <= d6) {
        qx = t.cx, qy = t.cy, qz = t.cz;
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        qx = t.ax + w * acx, qy = t.ay + w * acy, qz = t.az + w * acz;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        qx = t.bx + w * (t.cx - t.bx), qy = t.by + w * (t.cy - t.by), qz = t.bz + w * (t.cz - t.bz);
        return;
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    qx = t.ax + abx * v + acx * w, qy = t.ay + aby * v + acy * w, qz = t.az + abz * v + acz * w;
}
__device__ __forceinline__ double tri_dist2(const TriPlaced& t, double px, double py, double pz, double& qx, double& qy,
                                            double& qz) {
    tri_closest(t, px, py, pz, qx, qy, qz);
    return (px - qx) * (px - qx) + (py - qy) * (py - qy) + (pz - qz) * (pz - qz);
}
// radA: the sphere's radius + beta; the facet, like an analytical component, adds the margin beta4 once more
__device__ __forceinline__ bool tri_overlap_cd(const TriPlaced& t, double px, double py, double pz, double radA,
                                               float beta4) {
    double qx, qy, qz;
    const double reach = radA + (double)beta4;
    return tri_dist2(t, px, py, pz, qx, qy, qz) <= reach * reach;
}
__device__ __forceinline__ bool tri_overlap_dt(const TriPlaced& t, double xA, double yA, double zA, double radA,
                                               double& CPX, double& CPY, double& CPZ, float& nX, float& nY, float& nZ,
                                               double& depth) {
    double qx, qy, qz;
    const double d2 = tri_dist2(t, xA, yA, zA, qx, qy, qz);
    const double gap = sqrt(d2);
    const double od = (radA - gap) / 2.0;
    if (od < 0.0) return false;
    if (gap > 0.0) {
        nX = (float)(xA - qx);
        nY = (float)(yA - qy);
        nZ = (float)(zA - qz);
    } else {
        const double abx = t.bx - t.ax, aby = t.by - t.ay, abz = t.bz - t.az;
        const double acx = t.cx - t.ax, acy = t.cy - t.ay, acz = t.cz - t.az;
        nX = (float)(aby * acz - abz * acy);
        nY = (float)(abz * acx - abx * acz);
        nZ = (float)(abx * acy - aby * acx);
    }
    normalize_f(nX, nY, nZ);
    depth = od;
    CPX = xA - (double)nX * (gap + od);
    CPY = yA - (double)nY * (gap + od);
    CPZ = zA - (double)nZ * (gap + od);
    return true;
}

// Device error word bits (read by the host once per step; kernels never trap).
enum : uint32_t {
    ERR_CONTACT_CAPACITY = 1u << 0,
    ERR_SORT_LOOKBACK_TIMEOUT = 1u << 1,
    ERR_SCAN_LOOKBACK_TIMEOUT = 1u << 2,
    ERR_SEGMENT_TOO_LONG = 1u << 3,
    ERR_INDEX = 1u << 4,
};

// Index self-check: an out-of-range index sets ERR_INDEX, records (site, index, limit) of the first offender in
// err[1..3] and the caller skips the access.  err points to the handle's 4-word device error block.
__device__ __forceinline__ bool index_ok(uint32_t* err, uint32_t site, uint64_t idx, uint64_t limit) {
    if (idx < limit) return true;
    if (atomicOr(err, ERR_INDEX) & ERR_INDEX) return false;
    err[1] = site;
    err[2] = (uint32_t)idx;
    err[3] = (uint32_t)limit;
    return false;
}

}  // namespace deme_b200
