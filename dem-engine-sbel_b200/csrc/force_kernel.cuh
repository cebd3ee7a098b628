// force_kernel.cuh -- the fused force + collection kernel (one thread per contact): pose gather, overlap re-test,
// contact model, history update and accumulation of the owners' linear and angular accelerations (the reference's
// calculateContactForces + collectContactForces, src/kernel/DEMCalcForceKernels.cu:14-179,
// src/algorithms/DEMCubForceCollection.cu:20-158).
//
// The same source serves two builds: kernels.cu compiles it ahead of time with the built-in Hertz-Mindlin model,
// and the force-model compiler (force_jit.cu) compiles it at run time with NVRTC and DEME_USER_FORCE_MODEL
// defined, where the model block is a user's force-model string between generated wildcard loads and stores.
#pragma once
#include "kernels.cuh"

namespace deme_b200 {

// Block shapes (threads, resident blocks per SM; 64 registers a thread in each): 128 x 8 by default, where blocks
// wait less at the block-wide barriers (the voided-step check and the wall partials) than 256 x 4 or 512 x 2; the
// autotuner may pick another.  Run-time compiled user models use the default.
constexpr uint32_t kForceThreads = 128;
constexpr uint32_t kForceMinBlocks = 8;
// kNormalOnly: the built-in model as the frictionless Hertzian model (a scene with no contact wildcards).
template <bool kStore, uint32_t kThreads = kForceThreads, uint32_t kMinBlocks = kForceMinBlocks,
          bool kNormalOnly = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_force(SimConsts k, StateView s, ContactView c, uint32_t n,
                                                               bool has_hist, ContactOutputs out, AnalAccum aa) {
    // a device error earlier in the step (a list or pool outgrew its capacity inside a replayed graph) voids the
    // step: nothing is written, and the host redoes it from the untouched state
    if (__syncthreads_or(threadIdx.x == 0 && *k.err != 0u)) return;
    // blocks past the count (a launch that covers the list's capacity) have nothing to do; k_anal_reduce reads the
    // same count and skips their partials
    if (c.dN && blockIdx.x * blockDim.x >= min(n, *c.dN)) return;
    // analytical owners (walls) collect their reactions block-locally, then one fixed-order reduction
    extern __shared__ float s_anal[];  // 6 floats per analytical owner
    const bool partials = aa.nAO && !aa.direct;
    if (partials) {
        for (uint32_t t = threadIdx.x; t < 6u * aa.nAO; t += blockDim.x) s_anal[t] = 0.f;
        __syncthreads();
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // the count on the device bounds the launch (which may cover the list's capacity)
    const bool valid = i < (c.dN ? min(n, *c.dN) : n);
    uint32_t oA = 0xFFFFFFFFu, oB = 0xFFFFFFFFu;
    bool bSphere = false;
    float3 F = make_float3(0.f, 0.f, 0.f), T = make_float3(0.f, 0.f, 0.f);
    float3 cpA = make_float3(0.f, 0.f, 0.f), cpB = make_float3(0.f, 0.f, 0.f);
    float4 qA = make_float4(1.f, 0.f, 0.f, 0.f), qB = qA;
    bool active = false;
    bool ids_ok = valid;
    if (valid) {
        const int ct0 = c.type[i];
        ids_ok = index_ok(k.err, 8, c.idA[i], k.n_spheres) &&
                 index_ok(k.err, 9, c.idB[i],
                          ct0 == DEME_SPHERE_SPHERE_CONTACT ? k.n_spheres
                                                            : (ct0 == DEME_SPHERE_MESH_CONTACT ? k.n_tris : k.n_anal)) &&
                 index_ok(k.err, 10, ct0 == DEME_NOT_A_CONTACT || ct0 > DEME_SPHERE_CONE_CONTACT ? 1 : 0, 1);
    }
    if (ids_ok) {
        const uint32_t sA = c.idA[i];
        const uint32_t bId = c.idB[i];
        int ct = c.type[i];
        float4 hw = has_hist ? c.hist[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        ContactGeom g;
        // body A (always a sphere); body B's sphere record and owner id are fetched alongside, so that its owner
        // loads do not wait behind A's arithmetic
        const bool ssEarly = ct == DEME_SPHERE_SPHERE_CONTACT;
        oA = __ldg(s.sOwner + sA);
        const uint32_t oBEarly = ssEarly ? __ldg(s.sOwner + bId) : 0u;
        const float4 spA = __ldg(s.sph + sA);
        const float4 spBEarly = ssEarly ? __ldg(s.sph + bId) : make_float4(0.f, 0.f, 0.f, 0.f);
        const ushort4 lA = s.loc[oA];
        qA = s.quat[oA];
        const float4 vA = s.vel[oA];
        const float4 wA = s.omg[oA];
        double AOx, AOy, AOz;
        voxel_to_pos(k, s.voxel[oA], lA.x, lA.y, lA.z, AOx, AOy, AOz);
        // one rotation matrix per body serves every rotation by its orientation here (rot_matrix)
        const RotF RA = rot_matrix(qA.x, qA.y, qA.z, qA.w);
        RotF RB;
        float rx = spA.x, ry = spA.y, rz = spA.z;
        rot_apply(RA, rx, ry, rz);
        const double Ax = AOx + (double)rx, Ay = AOy + (double)ry, Az = AOz + (double)rz;
        g.ARadius = spA.w;
        g.AOwnerMass = vA.w;
        g.matA = s.sMat[sA];
        g.ALinVel = make_float3(vA.x, vA.y, vA.z);
        g.ARotVel = make_float3(wA.x, wA.y, wA.z);
        double BOx, BOy, BOz, CPx = 0, CPy = 0, CPz = 0, depth = 0;
        float nX = 0, nY = 0, nZ = 0;
        if (ct == DEME_SPHERE_SPHERE_CONTACT) {
            bSphere = true;
            oB = oBEarly;
            const float4 spB = spBEarly;
            const ushort4 lB = s.loc[oB];
            qB = s.quat[oB];
            const float4 vB = s.vel[oB];
            const float4 wB = s.omg[oB];
            voxel_to_pos(k, s.voxel[oB], lB.x, lB.y, lB.z, BOx, BOy, BOz);
            RB = rot_matrix(qB.x, qB.y, qB.z, qB.w);
            float bx = spB.x, by = spB.y, bz = spB.z;
            rot_apply(RB, bx, by, bz);
            const double Bx = BOx + (double)bx, By = BOy + (double)by, Bz = BOz + (double)bz;
            g.BRadius = spB.w;
            g.BOwnerMass = vB.w;
            g.matB = s.sMat[bId];
            g.BLinVel = make_float3(vB.x, vB.y, vB.z);
            g.BRotVel = make_float3(wB.x, wB.y, wB.z);
            // checkSpheresOverlap<double, float>, DEMHelperKernels.cu:233-264
            const double radA = (double)g.ARadius, radB = (double)g.BRadius;
            const double d2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
            if (d2 > (radA + radB) * (radA + radB)) {
                ct = DEME_NOT_A_CONTACT;
            } else {
                nX = (float)(Ax - Bx);
                nY = (float)(Ay - By);
                nZ = (float)(Az - Bz);
                normalize_f(nX, nY, nZ);
                depth = radA + radB - sqrt(d2);
                CPx = Bx + (radB - depth / 2.0) * (double)nX;
                CPy = By + (radB - depth / 2.0) * (double)nY;
                CPz = Bz + (radB - depth / 2.0) * (double)nZ;
            }
        } else if (ct == DEME_SPHERE_MESH_CONTACT) {
            // a mesh facet: a wall-like body B (huge radius) on the facet's owner
            const TriPlaced t = s.tri[bId];
            oB = t.owner;
            const ushort4 lB = s.loc[oB];
            qB = s.quat[oB];
            const float4 vB = s.vel[oB];
            const float4 wB = s.omg[oB];
            voxel_to_pos(k, s.voxel[oB], lB.x, lB.y, lB.z, BOx, BOy, BOz);
            RB = rot_matrix(qB.x, qB.y, qB.z, qB.w);
            g.BRadius = (float)kHugeFloat;
            g.BOwnerMass = t.mass;
            g.matB = t.material;
            g.BLinVel = make_float3(vB.x, vB.y, vB.z);
            g.BRotVel = make_float3(wB.x, wB.y, wB.z);
            if (!tri_overlap_dt(t, Ax, Ay, Az, (double)g.ARadius, CPx, CPy, CPz, nX, nY, nZ, depth))
                ct = DEME_NOT_A_CONTACT;
        } else {
            const AnalPlaced a = s.anal[bId];
            oB = a.owner;
            const ushort4 lB = s.loc[oB];
            qB = s.quat[oB];
            const float4 vB = s.vel[oB];
            const float4 wB = s.omg[oB];
            voxel_to_pos(k, s.voxel[oB], lB.x, lB.y, lB.z, BOx, BOy, BOz);
            RB = rot_matrix(qB.x, qB.y, qB.z, qB.w);
            g.BRadius = (float)kHugeFloat;
            g.BOwnerMass = a.mass;
            g.matB = a.material;
            g.BLinVel = make_float3(vB.x, vB.y, vB.z);
            g.BRotVel = make_float3(wB.x, wB.y, wB.z);
            ct = anal_overlap_dt(a, Ax, Ay, Az, (double)g.ARadius, CPx, CPy, CPz, nX, nY, nZ, depth);
        }
        if (ct != DEME_NOT_A_CONTACT) {
            active = true;
            float cax = (float)(CPx - AOx), cay = (float)(CPy - AOy), caz = (float)(CPz - AOz);
            float cbx = (float)(CPx - BOx), cby = (float)(CPy - BOy), cbz = (float)(CPz - BOz);
            rot_apply_t(RA, cax, cay, caz);
            rot_apply_t(RB, cbx, cby, cbz);
            cpA = make_float3(cax, cay, caz);
            cpB = make_float3(cbx, cby, cbz);
            g.B2A = make_float3(nX, nY, nZ);
            g.overlapDepth = depth;
            g.locCPA = cpA;
            g.locCPB = cpB;
            g.ARotCP = rot_cp_velocity(RA, g.ARotVel, cpA);
            g.BRotCP = rot_cp_velocity(RB, g.BRotVel, cpB);
#ifdef DEME_USER_FORCE_MODEL
            {
                // The names a DEM-Engine force-model string uses (calculateContactForces,
                // src/kernel/DEMCalcForceKernels.cu:14-179, and the ingredients of src/DEM/Models.h:197-234).
                const int myContactType = ct;
                const uint32_t myContactID = i;
                double3 contactPnt = make_double3(CPx, CPy, CPz);
                double3 AOwnerPos = make_double3(AOx, AOy, AOz), BOwnerPos = make_double3(BOx, BOy, BOz);
                double3 bodyAPos = make_double3(Ax, Ay, Az);
                float3 B2A = make_float3(nX, nY, nZ);
                double overlapDepth = depth;
                float AOwnerMass = g.AOwnerMass, BOwnerMass = g.BOwnerMass, ARadius = g.ARadius, BRadius = g.BRadius;
                float AoriQw = qA.x, AoriQx = qA.y, AoriQy = qA.z, AoriQz = qA.w;
                float BoriQw = qB.x, BoriQx = qB.y, BoriQy = qB.z, BoriQz = qB.w;
                uint32_t bodyAMatType = g.matA, bodyBMatType = g.matB;
                float ts = k.h;
                float3 ALinVel = g.ALinVel, BLinVel = g.BLinVel, ARotVel = g.ARotVel, BRotVel = g.BRotVel;
                uint32_t AOwnerFamily = lA.w, BOwnerFamily = s.loc[oB].w;
                float3 locCPA = cpA, locCPB = cpB;
                float3 force = make_float3(0.f, 0.f, 0.f), torque_only_force = make_float3(0.f, 0.f, 0.f);
                const float* E = s.mat.E;
                const float* nu = s.mat.nu;
                const float* CoR = s.mat.CoR;
                const float* mu = s.mat.mu;
                const float* Crr = s.mat.Crr;
                // contact wildcards in, the model, contact wildcards out (generated from the model string)
#include "deme_user_force_model.inc"
                F = force;
                T = torque_only_force;
                cpA = locCPA;
                cpB = locCPB;
            }
#else
            hertz_mindlin<kNormalOnly>(g, s.mat, k.h, F, T, hw.x, hw.y, hw.z, hw.w);
#endif
        } else {
            hw = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (has_hist) c.hist[i] = hw;
        if (kStore) {
            out.F[i] = make_float4(F.x, F.y, F.z, 0.f);
            out.TOF[i] = make_float4(T.x, T.y, T.z, 0.f);
            out.CPA[i] = make_float4(cpA.x, cpA.y, cpA.z, 0.f);
            out.CPB[i] = make_float4(cpB.x, cpB.y, cpB.z, 0.f);
        }
    }
    // owner contributions (forceToAcc / forceToAngAcc, src/kernel/DEMCollectForceKernels.cu:68-120): the
    // reference divides by the mass and the principal moments; this multiplies by their reciprocals (within one
    // rounding of the quotient), which saves a division sequence per component
    float4 aA = make_float4(0.f, 0.f, 0.f, 0.f), alA = aA, aB = aA, alB = aA;
    if (active) {
        const float4 mi = __ldg(s.invMoi + oA);
        const bool bOwnerCounts = bSphere || aa.nAO;
        aA = make_float4(F.x * mi.w, F.y * mi.w, F.z * mi.w, 0.f);
        float gx = F.x + T.x, gy = F.y + T.y, gz = F.z + T.z;
        // the matrices again from the quaternions (cached loads), rather than held through the contact model
        rot_apply_t(rot_matrix(qA.x, qA.y, qA.z, qA.w), gx, gy, gz);
        alA = make_float4((cpA.y * gz - cpA.z * gy) * mi.x, (cpA.z * gx - cpA.x * gz) * mi.y,
                          (cpA.x * gy - cpA.y * gx) * mi.z, 0.f);
        if (bOwnerCounts) {
            const float4 mj = __ldg(s.invMoi + oB);  // for an analytical owner, its owner mass (massOwnerBody)
            aB = make_float4(-F.x * mj.w, -F.y * mj.w, -F.z * mj.w, 0.f);
            float hx = -(F.x + T.x), hy = -(F.y + T.y), hz = -(F.z + T.z);
            rot_apply_t(rot_matrix(qB.x, qB.y, qB.z, qB.w), hx, hy, hz);
            alB = make_float4((cpB.y * hz - cpB.z * hy) * mj.x, (cpB.z * hx - cpB.x * hz) * mj.y,
                              (cpB.x * hy - cpB.y * hx) * mj.z, 0.f);
        }
    }
    // A side: contacts of one owner are adjacent (sorted by sphere id; a clump's spheres have consecutive ids).
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t key = ids_ok ? oA : 0xFFFFFFFFu;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t k2 = __shfl_down_sync(0xffffffffu, key, off);
        const float x0 = __shfl_down_sync(0xffffffffu, aA.x, off);
        const float x1 = __shfl_down_sync(0xffffffffu, aA.y, off);
        const float x2 = __shfl_down_sync(0xffffffffu, aA.z, off);
        const float y0 = __shfl_down_sync(0xffffffffu, alA.x, off);
        const float y1 = __shfl_down_sync(0xffffffffu, alA.y, off);
        const float y2 = __shfl_down_sync(0xffffffffu, alA.z, off);
        if (lane + off < 32 && k2 == key) {
            aA.x += x0;
            aA.y += x1;
            aA.z += x2;
            alA.x += y0;
            alA.y += y1;
            alA.z += y2;
        }
    }
    const uint32_t prevKey = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = (lane == 0) || (prevKey != key);
    if (head && key != 0xFFFFFFFFu) {
        atomicAdd(&s.acc[key], aA);
        atomicAdd(&s.alpha[key], alA);
    }
    if (active && bSphere) {
        atomicAdd(&s.acc[oB], aB);
        atomicAdd(&s.alpha[oB], alB);
    }
    if (aa.nAO && aa.direct && active && !bSphere) {
        atomicAdd(&s.acc[oB], aB);
        atomicAdd(&s.alpha[oB], alB);
    }
    if (partials) {
        if (active && !bSphere && index_ok(k.err, 11, oB - aa.nClumps, aa.nAO)) {
            float* slot = s_anal + 6u * (oB - aa.nClumps);
            atomicAdd(slot + 0, aB.x);
            atomicAdd(slot + 1, aB.y);
            atomicAdd(slot + 2, aB.z);
            atomicAdd(slot + 3, alB.x);
            atomicAdd(slot + 4, alB.y);
            atomicAdd(slot + 5, alB.z);
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < 6u * aa.nAO; t += blockDim.x)
            aa.partial[(size_t)blockIdx.x * 6u * aa.nAO + t] = s_anal[t];
    }
}

}  // namespace deme_b200
