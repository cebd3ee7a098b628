// family_change_kernel.cuh -- per-owner family changes on conditions written by the user (the reference's
// ChangeFamilyWhen, src/DEM/APIPublic.cpp:167-182, whose rules it pastes into applyFamilyChanges,
// src/kernel/DEMModeratorKernels.cu:9-38, through equipFamilyOnFlyChanges, src/DEM/APIPrivate.cpp:980-1003).
//
// Compiled only at run time with NVRTC (force_jit.cu): deme_family_change_rules.inc holds one block per rule,
//   if (family_code == FROM) { bool shouldMakeChange = false; { <condition, its `return` turned into
//   `shouldMakeChange =`> } if (shouldMakeChange) newFamily = TO; }
// A condition sees the names the reference gives it: pos (double3, the owner's position from the domain's lower
// corner, as voxelIDToPosition returns it), vel and acc (float3), mass, family_code, t (the time: a float advanced
// by h each step, as the reference's dT advances it) and h (the step).
// Rules test the family the owner had when the kernel started; when several apply, the last one wins.  The kernel
// runs after the forces and before the integration of a step, as the reference's routineChecks does.
#pragma once
#include "kernels.cuh"

namespace deme_b200 {

__global__ void __launch_bounds__(256) k_family_change(SimConsts k, StateView s, const float* time) {
    const uint32_t myOwner = blockIdx.x * blockDim.x + threadIdx.x;
    if (myOwner >= k.n_owners) return;
    if (*k.err != 0u) return;  // a voided step leaves the state as it was
    ushort4 l = s.loc[myOwner];
    const unsigned int family_code = l.w;
    double3 pos;
    voxel_to_pos(k, s.voxel[myOwner], l.x, l.y, l.z, pos.x, pos.y, pos.z);
    const float4 v4 = s.vel[myOwner];
    const float4 a4 = s.acc[myOwner];
    const float3 vel = make_float3(v4.x, v4.y, v4.z);
    const float3 acc = make_float3(a4.x, a4.y, a4.z);
    const float mass = v4.w;
    const float t = *time;
    const float h = k.h;
    unsigned int newFamily = family_code;
    (void)pos;
    (void)vel;
    (void)acc;
    (void)mass;
    (void)t;
    (void)h;
#include "deme_family_change_rules.inc"
    if (newFamily != family_code) {
        l.w = (unsigned short)newFamily;
        s.loc[myOwner] = l;
    }
}

}  // namespace deme_b200
