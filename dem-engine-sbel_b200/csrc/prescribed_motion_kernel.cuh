// prescribed_motion_kernel.cuh -- the integration kernel with prescribed motions written as expressions (the
// reference's SetFamilyPrescribedLinVel / SetFamilyPrescribedAngVel / SetFamilyPrescribedPosition strings, which
// equipFamilyPrescribedMotions pastes into applyPrescribedVel / applyPrescribedPos, src/DEM/APIPrivate.cpp:1005-1048
// and src/kernel/DEMIntegrationKernels.cu:5-44).
//
// Compiled only at run time with NVRTC (force_jit.cu).  deme_motion_vel.inc and deme_motion_pos.inc hold one
// `case FAMILY: { <component> = <expression>; ... LinPrescribed = ..; RotPrescribed = ..; break; }` per family.
// An expression sees t (float, the time at the start of the step), family, the components it prescribes (vX, vY,
// vZ, omgBarX, omgBarY, omgBarZ as float; X, Y, Z as double from the domain's lower corner) and deme::PI.  Families
// without expressions read the constant table, so they integrate exactly as in k_integrate.
#pragma once
#include "integrate_kernel.cuh"

namespace deme_b200 {

struct ExpressionMotion {
    TableMotion table;

    __device__ __forceinline__ void vel(unsigned int family, float t, float& vX, float& vY, float& vZ, float& omgBarX,
                                        float& omgBarY, float& omgBarZ, bool& LinPrescribed,
                                        bool& RotPrescribed) const {
        switch (family) {
#include "deme_motion_vel.inc"
            default:
                table.vel(family, t, vX, vY, vZ, omgBarX, omgBarY, omgBarZ, LinPrescribed, RotPrescribed);
        }
    }

    __device__ __forceinline__ void pos(unsigned int family, float t, double& X, double& Y, double& Z,
                                        bool& LinPrescribed, bool& RotPrescribed) const {
        switch (family) {
#include "deme_motion_pos.inc"
            default:
                table.pos(family, t, X, Y, Z, LinPrescribed, RotPrescribed);
        }
    }
};

__global__ void __launch_bounds__(256) k_integrate_motion(SimConsts k, StateView s, const float* time) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= k.n_owners) return;
    if (*k.err != 0u) return;  // a voided step leaves the state as it was
    integrate_owner(k, s, o, *time, ExpressionMotion{TableMotion{s.presc}});
}

}  // namespace deme_b200
