// integrate_kernel.cuh -- integrateOwners (src/kernel/DEMIntegrationKernels.cu:46-179) for one owner, as a template
// over the family prescription.
//
// kernels.cu instantiates it with the constant per-family table (TableMotion).  Prescribed motions written as
// expressions of the time are compiled at run time with NVRTC (force_jit.cu) into the same template: a generated
// `switch (family)` assigns the expressions, as the reference's applyPrescribedVel / applyPrescribedPos do with the
// strings that equipFamilyPrescribedMotions pastes into them (src/DEM/APIPrivate.cpp:1005-1048), and every other
// family falls back to the table.  Both builds use --fmad=false, so a family integrates identically in either.
//
// Quaternions are stored as float4 (x = w, y = x, z = y, w = z).
#pragma once
#include "kernels.cuh"

namespace deme_b200 {

// Constant-valued prescriptions from the per-family table.
struct TableMotion {
    const Prescription* presc;

    __device__ __forceinline__ void vel(unsigned int family, float t, float& vX, float& vY, float& vZ, float& omgBarX,
                                        float& omgBarY, float& omgBarZ, bool& LinPrescribed,
                                        bool& RotPrescribed) const {
        (void)t;
        const Prescription& pr = presc[family];
        if (!pr.used) return;
        if (pr.has_vel[0]) vX = pr.vel[0];
        if (pr.has_vel[1]) vY = pr.vel[1];
        if (pr.has_vel[2]) vZ = pr.vel[2];
        if (pr.has_omg[0]) omgBarX = pr.omg[0];
        if (pr.has_omg[1]) omgBarY = pr.omg[1];
        if (pr.has_omg[2]) omgBarZ = pr.omg[2];
        LinPrescribed = pr.lin_vel;
        RotPrescribed = pr.rot_vel;
    }

    __device__ __forceinline__ void pos(unsigned int family, float t, double& X, double& Y, double& Z,
                                        bool& LinPrescribed, bool& RotPrescribed) const {
        (void)t;
        const Prescription& pr = presc[family];
        if (!pr.used) return;
        if (pr.has_pos[0]) X = pr.pos[0];
        if (pr.has_pos[1]) Y = pr.pos[1];
        if (pr.has_pos[2]) Z = pr.pos[2];
        LinPrescribed = pr.lin_pos;
        RotPrescribed = pr.rot_pos;
    }
};

// One owner's step: prescribed or integrated velocities (integrateVel), then the position re-encoded on the voxel
// grid and the quaternion advanced by the exponential map (integratePos).  `t` is the time the prescriptions see.
template <class Motion>
__device__ __forceinline__ void integrate_owner(const SimConsts& k, const StateView& s, uint32_t o, float t,
                                                const Motion& motion) {
    ushort4 l = s.loc[o];
    const unsigned int family = l.w;
    float4 v = s.vel[o];
    float4 w = s.omg[o];
    const float4 a = s.acc[o];
    const float4 al = s.alpha[o];
    const float ovx = v.x, ovy = v.y, ovz = v.z, owx = w.x, owy = w.y, owz = w.z;
    bool linV = false, rotV = false, linP = false, rotP = false;
    motion.vel(family, t, v.x, v.y, v.z, w.x, w.y, w.z, linV, rotV);
    const float h = k.h;
    float ux = 0.f, uy = 0.f, uz = 0.f, qx = 0.f, qy = 0.f, qz = 0.f;
    if (!linV) {
        ux = (a.x + k.G[0]) * h;
        uy = (a.y + k.G[1]) * h;
        uz = (a.z + k.G[2]) * h;
        v.x += ux;
        v.y += uy;
        v.z += uz;
    }
    if (!rotV) {
        qx = al.x * h;
        qy = al.y * h;
        qz = al.z * h;
        w.x += qx;
        w.y += qy;
        w.z += qz;
    }
    float px, py, pz, rx, ry, rz;
    if (k.integrator == DEME_INTEGRATOR_FORWARD_EULER) {
        px = ovx; py = ovy; pz = ovz;
        rx = owx; ry = owy; rz = owz;
    } else if (k.integrator == DEME_INTEGRATOR_CENTERED_DIFFERENCE) {
        px = ovx + ux; py = ovy + uy; pz = ovz + uz;
        rx = owx + qx; ry = owy + qy; rz = owz + qz;
    } else {
        px = ovx + ux * 0.5f; py = ovy + uy * 0.5f; pz = ovz + uz * 0.5f;
        rx = owx + qx * 0.5f; ry = owy + qy * 0.5f; rz = owz + qz * 0.5f;
    }
    double X, Y, Z;
    uint64_t vox = s.voxel[o];
    voxel_to_pos(k, vox, l.x, l.y, l.z, X, Y, Z);
    motion.pos(family, t, X, Y, Z, linP, rotP);
    if (!linP) {
        X += (double)px * (double)h;
        Y += (double)py * (double)h;
        Z += (double)pz * (double)h;
    }
    uint16_t sx, sy, sz;
    pos_to_voxel(k, X, Y, Z, vox, sx, sy, sz);
    l.x = sx;
    l.y = sy;
    l.z = sz;
    float4 q = s.quat[o];
    if (!rotP) {
        double q0 = 1.0, q1 = rx, q2 = ry, q3 = rz;
        const double len = sqrt(q1 * q1 + q2 * q2 + q3 * q3);
        const double theta = 0.5 * (double)h * len;
        if (len > 0) {
            q0 = cos(theta);
            const double sn = sin(theta) / len;
            q1 *= sn;
            q2 *= sn;
            q3 *= sn;
        }
        const float a1 = q.x, b1 = q.y, c1 = q.z, d1 = q.w;
        const float a2 = (float)q0, b2 = (float)q1, c2 = (float)q2, d2 = (float)q3;
        q.x = a1 * a2 - b1 * b2 - c1 * c2 - d1 * d2;
        q.y = a1 * b2 + b1 * a2 + c1 * d2 - d1 * c2;
        q.z = a1 * c2 - b1 * d2 + c1 * a2 + d1 * b2;
        q.w = a1 * d2 + b1 * c2 - c1 * b2 + d1 * a2;
    }
    s.vel[o] = v;
    s.omg[o] = w;
    s.voxel[o] = vox;
    s.loc[o] = l;
    s.quat[o] = q;
}

}  // namespace deme_b200
