// force_model_hertz.cuh -- the built-in frictional Hertz-Mindlin contact model, restated operation by operation
// from the reference (src/kernel/DEMCustomizablePolicies/FullHertzianForceModel.cu:1-124 with
// matProxy2ContactParam, src/kernel/DEMHelperKernels.cu:316-339).  Every float/double promotion of the reference
// expression is written out explicitly so the result does not depend on compiler contraction.
//
// Inputs are the names the reference exposes to a force model; `force`, `torque_only_force` and the four contact
// wildcards (delta_tan_x/y/z, delta_time) are read-write.
#pragma once
#include "device_common.cuh"

namespace deme_b200 {

struct ContactGeom {
    float3 B2A;          // unit normal from B to A
    double overlapDepth;
    float3 locCPA, locCPB;
    float ARadius, BRadius, AOwnerMass, BOwnerMass;
    float3 ARotCP, BRotCP;  // rotational velocity of the contact point in the global frame: the owner's
                            // orientation applied to cross(omega, local contact point) (rot_cp_velocity)
    float3 ALinVel, BLinVel, ARotVel, BRotVel;
    uint32_t matA, matB;
};

struct MaterialTable {
    const float* E;
    const float* nu;
    const float* CoR;
    const float* mu;
    const float* Crr;
    // contact-pair parameters precomputed by contact_params for every (a, b) (two float4 per pair: E_cnt, G_cnt,
    // CoR_cnt, mu_cnt / Crr_cnt, beta), or null: then they are computed per contact
    const float4* pair = nullptr;
    uint32_t nM = 0;
};

// Contact-pair material parameters from the two materials (matProxy2ContactParam, DEMHelperKernels.cu:316-339):
// effective Young's and shear moduli, the smaller restitution and the larger friction coefficients, with the
// reference's double-precision intermediates.
template <typename T>
__device__ __forceinline__ void mat_proxy(T& E_cnt, T& G_cnt, T& CoR_cnt, T& mu_cnt, T& Crr_cnt, T E_A, T nu_A, T CoR_A,
                                          T mu_A, T Crr_A, T E_B, T nu_B, T CoR_B, T mu_B, T Crr_B) {
    const T invE = (T)((1. - (double)(nu_A * nu_A)) / (double)E_A + (1. - (double)(nu_B * nu_B)) / (double)E_B);
    E_cnt = (T)(1. / (double)invE);
    const T invG = (T)(2. * (2. - (double)nu_A) * (1. + (double)nu_A) / (double)E_A +
                       2. * (2. - (double)nu_B) * (1. + (double)nu_B) / (double)E_B);
    G_cnt = (T)(1. / (double)invG);
    CoR_cnt = CoR_A < CoR_B ? CoR_A : CoR_B;
    mu_cnt = mu_A > mu_B ? mu_A : mu_B;
    Crr_cnt = Crr_A > Crr_B ? Crr_A : Crr_B;
}

// The parameters of a contact between materials a and b that depend on nothing else: matProxy2ContactParam and
// the damping ratio beta = ln e / sqrt(ln^2 e + pi^2) of the pair's restitution coefficient, in the reference's
// precision (FullHertzianForceModel.cu).  The pair table is filled by this same function, so a table entry and an
// inline evaluation are bit-identical.
__device__ __forceinline__ void contact_params(const MaterialTable& m, uint32_t a, uint32_t b, float& E_cnt,
                                               float& G_cnt, float& CoR_cnt, float& mu_cnt, float& Crr_cnt,
                                               float& beta) {
    mat_proxy<float>(E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt, m.E[a], m.nu[a], m.CoR[a], m.mu[a], m.Crr[a], m.E[b],
                     m.nu[b], m.CoR[b], m.mu[b], m.Crr[b]);
    const float loge = (float)(((double)CoR_cnt < kTinyFloat) ? log(kTinyFloat) : (double)logf(CoR_cnt));
    beta = (float)((double)loge / sqrt((double)(loge * loge) + kPiSquared));
}

// kNormalOnly: the frictionless Hertzian model (FrictionlessHertzianForceModel.cu, the reference's
// UseFrictionlessHertzianModel): the same normal spring and damper, no rolling resistance, no tangential force and no
// contact history.  (The reference's file calls a material-proxy helper by a name its helper header does not define,
// mat2ProxyContactParam for matProxy2ContactParam, so its run-time build of that model fails; this is the model the
// file states, with the proxy overload for E and CoR, whose formulas are the full one's.)
template <bool kNormalOnly = false>
__device__ __forceinline__ void hertz_mindlin(const ContactGeom& g, const MaterialTable& m, float ts, float3& force,
                                              float3& torque_only_force, float& delta_tan_x, float& delta_tan_y,
                                              float& delta_tan_z, float& delta_time) {
    // material proxies
    float E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt, beta;
    if (m.pair) {
        const float4* e = m.pair + 2u * ((size_t)g.matA * m.nM + g.matB);
        const float4 p0 = __ldg(e), p1 = __ldg(e + 1);
        E_cnt = p0.x;
        G_cnt = p0.y;
        CoR_cnt = p0.z;
        mu_cnt = p0.w;
        Crr_cnt = p1.x;
        beta = p1.y;
    } else {
        contact_params(m, g.matA, g.matB, E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt, beta);
    }
    const float rAx = g.ARotCP.x, rAy = g.ARotCP.y, rAz = g.ARotCP.z;
    const float rBx = g.BRotCP.x, rBy = g.BRotCP.y, rBz = g.BRotCP.z;
    const float nX = g.B2A.x, nY = g.B2A.y, nZ = g.B2A.z;
    // normal part and history update
    const float vx = (g.ALinVel.x + rAx) - (g.BLinVel.x + rBx);
    const float vy = (g.ALinVel.y + rAy) - (g.BLinVel.y + rBy);
    const float vz = (g.ALinVel.z + rAz) - (g.BLinVel.z + rBz);
    const float proj = vx * nX + vy * nY + vz * nZ;
    const float vtx = vx - proj * nX, vty = vy - proj * nY, vtz = vz - proj * nZ;
    float dtx = delta_tan_x + ts * vtx, dty = delta_tan_y + ts * vty, dtz = delta_tan_z + ts * vtz;
    const float dproj = dtx * nX + dty * nY + dtz * nZ;
    dtx -= dproj * nX;
    dty -= dproj * nY;
    dtz -= dproj * nZ;
    delta_time += ts;
    const float mass_eff = (g.AOwnerMass * g.BOwnerMass) / (g.AOwnerMass + g.BOwnerMass);
    const float sqrt_Rd = (float)sqrt(g.overlapDepth * (double)(g.ARadius * g.BRadius) /
                                      (double)(g.ARadius + g.BRadius));
    const float Sn = (float)(2. * (double)E_cnt * (double)sqrt_Rd);
    const float k_n = (float)(kTwoOverThree * (double)Sn);
    const float gamma_n = (float)(kTwoTimesSqrtFiveOverSix * (double)beta * (double)sqrtf(Sn * mass_eff));
    const float scal = (float)((double)k_n * g.overlapDepth + (double)(gamma_n * proj));
    force.x += scal * nX;
    force.y += scal * nY;
    force.z += scal * nZ;
    if (kNormalOnly) return;
    // rolling resistance
    if ((double)Crr_cnt > 0.0) {
        bool add_rr = true;
        const float R_eff = sqrtf((g.ARadius * g.BRadius) / (g.ARadius + g.BRadius));
        const float kn_simple = (float)(kFourOverThree * (double)E_cnt * (double)sqrtf(R_eff));
        const float gn_simple =
            -2.f * sqrtf((float)(kFiveOverThree * (double)mass_eff * (double)E_cnt)) * beta * powf(R_eff, 0.25f);
        const float d_coeff = gn_simple / (2.f * sqrtf(kn_simple * mass_eff));
        if ((double)d_coeff < 1.0) {
            const float t_coll = (float)(kPi * (double)sqrtf(mass_eff / (kn_simple * (1.f - d_coeff * d_coeff))));
            if (delta_time <= t_coll) add_rr = false;
        }
        if (add_rr) {
            const float vrx = rBx - rAx, vry = rBy - rAy, vrz = rBz - rAz;
            const float vmag = sqrtf(vrx * vrx + vry * vry + vrz * vrz);
            if ((double)vmag > kTinyFloat) {
                const float s = Crr_cnt * sqrtf(force.x * force.x + force.y * force.y + force.z * force.z);
                torque_only_force.x = (vrx / vmag) * s;
                torque_only_force.y = (vry / vmag) * s;
                torque_only_force.z = (vrz / vmag) * s;
            }
        }
    }
    // tangential part with Coulomb cap
    if ((double)mu_cnt > 0.0) {
        const float kt = (float)(8. * (double)G_cnt * (double)sqrt_Rd);
        const float gt = (float)(-kTwoTimesSqrtFiveOverSix * (double)beta * (double)sqrtf(mass_eff * kt));
        const float nkt = -kt;
        float tfx = nkt * dtx - gt * vtx, tfy = nkt * dty - gt * vty, tfz = nkt * dtz - gt * vtz;
        const float ft = sqrtf(tfx * tfx + tfy * tfy + tfz * tfz);
        if ((double)ft > kTinyFloat) {
            const float ft_max = sqrtf(force.x * force.x + force.y * force.y + force.z * force.z) * mu_cnt;
            if (ft > ft_max) {
                const float r = ft_max / ft;
                tfx = r * tfx;
                tfy = r * tfy;
                tfz = r * tfz;
                dtx = (tfx + gt * vtx) / nkt;
                dty = (tfy + gt * vty) / nkt;
                dtz = (tfz + gt * vtz) / nkt;
            }
        } else {
            tfx = tfy = tfz = 0.f;
        }
        force.x += tfx;
        force.y += tfy;
        force.z += tfz;
    }
    delta_tan_x = dtx;
    delta_tan_y = dty;
    delta_tan_z = dtz;
}

}  // namespace deme_b200
