// adjoint_law.cuh -- reverse-mode derivative of one contact of the built-in frictional Hertz-Mindlin model, for the
// adjoint of the step (adjoint.cu).  The forward part restates force_model_hertz.cuh in double precision, taking
// the rotational velocities of both bodies at the contact point (ARotCP, BRotCP) as inputs; the reverse part
// propagates the gradients of the contact's force, torque-only force and updated history back to its inputs
// (normal, overlap, both linear and contact-point rotational velocities, the incoming history) and to the pair's
// material parameters (E*, G*, beta, mu, Crr).  Each reverse step is the derivative of the forward line it follows.
#pragma once
#include "device_common.cuh"

namespace deme_b200 {

struct dv3 {
    double x, y, z;
};
__device__ __forceinline__ dv3 mk(double x, double y, double z) { return dv3{x, y, z}; }
__device__ __forceinline__ dv3 operator+(dv3 a, dv3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ dv3 operator-(dv3 a, dv3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ dv3 operator-(dv3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ dv3 operator*(double s, dv3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ void operator+=(dv3& a, dv3 b) { a = a + b; }
__device__ __forceinline__ void operator-=(dv3& a, dv3 b) { a = a - b; }
__device__ __forceinline__ double dot(dv3 a, dv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ dv3 cross(dv3 a, dv3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm(dv3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ dv3 to_dv3(float4 v) { return mk(v.x, v.y, v.z); }

constexpr double kC5 = 1.825741858350554;  // 2 sqrt(5/6)
constexpr double kPi2 = 9.869604401089358;
constexpr double kTiny = 1e-12;

struct LawIn {
    dv3 n;         // unit normal B -> A
    double delta;  // overlap depth
    dv3 vA, vB;    // owner velocities
    dv3 WA, WB;    // rotational velocities at the contact point (w x r of each body)
    dv3 dtan;         // incoming tangential displacement history
    double tau;       // incoming contact duration
    double Es, Gs, be, mu, crr, meff, Rs, h;
    // floors in the derivatives at the law's non-smooth points (0 = exact): overlap relative to R* (the damping's
    // overlap^(1/4)), relative rolling speed (the rolling torque's direction), tangential force (the Coulomb cap)
    double floor_delta_rel, floor_roll_speed, floor_ft;
};

struct LawGrad {
    dv3 n;
    double delta;
    dv3 vA, vB, WA, WB, dtan;
    double tau, Es, Gs, be, mu, crr;
};

// Forward: contact force f, torque-only force t, updated history (dt3, tau2).  Reverse: given g_f, g_t and the
// gradients of the updated history, fills G.
__device__ __forceinline__ void law_vjp(const LawIn& in, dv3 g_f, dv3 g_t, dv3 g_dt3, double g_tau2, dv3& f_out,
                                        dv3& t_out, LawGrad& G) {
    const dv3 n = in.n;
    // ---- forward, keeping what the reverse pass needs ----
    const dv3 WA = in.WA, WB = in.WB;
    const dv3 vr = in.vA + WA - in.vB - WB;
    const double p = dot(vr, n);
    const dv3 vt = vr - p * n;
    const dv3 dt1 = in.dtan + in.h * vt;
    const double q = dot(dt1, n);
    const dv3 dt2 = dt1 - q * n;
    const double tau2 = in.tau + in.h;
    const double s = sqrt(in.delta * in.Rs);
    const double Sn = 2.0 * in.Es * s;
    const double kn = (2.0 / 3.0) * Sn;
    const double ssm = sqrt(Sn * in.meff);
    const double gn = kC5 * in.be * ssm;
    const double fnm = kn * in.delta + gn * p;
    const dv3 fn = fnm * n;
    const double nn = norm(n);  // 1 but for a wall direction rotated by a quaternion off unit length
    const double A = fabs(fnm) * nn;  // the length of the normal force, which sets the cap and the rolling torque
    // rolling resistance once the contact is older than the collision time
    const double Reff = sqrt(in.Rs);
    const double kns = (4.0 / 3.0) * in.Es * sqrt(Reff);
    const double gns = -2.0 * sqrt((5.0 / 3.0) * in.meff * in.Es) * in.be * sqrt(sqrt(Reff));  // Reff^(1/4)
    const double dc = gns / (2.0 * sqrt(kns * in.meff));
    bool roll = in.crr > 0.0;
    if (roll && dc < 1.0) {
        const double tcoll = 3.1415926535897932385 * sqrt(in.meff / (kns * (1.0 - dc * dc)));
        if (tau2 <= tcoll) roll = false;
    }
    const dv3 vroll = WB - WA;
    const double L = norm(vroll);
    roll = roll && L > kTiny;
    const dv3 e = roll ? (1.0 / L) * vroll : mk(0, 0, 0);
    t_out = roll ? (in.crr * A) * e : mk(0, 0, 0);
    // tangential with Coulomb cap
    const double kt = 8.0 * in.Gs * s;
    const double smk = sqrt(in.meff * kt);
    const double gt = -kC5 * in.be * smk;
    const dv3 Ft = (-kt) * dt2 - gt * vt;
    const double ft = norm(Ft);
    const bool big = in.mu > 0.0 && ft > kTiny;
    const bool cap = big && ft > A * in.mu;
    const double rr = cap ? A * in.mu / ft : 1.0;
    const dv3 Ftp = big ? rr * Ft : mk(0, 0, 0);
    f_out = fn + Ftp;

    // ---- reverse ----
    dv3 g_fn = g_f, g_Ftp = g_f;
    dv3 g_dt2 = mk(0, 0, 0), g_vt = mk(0, 0, 0), g_n = mk(0, 0, 0), g_WA = mk(0, 0, 0), g_WB = mk(0, 0, 0);
    double g_kt = 0.0, g_gt = 0.0, g_A = 0.0;
    G.mu = 0.0;
    if (cap) {  // dt3 = (Ftp + gt vt) / (-kt)
        const dv3 X = Ftp + gt * vt;
        g_Ftp -= (1.0 / kt) * g_dt3;
        g_gt += -dot(g_dt3, vt) / kt;
        g_vt += (-gt / kt) * g_dt3;
        g_kt += dot(g_dt3, X) / (kt * kt);
    } else {
        g_dt2 += g_dt3;
    }
    dv3 g_Ft = big ? rr * g_Ftp : mk(0, 0, 0);
    if (cap) {
        const double ftd = fmax(ft, in.floor_ft);
        const double g_rr = dot(g_Ftp, Ft);
        g_A += g_rr * in.mu / ftd;
        G.mu += g_rr * A / ftd;
        const double g_ft = -g_rr * A * in.mu / (ftd * ftd);
        g_Ft += (g_ft / ftd) * Ft;
    }
    g_kt += -dot(g_Ft, dt2);
    g_dt2 += (-kt) * g_Ft;
    g_gt += -dot(g_Ft, vt);
    g_vt += (-gt) * g_Ft;
    const double s_d = fmax(s, in.Rs * sqrt(in.floor_delta_rel));  // s = sqrt(delta R*), floored in derivatives
    const double smk_d = sqrt(in.meff * 8.0 * in.Gs * s_d);
    G.be = g_gt * (-kC5 * smk);
    g_kt += g_gt * (-kC5 * in.be * in.meff / (2.0 * (smk_d > 0.0 ? smk_d : 1.0)));
    G.Gs = 8.0 * s * g_kt;
    double g_s = 8.0 * in.Gs * g_kt;
    G.crr = 0.0;
    if (roll) {  // t = crr A e, e = vroll / |vroll|
        const double ge = dot(g_t, e);
        G.crr = A * ge;
        g_A += in.crr * ge;
        const dv3 g_e = (in.crr * A) * g_t;
        const dv3 g_vroll = (1.0 / fmax(L, in.floor_roll_speed)) * (g_e - dot(g_e, e) * e);
        g_WB += g_vroll;
        g_WA -= g_vroll;
    }
    const double g_fnm = g_A * nn * (fnm > 0.0 ? 1.0 : (fnm < 0.0 ? -1.0 : 0.0)) + dot(g_fn, n);
    g_n += fnm * g_fn + (g_A * fabs(fnm) / nn) * n;
    const double g_kn = g_fnm * in.delta;
    double g_delta = g_fnm * kn;
    const double g_gn = g_fnm * p;
    double g_p = g_fnm * gn;
    const double ssm_d = sqrt(2.0 * in.Es * s_d * in.meff);
    G.be += g_gn * kC5 * ssm;
    const double g_Sn = g_gn * kC5 * in.be * in.meff / (2.0 * (ssm_d > 0.0 ? ssm_d : 1.0)) + (2.0 / 3.0) * g_kn;
    G.Es = 2.0 * s * g_Sn;
    g_s += 2.0 * in.Es * g_Sn;
    g_delta += g_s * in.Rs / (2.0 * (s_d > 0.0 ? s_d : 1.0));
    G.tau = g_tau2;
    dv3 g_dt1 = g_dt2;
    const double g_q = -dot(g_dt2, n);
    g_n += (-q) * g_dt2;
    g_dt1 += g_q * n;
    g_n += g_q * dt1;
    G.dtan = g_dt1;
    g_vt += in.h * g_dt1;
    dv3 g_vr = g_vt;
    g_p += -dot(g_vt, n);
    g_n += (-p) * g_vt;
    g_vr += g_p * n;
    g_n += g_p * vr;
    g_WA += g_vr;
    g_WB -= g_vr;
    G.vA = g_vr;
    G.vB = -g_vr;
    G.WA = g_WA;
    G.WB = g_WB;
    G.n = g_n;
    G.delta = g_delta;
}

}  // namespace deme_b200
