// adjoint.cu -- adjoint of the DEM step for clumps and spheres with analytical walls (no reference counterpart).
//
// deme_adjoint_record runs the forward steps and keeps a checkpoint (owner state and the current contact list with
// its history) every K steps.  deme_adjoint_backward walks the checkpoints from the last: it restores one,
// recomputes its K steps with the production kernels while recording each step's state, angular accelerations and
// contact list, then runs the reverse pass over those steps.  Per step the contact set is the one the forward pass
// found, held fixed.  The reverse pass is
//   * k_adj_integrate: the Extended Taylor update (src/kernel/DEMIntegrationKernels.cu:46-179) reversed per owner:
//     x' = x + h v + h^2/2 a, v' = v + h a with a = F/m + g; w' = w + h alpha and q' = q (x) exp(h (w + h alpha/2))
//     with alpha = T / I from the owner-frame torque T (forceToAngAcc, src/kernel/DEMCollectForceKernels.cu:68-120).
//     It turns the state gradients into the gradients of the owner's summed force and owner-frame torque, and
//     gives the direct part of the step-start state gradients (orientation included);
//   * k_adj_contact: per contact, the derivative of the built-in frictional Hertz-Mindlin law (adjoint_law.cuh) and
//     of its geometry -- sphere centres X + R(q) r of clump members, the wall geometry of planes, cylinders and
//     cones (adjoint_rigid.cuh), lever arms and their owner-frame images, contact-point velocities R(q) (w x s),
//     owner-frame torques -- scattered onto both owners' position, velocity, quaternion and angular-velocity
//     gradients (summed per owner within a warp first), the gradient of the incoming history, and the
//     material-parameter gradients (FP64 accumulators);
//   * k_adj_hist_scatter: the history map (src/kernel/DEMHistoryMappingKernels.cu) reversed, so the incoming-history
//     gradient reaches the previous step's updated history.
// The state carried is the stored one: position, velocity, quaternion and owner-frame angular velocity.  At the
// interface angular velocities are in the world frame and quaternion gradients hold the world angular velocity
// fixed (k_adj_seed, k_adj_result).  Owners of prescribed families are driven: their recorded motion enters the
// contacts, and their gradients are 0.  The model is evaluated from the recorded FP32 state (sphere centres and
// wall placements formed as the forward step forms them); the state gradients are carried and accumulated in FP64
// (they sum many contributions of both signs), as are the material-parameter gradients.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "adjoint_rigid.cuh"
#include "handle.cuh"
#include "profiler.cuh"

using namespace deme_b200;

// struct Checkpoint: handle.cuh

// Per material, the terms matProxy2ContactParam (src/kernel/DEMHelperKernels.cu:316-339) combines per pair, in
// double: E* = 1 / (tE_A + tE_B), G* = 1 / (tG_A + tG_B), the damping ratio beta of a restitution coefficient and
// its derivative, and the derivatives dE = d tE / d(-E), dG = d tG / d(-E) for the material gradients.
struct MatAdj {
    double tE, tG, dE, dG, cor, be, dbe, mu, crr;
};

struct AdjointTape {
    int K = 0;
    int nSteps = 0;
    std::vector<Checkpoint> cps;  // cps[j]: state before step j*K
    Checkpoint fin;               // state after the last step
    // one segment of recorded steps
    double* X = nullptr;   // K x nO x 3 positions (world, relative to the domain corner)
    float4* V = nullptr;   // K x nO velocities
    float4* Q = nullptr;   // K x nO quaternions
    float4* W = nullptr;   // K x nO angular velocities (owner frame)
    float4* Al = nullptr;  // K x nO angular accelerations (owner frame) of the step's forces
    uint32_t poolCap = 0;
    uint32_t* cA = nullptr;
    uint32_t* cB = nullptr;
    uint8_t* cT = nullptr;
    float4* cH = nullptr;
    uint32_t* cM = nullptr;
    std::vector<uint32_t> stepN, stepBase;
    // reverse-pass buffers: 3 per owner, 4 for the quaternions
    double *lx = nullptr, *lv = nullptr, *lw = nullptr, *nlx = nullptr, *nlv = nullptr, *nlw = nullptr;
    double *lq = nullptr, *nlq = nullptr;
    double *lF = nullptr, *lT = nullptr;
    uint32_t gCap = 0;
    float4 *gA = nullptr, *gB = nullptr, *gC = nullptr;  // history gradients (current, previous, carried)
    double* gmat = nullptr;                             // nM x 4
    MatAdj* matAdj = nullptr;                           // nM per-material terms of the pair parameters
    double floors[3] = {1e-4, 1e-4, 1e-6};              // see deme_adjoint_set_floors
    uint32_t nO = 0;                                    // owners the per-owner buffers are sized for
    uint32_t maxN = 0;                                  // largest contact count seen at the checkpoints
};

namespace {

inline unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// State of every owner at a step start: position (double, kernel literals), velocity, quaternion, owner-frame
// angular velocity.
__global__ void k_adj_record_state(SimConsts k, StateView s, uint32_t nO, double* X, float4* V, float4* Q,
                                   float4* W) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nO) return;
    const ushort4 l = s.loc[o];
    double x, y, z;
    voxel_to_pos(k, s.voxel[o], l.x, l.y, l.z, x, y, z);
    X[3 * (size_t)o] = x;
    X[3 * (size_t)o + 1] = y;
    X[3 * (size_t)o + 2] = z;
    V[o] = s.vel[o];
    Q[o] = s.quat[o];
    W[o] = s.omg[o];
}

// Free owners are the clumps of families without a prescription; the scene check admits no partly prescribed one.
__device__ __forceinline__ bool owner_free(const StateView& s, uint32_t o, uint32_t nClumps) {
    return o < nClumps && !s.presc[s.loc[o].w].used;
}

__device__ __forceinline__ void add3(double* a, uint32_t o, dv3 g) {
    atomicAdd(a + 3 * (size_t)o, g.x);
    atomicAdd(a + 3 * (size_t)o + 1, g.y);
    atomicAdd(a + 3 * (size_t)o + 2, g.z);
}
__device__ __forceinline__ void add4(double* a, uint32_t o, const dq4& g) {
    atomicAdd(a + 4 * (size_t)o, g.w);
    atomicAdd(a + 4 * (size_t)o + 1, g.u.x);
    atomicAdd(a + 4 * (size_t)o + 2, g.u.y);
    atomicAdd(a + 4 * (size_t)o + 3, g.u.z);
}
__device__ __forceinline__ dv3 ld3(const double* a, uint32_t o) {
    return mk(a[3 * (size_t)o], a[3 * (size_t)o + 1], a[3 * (size_t)o + 2]);
}
__device__ __forceinline__ dq4 ld4(const double* a, uint32_t o) {
    return dq4{a[4 * (size_t)o], mk(a[4 * (size_t)o + 1], a[4 * (size_t)o + 2], a[4 * (size_t)o + 3])};
}
__device__ __forceinline__ void st3(double* a, uint32_t o, dv3 g) {
    a[3 * (size_t)o] = g.x;
    a[3 * (size_t)o + 1] = g.y;
    a[3 * (size_t)o + 2] = g.z;
}
__device__ __forceinline__ void st4(double* a, uint32_t o, const dq4& g) {
    a[4 * (size_t)o] = g.w;
    a[4 * (size_t)o + 1] = g.u.x;
    a[4 * (size_t)o + 2] = g.u.y;
    a[4 * (size_t)o + 3] = g.u.z;
}

// Reverse of one owner's step (the forward form is in the file header).  In: the gradients of the step-end state
// (lx, lv, lq, lw: position, velocity, quaternion, owner-frame angular velocity) and the recorded step-start
// quaternion, angular velocity and angular acceleration.  Out: the gradients of the owner's summed force (lF,
// world) and torque (lT, owner frame), and the direct part of the step-start state gradients.
__global__ void k_adj_integrate(StateView s, uint32_t nO, uint32_t nClumps, double h, const float4* Q,
                                const float4* W, const float4* Al, const double* lx, const double* lv,
                                const double* lq, const double* lw, double* lF, double* lT, double* nlx,
                                double* nlv, double* nlq, double* nlw) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nO) return;
    const dv3 zero = mk(0, 0, 0);
    if (!owner_free(s, o, nClumps)) {
        st3(lF, o, zero);
        st3(lT, o, zero);
        st3(nlx, o, zero);
        st3(nlv, o, zero);
        st3(nlw, o, zero);
        st4(nlq, o, dq4{0.0, zero});
        return;
    }
    const double m = s.vel[o].w;
    const float4 Mi = s.moi[o];
    const dv3 gx = ld3(lx, o), gv = ld3(lv, o), gw = ld3(lw, o);
    const dq4 gq = ld4(lq, o);
    // translation
    const dv3 ga = (0.5 * h * h) * gx + h * gv;
    st3(lF, o, (1.0 / m) * ga);
    st3(nlx, o, gx);
    st3(nlv, o, gv + h * gx);
    // rotation: r = w + h alpha / 2, p = exp(h r), q' = q (x) p, w' = w + h alpha
    const dq4 q = to_dq4(Q[o]);
    const float4 wf = W[o], af = Al[o];
    const dv3 w = mk(wf.x, wf.y, wf.z), al = mk(af.x, af.y, af.z);
    const dv3 r = w + (0.5 * h) * al;
    const double L = norm(r), th = 0.5 * h * L;
    dq4 p{1.0, zero};
    if (L > 0.0) p = dq4{cos(th), (sin(th) / L) * r};
    dq4 gq0, gp;
    qmul_vjp(q, p, gq, gq0, gp);
    const dv3 gr = qexp_vjp(r, h, gp);
    const dv3 gal = h * gw + (0.5 * h) * gr;
    st3(lT, o, mk(gal.x / Mi.x, gal.y / Mi.y, gal.z / Mi.z));
    st3(nlw, o, gw + gr);
    st4(nlq, o, gq0);
}

// The seed's angular-velocity gradient from the world frame to the owner frame, at the final state: w_world =
// R(q) w, so dL/dw = R(q)^T dL/dw_world and dL/dq gains the derivative of R(q) w.
__global__ void k_adj_seed(uint32_t nO, const float4* Q, const float4* W, double* lq, double* lw) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nO) return;
    const dq4 q = to_dq4(Q[o]);
    const float4 wf = W[o];
    const dv3 gW = ld3(lw, o);
    st3(lw, o, qrot_t(q, gW));
    dq4 gq = ld4(lq, o);
    gq += qrot_vjp(q, mk(wf.x, wf.y, wf.z), gW);
    st4(lq, o, gq);
}

// The result at the window start in the interface's variables: w = R(q)^T w_world, so dL/dw_world = R(q) dL/dw
// and the quaternion gradient at fixed w_world gains the derivative of R(q)^T w_world.  Driven owners get 0.
__global__ void k_adj_result(StateView s, uint32_t nO, uint32_t nClumps, const float4* Q, const float4* W,
                             double* lx, double* lv, double* lq, double* lw) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nO) return;
    const dv3 zero = mk(0, 0, 0);
    if (!owner_free(s, o, nClumps)) {
        st3(lx, o, zero);
        st3(lv, o, zero);
        st3(lw, o, zero);
        st4(lq, o, dq4{0.0, zero});
        return;
    }
    const dq4 q = to_dq4(Q[o]);
    const float4 wf = W[o];
    const dv3 gw = ld3(lw, o);
    const dv3 wW = qrot(q, mk(wf.x, wf.y, wf.z));
    st3(lw, o, qrot(q, gw));
    dq4 gq = ld4(lq, o);
    gq += qrot_vjp(q, gw, wW);
    st4(lq, o, gq);
}

__device__ __forceinline__ double dbeta_de(double e) {
    e = e > kTiny ? e : kTiny;
    const double le = log(e);
    const double d = le * le + kPi2;
    return (1.0 / e) * kPi2 / (d * sqrt(d));
}

__global__ void k_adj_mat_table(MaterialTable m, uint32_t nM, MatAdj* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nM) return;
    const double E = m.E[i], nu = m.nu[i], cor = m.CoR[i];
    MatAdj a;
    a.tE = (1.0 - nu * nu) / E;
    a.tG = 2.0 * (2.0 - nu) * (1.0 + nu) / E;
    a.dE = a.tE / E;
    a.dG = a.tG / E;
    a.cor = cor;
    const double le = log(cor > kTiny ? cor : kTiny);
    a.be = le / sqrt(le * le + kPi2);
    a.dbe = dbeta_de(cor);
    a.mu = m.mu[i];
    a.crr = m.Crr[i];
    out[i] = a;
}

// A sphere's offset from its owner as the forward step forms it: rotated in float (rot_f), then added in double.
__device__ __forceinline__ dv3 sphere_offset(float4 sp, float4 q) {
    float rx = sp.x, ry = sp.y, rz = sp.z;
    rot_f(rx, ry, rz, q.x, q.y, q.z, q.w);
    return mk(rx, ry, rz);
}

// One side's owner gradients (position 3, velocity 3, owner-frame angular velocity 3, quaternion 4) of every lane of
// a warp, summed per owner among the lanes that share it (a clump's contacts are adjacent in the list, and its
// neighbours recur) and added to the accumulators with one set of FP64 atomics per owner.  All 32 lanes call it;
// `key` is the owner, or kNoOwner for a lane with nothing to add.
constexpr uint32_t kNoOwner = 0xFFFFFFFFu;
constexpr int kOwnerGrad = 13;
__device__ __forceinline__ void warp_owner_add(const double (&v)[kOwnerGrad], uint32_t key, double* sw, double* nlx,
                                               double* nlv, double* nlw, double* nlq) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int c = 0; c < kOwnerGrad; c++) sw[c * 32 + lane] = v[c];
    __syncwarp();
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    if (key != kNoOwner && lane == (uint32_t)(__ffs(peers) - 1)) {
        double a[kOwnerGrad];
#pragma unroll
        for (int c = 0; c < kOwnerGrad; c++) a[c] = 0.0;
        for (uint32_t m = peers; m; m &= m - 1u) {
            const uint32_t b = (uint32_t)(__ffs(m) - 1);
#pragma unroll
            for (int c = 0; c < kOwnerGrad; c++) a[c] += sw[c * 32 + b];
        }
        add3(nlx, key, mk(a[0], a[1], a[2]));
        add3(nlv, key, mk(a[3], a[4], a[5]));
        add3(nlw, key, mk(a[6], a[7], a[8]));
        add4(nlq, key, dq4{a[9], mk(a[10], a[11], a[12])});
    }
    __syncwarp();
}
__device__ __forceinline__ void put_owner_grad(double (&v)[kOwnerGrad], dv3 x, dv3 vel, dv3 w, const dq4& q) {
    v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = vel.x, v[4] = vel.y, v[5] = vel.z, v[6] = w.x, v[7] = w.y, v[8] = w.z;
    v[9] = q.w, v[10] = q.u.x, v[11] = q.u.y, v[12] = q.u.z;
}

// Per contact of one recorded step: the law's derivative, scattered to both owners and to the material gradients.
// Geometry (checkSpheresOverlap / checkSphereEntityOverlap forms, src/kernel/DEMHelperKernels.cu:233-264, 394-445):
//   sphere pair:  c = X + R(q) r per side, d = cA - cB, D = |d|, n = d / D, delta = rA + rB - D,
//                 CP = cB + (rB - delta / 2) n;
//   wall:         gap, n at cA (wall_geom), delta = (rA - gap) / 2, CP = cA - n (gap + rA) / 2;
//   lever arms rAv = CP - XA, rBv = CP - XB, taken to the owner frames as s = R(q)^T r.
// As the forward step forms them (force_kernel.cuh): the rotational velocity at the contact point is R(q) (w x s)
// per body, and the owner-frame torques are sA x R(qA)^T (f + t) and sB x R(qB)^T -(f + t) (t: the torque-only
// force); lT carries the gradients of the owners' summed owner-frame torques.
// 128 threads, 5 blocks per SM: the register cap (102) spills to local memory, which costs less than running one
// block of 256 per SM at the kernel's natural 255 registers (turning drum, 100k clumps: 0.22 against 0.32 ms per
// step; 256 x 2 and 256 x 3 gave 0.25 and 0.24).
constexpr uint32_t kAdjContactThreads = 128;
__global__ void __launch_bounds__(kAdjContactThreads, 5) k_adj_contact(SimConsts k, StateView s, const MatAdj* matAdj,
                                                        const AnalRaw* raw, uint32_t n,
                                                     uint32_t nM, const uint32_t* cA, const uint32_t* cB,
                                                     const uint8_t* cT, const float4* cH, const double* X,
                                                     const float4* V, const float4* Q, const float4* W,
                                                     const double* lF, const double* lT, const float4* gHout,
                                                     float4* gHin, double* nlx, double* nlv, double* nlq, double* nlw,
                                                     double* gmat, double3 floors) {
    extern __shared__ double s_g[];  // nM x (E, CoR, mu, Crr), then kOwnerGrad x 32 per warp for warp_owner_add
    for (uint32_t t = threadIdx.x; t < 4u * nM; t += blockDim.x) s_g[t] = 0.0;
    double* s_w = s_g + 4u * nM + (threadIdx.x >> 5) * (kOwnerGrad * 32);
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double va[kOwnerGrad], vb[kOwnerGrad];
    uint32_t keyA = kNoOwner, keyB = kNoOwner;
    if (i < n) {
        const uint32_t sA = cA[i], bId = cB[i];
        const bool ss = cT[i] == DEME_SPHERE_SPHERE_CONTACT;
        bool ok = index_ok(k.err, 20, sA, k.n_spheres) && index_ok(k.err, 21, bId, ss ? k.n_spheres : k.n_anal);
        float4 gin = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ok) {
            const uint32_t oA = s.sOwner[sA];
            const float4 spA = s.sph[sA], qfA = Q[oA], wfA = W[oA];
            const dq4 qA = to_dq4(qfA);
            const dv3 XA = ld3(X, oA), wbA = mk(wfA.x, wfA.y, wfA.z);
            const dv3 cAc = XA + sphere_offset(spA, qfA);
            const double rA = (double)spA.w;
            const double mA = (double)s.vel[oA].w;
            const uint32_t matA = s.sMat[sA];
            LawIn in;
            dv3 in_rAv = mk(0, 0, 0), in_rBv = mk(0, 0, 0);
            uint32_t oB = 0, matB = 0;
            float4 spB = make_float4(0.f, 0.f, 0.f, 0.f), qfB = make_float4(1.f, 0.f, 0.f, 0.f);
            double rB = 0.0, mB = 1.0, D = 1.0, bb = 0.0, kk = 0.0;
            dv3 nrm = mk(0, 0, 0), XB = mk(0, 0, 0);
            WallGeom wg;
            bool active = false;
            if (ss) {
                oB = s.sOwner[bId];
                spB = s.sph[bId];
                qfB = Q[oB];
                XB = ld3(X, oB);
                const dv3 cBc = XB + sphere_offset(spB, qfB);
                rB = (double)spB.w;
                mB = (double)s.vel[oB].w;
                matB = s.sMat[bId];
                const dv3 d = cAc - cBc;
                D = norm(d);
                active = D <= rA + rB && D > 0.0;
                if (active) {
                    nrm = (1.0 / D) * d;
                    in.delta = rA + rB - D;
                    bb = rB - in.delta / 2.0;
                    const dv3 CP = cBc + bb * nrm;
                    in_rAv = CP - XA;
                    in_rBv = CP - XB;
                }
            } else {
                const AnalRaw ar = raw[bId];
                oB = ar.owner;
                qfB = Q[oB];
                XB = ld3(X, oB);
                // the wall placed as k_place_anal places it: reference point and direction rotated in float
                float px = ar.relX, py = ar.relY, pz = ar.relZ, dx = ar.rotX, dy = ar.rotY, dz = ar.rotZ;
                rot_f(px, py, pz, qfB.x, qfB.y, qfB.z, qfB.w);
                rot_f(dx, dy, dz, qfB.x, qfB.y, qfB.z, qfB.w);
                const dv3 P = XB + mk(px, py, pz), dir = mk(dx, dy, dz);
                rB = (double)1e15f;
                mB = (double)ar.mass;
                matB = ar.material;
                if (wall_geom(ar.type, ar.normal, (double)ar.size1, ar.c1, ar.c2, (double)ar.size2, (double)ar.size3, P,
                              dir, cAc, wg)) {
                    in.delta = (rA - wg.gap) / 2.0;
                    active = in.delta >= 0.0;
                    nrm = wg.n;
                    kk = (wg.gap + rA) / 2.0;
                    const dv3 CP = cAc - kk * nrm;
                    in_rAv = CP - XA;
                    in_rBv = CP - XB;
                }
            }
            if (active) {
                const float4 wfB = W[oB];
                const dv3 wbB = mk(wfB.x, wfB.y, wfB.z);
                const dq4 qB = to_dq4(qfB);
                const dv3 rAv = in_rAv, rBv = in_rBv;
                const dv3 sA = qrot_t(qA, rAv), sB = qrot_t(qB, rBv);
                in.n = nrm;
                in.vA = to_dv3(V[oA]);
                in.vB = to_dv3(V[oB]);
                in.WA = qrot(qA, cross(wbA, sA));
                in.WB = qrot(qB, cross(wbB, sB));
                const float4 hi = cH[i];
                in.dtan = mk(hi.x, hi.y, hi.z);
                in.tau = hi.w;
                in.meff = mA * mB / (mA + mB);
                in.Rs = rA * rB / (rA + rB);
                in.h = (double)k.h;
                in.floor_delta_rel = floors.x;
                in.floor_roll_speed = floors.y;
                in.floor_ft = floors.z;
                const MatAdj MA = matAdj[matA], MB = matAdj[matB];
                in.Es = 1.0 / (MA.tE + MB.tE);
                in.Gs = 1.0 / (MA.tG + MB.tG);
                const uint32_t corSrc = MA.cor < MB.cor ? matA : matB;
                in.be = MA.cor < MB.cor ? MA.be : MB.be;
                const double dbe = MA.cor < MB.cor ? MA.dbe : MB.dbe;
                in.mu = MA.mu > MB.mu ? MA.mu : MB.mu;
                const uint32_t muSrc = MA.mu > MB.mu ? matA : matB;
                in.crr = MA.crr > MB.crr ? MA.crr : MB.crr;
                const uint32_t crSrc = MA.crr > MB.crr ? matA : matB;
                // upstream gradients: forces (world) and owner-frame torques of both owners (driven owners carry 0)
                const dv3 gFA = ld3(lF, oA), gTA = ld3(lT, oA);
                const dv3 gFB = ss ? ld3(lF, oB) : mk(0, 0, 0), gTB = ss ? ld3(lT, oB) : mk(0, 0, 0);
                // torque sA x R^T u: its gradient with respect to u (= f + t) is R (gT x sA)
                const dv3 g_u = qrot(qA, cross(gTA, sA)) - qrot(qB, cross(gTB, sB));
                const float4 gho = gHout ? gHout[i] : make_float4(0.f, 0.f, 0.f, 0.f);
                dv3 f, t;
                LawGrad G;
                law_vjp(in, gFA - gFB + g_u, g_u, mk(gho.x, gho.y, gho.z), gho.w, f, t, G);
                const dv3 u = f + t;
                // A side: torque sA x bA (bA = R^T u) and contact-point velocity R (wA x sA), back to sA, wA, qA
                const dv3 bA = qrot_t(qA, u);
                dv3 g_sA = cross(bA, gTA);
                const dv3 gbA = cross(gTA, sA);
                dq4 gqA = qrot_vjp(qA, gbA, u);
                const dv3 gcA_ = qrot_t(qA, G.WA);
                gqA += qrot_vjp(qA, cross(wbA, sA), G.WA);
                const dv3 g_wbA = cross(sA, gcA_);
                g_sA += cross(gcA_, wbA);
                const dv3 g_rAv = qrot(qA, g_sA);  // sA = R^T rAv
                gqA += qrot_vjp(qA, g_sA, rAv);
                // B side likewise (torque -u); for a wall only the lever arm's path counts (its owner is driven)
                const dv3 gcB_ = qrot_t(qB, G.WB);
                dv3 g_sB = cross(gcB_, wbB);
                dq4 gqB = qrot_vjp(qB, cross(wbB, sB), G.WB);
                const dv3 g_wbB = cross(sB, gcB_);
                if (ss) {
                    const dv3 bB = qrot_t(qB, -u);
                    g_sB += cross(bB, gTB);
                    const dv3 gbB = cross(gTB, sB);
                    gqB += qrot_vjp(qB, gbB, -u);
                }
                const dv3 g_rBv = qrot(qB, g_sB);
                gqB += qrot_vjp(qB, g_sB, rBv);
                // geometry reversed: contact point, normal and depth back to the sphere centres and the owners
                const dv3 gCP = g_rAv + g_rBv;
                dv3 gcA;
                if (ss) {
                    const double g_delta = G.delta - 0.5 * dot(gCP, nrm);
                    const dv3 g_n = G.n + bb * gCP;
                    const dv3 g_d = (1.0 / D) * (g_n - dot(g_n, nrm) * nrm) + (-g_delta) * nrm;
                    gcA = g_d;
                    const dv3 gcB = gCP - g_d;
                    // owner B: its position directly and through its sphere centre, its offset's rotation
                    if (spB.x != 0.f || spB.y != 0.f || spB.z != 0.f) gqB += qrot_vjp(qB, mk(spB.x, spB.y, spB.z), gcB);
                    put_owner_grad(vb, gcB - g_rBv, G.vB, g_wbB, gqB);
                    keyB = oB;
                } else {
                    const double g_kk = -dot(gCP, nrm);
                    const dv3 g_n = G.n - kk * gCP;
                    const double g_gap = -0.5 * G.delta + 0.5 * g_kk;
                    gcA = gCP + wall_geom_vjp(wg, g_gap, g_n);
                }
                if (spA.x != 0.f || spA.y != 0.f || spA.z != 0.f) gqA += qrot_vjp(qA, mk(spA.x, spA.y, spA.z), gcA);
                put_owner_grad(va, gcA - g_rAv, G.vA, g_wbA, gqA);
                keyA = oA;
                gin = make_float4((float)G.dtan.x, (float)G.dtan.y, (float)G.dtan.z, (float)G.tau);
                // material parameters (matProxy2ContactParam's derivatives)
                const double Es2 = in.Es * in.Es, Gs2 = in.Gs * in.Gs;
                atomicAdd(&s_g[4 * matA], G.Es * Es2 * MA.dE + G.Gs * Gs2 * MA.dG);
                atomicAdd(&s_g[4 * matB], G.Es * Es2 * MB.dE + G.Gs * Gs2 * MB.dG);
                atomicAdd(&s_g[4 * corSrc + 1], G.be * dbe);
                atomicAdd(&s_g[4 * muSrc + 2], G.mu);
                atomicAdd(&s_g[4 * crSrc + 3], G.crr);
            }
        }
        gHin[i] = gin;
    }
    if (keyA == kNoOwner)
        for (int c = 0; c < kOwnerGrad; c++) va[c] = 0.0;
    if (keyB == kNoOwner)
        for (int c = 0; c < kOwnerGrad; c++) vb[c] = 0.0;
    warp_owner_add(va, keyA, s_w, nlx, nlv, nlw, nlq);
    warp_owner_add(vb, keyB, s_w, nlx, nlv, nlw, nlq);
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < 4u * nM; t += blockDim.x)
        if (s_g[t] != 0.0) atomicAdd(&gmat[t], s_g[t]);
}

// The history map reversed: the incoming-history gradient of a contact goes to its partner in the previous list.
__global__ void k_adj_hist_scatter(uint32_t n, const uint32_t* map, const float4* gHin, float4* gPrev, uint32_t nPrev,
                                   uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t m = map[i];
    if (m != DEME_NULL_MAPPING_PARTNER && index_ok(err, 22, m, nPrev)) gPrev[m] = gHin[i];
}

// Re-indexes history gradients from one list (CSR offsets `off` by sphere) to another holding the same contacts
// (the list a checkpoint stored and the one recomputed from it can differ in order or, rarely, in members).
__global__ void k_adj_rekey(uint32_t n, const uint32_t* A, const uint32_t* B, const uint8_t* T, const uint32_t* off,
                            const uint32_t* oB, const uint8_t* oT, uint32_t nOld, const float4* gOld, float4* gNew,
                            uint32_t nS, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t a = A[i];
    if (index_ok(err, 23, a, nS)) {
        uint32_t lo = off[a], hi = off[a + 1];
        if (hi > nOld) hi = nOld;
        const uint64_t key = ((uint64_t)(T[i] == DEME_SPHERE_SPHERE_CONTACT ? 1u : 0u) << 32) | B[i];
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            const uint64_t km = ((uint64_t)(oT[mid] == DEME_SPHERE_SPHERE_CONTACT ? 1u : 0u) << 32) | oB[mid];
            if (km < key)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo < min(off[a + 1], nOld) && oB[lo] == B[i] && oT[lo] == T[i]) g = gOld[lo];
    }
    gNew[i] = g;
}

}  // namespace

// ------------------------------------------------------------------------------------------------------ host ----

int32_t alloc_checkpoint(deme_handle* h, Checkpoint& c, uint32_t nContacts) {
    if (!c.voxel) {
        TRY(dalloc_n(h, &c.voxel, h->nO));
        TRY(dalloc_n(h, &c.loc, h->nO));
        TRY(dalloc_n(h, &c.quat, h->nO));
        TRY(dalloc_n(h, &c.vel, h->nO));
        TRY(dalloc_n(h, &c.omg, h->nO));
        TRY(dalloc_n(h, &c.off, (size_t)h->nS + 1));
    }
    if (nContacts > c.cap || !c.idA) {
        dfree(h, c.idA);
        dfree(h, c.idB);
        dfree(h, c.type);
        dfree(h, c.hist);
        c.idA = c.idB = nullptr;
        c.type = nullptr;
        c.hist = nullptr;
        const uint32_t cap = std::max<uint32_t>(nContacts + nContacts / 8 + 64, 64u);
        TRY(dalloc_n(h, &c.idA, cap));
        TRY(dalloc_n(h, &c.idB, cap));
        TRY(dalloc_n(h, &c.type, cap));
        TRY(dalloc_n(h, &c.hist, cap));
        c.cap = cap;
    }
    return DEME_OK;
}

void free_checkpoint(deme_handle* h, Checkpoint& c) {
    for (void* p : {(void*)c.voxel, (void*)c.loc, (void*)c.quat, (void*)c.vel, (void*)c.omg, (void*)c.off,
                    (void*)c.idA, (void*)c.idB, (void*)c.type, (void*)c.hist})
        dfree(h, p);
    c = Checkpoint{};
}

int32_t save_checkpoint(deme_handle* h, Checkpoint& c) {
    TRY(refresh_count(h));
    const uint32_t n = h->nContacts;
    TRY(alloc_checkpoint(h, c, n));
    cudaStream_t st = h->st_dt;
    const ContactBuf& L = h->lists[h->cur];
    CUDA_TRY(h, cudaMemcpyAsync(c.voxel, h->voxel, h->nO * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(c.loc, h->loc, h->nO * sizeof(ushort4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(c.quat, h->quat, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(c.vel, h->vel, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(c.omg, h->omg, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    if (n) {
        CUDA_TRY(h, cudaMemcpyAsync(c.idA, L.idA, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(c.idB, L.idB, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(c.type, L.type, n * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(c.hist, L.hist, n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    }
    CUDA_TRY(h, cudaMemcpyAsync(c.off, L.off, ((size_t)h->nS + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    c.n = n;
    c.steps = h->steps;
    c.t = h->t;
    c.tf = h->tf;
    return DEME_OK;
}

int32_t restore_checkpoint(deme_handle* h, const Checkpoint& c) {
    cudaStream_t st = h->st_dt;
    ContactBuf& L = h->lists[h->cur];
    TRY(ensure_list(h, L, c.n));
    h->analFresh = false;
    CUDA_TRY(h, cudaMemcpyAsync(h->voxel, c.voxel, h->nO * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(h->loc, c.loc, h->nO * sizeof(ushort4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(h->quat, c.quat, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(h->vel, c.vel, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(h->omg, c.omg, h->nO * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    if (c.n) {
        CUDA_TRY(h, cudaMemcpyAsync(L.idA, c.idA, c.n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(L.idB, c.idB, c.n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(L.type, c.type, c.n * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(L.hist, c.hist, c.n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    }
    CUDA_TRY(h, cudaMemcpyAsync(L.off, c.off, ((size_t)h->nS + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(L.dN, &c.n, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    h->nContacts = c.n;
    h->countStale = false;
    h->steps = c.steps;
    h->t = c.t;
    h->tf = c.tf;
    h->outsValid = false;
    return DEME_OK;
}

namespace {

// The scenes the adjoint covers: clumps (any number of member spheres, principal moments of inertia) of free
// families and analytical walls (planes, cylinders, cones) of families whose motion is prescribed, the built-in
// model, Extended Taylor integration, contact detection every step.  A clump of a prescribed family counts as
// driven when both its linear and its rotational motion are prescribed; a partial prescription, or a wall whose
// owner moves under the contact forces, is outside.
int32_t check_adjoint_scene(deme_handle* h) {
    if (h->userForce.lib) {
        h->err = "adjoint: only the built-in Hertz-Mindlin model is differentiated";
        return DEME_ERR_INVALID;
    }
    if (h->motion.lib || h->famRules.lib) {
        h->err = "adjoint: prescribed-motion expressions and family-change rules are not differentiated";
        return DEME_ERR_INVALID;
    }
    if (h->nT) {
        h->err = "adjoint: sphere--mesh contacts are not differentiated";
        return DEME_ERR_INVALID;
    }
    if (h->nW == 0) {
        h->err = "adjoint: the frictionless Hertzian model (no contact wildcards) is not differentiated";
        return DEME_ERR_INVALID;
    }
    if (h->params.integrator != DEME_INTEGRATOR_EXTENDED_TAYLOR || h->params.cd_update_freq > 1 || h->cdLag > 0) {
        h->err = "adjoint: needs Extended Taylor integration and synchronous contact detection every step";
        return DEME_ERR_INVALID;
    }
    std::vector<ushort4> loc(h->nO);
    std::vector<AnalRaw> anal(std::max(h->nA, 1u));
    std::vector<Prescription> presc(DEME_NUM_FAMILIES);
    CUDA_TRY(h, cudaMemcpy(loc.data(), h->loc, h->nO * sizeof(ushort4), cudaMemcpyDeviceToHost));
    if (h->nA) CUDA_TRY(h, cudaMemcpy(anal.data(), h->analRaw, h->nA * sizeof(AnalRaw), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(presc.data(), h->presc, DEME_NUM_FAMILIES * sizeof(Prescription), cudaMemcpyDeviceToHost));
    auto driven = [](const Prescription& p) {
        return p.used && (p.lin_vel || p.lin_pos) && (p.rot_vel || p.rot_pos);
    };
    for (uint32_t o = 0; o < h->nO; o++) {
        const Prescription& p = presc[loc[o].w];
        if (o < h->nClumps ? p.used && !driven(p) : !driven(p)) {
            h->err = o < h->nClumps ? "adjoint: a clump family is only partly prescribed"
                                    : "adjoint: walls must belong to families with prescribed motion";
            return DEME_ERR_INVALID;
        }
    }
    for (uint32_t a = 0; a < h->nA; a++)
        if (anal[a].type != DEME_ANAL_PLANE && anal[a].type != DEME_ANAL_CYLINDER && anal[a].type != DEME_ANAL_CONE) {
            h->err = "adjoint: walls must be planes, cylinders or cones";
            return DEME_ERR_INVALID;
        }
    return DEME_OK;
}

}  // namespace

void adjoint_release(deme_handle* h) {
    if (!h->adj) return;
    AdjointTape* t = h->adj;
    for (Checkpoint& c : t->cps) free_checkpoint(h, c);
    free_checkpoint(h, t->fin);
    for (void* p : {(void*)t->X, (void*)t->V, (void*)t->Q, (void*)t->W, (void*)t->Al, (void*)t->cA, (void*)t->cB,
                    (void*)t->cT, (void*)t->cH, (void*)t->cM, (void*)t->lx, (void*)t->lv, (void*)t->lw, (void*)t->nlx,
                    (void*)t->nlv, (void*)t->nlw, (void*)t->lq, (void*)t->nlq, (void*)t->lF, (void*)t->lT,
                    (void*)t->gA, (void*)t->gB, (void*)t->gC, (void*)t->gmat, (void*)t->matAdj})
        dfree(h, p);
    delete t;
    h->adj = nullptr;
}

extern "C" {

int32_t deme_set_material(deme_handle* h, uint32_t m, float E, float nu, float CoR, float mu, float Crr) {
    if (!h || m >= h->nM) return DEME_ERR_INVALID;
    const float v[5] = {E, nu, CoR, mu, Crr};
    for (int k = 0; k < 5; k++)
        CUDA_TRY(h, cudaMemcpy(h->mat + (size_t)k * h->nM + m, &v[k], sizeof(float), cudaMemcpyHostToDevice));
    return refresh_material_pairs(h);
}

int32_t deme_adjoint_set_floors(deme_handle* h, double overlap_rel, double roll_speed, double tangential_force) {
    if (!h || !(overlap_rel >= 0.0) || !(roll_speed >= 0.0) || !(tangential_force >= 0.0)) return DEME_ERR_INVALID;
    if (!h->adj) h->adj = new AdjointTape();
    h->adj->floors[0] = overlap_rel;
    h->adj->floors[1] = roll_speed;
    h->adj->floors[2] = tangential_force;
    return DEME_OK;
}

int32_t deme_adjoint_record(deme_handle* h, int32_t n_steps, int32_t checkpoint_every) {
    if (!h || n_steps <= 0 || checkpoint_every <= 0) return DEME_ERR_INVALID;
    TRY(check_adjoint_scene(h));
    // A tape of the same segment length and owner count is kept with its buffers (the segment records, the pair
    // pool, the checkpoints): allocating and freeing them at every window would cost more than the window.
    if (!h->adj || h->adj->K != checkpoint_every || h->adj->nO != h->nO) {
        double floors[3] = {1e-4, 1e-4, 1e-6};
        if (h->adj) std::copy(h->adj->floors, h->adj->floors + 3, floors);
        adjoint_release(h);
        h->adj = new AdjointTape();
        std::copy(floors, floors + 3, h->adj->floors);
        h->adj->K = checkpoint_every;
        h->adj->nO = h->nO;
    }
    AdjointTape* t = h->adj;
    t->nSteps = n_steps;
    const size_t nCp = (size_t)((n_steps + checkpoint_every - 1) / checkpoint_every);
    for (size_t j = nCp; j < t->cps.size(); j++) free_checkpoint(h, t->cps[j]);
    t->cps.resize(nCp);
    t->maxN = 0;
    for (int32_t s = 0; s < n_steps; s++) {
        if (s % checkpoint_every == 0) {
            Checkpoint& c = t->cps[(size_t)(s / checkpoint_every)];
            TRY(save_checkpoint(h, c));
            t->maxN = std::max(t->maxN, c.n);
        }
        TRY(deme_step(h, 1));
    }
    TRY(save_checkpoint(h, t->fin));
    t->maxN = std::max(t->maxN, t->fin.n);
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    return read_device_errors(h);
}

int32_t deme_adjoint_backward(deme_handle* h, const deme_adjoint_seed* seed, deme_adjoint_grads* out) {
    if (!h || !out) return DEME_ERR_INVALID;
    AdjointTape* t = h->adj;
    if (!t || t->cps.empty()) {
        h->err = "deme_adjoint_backward: no recorded window (call deme_adjoint_record first)";
        return DEME_ERR_STATE;
    }
    const uint32_t nO = h->nO, nM = std::max(h->nM, 1u);
    const int K = t->K, nSeg = (int)t->cps.size();
    cudaStream_t st = h->st_dt;
    const SimConsts& k = h->k;
    // buffers
    if (!t->lx) {
        for (double** p : {&t->lx, &t->lv, &t->lw, &t->nlx, &t->nlv, &t->nlw, &t->lF, &t->lT})
            TRY(dalloc_n(h, p, 3 * (size_t)nO));
        TRY(dalloc_n(h, &t->lq, 4 * (size_t)nO));
        TRY(dalloc_n(h, &t->nlq, 4 * (size_t)nO));
        TRY(dalloc_n(h, &t->gmat, 4 * (size_t)nM));
        TRY(dalloc_n(h, &t->matAdj, (size_t)nM));
        TRY(dalloc_n(h, &t->X, (size_t)K * nO * 3));
        TRY(dalloc_n(h, &t->V, (size_t)K * nO));
        TRY(dalloc_n(h, &t->Q, (size_t)K * nO));
        TRY(dalloc_n(h, &t->W, (size_t)K * nO));
        TRY(dalloc_n(h, &t->Al, (size_t)K * nO));
    }
    CUDA_TRY(h, cudaMemsetAsync(t->gmat, 0, 4 * (size_t)nM * sizeof(double), st));
    if (h->nM) k_adj_mat_table<<<nblk(h->nM, 64), 64, 0, st>>>(h->state_view().mat, h->nM, t->matAdj);
    {
        const double* src[4] = {seed ? seed->d_pos : nullptr, seed ? seed->d_vel : nullptr,
                                seed ? seed->d_angvel : nullptr, seed ? seed->d_quat : nullptr};
        double* dst[4] = {t->lx, t->lv, t->lw, t->lq};
        for (int a = 0; a < 4; a++) {
            const size_t bytes = (a == 3 ? 4 : 3) * (size_t)nO * sizeof(double);
            if (src[a])
                CUDA_TRY(h, cudaMemcpy(dst[a], src[a], bytes, cudaMemcpyHostToDevice));
            else
                CUDA_TRY(h, cudaMemset(dst[a], 0, bytes));
        }
        // the seed at the final state, its world-frame angular velocity gradient taken to the owner frame
        k_adj_seed<<<nblk(nO, 256), 256, 0, st>>>(nO, t->fin.quat, t->fin.omg, t->lq, t->lw);
    }
    uint32_t gCap = t->gCap;
    auto ensure_g = [&](uint32_t n) -> int32_t {
        if (n <= gCap && t->gA) return DEME_OK;
        // the carried buffer keeps its content across a resize
        const uint32_t cap = n + n / 4 + 1024;
        float4* nc = nullptr;
        TRY(dalloc_n(h, &nc, cap));
        if (t->gC && gCap) CUDA_TRY(h, cudaMemcpyAsync(nc, t->gC, gCap * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        dfree(h, t->gA);
        dfree(h, t->gB);
        dfree(h, t->gC);
        t->gA = t->gB = nullptr;
        TRY(dalloc_n(h, &t->gA, cap));
        TRY(dalloc_n(h, &t->gB, cap));
        t->gC = nc;
        gCap = t->gCap = cap;
        return DEME_OK;
    };
    {
        // the pair pool of one segment, sized once from the counts seen at the checkpoints (grown below if a step
        // holds more)
        const uint64_t want = std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)K * t->maxN * 9 / 8 + (uint64_t)K * 1024);
        if (t->poolCap < want) {
            dfree(h, t->cA);
            dfree(h, t->cB);
            dfree(h, t->cT);
            dfree(h, t->cH);
            dfree(h, t->cM);
            t->cA = t->cB = t->cM = nullptr;
            t->cT = nullptr;
            t->cH = nullptr;
            t->poolCap = 0;
            TRY(dalloc_n(h, &t->cA, want));
            TRY(dalloc_n(h, &t->cB, want));
            TRY(dalloc_n(h, &t->cT, want));
            TRY(dalloc_n(h, &t->cH, want));
            TRY(dalloc_n(h, &t->cM, want));
            t->poolCap = (uint32_t)want;
        }
    }
    const size_t contact_smem = (4 * (size_t)nM + (size_t)kOwnerGrad * kAdjContactThreads) * sizeof(double);
    if (contact_smem > 48 * 1024)
        CUDA_TRY(h, cudaFuncSetAttribute(k_adj_contact, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)contact_smem));
    for (int j = nSeg - 1; j >= 0; j--) {
        const Checkpoint& cp = t->cps[(size_t)j];
        const int len = std::min(K, t->nSteps - j * K);
        // ---- recompute the segment, recording every step's state and contacts ----
        TRY(restore_checkpoint(h, cp));
        t->stepN.assign((size_t)len, 0);
        t->stepBase.assign((size_t)len, 0);
        uint32_t base = 0;
        for (int s = 0; s < len; s++) {
            StateView sv = h->state_view();
            {
                ProfScope prof_(KID_ADJ_RECORD, st);
                k_adj_record_state<<<nblk(nO, 256), 256, 0, st>>>(k, sv, nO, t->X + (size_t)s * nO * 3,
                                                               t->V + (size_t)s * nO, t->Q + (size_t)s * nO,
                                                               t->W + (size_t)s * nO);
            }
            TRY(deme_detect_contacts(h));
            const uint32_t n = h->nContacts;
            if (base + n > t->poolCap) {  // grow the pool, keeping the steps recorded so far
                const uint32_t cap = std::max<uint32_t>((uint32_t)std::min<uint64_t>(0xFFFFFFF0ull,
                                                        (uint64_t)(base + n) * 3 / 2 + (uint64_t)len * 1024), 4096u);
                uint32_t *nA = nullptr, *nB = nullptr, *nM2 = nullptr;
                uint8_t* nT = nullptr;
                float4* nH = nullptr;
                TRY(dalloc_n(h, &nA, cap));
                TRY(dalloc_n(h, &nB, cap));
                TRY(dalloc_n(h, &nT, cap));
                TRY(dalloc_n(h, &nH, cap));
                TRY(dalloc_n(h, &nM2, cap));
                if (base) {
                    CUDA_TRY(h, cudaMemcpyAsync(nA, t->cA, base * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
                    CUDA_TRY(h, cudaMemcpyAsync(nB, t->cB, base * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
                    CUDA_TRY(h, cudaMemcpyAsync(nT, t->cT, base * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st));
                    CUDA_TRY(h, cudaMemcpyAsync(nH, t->cH, base * sizeof(float4), cudaMemcpyDeviceToDevice, st));
                    CUDA_TRY(h, cudaMemcpyAsync(nM2, t->cM, base * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
                }
                CUDA_TRY(h, cudaStreamSynchronize(st));
                dfree(h, t->cA);
                dfree(h, t->cB);
                dfree(h, t->cT);
                dfree(h, t->cH);
                dfree(h, t->cM);
                t->cA = nA;
                t->cB = nB;
                t->cT = nT;
                t->cH = nH;
                t->cM = nM2;
                t->poolCap = cap;
            }
            const ContactBuf& L = h->lists[h->cur];
            if (n) {
                ProfScope prof_(KID_ADJ_RECORD, st);
                CUDA_TRY(h, cudaMemcpyAsync(t->cA + base, L.idA, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
                CUDA_TRY(h, cudaMemcpyAsync(t->cB + base, L.idB, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
                CUDA_TRY(h, cudaMemcpyAsync(t->cT + base, L.type, n * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st));
                CUDA_TRY(h, cudaMemcpyAsync(t->cH + base, L.hist, n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
                CUDA_TRY(h, cudaMemcpyAsync(t->cM + base, L.mapping, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                            st));
            }
            t->stepN[(size_t)s] = n;
            t->stepBase[(size_t)s] = base;
            base += n;
            TRY(deme_compute_forces(h));
            CUDA_TRY(h, cudaMemcpyAsync(t->Al + (size_t)s * nO, h->alpha, nO * sizeof(float4),
                                        cudaMemcpyDeviceToDevice, st));
            TRY(deme_integrate(h));
        }
        uint32_t need = cp.n;
        for (uint32_t n : t->stepN) need = std::max(need, n);
        if (j < nSeg - 1) need = std::max(need, t->cps[(size_t)j + 1].n);
        TRY(ensure_g(need));
        // ---- the history gradient entering the segment's last step ----
        const float4* gOut = nullptr;
        if (j < nSeg - 1) {
            const Checkpoint& nx = t->cps[(size_t)j + 1];
            const uint32_t n = t->stepN[(size_t)len - 1], b = t->stepBase[(size_t)len - 1];
            if (n) {
                ProfScope prof_(KID_ADJ_HISTORY, st);
                k_adj_rekey<<<nblk(n, 256), 256, 0, st>>>(n, t->cA + b, t->cB + b, t->cT + b, nx.off, nx.idB, nx.type,
                                                          nx.n, t->gC, t->gA, h->nS, h->dErr);
                gOut = t->gA;
            }
        }
        // ---- reverse over the segment ----
        for (int s = len - 1; s >= 0; s--) {
            const uint32_t n = t->stepN[(size_t)s], b = t->stepBase[(size_t)s];
            StateView sv = h->state_view();
            const float4 *Qs = t->Q + (size_t)s * nO, *Ws = t->W + (size_t)s * nO;
            {
                ProfScope prof_(KID_ADJ_INTEGRATE, st);
                k_adj_integrate<<<nblk(nO, 256), 256, 0, st>>>(sv, nO, h->nClumps, (double)k.h, Qs, Ws,
                                                                t->Al + (size_t)s * nO, t->lx, t->lv, t->lq, t->lw,
                                                                t->lF, t->lT, t->nlx, t->nlv, t->nlq, t->nlw);
            }
            if (n) {
                ProfScope prof_(KID_ADJ_CONTACT, st);
                k_adj_contact<<<nblk(n, kAdjContactThreads), kAdjContactThreads, contact_smem, st>>>(
                    k, sv, t->matAdj, h->analRaw, n, nM, t->cA + b, t->cB + b, t->cT + b, t->cH + b, t->X + (size_t)s * nO * 3,
                    t->V + (size_t)s * nO, Qs, Ws, t->lF, t->lT, gOut, t->gB, t->nlx, t->nlv, t->nlq, t->nlw, t->gmat,
                    make_double3(t->floors[0], t->floors[1], t->floors[2]));
            }
            std::swap(t->lx, t->nlx);
            std::swap(t->lv, t->nlv);
            std::swap(t->lq, t->nlq);
            std::swap(t->lw, t->nlw);
            // incoming-history gradients go to the previous list (the previous step's, or the checkpoint's)
            const uint32_t nPrev = s > 0 ? t->stepN[(size_t)s - 1] : cp.n;
            float4* dst = s > 0 ? t->gA : t->gC;
            if (nPrev) CUDA_TRY(h, cudaMemsetAsync(dst, 0, nPrev * sizeof(float4), st));
            if (n && nPrev) {
                ProfScope prof_(KID_ADJ_HISTORY, st);
                k_adj_hist_scatter<<<nblk(n, 256), 256, 0, st>>>(n, t->cM + b, t->gB, dst, nPrev, h->dErr);
            }
            gOut = t->gA;
        }
        TRY(check_launch(h, "adjoint"));
    }
    // ---- results, in the interface's variables at the window start ----
    k_adj_result<<<nblk(nO, 256), 256, 0, st>>>(h->state_view(), nO, h->nClumps, t->cps[0].quat, t->cps[0].omg,
                                                 t->lx, t->lv, t->lq, t->lw);
    CUDA_TRY(h, cudaStreamSynchronize(st));
    TRY(check_launch(h, "adjoint"));
    double* dsts[4] = {out->d_pos0, out->d_vel0, out->d_angvel0, out->d_quat0};
    const double* srcs[4] = {t->lx, t->lv, t->lw, t->lq};
    for (int a = 0; a < 4; a++)
        if (dsts[a])
            CUDA_TRY(h, cudaMemcpy(dsts[a], srcs[a], (a == 3 ? 4 : 3) * (size_t)nO * sizeof(double),
                                   cudaMemcpyDeviceToHost));
    if (out->d_material)
        CUDA_TRY(h, cudaMemcpy(out->d_material, t->gmat, 4 * (size_t)h->nM * sizeof(double), cudaMemcpyDeviceToHost));
    TRY(restore_checkpoint(h, t->fin));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return read_device_errors(h);
}

}  // extern "C"
