// adjoint_rigid.cuh -- reverse-mode pieces of the rigid-body step for the adjoint (adjoint.cu): the orientation
// matrix of a quaternion and its derivative, the quaternion product and exponential map of the Extended Taylor
// orientation update (src/kernel/DEMIntegrationKernels.cu:46-179), and the geometry of the analytical walls
// (plane, cylinder, cone: the signed gap and the wall normal at a sphere centre).  Everything in double precision.
#pragma once
#include "adjoint_law.cuh"

namespace deme_b200 {

// Quaternion (w, x, y, z) = (w, u).
struct dq4 {
    double w;
    dv3 u;
};
__device__ __forceinline__ dq4 to_dq4(float4 q) { return dq4{(double)q.x, mk(q.y, q.z, q.w)}; }

// R(q) v with R(q) = (2 w^2 - 1) I + 2 u u^T + 2 w [u]x, the matrix applyOriQToVector3 forms (rot_matrix): the
// polynomial is used as it stands, so that a quaternion that has drifted off unit length is rotated -- and
// differentiated -- exactly as the forward step rotates it.
__device__ __forceinline__ dv3 qrot(const dq4& q, dv3 v) {
    return (2.0 * q.w * q.w - 1.0) * v + (2.0 * dot(q.u, v)) * q.u + (2.0 * q.w) * cross(q.u, v);
}
// R(q)^T v (the rotation by the conjugate quaternion).
__device__ __forceinline__ dv3 qrot_t(const dq4& q, dv3 v) {
    return (2.0 * q.w * q.w - 1.0) * v + (2.0 * dot(q.u, v)) * q.u - (2.0 * q.w) * cross(q.u, v);
}
// Gradient of g . R(q) v with respect to q: dR/dw = 4 w I + 2 [u]x, dR/du_j = 2 (e_j u^T + u e_j^T) + 2 w [e_j]x.
__device__ __forceinline__ dq4 qrot_vjp(const dq4& q, dv3 v, dv3 g) {
    dq4 r;
    r.w = 4.0 * q.w * dot(g, v) + 2.0 * dot(g, cross(q.u, v));
    r.u = (2.0 * dot(q.u, v)) * g + (2.0 * dot(g, q.u)) * v + (2.0 * q.w) * cross(v, g);
    return r;
}
__device__ __forceinline__ void operator+=(dq4& a, const dq4& b) {
    a.w += b.w;
    a.u += b.u;
}

// q' = q (x) p (Hamilton product).  Reverse: the gradients of q and p from that of q'.
__device__ __forceinline__ void qmul_vjp(const dq4& q, const dq4& p, const dq4& g, dq4& gq, dq4& gp) {
    gq.w = g.w * p.w + dot(g.u, p.u);
    gq.u = (-g.w) * p.u + p.w * g.u + cross(p.u, g.u);
    gp.w = g.w * q.w + dot(g.u, q.u);
    gp.u = (-g.w) * q.u + q.w * g.u + cross(g.u, q.u);
}

// p = (cos(h |r| / 2), sin(h |r| / 2) r / |r|), (1, 0) at r = 0.  Reverse: the gradient of r from that of p.
// With s(L) = sin(h L / 2) / L and theta = h L / 2: dp0/dr = -(h / 2) s r, dpv/dr = s I + (s'(L) / L) r r^T,
// s'(L) / L = (h / 2)^3 (theta cos theta - sin theta) / theta^3 (Taylor series below theta = 1e-2).
__device__ __forceinline__ dv3 qexp_vjp(dv3 r, double h, const dq4& g) {
    const double L = norm(r), hh = 0.5 * h, th = hh * L;
    double sinc, c3;  // sin(th) / th, (th cos th - sin th) / th^3
    if (th < 1e-2) {
        const double t2 = th * th;
        sinc = 1.0 - t2 / 6.0 + t2 * t2 / 120.0;
        c3 = -1.0 / 3.0 + t2 / 30.0 - t2 * t2 / 840.0;
    } else {
        sinc = sin(th) / th;
        c3 = (th * cos(th) - sin(th)) / (th * th * th);
    }
    const double s = hh * sinc, sp = hh * hh * hh * c3;
    return (-hh * s * g.w) * r + s * g.u + (sp * dot(r, g.u)) * r;
}

// Signed gap of a sphere centre c from an analytical wall and the wall's normal there (towards the sphere), with
// the reverse: the gradient of c from those of gap and normal.  P, d: the wall's reference point and direction
// (plane normal / axis) as the forward step places them; the curved forms follow curved_gap (device_common.cuh).
// wall_geom returns false where the forward step finds no contact geometry (no normal, or outside a cone's axial
// range).
struct WallGeom {
    double gap;
    dv3 n, a, u;  // normal; for the curved walls the axis and the radial unit vector
    double rho, t;
    int type, normal;
    double c1, c2;
};
__device__ __forceinline__ bool wall_geom(int type, int normalOut, double size1, double c1, double c2, double umin,
                                          double umax, dv3 P, dv3 d, dv3 c, WallGeom& g) {
    g.type = type;
    g.normal = normalOut;
    g.c1 = c1;
    g.c2 = c2;
    g.a = d;
    g.rho = 1.0;
    g.t = 0.0;
    g.u = mk(0, 0, 0);
    if (type == DEME_ANAL_PLANE) {
        g.gap = dot(c - P, d);
        g.n = d;
        return true;
    }
    const dv3 v = c - P;
    g.t = dot(v, d);
    const dv3 w = v - g.t * d;
    g.rho = norm(w);
    if (!(g.rho > 0.0)) return false;
    g.u = (1.0 / g.rho) * w;
    if (type == DEME_ANAL_CYLINDER) {
        g.gap = normalOut ? g.rho - size1 : size1 - g.rho;
        g.n = normalOut ? g.u : -g.u;
        return true;
    }
    if (type != DEME_ANAL_CONE) return false;
    const double uc = (g.t * c2 + g.rho * c1) * c2;
    if (uc < umin || uc > umax) return false;
    const double gg = g.t * c1 - g.rho * c2;
    const dv3 gv = c1 * d - c2 * g.u;
    g.gap = normalOut ? -gg : gg;
    g.n = normalOut ? -gv : gv;
    return true;
}
// Reverse, for a direction a of any length (a wall direction rotated by a quaternion off unit length is not quite
// unit): w = v - (v.a) a has dw/dv = I - a a^T; rho = |w|, u = w / rho give d rho / dw = u, d u / dw =
// (I - u u^T) / rho; t = v.a gives dt/dv = a.
__device__ __forceinline__ dv3 wall_geom_vjp(const WallGeom& g, double g_gap, dv3 g_n) {
    if (g.type == DEME_ANAL_PLANE) return g_gap * g.n;
    double g_rho, g_t = 0.0;
    dv3 g_u;
    if (g.type == DEME_ANAL_CYLINDER) {  // gap = s (rho - R), n = s u
        const double sg = g.normal ? 1.0 : -1.0;
        g_rho = sg * g_gap;
        g_u = sg * g_n;
    } else {  // gap = s (t c1 - rho c2), n = s (c1 a - c2 u)
        const double sg = g.normal ? -1.0 : 1.0;
        g_t = sg * g.c1 * g_gap;
        g_rho = -sg * g.c2 * g_gap;
        g_u = (-sg * g.c2) * g_n;
    }
    const dv3 g_w = g_rho * g.u + (1.0 / g.rho) * (g_u - dot(g_u, g.u) * g.u);
    return g_w - dot(g.a, g_w) * g.a + g_t * g.a;
}

}  // namespace deme_b200
