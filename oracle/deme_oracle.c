/*
 * deme_oracle.c -- CPU oracle (restatement) of the DEM-Engine per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker.  It is never linked into the product library.
 *
 * Every function restates one reference routine and cites it (paths relative to the reference's src/).
 * Arithmetic mirrors the reference kernels' float/double mix.  It is compiled with -ffp-contract=off, so every
 * multiply and add is rounded separately; the CUDA library is compiled with --fmad=false for the same reason.
 * Float-to-integer conversions saturate (NaN -> 0), which is what the GPU's cvt instructions do for the
 * reference's implicit conversions.
 *
 * New analytical shapes (cylinder, cone) have no reference counterpart; their formulas follow the reference's
 * plane convention (DEMHelperKernels.cu:356-445): contact when the signed gap is at most the (expanded) radius
 * plus the entity margin, overlap depth = half the penetration, contact point in the middle of the penetration.
 */
#include "deme_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TINY_FLOAT 1e-12
#define HUGE_FLOAT 1e15
/* Defines.h:30-35 */
static const double TWO_OVER_THREE = 0.666666666666667;
static const double FOUR_OVER_THREE = 1.333333333333333;
static const double FIVE_OVER_THREE = 1.666666666666667;
static const double TWO_TIMES_SQRT_FIVE_OVER_SIX = 1.825741858350554;
static const double PI_D = 3.1415926535897932385;
static const double PI_SQUARED = 9.869604401089358;

struct oracle_ctx {
    deme_sim_params p;
    uint32_t nO, nS, nA, nM;
    uint64_t* voxel;
    uint16_t *locX, *locY, *locZ;
    float *qw, *qx, *qy, *qz, *vX, *vY, *vZ, *wX, *wY, *wZ, *aX, *aY, *aZ, *alX, *alY, *alZ;
    uint8_t* fam;
    float *mass, *mXX, *mYY, *mZZ;
    uint32_t* sOwner;
    float *rX, *rY, *rZ, *rad;
    uint16_t* sMat;
    uint8_t *aType, *aNormal;
    uint16_t* aMat;
    uint32_t *oAFirst, *oACount; /* per owner analytical range (packed scenes), NULL = all */
    uint32_t* aOwner;
    float *aRX, *aRY, *aRZ, *aDX, *aDY, *aDZ, *aS1, *aS2, *aS3, *aMass;
    double *aC1, *aC2; /* cone: sin, cos of the half angle */
    float *E, *nu, *CoR, *mu, *Crr;
    /* mesh facets: owner, nodes in the owner frame (9 floats), material */
    uint32_t nT;
    uint32_t* tOwner;
    float* tNode;
    uint16_t* tMat;
    uint8_t* masks;
    deme_family_prescription presc[DEME_NUM_FAMILIES];
    int nW;
    /* current contact list */
    uint32_t nC, capC;
    uint32_t *idA, *idB, *map;
    uint8_t* type;
    float* wc;
    float *F, *TOF, *CPA, *CPB;
    /* previous kT product (history source) */
    uint32_t nPrev, capPrev;
    uint32_t *pA, *pB;
    uint8_t* pT;
    /* last bin assignment */
    uint16_t* nBins;
    uint8_t* nAnal;
    uint32_t nPairs, capPairs;
    uint32_t *pairBin, *pairSph;
    int maxInBin;
    double t;
    int64_t steps;
};

static int g_threads = 1;
int32_t orc_set_threads(int32_t n) {
    g_threads = n > 0 ? n : 1;
    return g_threads;
}

/* ---------- saturating conversions (PTX cvt.rzi semantics for the reference's implicit casts) ---------- */
static inline uint32_t sat_u32(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967296.0) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
static inline uint64_t sat_u64(double x) {
    if (!(x > 0.0)) return 0ull;
    if (x >= 18446744073709551616.0) return ~0ull;
    return (uint64_t)x;
}
static inline uint16_t sat_u16(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 65536.0) return 65535u;
    return (uint16_t)x;
}

/* ---------- DEMHelperKernels.cu helpers ---------- */
/* voxelIDToPosition, DEMHelperKernels.cu:93-110 (with IDChopper :67-77) */
static inline void voxel_to_pos(const deme_sim_params* p, uint64_t id, uint16_t sx, uint16_t sy, uint16_t sz,
                                double* X, double* Y, double* Z) {
    uint64_t vx = id & ((1ull << p->nvXp2) - 1ull);
    uint64_t vy = (id >> p->nvXp2) & ((1ull << p->nvYp2) - 1ull);
    uint64_t vz = id >> (p->nvXp2 + p->nvYp2);
    *X = (double)vx * p->voxel_size_kernel + (double)sx * p->l_kernel;
    *Y = (double)vy * p->voxel_size_kernel + (double)sy * p->l_kernel;
    *Z = (double)vz * p->voxel_size_kernel + (double)sz * p->l_kernel;
}
/* positionToVoxelID, DEMHelperKernels.cu:113-135 */
static inline void pos_to_voxel(const deme_sim_params* p, double X, double Y, double Z, uint64_t* id, uint16_t* sx,
                                uint16_t* sy, uint16_t* sz) {
    double vs = p->voxel_size_kernel, l = p->l_kernel;
    uint64_t nx = sat_u64(X / vs), ny = sat_u64(Y / vs), nz = sat_u64(Z / vs);
    *sx = sat_u16((X - (double)nx * vs) / l);
    *sy = sat_u16((Y - (double)ny * vs) / l);
    *sz = sat_u16((Z - (double)nz * vs) / l);
    uint64_t v = nx;
    v += ny << p->nvXp2;
    v += nz << (p->nvXp2 + p->nvYp2);
    *id = v;
}
/* applyOriQToVector3<float, float>, DEMHelperKernels.cu:137-148 */
static inline void rot_f(float* X, float* Y, float* Z, float w, float x, float y, float z) {
    float ox = *X, oy = *Y, oz = *Z;
    *X = (2.0f * (w * w + x * x) - 1.0f) * ox + (2.0f * (x * y - w * z)) * oy + (2.0f * (x * z + w * y)) * oz;
    *Y = (2.0f * (x * y + w * z)) * ox + (2.0f * (w * w + y * y) - 1.0f) * oy + (2.0f * (y * z - w * x)) * oz;
    *Z = (2.0f * (x * z - w * y)) * ox + (2.0f * (y * z + w * x)) * oy + (2.0f * (w * w + z * z) - 1.0f) * oz;
}
/* locateMaskPair, DEMHelperKernels.cu:51-56 */
static inline uint32_t mask_index(uint32_t i, uint32_t j) {
    if (i > j) {
        uint32_t t = i;
        i = j;
        j = t;
    }
    return (1u + j) * j / 2u + i;
}
/* normalizeVector3<float>, DEMHelperKernels.cu:156-166 */
static inline void normalize_f(float* x, float* y, float* z) {
    float m = sqrtf(*x * *x + *y * *y + *z * *z);
    *x /= m;
    *y /= m;
    *z /= m;
}

/* Owner position (double) and orientation. */
static inline void owner_pos(const oracle_ctx* c, uint32_t o, double* X, double* Y, double* Z) {
    voxel_to_pos(&c->p, c->voxel[o], c->locX[o], c->locY[o], c->locZ[o], X, Y, Z);
}
/* Sphere centre: owner position + rotated relative position (DEMBinSphereKernels.cu:39-51). */
static inline void sphere_pos(const oracle_ctx* c, uint32_t s, double* X, double* Y, double* Z) {
    uint32_t o = c->sOwner[s];
    double ox, oy, oz;
    owner_pos(c, o, &ox, &oy, &oz);
    float rx = c->rX[s], ry = c->rY[s], rz = c->rZ[s];
    rot_f(&rx, &ry, &rz, c->qw[o], c->qx[o], c->qy[o], c->qz[o]);
    *X = ox + (double)rx;
    *Y = oy + (double)ry;
    *Z = oz + (double)rz;
}
/* Analytical component placement (DEMBinSphereKernels.cu:84-104, DEMCalcForceKernels.cu:123-142). */
/* Analytical components the spheres of `owner` may meet: all, or the owner's range when independent scenes are packed
 * into one (their walls must not reach each other's spheres; no reference counterpart). */
static inline void anal_range(const oracle_ctx* c, uint32_t owner, uint32_t* k0, uint32_t* k1) {
    if (c->oAFirst && c->oACount) {
        *k0 = c->oAFirst[owner];
        *k1 = c->oAFirst[owner] + c->oACount[owner];
    } else {
        *k0 = 0;
        *k1 = c->nA;
    }
}

static inline void anal_place(const oracle_ctx* c, uint32_t k, double* X, double* Y, double* Z, float* dx, float* dy,
                              float* dz) {
    uint32_t o = c->aOwner[k];
    double ox, oy, oz;
    owner_pos(c, o, &ox, &oy, &oz);
    float rx = c->aRX[k], ry = c->aRY[k], rz = c->aRZ[k];
    float ex = c->aDX[k], ey = c->aDY[k], ez = c->aDZ[k];
    rot_f(&rx, &ry, &rz, c->qw[o], c->qx[o], c->qy[o], c->qz[o]);
    rot_f(&ex, &ey, &ez, c->qw[o], c->qx[o], c->qy[o], c->qz[o]);
    *X = ox + (double)rx;
    *Y = oy + (double)ry;
    *Z = oz + (double)rz;
    *dx = ex;
    *dy = ey;
    *dz = ez;
}

/* ---------- sphere--mesh contacts (no reference counterpart: the reference declares SPHERE_MESH_CONTACT, Defines.h:66,
 * but detects none).  Facet nodes placed like an analytical component (each node rotated in float, added to the owner
 * position in double); the closest point of the facet to the sphere centre by the region tests of Ericson's
 * closest-point-on-triangle algorithm (Real-Time Collision Detection, 5.1.5) in double; contact-detection reach =
 * expanded radius + margin; dynamics with the plane's conventions (half the overlap as the depth, the normal from the
 * closest point to the centre normalised in float, the face normal when the centre lies on the facet). ---------- */
typedef struct {
    double a[3], b[3], c[3];
} tri_placed;

static inline void tri_place(const oracle_ctx* c, uint32_t t, tri_placed* out) {
    uint32_t o = c->tOwner[t];
    double ox, oy, oz;
    owner_pos(c, o, &ox, &oy, &oz);
    const float* n = c->tNode + 9 * (size_t)t;
    double* dst[3] = {out->a, out->b, out->c};
    for (int k = 0; k < 3; k++) {
        float x = n[3 * k], y = n[3 * k + 1], z = n[3 * k + 2];
        rot_f(&x, &y, &z, c->qw[o], c->qx[o], c->qy[o], c->qz[o]);
        dst[k][0] = ox + (double)x;
        dst[k][1] = oy + (double)y;
        dst[k][2] = oz + (double)z;
    }
}

static void tri_closest(const tri_placed* t, double px, double py, double pz, double* q) {
    const double abx = t->b[0] - t->a[0], aby = t->b[1] - t->a[1], abz = t->b[2] - t->a[2];
    const double acx = t->c[0] - t->a[0], acy = t->c[1] - t->a[1], acz = t->c[2] - t->a[2];
    const double apx = px - t->a[0], apy = py - t->a[1], apz = pz - t->a[2];
    const double d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= 0.0 && d2 <= 0.0) {
        memcpy(q, t->a, sizeof(t->a));
        return;
    }
    const double bpx = px - t->b[0], bpy = py - t->b[1], bpz = pz - t->b[2];
    const double d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= 0.0 && d4 <= d3) {
        memcpy(q, t->b, sizeof(t->b));
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        q[0] = t->a[0] + v * abx;
        q[1] = t->a[1] + v * aby;
        q[2] = t->a[2] + v * abz;
        return;
    }
    const double cpx = px - t->c[0], cpy = py - t->c[1], cpz = pz - t->c[2];
    const double d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= 0.0 && d5 <= d6) {
        memcpy(q, t->c, sizeof(t->c));
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        q[0] = t->a[0] + w * acx;
        q[1] = t->a[1] + w * acy;
        q[2] = t->a[2] + w * acz;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        q[0] = t->b[0] + w * (t->c[0] - t->b[0]);
        q[1] = t->b[1] + w * (t->c[1] - t->b[1]);
        q[2] = t->b[2] + w * (t->c[2] - t->b[2]);
        return;
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    q[0] = t->a[0] + abx * v + acx * w;
    q[1] = t->a[1] + aby * v + acy * w;
    q[2] = t->a[2] + abz * v + acz * w;
}

static inline double tri_dist2(const tri_placed* t, double px, double py, double pz, double* q) {
    tri_closest(t, px, py, pz, q);
    return (px - q[0]) * (px - q[0]) + (py - q[1]) * (py - q[1]) + (pz - q[2]) * (pz - q[2]);
}

static inline int tri_overlap_cd(const tri_placed* t, double px, double py, double pz, double radA, float beta4) {
    double q[3];
    const double reach = radA + (double)beta4;
    return tri_dist2(t, px, py, pz, q) <= reach * reach;
}

static int tri_overlap_dt(const tri_placed* t, double xA, double yA, double zA, double radA, double* CPX, double* CPY,
                          double* CPZ, float* nX, float* nY, float* nZ, double* depth) {
    double q[3];
    const double d2 = tri_dist2(t, xA, yA, zA, q);
    const double gap = sqrt(d2);
    const double od = (radA - gap) / 2.0;
    if (od < 0.0) return DEME_NOT_A_CONTACT;
    if (gap > 0.0) {
        *nX = (float)(xA - q[0]);
        *nY = (float)(yA - q[1]);
        *nZ = (float)(zA - q[2]);
    } else {
        const double abx = t->b[0] - t->a[0], aby = t->b[1] - t->a[1], abz = t->b[2] - t->a[2];
        const double acx = t->c[0] - t->a[0], acy = t->c[1] - t->a[1], acz = t->c[2] - t->a[2];
        *nX = (float)(aby * acz - abz * acy);
        *nY = (float)(abz * acx - abx * acz);
        *nZ = (float)(abx * acy - aby * acx);
    }
    normalize_f(nX, nY, nZ);
    *depth = od;
    *CPX = xA - (double)*nX * (gap + od);
    *CPY = yA - (double)*nY * (gap + od);
    *CPZ = zA - (double)*nZ * (gap + od);
    return DEME_SPHERE_MESH_CONTACT;
}

/* Signed gap and outward (wall -> sphere) normal of the new curved shapes.  Returns 0 when undefined. */
static inline int curved_gap(int type, int normal_out, double xA, double yA, double zA, double xB, double yB,
                             double zB, double ax, double ay, double az, double size1, double c1, double c2,
                             double umin, double umax, double* gap, double* nx, double* ny, double* nz) {
    double vx = xA - xB, vy = yA - yB, vz = zA - zB;
    double t = vx * ax + vy * ay + vz * az;
    double wx = vx - t * ax, wy = vy - t * ay, wz = vz - t * az;
    double rho = sqrt(wx * wx + wy * wy + wz * wz);
    if (!(rho > 0.0)) return 0;
    double ux = wx / rho, uy = wy / rho, uz = wz / rho;
    if (type == DEME_ANAL_CYLINDER) {
        if (normal_out) {
            *gap = rho - size1;
            *nx = ux;
            *ny = uy;
            *nz = uz;
        } else {
            *gap = size1 - rho;
            *nx = -ux;
            *ny = -uy;
            *nz = -uz;
        }
        return 1;
    }
    /* cone: c1 = sin(half angle), c2 = cos(half angle); apex at B, axis along +a */
    double s = t * c2 + rho * c1;
    double uc = s * c2;
    if (uc < umin || uc > umax) return 0;
    double g = t * c1 - rho * c2;
    double gx = c1 * ax - c2 * ux, gy = c1 * ay - c2 * uy, gz = c1 * az - c2 * uz;
    if (normal_out) {
        *gap = -g;
        *nx = -gx;
        *ny = -gy;
        *nz = -gz;
    } else {
        *gap = g;
        *nx = gx;
        *ny = gy;
        *nz = gz;
    }
    return 1;
}

/* checkSphereEntityOverlap (CD form), DEMHelperKernels.cu:356-391, plus cylinder/cone. */
static inline int anal_overlap_cd(const oracle_ctx* c, uint32_t k, double xA, double yA, double zA, double radA,
                                  double xB, double yB, double zB, float dx, float dy, float dz, float beta4) {
    int tp = c->aType[k];
    if (tp == DEME_ANAL_PLANE) {
        double px = xA - xB, py = yA - yB, pz = zA - zB;
        double dist = px * (double)dx + py * (double)dy + pz * (double)dz;
        if (dist > radA + (double)beta4) return DEME_NOT_A_CONTACT;
        return DEME_SPHERE_PLANE_CONTACT;
    }
    if (tp == DEME_ANAL_CYLINDER || tp == DEME_ANAL_CONE) {
        double gap, nx, ny, nz;
        if (!curved_gap(tp, c->aNormal[k], xA, yA, zA, xB, yB, zB, (double)dx, (double)dy, (double)dz,
                        (double)c->aS1[k], c->aC1[k], c->aC2[k], (double)c->aS2[k], (double)c->aS3[k], &gap, &nx, &ny,
                        &nz))
            return DEME_NOT_A_CONTACT;
        if (gap > radA + (double)beta4) return DEME_NOT_A_CONTACT;
        return tp == DEME_ANAL_CYLINDER ? DEME_SPHERE_CYLINDER_CONTACT : DEME_SPHERE_CONE_CONTACT;
    }
    return DEME_NOT_A_CONTACT; /* PLATE always "no contact" in the reference (DEMHelperKernels.cu:385-387) */
}

/* checkSphereEntityOverlap (dT form), DEMHelperKernels.cu:394-445, plus cylinder/cone. */
static inline int anal_overlap_dt(const oracle_ctx* c, uint32_t k, double xA, double yA, double zA, double radA,
                                  double xB, double yB, double zB, float dx, float dy, float dz, float beta4,
                                  double* CPX, double* CPY, double* CPZ, float* nX, float* nY, float* nZ,
                                  double* depth) {
    int tp = c->aType[k];
    if (tp == DEME_ANAL_PLANE) {
        double px = xA - xB, py = yA - yB, pz = zA - zB;
        double ddx = (double)dx, ddy = (double)dy, ddz = (double)dz;
        double dist = px * ddx + py * ddy + pz * ddz;
        double od = (radA + (double)beta4 - dist) / 2.0;
        if (od < 0.0) return DEME_NOT_A_CONTACT;
        *depth = od;
        *CPX = xA - ddx * (dist + od);
        *CPY = yA - ddy * (dist + od);
        *CPZ = zA - ddz * (dist + od);
        *nX = (float)ddx;
        *nY = (float)ddy;
        *nZ = (float)ddz;
        return DEME_SPHERE_PLANE_CONTACT;
    }
    if (tp == DEME_ANAL_CYLINDER || tp == DEME_ANAL_CONE) {
        double gap, nx, ny, nz;
        if (!curved_gap(tp, c->aNormal[k], xA, yA, zA, xB, yB, zB, (double)dx, (double)dy, (double)dz,
                        (double)c->aS1[k], c->aC1[k], c->aC2[k], (double)c->aS2[k], (double)c->aS3[k], &gap, &nx, &ny,
                        &nz))
            return DEME_NOT_A_CONTACT;
        double od = (radA + (double)beta4 - gap) / 2.0;
        if (od < 0.0) return DEME_NOT_A_CONTACT;
        *depth = od;
        *CPX = xA - nx * (gap + od);
        *CPY = yA - ny * (gap + od);
        *CPZ = zA - nz * (gap + od);
        *nX = (float)nx;
        *nY = (float)ny;
        *nZ = (float)nz;
        return tp == DEME_ANAL_CYLINDER ? DEME_SPHERE_CYLINDER_CONTACT : DEME_SPHERE_CONE_CONTACT;
    }
    return DEME_NOT_A_CONTACT;
}

/* ---------- allocation helpers ---------- */
#define XALLOC(ptr, n) ((ptr) = calloc((size_t)(n) > 0 ? (size_t)(n) : 1, sizeof(*(ptr))))
#define XDUP(dst, src, n)                                                   \
    do {                                                                    \
        XALLOC(dst, n);                                                     \
        if ((src) && (n) > 0) memcpy((dst), (src), (size_t)(n) * sizeof(*(dst))); \
    } while (0)

static void grow_contacts(oracle_ctx* c, uint32_t n) {
    if (n <= c->capC) return;
    uint32_t cap = n + n / 4 + 16;
    c->idA = realloc(c->idA, cap * sizeof(uint32_t));
    c->idB = realloc(c->idB, cap * sizeof(uint32_t));
    c->map = realloc(c->map, cap * sizeof(uint32_t));
    c->type = realloc(c->type, cap);
    float* nwc = calloc((size_t)cap * (c->nW > 0 ? c->nW : 1), sizeof(float));
    for (int k = 0; k < c->nW; k++) memcpy(nwc + (size_t)k * cap, c->wc + (size_t)k * c->capC, c->nC * sizeof(float));
    free(c->wc);
    c->wc = nwc;
    c->F = realloc(c->F, (size_t)cap * 3 * sizeof(float));
    c->TOF = realloc(c->TOF, (size_t)cap * 3 * sizeof(float));
    c->CPA = realloc(c->CPA, (size_t)cap * 3 * sizeof(float));
    c->CPB = realloc(c->CPB, (size_t)cap * 3 * sizeof(float));
    memset(c->CPA + (size_t)c->capC * 3, 0, (size_t)(cap - c->capC) * 3 * sizeof(float));
    memset(c->CPB + (size_t)c->capC * 3, 0, (size_t)(cap - c->capC) * 3 * sizeof(float));
    c->capC = cap;
}

oracle_ctx* orc_create(const deme_sim_params* p, const deme_scene* s) {
    if (!p || !s) return NULL;
    oracle_ctx* c = calloc(1, sizeof(oracle_ctx));
    c->p = *p;
    c->nO = s->n_owners;
    c->nS = s->n_spheres;
    c->nA = s->n_anal;
    c->nM = s->n_materials;
    c->nW = p->n_contact_wildcards;
    uint32_t nO = c->nO, nS = c->nS, nA = c->nA, nM = c->nM;
    XDUP(c->voxel, s->voxel, nO);
    XDUP(c->locX, s->locX, nO);
    XDUP(c->locY, s->locY, nO);
    XDUP(c->locZ, s->locZ, nO);
    XDUP(c->qw, s->oriQw, nO);
    XDUP(c->qx, s->oriQx, nO);
    XDUP(c->qy, s->oriQy, nO);
    XDUP(c->qz, s->oriQz, nO);
    XDUP(c->vX, s->vX, nO);
    XDUP(c->vY, s->vY, nO);
    XDUP(c->vZ, s->vZ, nO);
    XDUP(c->wX, s->omgX, nO);
    XDUP(c->wY, s->omgY, nO);
    XDUP(c->wZ, s->omgZ, nO);
    XALLOC(c->aX, nO);
    XALLOC(c->aY, nO);
    XALLOC(c->aZ, nO);
    XALLOC(c->alX, nO);
    XALLOC(c->alY, nO);
    XALLOC(c->alZ, nO);
    XDUP(c->fam, s->family, nO);
    XDUP(c->mass, s->mass, nO);
    XDUP(c->mXX, s->mmiXX, nO);
    XDUP(c->mYY, s->mmiYY, nO);
    XDUP(c->mZZ, s->mmiZZ, nO);
    XDUP(c->sOwner, s->sphere_owner, nS);
    XDUP(c->rX, s->relX, nS);
    XDUP(c->rY, s->relY, nS);
    XDUP(c->rZ, s->relZ, nS);
    XDUP(c->rad, s->radius, nS);
    XALLOC(c->sMat, nS);
    for (uint32_t i = 0; i < nS; i++)
        c->sMat[i] = s->sphere_material_wide ? s->sphere_material_wide[i] : (uint16_t)s->sphere_material[i];
    XDUP(c->aType, s->anal_type, nA);
    XDUP(c->aOwner, s->anal_owner, nA);
    XDUP(c->aNormal, s->anal_normal, nA);
    XALLOC(c->aMat, nA);
    for (uint32_t i = 0; i < nA; i++)
        c->aMat[i] = s->anal_material_wide ? s->anal_material_wide[i] : (uint16_t)s->anal_material[i];
    c->oAFirst = c->oACount = NULL;
    if (s->owner_anal_first && s->owner_anal_count) {
        XDUP(c->oAFirst, s->owner_anal_first, nO);
        XDUP(c->oACount, s->owner_anal_count, nO);
    }
    XDUP(c->aRX, s->anal_relX, nA);
    XDUP(c->aRY, s->anal_relY, nA);
    XDUP(c->aRZ, s->anal_relZ, nA);
    XDUP(c->aDX, s->anal_rotX, nA);
    XDUP(c->aDY, s->anal_rotY, nA);
    XDUP(c->aDZ, s->anal_rotZ, nA);
    XDUP(c->aS1, s->anal_size1, nA);
    XDUP(c->aS2, s->anal_size2, nA);
    XDUP(c->aS3, s->anal_size3, nA);
    XDUP(c->aMass, s->anal_mass, nA);
    XALLOC(c->aC1, nA);
    XALLOC(c->aC2, nA);
    for (uint32_t k = 0; k < nA; k++) {
        c->aC1[k] = sin((double)c->aS1[k]);
        c->aC2[k] = cos((double)c->aS1[k]);
    }
    XDUP(c->E, s->mat_E, nM);
    XDUP(c->nu, s->mat_nu, nM);
    XDUP(c->CoR, s->mat_CoR, nM);
    XDUP(c->mu, s->mat_mu, nM);
    XDUP(c->Crr, s->mat_Crr, nM);
    c->nT = s->n_tris;
    if (c->nT) {
        XDUP(c->tOwner, s->tri_owner, c->nT);
        XDUP(c->tMat, s->tri_material, c->nT);
        XALLOC(c->tNode, 9 * (size_t)c->nT);
        for (uint32_t t = 0; t < c->nT; t++)
            for (int k = 0; k < 3; k++) {
                c->tNode[9 * (size_t)t + k] = s->tri_node1[3 * (size_t)t + k];
                c->tNode[9 * (size_t)t + 3 + k] = s->tri_node2[3 * (size_t)t + k];
                c->tNode[9 * (size_t)t + 6 + k] = s->tri_node3[3 * (size_t)t + k];
            }
    }
    XALLOC(c->masks, DEME_NUM_FAMILY_MASK);
    if (s->family_masks) memcpy(c->masks, s->family_masks, DEME_NUM_FAMILY_MASK);
    if (s->prescriptions) memcpy(c->presc, s->prescriptions, sizeof(c->presc));
    XALLOC(c->nBins, nS);
    XALLOC(c->nAnal, nS);
    grow_contacts(c, 16);
    return c;
}

void orc_destroy(oracle_ctx* c) {
    if (!c) return;
    void* ptrs[] = {c->voxel, c->locX,   c->locY,   c->locZ,   c->qw,     c->qx,     c->qy,     c->qz,    c->vX,
                    c->vY,    c->vZ,     c->wX,     c->wY,     c->wZ,     c->aX,     c->aY,     c->aZ,    c->alX,
                    c->alY,   c->alZ,    c->fam,    c->mass,   c->mXX,    c->mYY,    c->mZZ,    c->sOwner, c->rX,
                    c->rY,    c->rZ,     c->rad,    c->sMat,   c->aType,  c->aOwner, c->aNormal, c->aMat,  c->aRX,
                    c->aRY,   c->aRZ,    c->aDX,    c->aDY,    c->aDZ,    c->aS1,    c->aS2,    c->aS3,   c->aMass,
                    c->aC1,   c->aC2,    c->E,      c->nu,     c->CoR,    c->mu,     c->Crr,    c->masks, c->idA,
                    c->idB,   c->map,    c->type,   c->wc,     c->F,      c->TOF,    c->CPA,    c->CPB,   c->pA,
                    c->pB,    c->pT,     c->nBins,  c->nAnal,  c->pairBin, c->pairSph, c->oAFirst, c->oACount,
                    c->tOwner, c->tNode,  c->tMat};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    free(c);
}

/* ---------- stable LSD radix sort of (u32 key, u32 index) (cub::DeviceRadixSort::SortPairs is stable) ---------- */
static void stable_sort_u32(uint32_t* keys, uint32_t* vals, uint32_t n) {
    if (n < 2) return;
    uint32_t* k2 = malloc((size_t)n * sizeof(uint32_t));
    uint32_t* v2 = malloc((size_t)n * sizeof(uint32_t));
    for (int pass = 0; pass < 4; pass++) {
        int sh = pass * 8;
        size_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (uint32_t i = 0; i < n; i++) cnt[((keys[i] >> sh) & 255u) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (uint32_t i = 0; i < n; i++) {
            size_t d = cnt[(keys[i] >> sh) & 255u]++;
            k2[d] = keys[i];
            v2[d] = vals[i];
        }
        memcpy(keys, k2, (size_t)n * sizeof(uint32_t));
        memcpy(vals, v2, (size_t)n * sizeof(uint32_t));
    }
    free(k2);
    free(v2);
}

/* ---------- kT: contact detection (DEMCubContactDetection.cu:39-397) ---------- */
int32_t orc_detect_contacts(oracle_ctx* c) {
    const deme_sim_params* p = &c->p;
    uint32_t nS = c->nS;
    double bs = p->bin_size;
    uint32_t* binOff = calloc((size_t)nS + 1, sizeof(uint32_t));
    uint32_t* analOff = calloc((size_t)nS + 1, sizeof(uint32_t));
    uint32_t* nMeshS = calloc((size_t)nS + 1, sizeof(uint32_t));
    double* PX = malloc((size_t)nS * sizeof(double) * 3);
    /* getNumberOfBinsEachSphereTouches, DEMBinSphereKernels.cu:12-115 */
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (uint32_t s = 0; s < nS; s++) {
        double x, y, z;
        sphere_pos(c, s, &x, &y, &z);
        PX[3 * (size_t)s] = x;
        PX[3 * (size_t)s + 1] = y;
        PX[3 * (size_t)s + 2] = z;
        double myRadius = (double)c->rad[s];
        myRadius += (double)p->beta;
        double bx = x / bs, by = y / bs, bz = z / bs;
        double span = myRadius / bs;
        uint16_t nx = (uint16_t)(sat_u32(bx + span) - sat_u32(bx - span) + 1u);
        uint16_t ny = (uint16_t)(sat_u32(by + span) - sat_u32(by - span) + 1u);
        uint16_t nz = (uint16_t)(sat_u32(bz + span) - sat_u32(bz - span) + 1u);
        c->nBins[s] = (uint16_t)((int)nx * (int)ny * (int)nz);
        uint8_t cnt = 0;
        uint32_t sf = c->fam[c->sOwner[s]];
        uint32_t k0, k1;
        anal_range(c, c->sOwner[s], &k0, &k1);
        for (uint32_t k = k0; k < k1; k++) {
            uint32_t of = c->fam[c->aOwner[k]];
            if (c->masks[mask_index(sf, of)] != 0) continue;
            double ax, ay, az;
            float dx, dy, dz;
            anal_place(c, k, &ax, &ay, &az, &dx, &dy, &dz);
            if (anal_overlap_cd(c, k, x, y, z, myRadius, ax, ay, az, dx, dy, dz, p->beta)) cnt++;
        }
        c->nAnal[s] = cnt;
        uint32_t mcnt = 0;
        for (uint32_t t = 0; t < c->nT; t++) {
            if (c->masks[mask_index(sf, c->fam[c->tOwner[t]])] != 0) continue;
            tri_placed tp;
            tri_place(c, t, &tp);
            if (tri_overlap_cd(&tp, x, y, z, myRadius, p->beta)) mcnt++;
        }
        nMeshS[s] = mcnt;
    }
    /* ExclusiveScans, DEMCubContactDetection.cu:77-96 */
    for (uint32_t s = 0; s < nS; s++) {
        binOff[s + 1] = binOff[s] + c->nBins[s];
        analOff[s + 1] = analOff[s] + c->nAnal[s] + nMeshS[s];
    }
    uint32_t P = binOff[nS], nGeo = analOff[nS];
    if (P > c->capPairs) {
        c->capPairs = P + P / 4 + 16;
        c->pairBin = realloc(c->pairBin, (size_t)c->capPairs * sizeof(uint32_t));
        c->pairSph = realloc(c->pairSph, (size_t)c->capPairs * sizeof(uint32_t));
    }
    c->nPairs = P;
    uint32_t* gA = malloc(((size_t)nGeo + 1) * sizeof(uint32_t));
    uint32_t* gB = malloc(((size_t)nGeo + 1) * sizeof(uint32_t));
    uint8_t* gT = malloc((size_t)nGeo + 1);
    /* populateBinSphereTouchingPairs, DEMBinSphereKernels.cu:117-230 */
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (uint32_t s = 0; s < nS; s++) {
        double x = PX[3 * (size_t)s], y = PX[3 * (size_t)s + 1], z = PX[3 * (size_t)s + 2];
        double myRadius = (double)c->rad[s];
        myRadius += (double)p->beta;
        double bx = x / bs, by = y / bs, bz = z / bs, span = myRadius / bs;
        uint32_t off = binOff[s];
        for (uint32_t k = sat_u32(bz - span); k <= sat_u32(bz + span); k++)
            for (uint32_t j = sat_u32(by - span); j <= sat_u32(by + span); j++)
                for (uint32_t i = sat_u32(bx - span); i <= sat_u32(bx + span); i++) {
                    c->pairBin[off] = i + j * p->nbX + k * p->nbX * p->nbY;
                    c->pairSph[off] = s;
                    off++;
                }
        uint32_t goff = analOff[s];
        uint32_t sf = c->fam[c->sOwner[s]];
        uint32_t k0, k1;
        anal_range(c, c->sOwner[s], &k0, &k1);
        for (uint32_t k = k0; k < k1; k++) {
            uint32_t of = c->fam[c->aOwner[k]];
            if (c->masks[mask_index(sf, of)] != 0) continue;
            double ax, ay, az;
            float dx, dy, dz;
            anal_place(c, k, &ax, &ay, &az, &dx, &dy, &dz);
            int ct = anal_overlap_cd(c, k, x, y, z, myRadius, ax, ay, az, dx, dy, dz, p->beta);
            if (ct) {
                gA[goff] = s;
                gB[goff] = k;
                gT[goff] = (uint8_t)ct;
                goff++;
            }
        }
        /* sphere--mesh contacts after the analytical ones, by facet id */
        for (uint32_t t = 0; t < c->nT; t++) {
            if (c->masks[mask_index(sf, c->fam[c->tOwner[t]])] != 0) continue;
            tri_placed tp;
            tri_place(c, t, &tp);
            if (tri_overlap_cd(&tp, x, y, z, myRadius, p->beta)) {
                gA[goff] = s;
                gB[goff] = t;
                gT[goff] = DEME_SPHERE_MESH_CONTACT;
                goff++;
            }
        }
    }
    /* SortPairs by bin, DEMCubContactDetection.cu:119-129 */
    stable_sort_u32(c->pairBin, c->pairSph, P);
    /* Unique + RunLengthEncode + scan, DEMCubContactDetection.cu:135-169 */
    uint32_t nActive = 0;
    uint32_t* actStart = malloc(((size_t)P + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < P; i++)
        if (i == 0 || c->pairBin[i] != c->pairBin[i - 1]) actStart[nActive++] = i;
    actStart[nActive] = P;
    /* getNumberOfContactsEachBin / populateContactPairsEachBin (thread-per-bin form), DEMContactKernels.cu:12-221 */
    uint32_t* binCnt = calloc((size_t)nActive + 1, sizeof(uint32_t));
    int maxIn = 0;
    for (uint32_t b = 0; b < nActive; b++) {
        int nb = (int)(actStart[b + 1] - actStart[b]);
        if (nb > maxIn) maxIn = nb;
    }
    c->maxInBin = maxIn;
    /* two passes like the reference: count, scan, populate */
    for (int pass = 0; pass < 2; pass++) {
        uint32_t* outA = NULL;
        uint32_t* outB = NULL;
        uint32_t* binOut = NULL;
        if (pass == 1) {
            binOut = malloc(((size_t)nActive + 1) * sizeof(uint32_t));
            binOut[0] = 0;
            for (uint32_t b = 0; b < nActive; b++) binOut[b + 1] = binOut[b] + (uint32_t)(uint16_t)binCnt[b];
            uint32_t nSS = binOut[nActive];
            grow_contacts(c, nGeo + nSS);
            outA = c->idA + nGeo;
            outB = c->idB + nGeo;
            c->nC = nGeo + nSS;
        }
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 64)
        for (uint32_t b = 0; b < nActive; b++) {
            uint32_t st = actStart[b], nb = actStart[b + 1] - st;
            uint32_t binID = c->pairBin[st];
            uint32_t cnt = 0;
            uint32_t wr = pass == 1 ? binOut[b] : 0;
            for (uint32_t ia = 0; ia < nb; ia++) {
                uint32_t sa = c->pairSph[st + ia];
                uint32_t oa = c->sOwner[sa];
                float ra = c->rad[sa];
                ra += p->beta;
                double xa = PX[3 * (size_t)sa], ya = PX[3 * (size_t)sa + 1], za = PX[3 * (size_t)sa + 2];
                for (uint32_t ib = ia + 1; ib < nb; ib++) {
                    uint32_t sb = c->pairSph[st + ib];
                    uint32_t ob = c->sOwner[sb];
                    if (oa == ob) continue;
                    if (c->masks[mask_index(c->fam[oa], c->fam[ob])] != 0) continue;
                    float rb = c->rad[sb];
                    rb += p->beta;
                    double xb = PX[3 * (size_t)sb], yb = PX[3 * (size_t)sb + 1], zb = PX[3 * (size_t)sb + 2];
                    /* checkSpheresOverlap<double>, DEMHelperKernels.cu:195-222 */
                    double radA = (double)ra, radB = (double)rb;
                    double d2 = (xa - xb) * (xa - xb) + (ya - yb) * (ya - yb) + (za - zb) * (za - zb);
                    if (d2 > (radA + radB) * (radA + radB)) continue;
                    float nx = (float)(xa - xb), ny = (float)(ya - yb), nz = (float)(za - zb);
                    normalize_f(&nx, &ny, &nz);
                    double half = (radA + radB - sqrt(d2)) / (double)2;
                    double cx = xb + (radB - half) * (double)nx;
                    double cy = yb + (radB - half) * (double)ny;
                    double cz = zb + (radB - half) * (double)nz;
                    /* getPointBinID, DEMHelperKernels.cu:266-273 */
                    uint32_t cb = sat_u32(cx / bs) + sat_u32(cy / bs) * p->nbX + sat_u32(cz / bs) * p->nbX * p->nbY;
                    if (cb != binID) continue;
                    if (pass == 0) {
                        cnt++;
                    } else {
                        outA[wr] = sa;
                        outB[wr] = sb;
                        wr++;
                    }
                }
            }
            if (pass == 0) binCnt[b] = cnt;
        }
        free(binOut);
    }
    for (uint32_t i = 0; i < nGeo; i++) {
        c->idA[i] = gA[i];
        c->idB[i] = gB[i];
        c->type[i] = gT[i];
    }
    for (uint32_t i = nGeo; i < c->nC; i++) c->type[i] = DEME_SPHERE_SPHERE_CONTACT;
    /* two SortPairs keyed on idA (stable), DEMCubContactDetection.cu:237-258 */
    uint32_t n = c->nC;
    uint32_t* key = malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t* idx = malloc(((size_t)n + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) {
        key[i] = c->idA[i];
        idx[i] = i;
    }
    stable_sort_u32(key, idx, n);
    uint32_t* tB = malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint8_t* tT = malloc((size_t)n + 1);
    for (uint32_t i = 0; i < n; i++) {
        tB[i] = c->idB[idx[i]];
        tT[i] = c->type[idx[i]];
    }
    memcpy(c->idA, key, (size_t)n * sizeof(uint32_t));
    memcpy(c->idB, tB, (size_t)n * sizeof(uint32_t));
    memcpy(c->type, tT, n);
    free(tB);
    free(tT);
    free(key);
    free(idx);
    /* history map, DEMCubContactDetection.cu:266-372 and buildPersistentMap, DEMHistoryMappingKernels.cu:16-60 */
    if (c->nW > 0) {
        uint32_t* oldOff = calloc((size_t)nS + 2, sizeof(uint32_t));
        for (uint32_t i = 0; i < c->nPrev; i++)
            if (c->pA[i] < nS) oldOff[c->pA[i] + 1]++;
        for (uint32_t s = 0; s < nS; s++) oldOff[s + 1] += oldOff[s];
        for (uint32_t i = 0; i < n; i++) {
            uint32_t a = c->idA[i], partner = DEME_NULL_MAPPING_PARTNER;
            if (c->type[i] != DEME_NOT_A_CONTACT && a < nS) {
                for (uint32_t j = oldOff[a]; j < oldOff[a + 1]; j++)
                    if (c->pB[j] == c->idB[i] && c->pT[j] == c->type[i]) {
                        partner = j;
                        break;
                    }
            }
            c->map[i] = partner;
        }
        free(oldOff);
        /* rearrangeContactWildcards, DEMPrepForceKernels.cu:93-115 (dT side, migratePersistentContacts) */
        float* nwc = calloc((size_t)c->capC * c->nW, sizeof(float));
        for (int k = 0; k < c->nW; k++)
            for (uint32_t i = 0; i < n; i++)
                nwc[(size_t)k * c->capC + i] =
                    c->map[i] == DEME_NULL_MAPPING_PARTNER ? 0.f : c->wc[(size_t)k * c->capC + c->map[i]];
        free(c->wc);
        c->wc = nwc;
        /* previous_* := current list */
        if (n > c->capPrev) {
            c->capPrev = n + n / 4 + 16;
            c->pA = realloc(c->pA, (size_t)c->capPrev * sizeof(uint32_t));
            c->pB = realloc(c->pB, (size_t)c->capPrev * sizeof(uint32_t));
            c->pT = realloc(c->pT, c->capPrev);
        }
        memcpy(c->pA, c->idA, (size_t)n * sizeof(uint32_t));
        memcpy(c->pB, c->idB, (size_t)n * sizeof(uint32_t));
        memcpy(c->pT, c->type, n);
        c->nPrev = n;
    } else {
        for (uint32_t i = 0; i < n; i++) c->map[i] = DEME_NULL_MAPPING_PARTNER;
    }
    free(actStart);
    free(binCnt);
    free(gA);
    free(gB);
    free(gT);
    free(PX);
    free(binOff);
    free(analOff);
    free(nMeshS);
    return DEME_OK;
}

/* ---------- dT: forces (DEMCalcForceKernels.cu:14-179 + FullHertzianForceModel.cu) ---------- */
static void contact_force(oracle_ctx* c, uint32_t i) {
    const deme_sim_params* p = &c->p;
    int ctype = c->type[i];
    uint32_t sA = c->idA[i];
    uint32_t oA = c->sOwner[sA];
    float ARadius = c->rad[sA];
    float AOwnerMass = c->mass[oA];
    double AOx, AOy, AOz;
    owner_pos(c, oA, &AOx, &AOy, &AOz);
    float AQw = c->qw[oA], AQx = c->qx[oA], AQy = c->qy[oA], AQz = c->qz[oA];
    float rx = c->rX[sA], ry = c->rY[sA], rz = c->rZ[sA];
    rot_f(&rx, &ry, &rz, AQw, AQx, AQy, AQz);
    double Ax = AOx + (double)rx, Ay = AOy + (double)ry, Az = AOz + (double)rz;
    int matA = c->sMat[sA], matB;
    float BRadius, BOwnerMass;
    uint32_t oB;
    double BOx, BOy, BOz, Bx, By, Bz;
    double CPx = 0, CPy = 0, CPz = 0, depth = 0;
    float nX = 0, nY = 0, nZ = 0;
    if (ctype == DEME_SPHERE_SPHERE_CONTACT) {
        uint32_t sB = c->idB[i];
        oB = c->sOwner[sB];
        BRadius = c->rad[sB];
        BOwnerMass = c->mass[oB];
        owner_pos(c, oB, &BOx, &BOy, &BOz);
        float bx = c->rX[sB], by = c->rY[sB], bz = c->rZ[sB];
        rot_f(&bx, &by, &bz, c->qw[oB], c->qx[oB], c->qy[oB], c->qz[oB]);
        Bx = BOx + (double)bx;
        By = BOy + (double)by;
        Bz = BOz + (double)bz;
        matB = c->sMat[sB];
        /* checkSpheresOverlap<double, float>, DEMHelperKernels.cu:233-264 */
        double radA = (double)ARadius, radB = (double)BRadius;
        double d2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
        if (d2 > (radA + radB) * (radA + radB)) {
            ctype = DEME_NOT_A_CONTACT;
        } else {
            nX = (float)(Ax - Bx);
            nY = (float)(Ay - By);
            nZ = (float)(Az - Bz);
            normalize_f(&nX, &nY, &nZ);
            depth = radA + radB - sqrt(d2);
            CPx = Bx + (radB - depth / (double)2) * (double)nX;
            CPy = By + (radB - depth / (double)2) * (double)nY;
            CPz = Bz + (radB - depth / (double)2) * (double)nZ;
        }
    } else if (ctype == DEME_SPHERE_MESH_CONTACT) {
        uint32_t t = c->idB[i];
        oB = c->tOwner[t];
        matB = c->tMat[t];
        BOwnerMass = c->mass[oB];
        BRadius = (float)HUGE_FLOAT;
        owner_pos(c, oB, &BOx, &BOy, &BOz);
        tri_placed tp;
        tri_place(c, t, &tp);
        ctype = tri_overlap_dt(&tp, Ax, Ay, Az, (double)ARadius, &CPx, &CPy, &CPz, &nX, &nY, &nZ, &depth);
    } else {
        uint32_t k = c->idB[i];
        oB = c->aOwner[k];
        matB = c->aMat[k];
        BOwnerMass = c->aMass[k];
        BRadius = (float)HUGE_FLOAT;
        owner_pos(c, oB, &BOx, &BOy, &BOz);
        float dx, dy, dz;
        anal_place(c, k, &Bx, &By, &Bz, &dx, &dy, &dz);
        ctype = anal_overlap_dt(c, k, Ax, Ay, Az, (double)ARadius, Bx, By, Bz, dx, dy, dz, 0.0f, &CPx, &CPy, &CPz,
                                &nX, &nY, &nZ, &depth);
    }
    float BQw = c->qw[oB], BQx = c->qx[oB], BQy = c->qy[oB], BQz = c->qz[oB];
    float fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
    float dtx = 0, dty = 0, dtz = 0, dtime = 0;
    if (c->nW >= 4) {
        dtx = c->wc[0 * (size_t)c->capC + i];
        dty = c->wc[1 * (size_t)c->capC + i];
        dtz = c->wc[2 * (size_t)c->capC + i];
        dtime = c->wc[3 * (size_t)c->capC + i];
    }
    if (ctype != DEME_NOT_A_CONTACT) {
        float cax = (float)(CPx - AOx), cay = (float)(CPy - AOy), caz = (float)(CPz - AOz);
        float cbx = (float)(CPx - BOx), cby = (float)(CPy - BOy), cbz = (float)(CPz - BOz);
        rot_f(&cax, &cay, &caz, AQw, -AQx, -AQy, -AQz);
        rot_f(&cbx, &cby, &cbz, BQw, -BQx, -BQy, -BQz);
        /* FullHertzianForceModel.cu */
        float E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt;
        {
            float E_A = c->E[matA], nu_A = c->nu[matA], CoR_A = c->CoR[matA], mu_A = c->mu[matA], Crr_A = c->Crr[matA];
            float E_B = c->E[matB], nu_B = c->nu[matB], CoR_B = c->CoR[matB], mu_B = c->mu[matB], Crr_B = c->Crr[matB];
            /* matProxy2ContactParam, DEMHelperKernels.cu:316-339 */
            float invE = (float)((1. - (double)(nu_A * nu_A)) / (double)E_A + (1. - (double)(nu_B * nu_B)) / (double)E_B);
            E_cnt = (float)(1. / (double)invE);
            float invG = (float)(2. * (2. - (double)nu_A) * (1. + (double)nu_A) / (double)E_A +
                                 2. * (2. - (double)nu_B) * (1. + (double)nu_B) / (double)E_B);
            G_cnt = (float)(1. / (double)invG);
            CoR_cnt = CoR_A < CoR_B ? CoR_A : CoR_B;
            mu_cnt = mu_A > mu_B ? mu_A : mu_B;
            Crr_cnt = Crr_A > Crr_B ? Crr_A : Crr_B;
        }
        float AVx = c->vX[oA], AVy = c->vY[oA], AVz = c->vZ[oA];
        float BVx = c->vX[oB], BVy = c->vY[oB], BVz = c->vZ[oB];
        float AWx = c->wX[oA], AWy = c->wY[oA], AWz = c->wZ[oA];
        float BWx = c->wX[oB], BWy = c->wY[oB], BWz = c->wZ[oB];
        /* rotVelCP = cross(RotVel, locCP), mapped to global */
        float rAx = AWy * caz - AWz * cay, rAy = AWz * cax - AWx * caz, rAz = AWx * cay - AWy * cax;
        float rBx = BWy * cbz - BWz * cby, rBy = BWz * cbx - BWx * cbz, rBz = BWx * cby - BWy * cbx;
        rot_f(&rAx, &rAy, &rAz, AQw, AQx, AQy, AQz);
        rot_f(&rBx, &rBy, &rBz, BQw, BQx, BQy, BQz);
        float ts = p->h;
        float vx = (AVx + rAx) - (BVx + rBx), vy = (AVy + rAy) - (BVy + rBy), vz = (AVz + rAz) - (BVz + rBz);
        float proj = vx * nX + vy * nY + vz * nZ;
        float vtx = vx - proj * nX, vty = vy - proj * nY, vtz = vz - proj * nZ;
        dtx += ts * vtx;
        dty += ts * vty;
        dtz += ts * vtz;
        float dproj = dtx * nX + dty * nY + dtz * nZ;
        dtx -= dproj * nX;
        dty -= dproj * nY;
        dtz -= dproj * nZ;
        dtime += ts;
        float mass_eff = (AOwnerMass * BOwnerMass) / (AOwnerMass + BOwnerMass);
        float sqrt_Rd = (float)sqrt(depth * (double)(ARadius * BRadius) / (double)(ARadius + BRadius));
        float Sn = (float)(2. * (double)E_cnt * (double)sqrt_Rd);
        float loge = (float)(((double)CoR_cnt < TINY_FLOAT) ? log(TINY_FLOAT) : (double)logf(CoR_cnt));
        float beta = (float)((double)loge / sqrt((double)(loge * loge) + PI_SQUARED));
        float k_n = (float)(TWO_OVER_THREE * (double)Sn);
        float gamma_n = (float)(TWO_TIMES_SQRT_FIVE_OVER_SIX * (double)beta * (double)sqrtf(Sn * mass_eff));
        float scal = (float)((double)k_n * depth + (double)(gamma_n * proj));
        fx += scal * nX;
        fy += scal * nY;
        fz += scal * nZ;
        /* no contact wildcards: the frictionless Hertzian model (FrictionlessHertzianForceModel.cu), normal part only */
        const int normal_only = c->nW == 0;
        if (!normal_only && (double)Crr_cnt > 0.0) {
            int add_rr = 1;
            float R_eff = sqrtf((ARadius * BRadius) / (ARadius + BRadius));
            float kn_simple = (float)(FOUR_OVER_THREE * (double)E_cnt * (double)sqrtf(R_eff));
            float gn_simple = -2.f * sqrtf((float)(FIVE_OVER_THREE * (double)mass_eff * (double)E_cnt)) * beta *
                              powf(R_eff, 0.25f);
            float d_coeff = gn_simple / (2.f * sqrtf(kn_simple * mass_eff));
            if ((double)d_coeff < 1.0) {
                float t_coll = (float)(PI_D * (double)sqrtf(mass_eff / (kn_simple * (1.f - d_coeff * d_coeff))));
                if (dtime <= t_coll) add_rr = 0;
            }
            if (add_rr) {
                float vrx = rBx - rAx, vry = rBy - rAy, vrz = rBz - rAz;
                float vmag = sqrtf(vrx * vrx + vry * vry + vrz * vrz);
                if ((double)vmag > TINY_FLOAT) {
                    float fmag = sqrtf(fx * fx + fy * fy + fz * fz);
                    float s = Crr_cnt * fmag;
                    tx = (vrx / vmag) * s;
                    ty = (vry / vmag) * s;
                    tz = (vrz / vmag) * s;
                }
            }
        }
        if (!normal_only && (double)mu_cnt > 0.0) {
            float kt = (float)(8. * (double)G_cnt * (double)sqrt_Rd);
            float gt = (float)(-TWO_TIMES_SQRT_FIVE_OVER_SIX * (double)beta * (double)sqrtf(mass_eff * kt));
            float nkt = -kt;
            float tfx = nkt * dtx - gt * vtx, tfy = nkt * dty - gt * vty, tfz = nkt * dtz - gt * vtz;
            float ft = sqrtf(tfx * tfx + tfy * tfy + tfz * tfz);
            if ((double)ft > TINY_FLOAT) {
                float ft_max = sqrtf(fx * fx + fy * fy + fz * fz) * mu_cnt;
                if (ft > ft_max) {
                    float r = ft_max / ft;
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
            fx += tfx;
            fy += tfy;
            fz += tfz;
        }
        c->CPA[3 * (size_t)i] = cax;
        c->CPA[3 * (size_t)i + 1] = cay;
        c->CPA[3 * (size_t)i + 2] = caz;
        c->CPB[3 * (size_t)i] = cbx;
        c->CPB[3 * (size_t)i + 1] = cby;
        c->CPB[3 * (size_t)i + 2] = cbz;
    } else {
        dtx = dty = dtz = dtime = 0.f;
    }
    c->F[3 * (size_t)i] = fx;
    c->F[3 * (size_t)i + 1] = fy;
    c->F[3 * (size_t)i + 2] = fz;
    c->TOF[3 * (size_t)i] = tx;
    c->TOF[3 * (size_t)i + 1] = ty;
    c->TOF[3 * (size_t)i + 2] = tz;
    if (c->nW >= 4) {
        c->wc[0 * (size_t)c->capC + i] = dtx;
        c->wc[1 * (size_t)c->capC + i] = dty;
        c->wc[2 * (size_t)c->capC + i] = dtz;
        c->wc[3 * (size_t)c->capC + i] = dtime;
    }
}

/* ---------- dT: force collection (DEMCubForceCollection.cu:20-158, DEMCollectForceKernels.cu:11-133) ---------- */
static inline uint32_t owner_of_B(const oracle_ctx* c, uint32_t i) {
    if (c->type[i] == DEME_SPHERE_MESH_CONTACT) return c->tOwner[c->idB[i]];
    return c->type[i] == DEME_SPHERE_SPHERE_CONTACT ? c->sOwner[c->idB[i]] : c->aOwner[c->idB[i]];
}

int32_t orc_compute_forces(oracle_ctx* c) {
    uint32_t n = c->nC, nO = c->nO;
    /* prepareForceArrays, DEMPrepForceKernels.cu:23-31 */
    memset(c->aX, 0, nO * sizeof(float));
    memset(c->aY, 0, nO * sizeof(float));
    memset(c->aZ, 0, nO * sizeof(float));
    memset(c->alX, 0, nO * sizeof(float));
    memset(c->alY, 0, nO * sizeof(float));
    memset(c->alZ, 0, nO * sizeof(float));
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (uint32_t i = 0; i < n; i++) contact_force(c, i);
    if (n == 0) return DEME_OK;
    /* 2n contributions sorted (stably) by owner: A-side entries first, then B-side (SortPairs of idAOwner) */
    uint32_t* key = malloc((size_t)2 * n * sizeof(uint32_t));
    uint32_t* idx = malloc((size_t)2 * n * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) {
        key[i] = c->sOwner[c->idA[i]];
        idx[i] = i;
        key[n + i] = owner_of_B(c, i);
        idx[n + i] = n + i;
    }
    stable_sort_u32(key, idx, 2 * n);
    /* forceToAcc / forceToAngAcc then ReduceByKey (sequential order) and stashElem */
    uint32_t r = 0;
    while (r < 2 * n) {
        uint32_t o = key[r];
        float sx = 0, sy = 0, sz = 0, ax = 0, ay = 0, az = 0;
        int first = 1;
        for (; r < 2 * n && key[r] == o; r++) {
            uint32_t e = idx[r];
            uint32_t i = e < n ? e : e - n;
            float mod = e < n ? 1.f : -1.f;
            float m = c->mass[o];
            float Fx = c->F[3 * (size_t)i], Fy = c->F[3 * (size_t)i + 1], Fz = c->F[3 * (size_t)i + 2];
            float lx = (Fx * mod) / m, ly = (Fy * mod) / m, lz = (Fz * mod) / m;
            const float* cp = e < n ? c->CPA : c->CPB;
            float px = cp[3 * (size_t)i], py = cp[3 * (size_t)i + 1], pz = cp[3 * (size_t)i + 2];
            float gx = (Fx + c->TOF[3 * (size_t)i]) * mod, gy = (Fy + c->TOF[3 * (size_t)i + 1]) * mod,
                  gz = (Fz + c->TOF[3 * (size_t)i + 2]) * mod;
            rot_f(&gx, &gy, &gz, c->qw[o], -c->qx[o], -c->qy[o], -c->qz[o]);
            float cx = py * gz - pz * gy, cy = pz * gx - px * gz, cz = px * gy - py * gx;
            float wx = cx / c->mXX[o], wy = cy / c->mYY[o], wz = cz / c->mZZ[o];
            if (first) {
                sx = lx;
                sy = ly;
                sz = lz;
                ax = wx;
                ay = wy;
                az = wz;
                first = 0;
            } else {
                sx += lx;
                sy += ly;
                sz += lz;
                ax += wx;
                ay += wy;
                az += wz;
            }
        }
        c->aX[o] += sx;
        c->aY[o] += sy;
        c->aZ[o] += sz;
        c->alX[o] += ax;
        c->alY[o] += ay;
        c->alZ[o] += az;
    }
    free(key);
    free(idx);
    return DEME_OK;
}

/* ---------- dT: integration (DEMIntegrationKernels.cu:46-179) ---------- */
int32_t orc_integrate(oracle_ctx* c) {
    const deme_sim_params* p = &c->p;
    float h = p->h;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (uint32_t o = 0; o < c->nO; o++) {
        const deme_family_prescription* pr = &c->presc[c->fam[o]];
        int linV = 0, rotV = 0, linP = 0, rotP = 0;
        float ovx = c->vX[o], ovy = c->vY[o], ovz = c->vZ[o];
        float owx = c->wX[o], owy = c->wY[o], owz = c->wZ[o];
        /* applyPrescribedVel (_velPrescriptionStrategy_, APIPrivate.cpp:1014-1029) */
        if (pr->used) {
            if (pr->has_vel[0]) c->vX[o] = pr->vel[0];
            if (pr->has_vel[1]) c->vY[o] = pr->vel[1];
            if (pr->has_vel[2]) c->vZ[o] = pr->vel[2];
            if (pr->has_omg[0]) c->wX[o] = pr->omg[0];
            if (pr->has_omg[1]) c->wY[o] = pr->omg[1];
            if (pr->has_omg[2]) c->wZ[o] = pr->omg[2];
            linV = pr->lin_vel_prescribed;
            rotV = pr->rot_vel_prescribed;
        }
        float ux = 0, uy = 0, uz = 0, qx_ = 0, qy_ = 0, qz_ = 0;
        if (!linV) {
            ux = (c->aX[o] + p->G[0]) * h;
            uy = (c->aY[o] + p->G[1]) * h;
            uz = (c->aZ[o] + p->G[2]) * h;
            c->vX[o] += ux;
            c->vY[o] += uy;
            c->vZ[o] += uz;
        }
        if (!rotV) {
            qx_ = c->alX[o] * h;
            qy_ = c->alY[o] * h;
            qz_ = c->alZ[o] * h;
            c->wX[o] += qx_;
            c->wY[o] += qy_;
            c->wZ[o] += qz_;
        }
        float vx, vy, vz, wx, wy, wz;
        if (p->integrator == DEME_INTEGRATOR_FORWARD_EULER) {
            vx = ovx; vy = ovy; vz = ovz;
            wx = owx; wy = owy; wz = owz;
        } else if (p->integrator == DEME_INTEGRATOR_CENTERED_DIFFERENCE) {
            vx = ovx + ux; vy = ovy + uy; vz = ovz + uz;
            wx = owx + qx_; wy = owy + qy_; wz = owz + qz_;
        } else {
            vx = ovx + ux * 0.5f; vy = ovy + uy * 0.5f; vz = ovz + uz * 0.5f;
            wx = owx + qx_ * 0.5f; wy = owy + qy_ * 0.5f; wz = owz + qz_ * 0.5f;
        }
        /* integratePos */
        double X, Y, Z;
        owner_pos(c, o, &X, &Y, &Z);
        if (pr->used) {
            if (pr->has_pos[0]) X = pr->pos[0];
            if (pr->has_pos[1]) Y = pr->pos[1];
            if (pr->has_pos[2]) Z = pr->pos[2];
            linP = pr->lin_pos_prescribed;
            rotP = pr->rot_pos_prescribed;
        }
        if (!linP) {
            X += (double)vx * (double)h;
            Y += (double)vy * (double)h;
            Z += (double)vz * (double)h;
        }
        pos_to_voxel(p, X, Y, Z, &c->voxel[o], &c->locX[o], &c->locY[o], &c->locZ[o]);
        if (!rotP) {
            double q0 = 1, q1 = wx, q2 = wy, q3 = wz;
            double len = sqrt(q1 * q1 + q2 * q2 + q3 * q3);
            double theta = 0.5 * (double)h * len;
            if (len > 0) {
                q0 = cos(theta);
                double s = sin(theta) / len;
                q1 *= s;
                q2 *= s;
                q3 *= s;
            }
            float a1 = c->qw[o], b1 = c->qx[o], c1 = c->qy[o], d1 = c->qz[o];
            float a2 = (float)q0, b2 = (float)q1, c2 = (float)q2, d2 = (float)q3;
            c->qw[o] = a1 * a2 - b1 * b2 - c1 * c2 - d1 * d2;
            c->qx[o] = a1 * b2 + b1 * a2 + c1 * d2 - d1 * c2;
            c->qy[o] = a1 * c2 - b1 * d2 + c1 * a2 + d1 * b2;
            c->qz[o] = a1 * d2 + b1 * c2 - c1 * b2 + d1 * a2;
        }
    }
    c->t += (double)h;
    c->steps++;
    return DEME_OK;
}

int32_t orc_step(oracle_ctx* c, int32_t n) {
    for (int32_t k = 0; k < n; k++) {
        int f = c->p.cd_update_freq;
        if (f <= 0 || (c->steps % f) == 0) orc_detect_contacts(c);
        orc_compute_forces(c);
        orc_integrate(c);
    }
    return DEME_OK;
}

/* ---------- transfer ---------- */
#define CPY_OUT(dst, src, n) \
    if (dst) memcpy((dst), (src), (size_t)(n) * sizeof(*(src)))
int32_t orc_download_state(oracle_ctx* c, deme_state* o) {
    uint32_t n = c->nO;
    CPY_OUT(o->voxel, c->voxel, n);
    CPY_OUT(o->locX, c->locX, n);
    CPY_OUT(o->locY, c->locY, n);
    CPY_OUT(o->locZ, c->locZ, n);
    CPY_OUT(o->oriQw, c->qw, n);
    CPY_OUT(o->oriQx, c->qx, n);
    CPY_OUT(o->oriQy, c->qy, n);
    CPY_OUT(o->oriQz, c->qz, n);
    CPY_OUT(o->vX, c->vX, n);
    CPY_OUT(o->vY, c->vY, n);
    CPY_OUT(o->vZ, c->vZ, n);
    CPY_OUT(o->omgX, c->wX, n);
    CPY_OUT(o->omgY, c->wY, n);
    CPY_OUT(o->omgZ, c->wZ, n);
    CPY_OUT(o->aX, c->aX, n);
    CPY_OUT(o->aY, c->aY, n);
    CPY_OUT(o->aZ, c->aZ, n);
    CPY_OUT(o->alphaX, c->alX, n);
    CPY_OUT(o->alphaY, c->alY, n);
    CPY_OUT(o->alphaZ, c->alZ, n);
    CPY_OUT(o->family, c->fam, n);
    return DEME_OK;
}
#define CPY_IN(dst, src, n) \
    if (src) memcpy((dst), (src), (size_t)(n) * sizeof(*(dst)))
int32_t orc_upload_state(oracle_ctx* c, const deme_state* s) {
    uint32_t n = c->nO;
    CPY_IN(c->voxel, s->voxel, n);
    CPY_IN(c->locX, s->locX, n);
    CPY_IN(c->locY, s->locY, n);
    CPY_IN(c->locZ, s->locZ, n);
    CPY_IN(c->qw, s->oriQw, n);
    CPY_IN(c->qx, s->oriQx, n);
    CPY_IN(c->qy, s->oriQy, n);
    CPY_IN(c->qz, s->oriQz, n);
    CPY_IN(c->vX, s->vX, n);
    CPY_IN(c->vY, s->vY, n);
    CPY_IN(c->vZ, s->vZ, n);
    CPY_IN(c->wX, s->omgX, n);
    CPY_IN(c->wY, s->omgY, n);
    CPY_IN(c->wZ, s->omgZ, n);
    CPY_IN(c->aX, s->aX, n);
    CPY_IN(c->aY, s->aY, n);
    CPY_IN(c->aZ, s->aZ, n);
    CPY_IN(c->alX, s->alphaX, n);
    CPY_IN(c->alY, s->alphaY, n);
    CPY_IN(c->alZ, s->alphaZ, n);
    CPY_IN(c->fam, s->family, n);
    return DEME_OK;
}
uint32_t orc_num_contacts(oracle_ctx* c) { return c->nC; }
int32_t orc_download_contacts(oracle_ctx* c, deme_contacts* o) {
    o->n_contacts = c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    uint32_t n = c->nC;
    CPY_OUT(o->idA, c->idA, n);
    CPY_OUT(o->idB, c->idB, n);
    CPY_OUT(o->type, c->type, n);
    CPY_OUT(o->mapping, c->map, n);
    if (o->wildcards)
        for (int k = 0; k < c->nW; k++)
            memcpy(o->wildcards + (size_t)k * o->capacity, c->wc + (size_t)k * c->capC, (size_t)n * sizeof(float));
    return DEME_OK;
}
/* Inject a kT product with its history.  It also becomes the previous list of the next history map. */
int32_t orc_upload_contacts(oracle_ctx* c, const deme_contacts* in) {
    uint32_t n = in->n_contacts;
    grow_contacts(c, n);
    c->nC = n;
    memcpy(c->idA, in->idA, (size_t)n * sizeof(uint32_t));
    memcpy(c->idB, in->idB, (size_t)n * sizeof(uint32_t));
    memcpy(c->type, in->type, n);
    for (uint32_t i = 0; i < n; i++) c->map[i] = DEME_NULL_MAPPING_PARTNER;
    for (int k = 0; k < c->nW; k++) {
        if (in->wildcards)
            memcpy(c->wc + (size_t)k * c->capC, in->wildcards + (size_t)k * in->capacity, (size_t)n * sizeof(float));
        else
            memset(c->wc + (size_t)k * c->capC, 0, (size_t)n * sizeof(float));
    }
    if (n > c->capPrev) {
        c->capPrev = n + n / 4 + 16;
        c->pA = realloc(c->pA, (size_t)c->capPrev * sizeof(uint32_t));
        c->pB = realloc(c->pB, (size_t)c->capPrev * sizeof(uint32_t));
        c->pT = realloc(c->pT, c->capPrev);
    }
    memcpy(c->pA, c->idA, (size_t)n * sizeof(uint32_t));
    memcpy(c->pB, c->idB, (size_t)n * sizeof(uint32_t));
    memcpy(c->pT, c->type, n);
    c->nPrev = n;
    return DEME_OK;
}
int32_t orc_download_contact_forces(oracle_ctx* c, deme_contact_forces* o) {
    o->n_contacts = c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    size_t n3 = (size_t)c->nC * 3;
    CPY_OUT(o->force, c->F, n3);
    CPY_OUT(o->torque_only_force, c->TOF, n3);
    CPY_OUT(o->cpA, c->CPA, n3);
    CPY_OUT(o->cpB, c->CPB, n3);
    return DEME_OK;
}
int32_t orc_bin_assignment(oracle_ctx* c, uint16_t* n_bins, uint8_t* n_anal, uint32_t cap, uint32_t* bins,
                           uint32_t* spheres, uint32_t* n_pairs) {
    if (n_bins) memcpy(n_bins, c->nBins, (size_t)c->nS * sizeof(uint16_t));
    if (n_anal) memcpy(n_anal, c->nAnal, c->nS);
    if (n_pairs) *n_pairs = c->nPairs;
    if (bins && spheres) {
        if (cap < c->nPairs) return DEME_ERR_OVERFLOW;
        memcpy(bins, c->pairBin, (size_t)c->nPairs * sizeof(uint32_t));
        memcpy(spheres, c->pairSph, (size_t)c->nPairs * sizeof(uint32_t));
    }
    return DEME_OK;
}
/* Kinetic energy of clump owners (DEMOwnerQueryKernels.cu:10-37 per-owner term), summed in double. */
double orc_kinetic_energy(oracle_ctx* c) {
    double ke = 0;
    /* clump owners only (they are the owners the spheres reference; external and mesh objects follow them) */
    uint32_t nClumps = 0;
    for (uint32_t s = 0; s < c->nS; s++)
        if (c->sOwner[s] + 1 > nClumps) nClumps = c->sOwner[s] + 1;
    for (uint32_t o = 0; o < nClumps; o++) {
        double v2 = (double)c->vX[o] * c->vX[o] + (double)c->vY[o] * c->vY[o] + (double)c->vZ[o] * c->vZ[o];
        double r2 = (double)c->mXX[o] * c->wX[o] * c->wX[o] + (double)c->mYY[o] * c->wY[o] * c->wY[o] +
                    (double)c->mZZ[o] * c->wZ[o] * c->wZ[o];
        ke += 0.5 * (double)c->mass[o] * v2 + 0.5 * r2;
    }
    return ke;
}
int32_t orc_max_spheres_in_bin(oracle_ctx* c) { return c->maxInBin; }
double orc_time(oracle_ctx* c) { return c->t; }

/* ChangeClumpSizes (APIPublic.cpp:844-862): markOwnerToChange, then dTModifyComponents (DEMMiscKernels.cu:4-33):
 * relative positions and radii of the listed owners' spheres times the owner's factor (the last one given). */
int32_t orc_change_clump_sizes(oracle_ctx* c, uint32_t n, const uint32_t* owners, const float* factors) {
    float* fac = calloc((size_t)c->nO + 1, sizeof(float));
    uint8_t* mark = calloc((size_t)c->nO + 1, 1);
    for (uint32_t i = 0; i < n; i++) {
        if (owners[i] >= c->nO) {
            free(fac);
            free(mark);
            return DEME_ERR_INVALID;
        }
        mark[owners[i]] = 1;
        fac[owners[i]] = factors[i];
    }
    for (uint32_t s = 0; s < c->nS; s++) {
        uint32_t o = c->sOwner[s];
        if (!mark[o]) continue;
        float f = fac[o];
        c->rX[s] *= f;
        c->rY[s] *= f;
        c->rZ[s] *= f;
        c->rad[s] *= f;
    }
    free(fac);
    free(mark);
    return DEME_OK;
}

int32_t orc_set_family_prescription(oracle_ctx* c, int32_t family, const deme_family_prescription* p) {
    if (!c || !p || family < 0 || family >= DEME_NUM_FAMILIES) return DEME_ERR_INVALID;
    c->presc[family] = *p;
    return DEME_OK;
}
