// kernels.cu -- per-step kernels of the B200 DEM hot path.
//
// Contact detection (kT).  The reference assigns every sphere to all bins its expanded radius touches, sorts the
// (bin, sphere) pairs and tests all pairs inside each bin, keeping a pair only in the bin that holds its contact
// point (src/algorithms/DEMCubContactDetection.cu:39-233, src/kernel/DEMBinSphereKernels.cu,
// src/kernel/DEMContactKernels_Blockwise.cu).  That reports the pair (A < B) exactly when
//     owner(A) != owner(B), the family mask allows it, the double-precision overlap test of the expanded radii
//     passes, and bin(CP) lies in bin_range(A) and in bin_range(B) on every axis.
// This file enumerates candidates differently -- each sphere is sorted once into a home cell of a search grid
// whose cells are at least one expanded diameter wide, and each sphere scans the forward half (in cell order) of
// the cells its neighbours can live in, so every pair is tested once -- and then evaluates that same predicate
// with the reference's arithmetic.  The contact set is therefore the reference's, while the bin-pair list (about
// 8-30 pairs per sphere) and its 32-bit radix sort disappear.  Found pairs are counted per A, scanned into
// segments and placed; the list is then in canonical order: grouped by A (ascending), sphere--analytical contacts
// first, then sphere--sphere contacts by ascending B.
//
// Dynamics (dT).  One fused kernel per contact: pose gather, overlap re-test, Hertz-Mindlin, history update and
// accumulation of the owners' linear and angular accelerations (the reference's calculateContactForces +
// collectContactForces, src/kernel/DEMCalcForceKernels.cu:14-179, src/algorithms/DEMCubForceCollection.cu:20-158).
// Contacts sharing owner(A) are adjacent, so the A side is reduced inside the warp before one vector atomic per
// segment; the B side uses one float4 atomic per contact.  One kernel per owner integrates
// (src/kernel/DEMIntegrationKernels.cu:46-179) and clears the accumulators for the next step.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "force_jit.cuh"
#include "force_kernel.cuh"
#include "kernels.cuh"
#include "integrate_kernel.cuh"
#include "profiler.cuh"

namespace deme_b200 {

static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// The search grid of the scene that `owner` belongs to.  kPacked: several scenes, looked up through ownerScene (into
// `tmp`); otherwise the one grid in the kernel parameters, read from there as it is used.
template <bool kPacked>
__device__ __forceinline__ const SearchGrid& grid_of(const SimConsts& k, uint32_t owner, SearchGrid& tmp) {
    if (!kPacked) return k.grid0;
    tmp = k.grids[__ldg(k.ownerScene + owner)];
    return tmp;
}

// The analytical components the spheres of `owner` may meet: all of them, or the owner's range when the scene
// packs several independent scenes (their walls must not reach each other's spheres).
__device__ __forceinline__ uint2 anal_range(const StateView& s, uint32_t owner) {
    return s.ownerAnal ? s.ownerAnal[owner] : make_uint2(0u, s.nA);
}

// Sphere centre in double (owner position + rotated relative position), DEMBinSphereKernels.cu:39-51.
__device__ __forceinline__ void sphere_center(const SimConsts& k, const StateView& s, uint32_t sid, uint32_t& owner,
                                              float4& sp, double& X, double& Y, double& Z) {
    owner = s.sOwner[sid];
    sp = s.sph[sid];
    const uint64_t v = s.voxel[owner];
    const ushort4 l = s.loc[owner];
    const float4 q = s.quat[owner];
    double ox, oy, oz;
    voxel_to_pos(k, v, l.x, l.y, l.z, ox, oy, oz);
    float rx = sp.x, ry = sp.y, rz = sp.z;
    rot_f(rx, ry, rz, q.x, q.y, q.z, q.w);
    X = ox + (double)rx;
    Y = oy + (double)ry;
    Z = oz + (double)rz;
}

// ------------------------------------------------------------------------------------------------------------
__global__ void k_place_anal(SimConsts k, StateView s, const AnalRaw* raw, AnalPlaced* placed, uint32_t nA) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nA) return;
    const AnalRaw r = raw[i];
    const uint32_t o = r.owner;
    const ushort4 l = s.loc[o];
    const float4 q = s.quat[o];
    double ox, oy, oz;
    voxel_to_pos(k, s.voxel[o], l.x, l.y, l.z, ox, oy, oz);
    float rx = r.relX, ry = r.relY, rz = r.relZ, dx = r.rotX, dy = r.rotY, dz = r.rotZ;
    rot_f(rx, ry, rz, q.x, q.y, q.z, q.w);
    rot_f(dx, dy, dz, q.x, q.y, q.z, q.w);
    AnalPlaced a;
    a.x = ox + (double)rx;
    a.y = oy + (double)ry;
    a.z = oz + (double)rz;
    a.dx = dx;
    a.dy = dy;
    a.dz = dz;
    a.owner = o;
    a.type = r.type;
    a.normal = r.normal;
    a.material = r.material;
    a.mass = r.mass;
    a.size1 = (double)r.size1;
    a.c1 = r.c1;
    a.c2 = r.c2;
    a.umin = (double)r.size2;
    a.umax = (double)r.size3;
    placed[i] = a;
}

void launch_place_anal(const SimConsts& k, const StateView& s, const AnalRaw* raw, AnalPlaced* placed, uint32_t nA,
                       cudaStream_t st) {
    if (!(nA)) return;
    ProfScope prof_(KID_PLACE_ANAL, st);
    if (nA) k_place_anal<<<blocks_for(nA, 64), 64, 0, st>>>(k, s, raw, placed, nA);
}

// Mesh facets placed at the current poses (as k_place_anal places the analytical components): each node rotated
// by the owner's orientation in float, added to the owner position in double.
__global__ void k_place_tri(SimConsts k, StateView s, const TriRaw* raw, uint32_t nT) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nT) return;
    const TriRaw r = raw[i];
    const uint32_t o = r.owner;
    const ushort4 l = s.loc[o];
    const float4 q = s.quat[o];
    double ox, oy, oz;
    voxel_to_pos(k, s.voxel[o], l.x, l.y, l.z, ox, oy, oz);
    float ax = r.n1x, ay = r.n1y, az = r.n1z, bx = r.n2x, by = r.n2y, bz = r.n2z, cx = r.n3x, cy = r.n3y, cz = r.n3z;
    rot_f(ax, ay, az, q.x, q.y, q.z, q.w);
    rot_f(bx, by, bz, q.x, q.y, q.z, q.w);
    rot_f(cx, cy, cz, q.x, q.y, q.z, q.w);
    TriPlaced t;
    t.ax = ox + (double)ax;
    t.ay = oy + (double)ay;
    t.az = oz + (double)az;
    t.bx = ox + (double)bx;
    t.by = oy + (double)by;
    t.bz = oz + (double)bz;
    t.cx = ox + (double)cx;
    t.cy = oy + (double)cy;
    t.cz = oz + (double)cz;
    t.owner = o;
    t.material = r.material;
    t.pad = 0;
    t.mass = r.mass;
    s.tri[i] = t;
}

void launch_place_tri(const SimConsts& k, const StateView& s, const TriRaw* raw, cudaStream_t st) {
    if (!(k.n_tris)) return;
    ProfScope prof_(KID_PLACE_ANAL, st);
    k_place_tri<<<blocks_for(k.n_tris, 64), 64, 0, st>>>(k, s, raw, k.n_tris);
}

// Lane that owns entry p of a warp-wide list made of the lanes' runs in lane order (`pre`: exclusive prefix of the
// run lengths, 33 entries): the last lane whose prefix is <= p.
__device__ __forceinline__ uint32_t pool_owner(const uint32_t* pre, uint32_t p) {
    uint32_t L = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1)
        if (pre[L + step] <= p) L += step;
    return L;
}

constexpr uint32_t kMeshFindWarps = 4;  // k_mesh_find's warps per block

// Sphere--mesh contact search, one warp per facet, once the spheres are in cell order.  A sphere in cell c can touch
// facet t only if its centre lies within the reach (largest expanded radius + beta) of t, so the facet visits the
// cells of its reach box, less those whose box (open to the outside at the grid's faces, where cell_of clamps, and
// cut to the reach box) has its centre farther from t than the reach plus its half diagonal, and tests the spheres
// of each: family mask, then the exact test at the sphere's exact centre with its expanded radius + beta.  Every
// sphere lies in one home cell and the facet visits each cell once, so each (sphere, facet) pair is found once.  A
// pair adds one to the sphere's contact count and is appended to the mesh pool; entries past the pool's capacity
// are dropped and their total (counters[4]), read by the host, makes it grow the pool and search again.
__global__ void __launch_bounds__(kMeshFindWarps * 32) k_mesh_find(SimConsts k, StateView s, CDView cd) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (t >= k.n_tris) return;
    const TriPlaced tp = s.tri[t];
    const uint32_t famT = s.loc[tp.owner].w;
    const SearchGrid& g = k.grid0;
    const double cs = 1.0 / g.inv_cell;
    const double reach = (double)k.r_max_cd + (double)k.beta + 1e-6 * cs;
    const double lo[3] = {fmin(tp.ax, fmin(tp.bx, tp.cx)) - reach, fmin(tp.ay, fmin(tp.by, tp.cy)) - reach,
                          fmin(tp.az, fmin(tp.bz, tp.cz)) - reach};
    const double hi[3] = {fmax(tp.ax, fmax(tp.bx, tp.cx)) + reach, fmax(tp.ay, fmax(tp.by, tp.cy)) + reach,
                          fmax(tp.az, fmax(tp.bz, tp.cz)) + reach};
    const uint32_t gdim[3] = {g.gx, g.gy, g.gz};
    uint32_t c0[3], nc[3];
    for (int d = 0; d < 3; d++) {
        c0[d] = cell_of(lo[d], g.inv_cell, gdim[d]);
        const uint32_t c1 = cell_of(hi[d], g.inv_cell, gdim[d]);
        if (!(c1 >= c0[d])) return;  // a facet with non-finite nodes meets nothing
        nc[d] = c1 - c0[d] + 1u;
    }
    const uint64_t total = (uint64_t)nc[0] * nc[1] * nc[2];
    // the warp's cells 32 at a time, one a lane (reach test, then its sphere range); the batch's spheres are then
    // spread over the lanes, so that 32 sphere tests run side by side instead of one lane walking its cell's list
    __shared__ uint32_t s_pre[kMeshFindWarps][33], s_first[kMeshFindWarps][32];
    const uint32_t w = threadIdx.x >> 5;
    for (uint64_t cb = 0; cb < total; cb += 32u) {
        const uint64_t c = cb + lane;
        uint32_t first = 0, cnt = 0;
        if (c < total) {
            const uint32_t ci[3] = {c0[0] + (uint32_t)(c % nc[0]), c0[1] + (uint32_t)((c / nc[0]) % nc[1]),
                                    c0[2] + (uint32_t)(c / ((uint64_t)nc[0] * nc[1]))};
            double ctr[3], hd2 = 0.0;
            for (int d = 0; d < 3; d++) {
                const double b0 = ci[d] == 0u ? lo[d] : fmax(lo[d], (double)ci[d] * cs);
                const double b1 = ci[d] + 1u >= gdim[d] ? hi[d] : fmin(hi[d], (double)(ci[d] + 1u) * cs);
                ctr[d] = 0.5 * (b0 + b1);
                hd2 += 0.25 * (b1 - b0) * (b1 - b0);
            }
            double qx, qy, qz;
            const double lim = reach + sqrt(hd2);
            if (tri_dist2(tp, ctr[0], ctr[1], ctr[2], qx, qy, qz) <= lim * lim) {
                const uint32_t key = ci[0] + g.gx * (ci[1] + g.gy * ci[2]);
                first = cd.cellStart[key];
                const uint32_t e = min(cd.cellStart[key + 1], k.n_spheres);
                cnt = e > first ? e - first : 0u;
            }
        }
        uint32_t incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= (uint32_t)off) incl += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        s_pre[w][lane + 1] = incl;
        if (lane == 0) s_pre[w][0] = 0;
        s_first[w][lane] = first;
        __syncwarp();
        for (uint32_t q = lane; q < tot; q += 32u) {
            const uint32_t L = pool_owner(s_pre[w], q);
            const uint32_t p = s_first[w][L] + (q - s_pre[w][L]);
            if (s.masks[mask_index(cd.rngS[p].w, famT)] != 0) continue;
            const SphCD r = cd.recS[p];
            const uint32_t sid = __float_as_uint(cd.posFSorted[p].w) & k.id_mask;
            if (!index_ok(k.err, 19, sid, k.n_spheres)) continue;
            double rD = (double)s.sph[sid].w;
            rD += (double)k.beta;
            if (!tri_overlap_cd(tp, r.x, r.y, r.z, rD, k.beta)) continue;
            atomicAdd(&cd.cnt[sid], 1u);
            const uint32_t slot = atomicAdd(&cd.counters[4], 1u);
            if (slot < cd.meshCap) cd.meshPool[slot] = make_uint2(sid, t);
        }
        __syncwarp();  // the batch's shared entries are read before the next batch writes them
    }
}

void launch_mesh_find(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st) {
    if (!(k.n_tris)) return;
    ProfScope prof_(KID_MESH_FIND, st);
    k_mesh_find<<<blocks_for((size_t)k.n_tris * 32u, kMeshFindWarps * 32), kMeshFindWarps * 32, 0, st>>>(k, s, cd);
}

// Places the mesh pool's pairs in their spheres' segments of the new list, from the top like k_pair_scatter (the
// two share the spheres' counts), each facet id tagged with kMeshTag; k_pair_assemble sorts them ahead of the
// sphere partners.
__global__ void __launch_bounds__(256) k_mesh_scatter(SimConsts k, CDView cd, ContactView c, uint32_t nPairs,
                                                      uint32_t cap) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= min(nPairs, min(cd.counters[4], cd.meshCap))) return;
    const uint2 st = cd.meshPool[p];
    if (!index_ok(k.err, 15, st.x, k.n_spheres)) return;
    const uint32_t slot = atomicSub(&cd.cnt[st.x], 1u) - 1u;
    const uint32_t pos = c.off[st.x] + slot;
    if (!index_ok(k.err, 16, pos, cap)) return;
    c.idB[pos] = kMeshTag | st.y;
}

void launch_mesh_scatter(const SimConsts& k, const CDView& cd, const ContactView& c, uint32_t nPairs, uint32_t cap,
                         cudaStream_t st) {
    if (!(k.n_tris && nPairs)) return;
    ProfScope prof_(KID_PAIR_EMIT, st);
    k_mesh_scatter<<<blocks_for(nPairs, 256), 256, 0, st>>>(k, cd, c, nPairs, cap);
}

// ------------------------------------------------------------------------------------------------------------
// Per sphere: home cell and analytical-contact count (getNumberOfBinsEachSphereTouches's analytical loop,
// DEMBinSphereKernels.cu:72-113).  The exact position is not stored: the cell-order record writer forms it again
// from the owner pose (the same arithmetic, so the same bits), which costs less than writing and re-reading it.
template <bool kPacked>
__global__ void __launch_bounds__(256) k_sphere_prep(SimConsts k, StateView s, CDView cd) {
    const uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= k.n_spheres) return;
    uint32_t owner;
    float4 sp;
    double X, Y, Z;
    sphere_center(k, s, sid, owner, sp, X, Y, Z);
    SearchGrid tmp;
    const SearchGrid& g = grid_of<kPacked>(k, owner, tmp);
    const uint32_t cx = cell_of(kPacked ? X - g.ox : X, g.inv_cell, g.gx);
    const uint32_t cy = cell_of(kPacked ? Y - g.oy : Y, g.inv_cell, g.gy);
    const uint32_t cz = cell_of(kPacked ? Z - g.oz : Z, g.inv_cell, g.gz);
    const uint32_t key = (kPacked ? g.base : 0u) + cx + g.gx * (cy + g.gy * cz);
    cd.cellKey[sid] = key;
    cd.idSeq[sid] = sid;
    atomicAdd(&cd.cellCount[key], 1u);
    // sphere--analytical contacts (expanded radius in double, entity margin beta)
    double rD = (double)sp.w;
    rD += (double)k.beta;
    const uint32_t fam = s.loc[owner].w;
    uint32_t c = 0;
    const uint2 ar = anal_range(s, owner);
    for (uint32_t a = ar.x; a < ar.x + ar.y; a++) {
        const AnalPlaced ap = s.anal[a];
        if (s.masks[mask_index(fam, s.loc[ap.owner].w)] != 0) continue;
        if (anal_overlap_cd(ap, X, Y, Z, rD, k.beta) != DEME_NOT_A_CONTACT) c++;
    }
    cd.nAnal[sid] = (uint8_t)c;
    cd.cnt[sid] = c;  // the pair and mesh searches add the sphere partners (this sphere as A) and the facets
}

void launch_sphere_prep(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_SPHERE_PREP, st);
    if (k.ownerScene)
        k_sphere_prep<true><<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd);
    else
        k_sphere_prep<false><<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd);
}

__device__ __forceinline__ uint4 pack_ranges(const uint32_t lo[3], const uint32_t hi[3]) {
    return make_uint4(min(lo[0], 65535u) | (min(hi[0], 65535u) << 16), min(lo[1], 65535u) | (min(hi[1], 65535u) << 16),
                      min(lo[2], 65535u) | (min(hi[2], 65535u) << 16), 0u);
}
__device__ __forceinline__ bool in_range(uint32_t b, uint32_t packed) {
    return b >= (packed & 0xFFFFu) && b <= (packed >> 16);
}

// Cell-order copies of everything the contact search reads, so that a warp (neighbouring cells) reads contiguous
// memory: position + id + radius bound for the pre-filter, one 32-byte record (exact position, owner, expanded
// radius) for the overlap test, bin ranges + family for the contact-point test.  This writes those of sphere j
// (ID order) into slot i.
__device__ __forceinline__ void write_cell_records(const SimConsts& k, const StateView& s, const CDView& cd,
                                                   uint32_t i, uint32_t j) {
    uint32_t o;
    float4 sp;
    double X, Y, Z;
    sphere_center(k, s, j, o, sp, X, Y, Z);
    const float4 p = make_float4((float)X, (float)Y, (float)Z, 0.f);
    const float r = sp.w;
    float rf = r;
    rf += k.beta;
    // CD radius bound: q units of q_scale, rounded up and one unit over, so q * q_scale >= rf despite float rounding
    const uint32_t qMax = 0xFFFFFFFFu >> k.q_shift;
    const uint32_t q = k.q_scale > 0.f ? min(qMax, (uint32_t)ceilf(rf / k.q_scale) + 1u) : qMax;
    cd.posFSorted[i] = make_float4(p.x, p.y, p.z, __uint_as_float(j | (q << k.q_shift)));
    SphCD rec;
    rec.x = X;
    rec.y = Y;
    rec.z = Z;
    rec.owner = o;
    rec.rf = rf;
    cd.recS[i] = rec;
    // bin ranges of the expanded sphere (reference arithmetic), packed 16 bits per bound
    double rD = (double)r;
    rD += (double)k.beta;
    uint32_t lo[3], hi[3];
    bin_range(X, rD, k.bin_size, lo[0], hi[0]);
    bin_range(Y, rD, k.bin_size, lo[1], hi[1]);
    bin_range(Z, rD, k.bin_size, lo[2], hi[2]);
    uint4 g = pack_ranges(lo, hi);
    g.w = s.loc[o].w;
    cd.rngS[i] = g;
}

// After a radix sort by cell: slot i gathers sphere idSorted[i].
__global__ void k_gather_sorted(SimConsts k, StateView s, CDView cd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k.n_spheres) return;
    const uint32_t j = cd.idSorted[i];
    if (!index_ok(k.err, 1, j, k.n_spheres)) return;
    write_cell_records(k, s, cd, i, j);
}

// Counting sort of the spheres by home cell (a radix sort whose single digit spans the cell range): the histogram
// was taken in k_sphere_prep and scanned into cellStart; each sphere takes a slot of its cell by decrementing the
// cell's count.  The order inside a cell is not defined, which the search does not depend on (partner lists are
// sorted when the contact list is assembled).
// Sphere j takes its slot and writes its cell-order records there at once (coalesced reads of j's data, scattered
// record writes), so no index array is written and gathered again.
__global__ void k_cell_scatter(SimConsts k, StateView s, CDView cd) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k.n_spheres) return;
    const uint32_t key = cd.cellKey[j];
    // one atomic per distinct cell among the warp's spheres (a clump's spheres mostly share a cell); each sphere
    // then takes its own slot below the value the atomic returned
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(__activemask(), key);
    const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
    uint32_t top = 0;
    if (lane == leader) top = atomicSub(&cd.cellCount[key], (uint32_t)__popc(peers));
    top = __shfl_sync(peers, top, leader);
    const uint32_t slot = cd.cellStart[key] + top - 1u - (uint32_t)__popc(peers & ((1u << lane) - 1u));
    if (!index_ok(k.err, 1, slot, k.n_spheres)) return;
    write_cell_records(k, s, cd, slot, j);
}

void launch_cell_scatter(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_CELL_SCATTER, st);
    k_cell_scatter<<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd);
}

void launch_gather_sorted(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_GATHER, st);
    k_gather_sorted<<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd);
}

// One sphere as the exact pair test sees it (cell-order records).
struct SphRec {
    double x, y, z;
    uint4 rng;  // bin ranges of the expanded sphere, packed 16 bits per bound
    uint32_t owner, fam, id;
    float rf;  // expanded radius (radius + beta) in float, as the reference forms it
};

// Exact position, owner and expanded radius of cell-order sphere j (what the overlap test needs).
__device__ __forceinline__ void load_near(const CDView& cd, uint32_t j, SphRec& r) {
    const double2 xy = __ldg(reinterpret_cast<const double2*>(cd.recS) + 2 * (size_t)j);
    const uint4 zr = __ldg(reinterpret_cast<const uint4*>(cd.recS) + 2 * (size_t)j + 1);
    r.x = xy.x;
    r.y = xy.y;
    r.z = __hiloint2double((int)zr.y, (int)zr.x);
    r.owner = zr.z;
    r.rf = __uint_as_float(zr.w);
}

__device__ __forceinline__ SphRec load_rec(const SimConsts& k, const CDView& cd, uint32_t j) {
    SphRec r;
    load_near(cd, j, r);
    r.rng = __ldg(cd.rngS + j);
    r.fam = r.rng.w;
    r.id = __float_as_uint(__ldg(&cd.posFSorted[j].w)) & k.id_mask;
    return r;
}

// The reference's pair predicate (see the file comment) with a.id < b.id, in two parts: pair_near (owners,
// double-precision overlap of the expanded radii) and pair_bins (family mask, the contact point's bin inside both
// spheres' bin ranges).  The roles matter, because the contact point is formed from B's side exactly as the
// reference forms it.
__device__ __forceinline__ bool pair_near(const SphRec& a, const SphRec& b) {
    if (a.owner == b.owner) return false;
    // checkSpheresOverlap<double>, DEMHelperKernels.cu:195-222 (symmetric in a and b to the last bit)
    const double radA = (double)a.rf, radB = (double)b.rf;
    const double d2 = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
    return d2 <= (radA + radB) * (radA + radB);
}

__device__ __forceinline__ bool pair_bins(const SimConsts& k, const StateView& s, const SphRec& a, const SphRec& b) {
    if (s.masks[mask_index(a.fam, b.fam)] != 0) return false;
    const double radA = (double)a.rf, radB = (double)b.rf;
    const double d2 = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
    float nx = (float)(a.x - b.x), ny = (float)(a.y - b.y), nz = (float)(a.z - b.z);
    normalize_f(nx, ny, nz);
    const double half = (radA + radB - sqrt(d2)) / 2.0;
    const double cpx = b.x + (radB - half) * (double)nx;
    const double cpy = b.y + (radB - half) * (double)ny;
    const double cpz = b.z + (radB - half) * (double)nz;
    // getPointBinID, DEMHelperKernels.cu:266-273, tested per axis against both spheres' bin ranges
    const uint32_t bx = sat_u32(cpx / k.bin_size), by = sat_u32(cpy / k.bin_size), bz = sat_u32(cpz / k.bin_size);
    return in_range(bx, a.rng.x) && in_range(by, a.rng.y) && in_range(bz, a.rng.z) && in_range(bx, b.rng.x) &&
           in_range(by, b.rng.y) && in_range(bz, b.rng.z);
}

// Orders two records by sphere id (selects instead of branching, so a warp runs the test once).
__device__ __forceinline__ void order_pair(const SphRec& me, const SphRec& ot, SphRec& a, SphRec& b) {
    const bool lower = me.id < ot.id;
    a = lower ? me : ot;
    b = lower ? ot : me;
}

// Cells the neighbours of a sphere can live in.  Cell coordinates come from cell_of (a multiply by the
// reciprocal cell size); the search grid is this file's own construct, so only monotonicity matters: a sphere
// within `reach` of x has its home cell inside [cell_of(x - reach), cell_of(x + reach)].
struct SearchBox {
    uint32_t x0, x1, y0, y1, z0, z1, cy, cz;
};

template <bool kPacked>
__device__ __forceinline__ SearchBox search_box(const SimConsts& k, const SearchGrid& g, double x, double y, double z,
                                                float rf) {
    const double reach = (double)rf + (double)g.r_max_cd + (double)k.prefilter_abs;
    if (kPacked) {  // a single scene's grid starts at the domain's lower corner
        x -= g.ox;
        y -= g.oy;
        z -= g.oz;
    }
    SearchBox b;
    b.x0 = cell_of(x - reach, g.inv_cell, g.gx);
    b.x1 = cell_of(x + reach, g.inv_cell, g.gx);
    b.y0 = cell_of(y - reach, g.inv_cell, g.gy);
    b.y1 = cell_of(y + reach, g.inv_cell, g.gy);
    b.z0 = cell_of(z - reach, g.inv_cell, g.gz);
    b.z1 = cell_of(z + reach, g.inv_cell, g.gz);
    b.cy = cell_of(y, g.inv_cell, g.gy);
    b.cz = cell_of(z, g.inv_cell, g.gz);
    return b;
}

// Visits every candidate j of sphere i (cell-order index) in the FORWARD half of its neighbourhood: rows of cells
// after i's own row in cell order (all of their cells in the box), and in i's own row the spheres after i.  Every
// unordered pair of spheres within reach is visited exactly once, by the sphere that comes first in cell order.
// `visit(j)` receives the cell-order index of each candidate that passes the float pre-filter and lies outside
// the run of sphere ids `clump` (first, count) that shares i's owner (such pairs are never contacts).  The
// pre-filter has two levels: the distance against `lim2` (i's radius plus the largest radius), then, for the few
// candidates within it, against i's radius `rfA` plus the candidate's own radius bound from its record.
#ifndef DEME_FIND_UNROLL
#define DEME_FIND_UNROLL 2
#endif
template <bool kPacked, typename Visit>
__device__ __forceinline__ void for_each_forward_candidate(const SimConsts& k, const SearchGrid& g, const CDView& cd,
                                                           uint32_t i, const float4 fA, const SearchBox& b, float lim2,
                                                           float rfA, uint2 clump, Visit visit) {
    constexpr uint32_t U = DEME_FIND_UNROLL;
    // Rows in order: i's own row (from i + 1), the rest of its z layer, then the later layers.  The next row's
    // bounds are fetched before the current row is tested, and each row's candidates are loaded U at a time, so
    // several loads are in flight per lane.
    uint32_t cy = b.cy, cz = b.cz;
    uint32_t j0 = i + 1u;
    const uint32_t* cellStart = kPacked ? cd.cellStart + g.base : cd.cellStart;
    uint32_t j1 = __ldg(cellStart + g.gx * (cy + g.gy * cz) + b.x1 + 1);
    while (true) {
        uint32_t ny = cy + 1u, nz = cz;
        if (ny > b.y1) {
            ny = b.y0;
            nz++;
        }
        const bool more = nz <= b.z1;
        uint32_t nj0 = 0, nj1 = 0;
        if (more) {
            const uint32_t rowBase = g.gx * (ny + g.gy * nz);
            nj0 = __ldg(cellStart + rowBase + b.x0);
            nj1 = __ldg(cellStart + rowBase + b.x1 + 1);
        }
        if (!index_ok(k.err, 2, j1, (uint64_t)k.n_spheres + 1)) j1 = j0;
        for (uint32_t j = j0; j < j1; j += U) {
            float4 f[U];
#pragma unroll
            for (uint32_t u = 0; u < U; u++)
                f[u] = (j + u < j1) ? __ldg(cd.posFSorted + j + u) : make_float4(1e30f, 1e30f, 1e30f, 0.f);
#pragma unroll
            for (uint32_t u = 0; u < U; u++) {
                const float dx = fA.x - f[u].x, dy = fA.y - f[u].y, dz = fA.z - f[u].z;
                // explicit fused multiply-adds: the pre-filter only has to be conservative, its margin covers them
                const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
                // padding lanes sit 1e30 away and never pass; spheres of i's own clump are skipped by id
                if (d2 <= lim2) {
                    const uint32_t wv = __float_as_uint(f[u].w);
                    const float rb = (float)(wv >> k.q_shift) * k.q_scale;
                    const float lim = (rfA + rb) * 1.00001f + k.prefilter_abs;
                    if ((wv & k.id_mask) - clump.x >= clump.y && d2 <= lim * lim) visit(j + u);
                }
            }
        }
        if (!more) break;
        cy = ny;
        cz = nz;
        j0 = nj0;
        j1 = nj1;
    }
}

__device__ __forceinline__ float prefilter_lim2(const SimConsts& k, const SearchGrid& g, float rf) {
    const float lim = (rf + g.r_max_cd) * 1.00001f + k.prefilter_abs;
    return lim * lim;
}

// One search pass:
//   k_pair_find, threads in cell order (a warp shares neighbour cells): each lane runs the float pre-filter over
//   the forward half of its neighbourhood and keeps the survivors' cell-order indices in shared memory; with both
//   radii in the pre-filter nearly all survivors are contacts.  The warp then reserves pool slots for all its
//   (sphere, candidate) survivors with one atomic and runs the double-precision reference predicate on them at once,
//   spread over its lanes, while their records are still in cache: each slot receives the pair (A, B) with A < B
//   by sphere id, or kNoPair, and a found pair is counted on A (whose count was preset to A's number of analytical
//   contacts).  A lane with more survivors than it can hold is queued for k_pair_overflow, which searches it again
//   and tests its survivors the same way.
// (Testing the pool in a kernel of its own, one thread per entry, read the records back from DRAM: 0.195 + 0.103 ms
// against 0.282 ms for this form on the 3M-sphere drum.)


// The reference's pair predicate on a candidate (cell-order indices i, j): the pair (A, B) with A < B by sphere id,
// counted on A, or kNoPair.
__device__ __forceinline__ uint2 exact_test(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t i,
                                            uint32_t j) {
    uint2 out = make_uint2(kNoPair, kNoPair);
    if (index_ok(k.err, 17, i, k.n_spheres) && index_ok(k.err, 18, j, k.n_spheres)) {
        const SphRec me = load_rec(k, cd, i);
        const SphRec ot = load_rec(k, cd, j);
        if (pair_near(me, ot)) {
            SphRec a, b;
            order_pair(me, ot, a, b);
            if (pair_bins(k, s, a, b) && index_ok(k.err, 14, a.id, k.n_spheres)) {
                out = make_uint2(a.id, b.id);
                atomicAdd(&cd.cnt[a.id], 1u);
            }
        }
    }
    return out;
}

// The search comes in a few block shapes (warps per block, survivor slots per lane), chosen per scene by
// deme_autotune; every shape finds the same pairs.
#ifndef DEME_FIND_RESIDENT_WARPS
#define DEME_FIND_RESIDENT_WARPS 48
#endif
// kPersistent: a grid of a few blocks per SM that take tiles of kWarps * 32 consecutive cell-order spheres from a
// work counter (counters[2]) until none is left, instead of one block per tile: tiles of dense cells cost more, and
// the queue spreads them over the SMs as they free up.
template <uint32_t kWarps, uint32_t kSlots, bool kPersistent, bool kPacked>
__global__ void __launch_bounds__(kWarps * 32, DEME_FIND_RESIDENT_WARPS / kWarps)
    k_pair_find(SimConsts k, StateView s, CDView cd, uint32_t tempCap) {
    __shared__ uint32_t s_pre[kWarps][33];           // survivor prefix over lanes
    __shared__ uint32_t s_surv[kWarps][kSlots][32];  // survivors, [slot][lane]
    __shared__ uint32_t s_tile;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t tile = blockIdx.x;
    while (true) {
        if (kPersistent) {
            __syncthreads();  // every warp is done with the previous tile's shared slots
            if (threadIdx.x == 0) s_tile = atomicAdd(&cd.counters[2], 1u);
            __syncthreads();
            tile = s_tile;
            if ((uint64_t)tile * blockDim.x >= k.n_spheres) return;
        }
        const uint32_t i = tile * blockDim.x + threadIdx.x;
        bool valid = i < k.n_spheres;
        uint32_t nSurv = 0;
        if (valid) {
            const float4 fA = __ldg(cd.posFSorted + i);
            SphRec me;
            load_near(cd, i, me);
            me.id = __float_as_uint(fA.w) & k.id_mask;
            if (!index_ok(k.err, 12, me.id, k.n_spheres)) {
                valid = false;
            } else {
                SearchGrid tmp;
                const SearchGrid& g = grid_of<kPacked>(k, me.owner, tmp);
                const SearchBox b = search_box<kPacked>(k, g, me.x, me.y, me.z, me.rf);
                for_each_forward_candidate<kPacked>(k, g, cd, i, fA, b, prefilter_lim2(k, g, me.rf), me.rf,
                                           __ldg(cd.sClump + me.id), [&](uint32_t j) {
                    if (nSurv < kSlots) s_surv[w][nSurv][lane] = j;
                    nSurv++;
                });
            }
        }
        const bool ovf = valid && nSurv > kSlots;
        const uint32_t pool = (valid && !ovf) ? nSurv : 0u;
        uint32_t incl = pool;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= (uint32_t)off) incl += y;
        }
        const uint32_t totalSurv = __shfl_sync(0xffffffffu, incl, 31);
        s_pre[w][lane + 1] = incl;
        if (lane == 0) s_pre[w][0] = 0;
        __syncwarp();
        uint32_t base = 0;
        if (lane == 0 && totalSurv) base = atomicAdd(&cd.counters[0], totalSurv);
        base = __shfl_sync(0xffffffffu, base, 0);
        const uint32_t iWarp = i - lane;
        // the exact test of the warp's survivors right away, while their records are in cache
        for (uint32_t p = lane; p < totalSurv; p += 32) {
            const uint32_t L = pool_owner(s_pre[w], p);
            if (base + p < tempCap)
                cd.candTemp[base + p] = exact_test(k, s, cd, iWarp + L, s_surv[w][p - s_pre[w][L]][L]);
        }
        if (ovf) {
            const uint32_t o = atomicAdd(&cd.counters[1], 1u);
            cd.ovf[o] = i;  // cell-order index; k_pair_overflow searches it again
        }
        if (!kPersistent) return;
    }
}

namespace {
struct FindShape {
    uint32_t warps, slots;
    bool persistent;
};
// the sixth shape holds only two survivors per lane, so most spheres go through k_pair_overflow (it keeps that path
// covered by the shape-equivalence tests; the autotuner rarely keeps it); the last two take their tiles from a work
// queue (persistent blocks)
constexpr FindShape kFindShapes[] = {{4, 16, false}, {2, 16, false}, {8, 16, false}, {4, 8, false},
                                     {4, 24, false}, {4, 2, false},  {4, 16, true},  {8, 16, true}};
constexpr int kNumFindShapes = sizeof(kFindShapes) / sizeof(kFindShapes[0]);

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    }
    return n;
}

template <uint32_t kWarps, uint32_t kSlots, bool kPersistent>
void launch_find(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t tempCap, cudaStream_t st) {
    const uint32_t threads = kWarps * 32;
    const uint32_t tiles = blocks_for(k.n_spheres, threads);
    // persistent: as many blocks as stay resident (the kernel's launch bounds), at most one per tile
    const uint32_t grid = kPersistent ? std::min<uint32_t>(tiles, (uint32_t)sm_count() * (DEME_FIND_RESIDENT_WARPS /
                                                                                           kWarps))
                                      : tiles;
    if (k.ownerScene)
        k_pair_find<kWarps, kSlots, kPersistent, true><<<grid, threads, 0, st>>>(k, s, cd, tempCap);
    else
        k_pair_find<kWarps, kSlots, kPersistent, false><<<grid, threads, 0, st>>>(k, s, cd, tempCap);
}
}  // namespace

int find_shape_count() { return kNumFindShapes; }
void find_shape(int v, uint32_t* warps, uint32_t* slots, bool* persistent) {
    const FindShape f = kFindShapes[(v >= 0 && v < kNumFindShapes) ? v : 0];
    *warps = f.warps;
    *slots = f.slots;
    if (persistent) *persistent = f.persistent;
}

void launch_pair_find(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t tempCap, int shape,
                      cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_PAIR_COUNT, st);
    switch (shape) {
        case 1: launch_find<2, 16, false>(k, s, cd, tempCap, st); break;
        case 2: launch_find<8, 16, false>(k, s, cd, tempCap, st); break;
        case 3: launch_find<4, 8, false>(k, s, cd, tempCap, st); break;
        case 4: launch_find<4, 24, false>(k, s, cd, tempCap, st); break;
        case 5: launch_find<4, 2, false>(k, s, cd, tempCap, st); break;
        case 6: launch_find<4, 16, true>(k, s, cd, tempCap, st); break;
        case 7: launch_find<8, 16, true>(k, s, cd, tempCap, st); break;
        default: launch_find<4, 16, false>(k, s, cd, tempCap, st);
    }
}

// Spheres whose survivors k_pair_find could not hold: the same forward-half search, one thread per sphere, each
// survivor appended to the pair pool (after every entry of k_pair_find) and counted in counters[3], for
// k_pair_exact_tail to test one thread per entry.  (Testing them in this kernel, serially per sphere, made a dense
// start, where many spheres overflow, six times slower.)  Grid-stride over the device-side overflow count (no host
// round trip).
template <bool kPacked>
__global__ void __launch_bounds__(128) k_pair_overflow(SimConsts k, StateView s, CDView cd, uint32_t tempCap) {
    const uint32_t nOvf = *((volatile uint32_t*)&cd.counters[1]);
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < nOvf; o += gridDim.x * blockDim.x) {
        const uint32_t i = cd.ovf[o];
        if (!index_ok(k.err, 13, i, k.n_spheres)) continue;
        const float4 fA = __ldg(cd.posFSorted + i);
        SphRec me;
        load_near(cd, i, me);
        me.id = __float_as_uint(fA.w) & k.id_mask;
        if (!index_ok(k.err, 12, me.id, k.n_spheres)) continue;
        SearchGrid tmp;
        const SearchGrid& g = grid_of<kPacked>(k, me.owner, tmp);
        const SearchBox b = search_box<kPacked>(k, g, me.x, me.y, me.z, me.rf);
        for_each_forward_candidate<kPacked>(k, g, cd, i, fA, b, prefilter_lim2(k, g, me.rf), me.rf,
                                            __ldg(cd.sClump + me.id),
                                   [&](uint32_t j) {
            const uint32_t pos = atomicAdd(&cd.counters[0], 1u);
            atomicAdd(&cd.counters[3], 1u);
            if (pos < tempCap) cd.candTemp[pos] = make_uint2(i, j);  // tested by k_pair_exact_tail
        });
    }
}

// The overflow kernel's entries, the last counters[3] of the pool's counters[0]: the reference predicate, one thread
// per entry (grid-stride over the device-side counts), each rewritten in place as its verdict.
__global__ void __launch_bounds__(256) k_pair_exact_tail(SimConsts k, StateView s, CDView cd, uint32_t tempCap) {
    const uint32_t end = min(*((volatile uint32_t*)&cd.counters[0]), tempCap);
    const uint32_t nTail = *((volatile uint32_t*)&cd.counters[3]);
    const uint32_t first = *((volatile uint32_t*)&cd.counters[0]) - nTail;
    for (uint32_t p = first + blockIdx.x * blockDim.x + threadIdx.x; p < end; p += gridDim.x * blockDim.x) {
        const uint2 ij = cd.candTemp[p];
        cd.candTemp[p] = exact_test(k, s, cd, ij.x, ij.y);
    }
}

void launch_pair_overflow(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t tempCap, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_PAIR_OVERFLOW, st);
    if (k.ownerScene)
        k_pair_overflow<true><<<148, 128, 0, st>>>(k, s, cd, tempCap);
    else
        k_pair_overflow<false><<<148, 128, 0, st>>>(k, s, cd, tempCap);
    k_pair_exact_tail<<<4 * (uint32_t)sm_count(), 256, 0, st>>>(k, s, cd, tempCap);
}

// Presets every sphere's contact count to its number of analytical contacts (k_sphere_prep does the same; this is
// for a repeated search after the temporary list grew).
__global__ void k_cnt_init(uint32_t n, const uint8_t* __restrict__ nAnal, uint32_t* cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cnt[i] = nAnal[i];
}

void launch_cnt_init(const SimConsts& k, const CDView& cd, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_OTHER, st);
    k_cnt_init<<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k.n_spheres, cd.nAnal, cd.cnt);
}

// Places every found pair in A's segment of the new list.  After the scan A's count is no longer needed, so the
// slots after A's analytical contacts are handed out from the top by decrementing it (shared with the mesh pairs,
// k_mesh_scatter).
// The pool count is read on the device (counters[0]), so the launch may cover more threads than pairs; a pool that
// outgrew its buffer (only possible when the host did not see the count first) is flagged.
__global__ void __launch_bounds__(256) k_pair_scatter(SimConsts k, CDView cd, ContactView c, uint32_t nPairs,
                                                      uint32_t cap, uint32_t poolCap) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t pool = cd.counters[0];
    if (p == 0 && pool > poolCap) atomicOr(k.err, ERR_CONTACT_CAPACITY);
    if (p >= min(nPairs, min(pool, poolCap))) return;
    const uint2 ab = cd.candTemp[p];
    if (ab.x == kNoPair) return;  // a pool entry the exact test rejected
    if (!index_ok(k.err, 15, ab.x, k.n_spheres)) return;
    const uint32_t slot = atomicSub(&cd.cnt[ab.x], 1u) - 1u;
    const uint32_t pos = c.off[ab.x] + slot;
    if (!index_ok(k.err, 16, pos, cap)) return;
    c.idB[pos] = ab.y;
}

void launch_pair_scatter(const SimConsts& k, const CDView& cd, const ContactView& c, uint32_t nPairs, uint32_t cap,
                         uint32_t poolCap, cudaStream_t st) {
    if (!(nPairs)) return;
    ProfScope prof_(KID_PAIR_EMIT, st);
    k_pair_scatter<<<blocks_for(nPairs, 256), 256, 0, st>>>(k, cd, c, nPairs, cap, poolCap);
}

// Completes the canonical list: per sphere A (ID order), its sphere--analytical contacts by component id
// (populateBinSphereTouchingPairs, DEMBinSphereKernels.cu:186-228) in the first slots of its segment, then its
// sphere--mesh contacts by facet id, then its sphere partners sorted by ascending id.  The scatter kernels left the
// partners and the facets (tagged with kMeshTag) after the analytical contacts in no order; with meshes the tail is
// sorted on the ids with the tag bit flipped, which puts the facets first.
template <bool kMesh>
__global__ void __launch_bounds__(256) k_pair_assemble(SimConsts k, StateView s, CDView cd, ContactView c,
                                                       uint32_t cap) {
    const uint32_t A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= k.n_spheres) return;
    const uint32_t begin = c.off[A], end = c.off[A + 1];
    if (end > cap || begin > end) {
        atomicOr(k.err, ERR_CONTACT_CAPACITY);
        return;
    }
    const uint32_t nAn = cd.nAnal[A];
    const uint32_t anEnd = min(begin + nAn, end);
    uint32_t w = begin;
    if (nAn) {
        uint32_t owner;
        float4 sp;
        double X, Y, Z;
        sphere_center(k, s, A, owner, sp, X, Y, Z);
        double rD = (double)sp.w;
        rD += (double)k.beta;
        const uint32_t fam = s.loc[s.sOwner[A]].w;
        const uint2 ar = anal_range(s, s.sOwner[A]);
        for (uint32_t a = ar.x; a < ar.x + ar.y && w < anEnd; a++) {
            const AnalPlaced ap = s.anal[a];
            if (s.masks[mask_index(fam, s.loc[ap.owner].w)] != 0) continue;
            const int t = anal_overlap_cd(ap, X, Y, Z, rD, k.beta);
            if (t != DEME_NOT_A_CONTACT) {
                c.idA[w] = A;
                c.idB[w] = a;
                c.type[w] = (uint8_t)t;
                w++;
            }
        }
        if (w != anEnd) atomicOr(k.err, ERR_SEGMENT_TOO_LONG);
    }
    uint32_t* seg = c.idB + anEnd;
    const uint32_t n = end - anEnd;
    const uint32_t flip = kMesh ? kMeshTag : 0u;  // sort keys: facets below every sphere
    // a sorted key back to the contact it stands for
    auto put = [&](uint32_t i, uint32_t key) {
        const bool facet = kMesh && key < kMeshTag;
        seg[i] = facet ? key : key ^ flip;
        c.idA[anEnd + i] = A;
        c.type[anEnd + i] = facet ? DEME_SPHERE_MESH_CONTACT : DEME_SPHERE_SPHERE_CONTACT;
    };
    constexpr uint32_t kReg = 8;
    if (n <= kReg) {
        // short segments (nearly all): loaded at once, sorted in registers, stored at once
        uint32_t v[kReg];
#pragma unroll
        for (uint32_t i = 0; i < kReg; i++) v[i] = i < n ? seg[i] ^ flip : 0xFFFFFFFFu;
#pragma unroll
        for (uint32_t i = 1; i < kReg; i++) {
#pragma unroll
            for (uint32_t j = i; j > 0; j--) {
                const uint32_t a = v[j - 1], b = v[j];
                v[j - 1] = min(a, b);
                v[j] = max(a, b);
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < kReg; i++)
            if (i < n) put(i, v[i]);
    } else {
        if (kMesh)
            for (uint32_t i = 0; i < n; i++) seg[i] ^= flip;
        for (uint32_t i = 1; i < n; i++) {
            const uint32_t v = seg[i];
            uint32_t j = i;
            while (j > 0 && seg[j - 1] > v) {
                seg[j] = seg[j - 1];
                j--;
            }
            seg[j] = v;
        }
        for (uint32_t i = 0; i < n; i++) put(i, seg[i]);
    }
}

void launch_pair_assemble(const SimConsts& k, const StateView& s, const CDView& cd, const ContactView& c, uint32_t cap,
                          cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_PAIR_EMIT, st);
    if (k.n_tris)
        k_pair_assemble<true><<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd, c, cap);
    else
        k_pair_assemble<false><<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, cd, c, cap);
}

// ------------------------------------------------------------------------------------------------------------
// History map and wildcard remap: for each new contact, find (idB, type) in A's segment of the previous list
// (buildPersistentMap, src/kernel/DEMHistoryMappingKernels.cu:16-60; rearrangeContactWildcards,
// src/kernel/DEMPrepForceKernels.cu:93-115).  Segments of both lists are sorted by (group, idB), the groups being
// sphere--analytical, sphere--mesh and sphere--sphere contacts (contact_group), so a binary search finds the unique
// partner.
__global__ void __launch_bounds__(256) k_history(uint32_t n, ContactView cur, ContactView prev, bool has_hist,
                                                 uint32_t nS, uint32_t prevN, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (*err != 0u) return;  // a voided step (see k_force)
    // the counts on the device bound the launch (it may cover a list's capacity)
    if (cur.dN) n = min(n, *cur.dN);
    if (prev.dN) prevN = *prev.dN;
    if (i >= n) return;
    if (!has_hist) {
        // a model without contact wildcards keeps no history, and the reference builds no map for it
        // (DEMCubContactDetection.cu:267, isHistoryless)
        cur.mapping[i] = DEME_NULL_MAPPING_PARTNER;
        return;
    }
    const uint32_t A = cur.idA[i], B = cur.idB[i];
    const uint8_t t = cur.type[i];
    const uint64_t key = ((uint64_t)contact_group(t) << 32) | B;
    if (!index_ok(err, 5, A, nS)) return;
    uint32_t lo = prev.off[A], hi = prev.off[A + 1];
    if (!index_ok(err, 6, hi, (uint64_t)prevN + 1) || lo > hi) {
        cur.mapping[i] = DEME_NULL_MAPPING_PARTNER;
        if (has_hist) cur.hist[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    uint32_t partner = DEME_NULL_MAPPING_PARTNER;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint8_t tm = prev.type[mid];
        const uint64_t km = ((uint64_t)contact_group(tm) << 32) | prev.idB[mid];
        if (km < key) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    if (lo < prev.off[A + 1] && prev.idB[lo] == B && prev.type[lo] == t) partner = lo;
    if (partner != DEME_NULL_MAPPING_PARTNER && !index_ok(err, 7, partner, prevN)) partner = DEME_NULL_MAPPING_PARTNER;
    cur.mapping[i] = partner;
    if (has_hist) cur.hist[i] = partner == DEME_NULL_MAPPING_PARTNER ? make_float4(0.f, 0.f, 0.f, 0.f) : prev.hist[partner];
}

void launch_history(const SimConsts& k, const ContactView& cur, const ContactView& prev, uint32_t n, uint32_t prevN,
                    bool has_hist, cudaStream_t st) {
    if (!(n)) return;
    ProfScope prof_(KID_HISTORY, st);
    k_history<<<blocks_for(n, 256), 256, 0, st>>>(n, cur, prev, has_hist, k.n_spheres, prevN, k.err);
}

__global__ void k_count_by_sphere(const uint32_t* idA, uint32_t n, uint32_t* cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&cnt[idA[i]], 1u);
}
void launch_count_by_sphere(const uint32_t* idA, uint32_t n, uint32_t* cnt, cudaStream_t st) {
    if (!(n)) return;
    ProfScope prof_(KID_OTHER, st);
    if (n) k_count_by_sphere<<<blocks_for(n, 256), 256, 0, st>>>(idA, n, cnt);
}

// ------------------------------------------------------------------------------------------------------------
// Fused force + collection kernel.
// The per-block partials of each analytical owner summed in a fixed order (deterministic) into its accumulators,
// in two kernels so that the whole GPU takes part: block (owner component, chunk) sums the partials of a contiguous
// range of force blocks with a fixed tree, then one thread per owner component adds its chunk sums in order.
__global__ void k_anal_reduce(AnalAccum aa, uint32_t nBlocks, uint32_t forceThreads, const uint32_t* err,
                              const uint32_t* dN) {
    __shared__ float sh[256];
    if (__syncthreads_or(threadIdx.x == 0 && *err != 0u)) return;  // a voided step (see k_force)
    // only the force blocks that held contacts wrote partials
    if (dN) nBlocks = min(nBlocks, (*dN + forceThreads - 1) / forceThreads);
    const uint32_t sc = blockIdx.x, chunk = blockIdx.y;
    const uint32_t slot = sc / 6u, comp = sc % 6u;
    const uint32_t len = (nBlocks + kAnalChunks - 1u) / kAnalChunks;
    const uint32_t b0 = chunk * len, b1 = min(nBlocks, b0 + len);
    float v = 0.f;
    for (uint32_t b = b0 + threadIdx.x; b < b1; b += blockDim.x) v += aa.partial[(size_t)b * 6u * aa.nAO + 6u * slot + comp];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) aa.chunks[sc * kAnalChunks + chunk] = sh[0];
}
__global__ void k_anal_reduce_final(AnalAccum aa, float4* acc, float4* alpha, const uint32_t* err) {
    const uint32_t sc = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc >= 6u * aa.nAO || *err != 0u) return;
    float v = 0.f;
    for (uint32_t c = 0; c < kAnalChunks; c++) v += aa.chunks[sc * kAnalChunks + c];
    const uint32_t o = aa.nClumps + sc / 6u, comp = sc % 6u;
    float* dst = comp < 3 ? &acc[o].x : &alpha[o].x;
    dst[comp % 3] = v;
}

namespace {
struct ForceShape {
    uint32_t threads, minBlocks;
};
constexpr ForceShape kForceShapes[] = {{kForceThreads, kForceMinBlocks}, {256, 4}, {64, 16}};
constexpr int kNumForceShapes = sizeof(kForceShapes) / sizeof(kForceShapes[0]);

template <uint32_t T, uint32_t B>
void launch_force_shape(const SimConsts& k, const StateView& s, const ContactView& c, uint32_t n, bool has_hist,
                        const ContactOutputs* out, const AnalAccum& aa, size_t smem, cudaStream_t st) {
    const uint32_t nb = blocks_for(n, T);
    // no contact history: the built-in model is the frictionless Hertzian model (the reference's frictionless model
    // has no contact wildcards; the full one has four)
    if (!has_hist) {
        if (out)
            k_force<true, T, B, true><<<nb, T, smem, st>>>(k, s, c, n, has_hist, *out, aa);
        else
            k_force<false, T, B, true><<<nb, T, smem, st>>>(k, s, c, n, has_hist, ContactOutputs{}, aa);
    } else if (out) {
        k_force<true, T, B><<<nb, T, smem, st>>>(k, s, c, n, has_hist, *out, aa);
    } else {
        k_force<false, T, B><<<nb, T, smem, st>>>(k, s, c, n, has_hist, ContactOutputs{}, aa);
    }
}
}  // namespace

int force_shape_count() { return kNumForceShapes; }
uint32_t force_shape_threads(int shape) { return kForceShapes[(shape >= 0 && shape < kNumForceShapes) ? shape : 0].threads; }

void launch_force(const SimConsts& k, const StateView& s, const ContactView& c, uint32_t n, bool has_hist,
                  const ContactOutputs* out, const AnalAccum& aa, const UserForceKernel* user, int shape,
                  cudaStream_t st) {
    if (!(n)) return;
    if (user) shape = 0;  // run-time compiled models come in the default shape
    const uint32_t threads = force_shape_threads(shape);
    const uint32_t nb = blocks_for(n, threads);
    const bool partials = aa.nAO && !aa.direct;
    const size_t smem = partials ? 6u * aa.nAO * sizeof(float) : 0;
    {
        ProfScope prof_(KID_FORCE, st);
        if (user) {
            // the same kernel template compiled at run time around a user force model
            SimConsts ka = k;
            StateView sa = s;
            ContactView ca = c;
            uint32_t na = n;
            bool ha = has_hist;
            ContactOutputs oa = out ? *out : ContactOutputs{};
            AnalAccum aaa = aa;
            void* args[] = {&ka, &sa, &ca, &na, &ha, &oa, &aaa};
            cudaLaunchKernel((const void*)user->kern[out ? 1 : 0], dim3(nb), dim3(kForceThreads), args, smem, st);
        } else if (shape == 1) {
            launch_force_shape<256, 4>(k, s, c, n, has_hist, out, aa, smem, st);
        } else if (shape == 2) {
            launch_force_shape<64, 16>(k, s, c, n, has_hist, out, aa, smem, st);
        } else {
            launch_force_shape<kForceThreads, kForceMinBlocks>(k, s, c, n, has_hist, out, aa, smem, st);
        }
    }
    if (partials) {
        ProfScope prof_(KID_OTHER, st);
        k_anal_reduce<<<dim3(6u * aa.nAO, kAnalChunks), 256, 0, st>>>(aa, nb, threads, k.err, c.dN);
    }
    if (partials) {
        ProfScope prof_(KID_OTHER, st);
        k_anal_reduce_final<<<blocks_for(6u * aa.nAO, 128), 128, 0, st>>>(aa, s.acc, s.alpha, k.err);
    }
}

// the most force blocks any shape launches for n contacts (the wall partials are sized for it)
uint32_t force_blocks(uint32_t n) { return blocks_for(n, 64); }

// ChangeFamily (src/DEM/APIPublic.cpp:184-208): every owner of family `from` moves to family `to`.
__global__ void k_change_family(ushort4* loc, uint32_t n, uint32_t from, uint32_t to) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    ushort4 l = loc[o];
    if (l.w == from) {
        l.w = (unsigned short)to;
        loc[o] = l;
    }
}
void launch_change_family(ushort4* loc, uint32_t n, uint32_t from, uint32_t to, cudaStream_t st) {
    if (!n) return;
    ProfScope prof_(KID_OTHER, st);
    k_change_family<<<blocks_for(n, 256), 256, 0, st>>>(loc, n, from, to);
}

// One entry of the family-mask table, written in stream order (no host buffer has to outlive the call).
__global__ void k_set_mask(uint8_t* masks, uint32_t index, uint8_t value) { masks[index] = value; }
void launch_set_mask(uint8_t* masks, uint32_t index, uint8_t value, cudaStream_t st) {
    ProfScope prof_(KID_OTHER, st);
    k_set_mask<<<1, 1, 0, st>>>(masks, index, value);
}

// The simulation time on the device (read by the family-change rules and prescribed-motion expressions): a float
// advanced by h once per step, as the reference's dT advances timeElapsed (src/DEM/dT.cpp:1585).  A voided step
// does not advance it.
__global__ void k_advance_time(float* time, float h, const uint32_t* err) {
    if (*err == 0u) *time = *time + h;
}
void launch_advance_time(float* time, float h, const uint32_t* err, cudaStream_t st) {
    ProfScope prof_(KID_OTHER, st);
    k_advance_time<<<1, 1, 0, st>>>(time, h, err);
}
__global__ void k_set_time(float* time, float t) { *time = t; }

// The contact-pair parameter table of the built-in model (contact_params for every ordered material pair).
__global__ void k_material_pairs(MaterialTable m, uint32_t nM, float4* out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nM * nM) return;
    float E, G, CoR, mu, Crr, beta;
    contact_params(m, p / nM, p % nM, E, G, CoR, mu, Crr, beta);
    out[2u * p] = make_float4(E, G, CoR, mu);
    out[2u * p + 1u] = make_float4(Crr, beta, 0.f, 0.f);
}
void launch_material_pairs(const MaterialTable& m, uint32_t nM, float4* out, cudaStream_t st) {
    if (!nM || !out) return;
    ProfScope prof_(KID_OTHER, st);
    k_material_pairs<<<blocks_for(nM * nM, 256), 256, 0, st>>>(m, nM, out);
}
void launch_set_time(float* time, float t, cudaStream_t st) {
    ProfScope prof_(KID_OTHER, st);
    k_set_time<<<1, 1, 0, st>>>(time, t);
}

// End of a replayed window: counts the windows that completed without a device error.
__global__ void k_window_done(const uint32_t* err, uint32_t* done) {
    if (*err == 0u) atomicAdd(done, 1u);
}
void launch_window_done(const uint32_t* err, uint32_t* done, cudaStream_t st) {
    ProfScope prof_(KID_OTHER, st);
    k_window_done<<<1, 1, 0, st>>>(err, done);
}

// ------------------------------------------------------------------------------------------------------------
// integrateOwners (src/kernel/DEMIntegrationKernels.cu:46-179) with the constant prescription table.
__global__ void __launch_bounds__(512) k_integrate(SimConsts k, StateView s) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= k.n_owners) return;
    if (*k.err != 0u) return;  // a voided step (see k_force) leaves the state as it was
    integrate_owner(k, s, o, 0.f, TableMotion{s.presc});
}

void launch_integrate(const SimConsts& k, const StateView& s, uint32_t threads, cudaStream_t st) {
    if (!(k.n_owners)) return;
    ProfScope prof_(KID_INTEGRATE, st);
    if (k.n_owners) k_integrate<<<blocks_for(k.n_owners, threads), threads, 0, st>>>(k, s);
}

// Kinetic energy of clump owners: per-owner term of DEMOwnerQueryKernels.cu:10-37, summed in double.
__global__ void k_kinetic_energy(SimConsts k, StateView s, uint32_t nClumps, double* out) {
    __shared__ double sh[32];
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (o < nClumps) {
        const float4 v = s.vel[o], w = s.omg[o], I = s.moi[o];
        const double v2 = (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
        const double r2 = (double)I.x * w.x * w.x + (double)I.y * w.y * w.y + (double)I.z * w.z * w.z;
        e = 0.5 * (double)v.w * v2 + 0.5 * r2;
    }
    for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        e = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
        if (threadIdx.x == 0) atomicAdd(out, e);
    }
}

void launch_kinetic_energy(const SimConsts& k, const StateView& s, uint32_t n_clumps, double* out, cudaStream_t st) {
    if (!(true)) return;
    ProfScope prof_(KID_OTHER, st);
    cudaMemsetAsync(out, 0, sizeof(double), st);
    if (n_clumps) k_kinetic_energy<<<blocks_for(n_clumps, 256), 256, 0, st>>>(k, s, n_clumps, out);
}

// ------------------------------------------------------------------------------------------------------------
// Reference bin assignment (getNumberOfBinsEachSphereTouches / populateBinSphereTouchingPairs): parity path only.
__global__ void k_bin_count(SimConsts k, StateView s, uint16_t* nBins, uint8_t* nAnal) {
    const uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= k.n_spheres) return;
    uint32_t owner;
    float4 sp;
    double X, Y, Z;
    sphere_center(k, s, sid, owner, sp, X, Y, Z);
    double rD = (double)sp.w;
    rD += (double)k.beta;
    uint32_t lo[3], hi[3];
    bin_range(X, rD, k.bin_size, lo[0], hi[0]);
    bin_range(Y, rD, k.bin_size, lo[1], hi[1]);
    bin_range(Z, rD, k.bin_size, lo[2], hi[2]);
    const uint16_t nx = (uint16_t)(hi[0] - lo[0] + 1u), ny = (uint16_t)(hi[1] - lo[1] + 1u),
                   nz = (uint16_t)(hi[2] - lo[2] + 1u);
    nBins[sid] = (uint16_t)((int)nx * (int)ny * (int)nz);
    const uint32_t fam = s.loc[owner].w;
    uint32_t c = 0;
    const uint2 ar = anal_range(s, owner);
    for (uint32_t a = ar.x; a < ar.x + ar.y; a++) {
        const AnalPlaced ap = s.anal[a];
        if (s.masks[mask_index(fam, s.loc[ap.owner].w)] != 0) continue;
        if (anal_overlap_cd(ap, X, Y, Z, rD, k.beta) != DEME_NOT_A_CONTACT) c++;
    }
    nAnal[sid] = (uint8_t)c;
}

__global__ void k_bin_emit(SimConsts k, StateView s, const uint32_t* off, uint32_t* bins, uint32_t* sph) {
    const uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= k.n_spheres) return;
    uint32_t owner;
    float4 sp;
    double X, Y, Z;
    sphere_center(k, s, sid, owner, sp, X, Y, Z);
    double rD = (double)sp.w;
    rD += (double)k.beta;
    uint32_t lo[3], hi[3];
    bin_range(X, rD, k.bin_size, lo[0], hi[0]);
    bin_range(Y, rD, k.bin_size, lo[1], hi[1]);
    bin_range(Z, rD, k.bin_size, lo[2], hi[2]);
    uint32_t w = off[sid];
    for (uint32_t kk = lo[2]; kk <= hi[2]; kk++)
        for (uint32_t j = lo[1]; j <= hi[1]; j++)
            for (uint32_t i = lo[0]; i <= hi[0]; i++) {
                bins[w] = i + j * k.nbX + kk * k.nbX * k.nbY;
                sph[w] = sid;
                w++;
            }
}

void launch_bin_count(const SimConsts& k, const StateView& s, uint16_t* nBins, uint8_t* nAnal, cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_OTHER, st);
    if (k.n_spheres) k_bin_count<<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, nBins, nAnal);
}
void launch_bin_emit(const SimConsts& k, const StateView& s, const uint32_t* off, uint32_t* bins, uint32_t* sph,
                     cudaStream_t st) {
    if (!(k.n_spheres)) return;
    ProfScope prof_(KID_OTHER, st);
    if (k.n_spheres) k_bin_emit<<<blocks_for(k.n_spheres, 256), 256, 0, st>>>(k, s, off, bins, sph);
}

}  // namespace deme_b200
