// kernels.cuh -- device data views and host launchers of the per-step kernels.
#pragma once
#ifndef __CUDACC_RTC__
#include <cstdint>
#include <cuda_runtime.h>
#endif

#include "device_common.cuh"
#include "force_model_hertz.cuh"

namespace deme_b200 {

// Owner and sphere arrays in HBM (layout documented in device_common.cuh).
struct StateView {
    uint64_t* voxel;
    ushort4* loc;   // (locX, locY, locZ, family)
    float4* quat;   // (w, x, y, z)
    float4* vel;    // (vx, vy, vz, mass)
    float4* omg;    // (wx, wy, wz, 0)
    const float4* moi;
    const float4* invMoi;  // (1 / Ixx, 1 / Iyy, 1 / Izz, 1 / mass), for the accelerations of the force kernel
    float4* acc;    // force accumulators (a)
    float4* alpha;  // torque accumulators (alpha)
    const float4* sph;  // (relX, relY, relZ, radius)
    const uint32_t* sOwner;
    const uint16_t* sMat;
    const uint8_t* masks;
    MaterialTable mat;
    const AnalPlaced* anal;
    uint32_t nA;
    const Prescription* presc;  // DEME_NUM_FAMILIES entries
    const uint2* ownerAnal;     // per owner (first, count) of the analytical components it meets; null = all
    TriPlaced* tri;             // mesh facets placed at these poses (n_tris of them)
};

// Raw analytical component description (scene constants).
struct AnalRaw {
    float relX, relY, relZ, rotX, rotY, rotZ, size1, size2, size3, mass;
    uint32_t owner;
    uint8_t type, normal;
    uint16_t material;
    double c1, c2;
};

// Raw mesh facet (scene constants): the nodes in the owner frame (kT's relPosNode1..3), owner, material and the
// owner's mass.
struct TriRaw {
    float n1x, n1y, n1z, n2x, n2y, n2z, n3x, n3y, n3z, mass;
    uint32_t owner;
    uint16_t material, pad;
};

// Cell-order record of one sphere for the exact pair test: 32 bytes, read as two 16-byte loads.
struct __align__(16) SphCD {
    double x, y, z;
    uint32_t owner;
    float rf;  // radius + beta, added in float as the reference does
};

// Contact-detection work arrays.
struct CDView {
    float4* posFSorted;  // cell order: (x, y, z, sphere id bits)
    SphCD* recS;         // cell order: exact position, owner, expanded radius
    uint4* rngS;         // cell order: bin ranges of the expanded sphere, (lo | hi << 16) per axis; family in .w
    const uint2* sClump; // ID order: (first sphere, count) of the run of consecutive spheres sharing the owner
    uint32_t* cellKey;
    uint32_t* idSeq;
    uint32_t* keySorted;
    uint32_t* idSorted;
    uint32_t* cellCount;  // nCells + 1
    uint32_t* cellStart;  // nCells + 1
    uint8_t* nAnal;
    uint32_t* cnt;
    uint2* candTemp;      // pair pool: for each survivor of the candidate scan, the exact test's verdict: the
                          // pair (A, B), A < B by id, or kNoPair; in no particular order
    uint32_t* ovf;        // spheres with more pre-filter survivors than the candidate scan's slots hold
    uint32_t* counters;   // [0] pair-pool entries (survivors) appended, [1] overflow spheres, [2] the candidate
                          // scan's tile queue, [3] pool entries the overflow search appended (tested last),
                          // [4] mesh-pool entries appended
    // sphere--mesh contacts (n_tris > 0 only): the (sphere, facet) pairs the facet-driven search found, in no
    // particular order
    uint2* meshPool;
    uint32_t meshCap;
};

// One contact list (kT product) with its history wildcards.
struct ContactView {
    uint32_t* idA;
    uint32_t* idB;
    uint8_t* type;
    float4* hist;       // (delta_tan_x, delta_tan_y, delta_tan_z, delta_time)
    uint32_t* mapping;
    uint32_t* off;      // CSR offsets by sphere (nS + 1)
    uint32_t* dN;       // number of contacts, on the device (written by the scan that makes the offsets)
};

// Reactions on analytical owners (walls): block partials, reduced in fixed order.
struct AnalAccum {
    float* partial;     // blocks x nAO x 6
    float* chunks;      // (nAO x 6) x kAnalChunks sums of contiguous ranges of block partials
    uint32_t nClumps;   // analytical owners are [nClumps, nClumps + nAO)
    uint32_t nAO;
    bool direct;        // many analytical owners: float atomics onto their accumulators instead of partials
};

struct ContactOutputs {
    float4* F;
    float4* TOF;
    float4* CPA;
    float4* CPB;
};

#ifndef __CUDACC_RTC__
void launch_place_anal(const SimConsts& k, const StateView& s, const AnalRaw* raw, AnalPlaced* placed, uint32_t nA,
                       cudaStream_t st);
void launch_place_tri(const SimConsts& k, const StateView& s, const TriRaw* raw, cudaStream_t st);
// the sphere--mesh pairs, once the spheres are in cell order (adds to the spheres' contact counts)
void launch_mesh_find(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st);
// the mesh pool's pairs into their spheres' segments (after the contact offsets), tagged with kMeshTag
void launch_mesh_scatter(const SimConsts& k, const CDView& cd, const ContactView& c, uint32_t nPairs, uint32_t cap,
                         cudaStream_t st);
// a facet id placed in a segment before the assembly sorts it (sphere ids stay below it)
constexpr uint32_t kMeshTag = 0x80000000u;
void launch_sphere_prep(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st);
void launch_cell_scatter(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st);
void launch_gather_sorted(const SimConsts& k, const StateView& s, const CDView& cd, cudaStream_t st);
void launch_pair_find(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t tempCap, int shape,
                      cudaStream_t st);
int find_shape_count();  // block shapes of the candidate scan
// warps per block, survivor slots per lane and work-queue (persistent) form of shape v
void find_shape(int v, uint32_t* warps, uint32_t* slots, bool* persistent);
void launch_pair_overflow(const SimConsts& k, const StateView& s, const CDView& cd, uint32_t tempCap, cudaStream_t st);
// ranges the wall partials of the force blocks are first summed over (then the range sums, in order)
constexpr uint32_t kAnalChunks = 32;
// a pair-pool entry that the exact test rejected
constexpr uint32_t kNoPair = 0xFFFFFFFFu;
void launch_cnt_init(const SimConsts& k, const CDView& cd, cudaStream_t st);
void launch_pair_scatter(const SimConsts& k, const CDView& cd, const ContactView& c, uint32_t nPairs, uint32_t cap,
                         uint32_t poolCap, cudaStream_t st);
void launch_pair_assemble(const SimConsts& k, const StateView& s, const CDView& cd, const ContactView& c, uint32_t cap,
                          cudaStream_t st);
void launch_history(const SimConsts& k, const ContactView& cur, const ContactView& prev, uint32_t n, uint32_t prevN,
                    bool has_hist, cudaStream_t st);
void launch_count_by_sphere(const uint32_t* idA, uint32_t n, uint32_t* cnt, cudaStream_t st);
struct UserForceKernel;
void launch_force(const SimConsts& k, const StateView& s, const ContactView& c, uint32_t n, bool has_hist,
                  const ContactOutputs* out, const AnalAccum& aa, const UserForceKernel* user, int shape,
                  cudaStream_t st);
uint32_t force_blocks(uint32_t n);
int force_shape_count();                 // block shapes of the force kernel
uint32_t force_shape_threads(int shape);
void launch_window_done(const uint32_t* err, uint32_t* done, cudaStream_t st);
void launch_change_family(ushort4* loc, uint32_t n, uint32_t from, uint32_t to, cudaStream_t st);
void launch_set_mask(uint8_t* masks, uint32_t index, uint8_t value, cudaStream_t st);
void launch_advance_time(float* time, float h, const uint32_t* err, cudaStream_t st);
void launch_set_time(float* time, float t, cudaStream_t st);
// Scenes with at most this many materials keep a table of contact-pair parameters (2 float4 per ordered pair).
constexpr uint32_t kMaxPairTableMaterials = 256;
void launch_material_pairs(const MaterialTable& m, uint32_t nM, float4* out, cudaStream_t st);
void launch_integrate(const SimConsts& k, const StateView& s, uint32_t threads, cudaStream_t st);
void launch_kinetic_energy(const SimConsts& k, const StateView& s, uint32_t n_clumps, double* out, cudaStream_t st);

// Reference bin assignment (parity path).
void launch_bin_count(const SimConsts& k, const StateView& s, uint16_t* nBins, uint8_t* nAnal, cudaStream_t st);
void launch_bin_emit(const SimConsts& k, const StateView& s, const uint32_t* off, uint32_t* bins, uint32_t* sph,
                     cudaStream_t st);
#endif

}  // namespace deme_b200
