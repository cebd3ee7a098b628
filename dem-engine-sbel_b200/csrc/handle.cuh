// handle.cuh -- the solver handle behind the C ABI and the host helpers shared by capi.cu and adjoint.cu.
#pragma once
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/deme_b200.h"
#include "force_jit.cuh"
#include "kernels.cuh"

using namespace deme_b200;

struct AdjointTape;  // adjoint.cu

struct ContactBuf {
    uint32_t cap = 0;
    uint32_t* idA = nullptr;
    uint32_t* idB = nullptr;
    uint8_t* type = nullptr;
    float4* hist = nullptr;
    uint32_t* mapping = nullptr;
    uint32_t* off = nullptr;  // nS + 1, allocated once
    uint32_t* dN = nullptr;   // the list's contact count on the device, allocated once
    ContactView view() const { return ContactView{idA, idB, type, hist, mapping, off, dN}; }
};

// Owner state and contact list at one step (adjoint checkpoints, graph-replay rollback).
struct Checkpoint {
    uint64_t* voxel = nullptr;
    ushort4* loc = nullptr;
    float4* quat = nullptr;
    float4* vel = nullptr;
    float4* omg = nullptr;
    uint32_t n = 0, cap = 0;
    uint32_t* idA = nullptr;
    uint32_t* idB = nullptr;
    uint8_t* type = nullptr;
    float4* hist = nullptr;
    uint32_t* off = nullptr;
    int64_t steps = 0;
    double t = 0.0;
    float tf = 0.f;
};

struct deme_handle {
    std::string err;
    int device = 0;
    cudaStream_t st_dt = nullptr, st_kt = nullptr;
    cudaStream_t own_dt = nullptr, own_kt = nullptr;
    deme_sim_params params{};
    SimConsts k{};
    uint32_t nO = 0, nS = 0, nA = 0, nM = 0, nClumps = 0;
    int nW = 0;
    // scene and state
    uint64_t* voxel = nullptr;
    ushort4* loc = nullptr;
    float4* quat = nullptr;
    float4* vel = nullptr;
    float4* omg = nullptr;
    float4* moi = nullptr;
    float4* invMoi = nullptr;
    float4* acc = nullptr;
    float4* alpha = nullptr;
    float4* sph = nullptr;
    uint32_t* sOwner = nullptr;
    uint16_t* sMat = nullptr;
    uint8_t* masks = nullptr;
    float* mat = nullptr;  // 5 x nM
    float4* matPair = nullptr;  // contact-pair parameters, 2 x nM x nM (kMaxPairTableMaterials materials at most)
    AnalRaw* analRaw = nullptr;
    AnalPlaced* analPlaced = nullptr;
    bool analFresh = false;  // analPlaced holds the placement for the current poses (a detection of this step made it)
    Prescription* presc = nullptr;
    uint2* ownerAnal = nullptr;  // packed scenes: per owner (first, count) of its analytical components
    uint32_t nT = 0;             // mesh facets
    TriRaw* triRaw = nullptr;
    TriPlaced* triPlaced = nullptr;  // placed with analPlaced (analFresh covers both)
    // contact detection
    CDView cd{};
    uint32_t nCells = 0;
    uint32_t cellCap = 0;  // cells the cell arrays hold (the finest grid's count when they were sized)
    int cellBits = 0;
    SearchGrid* grids = nullptr;         // per scene (one for a plain run): see set_cell_grid
    uint32_t* ownerScene = nullptr;      // packed scenes: scene of each owner
    std::vector<double> sceneBox;        // per scene: lower and upper corner of its search grid (6 doubles)
    std::vector<float> sceneRmax;        // per scene: largest expanded radius
    uint32_t candCap = 0;
    ContactBuf lists[2];
    int cur = 0;
    uint32_t nContacts = 0;
    // per-contact outputs
    bool keepOutputs = false;
    bool useOnesweep = false;  // sort spheres by cell with the multi-pass onesweep instead of the counting sort
    uint32_t outCap = 0;
    ContactOutputs outs{nullptr, nullptr, nullptr, nullptr};
    bool outsValid = false;
    // scratch
    void* scratch = nullptr;
    size_t scratchBytes = 0;
    uint32_t* dTotal = nullptr;
    uint32_t* hTotal = nullptr;
    uint32_t* dErr = nullptr;
    uint32_t* hErr = nullptr;
    double* dKE = nullptr;
    double* hKE = nullptr;
    // ring of kinetic-energy results read without a wait (deme_kinetic_energy_enqueue / _collect)
    static constexpr int kKESlots = 4;
    double* dKERing = nullptr;
    double* hKERing = nullptr;
    cudaEvent_t keDone[kKESlots] = {};
    int64_t keSlotTicket[kKESlots] = {-1, -1, -1, -1};
    int64_t keTickets = 0;
    // pinned staging ring for deme_set_family_prescription: slot i may be rewritten once its copy has run
    static constexpr int kPrescSlots = 8;
    Prescription* hPresc = nullptr;
    cudaEvent_t prescDone[kPrescSlots] = {};
    int prescNext = 0;
    float* analPartial = nullptr;
    float* analChunks = nullptr;  // range sums of the wall partials (6 x analytical owners x kAnalChunks)
    size_t analPartialCap = 0;
    double t = 0.0;
    float tf = 0.f;  // the time as the reference's dT keeps it (a float, advanced by h each step): rules and
                     // prescribed-motion expressions see this one
    int64_t steps = 0;
    std::vector<void*> allocs;
    UserForceKernel userForce;  // a compiled force-model string, when one is set
    FamilyChangeKernel famRules;  // compiled ChangeFamilyWhen rules, when some are set
    MotionKernel motion;          // compiled prescribed-motion expressions, when some are set
    uint64_t jitGeneration = 0;   // counts changes of the run-time compiled kernels (recorded graphs hold them)
    float* dTime = nullptr;       // tf on the device (rules and expressions read it), advanced once per step
    AdjointTape* adj = nullptr;  // checkpoints of deme_adjoint_record
    // Asynchronous contact detection (kT on st_kt, dT on st_dt).  With cdLag > 0 a detection due at step k runs on
    // kT from a snapshot of the owner poses of step k while dT keeps stepping with the current list, and dT adopts
    // the new list at step k + cdLag.
    // search shape (deme_set_search_shape / deme_autotune): candidate-scan block shape and search-cell factor
    int32_t findShape = 0;
    float cellFactor = 1.f;
    // block shapes of the force kernel, the exact pair test and the integration (deme_set_kernel_shapes)
    int32_t forceShape = 0;
    uint32_t exactThreads = 256;
    uint32_t integrateThreads = 256;
    // CUDA-graph replay of whole steps (deme_set_graph): one executable graph per parity of `cur` at the start of
    // a detection window, keyed by everything its launches captured.
    bool useGraph = false;
    bool capturing = false;   // the step functions are being recorded: no host reads, launches cover capacities
    bool countStale = false;  // the list in use came out of a graph replay: its count is on the device only
    cudaGraphExec_t graphExec[2] = {nullptr, nullptr};
    int64_t graphKernels[2] = {0, 0};  // kernel launches recorded in each graph
    std::vector<uint8_t> graphKey[2];
    uint32_t* dWindows = nullptr;  // windows of a replayed batch that completed without a device error
    uint32_t* hWindows = nullptr;  // pinned: that count, then the error word
    int64_t graphReplays = 0, graphRollbacks = 0;
    int32_t cdLag = 0;
    bool cdPending = false;
    bool everDetected = false;
    int64_t cdAdoptStep = 0;
    uint64_t* kVoxel = nullptr;  // kT's snapshot of the owner poses (and families) of the detection step
    ushort4* kLoc = nullptr;
    float4* kQuat = nullptr;
    AnalPlaced* kAnalPlaced = nullptr;  // analytical components placed from that snapshot
    TriPlaced* kTriPlaced = nullptr;    // mesh facets placed from that snapshot
    uint32_t* hCounts = nullptr;        // pinned: total, pool count, overflow spheres, -, mesh pairs,
                                        // copied at the end of kT's part (8 words)
    cudaEvent_t evPose = nullptr, evCounts = nullptr, evListReady = nullptr, evListReleased = nullptr;
    StateView kt_view() const {
        StateView s = state_view();
        s.voxel = kVoxel;
        s.loc = kLoc;
        s.quat = kQuat;
        s.anal = kAnalPlaced;
        s.tri = kTriPlaced;
        return s;
    }

    StateView state_view() const {
        StateView s;
        s.voxel = voxel;
        s.loc = loc;
        s.quat = quat;
        s.vel = vel;
        s.omg = omg;
        s.moi = moi;
        s.invMoi = invMoi;
        s.acc = acc;
        s.alpha = alpha;
        s.sph = sph;
        s.sOwner = sOwner;
        s.sMat = sMat;
        s.masks = masks;
        s.mat = MaterialTable{mat, mat + nM, mat + 2 * nM, mat + 3 * nM, mat + 4 * nM, matPair, nM};
        s.anal = analPlaced;
        s.nA = nA;
        s.presc = presc;
        s.ownerAnal = ownerAnal;
        s.tri = triPlaced;
        return s;
    }
};

int32_t alloc_checkpoint(deme_handle* h, Checkpoint& c, uint32_t nContacts);
void free_checkpoint(deme_handle* h, Checkpoint& c);
int32_t save_checkpoint(deme_handle* h, Checkpoint& c);
int32_t restore_checkpoint(deme_handle* h, const Checkpoint& c);
int32_t refresh_count(deme_handle* h);
int32_t refresh_material_pairs(deme_handle* h);

#define CUDA_TRY(h, expr)                                                                        \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            (h)->err = std::string(#expr) + ": " + cudaGetErrorString(e_);                       \
            return e_ == cudaErrorMemoryAllocation ? DEME_ERR_OOM : DEME_ERR_CUDA;               \
        }                                                                                        \
    } while (0)

#define TRY(expr)                      \
    do {                               \
        int32_t s_ = (expr);           \
        if (s_ != DEME_OK) return s_;  \
    } while (0)

int32_t dalloc(deme_handle* h, void** p, size_t bytes);
void dfree(deme_handle* h, void* p);
int32_t check_launch(deme_handle* h, const char* what);
int32_t read_device_errors(deme_handle* h);
int32_t ensure_list(deme_handle* h, ContactBuf& b, uint32_t n);
void adjoint_release(deme_handle* h);  // adjoint.cu

template <typename T>
inline int32_t dalloc_n(deme_handle* h, T** p, size_t n) {
    return dalloc(h, reinterpret_cast<void**>(p), n * sizeof(T));
}
