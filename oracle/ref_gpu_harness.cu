// ref_gpu_harness.cu -- host driver that runs the reference's own kernels on the GPU.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  oracle/ref_gpu_build.py substitutes the reference's kernel templates
// (src/kernel/*.cu) the way its JitHelper does (src/core/utils/JitHelper.cpp:36-59) and compiles each program with
// NVRTC for sm_100a, as its jitify layer does at run time, into cubins under oracle/_ref/gpu-<key>/.  This driver
// loads those cubins and launches the reference's kernels in the order of its kT and dT threads on one stream:
//   * contactDetection (src/algorithms/DEMCubContactDetection.cu:39-397): bins per sphere, two scans, bin--sphere
//     pairs, a radix sort by bin, run-length encoding of active bins, the default block-per-bin contact kernels
//     (src/kernel/DEMContactKernels_Blockwise.cu) or the thread-per-bin ones (src/kernel/DEMContactKernels.cu),
//     two stable sorts by idA and the history map;
//   * the kT -> dT hand-over of the contact list and the dT -> kT hand-over of owner poses (src/DEM/kT.cpp:75-99,
//     src/DEM/dT.cpp:1202-1230);
//   * migratePersistentContacts, calculateForces and collectContactForces (src/DEM/dT.cpp:1258-1422,
//     src/algorithms/DEMCubForceCollection.cu:20-158): per-contact owner keys, per-side accelerations, a radix sort
//     and a reduce-by-key per quantity, then the stash;
//   * integrateOwners (src/kernel/DEMIntegrationKernels.cu:170-179).
// The device-wide primitives are CUB's, called as the reference's wrappers call them
// (src/algorithms/DEMCubWrappers.cu): ExclusiveScan with the output type's zero, SortPairs over all key bits,
// RunLengthEncode::Encode and ReduceByKey with a float3 sum.
//
// With `sync_each` set, the stream is synchronised after every launch and every primitive, as the reference's host
// code does; without it, only the count read-backs the next launch needs synchronise.
//
// The reference's contact kernels trap when a bin holds more than DEME_MAX_SPHERES_PER_BIN spheres
// (src/kernel/DEMContactKernels_Blockwise.cu:42-45, src/kernel/DEMContactKernels.cu:38-41).  Before they are launched this driver reduces the per-bin counts
// on the device, reads the maximum back and returns DEME_ERR_OVERFLOW without launching them if the limit would be
// exceeded, so that condition is never reached on the GPU.
#include <DEM/Defines.h>

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../include/deme_b200.h"

namespace {

struct Float3Sum {
    __host__ __device__ __forceinline__ float3 operator()(const float3& a, const float3& b) const {
        return make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
    }
};

struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
};

enum KernelId {
    K_BIN_COUNT,
    K_BIN_EMIT,
    K_CNT_EACH_BIN,
    K_POP_EACH_BIN,
    K_FILL_RL,
    K_BUILD_MAP,
    K_PREP_FORCE,
    K_REARRANGE_WC,
    K_CALC_FORCE,
    K_CASH_A,
    K_CASH_B,
    K_FORCE_TO_ACC,
    K_FORCE_TO_ANG_ACC,
    K_STASH,
    K_INTEGRATE,
    K_CNT_EACH_BIN_T,
    K_POP_EACH_BIN_T,
    K_COUNT
};

// program (cubin file stem) and kernel name of each entry; the lowered names come from the build's kernels.txt
const char* const kProgram[K_COUNT] = {
    "DEMBinSphereKernels",      "DEMBinSphereKernels",      "DEMContactKernels_Blockwise", "DEMContactKernels_Blockwise",
    "DEMHistoryMappingKernels", "DEMHistoryMappingKernels", "DEMPrepForceKernels",         "DEMPrepForceKernels",
    "DEMCalcForceKernels",      "DEMCollectForceKernels",   "DEMCollectForceKernels",      "DEMCollectForceKernels",
    "DEMCollectForceKernels",   "DEMCollectForceKernels",   "DEMIntegrationKernels",       "DEMContactKernels",
    "DEMContactKernels"};
const char* const kName[K_COUNT] = {"getNumberOfBinsEachSphereTouches",
                                    "populateBinSphereTouchingPairs",
                                    "getNumberOfContactsEachBin",
                                    "populateContactPairsEachBin",
                                    "fillRunLengthArray",
                                    "buildPersistentMap",
                                    "prepareForceArrays",
                                    "rearrangeContactWildcards",
                                    "calculateContactForces",
                                    "cashInOwnerIndexA",
                                    "cashInOwnerIndexB",
                                    "forceToAcc",
                                    "forceToAngAcc",
                                    "stashElem",
                                    "integrateOwners",
                                    "getNumberOfContactsEachBin",
                                    "populateContactPairsEachBin"};

inline unsigned blocks_for(size_t n, size_t per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

struct refg_ctx {
    std::string err;
    cudaStream_t stream = nullptr;
    bool sync_each = false;
    bool one_bin_per_thread = false;  // the reference's SetOneBinPerThread (src/DEM/API.h:140); default block per bin
    std::vector<cudaLibrary_t> libs;
    cudaKernel_t k[K_COUNT] = {};

    deme::DEMSimParams sp;
    deme::DEMDataKT kt;
    deme::DEMDataDT dt;
    deme::DEMSimParams* d_sp = nullptr;
    deme::DEMDataKT* d_kt = nullptr;
    deme::DEMDataDT* d_dt = nullptr;

    uint32_t nO = 0, nS = 0;
    int nW = 0;
    int cd_freq = 0;
    double t = 0;
    float tf = 0.f;  // the time as the reference's dT keeps it (float timeElapsed, src/DEM/dT.h:216)
    int64_t steps = 0;
    size_t nC = 0, nPrev = 0;

    std::vector<void*> owned;  // fixed-size device arrays
    // kT- and dT-side owner poses (dT integrates its own copy; kT reads the copy handed over before each CD)
    uint64_t* kVoxel = nullptr;
    uint16_t *kLocX = nullptr, *kLocY = nullptr, *kLocZ = nullptr;
    float *kQw = nullptr, *kQx = nullptr, *kQy = nullptr, *kQz = nullptr;
    uint8_t* kFam = nullptr;
    // growable arrays
    DBuf idA, idB, type, map;       // kT contact list
    DBuf pA, pB, pT;                // kT previous list
    DBuf dIdA, dIdB, dType, dMap;   // dT copy of the contact list
    DBuf F, TOF, CPA, CPB;          // dT per-contact outputs
    DBuf wc[DEME_MAX_WILDCARDS];    // dT wildcards
    DBuf newWc, sentry;
    DBuf numBins, numAnal, binScan, analScan, binIDs, sphIDs, pairBin, pairSph, activeBins, numSphBin, lookUp;
    DBuf numCnt, offs, newU, oldU, newRL, oldRL, newFull, oldFull, newScan, oldScan, sortTmpA, sortTmpB, sortTmpT;
    DBuf owners, ownersSorted, acc, accSorted, uniq, accOwner;
    DBuf cubTmp;
    size_t* d_count = nullptr;  // device-side count written by CUB (runs, maxima)
    uint32_t* d_max16 = nullptr;
    // phase profiling: events recorded at the phase boundaries of a step while `profiling` is set
    bool profiling = false;
    cudaEvent_t ev[11] = {};
};

namespace {

bool fail(refg_ctx* c, const char* what, cudaError_t e) {
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}
#define RG_TRY(expr)                                      \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return fail(c, #expr, e_); \
    } while (0)

bool grow(refg_ctx* c, DBuf& b, size_t bytes, bool keep) {
    if (bytes <= b.cap) return true;
    size_t cap = bytes + bytes / 4 + 256;
    void* p = nullptr;
    RG_TRY(cudaMalloc(&p, cap));
    if (keep && b.p && b.cap) RG_TRY(cudaMemcpyAsync(p, b.p, b.cap, cudaMemcpyDeviceToDevice, c->stream));
    if (b.p) {
        RG_TRY(cudaStreamSynchronize(c->stream));
        RG_TRY(cudaFree(b.p));
    }
    b.p = p;
    b.cap = cap;
    return true;
}

template <typename T>
T* P(DBuf& b) {
    return static_cast<T*>(b.p);
}

// Phase boundaries of a step: 0 start, 1 bins per sphere + scans + bin--sphere pairs, 2 sort by bin, 3 active bins,
// 4 pair kernels, 5 sort by idA, 6 history map, 7 hand-over + history remap, 8 force kernel, 9 force collection,
// 10 integration.
constexpr int kPhases = 10;
void mark(refg_ctx* c, int k) {
    if (c->profiling) cudaEventRecord(c->ev[k], c->stream);
}

bool sync_if(refg_ctx* c) {
    if (c->sync_each) RG_TRY(cudaStreamSynchronize(c->stream));
    return true;
}

bool launch(refg_ctx* c, KernelId id, unsigned grid, unsigned block, void** args) {
    if (grid == 0) return true;
    RG_TRY(cudaLaunchKernel((const void*)c->k[id], dim3(grid), dim3(block), args, 0, c->stream));
    return sync_if(c);
}

template <typename T>
bool read_back(refg_ctx* c, const T* dsrc, T& out) {
    RG_TRY(cudaMemcpyAsync(&out, dsrc, sizeof(T), cudaMemcpyDeviceToHost, c->stream));
    RG_TRY(cudaStreamSynchronize(c->stream));
    return true;
}

// CUB calls: size query, then the run, with the scratch growing as needed
template <typename F>
bool cub_call(refg_ctx* c, F&& f) {
    size_t bytes = 0;
    RG_TRY(f((void*)nullptr, bytes));
    if (!grow(c, c->cubTmp, bytes, false)) return false;
    size_t cap = c->cubTmp.cap;
    RG_TRY(f(c->cubTmp.p, cap));
    return sync_if(c);
}

template <typename TIn, typename TOut>
bool exclusive_scan(refg_ctx* c, const TIn* in, TOut* out, size_t n) {
    if (n == 0) return true;
    return cub_call(c, [&](void* tmp, size_t& bytes) {
        return cub::DeviceScan::ExclusiveScan(tmp, bytes, in, out, cuda::std::plus<>{}, (TOut)0, (int64_t)n,
                                              c->stream);
    });
}
template <typename K, typename V>
bool sort_pairs(refg_ctx* c, const K* kin, K* kout, const V* vin, V* vout, size_t n) {
    if (n == 0) return true;
    return cub_call(c, [&](void* tmp, size_t& bytes) {
        return cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, (int64_t)n, 0, (int)(sizeof(K) * 8),
                                               c->stream);
    });
}
template <typename K, typename C>
bool rle(refg_ctx* c, const K* in, K* uniq, C* counts, size_t n, size_t& runs) {
    runs = 0;
    if (n == 0) return true;
    if (!cub_call(c, [&](void* tmp, size_t& bytes) {
            return cub::DeviceRunLengthEncode::Encode(tmp, bytes, in, uniq, counts, c->d_count, (int64_t)n,
                                                      c->stream);
        }))
        return false;
    return read_back(c, c->d_count, runs);
}

// dT's owner state arrays and the rest of the fixed layout
template <typename T>
bool dev_copy(refg_ctx* c, T*& dst, const T* src, size_t n, size_t extra = 0) {
    size_t bytes = (n + extra) * sizeof(T);
    if (bytes == 0) bytes = sizeof(T);
    void* p = nullptr;
    RG_TRY(cudaMalloc(&p, bytes));
    c->owned.push_back(p);
    RG_TRY(cudaMemset(p, 0, bytes));
    if (src && n) RG_TRY(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice));
    dst = static_cast<T*>(p);
    return true;
}

bool upload_views(refg_ctx* c) {
    deme::DEMDataKT& kt = c->kt;
    kt.idGeometryA = P<uint32_t>(c->idA);
    kt.idGeometryB = P<uint32_t>(c->idB);
    kt.contactType = P<uint8_t>(c->type);
    kt.contactMapping = P<uint32_t>(c->map);
    kt.previous_idGeometryA = P<uint32_t>(c->pA);
    kt.previous_idGeometryB = P<uint32_t>(c->pB);
    kt.previous_contactType = P<uint8_t>(c->pT);
    deme::DEMDataDT& dt = c->dt;
    dt.idGeometryA = P<uint32_t>(c->dIdA);
    dt.idGeometryB = P<uint32_t>(c->dIdB);
    dt.contactType = P<uint8_t>(c->dType);
    dt.contactMapping = P<uint32_t>(c->dMap);
    dt.contactForces = P<float3>(c->F);
    dt.contactTorque_convToForce = P<float3>(c->TOF);
    dt.contactPointGeometryA = P<float3>(c->CPA);
    dt.contactPointGeometryB = P<float3>(c->CPB);
    for (int w = 0; w < c->nW; w++) dt.contactWildcards[w] = P<float>(c->wc[w]);
    RG_TRY(cudaMemcpyAsync(c->d_kt, &c->kt, sizeof(c->kt), cudaMemcpyHostToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->d_dt, &c->dt, sizeof(c->dt), cudaMemcpyHostToDevice, c->stream));
    return true;
}

// kT-side contact arrays for n contacts (contents not kept: they are rewritten by every CD)
bool ensure_kt_contacts(refg_ctx* c, size_t n) {
    n = n ? n : 1;
    return grow(c, c->idA, n * 4, true) && grow(c, c->idB, n * 4, true) && grow(c, c->type, n, true) &&
           grow(c, c->map, n * 4, false);
}
// dT-side arrays for n contacts; wildcards keep their contents (the history of the previous list)
bool ensure_dt_contacts(refg_ctx* c, size_t n) {
    n = n ? n : 1;
    bool ok = grow(c, c->dIdA, n * 4, false) && grow(c, c->dIdB, n * 4, false) && grow(c, c->dType, n, false) &&
              grow(c, c->dMap, n * 4, false) && grow(c, c->F, n * 12, false) && grow(c, c->TOF, n * 12, false) &&
              grow(c, c->CPA, n * 12, false) && grow(c, c->CPB, n * 12, false);
    for (int w = 0; ok && w < c->nW; w++) ok = grow(c, c->wc[w], n * 4, true);
    return ok;
}

bool load_kernels(refg_ctx* c, const char* dir) {
    std::ifstream names(std::string(dir) + "/kernels.txt");
    if (!names) {
        c->err = std::string("cannot open ") + dir + "/kernels.txt";
        return false;
    }
    // lines: <program> <name> <lowered name>
    std::vector<std::string> progs;
    std::string prog, name, lowered;
    std::vector<std::pair<std::string, std::string>> table[K_COUNT];
    struct Row {
        std::string prog, name, lowered;
    };
    std::vector<Row> rows;
    while (names >> prog >> name >> lowered) rows.push_back({prog, name, lowered});
    for (int id = 0; id < K_COUNT; id++) {
        const Row* hit = nullptr;
        for (const Row& r : rows)
            if (r.prog == kProgram[id] && r.name == kName[id]) hit = &r;
        if (!hit) {
            c->err = std::string("kernel ") + kName[id] + " missing from kernels.txt";
            return false;
        }
        size_t li = 0;
        for (; li < progs.size(); li++)
            if (progs[li] == hit->prog) break;
        if (li == progs.size()) {
            std::ifstream f(std::string(dir) + "/" + hit->prog + ".cubin", std::ios::binary);
            if (!f) {
                c->err = "cannot open cubin of " + hit->prog;
                return false;
            }
            std::stringstream ss;
            ss << f.rdbuf();
            std::string image = ss.str();
            cudaLibrary_t lib;
            RG_TRY(cudaLibraryLoadData(&lib, image.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
            c->libs.push_back(lib);
            progs.push_back(hit->prog);
        }
        RG_TRY(cudaLibraryGetKernel(&c->k[id], c->libs[li], hit->lowered.c_str()));
    }
    return true;
}

// Grid of the pair kernels as the reference sizes it (src/algorithms/DEMCubContactDetection.cu:177-180): one block
// per active bin, or one thread per active bin.
unsigned pair_grid(refg_ctx* c, size_t nActive) {
    return c->one_bin_per_thread ? blocks_for(nActive, DEME_KT_CD_NTHREADS_PER_BLOCK) : (unsigned)nActive;
}

bool do_detect(refg_ctx* c) {
    mark(c, 0);
    const size_t nS = c->nS;
    // dT -> kT hand-over of owner poses and families (dT::sendToTheirBuffer)
    const size_t nO = c->nO;
    RG_TRY(cudaMemcpyAsync(c->kVoxel, c->dt.voxelID, nO * 8, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kLocX, c->dt.locX, nO * 2, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kLocY, c->dt.locY, nO * 2, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kLocZ, c->dt.locZ, nO * 2, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kQw, c->dt.oriQw, nO * 4, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kQx, c->dt.oriQx, nO * 4, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kQy, c->dt.oriQy, nO * 4, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kQz, c->dt.oriQz, nO * 4, cudaMemcpyDeviceToDevice, c->stream));
    RG_TRY(cudaMemcpyAsync(c->kFam, c->dt.familyID, nO, cudaMemcpyDeviceToDevice, c->stream));
    if (!sync_if(c)) return false;

    // 1: bins each sphere touches, sphere--analytical counts
    if (!grow(c, c->numBins, (nS + 1) * 2, false) || !grow(c, c->numAnal, nS + 1, false) ||
        !grow(c, c->binScan, (nS + 1) * 4, false) || !grow(c, c->analScan, (nS + 1) * 4, false))
        return false;
    {
        void* numBins = c->numBins.p;
        void* numAnal = c->numAnal.p;
        void* args[] = {&c->d_sp, &c->d_kt, &numBins, &numAnal};
        if (!launch(c, K_BIN_COUNT, blocks_for(nS, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, args))
            return false;
    }
    // 2: scans and their totals
    if (!exclusive_scan(c, P<uint16_t>(c->numBins), P<uint32_t>(c->binScan), nS) ||
        !exclusive_scan(c, P<uint8_t>(c->numAnal), P<uint32_t>(c->analScan), nS))
        return false;
    uint32_t lastScan = 0, lastAnalScan = 0;
    uint16_t lastBins = 0;
    uint8_t lastAnal = 0;
    if (nS) {
        if (!read_back(c, P<uint32_t>(c->binScan) + nS - 1, lastScan) ||
            !read_back(c, P<uint16_t>(c->numBins) + nS - 1, lastBins) ||
            !read_back(c, P<uint32_t>(c->analScan) + nS - 1, lastAnalScan) ||
            !read_back(c, P<uint8_t>(c->numAnal) + nS - 1, lastAnal))
            return false;
    }
    const size_t nPairs = nS ? (size_t)lastScan + lastBins : 0;
    const size_t nGeo = nS ? (size_t)lastAnalScan + lastAnal : 0;
    if (!ensure_kt_contacts(c, nGeo) || !upload_views(c)) return false;
    // 3: bin--sphere pairs and sphere--analytical contacts
    if (!grow(c, c->binIDs, (nPairs + 1) * 4, false) || !grow(c, c->sphIDs, (nPairs + 1) * 4, false) ||
        !grow(c, c->pairBin, (nPairs + 1) * 4, false) || !grow(c, c->pairSph, (nPairs + 1) * 4, false))
        return false;
    {
        void* binScan = c->binScan.p;
        void* analScan = c->analScan.p;
        void* binIDs = c->binIDs.p;
        void* sphIDs = c->sphIDs.p;
        void* a = c->idA.p;
        void* b = c->idB.p;
        void* ty = c->type.p;
        void* args[] = {&c->d_sp, &c->d_kt, &binScan, &analScan, &binIDs, &sphIDs, &a, &b, &ty};
        if (!launch(c, K_BIN_EMIT, blocks_for(nS, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, args))
            return false;
    }
    mark(c, 1);
    // 4: sort by bin
    if (!sort_pairs(c, P<uint32_t>(c->binIDs), P<uint32_t>(c->pairBin), P<uint32_t>(c->sphIDs),
                    P<uint32_t>(c->pairSph), nPairs))
        return false;
    mark(c, 2);
    // 5: active bins, sphere counts per bin and their offsets
    if (!grow(c, c->activeBins, (nPairs + 1) * 4, false) || !grow(c, c->numSphBin, (nPairs + 1) * 2, false))
        return false;
    size_t nActive = 0;
    if (!rle(c, P<uint32_t>(c->pairBin), P<uint32_t>(c->activeBins), P<uint16_t>(c->numSphBin), nPairs, nActive))
        return false;
    if (!grow(c, c->lookUp, (nActive + 1) * 4, false)) return false;
    if (!exclusive_scan(c, P<uint16_t>(c->numSphBin), P<uint32_t>(c->lookUp), nActive)) return false;
    size_t nSS = 0;
    bool marked3 = false;
    if (nActive > 0) {
        // the reference's contact kernels trap above DEME_MAX_SPHERES_PER_BIN spheres in a bin: check first
        if (!cub_call(c, [&](void* tmp, size_t& bytes) {
                return cub::DeviceReduce::Max(tmp, bytes, P<uint16_t>(c->numSphBin), (uint16_t*)c->d_max16,
                                              (int64_t)nActive, c->stream);
            }))
            return false;
        uint16_t maxInBin = 0;
        if (!read_back(c, (const uint16_t*)c->d_max16, maxInBin)) return false;
        if (maxInBin > DEME_MAX_SPHERES_PER_BIN) {
            c->err = "a bin holds " + std::to_string(maxInBin) + " spheres, above the reference kernels' limit of " +
                     std::to_string(DEME_MAX_SPHERES_PER_BIN) + "; contact kernels not launched";
            return false;
        }
        mark(c, 3);
        marked3 = true;
        // 6: contacts per bin, offsets, then the pairs after the sphere--analytical contacts
        if (!grow(c, c->numCnt, (nActive + 1) * 2, false) || !grow(c, c->offs, (nActive + 1) * 4, false)) return false;
        {
            void* sph = c->pairSph.p;
            void* act = c->activeBins.p;
            void* nsb = c->numSphBin.p;
            void* lu = c->lookUp.p;
            void* cnt = c->numCnt.p;
            size_t na = nActive;
            void* args[] = {&c->d_sp, &c->d_kt, &sph, &act, &nsb, &lu, &cnt, &na};
            if (!launch(c, c->one_bin_per_thread ? K_CNT_EACH_BIN_T : K_CNT_EACH_BIN, pair_grid(c, nActive),
                        DEME_KT_CD_NTHREADS_PER_BLOCK, args))
                return false;
        }
        if (!exclusive_scan(c, P<uint16_t>(c->numCnt), P<uint32_t>(c->offs), nActive)) return false;
        uint16_t lastCnt = 0;
        uint32_t lastOff = 0;
        if (!read_back(c, P<uint16_t>(c->numCnt) + nActive - 1, lastCnt) ||
            !read_back(c, P<uint32_t>(c->offs) + nActive - 1, lastOff))
            return false;
        nSS = (size_t)lastCnt + lastOff;
        if (!ensure_kt_contacts(c, nGeo + nSS) || !upload_views(c)) return false;
        RG_TRY(cudaMemsetAsync(P<uint8_t>(c->type) + nGeo, deme::SPHERE_SPHERE_CONTACT, nSS, c->stream));
        if (!sync_if(c)) return false;
        {
            void* sph = c->pairSph.p;
            void* act = c->activeBins.p;
            void* nsb = c->numSphBin.p;
            void* lu = c->lookUp.p;
            void* off = c->offs.p;
            void* outA = P<uint32_t>(c->idA) + nGeo;
            void* outB = P<uint32_t>(c->idB) + nGeo;
            size_t na = nActive;
            void* args[] = {&c->d_sp, &c->d_kt, &sph, &act, &nsb, &lu, &off, &outA, &outB, &na};
            if (!launch(c, c->one_bin_per_thread ? K_POP_EACH_BIN_T : K_POP_EACH_BIN, pair_grid(c, nActive),
                        DEME_KT_CD_NTHREADS_PER_BLOCK, args))
                return false;
        }
    }
    if (!marked3) mark(c, 3);
    mark(c, 4);
    const size_t n = nGeo + nSS;
    c->nC = n;
    // 7: two stable sorts by idA (idB and the type as values), copied back
    if (n > 0) {
        if (!grow(c, c->sortTmpA, n * 4, false) || !grow(c, c->sortTmpB, n * 4, false) ||
            !grow(c, c->sortTmpT, n, false))
            return false;
        if (!sort_pairs(c, P<uint32_t>(c->idA), P<uint32_t>(c->sortTmpA), P<uint32_t>(c->idB), P<uint32_t>(c->sortTmpB),
                        n) ||
            !sort_pairs(c, P<uint32_t>(c->idA), P<uint32_t>(c->sortTmpA), P<uint8_t>(c->type), P<uint8_t>(c->sortTmpT),
                        n))
            return false;
        RG_TRY(cudaMemcpyAsync(c->idA.p, c->sortTmpA.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
        RG_TRY(cudaMemcpyAsync(c->idB.p, c->sortTmpB.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
        RG_TRY(cudaMemcpyAsync(c->type.p, c->sortTmpT.p, n, cudaMemcpyDeviceToDevice, c->stream));
        if (!sync_if(c)) return false;
        mark(c, 5);
        // 8: history map against the previous list
        if (c->nW > 0) {
            const size_t nSafe = nS;
            if (!grow(c, c->newU, (nSafe + 1) * 4, false) || !grow(c, c->oldU, (nSafe + 1) * 4, false) ||
                !grow(c, c->newRL, (nSafe + 1) * 2, false) || !grow(c, c->oldRL, (nSafe + 1) * 2, false) ||
                !grow(c, c->newFull, (nSafe + 1) * 2, false) || !grow(c, c->oldFull, (nSafe + 1) * 2, false) ||
                !grow(c, c->newScan, (nSafe + 1) * 4, false) || !grow(c, c->oldScan, (nSafe + 1) * 4, false))
                return false;
            size_t nNewU = 0, nOldU = 0;
            if (!rle(c, P<uint32_t>(c->idA), P<uint32_t>(c->newU), P<uint16_t>(c->newRL), n, nNewU) ||
                !rle(c, P<uint32_t>(c->pA), P<uint32_t>(c->oldU), P<uint16_t>(c->oldRL), c->nPrev, nOldU))
                return false;
            RG_TRY(cudaMemsetAsync(c->newFull.p, 0, nSafe * 2, c->stream));
            RG_TRY(cudaMemsetAsync(c->oldFull.p, 0, nSafe * 2, c->stream));
            if (!sync_if(c)) return false;
            {
                void* full = c->newFull.p;
                void* u = c->newU.p;
                void* rl = c->newRL.p;
                size_t m = nNewU;
                void* args[] = {&full, &u, &rl, &m};
                if (!launch(c, K_FILL_RL, blocks_for(nNewU, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK,
                            args))
                    return false;
            }
            {
                void* full = c->oldFull.p;
                void* u = c->oldU.p;
                void* rl = c->oldRL.p;
                size_t m = nOldU;
                void* args[] = {&full, &u, &rl, &m};
                if (!launch(c, K_FILL_RL, blocks_for(nOldU, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK,
                            args))
                    return false;
            }
            if (!exclusive_scan(c, P<uint16_t>(c->newFull), P<uint32_t>(c->newScan), nSafe) ||
                !exclusive_scan(c, P<uint16_t>(c->oldFull), P<uint32_t>(c->oldScan), nSafe))
                return false;
            {
                void* nf = c->newFull.p;
                void* of = c->oldFull.p;
                void* ns = c->newScan.p;
                void* os = c->oldScan.p;
                void* mp = c->map.p;
                size_t m = nSafe;
                void* args[] = {&nf, &of, &ns, &os, &mp, &c->d_kt, &m};
                if (!launch(c, K_BUILD_MAP, blocks_for(nSafe, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
                            args))
                    return false;
            }
            if (!grow(c, c->pA, n * 4, false) || !grow(c, c->pB, n * 4, false) || !grow(c, c->pT, n, false))
                return false;
            RG_TRY(cudaMemcpyAsync(c->pA.p, c->idA.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
            RG_TRY(cudaMemcpyAsync(c->pB.p, c->idB.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
            RG_TRY(cudaMemcpyAsync(c->pT.p, c->type.p, n, cudaMemcpyDeviceToDevice, c->stream));
            if (!sync_if(c)) return false;
        }
    }
    if (n == 0) mark(c, 5);
    mark(c, 6);
    const size_t nPrevForWc = c->nPrev;
    c->nPrev = n;
    // kT -> dT hand-over of the contact list (kT::sendToTheirBuffer)
    if (!ensure_dt_contacts(c, n) || !upload_views(c)) return false;
    if (n > 0) {
        RG_TRY(cudaMemcpyAsync(c->dIdA.p, c->idA.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
        RG_TRY(cudaMemcpyAsync(c->dIdB.p, c->idB.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
        RG_TRY(cudaMemcpyAsync(c->dType.p, c->type.p, n, cudaMemcpyDeviceToDevice, c->stream));
        if (c->nW > 0) RG_TRY(cudaMemcpyAsync(c->dMap.p, c->map.p, n * 4, cudaMemcpyDeviceToDevice, c->stream));
        if (!sync_if(c)) return false;
    }
    // dT: migratePersistentContacts
    if (c->nW > 0 && n > 0) {
        if (!grow(c, c->newWc, n * 4 * c->nW, false) || !grow(c, c->sentry, nPrevForWc + 1, false)) return false;
        {
            void* nw = c->newWc.p;
            void* se = c->sentry.p;
            unsigned nWc = (unsigned)c->nW;
            size_t m = n;
            void* args[] = {&c->d_dt, &nw, &se, &nWc, &m};
            if (!launch(c, K_REARRANGE_WC, blocks_for(n, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK, args))
                return false;
        }
        for (int w = 0; w < c->nW; w++)
            RG_TRY(cudaMemcpyAsync(c->wc[w].p, P<float>(c->newWc) + (size_t)w * n, n * 4, cudaMemcpyDeviceToDevice,
                                   c->stream));
        if (!sync_if(c)) return false;
    }
    mark(c, 7);
    return true;
}

bool do_forces(refg_ctx* c) {
    const size_t n = c->nC;
    {
        size_t m = n;
        void* args[] = {&c->d_sp, &c->d_dt, &m};
        size_t nPrep = n > c->nO ? n : c->nO;
        if (!launch(c, K_PREP_FORCE, blocks_for(nPrep, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK, args))
            return false;
    }
    if (n == 0) {
        mark(c, 8);
        mark(c, 9);
        return true;
    }
    {
        size_t m = n;
        void* args[] = {&c->d_sp, &c->d_dt, &m};
        if (!launch(c, K_CALC_FORCE, blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, args))
            return false;
    }
    mark(c, 8);
    // collectContactForces
    if (!grow(c, c->owners, 2 * n * 4, false) || !grow(c, c->ownersSorted, 2 * n * 4, false) ||
        !grow(c, c->acc, 2 * n * 12, false) || !grow(c, c->accSorted, 2 * n * 12, false) ||
        !grow(c, c->uniq, ((size_t)c->nO + 1) * 4, false) || !grow(c, c->accOwner, ((size_t)c->nO + 1) * 12, false))
        return false;
    const unsigned gb = blocks_for(n, DEME_NUM_BODIES_PER_BLOCK);
    uint32_t* idAOwner = P<uint32_t>(c->owners);
    uint32_t* idBOwner = idAOwner + n;
    {
        void* o = idAOwner;
        void* a = c->dIdA.p;
        void* so = (void*)c->dt.ownerClumpBody;
        void* ty = c->dType.p;
        size_t m = n;
        void* args[] = {&o, &a, &so, &ty, &m};
        if (!launch(c, K_CASH_A, gb, DEME_NUM_BODIES_PER_BLOCK, args)) return false;
    }
    {
        void* o = idBOwner;
        void* b = c->dIdB.p;
        void* so = (void*)c->dt.ownerClumpBody;
        void* ty = c->dType.p;
        size_t m = n;
        void* args[] = {&o, &b, &so, &ty, &m};
        if (!launch(c, K_CASH_B, gb, DEME_NUM_BODIES_PER_BLOCK, args)) return false;
    }
    auto reduce_stash = [&](float* o1, float* o2, float* o3) -> bool {
        if (!sort_pairs(c, P<uint32_t>(c->owners), P<uint32_t>(c->ownersSorted), P<float3>(c->acc),
                        P<float3>(c->accSorted), 2 * n))
            return false;
        if (!cub_call(c, [&](void* tmp, size_t& bytes) {
                return cub::DeviceReduce::ReduceByKey(tmp, bytes, P<uint32_t>(c->ownersSorted), P<uint32_t>(c->uniq),
                                                      P<float3>(c->accSorted), P<float3>(c->accOwner), c->d_count,
                                                      Float3Sum{}, (int64_t)(2 * n), c->stream);
            }))
            return false;
        size_t runs = 0;
        if (!read_back(c, c->d_count, runs)) return false;
        void* u = c->uniq.p;
        void* v = c->accOwner.p;
        size_t m = runs;
        void* args[] = {&o1, &o2, &o3, &u, &v, &m};
        return launch(c, K_STASH, blocks_for(runs, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, args);
    };
    for (int side = 0; side < 2; side++) {
        void* acc = P<float3>(c->acc) + side * n;
        void* f = c->F.p;
        void* o = side ? (void*)idBOwner : (void*)idAOwner;
        float sign = side ? -1.f : 1.f;
        size_t m = n;
        void* args[] = {&acc, &f, &o, &sign, &m, &c->d_dt};
        if (!launch(c, K_FORCE_TO_ACC, gb, DEME_NUM_BODIES_PER_BLOCK, args)) return false;
    }
    if (!reduce_stash(c->dt.aX, c->dt.aY, c->dt.aZ)) return false;
    for (int side = 0; side < 2; side++) {
        void* acc = P<float3>(c->acc) + side * n;
        void* cp = side ? c->CPB.p : c->CPA.p;
        void* qw = c->dt.oriQw;
        void* qx = c->dt.oriQx;
        void* qy = c->dt.oriQy;
        void* qz = c->dt.oriQz;
        void* f = c->F.p;
        void* tof = c->TOF.p;
        void* o = side ? (void*)idBOwner : (void*)idAOwner;
        float sign = side ? -1.f : 1.f;
        size_t m = n;
        void* args[] = {&acc, &cp, &qw, &qx, &qy, &qz, &f, &tof, &o, &sign, &m, &c->d_dt};
        if (!launch(c, K_FORCE_TO_ANG_ACC, gb, DEME_NUM_BODIES_PER_BLOCK, args)) return false;
    }
    if (!reduce_stash(c->dt.alphaX, c->dt.alphaY, c->dt.alphaZ)) return false;
    mark(c, 9);
    return true;
}

bool do_integrate(refg_ctx* c) {
    float t = c->tf;
    void* args[] = {&c->d_sp, &c->d_dt, &t};
    if (!launch(c, K_INTEGRATE, blocks_for(c->nO, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, args))
        return false;
    c->t += (double)c->sp.h;
    c->tf += c->sp.h;  // timeElapsed += simParams->h (src/DEM/dT.cpp:1585)
    c->steps++;
    return true;
}

bool do_create(refg_ctx* c, const char* dir, const deme_sim_params* p, const deme_scene* s) {
    RG_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    if (!load_kernels(c, dir)) return false;
    deme::DEMSimParams& sp = c->sp;
    std::memset(&sp, 0, sizeof(sp));
    sp.nvXp2 = p->nvXp2;
    sp.nvYp2 = p->nvYp2;
    sp.nvZp2 = p->nvZp2;
    sp.nbX = p->nbX;
    sp.nbY = p->nbY;
    sp.nbZ = p->nbZ;
    sp.l = p->l;
    sp.voxelSize = p->voxel_size;
    sp.binSize = p->bin_size;
    sp.nSpheresGM = s->n_spheres;
    sp.nAnalGM = (deme::objID_t)s->n_anal;
    sp.nOwnerBodies = s->n_owners;
    sp.LBFX = p->lbf[0];
    sp.LBFY = p->lbf[1];
    sp.LBFZ = p->lbf[2];
    sp.Gx = p->G[0];
    sp.Gy = p->G[1];
    sp.Gz = p->G[2];
    sp.h = p->h;
    sp.beta = p->beta;
    sp.nContactWildcards = p->n_contact_wildcards;
    c->nO = s->n_owners;
    c->nS = s->n_spheres;
    c->nW = p->n_contact_wildcards;
    c->cd_freq = p->cd_update_freq;
    const size_t nO = c->nO, nS = c->nS;
    std::memset(&c->kt, 0, sizeof(c->kt));
    std::memset(&c->dt, 0, sizeof(c->dt));
    deme::DEMDataDT& dt = c->dt;
    deme::DEMDataKT& kt = c->kt;
    bool ok = dev_copy(c, dt.voxelID, s->voxel, nO) && dev_copy(c, dt.locX, s->locX, nO) &&
              dev_copy(c, dt.locY, s->locY, nO) && dev_copy(c, dt.locZ, s->locZ, nO) &&
              dev_copy(c, dt.oriQw, s->oriQw, nO) && dev_copy(c, dt.oriQx, s->oriQx, nO) &&
              dev_copy(c, dt.oriQy, s->oriQy, nO) && dev_copy(c, dt.oriQz, s->oriQz, nO) &&
              dev_copy(c, dt.vX, s->vX, nO) && dev_copy(c, dt.vY, s->vY, nO) && dev_copy(c, dt.vZ, s->vZ, nO) &&
              dev_copy(c, dt.omgBarX, s->omgX, nO) && dev_copy(c, dt.omgBarY, s->omgY, nO) &&
              dev_copy(c, dt.omgBarZ, s->omgZ, nO) && dev_copy(c, dt.aX, (const float*)nullptr, nO, 1) &&
              dev_copy(c, dt.aY, (const float*)nullptr, nO, 1) && dev_copy(c, dt.aZ, (const float*)nullptr, nO, 1) &&
              dev_copy(c, dt.alphaX, (const float*)nullptr, nO, 1) &&
              dev_copy(c, dt.alphaY, (const float*)nullptr, nO, 1) &&
              dev_copy(c, dt.alphaZ, (const float*)nullptr, nO, 1) && dev_copy(c, dt.familyID, s->family, nO) &&
              dev_copy(c, dt.massOwnerBody, s->mass, nO) && dev_copy(c, dt.mmiXX, s->mmiXX, nO) &&
              dev_copy(c, dt.mmiYY, s->mmiYY, nO) && dev_copy(c, dt.mmiZZ, s->mmiZZ, nO) &&
              dev_copy(c, dt.ownerClumpBody, s->sphere_owner, nS) && dev_copy(c, dt.relPosSphereX, s->relX, nS) &&
              dev_copy(c, dt.relPosSphereY, s->relY, nS) && dev_copy(c, dt.relPosSphereZ, s->relZ, nS) &&
              dev_copy(c, dt.radiiSphere, s->radius, nS) && dev_copy(c, dt.sphereMaterialOffset, s->sphere_material, nS);
    if (!ok) return false;
    std::vector<uint8_t> masks(DEME_NUM_FAMILY_MASK, 0);
    if (s->family_masks) std::memcpy(masks.data(), s->family_masks, DEME_NUM_FAMILY_MASK);
    if (!dev_copy(c, dt.familyMasks, masks.data(), masks.size())) return false;
    // kT's own copies of the owner poses and families
    if (!dev_copy(c, c->kVoxel, s->voxel, nO) || !dev_copy(c, c->kLocX, s->locX, nO) ||
        !dev_copy(c, c->kLocY, s->locY, nO) || !dev_copy(c, c->kLocZ, s->locZ, nO) ||
        !dev_copy(c, c->kQw, s->oriQw, nO) || !dev_copy(c, c->kQx, s->oriQx, nO) ||
        !dev_copy(c, c->kQy, s->oriQy, nO) || !dev_copy(c, c->kQz, s->oriQz, nO) ||
        !dev_copy(c, c->kFam, s->family, nO))
        return false;
    kt.familyID = c->kFam;
    kt.voxelID = c->kVoxel;
    kt.locX = c->kLocX;
    kt.locY = c->kLocY;
    kt.locZ = c->kLocZ;
    kt.oriQw = c->kQw;
    kt.oriQx = c->kQx;
    kt.oriQy = c->kQy;
    kt.oriQz = c->kQz;
    kt.familyMasks = dt.familyMasks;
    kt.ownerClumpBody = dt.ownerClumpBody;
    kt.radiiSphere = dt.radiiSphere;
    kt.relPosSphereX = dt.relPosSphereX;
    kt.relPosSphereY = dt.relPosSphereY;
    kt.relPosSphereZ = dt.relPosSphereZ;
    void* p0 = nullptr;
    RG_TRY(cudaMalloc(&p0, sizeof(deme::DEMSimParams)));
    c->owned.push_back(p0);
    c->d_sp = (deme::DEMSimParams*)p0;
    RG_TRY(cudaMalloc(&p0, sizeof(deme::DEMDataKT)));
    c->owned.push_back(p0);
    c->d_kt = (deme::DEMDataKT*)p0;
    RG_TRY(cudaMalloc(&p0, sizeof(deme::DEMDataDT)));
    c->owned.push_back(p0);
    c->d_dt = (deme::DEMDataDT*)p0;
    RG_TRY(cudaMalloc(&p0, 64));
    c->owned.push_back(p0);
    c->d_count = (size_t*)p0;
    c->d_max16 = (uint32_t*)((char*)p0 + 32);
    RG_TRY(cudaMemcpy(c->d_sp, &sp, sizeof(sp), cudaMemcpyHostToDevice));
    if (!ensure_kt_contacts(c, 1) || !ensure_dt_contacts(c, 1) || !grow(c, c->pA, 4, false) ||
        !grow(c, c->pB, 4, false) || !grow(c, c->pT, 1, false))
        return false;
    if (!upload_views(c)) return false;
    RG_TRY(cudaStreamSynchronize(c->stream));
    return true;
}

int32_t status(refg_ctx* c, bool ok) {
    if (ok) return DEME_OK;
    return c->err.find("above the reference kernels' limit") != std::string::npos ? DEME_ERR_OVERFLOW : DEME_ERR_CUDA;
}

template <typename T>
bool copy_out(refg_ctx* c, T* dst, const T* src, size_t n) {
    if (dst && n) RG_TRY(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost));
    return true;
}
template <typename T>
bool copy_in(refg_ctx* c, T* dst, const T* src, size_t n) {
    if (src && n) RG_TRY(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return true;
}

}  // namespace

extern "C" {

/* Loads the cubins of `cubin_dir` and uploads the scene.  Returns the context even on failure (read
 * refg_get_error, then refg_destroy). */
int32_t refg_create(const char* cubin_dir, const deme_sim_params* p, const deme_scene* s, int32_t sync_each,
                    refg_ctx** out) {
    refg_ctx* c = new refg_ctx();
    c->sync_each = sync_each != 0;
    *out = c;
    return status(c, do_create(c, cubin_dir, p, s));
}

const char* refg_get_error(refg_ctx* c) { return c ? c->err.c_str() : "null context"; }

void refg_destroy(refg_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    DBuf* bufs[] = {&c->idA,     &c->idB,      &c->type,     &c->map,        &c->pA,         &c->pB,
                    &c->pT,      &c->dIdA,     &c->dIdB,     &c->dType,      &c->dMap,       &c->F,
                    &c->TOF,     &c->CPA,      &c->CPB,      &c->newWc,      &c->sentry,     &c->numBins,
                    &c->numAnal, &c->binScan,  &c->analScan, &c->binIDs,     &c->sphIDs,     &c->pairBin,
                    &c->pairSph, &c->activeBins, &c->numSphBin, &c->lookUp,  &c->numCnt,     &c->offs,
                    &c->newU,    &c->oldU,     &c->newRL,    &c->oldRL,      &c->newFull,    &c->oldFull,
                    &c->newScan, &c->oldScan,  &c->sortTmpA, &c->sortTmpB,   &c->sortTmpT,   &c->owners,
                    &c->ownersSorted, &c->acc, &c->accSorted, &c->uniq,      &c->accOwner,   &c->cubTmp};
    for (DBuf* b : bufs)
        if (b->p) cudaFree(b->p);
    for (int w = 0; w < DEME_MAX_WILDCARDS; w++)
        if (c->wc[w].p) cudaFree(c->wc[w].p);
    for (void* p : c->owned) cudaFree(p);
    for (cudaLibrary_t l : c->libs) cudaLibraryUnload(l);
    for (cudaEvent_t e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int32_t refg_detect_contacts(refg_ctx* c) { return status(c, do_detect(c)); }
int32_t refg_compute_forces(refg_ctx* c) { return status(c, do_forces(c)); }
int32_t refg_integrate(refg_ctx* c) { return status(c, do_integrate(c)); }

/* n steps: contact detection every cd_update_freq steps (every step when 0), forces, integration. */
int32_t refg_step(refg_ctx* c, int32_t n) {
    for (int32_t i = 0; i < n; i++) {
        if (c->cd_freq <= 0 || (c->steps % c->cd_freq) == 0)
            if (!do_detect(c)) return status(c, false);
        if (!do_forces(c) || !do_integrate(c)) return status(c, false);
    }
    return DEME_OK;
}

/* n steps with events at the phase boundaries; adds each phase's milliseconds to out[0..9]: bins per sphere and
 * bin--sphere pairs, sort by bin, active bins, pair kernels, sort by idA, history map, hand-over and history remap,
 * force kernel, force collection, integration. */
int32_t refg_profile_steps(refg_ctx* c, int32_t n, float* out) {
    for (int k = 0; k <= kPhases; k++)
        if (!c->ev[k] && cudaEventCreate(&c->ev[k]) != cudaSuccess) {
            c->err = "cudaEventCreate failed";
            return DEME_ERR_CUDA;
        }
    c->profiling = true;
    int32_t st = DEME_OK;
    for (int32_t i = 0; i < n && st == DEME_OK; i++) {
        if (c->cd_freq <= 0 || (c->steps % c->cd_freq) == 0) {
            if (!do_detect(c)) st = status(c, false);
        } else {
            for (int k = 0; k <= 7; k++) mark(c, k);
        }
        if (st == DEME_OK && (!do_forces(c) || !do_integrate(c))) st = status(c, false);
        mark(c, 10);
        if (cudaEventSynchronize(c->ev[10]) != cudaSuccess) {
            c->err = "cudaEventSynchronize failed";
            st = DEME_ERR_CUDA;
        }
        for (int k = 0; st == DEME_OK && k < kPhases; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]);
            out[k] += ms;
        }
    }
    c->profiling = false;
    return st;
}

/* Device time of n steps, measured with CUDA events on the driver's stream. */
int32_t refg_time_steps(refg_ctx* c, int32_t n, float* ms) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        c->err = "cudaEventCreate failed";
        return DEME_ERR_CUDA;
    }
    cudaStreamSynchronize(c->stream);
    cudaEventRecord(e0, c->stream);
    int32_t st = refg_step(c, n);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

int32_t refg_sync(refg_ctx* c) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        c->err = cudaGetErrorString(e);
        return DEME_ERR_CUDA;
    }
    return DEME_OK;
}

uint32_t refg_num_contacts(refg_ctx* c) { return (uint32_t)c->nC; }

int32_t refg_download_contacts(refg_ctx* c, deme_contacts* o) {
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DEME_ERR_CUDA;
    o->n_contacts = (uint32_t)c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    const size_t n = c->nC;
    bool ok = copy_out(c, o->idA, P<uint32_t>(c->dIdA), n) && copy_out(c, o->idB, P<uint32_t>(c->dIdB), n) &&
              copy_out(c, o->type, P<uint8_t>(c->dType), n);
    if (ok && o->mapping) {
        if (c->nW > 0)
            ok = copy_out(c, o->mapping, P<uint32_t>(c->dMap), n);
        else
            for (size_t i = 0; i < n; i++) o->mapping[i] = DEME_NULL_MAPPING_PARTNER;
    }
    for (int w = 0; ok && o->wildcards && w < c->nW; w++)
        ok = copy_out(c, o->wildcards + (size_t)w * o->capacity, P<float>(c->wc[w]), n);
    return status(c, ok);
}

int32_t refg_download_contact_forces(refg_ctx* c, deme_contact_forces* o) {
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DEME_ERR_CUDA;
    o->n_contacts = (uint32_t)c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    const size_t n3 = c->nC * 3;
    bool ok = copy_out(c, o->force, P<float>(c->F), n3) && copy_out(c, o->torque_only_force, P<float>(c->TOF), n3) &&
              copy_out(c, o->cpA, P<float>(c->CPA), n3) && copy_out(c, o->cpB, P<float>(c->CPB), n3);
    return status(c, ok);
}

int32_t refg_download_state(refg_ctx* c, deme_state* o) {
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DEME_ERR_CUDA;
    const size_t n = c->nO;
    const deme::DEMDataDT& d = c->dt;
    bool ok = copy_out(c, o->voxel, (const uint64_t*)d.voxelID, n) && copy_out(c, o->locX, d.locX, n) &&
              copy_out(c, o->locY, d.locY, n) && copy_out(c, o->locZ, d.locZ, n) &&
              copy_out(c, o->oriQw, d.oriQw, n) && copy_out(c, o->oriQx, d.oriQx, n) &&
              copy_out(c, o->oriQy, d.oriQy, n) && copy_out(c, o->oriQz, d.oriQz, n) &&
              copy_out(c, o->vX, d.vX, n) && copy_out(c, o->vY, d.vY, n) && copy_out(c, o->vZ, d.vZ, n) &&
              copy_out(c, o->omgX, d.omgBarX, n) && copy_out(c, o->omgY, d.omgBarY, n) &&
              copy_out(c, o->omgZ, d.omgBarZ, n) && copy_out(c, o->aX, d.aX, n) && copy_out(c, o->aY, d.aY, n) &&
              copy_out(c, o->aZ, d.aZ, n) && copy_out(c, o->alphaX, d.alphaX, n) &&
              copy_out(c, o->alphaY, d.alphaY, n) && copy_out(c, o->alphaZ, d.alphaZ, n) &&
              copy_out(c, o->family, d.familyID, n);
    return status(c, ok);
}

int32_t refg_upload_state(refg_ctx* c, const deme_state* s) {
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DEME_ERR_CUDA;
    const size_t n = c->nO;
    deme::DEMDataDT& d = c->dt;
    bool ok = copy_in(c, (uint64_t*)d.voxelID, s->voxel, n) && copy_in(c, d.locX, s->locX, n) &&
              copy_in(c, d.locY, s->locY, n) && copy_in(c, d.locZ, s->locZ, n) &&
              copy_in(c, d.oriQw, s->oriQw, n) && copy_in(c, d.oriQx, s->oriQx, n) &&
              copy_in(c, d.oriQy, s->oriQy, n) && copy_in(c, d.oriQz, s->oriQz, n) && copy_in(c, d.vX, s->vX, n) &&
              copy_in(c, d.vY, s->vY, n) && copy_in(c, d.vZ, s->vZ, n) && copy_in(c, d.omgBarX, s->omgX, n) &&
              copy_in(c, d.omgBarY, s->omgY, n) && copy_in(c, d.omgBarZ, s->omgZ, n) &&
              copy_in(c, d.aX, s->aX, n) && copy_in(c, d.aY, s->aY, n) && copy_in(c, d.aZ, s->aZ, n) &&
              copy_in(c, d.alphaX, s->alphaX, n) && copy_in(c, d.alphaY, s->alphaY, n) &&
              copy_in(c, d.alphaZ, s->alphaZ, n) && copy_in(c, d.familyID, s->family, n);
    return status(c, ok);
}

double refg_time(refg_ctx* c) { return c->t; }

/* Synchronise after every launch and primitive (as the reference's host code does) or only where a count is read. */
void refg_set_sync_each(refg_ctx* c, int32_t on) { c->sync_each = on != 0; }

/* The reference's two contact-kernel variants: block per active bin (default) or thread per active bin. */
void refg_set_one_bin_per_thread(refg_ctx* c, int32_t on) { c->one_bin_per_thread = on != 0; }

}  // extern "C"
