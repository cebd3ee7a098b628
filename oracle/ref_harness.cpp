// ref_harness.cpp -- host driver that runs the reference's own kernel code on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  oracle/ref_build.py substitutes the reference's kernel templates
// (src/kernel/*.cu) the way its JitHelper does and compiles them, together with this driver, into
// oracle/_ref/<hash>/libdeme_ref.so.  Kernels are launched by looping over (blockIdx, threadIdx) on host threads;
// the CUB device primitives of the reference (src/algorithms/DEMCubWrappers.cu) are replaced by their specified
// sequential behaviour: exclusive scans, stable radix sorts, unique/run-length encode and a left-to-right
// reduce-by-key.  The driver follows contactDetection (src/algorithms/DEMCubContactDetection.cu:39-397),
// migratePersistentContacts / calculateForces / integrateOwnerMotions (src/DEM/dT.cpp:1258-1432) and
// collectContactForces (src/algorithms/DEMCubForceCollection.cu:20-158).  The thread-per-bin contact kernels
// (src/kernel/DEMContactKernels.cu) are used: they implement the same test as the default block-per-bin kernels
// with a deterministic in-bin order.
#include <DEM/Defines.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/deme_b200.h"

thread_local dim3 blockIdx;
thread_local dim3 threadIdx;
thread_local dim3 blockDim;

// Kernels from the generated translation units.
void getNumberOfBinsEachSphereTouches(deme::DEMSimParams*, deme::DEMDataKT*, deme::binsSphereTouches_t*,
                                      deme::objID_t*);
void populateBinSphereTouchingPairs(deme::DEMSimParams*, deme::DEMDataKT*, deme::binSphereTouchPairs_t*,
                                    deme::binSphereTouchPairs_t*, deme::binID_t*, deme::bodyID_t*, deme::bodyID_t*,
                                    deme::bodyID_t*, deme::contact_t*);
void getNumberOfContactsEachBin(deme::DEMSimParams*, deme::DEMDataKT*, deme::bodyID_t*, deme::binID_t*,
                                deme::spheresBinTouches_t*, deme::binSphereTouchPairs_t*, deme::spheresBinTouches_t*,
                                size_t);
void populateContactPairsEachBin(deme::DEMSimParams*, deme::DEMDataKT*, deme::bodyID_t*, deme::binID_t*,
                                 deme::spheresBinTouches_t*, deme::binSphereTouchPairs_t*, deme::contactPairs_t*,
                                 deme::bodyID_t*, deme::bodyID_t*, size_t);
void fillRunLengthArray(deme::geoSphereTouches_t*, deme::bodyID_t*, deme::geoSphereTouches_t*, size_t);
void buildPersistentMap(deme::geoSphereTouches_t*, deme::geoSphereTouches_t*, deme::contactPairs_t*,
                        deme::contactPairs_t*, deme::contactPairs_t*, deme::DEMDataKT*, size_t);
void prepareForceArrays(deme::DEMSimParams*, deme::DEMDataDT*, size_t);
void rearrangeContactWildcards(deme::DEMDataDT*, float*, deme::notStupidBool_t*, unsigned int, size_t);
void calculateContactForces(deme::DEMSimParams*, deme::DEMDataDT*, size_t);
void cashInOwnerIndexA(deme::bodyID_t*, deme::bodyID_t*, deme::bodyID_t*, deme::contact_t*, size_t);
void cashInOwnerIndexB(deme::bodyID_t*, deme::bodyID_t*, deme::bodyID_t*, deme::contact_t*, size_t);
void forceToAcc(float3*, float3*, deme::bodyID_t*, float, size_t, deme::DEMDataDT*);
void forceToAngAcc(float3*, float3*, deme::oriQ_t*, deme::oriQ_t*, deme::oriQ_t*, deme::oriQ_t*, float3*, float3*,
                   deme::bodyID_t*, float, size_t, deme::DEMDataDT*);
void stashElem(float*, float*, float*, deme::bodyID_t*, float3*, size_t);
void integrateOwners(deme::DEMSimParams*, deme::DEMDataDT*, float);

namespace {
int g_threads = 1;

template <typename F>
void launch(size_t nBlocks, unsigned int nThreads, F&& body) {
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
    for (long long b = 0; b < (long long)nBlocks; b++) {
        blockDim = dim3(nThreads, 1, 1);
        blockIdx = dim3((unsigned int)b, 0, 0);
        for (unsigned int t = 0; t < nThreads; t++) {
            threadIdx = dim3(t, 0, 0);
            body();
        }
    }
}
inline size_t blocks_for(size_t n, size_t per) { return (n + per - 1) / per; }

// stable sort of (key, value) pairs, as cub::DeviceRadixSort::SortPairs over all key bits
template <typename K, typename V>
void stable_sort_pairs(const K* kin, K* kout, const V* vin, V* vout, size_t n) {
    std::vector<size_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return kin[a] < kin[b]; });
    for (size_t i = 0; i < n; i++) {
        kout[i] = kin[idx[i]];
        vout[i] = vin[idx[i]];
    }
}
template <typename T1, typename T2>
void exclusive_scan(const T1* in, T2* out, size_t n) {
    T2 acc = 0;
    for (size_t i = 0; i < n; i++) {
        out[i] = acc;
        acc = (T2)(acc + (T2)in[i]);
    }
}
// cub::DeviceRunLengthEncode::Encode
template <typename K, typename C>
size_t rle(const K* in, K* uniq, C* counts, size_t n) {
    size_t m = 0;
    for (size_t i = 0; i < n; i++) {
        if (i == 0 || in[i] != in[i - 1]) {
            uniq[m] = in[i];
            counts[m] = 0;
            m++;
        }
        counts[m - 1] = (C)(counts[m - 1] + 1);
    }
    return m;
}
}  // namespace

struct ref_ctx {
    deme::DEMSimParams sp;
    deme::DEMDataKT kt;
    deme::DEMDataDT dt;
    uint32_t nO, nS, nA;
    int nW;
    double t;
    float tf;  // the time as the reference's dT keeps it (float timeElapsed, src/DEM/dT.h:216)
    int64_t steps;
    int cd_freq;
    std::vector<uint64_t> voxel;
    std::vector<uint16_t> locX, locY, locZ;
    std::vector<float> qw, qx, qy, qz, vX, vY, vZ, wX, wY, wZ, aX, aY, aZ, alX, alY, alZ;
    std::vector<uint8_t> fam, masks;
    std::vector<float> mass, mXX, mYY, mZZ;
    std::vector<uint32_t> sOwner;
    std::vector<float> rX, rY, rZ, rad;
    std::vector<uint8_t> sMat;
    std::vector<uint32_t> idA, idB, map, pA, pB;
    std::vector<uint8_t> type, pT;
    std::vector<float> wc[DEME_MAX_WILDCARDS];
    std::vector<float3> F, TOF, CPA, CPB;
    std::vector<uint16_t> nBins;
    std::vector<uint8_t> nAnal;
    std::vector<uint32_t> pairBin, pairSph;
    void pack() {
        kt.familyID = fam.data();
        kt.voxelID = voxel.data();
        kt.locX = locX.data();
        kt.locY = locY.data();
        kt.locZ = locZ.data();
        kt.oriQw = qw.data();
        kt.oriQx = qx.data();
        kt.oriQy = qy.data();
        kt.oriQz = qz.data();
        kt.familyMasks = masks.data();
        kt.ownerClumpBody = sOwner.data();
        kt.radiiSphere = rad.data();
        kt.relPosSphereX = rX.data();
        kt.relPosSphereY = rY.data();
        kt.relPosSphereZ = rZ.data();
        kt.idGeometryA = idA.data();
        kt.idGeometryB = idB.data();
        kt.contactType = type.data();
        kt.previous_idGeometryA = pA.data();
        kt.previous_idGeometryB = pB.data();
        kt.previous_contactType = pT.data();
        kt.contactMapping = map.data();
        dt.familyID = fam.data();
        dt.voxelID = voxel.data();
        dt.locX = locX.data();
        dt.locY = locY.data();
        dt.locZ = locZ.data();
        dt.oriQw = qw.data();
        dt.oriQx = qx.data();
        dt.oriQy = qy.data();
        dt.oriQz = qz.data();
        dt.vX = vX.data();
        dt.vY = vY.data();
        dt.vZ = vZ.data();
        dt.omgBarX = wX.data();
        dt.omgBarY = wY.data();
        dt.omgBarZ = wZ.data();
        dt.aX = aX.data();
        dt.aY = aY.data();
        dt.aZ = aZ.data();
        dt.alphaX = alX.data();
        dt.alphaY = alY.data();
        dt.alphaZ = alZ.data();
        dt.idGeometryA = idA.data();
        dt.idGeometryB = idB.data();
        dt.contactType = type.data();
        dt.contactMapping = map.data();
        dt.familyMasks = masks.data();
        dt.contactForces = F.data();
        dt.contactTorque_convToForce = TOF.data();
        dt.contactPointGeometryA = CPA.data();
        dt.contactPointGeometryB = CPB.data();
        dt.ownerClumpBody = sOwner.data();
        dt.sphereMaterialOffset = sMat.data();
        dt.radiiSphere = rad.data();
        dt.relPosSphereX = rX.data();
        dt.relPosSphereY = rY.data();
        dt.relPosSphereZ = rZ.data();
        dt.massOwnerBody = mass.data();
        dt.mmiXX = mXX.data();
        dt.mmiYY = mYY.data();
        dt.mmiZZ = mZZ.data();
        for (int k = 0; k < nW; k++) dt.contactWildcards[k] = wc[k].data();
    }
    void resize_contacts(size_t n) {
        idA.resize(std::max<size_t>(n, 1));
        idB.resize(std::max<size_t>(n, 1));
        type.resize(std::max<size_t>(n, 1));
        map.resize(std::max<size_t>(n, 1));
        F.resize(std::max<size_t>(n, 1));
        TOF.resize(std::max<size_t>(n, 1));
        CPA.resize(std::max<size_t>(n, 1), make_float3(0, 0, 0));
        CPB.resize(std::max<size_t>(n, 1), make_float3(0, 0, 0));
        for (int k = 0; k < nW; k++) wc[k].resize(std::max<size_t>(n, 1), 0.f);
        pack();
    }
    size_t nC = 0, nPrev = 0;
};

extern "C" {

int32_t ref_set_threads(int32_t n) {
    g_threads = n > 0 ? n : 1;
    return g_threads;
}

ref_ctx* ref_create(const deme_sim_params* p, const deme_scene* s) {
    ref_ctx* c = new ref_ctx();
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
    c->nA = s->n_anal;
    c->nW = p->n_contact_wildcards;
    c->cd_freq = p->cd_update_freq;
    c->t = 0;
    c->tf = 0.f;
    c->steps = 0;
    uint32_t nO = c->nO, nS = c->nS;
    auto cp = [](auto& v, const auto* src, size_t n) {
        v.assign(std::max<size_t>(n, 1), 0);
        if (src && n) std::memcpy(v.data(), src, n * sizeof(*src));
    };
    cp(c->voxel, s->voxel, nO);
    cp(c->locX, s->locX, nO);
    cp(c->locY, s->locY, nO);
    cp(c->locZ, s->locZ, nO);
    cp(c->qw, s->oriQw, nO);
    cp(c->qx, s->oriQx, nO);
    cp(c->qy, s->oriQy, nO);
    cp(c->qz, s->oriQz, nO);
    cp(c->vX, s->vX, nO);
    cp(c->vY, s->vY, nO);
    cp(c->vZ, s->vZ, nO);
    cp(c->wX, s->omgX, nO);
    cp(c->wY, s->omgY, nO);
    cp(c->wZ, s->omgZ, nO);
    c->aX.assign(nO + 1, 0.f);
    c->aY.assign(nO + 1, 0.f);
    c->aZ.assign(nO + 1, 0.f);
    c->alX.assign(nO + 1, 0.f);
    c->alY.assign(nO + 1, 0.f);
    c->alZ.assign(nO + 1, 0.f);
    cp(c->fam, s->family, nO);
    cp(c->mass, s->mass, nO);
    cp(c->mXX, s->mmiXX, nO);
    cp(c->mYY, s->mmiYY, nO);
    cp(c->mZZ, s->mmiZZ, nO);
    cp(c->sOwner, s->sphere_owner, nS);
    cp(c->rX, s->relX, nS);
    cp(c->rY, s->relY, nS);
    cp(c->rZ, s->relZ, nS);
    cp(c->rad, s->radius, nS);
    cp(c->sMat, s->sphere_material, nS);
    c->masks.assign(DEME_NUM_FAMILY_MASK, 0);
    if (s->family_masks) std::memcpy(c->masks.data(), s->family_masks, DEME_NUM_FAMILY_MASK);
    c->nBins.assign(nS + 1, 0);
    c->nAnal.assign(nS + 1, 0);
    c->pA.assign(1, 0);
    c->pB.assign(1, 0);
    c->pT.assign(1, 0);
    c->resize_contacts(1);
    return c;
}

void ref_destroy(ref_ctx* c) { delete c; }

int32_t ref_detect_contacts(ref_ctx* c) {
    deme::DEMSimParams* sp = &c->sp;
    deme::DEMDataKT* kt = &c->kt;
    const size_t nS = c->nS;
    c->pack();
    // 1st step: bins each sphere touches, sphere--analytical counts
    std::vector<deme::binsSphereTouches_t>& numBins = c->nBins;
    std::vector<deme::objID_t>& numAnal = c->nAnal;
    launch(blocks_for(nS, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { getNumberOfBinsEachSphereTouches(sp, kt, numBins.data(), numAnal.data()); });
    // 2nd step: scans
    std::vector<deme::binSphereTouchPairs_t> binScan(nS + 1), analScan(nS + 1);
    exclusive_scan(numBins.data(), binScan.data(), nS);
    exclusive_scan(numAnal.data(), analScan.data(), nS);
    size_t P = nS ? (size_t)binScan[nS - 1] + numBins[nS - 1] : 0;
    size_t nGeo = nS ? (size_t)analScan[nS - 1] + numAnal[nS - 1] : 0;
    if (nGeo > c->idA.size()) c->resize_contacts(nGeo);
    // 3rd step: populate pairs
    std::vector<deme::binID_t> binIDs(P + 1);
    std::vector<deme::bodyID_t> sphIDs(P + 1);
    launch(blocks_for(nS, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, [&] {
        populateBinSphereTouchingPairs(sp, kt, binScan.data(), analScan.data(), binIDs.data(), sphIDs.data(),
                                       c->idA.data(), c->idB.data(), c->type.data());
    });
    // 4th step: sort by bin
    c->pairBin.assign(P + 1, 0);
    c->pairSph.assign(P + 1, 0);
    stable_sort_pairs(binIDs.data(), c->pairBin.data(), sphIDs.data(), c->pairSph.data(), P);
    // 5th step: active bins
    std::vector<deme::binID_t> activeBins(P + 1);
    std::vector<deme::spheresBinTouches_t> numSphBin(P + 1);
    size_t nActive = rle(c->pairBin.data(), activeBins.data(), numSphBin.data(), P);
    std::vector<deme::binSphereTouchPairs_t> lookUp(nActive + 1);
    exclusive_scan(numSphBin.data(), lookUp.data(), nActive);
    // 6th step: contact pairs
    size_t nSS = 0;
    if (nActive > 0) {
        std::vector<deme::spheresBinTouches_t> numCnt(nActive + 1);
        launch(blocks_for(nActive, DEME_KT_CD_NTHREADS_PER_BLOCK), DEME_KT_CD_NTHREADS_PER_BLOCK, [&] {
            getNumberOfContactsEachBin(sp, kt, c->pairSph.data(), activeBins.data(), numSphBin.data(), lookUp.data(),
                                       numCnt.data(), nActive);
        });
        std::vector<deme::contactPairs_t> offs(nActive + 1);
        exclusive_scan(numCnt.data(), offs.data(), nActive);
        nSS = (size_t)numCnt[nActive - 1] + offs[nActive - 1];
        if (nSS + nGeo > c->idA.size()) {
            c->resize_contacts(nSS + nGeo);
            kt = &c->kt;
        }
        for (size_t i = 0; i < nSS; i++) c->type[nGeo + i] = deme::SPHERE_SPHERE_CONTACT;
        deme::bodyID_t* outA = c->idA.data() + nGeo;
        deme::bodyID_t* outB = c->idB.data() + nGeo;
        launch(blocks_for(nActive, DEME_KT_CD_NTHREADS_PER_BLOCK), DEME_KT_CD_NTHREADS_PER_BLOCK, [&] {
            populateContactPairsEachBin(sp, kt, c->pairSph.data(), activeBins.data(), numSphBin.data(),
                                        lookUp.data(), offs.data(), outA, outB, nActive);
        });
    }
    size_t n = nGeo + nSS;
    c->nC = n;
    // sort by idA (two stable SortPairs in the reference; one stable permutation here)
    if (n > 0) {
        std::vector<deme::bodyID_t> a(c->idA.begin(), c->idA.begin() + n), b(n), bo(n);
        std::vector<deme::contact_t> tp(n);
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return a[x] < a[y]; });
        for (size_t i = 0; i < n; i++) {
            b[i] = c->idB[idx[i]];
            tp[i] = c->type[idx[i]];
        }
        for (size_t i = 0; i < n; i++) {
            c->idA[i] = a[idx[i]];
            c->idB[i] = b[i];
            c->type[i] = tp[i];
        }
        if (c->nW > 0) {
            // history map (DEMCubContactDetection.cu:266-372)
            size_t nSafe = nS;
            std::vector<deme::geoSphereTouches_t> newRL(nSafe + 1), oldRL(nSafe + 1), newFull(nSafe + 1, 0),
                oldFull(nSafe + 1, 0);
            std::vector<deme::bodyID_t> newU(nSafe + 1), oldU(nSafe + 1);
            size_t nNewU = rle(c->idA.data(), newU.data(), newRL.data(), n);
            size_t nOldU = rle(c->pA.data(), oldU.data(), oldRL.data(), c->nPrev);
            if (nNewU > 0)
                launch(blocks_for(nNewU, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK,
                       [&] { fillRunLengthArray(newFull.data(), newU.data(), newRL.data(), nNewU); });
            if (nOldU > 0)
                launch(blocks_for(nOldU, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK,
                       [&] { fillRunLengthArray(oldFull.data(), oldU.data(), oldRL.data(), nOldU); });
            std::vector<deme::contactPairs_t> newScan(nSafe + 1), oldScan(nSafe + 1);
            exclusive_scan(newFull.data(), newScan.data(), nSafe);
            exclusive_scan(oldFull.data(), oldScan.data(), nSafe);
            c->pack();
            kt = &c->kt;
            launch(blocks_for(nSafe, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, [&] {
                buildPersistentMap(newFull.data(), oldFull.data(), newScan.data(), oldScan.data(), c->map.data(), kt,
                                   nSafe);
            });
            c->pA.assign(c->idA.begin(), c->idA.begin() + n);
            c->pB.assign(c->idB.begin(), c->idB.begin() + n);
            c->pT.assign(c->type.begin(), c->type.begin() + n);
        }
    } else if (c->nW > 0) {
        c->pA.assign(1, 0);
        c->pB.assign(1, 0);
        c->pT.assign(1, 0);
    }
    c->nPrev = n;
    // dT side: migratePersistentContacts (rearrangeContactWildcards)
    if (c->nW > 0 && n > 0) {
        c->pack();
        std::vector<float> newWc((size_t)n * c->nW);
        std::vector<deme::notStupidBool_t> sentry(std::max<size_t>(c->wc[0].size(), 1));
        launch(blocks_for(n, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK, [&] {
            rearrangeContactWildcards(&c->dt, newWc.data(), sentry.data(), (unsigned)c->nW, n);
        });
        for (int k = 0; k < c->nW; k++)
            std::memcpy(c->wc[k].data(), newWc.data() + (size_t)k * n, n * sizeof(float));
    }
    return DEME_OK;
}

int32_t ref_compute_forces(ref_ctx* c) {
    c->pack();
    deme::DEMSimParams* sp = &c->sp;
    deme::DEMDataDT* dt = &c->dt;
    size_t n = c->nC;
    size_t nPrep = std::max<size_t>(c->nO, n);
    launch(blocks_for(nPrep, DEME_MAX_THREADS_PER_BLOCK), DEME_MAX_THREADS_PER_BLOCK,
           [&] { prepareForceArrays(sp, dt, n); });
    if (n == 0) return DEME_OK;
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { calculateContactForces(sp, dt, n); });
    // collectContactForces
    std::vector<deme::bodyID_t> owners(2 * n), ownersSorted(2 * n), uniq(2 * n);
    deme::bodyID_t* idAOwner = owners.data();
    deme::bodyID_t* idBOwner = owners.data() + n;
    deme::bodyID_t* ownerClumpBody = c->sOwner.data();
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { cashInOwnerIndexA(idAOwner, c->idA.data(), ownerClumpBody, c->type.data(), n); });
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { cashInOwnerIndexB(idBOwner, c->idB.data(), ownerClumpBody, c->type.data(), n); });
    std::vector<float3> acc(2 * n), accSorted(2 * n), accOwner(2 * n);
    auto reduce_stash = [&](float* o1, float* o2, float* o3) {
        stable_sort_pairs(owners.data(), ownersSorted.data(), acc.data(), accSorted.data(), 2 * n);
        size_t runs = 0;
        for (size_t i = 0; i < 2 * n; i++) {
            if (i == 0 || ownersSorted[i] != ownersSorted[i - 1]) {
                uniq[runs] = ownersSorted[i];
                accOwner[runs] = accSorted[i];
                runs++;
            } else {
                float3& s = accOwner[runs - 1];
                s = make_float3(s.x + accSorted[i].x, s.y + accSorted[i].y, s.z + accSorted[i].z);
            }
        }
        launch(blocks_for(runs, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
               [&] { stashElem(o1, o2, o3, uniq.data(), accOwner.data(), runs); });
    };
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { forceToAcc(acc.data(), c->F.data(), idAOwner, 1.f, n, dt); });
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { forceToAcc(acc.data() + n, c->F.data(), idBOwner, -1.f, n, dt); });
    reduce_stash(c->aX.data(), c->aY.data(), c->aZ.data());
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, [&] {
        forceToAngAcc(acc.data(), c->CPA.data(), c->qw.data(), c->qx.data(), c->qy.data(), c->qz.data(), c->F.data(),
                      c->TOF.data(), idAOwner, 1.f, n, dt);
    });
    launch(blocks_for(n, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK, [&] {
        forceToAngAcc(acc.data() + n, c->CPB.data(), c->qw.data(), c->qx.data(), c->qy.data(), c->qz.data(),
                      c->F.data(), c->TOF.data(), idBOwner, -1.f, n, dt);
    });
    reduce_stash(c->alX.data(), c->alY.data(), c->alZ.data());
    return DEME_OK;
}

int32_t ref_integrate(ref_ctx* c) {
    c->pack();
    launch(blocks_for(c->nO, DEME_NUM_BODIES_PER_BLOCK), DEME_NUM_BODIES_PER_BLOCK,
           [&] { integrateOwners(&c->sp, &c->dt, c->tf); });
    c->t += (double)c->sp.h;
    c->tf += c->sp.h;  // timeElapsed += simParams->h (src/DEM/dT.cpp:1585)
    c->steps++;
    return DEME_OK;
}

int32_t ref_step(ref_ctx* c, int32_t n) {
    for (int32_t k = 0; k < n; k++) {
        if (c->cd_freq <= 0 || (c->steps % c->cd_freq) == 0) ref_detect_contacts(c);
        ref_compute_forces(c);
        ref_integrate(c);
    }
    return DEME_OK;
}

#define RCPY_OUT(dst, vec, n) \
    if (dst) std::memcpy((dst), (vec).data(), (size_t)(n) * sizeof((vec)[0]))
#define RCPY_IN(vec, src, n) \
    if (src) std::memcpy((vec).data(), (src), (size_t)(n) * sizeof((vec)[0]))

int32_t ref_download_state(ref_ctx* c, deme_state* o) {
    uint32_t n = c->nO;
    RCPY_OUT(o->voxel, c->voxel, n);
    RCPY_OUT(o->locX, c->locX, n);
    RCPY_OUT(o->locY, c->locY, n);
    RCPY_OUT(o->locZ, c->locZ, n);
    RCPY_OUT(o->oriQw, c->qw, n);
    RCPY_OUT(o->oriQx, c->qx, n);
    RCPY_OUT(o->oriQy, c->qy, n);
    RCPY_OUT(o->oriQz, c->qz, n);
    RCPY_OUT(o->vX, c->vX, n);
    RCPY_OUT(o->vY, c->vY, n);
    RCPY_OUT(o->vZ, c->vZ, n);
    RCPY_OUT(o->omgX, c->wX, n);
    RCPY_OUT(o->omgY, c->wY, n);
    RCPY_OUT(o->omgZ, c->wZ, n);
    RCPY_OUT(o->aX, c->aX, n);
    RCPY_OUT(o->aY, c->aY, n);
    RCPY_OUT(o->aZ, c->aZ, n);
    RCPY_OUT(o->alphaX, c->alX, n);
    RCPY_OUT(o->alphaY, c->alY, n);
    RCPY_OUT(o->alphaZ, c->alZ, n);
    RCPY_OUT(o->family, c->fam, n);
    return DEME_OK;
}
int32_t ref_upload_state(ref_ctx* c, const deme_state* s) {
    uint32_t n = c->nO;
    RCPY_IN(c->voxel, s->voxel, n);
    RCPY_IN(c->locX, s->locX, n);
    RCPY_IN(c->locY, s->locY, n);
    RCPY_IN(c->locZ, s->locZ, n);
    RCPY_IN(c->qw, s->oriQw, n);
    RCPY_IN(c->qx, s->oriQx, n);
    RCPY_IN(c->qy, s->oriQy, n);
    RCPY_IN(c->qz, s->oriQz, n);
    RCPY_IN(c->vX, s->vX, n);
    RCPY_IN(c->vY, s->vY, n);
    RCPY_IN(c->vZ, s->vZ, n);
    RCPY_IN(c->wX, s->omgX, n);
    RCPY_IN(c->wY, s->omgY, n);
    RCPY_IN(c->wZ, s->omgZ, n);
    RCPY_IN(c->aX, s->aX, n);
    RCPY_IN(c->aY, s->aY, n);
    RCPY_IN(c->aZ, s->aZ, n);
    RCPY_IN(c->alX, s->alphaX, n);
    RCPY_IN(c->alY, s->alphaY, n);
    RCPY_IN(c->alZ, s->alphaZ, n);
    RCPY_IN(c->fam, s->family, n);
    return DEME_OK;
}
uint32_t ref_num_contacts(ref_ctx* c) { return (uint32_t)c->nC; }
int32_t ref_download_contacts(ref_ctx* c, deme_contacts* o) {
    o->n_contacts = (uint32_t)c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    size_t n = c->nC;
    RCPY_OUT(o->idA, c->idA, n);
    RCPY_OUT(o->idB, c->idB, n);
    RCPY_OUT(o->type, c->type, n);
    if (o->mapping) {
        if (c->nW > 0)
            std::memcpy(o->mapping, c->map.data(), n * sizeof(uint32_t));
        else
            for (size_t i = 0; i < n; i++) o->mapping[i] = DEME_NULL_MAPPING_PARTNER;
    }
    if (o->wildcards)
        for (int k = 0; k < c->nW; k++)
            std::memcpy(o->wildcards + (size_t)k * o->capacity, c->wc[k].data(), n * sizeof(float));
    return DEME_OK;
}
int32_t ref_upload_contacts(ref_ctx* c, const deme_contacts* in) {
    size_t n = in->n_contacts;
    c->resize_contacts(std::max<size_t>(n, c->idA.size()));
    c->nC = n;
    std::memcpy(c->idA.data(), in->idA, n * sizeof(uint32_t));
    std::memcpy(c->idB.data(), in->idB, n * sizeof(uint32_t));
    std::memcpy(c->type.data(), in->type, n);
    for (int k = 0; k < c->nW; k++) {
        if (in->wildcards)
            std::memcpy(c->wc[k].data(), in->wildcards + (size_t)k * in->capacity, n * sizeof(float));
        else
            std::fill(c->wc[k].begin(), c->wc[k].begin() + n, 0.f);
    }
    c->pA.assign(c->idA.begin(), c->idA.begin() + std::max<size_t>(n, 1));
    c->pB.assign(c->idB.begin(), c->idB.begin() + std::max<size_t>(n, 1));
    c->pT.assign(c->type.begin(), c->type.begin() + std::max<size_t>(n, 1));
    c->nPrev = n;
    return DEME_OK;
}
int32_t ref_download_contact_forces(ref_ctx* c, deme_contact_forces* o) {
    o->n_contacts = (uint32_t)c->nC;
    if (o->capacity < c->nC) return DEME_ERR_OVERFLOW;
    size_t n3 = c->nC * 3;
    if (o->force) std::memcpy(o->force, c->F.data(), n3 * sizeof(float));
    if (o->torque_only_force) std::memcpy(o->torque_only_force, c->TOF.data(), n3 * sizeof(float));
    if (o->cpA) std::memcpy(o->cpA, c->CPA.data(), n3 * sizeof(float));
    if (o->cpB) std::memcpy(o->cpB, c->CPB.data(), n3 * sizeof(float));
    return DEME_OK;
}
int32_t ref_bin_assignment(ref_ctx* c, uint16_t* n_bins, uint8_t* n_anal, uint32_t cap, uint32_t* bins,
                           uint32_t* spheres, uint32_t* n_pairs) {
    size_t P = c->pairBin.size() ? c->pairBin.size() - 1 : 0;
    if (n_bins) std::memcpy(n_bins, c->nBins.data(), c->nS * sizeof(uint16_t));
    if (n_anal) std::memcpy(n_anal, c->nAnal.data(), c->nS);
    if (n_pairs) *n_pairs = (uint32_t)P;
    if (bins && spheres) {
        if (cap < P) return DEME_ERR_OVERFLOW;
        std::memcpy(bins, c->pairBin.data(), P * sizeof(uint32_t));
        std::memcpy(spheres, c->pairSph.data(), P * sizeof(uint32_t));
    }
    return DEME_OK;
}
double ref_time(ref_ctx* c) { return c->t; }

}  // extern "C"
