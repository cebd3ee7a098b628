// capi.cu -- the solver handle behind the C ABI (include/deme_b200.h).
//
// One handle owns all device arrays of one scene on one GPU.  The reference keeps the same data in managed
// vectors of its two worker threads (src/DEM/dT.h:88-247, src/DEM/kT.h) and copies it between them every step;
// here kT and dT share one HBM address space, so the kT product is a double-buffered contact list whose roles
// swap by pointer, and nothing is copied between the halves.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/deme_b200.h"
#include "force_jit.cuh"
#include "handle.cuh"
#include "kernels.cuh"
#include "primitives.cuh"
#include "profiler.cuh"

int32_t dalloc(deme_handle* h, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        h->err = std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
        return DEME_ERR_OOM;
    }
    h->allocs.push_back(*p);
    return DEME_OK;
}
void dfree(deme_handle* h, void* p) {
    if (!p) return;
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if (it != h->allocs.end()) h->allocs.erase(it);
    cudaFree(p);
}

int32_t check_launch(deme_handle* h, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        h->err = std::string(what) + ": " + cudaGetErrorString(e);
        return DEME_ERR_CUDA;
    }
    return DEME_OK;
}

int32_t read_device_errors(deme_handle* h) {
    CUDA_TRY(h, cudaMemcpyAsync(h->hErr, h->dErr, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st_dt));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    if (*h->hErr) {
        uint32_t e = *h->hErr;
        uint32_t w[4] = {0, 0, 0, 0};
        cudaMemcpy(w, h->dErr, sizeof(w), cudaMemcpyDeviceToHost);
        h->err = "device error word " + std::to_string(e) +
                 ((e & ERR_SORT_LOOKBACK_TIMEOUT) ? " (radix sort look-back timed out)" : "") +
                ((e & ERR_SCAN_LOOKBACK_TIMEOUT) ? " (scan look-back timed out)" : "") +
                 ((e & ERR_CONTACT_CAPACITY) ? " (contact capacity exceeded)" : "") +
                 ((e & ERR_SEGMENT_TOO_LONG) ? " (contact segment mismatch)" : "") +
                 ((e & ERR_INDEX) ? " (index out of range at site " + std::to_string(w[1]) + ": " +
                                        std::to_string(w[2]) + " >= " + std::to_string(w[3]) + ")"
                                  : "");
        *h->hErr = 0;
        cudaMemsetAsync(h->dErr, 0, 4 * sizeof(uint32_t), h->st_dt);
        return (e & (ERR_SORT_LOOKBACK_TIMEOUT | ERR_SCAN_LOOKBACK_TIMEOUT)) ? DEME_ERR_TIMEOUT : DEME_ERR_OVERFLOW;
    }
    return DEME_OK;
}

static int32_t ensure_scratch(deme_handle* h, size_t bytes) {
    if (bytes <= h->scratchBytes) return DEME_OK;
    dfree(h, h->scratch);
    h->scratch = nullptr;
    h->scratchBytes = 0;
    TRY(dalloc(h, &h->scratch, bytes));
    h->scratchBytes = bytes;
    return DEME_OK;
}

int32_t ensure_list(deme_handle* h, ContactBuf& b, uint32_t n) {
    if (n <= b.cap) return DEME_OK;
    uint32_t cap = std::max<uint32_t>(1024u, (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)n * 5 / 4 + 64));
    dfree(h, b.idA);
    dfree(h, b.idB);
    dfree(h, b.type);
    dfree(h, b.hist);
    dfree(h, b.mapping);
    b.idA = b.idB = b.mapping = nullptr;
    b.type = nullptr;
    b.hist = nullptr;
    b.cap = 0;
    TRY(dalloc_n(h, &b.idA, cap));
    TRY(dalloc_n(h, &b.idB, cap));
    TRY(dalloc_n(h, &b.type, cap));
    TRY(dalloc_n(h, &b.hist, cap));
    TRY(dalloc_n(h, &b.mapping, cap));
    b.cap = cap;
    return DEME_OK;
}

// Grows a list that is in use, keeping its contents (ids, history, mapping).
static int32_t ensure_list_keep(deme_handle* h, ContactBuf& b, uint32_t n, uint32_t used, cudaStream_t st) {
    if (n <= b.cap) return DEME_OK;
    ContactBuf old = b;
    ContactBuf grown = b;
    const uint32_t cap = std::max<uint32_t>(1024u, (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)n * 5 / 4 + 64));
    TRY(dalloc_n(h, &grown.idA, cap));
    TRY(dalloc_n(h, &grown.idB, cap));
    TRY(dalloc_n(h, &grown.type, cap));
    TRY(dalloc_n(h, &grown.hist, cap));
    TRY(dalloc_n(h, &grown.mapping, cap));
    grown.cap = cap;
    if (used) {
        CUDA_TRY(h, cudaMemcpyAsync(grown.idA, old.idA, used * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(grown.idB, old.idB, used * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(grown.type, old.type, used * sizeof(uint8_t), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(grown.hist, old.hist, used * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(grown.mapping, old.mapping, used * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));
    dfree(h, old.idA);
    dfree(h, old.idB);
    dfree(h, old.type);
    dfree(h, old.hist);
    dfree(h, old.mapping);
    b = grown;
    return DEME_OK;
}

// The built-in model's contact-pair parameters, recomputed whenever a material changes.
int32_t refresh_material_pairs(deme_handle* h) {
    if (!h->matPair) return DEME_OK;
    launch_material_pairs(h->state_view().mat, h->nM, h->matPair, h->st_dt);
    return check_launch(h, "material_pairs");
}

// The count of the list in use, read back after a graph replay produced it on the device.
int32_t refresh_count(deme_handle* h) {
    if (!h->countStale) return DEME_OK;
    CUDA_TRY(h, cudaMemcpyAsync(h->hTotal + 3, h->lists[h->cur].dN, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st_dt));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    h->nContacts = h->hTotal[3];
    h->countStale = false;
    return DEME_OK;
}

static int32_t ensure_cand(deme_handle* h, uint32_t n) {
    if (n <= h->candCap) return DEME_OK;
    const uint32_t cap = std::max<uint32_t>(1024u, (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)n * 5 / 4 + 64));
    dfree(h, h->cd.candTemp);
    h->cd.candTemp = nullptr;
    h->candCap = 0;
    TRY(dalloc_n(h, &h->cd.candTemp, cap));
    h->candCap = cap;
    return DEME_OK;
}

// Room for n (sphere, facet) pairs in the mesh pool.
static int32_t ensure_mesh_pool(deme_handle* h, uint32_t n) {
    if (n <= h->cd.meshCap && h->cd.meshPool) return DEME_OK;
    const uint32_t cap = std::max<uint32_t>(1024u, (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)n * 5 / 4 + 64));
    dfree(h, h->cd.meshPool);
    h->cd.meshPool = nullptr;
    h->cd.meshCap = 0;
    TRY(dalloc_n(h, &h->cd.meshPool, cap));
    h->cd.meshCap = cap;
    return DEME_OK;
}

// A search's counts (total, pool, overflow spheres, -, mesh pairs) fit the buffers it wrote into.
static bool search_fits(const deme_handle* h, const uint32_t* c) {
    return c[1] <= h->candCap && (!h->nT || c[4] <= h->cd.meshCap);
}
static int32_t grow_search(deme_handle* h, const uint32_t* c) {
    TRY(ensure_cand(h, c[1]));
    if (h->nT) TRY(ensure_mesh_pool(h, c[4]));
    return DEME_OK;
}

static int32_t ensure_outputs(deme_handle* h, uint32_t n) {
    if (n <= h->outCap) return DEME_OK;
    uint32_t cap = std::max<uint32_t>(1024u, n + n / 4);
    dfree(h, h->outs.F);
    dfree(h, h->outs.TOF);
    dfree(h, h->outs.CPA);
    dfree(h, h->outs.CPB);
    h->outs = ContactOutputs{nullptr, nullptr, nullptr, nullptr};
    h->outCap = 0;
    TRY(dalloc_n(h, &h->outs.F, cap));
    TRY(dalloc_n(h, &h->outs.TOF, cap));
    TRY(dalloc_n(h, &h->outs.CPA, cap));
    TRY(dalloc_n(h, &h->outs.CPB, cap));
    h->outCap = cap;
    return DEME_OK;
}

extern "C" {

int32_t deme_abi_version(void) { return DEME_B200_ABI_VERSION; }

const char* deme_status_string(int32_t s) {
    switch (s) {
        case DEME_OK: return "DEME_OK";
        case DEME_ERR_INVALID: return "DEME_ERR_INVALID";
        case DEME_ERR_CUDA: return "DEME_ERR_CUDA";
        case DEME_ERR_OOM: return "DEME_ERR_OOM";
        case DEME_ERR_OVERFLOW: return "DEME_ERR_OVERFLOW";
        case DEME_ERR_NVRTC: return "DEME_ERR_NVRTC";
        case DEME_ERR_TIMEOUT: return "DEME_ERR_TIMEOUT";
        case DEME_ERR_STATE: return "DEME_ERR_STATE";
        case DEME_ERR_NO_DEVICE: return "DEME_ERR_NO_DEVICE";
        case DEME_ERR_TOO_LARGE: return "DEME_ERR_TOO_LARGE";
        default: return "unknown";
    }
}

const char* deme_get_error(deme_handle* h) { return h ? h->err.c_str() : "null handle"; }

// Search cells: per scene, cubes of edge cell_factor x max(bin size, the scene's largest expanded diameter) over the
// scene's box (the user's domain, or the voxel world, when the run holds one scene), coarsened together while there
// would be more than 2^26 cells in all.  Factor 1 gives the most cells, which the cell arrays are sized for; any
// factor >= 1 finds the same pairs.  The grid table goes to the device (h->grids).
static int32_t set_cell_grid(deme_handle* h, double cell_factor) {
    const deme_sim_params* p = &h->params;
    const double factor = std::max(cell_factor, 1.0);
    const uint32_t nG = (uint32_t)h->sceneRmax.size();
    std::vector<SearchGrid> g(nG);
    double grow = 1.0;
    uint64_t total = 0;
    while (true) {
        total = 0;
        for (uint32_t sc = 0; sc < nG; sc++) {
            double cs = std::max(p->bin_size, 2.0 * (double)h->sceneRmax[sc]) * (1.0 + 1e-6) * factor * grow;
            if (!(cs > 0.0)) cs = 1.0;
            const double* lo = &h->sceneBox[6 * (size_t)sc];
            uint64_t n[3];
            for (int a = 0; a < 3; a++) n[a] = (uint64_t)std::ceil(std::max(lo[3 + a] - lo[a], 0.0) / cs) + 1;
            SearchGrid& q = g[sc];
            q = SearchGrid{};
            q.ox = lo[0];
            q.oy = lo[1];
            q.oz = lo[2];
            q.inv_cell = 1.0 / cs;
            q.gx = (uint32_t)std::min<uint64_t>(n[0], 1u << 26);
            q.gy = (uint32_t)std::min<uint64_t>(n[1], 1u << 26);
            q.gz = (uint32_t)std::min<uint64_t>(n[2], 1u << 26);
            q.base = (uint32_t)std::min<uint64_t>(total, 0xFFFFFFFFull);
            q.r_max_cd = h->sceneRmax[sc];
            total += (uint64_t)q.gx * q.gy * q.gz;
        }
        if (total <= (1ull << 26)) break;
        grow *= 1.25;
    }
    h->nCells = (uint32_t)total;
    h->cellBits = 1;
    while ((1ull << h->cellBits) < h->nCells) h->cellBits++;
    h->cellFactor = (float)factor;
    if (!h->grids) TRY(dalloc_n(h, &h->grids, std::max(nG, 1u)));
    CUDA_TRY(h, cudaMemcpy(h->grids, g.data(), nG * sizeof(SearchGrid), cudaMemcpyHostToDevice));
    h->k.grids = h->grids;
    h->k.grid0 = g[0];  // a run of one scene reads its grid from here; its origin is the domain's corner, base 0
    return DEME_OK;
}

// The scenes' boxes and largest expanded radii for the search grids: one scene spanning the domain, or, when the
// scene packs several independent scenes (owner_scene), one box per scene (scene_box, or the bounding box of the
// scene's initial owner positions widened by its clump reach and half its size).
static int32_t set_scene_boxes(deme_handle* h, const deme_scene* s) {
    const deme_sim_params* p = &h->params;
    const double world[3] = {p->voxel_size * std::ldexp(1.0, p->nvXp2), p->voxel_size * std::ldexp(1.0, p->nvYp2),
                             p->voxel_size * std::ldexp(1.0, p->nvZp2)};
    if (!s->owner_scene) {
        h->sceneRmax.assign(1, h->k.r_max_cd);
        h->sceneBox.assign(6, 0.0);
        for (int a = 0; a < 3; a++) h->sceneBox[3 + a] = p->domain[a] > 0.f ? (double)p->domain[a] : world[a];
        return DEME_OK;
    }
    uint32_t nG = 0;
    for (uint32_t o = 0; o < h->nO; o++) nG = std::max(nG, s->owner_scene[o] + 1);
    if (nG > (1u << 20)) {
        h->err = "owner_scene: more than 2^20 scenes";
        return DEME_ERR_INVALID;
    }
    h->sceneRmax.assign(nG, 0.f);
    std::vector<float> reach(nG, 0.f);
    for (uint32_t i = 0; i < h->nS; i++) {
        const uint32_t sc = s->owner_scene[s->sphere_owner[i]];
        float r = s->radius[i];
        r += p->beta;
        h->sceneRmax[sc] = std::max(h->sceneRmax[sc], r);
        const float rel = std::sqrt(s->relX[i] * s->relX[i] + s->relY[i] * s->relY[i] + s->relZ[i] * s->relZ[i]);
        reach[sc] = std::max(reach[sc], rel + r);
    }
    h->sceneBox.assign(6 * (size_t)nG, 0.0);
    if (s->scene_box) {
        for (size_t i = 0; i < 6 * (size_t)nG; i++) h->sceneBox[i] = (double)s->scene_box[i];
        return DEME_OK;
    }
    std::vector<double> lo(3 * (size_t)nG, 1e300), hi(3 * (size_t)nG, -1e300);
    const uint64_t mx = (1ull << p->nvXp2) - 1, my = (1ull << p->nvYp2) - 1;
    for (uint32_t o = 0; o < h->nClumps; o++) {
        const uint32_t sc = s->owner_scene[o];
        const uint64_t v = s->voxel[o];
        const double x[3] = {(double)(v & mx) * p->voxel_size + s->locX[o] * p->l,
                             (double)((v >> p->nvXp2) & my) * p->voxel_size + s->locY[o] * p->l,
                             (double)(v >> (p->nvXp2 + p->nvYp2)) * p->voxel_size + s->locZ[o] * p->l};
        for (int a = 0; a < 3; a++) {
            lo[3 * sc + a] = std::min(lo[3 * sc + a], x[a]);
            hi[3 * sc + a] = std::max(hi[3 * sc + a], x[a]);
        }
    }
    for (uint32_t sc = 0; sc < nG; sc++)
        for (int a = 0; a < 3; a++) {
            double l0 = lo[3 * sc + a], h0 = hi[3 * sc + a];
            if (l0 > h0) l0 = h0 = 0.0;  // a scene without clumps
            const double pad = reach[sc] + 0.25 * (h0 - l0);
            h->sceneBox[6 * sc + a] = l0 - pad;
            h->sceneBox[6 * sc + 3 + a] = h0 + pad;
        }
    return DEME_OK;
}

// The sphere id in the low bits of a cell-order record's last word and a CD radius bound in the bits above (at
// least 4 of them; with fewer the bound is r_max_cd for every sphere).
static void radius_bounds(SimConsts& k, uint32_t nS, float rmax) {
    uint32_t idBits = 1;
    while (idBits < 31 && (1ull << idBits) < (uint64_t)nS) idBits++;
    if (32 - idBits >= 4) {
        k.q_shift = idBits;
        k.q_scale = rmax / (float)((1u << (32 - idBits)) - 1u);
    } else {
        k.q_shift = 31;
        k.q_scale = rmax;
    }
    k.id_mask = (1u << k.q_shift) - 1u;
}

static int32_t create_impl(deme_handle* h, const deme_sim_params* p, const deme_scene* s) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        h->err = "no CUDA device";
        return DEME_ERR_NO_DEVICE;
    }
    CUDA_TRY(h, cudaGetDevice(&h->device));
    h->params = *p;
    h->nO = s->n_owners;
    h->nS = s->n_spheres;
    h->nA = s->n_anal;
    h->nM = s->n_materials;
    h->nW = p->n_contact_wildcards;
    if (h->nW != 0 && h->nW != 4) {
        h->err = "the built-in models use 0 or 4 contact wildcards";
        return DEME_ERR_INVALID;
    }
    if (p->nbX > 65535u || p->nbY > 65535u || p->nbZ > 65535u) {
        h->err = "more than 65535 bins along an axis: enlarge the bin size";
        return DEME_ERR_INVALID;
    }
    if ((int)p->nvXp2 + (int)p->nvYp2 + (int)p->nvZp2 > 64) {
        h->err = "voxel bits nvXp2 + nvYp2 + nvZp2 exceed 64: voxel ids would wrap";
        return DEME_ERR_INVALID;
    }
    if (s->owner_anal_first && s->owner_anal_count) {
        // packed scenes: each owner meets only its own range of components (at most 255 of them)
        for (uint32_t o = 0; o < h->nO; o++)
            if (s->owner_anal_count[o] > 255 || (uint64_t)s->owner_anal_first[o] + s->owner_anal_count[o] > h->nA) {
                h->err = "owner analytical range out of bounds or wider than 255 components";
                return DEME_ERR_INVALID;
            }
    } else if (h->nA > 255) {
        h->err = "at most 255 analytical components";
        return DEME_ERR_INVALID;
    }
    const uint32_t nO = h->nO, nS = h->nS, nA = h->nA, nM = h->nM;
    // clumps are the owners referenced by spheres; analytical owners follow them
    uint32_t nClumps = 0;
    for (uint32_t i = 0; i < nS; i++) nClumps = std::max(nClumps, s->sphere_owner[i] + 1);
    for (uint32_t i = 0; i < nA; i++)
        if (s->anal_owner[i] < nClumps || s->anal_owner[i] >= nO) {
            h->err = "analytical owners must follow the clump owners";
            return DEME_ERR_INVALID;
        }
    for (uint32_t i = 0; i < nS; i++)
        if (s->sphere_owner[i] >= nO ||
            (s->sphere_material_wide ? s->sphere_material_wide[i] : s->sphere_material[i]) >= std::max(nM, 1u)) {
            h->err = "sphere owner or material out of range";
            return DEME_ERR_INVALID;
        }
    for (uint32_t i = 1; i < nS; i++)
        if (s->sphere_owner[i] < s->sphere_owner[i - 1]) {
            h->err = "spheres must be grouped by owner in ascending owner order";
            return DEME_ERR_INVALID;
        }
    h->nClumps = nClumps;
    h->nT = s->n_tris;
    if (h->nT) {
        if (s->owner_scene || s->owner_anal_first) {
            h->err = "mesh facets are not supported together with packed scenes";
            return DEME_ERR_INVALID;
        }
        if (!s->tri_owner || !s->tri_node1 || !s->tri_node2 || !s->tri_node3 || !s->tri_material) {
            h->err = "n_tris > 0 needs tri_owner, tri_node1..3 and tri_material";
            return DEME_ERR_INVALID;
        }
        for (uint32_t i = 0; i < h->nT; i++) {
            if (s->tri_owner[i] < nClumps || s->tri_owner[i] >= nO || s->tri_material[i] >= std::max(nM, 1u)) {
                h->err = "mesh facet owner (must follow the clump owners) or material out of range";
                return DEME_ERR_INVALID;
            }
            // a facet of zero area has no closest-point region test that is defined everywhere
            const float *a = s->tri_node1 + 3 * (size_t)i, *b = s->tri_node2 + 3 * (size_t)i,
                        *c = s->tri_node3 + 3 * (size_t)i;
            const double u[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
            const double v[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
            const double n[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
            if (!(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] > 0.0)) {
                h->err = "mesh facet " + std::to_string(i) + " has zero area (or non-finite nodes)";
                return DEME_ERR_INVALID;
            }
        }
    }
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->own_dt, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->own_kt, cudaStreamNonBlocking));
    h->st_dt = h->own_dt;
    h->st_kt = h->own_kt;

    // ---- constants and the contact search grid ----
    SimConsts& k = h->k;
    k.nvXp2 = p->nvXp2;
    k.nvYp2 = p->nvYp2;
    k.l_kernel = p->l_kernel;
    k.voxel_kernel = p->voxel_size_kernel;
    k.bin_size = p->bin_size;
    k.nbX = p->nbX;
    k.nbY = p->nbY;
    k.nbZ = p->nbZ;
    k.beta = p->beta;
    k.h = p->h;
    k.G[0] = p->G[0];
    k.G[1] = p->G[1];
    k.G[2] = p->G[2];
    k.integrator = p->integrator;
    k.n_spheres = nS;
    k.n_owners = nO;
    k.n_anal = nA;
    k.n_tris = h->nT;
    float rmax = 0.f;
    for (uint32_t i = 0; i < nS; i++) {
        float r = s->radius[i];
        r += p->beta;
        rmax = std::max(rmax, r);
    }
    k.r_max_cd = rmax;
    const double world[3] = {p->voxel_size * std::ldexp(1.0, p->nvXp2), p->voxel_size * std::ldexp(1.0, p->nvYp2),
                             p->voxel_size * std::ldexp(1.0, p->nvZp2)};
    const double wmax = std::max(world[0], std::max(world[1], world[2]));
    if (s->owner_scene) {
        TRY(dalloc_n(h, &h->ownerScene, std::max(nO, 1u)));
        CUDA_TRY(h, cudaMemcpy(h->ownerScene, s->owner_scene, nO * sizeof(uint32_t), cudaMemcpyHostToDevice));
        k.ownerScene = h->ownerScene;
    }
    TRY(set_scene_boxes(h, s));
    k.prefilter_abs = (float)(4e-7 * wmax + 1e-9);
    radius_bounds(k, nS, rmax);
    TRY(set_cell_grid(h, 1.0));
    h->cellCap = h->nCells;  // the cell arrays below are sized for the finest grid (factor 1)

    // ---- device arrays ----
    TRY(dalloc_n(h, &h->voxel, nO));
    TRY(dalloc_n(h, &h->loc, nO));
    TRY(dalloc_n(h, &h->quat, nO));
    TRY(dalloc_n(h, &h->vel, nO));
    TRY(dalloc_n(h, &h->omg, nO));
    TRY(dalloc_n(h, &h->moi, nO));
    TRY(dalloc_n(h, &h->invMoi, nO));
    TRY(dalloc_n(h, &h->acc, nO));
    TRY(dalloc_n(h, &h->alpha, nO));
    TRY(dalloc_n(h, &h->sph, nS));
    TRY(dalloc_n(h, &h->sOwner, nS));
    TRY(dalloc_n(h, &h->sMat, nS));
    TRY(dalloc_n(h, &h->masks, DEME_NUM_FAMILY_MASK));
    TRY(dalloc_n(h, &h->mat, 5 * std::max(nM, 1u)));
    if (nM && nM <= kMaxPairTableMaterials) TRY(dalloc_n(h, &h->matPair, 2 * (size_t)nM * nM));
    TRY(dalloc_n(h, &h->analRaw, std::max(nA, 1u)));
    TRY(dalloc_n(h, &h->analPlaced, std::max(nA, 1u)));
    TRY(dalloc_n(h, &h->presc, DEME_NUM_FAMILIES));
    {
        std::vector<ushort4> loc(nO);
        std::vector<float4> quat(nO), vel(nO), omg(nO), moi(nO), invMoi(nO);
        for (uint32_t o = 0; o < nO; o++) {
            loc[o] = make_ushort4(s->locX[o], s->locY[o], s->locZ[o], s->family[o]);
            quat[o] = make_float4(s->oriQw[o], s->oriQx[o], s->oriQy[o], s->oriQz[o]);
            vel[o] = make_float4(s->vX[o], s->vY[o], s->vZ[o], s->mass[o]);
            omg[o] = make_float4(s->omgX[o], s->omgY[o], s->omgZ[o], 0.f);
            moi[o] = make_float4(s->mmiXX[o], s->mmiYY[o], s->mmiZZ[o], 0.f);
            invMoi[o] = make_float4(1.f / s->mmiXX[o], 1.f / s->mmiYY[o], 1.f / s->mmiZZ[o], 1.f / s->mass[o]);
        }
        CUDA_TRY(h, cudaMemcpy(h->voxel, s->voxel, nO * sizeof(uint64_t), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->loc, loc.data(), nO * sizeof(ushort4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->quat, quat.data(), nO * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->vel, vel.data(), nO * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->omg, omg.data(), nO * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->moi, moi.data(), nO * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->invMoi, invMoi.data(), nO * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemset(h->acc, 0, nO * sizeof(float4)));
        CUDA_TRY(h, cudaMemset(h->alpha, 0, nO * sizeof(float4)));
        std::vector<float4> sph(nS);
        for (uint32_t i = 0; i < nS; i++) sph[i] = make_float4(s->relX[i], s->relY[i], s->relZ[i], s->radius[i]);
        CUDA_TRY(h, cudaMemcpy(h->sph, sph.data(), nS * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->sOwner, s->sphere_owner, nS * sizeof(uint32_t), cudaMemcpyHostToDevice));
        {
            std::vector<uint16_t> mat16(std::max(nS, 1u));
            for (uint32_t i = 0; i < nS; i++)
                mat16[i] = s->sphere_material_wide ? s->sphere_material_wide[i] : (uint16_t)s->sphere_material[i];
            CUDA_TRY(h, cudaMemcpy(h->sMat, mat16.data(), nS * sizeof(uint16_t), cudaMemcpyHostToDevice));
        }
        if (s->owner_anal_first && s->owner_anal_count) {
            std::vector<uint2> rg(nO);
            for (uint32_t o = 0; o < nO; o++) rg[o] = make_uint2(s->owner_anal_first[o], s->owner_anal_count[o]);
            TRY(dalloc_n(h, &h->ownerAnal, nO));
            CUDA_TRY(h, cudaMemcpy(h->ownerAnal, rg.data(), nO * sizeof(uint2), cudaMemcpyHostToDevice));
        }
        std::vector<uint8_t> masks(DEME_NUM_FAMILY_MASK, 0);
        if (s->family_masks) std::memcpy(masks.data(), s->family_masks, DEME_NUM_FAMILY_MASK);
        CUDA_TRY(h, cudaMemcpy(h->masks, masks.data(), DEME_NUM_FAMILY_MASK, cudaMemcpyHostToDevice));
        std::vector<float> mat(5 * std::max(nM, 1u), 0.f);
        for (uint32_t m = 0; m < nM; m++) {
            mat[m] = s->mat_E[m];
            mat[nM + m] = s->mat_nu[m];
            mat[2 * nM + m] = s->mat_CoR[m];
            mat[3 * nM + m] = s->mat_mu[m];
            mat[4 * nM + m] = s->mat_Crr[m];
        }
        CUDA_TRY(h, cudaMemcpy(h->mat, mat.data(), mat.size() * sizeof(float), cudaMemcpyHostToDevice));
        TRY(refresh_material_pairs(h));
        std::vector<AnalRaw> raw(std::max(nA, 1u));
        for (uint32_t a = 0; a < nA; a++) {
            AnalRaw r{};
            r.relX = s->anal_relX[a];
            r.relY = s->anal_relY[a];
            r.relZ = s->anal_relZ[a];
            r.rotX = s->anal_rotX[a];
            r.rotY = s->anal_rotY[a];
            r.rotZ = s->anal_rotZ[a];
            r.size1 = s->anal_size1[a];
            r.size2 = s->anal_size2[a];
            r.size3 = s->anal_size3[a];
            r.mass = s->anal_mass[a];
            r.owner = s->anal_owner[a];
            r.type = s->anal_type[a];
            r.normal = s->anal_normal[a];
            r.material = s->anal_material_wide ? s->anal_material_wide[a] : (uint16_t)s->anal_material[a];
            // cone wall: sin and cos of the half angle, computed once on the host
            r.c1 = std::sin((double)r.size1);
            r.c2 = std::cos((double)r.size1);
            if (r.material >= std::max(nM, 1u)) {
                h->err = "analytical material out of range";
                return DEME_ERR_INVALID;
            }
            raw[a] = r;
        }
        CUDA_TRY(h, cudaMemcpy(h->analRaw, raw.data(), raw.size() * sizeof(AnalRaw), cudaMemcpyHostToDevice));
        if (h->nT) {
            std::vector<TriRaw> tr(h->nT);
            for (uint32_t i = 0; i < h->nT; i++) {
                TriRaw t{};
                const float *a = s->tri_node1 + 3 * (size_t)i, *b = s->tri_node2 + 3 * (size_t)i,
                            *c = s->tri_node3 + 3 * (size_t)i;
                t.n1x = a[0], t.n1y = a[1], t.n1z = a[2];
                t.n2x = b[0], t.n2y = b[1], t.n2z = b[2];
                t.n3x = c[0], t.n3y = c[1], t.n3z = c[2];
                t.owner = s->tri_owner[i];
                t.mass = s->mass[t.owner];
                t.material = s->tri_material[i];
                tr[i] = t;
            }
            TRY(dalloc_n(h, &h->triRaw, h->nT));
            TRY(dalloc_n(h, &h->triPlaced, h->nT));
            CUDA_TRY(h, cudaMemcpy(h->triRaw, tr.data(), tr.size() * sizeof(TriRaw), cudaMemcpyHostToDevice));
        }
        std::vector<Prescription> pr(DEME_NUM_FAMILIES);
        for (int f = 0; f < DEME_NUM_FAMILIES; f++) {
            Prescription q{};
            if (s->prescriptions) {
                const deme_family_prescription& src = s->prescriptions[f];
                q.used = src.used;
                q.lin_vel = src.lin_vel_prescribed;
                q.rot_vel = src.rot_vel_prescribed;
                q.lin_pos = src.lin_pos_prescribed;
                q.rot_pos = src.rot_pos_prescribed;
                for (int c = 0; c < 3; c++) {
                    q.has_vel[c] = src.has_vel[c];
                    q.has_omg[c] = src.has_omg[c];
                    q.has_pos[c] = src.has_pos[c];
                    q.vel[c] = src.vel[c];
                    q.omg[c] = src.omg[c];
                    q.pos[c] = src.pos[c];
                }
            }
            pr[f] = q;
        }
        CUDA_TRY(h, cudaMemcpy(h->presc, pr.data(), pr.size() * sizeof(Prescription), cudaMemcpyHostToDevice));
    }
    // ---- contact-detection work arrays ----
    CDView& cd = h->cd;
    TRY(dalloc_n(h, &cd.posFSorted, nS));
    TRY(dalloc_n(h, &cd.recS, nS));
    TRY(dalloc_n(h, &cd.rngS, nS));
    {
        // runs of consecutive spheres sharing an owner: the search skips them by id
        uint2* dClump = nullptr;
        TRY(dalloc_n(h, &dClump, std::max(nS, 1u)));
        std::vector<uint2> runs(nS);
        for (uint32_t i = 0; i < nS;) {
            uint32_t e = i + 1;
            while (e < nS && s->sphere_owner[e] == s->sphere_owner[i]) e++;
            for (uint32_t q = i; q < e; q++) runs[q] = make_uint2(i, e - i);
            i = e;
        }
        if (nS) CUDA_TRY(h, cudaMemcpy(dClump, runs.data(), nS * sizeof(uint2), cudaMemcpyHostToDevice));
        cd.sClump = dClump;
    }
    TRY(dalloc_n(h, &cd.cellKey, nS));
    TRY(dalloc_n(h, &cd.idSeq, nS));
    TRY(dalloc_n(h, &cd.keySorted, nS));
    TRY(dalloc_n(h, &cd.idSorted, nS));
    TRY(dalloc_n(h, &cd.cellCount, (size_t)h->nCells + 1));
    TRY(dalloc_n(h, &cd.cellStart, (size_t)h->nCells + 1));
    TRY(dalloc_n(h, &cd.nAnal, nS));
    TRY(dalloc_n(h, &cd.cnt, (size_t)nS + 1));
    // cnt[nS] stays 0 so the scan over nS + 1 entries leaves the total in off[nS]
    CUDA_TRY(h, cudaMemset(cd.cnt, 0, ((size_t)nS + 1) * sizeof(uint32_t)));
    TRY(dalloc_n(h, &cd.ovf, nS + 1));
    TRY(dalloc_n(h, &cd.counters, 8));
    CUDA_TRY(h, cudaMemset(cd.counters, 0, 8 * sizeof(uint32_t)));
    TRY(ensure_cand(h, std::max<uint32_t>(1024u, 2u * nS)));
    if (h->nT) TRY(ensure_mesh_pool(h, std::max<uint32_t>(1024u, 2u * h->nT)));
    for (int b = 0; b < 2; b++) {
        TRY(dalloc_n(h, &h->lists[b].off, (size_t)nS + 1));
        CUDA_TRY(h, cudaMemset(h->lists[b].off, 0, ((size_t)nS + 1) * sizeof(uint32_t)));
        TRY(dalloc_n(h, &h->lists[b].dN, 1));
        CUDA_TRY(h, cudaMemset(h->lists[b].dN, 0, sizeof(uint32_t)));
        TRY(ensure_list(h, h->lists[b], std::max<uint32_t>(1024u, 4u * nS)));
    }
    TRY(ensure_scratch(h, std::max({radix_sort_scratch_bytes(nS), scan_scratch_bytes(std::max(h->nCells + 1, nS + 1)),
                                    scan_onepass_scratch_bytes(std::max(h->nCells + 1, nS + 1))})));
    TRY(dalloc_n(h, &h->dTotal, 4));
    TRY(dalloc_n(h, &h->dErr, 4));
    h->k.err = h->dErr;
    TRY(dalloc_n(h, &h->dKE, 2));
    CUDA_TRY(h, cudaMemset(h->dErr, 0, 4 * sizeof(uint32_t)));
    CUDA_TRY(h, cudaMallocHost(&h->hTotal, 8 * sizeof(uint32_t)));
    CUDA_TRY(h, cudaMallocHost(&h->hErr, 4 * sizeof(uint32_t)));
    CUDA_TRY(h, cudaMallocHost(&h->hKE, 2 * sizeof(double)));
    *h->hErr = 0;
    CUDA_TRY(h, cudaDeviceSynchronize());
    return DEME_OK;
}

int32_t deme_create(const deme_sim_params* params, const deme_scene* scene, deme_handle** out) {
    if (!params || !scene || !out) return DEME_ERR_INVALID;
    *out = nullptr;
    deme_handle* h = new deme_handle();
    int32_t st = create_impl(h, params, scene);
    if (st != DEME_OK) {
        // keep the handle so the caller can read the message; it owns no live work
        *out = h;
        return st;
    }
    *out = h;
    return DEME_OK;
}

void deme_destroy(deme_handle* h) {
    if (!h) return;
    if (h->cdPending && h->st_kt) cudaStreamSynchronize(h->st_kt);
    if (h->own_dt) cudaStreamSynchronize(h->own_dt);
    if (h->own_kt) cudaStreamSynchronize(h->own_kt);
    adjoint_release(h);  // frees its arrays through dfree, so before the bulk free below
    for (void* p : h->allocs) cudaFree(p);
    h->allocs.clear();
    if (h->hTotal) cudaFreeHost(h->hTotal);
    if (h->hErr) cudaFreeHost(h->hErr);
    if (h->hKE) cudaFreeHost(h->hKE);
    if (h->hKERing) cudaFreeHost(h->hKERing);
    for (cudaEvent_t e : h->keDone)
        if (e) cudaEventDestroy(e);
    if (h->hPresc) cudaFreeHost(h->hPresc);
    for (cudaEvent_t e : h->prescDone)
        if (e) cudaEventDestroy(e);
    if (h->hCounts) cudaFreeHost(h->hCounts);
    for (cudaEvent_t e : {h->evPose, h->evCounts, h->evListReady, h->evListReleased})
        if (e) cudaEventDestroy(e);
    for (cudaGraphExec_t g : h->graphExec)
        if (g) cudaGraphExecDestroy(g);
    if (h->hWindows) cudaFreeHost(h->hWindows);
    if (h->own_dt) cudaStreamDestroy(h->own_dt);
    if (h->own_kt) cudaStreamDestroy(h->own_kt);
    release_user_force_model(h->userForce);
    release_family_change_rules(h->famRules);
    release_prescribed_motion(h->motion);
    delete h;
}

int32_t deme_set_force_model(deme_handle* h, const char* src, const char* const* names, int32_t n) {
    if (!h) return DEME_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    if (src == nullptr) {
        // back to the built-in frictional Hertz-Mindlin model and its four history wildcards
        release_user_force_model(h->userForce);
        h->jitGeneration++;
        h->nW = h->params.n_contact_wildcards;
        return DEME_OK;
    }
    std::string err;
    const int32_t rc = compile_user_force_model(src, names, n, h->userForce, err);
    if (rc != DEME_OK) {
        h->err = err;
        return rc;
    }
    h->jitGeneration++;
    h->nW = h->userForce.n_wildcards;
    h->outsValid = false;
    return DEME_OK;
}

static int32_t cd_finish(deme_handle* h);

int32_t deme_set_streams(deme_handle* h, void* kT_stream, void* dT_stream) {
    if (!h) return DEME_ERR_INVALID;
    TRY(cd_finish(h));
    h->st_kt = kT_stream ? (cudaStream_t)kT_stream : h->own_kt;
    h->st_dt = dT_stream ? (cudaStream_t)dT_stream : h->own_dt;
    return DEME_OK;
}

int32_t deme_set_cell_sort(deme_handle* h, int32_t onesweep) {
    if (!h) return DEME_ERR_INVALID;
    h->useOnesweep = onesweep != 0;
    return DEME_OK;
}

int32_t deme_keep_contact_forces(deme_handle* h, int32_t enable) {
    if (!h) return DEME_ERR_INVALID;
    h->keepOutputs = enable != 0;
    return DEME_OK;
}

// ---------------------------------------------------------------------------------------------------- kT ----
// Contact search up to the per-sphere offsets of the new list (into lists[cur ^ 1].off, its count into .dN), for the
// poses in `s`, with the analytical components placed into `anal` (and the mesh facets into s.tri).  The pair total,
// the pool count, its overflow counter and the mesh-pair count are copied to `hCnt` (pinned, unless null; words 0,
// 1, 2 and 4) at the end, on `st`; nothing here waits for the device.
static int32_t cd_search(deme_handle* h, const StateView& s, AnalPlaced* anal, cudaStream_t st, bool retry,
                         uint32_t* hCnt) {
    const SimConsts& k = h->k;
    CDView& cd = h->cd;
    launch_place_anal(k, s, h->analRaw, anal, h->nA, st);
    launch_place_tri(k, s, h->triRaw, st);
    // the forces of this step, on the same poses, reuse the placement
    if (anal == h->analPlaced) h->analFresh = true;
    CUDA_TRY(h, cudaMemsetAsync(cd.cellCount, 0, ((size_t)h->nCells + 1) * sizeof(uint32_t), st));
    launch_sphere_prep(k, s, cd, st);
    exclusive_scan_u32_onepass(cd.cellCount, h->nCells + 1, cd.cellStart, nullptr, h->scratch, h->dErr, st);
    if (h->useOnesweep) {
        radix_sort_pairs(cd.cellKey, cd.idSeq, cd.keySorted, cd.idSorted, h->nS, h->cellBits, h->scratch, h->dErr, st);
        launch_gather_sorted(k, s, cd, st);
    } else {
        launch_cell_scatter(k, s, cd, st);  // counting sort and record writes in one pass
    }
    ContactBuf& nb = h->lists[h->cur ^ 1];
    // pool, overflow spheres, tile queue, overflow entries, mesh pairs
    CUDA_TRY(h, cudaMemsetAsync(cd.counters, 0, 5 * sizeof(uint32_t), st));
    if (retry) launch_cnt_init(k, cd, st);
    launch_mesh_find(k, s, cd, st);
    launch_pair_find(k, s, cd, h->candCap, h->findShape, st);
    launch_pair_overflow(k, s, cd, h->candCap, st);
    TRY(check_launch(h, "contact search"));
    exclusive_scan_u32_onepass(cd.cnt, h->nS + 1, nb.off, nb.dN, h->scratch, h->dErr, st);
    if (hCnt) {
        CUDA_TRY(h, cudaMemcpyAsync(hCnt + 1, cd.counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        if (h->nT) CUDA_TRY(h, cudaMemcpyAsync(hCnt + 4, cd.counters + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(hCnt, nb.dN, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    }
    return DEME_OK;
}

// Writes the new list (n contacts, pool of `pool` pairs) in canonical order into lists[cur ^ 1], on `st`.  While a
// graph is recorded the counts are unknown: n and pool are the capacities, and the kernels read the counts on the
// device.
static int32_t cd_assemble(deme_handle* h, const StateView& s, uint32_t n, uint32_t pool, uint32_t meshPairs,
                           cudaStream_t st) {
    ContactBuf& nb = h->lists[h->cur ^ 1];
    if (!h->capturing) TRY(ensure_list(h, nb, n));
    launch_pair_scatter(h->k, h->cd, nb.view(), pool, nb.cap, h->candCap, st);
    launch_mesh_scatter(h->k, h->cd, nb.view(), meshPairs, nb.cap, st);
    launch_pair_assemble(h->k, s, h->cd, nb.view(), nb.cap, st);
    return check_launch(h, "contact assembly");
}

// History map of the new list against the list in use, remapped history, and the switch to the new list (on dT).
static int32_t cd_adopt(deme_handle* h, uint32_t n) {
    ContactBuf& nb = h->lists[h->cur ^ 1];
    ContactBuf& pb = h->lists[h->cur];
    launch_history(h->k, nb.view(), pb.view(), h->capturing ? nb.cap : n, h->capturing ? pb.cap : h->nContacts,
                   h->nW > 0, h->st_dt);
    TRY(check_launch(h, "contact history"));
    h->cur ^= 1;
    h->nContacts = n;
    h->outsValid = false;
    return DEME_OK;
}

// Synchronous detection on dT's stream from the current poses (DoStepDynamics with CD due this step).
static int32_t cd_sync(deme_handle* h) {
    cudaStream_t st = h->st_dt;
    StateView s = h->state_view();
    if (h->capturing) {
        // recorded into a graph: no host read; launches cover the capacities, kernels read the counts
        TRY(cd_search(h, s, h->analPlaced, st, false, nullptr));
        TRY(cd_assemble(h, s, h->lists[h->cur ^ 1].cap, h->candCap, h->cd.meshCap, st));
        return cd_adopt(h, h->lists[h->cur ^ 1].cap);
    }
    TRY(refresh_count(h));
    uint32_t n = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        TRY(cd_search(h, s, h->analPlaced, st, attempt > 0, h->hTotal));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        n = h->hTotal[0];
        if (search_fits(h, h->hTotal)) break;
        // the pair pool (or the mesh pool) outgrew its buffer: grow and search again
        TRY(grow_search(h, h->hTotal));
    }
    if (!search_fits(h, h->hTotal)) {
        h->err = "contact search: pair list still over capacity after growing";
        return DEME_ERR_OVERFLOW;
    }
    TRY(cd_assemble(h, s, n, h->hTotal[1], h->nT ? h->hTotal[4] : 0u, st));
    TRY(cd_adopt(h, n));
    return read_device_errors(h);
}

static int32_t ensure_async(deme_handle* h) {
    if (h->kVoxel) return DEME_OK;
    TRY(dalloc_n(h, &h->kVoxel, std::max(h->nO, 1u)));
    TRY(dalloc_n(h, &h->kLoc, std::max(h->nO, 1u)));
    TRY(dalloc_n(h, &h->kQuat, std::max(h->nO, 1u)));
    TRY(dalloc_n(h, &h->kAnalPlaced, std::max(h->nA, 1u)));
    if (h->nT) TRY(dalloc_n(h, &h->kTriPlaced, h->nT));
    CUDA_TRY(h, cudaMallocHost(&h->hCounts, 8 * sizeof(uint32_t)));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->evPose, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->evCounts, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->evListReady, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->evListReleased, cudaEventDisableTiming));
    // nothing has read a list yet: the first search may write lists[cur ^ 1] at once
    CUDA_TRY(h, cudaEventRecord(h->evListReleased, h->st_dt));
    return DEME_OK;
}

// kT's part of an asynchronous detection: snapshot of the poses dT has reached, then the search on st_kt.
static int32_t cd_start(deme_handle* h) {
    TRY(ensure_async(h));
    cudaStream_t kt = h->st_kt;
    CUDA_TRY(h, cudaEventRecord(h->evPose, h->st_dt));
    CUDA_TRY(h, cudaStreamWaitEvent(kt, h->evPose, 0));
    // lists[cur ^ 1] was last read by dT's history map at the previous adoption
    CUDA_TRY(h, cudaStreamWaitEvent(kt, h->evListReleased, 0));
    const size_t nO = h->nO;
    CUDA_TRY(h, cudaMemcpyAsync(h->kVoxel, h->voxel, nO * sizeof(uint64_t), cudaMemcpyDeviceToDevice, kt));
    CUDA_TRY(h, cudaMemcpyAsync(h->kLoc, h->loc, nO * sizeof(ushort4), cudaMemcpyDeviceToDevice, kt));
    CUDA_TRY(h, cudaMemcpyAsync(h->kQuat, h->quat, nO * sizeof(float4), cudaMemcpyDeviceToDevice, kt));
    TRY(cd_search(h, h->kt_view(), h->kAnalPlaced, kt, false, h->hCounts));
    CUDA_TRY(h, cudaEventRecord(h->evCounts, kt));
    h->cdPending = true;
    h->cdAdoptStep = h->steps + h->cdLag;
    return DEME_OK;
}

// dT adopts the list kT found: wait for kT's counts, assemble on kT, history map and switch on dT.
static int32_t cd_finish(deme_handle* h) {
    if (!h->cdPending) return DEME_OK;
    h->cdPending = false;
    cudaStream_t kt = h->st_kt;
    CUDA_TRY(h, cudaEventSynchronize(h->evCounts));
    const StateView ks = h->kt_view();
    if (!search_fits(h, h->hCounts)) {
        // pool overflow: grow and search the same snapshot again (it is untouched until the next detection)
        TRY(grow_search(h, h->hCounts));
        TRY(cd_search(h, ks, h->kAnalPlaced, kt, true, h->hCounts));
        CUDA_TRY(h, cudaStreamSynchronize(kt));
        if (!search_fits(h, h->hCounts)) {
            h->err = "contact search: pair list still over capacity after growing";
            return DEME_ERR_OVERFLOW;
        }
    }
    const uint32_t n = h->hCounts[0];
    TRY(cd_assemble(h, ks, n, h->hCounts[1], h->nT ? h->hCounts[4] : 0u, kt));
    CUDA_TRY(h, cudaEventRecord(h->evListReady, kt));
    CUDA_TRY(h, cudaStreamWaitEvent(h->st_dt, h->evListReady, 0));
    TRY(cd_adopt(h, n));
    CUDA_TRY(h, cudaEventRecord(h->evListReleased, h->st_dt));
    return DEME_OK;
}

// A pending asynchronous detection is dropped (its snapshot no longer describes the state).
static int32_t cd_cancel(deme_handle* h) {
    if (!h->cdPending) return DEME_OK;
    h->cdPending = false;
    CUDA_TRY(h, cudaStreamSynchronize(h->st_kt));
    return DEME_OK;
}

int32_t deme_set_async_cd(deme_handle* h, int32_t lag) {
    if (!h) return DEME_ERR_INVALID;
    const int32_t f = h->params.cd_update_freq;
    if (lag < 0 || (lag > 0 && f > 0 && lag > f) || (lag > 1 && f <= 0)) {
        h->err = "asynchronous detection lag must lie in [0, cd_update_freq] (0 or 1 with detection every step)";
        return DEME_ERR_INVALID;
    }
    TRY(cd_finish(h));
    h->cdLag = lag;
    return DEME_OK;
}

int32_t deme_detect_contacts(deme_handle* h) {
    if (!h) return DEME_ERR_INVALID;
    TRY(cd_finish(h));
    return cd_sync(h);
}

// ---------------------------------------------------------------------------------------------------- dT ----
int32_t deme_compute_forces(deme_handle* h) {
    if (!h) return DEME_ERR_INVALID;
    cudaStream_t st = h->st_dt;
    const SimConsts& k = h->k;
    StateView s = h->state_view();
    if (!h->analFresh) {
        launch_place_anal(k, s, h->analRaw, h->analPlaced, h->nA, st);
        launch_place_tri(k, s, h->triRaw, st);
    }
    h->analFresh = false;
    // prepareForceArrays (src/kernel/DEMPrepForceKernels.cu:23-31): accumulators start from zero every step
    CUDA_TRY(h, cudaMemsetAsync(h->acc, 0, h->nO * sizeof(float4), st));
    CUDA_TRY(h, cudaMemsetAsync(h->alpha, 0, h->nO * sizeof(float4), st));
    const ContactBuf& c = h->lists[h->cur];
    // while a graph is recorded the count is unknown: the launch covers the list's capacity
    if (!h->capturing) TRY(refresh_count(h));
    const uint32_t nL = h->capturing ? c.cap : h->nContacts;
    const ContactOutputs* out = nullptr;
    if (h->keepOutputs) {
        if (!h->capturing) TRY(ensure_outputs(h, nL));
        out = &h->outs;
    }
    AnalAccum aa{nullptr, nullptr, h->nClumps, h->nO - h->nClumps, h->nO - h->nClumps > 64};
    if (aa.nAO && !aa.direct) {
        if (!h->analChunks) {
            if (h->capturing) {
                h->err = "graph recording: wall partial sums not allocated";
                return DEME_ERR_STATE;
            }
            TRY(dalloc_n(h, &h->analChunks, (size_t)6u * aa.nAO * kAnalChunks));
        }
        aa.chunks = h->analChunks;
        const size_t need = (size_t)force_blocks(std::max(nL, 1u)) * 6u * aa.nAO;
        if (need > h->analPartialCap && h->capturing) {
            h->err = "graph recording: wall partials not sized for the list capacity";
            return DEME_ERR_STATE;
        }
        if (need > h->analPartialCap) {
            dfree(h, h->analPartial);
            h->analPartial = nullptr;
            h->analPartialCap = 0;
            TRY(dalloc_n(h, &h->analPartial, need + need / 4 + 64));
            h->analPartialCap = need + need / 4 + 64;
        }
        aa.partial = h->analPartial;
    }
    launch_force(k, s, c.view(), nL, h->nW > 0, out, aa, h->userForce.lib ? &h->userForce : nullptr, h->forceShape,
                 st);
    TRY(check_launch(h, "force"));
    h->outsValid = out != nullptr;
    return DEME_OK;
}

// The time as the reference's dT advances it: a float plus the step, once per step.
static void advance_host_time(deme_handle* h) {
    h->t += (double)h->k.h;
    h->tf = h->tf + h->k.h;
}

// Family-change rules and prescribed-motion expressions read the time from the device.
static bool needs_device_time(const deme_handle* h) { return h->famRules.kern || h->motion.kern; }

int32_t deme_integrate(deme_handle* h) {
    if (!h) return DEME_ERR_INVALID;
    h->analFresh = false;  // the poses move
    cudaStream_t st = h->st_dt;
    if (h->motion.kern) {
        SimConsts k = h->k;
        StateView s = h->state_view();
        const float* t = h->dTime;
        void* args[] = {&k, &s, &t};
        if (h->nO) {
            ProfScope prof_(KID_INTEGRATE, st);
            CUDA_TRY(h, cudaLaunchKernel((const void*)h->motion.kern, dim3((h->nO + 255) / 256), dim3(256), args, 0,
                                         st));  // ProfScope counts the launch
        }
    } else {
        launch_integrate(h->k, h->state_view(), h->integrateThreads, st);
    }
    if (needs_device_time(h)) launch_advance_time(h->dTime, h->k.h, h->dErr, st);
    TRY(check_launch(h, "integrate"));
    advance_host_time(h);
    h->steps++;
    return DEME_OK;
}

// ChangeFamilyWhen rules between the forces and the integration of a step (routineChecks, src/DEM/dT.cpp:1434-1444),
// then the device time advances with the step.
static int32_t apply_family_rules(deme_handle* h) {
    if (!h->famRules.kern) return DEME_OK;
    SimConsts k = h->k;
    StateView s = h->state_view();
    const float* t = h->dTime;
    void* args[] = {&k, &s, &t};
    CUDA_TRY(h, cudaLaunchKernel((const void*)h->famRules.kern, dim3((h->nO + 255) / 256), dim3(256), args, 0,
                                 h->st_dt));
    add_launches(1);
    return DEME_OK;
}

// One step launched function by function (DoStepDynamics).
static int32_t step_plain(deme_handle* h) {
    const int f = h->params.cd_update_freq;
    const bool due = f <= 0 || (h->steps % f) == 0;
    if (h->cdLag > 0) {
        // kT/dT on two streams: adopt what kT found cdLag steps ago, then hand kT the poses of this step.  The
        // first detection of a run is adopted at once, so no step runs without a contact list.
        if (h->cdPending && h->steps >= h->cdAdoptStep) TRY(cd_finish(h));
        if (due) {
            TRY(cd_finish(h));
            TRY(cd_start(h));
            if (h->steps == 0 || !h->everDetected) TRY(cd_finish(h));
            h->everDetected = true;
        }
    } else if (due) {
        TRY(cd_sync(h));
        h->everDetected = true;
    }
    TRY(deme_compute_forces(h));
    TRY(apply_family_rules(h));
    TRY(deme_integrate(h));
    return DEME_OK;
}

// ------------------------------------------------------------------------------------------ graph replay ----
// With deme_set_graph, a window of cd_update_freq steps (a detection, then forces and integration each step) is
// recorded once into a CUDA graph and replayed.  Nothing in a window reads the device from the host: the launches
// cover the lists' capacities and the kernels read the counts the scans left on the device.  The capacities are
// fixed before recording with headroom; a window whose lists or pair pool outgrow them sets the device error word.
// From then on every force, history and integration kernel of the batch returns at once, so the state stays that
// of the last completed window (each window ends by counting itself done when the error word is clear), and the
// host redoes the remaining steps one by one, which grows the buffers.

static std::vector<uint8_t> graph_key(const deme_handle* h) {
    std::vector<uint8_t> key;
    auto put = [&](const void* p, size_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        key.insert(key.end(), b, b + n);
    };
    put(&h->k, sizeof(h->k));
    for (int b = 0; b < 2; b++) {
        const ContactView v = h->lists[b].view();
        put(&v, sizeof(v));
        put(&h->lists[b].cap, sizeof(uint32_t));
    }
    put(&h->cd, sizeof(h->cd));
    put(&h->candCap, sizeof(h->candCap));
    put(&h->st_dt, sizeof(h->st_dt));
    put(&h->keepOutputs, sizeof(h->keepOutputs));
    put(&h->outs, sizeof(h->outs));
    put(&h->analPartial, sizeof(h->analPartial));
    put(&h->analPartialCap, sizeof(h->analPartialCap));
    put(&h->analPlaced, sizeof(h->analPlaced));
    put(&h->scratch, sizeof(h->scratch));
    put(&h->useOnesweep, sizeof(h->useOnesweep));
    put(&h->nW, sizeof(h->nW));
    const void* lib = h->userForce.lib;
    put(&lib, sizeof(lib));
    const void* rules = h->famRules.lib;
    put(&rules, sizeof(rules));
    const void* motion = h->motion.lib;
    put(&motion, sizeof(motion));
    put(&h->jitGeneration, sizeof(h->jitGeneration));  // a new image may load where a released one was
    put(&h->params.cd_update_freq, sizeof(h->params.cd_update_freq));
    put(&h->findShape, sizeof(h->findShape));
    put(&h->cellFactor, sizeof(h->cellFactor));
    put(&h->nCells, sizeof(h->nCells));  // recorded as the cell scan's length (deme_change_clump_sizes changes it)
    put(&h->cellBits, sizeof(h->cellBits));
    put(&h->forceShape, sizeof(h->forceShape));
    put(&h->exactThreads, sizeof(h->exactThreads));
    put(&h->integrateThreads, sizeof(h->integrateThreads));
    return key;
}

// Capacities a window needs, fixed before recording: both lists and the pair pool at 1.25 times the current count
// plus 4,096 (twice the sphere count before the first detection), per-contact outputs and wall partials for the
// list capacity.  A window that outgrows them is redone step by step, which grows them.
static int32_t graph_prepare(deme_handle* h) {
    TRY(refresh_count(h));
    const uint32_t n = h->nContacts;
    const uint64_t want64 = std::max<uint64_t>((uint64_t)n + n / 4 + 4096u, h->everDetected ? 0ull : 2ull * h->nS);
    const uint32_t want = (uint32_t)std::min<uint64_t>(want64, 0xF0000000ull);
    TRY(ensure_list_keep(h, h->lists[h->cur], want, n, h->st_dt));
    TRY(ensure_list(h, h->lists[h->cur ^ 1], want));
    TRY(ensure_cand(h, std::max<uint32_t>(want, h->hTotal[1] + h->hTotal[1] / 4 + 4096u)));
    if (!h->dWindows) {
        TRY(dalloc_n(h, &h->dWindows, 1));
        CUDA_TRY(h, cudaMallocHost(&h->hWindows, 2 * sizeof(uint32_t)));
    }
    const uint32_t cap = std::max(h->lists[0].cap, h->lists[1].cap);
    if (h->keepOutputs) TRY(ensure_outputs(h, cap));
    const uint32_t nAO = h->nO - h->nClumps;
    if (nAO && nAO <= 64) {
        const size_t need = (size_t)force_blocks(cap) * 6u * nAO;
        if (need > h->analPartialCap) {
            dfree(h, h->analPartial);
            h->analPartial = nullptr;
            h->analPartialCap = 0;
            TRY(dalloc_n(h, &h->analPartial, need + need / 4 + 64));
            h->analPartialCap = need + need / 4 + 64;
        }
        if (!h->analChunks) TRY(dalloc_n(h, &h->analChunks, (size_t)6u * nAO * kAnalChunks));
    }
    return DEME_OK;
}

static int32_t graph_capture(deme_handle* h, int p) {
    const int f = std::max(1, h->params.cd_update_freq);
    // the host's bookkeeping is put back after recording: the replays do the work
    const int cur0 = h->cur;
    const uint32_t n0 = h->nContacts;
    const int64_t steps0 = h->steps;
    const double t0 = h->t;
    const float tf0 = h->tf;
    const bool outs0 = h->outsValid, stale0 = h->countStale;
    CUDA_TRY(h, cudaStreamBeginCapture(h->st_dt, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    const int64_t launches0 = launch_count();
    int32_t st = DEME_OK;
    for (int i = 0; i < f && st == DEME_OK; i++) {
        if (i == 0) st = cd_sync(h);
        if (st == DEME_OK) st = deme_compute_forces(h);
        if (st == DEME_OK) st = apply_family_rules(h);
        if (st == DEME_OK) st = deme_integrate(h);
    }
    if (st == DEME_OK) launch_window_done(h->dErr, h->dWindows, h->st_dt);
    h->capturing = false;
    // recording counted its launches once; the replays add them back each time they run
    const int64_t recorded = launch_count() - launches0;
    add_launches(-recorded);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->st_dt, &g);
    h->cur = cur0;
    h->nContacts = n0;
    h->steps = steps0;
    h->t = t0;
    h->tf = tf0;
    h->outsValid = outs0;
    h->countStale = stale0;
    if (st != DEME_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (st == DEME_OK) h->err = std::string("graph recording: ") + cudaGetErrorString(e);
        return st != DEME_OK ? st : DEME_ERR_CUDA;
    }
    if (h->graphExec[p]) {
        cudaGraphExecDestroy(h->graphExec[p]);
        h->graphExec[p] = nullptr;
    }
    const cudaError_t ei = cudaGraphInstantiate(&h->graphExec[p], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        h->graphExec[p] = nullptr;
        h->err = std::string("graph instantiation: ") + cudaGetErrorString(ei);
        return DEME_ERR_CUDA;
    }
    h->graphKey[p] = graph_key(h);
    h->graphKernels[p] = recorded;
    return DEME_OK;
}

static int32_t step_graph(deme_handle* h, int32_t n_steps) {
    const int f = std::max(1, h->params.cd_update_freq);
    while (n_steps > 0 && h->steps % f != 0) {
        TRY(step_plain(h));
        n_steps--;
    }
    const int32_t windows = n_steps / f;
    if (windows > 0) {
        TRY(graph_prepare(h));
        const int cur0 = h->cur;
        const int64_t steps0 = h->steps;
        const double t0 = h->t;
        const float tf0 = h->tf;
        CUDA_TRY(h, cudaMemsetAsync(h->dWindows, 0, sizeof(uint32_t), h->st_dt));
        for (int32_t w = 0; w < windows; w++) {
            const int p = h->cur;
            if (!h->graphExec[p] || h->graphKey[p] != graph_key(h)) TRY(graph_capture(h, p));
            CUDA_TRY(h, cudaGraphLaunch(h->graphExec[p], h->st_dt));
            add_launches(h->graphKernels[p]);
            h->cur ^= 1;
            h->steps += f;
            for (int i = 0; i < f; i++) advance_host_time(h);  // as deme_integrate adds it, step by step
            h->countStale = true;
            h->outsValid = h->keepOutputs;
            h->everDetected = true;
            h->graphReplays++;
        }
        CUDA_TRY(h, cudaMemcpyAsync(h->hWindows, h->dWindows, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st_dt));
        CUDA_TRY(h, cudaMemcpyAsync(h->hWindows + 1, h->dErr, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st_dt));
        // the count of the list in use comes back with them, so the next call needs no read of its own
        CUDA_TRY(h, cudaMemcpyAsync(h->hTotal + 3, h->lists[h->cur].dN, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                    h->st_dt));
        CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
        if (!h->hWindows[1]) {
            h->nContacts = h->hTotal[3];
            h->countStale = false;
        }
        if (h->hWindows[1]) {
            // a list or the pair pool outgrew its capacity in window `done`: the state and the list in use are those
            // its detection started from; redo the rest step by step
            const int32_t done = (int32_t)h->hWindows[0];
            CUDA_TRY(h, cudaMemset(h->dErr, 0, 4 * sizeof(uint32_t)));
            h->cur = cur0 ^ (done & 1);
            h->steps = steps0 + (int64_t)done * f;
            h->t = t0;
            h->tf = tf0;
            for (int32_t i = 0; i < done * f; i++) advance_host_time(h);
            if (needs_device_time(h)) launch_set_time(h->dTime, h->tf, h->st_dt);
            h->outsValid = false;
            h->graphRollbacks++;
            for (int32_t i = 0; i < (windows - done) * f; i++) TRY(step_plain(h));
        }
        n_steps -= windows * f;
    }
    while (n_steps-- > 0) TRY(step_plain(h));
    return DEME_OK;
}

int32_t deme_set_graph(deme_handle* h, int32_t enable) {
    if (!h) return DEME_ERR_INVALID;
    TRY(cd_finish(h));
    h->useGraph = enable != 0;
    return DEME_OK;
}

int32_t deme_graph_stats(deme_handle* h, int64_t* replays, int64_t* rollbacks) {
    if (!h) return DEME_ERR_INVALID;
    if (replays) *replays = h->graphReplays;
    if (rollbacks) *rollbacks = h->graphRollbacks;
    return DEME_OK;
}

// ------------------------------------------------------------------------------------------ family changes ----
// The device copy of the time, allocated with the first rule or expression and started from the host's.
static int32_t ensure_device_time(deme_handle* h, bool needed) {
    if (!needed || h->dTime) return DEME_OK;
    TRY(dalloc_n(h, &h->dTime, 1));
    launch_set_time(h->dTime, h->tf, h->st_dt);
    return check_launch(h, "set_time");
}

int32_t deme_set_family_change_rules(deme_handle* h, int32_t n, const uint32_t* from, const uint32_t* to,
                                     const char* const* conditions) {
    if (!h || n < 0) return DEME_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(cd_finish(h));
    TRY(ensure_device_time(h, n > 0));
    std::string err;
    const int32_t rc = compile_family_change_rules(n, from, to, conditions, h->famRules, err);
    if (rc != DEME_OK) h->err = err;
    else h->jitGeneration++;
    return rc;
}

int32_t deme_set_prescribed_motion(deme_handle* h, int32_t n, const deme_motion_expressions* m) {
    if (!h || n < 0 || (n > 0 && !m)) return DEME_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(cd_finish(h));
    TRY(ensure_device_time(h, n > 0));
    std::string err;
    const int32_t rc = compile_prescribed_motion(n, m, h->motion, err);
    if (rc != DEME_OK) h->err = err;
    else h->jitGeneration++;
    return rc;
}

int32_t deme_change_family(deme_handle* h, uint32_t from, uint32_t to) {
    if (!h) return DEME_ERR_INVALID;
    if (from > 255u || to > 255u) {
        h->err = "family numbers lie in [0, 255]";
        return DEME_ERR_INVALID;
    }
    TRY(cd_finish(h));
    launch_change_family(h->loc, h->nO, from, to, h->st_dt);
    return check_launch(h, "change_family");
}

int32_t deme_set_family_contact(deme_handle* h, uint32_t a, uint32_t b, int32_t prevent) {
    if (!h) return DEME_ERR_INVALID;
    if (a > 255u || b > 255u) {
        h->err = "family numbers lie in [0, 255]";
        return DEME_ERR_INVALID;
    }
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    const uint32_t index = (1u + hi) * hi / 2u + lo;  // the device's mask_index
    if (index >= DEME_NUM_FAMILY_MASK) {
        h->err = "family mask entry out of range";
        return DEME_ERR_INVALID;
    }
    TRY(cd_finish(h));
    launch_set_mask(h->masks, index, prevent ? 1u : 0u, h->st_dt);
    return check_launch(h, "set_family_contact");
}

int32_t deme_change_clump_sizes(deme_handle* h, uint32_t n, const uint32_t* owners, const float* factors) {
    if (!h || (n && (!owners || !factors))) return DEME_ERR_INVALID;
    if (h->ownerScene) {
        h->err = "change_clump_sizes: not with packed scenes";
        return DEME_ERR_INVALID;
    }
    std::vector<float> fac(h->nClumps, 1.f);
    std::vector<uint8_t> mark(h->nClumps, 0);
    for (uint32_t i = 0; i < n; i++) {
        if (owners[i] >= h->nClumps || !(factors[i] > 0.f)) {
            h->err = "change_clump_sizes: owner is not a clump, or factor not positive";
            return DEME_ERR_INVALID;
        }
        mark[owners[i]] = 1;
        fac[owners[i]] = factors[i];  // a clump listed twice takes its last factor
    }
    TRY(cd_finish(h));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    const uint32_t nS = h->nS;
    std::vector<float4> sph(nS);
    std::vector<uint32_t> own(nS);
    if (nS) {
        CUDA_TRY(h, cudaMemcpy(sph.data(), h->sph, nS * sizeof(float4), cudaMemcpyDeviceToHost));
        CUDA_TRY(h, cudaMemcpy(own.data(), h->sOwner, nS * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    // the components' relative positions and radii times the factor, in float (dTModifyComponents,
    // src/kernel/DEMMiscKernels.cu:18-33); masses and moments stay
    float rmax = 0.f;
    for (uint32_t i = 0; i < nS; i++) {
        float4& q = sph[i];
        if (own[i] < h->nClumps && mark[own[i]]) {
            const float f = fac[own[i]];
            q.x *= f;
            q.y *= f;
            q.z *= f;
            q.w *= f;
        }
        float r = q.w;
        r += h->params.beta;
        rmax = std::max(rmax, r);
    }
    if (nS) CUDA_TRY(h, cudaMemcpy(h->sph, sph.data(), nS * sizeof(float4), cudaMemcpyHostToDevice));
    // the search grid follows the largest expanded radius; its arrays grow if the finest grid has more cells now
    h->k.r_max_cd = rmax;
    radius_bounds(h->k, nS, rmax);
    h->sceneRmax.assign(1, rmax);
    const float factor = h->cellFactor;
    TRY(set_cell_grid(h, 1.0));
    if (h->nCells > h->cellCap) {
        dfree(h, h->cd.cellCount);
        dfree(h, h->cd.cellStart);
        h->cd.cellCount = h->cd.cellStart = nullptr;
        TRY(dalloc_n(h, &h->cd.cellCount, (size_t)h->nCells + 1));
        TRY(dalloc_n(h, &h->cd.cellStart, (size_t)h->nCells + 1));
        TRY(ensure_scratch(h, std::max(scan_scratch_bytes(h->nCells + 1), scan_onepass_scratch_bytes(h->nCells + 1))));
        h->cellCap = h->nCells;
    }
    TRY(set_cell_grid(h, factor));
    h->outsValid = false;
    return DEME_OK;
}

// ------------------------------------------------------------------------------------------- search shape ----
int32_t deme_set_search_shape(deme_handle* h, int32_t shape, float cell_factor) {
    if (!h) return DEME_ERR_INVALID;
    if (shape < 0 || shape >= find_shape_count() || !(cell_factor >= 1.f) || cell_factor > 4.f) {
        h->err = "search shape out of range (shape index in [0, deme_search_shape_count), cell factor in [1, 4])";
        return DEME_ERR_INVALID;
    }
    TRY(cd_finish(h));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    h->findShape = shape;
    return set_cell_grid(h, cell_factor);
}

int32_t deme_search_shape_count(void) { return find_shape_count(); }

int32_t deme_force_shape_count(void) { return force_shape_count(); }

int32_t deme_set_kernel_shapes(deme_handle* h, int32_t force_shape, int32_t exact_threads, int32_t integrate_threads) {
    if (!h) return DEME_ERR_INVALID;
    auto ok_threads = [](int32_t t) { return t >= 32 && t <= 512 && t % 32 == 0; };
    if (force_shape < 0 || force_shape >= force_shape_count() || !ok_threads(exact_threads) ||
        !ok_threads(integrate_threads)) {
        h->err = "kernel shapes out of range (force shape < deme_force_shape_count(), threads 32..512 in steps of 32)";
        return DEME_ERR_INVALID;
    }
    TRY(cd_finish(h));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    h->forceShape = force_shape;
    h->exactThreads = (uint32_t)exact_threads;
    h->integrateThreads = (uint32_t)integrate_threads;
    return DEME_OK;
}

// Times every (candidate-scan shape, cell factor) pair on a few steps from the same state, keeps the fastest and
// puts the state back.  Every pair gives the same contact lists, so only the time differs.
int32_t deme_autotune(deme_handle* h, int32_t steps_per_trial, deme_tuning* out) {
    if (!h) return DEME_ERR_INVALID;
    const int32_t steps = steps_per_trial > 0 ? steps_per_trial : 5;
    TRY(cd_finish(h));
    Checkpoint ck;
    TRY(save_checkpoint(h, ck));
    const int cur0 = h->cur;
    const bool graph0 = h->useGraph;
    h->useGraph = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(h, cudaEventCreate(&e0));
    CUDA_TRY(h, cudaEventCreate(&e1));
    int trials = 0;
    int32_t st = DEME_OK;
    // one trial: the current shapes on `steps` steps from the checkpoint (after one untimed step that settles the
    // buffer sizes for them)
    auto trial = [&](float& ms) -> int32_t {
        h->cur = cur0;
        TRY(restore_checkpoint(h, ck));
        TRY(step_plain(h));
        cudaEventRecord(e0, h->st_dt);
        for (int32_t i = 0; i < steps; i++) TRY(step_plain(h));
        cudaEventRecord(e1, h->st_dt);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)steps;
        trials++;
        return DEME_OK;
    };
    // A shape replaces the one kept so far only when it is at least 1 % faster: trials of a few steps spread by
    // about that much, and the defaults win ties.
    constexpr float kMargin = 0.99f;
    // 1. candidate-scan shape x cell factor, with the default shapes of the other kernels
    const float factors[] = {1.f, 1.25f, 1.5f};
    h->forceShape = 0;
    h->exactThreads = h->integrateThreads = 256;
    float best = 3.4e38f, dflt = 0.f;
    int bestShape = 0;
    float bestFactor = 1.f;
    for (int v = 0; v < find_shape_count() && st == DEME_OK; v++) {
        for (float f : factors) {
            h->findShape = v;
            if ((st = set_cell_grid(h, f)) != DEME_OK) break;
            float ms = 0.f;
            if ((st = trial(ms)) != DEME_OK) break;
            if (v == 0 && f == 1.f) dflt = ms;
            if (ms < best * kMargin || (v == 0 && f == 1.f)) {
                best = ms;
                bestShape = v;
                bestFactor = f;
            }
        }
    }
    if (st == DEME_OK) {
        h->findShape = bestShape;
        st = set_cell_grid(h, bestFactor);
    }
    // 2. force shape, 3. threads of the exact test, 4. threads of the integration, one after the other
    int bestForce = 0;
    for (int v = 1; v < force_shape_count() && st == DEME_OK; v++) {
        h->forceShape = v;
        float ms = 0.f;
        if ((st = trial(ms)) != DEME_OK) break;
        if (ms < best * kMargin) {
            best = ms;
            bestForce = v;
        }
    }
    h->forceShape = bestForce;
    const uint32_t threads[] = {128, 512};
    for (uint32_t* knob : {&h->integrateThreads}) {
        const uint32_t keep = *knob;
        uint32_t pick = keep;
        for (uint32_t t : threads) {
            if (st != DEME_OK) break;
            *knob = t;
            float ms = 0.f;
            if ((st = trial(ms)) != DEME_OK) break;
            if (ms < best * kMargin) {
                best = ms;
                pick = t;
            }
        }
        *knob = pick;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->cur = cur0;
    const int32_t rs = restore_checkpoint(h, ck);
    free_checkpoint(h, ck);
    h->useGraph = graph0;
    if (st != DEME_OK) return st;
    TRY(rs);
    if (out) {
        uint32_t w = 0, slots = 0;
        bool persistent = false;
        find_shape(bestShape, &w, &slots, &persistent);
        out->shape = bestShape;
        out->find_warps = (int32_t)w;
        out->find_slots = (int32_t)slots;
        out->find_persistent = persistent ? 1 : 0;
        out->cell_factor = bestFactor;
        out->ms_per_step = best;
        out->ms_per_step_default = dflt;
        out->trials = trials;
        out->force_shape = h->forceShape;
        out->force_threads = (int32_t)force_shape_threads(h->forceShape);
        out->exact_threads = (int32_t)h->exactThreads;
        out->integrate_threads = (int32_t)h->integrateThreads;
    }
    return DEME_OK;
}

int32_t deme_step(deme_handle* h, int32_t n_steps) {
    if (!h) return DEME_ERR_INVALID;
    // rules and expressions read the time on the device: start it from the host's (a kernel argument, so no
    // staging buffer is read after this call returns)
    if (needs_device_time(h)) launch_set_time(h->dTime, h->tf, h->st_dt);
    // (scenes with mesh facets step without graphs: their cell lists may need to grow inside a window)
    if (h->useGraph && h->cdLag == 0 && h->nT == 0 && !prof_timing()) {
        TRY(step_graph(h, n_steps));
    } else {
        for (int32_t i = 0; i < n_steps; i++) TRY(step_plain(h));
    }
    return check_launch(h, "step");
}

int32_t deme_sync(deme_handle* h) {
    if (!h) return DEME_ERR_INVALID;
    TRY(cd_finish(h));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_kt));
    return read_device_errors(h);
}

// ---------------------------------------------------------------------------------------------- transfer ----
// Owners [first, first + count) between the device arrays and a deme_state whose arrays hold `count` entries (any
// array may be NULL).  An upload reads the packed records back first, so fields the caller leaves NULL keep their
// device values.
static int32_t transfer_state(deme_handle* h, uint32_t first, uint32_t count, deme_state* o, const deme_state* in) {
    if ((uint64_t)first + count > h->nO) {
        h->err = "owner range [" + std::to_string(first) + ", " + std::to_string((uint64_t)first + count) +
                 ") beyond the " + std::to_string(h->nO) + " owners";
        return DEME_ERR_INVALID;
    }
    if (in) {
        TRY(cd_cancel(h));
        h->analFresh = false;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    const uint32_t n = count;
    if (n == 0) return DEME_OK;
    std::vector<ushort4> loc(n);
    std::vector<float4> q(n), v(n), w(n), a(n), al(n);
    CUDA_TRY(h, cudaMemcpy(loc.data(), h->loc + first, n * sizeof(ushort4), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(q.data(), h->quat + first, n * sizeof(float4), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(v.data(), h->vel + first, n * sizeof(float4), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(w.data(), h->omg + first, n * sizeof(float4), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(a.data(), h->acc + first, n * sizeof(float4), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(al.data(), h->alpha + first, n * sizeof(float4), cudaMemcpyDeviceToHost));
    if (o) {
        if (o->voxel)
            CUDA_TRY(h, cudaMemcpy(o->voxel, h->voxel + first, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++) {
            if (o->locX) o->locX[i] = loc[i].x;
            if (o->locY) o->locY[i] = loc[i].y;
            if (o->locZ) o->locZ[i] = loc[i].z;
            if (o->family) o->family[i] = (uint8_t)loc[i].w;
            if (o->oriQw) o->oriQw[i] = q[i].x;
            if (o->oriQx) o->oriQx[i] = q[i].y;
            if (o->oriQy) o->oriQy[i] = q[i].z;
            if (o->oriQz) o->oriQz[i] = q[i].w;
            if (o->vX) o->vX[i] = v[i].x;
            if (o->vY) o->vY[i] = v[i].y;
            if (o->vZ) o->vZ[i] = v[i].z;
            if (o->omgX) o->omgX[i] = w[i].x;
            if (o->omgY) o->omgY[i] = w[i].y;
            if (o->omgZ) o->omgZ[i] = w[i].z;
            if (o->aX) o->aX[i] = a[i].x;
            if (o->aY) o->aY[i] = a[i].y;
            if (o->aZ) o->aZ[i] = a[i].z;
            if (o->alphaX) o->alphaX[i] = al[i].x;
            if (o->alphaY) o->alphaY[i] = al[i].y;
            if (o->alphaZ) o->alphaZ[i] = al[i].z;
        }
        return DEME_OK;
    }
    const deme_state* s = in;
    for (uint32_t i = 0; i < n; i++) {
        if (s->locX) loc[i].x = s->locX[i];
        if (s->locY) loc[i].y = s->locY[i];
        if (s->locZ) loc[i].z = s->locZ[i];
        if (s->family) loc[i].w = s->family[i];
        if (s->oriQw) q[i].x = s->oriQw[i];
        if (s->oriQx) q[i].y = s->oriQx[i];
        if (s->oriQy) q[i].z = s->oriQy[i];
        if (s->oriQz) q[i].w = s->oriQz[i];
        if (s->vX) v[i].x = s->vX[i];
        if (s->vY) v[i].y = s->vY[i];
        if (s->vZ) v[i].z = s->vZ[i];
        if (s->omgX) w[i].x = s->omgX[i];
        if (s->omgY) w[i].y = s->omgY[i];
        if (s->omgZ) w[i].z = s->omgZ[i];
        if (s->aX) a[i].x = s->aX[i];
        if (s->aY) a[i].y = s->aY[i];
        if (s->aZ) a[i].z = s->aZ[i];
        if (s->alphaX) al[i].x = s->alphaX[i];
        if (s->alphaY) al[i].y = s->alphaY[i];
        if (s->alphaZ) al[i].z = s->alphaZ[i];
    }
    if (s->voxel) CUDA_TRY(h, cudaMemcpy(h->voxel + first, s->voxel, n * sizeof(uint64_t), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->loc + first, loc.data(), n * sizeof(ushort4), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->quat + first, q.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->vel + first, v.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->omg + first, w.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->acc + first, a.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->alpha + first, al.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    return DEME_OK;
}

int32_t deme_download_state(deme_handle* h, deme_state* o) {
    if (!h || !o) return DEME_ERR_INVALID;
    return transfer_state(h, 0, h->nO, o, nullptr);
}

int32_t deme_upload_state(deme_handle* h, const deme_state* s) {
    if (!h || !s) return DEME_ERR_INVALID;
    return transfer_state(h, 0, h->nO, nullptr, s);
}

int32_t deme_download_state_range(deme_handle* h, uint32_t first, uint32_t count, deme_state* o) {
    if (!h || !o) return DEME_ERR_INVALID;
    return transfer_state(h, first, count, o, nullptr);
}

int32_t deme_upload_state_range(deme_handle* h, uint32_t first, uint32_t count, const deme_state* s) {
    if (!h || !s) return DEME_ERR_INVALID;
    return transfer_state(h, first, count, nullptr, s);
}

int32_t deme_get_num_contacts(deme_handle* h, uint32_t* n) {
    if (!h || !n) return DEME_ERR_INVALID;
    TRY(refresh_count(h));
    *n = h->nContacts;
    return DEME_OK;
}

int32_t deme_download_contacts(deme_handle* h, deme_contacts* o) {
    if (!h || !o) return DEME_ERR_INVALID;
    TRY(refresh_count(h));
    const uint32_t n = h->nContacts;
    o->n_contacts = n;
    if (o->capacity < n) return DEME_ERR_OVERFLOW;
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    const ContactBuf& c = h->lists[h->cur];
    if (n == 0) return DEME_OK;
    if (o->idA) CUDA_TRY(h, cudaMemcpy(o->idA, c.idA, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (o->idB) CUDA_TRY(h, cudaMemcpy(o->idB, c.idB, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (o->type) CUDA_TRY(h, cudaMemcpy(o->type, c.type, n, cudaMemcpyDeviceToHost));
    if (o->mapping) CUDA_TRY(h, cudaMemcpy(o->mapping, c.mapping, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (o->wildcards && h->nW > 0) {
        std::vector<float4> hw(n);
        CUDA_TRY(h, cudaMemcpy(hw.data(), c.hist, n * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++) {
            o->wildcards[i] = hw[i].x;
            o->wildcards[(size_t)o->capacity + i] = hw[i].y;
            o->wildcards[2 * (size_t)o->capacity + i] = hw[i].z;
            o->wildcards[3 * (size_t)o->capacity + i] = hw[i].w;
        }
    }
    return DEME_OK;
}

int32_t deme_upload_contacts(deme_handle* h, const deme_contacts* in) {
    if (!h || !in) return DEME_ERR_INVALID;
    TRY(cd_cancel(h));
    const uint32_t n = in->n_contacts;
    for (uint32_t i = 0; i < n; i++) {
        const uint8_t t = in->type[i];
        const uint32_t limB = t == DEME_SPHERE_SPHERE_CONTACT ? h->nS : (t == DEME_SPHERE_MESH_CONTACT ? h->nT : h->nA);
        if (t == DEME_NOT_A_CONTACT || t > DEME_SPHERE_CONE_CONTACT) {
            h->err = "contact type out of range";
            return DEME_ERR_INVALID;
        }
        if (in->idA[i] >= h->nS || in->idB[i] >= limB) {
            h->err = "contact ids out of range";
            return DEME_ERR_INVALID;
        }
    }
    // canonical order: (idA, group, idB), groups sphere--analytical, sphere--mesh, sphere--sphere
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) {
        const uint32_t ga = contact_group(in->type[a]), gb = contact_group(in->type[b]);
        if (in->idA[a] != in->idA[b]) return in->idA[a] < in->idA[b];
        if (ga != gb) return ga < gb;
        return in->idB[a] < in->idB[b];
    });
    std::vector<uint32_t> A(n), B(n), off(h->nS + 1, 0);
    std::vector<uint8_t> T(n);
    std::vector<float4> hw(n, make_float4(0.f, 0.f, 0.f, 0.f));
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t j = perm[i];
        A[i] = in->idA[j];
        B[i] = in->idB[j];
        T[i] = in->type[j];
        if (in->wildcards && h->nW > 0)
            hw[i] = make_float4(in->wildcards[j], in->wildcards[(size_t)in->capacity + j],
                                in->wildcards[2 * (size_t)in->capacity + j], in->wildcards[3 * (size_t)in->capacity + j]);
        off[A[i] + 1]++;
    }
    for (uint32_t s = 0; s < h->nS; s++) off[s + 1] += off[s];
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    ContactBuf& c = h->lists[h->cur];
    TRY(ensure_list(h, c, n));
    if (n) {
        CUDA_TRY(h, cudaMemcpy(c.idA, A.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(c.idB, B.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(c.type, T.data(), n, cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(c.hist, hw.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
        std::vector<uint32_t> nul(n, DEME_NULL_MAPPING_PARTNER);
        CUDA_TRY(h, cudaMemcpy(c.mapping, nul.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    CUDA_TRY(h, cudaMemcpy(c.off, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(c.dN, &n, sizeof(uint32_t), cudaMemcpyHostToDevice));
    h->nContacts = n;
    h->countStale = false;
    h->outsValid = false;
    return DEME_OK;
}

int32_t deme_download_contact_forces(deme_handle* h, deme_contact_forces* o) {
    if (!h || !o) return DEME_ERR_INVALID;
    TRY(refresh_count(h));
    const uint32_t n = h->nContacts;
    o->n_contacts = n;
    if (o->capacity < n) return DEME_ERR_OVERFLOW;
    if (!h->outsValid) {
        h->err = "per-contact forces were not kept: call deme_keep_contact_forces(h, 1) before deme_compute_forces";
        return DEME_ERR_STATE;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    std::vector<float4> tmp(n);
    float* dst[4] = {o->force, o->torque_only_force, o->cpA, o->cpB};
    float4* src[4] = {h->outs.F, h->outs.TOF, h->outs.CPA, h->outs.CPB};
    for (int a = 0; a < 4; a++) {
        if (!dst[a] || n == 0) continue;
        CUDA_TRY(h, cudaMemcpy(tmp.data(), src[a], n * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++) {
            dst[a][3 * (size_t)i] = tmp[i].x;
            dst[a][3 * (size_t)i + 1] = tmp[i].y;
            dst[a][3 * (size_t)i + 2] = tmp[i].z;
        }
    }
    return DEME_OK;
}

int32_t deme_set_family_prescription(deme_handle* h, int32_t family, const deme_family_prescription* src) {
    if (!h || !src || family < 0 || family >= DEME_NUM_FAMILIES) return DEME_ERR_INVALID;
    if (!h->hPresc) {
        // the events first: the ring counts as set up (hPresc non-null) only once every slot has its event
        for (cudaEvent_t& e : h->prescDone)
            if (!e) CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        Prescription* ring = nullptr;
        CUDA_TRY(h, cudaMallocHost(&ring, deme_handle::kPrescSlots * sizeof(Prescription)));
        h->hPresc = ring;
    }
    // a ring of staging slots: only a slot whose earlier copy has not run yet is waited for
    const int slot = h->prescNext;
    h->prescNext = (slot + 1) % deme_handle::kPrescSlots;
    CUDA_TRY(h, cudaEventSynchronize(h->prescDone[slot]));
    Prescription& q = h->hPresc[slot];
    q = Prescription{};
    q.used = src->used;
    q.lin_vel = src->lin_vel_prescribed;
    q.rot_vel = src->rot_vel_prescribed;
    q.lin_pos = src->lin_pos_prescribed;
    q.rot_pos = src->rot_pos_prescribed;
    for (int c = 0; c < 3; c++) {
        q.has_vel[c] = src->has_vel[c];
        q.has_omg[c] = src->has_omg[c];
        q.has_pos[c] = src->has_pos[c];
        q.vel[c] = src->vel[c];
        q.omg[c] = src->omg[c];
        q.pos[c] = src->pos[c];
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->presc + family, &q, sizeof(Prescription), cudaMemcpyHostToDevice, h->st_dt));
    CUDA_TRY(h, cudaEventRecord(h->prescDone[slot], h->st_dt));
    return DEME_OK;
}

int32_t deme_set_time_step(deme_handle* h, float h_step) {
    if (!h || !(h_step > 0.f)) return DEME_ERR_INVALID;
    h->params.h = h_step;
    h->k.h = h_step;
    return DEME_OK;
}

int32_t deme_get_time(deme_handle* h, double* t, int64_t* steps) {
    if (!h) return DEME_ERR_INVALID;
    if (t) *t = h->t;
    if (steps) *steps = h->steps;
    return DEME_OK;
}

int32_t deme_set_time(deme_handle* h, double t, float t_float, int64_t steps) {
    if (!h || steps < 0) return DEME_ERR_INVALID;
    TRY(cd_finish(h));
    h->t = t;
    h->tf = t_float;
    h->steps = steps;
    if (h->dTime) launch_set_time(h->dTime, h->tf, h->st_dt);
    return check_launch(h, "set_time");
}

int32_t deme_get_time_float(deme_handle* h, float* t_float) {
    if (!h || !t_float) return DEME_ERR_INVALID;
    *t_float = h->tf;
    return DEME_OK;
}

int32_t deme_kinetic_energy(deme_handle* h, double* ke) {
    if (!h || !ke) return DEME_ERR_INVALID;
    launch_kinetic_energy(h->k, h->state_view(), h->nClumps, h->dKE, h->st_dt);
    CUDA_TRY(h, cudaMemcpyAsync(h->hKE, h->dKE, sizeof(double), cudaMemcpyDeviceToHost, h->st_dt));
    CUDA_TRY(h, cudaStreamSynchronize(h->st_dt));
    *ke = *h->hKE;
    return DEME_OK;
}

int32_t deme_kinetic_energy_enqueue(deme_handle* h, int64_t* ticket) {
    if (!h || !ticket) return DEME_ERR_INVALID;
    if (!h->hKERing) {
        // the events first: the ring counts as set up (hKERing non-null) only once every slot has its event
        for (cudaEvent_t& e : h->keDone)
            if (!e) CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        if (!h->dKERing) TRY(dalloc_n(h, &h->dKERing, deme_handle::kKESlots));
        double* ring = nullptr;
        CUDA_TRY(h, cudaMallocHost(&ring, deme_handle::kKESlots * sizeof(double)));
        h->hKERing = ring;
    }
    const int64_t t = h->keTickets++;
    const int slot = (int)(t % deme_handle::kKESlots);
    // the slot's previous result has landed in host memory before it is reused
    CUDA_TRY(h, cudaEventSynchronize(h->keDone[slot]));
    launch_kinetic_energy(h->k, h->state_view(), h->nClumps, h->dKERing + slot, h->st_dt);
    CUDA_TRY(h, cudaMemcpyAsync(h->hKERing + slot, h->dKERing + slot, sizeof(double), cudaMemcpyDeviceToHost,
                                h->st_dt));
    CUDA_TRY(h, cudaEventRecord(h->keDone[slot], h->st_dt));
    h->keSlotTicket[slot] = t;
    *ticket = t;
    return DEME_OK;
}

int32_t deme_kinetic_energy_collect(deme_handle* h, int64_t ticket, double* ke) {
    if (!h || !ke || ticket < 0) return DEME_ERR_INVALID;
    const int slot = (int)(ticket % deme_handle::kKESlots);
    if (!h->hKERing || h->keSlotTicket[slot] != ticket) {
        h->err = "deme_kinetic_energy_collect: unknown ticket, or its slot was reused by a later enqueue";
        return DEME_ERR_STATE;
    }
    CUDA_TRY(h, cudaEventSynchronize(h->keDone[slot]));
    *ke = h->hKERing[slot];
    return DEME_OK;
}

int32_t deme_bin_assignment(deme_handle* h, uint16_t* n_bins, uint8_t* n_anal, uint32_t pair_capacity,
                            uint32_t* bin_ids, uint32_t* sphere_ids, uint32_t* n_pairs) {
    if (!h) return DEME_ERR_INVALID;
    cudaStream_t st = h->st_dt;
    const uint32_t nS = h->nS;
    StateView s = h->state_view();
    launch_place_anal(h->k, s, h->analRaw, h->analPlaced, h->nA, st);
    uint16_t* dNb = nullptr;
    uint8_t* dNa = nullptr;
    uint32_t* dOff = nullptr;
    TRY(dalloc_n(h, &dNb, nS + 1));
    TRY(dalloc_n(h, &dNa, nS + 1));
    TRY(dalloc_n(h, &dOff, nS + 1));
    int32_t rc = DEME_OK;
    do {
        launch_bin_count(h->k, s, dNb, dNa, st);
        exclusive_scan_u16(dNb, nS, dOff, h->dTotal, h->scratch, st);
        if (cudaMemcpyAsync(h->hTotal, h->dTotal, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            h->err = "bin assignment count failed";
            rc = DEME_ERR_CUDA;
            break;
        }
        const uint32_t P = nS ? *h->hTotal : 0;
        if (n_pairs) *n_pairs = P;
        if (n_bins && nS) cudaMemcpy(n_bins, dNb, nS * sizeof(uint16_t), cudaMemcpyDeviceToHost);
        if (n_anal && nS) cudaMemcpy(n_anal, dNa, nS, cudaMemcpyDeviceToHost);
        if (!bin_ids || !sphere_ids) break;
        if (pair_capacity < P) {
            rc = DEME_ERR_OVERFLOW;
            break;
        }
        uint32_t *kb = nullptr, *vb = nullptr, *ko = nullptr, *vo = nullptr;
        void* sc = nullptr;
        if ((rc = dalloc_n(h, &kb, P + 1)) || (rc = dalloc_n(h, &vb, P + 1)) || (rc = dalloc_n(h, &ko, P + 1)) ||
            (rc = dalloc_n(h, &vo, P + 1)) || (rc = dalloc(h, &sc, radix_sort_scratch_bytes(P))))
            break;
        launch_bin_emit(h->k, s, dOff, kb, vb, st);
        int bits = 1;
        const uint64_t nb = (uint64_t)h->k.nbX * h->k.nbY * h->k.nbZ;
        while (bits < 32 && (1ull << bits) < nb) bits++;
        radix_sort_pairs(kb, vb, ko, vo, P, bits, sc, h->dErr, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            h->err = "bin assignment sort failed";
            rc = DEME_ERR_CUDA;
        } else if (P) {
            cudaMemcpy(bin_ids, ko, P * sizeof(uint32_t), cudaMemcpyDeviceToHost);
            cudaMemcpy(sphere_ids, vo, P * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        }
        dfree(h, kb);
        dfree(h, vb);
        dfree(h, ko);
        dfree(h, vo);
        dfree(h, sc);
    } while (0);
    dfree(h, dNb);
    dfree(h, dNa);
    dfree(h, dOff);
    if (rc != DEME_OK) return rc;
    return read_device_errors(h);
}

int32_t deme_radix_sort_pairs_device(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, int32_t key_bits, void* scratch,
                                     size_t scratch_bytes, void* stream) {
    if (scratch_bytes < radix_sort_scratch_bytes(n) + 16) return DEME_ERR_INVALID;
    // the error word lives at the end of the caller's scratch
    uint32_t* err = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(scratch) + radix_sort_scratch_bytes(n));
    cudaStream_t st = (cudaStream_t)stream;
    cudaMemsetAsync(err, 0, sizeof(uint32_t), st);
    radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, key_bits, scratch, err, st);
    return cudaGetLastError() == cudaSuccess ? DEME_OK : DEME_ERR_CUDA;
}

size_t deme_radix_sort_scratch_bytes(uint32_t n) { return radix_sort_scratch_bytes(n) + 16; }

}  // extern "C"
