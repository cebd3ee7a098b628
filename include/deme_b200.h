/*
 * deme_b200.h -- C ABI of the B200-native DEM-Engine hot path.
 *
 * The reference solver (DEM-Engine, `deme::DEMSolver`, src/DEM/API.h:44-887) has no C ABI: its kernels are
 * reachable only through the C++ class and its two worker threads (kT: contact detection, dT: dynamics).
 * This header is the drop-in boundary for that per-step path.  Each entry point names the reference
 * interface it replaces.  The C++ `deme::DEMSolver` facade in dem-engine-sbel_b200/csrc/solver/ is
 * written on top of these calls and keeps the reference's method names.
 *
 * Conventions
 *   - plain C structs of host pointers plus counts; caller-owned host buffers, solver-owned device buffers;
 *   - every entry point returns a deme_status; nothing throws and no kernel traps;
 *   - one handle per host thread (not re-entrant);
 *   - ID widths and array layouts follow src/DEM/VariableTypes.h:11-49 and src/DEM/Defines.h:154-383.
 */
#ifndef DEME_B200_H
#define DEME_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEME_B200_ABI_VERSION 5

/* Status codes (the reference throws std::runtime_error instead: src/DEM/Structs.h:129-141, src/core/utils/GpuError.h:13-27). */
typedef enum {
    DEME_OK = 0,
    DEME_ERR_INVALID = 1,     /* bad argument or inconsistent scene */
    DEME_ERR_CUDA = 2,        /* CUDA runtime error; the handle should be destroyed */
    DEME_ERR_OOM = 3,         /* device allocation failed */
    DEME_ERR_OVERFLOW = 4,    /* a device-side capacity check failed (reported, never trapped) */
    DEME_ERR_NVRTC = 5,       /* the user force model did not compile */
    DEME_ERR_TIMEOUT = 6,     /* a bounded device wait gave up */
    DEME_ERR_STATE = 7,       /* call made in the wrong lifecycle state */
    DEME_ERR_NO_DEVICE = 8,   /* no CUDA device is visible */
    DEME_ERR_TOO_LARGE = 9    /* input larger than a fixed capacity (nothing was launched) */
} deme_status;

/* Contact types (src/DEM/Defines.h:63-67).  Cylinder and cone are additions of this build; sphere--mesh contacts
 * are detected here (the reference declares the type but detects none). */
#define DEME_NOT_A_CONTACT 0
#define DEME_SPHERE_SPHERE_CONTACT 1
#define DEME_SPHERE_MESH_CONTACT 2
#define DEME_SPHERE_PLANE_CONTACT 3
#define DEME_SPHERE_PLATE_CONTACT 4
#define DEME_SPHERE_CYLINDER_CONTACT 5
#define DEME_SPHERE_CONE_CONTACT 6

/* Analytical component types (src/DEM/Defines.h:60-61, plus the two new shapes). */
#define DEME_ANAL_PLANE 0
#define DEME_ANAL_PLATE 1
#define DEME_ANAL_CYLINDER 2
#define DEME_ANAL_CONE 3

/* Integrators (src/DEM/Defines.h:106, TIME_INTEGRATOR). */
#define DEME_INTEGRATOR_FORWARD_EULER 0
#define DEME_INTEGRATOR_CENTERED_DIFFERENCE 1
#define DEME_INTEGRATOR_EXTENDED_TAYLOR 2

/* NULL_MAPPING_PARTNER (src/DEM/Defines.h:80-81).  The reference's expression `(1 << 31) + (1 << 31 - 1)` parses as
 * (1 << 31) + (1 << 30) because `-` binds tighter than `<<`, so its value is 0xC0000000, kept here bit for bit. */
#define DEME_NULL_MAPPING_PARTNER 0xC0000000u
/* Family-mask table size.  The reference sizes it (255*256)/2 = 32640 (src/DEM/APIPrivate.cpp:588) but indexes up to
 * 32895 for family 255 (src/kernel/DEMHelperKernels.cu:51-56); this build stores 32896 entries, tail = allow. */
#define DEME_NUM_FAMILY_MASK 32896
#define DEME_NUM_FAMILIES 256
#define DEME_RESERVED_FAMILY 255
#define DEME_MAX_WILDCARDS 8

/* Simulation parameters: the fields of deme::DEMSimParams (src/DEM/Defines.h:154-211) plus the two JIT literals.
 * `l_kernel` and `voxel_size_kernel` are the values the reference's kernels see: it substitutes `_l_` and
 * `_voxelSize_` as std::fixed 17-decimal text (src/DEM/APIPrivate.cpp:1358-1359, src/DEM/HostSideHelpers.hpp:396-401),
 * while host-side initial encoding uses the exact doubles `l` and `voxel_size` (src/DEM/dT.cpp:572-575). */
typedef struct {
    uint8_t nvXp2, nvYp2, nvZp2, pad0;
    uint32_t nbX, nbY, nbZ;
    double l;
    double voxel_size;
    double l_kernel;
    double voxel_size_kernel;
    double bin_size;
    float lbf[3];
    float G[3];
    float h;          /* time step (float, as DEMSimParams::h) */
    float beta;       /* contact-detection expand factor (DEMSimParams::beta) */
    int32_t integrator;
    int32_t cd_update_freq;  /* 0: contact detection every step (src/DEM/API.h:82, SetCDUpdateFreq) */
    int32_t n_contact_wildcards; /* 4 for the built-in Hertz-Mindlin model, 0 for frictionless */
    int32_t pad1;
    float domain[3];  /* user-instructed domain size (InstructBoxDomainDimension); bounds the contact search grid */
    float pad2;
} deme_sim_params;

/* Per-family prescription.  The reference jitifies these as C expression strings
 * (src/DEM/APIPrivate.cpp:1005-1048); this struct carries the constant-valued form.  `has_*` marks the
 * components the user prescribed ("none" in the reference leaves a component free). */
typedef struct {
    uint8_t used;
    uint8_t lin_vel_prescribed;
    uint8_t rot_vel_prescribed;
    uint8_t lin_pos_prescribed;
    uint8_t rot_pos_prescribed;
    uint8_t has_vel[3];
    uint8_t has_omg[3];
    uint8_t has_pos[3];
    uint8_t pad[4];
    float vel[3];
    float omg[3];
    double pos[3];
} deme_family_prescription;

/* Scene: the flattened arrays dT/kT receive at Initialize (src/DEM/dT.cpp:480-640), as host pointers. */
typedef struct {
    uint32_t n_owners;
    uint32_t n_spheres;
    uint32_t n_anal;
    uint32_t n_materials;
    /* owners (clumps first, then analytical owners: src/DEM/dT.cpp:622-640) */
    const uint64_t* voxel;
    const uint16_t* locX;
    const uint16_t* locY;
    const uint16_t* locZ;
    const float* oriQw;
    const float* oriQx;
    const float* oriQy;
    const float* oriQz;
    const float* vX;
    const float* vY;
    const float* vZ;
    const float* omgX;
    const float* omgY;
    const float* omgZ;
    const uint8_t* family;
    const float* mass;
    const float* mmiXX;
    const float* mmiYY;
    const float* mmiZZ;
    /* spheres (flattened clump components: ClumpCompAcqStratAllFlatten.cu) */
    const uint32_t* sphere_owner;
    const float* relX;
    const float* relY;
    const float* relZ;
    const float* radius;
    const uint8_t* sphere_material;
    /* analytical components (AnalyticalCompDefJitify.cu) */
    const uint8_t* anal_type;
    const uint32_t* anal_owner;
    const uint8_t* anal_normal;
    const uint8_t* anal_material;
    const float* anal_relX;
    const float* anal_relY;
    const float* anal_relZ;
    const float* anal_rotX;
    const float* anal_rotY;
    const float* anal_rotZ;
    const float* anal_size1;
    const float* anal_size2;
    const float* anal_size3;
    const float* anal_mass;
    /* materials (keys E, nu, CoR, mu, Crr: src/DEM/AuxClasses.cpp:222) */
    const float* mat_E;
    const float* mat_nu;
    const float* mat_CoR;
    const float* mat_mu;
    const float* mat_Crr;
    /* families */
    const uint8_t* family_masks;                        /* DEME_NUM_FAMILY_MASK entries, 1 = prevent contact */
    const deme_family_prescription* prescriptions;      /* DEME_NUM_FAMILIES entries */
    /* Extensions for many independent scenes packed into one (no reference counterpart); NULL = unused. */
    const uint16_t* sphere_material_wide;  /* per sphere, replaces sphere_material (up to 65536 materials) */
    const uint16_t* anal_material_wide;    /* per component, replaces anal_material */
    const uint32_t* owner_anal_first;      /* per owner: its spheres meet only the analytical components */
    const uint32_t* owner_anal_count;      /*   [first, first + count) (then n_anal may exceed 255) */
    const uint32_t* owner_scene;           /* per owner: the scene it belongs to (0 .. n_scenes - 1); each scene gets
                                              a search grid of its own, sized by its own spheres */
    const float* scene_box;                /* n_scenes x 6: lower and upper corner of each scene's search grid,
                                              relative to the domain's lower corner (NULL: from the initial poses) */
    /* Mesh facets (triangles) of mesh-represented owners: DEMMeshConnected (src/DEM/BdrsAndObjs.h:173-300), kT's
     * ownerMesh and relPosNode1..3 (src/DEM/kT.cpp:603-625).  Mesh owners follow the clump owners, like the
     * analytical owners.  The reference declares the sphere--mesh contact type (src/DEM/Defines.h:66) but detects no
     * such contact; here every facet a sphere touches is one DEME_SPHERE_MESH_CONTACT with idB = the facet id.
     * 0 / NULL: no meshes.  Not with the packed-scene extensions above. */
    uint32_t n_tris;
    const uint32_t* tri_owner;    /* per facet: its owner (n_clumps <= owner < n_owners) */
    const float* tri_node1;       /* n_tris x 3 (x, y, z interleaved): the nodes in the owner frame */
    const float* tri_node2;
    const float* tri_node3;
    const uint16_t* tri_material; /* per facet */
} deme_scene;

/* Mutable owner state (download/upload).  Any pointer may be NULL to skip that array. */
typedef struct {
    uint64_t* voxel;
    uint16_t* locX;
    uint16_t* locY;
    uint16_t* locZ;
    float* oriQw;
    float* oriQx;
    float* oriQy;
    float* oriQz;
    float* vX;
    float* vY;
    float* vZ;
    float* omgX;
    float* omgY;
    float* omgZ;
    float* aX;
    float* aY;
    float* aZ;
    float* alphaX;
    float* alphaY;
    float* alphaZ;
    uint8_t* family;
} deme_state;

/* Contact list (kT product, src/DEM/Defines.h:242-245).  Order: sorted by idA; inside one idA, sphere--analytical
 * contacts first (ascending component id), then sphere--mesh contacts (ascending facet id), then sphere--sphere
 * contacts (ascending idB).  The reference sorts by idA
 * only, so its in-segment order is a permutation of this one. */
typedef struct {
    uint32_t capacity;       /* elements available in each caller array (in) */
    uint32_t n_contacts;     /* contacts in the list (out) */
    uint32_t* idA;
    uint32_t* idB;
    uint8_t* type;
    uint32_t* mapping;       /* index into the previous list, or DEME_NULL_MAPPING_PARTNER */
    float* wildcards;        /* n_contact_wildcards x capacity, row-major by wildcard (may be NULL) */
} deme_contacts;

/* Per-contact dT outputs (contactForces, contactTorque_convToForce, contactPointGeometryA/B in DEMDataDT). */
typedef struct {
    uint32_t capacity;
    uint32_t n_contacts;
    float* force;            /* 3 x n, interleaved xyz */
    float* torque_only_force;
    float* cpA;
    float* cpB;
} deme_contact_forces;

typedef struct deme_handle deme_handle;

/* The entry points (the run-time compiler of force models reads this header for its types only). */
#ifndef __CUDACC_RTC__

/* Version and error text. */
int32_t deme_abi_version(void);
const char* deme_status_string(int32_t status);

/* Create a solver on the current CUDA device and upload the scene.
 * Replaces DEMSolver::Initialize -> allocateGPUArrays/initializeGPUArrays (src/DEM/APIPublic.cpp:659-693,
 * src/DEM/APIPrivate.cpp:760-818). */
int32_t deme_create(const deme_sim_params* params, const deme_scene* scene, deme_handle** out);
void deme_destroy(deme_handle* h);
/* Last error message of this handle (static storage, valid until the next call on it). */
const char* deme_get_error(deme_handle* h);

/* Force model.  src == NULL selects the built-in frictional Hertz-Mindlin model (FullHertzianForceModel.cu);
 * otherwise `src` is a user force-model snippet compiled with NVRTC into the force-kernel template, with the
 * given per-contact wildcard names (DefineContactForceModel, src/DEM/APIPublic.cpp:116-121;
 * DEMForceModel::SetPerContactWildcards, src/DEM/AuxClasses.cpp:256-266).
 * In scope, with the reference's names: force, torque_only_force (outputs), B2A, overlapDepth, contactPnt,
 * AOwnerPos, BOwnerPos, bodyAPos, ARadius, BRadius, AOwnerMass, BOwnerMass, AoriQw..AoriQz, BoriQw..BoriQz,
 * locCPA, locCPB, bodyAMatType, bodyBMatType, the material arrays E, nu, CoR, mu, Crr, ts, ALinVel, BLinVel,
 * ARotVel, BRotVel, AOwnerFamily, BOwnerFamily, myContactType, myContactID, and each wildcard as a float; helpers
 * float3 arithmetic, dot, cross, length, normalize, applyOriQToVector3, matProxy2ContactParam, deme:: constants.
 * At most 4 wildcards (DEME_ERR_INVALID beyond).  A string that does not compile returns DEME_ERR_NVRTC and
 * deme_get_error holds the compiler log (lines of the string are reported as "force_model_string"). */
int32_t deme_set_force_model(deme_handle* h, const char* src, const char* const* wildcard_names, int32_t n_wildcards);

/* Contact detection on the current state (kT: contactDetection, src/algorithms/DEMCubContactDetection.cu:39-397),
 * including the history map against the previous list and the wildcard remap
 * (dT::migratePersistentContacts, src/DEM/dT.cpp:1258-1347). */
int32_t deme_detect_contacts(deme_handle* h);
/* Forces and their collection onto owners for the current contact list (dT::calculateForces,
 * src/DEM/dT.cpp:1349-1422, collectContactForces, src/algorithms/DEMCubForceCollection.cu:20-158). */
int32_t deme_compute_forces(deme_handle* h);
/* Owner integration (integrateOwners, src/kernel/DEMIntegrationKernels.cu:170-179). */
int32_t deme_integrate(deme_handle* h);
/* n full steps (contact detection every cd_update_freq steps, forces, integration), as DoDynamics
 * (src/DEM/APIPublic.cpp:871-892) driven by DoStepDynamics. */
int32_t deme_step(deme_handle* h, int32_t n_steps);
/* Block until all work of this handle is done. */
int32_t deme_sync(deme_handle* h);

/* State and contact transfer (GetOwner* / SetOwner*, src/DEM/API.h:196-214; WriteContactFile, API.h:324). */
int32_t deme_download_state(deme_handle* h, deme_state* out);
int32_t deme_upload_state(deme_handle* h, const deme_state* in);
/* The same for owners [first, first + count) only; the arrays of the struct hold `count` entries.  An upload
 * leaves the fields whose arrays are NULL as they were.  This is what one owner's GetOwner* / SetOwner* costs in
 * the reference (dT::getOwnerPos / setOwnerPos and their siblings, src/DEM/dT.cpp:1705-1810). */
int32_t deme_download_state_range(deme_handle* h, uint32_t first, uint32_t count, deme_state* out);
int32_t deme_upload_state_range(deme_handle* h, uint32_t first, uint32_t count, const deme_state* in);
int32_t deme_get_num_contacts(deme_handle* h, uint32_t* n);
int32_t deme_download_contacts(deme_handle* h, deme_contacts* out);
/* Replace the current contact list and its wildcards (history); mapping is ignored.  Used to inject identical
 * kT products into dT for parity checks.  The list may come in any order (it is put in the canonical order);
 * idB must be below the count of its kind (spheres, analytical components or mesh facets) and the type one of
 * the contact types above, else DEME_ERR_INVALID. */
int32_t deme_upload_contacts(deme_handle* h, const deme_contacts* in);
int32_t deme_download_contact_forces(deme_handle* h, deme_contact_forces* out);
/* Keep the per-contact force, torque-only force and local contact points of the next deme_compute_forces calls so
 * deme_download_contact_forces can return them (the fused hot path does not store them by default). */
int32_t deme_keep_contact_forces(deme_handle* h, int32_t enable);
/* How contact detection orders spheres by search cell: 0 (default) a one-pass counting sort (a radix sort whose single
 * digit spans the cell range), 1 the multi-pass onesweep radix sort.  Both give the same contact list. */
int32_t deme_set_cell_sort(deme_handle* h, int32_t onesweep);

/* Streams: kT (contact detection) and dT (dynamics) work queues; NULL restores the handle's own streams.
 * The two workers of the reference are host threads with one stream each (src/core/utils/GpuManager.cpp:8-32). */
int32_t deme_set_streams(deme_handle* h, void* kT_stream, void* dT_stream);

/* kT and dT as concurrent producer and consumer (the reference's asynchronous kT/dT threads with drift limit
 * cd_update_freq, src/DEM/dT.cpp:1446-1586, src/DEM/kT.cpp:101-188, src/core/utils/ThreadManager.h:37-94), made
 * deterministic.  With lag > 0, a detection due at step k runs on the kT stream from a snapshot of the owner poses of
 * step k while dT keeps stepping with the current list; dT adopts the new list at step k + lag (history remapped from
 * the list it replaces).  dT therefore uses lists up to lag + cd_update_freq - 1 steps old, which the expand factor
 * (SetExpandFactor / SetMaxVelocity) must cover, as in the reference.  lag lies in [0, cd_update_freq] (0 or 1 when
 * detection runs every step); 0 (the default) detects synchronously.  The first detection of a run is adopted at
 * once.  Uploading state or contacts drops a pending detection; deme_detect_contacts and deme_sync adopt it first. */
int32_t deme_set_async_cd(deme_handle* h, int32_t lag);

/* Family changes.  deme_change_family moves every owner of family `from` to family `to` now (ChangeFamily,
 * src/DEM/APIPublic.cpp:184-208).  deme_set_family_change_rules compiles n rules with NVRTC (ChangeFamilyWhen,
 * src/DEM/APIPublic.cpp:167-182, applied by applyFamilyChanges, src/kernel/DEMModeratorKernels.cu:9-38): at every
 * step, after the forces and before the integration, an owner of family from[i] moves to to[i] when conditions[i]
 * returns true.  A condition is a code block that ends with `return <bool>;` and may use pos (double3, the owner's
 * position from the domain's lower corner), vel, acc (float3), mass, family_code, t (time) and h (step), with the
 * float3 helpers force models have.  Rules test the family the owner had at the start of the step; when several
 * apply, the last one wins.  n = 0 removes the rules.  A rule that does not compile returns DEME_ERR_NVRTC with the
 * log. */
int32_t deme_change_family(deme_handle* h, uint32_t from, uint32_t to);
/* Contact between families a and b (either order) on a created solver: prevent = 1 disables it, 0 enables it
 * (DisableContactBetweenFamilies / EnableContactBetweenFamilies on an initialized DEMSolver, src/DEM/APIPublic.cpp:
 * 431-468, which write the workers' family-mask tables directly).  Ordered on the dynamics stream; the next contact
 * detection uses it. */
int32_t deme_set_family_contact(deme_handle* h, uint32_t a, uint32_t b, int32_t prevent);
/* ChangeClumpSizes (src/DEM/APIPublic.cpp:844-862; dTModifyComponents / kTModifyComponents,
 * src/kernel/DEMMiscKernels.cu:18-52): the component spheres of each listed clump owner get their relative positions
 * and radii multiplied by its factor (float products; a clump listed twice takes its last factor); masses and
 * moments of inertia stay.  The search grid follows the new largest radius.  Contacts are found anew at the next
 * detection.  Not with packed scenes. */
int32_t deme_change_clump_sizes(deme_handle* h, uint32_t n, const uint32_t* owners, const float* factors);
int32_t deme_set_family_change_rules(deme_handle* h, int32_t n, const uint32_t* from, const uint32_t* to,
                                     const char* const* conditions);

/* Whole steps as CUDA graphs (no reference counterpart: its host code launches and synchronises kernel by kernel,
 * src/DEM/dT.cpp:1446-1586).  With enable != 0, deme_step records a window of cd_update_freq steps (one detection,
 * then forces and integration each step) into a CUDA graph once and replays it; nothing in a window waits for the
 * host.  Launches cover the contact lists' capacities, sized before recording at 1.25 times the current count
 * plus 4,096 (twice the sphere count before the first detection), and the kernels read the counts on the device.  A window in which a list or the
 * pair pool outgrows its capacity sets the device error word, after which every force, history and integration
 * kernel of the batch returns at once; the host then redoes the remaining steps one by one from the state of the
 * last completed window, so results do not depend on the mode.  Steps before the next detection step, and those left after the last whole
 * window, run step by step.  A graph is recorded again whenever anything it captured changes (buffers, streams,
 * time step, force model, stored outputs).  Not used with deme_set_async_cd lag > 0 or while per-kernel timing
 * (deme_kernel_timing) is on.  Helps small scenes, whose steps are bound by launch latency. */
int32_t deme_set_graph(deme_handle* h, int32_t enable);
/* Windows replayed from graphs and batches rolled back, since the handle was created. */
int32_t deme_graph_stats(deme_handle* h, int64_t* replays, int64_t* rollbacks);

/* Search shape (no reference counterpart: the reference's bin size, SetInitBinSize, sets both its bins and its
 * work per thread).  `shape` picks a block shape of the candidate scan (index < deme_search_shape_count();
 * 0, the default, is 4 warps with 16 survivor slots per lane; the last two take their tiles of spheres from a work
 * queue, with a few persistent blocks per SM) and `cell_factor` in [1, 4] scales the search cells (edge
 * cell_factor x max(bin size, the scene's largest expanded diameter)).  Every shape finds the same contacts. */
int32_t deme_set_search_shape(deme_handle* h, int32_t shape, float cell_factor);
int32_t deme_search_shape_count(void);
/* Block shapes of the other per-step kernels (no reference counterpart): `force_shape` < deme_force_shape_count()
 * (0, the default: 128 threads, 8 blocks per SM; 1: 256 x 4; 2: 64 x 16), and the threads per block of the
 * integration (32 to 512, multiples of 32; 256 by default).  `exact_threads` is checked and kept but no longer used:
 * the exact pair test runs inside the candidate scan.  They change speed only. */
int32_t deme_set_kernel_shapes(deme_handle* h, int32_t force_shape, int32_t exact_threads, int32_t integrate_threads);
int32_t deme_force_shape_count(void);

typedef struct {
    int32_t shape;         /* index passed to deme_set_search_shape */
    int32_t find_warps;    /* warps per block of the candidate scan */
    int32_t find_slots;    /* survivor slots per lane */
    float cell_factor;
    float ms_per_step;     /* the chosen shapes' time per step in the trials */
    float ms_per_step_default;
    int32_t trials;
    int32_t find_persistent;    /* the candidate scan takes its tiles from a work queue */
    int32_t force_shape;        /* arguments of deme_set_kernel_shapes */
    int32_t force_threads;
    int32_t exact_threads;
    int32_t integrate_threads;
} deme_tuning;

/* Autotuner: times every search shape with cell factors 1, 1.25 and 1.5, then (with the best of those) every force
 * shape, then 128, 256 and 512 threads per block for the integration, each trial on
 * `steps_per_trial` steps (5 when <= 0) from the current state; keeps the fastest, and restores the state and
 * contact history, so the run continues as if it had not been called.  `out` may be NULL. */
int32_t deme_autotune(deme_handle* h, int32_t steps_per_trial, deme_tuning* out);

/* Change one family's prescription between steps (the constant-valued form of SetFamilyPrescribedLinVel /
 * SetFamilyPrescribedAngVel / SetFamilyFixed, src/DEM/APIPublic.cpp:145-252, which the reference can only change by
 * re-jitifying).  The value is staged through pinned memory and applied in stream order. */
int32_t deme_set_family_prescription(deme_handle* h, int32_t family, const deme_family_prescription* p);

/* A family's prescribed motion written as C expressions: SetFamilyPrescribedLinVel / SetFamilyPrescribedAngVel /
 * SetFamilyPrescribedPosition with strings that are not constants (src/DEM/APIPublic.cpp:210-273).  Each non-NULL
 * string is pasted into the integration kernel as `vX = <string>;` (lin_vel), `omgBarX = <string>;` (ang_vel) or
 * `X = <string>;` (lin_pos, measured from the domain's lower corner), the way equipFamilyPrescribedMotions pastes
 * them (src/DEM/APIPrivate.cpp:1005-1048).  An expression sees t (float: the time at the start of the step,
 * accumulated in float as the reference's dT accumulates it), family, the components it prescribes and deme::PI.
 * NULL leaves a component free (the reference's "none"). */
typedef struct {
    int32_t family;
    uint8_t lin_vel_prescribed; /* the family's linear velocity is dictated, not integrated */
    uint8_t rot_vel_prescribed;
    uint8_t lin_pos_prescribed;
    uint8_t rot_pos_prescribed;
    const char* lin_vel[3];
    const char* ang_vel[3];
    const char* lin_pos[3];
} deme_motion_expressions;

/* Compiles the prescribed motions of n families (each at most once) with NVRTC into the integration kernel; from
 * the next step those families follow their expressions instead of their constant table entries.  n = 0 returns
 * every family to its table entry.  A set that does not compile returns DEME_ERR_NVRTC with the compiler's log in
 * deme_get_error and leaves the previous set in place. */
int32_t deme_set_prescribed_motion(deme_handle* h, int32_t n, const deme_motion_expressions* m);

/* Instrumentation.  deme_launch_count: kernels launched by this library in this process.  deme_kernel_timing(1)
 * brackets every launch with CUDA events on its stream; deme_kernel_times sums them per kernel name.  (The reference
 * keeps host wall-clock timers per phase instead: src/DEM/kT.h:179-181, src/DEM/dT.h:253-255.) */
int64_t deme_launch_count(void);
int32_t deme_kernel_timing(int32_t enable);
int32_t deme_kernel_times(int32_t cap, const char** names, double* total_ms, int64_t* launches, int32_t* n_out);

/* Change the time step between steps (SetInitTimeStep followed by UpdateSimParams, src/DEM/API.h:61, 399). */
int32_t deme_set_time_step(deme_handle* h, float h_step);

/* Simulation time advanced so far and step counter. */
int32_t deme_get_time(deme_handle* h, double* t, int64_t* steps);
/* The time as the reference's dT keeps it (timeElapsed, a float advanced by h every step, src/DEM/dT.h:216): what
 * prescribed-motion expressions and family-change rules see. */
int32_t deme_get_time_float(deme_handle* h, float* t_float);
/* Sets the time (double and the reference's float), and the step counter that schedules contact detection.  Used to
 * carry a run over into a new handle (UpdateClumps, src/DEM/APIPublic.cpp:792-843, keeps the simulation time). */
int32_t deme_set_time(deme_handle* h, double t, float t_float, int64_t steps);
/* Sum of 0.5 m v^2 + 0.5 I omega^2 over clump owners (DEMOwnerQueryKernels.cu:10-37 computes the per-owner term;
 * the reference's GetTotalKineticEnergy returns 0, src/DEM/dT.cpp:154-171). */
int32_t deme_kinetic_energy(deme_handle* h, double* ke);
/* The same sum without waiting for it (no reference counterpart): _enqueue launches it on the handle's stream after
 * the work queued so far, copies the result to pinned host memory and returns a ticket; _collect waits for that
 * copy and returns the value.  Up to 4 results can be outstanding: a fifth enqueue reuses the oldest slot, and
 * collecting a ticket whose slot was reused returns DEME_ERR_STATE.  A caller that steps and reads the energy every
 * step can so collect step k's value after queueing step k + 1, keeping the GPU busy while it reads. */
int32_t deme_kinetic_energy_enqueue(deme_handle* h, int64_t* ticket);
int32_t deme_kinetic_energy_collect(deme_handle* h, int64_t ticket, double* ke);

/* Bin assignment of the reference (getNumberOfBinsEachSphereTouches / populateBinSphereTouchingPairs, radix sort
 * by bin: src/kernel/DEMBinSphereKernels.cu:12-230, src/algorithms/DEMCubContactDetection.cu:59-129) on the current
 * state.  Fills per-sphere bin counts and, if pair arrays are given with enough capacity, the (bin, sphere) pairs
 * sorted by bin (stable).  *n_pairs receives the pair count. */
int32_t deme_bin_assignment(deme_handle* h, uint16_t* n_bins_per_sphere, uint8_t* n_anal_per_sphere,
                            uint32_t pair_capacity, uint32_t* bin_ids, uint32_t* sphere_ids, uint32_t* n_pairs);

/* Stable radix sort of (key, value) u32 pairs held in device memory (project-written onesweep sort; replaces
 * cub::DeviceRadixSort::SortPairs, src/algorithms/DEMCubWrappers.cu:43-59).  Sorts bits [0, key_bits).
 * The call returns once the work is queued on `stream`; its error word sits in the last 16 bytes of `scratch`
 * (offset deme_radix_sort_scratch_bytes(n) - 16) and is read with deme_radix_sort_status. */
int32_t deme_radix_sort_pairs_device(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, int32_t key_bits, void* scratch,
                                     size_t scratch_bytes, void* stream);
size_t deme_radix_sort_scratch_bytes(uint32_t n);

/* Outcome of the last sort queued on `stream`: scratch = the buffer given to deme_radix_sort_pairs_device for n
 * pairs, or NULL for deme_radix_sort_pairs_static.  Waits for `stream`, stores the sort's error word in *word (may
 * be NULL) and returns DEME_OK when it is 0, DEME_ERR_TIMEOUT when a bounded look-back wait of the sort ran out (the
 * output is then not in order; sorting again is safe, since every sort clears the word first).  No counterpart
 * in the reference, whose CUB sort reports nothing on the device (src/algorithms/DEMCubWrappers.cu:43-59).
 * Allocates nothing. */
int32_t deme_radix_sort_status(const void* scratch, uint32_t n, void* stream, uint32_t* word);

/* ---- Adjoint of the step (no reference counterpart) ----------------------------------------------------------
 * For scenes of clumps (or single spheres) with analytical walls (planes, cylinders, cones), the built-in
 * Hertz-Mindlin model, Extended Taylor integration and contact detection every step.  Clump families are free or
 * driven (linear and rotational motion both prescribed); wall families are driven.  deme_adjoint_record runs
 * n_steps forward from the current state, keeping a checkpoint every `checkpoint_every` steps;
 * deme_adjoint_backward takes the gradient of a loss with respect to the final state and returns it with respect to
 * the state before the window and to the material parameters, recomputing each window segment from its checkpoint.
 * The contact set of each step is the one the forward pass found.  Angular velocities are in the world frame
 * (w_world = R(q) w_owner); quaternion gradients (w, x, y, z) hold the world angular velocity fixed.  Driven owners
 * get 0.  The model runs on the recorded FP32 state; gradients are accumulated in FP64.  The handle ends at the
 * recorded final state. */
typedef struct {
    const double* d_pos;     /* n_owners x 3, dL/d(final position); NULL = 0 */
    const double* d_vel;     /* n_owners x 3, dL/d(final velocity); NULL = 0 */
    const double* d_angvel;  /* n_owners x 3, dL/d(final angular velocity, world frame); NULL = 0 */
    const double* d_quat;    /* n_owners x 4, dL/d(final quaternion w, x, y, z); NULL = 0 */
} deme_adjoint_seed;

typedef struct {
    double* d_pos0;      /* n_owners x 3 (may be NULL) */
    double* d_vel0;      /* n_owners x 3 (may be NULL) */
    double* d_angvel0;   /* n_owners x 3 (may be NULL) */
    double* d_material;  /* n_materials x 4: dL/dE, dL/dCoR, dL/dmu, dL/dCrr (may be NULL) */
    double* d_quat0;     /* n_owners x 4 (may be NULL) */
} deme_adjoint_grads;

int32_t deme_adjoint_record(deme_handle* h, int32_t n_steps, int32_t checkpoint_every);
int32_t deme_adjoint_backward(deme_handle* h, const deme_adjoint_seed* seed, deme_adjoint_grads* out);
/* Floors in the adjoint's derivatives at the contact law's non-smooth points: overlap relative to R* (the damping's
 * overlap^(1/4) is unbounded in slope at contact onset), relative rolling speed in m/s (the rolling torque's
 * direction flips through zero speed) and tangential force in N (the Coulomb cap's 1/|Ft|).  Where a floor binds,
 * the gradient is that of the smoothed law; the exact derivative there only describes a neighbourhood far smaller
 * than any useful parameter change.  Defaults 1e-4, 1e-4, 1e-6; zeros give the exact derivative. */
int32_t deme_adjoint_set_floors(deme_handle* h, double overlap_rel, double roll_speed, double tangential_force);
/* Replaces material m's properties (LoadMaterial keys E, nu, CoR, mu, Crr) for the following steps. */
int32_t deme_set_material(deme_handle* h, uint32_t m, float E, float nu, float CoR, float mu, float Crr);

/* Largest n deme_radix_sort_pairs_static accepts. */
#define DEME_SORT_STATIC_MAX_N 1048576u

/* The same stable sort for callers that cannot allocate device memory; it has no counterpart in the reference.
 * Such callers are, for example, a host application that has reserved the GPU's memory for its own pool (a coupled
 * fluid solver, or a framework whose caching allocator owns the HBM), or per-step code that must not call
 * cudaMalloc because it synchronises the device.
 * It allocates nothing: its scratch is a fixed 8.5 MiB __device__ array inside this library, which every GPU that
 * loads the library holds until the process exits.  The caller passes device inputs and outputs (outputs must not
 * alias inputs); nothing needs to be zeroed beforehand, each call clears what its kernels read on `stream`.
 * - n > DEME_SORT_STATIC_MAX_N returns DEME_ERR_TOO_LARGE and launches nothing; key_bits outside [0, 32] returns
 *   DEME_ERR_INVALID.
 * - The first call on each device (with that device current) looks up the scratch address; make it before any
 *   stream capture.  A first call on a capturing stream returns DEME_ERR_STATE.
 * - All calls on one device share the scratch: calls that overlap in time (other streams, other threads) race and
 *   corrupt each other's results.  Serialise them, e.g. one stream per device.
 * - The sort's error word stays in the scratch until the next call: deme_radix_sort_status(NULL, n, stream, &w)
 *   reports whether the last sort completed in order.
 * - The scratch address is kept for the life of the process: calls after cudaDeviceReset are not supported. */
int32_t deme_radix_sort_pairs_static(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, int32_t key_bits, void* stream);

#endif /* __CUDACC_RTC__ */

#ifdef __cplusplus
}
#endif

#endif /* DEME_B200_H */
