/*
 * deme_oracle.h -- CPU oracle for the DEM-Engine per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference algorithm, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  The product path never links it.
 *
 * The contact list it produces keeps the reference's order: sphere--analytical contacts first (sphere order),
 * then sphere--sphere contacts per active bin (ascending bin id, in-bin pair loop order of the thread-per-bin
 * kernel), then a stable sort by idA (src/algorithms/DEMCubContactDetection.cu:99-264).
 */
#ifndef DEME_ORACLE_H
#define DEME_ORACLE_H

#include "../include/deme_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

oracle_ctx* orc_create(const deme_sim_params* p, const deme_scene* s);
void orc_destroy(oracle_ctx* c);
int32_t orc_set_threads(int32_t n);

int32_t orc_detect_contacts(oracle_ctx* c);
int32_t orc_compute_forces(oracle_ctx* c);
int32_t orc_integrate(oracle_ctx* c);
int32_t orc_step(oracle_ctx* c, int32_t n);

int32_t orc_download_state(oracle_ctx* c, deme_state* out);
int32_t orc_upload_state(oracle_ctx* c, const deme_state* in);
uint32_t orc_num_contacts(oracle_ctx* c);
int32_t orc_download_contacts(oracle_ctx* c, deme_contacts* out);
int32_t orc_upload_contacts(oracle_ctx* c, const deme_contacts* in);
int32_t orc_download_contact_forces(oracle_ctx* c, deme_contact_forces* out);
int32_t orc_bin_assignment(oracle_ctx* c, uint16_t* n_bins, uint8_t* n_anal, uint32_t cap, uint32_t* bins,
                           uint32_t* spheres, uint32_t* n_pairs);
double orc_kinetic_energy(oracle_ctx* c);
int32_t orc_max_spheres_in_bin(oracle_ctx* c);
double orc_time(oracle_ctx* c);
/* Replaces one family's constant prescription (deme_set_family_prescription's counterpart); a test that checks
 * prescribed-motion expressions sets, before each step, the values the expressions take at that step's time. */
int32_t orc_set_family_prescription(oracle_ctx* c, int32_t family, const deme_family_prescription* p);
int32_t orc_change_clump_sizes(oracle_ctx* c, uint32_t n, const uint32_t* owners, const float* factors);

#ifdef __cplusplus
}
#endif
#endif
