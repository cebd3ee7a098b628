// profiler.cuh -- launch counting and per-kernel CUDA-event timing (process-wide, single host thread).
//
// Every launcher in kernels.cu and primitives.cu counts its launches.  When timing is on, each launch is bracketed
// by two events recorded on the stream it is launched on, so durations are device times of that kernel alone.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace deme_b200 {

enum KernelId : int {
    KID_PLACE_ANAL = 0,
    KID_SPHERE_PREP,
    KID_SCAN,
    KID_SORT_HIST,
    KID_SORT_PASS,
    KID_GATHER,
    KID_PAIR_COUNT,
    KID_PAIR_EMIT,
    KID_PAIR_OVERFLOW,
    KID_CELL_SCATTER,
    KID_HISTORY,
    KID_FORCE,
    KID_INTEGRATE,
    KID_PAIR_EXACT,
    KID_OTHER,
    KID_ADJ_RECORD,     // adjoint: per-step records of the recomputed segment (state, accelerations, contact list)
    KID_ADJ_INTEGRATE,  // adjoint: reverse integration
    KID_ADJ_CONTACT,    // adjoint: reverse contact law and geometry
    KID_ADJ_HISTORY,    // adjoint: reverse history map and re-keying at segment boundaries
    KID_MESH_FIND,      // sphere--mesh search (facet-driven)
    KID_COUNT
};

const char* kernel_name(int id);
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st);
int64_t launch_count();
void add_launches(int64_t n);  // kernels a replayed CUDA graph ran (recorded once, counted at every replay)
bool prof_timing();  // per-kernel timing is on (its events are recorded at launch time, so graphs are not used)

struct ProfScope {
    int id;
    cudaStream_t st;
    ProfScope(int i, cudaStream_t s) : id(i), st(s) { prof_begin(i, s); }
    ~ProfScope() { prof_end(id, st); }
};

}  // namespace deme_b200
