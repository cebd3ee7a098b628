// profiler.cu -- see profiler.cuh.
#include <atomic>
#include <vector>

#include "../../include/deme_b200.h"
#include "profiler.cuh"

namespace deme_b200 {

namespace {
std::atomic<int64_t> g_launches{0};
bool g_timing = false;
struct Pending {
    int id;
    cudaEvent_t a, b;
};
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_open;
double g_ms[KID_COUNT];
int64_t g_cnt[KID_COUNT];
const char* g_names[KID_COUNT] = {"place_anal",    "sphere_prep",   "scan",          "sort_histogram",
                                  "sort_onesweep", "gather_sorted", "pair_find",     "pair_assemble",
                                  "pair_overflow", "cell_scatter",  "history",       "force",
                                  "integrate",     "pair_exact",    "other",         "adj_record",
                                  "adj_integrate", "adj_contact",   "adj_history",   "mesh_find"};
}  // namespace

const char* kernel_name(int id) { return (id >= 0 && id < KID_COUNT) ? g_names[id] : "?"; }

void prof_begin(int id, cudaStream_t st) {
    g_launches++;
    if (!g_timing) return;
    cudaEvent_t a;
    cudaEventCreate(&a);
    cudaEventRecord(a, st);
    g_open.push_back(a);
}

void prof_end(int id, cudaStream_t st) {
    if (!g_timing || g_open.empty()) return;
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, st);
    g_pending.push_back(Pending{id, g_open.back(), b});
    g_open.pop_back();
}

int64_t launch_count() { return g_launches.load(); }

void add_launches(int64_t n) { g_launches += n; }

bool prof_timing() { return g_timing; }

}  // namespace deme_b200

using namespace deme_b200;

extern "C" {

int64_t deme_launch_count(void) { return launch_count(); }

int32_t deme_kernel_timing(int32_t enable) {
    if (enable) {
        for (auto& p : g_pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        g_pending.clear();
        for (int i = 0; i < KID_COUNT; i++) {
            g_ms[i] = 0.0;
            g_cnt[i] = 0;
        }
    }
    g_timing = enable != 0;
    return DEME_OK;
}

int32_t deme_kernel_times(int32_t cap, const char** names, double* total_ms, int64_t* launches, int32_t* n_out) {
    for (auto& p : g_pending) {
        float ms = 0.f;
        cudaEventSynchronize(p.b);
        cudaEventElapsedTime(&ms, p.a, p.b);
        g_ms[p.id] += ms;
        g_cnt[p.id] += 1;
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    g_pending.clear();
    int n = 0;
    for (int i = 0; i < KID_COUNT && n < cap; i++) {
        if (names) names[n] = g_names[i];
        if (total_ms) total_ms[n] = g_ms[i];
        if (launches) launches[n] = g_cnt[i];
        n++;
    }
    if (n_out) *n_out = n;
    return DEME_OK;
}

}  // extern "C"
