// force_jit.cuh -- run-time compilation of a user force-model string into the force kernel (host side).
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/deme_b200.h"

namespace deme_b200 {

// Maximum number of per-contact wildcards a force model can declare: they live in the contact's float4 history.
constexpr int kMaxContactWildcards = 4;

struct UserForceKernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern[2] = {nullptr, nullptr};  // [0]: no per-contact outputs, [1]: stores force / contact points
    int n_wildcards = 0;
};

// Compiles `model` (the body of a DEM-Engine force-model string) for this device with NVRTC into the force-kernel
// template.  `names` are the per-contact wildcards; like the reference, they are assigned storage slots in sorted
// order.  On failure returns a DEME_ERR_* code and fills `err` (the compiler log for a model that does not compile).
int32_t compile_user_force_model(const char* model, const char* const* names, int32_t n, UserForceKernel& out,
                                 std::string& err);
void release_user_force_model(UserForceKernel& k);

// Family-change rules (ChangeFamilyWhen) compiled into k_family_change (family_change_kernel.cuh).
struct FamilyChangeKernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
};
// n rules: owners of family from[i] move to family to[i] when conditions[i] (a code block whose `return` gives the
// decision) holds.  On failure returns a DEME_ERR_* code and fills `err` (the compiler log).
int32_t compile_family_change_rules(int32_t n, const uint32_t* from, const uint32_t* to,
                                    const char* const* conditions, FamilyChangeKernel& out, std::string& err);
void release_family_change_rules(FamilyChangeKernel& k);

// Prescribed motions written as expressions (SetFamilyPrescribedLinVel / AngVel / Position with strings that are not
// constants) compiled into k_integrate_motion (prescribed_motion_kernel.cuh).
struct MotionKernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
};
// n families' expressions; n <= 0 releases the kernel.  On failure returns a DEME_ERR_* code and fills `err` (the
// compiler log for an expression that does not compile); `out` is then unchanged.
int32_t compile_prescribed_motion(int32_t n, const deme_motion_expressions* m, MotionKernel& out, std::string& err);
void release_prescribed_motion(MotionKernel& k);

}  // namespace deme_b200
