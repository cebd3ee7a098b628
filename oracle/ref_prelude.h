// ref_prelude.h -- lets the reference's kernel sources (text of src/kernel/*.cu, after the same placeholder
// substitution its JitHelper performs, src/core/utils/JitHelper.cpp:36-59) compile as host C++ with g++.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref): the reference run on the CPU, used to pin the C oracle.
// Nothing here is reference source; the generated translation units include this header first.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include <vector_functions.h>
#include <vector_types.h>

// Each reference JIT program is its own device module, so its jitified constant arrays are module-local:
// give them internal linkage here.
#undef __constant__
#define __constant__ static
#undef __shared__
#define __shared__

// Launch emulation: the harness sets these per emulated thread.
extern thread_local dim3 blockIdx;
extern thread_local dim3 threadIdx;
extern thread_local dim3 blockDim;

// Unqualified math calls in the kernels resolve to the float overloads, as they do in CUDA device code.
using std::abs;
using std::cos;
using std::log;
using std::max;
using std::min;
using std::sin;
using std::sqrt;

inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline void __threadfence() {}
namespace cub {
inline void ThreadTrap() { std::abort(); }
}  // namespace cub
