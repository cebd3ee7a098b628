// force_model_api.cuh -- what a DEM-Engine force-model string can call, for the run-time compiled force kernel.
//
// A force-model string (DEMSolver::DefineContactForceModel, src/DEM/APIPublic.cpp:116-121) is C++ that runs inside
// the force kernel with the kernel's variables in scope (see force_kernel.cuh) and may call the reference's vector
// helpers (its thirdparty helper_math: float3 arithmetic, dot, cross, length, normalize), applyOriQToVector3 and
// matProxy2ContactParam (src/kernel/DEMHelperKernels.cu:316-339, 394-445), and use the deme:: constants of
// src/DEM/Defines.h.  This header provides those names, written for this project; it is compiled only into the
// NVRTC build of the force kernel.
#pragma once
#include "force_model_hertz.cuh"

namespace deme {
typedef float oriQ_t;
typedef uint8_t family_t;
typedef uint32_t bodyID_t;
typedef uint32_t materialsOffset_t;
// src/DEM/Defines.h:30-35
constexpr double PI = 3.1415926535897932385;
constexpr double PI_SQUARED = 9.869604401089358;
constexpr double TWO_OVER_THREE = 0.666666666666667;
constexpr double FOUR_OVER_THREE = 1.333333333333333;
constexpr double FIVE_OVER_THREE = 1.666666666666667;
constexpr double TWO_TIMES_SQRT_FIVE_OVER_SIX = 1.825741858350554;
constexpr int NOT_A_CONTACT = DEME_NOT_A_CONTACT;
constexpr int SPHERE_SPHERE_CONTACT = DEME_SPHERE_SPHERE_CONTACT;
constexpr int SPHERE_PLANE_CONTACT = DEME_SPHERE_PLANE_CONTACT;
}  // namespace deme

#ifndef DEME_TINY_FLOAT
#define DEME_TINY_FLOAT 1e-12
#endif
#ifndef DEME_HUGE_FLOAT
#define DEME_HUGE_FLOAT 1e15
#endif

// float3 arithmetic
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ void operator+=(float3& a, float3 b) { a = a + b; }
__device__ __forceinline__ void operator-=(float3& a, float3 b) { a = a - b; }
__device__ __forceinline__ void operator*=(float3& a, float s) { a = a * s; }
__device__ __forceinline__ void operator/=(float3& a, float s) { a = a / s; }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return a * (1.0f / sqrtf(dot(a, a))); }

// double3 - double3 gives a float3 (differences of nearby points), as in the reference's model dialect
__device__ __forceinline__ float3 operator-(double3 a, double3 b) {
    return make_float3((float)(a.x - b.x), (float)(a.y - b.y), (float)(a.z - b.z));
}

// Rotate (X, Y, Z) by the unit quaternion (w, x, y, z); the float case is the rotation the kernels use.
template <typename T1, typename T2>
__device__ __forceinline__ void applyOriQToVector3(T1& X, T1& Y, T1& Z, T2 w, T2 x, T2 y, T2 z) {
    float fx = (float)X, fy = (float)Y, fz = (float)Z;
    deme_b200::rot_f(fx, fy, fz, (float)w, (float)x, (float)y, (float)z);
    X = (T1)fx;
    Y = (T1)fy;
    Z = (T1)fz;
}

template <typename T>
__device__ __forceinline__ void matProxy2ContactParam(T& E_eff, T& G_eff, T& CoR_cnt, T& mu_cnt, T& Crr_cnt, T E_A,
                                                      T nu_A, T CoR_A, T mu_A, T Crr_A, T E_B, T nu_B, T CoR_B,
                                                      T mu_B, T Crr_B) {
    deme_b200::mat_proxy<T>(E_eff, G_eff, CoR_cnt, mu_cnt, Crr_cnt, E_A, nu_A, CoR_A, mu_A, Crr_A, E_B, nu_B, CoR_B,
                            mu_B, Crr_B);
}
