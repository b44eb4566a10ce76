// Device helpers shared by the kernel files of the phx library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "phx_internal.h"

namespace phx {

static constexpr int kThreads = 256;

template <class T> __device__ __forceinline__ T ld(const T *p) { return __ldg(p); }
// Loads of data written earlier in the same kernel by other blocks: bypass L1.
template <class T> __device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// Vector loads of 4- or 8-element records (16-byte aligned).
__device__ __forceinline__ void ld4(const double *p, double *o)
{
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, float *o)
{
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
template <class T>
__device__ __forceinline__ void ld8(const T *p, T *o) { ld4(p, o); ld4(p + 4, o + 4); }
__device__ __forceinline__ void ld4cg(const double *p, double *o)
{
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void ld4cg(const float *p, float *o)
{
    const float4 a = __ldcg(reinterpret_cast<const float4 *>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
template <class T>
__device__ __forceinline__ void ld8cg(const T *p, T *o) { ld4cg(p, o); ld4cg(p + 4, o + 4); }
__device__ __forceinline__ void st4(double *p, const double *v)
{
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(float *p, const float *v)
{
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
}
template <class T>
__device__ __forceinline__ void st8(T *p, const T *v) { st4(p, v); st4(p + 4, v + 4); }

// Writes state, c2 = |gamma p / rho| and total enthalpy of a cell record
// (slot 7, the limiter, is left untouched).  c2 and the enthalpy are the
// per-cell factors MXDQ_STD forms (Jacobian.cpp:22-23, PerfectGas.cpp:384-394).
template <class T>
__device__ __forceinline__ void put_state(T *rec, const T *q, T gm)
{
    const T c2 = fabs(gm * q[4] / q[0]);
    const T hm = (gm / (gm - T(1))) * (q[4] / q[0]) + T(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    T v[4] = {q[0], q[1], q[2], q[3]};
    st4(rec, v);
    rec[4] = q[4];
    rec[5] = c2;
    rec[6] = hm;
}

// Temperature (ComputeGamaAndTemperature, NSSolverUnstruct.cpp:4717-4730) and
// Sutherland viscosity (ComputeViscousCoefficientWithoutChemical, :6722-6747),
// formed on the fly from a cell record wherever they are needed.
template <class T>
__device__ __forceinline__ T temperature(const T *q, T coef) { return q[4] / (coef * q[0]); }
template <class T>
__device__ __forceinline__ T sutherland(T t, T s) { return t * sqrt(t) * (T(1) + s) / (t + s); }

__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Per-cell completion flags of the LU-SGS dataflow sweeps (release / acquire at
// device scope), and the sweep geometry: a lane group of kGroup lanes per cell,
// kSweepPad groups per warp.
static constexpr long long kSpinLimit = 20000000LL;   // ~1-2 s of polling per wait
static constexpr int kSweepThreads = 256;
static constexpr int kGroup = kSweepGroup;            // lanes per cell
static_assert(kGroup * kSweepPad == 32, "one warp holds kSweepPad lane groups");

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace phx
