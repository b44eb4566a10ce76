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

// IEEE division on both paths, for the LU-SGS sweeps: the files holding the
// face and SA passes are compiled with approximate FP32 division.
__device__ __forceinline__ float idiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double idiv(double a, double b) { return a / b; }

// Sweep geometry of the LU-SGS dataflow sweeps: a slot of kSweepLanes lanes
// per schedule position, kSweepSlots slots per warp.  Every wait is bounded by
// NsConst::spinLimit polls (phx_set_wait_limit).
static constexpr int kSweepThreads = 256;
static_assert(kSweepLanes * kSweepSlots == 32, "one warp holds kSweepSlots slots");
static_assert(kSweepMaxEntries == 2 * kSweepLanes, "a cell spans at most two adjacent slots");

// Write-once sweep records.  Before a sweep every element of its output
// records holds the sentinel, a NaN whose sign and payload no arithmetic
// result carries (the GPU's NaN results are the positive canonical NaN, and
// producers map the sentinel pattern itself to that NaN).  During the sweep
// each element is stored once, so a reader that sees anything but the
// sentinel sees the final value: the data is its own completion flag, and
// neither a fence between the producer's stores nor a second load after the
// wait sits on the sweep's critical path.  Stores and polling loads are
// relaxed at device scope (coherent in L2, not cached in L1).
static constexpr unsigned kSentinelF = 0xffc0e1a5u;
static constexpr unsigned long long kSentinelD = 0xfff80000d0e1a5c3ull;

template <class T> __device__ __forceinline__ T sweep_sentinel();
template <> __device__ __forceinline__ float sweep_sentinel<float>() { return __uint_as_float(kSentinelF); }
template <> __device__ __forceinline__ double sweep_sentinel<double>()
{
    return __longlong_as_double((long long)kSentinelD);
}
__device__ __forceinline__ bool is_sentinel(float v) { return __float_as_uint(v) == kSentinelF; }
__device__ __forceinline__ bool is_sentinel(double v)
{
    return (unsigned long long)__double_as_longlong(v) == kSentinelD;
}
// a computed value as stored: the sentinel pattern becomes the canonical NaN
__device__ __forceinline__ float unsentinel(float v) { return is_sentinel(v) ? __int_as_float(0x7fffffff) : v; }
__device__ __forceinline__ double unsentinel(double v)
{
    return is_sentinel(v) ? __longlong_as_double(0x7fffffffffffffffLL) : v;
}

__device__ __forceinline__ float ld_poll(const float *p)
{
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ double ld_poll(const double *p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(float *p, float v)
{
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(double *p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// Polls the first five elements of an 8-element record; true once none of
// them is the sentinel (o then holds the final values).
__device__ __forceinline__ bool poll5(const float *p, float *o)
{
    asm volatile("ld.relaxed.gpu.global.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3])
                 : "l"(p)
                 : "memory");
    o[4] = ld_poll(p + 4);
    return !(is_sentinel(o[0]) | is_sentinel(o[1]) | is_sentinel(o[2]) | is_sentinel(o[3]) | is_sentinel(o[4]));
}
__device__ __forceinline__ bool poll5(const double *p, double *o)
{
    asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(o[0]), "=d"(o[1]) : "l"(p) : "memory");
    asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(o[2]), "=d"(o[3]) : "l"(p + 2) : "memory");
    o[4] = ld_poll(p + 4);
    return !(is_sentinel(o[0]) | is_sentinel(o[1]) | is_sentinel(o[2]) | is_sentinel(o[3]) | is_sentinel(o[4]));
}

// Publishes the five values of an 8-element record (slots 5-7 zero).
__device__ __forceinline__ void publish5(float *p, const float *v)
{
    asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(unsentinel(v[0])),
                 "f"(unsentinel(v[1])), "f"(unsentinel(v[2])), "f"(unsentinel(v[3]))
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p + 4), "f"(unsentinel(v[4])),
                 "f"(0.0f), "f"(0.0f), "f"(0.0f)
                 : "memory");
}
__device__ __forceinline__ void publish5(double *p, const double *v)
{
    asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(unsentinel(v[0])),
                 "d"(unsentinel(v[1]))
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1, %2};" ::"l"(p + 2), "d"(unsentinel(v[2])),
                 "d"(unsentinel(v[3]))
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1, %2};" ::"l"(p + 4), "d"(unsentinel(v[4])), "d"(0.0)
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1, %2};" ::"l"(p + 6), "d"(0.0), "d"(0.0) : "memory");
}

}  // namespace phx
