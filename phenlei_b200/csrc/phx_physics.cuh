// Device-side physics of the NS path, templated on the working precision T
// (double for the FP64 path, float for the mixed path).  Each function states
// the reference routine whose arithmetic it follows, in the same operation
// order, so that the FP64 path agrees with the reference to rounding.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "phx_internal.h"

namespace phx {

template <class T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }
template <class T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }

// Harten entropy fix (API/Physics/include/Flux_RoeEntropyCorrection.h:66-74).
template <class T>
__device__ __forceinline__ T harten(T e, T lim)
{
    T a = fabs(e);
    if (a < lim) a = T(0.5) * (e * e + lim * lim) / lim;
    return a;
}

// Roe flux in conservative jump form per unit face area
// (Roe_Scheme_ConservativeForm, API/Physics/src/Flux_Inviscid.cpp:136-399,
// perfect gas, static grid, entropy fix method 3).
template <class T>
__device__ __forceinline__ void roe_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn,
                                         T acoustic, T convective, T *f)
{
    const T LITTLE = T(1.0e-10);
    T rL = tmax(ql[0], LITTLE), uL = ql[1], vL = ql[2], wL = ql[3], pL = tmax(ql[4], LITTLE);
    T rR = tmax(qr[0], LITTLE), uR = qr[1], vR = qr[2], wR = qr[3], pR = tmax(qr[4], LITTLE);
    T v2L = uL * uL + vL * vL + wL * wL;
    T v2R = uR * uR + vR * vR + wR * wR;
    T hL = (gl / (gl - T(1))) * (pL / rL) + T(0.5) * v2L;
    T hR = (gr / (gr - T(1))) * (pR / rR) + T(0.5) * v2R;
    T vnL = xsn * uL + ysn * vL + zsn * wL;
    T vnR = xsn * uR + ysn * vR + zsn * wR;
    T rvnL = rL * vnL, rvnR = rR * vnR;
    f[0] = T(0.5) * (rvnL + rvnR);
    f[1] = T(0.5) * (rvnL * uL + xsn * pL + rvnR * uR + xsn * pR);
    f[2] = T(0.5) * (rvnL * vL + ysn * pL + rvnR * vR + ysn * pR);
    f[3] = T(0.5) * (rvnL * wL + zsn * pL + rvnR * wR + zsn * pR);
    f[4] = T(0.5) * (rvnL * hL + rvnR * hR);
    T ratio = sqrt(rR / rL);
    T coef = T(1) / (T(1) + ratio);
    T um = (uL + uR * ratio) * coef;
    T vm = (vL + vR * ratio) * coef;
    T wm = (wL + wR * ratio) * coef;
    T pm = (pL + pR * ratio) * coef;
    T rm = sqrt(rL * rR);
    T gama = (gl + gr * ratio) * coef;
    T gm1 = gama - T(1);
    T v2 = um * um + vm * vm + wm * wm;
    T hm = gama / gm1 * pm / rm + T(0.5) * v2;
    T vn = xsn * um + ysn * vm + zsn * wm;
    T c2 = gm1 * (hm - T(0.5) * v2);
    T cm = sqrt(fabs(c2));
    T EL = (T(1) / (gl - T(1))) * (pL / rL) + T(0.5) * v2L;
    T ER = (T(1) / (gr - T(1))) * (pR / rR) + T(0.5) * v2R;
    T dq0 = rR - rL, dq1 = rR * uR - rL * uL, dq2 = rR * vR - rL * vL, dq3 = rR * wR - rL * wL;
    T dq4 = rR * ER - rL * EL;
    T maxe = fabs(vn) + cm;
    T e1 = harten(fabs(vn), convective * maxe);
    T e2 = harten(fabs(vn + cm), acoustic * maxe);
    T e3 = harten(fabs(vn - cm), acoustic * maxe);
    T xi1 = (T(2) * e1 - e2 - e3) / (T(2) * c2);
    T xi2 = (e2 - e3) / (T(2) * cm);
    T dc = vn * dq0 - xsn * dq1 - ysn * dq2 - zsn * dq3;
    T c2dc = c2 * dc;
    T dh = -gm1 * (um * dq1 + vm * dq2 + wm * dq3 - dq4) + T(0.5) * gm1 * v2 * dq0;
    f[0] -= T(0.5) * (e1 * dq0 - dh * xi1 - dc * xi2);
    f[1] -= T(0.5) * (e1 * dq1 + (xsn * c2dc - um * dh) * xi1 + (xsn * dh - um * dc) * xi2);
    f[2] -= T(0.5) * (e1 * dq2 + (ysn * c2dc - vm * dh) * xi1 + (ysn * dh - vm * dc) * xi2);
    f[3] -= T(0.5) * (e1 * dq3 + (zsn * c2dc - wm * dh) * xi1 + (zsn * dh - wm * dc) * xi2);
    f[4] -= T(0.5) * (e1 * dq4 + (vn * c2dc - hm * dh) * xi1 + (vn * dh - hm * dc) * xi2);
}

// VenFun (API/Math/include/Math_Limiter.h:174-180).
template <class T>
__device__ __forceinline__ T venfun(T x, T y, T eps)
{
    T x2 = x * x, xy = x * y, y2 = y * y;
    return (x2 + eps + T(2) * xy) / (x2 + T(2) * y2 + xy + eps);
}

// RoeAveragedVariables (API/Physics/src/Flux_Inviscid.cpp:15440-15465).
template <class T>
__device__ __forceinline__ void roe_average(const T *a, T ga, const T *b, T gb, T *o)
{
    T hL = ga / (ga - T(1)) * a[4] / a[0] + T(0.5) * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
    T hR = gb / (gb - T(1)) * b[4] / b[0] + T(0.5) * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]);
    T t0 = sqrt(b[0] / a[0]);
    T t1 = T(1) / (T(1) + t0);
    o[0] = sqrt(b[0] * a[0]);
    o[1] = (a[1] + b[1] * t0) * t1;
    o[2] = (a[2] + b[2] * t0) * t1;
    o[3] = (a[3] + b[3] * t0) * t1;
    T hm = (hL + hR * t0) * t1;
    o[4] = o[0] * (hm - T(0.5) * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3])) * (ga - T(1)) / ga;
}

// MXDQ_STD with ipn = -1 (API/Physics/src/Jacobian.cpp:13-86) and
// PerfectGas::ComputeTotalEnthalpyAndDH (API/Physics/src/PerfectGas.cpp:368-395):
// the split flux-Jacobian product used by the LU-SGS sweeps.
template <class T>
__device__ __forceinline__ void mxdq(const T *prim, T nx, T ny, T nz, T area, T gama, const T *dq, T *f, T radius)
{
    T rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    T c2 = fabs(gama * pm / rm);
    T cm = sqrt(c2);
    T cits = nx * um + ny * vm + nz * wm;
    T ipnrad = -radius / tmax(T(kSmall), area);
    T l1 = T(0.5) * (cits + ipnrad);
    T l2 = T(0.5) * (cits + cm + ipnrad);
    T l3 = T(0.5) * (cits - cm + ipnrad);
    T x1 = (l1 + l1 - l2 - l3) / (c2 + c2);
    T x2 = (l2 - l3) / (cm + cm);
    T dc = cits * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
    T c2dc = c2 * dc;
    T v2 = um * um + vm * vm + wm * wm;
    T g1 = gama - T(1);
    T dh = -g1 * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
    dh += T(0.5) * g1 * v2 * dq[0];
    T hm = (gama / g1) * (pm / rm) + T(0.5) * v2;
    T a = dh * x1 + dc * x2;
    T b = c2dc * x1 + dh * x2;
    f[0] = (l1 * dq[0] - a) * area;
    f[1] = (l1 * dq[1] - um * a + nx * b) * area;
    f[2] = (l1 * dq[2] - vm * a + ny * b) * area;
    f[3] = (l1 * dq[3] - wm * a + nz * b) * area;
    f[4] = (l1 * dq[4] - hm * a + cits * b) * area;
}

}  // namespace phx
