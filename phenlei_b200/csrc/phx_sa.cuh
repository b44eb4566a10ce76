// Spalart-Allmaras device functions shared by the SA kernels and the MLP
// source kernels: PositiveSA and the exact source of
// SourceFluxOneEquationOriginal (NSMB formation).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "phx_internal.h"
#include "phx_physics.cuh"

namespace phx {

// PositiveSA (CFD/TurbSolver/include/TurbSolver.h:103-116).
template <class T>
__device__ __forceinline__ T positive_sa(T nue, T visl, T rho)
{
    if (nue < T(0)) {
        const T xsi = nue / (visl / rho);
        const T xsi3 = xsi * xsi * xsi;
        return nue * (T(16) + xsi3) / (T(16) - xsi3);
    }
    return nue;
}

// Exact SA source and its implicit part per unit volume
// (SourceFluxOneEquationOriginal, CFD/TurbSolver/src/TurbSolverUnstr.cpp:
// 2702-2916, NSMB formation, ft2 = 0): src = production - wall destruction,
// spec = the spectral-radius contribution (part1 + part2).
template <class T>
__device__ __forceinline__ void sa_source_exact(T nue, T omega, T olam, T odist2, T grd2, T oRe, T &src, T &spec)
{
    const T karm = T(0.41), cb1 = T(0.1355), cb2 = T(0.622), cv1 = T(7.1), cw2 = T(0.3), cw3 = T(2.0);
    const T sigma = T(2.0 / 3.0);
    const T kap2 = karm * karm, okap2 = T(1) / kap2;
    const T cw1 = cb1 * okap2 + (T(1) + cb2) / sigma;
    const T cv13 = cv1 * cv1 * cv1;
    const T cw36 = pow(cw3, T(6));
    const T or6 = T(1) / T(6);
    const T ct3 = T(1.2);
    const T saC2 = T(0.7), saC3 = T(0.9);
    const T cw1kap2 = cw1 * kap2;
    (void)grd2;
    const T xsi = nue * olam + (T)kSmall;
    const T xsi3 = xsi * xsi * xsi;
    const T fv1 = xsi3 / (xsi3 + cv13);
    const T fv2 = T(1) - xsi / (T(1) + xsi * fv1);
    const T rs = nue * okap2 * odist2 * oRe;
    const T nuetrs = nue * rs;
    const T sbar = rs * fv2;
    T std_;
    if (sbar >= -saC2 * omega) std_ = omega + sbar;
    else std_ = omega + omega * (saC2 * saC2 * omega + saC3 * sbar) / ((saC3 - T(2) * saC2) * omega - sbar);
    const T ostd = T(1) / (std_ + (T)kSmall);
    T r = rs * ostd;
    r = tmin(r, T(10));
    const T r5 = pow(r, T(5));
    const T gg = r + cw2 * (r5 * r - r);
    const T g6 = pow(gg, T(6));
    const T fw = gg * pow((T(1) + cw36) / (g6 + cw36), or6);
    const T ft2 = T(0);
    T production = cb1 * (T(1) - ft2) * std_ * nue;
    T walldest = (cw1kap2 * fw - cb1 * ft2) * nuetrs;
    const T destrAlpha = T(50);
    if (nue < T(0)) {
        production = cb1 * (T(1) - ct3) * omega * nue;
        walldest = -destrAlpha * cw1kap2 * nuetrs;
    }
    src = production - walldest;
    const T dfv2dk = (T(3) * cv13 * pow(fv1 / (xsi + (T)kSmall), T(2)) - T(1)) / pow(T(1) + xsi * fv1, T(2));
    const T dsdnu = oRe * okap2 * odist2 * (fv2 + xsi * dfv2dk);
    const T dfwdg = fw / (gg + (T)kSmall) * (T(1) - g6 / (g6 + cw36));
    const T dgdr = T(1) + cw2 * (T(6) * r5 - T(1));
    const T drdnu = oRe * okap2 * odist2 * ostd * (T(1) - nue * ostd * dsdnu);
    const T dfwdnu = dfwdg * dgdr * drdnu;
    T prod = cb1 * (T(1) - ft2) * std_;
    T dest = (cw1 * fw - cb1 * ft2 * okap2) * nue * odist2 * oRe;
    T prodp = cb1 * ((T(1) - ft2) * dsdnu);
    T destp = (cw1 * (fw + dfwdnu * nue) - cb1 * ft2 * okap2) * odist2 * oRe;
    if (nue < T(0)) {
        prod = cb1 * (T(1) - ct3) * omega;
        dest = -destrAlpha * cw1 * nue * odist2 * oRe;
        prodp = cb1 * ((T(1) - ct3) * dsdnu);
        destp = -destrAlpha * cw1 * odist2 * oRe;
    }
    const T prde = prod - dest;
    const T prdep = prodp - destp;
    const T part1 = -T(0.5) * (prde - fabs(prde));
    const T part2 = -T(0.5) * (prdep - fabs(prdep)) * nue;
    spec = part1 + part2;
}

// The exact source evaluated in FP64 for either working precision.  In the
// free stream (Omega = 0) the implicit part multiplies d fw / dg = 0 by a
// d r / d nu~ of order 1e48 / d^4, which overflows FP32 to 0 * inf = NaN; in
// FP64 the product is the finite zero the reference computes.
template <class T>
__device__ __forceinline__ void sa_source_fp64(T nue, T omega, T olam, double d, T grd2, double oRe, T &src, T &spec)
{
    double s, p;
    sa_source_exact<double>((double)nue, (double)omega, (double)olam, 1.0 / (d * d), (double)grd2, oRe, s, p);
    src = (T)s;
    spec = (T)p;
}

}  // namespace phx
