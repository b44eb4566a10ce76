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

// The other schemes of GetINVScheme (API/Physics/src/Flux_Inviscid.cpp:88-134),
// perfect gas, static grid (face velocity 0), no preconditioning; each
// writes the flux per unit face area to f[0..4].

// Steger_Scheme (Flux_Inviscid.cpp:12467-12694), entropy fix method 3 (none):
// one side's split flux; sgn = +1 keeps the positive eigenvalues (left
// state), -1 the negative ones (right state).
template <class T>
__device__ __forceinline__ void steger_side(const T *q, T g, T xsn, T ysn, T zsn, T sgn, T *f)
{
    const T r = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
    const T v2 = u * u + v * v + w * w;
    const T h = (g / (g - T(1))) * (p / r) + T(0.5) * v2;
    const T e = h - p / (r + T(kSmall));
    const T vn = xsn * u + ysn * v + zsn * w;
    const T c2 = g * p / r;
    const T c = sqrt(fabs(c2));
    T l1 = vn, l2 = vn + c, l3 = vn - c;
    l1 = T(0.5) * (l1 + sgn * fabs(l1));
    l2 = T(0.5) * (l2 + sgn * fabs(l2));
    l3 = T(0.5) * (l3 + sgn * fabs(l3));
    const T c2g = c2 / g;
    const T xi1 = c2g * (l1 + l1 - l2 - l3) / (c2 + c2);
    const T xi2 = c2g * (l2 - l3) / (c + c);
    const T ex = l1 - xi1;
    f[0] = r * ex;
    f[1] = r * (ex * u + xi2 * xsn);
    f[2] = r * (ex * v + xi2 * ysn);
    f[3] = r * (ex * w + xi2 * zsn);
    f[4] = r * (l1 * e - xi1 * h + xi2 * vn);
}

// Vanleer_Scheme (Flux_Inviscid.cpp:12697-12950, nPrecondition = 0): one
// side's Van Leer split flux (kLeft: F+ of the left state, else F- of the right).
template <class T, bool kLeft>
__device__ __forceinline__ void vanleer_side(const T *q, T g, T xsn, T ysn, T zsn, T *f)
{
    const T r = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
    const T v2 = u * u + v * v + w * w;
    const T h = (g / (g - T(1))) * (p / r) + T(0.5) * v2;
    const T vn = xsn * u + ysn * v + zsn * w;
    const T rvn = r * vn;
    const T c = sqrt(fabs(g * p / r));
    const T mach = vn / c;
    if (kLeft ? mach > T(1) : mach < T(-1)) {
        f[0] = rvn;
        f[1] = rvn * u + xsn * p;
        f[2] = rvn * v + ysn * p;
        f[3] = rvn * w + zsn * p;
        f[4] = rvn * h;
    } else if (kLeft ? mach < T(-1) : mach > T(1)) {
        f[0] = f[1] = f[2] = f[3] = f[4] = T(0);
    } else {
        const T fm = kLeft ? T(0.25) * r * c * (mach + T(1)) * (mach + T(1))
                           : T(-0.25) * r * c * (mach - T(1)) * (mach - T(1));
        const T t = kLeft ? (-vn + T(2) * c) / g : (-vn - T(2) * c) / g;
        f[0] = fm;
        f[1] = fm * (u + xsn * t);
        f[2] = fm * (v + ysn * t);
        f[3] = fm * (w + zsn * t);
        f[4] = fm * h;
    }
}

// GetAngleOfTwoVector (API/DataStruct/include/PHMatrix.h:203-217): the dot
// product over both norms (sums from zero), clamped, acos.
template <class T>
__device__ __forceinline__ T angle_of(const T *a, const T *b)
{
    T dot = T(0), na = T(0), nb = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) dot += a[i] * b[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) na += a[i] * a[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) nb += b[i] * b[i];
    const T c = dot / sqrt(na) / sqrt(nb);
    if (c > T(1)) return T(0);
    if (c < T(-1)) return T(3.141592653589793);
    return acos(c);
}

// Rotate_Vanleer_Scheme (Flux_Inviscid.cpp:12952-13180): Van Leer's splitting
// along n1, the direction of the velocity jump across the face (x when there
// is none), turned to the face normal's side, and along n2, normal to n1 in
// the plane of n1 and the face normal (y when n1 is the normal), each weighted
// by the cosine of its angle to the face normal (CrossProduct,
// API/Math/src/Math_BasisFunction.cpp:98-104).
template <class T>
__device__ __forceinline__ void vanleer_rotate_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn,
                                                    T *f)
{
    const T n[3] = {xsn, ysn, zsn};
    T n1[3], n2[3];
    const T du = qr[1] - ql[1], dv = qr[2] - ql[2], dw = qr[3] - ql[3];
    if (du == T(0) && dv == T(0) && dw == T(0)) {
        n1[0] = T(1); n1[1] = T(0); n1[2] = T(0);
    } else {
        const T sqdv = sqrt(du * du + dv * dv + dw * dw);
        n1[0] = du / sqdv; n1[1] = dv / sqdv; n1[2] = dw / sqdv;
    }
    T angle1 = angle_of<T>(n1, n);
    if (cos(angle1) < T(0)) {
        n1[0] = -n1[0]; n1[1] = -n1[1]; n1[2] = -n1[2];
        angle1 = angle_of<T>(n1, n);
    }
    if (fabs(n1[0] - xsn) < T(1.0e-8) && fabs(n1[1] - ysn) < T(1.0e-8) && fabs(n1[2] - zsn) < T(1.0e-8)) {
        n2[0] = T(0); n2[1] = T(1); n2[2] = T(0);
    } else {
        const T t[3] = {n1[1] * n[2] - n1[2] * n[1], n1[2] * n[0] - n1[0] * n[2], n1[0] * n[1] - n1[1] * n[0]};
        n2[0] = t[1] * n1[2] - t[2] * n1[1];
        n2[1] = t[2] * n1[0] - t[0] * n1[2];
        n2[2] = t[0] * n1[1] - t[1] * n1[0];
    }
    T nn = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) nn += n2[i] * n2[i];
    const T normn2 = sqrt(nn);
    const T sgn = cos(angle_of<T>(n2, n)) < T(0) ? T(-1) : T(1);
#pragma unroll
    for (int i = 0; i < 3; ++i) n2[i] = (sgn * n2[i]) / normn2;
    const T angle2 = angle_of<T>(n2, n);
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
        const T *d = dir == 0 ? n1 : n2;
        T a[5], b[5];
        vanleer_side<T, true>(ql, gl, d[0], d[1], d[2], a);
        vanleer_side<T, false>(qr, gr, d[0], d[1], d[2], b);
        const T c = cos(dir == 0 ? angle1 : angle2);
#pragma unroll
        for (int k = 0; k < 5; ++k) f[k] = f[k] + c * (a[k] + b[k]);
    }
}

// The rotated Van Leer flux formed in FP64 on both paths: the rotation
// degenerates in single precision (its 1e-8 test of n1 against the normal
// lies below FP32 resolution, and a zero cross product then divides 0 by 0).
template <class T>
__device__ __forceinline__ void vanleer_rotate_flux_fp64(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn,
                                                         T *f)
{
    double dl[5], dr[5], fd[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { dl[k] = (double)ql[k]; dr[k] = (double)qr[k]; }
    vanleer_rotate_flux<double>(dl, dr, (double)gl, (double)gr, (double)xsn, (double)ysn, (double)zsn, fd);
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = (T)fd[k];
}

// Hlle_Scheme (Flux_Inviscid.cpp:13917-14077): HLLE with signal speeds from
// the Roe average and both sides; conserved jump as
// PerfectGas::Primitive2Conservative (PerfectGas.cpp:284-323) forms it.
template <class T>
__device__ __forceinline__ void hlle_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn, T *f)
{
    const T rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    const T rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    const T v2l = ul * ul + vl * vl + wl * wl;
    const T v2r = ur * ur + vr * vr + wr * wr;
    const T hl = (gl / (gl - T(1))) * (pl / rl) + T(0.5) * v2l;
    const T hr = (gr / (gr - T(1))) * (pr / rr) + T(0.5) * v2r;
    const T ratio = sqrt(rr / rl);
    const T coef = T(1) / (T(1) + ratio);
    const T rm = sqrt(rl * rr);
    const T um = (ul + ur * ratio) * coef;
    const T vm = (vl + vr * ratio) * coef;
    const T wm = (wl + wr * ratio) * coef;
    const T pm = (pl + pr * ratio) * coef;
    const T gm = (gl + gr * ratio) * coef;
    const T vnl = xsn * ul + ysn * vl + zsn * wl;
    const T vnr = xsn * ur + ysn * vr + zsn * wr;
    const T rvnl = rl * vnl, rvnr = rr * vnr;
    const T vn = xsn * um + ysn * vm + zsn * wm;
    const T cl = sqrt(gl * pl / (rl + T(kSmall)));
    const T cr = sqrt(gr * pr / (rr + T(kSmall)));
    const T cm = sqrt(gm * pm / (rm + T(kSmall)));
    const T fl[5] = {rvnl, rvnl * ul + xsn * pl, rvnl * vl + ysn * pl, rvnl * wl + zsn * pl, rvnl * hl};
    const T fr[5] = {rvnr, rvnr * ur + xsn * pr, rvnr * vr + ysn * pr, rvnr * wr + zsn * pr, rvnr * hr};
    const T el = (pl / rl) / (gl - T(1)) + T(0.5) * v2l;
    const T er = (pr / rr) / (gr - T(1)) + T(0.5) * v2r;
    const T cvl[5] = {rl, rl * ul, rl * vl, rl * wl, rl * el};
    const T cvr[5] = {rr, rr * ur, rr * vr, rr * wr, rr * er};
    const T bm = tmin(T(0), tmin(vn - cm, vnl - cl));
    const T bp = tmax(T(0), tmax(vn + cm, vnr + cr));
    const T c1 = bp * bm / (bp - bm + T(kSmall));
    const T c2 = T(-0.5) * (bp + bm) / (bp - bm + T(kSmall));
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = T(0.5) * (fl[k] + fr[k]) + c1 * (cvr[k] - cvl[k]) + c2 * (fr[k] - fl[k]);
}

// Ausmdv_Scheme (Flux_Inviscid.cpp:13191-13461): AUSMD / AUSMV blended by the
// pressure jump, the Haenel / Van Leer flux at shocks, and its entropy fix.
template <class T>
__device__ __forceinline__ void ausmdv_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn, T *f)
{
    const T rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    const T rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    const T gama = T(0.5) * (gl + gr);
    const T v2l = ul * ul + vl * vl + wl * wl;
    const T v2r = ur * ur + vr * vr + wr * wr;
    const T hl = (gl / (gl - T(1))) * (pl / rl) + T(0.5) * v2l;
    const T hr = (gr / (gr - T(1))) * (pr / rr) + T(0.5) * v2r;
    const T vnl = xsn * ul + ysn * vl + zsn * wl;
    const T vnr = xsn * ur + ysn * vr + zsn * wr;
    const T orl = T(1) / (rl + T(kSmall)), orr = T(1) / (rr + T(kSmall));
    const T cl = sqrt(gama * pl * orl), cr = sqrt(gama * pr * orr);
    const T cm = tmax(cl, cr);
    const T ocm = T(1) / (cm + T(kSmall));
    const T ssw = ((vnl > cl && vnr < cr) || (vnl > -cl && vnr < -cr)) ? T(1) : T(0);
    const T ssw_a = T(1) - ssw;
    // Haenel / Van Leer with each side's sound speed
    T ml = vnl / cl, mr = vnr / cr;
    T mla = fabs(ml), mra = fabs(mr);
    T mpl, ppl, mmr, pmr;
    if (mla >= T(1)) { mpl = T(0.5) * (ml + mla); ppl = T(0.5) * (T(1) + ml / (mla + T(kSmall))); }
    else { const T t = T(0.25) * ((ml + T(1)) * (ml + T(1))); mpl = t; ppl = t * (T(2) - ml); }
    if (mra >= T(1)) { mmr = T(0.5) * (mr - mra); pmr = T(0.5) * (T(1) - mr / (mra + T(kSmall))); }
    else { const T t = T(0.25) * ((mr - T(1)) * (mr - T(1))); mmr = -t; pmr = t * (T(2) + mr); }
    const T p12 = ppl * pl + pmr * pr;
    const T rvnl_v = cl * rl * mpl, rvnr_v = cr * rr * mmr;
    // AUSMD / AUSMV with the common sound speed
    ml = vnl * ocm; mla = fabs(ml);
    mr = vnr * ocm; mra = fabs(mr);
    const T r1 = pl * orl, r2 = pr * orr, r3 = T(2) / (r1 + r2);
    const T al = r1 * r3, ar = r2 * r3;
    if (mla >= T(1)) mpl = T(0.5) * (ml + mla);
    else { const T t = T(0.25) * ((ml + T(1)) * (ml + T(1))); mpl = al * t + (T(1) - al) * (T(0.5) * (ml + mla)); }
    if (mra >= T(1)) mmr = T(0.5) * (mr - mra);
    else { const T t = T(0.25) * ((mr - T(1)) * (mr - T(1))); mmr = -ar * t + (T(1) - ar) * (T(0.5) * (mr - mra)); }
    T rvnl_d = cm * rl * mpl, rvnr_d = cm * rr * mmr;
    const T rvn = rvnl_d + rvnr_d;
    rvnl_d = T(0.5) * (rvn + fabs(rvn));
    rvnr_d = T(0.5) * (rvn - fabs(rvn));
    T rvnl = rvnl_v, rvnr = rvnr_v;
    const T sw = T(0.5) * tmin(T(1), T(10) * fabs(pr - pl) / tmin(pl, pr));
    T rvvn = ssw * (rvnl_v * vnl + rvnr_v * vnr);
    rvvn += (T(0.5) - sw) * ssw_a * (rvnl_d * vnl + rvnr_d * vnr) +
            (T(0.5) + sw) * ssw_a * cm * (rl * mpl * vnl + rr * mmr * vnr);
    const bool a = (vnl - cl) < T(0) && (vnr - cr) > T(0);
    const bool b = (vnl + cl) < T(0) && (vnr + cr) > T(0);
    if (a != b) {
        const T t = a ? ssw_a * T(0.125) * ((vnr - cr) - (vnl - cl)) : ssw_a * T(0.125) * ((vnr + cr) - (vnl + cl));
        rvnl += t * rl;
        rvnr -= t * rr;
    }
    rvvn += p12;
    f[0] = rvnl + rvnr;
    f[1] = rvnl * (ul - xsn * vnl) + rvnr * (ur - xsn * vnr) + rvvn * xsn;
    f[2] = rvnl * (vl - ysn * vnl) + rvnr * (vr - ysn * vnr) + rvvn * ysn;
    f[3] = rvnl * (wl - zsn * vnl) + rvnr * (wr - zsn * vnr) + rvvn * zsn;
    f[4] = rvnl * hl + rvnr * hr;
}

// FMmpn / FMppn (Flux_Inviscid.cpp:14079-14107): split Mach number and
// pressure polynomials; ipn = +1 for the left side, -1 for the right.
template <class T>
__device__ __forceinline__ T fm_mpn(T m, T ipn)
{
    if (fabs(m) >= T(1)) return T(0.5) * (m + ipn * fabs(m));
    return ipn * T(0.25) * ((m + ipn) * (m + ipn));
}

template <class T>
__device__ __forceinline__ T fm_ppn(T m, T ipn)
{
    if (fabs(m) >= T(1)) return T(0.5) * (m + ipn * fabs(m)) / m;
    return ipn * T(0.25) * ((m + ipn) * (m + ipn)) * (T(2) * ipn - m);
}

// AusmpwPlus_Scheme (Flux_Inviscid.cpp:13628-13915): AUSMPW+ with the mean
// sound speed 0.5 (a_L + a_R) and the weight 1 - min(p_L/p_R, p_R/p_L)^3 * lim
// (lim = AusmpwPlusLimiter).
template <class T>
__device__ __forceinline__ void ausmpwp_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn, T lim,
                                             T *f)
{
    const T rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    const T rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    const T v2l = ul * ul + vl * vl + wl * wl;
    const T v2r = ur * ur + vr * vr + wr * wr;
    const T hl = (gl / (gl - T(1))) * (pl / rl) + T(0.5) * v2l;
    const T hr = (gr / (gr - T(1))) * (pr / rr) + T(0.5) * v2r;
    const T al = sqrt(gl * (pl / (rl + T(kSmall))));
    const T ar = sqrt(gr * (pr / (rr + T(kSmall))));
    const T vnl = xsn * ul + ysn * vl + zsn * wl;
    const T vnr = xsn * ur + ysn * vr + zsn * wr;
    const T minplr = tmin(pl / (pr + T(kSmall)), pr / (pl + T(kSmall)));
    const T c12 = T(0.5) * (al + ar);
    const T ocm = T(1) / c12;
    const T ml = vnl * ocm, mr = vnr * ocm;
    const T fm4l = fm_mpn(ml, T(1)), fm4r = fm_mpn(mr, T(-1));
    const T fp5l = fm_ppn(ml, T(1)), fp5r = fm_ppn(mr, T(-1));
    const T m12 = fm4l + fm4r;
    const T p12 = fp5l * pl + fp5r * pr;
    const T fw = T(1) - minplr * minplr * minplr * lim;
    const T op12 = T(1) / (p12 + T(kSmall));
    T fl = T(0), fr = T(0);
    if (p12 != T(0)) {
        if (fabs(ml) <= T(1)) fl = pl * op12 - T(1);
        if (fabs(mr) <= T(1)) fr = pr * op12 - T(1);
    }
    T mpl, mmr;
    if (m12 >= T(0)) {
        const T o = T(1) + fr;
        mpl = fm4l + fm4r * ((T(1) - fw) * o - fl);
        mmr = fm4r * fw * o;
    } else {
        const T o = T(1) + fl;
        mpl = fm4l * fw * o;
        mmr = fm4r + fm4l * ((T(1) - fw) * o - fr);
    }
    f[0] = c12 * (mpl * rl + mmr * rr);
    f[1] = c12 * (mpl * rl * ul + mmr * rr * ur) + p12 * xsn;
    f[2] = c12 * (mpl * rl * vl + mmr * rr * vr) + p12 * ysn;
    f[3] = c12 * (mpl * rl * wl + mmr * rr * wr) + p12 * zsn;
    f[4] = c12 * (mpl * rl * hl + mmr * rr * hr);
}

// Ausmpw_Scheme (Flux_Inviscid.cpp:13463-13626): AUSMPW.  It differs from
// AUSMPW+ in its sound speeds (gamma p (1 / (rho + SMALL)), mean
// 1 / (0.5 (a_L + a_R) + SMALL)), in a pressure weight without limiter, and in
// the pressure corrections, taken for |M| < 1 with no test of p12.  Its split
// polynomials (FMSplit4 / FPSplit5 with beta = alpha = 0) are FMmpn / FMppn.
template <class T>
__device__ __forceinline__ void ausmpw_flux(const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn, T *f)
{
    const T rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    const T rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    const T v2l = ul * ul + vl * vl + wl * wl;
    const T v2r = ur * ur + vr * vr + wr * wr;
    const T hl = (gl / (gl - T(1))) * (pl / rl) + T(0.5) * v2l;
    const T hr = (gr / (gr - T(1))) * (pr / rr) + T(0.5) * v2r;
    const T vnl = xsn * ul + ysn * vl + zsn * wl;
    const T vnr = xsn * ur + ysn * vr + zsn * wr;
    const T orl = T(1) / (rl + T(kSmall)), orr = T(1) / (rr + T(kSmall));
    const T cl = sqrt(gl * pl * orl), cr = sqrt(gr * pr * orr);
    const T cm = T(0.5) * (cl + cr);
    const T ocm = T(1) / (cm + T(kSmall));
    const T ml = vnl * ocm, mr = vnr * ocm;
    const T fm4l = fm_mpn(ml, T(1)), fm4r = fm_mpn(mr, T(-1));
    const T fp5l = fm_ppn(ml, T(1)), fp5r = fm_ppn(mr, T(-1));
    const T m12 = fm4l + fm4r;
    const T p12 = fp5l * pl + fp5r * pr;
    const T minplr = tmin(pl / (pr + T(kSmall)), pr / (pl + T(kSmall)));
    const T fw = T(1) - minplr * minplr * minplr;
    const T op12 = T(1) / (p12 + T(kSmall));
    T fl = T(0), fr = T(0);
    if (fabs(ml) < T(1)) fl = pl * op12 - T(1);
    if (fabs(mr) < T(1)) fr = pr * op12 - T(1);
    T mpl, mmr;
    if (m12 >= T(0)) {
        const T o = T(1) + fr;
        mpl = fm4l + fm4r * ((T(1) - fw) * o - fl);
        mmr = fm4r * fw * o;
    } else {
        const T o = T(1) + fl;
        mpl = fm4l * fw * o;
        mmr = fm4r + fm4l * ((T(1) - fw) * o - fr);
    }
    f[0] = cm * (mpl * rl + mmr * rr);
    f[1] = cm * (mpl * rl * ul + mmr * rr * ur) + p12 * xsn;
    f[2] = cm * (mpl * rl * vl + mmr * rr * vr) + p12 * ysn;
    f[3] = cm * (mpl * rl * wl + mmr * rr * wr) + p12 * zsn;
    f[4] = cm * (mpl * rl * hl + mmr * rr * hr);
}

// Non-Roe scheme selected by uns_scheme_name (PHX_SCHEME_*); uniform across a launch.
template <class T>
__device__ __forceinline__ void other_flux(int scheme, const T *ql, const T *qr, T gl, T gr, T xsn, T ysn, T zsn,
                                           T ausmpwLim, T *f)
{
    if (scheme == PHX_SCHEME_STEGER || scheme == PHX_SCHEME_VANLEER) {
        T a[5], b[5];
        if (scheme == PHX_SCHEME_STEGER) {
            steger_side<T>(ql, gl, xsn, ysn, zsn, T(1), a);
            steger_side<T>(qr, gr, xsn, ysn, zsn, T(-1), b);
        } else {
            vanleer_side<T, true>(ql, gl, xsn, ysn, zsn, a);
            vanleer_side<T, false>(qr, gr, xsn, ysn, zsn, b);
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) f[k] = a[k] + b[k];
    } else if (scheme == PHX_SCHEME_HLLE) {
        hlle_flux<T>(ql, qr, gl, gr, xsn, ysn, zsn, f);
    } else if (scheme == PHX_SCHEME_AUSMDV) {
        ausmdv_flux<T>(ql, qr, gl, gr, xsn, ysn, zsn, f);
    } else if (scheme == PHX_SCHEME_AUSMPW) {
        ausmpw_flux<T>(ql, qr, gl, gr, xsn, ysn, zsn, f);
    } else {
        ausmpwp_flux<T>(ql, qr, gl, gr, xsn, ysn, zsn, ausmpwLim, f);
    }
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
