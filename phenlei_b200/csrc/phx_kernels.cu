// sm_100a kernels of the NS per-iteration path (storage layout: see
// phx_internal.h).
//
// Per-cell sums are owner-computes gathers over the cell's faces in the
// reference's face order, so no atomics touch the state and the FP64 path
// keeps the reference's accumulation order.  Face metrics stay FP64; the
// working state T is double (FP64 path) or float (mixed path).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "phx_internal.h"
#include "phx_device.cuh"
#include "phx_physics.cuh"

namespace phx {

// ---------------------------------------------------------------------------
// Boundary: ghost-cell state per boundary face (NSSolverUnstruct::Boundary,
// NSSolverUnstruct.cpp:13404-13515): SymmetryBCRegion (:19413),
// ViscousAdiabaticWallBCRegion (:20988), FarfieldBCRegion (:21195).
// Computed in FP64 from the FP64 master state.  Interface ghosts keep the
// state the last halo exchange gave them (Boundary skips INTERFACE faces,
// :13474); their working record and laminar viscosity are formed from it.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) boundary_kernel(DevGrid g, NsConst c, double *q, Work<T> w,
                                                            bool writeVisl)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nBFace) return;
    const int nt = g.nTotal;
    const int le = g.lr[f].x, re = g.nCell + f;
    const double r = q[le], u = q[nt + le], v = q[2 * nt + le], wv = q[3 * nt + le], p = q[4 * nt + le];
    double fr[4];
    ld4(g.frec + (size_t)f * kF, fr);
    const double xn = fr[0], yn = fr[1], zn = fr[2];
    double o[5] = {r, u, v, wv, p};
    const int kind = g.bkind[f];
    if (kind == BK_INTERFACE) {
#pragma unroll
        for (int k = 0; k < 5; ++k) o[k] = q[k * nt + re];
    } else if (kind == BK_SYMMETRY) {
        const double vn = xn * u + yn * v + zn * wv;
        o[1] = u - 2.0 * xn * vn;
        o[2] = v - 2.0 * yn * vn;
        o[3] = wv - 2.0 * zn * vn;
    } else if (kind == BK_WALL) {
        o[1] = -u; o[2] = -v; o[3] = -wv;
    } else if (kind == BK_FARFIELD) {
        const double *pi = c.primInf;
        const double rO = pi[0], uO = pi[1], vO = pi[2], wO = pi[3], pO = pi[4];
        const double gl = c.gama;
        const double cO = sqrt(fabs(gl * pO / rO));
        const double vnO = xn * uO + yn * vO + zn * wO;
        const double vnI = xn * u + yn * v + zn * wv;
        const double cI = sqrt(fabs(gl * p / r));
        const double gm1 = gl - 1.0;
        const double velI = sqrt(u * u + v * v + wv * wv);
        if (velI > cI) {
            if (vnI < 0.0) { for (int k = 0; k < 5; ++k) o[k] = pi[k]; }
        } else {
            const double Rp = vnI + 2.0 * cI / gm1;
            const double Rm = vnO - 2.0 * cO / gm1;
            const double vnB = 0.5 * (Rp + Rm);
            const double cB = 0.25 * (Rp - Rm) * gm1;
            double s, vtx, vty, vtz;
            if (vnB >= 0.0) {
                s = p / pow(r, gl);
                vtx = u - xn * vnI; vty = v - yn * vnI; vtz = wv - zn * vnI;
            } else {
                s = pO / pow(rO, gl);
                vtx = uO - xn * vnO; vty = vO - yn * vnO; vtz = wO - zn * vnO;
            }
            const double rB = pow((cB * cB / (s * gl)), 1.0 / gm1);
            o[0] = rB;
            o[1] = vtx + xn * vnB;
            o[2] = vty + yn * vnB;
            o[3] = vtz + zn * vnB;
            o[4] = cB * cB * rB / gl;
        }
    }
    T t[5];
    for (int k = 0; k < 5; ++k) {
        q[k * nt + re] = o[k];
        t[k] = (T)o[k];
    }
    put_state<T>(w.qrec + (size_t)re * kQ, t, (T)c.gama);
    // laminar viscosity of the ghost for the SA step (NS ComputeViscousCoeff
    // covers the ghosts, NSSolverUnstruct.cpp:6733-6745)
    if (w.trec && writeVisl) w.trec[(size_t)re * kTr + 2] = sutherland(temperature(t, (T)c.coefState), (T)c.tsuth);
}

template <class T>
void launch_boundary(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s)
{
    if (g.nBFace == 0) return;
    boundary_kernel<T><<<(g.nBFace + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, q64, w, true);
}

template <class T>
void launch_boundary_post(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s)
{
    if (g.nBFace == 0) return;
    boundary_kernel<T><<<(g.nBFace + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, q64, w, false);
}

template <class T>
__global__ void __launch_bounds__(kThreads) sync_qrec_kernel(DevGrid g, NsConst c, const double *q, Work<T> w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nTotal) return;
    const int nt = g.nTotal;
    T t[5];
    for (int k = 0; k < 5; ++k) t[k] = (T)q[k * nt + i];
    put_state<T>(w.qrec + (size_t)i * kQ, t, (T)c.gama);
}

template <class T>
void launch_sync_qrec(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w, cudaStream_t s)
{
    sync_qrec_kernel<T><<<(g.nTotal + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, q64, w);
}

// ---------------------------------------------------------------------------
// Gradient + limiter, fused per cell:
//  Green-Gauss cell gradient (UnstructGrid::CompGradientGGCell,
//  Geo_UnstructGrid.cpp:3220-3284) or least-squares gradient
//  (CompGradientLSQ, :3996-4085, weights of ComputeWeight :3761-3935) of the 5
//  primitives, and for viscous runs of the temperature (GetGradientField,
//  NSSolverUnstruct.cpp:18244-18330), accumulated in the reference's face
//  order; then the scalar Venkatakrishnan limiter from rho and p
//  (Limiter::VencatLimiter7, Limiter.cpp:1091-1200, neighbour min/max of
//  Limiter::MinMaxDiff :1202-1252 over interior faces), zeroed next to
//  far-field boundaries (SetLimitBoundary, Geo_UnstructGrid.cpp:10744-10775).
// ---------------------------------------------------------------------------
// GG-node node values (NSSolverUnstruct::ComputeNodeValue,
// NSSolverUnstruct.cpp:4734-5080, and ModifyNodeValue :5083-5116) of the
// current state: per node the 1/distance-weighted sum of its contributions in
// the reference's order (a boundary face gives 0.5 (owner + ghost), a cell its
// value) over the weight sum, 0 where the sum is not above SMALL.  The
// reference forms node values in PostSolve after the update and the boundary
// but without recomputing the temperature (Controller::PostSolve,
// Controller.cpp:5063-5205; SetBoundaryValueOfField :1467-1491), so the
// temperature node values its next gradient reads are those of the previous
// state: slot 6 takes slot 5 of the previous call (havePrev), or this state's
// after a state import, as at initialisation (NSSolver::InitDependentVariables,
// NSSolver.cpp:757-790).
template <class T>
__global__ void __launch_bounds__(kThreads) node_value_kernel(DevGrid g, NsConst c, Work<T> w, int havePrev)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nNode) return;
    const T coef = (T)c.coefState;
    T acc[6] = {0, 0, 0, 0, 0, 0};
    const int j1 = ld(g.node_off + n + 1);
    for (int j = ld(g.node_off + n); j < j1; ++j) {
        const int src = ld(g.node_src + j);
        const T wt = (T)ld(g.node_w + j);
        T v[6];
        if (src < 0) {
            const int fs = src & 0x7fffffff;
            const int le = ld(&g.lr[fs].x), re = g.nCell + fs;
            T ql[8], qg[8];
            ld8(w.qrec + (size_t)le * kQ, ql);
            ld8(w.qrec + (size_t)re * kQ, qg);
#pragma unroll
            for (int k = 0; k < 5; ++k) v[k] = T(0.5) * (ql[k] + qg[k]);
            v[5] = T(0.5) * (temperature(ql, coef) + temperature(qg, coef));
        } else {
            T qc[8];
            ld8(w.qrec + (size_t)src * kQ, qc);
#pragma unroll
            for (int k = 0; k < 5; ++k) v[k] = qc[k];
            v[5] = temperature(qc, coef);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] += v[k] * wt;
    }
    const double ws = ld(g.node_wsum + n);
    T o[8];
#pragma unroll
    for (int k = 0; k < 6; ++k) o[k] = ws > kSmall ? acc[k] / (T)ws : T(0);
    T *r = w.nrec + (size_t)n * kN;
    o[6] = havePrev ? r[5] : o[5];
    o[7] = T(0);
    st8(r, o);
}

// kGrad: 0 GG-cell, 1 least squares, 2 GG-node.
template <class T, bool kTemp, int kGrad>
__global__ void __launch_bounds__(kThreads) gradient_limiter_kernel(DevGrid g, NsConst c, Work<T> w)
{
    constexpr bool kLsq = kGrad == 1;
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.nCell) return;
    constexpr int NV = kTemp ? 6 : 5;   // variable 5: temperature
    T qc[8];
    ld8(w.qrec + (size_t)cell * kQ, qc);
    const T coef = (T)c.coefState;
    T vc[NV];
#pragma unroll
    for (int k = 0; k < 5; ++k) vc[k] = qc[k];
    if (kTemp) vc[NV - 1] = temperature(qc, coef);
    double xc[4];
    ld4(g.xrec + (size_t)cell * kX, xc);
    T gx[NV], gy[NV], gz[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) gx[k] = gy[k] = gz[k] = T(0);
    T rmin = qc[0], rmax = qc[0], pmin = qc[4], pmax = qc[4];
    const int j0 = g.c2f_off[cell], j1 = g.c2f_off[cell + 1];
    for (int j = j0; j < j1; ++j) {
        const int f = ld(g.c2f + j);
        const int2 lr = ld(g.lr + f);
        const bool isLeft = (lr.x == cell);
        const int nb = isLeft ? lr.y : lr.x;
        T qn[8];
        ld8(w.qrec + (size_t)nb * kQ, qn);
        T vn[NV];
#pragma unroll
        for (int k = 0; k < 5; ++k) vn[k] = qn[k];
        if (kTemp) vn[NV - 1] = temperature(qn, coef);
        if (kLsq) {
            // (q[re] - q[le]) (x[re] - x[le]) iwt in the face's own orientation,
            // added to both sides
            double xn[4];
            ld4(g.xrec + (size_t)nb * kX, xn);
            const double iw = ld(g.frec + (size_t)f * kF + 7);
            const T dx = (T)(isLeft ? xn[0] - xc[0] : xc[0] - xn[0]);
            const T dy = (T)(isLeft ? xn[1] - xc[1] : xc[1] - xn[1]);
            const T dz = (T)(isLeft ? xn[2] - xc[2] : xc[2] - xn[2]);
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const T dq = (T)iw * (isLeft ? vn[k] - vc[k] : vc[k] - vn[k]);
                gx[k] += dq * dx; gy[k] += dq * dy; gz[k] += dq * dz;
            }
        } else {
            double fr[4];
            ld4(g.frec + (size_t)f * kF, fr);
            const double a = fr[3];
            const T nx = (T)(fr[0] * a), ny = (T)(fr[1] * a), nz = (T)(fr[2] * a);
            T qf[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) qf[k] = T(0.5) * (isLeft ? (vc[k] + vn[k]) : (vn[k] + vc[k]));
            if (kGrad == 2 && (f >= g.nBFace || ld(g.btype + f) == PHX_BC_SYMMETRY)) {
                // UnstructGrid::CompGradientGGNode_NEW (Geo_UnstructGrid.cpp:4202-4309):
                // the average of the face's node values, in the face's node order
                T sn[NV];
#pragma unroll
                for (int k = 0; k < NV; ++k) sn[k] = T(0);
                const int a0 = ld(g.fn_off + f), a1 = ld(g.fn_off + f + 1);
                for (int a = a0; a < a1; ++a) {
                    T r[8];
                    ld8(w.nrec + (size_t)ld(g.fn_idx + a) * kN, r);
#pragma unroll
                    for (int k = 0; k < 5; ++k) sn[k] += r[k];
                    if (kTemp) sn[NV - 1] += r[6];
                }
                const T cnt = (T)(a1 - a0);
#pragma unroll
                for (int k = 0; k < NV; ++k) qf[k] = sn[k] / cnt;
            }
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                if (isLeft) { gx[k] += qf[k] * nx; gy[k] += qf[k] * ny; gz[k] += qf[k] * nz; }
                else { gx[k] -= qf[k] * nx; gy[k] -= qf[k] * ny; gz[k] -= qf[k] * nz; }
            }
        }
        if (f >= g.nBFace || ld(g.bkind + f) == BK_INTERFACE) {   // MinMaxDiff reads interface ghosts
            rmin = tmin(rmin, qn[0]); rmax = tmax(rmax, qn[0]);
            pmin = tmin(pmin, qn[4]); pmax = tmax(pmax, qn[4]);
        }
    }
    if (kLsq) {
        double m6[8];
        ld8(g.lsq + (size_t)cell * 8, m6);
        const T ixx = (T)m6[0], iyy = (T)m6[1], izz = (T)m6[2], ixy = (T)m6[3], ixz = (T)m6[4], iyz = (T)m6[5];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const T tx = gx[k], ty = gy[k], tz = gz[k];
            gx[k] = ixx * tx + ixy * ty + ixz * tz;
            gy[k] = ixy * tx + iyy * ty + iyz * tz;
            gz[k] = ixz * tx + iyz * ty + izz * tz;
        }
    } else if (kGrad == 2) {
        const T vol = (T)xc[3];
#pragma unroll
        for (int k = 0; k < NV; ++k) { gx[k] /= vol; gy[k] /= vol; gz[k] /= vol; }
    } else {
        const T ovol = T(1) / (T)xc[3];
#pragma unroll
        for (int k = 0; k < NV; ++k) { gx[k] *= ovol; gy[k] *= ovol; gz[k] *= ovol; }
    }
    T gr[kG];
#pragma unroll
    for (int k = 0; k < 5; ++k) { gr[3 * k] = gx[k]; gr[3 * k + 1] = gy[k]; gr[3 * k + 2] = gz[k]; }
    gr[15] = T(0);
    T *go = w.grec + (size_t)cell * kG;
    st8(go, gr);
    st8(go + 8, gr + 8);
    if (kTemp) {
        gr[16] = gx[NV - 1]; gr[17] = gy[NV - 1]; gr[18] = gz[NV - 1]; gr[19] = T(0);
        st4(go + 16, gr + 16);
        // laminar viscosity of this NS step, read by the SA step after the update
        if (w.trec) w.trec[(size_t)cell * kTr + 2] = sutherland(vc[NV - 1], (T)c.tsuth);
    }
    T lim = T(1);
    if (c.limiter != PHX_LIMITER_NOLIM && c.firstOrder) {
        lim = T(0);
    } else if (c.limiter == PHX_LIMITER_BARTH) {
        // Limiter::BarthLimiter (Limiter.cpp:157-262) from rho and p: the face
        // extrapolation clipped to the neighbour min/max difference; a face whose
        // centre lies behind the cell's outward normal zeroes the limiter.  Each
        // candidate is >= 0, so visiting rho and p per face gives the reference's
        // two passes' minimum.
        const T dminr = rmin - qc[0], dmaxr = rmax - qc[0];
        const T dminp = pmin - qc[4], dmaxp = pmax - qc[4];
        const T small = (T)kSmall;
        for (int j = j0; j < j1; ++j) {
            const int f = ld(g.c2f + j);
            double fn[4], fc[4];
            ld4(g.frec + (size_t)f * kF, fn);
            ld4(g.frec + (size_t)f * kF + 4, fc);
            const T dx = (T)(fc[0] - xc[0]), dy = (T)(fc[1] - xc[1]), dz = (T)(fc[2] - xc[2]);
            const T ds = sqrt(dx * dx + dy * dy + dz * dz);
            const T nd = (T)fn[0] * dx + (T)fn[1] * dy + (T)fn[2] * dz;
            const T dot = (ld(g.lr + f).x == cell ? nd : -nd) / (ds + small);
            if (dot < T(0)) { lim = T(0); continue; }
            T d = gx[0] * dx + gy[0] * dy + gz[0] * dz;
            if (d > dmaxr) lim = tmin(lim, dmaxr / (d + small));
            else if (d < dminr) lim = tmin(lim, dminr / (d + small));
            d = gx[4] * dx + gy[4] * dy + gz[4] * dz;
            if (d > dmaxp) lim = tmin(lim, dmaxp / (d + small));
            else if (d < dminp) lim = tmin(lim, dminp / (d + small));
        }
        if (g.farfield_adj[cell]) lim = T(0);
    } else if (c.limiter == PHX_LIMITER_VENCAT) {
        const T vp = (T)ld(g.volpow + cell);
        T er = (T)c.venkatK3 * qc[0]; er = er * qc[0]; er = er * vp;
        T ep = (T)c.venkatK3 * qc[4]; ep = ep * qc[4]; ep = ep * vp;
        const T dminr = rmin - qc[0], dmaxr = rmax - qc[0];
        const T dminp = pmin - qc[4], dmaxp = pmax - qc[4];
        const T small = (T)kSmall;
        for (int j = j0; j < j1; ++j) {
            const int f = ld(g.c2f + j);
            double fc[4];
            ld4(g.frec + (size_t)f * kF + 4, fc);
            const T dx = (T)(fc[0] - xc[0]), dy = (T)(fc[1] - xc[1]), dz = (T)(fc[2] - xc[2]);
            T d = gx[0] * dx + gy[0] * dy + gz[0] * dz;
            if (d > small) lim = tmin(lim, venfun(dmaxr, d, er));
            else if (d < -small) lim = tmin(lim, venfun(dminr, d, er));
            d = gx[4] * dx + gy[4] * dy + gz[4] * dz;
            if (d > small) lim = tmin(lim, venfun(dmaxp, d, ep));
            else if (d < -small) lim = tmin(lim, venfun(dminp, d, ep));
        }
        if (g.farfield_adj[cell]) lim = T(0);
    }
    w.qrec[(size_t)cell * kQ + 7] = lim;
}

template <class T>
void launch_gradient_limiter(const DevGrid &g, const NsConst &c, const Work<T> &w, int nodePrev, cudaStream_t s)
{
    const int blocks = (g.nCell + kThreads - 1) / kThreads;
    if (c.gradient == 2)
        node_value_kernel<T><<<(g.nNode + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, w, nodePrev);
    if (c.viscous) {
        if (c.gradient == 1) gradient_limiter_kernel<T, true, 1><<<blocks, kThreads, 0, s>>>(g, c, w);
        else if (c.gradient == 2) gradient_limiter_kernel<T, true, 2><<<blocks, kThreads, 0, s>>>(g, c, w);
        else gradient_limiter_kernel<T, true, 0><<<blocks, kThreads, 0, s>>>(g, c, w);
    } else {
        if (c.gradient == 1) gradient_limiter_kernel<T, false, 1><<<blocks, kThreads, 0, s>>>(g, c, w);
        else if (c.gradient == 2) gradient_limiter_kernel<T, false, 2><<<blocks, kThreads, 0, s>>>(g, c, w);
        else gradient_limiter_kernel<T, false, 0><<<blocks, kThreads, 0, s>>>(g, c, w);
    }
}

// ---------------------------------------------------------------------------
// Residual, pass 1 (one thread per face): MUSCL face states (GetQlQr /
// ReConstructFaceValue, NSSolverUnstruct.cpp:5507, :13991-14193), the wall /
// symmetry face fix (BoundaryQlQrFix, :13725-13951), the inviscid flux (Roe,
// with kScheme = 1 the other scheme uns_scheme_name selects, with kScheme = 2
// the rotated Van Leer scheme in an instantiation of its own) times the face area
// (InviscidFluxWrap, :14466-14488), the face term of the inviscid
// spectral radius (SpectrumRadiusInviscid, :5749-5850), and the dq-independent
// LU-SGS factors of both face uses (RoeAveragedVariables + GetRad +
// MXDQ_STD, :15097-15116, Jacobian.cpp:27-47).
// ---------------------------------------------------------------------------

// dq-independent part of the neighbour's MXDQ_STD term for the use (cell ->
// neighbour, normal pointing from cell to neighbour).
template <class T>
__device__ __forceinline__ void lusgs_coef(const T *qc, const T *qn, T nx, T ny, T nz, T area, T gm, T *o)
{
    T fp[5];
    roe_average<T>(qc, gm, qn, gm, fp);
    const T vn = nx * fp[1] + ny * fp[2] + nz * fp[3];
    const T rad = (fabs(vn) + sqrt(gm * fp[4] / fp[0])) * area;
    const T c2 = fabs(gm * qn[4] / qn[0]);
    const T cm = sqrt(c2);
    const T cits = nx * qn[1] + ny * qn[2] + nz * qn[3];
    const T ipnrad = -rad / tmax(T(kSmall), area);
    const T a1 = T(0.5) * (cits + ipnrad);
    const T a2 = T(0.5) * (cits + cm + ipnrad);
    const T a3 = T(0.5) * (cits - cm + ipnrad);
    o[0] = a1;
    o[1] = (a1 + a1 - a2 - a3) / (c2 + c2);
    o[2] = (a2 - a3) / (cm + cm);
    o[3] = T(0);
}

// MUSCL state of one side (boundary ghosts carry a zero gradient, so their
// state is used as is; an interface ghost has the neighbouring zone's
// gradient, limiter and centre, and is reconstructed like a cell).
template <class T>
__device__ __forceinline__ void reconstruct(const DevGrid &g, const Work<T> &w, int cell, const double *fc, T lim,
                                            const T *qs, T *qo, bool interfaceGhost = false)
{
#pragma unroll
    for (int k = 0; k < 5; ++k) qo[k] = qs[k];
    if (cell >= g.nCell && !interfaceGhost) return;
    double xc[4];
    ld4(g.xrec + (size_t)cell * kX, xc);
    const T dx = (T)(fc[0] - xc[0]), dy = (T)(fc[1] - xc[1]), dz = (T)(fc[2] - xc[2]);
    T gr[16];
    const T *gp = w.grec + (size_t)cell * kG;
    ld8(gp, gr);
    ld8(gp + 8, gr + 8);
    T tr[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) tr[k] = qs[k] + lim * (gr[3 * k] * dx + gr[3 * k + 1] * dy + gr[3 * k + 2] * dz);
    if (tr[0] > T(0) && tr[4] > T(0)) {
#pragma unroll
        for (int k = 0; k < 5; ++k) qo[k] = tr[k];
    }
}

// Gradients of u, v, w (9 values) and of the temperature (3) of one side of
// a face; a boundary ghost has the owner's gradient (least squares, GG-node)
// or none (GG-cell), as the reference's gradient routines leave them; an
// interface ghost has the neighbouring zone's.
template <class T>
__device__ __forceinline__ void side_gradients(const DevGrid &g, const NsConst &c, const Work<T> &w, int cell,
                                               int owner, T *gv, T *gt, bool interfaceGhost = false)
{
    const int src = (cell < g.nCell || interfaceGhost) ? cell : (c.gradient != 0 ? owner : -1);
    if (src < 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) gv[k] = T(0);
        gt[0] = gt[1] = gt[2] = T(0);
        return;
    }
    const T *gp = w.grec + (size_t)src * kG;
    T a[16];
    ld8(gp, a);
    ld8(gp + 8, a + 8);
#pragma unroll
    for (int k = 0; k < 9; ++k) gv[k] = a[3 + k];
    T b[4];
    ld4(gp + 16, b);
    gt[0] = b[0]; gt[1] = b[1]; gt[2] = b[2];
}

// Viscous flux of one face times the area, F1..F4 (F0 is zero), and the
// face's viscous spectral-radius term, which is also the LU-SGS viscous
// factor of both face uses (SpectrumRadiusViscous method 2,
// NSSolverUnstruct.cpp:5930-5960; SolveLUSGSForward :15339-15357).
// FaceWeight (Geo_UnstructGrid.cpp:2420-2478), GetVisFaceValue
// (NSSolverUnstruct.cpp:7126-7375, static adiabatic walls) and ComputeVisflux
// (:12977-13378, perfect gas).  Geometry is formed in FP64.
template <class T>
__device__ __forceinline__ void viscous_face(const DevGrid &g, const NsConst &c, const Work<T> &w, int f, int le,
                                             int re, const double *fr, const T *qL, const T *qR, T *fv, T &vspec)
{
    // interface faces are interior faces here (FaceWeight, Geo_UnstructGrid.cpp:2475;
    // GetVisFaceValue and ComputeVisflux, NSSolverUnstruct.cpp:7292, :13261)
    const bool itf = f < g.nBFace && g.bkind[f] == BK_INTERFACE;
    const bool bnd = f < g.nBFace && !itf;
    const bool wall = bnd && g.bkind[f] == BK_WALL;
    double xl[4], xr[4];
    ld4(g.xrec + (size_t)le * kX, xl);
    ld4(g.xrec + (size_t)re * kX, xr);
    const double nxs = fr[0], nys = fr[1], nzs = fr[2], area = fr[3];
    const T coef = (T)c.coefState, S = (T)c.tsuth;
    const T tl0 = temperature(qL, coef), tr0 = temperature(qR, coef);
    const T mul = T(0.5) * (sutherland(tl0, S) + sutherland(tr0, S));
    const T mut = w.trec ? T(0.5) * (w.trec[(size_t)le * kTr + 1] + w.trec[(size_t)re * kTr + 1]) : T(0);
    // spectral radius / LU-SGS viscous factor
    {
        const double ds = fabs(nxs * (xr[0] - xl[0]) + nys * (xr[1] - xl[1]) + nzs * (xr[2] - xl[2]));
        const T rho = T(0.5) * (qL[0] + qR[0]);
        T vs = T(2) * (mul + mut) / (rho * (T)ds * (T)c.reynolds + (T)kSmall);
        vs *= T(0.5) * (T)area;
        vspec = vs;
    }
    // FaceWeight
    double dwl = 1.0, dwr = 0.0;
    if (!bnd) {
        const double ax = fr[4] - xl[0], ay = fr[5] - xl[1], az = fr[6] - xl[2];
        const double bx = fr[4] - xr[0], by = fr[5] - xr[1], bz = fr[6] - xr[2];
        const double d1 = sqrt(ax * ax + ay * ay + az * az), d2 = sqrt(bx * bx + by * by + bz * bz);
        const double dl = 1.0 / (d1 + d2 + kSmall);
        dwl = d2 * dl;
        dwr = d1 * dl;
    }
    // tangents
    double t1x, t1y, t1z;
    if (fabs(nxs) > kSmall) { t1x = nys; t1y = -nxs; t1z = 0.0; }
    else if (fabs(nys) > kSmall) { t1x = -nys; t1y = nxs; t1z = 0.0; }
    else if (fabs(nzs) > kSmall) { t1x = 0.0; t1y = -nzs; t1z = nys; }
    else { fv[0] = fv[1] = fv[2] = fv[3] = T(0); return; }
    const double on = 1.0 / sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    t1x *= on; t1y *= on; t1z *= on;
    const double t2x = nys * t1z - nzs * t1y, t2y = nzs * t1x - nxs * t1z, t2z = nxs * t1y - nys * t1x;
    const double dxL = xl[0] - fr[4], dyL = xl[1] - fr[5], dzL = xl[2] - fr[6];
    const double dxR = xr[0] - fr[4], dyR = xr[1] - fr[5], dzR = xr[2] - fr[6];
    const double dL = nxs * dxL + nys * dyL + nzs * dzL;
    const double dR = nxs * dxR + nys * dyR + nzs * dzR;
    const int vf = g.vflag[f];
    T gvl[9], gtl[3], gvr[9], gtr[3];
    side_gradients<T>(g, c, w, le, le, gvl, gtl);
    side_gradients<T>(g, c, w, re, le, gvr, gtr, itf);
    T f1[3] = {qL[1], qL[2], qL[3]}, f2[3] = {qR[1], qR[2], qR[3]};
    T tL = tl0, tR = tr0;
    T fm[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) fm[k] = T(0.5) * (f1[k] + f2[k]);
    const T tmf = T(0.5) * (tl0 + tr0);
    T tM = tmf;
    if (vf & 1) {
        const T xnl = (T)(nxs * dL - dxL), ynl = (T)(nys * dL - dyL), znl = (T)(nzs * dL - dzL);
        const T xnr = (T)(nxs * dR - dxR), ynr = (T)(nys * dR - dyR), znr = (T)(nzs * dR - dzR);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            f1[k] += gvl[3 * k] * xnl + gvl[3 * k + 1] * ynl + gvl[3 * k + 2] * znl;
            f2[k] += gvr[3 * k] * xnr + gvr[3 * k + 1] * ynr + gvr[3 * k + 2] * znr;
        }
        tL += gtl[0] * xnl + gtl[1] * ynl + gtl[2] * znl;
        tR += gtr[0] * xnr + gtr[1] * ynr + gtr[2] * znr;
        if (tL < (T)kSmall) tL = tl0;
        if (tR < (T)kSmall) tR = tr0;
        // face values of GetVisFaceValue: the mean, no-slip at walls
#pragma unroll
        for (int k = 0; k < 3; ++k) fm[k] = wall ? T(0) : T(0.5) * (qL[k + 1] + qR[k + 1]);
        tM = tmf;
    }
    T dfdn[3] = {0, 0, 0}, dtdn = T(0);
    if (vf & 2) {
        const T dLt = (T)dL, dRt = (T)dR;
        T wL = dLt * dLt / (dLt * dLt + dRt * dRt);
        T wR = T(1) - wL;
        if (bnd) { wL = T(1); wR = T(0); }
#pragma unroll
        for (int k = 0; k < 3; ++k) dfdn[k] = wL * ((f1[k] - fm[k]) / dLt) + wR * ((f2[k] - fm[k]) / dRt);
        dtdn = ((tL - tM) / dLt) * wL + ((tR - tM) / dRt) * wR;
    }
    T gx[3], gy[3], gz[3];
    const T wl = (T)dwl, wr = (T)dwr;
    const T n1 = (T)nxs, n2 = (T)nys, n3 = (T)nzs;
    const T a1 = (T)t1x, a2 = (T)t1y, a3 = (T)t1z, b1 = (T)t2x, b2 = (T)t2y, b3 = (T)t2z;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const T fx = wl * gvl[3 * k] + wr * gvr[3 * k];
        const T fy = wl * gvl[3 * k + 1] + wr * gvr[3 * k + 1];
        const T fz = wl * gvl[3 * k + 2] + wr * gvr[3 * k + 2];
        const T d1 = a1 * fx + a2 * fy + a3 * fz;
        const T d2 = b1 * fx + b2 * fy + b3 * fz;
        gx[k] = n1 * dfdn[k] + a1 * d1 + b1 * d2;
        gy[k] = n2 * dfdn[k] + a2 * d1 + b2 * d2;
        gz[k] = n3 * dfdn[k] + a3 * d1 + b3 * d2;
    }
    const T kcp = (mul * (T)c.oPrl + mut * (T)c.oPrt) * (T)c.cp;
    const T qn = kcp * dtdn;
    const T div = T(2.0 / 3.0) * (gx[0] + gy[1] + gz[2]);
    const T vis = mul + mut;
    const T txx = vis * (T(2) * gx[0] - div), tyy = vis * (T(2) * gy[1] - div), tzz = vis * (T(2) * gz[2] - div);
    const T txy = vis * (gy[0] + gx[1]), txz = vis * (gz[0] + gx[2]), tyz = vis * (gz[1] + gy[2]);
    const T v1 = n1 * txx + n2 * txy + n3 * txz;
    const T v2 = n1 * txy + n2 * tyy + n3 * tyz;
    const T v3 = n1 * txz + n2 * tyz + n3 * tzz;
    const T v4 = fm[0] * v1 + fm[1] * v2 + fm[2] * v3 + qn;
    const T sc = -(T)c.oRe * (T)area;
    fv[0] = sc * v1; fv[1] = sc * v2; fv[2] = sc * v3; fv[3] = sc * v4;
}

// Three blocks per SM on the mixed path (at most 85 registers): the face pass
// is latency-bound on its arithmetic, and 16M cells take 5.3 ms against 6.2 ms
// at the two blocks its natural 101 registers allow.
template <class T, bool kVisc, int kScheme>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 3 : 1) face_flux_kernel(DevGrid g, NsConst c, Work<T> w)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nFace) return;
    const int2 lr = ld(g.lr + f);
    const int le = lr.x, re = lr.y;
    double fr[8];
    ld8(g.frec + (size_t)f * kF, fr);
    T qL[8], qR[8];
    ld8(w.qrec + (size_t)le * kQ, qL);
    ld8(w.qrec + (size_t)re * kQ, qR);
    T limL = qL[7], limR = qR[7];
    if (c.reconMethod == 1) { const T m = tmin(limL, limR); limL = limR = m; }
    T ql[5], qr[5];
    if (kScheme != 0 && c.firstOrder) {
#pragma unroll
        for (int k = 0; k < 5; ++k) { ql[k] = qL[k]; qr[k] = qR[k]; }
    } else {
        reconstruct<T>(g, w, le, fr + 4, limL, qL, ql);
        reconstruct<T>(g, w, re, fr + 4, limR, qR, qr, f < g.nBFace && g.bkind[f] == BK_INTERFACE);
    }
    const T xn = (T)fr[0], yn = (T)fr[1], zn = (T)fr[2], area = (T)fr[3];
    if (f < g.nBFace) {
        const int bt = g.btype[f];
        if (bt == PHX_BC_SOLID_SURFACE || bt == PHX_BC_SYMMETRY) {
#pragma unroll
            for (int k = 0; k < 5; ++k) { const T a = T(0.5) * (qL[k] + qR[k]); ql[k] = a; qr[k] = a; }
            if (bt == PHX_BC_SYMMETRY) {
                const T vn = T(2) * (xn * ql[1] + yn * ql[2] + zn * ql[3]);
                qr[1] = ql[1] - vn * xn; qr[2] = ql[2] - vn * yn; qr[3] = ql[3] - vn * zn;
            } else if (g.bkind[f] == BK_WALL) {
                ql[1] = ql[2] = ql[3] = T(0);
                qr[1] = qr[2] = qr[3] = T(0);
            }
        }
    }
    const T gm = (T)c.gama;
    T fl[8];
    if (kScheme == 0) roe_flux<T>(ql, qr, gm, gm, xn, yn, zn, (T)c.acoustic, (T)c.convective, fl);
    else if (kScheme == 2) vanleer_rotate_flux_fp64<T>(ql, qr, gm, gm, xn, yn, zn, fl);
    else other_flux<T>(c.scheme, ql, qr, gm, gm, xn, yn, zn, (T)c.ausmpwLim, fl);
#pragma unroll
    for (int k = 0; k < 5; ++k) fl[k] *= area;
    // inviscid spectral radius term from the face-mean state
    {
        const T vnl = xn * qL[1] + yn * qL[2] + zn * qL[3];
        const T vnr = xn * qR[1] + yn * qR[2] + zn * qR[3];
        const T gmm = T(0.5) * (gm + gm);
        const T pm = T(0.5) * (qL[4] + qR[4]);
        const T rm = T(0.5) * (qL[0] + qR[0]);
        const T vn = T(0.5) * (vnl + vnr);
        const T cm = sqrt(gmm * pm / rm);
        fl[5] = T(0.5) * area * (fabs(vn) + cm);
    }
    T vspec = T(0);
    if (kVisc) {
        T fv[4];
        viscous_face<T>(g, c, w, f, le, re, fr, qL, qR, fv, vspec);
        T vr[8] = {fv[0], fv[1], fv[2], fv[3], T(0), T(0), T(0), T(0)};
        st8(w.flux + (size_t)f * kFlux + 8, vr);
    }
    fl[6] = vspec;
    fl[7] = T(0);
    st8(w.flux + (size_t)f * kFlux, fl);
    // LU-SGS factors: side 0 = the left cell's view, side 1 = the right cell's
    T cf[4];
    lusgs_coef<T>(qL, qR, xn, yn, zn, area, gm, cf);
    cf[3] = vspec;
    st4(w.coef + (size_t)(2 * f) * kCoef, cf);
    if (f >= g.nBFace) {
        lusgs_coef<T>(qR, qL, -xn, -yn, -zn, area, gm, cf);
        cf[3] = vspec;
        st4(w.coef + (size_t)(2 * f + 1) * kCoef, cf);
    }
}

// Residual, pass 2 (one thread per cell): res gathered from the face fluxes
// in the reference's face order with the sign LoadFlux applies
// (NSSolverUnstruct.cpp:6435-6495), the inviscid spectral radius, and the
// local time step (LocalTimeStep / LimitCFL, :5999-6118) with its device-wide
// minimum (Controller::ComputeMinTimeStep, Controller.cpp:706-752).
__device__ __forceinline__ void atomic_min_pos_double(unsigned long long *addr, double v)
{
    atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

template <class T, bool kVisc>
__global__ void __launch_bounds__(kThreads) cell_residual_kernel(DevGrid g, NsConst c, Work<T> w, Reduce *red, double cfl)
{
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    double mydt = kLarge;
    if (cell < g.nCell) {
        T res[5] = {0, 0, 0, 0, 0};
        T spec = T(0), vis = T(0);
        const int j0 = g.c2f_off[cell], j1 = g.c2f_off[cell + 1];
        for (int j = j0; j < j1; ++j) {
            const int f = ld(g.c2f + j);
            const bool isLeft = ld(&g.lr[f].x) == cell;
            T fl[8];
            ld8(w.flux + (size_t)f * kFlux, fl);
            if (isLeft) {
#pragma unroll
                for (int k = 0; k < 5; ++k) res[k] -= fl[k];
            } else {
#pragma unroll
                for (int k = 0; k < 5; ++k) res[k] += fl[k];
            }
            spec += fl[5];
            if (kVisc) vis += fl[6];
        }
        if (kVisc) {
            // ViscousFlux is loaded after InviscidFlux (NSSolver::UpdateResiduals,
            // NSSolver.cpp:71-80): a second pass in the same face order
            for (int j = j0; j < j1; ++j) {
                const int f = ld(g.c2f + j);
                const bool isLeft = ld(&g.lr[f].x) == cell;
                T fv[4];
                ld4(w.flux + (size_t)f * kFlux + 8, fv);
                if (isLeft) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) res[k + 1] -= fv[k];
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) res[k + 1] += fv[k];
                }
            }
        }
        T tot = spec;
        if (c.viscous) tot += vis;
        double cc = cfl;
        const double pc = (double)w.qrec[(size_t)cell * kQ + 4];
        const double plo = 0.001 * c.pTotal, phi = 0.02 * c.pTotal;
        if (pc < plo) cc = c.cflStart;
        else if (pc < phi) cc = (pc - phi) * (cfl - c.cflStart) / (phi - plo) + cfl;
        const double sk = ld(g.skew + cell);
        if (sk < 0.1) cc *= 0.1;
        else if (sk < 10.0) cc *= (1.0 - exp(0.0 - sk));
        const T vol = (T)ld(&g.xrec[(size_t)cell * kX + 3]);
        const T dt = (T)cc * vol / tot;
        w.dtraw[cell] = dt;
        mydt = (double)dt;
        // reciprocal of the LU-SGS diagonal for the unclamped time step, formed
        // as the sweep forms it (the sweep recomputes it where ktmax clamps dt)
        T dd = idiv(T(1), idiv(dt, vol));
        dd += spec;
        if (c.viscous) dd += vis;
        T out[8] = {res[0], res[1], res[2], res[3], res[4], idiv(T(1), dd), spec, vis};
        st8(w.crec + (size_t)cell * kC, out);
    }
    // block minimum, then one atomic per block, skipped when it cannot lower
    // the running minimum (positive doubles order like their bit patterns)
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(0xffffffffu, mydt, o));
    __shared__ double wmin[kThreads / 32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = mydt;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wmin[0];
        for (int i = 1; i < kThreads / 32; ++i) m = fmin(m, wmin[i]);
        const unsigned long long cur = *(volatile unsigned long long *)&red->mindt_bits;
        if (m < kLarge && (unsigned long long)__double_as_longlong(m) < cur) atomic_min_pos_double(&red->mindt_bits, m);
    }
}

template <class T>
void launch_residual(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, double cfl, cudaStream_t s)
{
    const int fb = (g.nFace + kThreads - 1) / kThreads, cb = (g.nCell + kThreads - 1) / kThreads;
    const int kind = c.scheme == PHX_SCHEME_ROE ? 0 : c.scheme == PHX_SCHEME_VANLEER_ROTATE ? 2 : 1;
    if (c.viscous) {
        if (kind == 0) face_flux_kernel<T, true, 0><<<fb, kThreads, 0, s>>>(g, c, w);
        else if (kind == 2) face_flux_kernel<T, true, 2><<<fb, kThreads, 0, s>>>(g, c, w);
        else face_flux_kernel<T, true, 1><<<fb, kThreads, 0, s>>>(g, c, w);
        cell_residual_kernel<T, true><<<cb, kThreads, 0, s>>>(g, c, w, red, cfl);
    } else {
        if (kind == 0) face_flux_kernel<T, false, 0><<<fb, kThreads, 0, s>>>(g, c, w);
        else if (kind == 2) face_flux_kernel<T, false, 2><<<fb, kThreads, 0, s>>>(g, c, w);
        else face_flux_kernel<T, false, 1><<<fb, kThreads, 0, s>>>(g, c, w);
        cell_residual_kernel<T, false><<<cb, kThreads, 0, s>>>(g, c, w, red, cfl);
    }
}

// ---------------------------------------------------------------------------
// LU-SGS (Controller::LUSGS, Controller.cpp:1878-1955) as a dataflow
// computation.  The forward sweep of the reference visits cells in
// increasing number and uses the just-updated dq of lower-numbered face
// neighbours; the backward sweep the reverse.  Here the forward sweep writes
// each cell's dq and delta flux into write-once records (dqfwd, dflux) and
// the backward sweep writes the final dq into dqrec; all three are filled
// with the sentinel before the sweep (sweep_reset_kernel), so a cell waits
// only on the records of the neighbours it reads, polling the data itself,
// and sees exactly the values the sequential sweep of the reference sees,
// with no device-wide barrier and no completion flags.  Lane groups (one per
// cell) take schedule positions in level order (forward positions, then
// backward positions), the four groups of a warp four consecutive positions
// of one level (levels are padded to multiples of four), so a warp only
// waits on cells of earlier levels, held by other warps or by its own
// earlier rounds.  All warps are co-resident (cooperative launch), so the
// wait graph cannot cycle: the warp holding the lowest unfinished position
// always has its inputs.  Every wait is bounded: a timeout sets
// Reduce::error and the kernel gives up.  The dq-independent MXDQ_STD
// factors were computed by the residual pass.
// ---------------------------------------------------------------------------

// Ghost-cell dq of a boundary face from the owner's forward dq dl
// (SetGhostDQLUSGS, NSSolverUnstruct.cpp:14767-14810; SetSymmBCGhostDQLUSGS
// :14812-14915; SetWallBCGhostDQLUSGS :14917-15006; far field 0).  The
// dq-independent terms of the symmetry ghost (the owner's conservative state
// Q, p_ghost / (gamma - 1), rho |u|^2 of the ghost) were formed before the
// wait by ghost_static.
template <class T>
struct GhostStatic {
    T Q[5];
    T pmg, rmu2;
};

template <class T>
__device__ __forceinline__ void ghost_static(const T *ql, const T *qg, T gm, GhostStatic<T> &s)
{
    const T r = ql[0], u = ql[1], v = ql[2], ww = ql[3], pp = ql[4];
    const T em = idiv(idiv(pp, r), gm - T(1)) + T(0.5) * (u * u + v * v + ww * ww);
    s.Q[0] = r; s.Q[1] = r * u; s.Q[2] = r * v; s.Q[3] = r * ww; s.Q[4] = r * em;
    const T rm = qg[0], um = qg[1], vm = qg[2], wm = qg[3], pm = qg[4];
    s.pmg = idiv(pm, gm - T(1));
    s.rmu2 = rm * (um * um + vm * vm + wm * wm);
}

template <class T>
__device__ __forceinline__ void ghost_dq(int kind, T xn, T yn, T zn, const GhostStatic<T> &s, const T *dl, T *o)
{
#pragma unroll
    for (int k = 0; k < 5; ++k) o[k] = T(0);
    if (kind == BK_SYMMETRY) {
        T Q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) Q[k] = s.Q[k] + dl[k];
        o[0] = dl[0];
        T rvn = T(2) * (xn * dl[1] + yn * dl[2] + zn * dl[3]);
        o[1] = dl[1] - xn * rvn;
        o[2] = dl[2] - yn * rvn;
        o[3] = dl[3] - zn * rvn;
        rvn = T(2) * (xn * Q[1] + yn * Q[2] + zn * Q[3]);
        const T ru = Q[1] - xn * rvn, rv = Q[2] - yn * rvn, rw = Q[3] - zn * rvn;
        const T rq0 = idiv(T(1), Q[0]);   // one division on the sweep's critical path, not two
        const T pnew = Q[4] - T(0.5) * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) * rq0;
        o[4] = pnew - s.pmg + T(0.5) * ((ru * ru + rv * rv + rw * rw) * rq0 - s.rmu2);
    } else if (kind == BK_WALL) {
        o[0] = dl[0]; o[1] = -dl[1]; o[2] = -dl[2]; o[3] = -dl[3]; o[4] = dl[4];
    }
}

// Static inputs of one schedule slot for one lane: the slot, this lane's
// neighbour entry with its face, MXDQ factors and the neighbour's record,
// and (lane 0 of the cell's first slot) the cell's residual record, time step
// and volume.  Loaded into registers one round before the slot is processed,
// so that only the neighbours' dq are waited for.
template <class T>
struct SweepIn {
    int cell, count;   // cell < 0: idle slot; count < 0: second slot of a two-slot cell
    int nb, kind;      // neighbour storage index (-1: no entry); boundary kind of a ghost entry
    T nx, ny, nz, area;
    T cf[4];
    T qn[8];
    T ql[5];           // ghost entries: the owner cell's state
    T cr[8];
    T dt, vol;
};

template <class T, bool kForward>
__device__ __forceinline__ void sweep_load(const DevGrid &g, const Work<T> &w, int2 info, int4 en, int lane,
                                           SweepIn<T> &s)
{
    s.cell = info.x;
    s.count = info.y;
    s.nb = -1;
    s.kind = -1;
    const int nc = g.nCell;
    if (info.x >= 0 && en.x >= 0) {
        s.nb = en.x;
        const int f = en.y & 0x7fffffff;
        const T sgn = en.y < 0 ? T(-1) : T(1);
        double fr[4];
        ld4(g.frec + (size_t)f * kF, fr);
        s.nx = sgn * (T)fr[0]; s.ny = sgn * (T)fr[1]; s.nz = sgn * (T)fr[2]; s.area = (T)fr[3];
        ld4(w.coef + (size_t)en.z * kCoef, s.cf);
        ld8(w.qrec + (size_t)en.x * kQ, s.qn);
        if (!kForward && en.x >= nc) {
            s.kind = ld(g.bkind + (en.x - nc));
            T q8[8];
            ld8(w.qrec + (size_t)info.x * kQ, q8);
#pragma unroll
            for (int k = 0; k < 5; ++k) s.ql[k] = q8[k];
        }
    }
    if (info.x >= 0 && info.y >= 0 && lane == 0) {
        ld8(w.crec + (size_t)info.x * kC, s.cr);
        s.dt = w.dtraw[info.x];
        s.vol = (T)g.xrec[(size_t)info.x * kX + 3];
    }
}

// One schedule slot of a sweep, processed by kSweepLanes lanes (one lane per
// neighbour entry; a cell with more entries spans two adjacent slots, whose
// first slot's lane 0 sums all of them).  The eight slots of a warp run in
// lockstep: the warp polls until every lane's inputs are final, so no slot
// ever spins while a sibling in the same warp is ready to work, and every
// shuffle uses the full warp mask.  s.cell < 0 marks an idle slot (the
// warp's trip count is uniform).
template <class T, bool kForward>
__device__ __forceinline__ bool sweep_position(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red,
                                               double mindt, const SweepIn<T> &s, int lane, int base)
{
    const int nc = g.nCell;
    const int cell = s.cell;
    const bool live = cell >= 0;
    const bool lead = live && s.count >= 0;   // the cell's first slot
    const int e1 = lead ? s.count : 0;
    const bool has = live && s.nb >= 0;
    // wait for the inputs other positions write: the neighbour's dq (forward:
    // its forward dq; backward: its final dq; a boundary ghost's comes from
    // this cell's forward dq) and, backward, this cell's forward delta flux.
    // An interface ghost holds the neighbouring zone's forward dq, set by the
    // halo exchange between the sweeps (SetGhostDQLUSGS leaves it to
    // CommunicationDQ, Controller.cpp:1917-1924).
    const bool ghost = !kForward && has && s.nb >= nc;
    const bool itfGhost = ghost && s.kind == BK_INTERFACE;
    const T *src1 = !has ? nullptr
                         : (ghost && !itfGhost) ? w.dqfwd + (size_t)cell * kD
                                                : (kForward || itfGhost ? w.dqfwd : w.dqrec) + (size_t)s.nb * kD;
    const T *src2 = (!kForward && lead && lane == 0) ? w.dflux + (size_t)cell * kD : nullptr;
    T v1[5], fl[5];
    bool r1 = !src1 || poll5(src1, v1);
    bool r2 = !src2 || poll5(src2, fl);
    const T gm = (T)c.gama;
    // dq-independent terms, formed while the first poll is in flight:
    // the reciprocal of the diagonal (NSSolverUnstruct.cpp:15867-15935),
    // 1 / (dt' / vol) + spectral radii, dt' = min(dt, ktmax min dt)
    // (ReduceMaxTimeStep, :5717-5745) -- formed by the residual pass for the
    // raw dt, here only where the clamp applies -- and the symmetry ghost's
    // static terms.  dq is then (res - flux) times the reciprocal: IEEE
    // divisions after the wait held the publishing lanes for up to 2 us
    // (per-cell timestamps), on the critical path of every level.
    T rd = T(1);
    if (lead && lane == 0) {
        const T clamp = (T)(c.ktmax * mindt);
        if (c.ktmax > 0 && s.dt > clamp) {
            // the clamp applies: the residual pass's reciprocal is for the raw dt
            const T dt = idiv(clamp, s.vol);
            T d = idiv(T(1), dt);
            d += s.cr[6];
            if (c.viscous) d += s.cr[7];
            rd = idiv(T(1), d);
        } else {
            rd = s.cr[5];
        }
    }
    GhostStatic<T> gs;
    if (ghost && s.kind == BK_SYMMETRY) ghost_static<T>(s.ql, s.qn, gm, gs);
    // fault injection (phx_fault_hold_cell): the held cell's lead lane waits on
    // nothing that is ever set, so its wait runs out
    if (kForward && lead && lane == 0 && cell == c.holdCell) r2 = false;
    long long spins = 0;
    while (!__all_sync(0xffffffffu, r1 && r2)) {
        ++spins;
        if (spins > c.spinLimit) {
            if ((threadIdx.x & 31) == 0) atomicExch(&red->error, PHX_ERR_TIMEOUT);
            return false;
        }
        if ((spins & 1023) == 0 && __any_sync(0xffffffffu, ((volatile int *)&red->error)[0] != 0)) return false;
        if (spins > 8) __nanosleep(20);
        if (!r1) r1 = poll5(src1, v1);
        if (!r2 && src2) r2 = poll5(src2, fl);
    }
    T df[5] = {0, 0, 0, 0, 0};
    if (has) {
        T dq[5];
        if (ghost && !itfGhost) {
            ghost_dq<T>(s.kind, s.nx, s.ny, s.nz, gs, v1, dq);
        } else {
#pragma unroll
            for (int k = 0; k < 5; ++k) dq[k] = v1[k];
        }
        const T nx = s.nx, ny = s.ny, nz = s.nz, area = s.area;
        const T um = s.qn[1], vm = s.qn[2], wm = s.qn[3], c2 = s.qn[5], hm = s.qn[6];
        const T *cf = s.cf;
        const T cits = nx * um + ny * vm + nz * wm;
        const T dc = cits * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
        const T c2dc = c2 * dc;
        const T v2 = um * um + vm * vm + wm * wm;
        const T g1 = gm - T(1);
        T dh = -g1 * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
        dh += T(0.5) * g1 * v2 * dq[0];
        const T a = dh * cf[1] + dc * cf[2];
        const T b = c2dc * cf[1] + dh * cf[2];
        df[0] = (cf[0] * dq[0] - a) * area;
        df[1] = (cf[0] * dq[1] - um * a + nx * b) * area;
        df[2] = (cf[0] * dq[2] - vm * a + ny * b) * area;
        df[3] = (cf[0] * dq[3] - wm * a + nz * b) * area;
        df[4] = (cf[0] * dq[4] - hm * a + cits * b) * area;
        if (c.viscous) {
            // viscous part of the delta flux (SolveLUSGSForward, :15339-15357)
#pragma unroll
            for (int m = 0; m < 5; ++m) df[m] -= cf[3] * dq[m];
        }
    }
    // in-order accumulation (entries are in the cell's face order; lanes
    // past the cell's entry count are skipped); the second slot's lanes only
    // when the warp holds a two-slot cell
    T rhs0[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kSweepLanes; ++k) {
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const T v = __shfl_sync(0xffffffffu, df[m], base + k);
            if (k < e1) rhs0[m] += v;
        }
    }
    if (__any_sync(0xffffffffu, e1 > kSweepLanes)) {
#pragma unroll
        for (int k = kSweepLanes; k < kSweepMaxEntries; ++k) {
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const T v = __shfl_sync(0xffffffffu, df[m], (base + k) & 31);
                if (k < e1) rhs0[m] += v;
            }
        }
    }
    if (lead && lane == 0) {
        T o[5];
        if (kForward) {
            // dq = (res - Ux - L dq) / D, Ux = 0 for a single sweep
            // (LUSGSInitialization, Controller.cpp:1765-1777)
            T fo[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) { o[k] = (s.cr[k] - T(0) - rhs0[k]) * rd; fo[k] = T(0) + rhs0[k]; }
            publish5(w.dflux + (size_t)cell * kD, fo);
            publish5(w.dqfwd + (size_t)cell * kD, o);
        } else {
#pragma unroll
            for (int k = 0; k < 5; ++k) o[k] = (s.cr[k] - fl[k] - rhs0[k]) * rd;
            publish5(w.dqrec + (size_t)cell * kD, o);
        }
    }
    return true;
}

// One sweep over the schedule: rounds of ngroups positions.  The entries
// ({cell, count} and this lane's neighbour entry) are loaded two rounds
// ahead and the records they point to one round ahead (into registers, and
// into L2 a round before that), so a position starts by polling.
template <class T, bool kForward>
__device__ __forceinline__ bool sweep_all(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red,
                                          double mindt, int group, int wgroup0, int ngroups, int lane, int base)
{
    const int npos = kForward ? g.nFwdPos : g.nBwdPos;
    const int2 *pinfo = kForward ? g.fwd_pinfo : g.bwd_pinfo;
    const int4 *ent = kForward ? g.fwd_ent : g.bwd_ent;
    auto entry = [&](int p, int2 &info, int4 &en) {
        info = make_int2(-1, 0);
        en = make_int4(-1, 0, 0, 0);
        if (p < npos) { info = __ldg(pinfo + p); en = __ldg(ent + (size_t)p * kSweepLanes + lane); }
    };
    int p = group;
    int2 info;
    int4 en;
    entry(p, info, en);
    SweepIn<T> cur;
    sweep_load<T, kForward>(g, w, info, en, lane, cur);
    entry(p + ngroups, info, en);   // entries of the next round
    for (int p0 = wgroup0; p0 < npos; p0 += ngroups) {
        SweepIn<T> nxt;
        sweep_load<T, kForward>(g, w, info, en, lane, nxt);
        entry(p + 2 * ngroups, info, en);
        if (!sweep_position<T, kForward>(g, c, w, red, mindt, cur, lane, base)) return false;
        // the records of the round after next into L2 (its entries have arrived)
        if (en.x >= 0) {
            prefetch_l2(g.frec + (size_t)(en.y & 0x7fffffff) * kF);
            prefetch_l2(w.coef + (size_t)en.z * kCoef);
            prefetch_l2(w.qrec + (size_t)en.x * kQ);
        }
        if (lane == 0 && info.x >= 0 && info.y >= 0) {
            prefetch_l2(w.crec + (size_t)info.x * kC);
            prefetch_l2(w.dtraw + info.x);
        }
        cur = nxt;
        p += ngroups;
    }
    return true;
}

template <class T>
__global__ void __launch_bounds__(kSweepThreads) lusgs_kernel(DevGrid g, NsConst c, Work<T> w, Reduce *red,
                                                              int sweeps)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = tid / kSweepLanes, lane = tid % kSweepLanes;   // slot lane group
    const int ngroups = (gridDim.x * blockDim.x) / kSweepLanes;
    const int wgroup0 = group & ~(kSweepSlots - 1);   // first group of this warp
    const int base = (threadIdx.x & 31) & ~(kSweepLanes - 1);
    const double mindt = __longlong_as_double((long long)red->mindt_bits);
    if ((sweeps & kSweepForward) && !sweep_all<T, true>(g, c, w, red, mindt, group, wgroup0, ngroups, lane, base))
        return;
    if (sweeps & kSweepBackward) sweep_all<T, false>(g, c, w, red, mindt, group, wgroup0, ngroups, lane, base);
}

// Fills the sweep's output records (forward dq, forward delta flux, final dq)
// with the sentinel: 8-element records, 16-byte stores.
template <class T>
__global__ void __launch_bounds__(kThreads) sweep_reset_kernel(int n, T *a, T *b, T *c)
{
    const T s = sweep_sentinel<T>();
    const long long tot = (long long)n * kD;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i * 4 < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const T v[4] = {s, s, s, s};
        st4(a + i * 4, v);
        st4(b + i * 4, v);
        st4(c + i * 4, v);
    }
}

// Grid of the sweeps: every resident lane group (cooperative launch), at most
// one group per schedule position.
template <class K>
static int sweep_blocks(K kernel, int &perSM, const DevGrid &g, int numSMs)
{
    if (perSM < 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, kSweepThreads, 0);
        if (perSM < 1) perSM = 1;
    }
    int blocks = numSMs * perSM;
    const int npos = g.nFwdPos > g.nBwdPos ? g.nFwdPos : g.nBwdPos;
    const int need = (int)(((long long)npos * kSweepLanes + kSweepThreads - 1) / kSweepThreads);
    if (blocks > need) blocks = need;
    // PHX_LUSGS_MAX_BLOCKS caps the grid (tuning; tests of many positions per group)
    if (const char *cap = getenv("PHX_LUSGS_MAX_BLOCKS")) {
        const int v = atoi(cap);
        if (v > 0 && blocks > v) blocks = v;
    }
    return blocks < 1 ? 1 : blocks;
}

template <class T>
int launch_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, int numSMs, cudaStream_t s,
                 int sweeps)
{
    // residency of the cooperative launch, per device (a process may drive several)
    static int perSMcache[kMaxDevices][2];
    static bool init = false;
    if (!init) {
        for (auto &d : perSMcache) d[0] = d[1] = -1;
        init = true;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
    const int blocks = sweep_blocks(lusgs_kernel<T>, perSMcache[dev][sizeof(T) == 8 ? 0 : 1], g, numSMs);
    const long long quads = (long long)g.nCell * kD / 4;
    const int rb = (int)std::min<long long>((quads + kThreads - 1) / kThreads, (long long)numSMs * 16);
    if (sweeps & kSweepForward)
        sweep_reset_kernel<T><<<rb > 0 ? rb : 1, kThreads, 0, s>>>(g.nCell, w.dqfwd, w.dflux, w.dqrec);
    DevGrid gg = g;
    NsConst cc = c;
    Work<T> ww = w;
    Reduce *rr = red;
    int sw = sweeps;
    void *args[] = {&gg, &cc, &ww, &rr, &sw};
    const cudaError_t e =
        cudaLaunchCooperativeKernel((void *)lusgs_kernel<T>, dim3(blocks), dim3(kSweepThreads), args, 0, s);
    return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// Update (NSSolverUnstruct::UpdateFlowField, NSSolverUnstruct.cpp:14587-14765):
// Q_cons (FP64, from the FP64 master primitive state) += dq, back to
// primitive.  Cells whose density or pressure drop below 1e-6 of the free
// stream are listed for the ordered SolutionFix pass.  Also reduces the
// residual monitor sum res_m^2 in FP64 (Residual.cpp:534-600).  q_old is read
// and q_new written (ghosts copied), so the repair pass can see the
// pre-update state of neighbours that come later in the reference's order,
// as the in-place sequential loop of the reference does.
// ---------------------------------------------------------------------------
// Cells the ordered repair pass takes per iteration; more than that means the
// run has diverged: the pass sets PHX_ERR_NUMERIC and leaves the state alone.
static constexpr int kMaxNeg = 4096;

template <class T>
__global__ void __launch_bounds__(kThreads) update_kernel(DevGrid g, NsConst c, Work<T> w, const double *qo,
                                                          double *qn, Reduce *red, int *neglist)
{
    const int nt = g.nTotal, nc = g.nCell;
    const int n = nc > g.nBFace ? nc : g.nBFace;
    const double gm = c.gama;
    double rs[5] = {0, 0, 0, 0, 0};
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < n; cell += gridDim.x * blockDim.x) {
        if (cell < nc) {
            const double r = qo[cell], u = qo[nt + cell], v = qo[2 * nt + cell], ww = qo[3 * nt + cell],
                         p = qo[4 * nt + cell];
            const double em = (p / r) / (gm - 1.0) + 0.5 * (u * u + v * v + ww * ww);
            double Q[5] = {r, r * u, r * v, r * ww, r * em};
            T dq[8];
            ld8(w.dqrec + (size_t)cell * kD, dq);
#pragma unroll
            for (int k = 0; k < 5; ++k) Q[k] += (double)dq[k];
            double prim[5];
            if (Q[0] <= 0.0) {
                prim[0] = Q[0]; prim[1] = u; prim[2] = v; prim[3] = ww; prim[4] = p;
            } else {
                const double od = 1.0 / Q[0];
                const double um = Q[1] * od, vm = Q[2] * od, wm = Q[3] * od;
                const double ie = Q[4] - 0.5 * Q[0] * (um * um + vm * vm + wm * wm);
                prim[0] = Q[0]; prim[1] = um; prim[2] = vm; prim[3] = wm; prim[4] = (gm - 1.0) * ie;
            }
            if (prim[0] < 1.0e-6 * c.primInf[0] || prim[4] < 1.0e-6 * c.primInf[4]) {
                const int slot = atomicAdd(&red->negcount, 1);
                if (slot < kMaxNeg) neglist[slot] = cell;
            }
            T t[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                qn[k * nt + cell] = prim[k];
                t[k] = (T)prim[k];
            }
            put_state<T>(w.qrec + (size_t)cell * kQ, t, (T)gm);
            T cr[8];
            ld8(w.crec + (size_t)cell * kC, cr);
#pragma unroll
            for (int k = 0; k < 5; ++k) rs[k] += (double)cr[k] * (double)cr[k];
        }
        if (cell < g.nBFace) {
            const int gc = nc + cell;
#pragma unroll
            for (int k = 0; k < 5; ++k) qn[k * nt + gc] = qo[k * nt + gc];
        }
    }
    // residual monitor sums: warp shuffle, then one FP64 atomic per block and variable
    __shared__ double part[kThreads / 32][5];
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = rs[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (ln == 0) part[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) v += part[i][threadIdx.x];
        if (v != 0.0) atomicAdd(&red->resnorm[threadIdx.x], v);
    }
}

template <class T>
void launch_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new,
                   Reduce *red, int *neglist, int numSMs, cudaStream_t s)
{
    const int n = g.nCell > g.nBFace ? g.nCell : g.nBFace;
    int blocks = (n + kThreads - 1) / kThreads;
    if (blocks > numSMs * 8) blocks = numSMs * 8;
    update_kernel<T><<<blocks, kThreads, 0, s>>>(g, c, w, q64, q64_new, red, neglist);
}

// SolutionFix (NSSolverUnstruct.cpp:14509-14585) for the listed cells, in the
// reference's cell order: neighbour averages of rho,u,v,w,p (|rho|, |p|),
// neighbours earlier in the reference's order taken after their update,
// later ones before.  One block: the list (at most kMaxNeg cells; empty in
// healthy runs) is sorted by reference number with a bitonic sort in shared
// memory, then one thread repairs the cells in that order.
static constexpr int kFixThreads = 1024;

template <class T>
__global__ void __launch_bounds__(kFixThreads) solution_fix_kernel(DevGrid g, NsConst c, Work<T> w, const double *qo,
                                                                   double *qn, Reduce *red, int *neglist)
{
    __shared__ int key[kMaxNeg], val[kMaxNeg];
    const int n = red->negcount;
    if (n <= 0) return;
    if (n > kMaxNeg) {
        if (threadIdx.x == 0) red->error = PHX_ERR_NUMERIC;
        return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int v = i < n ? neglist[i] : -1;
        key[i] = i < n ? g.orig[v] : 0x7fffffff;
        val[i] = v;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    if ((key[i] > key[l]) == up) {
                        const int tk = key[i]; key[i] = key[l]; key[l] = tk;
                        const int tv = val[i]; val[i] = val[l]; val[l] = tv;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;
    const int nt = g.nTotal;
    const double rlim = 1.0e-6 * c.primInf[0], plim = 1.0e-6 * c.primInf[4];
    for (int i = 0; i < n; ++i) {
        const int cell = val[i];
        const int oc = key[i];
        double acc[5] = {0, 0, 0, 0, 0}, wsum = 0.0;
        for (int j = g.c2f_off[cell]; j < g.c2f_off[cell + 1]; ++j) {
            const int f = g.c2f[j];
            const int2 lr = g.lr[f];
            const int nb = (cell == lr.x) ? lr.y : lr.x;
            const double *src = (g.orig[nb] < oc) ? qn : qo;
            if (src[nb] < rlim || src[4 * nt + nb] < plim) continue;
            wsum += 1.0;
            for (int k = 0; k < 5; ++k) {
                double fv = src[k * nt + nb];
                if (k == 0 || k == 4) fv = fabs(fv);
                acc[k] += fv;
            }
        }
        double prim[5];
        if (wsum > 0.0) { const double o = 1.0 / wsum; for (int k = 0; k < 5; ++k) prim[k] = acc[k] * o; }
        else for (int k = 0; k < 5; ++k) prim[k] = c.primInf[k];
        T t[5];
        for (int k = 0; k < 5; ++k) { qn[k * nt + cell] = prim[k]; t[k] = (T)prim[k]; }
        put_state<T>(w.qrec + (size_t)cell * kQ, t, (T)c.gama);
    }
}

template <class T>
void launch_solution_fix(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new,
                         Reduce *red, int *neglist, cudaStream_t s)
{
    solution_fix_kernel<T><<<1, kFixThreads, 0, s>>>(g, c, w, q64, q64_new, red, neglist);
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference order (API) and storage order.
// ---------------------------------------------------------------------------
template <class T>
__global__ void export_kernel(DevGrid g, const T *rec, int stride, int first, int count, int step, int n, double *out,
                              int outLen)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = g.orig[i];
    for (int k = 0; k < count; ++k) out[(size_t)k * outLen + o] = (double)rec[(size_t)i * stride + first + k * step];
}

template <class T>
void launch_export(const DevGrid &g, const T *rec, int stride, int first, int count, int step, int n, double *out,
                   int outLen, cudaStream_t s)
{
    export_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, rec, stride, first, count, step, n, out,
                                                                       outLen);
}

__global__ void import_q_kernel(DevGrid g, const double *in, double *q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nTotal) return;
    const int o = g.orig[i], nt = g.nTotal;
    for (int k = 0; k < 5; ++k) q[(size_t)k * nt + i] = in[(size_t)k * nt + o];
}

__global__ void export_q_kernel(DevGrid g, const double *q, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nTotal) return;
    const int o = g.orig[i], nt = g.nTotal;
    for (int k = 0; k < 5; ++k) out[(size_t)k * nt + o] = q[(size_t)k * nt + i];
}

void launch_import_q(const DevGrid &g, const double *in, double *q64, cudaStream_t s)
{
    import_q_kernel<<<(g.nTotal + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, in, q64);
}

void launch_export_q(const DevGrid &g, const double *q64, double *out, cudaStream_t s)
{
    export_q_kernel<<<(g.nTotal + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, q64, out);
}

static __global__ void reset_reduce_kernel(Reduce *r)
{
    r->mindt_bits = 0x7FEFFFFFFFFFFFFFULL;  // largest finite double
    for (int k = 0; k < 5; ++k) r->resnorm[k] = 0.0;
    r->negcount = 0;
}

static __global__ void finish_step_kernel(Reduce *r, double *hist, int i, double ncell)
{
    const double v = sqrt(r->resnorm[0] / ncell);
    if ((!(v == v) || v > 1.0e300) && r->error == 0) r->error = PHX_ERR_NUMERIC;
    if (hist) hist[i] = v;
}

// Residual monitor of the current residual record: out[m] += sum_c res_m^2
// (FP64; block sums, one atomic per block and equation; out zeroed first).
template <class T>
__global__ void __launch_bounds__(kThreads) resnorm_kernel(DevGrid g, Work<T> w, double *out)
{
    double s[5] = {0, 0, 0, 0, 0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.nCell; c += gridDim.x * blockDim.x) {
        T cr[8];
        ld8(w.crec + (size_t)c * kC, cr);
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] += (double)cr[k] * (double)cr[k];
    }
    __shared__ double part[kThreads / 32][5];
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (ln == 0) part[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) v += part[i][threadIdx.x];
        if (v != 0.0) atomicAdd(out + threadIdx.x, v);
    }
}

template <class T>
void launch_resnorm(const DevGrid &g, const Work<T> &w, double *out, int numSMs, cudaStream_t s)
{
    cudaMemsetAsync(out, 0, sizeof(double) * 5, s);
    int blocks = (g.nCell + kThreads - 1) / kThreads;
    if (blocks > numSMs * 8) blocks = numSMs * 8;
    resnorm_kernel<T><<<blocks, kThreads, 0, s>>>(g, w, out);
}
template void launch_resnorm<double>(const DevGrid &, const Work<double> &, double *, int, cudaStream_t);
template void launch_resnorm<float>(const DevGrid &, const Work<float> &, double *, int, cudaStream_t);

void launch_reset_reduce(Reduce *r, cudaStream_t s) { reset_reduce_kernel<<<1, 1, 0, s>>>(r); }
void launch_finish_step(Reduce *r, double *hist, int i, double ncell, cudaStream_t s)
{
    finish_step_kernel<<<1, 1, 0, s>>>(r, hist, i, ncell);
}

// Explicit instantiations for the FP64 and mixed paths.
#define PHX_INSTANTIATE(T)                                                                                         \
    template void launch_boundary<T>(const DevGrid &, const NsConst &, double *, const Work<T> &, cudaStream_t);   \
    template void launch_gradient_limiter<T>(const DevGrid &, const NsConst &, const Work<T> &, int, cudaStream_t); \
    template void launch_residual<T>(const DevGrid &, const NsConst &, const Work<T> &, Reduce *, double,           \
                                     cudaStream_t);                                                                 \
    template int launch_lusgs<T>(const DevGrid &, const NsConst &, const Work<T> &, Reduce *, int, cudaStream_t,   \
                                 int);                                                                             \
    template void launch_boundary_post<T>(const DevGrid &, const NsConst &, double *, const Work<T> &,           \
                                          cudaStream_t);                                                            \
    template void launch_update<T>(const DevGrid &, const NsConst &, const Work<T> &, const double *, double *,     \
                                   Reduce *, int *, int, cudaStream_t);                                             \
    template void launch_solution_fix<T>(const DevGrid &, const NsConst &, const Work<T> &, const double *,         \
                                         double *, Reduce *, int *, cudaStream_t);                                  \
    template void launch_sync_qrec<T>(const DevGrid &, const NsConst &, const double *, const Work<T> &,            \
                                      cudaStream_t);                                                                \
    template void launch_export<T>(const DevGrid &, const T *, int, int, int, int, int, double *, int, cudaStream_t);
PHX_INSTANTIATE(double)
PHX_INSTANTIATE(float)

}  // namespace phx
