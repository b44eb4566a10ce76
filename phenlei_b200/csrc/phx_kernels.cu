// sm_100a kernels of the NS per-iteration path.
//
// Every kernel is owner-computes over cells: a cell gathers from its faces in
// ascending face order (the order LoadFlux and the Green-Gauss loop of the
// reference accumulate in), so no atomics touch the state and the FP64 path
// reproduces the reference's summation order.  Face metrics stay FP64; the
// working state T is double (FP64 path) or float (mixed path).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "phx_internal.h"
#include "phx_physics.cuh"

namespace phx {

static constexpr int kThreads = 256;

template <class T> __device__ __forceinline__ T ld(const T *p) { return __ldg(p); }
// Loads of data written earlier in the same kernel by other blocks: bypass L1.
template <class T> __device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// Boundary: ghost-cell state per boundary face (NSSolverUnstruct::Boundary,
// NSSolverUnstruct.cpp:13404-13515): SymmetryBCRegion (:19413),
// ViscousAdiabaticWallBCRegion (:20988), FarfieldBCRegion (:21195).
// Computed in FP64 from the FP64 master state.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) boundary_kernel(DevGrid g, NsConst c, double *q, T *qw, T *c2o, T *hmo)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nBFace) return;
    const int nt = g.nTotal;
    const int le = g.left[f], re = g.nCell + f;
    double r = q[le], u = q[nt + le], v = q[2 * nt + le], w = q[3 * nt + le], p = q[4 * nt + le];
    double xn = g.xfn[f], yn = g.yfn[f], zn = g.zfn[f];
    double o[5] = {r, u, v, w, p};
    int kind = g.bkind[f];
    if (kind == BK_SYMMETRY) {
        double vn = xn * u + yn * v + zn * w;
        o[1] = u - 2.0 * xn * vn;
        o[2] = v - 2.0 * yn * vn;
        o[3] = w - 2.0 * zn * vn;
    } else if (kind == BK_WALL) {
        o[1] = -u; o[2] = -v; o[3] = -w;
    } else if (kind == BK_FARFIELD) {
        const double *pi = c.primInf;
        double rO = pi[0], uO = pi[1], vO = pi[2], wO = pi[3], pO = pi[4];
        double gl = c.gama;
        double cO = sqrt(fabs(gl * pO / rO));
        double vnO = xn * uO + yn * vO + zn * wO;
        double vnI = xn * u + yn * v + zn * w;
        double cI = sqrt(fabs(gl * p / r));
        double gm1 = gl - 1.0;
        double velI = sqrt(u * u + v * v + w * w);
        if (velI > cI) {
            if (vnI < 0.0) { for (int k = 0; k < 5; ++k) o[k] = pi[k]; }
        } else {
            double Rp = vnI + 2.0 * cI / gm1;
            double Rm = vnO - 2.0 * cO / gm1;
            double vnB = 0.5 * (Rp + Rm);
            double cB = 0.25 * (Rp - Rm) * gm1;
            double s, vtx, vty, vtz;
            if (vnB >= 0.0) {
                s = p / pow(r, gl);
                vtx = u - xn * vnI; vty = v - yn * vnI; vtz = w - zn * vnI;
            } else {
                s = pO / pow(rO, gl);
                vtx = uO - xn * vnO; vty = vO - yn * vnO; vtz = wO - zn * vnO;
            }
            double rB = pow((cB * cB / (s * gl)), 1.0 / gm1);
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
        if ((void *)qw != (void *)q) qw[k * nt + re] = t[k];
    }
    // squared sound speed and total enthalpy of the ghost for the LU-SGS sweep
    const T gm = (T)c.gama;
    c2o[re] = fabs(gm * t[4] / t[0]);
    hmo[re] = (gm / (gm - T(1))) * (t[4] / t[0]) + T(0.5) * (t[1] * t[1] + t[2] * t[2] + t[3] * t[3]);
}

template <class T>
void launch_boundary(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s)
{
    if (g.nBFace == 0) return;
    boundary_kernel<T><<<(g.nBFace + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, q64, w.qw, w.c2, w.hm);
}

// ---------------------------------------------------------------------------
// Gradient + limiter, fused per cell:
//  Green-Gauss cell gradient (UnstructGrid::CompGradientGGCell,
//  Geo_UnstructGrid.cpp:3220-3284) of the 5 primitives; then the scalar
//  Venkatakrishnan limiter from rho and p (Limiter::VencatLimiter7,
//  Limiter.cpp:1091-1200, neighbour min/max of Limiter::MinMaxDiff
//  :1202-1252 over interior faces), zeroed next to far-field boundaries
//  (SetLimitBoundary, Geo_UnstructGrid.cpp:10744-10775).
// ---------------------------------------------------------------------------
// Cells are processed by groups of kLanes lanes; lane k takes the k-th face of
// the cell's ascending face list, and lane 0 adds the lanes' terms in face
// order, so sums keep the reference's accumulation order.
static constexpr int kLanes = 8;

template <class T>
__global__ void __launch_bounds__(kThreads) gradient_limiter_kernel(DevGrid g, NsConst c, Work<T> w)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int cell = tid / kLanes, lane = tid % kLanes;
    const int base = (threadIdx.x & 31) & ~(kLanes - 1);
    const unsigned full = 0xffffffffu;
    const int nt = g.nTotal, nc = g.nCell;
    const bool valid = cell < nc;
    const T *q = w.qw;
    int j0 = 0, j1 = 0;
    if (valid) { j0 = g.c2f_off[cell]; j1 = g.c2f_off[cell + 1]; }
    const int j = j0 + lane;
    const bool act = valid && j < j1;
    T qc[5] = {0, 0, 0, 0, 0};
    if (valid) {
#pragma unroll
        for (int k = 0; k < 5; ++k) qc[k] = q[k * nt + cell];
    }
    // this lane's face: signed contributions qf * n A, neighbour rho and p
    T cx[5] = {0, 0, 0, 0, 0}, cy[5] = {0, 0, 0, 0, 0}, cz[5] = {0, 0, 0, 0, 0};
    T rn = qc[0], pn = qc[4];
    int f = 0;
    bool interior = false, isLeft = true;
    if (act) {
        f = ld(g.c2f + j);
        const int le = ld(g.left + f);
        isLeft = (le == cell);
        const int nb = isLeft ? (f < g.nBFace ? nc + f : ld(g.right + f)) : le;
        const double a = ld(g.area + f);
        const T nx = (T)(ld(g.xfn + f) * a), ny = (T)(ld(g.yfn + f) * a), nz = (T)(ld(g.zfn + f) * a);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const T qn = q[k * nt + nb];
            const T qf = T(0.5) * (isLeft ? (qc[k] + qn) : (qn + qc[k]));
            cx[k] = qf * nx; cy[k] = qf * ny; cz[k] = qf * nz;
        }
        interior = f >= g.nBFace;
        if (interior) { rn = q[nb]; pn = q[4 * nt + nb]; }
    }
    const unsigned actm = __ballot_sync(full, act);
    const unsigned leftm = __ballot_sync(full, isLeft);
    T gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kLanes; ++k) {
        const int src = base + k;
        const bool on = (actm >> src) & 1u;
        const bool lf = (leftm >> src) & 1u;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const T vx = __shfl_sync(full, cx[m], src), vy = __shfl_sync(full, cy[m], src), vz = __shfl_sync(full, cz[m], src);
            if (on) {
                if (lf) { gx[m] += vx; gy[m] += vy; gz[m] += vz; }
                else { gx[m] -= vx; gy[m] -= vy; gz[m] -= vz; }
            }
        }
    }
    // neighbour min / max of rho and p over interior faces (order-free)
    T rmin = interior ? rn : qc[0], rmax = rmin, pmin = interior ? pn : qc[4], pmax = pmin;
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) {
        rmin = tmin(rmin, __shfl_xor_sync(full, rmin, o));
        rmax = tmax(rmax, __shfl_xor_sync(full, rmax, o));
        pmin = tmin(pmin, __shfl_xor_sync(full, pmin, o));
        pmax = tmax(pmax, __shfl_xor_sync(full, pmax, o));
    }
    rmin = tmin(rmin, qc[0]); rmax = tmax(rmax, qc[0]);
    pmin = tmin(pmin, qc[4]); pmax = tmax(pmax, qc[4]);
    T ovol = T(1);
    if (valid) ovol = T(1) / (T)ld(g.vol + cell);
#pragma unroll
    for (int k = 0; k < 5; ++k) { gx[k] *= ovol; gy[k] *= ovol; gz[k] *= ovol; }
    if (valid && lane == 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            w.grad[(0 * 5 + k) * nc + cell] = gx[k];
            w.grad[(1 * 5 + k) * nc + cell] = gy[k];
            w.grad[(2 * 5 + k) * nc + cell] = gz[k];
        }
    }
    // Venkatakrishnan limiter: every lane holds the group's gradient (each lane
    // accumulated the same terms in the same order)
    T lim = T(1);
    if (c.limiter == 1 && act) {
        const T vp = (T)ld(g.volpow + cell);
        T er = (T)c.venkatK3 * qc[0]; er = er * qc[0]; er = er * vp;
        T ep = (T)c.venkatK3 * qc[4]; ep = ep * qc[4]; ep = ep * vp;
        const T dminr = rmin - qc[0], dmaxr = rmax - qc[0];
        const T dminp = pmin - qc[4], dmaxp = pmax - qc[4];
        const double xc = ld(g.xcc + cell), yc = ld(g.ycc + cell), zc = ld(g.zcc + cell);
        const T small = (T)kSmall;
        const T dx = (T)(ld(g.xfc + f) - xc), dy = (T)(ld(g.yfc + f) - yc), dz = (T)(ld(g.zfc + f) - zc);
        T d = gx[0] * dx + gy[0] * dy + gz[0] * dz;
        if (d > small) lim = tmin(lim, venfun(dmaxr, d, er));
        else if (d < -small) lim = tmin(lim, venfun(dminr, d, er));
        d = gx[4] * dx + gy[4] * dy + gz[4] * dz;
        if (d > small) lim = tmin(lim, venfun(dmaxp, d, ep));
        else if (d < -small) lim = tmin(lim, venfun(dminp, d, ep));
    }
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) lim = tmin(lim, __shfl_xor_sync(full, lim, o));
    if (valid && lane == 0) {
        if (c.limiter == 1 && g.farfield_adj[cell]) lim = T(0);
        w.limit[cell] = lim;
    }
}

template <class T>
void launch_gradient_limiter(const DevGrid &g, const NsConst &c, const Work<T> &w, cudaStream_t s)
{
    const long long threads = (long long)g.nCell * kLanes;
    gradient_limiter_kernel<T><<<(unsigned)((threads + kThreads - 1) / kThreads), kThreads, 0, s>>>(g, c, w);
}

// ---------------------------------------------------------------------------
// Residual: for every face of the cell, the MUSCL face states
// (GetQlQr / ReConstructFaceValue, NSSolverUnstruct.cpp:5507, :13991-14193),
// the wall / symmetry face fix (BoundaryQlQrFix, :13725-13951), the Roe flux
// times the face area (InviscidFluxWrap, :14466-14488), gathered into res with
// the sign LoadFlux applies (:6435-6495); the inviscid spectral radius
// (SpectrumRadiusInviscid, :5749-5850); and in the epilogue the local time
// step (LocalTimeStep / LimitCFL, :5999-6118) with its device-wide minimum
// (Controller::ComputeMinTimeStep, Controller.cpp:706-752).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void load_side(const DevGrid &g, const Work<T> &w, int cell, int face, T lim, T *qo)
{
    const int nt = g.nTotal, nc = g.nCell;
    T qs[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) qs[k] = w.qw[k * nt + cell];
    if (cell < nc) {
        const T dx = (T)(ld(g.xfc + face) - ld(g.xcc + cell));
        const T dy = (T)(ld(g.yfc + face) - ld(g.ycc + cell));
        const T dz = (T)(ld(g.zfc + face) - ld(g.zcc + cell));
        T tr[5];
#pragma unroll
        for (int k = 0; k < 5; ++k)
            tr[k] = qs[k] + lim * (w.grad[(0 * 5 + k) * nc + cell] * dx + w.grad[(1 * 5 + k) * nc + cell] * dy +
                                   w.grad[(2 * 5 + k) * nc + cell] * dz);
        if (tr[0] > T(0) && tr[4] > T(0)) {
#pragma unroll
            for (int k = 0; k < 5; ++k) qs[k] = tr[k];
        }
    }
    // ghost cells carry a zero gradient (CompGradientGGCell never writes them),
    // so their reconstruction returns the ghost state itself
#pragma unroll
    for (int k = 0; k < 5; ++k) qo[k] = qs[k];
}

template <class T>
__device__ __forceinline__ void face_flux(const DevGrid &g, const NsConst &c, const Work<T> &w, int f, T *fa)
{
    const int nc = g.nCell, nt = g.nTotal;
    const int le = ld(g.left + f);
    const int re = f < g.nBFace ? nc + f : ld(g.right + f);
    T limL = w.limit[le], limR = w.limit[re];
    if (c.reconMethod == 1) { T m = tmin(limL, limR); limL = limR = m; }
    T ql[5], qr[5];
    load_side(g, w, le, f, limL, ql);
    load_side(g, w, re, f, limR, qr);
    const T xn = (T)ld(g.xfn + f), yn = (T)ld(g.yfn + f), zn = (T)ld(g.zfn + f);
    if (f < g.nBFace) {
        const int kind = g.bkind[f];
        const int bt = g.btype[f];
        if (bt == PHX_BC_SOLID_SURFACE || bt == PHX_BC_SYMMETRY) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                T a = T(0.5) * (w.qw[k * nt + le] + w.qw[k * nt + re]);
                ql[k] = a; qr[k] = a;
            }
            if (bt == PHX_BC_SYMMETRY) {
                T vn = T(2) * (xn * ql[1] + yn * ql[2] + zn * ql[3]);
                qr[1] = ql[1] - vn * xn; qr[2] = ql[2] - vn * yn; qr[3] = ql[3] - vn * zn;
            } else if (kind == BK_WALL) {
                ql[1] = ql[2] = ql[3] = T(0);
                qr[1] = qr[2] = qr[3] = T(0);
            }
        }
    }
    const T gm = (T)c.gama;
    roe_flux<T>(ql, qr, gm, gm, xn, yn, zn, (T)c.acoustic, (T)c.convective, fa);
    const T a = (T)ld(g.area + f);
#pragma unroll
    for (int k = 0; k < 5; ++k) fa[k] *= a;
}

template <class T>
__device__ __forceinline__ void lusgs_coef(const T *qc, const T *qn, T nx, T ny, T nz, T area, T gm, T *l1, T *x1,
                                           T *x2);

__device__ __forceinline__ void atomic_min_pos_double(unsigned long long *addr, double v)
{
    atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

template <class T>
__global__ void __launch_bounds__(kThreads) residual_kernel(DevGrid g, NsConst c, Work<T> w, Reduce *red, double cfl)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int cell = tid / kLanes, lane = tid % kLanes;
    const int base = (threadIdx.x & 31) & ~(kLanes - 1);
    const unsigned full = 0xffffffffu;
    const int nt = g.nTotal, nc = g.nCell;
    const bool valid = cell < nc;
    int j0 = 0, j1 = 0;
    if (valid) { j0 = g.c2f_off[cell]; j1 = g.c2f_off[cell + 1]; }
    const int j = j0 + lane;
    const bool act = valid && j < j1;
    T fa[5] = {0, 0, 0, 0, 0};
    T sp = T(0);
    bool isLeft = true;
    if (act) {
        const int f = ld(g.c2f + j);
        const int le = ld(g.left + f);
        isLeft = (le == cell);
        face_flux<T>(g, c, w, f, fa);
        // inviscid spectral radius from the face-mean state
        const int re = f < g.nBFace ? nc + f : ld(g.right + f);
        const T xn = (T)ld(g.xfn + f), yn = (T)ld(g.yfn + f), zn = (T)ld(g.zfn + f);
        const T *q = w.qw;
        T vnl = xn * q[nt + le] + yn * q[2 * nt + le] + zn * q[3 * nt + le];
        T vnr = xn * q[nt + re] + yn * q[2 * nt + re] + zn * q[3 * nt + re];
        T gm = T(0.5) * ((T)c.gama + (T)c.gama);
        T pm = T(0.5) * (q[4 * nt + le] + q[4 * nt + re]);
        T rm = T(0.5) * (q[le] + q[re]);
        T vn = T(0.5) * (vnl + vnr);
        T cm = sqrt(gm * pm / rm);
        const T area = (T)ld(g.area + f);
        sp = T(0.5) * area * (fabs(vn) + cm);
        // LU-SGS factors of the neighbour across this face, as seen from this cell
        const int nbr = isLeft ? re : le;
        const T sg = isLeft ? T(1) : T(-1);
        T qc[5], qn[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) { qc[k] = q[k * nt + cell]; qn[k] = q[k * nt + nbr]; }
        T l1, x1, x2;
        lusgs_coef<T>(qc, qn, sg * xn, sg * yn, sg * zn, area, (T)c.gama, &l1, &x1, &x2);
        w.coef[j] = l1;
        w.coef[g.c2fLen + j] = x1;
        w.coef[2 * g.c2fLen + j] = x2;
    }
    // LoadFlux order: lane 0 adds the faces in ascending face order
    const unsigned actm = __ballot_sync(full, act);
    const unsigned leftm = __ballot_sync(full, isLeft);
    T res[5] = {0, 0, 0, 0, 0};
    T spec = T(0);
#pragma unroll
    for (int k = 0; k < kLanes; ++k) {
        const int src = base + k;
        const bool on = (actm >> src) & 1u;
        const bool lf = (leftm >> src) & 1u;
        T v[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) v[m] = __shfl_sync(full, fa[m], src);
        const T vs = __shfl_sync(full, sp, src);
        if (on) {
            if (lf) {
#pragma unroll
                for (int m = 0; m < 5; ++m) res[m] -= v[m];
            } else {
#pragma unroll
                for (int m = 0; m < 5; ++m) res[m] += v[m];
            }
            spec += vs;
        }
    }
    double mydt = kLarge;
    if (valid && lane == 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k) w.res[k * nc + cell] = res[k];
        w.invspec[cell] = spec;
        if (c.viscous) spec += w.visspec[cell];
        const T *q = w.qw;
        const T gm = (T)c.gama;
        const T r = q[cell], u = q[nt + cell], v = q[2 * nt + cell], ww = q[3 * nt + cell], p = q[4 * nt + cell];
        w.c2[cell] = fabs(gm * p / r);
        w.hm[cell] = (gm / (gm - T(1))) * (p / r) + T(0.5) * (u * u + v * v + ww * ww);
        // LimitCFL: pressure- and skewness-based CFL of the cell
        double cc = cfl;
        const double pc = (double)p;
        const double plo = 0.001 * c.pTotal, phi = 0.02 * c.pTotal;
        if (pc < plo) cc = c.cflStart;
        else if (pc < phi) cc = (pc - phi) * (cfl - c.cflStart) / (phi - plo) + cfl;
        const double sk = ld(g.skew + cell);
        if (sk < 0.1) cc *= 0.1;
        else if (sk < 10.0) cc *= (1.0 - exp(0.0 - sk));
        T dt = (T)cc * (T)ld(g.vol + cell) / spec;
        w.dtraw[cell] = dt;
        mydt = (double)dt;
    }
    // device-wide minimum of dt (positive doubles order like unsigned integers)
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(full, mydt, o));
    if ((threadIdx.x & 31) == 0 && mydt < kLarge) atomic_min_pos_double(&red->mindt_bits, mydt);
}

template <class T>
void launch_residual(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, double cfl, cudaStream_t s)
{
    const long long threads = (long long)g.nCell * kLanes;
    residual_kernel<T><<<(unsigned)((threads + kThreads - 1) / kThreads), kThreads, 0, s>>>(g, c, w, red, cfl);
}

// ---------------------------------------------------------------------------
// LU-SGS (Controller::LUSGS, Controller.cpp:1878-1955): one persistent
// cooperative kernel runs the diagonal, the forward sweep level by level, the
// ghost-cell dq and the backward sweep level by level.  Levels come from the
// reference's own cell order (a cell depends on its face neighbours of lower
// index in the forward sweep, higher index in the backward sweep), so every
// cell sees exactly the neighbour values the sequential sweep of the
// reference sees.  The dq-independent factors of MXDQ_STD (Roe-averaged
// spectral radius, split eigenvalue, weights) were computed by the residual
// pass, so the sequential critical path is multiply-adds only.  Between levels
// a device-wide barrier on a monotonic counter; every wait is bounded (a
// timeout sets Reduce::error and the kernel returns).
// ---------------------------------------------------------------------------
static constexpr long long kSpinLimit = 50000000LL;  // a few seconds of polling
static constexpr int kSweepThreads = 512;

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(Reduce *red, unsigned int &target, int nblocks)
{
    if (nblocks == 1) { __syncthreads(); return true; }
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        target += (unsigned int)nblocks;
        __threadfence();
        atomicAdd(&red->barrier, 1u);
        long long spins = 0;
        while (ld_acquire(&red->barrier) < target) {
            __nanosleep(20);
            if (++spins > kSpinLimit || ((volatile int *)&red->error)[0] != 0) {
                atomicExch(&red->error, PHX_ERR_TIMEOUT);
                ok = 0;
                break;
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

// dq-independent part of the neighbour's MXDQ_STD term for the use (cell ->
// neighbour across face f): Roe-averaged spectral radius (RoeAveragedVariables
// + GetRad, NSSolverUnstruct.cpp:15097-15116, 15297-15313) and the split
// eigenvalue l1 and weights x1, x2 of MXDQ_STD (Jacobian.cpp:27-47).
template <class T>
__device__ __forceinline__ void lusgs_coef(const T *qc, const T *qn, T nx, T ny, T nz, T area, T gm, T *l1, T *x1,
                                           T *x2)
{
    T fp[5];
    roe_average<T>(qc, gm, qn, gm, fp);
    T vn = nx * fp[1] + ny * fp[2] + nz * fp[3];
    T rad = (fabs(vn) + sqrt(gm * fp[4] / fp[0])) * area;
    T c2 = fabs(gm * qn[4] / qn[0]);
    T cm = sqrt(c2);
    T cits = nx * qn[1] + ny * qn[2] + nz * qn[3];
    T ipnrad = -rad / tmax(T(kSmall), area);
    T a1 = T(0.5) * (cits + ipnrad);
    T a2 = T(0.5) * (cits + cm + ipnrad);
    T a3 = T(0.5) * (cits - cm + ipnrad);
    *l1 = a1;
    *x1 = (a1 + a1 - a2 - a3) / (c2 + c2);
    *x2 = (a2 - a3) / (cm + cm);
}

// MXDQ_STD (Jacobian.cpp:48-86) with the precomputed factors.
template <class T>
__device__ __forceinline__ void mxdq_apply(const Work<T> &w, int nt, int nb, T nx, T ny, T nz, T area, T gm, T l1,
                                           T x1, T x2, const T *dq, T *f)
{
    const T um = w.qw[nt + nb], vm = w.qw[2 * nt + nb], wm = w.qw[3 * nt + nb];
    const T c2 = w.c2[nb], hm = w.hm[nb];
    const T cits = nx * um + ny * vm + nz * wm;
    const T dc = cits * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
    const T c2dc = c2 * dc;
    const T v2 = um * um + vm * vm + wm * wm;
    const T g1 = gm - T(1);
    T dh = -g1 * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
    dh += T(0.5) * g1 * v2 * dq[0];
    const T a = dh * x1 + dc * x2;
    const T b = c2dc * x1 + dh * x2;
    f[0] = (l1 * dq[0] - a) * area;
    f[1] = (l1 * dq[1] - um * a + nx * b) * area;
    f[2] = (l1 * dq[2] - vm * a + ny * b) * area;
    f[3] = (l1 * dq[3] - wm * a + nz * b) * area;
    f[4] = (l1 * dq[4] - hm * a + cits * b) * area;
}

// Ghost-cell dq between the sweeps (SetGhostDQLUSGS, NSSolverUnstruct.cpp:14767-14810;
// SetSymmBCGhostDQLUSGS :14812-14915; SetWallBCGhostDQLUSGS :14917-15006; far field 0).
template <class T>
__device__ void ghost_dq(const DevGrid &g, const NsConst &c, const Work<T> &w, int f)
{
    const int nt = g.nTotal, nc = g.nCell;
    const int le = g.left[f], re = nc + f;
    const int kind = g.bkind[f];
    T *dq = w.dq;
    T dl[5];
    for (int k = 0; k < 5; ++k) dl[k] = ldcg(dq + k * nt + le);
    if (kind == BK_SYMMETRY) {
        const T *q = w.qw;
        T r = q[le], u = q[nt + le], v = q[2 * nt + le], ww = q[3 * nt + le], pp = q[4 * nt + le];
        T gm = (T)c.gama;
        T em = (pp / r) / (gm - T(1)) + T(0.5) * (u * u + v * v + ww * ww);
        T Q[5] = {r, r * u, r * v, r * ww, r * em};
        for (int k = 0; k < 5; ++k) Q[k] += dl[k];
        T rm = q[re], um = q[nt + re], vm = q[2 * nt + re], wm = q[3 * nt + re], pm = q[4 * nt + re];
        T xn = (T)g.xfn[f], yn = (T)g.yfn[f], zn = (T)g.zfn[f];
        dq[re] = dl[0];
        T rvn = T(2) * (xn * dl[1] + yn * dl[2] + zn * dl[3]);
        dq[nt + re] = dl[1] - xn * rvn;
        dq[2 * nt + re] = dl[2] - yn * rvn;
        dq[3 * nt + re] = dl[3] - zn * rvn;
        rvn = T(2) * (xn * Q[1] + yn * Q[2] + zn * Q[3]);
        T ru = Q[1] - xn * rvn, rv = Q[2] - yn * rvn, rw = Q[3] - zn * rvn;
        T pnew = Q[4] - T(0.5) * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0];
        T g1 = gm - T(1);
        dq[4 * nt + re] = pnew - pm / g1 + T(0.5) * ((ru * ru + rv * rv + rw * rw) / Q[0] - rm * (um * um + vm * vm + wm * wm));
    } else if (kind == BK_WALL) {
        dq[re] = dl[0];
        dq[nt + re] = -dl[1];
        dq[2 * nt + re] = -dl[2];
        dq[3 * nt + re] = -dl[3];
        dq[4 * nt + re] = dl[4];
    } else {
        for (int k = 0; k < 5; ++k) dq[k * nt + re] = T(0);
    }
}

// A sweep is processed by groups of kGroup lanes, one cell per group: lane k
// takes the k-th face of the cell, computes the neighbour's delta flux if the
// neighbour is on the sweep's side, and lane 0 adds the lanes' terms in face
// order (the reference's order).  All loads that do not depend on dq are
// issued for the next level before the barrier (Slot), so after the barrier
// only the neighbours' dq are read.
static constexpr int kGroup = 8;

template <class T>
struct Slot {
    int cell;          // -1: no cell for this group at this position
    int nb;            // neighbour index, -1 if this lane has no entry
    T nx, ny, nz, area, l1, x1, x2, um, vm, wm, c2, hm;
    T r[5];            // lane 0: res (forward) or res - carried delta flux (backward)
    T diag;            // lane 0
};

// Loads everything the position needs except the neighbours' dq (which the
// previous level produces): issued one level ahead, before the barrier.
template <class T, bool kForward>
__device__ __forceinline__ void load_slot(const DevGrid &g, const Work<T> &w, int level_pos_end, int pos, int lane,
                                          Slot<T> &s)
{
    const int nt = g.nTotal, nc = g.nCell, len = g.c2fLen;
    s.cell = -1;
    s.nb = -1;
    if (pos >= level_pos_end) return;
    const int *cells = kForward ? g.fwd_cells : g.bwd_cells;
    const int *eoff = kForward ? g.fwd_eoff : g.bwd_eoff;
    const int cell = cells[pos];
    s.cell = cell;
    const int e = eoff[pos] + lane;
    if (e < eoff[pos + 1]) {
        const int nb = (kForward ? g.fwd_enb : g.bwd_enb)[e];
        const int fs = (kForward ? g.fwd_ef : g.bwd_ef)[e];
        const int j = (kForward ? g.fwd_ej : g.bwd_ej)[e];
        const int f = fs & 0x7fffffff;
        const T sgn = fs < 0 ? T(-1) : T(1);
        s.nb = nb;
        s.nx = sgn * (T)ld(g.xfn + f);
        s.ny = sgn * (T)ld(g.yfn + f);
        s.nz = sgn * (T)ld(g.zfn + f);
        s.area = (T)ld(g.area + f);
        s.l1 = w.coef[j];
        s.x1 = w.coef[len + j];
        s.x2 = w.coef[2 * len + j];
        s.um = w.qw[nt + nb];
        s.vm = w.qw[2 * nt + nb];
        s.wm = w.qw[3 * nt + nb];
        s.c2 = w.c2[nb];
        s.hm = w.hm[nb];
    }
    if (lane == 0) {
        s.diag = ldcg(w.diag + cell);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            T rv = w.res[k * nc + cell];
            if (!kForward) rv = rv - ldcg(w.dflux + k * nc + cell);
            s.r[k] = kForward ? (rv - T(0)) : rv;
        }
    }
}

template <class T, bool kForward>
__device__ __forceinline__ void process_slot(const DevGrid &g, const NsConst &c, const Work<T> &w, const Slot<T> &s,
                                             int lane)
{
    const unsigned full = 0xffffffffu;
    const int nt = g.nTotal, nc = g.nCell;
    T df[5] = {0, 0, 0, 0, 0};
    const bool active = s.cell >= 0 && s.nb >= 0;
    if (active) {
        T dq[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) dq[k] = ldcg(w.dq + k * nt + s.nb);
        const T gm = (T)c.gama;
        const T cits = s.nx * s.um + s.ny * s.vm + s.nz * s.wm;
        const T dc = cits * dq[0] - s.nx * dq[1] - s.ny * dq[2] - s.nz * dq[3];
        const T c2dc = s.c2 * dc;
        const T v2 = s.um * s.um + s.vm * s.vm + s.wm * s.wm;
        const T g1 = gm - T(1);
        T dh = -g1 * (s.um * dq[1] + s.vm * dq[2] + s.wm * dq[3] - dq[4]);
        dh += T(0.5) * g1 * v2 * dq[0];
        const T a = dh * s.x1 + dc * s.x2;
        const T b = c2dc * s.x1 + dh * s.x2;
        df[0] = (s.l1 * dq[0] - a) * s.area;
        df[1] = (s.l1 * dq[1] - s.um * a + s.nx * b) * s.area;
        df[2] = (s.l1 * dq[2] - s.vm * a + s.ny * b) * s.area;
        df[3] = (s.l1 * dq[3] - s.wm * a + s.nz * b) * s.area;
        df[4] = (s.l1 * dq[4] - s.hm * a + cits * b) * s.area;
    }
    // In-order accumulation on lane 0 of the group.  Entries are compact and in
    // face order, so the active lanes of a group are 0..n-1; the trip count is
    // the warp's maximum (uniform across the warp).
    const unsigned act = __ballot_sync(full, active);
    const int base = (threadIdx.x & 31) & ~(kGroup - 1);
    const int ncnt = __popc((act >> base) & ((1u << kGroup) - 1u));
    const int wmax = __reduce_max_sync(full, (unsigned)ncnt);
    T rhs0[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < wmax; ++k) {
        T v[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) v[m] = __shfl_sync(full, df[m], base + k);
        if (k < ncnt) {
#pragma unroll
            for (int m = 0; m < 5; ++m) rhs0[m] += v[m];
        }
    }
    if (lane == 0 && s.cell >= 0) {
        const int cell = s.cell;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            w.dq[k * nt + cell] = (s.r[k] - rhs0[k]) / s.diag;
            if (kForward) w.dflux[k * nc + cell] = T(0) + rhs0[k];
        }
    }
}

template <class T, bool kForward>
__device__ __forceinline__ bool run_sweep(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red,
                                          unsigned &target, int group, int ngroups, int lane)
{
    const int nlev = kForward ? g.nFwdLevels : g.nBwdLevels;
    const int *off = kForward ? g.fwd_off : g.bwd_off;
    const int warpGroup0 = group - ((threadIdx.x & 31) / kGroup);
    Slot<T> cur, nxt;
    load_slot<T, kForward>(g, w, off[1], off[0] + group, lane, cur);
    for (int L = 0; L < nlev; ++L) {
        const int b = off[L], e = off[L + 1];
        // next level's dq-independent data, in flight while this level runs
        if (L + 1 < nlev) load_slot<T, kForward>(g, w, off[L + 2], off[L + 1] + group, lane, nxt);
        process_slot<T, kForward>(g, c, w, cur, lane);
        // Levels wider than the grid: further rounds, warp-uniform trip count
        // (process_slot uses full-warp collectives).
        for (int round = b + ngroups; round + warpGroup0 < e; round += ngroups) {
            Slot<T> extra;
            load_slot<T, kForward>(g, w, e, round + group, lane, extra);
            process_slot<T, kForward>(g, c, w, extra, lane);
        }
        if (!grid_sync(red, target, gridDim.x)) return false;
        cur = nxt;
    }
    return true;
}

template <class T>
__global__ void __launch_bounds__(kSweepThreads, 1) lusgs_kernel(DevGrid g, NsConst c, Work<T> w, Reduce *red)
{
    const int nc = g.nCell;
    const int stride = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = tid / kGroup, lane = tid % kGroup, ngroups = stride / kGroup;
    unsigned int target = 0;
    const double mindt = __longlong_as_double((long long)red->mindt_bits);

    // Diagonal (NSSolverUnstruct.cpp:15867-15935); single sweep: dq starts
    // from res, the carried delta flux from zero (LUSGSInitialization,
    // Controller.cpp:1765-1777).
    for (int cell = tid; cell < nc; cell += stride) {
        T dt = w.dtraw[cell];
        if (c.ktmax > 0) dt = tmin(dt, (T)(c.ktmax * mindt));
        dt /= (T)g.vol[cell];
        T d = T(1) / dt;
        d += w.invspec[cell];
        if (c.viscous) d += w.visspec[cell];
        w.diag[cell] = d;
    }
    if (!grid_sync(red, target, gridDim.x)) return;
    if (!run_sweep<T, true>(g, c, w, red, target, group, ngroups, lane)) return;
    for (int f = tid; f < g.nBFace; f += stride) ghost_dq<T>(g, c, w, f);
    if (!grid_sync(red, target, gridDim.x)) return;
    run_sweep<T, false>(g, c, w, red, target, group, ngroups, lane);
}

static __global__ void reset_barrier_kernel(Reduce *r) { r->barrier = 0u; }

template <class T>
int launch_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, Reduce *red, int numSMs,
                 cudaStream_t s)
{
    (void)q64;
    static int perSMcache[2] = {-1, -1};
    int &perSM = perSMcache[sizeof(T) == 8 ? 0 : 1];
    if (perSM < 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, lusgs_kernel<T>, kSweepThreads, 0);
        if (perSM < 1) perSM = 1;
    }
    // one group per cell of the widest level; never more blocks than can be co-resident
    const long long threads = (long long)g.maxLevelWidth * kGroup;
    int blocks = (int)((threads + kSweepThreads - 1) / kSweepThreads);
    if (blocks > numSMs * perSM) blocks = numSMs * perSM;
    // PHX_LUSGS_MAX_BLOCKS caps the sweep grid (tuning, and tests of levels
    // wider than the grid on small meshes)
    if (const char *cap = getenv("PHX_LUSGS_MAX_BLOCKS")) {
        const int v = atoi(cap);
        if (v > 0 && blocks > v) blocks = v;
    }
    if (blocks < 1) blocks = 1;
    reset_barrier_kernel<<<1, 1, 0, s>>>(red);
    DevGrid gg = g;
    NsConst cc = c;
    Work<T> ww = w;
    Reduce *rr = red;
    void *args[] = {&gg, &cc, &ww, &rr};
    cudaError_t e = cudaLaunchCooperativeKernel((void *)lusgs_kernel<T>, dim3(blocks), dim3(kSweepThreads), args, 0, s);
    return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// Update (NSSolverUnstruct::UpdateFlowField, NSSolverUnstruct.cpp:14587-14765):
// Q_cons (FP64, from the FP64 master primitive state) += dq, back to
// primitive.  Cells whose density or pressure drop below 1e-6 of the free
// stream are listed for the ordered SolutionFix pass.  Also reduces the
// residual monitor sum res_m^2 in FP64 (Residual.cpp:534-600).
// q_old is read, q_new written (ghosts copied), so the repair pass can see
// the pre-update state of higher-index neighbours as the in-place sequential
// loop of the reference does.
// ---------------------------------------------------------------------------
static constexpr int kMaxNeg = 1 << 16;

template <class T>
__global__ void __launch_bounds__(kThreads) update_kernel(DevGrid g, NsConst c, Work<T> w, const double *qo,
                                                          double *qn, T *qw_out, Reduce *red, int *neglist)
{
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = g.nTotal, nc = g.nCell;
    double rs[5] = {0, 0, 0, 0, 0};
    if (cell < nc) {
        double r = qo[cell], u = qo[nt + cell], v = qo[2 * nt + cell], ww = qo[3 * nt + cell], p = qo[4 * nt + cell];
        const double gm = c.gama;
        double em = (p / r) / (gm - 1.0) + 0.5 * (u * u + v * v + ww * ww);
        double Q[5] = {r, r * u, r * v, r * ww, r * em};
#pragma unroll
        for (int k = 0; k < 5; ++k) Q[k] += (double)w.dq[k * nt + cell];
        double prim[5];
        if (Q[0] <= 0.0) {
            prim[0] = Q[0]; prim[1] = u; prim[2] = v; prim[3] = ww; prim[4] = p;
        } else {
            double od = 1.0 / Q[0];
            double um = Q[1] * od, vm = Q[2] * od, wm = Q[3] * od;
            double ie = Q[4] - 0.5 * Q[0] * (um * um + vm * vm + wm * wm);
            prim[0] = Q[0]; prim[1] = um; prim[2] = vm; prim[3] = wm; prim[4] = (gm - 1.0) * ie;
        }
        if (prim[0] < 1.0e-6 * c.primInf[0] || prim[4] < 1.0e-6 * c.primInf[4]) {
            int slot = atomicAdd(&red->negcount, 1);
            if (slot < kMaxNeg) neglist[slot] = cell;
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            qn[k * nt + cell] = prim[k];
            if ((void *)qw_out != (void *)qn) qw_out[k * nt + cell] = (T)prim[k];
            double rv = (double)w.res[k * nc + cell];
            rs[k] = rv * rv;
        }
    }
    if (cell < g.nBFace) {
        const int gc = nc + cell;
#pragma unroll
        for (int k = 0; k < 5; ++k) qn[k * nt + gc] = qo[k * nt + gc];
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = rs[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&red->resnorm[k], v);
    }
}

template <class T>
void launch_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new, T *qw_out,
                   Reduce *red, int *neglist, cudaStream_t s)
{
    int n = g.nCell > g.nBFace ? g.nCell : g.nBFace;
    update_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, w, q64, q64_new, qw_out, red, neglist);
}

// SolutionFix (NSSolverUnstruct.cpp:14509-14585) for the listed cells, in
// ascending cell order: neighbour averages of rho,u,v,w,p (|rho|, |p|),
// lower-index neighbours taken after their update, higher-index ones before.
// One thread: the list is empty in healthy runs and short otherwise.
template <class T>
__global__ void solution_fix_kernel(DevGrid g, NsConst c, const double *qo, double *qn, T *qw_out, Reduce *red,
                                    int *neglist)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int n = red->negcount;
    if (n <= 0) return;
    if (n > kMaxNeg) { red->error = PHX_ERR_NUMERIC; n = kMaxNeg; }
    for (int i = 1; i < n; ++i) {  // insertion sort (short list)
        int v = neglist[i], j = i - 1;
        while (j >= 0 && neglist[j] > v) { neglist[j + 1] = neglist[j]; --j; }
        neglist[j + 1] = v;
    }
    const int nt = g.nTotal, nc = g.nCell;
    const double rlim = 1.0e-6 * c.primInf[0], plim = 1.0e-6 * c.primInf[4];
    for (int i = 0; i < n; ++i) {
        const int cell = neglist[i];
        double acc[5] = {0, 0, 0, 0, 0}, wsum = 0.0;
        for (int j = g.c2f_off[cell]; j < g.c2f_off[cell + 1]; ++j) {
            const int f = g.c2f[j];
            const int le = g.left[f], re = f < g.nBFace ? nc + f : g.right[f];
            const int nb = (cell == le) ? re : le;
            const double *src = (nb < cell) ? qn : qo;
            if (src[nb] < rlim || src[4 * nt + nb] < plim) continue;
            wsum += 1.0;
            for (int k = 0; k < 5; ++k) {
                double fv = src[k * nt + nb];
                if (k == 0 || k == 4) fv = fabs(fv);
                acc[k] += fv;
            }
        }
        double prim[5];
        if (wsum > 0.0) { double o = 1.0 / wsum; for (int k = 0; k < 5; ++k) prim[k] = acc[k] * o; }
        else for (int k = 0; k < 5; ++k) prim[k] = c.primInf[k];
        for (int k = 0; k < 5; ++k) {
            qn[k * nt + cell] = prim[k];
            if ((void *)qw_out != (void *)qn) qw_out[k * nt + cell] = (T)prim[k];
        }
    }
}

template <class T>
void launch_solution_fix(const DevGrid &g, const NsConst &c, const double *q64, double *q64_new, T *qw_out,
                         Reduce *red, int *neglist, cudaStream_t s)
{
    solution_fix_kernel<T><<<1, 32, 0, s>>>(g, c, q64, q64_new, qw_out, red, neglist);
}

// Explicit instantiations for the FP64 and mixed paths.
#define PHX_INSTANTIATE(T)                                                                                      \
    template void launch_boundary<T>(const DevGrid &, const NsConst &, double *, const Work<T> &, cudaStream_t);\
    template void launch_gradient_limiter<T>(const DevGrid &, const NsConst &, const Work<T> &, cudaStream_t);   \
    template void launch_residual<T>(const DevGrid &, const NsConst &, const Work<T> &, Reduce *, double,        \
                                     cudaStream_t);                                                              \
    template int launch_lusgs<T>(const DevGrid &, const NsConst &, const Work<T> &, const double *, Reduce *, int, \
                                 cudaStream_t);                                                                  \
    template void launch_update<T>(const DevGrid &, const NsConst &, const Work<T> &, const double *, double *, T *, \
                                   Reduce *, int *, cudaStream_t);                                               \
    template void launch_solution_fix<T>(const DevGrid &, const NsConst &, const double *, double *, T *, Reduce *, \
                                         int *, cudaStream_t);
PHX_INSTANTIATE(double)
PHX_INSTANTIATE(float)

}  // namespace phx
