// sm_100a kernels of the Spalart-Allmaras step (TurbSolverUnstr, one equation,
// NSMB formation, RANS length scale = wall distance, no wall function).
//
// The step runs after the NS update and the NS PostSolve boundary, as
// Simulation::SolveSteady orders the solvers (Main/src/Simulation.cpp:1527-1560).
// Like the reference it reads the NS velocity gradients and the laminar
// viscosity of the NS step (formed before the update) together with the
// updated density and velocity.  Per-cell sums are owner-computes gathers in
// the reference's face order; the LU-SGS sweeps use the NS dataflow schedule.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "phx_device.cuh"
#include "phx_internal.h"
#include "phx_physics.cuh"
#include "phx_mlp.h"
#include "phx_sa.cuh"

namespace phx {

// ---------------------------------------------------------------------------
// TurbSolverUnstr::Boundary (TurbSolverUnstr.cpp:5919-6019): OutflowBCRegion
// (copy; symmetry too, 6021-6048), WallBCRegion (6116-6160: nu~ and eddy
// viscosity reflected), FarfieldBCRegion (6546-6640: the Riemann-invariant
// normal velocity picks the interior copy or the free stream).  The far-field
// decision is made in FP64 from the master state.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) sa_boundary_kernel(DevGrid g, NsConst c, const double *q, Work<T> w,
                                                               TurbWork<T> t)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nBFace) return;
    const int nt = g.nTotal;
    // interface ghosts keep nu~ and the eddy viscosity of the last halo
    // exchange (TurbSolverUnstr::Boundary skips INTERFACE faces)
    if (g.bkind[f] == BK_INTERFACE) return;
    const int le = g.lr[f].x, re = g.nCell + f;
    T *tl = w.trec + (size_t)le * kTr;
    T *tg = w.trec + (size_t)re * kTr;
    const int bt = g.btype[f];
    double nu = t.qt64[le];
    T vist = tl[1];
    if (bt == PHX_BC_SOLID_SURFACE) {
        nu = -nu;
        vist = -vist;
    } else if (bt == PHX_BC_FARFIELD) {
        double fr[4];
        ld4(g.frec + (size_t)f * kF, fr);
        const double *pi = c.primInf;
        const double rin = q[le], uin = q[nt + le], vin = q[2 * nt + le], win = q[3 * nt + le], pin = q[4 * nt + le];
        const double vno = fr[0] * pi[1] + fr[1] * pi[2] + fr[2] * pi[3] - 0.0;
        const double vni = fr[0] * uin + fr[1] * vin + fr[2] * win - 0.0;
        const double vei = sqrt(uin * uin + vin * vin + win * win);
        const double ga = c.gama;
        const double coo = sqrt(fabs(c.gama * pi[4] / pi[0]));
        const double cin = sqrt(fabs(ga * pin / rin));
        bool exitFace;
        if (vei > cin) {
            exitFace = vni >= 0.0;
        } else {
            const double riemp = vni + 2.0 * cin / (ga - 1.0);
            const double riemm = vno - 2.0 * coo / (c.gama - 1.0);
            exitFace = 0.5 * (riemp + riemm) >= 0.0;
        }
        if (!exitFace) {
            nu = c.nutInf;
            vist = (T)c.vistInf;
        }
    }
    t.qt64[re] = nu;
    tg[0] = (T)nu;
    tg[1] = vist;
}

template <class T>
void launch_sa_boundary(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w,
                        const TurbWork<T> &t, cudaStream_t s)
{
    if (g.nBFace == 0) return;
    sa_boundary_kernel<T><<<(g.nBFace + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, q64, w, t);
}

// ---------------------------------------------------------------------------
// Eddy viscosity (TurbSolverUnstr::Viscosity, 1eq-sa branch, :6910-6960) and
// the gradient of nu~ (GetGradientField, :8652-8700: GG-cell or least
// squares, as the NS gradient), fused per cell.
// ---------------------------------------------------------------------------
// GG-node node values of nu~ (TurbSolverUnstr::ComputeQTurbNodeValue,
// TurbSolverUnstr.cpp:3480-3814, ModifyQTurbNodeValue :3816-3845): per node
// the sum of its {owner, other side} pairs in the reference's order over twice
// their number, 0 for a node without pairs.
template <class T>
__global__ void __launch_bounds__(kThreads) turb_node_kernel(DevGrid g, Work<T> w, TurbWork<T> t)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nNode) return;
    const int j0 = ld(g.tn_off + n), j1 = ld(g.tn_off + n + 1);
    T acc = T(0);
    for (int j = j0; j < j1; ++j) {
        const int2 pr = ld(g.tn_pairs + j);
        acc += w.trec[(size_t)pr.x * kTr];
        acc += w.trec[(size_t)pr.y * kTr];
    }
    t.qtnode[n] = j1 > j0 ? idiv(acc, (T)(2 * (j1 - j0))) : T(0);
}

template <class T>
void launch_turb_node_values(const DevGrid &g, const Work<T> &w, const TurbWork<T> &t, cudaStream_t s)
{
    turb_node_kernel<T><<<(g.nNode + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, w, t);
}

// kGrad: 0 GG-cell, 1 least squares, 2 GG-node.
template <class T, int kGrad>
__global__ void __launch_bounds__(kThreads) sa_visc_grad_kernel(DevGrid g, NsConst c, Work<T> w, TurbWork<T> t)
{
    constexpr bool kLsq = kGrad == 1;
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.nCell) return;
    T tr[4];
    ld4(w.trec + (size_t)cell * kTr, tr);
    const T nue = tr[0];
    const T rho = w.qrec[(size_t)cell * kQ];
    T vist = T(0);
    if (nue > T(0)) {
        const T cv13 = T(7.1) * T(7.1) * T(7.1);
        const T ld_ = nue * rho / (tr[2] + (T)kSmall);
        const T ld3 = ld_ * ld_ * ld_;
        const T fv1 = ld3 / (ld3 + cv13);
        vist = rho * fv1 * nue;
    }
    w.trec[(size_t)cell * kTr + 1] = vist;
    double xc[4];
    ld4(g.xrec + (size_t)cell * kX, xc);
    T gx = T(0), gy = T(0), gz = T(0);
    const int j0 = g.c2f_off[cell], j1 = g.c2f_off[cell + 1];
    for (int j = j0; j < j1; ++j) {
        const int f = ld(g.c2f + j);
        const int2 lr = ld(g.lr + f);
        const bool isLeft = (lr.x == cell);
        const int nb = isLeft ? lr.y : lr.x;
        const T vn = ldcg(w.trec + (size_t)nb * kTr);   // slot 1 of the rows is written by this kernel
        if (kLsq) {
            double xn[4];
            ld4(g.xrec + (size_t)nb * kX, xn);
            const double iw = ld(g.frec + (size_t)f * kF + 7);
            const T dx = (T)(isLeft ? xn[0] - xc[0] : xc[0] - xn[0]);
            const T dy = (T)(isLeft ? xn[1] - xc[1] : xc[1] - xn[1]);
            const T dz = (T)(isLeft ? xn[2] - xc[2] : xc[2] - xn[2]);
            const T dq = (T)iw * (isLeft ? vn - nue : nue - vn);
            gx += dq * dx; gy += dq * dy; gz += dq * dz;
        } else {
            double fr[4];
            ld4(g.frec + (size_t)f * kF, fr);
            const double a = fr[3];
            const T nx = (T)(fr[0] * a), ny = (T)(fr[1] * a), nz = (T)(fr[2] * a);
            T qf = T(0.5) * (isLeft ? (nue + vn) : (vn + nue));
            if (kGrad == 2 && (f >= g.nBFace || ld(g.btype + f) == PHX_BC_SYMMETRY)) {
                // UnstructGrid::CompGradientGGNode_NEW (Geo_UnstructGrid.cpp:4202-4309)
                const int a0 = ld(g.fn_off + f), a1 = ld(g.fn_off + f + 1);
                T sn = T(0);
                for (int k = a0; k < a1; ++k) sn += t.qtnode[ld(g.fn_idx + k)];
                qf = sn / (T)(a1 - a0);
            }
            if (isLeft) { gx += qf * nx; gy += qf * ny; gz += qf * nz; }
            else { gx -= qf * nx; gy -= qf * ny; gz -= qf * nz; }
        }
    }
    if (kLsq) {
        double m6[8];
        ld8(g.lsq + (size_t)cell * 8, m6);
        const T tx = gx, ty = gy, tz = gz;
        gx = (T)m6[0] * tx + (T)m6[3] * ty + (T)m6[4] * tz;
        gy = (T)m6[3] * tx + (T)m6[1] * ty + (T)m6[5] * tz;
        gz = (T)m6[4] * tx + (T)m6[5] * ty + (T)m6[2] * tz;
    } else if (kGrad == 2) {
        const T vol = (T)xc[3];
        gx /= vol; gy /= vol; gz /= vol;
    } else {
        const T ovol = T(1) / (T)xc[3];
        gx *= ovol; gy *= ovol; gz *= ovol;
    }
    T o[4] = {gx, gy, gz, T(0)};
    st4(t.tgrad + (size_t)cell * kTg, o);
}

// ---------------------------------------------------------------------------
// SA face pass (one thread per face):
//  * convection: GetQlQrTurbulence / GetQlQrNS (TurbSolverUnstr.cpp:4978-5140;
//    boundary faces take the face average, symmetry copies the left nu~)
//    and NNDFlux (:5721-5805, first-order upwind, rhoFlag = 0);
//  * diffusion: mlt of GetVisFaceValue (:3960-3990) and the NSMB branch of
//    ComputeVisflux (:4438-4674): flux1 for both sides, flux2 times the side's
//    own (visl / rho + PositiveSA(nu~));
//  * SpectrumRadiusOfOneEquation, NSMB branch (:4690-4855): upwind Jacobians,
//    the diffusion spectral term and the face matrices mat_turbl / mat_turbr,
//    stored per face use for the sweeps.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) sa_face_kernel(DevGrid g, NsConst c, Work<T> w, TurbWork<T> t)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nFace) return;
    const int2 lr = ld(g.lr + f);
    const int le = lr.x, re = lr.y;
    // interface faces are interior faces for the face states (GetQlQrTurbulence,
    // GetQlQrNS, TurbSolverUnstr.cpp:5041, :5125) and the normal derivative (:4569)
    const bool bnd = f < g.nBFace && g.bkind[f] != BK_INTERFACE;
    const int bt = bnd ? g.btype[f] : 0;
    double fr[8];
    ld8(g.frec + (size_t)f * kF, fr);
    T qL[8], qR[8], tl[4], tr[4];
    ld8(w.qrec + (size_t)le * kQ, qL);
    ld8(w.qrec + (size_t)re * kQ, qR);
    ld4(w.trec + (size_t)le * kTr, tl);
    ld4(w.trec + (size_t)re * kTr, tr);
    const T nx = (T)fr[0], ny = (T)fr[1], nz = (T)fr[2], area = (T)fr[3];
    const T oRe = (T)c.oRe;
    const T cb2 = T(0.622);
    const T osigma = T(1) / T(2.0 / 3.0);
    T out[8];
    // convection
    {
        T ql = tl[0], qr = tr[0];
        T pl[4] = {qL[0], qL[1], qL[2], qL[3]}, pr[4] = {qR[0], qR[1], qR[2], qR[3]};
        if (bnd) {
            if (bt == PHX_BC_SYMMETRY) qr = ql;
            else { const T a = T(0.5) * (qr + ql); qr = a; ql = a; }
#pragma unroll
            for (int k = 0; k < 4; ++k) { const T a = T(0.5) * (pr[k] + pl[k]); pr[k] = a; pl[k] = a; }
        }
        const T vnl = nx * pl[1] + ny * pl[2] + nz * pl[3] - T(0);
        const T vnr = nx * pr[1] + ny * pr[2] + nz * pr[3] - T(0);
        const T vnll = T(0.5) * (vnl + fabs(vnl));
        const T vnrr = T(0.5) * (vnr - fabs(vnr));
        out[0] = (vnll * ql + vnrr * qr) * area;
    }
    // diffusion: the face value mlt takes interface faces as boundary faces
    // (GetVisFaceValue's mlt loop, TurbSolverUnstr.cpp:3990-4003); the normal
    // derivative below takes them as interior faces (:4569)
    {
        T nl = tl[0], nr = tr[0];
        const T vl = tl[2], vr = tr[2], rl = qL[0], rr = qR[0];
        if (f < g.nBFace) {
            if (nl < T(0)) {
                nl = positive_sa(nl, vl, rl);
                if (bt == PHX_BC_SOLID_SURFACE) nr = -nl;
            }
        } else {
            nl = positive_sa(nl, vl, rl);
            nr = positive_sa(nr, vr, rr);
        }
        const T mlt = osigma * T(0.5) * (vl / rl + vr / rr + nl + nr);
        T dfdn = T(0);
        if (g.vflag[f] & 4) {
            double xl[4], xr[4];
            ld4(g.xrec + (size_t)le * kX, xl);
            ld4(g.xrec + (size_t)re * kX, xr);
            const double dL = fr[0] * (xl[0] - fr[4]) + fr[1] * (xl[1] - fr[5]) + fr[2] * (xl[2] - fr[6]);
            const double dR = fr[0] * (xr[0] - fr[4]) + fr[1] * (xr[1] - fr[5]) + fr[2] * (xr[2] - fr[6]);
            const T f1 = tl[0], f2 = tr[0];
            const T fm = T(0.5) * (f1 + f2);
            const T dLt = (T)dL, dRt = (T)dR;
            const T d1 = (f1 - fm) / dLt, d2 = (f2 - fm) / dRt;
            const T wl = dLt * dLt / (dLt * dLt + dRt * dRt);
            const T wr = T(1) - wl;
            dfdn = wl * d1 + wr * d2;
            if (bnd && bt != PHX_BC_SYMMETRY) {
                const double nd = (xr[0] - xl[0]) * fr[0] + (xr[1] - xl[1]) * fr[1] + (xr[2] - xl[2]) * fr[2];
                dfdn = (f2 - f1) / (T)nd;
            }
        }
        out[1] = -oRe * (T(1) + cb2) * mlt * dfdn * area;
        out[2] = oRe * cb2 * osigma * dfdn * area;
    }
    // spectral radius and face matrices
    T matR, matL;
    {
        const T vnl = nx * qL[1] + ny * qL[2] + nz * qL[3] - T(0);
        const T vnr = nx * qR[1] + ny * qR[2] + nz * qR[3] - T(0);
        const T ijl = vnl > T(0) ? qL[0] * vnl * area : T(0);
        const T ijr = vnr < T(0) ? qR[0] * vnr * area : T(0);
        const T orl = T(1) / (qL[0] + (T)kSmall), orr = T(1) / (qR[0] + (T)kSmall);
        const T nuel = positive_sa(tl[0], tl[2], qL[0]);
        T nuer = positive_sa(tr[0], tr[2], qR[0]);
        if (bnd && bt == PHX_BC_SOLID_SURFACE) nuer = -nuel;
        const T effl = tl[2] * orl + fabs(nuel);
        const T effr = tr[2] * orr + fabs(nuer);
        const T eff = T(0.5) * (effl + effr);
        const T ovol = T(1) / (T(0.5) * ((T)g.xrec[(size_t)le * kX + 3] + (T)g.xrec[(size_t)re * kX + 3]));
        const T ns2 = area * area;
        const T vterm = oRe * ovol * (T(1) + cb2) * (osigma * eff * ns2);
        out[3] = ijl;
        out[4] = ijr;
        out[5] = vterm;
        out[6] = out[7] = T(0);
        matR = ijr;
        matL = -ijl;
        matL += -oRe * ovol * (T(1) + cb2) * (osigma * eff * ns2);
        matR += -oRe * ovol * (T(1) + cb2) * (osigma * eff * ns2);
        const T cl = cb2 * osigma * effl, cr = cb2 * osigma * effr;
        matL += oRe * ovol * ns2 * cl;
        matR += oRe * ovol * ns2 * cr;
    }
    st8(t.tface + (size_t)f * kTf, out);
    t.tcoef[2 * (size_t)f] = matR;
    if (!bnd) t.tcoef[2 * (size_t)f + 1] = matL;
}

// ---------------------------------------------------------------------------
// SA cell pass (one thread per cell): InitSpectrum (TurbSolverUnstr.cpp:
// 1025-1072) with the NS step's final dt, the exact source and its implicit
// part (SourceFluxOneEquationOriginal, :2702-2916, NSMB formation: the cb2
// gradient term is carried by the diffusion flux), then the face terms in the
// reference's order: convection over all faces (InviscidFlux), diffusion over
// all faces (ViscousFlux), and, into the spectral radius, the Jacobians of
// SpectrumRadiusOfOneEquation (called by Diagonal before the sweeps).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) sa_cell_kernel(DevGrid g, NsConst c, Work<T> w, TurbWork<T> t,
                                                           const Reduce *red)
{
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.nCell) return;
    T tr[4];
    ld4(w.trec + (size_t)cell * kTr, tr);
    const T nue = tr[0], visl = tr[2];
    const T rho = w.qrec[(size_t)cell * kQ];
    const double vol = ld(g.xrec + (size_t)cell * kX + 3);
    // velocity gradients of the NS step
    T gr[16];
    const T *gp = w.grec + (size_t)cell * kG;
    ld8(gp, gr);
    ld8(gp + 8, gr + 8);
    const T dudy = gr[4], dudz = gr[5], dvdx = gr[6], dvdz = gr[8], dwdx = gr[9], dwdy = gr[10];
    const T omega = sqrt((dwdy - dvdz) * (dwdy - dvdz) + (dudz - dwdx) * (dudz - dwdx) + (dvdx - dudy) * (dvdx - dudy));
    T tg[4];
    ld4(t.tgrad + (size_t)cell * kTg, tg);
    const T grd2 = tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2];
    const T olam = rho / (visl + (T)kSmall);
    const double d = ld(g.walldist + cell);
    T src, sspec;
    sa_source_fp64<T>(nue, omega, olam, d, grd2, c.oRe, src, sspec);
    if (c.saSource) {
        // learned source; NaN marks the cells that take the exact source
        const T s = t.tsrc[cell];
        if (s == s) src = s;
    }
    // NS dt after ReduceMaxTimeStep: min(dt, ktmax dt_min) / vol
    T dt = w.dtraw[cell];
    const double mindt = __longlong_as_double((long long)red->mindt_bits);
    if (c.ktmax > 0) dt = tmin(dt, (T)(c.ktmax * mindt));
    dt /= (T)vol;
    T res = T(-0.0);
    res += src * (T)vol;
    T spec = T(0) * (T)vol + T(1) / ((T)c.turbCflScale * dt + (T)kSmall);
    spec += sspec * (T)vol;
    const int j0 = g.c2f_off[cell], j1 = g.c2f_off[cell + 1];
    for (int j = j0; j < j1; ++j) {
        const int f = ld(g.c2f + j);
        const bool isLeft = ld(&g.lr[f].x) == cell;
        const T fl = ld(t.tface + (size_t)f * kTf);
        if (isLeft) res -= fl;
        else res += fl;
    }
    const T own = visl / rho + positive_sa(nue, visl, rho);
    for (int j = j0; j < j1; ++j) {
        const int f = ld(g.c2f + j);
        const bool isLeft = ld(&g.lr[f].x) == cell;
        T tf[8];
        ld8(t.tface + (size_t)f * kTf, tf);
        if (isLeft) { res -= tf[1]; res -= tf[2] * own; }
        else { res += tf[1]; res += tf[2] * own; }
    }
    for (int j = j0; j < j1; ++j) {
        const int f = ld(g.c2f + j);
        const bool isLeft = ld(&g.lr[f].x) == cell;
        T tf[8];
        ld8(t.tface + (size_t)f * kTf, tf);
        if (isLeft) spec += tf[3];
        else spec -= tf[4];
        spec += tf[5];
    }
    T o[4] = {res, spec, idiv(T(1), spec), T(0)};   // the sweep multiplies by the reciprocal
    st4(t.tcrec + (size_t)cell * kTc, o);
}

template <class T>
void launch_sa_residual(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w,
                        const TurbWork<T> &t, Reduce *red, const MlpDev *mlp, unsigned long long *nmlp, int numSMs,
                        cudaStream_t s)
{
    const int cb = (g.nCell + kThreads - 1) / kThreads, fb = (g.nFace + kThreads - 1) / kThreads;
    // Controller::UpdateResiduals(TURB): boundary, Viscosity + gradient, then
    // TurbSolver::UpdateResiduals repeats the boundary (ghost eddy viscosity of
    // the new interior values)
    launch_sa_boundary<T>(g, c, q64, w, t, s);
    if (c.gradient == 1) sa_visc_grad_kernel<T, 1><<<cb, kThreads, 0, s>>>(g, c, w, t);
    else if (c.gradient == 2) sa_visc_grad_kernel<T, 2><<<cb, kThreads, 0, s>>>(g, c, w, t);
    else sa_visc_grad_kernel<T, 0><<<cb, kThreads, 0, s>>>(g, c, w, t);
    launch_sa_boundary<T>(g, c, q64, w, t, s);
    sa_face_kernel<T><<<fb, kThreads, 0, s>>>(g, c, w, t);
    if (c.saSource && mlp) launch_mlp_source<T>(g, c, w, t, *mlp, red, nmlp, numSMs, s);
    sa_cell_kernel<T><<<cb, kThreads, 0, s>>>(g, c, w, t, red);
}

// ---------------------------------------------------------------------------
// Scalar LU-SGS of the SA equation (SolveLUSGSForward / Backward,
// TurbSolverUnstr.cpp:1400-1638): dq = (res - L/U dq - rhs0) / spec_turb with
// the face matrices of each face use.  Same dataflow schedule, write-once
// records and bounded waits as the NS sweep (phx_kernels.cu): tdqf (forward
// dq), tdfl (forward delta flux) and tdq (final dq) hold the sentinel until
// written.  dq of the ghosts is the ghost residual, which is zero, so ghost
// entries of the backward sweep add nothing and are skipped; an interface
// ghost's too, as the reference exchanges no SA dq between the sweeps
// (Controller::CommunicationDQ, CFD/Solver/src/Controller.cpp:2874-2880).
// ---------------------------------------------------------------------------
// Static inputs of one slot for one lane (loaded a round ahead): neighbour
// (-1: none or a ghost), its face matrix, and (lane 0 of the cell's first
// slot) the cell's residual and the reciprocal of its spectral radius.
template <class T>
struct SaSweepIn {
    int cell, count, nb;
    T mat, res, rspec;
};

template <class T>
__device__ __forceinline__ void sa_sweep_load(const DevGrid &g, const TurbWork<T> &t, int2 info, int4 en, int lane,
                                              SaSweepIn<T> &s)
{
    s.cell = info.x;
    s.count = info.y;
    s.nb = -1;
    if (info.x >= 0 && en.x >= 0 && en.x < g.nCell) {
        s.nb = en.x;
        s.mat = t.tcoef[en.z];
    }
    if (info.x >= 0 && info.y >= 0 && lane == 0) {
        T cr[4];
        ld4(t.tcrec + (size_t)info.x * kTc, cr);
        s.res = cr[0];
        s.rspec = cr[2];
    }
}

template <class T, bool kForward>
__device__ __forceinline__ bool sa_sweep_position(const TurbWork<T> &t, Reduce *red, const SaSweepIn<T> &s, int lane,
                                                  int base, long long spinLimit)
{
    const int cell = s.cell;
    const bool live = cell >= 0;
    const bool lead = live && s.count >= 0;   // the cell's first slot
    const int e1 = lead ? s.count : 0;
    const bool has = live && s.nb >= 0;
    // the neighbour's dq (forward: its forward dq; backward: its final dq)
    // and, backward, this cell's forward delta flux
    const T *src1 = has ? (kForward ? t.tdqf : t.tdq) + s.nb : nullptr;
    const T *src2 = (!kForward && lead && lane == 0) ? t.tdfl + cell : nullptr;
    T v1 = T(0), fl = T(0);
    bool r1 = true, r2 = true;
    if (src1) { v1 = ld_poll(src1); r1 = !is_sentinel(v1); }
    if (src2) { fl = ld_poll(src2); r2 = !is_sentinel(fl); }
    // the SA cell pass formed the reciprocal of the spectral radius (a division
    // on the sweep's critical path costs up to microseconds; see the NS sweep)
    const T rspec = s.rspec;
    long long spins = 0;
    while (!__all_sync(0xffffffffu, r1 && r2)) {
        ++spins;
        if (spins > spinLimit) {
            if ((threadIdx.x & 31) == 0) atomicExch(&red->error, PHX_ERR_TIMEOUT);
            return false;
        }
        if ((spins & 1023) == 0 && __any_sync(0xffffffffu, ((volatile int *)&red->error)[0] != 0)) return false;
        if (spins > 8) __nanosleep(20);
        if (!r1) { v1 = ld_poll(src1); r1 = !is_sentinel(v1); }
        if (!r2) { fl = ld_poll(src2); r2 = !is_sentinel(fl); }
    }
    const T df = has ? s.mat * v1 : T(0);
    T rhs0 = T(0);
#pragma unroll
    for (int k = 0; k < kSweepLanes; ++k) {
        const T v = __shfl_sync(0xffffffffu, df, base + k);
        if (k < e1) rhs0 += v;
    }
    if (__any_sync(0xffffffffu, e1 > kSweepLanes)) {
#pragma unroll
        for (int k = kSweepLanes; k < kSweepMaxEntries; ++k) {
            const T v = __shfl_sync(0xffffffffu, df, (base + k) & 31);
            if (k < e1) rhs0 += v;
        }
    }
    if (lead && lane == 0) {
        if (kForward) {
            st_relaxed(t.tdfl + cell, unsentinel(T(0) + rhs0));
            st_relaxed(t.tdqf + cell, unsentinel((s.res - T(0) - rhs0) * rspec));
        } else {
            st_relaxed(t.tdq + cell, unsentinel((s.res - fl - rhs0) * rspec));
        }
    }
    return true;
}

// Rounds of ngroups positions; entries loaded two rounds ahead, the face
// matrices and residual records one round ahead.
template <class T, bool kForward>
__device__ __forceinline__ bool sa_sweep_all(const DevGrid &g, const TurbWork<T> &t, Reduce *red, int group,
                                             int wgroup0, int ngroups, int lane, int base, long long spinLimit)
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
    SaSweepIn<T> cur;
    sa_sweep_load<T>(g, t, info, en, lane, cur);
    entry(p + ngroups, info, en);
    for (int p0 = wgroup0; p0 < npos; p0 += ngroups) {
        SaSweepIn<T> nxt;
        sa_sweep_load<T>(g, t, info, en, lane, nxt);
        entry(p + 2 * ngroups, info, en);
        if (!sa_sweep_position<T, kForward>(t, red, cur, lane, base, spinLimit)) return false;
        if (en.x >= 0 && en.x < g.nCell) prefetch_l2(t.tcoef + en.z);
        if (lane == 0 && info.x >= 0 && info.y >= 0) prefetch_l2(t.tcrec + (size_t)info.x * kTc);
        cur = nxt;
        p += ngroups;
    }
    return true;
}

template <class T>
__global__ void __launch_bounds__(kSweepThreads) sa_lusgs_kernel(DevGrid g, TurbWork<T> t, Reduce *red,
                                                                 long long spinLimit, int sweeps)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int group = tid / kSweepLanes, lane = tid % kSweepLanes;
    const int ngroups = (gridDim.x * blockDim.x) / kSweepLanes;
    const int wgroup0 = group & ~(kSweepSlots - 1);
    const int base = (threadIdx.x & 31) & ~(kSweepLanes - 1);
    if ((sweeps & kSweepForward) && !sa_sweep_all<T, true>(g, t, red, group, wgroup0, ngroups, lane, base, spinLimit))
        return;
    if (sweeps & kSweepBackward) sa_sweep_all<T, false>(g, t, red, group, wgroup0, ngroups, lane, base, spinLimit);
}

// Fills the SA sweep's output records with the sentinel.
template <class T>
__global__ void __launch_bounds__(kThreads) sa_sweep_reset_kernel(int n, T *a, T *b, T *c)
{
    const T s = sweep_sentinel<T>();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i] = s;
        b[i] = s;
        c[i] = s;
    }
}

template <class T>
int launch_sa_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, Reduce *red,
                    int numSMs, cudaStream_t s, int sweeps)
{
    (void)w;
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
    int &resident = perSMcache[dev][sizeof(T) == 8 ? 0 : 1];
    if (resident < 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, sa_lusgs_kernel<T>, kSweepThreads, 0);
        if (resident < 1) resident = 1;
    }
    // at most two blocks per SM: the scalar sweep does little work per poll,
    // and more polling slots only load L2 (16M cells: 4.1 ms at two blocks per
    // SM against 4.5 ms at six); PHX_SA_SWEEP_BLOCKS_PER_SM changes the cap
    // (tuning)
    int cap = 2;
    if (const char *e = getenv("PHX_SA_SWEEP_BLOCKS_PER_SM")) cap = atoi(e) > 0 ? atoi(e) : cap;
    const int perSM = resident < cap ? resident : cap;
    int blocks = numSMs * perSM;
    const int npos = g.nFwdPos > g.nBwdPos ? g.nFwdPos : g.nBwdPos;
    const int need = (int)(((long long)npos * kSweepLanes + kSweepThreads - 1) / kSweepThreads);
    if (blocks > need) blocks = need;
    if (const char *cap = getenv("PHX_LUSGS_MAX_BLOCKS")) {
        const int v = atoi(cap);
        if (v > 0 && blocks > v) blocks = v;
    }
    if (blocks < 1) blocks = 1;
    const int rb = std::min((g.nCell + kThreads - 1) / kThreads, numSMs * 16);
    if (sweeps & kSweepForward)
        sa_sweep_reset_kernel<T><<<rb > 0 ? rb : 1, kThreads, 0, s>>>(g.nCell, t.tdqf, t.tdfl, t.tdq);
    DevGrid gg = g;
    TurbWork<T> tt = t;
    Reduce *rr = red;
    long long lim = c.spinLimit;
    int sw = sweeps;
    void *args[] = {&gg, &tt, &rr, &lim, &sw};
    const cudaError_t e =
        cudaLaunchCooperativeKernel((void *)sa_lusgs_kernel<T>, dim3(blocks), dim3(kSweepThreads), args, 0, s);
    return e == cudaSuccess ? 0 : (int)e;
}

// UpdateFlowField (TurbSolverUnstr.cpp:1180-1230; RANS without qTurbLimit: no
// clipping): FP64 master nu~ += dq.
template <class T>
__global__ void __launch_bounds__(kThreads) sa_update_kernel(DevGrid g, Work<T> w, TurbWork<T> t)
{
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.nCell) return;
    const double v = t.qt64[cell] + (double)t.tdq[cell];
    t.qt64[cell] = v;
    w.trec[(size_t)cell * kTr] = (T)v;
}

template <class T>
void launch_sa_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, cudaStream_t s)
{
    (void)c;
    sa_update_kernel<T><<<(g.nCell + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, w, t);
}

template <class T>
__global__ void __launch_bounds__(kThreads) import_turb_kernel(DevGrid g, const double *in, TurbWork<T> t, Work<T> w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nTotal) return;
    const double v = in[g.orig[i]];
    t.qt64[i] = v;
    w.trec[(size_t)i * kTr] = (T)v;
}

template <class T>
void launch_import_turb(const DevGrid &g, const double *in, const TurbWork<T> &t, const Work<T> &w, cudaStream_t s)
{
    import_turb_kernel<T><<<(g.nTotal + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, in, t, w);
}

// trec slot 1 (eddy viscosity) of cells and ghosts from a reference-order array.
template <class T>
__global__ void __launch_bounds__(kThreads) import_vist_kernel(DevGrid g, const double *in, Work<T> w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nTotal) return;
    w.trec[(size_t)i * kTr + 1] = (T)in[g.orig[i]];
}

template <class T>
void launch_import_vist(const DevGrid &g, const double *in, const Work<T> &w, cudaStream_t s)
{
    import_vist_kernel<T><<<(g.nTotal + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, in, w);
}

#define PHX_SA_INSTANTIATE(T)                                                                                     \
    template void launch_sa_boundary<T>(const DevGrid &, const NsConst &, const double *, const Work<T> &,        \
                                        const TurbWork<T> &, cudaStream_t);                                       \
    template void launch_sa_residual<T>(const DevGrid &, const NsConst &, const double *, const Work<T> &,        \
                                        const TurbWork<T> &, Reduce *, const MlpDev *, unsigned long long *, int, \
                                        cudaStream_t);                                                            \
    template int launch_sa_lusgs<T>(const DevGrid &, const NsConst &, const Work<T> &, const TurbWork<T> &,       \
                                    Reduce *, int, cudaStream_t, int);                                            \
    template void launch_sa_update<T>(const DevGrid &, const NsConst &, const Work<T> &, const TurbWork<T> &,     \
                                      cudaStream_t);                                                              \
    template void launch_turb_node_values<T>(const DevGrid &, const Work<T> &, const TurbWork<T> &, cudaStream_t); \
    template void launch_import_turb<T>(const DevGrid &, const double *, const TurbWork<T> &, const Work<T> &,    \
                                        cudaStream_t);                                                            \
    template void launch_import_vist<T>(const DevGrid &, const double *, const Work<T> &, cudaStream_t);
PHX_SA_INSTANTIATE(double)
PHX_SA_INSTANTIATE(float)

}  // namespace phx

namespace phx {

// ---------------------------------------------------------------------------
// Wall force sums (NSSolverUnstruct::AirForceCoefParts, NSSolverUnstruct.cpp:
// 16026-16240, all solid walls, torque reference at the origin): pressure
// force 2 (p - p_inf) n A of the wall cell, viscous stress from the NS step's
// velocity gradient corrected along the cell-to-ghost line (CorrectGradient,
// API/Physics/src/GradientOperation.cpp:21-31) and the NS step's laminar
// viscosity.  FP64 on both paths: per-face terms, block sums, one FP64 atomic
// per block and value.  out[15]: CA_f CA_p CN_f CN_p CZ_f CZ_p cpx cpy cpz
// Cl_f Cl_p Cn_f Cn_p Cm_f Cm_p.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) forces_kernel(DevGrid g, NsConst c, Work<T> w, const double *q,
                                                          double *out)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    double v[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) v[k] = 0.0;
    if (f < g.nBFace && g.btype[f] == PHX_BC_SOLID_SURFACE) {
        const int nt = g.nTotal;
        const int le = g.lr[f].x, re = g.nCell + f;
        double fr[8];
        ld8(g.frec + (size_t)f * kF, fr);
        const double nx = fr[0] * fr[3], ny = fr[1] * fr[3], nz = fr[2] * fr[3];
        const double cp = 2.0 * (q[4 * nt + le] - c.primInf[4]);
        const double dpx = nx * cp, dpy = ny * cp, dpz = nz * cp;
        const double xc = fr[4], yc = fr[5], zc = fr[6];
        v[1] = dpx; v[3] = dpy; v[5] = dpz;
        v[6] = dpx; v[7] = dpy; v[8] = dpz;
        v[10] = yc * dpz - zc * dpy;
        v[12] = zc * dpx - xc * dpz;
        v[14] = xc * dpy - yc * dpx;
        if (c.viscous) {
            T gr[16];
            const T *gp = w.grec + (size_t)le * kG;
            ld8(gp, gr);
            ld8(gp + 8, gr + 8);
            double gu[3] = {gr[3], gr[4], gr[5]}, gv[3] = {gr[6], gr[7], gr[8]}, gw[3] = {gr[9], gr[10], gr[11]};
            double xl[4], xr[4];
            ld4(g.xrec + (size_t)le * kX, xl);
            ld4(g.xrec + (size_t)re * kX, xr);
            double dx = xr[0] - xl[0], dy = xr[1] - xl[1], dz = xr[2] - xl[2];
            const double ods = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
            dx *= ods; dy *= ods; dz *= ods;
            double *gs[3] = {gu, gv, gw};
            for (int k = 0; k < 3; ++k) {
                double *gg = gs[k];
                const double fold = gg[0] * dx + gg[1] * dy + gg[2] * dz;
                const double fnew = (q[(k + 1) * nt + re] - q[(k + 1) * nt + le]) * ods;
                const double df = fnew - fold;
                gg[0] += df * dx; gg[1] += df * dy; gg[2] += df * dz;
            }
            const double vis = (double)w.trec[(size_t)le * kTr + 2];
            const double c23 = 2.0 / 3.0;
            const double txx = vis * c23 * (2.0 * gu[0] - gv[1] - gw[2]);
            const double tyy = vis * c23 * (2.0 * gv[1] - gw[2] - gu[0]);
            const double tzz = vis * c23 * (2.0 * gw[2] - gu[0] - gv[1]);
            const double txy = vis * (gu[1] + gv[0]), txz = vis * (gu[2] + gw[0]), tyz = vis * (gv[2] + gw[1]);
            const double fvx = -2.0 * (nx * txx + ny * txy + nz * txz) * c.oRe;
            const double fvy = -2.0 * (nx * txy + ny * tyy + nz * tyz) * c.oRe;
            const double fvz = -2.0 * (nx * txz + ny * tyz + nz * tzz) * c.oRe;
            v[0] = fvx; v[2] = fvy; v[4] = fvz;
            v[9] = yc * fvz - zc * fvy;
            v[11] = zc * fvx - xc * fvz;
            v[13] = xc * fvy - yc * fvx;
        }
    }
    __shared__ double part[kThreads / 32][15];
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        double s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (ln == 0) part[wid][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < 15) {
        double s = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) s += part[i][threadIdx.x];
        if (s != 0.0) atomicAdd(out + threadIdx.x, s);
    }
}

template <class T>
void launch_forces(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *out,
                   cudaStream_t s)
{
    cudaMemsetAsync(out, 0, sizeof(double) * 16, s);
    if (g.nBFace == 0) return;
    forces_kernel<T><<<(g.nBFace + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, w, q64, out);
}

template void launch_forces<double>(const DevGrid &, const NsConst &, const Work<double> &, const double *, double *,
                                    cudaStream_t);
template void launch_forces<float>(const DevGrid &, const NsConst &, const Work<float> &, const double *, double *,
                                   cudaStream_t);

}  // namespace phx
