// Internal definitions of the phx library: the device-side grid, the
// working arrays of one precision, and the kernel launchers.
//
// Storage layout.  The API speaks the reference's layout (original cell and
// face numbers, structure-of-arrays).  On the device, cells are stored in a
// space-filling-curve (Morton) order of their centroids and faces grouped by
// their storage owner, so that face neighbours lie close in memory; gathered
// per-cell and per-face data are array-of-structs records read with vector
// loads.  The reference's numbering is kept wherever it decides an order:
// every cell's face list is sorted by the reference face number (the order
// LoadFlux and the Green-Gauss loop accumulate in), and the LU-SGS level
// schedules come from the reference cell numbers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/phx.h"

namespace phx {

constexpr double kSmall = 1.0e-40;  // API/Common/include/Precision.h:27 (SMALL, TINY)
constexpr double kLarge = 1.0e40;   // Precision.h:26 (LARGE)

// Boundary handling classes, resolved once from (bcType, viscousType) the way
// NSSolverUnstruct::Boundary dispatches (NSSolverUnstruct.cpp:13469-13512).
enum BcKind : int32_t {
    BK_SYMMETRY = 0,   // SymmetryBCRegion (also inviscid solid walls)
    BK_WALL = 1,       // ViscousAdiabaticWallBCRegion
    BK_FARFIELD = 2,   // FarfieldBCRegion
    BK_EXTRAP = 3,     // OutflowBCRegion / extrapolation
};

// Record strides (elements).
constexpr int kQ = 8;      // qrec: rho u v w p | c2 hm | limiter
constexpr int kG = 20;     // grec: (d/dx, d/dy, d/dz) of var k at 3k..3k+2 | pad | temperature gradient 16..18 | pad
constexpr int kC = 8;      // crec: res0..4 | diag | inviscid | viscous spectral radius
constexpr int kD = 8;      // dqrec / dflux: 5 values | pad
constexpr int kF = 8;      // frec (FP64): nx ny nz area xfc yfc zfc | least-squares face weight
constexpr int kX = 4;      // xrec (FP64): xcc ycc zcc vol
constexpr int kFlux = 16;  // face flux record: inviscid F0..4 (times area) | inviscid and viscous
                           // spectral parts | pad | viscous F1..4 (times area; F0 is zero) | pad
constexpr int kCoef = 4;   // LU-SGS factors per face use: l1 x1 x2 | viscous spectral term
constexpr int kSweepPad = 4; // LU-SGS lane groups per warp: schedule levels are padded to this multiple

// Read-only device grid (FP64 metrics, connectivity, schedules), storage order.
struct DevGrid {
    int nCell, nBFace, nFace, nTotal;
    const int2 *lr;              // [nFace] left, right (boundary face f: right = nCell + f)
    const double *frec;          // [nFace][kF]
    const double *xrec;          // [nTotal][kX]
    const double *skew;          // [nCell]
    const double *volpow;        // [nCell] pow(pow(vol, 1/3), 3) as VencatLimiter7 forms it
    const double *walldist;      // [nCell]
    const double *lsq;           // [nCell][8] inverse least-squares matrix ixx iyy izz ixy ixz iyz | pad (lsq only)
    // [nFace] viscous-flux geometry switches of ComputeVisflux: bit 0 = both
    // centre angles above skewnessAngle (project the cell values onto the
    // normal line), bit 1 = both angles positive and |dL|, |dR| > TINY (form
    // the normal derivative); pure geometry, decided on the host
    const uint8_t *vflag;
    const int *c2f_off, *c2f;    // faces of each cell, ordered by the reference face number
    const int *orig;             // [nTotal] reference number of each cell (ghost: nCell + reference face)
    const int32_t *bkind;        // [nBFace] BcKind
    const int32_t *btype;        // [nBFace] bcType
    const uint8_t *farfield_adj; // [nCell] 1 if the cell touches a limiter-zeroing boundary
    // LU-SGS schedules: cells by level, and per schedule position the
    // neighbours on the sweep's side (in the cell's face order) as entries
    // eoff[i]..eoff[i+1]: neighbour, face (sign bit set when the normal points
    // into the cell), and the index of the face use's factors (2 f + side).
    const int *fwd_cells, *fwd_off, *fwd_eoff, *fwd_enb, *fwd_ef, *fwd_ec;
    const int *bwd_cells, *bwd_off, *bwd_eoff, *bwd_enb, *bwd_ef, *bwd_ec;
    int nFwdLevels, nBwdLevels;
    int nFwdPos, nBwdPos;        // schedule positions incl. idle padding (-1 cells)
    int maxLevelWidth;           // widest LU-SGS level (cells)
    double avgVol;
};

// Scalars of the NS path (derived from phx_params as the reference's
// Param_NSSolverUnstruct and PerfectGas do).
struct NsConst {
    double gama, coefState, pTotal;
    double primInf[5];
    double acoustic, convective;   // Roe entropy-fix coefficients
    double venkatK3;               // K^3 / (avgVol^(1/3))^3, as VencatLimiter7 forms it
    int viscous;                   // viscousType
    int limiter;                   // 0 none, 1 vencat
    int reconMethod;
    double cflStart, cflEnd;
    int cflVaryStep;
    double ktmax;
    int nSweeps;
    double lusgsTol;
    double reynolds;
    int gradient;                  // 0 Green-Gauss cell, 1 least squares
    // viscous terms (Param_NSSolverUnstruct / PerfectGas): 1/Re, 1/Pr, 1/Pr_t,
    // cp = 1 / ((gamma - 1) M^2), Sutherland constant over the reference
    // temperature, skewness switch of the viscous flux (degrees)
    double oRe, oPrl, oPrt, cp, tsuth, skewAngle;
};

// Working arrays of one precision T (double: FP64 path, float: mixed path).
template <class T>
struct Work {
    T *qrec;        // [nTotal][kQ] working state, c2 = |gamma p / rho|, total enthalpy, limiter
    T *grec;        // [nCell][kG] primitive gradients
    T *flux;        // [nFace][kFlux] face flux times area and inviscid spectral radius term
    T *coef;        // [2 nFace][kCoef] LU-SGS factors of each face use (side 0: the left cell's view)
    T *crec;        // [nCell][kC] residual, diagonal, spectral radii
    T *dtraw;       // [nCell] CFL * vol / spectral radius, before the ktmax clamp
    T *dqrec;       // [nTotal][kD] LU-SGS dq
    T *dflux;       // [nCell][kD] delta flux carried from the forward to the backward sweep
};

struct Reduce {
    unsigned long long mindt_bits;  // min over cells of dtraw (positive doubles order as integers)
    double resnorm[5];
    int negcount;
    unsigned int barrier;           // monotonic arrival counter of the LU-SGS grid barrier
    int error;                      // PHX_ERR_TIMEOUT / PHX_ERR_NUMERIC
};

// Kernel launchers (phx_kernels.cu).
template <class T>
void launch_boundary(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s);
template <class T>
void launch_gradient_limiter(const DevGrid &g, const NsConst &c, const Work<T> &w, cudaStream_t s);
template <class T>
void launch_residual(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, double cfl, cudaStream_t s);
template <class T>
int launch_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, int *flagF, int *flagB, int epoch,
                 int numSMs, cudaStream_t s);
template <class T>
void launch_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new,
                   Reduce *red, int *neglist, int numSMs, cudaStream_t s);
template <class T>
void launch_solution_fix(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new,
                         Reduce *red, int *neglist, cudaStream_t s);
// Refreshes qrec (state, c2, hm) of all cells and ghosts from the FP64 master state.
template <class T>
void launch_sync_qrec(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w, cudaStream_t s);
// Export of record fields into reference-order SoA: out[k * outLen +
// orig[i]] = rec[i * stride + first + k * step] for k < count, i < n.
template <class T>
void launch_export(const DevGrid &g, const T *rec, int stride, int first, int count, int step, int n, double *out,
                   int outLen, cudaStream_t s);
// q64[k][i] = in[k][orig[i]] and the inverse.
void launch_import_q(const DevGrid &g, const double *in, double *q64, cudaStream_t s);
void launch_export_q(const DevGrid &g, const double *q64, double *out, cudaStream_t s);
void launch_reset_reduce(Reduce *r, cudaStream_t s);
void launch_finish_step(Reduce *r, double *hist, int i, double ncell, cudaStream_t s);

}  // namespace phx
