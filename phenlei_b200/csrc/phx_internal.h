// Internal definitions of the phx library: the device-side grid, the
// working arrays of one precision, and the kernel launchers.
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

// Per-boundary-face flags used by BoundaryQlQrFix / SetLimitBoundary / ghost dq.
struct BFaceInfo {
    int32_t kind;       // BcKind
    int32_t bcType;     // the reference bcType
};

// Read-only device grid (FP64 metrics, connectivity, schedules).
struct DevGrid {
    int nCell, nBFace, nFace, nTotal;
    const int *left, *right;                 // right of boundary face f = nCell + f
    const double *xfn, *yfn, *zfn, *area;    // [nFace]
    const double *xfc, *yfc, *zfc;           // [nFace]
    const double *xcc, *ycc, *zcc, *vol;     // [nTotal]
    const double *skew;                      // [nCell]
    const double *volpow;                    // [nCell] pow(pow(vol, 1/3), 3) as VencatLimiter7 forms it
    const double *walldist;                  // [nCell]
    const int *c2f_off, *c2f;                // ascending face lists per cell
    const int32_t *bkind;                    // [nBFace] BcKind
    const int32_t *btype;                    // [nBFace] bcType
    const uint8_t *farfield_adj;             // [nCell] 1 if the cell touches a limiter-zeroing boundary
    const int *fwd_cells, *fwd_off;          // LU-SGS forward schedule: cells by level
    const int *bwd_cells, *bwd_off;          // backward schedule
    // Per sweep, in schedule order: for position i the neighbours on the
    // sweep's side, in the cell's face order, as entries eoff[i]..eoff[i+1]:
    // neighbour cell, face (sign bit set when the normal points into the
    // cell), and the slot j of the face in the cell's face list.
    const int *fwd_eoff, *fwd_enb, *fwd_ef, *fwd_ej;
    const int *bwd_eoff, *bwd_enb, *bwd_ef, *bwd_ej;
    int nFwdLevels, nBwdLevels;
    int c2fLen;                              // c2f_off[nCell]
    int maxLevelWidth;                       // widest LU-SGS level (cells)
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
};

// Working arrays of one precision T.  In FP64 mode qw aliases q64.
template <class T>
struct Work {
    T *qw;          // [5][nTotal] working primitive state
    T *grad;        // [15][nCell]: d/dx of 5 vars, then d/dy, then d/dz
    T *limit;       // [nTotal]
    T *res;         // [5][nCell]
    T *invspec;     // [nCell] inviscid spectral radius ("invSpectralRadius")
    T *visspec;     // [nCell] viscous spectral radius ("visSpectralRadius"), viscous runs only
    T *dtraw;       // [nCell] CFL * vol / spec before the ktmax clamp
    T *dq;          // [5][nTotal]
    T *dflux;       // [5][nCell] LU-SGS delta flux carried between sweeps
    T *diag;        // [nCell]
    // LU-SGS coefficients that do not depend on dq, filled by the residual
    // pass: per (cell, face slot) of the cell-to-face list the split
    // eigenvalue l1 and the MXDQ weights x1, x2 of the neighbour across that
    // face; per cell the squared sound speed and total enthalpy.
    T *coef;        // [3][c2fLen]
    T *c2;          // [nTotal]
    T *hm;          // [nTotal]
};

struct Reduce {
    unsigned long long mindt_bits;  // min over cells of dtraw (positive doubles order as integers)
    double resnorm[5];
    int negcount;
    unsigned int barrier;           // monotonic arrival counter of the LU-SGS grid barrier
    int error;                      // PHX_ERR_TIMEOUT when a bounded wait gave up
    int step;                       // outer step (CFL ramp)
};

// Kernel launchers (phx_kernels.cu).
template <class T>
void launch_boundary(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s);
template <class T>
void launch_gradient_limiter(const DevGrid &g, const NsConst &c, const Work<T> &w, cudaStream_t s);
template <class T>
void launch_residual(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, double cfl, cudaStream_t s);
template <class T>
int launch_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, Reduce *red,
                 int numSMs, cudaStream_t s);
template <class T>
void launch_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *q64_new, T *qw_out,
                   Reduce *red, int *neglist, cudaStream_t s);
template <class T>
void launch_solution_fix(const DevGrid &g, const NsConst &c, const double *q64, double *q64_new, T *qw_out,
                         Reduce *red, int *neglist, cudaStream_t s);

}  // namespace phx
