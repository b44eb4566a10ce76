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
    BK_INTERFACE = 4,  // a face cut by a partition (PHENGLEI::INTERFACE): the ghost is the neighbouring part's
                       // cell, filled by halo exchanges; every pass but the boundary treats the face as interior
};

// Record strides (elements).
constexpr int kQ = 8;      // qrec: rho u v w p | c2 hm | limiter
constexpr int kG = 20;     // grec: (d/dx, d/dy, d/dz) of var k at 3k..3k+2 | pad | temperature gradient 16..18 | pad
constexpr int kC = 8;      // crec: res0..4 | 1 / LU-SGS diagonal (unclamped dt) | inviscid | viscous spectral radius
constexpr int kD = 8;      // dqrec / dflux: 5 values | pad
constexpr int kF = 8;      // frec (FP64): nx ny nz area xfc yfc zfc | least-squares face weight
constexpr int kX = 4;      // xrec (FP64): xcc ycc zcc vol
constexpr int kFlux = 16;  // face flux record: inviscid F0..4 (times area) | inviscid and viscous
                           // spectral parts | pad | viscous F1..4 (times area; F0 is zero) | pad
constexpr int kN = 8;      // nrec (GG-node): q node values (5), temperature node values of this
                           // iteration's state, those the gradient uses (the previous state's), pad
constexpr int kCoef = 4;   // LU-SGS factors per face use: l1 x1 x2 | viscous spectral term
constexpr int kSweepLanes = 4;   // LU-SGS lanes (neighbour entries) per schedule slot
constexpr int kSweepSlots = 8;   // slots per warp: schedule levels are padded to this multiple
constexpr int kSweepMaxEntries = 2 * kSweepLanes;   // entries of a cell: one slot, or two adjacent slots
constexpr long long kDefaultSpinLimit = 20000000LL;   // polls per dependency wait (~1-2 s)
constexpr int kMaxDevices = 64;                       // per-device launch caches
// Spalart-Allmaras records
constexpr int kTr = 4;     // trec: nu~ | eddy viscosity | laminar viscosity of the NS step | pad
constexpr int kTg = 4;     // tgrad: d nu~ / dx, dy, dz | pad
constexpr int kTc = 4;     // tcrec: res_turb | spec_turb | pad
constexpr int kTf = 8;     // tface: convective flux | diffusion flux1, flux2 | upwind Jacobians L, R |
                           // diffusion spectral term | pad

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
    // the normal derivative), bit 2 = both angles above turbSkewnessAngle and
    // |dL|, |dR| > TINY (the SA diffusion's normal derivative); pure geometry,
    // decided on the host
    const uint8_t *vflag;
    const int *c2f_off, *c2f;    // faces of each cell, ordered by the reference face number
    const int *orig;             // [nTotal] reference number of each cell (ghost: nCell + reference face)
    const int32_t *bkind;        // [nBFace] BcKind
    const int32_t *btype;        // [nBFace] bcType
    const uint8_t *farfield_adj; // [nCell] 1 if the cell touches a limiter-zeroing boundary
    // LU-SGS schedules, slots in level order (levels padded with idle slots):
    // pinfo = {storage cell or -1, entry count}, {cell, -1} on the second slot
    // of a cell with more than kSweepLanes entries; ent = kSweepLanes entries
    // per slot, the neighbours on the sweep's side in the cell's face order:
    // {neighbour (-1: unused lane), face (sign bit set when the normal points
    // into the cell), index of the face use's factors (2 f + side), 0}.
    const int2 *fwd_pinfo, *bwd_pinfo;
    const int4 *fwd_ent, *bwd_ent;
    // GG-node (gradientName 2): per storage node, its contributions {storage
    // cell, or storage boundary face with the sign bit set} with 1/distance
    // weights in the reference's order and their sum; per storage face, its
    // storage nodes in the face's node order
    int nNode;
    const int *node_off, *node_src;
    const double *node_w, *node_wsum;
    const int *fn_off, *fn_idx;
    // GG-node of the SA variable: per storage node, the {owner, other side}
    // pairs whose values it averages, in the reference's order
    const int *tn_off;
    const int2 *tn_pairs;
    int nFwdLevels, nBwdLevels;
    int nFwdPos, nBwdPos;        // schedule slots incl. idle padding (-1 cells)
    double avgVol;
};

// Scalars of the NS path (derived from phx_params as the reference's
// Param_NSSolverUnstruct and PerfectGas do).
struct NsConst {
    double gama, coefState, pTotal;
    double primInf[5];
    double acoustic, convective;   // Roe entropy-fix coefficients
    int scheme;                    // PHX_SCHEME_* in use (Van Leer during the flow initialisation)
    int firstOrder;                // flow initialisation: no reconstruction, zero limiter
    double ausmpwLim;              // AusmpwPlusLimiter
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
    // Spalart-Allmaras (viscousType 3): free-stream nu~ and eddy viscosity of
    // far-field inflow ghosts, turbCFLScale
    double nutInf, vistInf, turbCflScale;
    int saSource;                  // 0 exact source, 1 learned source (exact for nu~ <= 0), 2 learned inside its
                                   // training hull, exact outside
    long long spinLimit;           // polls per device-side dependency wait before PHX_ERR_TIMEOUT
    int holdCell;                  // fault injection: storage cell whose forward LU-SGS result never comes (the
                                   // wait on it runs out); -1 off
};

// Working arrays of one precision T (double: FP64 path, float: mixed path).
template <class T>
struct Work {
    T *qrec;        // [nTotal][kQ] working state, c2 = |gamma p / rho|, total enthalpy, limiter
    T *grec;        // [nTotal][kG] primitive gradients (ghost rows: interface ghosts only, from the halo exchange)
    T *flux;        // [nFace][kFlux] face flux times area and inviscid spectral radius term
    T *coef;        // [2 nFace][kCoef] LU-SGS factors of each face use (side 0: the left cell's view)
    T *crec;        // [nCell][kC] residual, diagonal, spectral radii
    T *dtraw;       // [nCell] CFL * vol / spectral radius, before the ktmax clamp
    T *dqrec;       // [nTotal][kD] LU-SGS dq (backward sweep; write-once per sweep)
    T *dqfwd;       // [nTotal][kD] forward-sweep dq (write-once per sweep; ghost rows: interface ghosts, from
                    // the halo exchange between the sweeps)
    T *dflux;       // [nCell][kD] delta flux carried from the forward to the backward sweep (write-once)
    T *trec;        // [nTotal][kTr] SA variable, eddy and laminar viscosity (SA runs; else null)
    T *nrec;        // [nNode][kN] GG-node node values (GG-node runs; else null)
};

// Spalart-Allmaras working arrays (one precision T; the FP64 master nu~ is qt64).
template <class T>
struct TurbWork {
    double *qt64;   // [nTotal] master nu~
    T *tgrad;       // [nCell][kTg] gradient of nu~
    T *tcrec;       // [nCell][kTc] residual, spectral radius, its reciprocal, pad
    T *tface;       // [nFace][kTf] face terms
    T *tcoef;       // [2 nFace] LU-SGS matrix of each face use (side 0: left cell's view = mat_turbr)
    T *tdq;         // [nCell] LU-SGS dq (backward sweep; write-once per sweep)
    T *tdqf;        // [nCell] forward-sweep dq (write-once per sweep)
    T *tdfl;        // [nCell] forward delta flux (write-once per sweep)
    T *tsrc;        // [nCell] source computed by the learned-source kernel (sa_source != 0)
    T *qtnode;      // [nNode] GG-node node values of nu~ for the next SA gradient (GG-node runs; else null)
};

struct Reduce {
    unsigned long long mindt_bits;  // min over cells of dtraw (positive doubles order as integers)
    double resnorm[5];
    int negcount;
    int error;                      // PHX_ERR_TIMEOUT / PHX_ERR_NUMERIC
};

// Kernel launchers (phx_kernels.cu).
template <class T>
void launch_boundary(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s);
template <class T>
void launch_gradient_limiter(const DevGrid &g, const NsConst &c, const Work<T> &w, int nodePrev, cudaStream_t s);
template <class T>
void launch_residual(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, double cfl, cudaStream_t s);
// LU-SGS sweeps: bit 0 of `sweeps` runs the forward sweep (after resetting
// the sweep records), bit 1 the backward sweep; 3 runs both in one launch.
constexpr int kSweepForward = 1, kSweepBackward = 2, kSweepBoth = 3;
template <class T>
int launch_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, Reduce *red, int numSMs, cudaStream_t s,
                 int sweeps = kSweepBoth);
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
// out[m] = sum over cells of res_m^2 (FP64 device reduction of the residual record).
template <class T>
void launch_resnorm(const DevGrid &g, const Work<T> &w, double *out, int numSMs, cudaStream_t s);
// NS boundary after the update (Controller::PostSolve): ghost states only,
// the laminar viscosity of the ghosts keeps its value of the NS step.
template <class T>
void launch_boundary_post(const DevGrid &g, const NsConst &c, double *q64, const Work<T> &w, cudaStream_t s);
// Spalart-Allmaras step (phx_sa.cu).
template <class T>
void launch_sa_boundary(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w,
                        const TurbWork<T> &t, cudaStream_t s);
struct MlpDev;
template <class T>
void launch_sa_residual(const DevGrid &g, const NsConst &c, const double *q64, const Work<T> &w,
                        const TurbWork<T> &t, Reduce *red, const MlpDev *mlp, unsigned long long *nmlp, int numSMs,
                        cudaStream_t s);
// Learned SA source (phx_mlp.cu): source of every cell into t.tsrc; training-sample capture.
template <class T>
void launch_mlp_source(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t,
                       const MlpDev &mlp, Reduce *red, unsigned long long *nmlp, int numSMs, cudaStream_t s);
template <class T>
void launch_mlp_capture(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, float *feat,
                        float *targ, int *cells, float *scales, long long cap, unsigned long long *count,
                        cudaStream_t s);
template <class T>
void launch_turb_node_values(const DevGrid &g, const Work<T> &w, const TurbWork<T> &t, cudaStream_t s);
template <class T>
int launch_sa_lusgs(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, Reduce *red,
                    int numSMs, cudaStream_t s, int sweeps = kSweepBoth);
template <class T>
void launch_sa_update(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, cudaStream_t s);
// Wall force sums (16 doubles, the last zero) of the current state.
template <class T>
void launch_forces(const DevGrid &g, const NsConst &c, const Work<T> &w, const double *q64, double *out,
                   cudaStream_t s);
// qt64[i] = in[orig[i]] and the working copy in trec, cells and ghosts.
template <class T>
void launch_import_turb(const DevGrid &g, const double *in, const TurbWork<T> &t, const Work<T> &w, cudaStream_t s);
void launch_finish_step(Reduce *r, double *hist, int i, double ncell, cudaStream_t s);
// trec slot 1 (eddy viscosity) of cells and ghosts from in[orig[i]].
template <class T>
void launch_import_vist(const DevGrid &g, const double *in, const Work<T> &w, cudaStream_t s);
// Halo exchange of a partitioned grid (phx_halo.cu): pack gathers rows of
// the cells `send` (storage indices) into buf, unpack scatters rows of buf
// into the ghosts `recv` (storage indices); `field` is a PHX_HALO_* code and
// a row holds halo_row_bytes<T>(field) bytes.
template <class T>
size_t halo_row_bytes(int field);
template <class T>
void launch_halo_pack(const DevGrid &g, int field, const double *q64, const Work<T> &w, const TurbWork<T> &t,
                      const int *send, int n, unsigned char *buf, cudaStream_t s);
template <class T>
void launch_halo_unpack(const DevGrid &g, const NsConst &c, int field, double *q64, const Work<T> &w,
                        const TurbWork<T> &t, const int *recv, int n, const unsigned char *buf, cudaStream_t s);

}  // namespace phx
