/* phx — B200-native (sm_100a) per-iteration hot path of PHengLEI's unstructured
 * compressible NS solver (NSSolverUnstruct) and its Spalart-Allmaras solver
 * (TurbSolverUnstr), exposed as a C ABI.
 *
 * Plain pointers and sizes only; no exceptions cross the boundary; every call
 * returns PHX_OK or a negative error code and leaves a message in
 * phx_last_error().  One context per host thread; all device work of a
 * context is issued on its stream (phx_set_stream); calls are synchronous with
 * respect to the host only where they return data to host memory.
 *
 * Each entry point names the reference solver method(s) it replaces (file:line
 * in the reference project).  The reference's own accelerator hook pattern is
 * `#ifdef USE_CUDA CallGPUxxx(grid, ...); return; #endif` at the top of those
 * methods (e.g. CFD/NSSolver/src/NSSolverUnstruct.cpp:13406-13412); a
 * `#ifdef USE_PHX` block in the same place calls the entry point below that
 * names the method, on the context the solver keeps for its grid.
 *
 * Layout conventions (the reference's, API/Geometry/include/Geo_UnstructGrid.h):
 *  - faces: boundary faces first (nBFace of them), then interior faces;
 *  - the face normal points from the left to the right cell;
 *  - cell fields hold nTotal = nCell + nBFace entries; the ghost cell of
 *    boundary face f is nCell + f;
 *  - multi-variable fields are structure-of-arrays [var][nTotal], primitive
 *    variables (rho, u, v, w, p), non-dimensionalised by the free stream. */
#ifndef PHX_H
#define PHX_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHX_OK 0
#define PHX_ERR_ARG -1       /* invalid argument (null pointer, bad size, unsupported option) */
#define PHX_ERR_CUDA -2      /* a CUDA runtime call failed */
#define PHX_ERR_TIMEOUT -3   /* a bounded device-side wait gave up (level barrier) */
#define PHX_ERR_NUMERIC -4   /* NaN / divergence detected in a reduction */
#define PHX_ERR_STATE -5     /* call out of order (e.g. no state uploaded) */

/* precision modes */
#define PHX_FP64 0   /* everything in FP64 (the reference's PH_DOUBLE_PREC) */
#define PHX_MIXED 1  /* FP32 flux/gradient/limiter/LU-SGS, FP64 metrics, update and reductions */

/* boundary condition codes: the reference's bcType values
 * (API/Geometry/include/Geo_SimpleBC.h:32-39) */
/* Inviscid schemes (uns_scheme_name; GetSchemeID / GetINVScheme,
 * API/Physics/src/Flux_Inviscid.cpp:16-134) */
#define PHX_SCHEME_ROE 0          /* "roe" */
#define PHX_SCHEME_AUSMPW_PLUS 1  /* "ausmpw+" */
#define PHX_SCHEME_STEGER 2       /* "steger" */
#define PHX_SCHEME_VANLEER 3      /* "vanleer" */
#define PHX_SCHEME_HLLE 4         /* "hlle" */
#define PHX_SCHEME_AUSMDV 5       /* "ausmdv" */
#define PHX_SCHEME_AUSMPW 6       /* "ausmpw" */
#define PHX_SCHEME_VANLEER_ROTATE 7 /* "vanleer_Rotate" */

/* Limiters (uns_limiter_name; GetLimiterID, API/Physics/src/Limiter.cpp:1279-1300) */
#define PHX_LIMITER_NOLIM 0       /* "nolim" */
#define PHX_LIMITER_VENCAT 1      /* "vencat" (ivencat 7) */
#define PHX_LIMITER_FIRST 2       /* "1st": first order */
#define PHX_LIMITER_BARTH 3       /* "barth" */

#define PHX_BC_EXTRAPOLATION 1
#define PHX_BC_SOLID_SURFACE 2
#define PHX_BC_SYMMETRY 3
#define PHX_BC_FARFIELD 4
#define PHX_BC_OUTFLOW 6
/* PHENGLEI::INTERFACE (Geo_SimpleBC.h:32): the faces of a zone cut by a
 * partition.  The ghost of such a face is the neighbouring zone's cell: its
 * values come from halo exchanges (phx_set_halo / phx_halo_pack /
 * phx_halo_unpack), never from the boundary pass, and every other pass treats
 * the face as an interior face. */
#define PHX_BC_INTERFACE -1

/* Halo fields, the interface data the reference uploads between zones: */
#define PHX_HALO_Q 0         /* FP64 state (NSSolver::PostSolve, CFD/NSSolver/src/NSSolver.cpp:139-142) */
#define PHX_HALO_GRADIENT 1  /* primitive and temperature gradients with the limiter
                                (Controller::ComputeGradient, CFD/Solver/src/Controller.cpp:1288, :1321) */
#define PHX_HALO_DQ 2        /* forward-sweep dq between the LU-SGS sweeps (Controller::LUSGS, :1917-1924) */
#define PHX_HALO_TURB 3      /* nu~ and eddy viscosity (TurbSolverUnstr::UploadInterfaceValue,
                                CFD/TurbSolver/src/TurbSolverUnstr.cpp:7130-7145) */

/* state selectors for phx_set_state / phx_get_state */
#define PHX_Q 0          /* primitive state [5][nTotal] */
#define PHX_RES 1        /* residual [5][nTotal] (the reference's "res") */
#define PHX_DT 2         /* time step / volume [nTotal] (the reference's "dt") */
#define PHX_LIMIT 3      /* scalar limiter [nTotal] ("limit2D" row 0) */
#define PHX_GRADX 4      /* primitive gradients [5][nTotal] ("gradPrimtiveVarX/Y/Z") */
#define PHX_GRADY 5
#define PHX_GRADZ 6
#define PHX_DQ 7         /* LU-SGS increment of the conservative variables [5][nTotal] */
#define PHX_INVSPEC 8    /* inviscid spectral radius [nCell] ("invSpectralRadius") */
#define PHX_VISSPEC 9    /* viscous spectral radius [nCell] ("visSpectralRadius") */
#define PHX_Q_TURB 10    /* SA working variable nu~ [nTotal] ("q_turb") */
#define PHX_VISL 11      /* laminar viscosity [nTotal] ("visl") */
#define PHX_VIST 12      /* eddy viscosity [nTotal] ("vist") */
#define PHX_RES_TURB 13  /* SA residual [nTotal] */
#define PHX_GEOM 14      /* geometry, see phx_get_geometry */
#define PHX_GRAD_TURB 16 /* gradient of nu~ of the last SA residual [3][nTotal] (x, y, z; ghosts 0) */
#define PHX_SA_SRC 15    /* learned SA source per unit volume of the last SA residual [nCell] (learned-source runs;
                            NaN where the cell took the exact source) */

typedef struct phx_ctx phx_ctx;

/* Grid, as UnstructGrid holds it (Geo_UnstructGrid.h).  Host arrays are read
 * during phx_ctx_create only. */
typedef struct {
    int64_t n_node, n_face, n_cell, n_bface;
    const double *x, *y, *z;              /* [n_node] node coordinates */
    const int32_t *face_nnode;            /* [n_face] node_number_of_each_face */
    const int32_t *face2node;             /* [sum face_nnode] */
    const int32_t *left_cell;             /* [n_face] leftCellOfFace */
    const int32_t *right_cell;            /* [n_face] rightCellOfFace (boundary: ignored) */
    const int32_t *cell_nnode;            /* [n_cell] node_number_of_each_cell */
    const int32_t *cell2node;             /* [sum cell_nnode] (sorted node set per cell) */
    int32_t n_region;                     /* boundary regions (UnstructBCSet) */
    const int32_t *region_type;           /* [n_region] bcType */
    const int32_t *bface_region;          /* [n_bface] region of each boundary face */
    const double *wall_dist;              /* [n_cell] wall distance, or NULL to compute */
} phx_grid_desc;

/* Parameters: the hypara keys of the reference (PHengLEI/examples/bin/cfd_para.hypara)
 * that the path reads, with the same meaning.  String keys become codes. */
typedef struct {
    int32_t precision;          /* PHX_FP64 or PHX_MIXED */
    double refGama;             /* ratio of specific heats */
    double refMachNumber;
    double attackd, angleSlide; /* degrees */
    int32_t viscousType;        /* 0 inviscid, 1 laminar, 3 one-equation SA */
    double refReNumber;         /* Reynolds number per unit grid length */
    double refDimensionalTemperature;
    double prl, prt;            /* laminar / turbulent Prandtl numbers */
    double tsuth;               /* Sutherland constant, K */
    double wallTemperature;     /* <= 0: adiabatic wall */
    int32_t gradientName;       /* 0 "ggcell", 1 "lsq", 2 "ggnode" */
    int32_t uns_limiter_name;   /* PHX_LIMITER_* (scalar limiter from rho and p) */
    int32_t ivencat;            /* Venkatakrishnan variant (7 supported) */
    double venkatCoeff;
    int32_t reconmeth;          /* 0 own limiter, 1 min of both sides */
    int32_t uns_scheme_name;    /* PHX_SCHEME_* */
    int32_t roeEntropyFixMethod;/* 3 (Harten) supported */
    double roeEntropyScale;
    double CFLStart, CFLEnd;
    int32_t CFLVaryStep;
    double ktmax;
    int32_t nLUSGSSweeps;
    double LUSGSTolerance;
    double skewnessAngle;
    double muoo;                /* SA free-stream nu~ / nu */
    double turbCFLScale;
    int32_t sa_source;          /* 0 exact SA source, 1 MLP, 2 MLP with exact fallback */
    double turbSkewnessAngle;   /* SA diffusion skewness switch, degrees */
    double freeStreamViscosity; /* eddy viscosity of far-field inflow ghosts (SA) */
    double AusmpwPlusLimiter;   /* weight limiter of the AUSMPW+ scheme */
    int32_t flowInitStep;       /* outer steps 1..flowInitStep run first order with Van Leer's flux */
    int32_t flowInitMethod;     /* 0 or 2 (1: boundary-layer start, 3: GMRES start, not supported) */
} phx_params;

/* Fills `p` with the reference's defaults for every key. */
void phx_default_params(phx_params *p);

/* Creates a context: uploads the grid, computes the FP64 metrics on the
 * device side of the context (face normals/areas/centres, cell centres and
 * volumes, skewness, wall distance), the cell-to-face lists and the LU-SGS
 * level schedules, and initialises the state to the free stream.
 * Replaces: Simulation::RunCFD grid set-up (Main/src/Simulation.cpp:205-260),
 * UnstructGrid::ComputeMetrics (API/Geometry/src/Geo_UnstructGrid.cpp:5695),
 * NSSolverUnstruct::AllocateGlobalVar / InitFlow, GPUGeomInfoAllocCopy. */
int phx_ctx_create(const phx_grid_desc *grid, const phx_params *params, phx_ctx **out);
int phx_ctx_destroy(phx_ctx *ctx);
const char *phx_last_error(const phx_ctx *ctx);
/* cudaStream_t as void*; NULL = the legacy default stream. */
int phx_set_stream(phx_ctx *ctx, void *stream);
/* Device on which the context was created. */
int phx_device(const phx_ctx *ctx);

/* Host <-> device state copies in the reference SoA layout.  n is the element
 * count of the host array (checked against the selector's size).  PHX_Q,
 * PHX_Q_TURB and PHX_VIST can be set; every selector can be read. */
int phx_set_state(phx_ctx *ctx, int which, const double *host, int64_t n);
int phx_get_state(phx_ctx *ctx, int which, double *host, int64_t n);
/* Device-pointer variants (FP64 device memory of the same layout). */
int phx_set_state_device(phx_ctx *ctx, int which, const double *dev, int64_t n);
int phx_get_state_device(phx_ctx *ctx, int which, double *dev, int64_t n);
/* Geometry as computed by the context: names "xfn","yfn","zfn","area","xfc",
 * "yfc","zfc" ([n_face]), "xcc","ycc","zcc","vol" ([nTotal]), "skew",
 * "walldist" ([n_cell]). */
int phx_get_geometry(phx_ctx *ctx, const char *name, double *host, int64_t n);

/* --- NS residual phases ---------------------------------------------------- */

/* Ghost-cell state of every boundary face.
 * Replaces NSSolverUnstruct::Boundary (CFD/NSSolver/src/NSSolverUnstruct.cpp:13404). */
int phx_ns_boundary(phx_ctx *ctx);

/* Gas state (gamma, T), laminar viscosity, primitive and temperature gradients
 * and the limiter.  Replaces NSSolverUnstruct::ComputeGamaAndTemperature
 * (:4666), ComputeViscousCoefficientWithoutChemical (:6722), ComputeGradient /
 * GetGradientField (:18171/:18244) and ComputeLimiter (:18189). */
int phx_ns_gradient_limiter(phx_ctx *ctx);

/* Inviscid and viscous face fluxes summed into res, the spectral radii and the
 * local time step (with the ktmax clamp).  Replaces NSSolver::UpdateResiduals
 * (CFD/NSSolver/src/NSSolver.cpp:71): InviscidFlux (NSSolverUnstruct.cpp:6912),
 * ViscousFlux (:7058), LoadFlux (:6435); plus SpectrumRadius (:15795),
 * NSSolver::TimeStep (NSSolver.cpp:51) and ReduceMaxTimeStep (:5717). */
int phx_ns_residual(phx_ctx *ctx);

/* Implicit LU-SGS solve for dq.  Replaces Controller::LUSGS
 * (CFD/Solver/src/Controller.cpp:1878): Diagonal (NSSolverUnstruct.cpp:15867),
 * SolveLUSGSForward (:15118), SetGhostDQLUSGS (:14767), SolveLUSGSBackward (:15446). */
int phx_ns_lusgs(phx_ctx *ctx);

/* Q += dq in conservative variables, back to primitive, positivity repair.
 * Replaces NSSolverUnstruct::UpdateFlowField (:14587) and SolutionFix (:14509). */
int phx_ns_update(phx_ctx *ctx);

/* Spalart-Allmaras step (viscousType = 3), run after phx_ns_update of the
 * same outer iteration, as Simulation::SolveSteady orders the solvers
 * (Main/src/Simulation.cpp:1527-1560).
 * phx_sa_boundary replaces TurbSolverUnstr::Boundary
 * (CFD/TurbSolver/src/TurbSolverUnstr.cpp:5919), after the NS PostSolve
 * boundary of the updated NS state (Controller::PostSolve,
 * CFD/Solver/src/Controller.cpp:5063).
 * phx_sa_residual replaces Controller::UpdateResiduals for TURB_SOLVER:
 * Viscosity (:6910), GetGradientField (:8652), TurbSolver::UpdateResiduals
 * (CFD/TurbSolver/src/TurbSolver.cpp:316: InitSpectrum :1025, SourceFlux
 * :2342, InviscidFlux :5187, ViscousFlux :3856) and Diagonal (:4675).
 * phx_sa_lusgs replaces SolveLUSGSForward / Backward (:1400, :1521).
 * phx_sa_update replaces UpdateFlowField (:1180) and the PostSolve boundary. */
int phx_sa_boundary(phx_ctx *ctx);
int phx_sa_residual(phx_ctx *ctx);
int phx_sa_lusgs(phx_ctx *ctx);
int phx_sa_update(phx_ctx *ctx);

/* Learned SA source (sa_source = 1: the MLP for every cell with nu~ > 0;
 * 2: the MLP inside its training hull, the exact source outside; the exact
 * source is always used for nu~ <= 0).  The MLP replaces production - wall
 * destruction of SourceFluxOneEquationOriginal (TurbSolverUnstr.cpp:2702);
 * the implicit part of the source stays exact.
 * phx_sa_capture writes, for every cell with nu~ > 0 after an SA residual,
 * the 6 raw input features ([count][6]) and the target of the exact source,
 * and optionally (non-NULL) each sample's reference cell number and the scale
 * that turns a network output into a source (source = target * scale).
 * phx_mlp_train trains the 6-64-64-64-1 SiLU network on the GPU (Adam, MSE;
 * seeded) and installs it; phx_mlp_get / phx_mlp_set move the model as a flat
 * float blob of phx_mlp_blob_size() values (weights, normalisation, hull).
 * phx_mlp_cells returns the running count of cells that used the MLP. */
int phx_sa_capture(phx_ctx *ctx, float *features, float *targets, int32_t *cells, float *scales, int64_t capacity,
                   int64_t *count);
int phx_mlp_train(phx_ctx *ctx, const float *features, const float *targets, int64_t n, int epochs, int batch,
                  double lr, uint64_t seed, double *final_loss);
int phx_mlp_get(phx_ctx *ctx, float *blob, int64_t n);
int phx_mlp_set(phx_ctx *ctx, const float *blob, int64_t n);
int64_t phx_mlp_blob_size(void);
/* One batch through the training kernels of phx_mlp_train, for checking them:
 * params is the flat weight vector (w1 [64][6], b1 [64], w2 [64][64], b2, w3
 * [64][64], b3, w4 [64], b4; phx_mlp_param_count() values, the first part of
 * the model blob), x the standardised inputs [n][6], y the scaled targets [n];
 * writes the mean squared error and its gradient with respect to params.  No
 * counterpart in the reference (its SA source has no learned part). */
int64_t phx_mlp_param_count(void);
int phx_mlp_loss_grad(const float *params, int64_t nparam, const float *x, const float *y, int64_t n, float *grad,
                      double *loss);
int phx_mlp_cells(phx_ctx *ctx, uint64_t *count);

/* nsteps outer iterations of the NS solver (and the SA solver when
 * viscousType = 3): the sequence of Controller::Relaxation with tscheme =
 * LU_SGS (Controller.cpp:549-587), driven as Simulation::SolveSteady
 * (Main/src/Simulation.cpp:1527).  If res_hist is not NULL it receives, per
 * step, the residual monitor of NSSolverUnstruct::GetResidual (:14258,
 * API/Physics/src/Residual.cpp:534): sqrt(sum res_rho^2 / nCell). */
int phx_ns_relaxation(phx_ctx *ctx, int nsteps, double *res_hist);

/* Wall force sums of the current state (NSSolverUnstruct::AirForceCoefParts,
 * CFD/NSSolver/src/NSSolverUnstruct.cpp:16026, all solid walls, torque
 * reference at the origin): out = CA_f CA_p CN_f CN_p CZ_f CZ_p cpx cpy cpz
 * Cl_f Cl_p Cn_f Cn_p Cm_f Cm_p 0, FP64 device reduction.  CL and CD follow
 * as in Force.cpp:441-536: scale by 1 / forceReferenceArea, then
 * CL = -sin(a) CFx + cos(a) CFy, CD = cos(a) cos(b) CFx + sin(a) cos(b) CFy + sin(b) CFz. */
int phx_forces(phx_ctx *ctx, double out[16]);

/* Residual monitor of the current res, per equation: out[m] =
 * sqrt(sum res_m^2 / nCell) (FP64 device reduction). */
int phx_residual_norm(phx_ctx *ctx, double out[5]);

/* Allocation-free residual monitor (no counterpart in the reference, whose
 * GetResidual reduces on the host): out_host[m] = sqrt(sum_{c < n_cell}
 * res_dev[m * n_total + c]^2 / n_cell) for m < nvar, over a device residual in
 * the reference's SoA layout, on `stream` (NULL: the default stream).  Needs no
 * context and allocates nothing: the partial sums live in a fixed 64 KiB
 * device array of the library (at most 8 variables; larger nvar is rejected
 * with PHX_ERR_ARG; any n_cell).  The first call on a device looks the array
 * up, so make it before any stream capture.  Each call waits for `stream` to
 * finish before it returns.  A CUDA error the calling thread left unchecked is
 * reported as PHX_ERR_CUDA and left in place, with nothing launched.  Calls
 * that overlap on one device share the array and race: serialise them. */
int phx_residual_norm_noalloc(const double *res_dev, int64_t n_cell, int64_t n_total, int nvar, double *out_host,
                              void *stream);

/* Bound on every device-side dependency wait of the LU-SGS sweeps, in polls
 * (default 20,000,000, about one to two seconds).  A wait that runs out ends
 * its sweep: the step's call returns PHX_ERR_TIMEOUT, the status is cleared,
 * and the context stays usable (its state is then undefined until the next
 * phx_set_state).  No counterpart in the reference, whose sweeps are
 * sequential host loops (Controller::LUSGS, Controller.cpp:1878). */
int phx_set_wait_limit(phx_ctx *ctx, int64_t polls);

/* Failure-detection hook for tests: the forward LU-SGS result of reference
 * cell `cell` never comes (-1: off), so the wait on it runs out and the step
 * returns PHX_ERR_TIMEOUT instead of hanging.  Nothing faults: the sweep
 * stops at its next level boundary.  No counterpart in the reference. */
int phx_fault_hold_cell(phx_ctx *ctx, int32_t cell);

/* --- partitioned grids (zones joined by PHX_BC_INTERFACE faces) ------------
 * One context per zone.  A partitioned step runs the phases one by one with
 * the reference's exchanges between them (Controller::Relaxation,
 * CFD/Solver/src/Controller.cpp:549-587; the interface communication of
 * Controller::CommunicationInterfaceData, :3389): boundary, gradient and
 * limiter, HALO GRADIENT, residual, the minimum time step over all zones,
 * forward sweep, HALO DQ (when swapDq is set, as the reference's parameter
 * file sets it), backward sweep, update, HALO Q; with SA: SA residual, SA
 * forward and backward sweeps, SA update, HALO TURB.  The SA dq is not
 * exchanged (Controller::CommunicationDQ, Controller.cpp:2874-2880, serves the
 * NS solver only), and the gradient of nu~ needs no exchange here: only its
 * own cell reads it.  The fused
 * phx_ns_relaxation, phx_ns_lusgs and phx_sa_lusgs refuse a context with
 * interface faces (PHX_ERR_STATE).  GG-node gradients are not supported
 * across zones (PHX_ERR_ARG at creation). */

/* Region::SwapGeometry (API/Physics/src/Region.cpp:3257-3268) and
 * Region::ComputeGlobalGridSize (:2655-2734): the cell centres and volumes of
 * the neighbouring zones' cells behind n interface faces bfaces[] (this
 * zone's boundary face numbers) become their ghosts' (UnstructGrid::
 * TranslateCellCenter, API/Geometry/src/Geo_UnstructGrid.cpp:4500-4541), and
 * the least-squares weights and viscous-flux switches are formed again;
 * avg_vol > 0 replaces the average cell volume the Venkatakrishnan limiter
 * scales with (the average over all zones).  Host arrays. */
int phx_swap_geometry(phx_ctx *ctx, int64_t n, const int32_t *bfaces, const double *xcc, const double *ycc,
                      const double *zcc, const double *vol, double avg_vol);

/* The halo plan of this zone: the n_send cells (this zone's cell numbers)
 * whose values the neighbouring zones receive, and the n_recv interface faces
 * (boundary face numbers) whose ghosts receive, each in the caller's order
 * (concatenated over the neighbours).  A cell is listed once per interface
 * face behind it, so n_send may exceed the cell count; each interface face is
 * listed once at most.  Host arrays, copied. */
int phx_set_halo(phx_ctx *ctx, int64_t n_send, const int32_t *send_cells, int64_t n_recv,
                 const int32_t *recv_bfaces);
/* Bytes of one row of a halo field (it depends on the precision). */
int64_t phx_halo_row_bytes(const phx_ctx *ctx, int field);
/* Gathers the send cells' rows of `field` into buf_dev (n_send rows), or
 * scatters buf_dev (n_recv rows) into the receiving ghosts, on the context's
 * stream.  Device buffers; the caller moves the rows between the zones
 * (peer copies, NCCL). */
int phx_halo_pack(phx_ctx *ctx, int field, void *buf_dev);
int phx_halo_unpack(phx_ctx *ctx, int field, const void *buf_dev);

/* The two LU-SGS sweeps of phx_ns_lusgs / phx_sa_lusgs as separate calls,
 * for the dq exchange between them (Controller::LUSGS, Controller.cpp:1917-1924;
 * CommunicationDQ :2874).  The NS backward sweep reads the interface ghosts'
 * dq from HALO DQ (zero without the exchange); the SA backward sweep, like the
 * reference's, takes an interface ghost's dq as zero. */
int phx_ns_lusgs_forward(phx_ctx *ctx);
int phx_ns_lusgs_backward(phx_ctx *ctx);
int phx_sa_lusgs_forward(phx_ctx *ctx);
int phx_sa_lusgs_backward(phx_ctx *ctx);

/* The smallest raw local time step of this zone after phx_ns_residual
 * (synchronises), and the minimum over all zones that the ktmax clamp of the
 * sweeps then uses (Controller::GetGlobalMinTimeStep, Controller.cpp:720-751). */
int phx_ns_min_timestep(phx_ctx *ctx, double *out);
int phx_ns_set_min_timestep(phx_ctx *ctx, double value);

/* Status of the device work issued so far (synchronises): PHX_ERR_TIMEOUT if
 * a sweep's bounded dependency wait ran out, PHX_ERR_NUMERIC if the positivity
 * repair overflowed, else PHX_OK; the status is cleared once reported.  The
 * phase calls above only launch; phx_ns_relaxation checks the same status
 * itself. */
int phx_step_status(phx_ctx *ctx);

/* Restart files.  phx_write_restart writes what the reference's restart holds
 * (NSSolverUnstruct::DumpRestartH5, CFD/NSSolver/src/NSSolverUnstruct.cpp:1247-1320;
 * TurbSolverUnstr::DumpRestartH5, CFD/TurbSolver/src/TurbSolverUnstr.cpp:506-560):
 * the outer step (outnstep), the primitive state q of cells and ghosts and,
 * with SA, q_turb and the eddy viscosity (visturb), in FP64, plus the
 * learned-source model when one is set; in a binary layout of its own (this
 * library reads no HDF5).  phx_read_restart loads such a file into a context
 * of the same grid (PHX_ERR_ARG when the cell or boundary-face counts differ,
 * as ReadRestartH5 checks nTotalCell, TurbSolverUnstr.cpp:669-676), so the run
 * continues from that step: an uninterrupted run and a restarted one give the
 * same state bit for bit (GG-cell and least-squares gradients; GG-node forms
 * its node values from the loaded state, as the reference's restart does). */
int phx_write_restart(phx_ctx *ctx, const char *path);
int phx_read_restart(phx_ctx *ctx, const char *path);

/* Outer step counter (drives the CFL ramp of NSSolver::ComputeCFL). */
int phx_set_step(phx_ctx *ctx, int step);
int phx_get_step(const phx_ctx *ctx);

/* Number of kernel launches the context has issued so far (for accounting). */
int64_t phx_launch_count(const phx_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
