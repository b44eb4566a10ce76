/* Oracle: a plain-C, single-threaded restatement of the reference's
 * unstructured NS / SA per-iteration path (PHengLEI NSSolverUnstruct /
 * TurbSolverUnstr).  TEST INFRASTRUCTURE ONLY: it is the parity checker for
 * the CUDA product and the timed CPU baseline ("port"); the product never
 * links, loads or calls it.  Each function cites the reference lines it
 * restates.  Arrays are the reference's SoA layout: cell fields hold nTotal =
 * nCell + nBFace entries, the ghost cell of boundary face f being nCell + f;
 * multi-variable fields are [var][nTotal]. */
#ifndef PHX_ORACLE_H
#define PHX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary condition codes (API/Geometry/include/Geo_SimpleBC.h:32-39). */
enum { OX_BC_EXTRAPOLATION = 1, OX_BC_SOLID_SURFACE = 2, OX_BC_SYMMETRY = 3,
       OX_BC_FARFIELD = 4, OX_BC_INFLOW = 5, OX_BC_OUTFLOW = 6 };
/* PHENGLEI::INTERFACE (Geo_SimpleBC.h:32): a face cut by the partition; its
 * ghost holds the neighbouring part's cell, filled by the caller's halo
 * exchange (Geo_UnstructGrid.cpp:10806-10990). */
enum { OX_BC_INTERFACE = -1 };

typedef struct {
    int n_node, n_face, n_cell, n_bface;
    const double *x, *y, *z;
    const int *face_off;     /* [n_face+1] offsets into face2node */
    const int *face2node;
    const int *left, *right; /* right of boundary face f = n_cell + f */
    const int *cell_off;     /* [n_cell+1] offsets into cell2node */
    const int *cell2node;
    int n_region;
    const int *region_type;  /* [n_region] bcType, regions in the solver's order */
    const int *bface_region; /* [n_bface] region index */
} ox_grid;

typedef struct {
    double *xfn, *yfn, *zfn, *area;   /* [n_face] */
    double *xfc, *yfc, *zfc;          /* [n_face] */
    double *xcc, *ycc, *zcc, *vol;    /* [nTotal] */
    double *skew;                     /* [n_cell] degrees, 90 = orthogonal */
    double *walldist;                 /* [n_cell] or NULL */
    double avg_vol;
    /* cell -> face lists in ascending face order, [n_cell+1] offsets */
    int *c2f_off, *c2f;
    /* least-squares weights (UnstructGrid::ComputeWeight,
     * Geo_UnstructGrid.cpp:3761-3935): iwt [n_face], inverse normal matrix
     * ixx..iyz [n_cell]; filled when non-NULL */
    double *iwt, *ixx, *iyy, *izz, *ixy, *ixz, *iyz;
} ox_metrics;

typedef struct {
    double gama;            /* refGama */
    double mach, attack, sideslip;  /* attack / sideslip in radians */
    double prim_inf[5];     /* non-dimensional freestream primitive state */
    double coef_state;      /* 1 / (gama M^2) */
    double p_total;         /* pTotal of PerfectGas::ComputePTotal */
    int viscous;            /* 0 inviscid, 1 laminar, 3 SA */
    double reynolds;        /* refReNumber (non-dimensional, per unit grid length) */
    double prandtl, prandtl_turb;
    double tsuth_nd;        /* Sutherland constant / reference temperature */
    double wall_temperature;/* <= 0: adiabatic */
    int gradient;           /* 0 ggcell, 1 lsq, 2 ggnode */
    int limiter;            /* OX_LIMITER_*: uns_limiter_name (scalar limiter from rho and p) */
    double venkat_coeff;
    int recon_method;       /* reconmeth: 0 own limiter, 1 min(L,R) */
    int scheme;             /* OX_SCHEME_*: uns_scheme_name */
    int entropy_fix;        /* roeEntropyFixMethod (3 supported) */
    double entropy_acoustic, entropy_convective;
    double cfl_start, cfl_end;
    int cfl_vary_step;
    double ktmax;
    int n_sweeps;           /* nLUSGSSweeps */
    double lusgs_tol;
    double skewness_angle;  /* viscous-flux skewness switch, degrees */
    /* Spalart-Allmaras (viscous == 3; Param_TurbSolver.cpp:20-280) */
    double nut_inf;         /* freeStreamTurbVar[ISA] = muoo / (rho_inf + SMALL) */
    double vist_inf;        /* freeStreamViscosity (far-field inflow ghost eddy viscosity) */
    double turb_cfl_scale;  /* turbCFLScale */
    double turb_skew_angle; /* turbSkewnessAngle, degrees */
    double ausmpw_limiter;  /* AusmpwPlusLimiter (Param_CFDSolver.cpp:116-120) */
    int flow_init_step;     /* flowInitStep: outer steps 1..flow_init_step run first order with Van Leer */
    int first_order;        /* set by ox_ns_iteration on its copy while isInIniting holds */
} ox_params;

/* uns_limiter_name (GetLimiterID, API/Physics/src/Limiter.cpp:1279-1300; vencat with ivencat 7) */
enum { OX_LIMITER_NOLIM = 0, OX_LIMITER_VENCAT = 1, OX_LIMITER_FIRST = 2, OX_LIMITER_BARTH = 3 };

/* uns_scheme_name (GetSchemeID, API/Physics/src/Flux_Inviscid.cpp:16-86) */
enum { OX_SCHEME_ROE = 0, OX_SCHEME_AUSMPW_PLUS = 1, OX_SCHEME_STEGER = 2, OX_SCHEME_VANLEER = 3,
       OX_SCHEME_HLLE = 4, OX_SCHEME_AUSMDV = 5, OX_SCHEME_AUSMPW = 6, OX_SCHEME_VANLEER_ROTATE = 7 };

/* Grid metrics: API/Geometry/src/Geo_UnstructGrid.cpp:5911-6156 (faces),
 * 6545-6819 (cells), 2206-2340 (skewness), Region.cpp:2655-2734 (avg volume),
 * Geo_UnstructGrid.cpp:1246-1304 (cell2face). */
void ox_compute_metrics(const ox_grid *g, ox_metrics *m);
/* UnstructGrid::ComputeWeight again, after the caller has set the interface
 * ghosts' centres to the neighbouring cells' (Region::SwapGeometry,
 * API/Physics/src/Region.cpp:3257-3268). */
void ox_lsq_weights(const ox_grid *g, ox_metrics *m);

/* One full outer iteration of NSSolverUnstruct (Controller::Relaxation
 * tscheme=LU_SGS, CFD/Solver/src/Controller.cpp:549-587) at outer step
 * `step` (1-based, drives the CFL ramp).  q [5][nTotal] is updated in place.
 * Work arrays (may be NULL to use internal scratch): see ox_ns_work. */
typedef struct {
    double *gama, *t;            /* [nTotal] */
    double *dqdx, *dqdy, *dqdz;  /* [5][nTotal] */
    double *limit;               /* [nTotal] scalar limiter */
    double *res;                 /* [5][nTotal] */
    double *inv_spec, *vis_spec; /* [n_cell] */
    double *dt;                  /* [nTotal] dt / vol after the reduction */
    double *dq;                  /* [5][nTotal] */
    double *visl, *vist;         /* [nTotal] */
    double *dtdx, *dtdy, *dtdz;  /* [nTotal] temperature gradient */
    double res_norm;             /* sqrt(sum res_rho^2 / nCell) */
    int n_negative;              /* cells repaired by SolutionFix */
    /* Spalart-Allmaras working variable nu~ and its solver arrays */
    double *qt, *res_t, *spec_t, *dqt;  /* [nTotal] */
    double *matl, *matr;                /* [n_face] mat_turbl / mat_turbr */
    double *dntx, *dnty, *dntz;         /* [nTotal] gradient of nu~ */
    double *qnode;                      /* [5][n_node] GG-node node values of the last gradient, or NULL */
    double *tnode_prev;                 /* [n_node] GG-node temperature node values for the next iteration */
    int have_tnode_prev;                /* 0 after initialisation or a state load */
    double *qtnode;                     /* [n_node] GG-node node values of nu~ for the next SA gradient */
    int have_qtnode;                    /* 0 after initialisation or a state load */
} ox_ns_work;

void ox_ns_iteration(const ox_grid *g, const ox_metrics *m, const ox_params *p,
                     int step, double *q, ox_ns_work *w);

/* Individual phases (for per-kernel parity tests). */
void ox_ns_boundary(const ox_grid *g, const ox_metrics *m, const ox_params *p, double *q, const double *gama);
void ox_gamma_temperature(const ox_grid *g, const ox_params *p, const double *q, double *gama, double *t);
void ox_gradient(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *f,
                 double *dfdx, double *dfdy, double *dfdz);
void ox_node_values(const ox_grid *g, const ox_metrics *m, const double *f, int nv, const double *t, double *fn,
                    double *tn);
void ox_gradient_ggnode(const ox_grid *g, const ox_metrics *m, const double *q, const double *qn, double *dx,
                        double *dy, double *dz);
void ox_qturb_node_values(const ox_grid *g, const double *qt, double *qn);
void ox_limiter(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                const double *dqdx, const double *dqdy, const double *dqdz, double *limit);
void ox_inviscid_flux(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                      const double *gama, const double *dqdx, const double *dqdy, const double *dqdz,
                      const double *limit, double *res);
void ox_spectrum(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                 const double *gama, const double *visl, const double *vist, double *inv_spec, double *vis_spec);
double ox_cfl(const ox_params *p, int step);
void ox_timestep(const ox_grid *g, const ox_metrics *m, const ox_params *p, int step, const double *q,
                 const double *inv_spec, const double *vis_spec, double *dt);
/* ox_timestep in two halves for a partitioned run: the CFL-scaled
 * vol / spectral radius of every cell, returning their minimum; then the
 * ktmax clamp from the minimum over all zones (Controller::GetGlobalMinTimeStep,
 * Controller.cpp:720-751, PH_CompareMaxMin) and the division by the volume. */
double ox_timestep_raw(const ox_grid *g, const ox_metrics *m, const ox_params *p, int step, const double *q,
                       const double *inv_spec, const double *vis_spec, double *dt);
void ox_timestep_clamp(const ox_grid *g, const ox_metrics *m, const ox_params *p, double mindt, double *dt);
/* The two halves of a single LU-SGS sweep, for a partitioned run
 * (Controller::LUSGS, Controller.cpp:1917-1924): the forward sweep then
 * SetGhostDQLUSGS (interface ghosts get dq = 0, its default branch); the
 * caller fills the interface ghosts with the neighbours' forward dq
 * (CommunicationDQ); then the backward sweep.  dflux [5][nTotal] carries the
 * forward sweep's lower fluxes; both need n_sweeps == 1. */
void ox_lusgs_forward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                      const double *gama, const double *visl, const double *vist, const double *res,
                      const double *dt, const double *inv_spec, const double *vis_spec, double *dq, double *dflux);
void ox_lusgs_backward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                       const double *gama, const double *visl, const double *vist, const double *res,
                       const double *dt, const double *inv_spec, const double *vis_spec, double *dq, double *dflux);
void ox_lusgs(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *gama,
              const double *t, const double *visl, const double *vist, const double *res, const double *dt,
              const double *inv_spec, const double *vis_spec, double *dq);
int ox_update(const ox_grid *g, const ox_metrics *m, const ox_params *p, double *q, const double *gama,
              const double *dq);
double ox_residual_norm(const ox_grid *g, const double *res);
void ox_viscosity(const ox_grid *g, const ox_params *p, const double *t, double *visl, double *vist);
/* Wall force sums of NSSolverUnstruct::AirForceCoefParts (NSSolverUnstruct.cpp:
 * 16026-16240, all solid-wall faces, torque reference at the origin): out[16] =
 * CA_f CA_p CN_f CN_p CZ_f CZ_p cpx cpy cpz Cl_f Cl_p Cn_f Cn_p Cm_f Cm_p 0,
 * from the current state, the NS step's gradients and laminar viscosity. */
void ox_forces(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const ox_ns_work *w,
               double *out);
/* One outer step of TurbSolverUnstr (SA, NSMB formation), run after the NS
 * step of the same outer iteration (Simulation::SolveSteady,
 * Main/src/Simulation.cpp:1527-1560). */
void ox_sa_step(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w);
/* ox_sa_step in the phases a partitioned run exchanges between
 * (Controller.cpp:1288 gradient of nu~, :1917-1924 dq between the sweeps,
 * TurbSolver::PostSolve q_turb and vist; TurbSolverUnstr::SetGhostDQLUSGS
 * leaves interface ghosts to that exchange, TurbSolverUnstr.cpp:1660).
 * dfl [nTotal] carries the forward sweep's lower fluxes. */
void ox_sa_gradient_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w);
void ox_sa_residual_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w);
void ox_sa_lusgs_forward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl);
void ox_sa_lusgs_backward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl);
void ox_sa_post_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w);
void ox_sa_boundary(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *gama,
                    double *qt, double *vist);
void ox_viscous_flux(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *t,
                     const double *visl, const double *vist, const double *dqdx, const double *dqdy,
                     const double *dqdz, const double *dtdx, const double *dtdy, const double *dtdz, double *res);

#ifdef __cplusplus
}
#endif
#endif
