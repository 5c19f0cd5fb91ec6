/*
 * fivo2d.h — C ABI of the B200 finite-volume stage for FiVoHydro's 2+1D solver.
 *
 * The library replaces, behind plain pointers and sizes, the Julia functions the
 * 2+1D driver `run_sim_2d!` (main2D.jl:371-561) calls once per time step:
 *
 *   step_ssprk2_2d! / step_ssprk3_2d!   src2d/timestepper2d.jl:74-103, 148-188
 *   rhs_2d!                             src2d/rhs2d.jl:169-249
 *   update_primitives_2d!               src2d/rhs2d.jl:57-65
 *   relax_dissipative_2d!               src2d/dissipation2d.jl:293-363
 *   compute_dt_2d                       src2d/timestepper2d.jl:37-47
 *   project_shear!                      main2D.jl:332-358
 *   prim_to_cons_2d! (IC path)          src2d/primrec2d.jl:753-796
 *   finalize_ic!                        main2D.jl:164-171
 *
 * Conventions
 *   - State U is the reference's `Matrix{Float64}(nv, Ntot)`: column-major, so
 *     cell i, field a lives at U[i*nv + a] (AoS per cell). Flat cell index
 *     i = ix*Nytot + iy (0-based; y is the fast index), src2d/grid2d.jl:85.
 *   - Field order is StateLayout2D's (src2d/state_layout2d.jl:61-84):
 *     Dtau, Sx, Sy, E, [nux, nuy], [Pi], [pixx, pixy, piyy, pieta],
 *     [pQxx, pQxy, pQyy, pQeta, PiQ] (the last five when consistent_m2 = 1).
 *   - Every function returns an int status: FIVO_OK (0) or a positive error
 *     code; fivo_last_error() returns the message of the last failure on the
 *     calling thread. A time step that the scheme cannot accept is NOT an
 *     error: it reports ok = 0, as step_ssprk2_2d! returns (false, Δ).
 *   - All host pointers are only read or written during the call.
 *   - One context owns one CUDA stream on the device that was current when the
 *     context was created; calls are synchronous unless named *_async.
 */
#ifndef FIVO2D_H
#define FIVO2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FIVO_ABI_VERSION 2

/* status codes */
#define FIVO_OK              0
#define FIVO_ERR_ARG         1   /* invalid argument / size mismatch          */
#define FIVO_ERR_CONFIG      2   /* model knob not implemented (reference refuses it too) */
#define FIVO_ERR_CUDA        3   /* CUDA runtime error                        */
#define FIVO_ERR_NOMEM       4   /* device allocation failed                  */
#define FIVO_ERR_DEVICE      5   /* a device-side loop hit its iteration cap  */

/* equation of state: src/eos.jl:39-84 (ConformalHQEOS), :318-519 (LatticeHRGEOS) */
#define FIVO_EOS_CONFORMAL_HQ  0
#define FIVO_EOS_LATTICE_HRG   1

/* shear / bulk transport models: src/primitives.jl:47-108 */
#define FIVO_SHEAR_ZERO        0   /* ZeroViscosity                             */
#define FIVO_SHEAR_QGP         1   /* QGPViscosity(eta/s, C_s)                  */
#define FIVO_BULK_ZERO         0   /* ZeroBulkViscosity                         */
#define FIVO_BULK_LORENTZ      1   /* SimpleBulkViscosity: Lorentzian at 0.175 GeV */
#define FIVO_BULK_GAUSS        2   /* Gaussian zeta/s(T) peak (new BulkViscosity subtype) */

/* boundary conditions: src2d/bc2d.jl:14-65 */
#define FIVO_BC_OUTFLOW        0
#define FIVO_BC_PERIODIC       1

/* integrators: main2D.jl:382 */
#define FIVO_SSPRK2            2
#define FIVO_SSPRK3            3

/* Terms register bits, in the field order of `Terms` (src/terms.jl:82-104). */
#define FIVO_TERM_NU_GRADALPHA     (1u << 0)
#define FIVO_TERM_FM_GRADT         (1u << 1)
#define FIVO_TERM_FM_INERTIAL      (1u << 2)
#define FIVO_TERM_FM_NU_GRADU      (1u << 3)
#define FIVO_TERM_FM_EXPANSION     (1u << 4)
#define FIVO_TERM_FM_DLNH          (1u << 5)
#define FIVO_TERM_M2_NU_GRADIENT   (1u << 6)
#define FIVO_TERM_M2_BG_GRADU      (1u << 7)
#define FIVO_TERM_M2_BG_DLNT       (1u << 8)
#define FIVO_TERM_M2_BG_DALPHA     (1u << 9)
#define FIVO_TERM_M2_EXPANSION     (1u << 10)
#define FIVO_TERM_M2_PI_SIGMA      (1u << 11)
#define FIVO_TERM_M2_PIQ_SIGMA     (1u << 12)
#define FIVO_TERM_M2_VORTICITY     (1u << 13)
#define FIVO_TERM_M2_PROJECTOR     (1u << 14)
#define FIVO_TERM_M2_ACCEL_NU      (1u << 15)
#define FIVO_TERM_M2_NU_GRADTH     (1u << 16)
#define FIVO_TERM_SHEAR_VORTICITY  (1u << 17)
/* Terms() defaults: every term on except m2_vorticity and shear_vorticity */
#define FIVO_TERMS_DEFAULT         0x1DFFFu

/*
 * Flattened IdealDiffVisc2DModel (src2d/primitives2d.jl:41-210) plus the EOS,
 * transport models and layout switches of build_model_2d (main2D.jl:85-123).
 * fivo_params_default() fills the reference's keyword defaults.
 * Doubles first, then 32-bit integers, so the struct has no interior padding.
 */
typedef struct fivo_params {
  /* --- EOS --- */
  double g_eff;             /* ConformalHQEOS g_eff (default 40)                 */
  double m_hq;              /* heavy-quark mass [GeV] (1.5)                      */
  double g_hq;              /* heavy-quark degeneracy (6)                        */
  double lhrg_a[4];         /* LatticeHRGEOS a1..a4                              */
  double lhrg_b[4];         /* LatticeHRGEOS b1..b4                              */
  double lhrg_c, lhrg_d;    /* LatticeHRGEOS c, d                                */
  double canon_factor;      /* LatticeHRGEOS canonical suppression I1/I0         */
  /* --- charge diffusion --- */
  double kappa_coeff;       /* D_s T [GeV fm]                                    */
  double tauN_coeff;        /* multiplies tau_n (1)                              */
  double deltaN_factor;     /* delta_N = factor * tau_n (0)                      */
  double nu_clip_factor;    /* |nu| <= f n u^tau, off when <= 0 (-1)             */
  double vacuum_n_lo;       /* charge-sector density ramp (1e-6)                 */
  double vacuum_n_hi;       /* (2e-3)                                            */
  /* --- shear --- */
  double eta_over_s;        /* QGPViscosity eta/s                                */
  double tauShear_coeff;    /* QGPViscosity C_s                                  */
  double deltaShear_factor; /* delta_pipi = factor * tau_pi (4/3)                */
  double taupi_pi_factor;   /* tau_pipi = factor * tau_pi (0)                    */
  double lambda_pi_Pi_factor; /* lambda_piPi = factor * tau_pi (0)               */
  double pi_clip_factor;    /* |pi^ij| <= f |P|, off when <= 0 (-1)              */
  /* --- bulk --- */
  double zeta_over_s;       /* peak zeta/s                                       */
  double tauPi_coeff;       /* C_zeta (15)                                       */
  double bulk_T0;           /* peak position [GeV] (Lorentzian: 0.175)           */
  double bulk_width;        /* width [GeV] (Lorentzian: 0.024)                   */
  double deltaPi_factor;    /* delta_PiPi = factor * tau_Pi (0)                  */
  double lambda_Pi_pi_factor; /* lambda_Pipi = factor * tau_Pi (0)              */
  double Pi_clip_factor;    /* |Pi| <= f |P|, off when <= 0 (-1)                 */
  /* --- domain / vacuum --- */
  double r_domain;          /* evolve only r <= r_domain (+Inf = whole box)      */
  double T_vac_cut;         /* vacuum cut temperature [GeV] (0.05)               */
  double E_vac_cut;         /* vacuum cut energy; <= 0 derives it from T_vac_cut */
  /* --- primitive recovery numerics (src2d/primrec2d.jl:465-472) --- */
  double primrec_tol;       /* row-scaled residual tolerance (1e-12)             */
  /* --- charm second moment --- */
  double transport_mass;    /* charm mass of the m2 transport coefficients [GeV];
                               <= 0 takes the EOS mass m_hq (0)                   */
  /* --- integers --- */
  int32_t eos_kind;         /* FIVO_EOS_*                                        */
  int32_t hq_times_fmGeV3;  /* multiply HQ (P,n,e) by fmGeV3                     */
  int32_t with_charge;      /* layout: nux, nuy present                          */
  int32_t enable_diff;
  int32_t enable_shear;     /* also: layout carries pixx, pixy, piyy, pieta      */
  int32_t enable_bulk;      /* also: layout carries Pi                           */
  int32_t shear_kind;       /* FIVO_SHEAR_*                                      */
  int32_t bulk_kind;        /* FIVO_BULK_*                                       */
  int32_t advect_nu, relax_advect_nu;
  int32_t advect_pi, relax_advect_pi;
  int32_t advect_Pi, relax_advect_Pi;
  int32_t vacuum_ramp_relax;
  int32_t shear_projected_deriv, diff_projected_deriv;
  int32_t shear_constraint_project; /* 1 = :project, 0 = :monitor                */
  int32_t consistent_fm, consistent_m2; /* charm closures (first, second moment);
                               consistent_m2 adds the five rows pQxx..PiQ          */
  int32_t primrec_maxit;    /* Newton iteration cap (80)                         */
  uint32_t terms;           /* FIVO_TERM_* bitmask                               */
  int32_t relax_advect_m2;  /* tau_M u^k d_k of the m2 rows inside the relaxation (1) */
  int32_t reserved0;        /* 0                                                 */
} fivo_params;

/* Diagnostics of the last call (run_sim_2d! NamedTuple, main2D.jl:558-560). */
typedef struct fivo_counters {
  int64_t nprimfail;        /* recovery failures (non-vacuum), last pass         */
  int64_t nvacuum;          /* PRR_VACUUM cells, last pass                       */
  int64_t primfail_index;   /* one representative failing cell, -1 if none      */
  int32_t primfail_reason;  /* its PrimRecReason (src/constants.jl:51-62)        */
  int32_t pad0;
  double  primfail_resnorm; /* its scaled residual                               */
  double  amax;             /* largest HLLE signal speed of the last rhs         */
  int64_t nmood;            /* MOOD stage retries in the last step               */
  int64_t nhalve;           /* dt halvings in the last step                      */
} fivo_counters;

/* Result of fivo_run (run_sim_2d!, main2D.jl:558-560). */
typedef struct fivo_run_result {
  int32_t ok;
  int32_t pad0;
  double  tau;
  int64_t nsteps;
  int64_t nprimfail;
  int64_t nvacuum;
  double  max_shear_res;
  double  maxu;
  double  dQ, Q0, Q1;
  double  minPtot;
} fivo_run_result;

/* CUDA-event timing of the library's kernels (fivo_profile), by kernel class:
 *   PRIM_FAST  recovery of every cell from its warm start, small iteration budget
 *   PRIM_SLOW  full cons_to_prim_2d! of the cells the fast pass deferred
 *   FACES      MUSCL + prim->cons + HLLE, x then y faces
 *   UPDATE     flux divergence + source, stage combination, floors, bounds
 *   ADM_SLOW   the inversions of cell_admissible_2d the update deferred
 *   RELAX      relaxation + shear projection
 *   OTHER      boundary frames, copies, masks, flag resets
 * launches[k] counts launch brackets of class k (FACES launches two kernels per
 * bracket); units[k] the cells (faces, for FACES) those launches processed. */
#define FIVO_KCLASS_PRIM_FAST 0
#define FIVO_KCLASS_PRIM_SLOW 1
#define FIVO_KCLASS_FACES     2
#define FIVO_KCLASS_UPDATE    3
#define FIVO_KCLASS_ADM_SLOW  4
#define FIVO_KCLASS_RELAX     5
#define FIVO_KCLASS_OTHER     6
#define FIVO_KCLASS_N         8
typedef struct fivo_kernel_times {
  int64_t launches[FIVO_KCLASS_N];
  double  ms[FIVO_KCLASS_N];
  int64_t units[FIVO_KCLASS_N];
  int64_t total_launches;   /* every kernel this context launched while enabled */
} fivo_kernel_times;

typedef struct fivo_ctx fivo_ctx;

/* --- library --- */
int         fivo_abi_version(void);
const char* fivo_last_error(void);
void        fivo_params_default(fivo_params* p);

/* --- context (Grid2D + Work2D mirror), src2d/grid2d.jl:52-71, src2d/work2d.jl:15-139 --- */
int  fivo_ctx_create(const fivo_params* p, int nx, int ny, int nghost,
                     double xmax, double ymax, fivo_ctx** out);
int  fivo_ctx_destroy(fivo_ctx* ctx);
int  fivo_ctx_info(const fivo_ctx* ctx, int* nv, int64_t* ntot, double* E_vac_cut);
/* Copy everything that determines the next steps of src into dst (state
 * buffers, primitives, warm starts and history, masks, the last signal speed
 * and the run bookkeeping): dst then advances to the same bits as src. Both
 * contexts must come from the same parameters and grid. A device-memory
 * checkpoint; no counterpart in the reference (Julia copies the arrays). */
int  fivo_ctx_clone_state(fivo_ctx* dst, const fivo_ctx* src);

/* --- state and history transfer --- */
int  fivo_upload_state(fivo_ctx* ctx, const double* U, int nv, int64_t ntot);
int  fivo_download_state(fivo_ctx* ctx, double* U, int nv, int64_t ntot);
/* Warm starts and dtau history (Work2D x0_*, *_prev); any pointer may be NULL. */
int  fivo_upload_history(fivo_ctx* ctx, int64_t ntot,
                         const double* x0_yT, const double* x0_phi,
                         const double* x0_ux, const double* x0_uy,
                         const double* ux_prev, const double* uy_prev,
                         const double* alpha_prev, const double* T_prev);
int  fivo_download_history(fivo_ctx* ctx, int64_t ntot,
                           double* x0_yT, double* x0_phi, double* x0_ux, double* x0_uy,
                           double* ux_prev, double* uy_prev,
                           double* alpha_prev, double* T_prev);
/* The charge-current history of the charm second moment (Work2D nux_prev,
 * nuy_prev, src2d/work2d.jl:46-47: nu after the previous relaxation, for d_tau nu);
 * any pointer may be NULL. Meaningful when consistent_m2 = 1. */
int  fivo_upload_nu_history(fivo_ctx* ctx, int64_t ntot, const double* nux_prev, const double* nuy_prev);
int  fivo_download_nu_history(fivo_ctx* ctx, int64_t ntot, double* nux_prev, double* nuy_prev);
/* NaN-seed every history vector (run_sim_2d! reset_history, main2D.jl:407-415). */
int  fivo_reset_history(fivo_ctx* ctx);
/* Cell primitives of the last recovery (Work2D yT..ok); any pointer may be NULL. */
int  fivo_get_primitives(fivo_ctx* ctx, int64_t ntot,
                         double* yT, double* phi, double* mu, double* alpha,
                         double* ux, double* uy, double* P, double* n, double* e,
                         uint8_t* ok);
int  fivo_get_counters(fivo_ctx* ctx, fivo_counters* out);

/* --- the stage --- */
/* rhs_2d!: BCs, primitive pass, MUSCL, HLLE, sources. mask = force_first_order
 * (Ntot bytes, NULL = none). dU (nv x Ntot AoS, may be NULL) receives the RHS. */
int  fivo_rhs(fivo_ctx* ctx, double tau, int bc, const uint8_t* mask, double* dU);
/* step_ssprk2_2d! / step_ssprk3_2d! on the resident state. */
int  fivo_step(fivo_ctx* ctx, int integrator, double tau, double dtau,
               int max_halve, int max_mood, int bc, double* dtau_used, int* ok);
/* update_primitives_2d!: BCs + primitive pass; returns the failure count. */
int  fivo_update_primitives(fivo_ctx* ctx, double tau, int bc, int64_t* nprimfail);
/* relax_dissipative_2d!: operator-split IS/DNMR relaxation, once per step. */
int  fivo_relax(fivo_ctx* ctx, double tau, double dtau);
/* project_shear!: pieta from tracelessness; returns max and mean residual. */
int  fivo_project_shear(fivo_ctx* ctx, double* max_res, double* mean_res);
/* compute_dt_2d from the amax of the last rhs. */
int  fivo_compute_dt(fivo_ctx* ctx, double tau, double cfl, double cfltau, double* dt);
/* run_sim_2d! (main2D.jl:371-561) on the resident state, without dumps. */
int  fivo_run(fivo_ctx* ctx, double tau0, double taufinal, double cfl, double cfltau,
              int integrator, int bc, int64_t max_steps, int reset_history,
              fivo_run_result* out);

/* The loop body of run_sim_2d! (main2D.jl:436-513) from tau for at most
 * max_steps steps (and not past taufinal), continuing the history and the
 * signal speed of the previous call: no initial rhs, no history reset, no
 * end-of-run diagnostics. out->tau is the new time, out->nsteps the steps taken.
 * A host that calls on_dump between chunks uses this instead of fivo_run. */
int  fivo_advance(fivo_ctx* ctx, double tau, double taufinal, double cfl, double cfltau,
                  int integrator, int bc, int64_t max_steps, fivo_run_result* out);
/* The end-of-run diagnostics of run_sim_2d! (main2D.jl:532-556) on the resident
 * state and primitives: *Q = sum of Dtau over the interior, *maxu = max |u|
 * over the interior, *minPtot = min(P + Pi) over interior cells with P > 0.
 * A host that ran fivo_advance chunks forms dQ from this Q and fivo_run's Q0. */
int  fivo_run_diagnostics(fivo_ctx* ctx, double* Q, double* maxu, double* minPtot);

/* --- initial conditions --- */
/* finalize_ic! (main2D.jl:164-171) on the resident state. */
int  fivo_finalize_ic(fivo_ctx* ctx, double tau0, int bc);
/* set_cell! / prim_to_cons_2d! for ncell cells at once (main2D.jl:142-154):
 * inputs are per-cell arrays (T, alpha = mu/T, ux, uy, Pi, pixx, pixy, piyy,
 * nux, nuy; the dissipative ones may be NULL = 0); pieta comes from
 * tracelessness. U receives nv x ncell (AoS), ok one byte per cell. */
int  fivo_set_cells(const fivo_params* p, int64_t ncell, double tau,
                    const double* T, const double* alpha,
                    const double* ux, const double* uy,
                    const double* Pi, const double* pixx, const double* pixy,
                    const double* piyy, const double* nux, const double* nuy,
                    double* U, uint8_t* ok);

/* --- equation of state (for IC builders and tests) --- */
/* eos_Pne (src/eos.jl:53-84, 483-519) for n points. */
/* The MC-Glauber initial condition of the event-by-event workload, built on the
 * device into the context's state (the reference's IC builder is not public; the
 * same construction runs on the host in fivo2d.ic.glauber_fields): Gaussian
 * deposits of width `width` of npart participants (x, y pairs, with weights) and
 * nbin binary collisions (x, y pairs) at every cell centre; energy density
 * e = e_edge + (e(Tpeak) - e_edge) s / max s over the light-sector e(T), with
 * e_edge = e(T_edge); T by 90-step bisection of e(T); charm density
 * n = n(T_edge, alpha_edge) + a part proportional to the binary density with
 * tau0 * sum dx dy = ncharm over the interior; alpha = log(n / n(T, alpha = 0)),
 * floored at alpha_min where it is not finite; u = 0 and no dissipative parts;
 * then set_cell! and finalize_ic! (main2D.jl:142-171) with boundary bc.
 * (T_edge, alpha_edge) is the edge state the event is laid on (the reference's
 * production profile carries T = 0.12786 GeV, alpha = 1.8878 at its edge,
 * data/initial_profiles_physical.csv); T_edge <= 0 builds it on vacuum instead.
 * T_out, alpha_out (Ntot each, may be NULL) receive the fields.
 * LatticeHRGEOS only. No counterpart in the reference. */
int  fivo_glauber_ic(fivo_ctx* ctx, double tau0, const double* parts, const double* weights,
                     int64_t npart, const double* binary, int64_t nbin, double width, double Tpeak,
                     double ncharm, double alpha_min, double T_edge, double alpha_edge, int bc,
                     double* T_out, double* alpha_out);
int  fivo_eos_Pne(const fivo_params* p, int64_t n, const double* T, const double* mu,
                  double* P, double* nq, double* e);

/* --- one-cell recovery (src2d/primrec2d.jl:465-486) for n independent cells --- */
/* cons[k*11 + j] = (D, Sx, Sy, E, nux, nuy, Pi, pixx, pixy, piyy, pieta) of cell k;
 * warm[k*4 + j] = (yT0, phi0, ux0, uy0) or NULL for a cold start.
 * prim[k*7 + j] = (T, mu, ux, uy, n, e, P); ok and reason one byte per cell. */
int  fivo_cons_to_prim(const fivo_params* p, int64_t n, double tau,
                       const double* cons, const double* warm,
                       double* prim, uint8_t* ok, uint8_t* reason);

/* --- rhs without device allocation --- */
/* No counterpart in the reference: an extra entry point for hosts that cannot
 * allocate device memory (see the comment block in fivo2d.cu). One rhs_2d!
 * evaluation with a cold-started recovery (no warm starts are kept), reading the
 * state U and writing the right-hand side dU, both caller-owned device buffers of
 * nv planes x Ntot doubles (plane a at ptr + a*Ntot). The ghost frame of U is
 * refilled in place, as rhs_2d! does. *amax (host) receives the largest HLLE
 * signal speed. counters (host, may be NULL) receives the primitive pass's
 * bookkeeping as fivo_get_counters reports it after fivo_rhs: nprimfail,
 * nvacuum, one failing cell and its reason, amax (failed cells are floored to
 * the cold vacuum state and the call still returns FIVO_OK, as rhs_2d! does).
 * stream may be NULL (the default stream); the call waits for it before
 * returning. Work memory is a fixed file-scope device array, so Ntot =
 * (nx+6)*(ny+6) must not exceed FIVO_NOALLOC_MAX_CELLS; concurrent calls on
 * overlapping streams race on it. */
#define FIVO_NOALLOC_MAX_CELLS 160000
int  fivo_rhs_noalloc(const fivo_params* p, int nx, int ny, double xmax, double ymax,
                      double tau, int bc, double* U, double* dU, double* amax,
                      fivo_counters* counters, void* stream);

/* --- batches of events (event-by-event hydro, uneven grids) ---
 * One context per event (same model, own grid), each on its own stream, driven
 * by nworkers host threads (<= 0: min(nevents, 32)); their waits block instead
 * of spinning. Event k's context (fivo_batch_event) takes the usual calls:
 * fivo_set_cells/fivo_upload_state for its IC, fivo_download_state, ... The
 * run and advance calls are run_sim_2d! and its loop body on every event at
 * once; results[k] and status[k] (may be NULL) are event k's. A run's outcome
 * per event is bitwise that of a separate fivo_run on the same context.
 * The reference has no batch driver (a Julia user loops over run_sim_2d!). */
typedef struct fivo_batch fivo_batch;
int  fivo_batch_create(const fivo_params* p, int nevents, const int* nx, const int* ny,
                       const double* xmax, const double* ymax, int nghost, int nworkers,
                       fivo_batch** out);
int  fivo_batch_destroy(fivo_batch* b);
int  fivo_batch_event(fivo_batch* b, int k, fivo_ctx** ctx);
int  fivo_batch_run(fivo_batch* b, double tau0, double taufinal, double CFL, double CFLtau,
                    int integrator, int bc, int64_t max_steps, int reset_history,
                    fivo_run_result* results, int* status);
int  fivo_batch_advance(fivo_batch* b, const double* tau, double taufinal, double CFL,
                        double CFLtau, int integrator, int bc, int64_t max_steps,
                        fivo_run_result* results, int* status);

/* Lockstep mode of a batch (enable != 0): fivo_batch_run and fivo_batch_advance
 * take every event's step at the same time, each kernel of the step launched
 * once over the blocks of all events (the deferred recoveries and admissibility
 * inversions as persistent kernels over the union of the events' queues), with
 * ONE host read for the whole batch per step: the post-step pass
 * (update_primitives_2d! + relax_dissipative_2d!, main2D.jl:486-502) follows in
 * the same sequence, speculating that the step is accepted. An event whose
 * optimistic step has an inadmissible cell is undone (speculation included) and
 * stepped alone by the usual stage-by-stage procedure with MOOD and halving; events that have
 * reached taufinal or max_steps sit out the launches. Results per event are
 * bitwise those of separate fivo_run calls. flags: FIVO_LOCKSTEP_GRAPHS
 * replays each launch sequence as a captured CUDA graph; FIVO_LOCKSTEP_TUNE
 * times the candidate schedules (block order of the events, blocks of the
 * persistent deferred pass, the face pass's two directions in one launch or two)
 * on the first 16 steps of the next run and keeps the fastest. Every event must use the same recovery (the plain one, or one
 * learned guess in one mode: its batched kernels take the network's tiles over
 * the events' cells or over the union of their deferred cells) and the same
 * precision. Replaces the reference's per-event loop over run_sim_2d!. */
#define FIVO_LOCKSTEP_GRAPHS 1
#define FIVO_LOCKSTEP_TUNE   2
int  fivo_batch_set_lockstep(fivo_batch* b, int enable, int flags);

#define FIVO_LOCKSTEP_MAXCAND 16
typedef struct fivo_lockstep_info {
  int32_t enabled, flags;
  int32_t ncand;            /* candidate schedules */
  int32_t chosen;           /* index of the kept one, -1 before tuning */
  int32_t cand_order[FIVO_LOCKSTEP_MAXCAND];    /* 0: events in batch order, 1: largest grid first */
  int32_t cand_slow[FIVO_LOCKSTEP_MAXCAND];     /* persistent deferred-pass blocks per SM */
  int32_t cand_fused[FIVO_LOCKSTEP_MAXCAND];    /* 1: both face directions in one launch */
  double  cand_ms[FIVO_LOCKSTEP_MAXCAND];       /* best step time measured (device, ms) */
  int64_t steps;            /* lockstep steps taken (batch-wide) */
  int64_t fallbacks;        /* event steps redone stage by stage */
  double  ms_step, ms_post; /* device time of the step and post-step launch sequences */
  int64_t kernels;          /* kernels launched by the sequences (graph nodes replayed included) */
} fivo_lockstep_info;
int  fivo_batch_lockstep_info(fivo_batch* b, fivo_lockstep_info* out);

/* One context through the same launch sequences (mode 1): fivo_run and
 * fivo_advance take each step as a batch of this one context, the step and the
 * post-step pass replayed as one CUDA graph on the context's stream (one graph
 * launch and one host read per step instead of about 32 kernel launches),
 * with the default schedule and the global-load face pass; mode 2 launches the
 * same sequences kernel by kernel; mode 0 (the default) is the context's own
 * per-kernel path. Results are the same bits in every mode. While fivo_profile
 * is on the per-kernel path is taken. fivo_ctx_lockstep_info reports the
 * sequences. Replaces nothing in the reference: its step is a sequence of Julia
 * calls (main2D.jl:436-513). */
int  fivo_ctx_set_graphs(fivo_ctx* c, int mode);
int  fivo_ctx_lockstep_info(fivo_ctx* c, fivo_lockstep_info* out);

/* --- the learned starting guess of the primitive recovery (no counterpart in
 * the reference: its Newton starts from the previous step's primitives or the
 * closed-form seed, src2d/primrec2d.jl:300-347,465-486) ---
 * An MLP 8 -> 64 -> 64 -> 3 (GELU; BF16 weights, FP32 accumulation on the
 * tensor cores) maps a cell's normalised (log E, S^x/E, S^y/E, Pi/E, pi^xx/E,
 * pi^xy/E, pi^yy/E, |S|/E) to (log T - log(E)/4, u^x, u^y); the charm chemical
 * potential of the guess follows in closed form from N^tau. A context with a
 * guess attached starts each cell's Newton there; a cell whose residual is above
 * 1e-10 after 3 updates falls back to the plain warm-started recovery. Results
 * then agree with the plain path to the recovery tolerance, not bitwise.
 * Parameters: FIVO_GUESS_NPARAM floats, W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[16][64] b3[16] (W[out][in]; columns 8..15 of W1, rows 3..15 of W3 and
 * b3[3..15] are padding and stay 0). Normalisation: FIVO_GUESS_NNORM floats,
 * in_mean[8] in_istd[8] out_mean[3] out_std[3]. A sample is 11 floats: the 8
 * raw features and the 3 raw targets. */
#define FIVO_GUESS_NPARAM 6288
#define FIVO_GUESS_NNORM 22
#define FIVO_GUESS_NSAMP 11
typedef struct fivo_guess fivo_guess;
typedef struct {
  uint64_t it_fast, n_fast;      /* Newton updates / attempts of the warm-started pass   */
  uint64_t it_learn, n_learn;    /* ... of the attempts from the learned guess           */
  uint64_t ok_learn;             /* learned attempts accepted                             */
  uint64_t it_fb, n_fb;          /* warm attempts after a rejected learned guess          */
  uint64_t deferred;             /* cells deferred to the slow pass                       */
} fivo_newton_stats;
/* on the device of `ctx_or_null` (the current device when NULL); weights drawn
 * from a seeded uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)), identity normalisation */
int  fivo_guess_create(fivo_ctx* ctx_or_null, uint64_t seed, fivo_guess** out);
int  fivo_guess_destroy(fivo_guess* g);
int  fivo_guess_set_params(fivo_guess* g, const float* params, const float* norm);
int  fivo_guess_get_params(fivo_guess* g, float* params, float* norm);
/* the device sample store: capacity in samples; set/get copy host samples in/out */
int  fivo_guess_reserve(fivo_guess* g, int64_t capacity);
int  fivo_guess_set_samples(fivo_guess* g, const float* samples, int64_t n);
int  fivo_guess_get_samples(fivo_guess* g, float* samples, int64_t n);
int  fivo_guess_nsamples(fivo_guess* g, int64_t* n);
/* append the (features, targets) pairs of ctx's interior cells: the features
 * from its current state, the targets from its last primitive pass, so that
 * pass must be of the current state (fivo_update_primitives after a step, whose
 * relaxation moved the dissipative rows); every stride-th cell from phase;
 * stops at capacity */
int  fivo_guess_harvest(fivo_ctx* ctx, fivo_guess* g, double tau, int stride, int phase);
/* normalisation = the mean and standard deviation of the stored samples */
int  fivo_guess_fit_norm(fivo_guess* g);
/* steps of Adam (beta 0.9, 0.999, eps 1e-8) on the mean-squared error of the
 * normalised outputs, batch = 128 * ctas_per_step samples drawn with a seeded
 * hash; loss_out[0] = the loss of the first step, loss_out[1] = of the last */
int  fivo_guess_train(fivo_guess* g, int steps, int ctas_per_step, float lr, uint64_t seed,
                      double* loss_out);
/* the gradient of the mean-squared error over n samples (n % 128 == 0, taken in
 * order) with respect to every parameter, and that loss; no update */
int  fivo_guess_grad(fivo_guess* g, const float* samples, int64_t n, float* grad, double* loss);
/* normalised outputs out[k*3 + o] for raw features raw[k*8 + q] */
int  fivo_guess_forward(fivo_guess* g, const float* raw, int64_t n, float* out);
/* attach (g) or detach (NULL) the guess; the context keeps no ownership */
int  fivo_ctx_set_guess(fivo_ctx* ctx, fivo_guess* g);
/* where the attached guess is used. FIVO_GUESS_EVERY_CELL (the default): the network's
 * guess is the starting point of every cell's Newton, the previous step's warm start
 * its per-cell fallback. FIVO_GUESS_DEFERRED: the warm starts run first as in the plain
 * path, and the network's guess is tried on the cells the warm start leaves (no warm
 * start, over the fast budget, failed) before the full cons_to_prim_2d!. */
#define FIVO_GUESS_EVERY_CELL 0
#define FIVO_GUESS_DEFERRED   1
int  fivo_ctx_set_guess_mode(fivo_ctx* ctx, int mode);
int  fivo_newton_stats_read(fivo_ctx* ctx, fivo_newton_stats* out, int reset);

/* --- mixed precision (no counterpart in the reference, which is FP64 throughout) ---
 * FIVO_PRECISION_FP32_FACES runs the face pass of rhs_2d! (MUSCL reconstruction,
 * the EOS at the faces, physical fluxes, wave speeds, HLLE) in FP32 and stores FP32
 * face fluxes; the recovery, the divergence and sources, the SSPRK combination,
 * the floors and the relaxation stay FP64. Results then differ from the FP64 path
 * at the FP32 rounding level of the fluxes (not bitwise).
 * FIVO_PRECISION_FP32 adds the relaxation's sources in FP32 (kinematics, the
 * Navier-Stokes targets, the projected-derivative, advection and coupling terms and
 * the consistent first moment's sources); the transport coefficients and the
 * backward-Euler update of each dissipative field stay FP64. Not available with
 * consistent_m2 (FIVO_ERR_CONFIG). */
#define FIVO_PRECISION_FP64        0
#define FIVO_PRECISION_FP32_FACES  1
#define FIVO_PRECISION_FP32        2
int  fivo_ctx_set_precision(fivo_ctx* ctx, int mode);

/* --- which kernel runs the FP64 face pass of rhs_2d! (_faces_2d!, src2d/rhs2d.jl:282-371) ---
 * Both give the same bits. FIVO_FACES_GLOBAL reads each face's stencil from global
 * memory; FIVO_FACES_TILE_* stages a halo tile of every plane the faces read in
 * shared memory by TMA first (needs Ny + 6 even), in tiles of TX x TY faces:
 * 0 = 4 x 32, 1 = 2 x 64, 2 = 8 x 16, 3 = 8 x 32. FIVO_FACES_AUTO (the default) times
 * every candidate on the context's first stage and keeps the fastest, one choice
 * per grid and layout shared by the contexts of the process. x_cfg and y_cfg are
 * the x- and y-face passes; fivo_ctx_face_pass reports the current choice. */
#define FIVO_FACES_AUTO    (-2)
#define FIVO_FACES_GLOBAL  (-1)
int  fivo_ctx_set_face_pass(fivo_ctx* ctx, int x_cfg, int y_cfg);
int  fivo_ctx_face_pass(fivo_ctx* ctx, int* x_cfg, int* y_cfg);

/* --- the freeze-out surface and its Cooper-Frye pion yield (freezeout2d.jl) ---
 * The surface tau = tau_fo(x, y) over ctx's interior cells: each record takes the
 * primitives of ctx's last primitive pass (fivo_update_primitives first, as
 * freeze_surface does after each chunk of the run) and, per cell, keeps the last
 * downward crossing of T_fo, interpolated linearly between records, with the flow
 * at that record (freezeout2d.jl:94-115). Arrays are Nx x Ny, cell (a, b) at
 * a * Ny + b; tau_fo is NaN where the cell has not frozen. counts = (cells ever
 * above T_fo, cells frozen, re-heatings after freezing). */
typedef struct fivo_fo fivo_fo;
typedef struct {
  double T_fo;       /* GeV (0.156)                                    */
  double m;          /* particle mass, GeV (pion: 0.138)               */
  double pt_lo, pt_hi;  /* p_T range, GeV (0.1, 5.0)                   */
  double eta_max;    /* |eta| <= eta_max (6)                           */
  double f_yield;    /* overall factor (2 charge states x 2.5 feed-down) */
  int32_t n_eta, n_pt, n_phi, pad;   /* grid (40, 40, 24)              */
} fivo_cf_params;
void fivo_cf_params_default(fivo_cf_params* p);
int  fivo_fo_create(fivo_ctx* ctx, double T_fo, fivo_fo** out);
int  fivo_fo_destroy(fivo_fo* f);
int  fivo_fo_reset(fivo_fo* f);
int  fivo_fo_record(fivo_fo* f, fivo_ctx* ctx, double tau);
int  fivo_fo_surface(fivo_fo* f, double* tau_fo, double* uxf, double* uyf, int64_t* counts);
int  fivo_fo_set_surface(fivo_fo* f, const double* tau_fo, const double* uxf, const double* uyf);
/* pion_yield (freezeout2d.jl:144-190): out = (dN/dy Boltzmann, dN/dy Bose,
 * negative-dSigma fraction of the Boltzmann integrand); one-sided tau_fo gradients
 * at the rim of the frozen region, cells without a gradient skipped */
int  fivo_cooper_frye(fivo_fo* f, const fivo_cf_params* p, double* out);

/* --- streams, synchronisation, timing --- */
int  fivo_sync(fivo_ctx* ctx);
/* Run the context's later calls on a caller's CUDA stream (a cudaStream_t of
 * the context's device, e.g. CUDA.jl's or torch's); NULL restores its own. */
int  fivo_ctx_set_stream(fivo_ctx* ctx, void* stream);
/* Enable (1) or disable (0) per-kernel CUDA-event timing. */
int  fivo_profile(fivo_ctx* ctx, int enable);
/* Accumulated kernel times since enabling or the last reset. */
int  fivo_profile_read(fivo_ctx* ctx, fivo_kernel_times* out, int reset);

#ifdef __cplusplus
}
#endif
#endif /* FIVO2D_H */
