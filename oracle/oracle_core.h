/*
 * oracle/oracle_core.h — CPU restatement of FiVoHydro's 2+1D finite-volume stage.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle for the CUDA library: a
 * line-by-line C++ restatement of the reference's Julia (the src2d files, the EOS and
 * transport parts of src/, and the driver loop of main2D.jl). Each function
 * cites the file:line it follows. Expressions keep Julia's evaluation order
 * (n-ary + and * fold left; `2x` is 2*x; `x^2` is x*x, `x^3` is x*x*x, `x^4` is
 * pow_body). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.
 *
 * Parity pin: the reference cannot run here (no Julia), so the restatement is
 * pinned against the reference's own published gate numbers (README2D.md:273-275:
 * Gubser L2 sequence and orders, Bjorken orders) and its round-trip gates
 * (test/test_primrec2d.jl), which the tests re-run on this code.
 */
#ifndef FIVO_ORACLE_CORE_H
#define FIVO_ORACLE_CORE_H

#include <cstdint>
#include <vector>
#include "jlmath.h"
#include "../include/fivo2d.h"

namespace orc {

/* src/constants.jl:11-44 */
static const double HBARC = 0.1973269804;
static const double FMGEV = 1.0 / 0.1973269804;
static const double INVFMGEV = 0.1973269804;
static const double FMGEV3 = (FMGEV * FMGEV) * FMGEV;   /* (1/ħc)^3, literal_pow Val{3} */
static const double T_MIN = 1e-20;
static const double T_SOLVE_MAX = 10.0;
static const double PHI_CAP = 10000.0;
static const double E_VAC = 1e-20;
static const double D_VAC = 0.0;
static const double E_FLOOR = 1e-20;
static const double CHI_SRE = 0.99999999;
static const double TINY = 1e-300;
static const double EPS_POS = 1e-50;
static const double U_CAP_2D = 1.0e4;          /* src2d/primrec2d.jl:265 */
static const double SR_MARGIN_2D = 0.98;       /* src2d/floors2d.jl:270 */
static const double PI2 = O_PI * O_PI;         /* const π2 = π^2, src/eos.jl:8 */

static inline double posden(double x) { return x > EPS_POS ? x : EPS_POS; }
static inline double safe_inv(double x) { return 1.0 / posden(x); }
static inline double safe_div(double a, double b) { return a / posden(b); }
static inline double safe_sqrt(double x) { return x <= 0 ? 0.0 : std::sqrt(x); }

enum PrimRecReason : uint8_t {
  PRR_UNSET = 0, PRR_VACUUM = 1, PRR_CONVERGED = 2, PRR_NONFINITE_INITIAL = 3,
  PRR_NONFINITE_JACOBIAN = 4, PRR_LINSOLVE_FAILED = 5, PRR_LINESEARCH_FAILED = 6,
  PRR_EOS_INVALID = 7, PRR_RESIDUAL_TOO_LARGE = 8, PRR_MAXIT = 9
};

struct Grid {                 /* src2d/grid2d.jl:19-71 */
  int Nx, Ny, ng;
  double xmin, xmax, ymin, ymax, dx, dy;
  int Nxtot, Nytot;
  int64_t Ntot;
  std::vector<double> xC, yC;
  inline int64_t lin(int ix, int iy) const { return (int64_t)ix * Nytot + iy; }  /* 0-based */
};

struct Layout {               /* src2d/state_layout2d.jl:23-84 (0-based rows) */
  int nv;
  int iDtau, iSx, iSy, iE;
  bool hasNu; int iNux, iNuy;
  bool hasPi; int iPi;
  bool hasShear; int iPixx, iPixy, iPiyy, iPieta;
  bool hasM2; int iPQxx, iPQxy, iPQyy, iPQeta, iPiQ;
};

struct EOSCache {             /* src2d/primrec2d.jl:115-130 */
  double T[4], Pl[4], el[4], K2[4];
  int next;
  void reset() { for (int j = 0; j < 4; ++j) T[j] = O_NAN; next = 0; }
};

struct Model {
  fivo_params p;
  Layout L;
  double E_vac_cut;
};

struct Prim {                 /* PrimIdealVisc2D, src2d/primitives2d.jl:10-26 */
  double T, mu, ux, uy, n, e, P, nux, nuy, Pi, pixx, pixy, piyy, pieta;
  bool ok;
};

struct RecoveryOut { double T, mu, ux, uy, n, e, P; bool ok; uint8_t reason; double resnorm; int iters; };

struct Work {                 /* src2d/work2d.jl:15-139 */
  std::vector<double> yT, phi, mu, alpha, ux, uy, P, n, e;
  std::vector<uint8_t> ok;
  std::vector<double> x0_yT, x0_phi, x0_ux, x0_uy;
  std::vector<double> ux_prev, uy_prev, alpha_prev, T_prev;
  std::vector<double> nux_prev, nuy_prev;                      /* the charm second moment's d_tau nu */
  std::vector<double> sigx, sigy, ULpx, URpx, ULpy, URpy;      /* 4 x Ntot */
  std::vector<double> ULcx, URcx, ULcy, URcy, Fhx, Fhy, S, diss_snap, k, U1, U2;  /* nv x Ntot */
  std::vector<uint8_t> bad, bad_tmp;
  std::vector<double> theta, vxC, vyC;
  std::vector<double> slope_tmp, alphaFx, alphaFy, gradAx, gradAy;
  std::vector<double> shear_res;
  int64_t nprimfail, nvacuum, primfail_i; int primfail_reason; double primfail_resnorm;
  double amax;
  int64_t nmood, nhalve;
};

/* API used by the extern "C" wrapper and the tests */
bool make_model(const fivo_params& p, Model& m, const char** err);
void make_grid(int Nx, int Ny, int ng, double xmax, double ymax, Grid& g);
void make_work(const Grid& g, const Model& m, Work& w);

void eos_Pne(double T, double mu, const fivo_params& e, double* P, double* n, double* en);
double eos_cs2(double T, double mu, const fivo_params& e);
RecoveryOut cons_to_prim_2d(double D, double Sx, double Sy, double E, double nux, double nuy,
                            double Pi, double pixx, double pixy, double piyy, double pieta,
                            double tau, const fivo_params& e, double yT0, double phi0,
                            double ux0, double uy0, int maxit, double tol);
bool prim_to_cons_2d(double* Ucol, double T, double mu, double ux, double uy, double nux,
                     double nuy, double Pi, double pixx, double pixy, double piyy, double pieta,
                     double tau, const fivo_params& e, const Layout& L, Prim* out);
void apply_bc_2d(double* U, const Grid& g, const Layout& L, int bc);
int64_t update_primitives_2d(double* U, const Grid& g, double tau, const Model& m, Work& w, int bc);
void rhs_2d(double* dU, double* U, const Grid& g, double tau, const Model& m, Work& w, int bc,
            double Emin, const uint8_t* force_first_order);
double compute_dt_2d(const Work& w, const Grid& g, double tau, double CFL, double CFLtau);
bool step_ssprk2_2d(double* U, const Grid& g, double tau, double dtau, const Model& m, Work& w,
                    int bc, int max_halve, int max_mood, double* used);
bool step_ssprk3_2d(double* U, const Grid& g, double tau, double dtau, const Model& m, Work& w,
                    int bc, int max_halve, double* used);
int64_t relax_dissipative_2d(double* U, const Grid& g, double tau, double dtau, const Model& m, Work& w);
void project_shear(double* U, const Grid& g, const Work& w, const Model& m, double* maxr, double* meanr);
void finalize_ic(double* U, const Grid& g, const Model& m, int bc, double Emin, double tau0);
void advance_sim_2d(double* U, const Grid& g, const Model& m, Work& w, double tau, double taufinal,
                    double CFL, double CFLtau, int integrator, int bc, int64_t max_steps,
                    int64_t* nsteps_run, fivo_run_result* res);
void run_sim_2d(double* U, const Grid& g, const Model& m, Work& w, double tau0, double taufinal,
                double CFL, double CFLtau, int integrator, int bc, bool reset_history,
                int64_t max_steps, fivo_run_result* res);

/* the consistent charm first moment (src2d/hq_consistent_firstmoment2d.jl) */
void cfm_h_hprime(double T, const fivo_params& p, double* h, double* hp);
double cfm_dn_dT(double T, double n, const fivo_params& p);
void cfm_diff_coeffs(double T, double mu, double n, const fivo_params& p, double* kappa, double* taun,
                     double* dN);
void cfm_source(double ux, double uy, double ut, double T, double dxT, double dyT, double dtT, double nux,
                double nuy, double n, double dn_dT, double tn, double Ds, double hp, double th, double ax,
                double ay, double dxux, double dxuy, double dyux, double dyuy, uint32_t terms, double* sx,
                double* sy);

/* cell-level functions of the relaxation, for the gate tests */
void cell_shear_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p, double* out3);
void cell_bulk_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p, double* out2);
void cell_diff_tauN(double T, double alpha, const fivo_params& p, double DsT, double tauD, double* taun,
                    double* norm);
double cell_vacuum_weight(double n, const fivo_params& p);
double cell_entropy(double T, double mu, double n, double en, double P);
void cell_ns_shear_target(const double* kin12, double* out4);
double cell_project_traceless(double ux, double uy, double ut, double pixx, double pixy, double piyy);
void cell_ns_diffusion_target(double ux, double uy, double ut, double dxa, double dya, double dta, double kappa,
                              double* out2);
void cell_pi_sigma(const double* in10, double* out4);
void cell_shear_tensor(double ux, double uy, double ut, double tau, double pixx, double pixy, double piyy,
                       double pieta, double* out7);

/* the consistent charm second moment (src2d/hq_consistent_m2_2d.jl), for the gate tests:
 * in[44] = the 44 positional arguments of consistent_m2_source_2d in their order;
 * out[5] = (dpxx, dpxy, dpyy, dPiQ, geo) */
void m2_source(const double* in44, uint32_t terms, double* out5);
void m2_coeffs(double T, double n, double tn, double Ds, double h, double m, double* out5);
double m2_tauM(double T, double tn, double m);
void m2_sigma_nu(const double* in18, double* out4);
void m2_rank1_traceless(const double* in7, double* out3);

}  // namespace orc
#endif
