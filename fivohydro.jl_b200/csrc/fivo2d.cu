/*
 * fivo2d.cu — the C ABI of include/fivo2d.h on one B200 (sm_100a).
 *
 * A context mirrors Grid2D + Work2D (src2d/grid2d.jl, src2d/work2d.jl) in HBM:
 * four state buffers (U, U1, U2 and a scratch) of nv planes each, the cell
 * primitives, warm starts and dtau history, three MOOD masks and a flag block.
 * The RK buffers are addressed by role indices, so "copy U1 into U" is a role
 * swap, and the relaxation double-buffers only the dissipative planes.
 *
 * Control flow (halving, MOOD escalation, the time loop) stays on the host,
 * exactly as in src2d/timestepper2d.jl and main2D.jl:371-561; the device
 * reports the admissibility count and the signal speed after every stage.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "freezeout.cuh"
#include "face32.cuh"
#include "facetile.cuh"
#include "relax32.cuh"
#include "batch.cuh"

using namespace fv;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return fail(FIVO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CKL()                                                                             \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess)                                                                \
      return fail(FIVO_ERR_CUDA, std::string("kernel launch at fivo2d.cu:") + std::to_string(__LINE__) + ": " + \
                                     cudaGetErrorString(e_));                             \
  } while (0)

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

/* history planes of a context: x0_yT, x0_phi, x0_ux, x0_uy, ux_prev, uy_prev,
 * alpha_prev, T_prev, nux_prev, nuy_prev */
constexpr size_t NHIST = 10;

/* reject_unwired_knobs_2d + check_terms (src2d/primitives2d.jl:246-272, src/terms.jl) */
int validate(const fivo_params* p) {
  if (p->consistent_fm && p->tauN_coeff != 1.0)   /* reject_unwired_knobs_2d, src2d/primitives2d.jl:263-269 */
    return fail(FIVO_ERR_CONFIG, "tauN_coeff cannot be combined with consistent_fm = true (the closure ties "
                                 "tau_n = D_s h / T with h in closed form)");
  if (p->eos_kind != FIVO_EOS_CONFORMAL_HQ && p->eos_kind != FIVO_EOS_LATTICE_HRG)
    return fail(FIVO_ERR_CONFIG, "unknown eos_kind");
  if (p->enable_shear && p->shear_kind != FIVO_SHEAR_QGP && p->shear_kind != FIVO_SHEAR_ZERO)
    return fail(FIVO_ERR_CONFIG, "unknown shear_kind");
  if (p->enable_bulk && (p->bulk_kind < FIVO_BULK_ZERO || p->bulk_kind > FIVO_BULK_GAUSS))
    return fail(FIVO_ERR_CONFIG, "unknown bulk_kind");
  if (p->enable_bulk && p->bulk_kind == FIVO_BULK_GAUSS && !(p->bulk_width > 0))
    return fail(FIVO_ERR_CONFIG, "GaussianBulkViscosity needs bulk_width > 0");
  if (p->enable_diff && !p->with_charge)
    return fail(FIVO_ERR_CONFIG, "enable_diff needs a layout with charge (with_charge = true)");
  /* a term switched away from its default whose sector is off cannot act */
  const uint32_t diff = (p->terms ^ FIVO_TERMS_DEFAULT);
  const uint32_t fm = 0x3Eu, m2 = 0x1FFC0u;
  if ((diff & FIVO_TERM_NU_GRADALPHA) && !p->enable_diff)
    return fail(FIVO_ERR_CONFIG, "Terms: nu_gradalpha switched but enable_diff is off");
  if ((diff & FIVO_TERM_SHEAR_VORTICITY) && !p->enable_shear)
    return fail(FIVO_ERR_CONFIG, "Terms: shear_vorticity switched but enable_shear is off");
  if ((diff & fm) && !p->consistent_fm)
    return fail(FIVO_ERR_CONFIG, "Terms: a consistent-first-moment term is switched but consistent_fm is off");
  if ((diff & m2) && !p->consistent_m2)
    return fail(FIVO_ERR_CONFIG, "Terms: a second-moment term is switched but consistent_m2 is off");
  if (p->primrec_maxit < 1 || !(p->primrec_tol > 0))
    return fail(FIVO_ERR_CONFIG, "primrec_maxit must be >= 1 and primrec_tol > 0");
  return FIVO_OK;
}

/* Layout, grid and derived constants. The derived constants are the same
 * expressions the per-call code of the reference evaluates, computed once. */
DevParams make_devparams(const fivo_params* p, int nx, int ny, int ng, double xmax, double ymax) {
  DevParams d;
  std::memset(&d, 0, sizeof(d));
  d.p = *p;
  int k = 0;
  d.iDtau = k++; d.iSx = k++; d.iSy = k++; d.iE = k++;
  d.hasNu = p->with_charge != 0; d.iNux = d.hasNu ? k++ : -1; d.iNuy = d.hasNu ? k++ : -1;
  d.hasPi = p->enable_bulk != 0; d.iPi = d.hasPi ? k++ : -1;
  d.hasShear = p->enable_shear != 0;
  d.iPixx = d.hasShear ? k++ : -1; d.iPixy = d.hasShear ? k++ : -1;
  d.iPiyy = d.hasShear ? k++ : -1; d.iPieta = d.hasShear ? k++ : -1;
  d.nvf = k;
  /* the charm second moment's rows follow the medium's (make_layout2d with_m2) */
  d.hasM2 = p->consistent_m2 != 0;
  d.iPQxx = d.hasM2 ? k++ : -1; d.iPQxy = d.hasM2 ? k++ : -1; d.iPQyy = d.hasM2 ? k++ : -1;
  d.iPQeta = d.hasM2 ? k++ : -1; d.iPiQ = d.hasM2 ? k++ : -1;
  d.nv = k;
  d.ncharge = (p->eos_kind == FIVO_EOS_CONFORMAL_HQ) ? (p->g_hq > 0.0) : 1;
  d.Nx = nx; d.Ny = ny; d.ng = ng; d.Nxtot = nx + 2 * ng; d.Nytot = ny + 2 * ng;
  d.Ntot = (long long)d.Nxtot * d.Nytot;
  d.xmin = -xmax; d.ymin = -ymax;
  d.dx = (xmax - d.xmin) / nx; d.dy = (ymax - d.ymin) / ny;
  const double fmgev = 1.0 / 0.1973269804;
  d.fmgev3 = (fmgev * fmgev) * fmgev;
  d.pi2 = FX_PI * FX_PI;
  d.aSB = (d.pi2 / 90.0) * p->g_eff;
  double m = p->m_hq, g = p->g_hq;
  d.A_conf = (g * (m * m)) / (2.0 * d.pi2);
  d.A_lhrg = ((p->canon_factor * g) * (m * m)) / (2.0 * d.pi2);
  d.lA = 0.01 * (p->lhrg_d * p->lhrg_d);
  d.lB = 0.1 * (p->lhrg_c * p->lhrg_c);
  d.log_T_min = fx_log(FV_T_MIN);
  d.log_T_solve_max = fx_log(FV_T_SOLVE_MAX);
  d.log_seed_T = fx_log(jmax(0.15, FV_T_MIN));
  /* build_model_2d derives E_vac_cut from T_vac_cut (main2D.jl:102-108) */
  if (p->E_vac_cut > 0.0) d.E_vac_cut = p->E_vac_cut;
  else {
    double P, n, e;
    if (p->eos_kind == FIVO_EOS_CONFORMAL_HQ) eos_Pne<FIVO_EOS_CONFORMAL_HQ>(p->T_vac_cut, 0.0, d, &P, &n, &e);
    else eos_Pne<FIVO_EOS_LATTICE_HRG>(p->T_vac_cut, 0.0, d, &P, &n, &e);
    d.E_vac_cut = e;
  }
  return d;
}

}  // namespace

struct fivo_ctx {
  DevParams dp;
  int device = 0;
  cudaStream_t st = nullptr;
  double* slab = nullptr;
  DevState S[4];
  int iU = 0, iU1 = 1, iU2 = 2, iT = 3;
  double* pbuf = nullptr;
  DevPrims w;
  double* hbuf = nullptr;
  DevHist h;
  uint8_t* masks = nullptr;   /* bad | mask | tmp, Ntot bytes each */
  DevFlags* fl = nullptr;
  DevFlags* flh = nullptr;    /* pinned mirror */
  double* dU = nullptr;       /* lazily allocated RHS planes for fivo_rhs */
  double* part = nullptr;     /* per-warp partial sums of the run diagnostics */
  cudaEvent_t ev_sync = nullptr;   /* set: waits block the host thread (batch workers) */
  double* fh = nullptr;       /* face fluxes: x faces then y faces, nv planes each */
  unsigned int* queues = nullptr;  /* deferred recoveries | deferred admissibility tests */
  int nsm = 148;
  double* stage = nullptr;    /* nv x Ntot AoS staging for uploads and downloads */
  bool hist_valid = false;
  long long nsteps_run = 0;            /* accepted steps since fivo_run started */
  fivo_counters cnt;
  cudaStream_t own_st = nullptr;       /* the context's own stream (st may be a caller's) */
  /* per-kernel CUDA-event timing (fivo_profile) */
  bool profiling = false;
  struct Pend { int cls, nk; long long units; cudaEvent_t a, b; };
  std::vector<Pend> pend;
  std::vector<cudaEvent_t> pool;
  fivo_kernel_times kt;
  int64_t tot_base_p = 0, tot_base_a = 0;   /* device deferred-cell totals at the last reset */
  /* the learned recovery guess (fivo_ctx_set_guess): k_prim_learned replaces k_prim_fast */
  bool learned = false;
  int guess_mode = FIVO_GUESS_EVERY_CELL;
  guess::Net gnet{};
  int64_t stats_base_p = 0;                 /* deferred-cell total at the last Newton-statistics reset */
  /* the mixed-precision face pass (fivo_ctx_set_precision): FP32 face fluxes */
  int precision = FIVO_PRECISION_FP64;
  float* fh32 = nullptr;                    /* x faces then y faces, nv FP32 planes each */
  double* x0save = nullptr;                 /* the warm starts before an optimistic step */
  double* hsave = nullptr;                  /* history planes before a lockstep step with speculation */
  /* the face pass (x, y): -2 not chosen yet, -1 k_faces, k >= 0 k_faces_tile of FT_SHAPES[k];
   * the tensor maps of the chosen shape: the primitive planes, and the dissipative
   * planes of each of the four state buffers */
  int ft_cfg[2] = {-2, -2};
  /* fivo_ctx_set_graphs: fivo_run / fivo_advance through the lockstep launch
   * sequences of a batch of this one context, replayed as CUDA graphs */
  int graphs = 0;                 /* 1: graphs; 2: the same sequences launched kernel by kernel */
  fivo_batch* solo = nullptr;
  CUtensorMap ft_prim[2][5];
  CUtensorMap ft_slab[2][4 * FV_MAXP];   /* every plane of the state slab: the relaxation swaps
                                           the dissipative planes between state buffers */
};

namespace {

const long long REP_NONE = 0x7fffffffffffffffLL;

/* ------------------------------------------------------------ kernel timing */

cudaEvent_t pool_get(fivo_ctx* c) {
  if (!c->pool.empty()) { cudaEvent_t e = c->pool.back(); c->pool.pop_back(); return e; }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

/* bracket nk launches of kernel class cls (FIVO_KCLASS_*) that process `units` cells or faces */
struct KTimer {
  fivo_ctx* c; int cls, nk; long long units; cudaEvent_t a = nullptr;
  KTimer(fivo_ctx* c_, int cls_, int nk_ = 1, long long units_ = 0) : c(c_), cls(cls_), nk(nk_), units(units_) {
    if (!c->profiling) return;
    a = pool_get(c);
    cudaEventRecord(a, c->st);
  }
  ~KTimer() {
    if (!c->profiling || !a) return;
    cudaEvent_t b = pool_get(c);
    cudaEventRecord(b, c->st);
    c->pend.push_back({cls, nk, units, a, b});
  }
};

/* after a stream synchronisation: fold finished launches into the totals */
void prof_flush(fivo_ctx* c) {
  for (auto& q : c->pend) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, q.a, q.b) == cudaSuccess) c->kt.ms[q.cls] += ms;
    c->kt.launches[q.cls] += 1;
    c->kt.total_launches += q.nk;
    c->kt.units[q.cls] += q.units;
    c->pool.push_back(q.a);
    c->pool.push_back(q.b);
  }
  c->pend.clear();
}

cudaError_t ctx_sync(fivo_ctx* c) {
  cudaError_t e;
  if (c->ev_sync) {   /* blocking wait: the host thread sleeps instead of spinning */
    e = cudaEventRecord(c->ev_sync, c->st);
    if (e == cudaSuccess) e = cudaEventSynchronize(c->ev_sync);
  } else {
    e = cudaStreamSynchronize(c->st);
  }
  if (e == cudaSuccess) prof_flush(c);
  return e;
}

/* ---------------------------------------------------------- launch helpers */

int launch_bc(fivo_ctx* c, const DevState& U, int bc) {
  const DevParams& d = c->dp;
  long long nframe = d.Ntot - (long long)d.Nx * d.Ny;
  KTimer t_(c, FIVO_KCLASS_OTHER);
  k_bc<<<nblk(nframe, 256), 256, 0, c->st>>>(d, U, bc);
  CKL();
  return FIVO_OK;
}

/* what: see k_reset_flags. amax is reset to 0 only by an rhs pass (rhs_2d!
 * fills amax_tls, src2d/rhs2d.jl:193); other passes leave it alone. */
int reset_flags(fivo_ctx* c, int what) {
  KTimer t_(c, FIVO_KCLASS_OTHER);
  k_reset_flags<<<1, 32, 0, c->st>>>(c->fl, what, 0ULL);
  CKL();
  return FIVO_OK;
}

/* shared memory a block of the learned pass holds, static and reserved: with one
 * KB per block reserved by the hardware, 5 blocks (255 KB) do not fit in the 228 KB
 * of an SM and 4 (204 KB) do */
constexpr int LEARNED_SMEM = 50 * 1024;

template <int EOS, bool NCH>
int launch_primitive_t(fivo_ctx* c, const DevState& U, double tau) {
  const DevParams& d = c->dp;
  unsigned int* q = c->queues;
  if (c->learned && c->guess_mode == FIVO_GUESS_DEFERRED) {
    /* the plain fast pass, the network's guess for the cells it deferred, then the
     * full recovery of what is left (second queue) */
    unsigned int* q2 = c->queues + 2 * d.Ntot;
    {
      KTimer t_(c, FIVO_KCLASS_PRIM_FAST, 1, d.Ntot);
      k_prim_fast<EOS, NCH><<<nblk(d.Ntot, 128), 128, 0, c->st>>>(d, U, c->w, c->h, tau, c->fl, q);
      CKL();
    }
    {
      const int dyn = LEARNED_SMEM - (int)sizeof(guess::FwdSmem) - 128;
      CK(cudaFuncSetAttribute(k_prim_learned_retry<EOS, NCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
      KTimer t_(c, FIVO_KCLASS_PRIM_SLOW);
      k_prim_learned_retry<EOS, NCH><<<nblk(d.Ntot, 128), 128, dyn, c->st>>>(d, U, c->w, c->h, tau, c->fl, q, q2,
                                                                               c->gnet);
      CKL();
    }
    {
      KTimer t_(c, FIVO_KCLASS_PRIM_SLOW);
      k_prim_slow<EOS, NCH><<<2 * c->nsm, 128, 0, c->st>>>(d, U, c->w, c->h, tau, c->fl, q2, &c->fl->qcount_q,
                                                           &c->fl->qnext_q);
      CKL();
    }
    return FIVO_OK;
  }
  if (c->learned) {
    /* at most 4 blocks per SM (4 x 128 tensor-memory columns): the launch reserves
     * shared memory up to LEARNED_SMEM per block */
    CK(cudaFuncSetAttribute(k_prim_learned<EOS, NCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            LEARNED_SMEM - (int)sizeof(guess::FwdSmem)));
    KTimer t_(c, FIVO_KCLASS_PRIM_FAST, 1, d.Ntot);
    k_prim_learned<EOS, NCH><<<nblk(d.Ntot, 128), 128, LEARNED_SMEM - sizeof(guess::FwdSmem), c->st>>>(
        d, U, c->w, c->h, tau, c->fl, q, c->gnet);
    CKL();
  } else {
    KTimer t_(c, FIVO_KCLASS_PRIM_FAST, 1, d.Ntot);
    k_prim_fast<EOS, NCH><<<nblk(d.Ntot, 128), 128, 0, c->st>>>(d, U, c->w, c->h, tau, c->fl, q);
    CKL();
  }
  {
    KTimer t_(c, FIVO_KCLASS_PRIM_SLOW);
    k_prim_slow<EOS, NCH><<<2 * c->nsm, 128, 0, c->st>>>(d, U, c->w, c->h, tau, c->fl, q, &c->fl->qcount_p,
                                                         &c->fl->qnext_p);
    CKL();
  }
  return FIVO_OK;
}

/* _primitive_pass!: the two-phase recovery (k_prim_fast, then k_prim_slow on
 * the cells it deferred). The flag block's pass counters must be reset first. */
int launch_primitive(fivo_ctx* c, const DevState& U, double tau) {
  const DevParams& d = c->dp;
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG) return launch_primitive_t<FIVO_EOS_LATTICE_HRG, true>(c, U, tau);
  if (d.ncharge) return launch_primitive_t<FIVO_EOS_CONFORMAL_HQ, true>(c, U, tau);
  return launch_primitive_t<FIVO_EOS_CONFORMAL_HQ, false>(c, U, tau);
}

/* ------------------------------------------------------------ the face pass
 * Two implementations with the same arithmetic (face_flux_pair): k_faces, whose
 * lanes read their stencils from global memory, and k_faces_tile, which stages
 * a halo tile of every plane it reads in shared memory by TMA first. The tile
 * path needs 16-byte row pitches (Nytot even). Which one runs, and with which
 * tile shape, is chosen per grid and layout by timing every candidate on the
 * context's first stage (tune_faces); the choice is shared by contexts of the
 * same shape. */
struct FtShape { int tx, ty; };
constexpr FtShape FT_SHAPES[] = {{4, 32}, {2, 64}, {8, 16}, {8, 32}};
constexpr int FT_NSHAPES = (int)(sizeof(FT_SHAPES) / sizeof(FT_SHAPES[0]));

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

/* the tensor map of one Nxtot x Nytot plane (y contiguous) with the box of a tile
 * of shape sh in direction dir (0 = x faces) */
bool encode_plane(CUtensorMap* m, const double* plane, const DevParams& d, FtShape sh, int dir) {
  EncodeTiledFn fn = encode_tiled_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)d.Nytot, (cuuint64_t)d.Nxtot};
  const cuuint64_t strides[1] = {(cuuint64_t)d.Nytot * 8};
  const cuuint32_t box[2] = {(cuuint32_t)(dir == 0 ? sh.ty : sh.ty + 4), (cuuint32_t)(dir == 0 ? sh.tx + 3 : sh.tx)};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(plane), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

/* the dissipative planes of a state, in face_flux_pair's slot order */
void dis_planes(const DevParams& d, const DevState& U, const double* out[7]) {
  out[0] = d.hasNu ? U.f[d.iNux] : nullptr;
  out[1] = d.hasNu ? U.f[d.iNuy] : nullptr;
  out[2] = d.hasPi ? U.f[d.iPi] : nullptr;
  out[3] = d.hasShear ? U.f[d.iPixx] : nullptr;
  out[4] = d.hasShear ? U.f[d.iPixy] : nullptr;
  out[5] = d.hasShear ? U.f[d.iPiyy] : nullptr;
  out[6] = d.hasShear ? U.f[d.iPieta] : nullptr;
}

/* encode the maps of shape index k for direction dir into the context: the primitive
 * planes and every plane of the state slab */
bool ft_encode(fivo_ctx* c, int dir, int k) {
  const DevParams& d = c->dp;
  const FtShape sh = FT_SHAPES[k];
  const double* prim[5] = {c->w.yT, c->w.phi, c->w.ux, c->w.uy, c->w.mu};
  for (int q = 0; q < 5; ++q)
    if (!encode_plane(&c->ft_prim[dir][q], prim[q], d, sh, dir)) return false;
  for (int p = 0; p < 4 * d.nv; ++p)
    if (!encode_plane(&c->ft_slab[dir][p], c->slab + (size_t)p * d.Ntot, d, sh, dir)) return false;
  return true;
}

/* the launch's maps: the primitives, then the dissipative rows of U that exist (found by
 * their place in the slab); false when a plane is not in the slab */
bool ft_maps(const fivo_ctx* c, int dir, const DevState& U, FaceTileMaps* m) {
  const DevParams& d = c->dp;
  for (int q = 0; q < 5; ++q) m->map[q] = c->ft_prim[dir][q];
  const double* dp[7];
  dis_planes(d, U, dp);
  int np = 5;
  for (int j = 0; j < 7; ++j) {
    if (!dp[j]) { m->dis_plane[j] = -1; continue; }
    const long long off = dp[j] - c->slab;
    if (off < 0 || off % d.Ntot != 0 || off / d.Ntot >= 4LL * d.nv) return false;
    m->map[np] = c->ft_slab[dir][off / d.Ntot];
    m->dis_plane[j] = np;
    ++np;
  }
  m->nplanes = np;
  return true;
}

template <int EOS, bool XDIR, int TX, int TY>
int launch_tile(fivo_ctx* c, const StageArgs& a, const FaceTileMaps& m, double* Fh) {
  const DevParams& d = c->dp;
  const int smem = ft_smem_bytes(XDIR, TX, TY, m.nplanes);
  CK(cudaFuncSetAttribute(k_faces_tile<EOS, XDIR, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const dim3 grid(XDIR ? (d.Nytot + TY - 1) / TY : (d.Nytot - 1 + TY - 1) / TY,
                  XDIR ? (d.Nxtot - 1 + TX - 1) / TX : (d.Nxtot + TX - 1) / TX);
  k_faces_tile<EOS, XDIR, TX, TY><<<grid, 2 * TX * TY, smem, c->st>>>(d, m, a.tau, a.ffo, Fh, c->fl);
  CKL();
  return FIVO_OK;
}

/* one direction of the face pass with configuration cfg (-1: k_faces) */
template <int EOS, bool XDIR>
int launch_faces_dir(fivo_ctx* c, const StageArgs& a, int cfg, double* Fh) {
  const DevParams& d = c->dp;
  FaceTileMaps m;
  if (cfg < 0 || !ft_maps(c, XDIR ? 0 : 1, a.Ub, &m)) {
    const long long nf = XDIR ? (long long)(d.Nxtot - 1) * d.Nytot : (long long)d.Nxtot * (d.Nytot - 1);
    k_faces<EOS, XDIR><<<nblk(2 * nf, 128), 128, 0, c->st>>>(d, a.Ub, a.w, a.tau, a.ffo, Fh, c->fl);
    CKL();
    return FIVO_OK;
  }
  switch (cfg) {
    case 0: return launch_tile<EOS, XDIR, 4, 32>(c, a, m, Fh);
    case 1: return launch_tile<EOS, XDIR, 2, 64>(c, a, m, Fh);
    case 2: return launch_tile<EOS, XDIR, 8, 16>(c, a, m, Fh);
    default: return launch_tile<EOS, XDIR, 8, 32>(c, a, m, Fh);
  }
}

std::mutex g_ft_mu;
std::vector<std::pair<std::vector<long long>, std::pair<int, int>>> g_ft_choice;

/* the choice of the face pass for this context: cached per (grid, EOS, layout),
 * else timed here: each candidate once to warm up, then the best of three */
template <int EOS>
int tune_faces(fivo_ctx* c, const StageArgs& a, double* fhx, double* fhy) {
  const DevParams& d = c->dp;
  const std::vector<long long> key = {d.Nxtot, d.Nytot, EOS, d.nv, d.hasNu, d.hasPi, d.hasShear, c->device};
  {
    std::lock_guard<std::mutex> lk(g_ft_mu);
    for (auto& e : g_ft_choice)
      if (e.first == key) { c->ft_cfg[0] = e.second.first; c->ft_cfg[1] = e.second.second; break; }
  }
  const bool tile_ok = (d.Nytot % 2 == 0) && encode_tiled_fn() != nullptr;
  if (c->ft_cfg[0] == -2) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int dir = 0; dir < 2; ++dir) {
      double* Fh = dir == 0 ? fhx : fhy;
      int best = -1;
      float best_ms = 1e30f, glob_ms = 1e30f;
      for (int cfg = -1; cfg < (tile_ok ? FT_NSHAPES : 0); ++cfg) {
        if (cfg >= 0 && !ft_encode(c, dir, cfg)) continue;
        float tmin = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
          CK(cudaEventRecord(e0, c->st));
          int rc = dir == 0 ? launch_faces_dir<EOS, true>(c, a, cfg, Fh) : launch_faces_dir<EOS, false>(c, a, cfg, Fh);
          if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
          CK(cudaEventRecord(e1, c->st));
          CK(cudaEventSynchronize(e1));
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          if (rep > 0) tmin = std::min(tmin, ms);
        }
        /* a tile shape replaces the global-load kernel only when it is clearly faster
         * (3 %): the two are often within the timing noise of each other */
        if (cfg < 0 ? tmin < best_ms : tmin < best_ms && tmin < 0.97f * glob_ms) { best_ms = tmin; best = cfg; }
        if (cfg < 0) glob_ms = tmin;
      }
      c->ft_cfg[dir] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(g_ft_mu);
    g_ft_choice.push_back({key, {c->ft_cfg[0], c->ft_cfg[1]}});
  }
  for (int dir = 0; dir < 2; ++dir)
    if (c->ft_cfg[dir] >= 0 && !(tile_ok && ft_encode(c, dir, c->ft_cfg[dir]))) c->ft_cfg[dir] = -1;
  return FIVO_OK;
}

/* rhs_2d! + combination + sanitiser + admissibility: the face pass (x, y), k_update,
 * and k_adm_slow for the cells whose admissibility needs an inversion. */
template <int EOS, bool NCH>
int launch_stage_t(fivo_ctx* c, const StageArgs& a) {
  const DevParams& d = c->dp;
  double* fhx = c->fh;
  double* fhy = c->fh + (size_t)d.nv * d.Ntot;
  float* fhx32 = c->fh32;
  float* fhy32 = c->fh32 ? c->fh32 + (size_t)d.nv * d.Ntot : nullptr;
  const bool f32 = c->precision != FIVO_PRECISION_FP64;
  {
    long long nfx = (long long)(d.Nxtot - 1) * d.Nytot, nfy = (long long)d.Nxtot * (d.Nytot - 1);
    KTimer t_(c, FIVO_KCLASS_FACES, 2, nfx + nfy);
    if (f32) {
      f32::k_faces32<EOS, true><<<nblk(2 * nfx, 128), 128, 0, c->st>>>(d, a.Ub, a.w, a.tau, a.ffo, fhx32, c->fl);
      CKL();
      f32::k_faces32<EOS, false><<<nblk(2 * nfy, 128), 128, 0, c->st>>>(d, a.Ub, a.w, a.tau, a.ffo, fhy32, c->fl);
      CKL();
    } else {
      int rc;
      if (c->ft_cfg[0] == -2 && (rc = tune_faces<EOS>(c, a, fhx, fhy))) return rc;
      if ((rc = launch_faces_dir<EOS, true>(c, a, c->ft_cfg[0], fhx))) return rc;
      if ((rc = launch_faces_dir<EOS, false>(c, a, c->ft_cfg[1], fhy))) return rc;
    }
  }
  unsigned int* aq = c->queues + d.Ntot;
  {
    KTimer t_(c, FIVO_KCLASS_UPDATE, 1, (long long)d.Nx * d.Ny);
    const unsigned gu = nblk((long long)d.Nx * d.Ny, 128);
    const bool full = d.hasNu && d.hasPi && d.hasShear;   /* the rows at fixed places (k_update FULL) */
    if (f32 && full)
      k_update<EOS, NCH, float, true><<<gu, 128, 0, c->st>>>(d, a, fhx32, fhy32, aq);
    else if (f32)
      k_update<EOS, NCH, float><<<gu, 128, 0, c->st>>>(d, a, fhx32, fhy32, aq);
    else if (full)
      k_update<EOS, NCH, double, true><<<gu, 128, 0, c->st>>>(d, a, fhx, fhy, aq);
    else
      k_update<EOS, NCH><<<gu, 128, 0, c->st>>>(d, a, fhx, fhy, aq);
    CKL();
  }
  if (a.mode != COMB_RHS_ONLY) {
    KTimer t_(c, FIVO_KCLASS_ADM_SLOW);
    k_adm_slow<EOS, NCH><<<c->nsm, 128, 0, c->st>>>(d, a.Uout, a.tau_state, a.bad, c->fl, aq);
    CKL();
  }
  return FIVO_OK;
}

int launch_stage(fivo_ctx* c, const StageArgs& a) {
  if (c->dp.p.eos_kind == FIVO_EOS_LATTICE_HRG) return launch_stage_t<FIVO_EOS_LATTICE_HRG, true>(c, a);
  if (c->dp.ncharge) return launch_stage_t<FIVO_EOS_CONFORMAL_HQ, true>(c, a);
  return launch_stage_t<FIVO_EOS_CONFORMAL_HQ, false>(c, a);
}

int parse_flags(fivo_ctx* c, bool read_amax);

int sync_flags(fivo_ctx* c, bool read_amax) {
  CK(cudaMemcpyAsync(c->flh, c->fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return parse_flags(c, read_amax);
}

/* the host mirror c->flh of the flag block, just read back: errors, counters, amax */
int parse_flags(fivo_ctx* c, bool read_amax) {
  const DevFlags& f = *c->flh;
  if (f.status == 3) return fail(FIVO_ERR_DEVICE, "learned recovery guess: a tensor-core wait gave up");
  if (f.status == 4) return fail(FIVO_ERR_DEVICE, "face pass: a tile copy to shared memory did not complete");
  c->cnt.nprimfail = f.nprimfail;
  c->cnt.nvacuum = f.nvacuum;
  if (f.rep != (unsigned long long)REP_NONE) {
    c->cnt.primfail_index = (int64_t)(f.rep >> 8);
    c->cnt.primfail_reason = (int32_t)(f.rep & 0xff);
  } else {
    c->cnt.primfail_index = -1;
    c->cnt.primfail_reason = 0;
  }
  c->cnt.primfail_resnorm = fx::nan_();
  if (read_amax) {
    uint64_t ab = f.amax_bits;
    double am; std::memcpy(&am, &ab, 8);
    c->cnt.amax = am;
  }
  return FIVO_OK;
}

/* rhs_2d! + combination + sanitize + admissibility on the given roles.
 * ub = base (and combination input), uo = output, uold = blend partner.
 * Returns FIVO_OK; *nbad = inadmissible interior cells. With sync = false the
 * host does not wait (nbad is not read), and with first = false the device's
 * count of inadmissible cells carries on from the previous stage, so a chain of
 * stages can be checked once at its end. With bc_in = false the input's ghost frame is
 * taken as filled: the previous stage's output got the same (idempotent) fill. */
int run_stage(fivo_ctx* c, int ub, int uo, int uold, double tau, double tau_state, double dt, double wold,
              double wnew, int mode, const uint8_t* mask, int bc, long long* nbad, double* dU,
              bool sync = true, bool first = true, bool bc_in = true) {
  int rc;
  if (bc_in && (rc = launch_bc(c, c->S[ub], bc))) return rc;
  if ((rc = reset_flags(c, first ? (1 | 2 | 64) : (1 | 2)))) return rc;
  if ((rc = launch_primitive(c, c->S[ub], tau))) return rc;
  StageArgs a;
  a.Ub = c->S[ub]; a.Uold = c->S[uold]; a.Uout = c->S[uo]; a.w = c->w; a.ffo = mask;
  a.bad = c->masks; a.dU = dU; a.tau = tau; a.tau_state = tau_state; a.dt = dt; a.wold = wold;
  a.wnew = wnew; a.mode = mode; a.fl = c->fl;
  if ((rc = launch_stage(c, a))) return rc;
  if (mode != COMB_RHS_ONLY)
    if ((rc = launch_bc(c, c->S[uo], bc))) return rc;
  if (!sync) return FIVO_OK;
  if ((rc = sync_flags(c, true))) return rc;
  if (nbad) *nbad = c->flh->nbad;
  return FIVO_OK;
}

/* _stage_2d! with the MOOD escalation, src2d/timestepper2d.jl:113-140 */
int stage_mood(fivo_ctx* c, int ub, int uo, int uold, double tau, double tau_state, double dt, double wold,
               double wnew, int bc, int max_mood, bool* ok) {
  const DevParams& d = c->dp;
  const uint8_t* mask = nullptr;
  uint8_t* bad = c->masks;
  uint8_t* m1 = c->masks + d.Ntot;
  uint8_t* m2 = c->masks + 2 * d.Ntot;
  int mode = (wnew == 0.0) ? COMB_EULER : COMB_BLEND;
  for (int attempt = 0; attempt <= max_mood; ++attempt) {
    long long nbad = 0;
    int rc = run_stage(c, ub, uo, uold, tau, tau_state, dt, wold, wnew, mode, mask, bc, &nbad, nullptr);
    if (rc) return rc;
    if (nbad == 0) { *ok = true; return FIVO_OK; }
    if (attempt == max_mood) { *ok = false; return FIVO_OK; }
    c->cnt.nmood += 1;
    /* expand_bad_2d!(radius = 1 + attempt): bad -> m1 -> m2 -> ... */
    const uint8_t* src = bad;
    uint8_t* dst = m1;
    for (int r = 0; r < 1 + attempt; ++r) {
      KTimer t_(c, FIVO_KCLASS_OTHER);
      k_expand_bad<<<nblk(d.Ntot, 256), 256, 0, c->st>>>(d, src, dst);
      CKL();
      src = dst;
      dst = (dst == m1) ? m2 : m1;
    }
    mask = src;
  }
  *ok = false;
  return FIVO_OK;
}

/* The warm starts x0_* (four contiguous planes of the history block) are updated by
 * every recovery pass, so an optimistic step that is thrown away must leave them as
 * they were for the stage-by-stage procedure to take the reference's path. */
int save_warm(fivo_ctx* c) {
  const size_t bytes = 4 * (size_t)c->dp.Ntot * sizeof(double);
  if (!c->x0save && cudaMalloc(&c->x0save, bytes) != cudaSuccess) {
    c->x0save = nullptr;
    return fail(FIVO_ERR_NOMEM, "device allocation failed");
  }
  CK(cudaMemcpyAsync(c->x0save, c->h.x0_yT, bytes, cudaMemcpyDeviceToDevice, c->st));
  return FIVO_OK;
}
int restore_warm(fivo_ctx* c) {
  const size_t bytes = 4 * (size_t)c->dp.Ntot * sizeof(double);
  CK(cudaMemcpyAsync(c->h.x0_yT, c->x0save, bytes, cudaMemcpyDeviceToDevice, c->st));
  return FIVO_OK;
}

int copy_state(fivo_ctx* c, int dst, int src) {
  const DevParams& d = c->dp;
  KTimer t_(c, FIVO_KCLASS_OTHER);
  k_copy_planes<<<nblk(d.Ntot, 256), 256, 0, c->st>>>(c->S[dst], c->S[src], 0, d.nv, d.Ntot);
  CKL();
  return FIVO_OK;
}

int step2_rest(fivo_ctx* c, double tau, double D, int max_halve, int max_mood, int bc, double* used, int* okout);
int step3_rest(fivo_ctx* c, double tau, double D, int max_halve, int bc, double* used, int* okout);

/* step_ssprk2_2d!, src2d/timestepper2d.jl:74-103 */
int step2(fivo_ctx* c, double tau, double dtau, int max_halve, int max_mood, int bc, double* used, int* okout) {
  double D = dtau;
  c->cnt.nmood = 0; c->cnt.nhalve = 0;
  /* Optimistic first pass: both stages at the full step without a host read in
   * between, their inadmissible cells counted together. Nothing inadmissible: the
   * step is the one the stage-by-stage procedure below takes (same kernels on the
   * same inputs). Otherwise the state is restored and that procedure runs. */
  {
    int rc;
    long long nbad = 0;
    if ((rc = save_warm(c))) return rc;
    if ((rc = copy_state(c, c->iU2, c->iU))) return rc;
    if ((rc = run_stage(c, c->iU, c->iU1, c->iU2, tau, tau + D, D, 1.0, 0.0, COMB_EULER, nullptr, bc, nullptr,
                        nullptr, false, true))) return rc;
    if ((rc = run_stage(c, c->iU1, c->iT, c->iU2, tau + D, tau + D, D, 0.5, 0.5, COMB_BLEND, nullptr, bc, &nbad,
                        nullptr, true, false, false))) return rc;
    if (nbad == 0) { std::swap(c->iU, c->iT); *used = D; *okout = 1; return FIVO_OK; }
    if ((rc = restore_warm(c))) return rc;
  }
  return step2_rest(c, tau, D, max_halve, max_mood, bc, used, okout);
}

/* step_ssprk2_2d!'s stage-by-stage procedure with MOOD and halving (after the
 * optimistic pass found an inadmissible cell and was undone) */
int step2_rest(fivo_ctx* c, double tau, double D, int max_halve, int max_mood, int bc, double* used, int* okout) {
  for (int h = 0; h <= max_halve; ++h) {
    int rc;
    if ((rc = copy_state(c, c->iU2, c->iU))) return rc;
    bool ok1 = false, ok2 = false;
    if ((rc = stage_mood(c, c->iU, c->iU1, c->iU2, tau, tau + D, D, 1.0, 0.0, bc, max_mood, &ok1))) return rc;
    if (ok1) {
      if ((rc = stage_mood(c, c->iU1, c->iT, c->iU2, tau + D, tau + D, D, 0.5, 0.5, bc, max_mood, &ok2))) return rc;
      if (ok2) { std::swap(c->iU, c->iT); *used = D; *okout = 1; return FIVO_OK; }
    }
    std::swap(c->iU, c->iU2);   /* copyto!(U, work.U2) */
    D *= 0.5;
    c->cnt.nhalve += 1;
  }
  *used = D; *okout = 0;
  return FIVO_OK;
}

/* step_ssprk3_2d!, src2d/timestepper2d.jl:148-188 */
int step3(fivo_ctx* c, double tau, double dtau, int max_halve, int bc, double* used, int* okout) {
  double D = dtau;
  c->cnt.nmood = 0; c->cnt.nhalve = 0;
  /* Optimistic first pass (as in step2): the three stages at the full step, one
   * host read at the end; any inadmissible cell restores the state and the
   * stage-by-stage procedure below takes the step. */
  {
    int rc;
    long long nbad = 0;
    if ((rc = save_warm(c))) return rc;
    if ((rc = copy_state(c, c->iU2, c->iU))) return rc;
    if ((rc = run_stage(c, c->iU, c->iU1, c->iU2, tau, tau + D, D, 1.0, 0.0, COMB_EULER, nullptr, bc, nullptr,
                        nullptr, false, true))) return rc;
    if ((rc = run_stage(c, c->iU1, c->iT, c->iU2, tau + D, tau + D, D, 0.75, 0.25, COMB_BLEND, nullptr, bc, nullptr,
                        nullptr, false, false, false))) return rc;
    std::swap(c->iU1, c->iT);
    if ((rc = run_stage(c, c->iU1, c->iT, c->iU2, tau + (0.5 * D), tau + D, D, 0.0, 0.0, COMB_THIRD, nullptr, bc,
                        &nbad, nullptr, true, false, false))) return rc;
    std::swap(c->iU, c->iT);
    if (nbad == 0) { *used = D; *okout = 1; return FIVO_OK; }
    std::swap(c->iU, c->iU2);    /* the state before the step */
    if ((rc = restore_warm(c))) return rc;
  }
  return step3_rest(c, tau, D, max_halve, bc, used, okout);
}

/* step_ssprk3_2d!'s stage-by-stage procedure with halving (after the optimistic
 * pass found an inadmissible cell and was undone) */
int step3_rest(fivo_ctx* c, double tau, double D, int max_halve, int bc, double* used, int* okout) {
  for (int h = 0; h <= max_halve; ++h) {
    int rc;
    long long nbad = 0;
    if ((rc = copy_state(c, c->iU2, c->iU))) return rc;
    if ((rc = run_stage(c, c->iU, c->iU1, c->iU2, tau, tau + D, D, 1.0, 0.0, COMB_EULER, nullptr, bc, &nbad, nullptr))) return rc;
    if (nbad) { std::swap(c->iU, c->iU2); D *= 0.5; c->cnt.nhalve += 1; continue; }
    if ((rc = run_stage(c, c->iU1, c->iT, c->iU2, tau + D, tau + D, D, 0.75, 0.25, COMB_BLEND, nullptr, bc, &nbad, nullptr))) return rc;
    std::swap(c->iU1, c->iT);
    if (nbad) { std::swap(c->iU, c->iU2); D *= 0.5; c->cnt.nhalve += 1; continue; }
    if ((rc = run_stage(c, c->iU1, c->iT, c->iU2, tau + (0.5 * D), tau + D, D, 0.0, 0.0, COMB_THIRD, nullptr, bc, &nbad, nullptr))) return rc;
    std::swap(c->iU, c->iT);
    if (!nbad) { *used = D; *okout = 1; return FIVO_OK; }
    std::swap(c->iU, c->iU2);
    D *= 0.5;
    c->cnt.nhalve += 1;
  }
  *used = D; *okout = 0;
  return FIVO_OK;
}

/* update_primitives_2d!, src2d/rhs2d.jl:57-65. bc_in = false: the state's ghost
 * frame is already filled (a step's last stage filled it). */
int update_prims(fivo_ctx* c, double tau, int bc, bool bc_in = true) {
  int rc;
  if (bc_in && (rc = launch_bc(c, c->S[c->iU], bc))) return rc;
  if ((rc = reset_flags(c, 1 | 64))) return rc;
  if ((rc = launch_primitive(c, c->S[c->iU], tau))) return rc;
  return FIVO_OK;
}

/* relax_dissipative_2d! (+ project_shear! when project != 0) on U */
int relax_project(fivo_ctx* c, double tau, double D, int do_relax, int do_project) {
  const DevParams& d = c->dp;
  if (d.nv <= 4) return FIVO_OK;
  DevState Uq = c->S[c->iU], Uo = c->S[c->iT];
  int rc = reset_flags(c, 4);
  if (rc) return rc;
  unsigned g = nblk(d.Ntot, 128);
  {
  KTimer t_(c, FIVO_KCLASS_RELAX, 1, d.Ntot);
  if (c->precision == FIVO_PRECISION_FP32 && do_relax) {
    if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG)
      k_relax32<FIVO_EOS_LATTICE_HRG><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
    else
      k_relax32<FIVO_EOS_CONFORMAL_HQ><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
  } else if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG) {
    if (d.hasM2)
      k_relax<FIVO_EOS_LATTICE_HRG, true><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
    else
      k_relax<FIVO_EOS_LATTICE_HRG, false><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
  } else {
    if (d.hasM2)
      k_relax<FIVO_EOS_CONFORMAL_HQ, true><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
    else
      k_relax<FIVO_EOS_CONFORMAL_HQ, false><<<g, 128, 0, c->st>>>(d, Uq, Uo, c->w, c->h, tau, D, do_relax, do_project, c->fl);
  }
  CKL();
  }
  /* the dissipative planes of U are now those of the scratch state */
  for (int a = 4; a < d.nv; ++a) std::swap(c->S[c->iU].f[a], c->S[c->iT].f[a]);
  if (do_relax) {
    CK(cudaMemcpyAsync(c->h.ux_prev, c->w.ux, d.Ntot * 8, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->h.uy_prev, c->w.uy, d.Ntot * 8, cudaMemcpyDeviceToDevice, c->st));
  }
  return FIVO_OK;
}

int read_shear(fivo_ctx* c, double* maxr, double* meanr) {
  CK(cudaMemcpyAsync(c->flh, c->fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  uint64_t b = c->flh->shear_max_bits;
  double m; std::memcpy(&m, &b, 8);
  if (maxr) *maxr = m;
  long long cnt = (long long)c->dp.Nx * c->dp.Ny;
  if (meanr) *meanr = cnt > 0 ? c->flh->shear_sum / cnt : 0.0;
  return FIVO_OK;
}

int fill_nan(fivo_ctx* c, double* p, long long n) {
  KTimer t_(c, FIVO_KCLASS_OTHER);
  k_fill_nan<<<nblk(n, 256), 256, 0, c->st>>>(p, n);
  CKL();
  return FIVO_OK;
}

int reset_history(fivo_ctx* c) {
  int rc;
  c->nsteps_run = 0;
  /* x0_* and the six *_prev planes are contiguous in hbuf */
  if ((rc = fill_nan(c, c->hbuf, NHIST * c->dp.Ntot))) return rc;
  c->hist_valid = false;
  return FIVO_OK;
}

int diag(fivo_ctx* c, bool want_u, double* sumD, double* maxu, double* minPtot) {
  const DevParams& d = c->dp;
  int rc = reset_flags(c, 8);
  if (rc) return rc;
  const long long nwarps = (long long)nblk((long long)d.Nx * d.Ny, 256) * 8;
  KTimer t_(c, FIVO_KCLASS_OTHER, 2);
  k_diag<<<nblk((long long)d.Nx * d.Ny, 256), 256, 0, c->st>>>(d, c->S[c->iU], c->w, c->fl, want_u ? 1 : 0, c->part);
  CKL();
  k_sum_parts<<<1, 256, 0, c->st>>>(c->part, nwarps, &c->fl->sumD);
  CKL();
  CK(cudaMemcpyAsync(c->flh, c->fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  *sumD = c->flh->sumD;
  if (maxu) *maxu = c->flh->maxu;
  if (minPtot) *minPtot = c->flh->minPtot;
  return FIVO_OK;
}

}  // namespace

/* ==================================================================== ABI */

extern "C" {

int fivo_abi_version(void) { return FIVO_ABI_VERSION; }

const char* fivo_last_error(void) { return g_err.c_str(); }

void fivo_params_default(fivo_params* p) {
  std::memset(p, 0, sizeof(*p));
  /* LatticeHRGEOS() (src/eos.jl:318-345) */
  const double a[4] = {-15.526548963383643, 18.6159584620131, -10.731808109698516, 2.7413302179949346};
  const double b[4] = {-3.3147904483107595, 5.310983721567554, -4.653922019495976, 1.8600649533271152};
  for (int k = 0; k < 4; ++k) { p->lhrg_a[k] = a[k]; p->lhrg_b[k] = b[k]; }
  p->lhrg_c = -1.0465330501411811; p->lhrg_d = 0.09551531822245873;
  p->g_eff = 40.0; p->m_hq = 1.5; p->g_hq = 6.0;
  p->canon_factor = 0.9524014587885937;
  p->eos_kind = FIVO_EOS_LATTICE_HRG; p->hq_times_fmGeV3 = 1;
  /* IdealDiffVisc2DModel / build_model_2d defaults (src2d/primitives2d.jl:41-210, main2D.jl:85-93) */
  p->with_charge = 1;
  p->tauN_coeff = 1.0; p->nu_clip_factor = -1.0; p->vacuum_n_lo = 1e-6; p->vacuum_n_hi = 2e-3;
  p->eta_over_s = 0.1; p->tauShear_coeff = 0.2; p->deltaShear_factor = 4.0 / 3.0; p->pi_clip_factor = -1.0;
  p->zeta_over_s = 0.1; p->tauPi_coeff = 15.0; p->bulk_T0 = 0.175; p->bulk_width = 0.024;
  p->Pi_clip_factor = -1.0;
  p->r_domain = fx::inf_(); p->T_vac_cut = 0.05; p->E_vac_cut = -1.0;
  p->primrec_tol = 1e-12; p->primrec_maxit = 80;
  p->relax_advect_nu = 1; p->relax_advect_pi = 1; p->relax_advect_Pi = 1; p->vacuum_ramp_relax = 1;
  p->relax_advect_m2 = 1;
  p->shear_projected_deriv = 1; p->diff_projected_deriv = 1; p->shear_constraint_project = 1;
  p->terms = FIVO_TERMS_DEFAULT;
}

int fivo_ctx_create(const fivo_params* p, int nx, int ny, int nghost, double xmax, double ymax, fivo_ctx** out) {
  if (!p || !out) return fail(FIVO_ERR_ARG, "null argument");
  *out = nullptr;
  if (nx <= 8 || ny <= 8) return fail(FIVO_ERR_ARG, "make_grid2d: Nx and Ny must exceed 8");
  if (nghost != 3) return fail(FIVO_ERR_ARG, "the stage is built for nghost = 3");
  if (!(xmax > 0) || !(ymax > 0)) return fail(FIVO_ERR_ARG, "xmax and ymax must be positive");
  int rc = validate(p);
  if (rc) return rc;
  fivo_ctx* c = new fivo_ctx();
  c->dp = make_devparams(p, nx, ny, nghost, xmax, ymax);
  const DevParams& d = c->dp;
  std::memset(&c->cnt, 0, sizeof(c->cnt));
  c->cnt.primfail_index = -1;
  auto cleanup = [&](int code) { fivo_ctx_destroy(c); return code; };
  if (cudaGetDevice(&c->device) != cudaSuccess) return cleanup(fail(FIVO_ERR_CUDA, "no CUDA device"));
  if (cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_CUDA, "cudaStreamCreate failed"));
  c->st = c->own_st;
  std::memset(&c->kt, 0, sizeof(c->kt));
  size_t N = (size_t)d.Ntot;
  if (cudaMalloc(&c->slab, 4 * (size_t)d.nv * N * 8) != cudaSuccess ||
      cudaMalloc(&c->pbuf, 9 * N * 8 + N) != cudaSuccess ||
      cudaMalloc(&c->hbuf, NHIST * N * 8) != cudaSuccess ||
      cudaMalloc(&c->masks, 3 * N) != cudaSuccess ||
      cudaMalloc(&c->fl, sizeof(DevFlags)) != cudaSuccess ||
      cudaMalloc(&c->stage, (size_t)d.nv * N * 8) != cudaSuccess ||
      cudaMalloc(&c->fh, 2 * (size_t)d.nv * N * 8) != cudaSuccess ||
      cudaMalloc(&c->queues, 3 * N * sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&c->part, (size_t)nblk((long long)d.Nx * d.Ny, 256) * 8 * sizeof(double)) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_NOMEM, "device allocation failed"));
  if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || c->nsm < 1)
    c->nsm = 148;
  if (cudaMallocHost(&c->flh, sizeof(DevFlags)) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_NOMEM, "pinned allocation failed"));
  for (int s = 0; s < 4; ++s)
    for (int a = 0; a < FV_MAXP; ++a) c->S[s].f[a] = a < d.nv ? c->slab + ((size_t)s * d.nv + a) * N : nullptr;
  double* q = c->pbuf;
  c->w.yT = q; q += N; c->w.phi = q; q += N; c->w.mu = q; q += N; c->w.alpha = q; q += N;
  c->w.ux = q; q += N; c->w.uy = q; q += N; c->w.P = q; q += N; c->w.n = q; q += N; c->w.e = q; q += N;
  c->w.ok = (uint8_t*)q;
  q = c->hbuf;
  c->h.x0_yT = q; q += N; c->h.x0_phi = q; q += N; c->h.x0_ux = q; q += N; c->h.x0_uy = q; q += N;
  c->h.ux_prev = q; q += N; c->h.uy_prev = q; q += N; c->h.alpha_prev = q; q += N; c->h.T_prev = q; q += N;
  c->h.nux_prev = q; q += N; c->h.nuy_prev = q;
  /* Work2D(): zeros, NaN history (src2d/work2d.jl:115-139) */
  if (cudaMemsetAsync(c->slab, 0, 4 * (size_t)d.nv * N * 8, c->st) != cudaSuccess ||
      cudaMemsetAsync(c->pbuf, 0, 9 * N * 8 + N, c->st) != cudaSuccess ||
      cudaMemsetAsync(c->masks, 0, 3 * N, c->st) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_CUDA, "memset failed"));
  if ((rc = reset_history(c))) return cleanup(rc);
  if ((rc = reset_flags(c, 1 | 2 | 4 | 8 | 16 | 32 | 64))) return cleanup(rc);
  if (ctx_sync(c) != cudaSuccess) return cleanup(fail(FIVO_ERR_CUDA, "sync failed"));
  *out = c;
  return FIVO_OK;
}

void solo_destroy(fivo_batch* b);

int fivo_ctx_destroy(fivo_ctx* c) {
  if (!c) return FIVO_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  solo_destroy(c->solo);
  for (auto& q : c->pend) { cudaEventDestroy(q.a); cudaEventDestroy(q.b); }
  for (auto e : c->pool) cudaEventDestroy(e);
  cudaFree(c->slab); cudaFree(c->pbuf); cudaFree(c->hbuf); cudaFree(c->masks); cudaFree(c->fl);
  cudaFree(c->dU); cudaFree(c->stage); cudaFree(c->fh); cudaFree(c->queues); cudaFree(c->part);
  cudaFree(c->fh32); cudaFree(c->x0save); cudaFree(c->hsave);
  if (c->flh) cudaFreeHost(c->flh);
  if (c->own_st) cudaStreamDestroy(c->own_st);
  if (c->ev_sync) cudaEventDestroy(c->ev_sync);
  delete c;
  return FIVO_OK;
}

int fivo_ctx_info(const fivo_ctx* c, int* nv, int64_t* ntot, double* evac) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (nv) *nv = c->dp.nv;
  if (ntot) *ntot = c->dp.Ntot;
  if (evac) *evac = c->dp.E_vac_cut;
  return FIVO_OK;
}

int fivo_ctx_clone_state(fivo_ctx* dst, const fivo_ctx* src) {
  if (!dst || !src) return fail(FIVO_ERR_ARG, "null context");
  if (dst == src) return FIVO_OK;
  const DevParams& a = dst->dp;
  const DevParams& b = src->dp;
  if (a.Nx != b.Nx || a.Ny != b.Ny || a.nv != b.nv || a.dx != b.dx || a.dy != b.dy ||
      std::memcmp(&a.p, &b.p, sizeof(fivo_params)) != 0)
    return fail(FIVO_ERR_ARG, "fivo_ctx_clone_state: contexts differ in parameters or grid");
  if (dst->device != src->device) return fail(FIVO_ERR_ARG, "fivo_ctx_clone_state: contexts on different devices");
  const size_t N = (size_t)a.Ntot;
  CK(cudaStreamSynchronize(src->st));
  CK(cudaMemcpyAsync(dst->slab, src->slab, 4 * (size_t)a.nv * N * 8, cudaMemcpyDeviceToDevice, dst->st));
  CK(cudaMemcpyAsync(dst->pbuf, src->pbuf, 9 * N * 8 + N, cudaMemcpyDeviceToDevice, dst->st));
  CK(cudaMemcpyAsync(dst->hbuf, src->hbuf, NHIST * N * 8, cudaMemcpyDeviceToDevice, dst->st));
  CK(cudaMemcpyAsync(dst->masks, src->masks, 3 * N, cudaMemcpyDeviceToDevice, dst->st));
  /* the role indices and the plane permutation of the relaxation double buffer */
  for (int s = 0; s < 4; ++s)
    for (int k = 0; k < FV_MAXP; ++k)
      dst->S[s].f[k] = src->S[s].f[k] ? dst->slab + (src->S[s].f[k] - src->slab) : nullptr;
  dst->iU = src->iU; dst->iU1 = src->iU1; dst->iU2 = src->iU2; dst->iT = src->iT;
  dst->hist_valid = src->hist_valid;
  dst->nsteps_run = src->nsteps_run;
  dst->cnt = src->cnt;
  CK(ctx_sync(dst));
  return FIVO_OK;
}

int fivo_upload_state(fivo_ctx* c, const double* U, int nv, int64_t ntot) {
  if (!c || !U) return fail(FIVO_ERR_ARG, "null argument");
  if (nv != c->dp.nv || ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "state size mismatch");
  /* stage the AoS block, then transpose into the U planes */
  double* stage = c->stage;
  CK(cudaMemcpyAsync(stage, U, (size_t)nv * ntot * 8, cudaMemcpyHostToDevice, c->st));
  { KTimer t_(c, FIVO_KCLASS_OTHER);
  k_aos_to_soa<<<nblk((long long)nv * ntot, 256), 256, 0, c->st>>>(c->S[c->iU], stage, nv, ntot);
  CKL(); }
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_download_state(fivo_ctx* c, double* U, int nv, int64_t ntot) {
  if (!c || !U) return fail(FIVO_ERR_ARG, "null argument");
  if (nv != c->dp.nv || ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "state size mismatch");
  double* stage = c->stage;
  { KTimer t_(c, FIVO_KCLASS_OTHER);
  k_soa_to_aos<<<nblk((long long)nv * ntot, 256), 256, 0, c->st>>>(c->S[c->iU], stage, nv, ntot);
  CKL(); }
  CK(cudaMemcpyAsync(U, stage, (size_t)nv * ntot * 8, cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_upload_history(fivo_ctx* c, int64_t ntot, const double* x0_yT, const double* x0_phi,
                        const double* x0_ux, const double* x0_uy, const double* ux_prev,
                        const double* uy_prev, const double* alpha_prev, const double* T_prev) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "history size mismatch");
  const double* src[8] = {x0_yT, x0_phi, x0_ux, x0_uy, ux_prev, uy_prev, alpha_prev, T_prev};
  double* dst[8] = {c->h.x0_yT, c->h.x0_phi, c->h.x0_ux, c->h.x0_uy, c->h.ux_prev, c->h.uy_prev,
                    c->h.alpha_prev, c->h.T_prev};
  for (int k = 0; k < 8; ++k)
    if (src[k]) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)ntot * 8, cudaMemcpyHostToDevice, c->st));
  if (alpha_prev) c->hist_valid = fx::isfinite_(alpha_prev[0]);
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_download_history(fivo_ctx* c, int64_t ntot, double* x0_yT, double* x0_phi, double* x0_ux,
                          double* x0_uy, double* ux_prev, double* uy_prev, double* alpha_prev, double* T_prev) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "history size mismatch");
  double* dst[8] = {x0_yT, x0_phi, x0_ux, x0_uy, ux_prev, uy_prev, alpha_prev, T_prev};
  const double* src[8] = {c->h.x0_yT, c->h.x0_phi, c->h.x0_ux, c->h.x0_uy, c->h.ux_prev, c->h.uy_prev,
                          c->h.alpha_prev, c->h.T_prev};
  for (int k = 0; k < 8; ++k)
    if (dst[k]) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)ntot * 8, cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_upload_nu_history(fivo_ctx* c, int64_t ntot, const double* nux_prev, const double* nuy_prev) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "history size mismatch");
  if (nux_prev) CK(cudaMemcpyAsync(c->h.nux_prev, nux_prev, (size_t)ntot * 8, cudaMemcpyHostToDevice, c->st));
  if (nuy_prev) CK(cudaMemcpyAsync(c->h.nuy_prev, nuy_prev, (size_t)ntot * 8, cudaMemcpyHostToDevice, c->st));
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_download_nu_history(fivo_ctx* c, int64_t ntot, double* nux_prev, double* nuy_prev) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "history size mismatch");
  if (nux_prev) CK(cudaMemcpyAsync(nux_prev, c->h.nux_prev, (size_t)ntot * 8, cudaMemcpyDeviceToHost, c->st));
  if (nuy_prev) CK(cudaMemcpyAsync(nuy_prev, c->h.nuy_prev, (size_t)ntot * 8, cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_reset_history(fivo_ctx* c) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  int rc = reset_history(c);
  if (rc) return rc;
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_get_primitives(fivo_ctx* c, int64_t ntot, double* yT, double* phi, double* mu, double* alpha,
                        double* ux, double* uy, double* P, double* n, double* e, uint8_t* ok) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (ntot != c->dp.Ntot) return fail(FIVO_ERR_ARG, "size mismatch");
  double* dst[9] = {yT, phi, mu, alpha, ux, uy, P, n, e};
  const double* src[9] = {c->w.yT, c->w.phi, c->w.mu, c->w.alpha, c->w.ux, c->w.uy, c->w.P, c->w.n, c->w.e};
  for (int k = 0; k < 9; ++k)
    if (dst[k]) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)ntot * 8, cudaMemcpyDeviceToHost, c->st));
  if (ok) CK(cudaMemcpyAsync(ok, c->w.ok, (size_t)ntot, cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_get_counters(fivo_ctx* c, fivo_counters* out) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  *out = c->cnt;
  return FIVO_OK;
}

int fivo_rhs(fivo_ctx* c, double tau, int bc, const uint8_t* mask, double* dU) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  const DevParams& d = c->dp;
  const uint8_t* dmask = nullptr;
  if (mask) {
    CK(cudaMemcpyAsync(c->masks + d.Ntot, mask, (size_t)d.Ntot, cudaMemcpyHostToDevice, c->st));
    dmask = c->masks + d.Ntot;
  }
  if (dU && !c->dU) CK(cudaMalloc(&c->dU, (size_t)d.nv * d.Ntot * 8));
  if (dU) CK(cudaMemsetAsync(c->dU, 0, (size_t)d.nv * d.Ntot * 8, c->st));
  int rc = run_stage(c, c->iU, c->iT, c->iU, tau, tau, 0.0, 0.0, 0.0, COMB_RHS_ONLY, dmask, bc, nullptr,
                     dU ? c->dU : nullptr);
  if (rc) return rc;
  if (dU) {
    /* planes -> AoS on the host side */
    std::vector<double> tmp((size_t)d.nv * d.Ntot);
    CK(cudaMemcpy(tmp.data(), c->dU, tmp.size() * 8, cudaMemcpyDeviceToHost));
    for (long long i = 0; i < d.Ntot; ++i)
      for (int a = 0; a < d.nv; ++a) dU[i * d.nv + a] = tmp[(size_t)a * d.Ntot + i];
  }
  return FIVO_OK;
}

int fivo_step(fivo_ctx* c, int integrator, double tau, double dtau, int max_halve, int max_mood, int bc,
              double* dtau_used, int* ok) {
  if (!c || !dtau_used || !ok) return fail(FIVO_ERR_ARG, "null argument");
  if (integrator == FIVO_SSPRK3) return step3(c, tau, dtau, max_halve, bc, dtau_used, ok);
  if (integrator == FIVO_SSPRK2) return step2(c, tau, dtau, max_halve, max_mood, bc, dtau_used, ok);
  return fail(FIVO_ERR_ARG, "integrator must be FIVO_SSPRK2 or FIVO_SSPRK3");
}

int fivo_update_primitives(fivo_ctx* c, double tau, int bc, int64_t* nprimfail) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  int rc = update_prims(c, tau, bc);
  if (rc) return rc;
  if ((rc = sync_flags(c, false))) return rc;
  if (nprimfail) *nprimfail = c->cnt.nprimfail;
  return FIVO_OK;
}

int fivo_relax(fivo_ctx* c, double tau, double dtau) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  const fivo_params& p = c->dp.p;
  if (!(p.enable_shear || p.enable_bulk || p.enable_diff)) return FIVO_OK;
  int rc = relax_project(c, tau, dtau, 1, 0);
  if (rc) return rc;
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_project_shear(fivo_ctx* c, double* max_res, double* mean_res) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (!c->dp.hasShear) { if (max_res) *max_res = 0.0; if (mean_res) *mean_res = 0.0; return FIVO_OK; }
  int rc = relax_project(c, 0.0, 1.0, 0, 1);
  if (rc) return rc;
  return read_shear(c, max_res, mean_res);
}

int fivo_compute_dt(fivo_ctx* c, double tau, double cfl, double cfltau, double* dt) {
  if (!c || !dt) return fail(FIVO_ERR_ARG, "null argument");
  /* compute_dt_2d, src2d/timestepper2d.jl:37-47 */
  double amax = 0.0;
  if (c->cnt.amax > amax) amax = c->cnt.amax;
  amax = jmax(amax, 1e-6);
  double dt_cfl = (cfl * jmin(c->dp.dx, c->dp.dy)) / amax;
  double dt_tau = cfltau * tau;
  *dt = jmin(dt_cfl, dt_tau);
  return FIVO_OK;
}

namespace {
/* run_sim_2d!'s while loop (main2D.jl:436-513) */
int advance_loop(fivo_ctx* c, double tau, double taufinal, double cfl, double cfltau, int integrator, int bc,
                 int64_t max_steps, fivo_run_result* out) {
  const DevParams& d = c->dp;
  const fivo_params& p = d.p;
  int rc;
  int64_t nsteps = 0, nprimfail = 0, nvacuum = 0;
  double max_shear_res = 0.0;
  const bool any_sector = p.enable_shear || p.enable_bulk || p.enable_diff;
  out->ok = 1;
  while (tau < taufinal && nsteps < max_steps) {
    double D;
    fivo_compute_dt(c, tau, cfl, cfltau, &D);
    D = jmin(D, taufinal - tau);
    if (D <= 0) break;
    if (c->hist_valid || c->nsteps_run > 0) {
      KTimer t_(c, FIVO_KCLASS_OTHER);
      k_snapshot<<<nblk(d.Ntot, 256), 256, 0, c->st>>>(d, c->w, c->h);
      CKL();
      c->hist_valid = true;
    }
    double used = 0.0;
    int ok = 0;
    if (integrator == FIVO_SSPRK3) rc = step3(c, tau, D, 12, bc, &used, &ok);
    else rc = step2(c, tau, D, 12, 2, bc, &used, &ok);
    if (rc) return rc;
    if (!ok) { out->ok = 0; break; }
    tau += used;
    nsteps += 1;
    c->nsteps_run += 1;
    if (any_sector) {
      if ((rc = update_prims(c, tau, bc, false))) return rc;
      if ((rc = relax_project(c, tau, used, 1, d.hasShear))) return rc;
      if ((rc = sync_flags(c, false))) return rc;
      if (d.hasShear) {
        uint64_t b = c->flh->shear_max_bits;
        double r; std::memcpy(&r, &b, 8);
        max_shear_res = jmax(max_shear_res, r);
      }
    } else if (d.hasShear) {
      if ((rc = relax_project(c, tau, used, 0, 1))) return rc;
      double r;
      if ((rc = read_shear(c, &r, nullptr))) return rc;
      max_shear_res = jmax(max_shear_res, r);
    }
    nprimfail += c->cnt.nprimfail;
    nvacuum += c->cnt.nvacuum;
  }
  out->tau = tau; out->nsteps = nsteps; out->nprimfail = nprimfail; out->nvacuum = nvacuum;
  out->max_shear_res = max_shear_res;
  return FIVO_OK;
}
}  // namespace

int solo_advance(fivo_ctx* c, double tau, double taufinal, double cfl, double cfltau, int integrator, int bc,
                 int64_t max_steps, fivo_run_result* out);

namespace {
/* run_sim_2d! before its loop: the history reset, one RHS pass to populate the
 * primitives and signal speeds (main2D.jl:418), the initial total charge */
int run_begin(fivo_ctx* c, double tau0, int bc, int reset_hist, double* Qin) {
  int rc;
  if (reset_hist && (rc = reset_history(c))) return rc;
  c->nsteps_run = 0;
  if ((rc = run_stage(c, c->iU, c->iT, c->iU, tau0, tau0, 0.0, 0.0, 0.0, COMB_RHS_ONLY, nullptr, bc, nullptr, nullptr))) return rc;
  return diag(c, false, Qin, nullptr, nullptr);
}

/* run_sim_2d! after its loop: the result's bulk diagnostics */
int run_end(fivo_ctx* c, double Qin, fivo_run_result* out) {
  int rc;
  out->Q0 = Qin;
  if (!out->ok) {
    out->maxu = fx::nan_(); out->dQ = fx::nan_(); out->Q1 = fx::nan_(); out->minPtot = fx::nan_();
    return FIVO_OK;
  }
  double Qout = 0.0, maxu = 0.0, minPtot = 0.0;
  if ((rc = diag(c, true, &Qout, &maxu, &minPtot))) return rc;
  out->maxu = maxu;
  out->dQ = fx::fabs_(Qin) > 0 ? fx::fabs_(Qout - Qin) / fx::fabs_(Qin) : 0.0;
  out->Q1 = Qout; out->minPtot = minPtot;
  return FIVO_OK;
}
}  // namespace

int fivo_run(fivo_ctx* c, double tau0, double taufinal, double cfl, double cfltau, int integrator, int bc,
             int64_t max_steps, int reset_hist, fivo_run_result* out) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  if (integrator != FIVO_SSPRK2 && integrator != FIVO_SSPRK3)
    return fail(FIVO_ERR_ARG, "integrator must be FIVO_SSPRK2 or FIVO_SSPRK3");
  int rc;
  std::memset(out, 0, sizeof(*out));
  double Qin = 0.0;
  if ((rc = run_begin(c, tau0, bc, reset_hist, &Qin))) return rc;
  if (c->graphs && !c->profiling) rc = solo_advance(c, tau0, taufinal, cfl, cfltau, integrator, bc, max_steps, out);
  else rc = advance_loop(c, tau0, taufinal, cfl, cfltau, integrator, bc, max_steps, out);
  if (rc) return rc;
  return run_end(c, Qin, out);
}

int fivo_advance(fivo_ctx* c, double tau, double taufinal, double cfl, double cfltau, int integrator, int bc,
                 int64_t max_steps, fivo_run_result* out) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  if (integrator != FIVO_SSPRK2 && integrator != FIVO_SSPRK3)
    return fail(FIVO_ERR_ARG, "integrator must be FIVO_SSPRK2 or FIVO_SSPRK3");
  std::memset(out, 0, sizeof(*out));
  if (c->graphs && !c->profiling) return solo_advance(c, tau, taufinal, cfl, cfltau, integrator, bc, max_steps, out);
  return advance_loop(c, tau, taufinal, cfl, cfltau, integrator, bc, max_steps, out);
}

int fivo_run_diagnostics(fivo_ctx* c, double* Q, double* maxu, double* minPtot) {
  if (!c || !Q || !maxu || !minPtot) return fail(FIVO_ERR_ARG, "null argument");
  return diag(c, true, Q, maxu, minPtot);
}

int fivo_finalize_ic(fivo_ctx* c, double tau0, int bc) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  const DevParams& d = c->dp;
  { KTimer t_(c, FIVO_KCLASS_OTHER);
  k_finalize_ic<<<nblk((long long)d.Nx * d.Ny, 256), 256, 0, c->st>>>(d, c->S[c->iU], tau0);
  CKL(); }
  int rc = launch_bc(c, c->S[c->iU], bc);
  if (rc) return rc;
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_sync(fivo_ctx* c) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_ctx_set_stream(fivo_ctx* c, void* stream) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  CK(ctx_sync(c));
  c->st = stream ? (cudaStream_t)stream : c->own_st;
  return FIVO_OK;
}

int fivo_profile(fivo_ctx* c, int enable) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  CK(ctx_sync(c));
  c->profiling = enable != 0;
  return FIVO_OK;
}

int fivo_profile_read(fivo_ctx* c, fivo_kernel_times* out, int reset) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(c->flh, c->fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  /* deferred cells are counted on the device; the profile owns those totals */
  c->kt.units[FIVO_KCLASS_PRIM_SLOW] = (int64_t)c->flh->tot_p - c->tot_base_p;
  c->kt.units[FIVO_KCLASS_ADM_SLOW] = (int64_t)c->flh->tot_a - c->tot_base_a;
  *out = c->kt;
  if (reset) {
    std::memset(&c->kt, 0, sizeof(c->kt));
    c->tot_base_p = (int64_t)c->flh->tot_p;
    c->tot_base_a = (int64_t)c->flh->tot_a;
  }
  return FIVO_OK;
}

/* ------------------------------------------------- batched one-shot helpers */

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};
int up(DevBuf& b, const double* src, long long n) {
  if (!src) return FIVO_OK;
  CK(cudaMalloc(&b.p, n * 8));
  CK(cudaMemcpy(b.p, src, n * 8, cudaMemcpyHostToDevice));
  return FIVO_OK;
}
}  // namespace

int fivo_set_cells(const fivo_params* p, int64_t ncell, double tau, const double* T, const double* alpha,
                   const double* ux, const double* uy, const double* Pi, const double* pixx, const double* pixy,
                   const double* piyy, const double* nux, const double* nuy, double* U, uint8_t* ok) {
  if (!p || !T || !alpha || !ux || !uy || !U || !ok) return fail(FIVO_ERR_ARG, "null argument");
  if (ncell <= 0) return FIVO_OK;
  int rc = validate(p);
  if (rc) return rc;
  DevParams d = make_devparams(p, 9, 9, 3, 1.0, 1.0);
  DevBuf bT, ba, bx, by, bP, bxx, bxy, byy, bnx, bny, bU, bok;
  const double* srcs[10] = {T, alpha, ux, uy, Pi, pixx, pixy, piyy, nux, nuy};
  DevBuf* bufs[10] = {&bT, &ba, &bx, &by, &bP, &bxx, &bxy, &byy, &bnx, &bny};
  for (int k = 0; k < 10; ++k) if ((rc = up(*bufs[k], srcs[k], ncell))) return rc;
  CK(cudaMalloc(&bU.p, (size_t)ncell * d.nv * 8));
  CK(cudaMemcpy(bU.p, U, (size_t)ncell * d.nv * 8, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&bok.p, (size_t)ncell));
  auto P_ = [](DevBuf& b) { return (const double*)b.p; };
  if (p->eos_kind == FIVO_EOS_LATTICE_HRG)
    k_set_cells<FIVO_EOS_LATTICE_HRG><<<nblk(ncell, 128), 128>>>(d, ncell, tau, P_(bT), P_(ba), P_(bx), P_(by), P_(bP), P_(bxx), P_(bxy), P_(byy), P_(bnx), P_(bny), (double*)bU.p, (uint8_t*)bok.p);
  else
    k_set_cells<FIVO_EOS_CONFORMAL_HQ><<<nblk(ncell, 128), 128>>>(d, ncell, tau, P_(bT), P_(ba), P_(bx), P_(by), P_(bP), P_(bxx), P_(bxy), P_(byy), P_(bnx), P_(bny), (double*)bU.p, (uint8_t*)bok.p);
  CKL();
  CK(cudaMemcpy(U, bU.p, (size_t)ncell * d.nv * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ok, bok.p, (size_t)ncell, cudaMemcpyDeviceToHost));
  return FIVO_OK;
}

int fivo_glauber_ic(fivo_ctx* c, double tau0, const double* parts, const double* weights, int64_t npart,
                    const double* binary, int64_t nbin, double width, double Tpeak, double ncharm,
                    double alpha_min, double T_edge, double alpha_edge, int bc, double* T_out,
                    double* alpha_out) {
  if (!c || !parts || !weights || (nbin > 0 && !binary)) return fail(FIVO_ERR_ARG, "null argument");
  const DevParams& d = c->dp;
  if (d.p.eos_kind != FIVO_EOS_LATTICE_HRG)
    return fail(FIVO_ERR_CONFIG, "fivo_glauber_ic: the MC-Glauber initial condition is built for LatticeHRGEOS");
  if (npart < 1 || nbin < 0 || !(width > 0) || !(Tpeak > 0) || !(tau0 > 0))
    return fail(FIVO_ERR_ARG, "fivo_glauber_ic: need npart >= 1, nbin >= 0, width > 0, Tpeak > 0, tau0 > 0");
  const long long N = d.Ntot;
  int rc;
  DevBuf bp, bw, bb, planes, aos, zero, okb, scal;
  if ((rc = up(bp, parts, 2 * npart)) || (rc = up(bw, weights, npart))) return rc;
  if (nbin > 0 && (rc = up(bb, binary, 2 * nbin))) return rc;
  CK(cudaMalloc(&planes.p, 4 * (size_t)N * 8));
  CK(cudaMalloc(&aos.p, (size_t)N * d.nv * 8));
  CK(cudaMalloc(&zero.p, (size_t)N * 8));
  CK(cudaMalloc(&okb.p, (size_t)N));
  CK(cudaMalloc(&scal.p, 16));
  double* s = (double*)planes.p;
  double* nb = s + N;
  double* T = s + 2 * N;
  double* al = s + 3 * N;
  unsigned long long* mx = (unsigned long long*)scal.p;
  double* interior = (double*)scal.p + 1;
  CK(cudaMemsetAsync(scal.p, 0, 16, c->st));
  CK(cudaMemsetAsync(aos.p, 0, (size_t)N * d.nv * 8, c->st));
  CK(cudaMemsetAsync(zero.p, 0, (size_t)N * 8, c->st));
  /* e_peak: the light-sector energy density at Tpeak (the same functions on the host) */
  double Pl, dP;
  const double Tp = jmax(Tpeak, FV_T_MIN);
  light_eos<3>(Tp, d, &Pl, &dP, nullptr);
  const double e_peak = (-Pl) + (Tp * dP);
  /* the edge state: its light-sector energy density and charm density n(T_edge, alpha_edge) */
  double e_edge = 0.0, n_edge = 0.0;
  if (T_edge > 0) {
    double Pe, dPe;
    light_eos<3>(T_edge, d, &Pe, &dPe, nullptr);
    e_edge = (-Pe) + (T_edge * dPe);
    const double x = lhrg_x(T_edge, d);
    double P0, n0, e0;
    lhrg_assemble(T_edge, 0.0, d, x, Pe, e_edge, lhrg_K2(x), &P0, &n0, &e0);
    n_edge = n0 * fx_exp(alpha_edge);
  }
  const long long nw = (long long)nblk(N, 256) * 8;
  DevBuf partb;
  CK(cudaMalloc(&partb.p, (size_t)nw * 8));
  {
    KTimer t_(c, FIVO_KCLASS_OTHER, 5);
    k_glauber_deposit<<<nblk(N, 128), 128, 0, c->st>>>(d, (const double*)bp.p, (const double*)bw.p, npart, width, s);
    CKL();
    k_glauber_deposit<<<nblk(N, 128), 128, 0, c->st>>>(d, (const double*)bb.p, nullptr, nbin, width, nb);
    CKL();
    k_glauber_reduce<<<nblk(N, 256), 256, 0, c->st>>>(d, s, nb, mx, (double*)partb.p);
    CKL();
    k_sum_parts<<<1, 256, 0, c->st>>>((const double*)partb.p, nw, interior);
    CKL();
    k_glauber_fields<<<nblk(N, 128), 128, 0, c->st>>>(d, s, nb, mx, interior, e_peak, e_edge, n_edge, tau0, ncharm,
                                                      alpha_min, T, al);
    CKL();
  }
  {
    KTimer t_(c, FIVO_KCLASS_OTHER, 2);
    const double* z = (const double*)zero.p;
    k_set_cells<FIVO_EOS_LATTICE_HRG><<<nblk(N, 128), 128, 0, c->st>>>(d, N, tau0, T, al, z, z, nullptr, nullptr, nullptr,
                                                                      nullptr, nullptr, nullptr, (double*)aos.p,
                                                                      (uint8_t*)okb.p);
    CKL();
    k_aos_to_soa<<<nblk(N * d.nv, 256), 256, 0, c->st>>>(c->S[c->iU], (const double*)aos.p, d.nv, N);
    CKL();
  }
  if (T_out) CK(cudaMemcpyAsync(T_out, T, (size_t)N * 8, cudaMemcpyDeviceToHost, c->st));
  if (alpha_out) CK(cudaMemcpyAsync(alpha_out, al, (size_t)N * 8, cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  return fivo_finalize_ic(c, tau0, bc);
}

int fivo_eos_Pne(const fivo_params* p, int64_t n, const double* T, const double* mu, double* P, double* nq,
                 double* e) {
  if (!p || !T || !mu || !P || !nq || !e) return fail(FIVO_ERR_ARG, "null argument");
  if (n <= 0) return FIVO_OK;
  int rc = validate(p);
  if (rc) return rc;
  DevParams d = make_devparams(p, 9, 9, 3, 1.0, 1.0);
  DevBuf bT, bm, bo;
  if ((rc = up(bT, T, n)) || (rc = up(bm, mu, n))) return rc;
  CK(cudaMalloc(&bo.p, 3 * (size_t)n * 8));
  double* o = (double*)bo.p;
  if (p->eos_kind == FIVO_EOS_LATTICE_HRG)
    k_eos<FIVO_EOS_LATTICE_HRG><<<nblk(n, 128), 128>>>(d, n, (const double*)bT.p, (const double*)bm.p, o, o + n, o + 2 * n);
  else
    k_eos<FIVO_EOS_CONFORMAL_HQ><<<nblk(n, 128), 128>>>(d, n, (const double*)bT.p, (const double*)bm.p, o, o + n, o + 2 * n);
  CKL();
  CK(cudaMemcpy(P, o, n * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nq, o + n, n * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(e, o + 2 * n, n * 8, cudaMemcpyDeviceToHost));
  return FIVO_OK;
}

int fivo_cons_to_prim(const fivo_params* p, int64_t n, double tau, const double* cons, const double* warm,
                      double* prim, uint8_t* ok, uint8_t* reason) {
  if (!p || !cons || !prim || !ok) return fail(FIVO_ERR_ARG, "null argument");
  if (n <= 0) return FIVO_OK;
  int rc = validate(p);
  if (rc) return rc;
  DevParams d = make_devparams(p, 9, 9, 3, 1.0, 1.0);
  DevBuf bc, bw, bp, bo, br;
  if ((rc = up(bc, cons, 11 * n)) || (rc = up(bw, warm, 4 * n))) return rc;
  CK(cudaMalloc(&bp.p, 7 * (size_t)n * 8));
  CK(cudaMalloc(&bo.p, (size_t)n));
  CK(cudaMalloc(&br.p, (size_t)n));
  const double* c_ = (const double*)bc.p;
  const double* w_ = (const double*)bw.p;
  if (p->eos_kind == FIVO_EOS_LATTICE_HRG)
    k_cons_to_prim<FIVO_EOS_LATTICE_HRG, true><<<nblk(n, 128), 128>>>(d, n, tau, c_, w_, (double*)bp.p, (uint8_t*)bo.p, (uint8_t*)br.p);
  else if (d.ncharge)
    k_cons_to_prim<FIVO_EOS_CONFORMAL_HQ, true><<<nblk(n, 128), 128>>>(d, n, tau, c_, w_, (double*)bp.p, (uint8_t*)bo.p, (uint8_t*)br.p);
  else
    k_cons_to_prim<FIVO_EOS_CONFORMAL_HQ, false><<<nblk(n, 128), 128>>>(d, n, tau, c_, w_, (double*)bp.p, (uint8_t*)bo.p, (uint8_t*)br.p);
  CKL();
  CK(cudaMemcpy(prim, bp.p, 7 * (size_t)n * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ok, bo.p, (size_t)n, cudaMemcpyDeviceToHost));
  if (reason) CK(cudaMemcpy(reason, br.p, (size_t)n, cudaMemcpyDeviceToHost));
  return FIVO_OK;
}

}  /* extern "C" */

/* ======================================================== rhs without allocation
 *
 * Some hosts cannot call cudaMalloc: a Julia driver whose device memory is owned
 * by CUDA.jl's pool allocator, or a long-running service that forbids device
 * allocation after start-up so its memory footprint stays fixed. fivo_rhs_noalloc serves them: its work
 * memory (the cell primitives, the warm-start planes it starts cold from, and
 * the flag block) is the file-scope array below, sized for
 * FIVO_NOALLOC_MAX_CELLS cells (about 17 MB). The array exists on every GPU
 * that loads this library until the process exits. The first call on a device
 * looks up its device address (cudaGetSymbolAddress) and keeps it for the life of
 * the process, so make that first call before any stream capture, and do not use
 * the library across a cudaDeviceReset (the kept address would be stale). Every
 * call shares the array and it keeps the last call's contents, so each call clears
 * what must start cleared (flags, warm starts); calls whose work overlaps on the
 * GPU race on it. A call is synchronous: it waits for its stream to read back the
 * signal speed and the recovery counters.
 */

namespace {
constexpr size_t NOALLOC_PLANE_BYTES = (size_t)FIVO_NOALLOC_MAX_CELLS * 8;
/* 9 primitive planes + 4 warm-start planes (doubles), the ok bytes, the flags */
constexpr size_t NOALLOC_BYTES = 13 * NOALLOC_PLANE_BYTES + (((size_t)FIVO_NOALLOC_MAX_CELLS + 255) / 256) * 256 +
                                 ((sizeof(DevFlags) + 255) / 256) * 256;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[128] = {nullptr};

int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(FIVO_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = (unsigned char*)p;
  }
  *out = g_noalloc_ptr[dev];
  return FIVO_OK;
}
}  // namespace

extern "C" int fivo_rhs_noalloc(const fivo_params* p, int nx, int ny, double xmax, double ymax, double tau,
                                int bc, double* U, double* dU, double* amax, fivo_counters* counters,
                                void* stream) {
  if (!p || !U || !dU || !amax) return fail(FIVO_ERR_ARG, "null argument");
  if (nx <= 8 || ny <= 8) return fail(FIVO_ERR_ARG, "make_grid2d: Nx and Ny must exceed 8");
  if (!(xmax > 0) || !(ymax > 0)) return fail(FIVO_ERR_ARG, "xmax and ymax must be positive");
  const long long ntot = (long long)(nx + 6) * (ny + 6);
  if (ntot > FIVO_NOALLOC_MAX_CELLS)
    return fail(FIVO_ERR_ARG, "fivo_rhs_noalloc: (nx+6)*(ny+6) = " + std::to_string(ntot) +
                                  " cells exceeds FIVO_NOALLOC_MAX_CELLS = " +
                                  std::to_string((long long)FIVO_NOALLOC_MAX_CELLS));
  int rc = validate(p);
  if (rc) return rc;
  unsigned char* base = nullptr;
  if ((rc = noalloc_scratch(&base))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  DevParams d = make_devparams(p, nx, ny, 3, xmax, ymax);
  const size_t N = (size_t)d.Ntot;
  DevState S;
  for (int a = 0; a < FV_MAXP; ++a) S.f[a] = a < d.nv ? U + (size_t)a * N : nullptr;
  double* q = (double*)base;
  DevPrims w;
  w.yT = q; q += N; w.phi = q; q += N; w.mu = q; q += N; w.alpha = q; q += N;
  w.ux = q; q += N; w.uy = q; q += N; w.P = q; q += N; w.n = q; q += N; w.e = q; q += N;
  DevHist h;
  h.x0_yT = q; q += N; h.x0_phi = q; q += N; h.x0_ux = q; q += N; h.x0_uy = q; q += N;
  h.ux_prev = h.uy_prev = h.alpha_prev = h.T_prev = h.nux_prev = h.nuy_prev = nullptr;
  unsigned char* okb = base + 13 * NOALLOC_PLANE_BYTES;
  w.ok = (uint8_t*)okb;
  DevFlags* fl = (DevFlags*)(okb + (((size_t)FIVO_NOALLOC_MAX_CELLS + 255) / 256) * 256);
  /* clear what the pass must start from: NaN warm starts (a cold start), the flags */
  k_fill_nan<<<nblk(4 * (long long)N, 256), 256, 0, st>>>(h.x0_yT, 4 * (long long)N);
  CKL();
  k_reset_flags<<<1, 32, 0, st>>>(fl, 1 | 2 | 4 | 8 | 64, 0ULL);
  CKL();
  CK(cudaMemsetAsync(dU, 0, (size_t)d.nv * N * 8, st));
  /* rhs_2d!: BCs, primitive pass, faces + sources (src2d/rhs2d.jl:169-249) */
  long long nframe = d.Ntot - (long long)d.Nx * d.Ny;
  k_bc<<<nblk(nframe, 256), 256, 0, st>>>(d, S, bc);
  CKL();
  unsigned g = nblk(d.Ntot, 128);
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG)
    k_primitive<FIVO_EOS_LATTICE_HRG, true><<<g, 128, 0, st>>>(d, S, w, h, tau, fl);
  else if (d.ncharge)
    k_primitive<FIVO_EOS_CONFORMAL_HQ, true><<<g, 128, 0, st>>>(d, S, w, h, tau, fl);
  else
    k_primitive<FIVO_EOS_CONFORMAL_HQ, false><<<g, 128, 0, st>>>(d, S, w, h, tau, fl);
  CKL();
  StageArgs a;
  a.Ub = S; a.Uold = S; a.Uout = S; a.w = w; a.ffo = nullptr; a.bad = nullptr; a.dU = dU;
  a.tau = tau; a.tau_state = tau; a.dt = 0.0; a.wold = 0.0; a.wnew = 0.0; a.mode = COMB_RHS_ONLY; a.fl = fl;
  size_t smem = (size_t)(ST_NFX + ST_NFY) * d.nvf * sizeof(double);
  dim3 grid((d.Nxtot + ST_CX - 1) / ST_CX, (d.Nytot + ST_CY - 1) / ST_CY);
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG) {
    CK(cudaFuncSetAttribute(k_stage<FIVO_EOS_LATTICE_HRG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_stage<FIVO_EOS_LATTICE_HRG, true><<<grid, 256, smem, st>>>(d, a);
  } else if (d.ncharge) {
    CK(cudaFuncSetAttribute(k_stage<FIVO_EOS_CONFORMAL_HQ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_stage<FIVO_EOS_CONFORMAL_HQ, true><<<grid, 256, smem, st>>>(d, a);
  } else {
    CK(cudaFuncSetAttribute(k_stage<FIVO_EOS_CONFORMAL_HQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_stage<FIVO_EOS_CONFORMAL_HQ, false><<<grid, 256, smem, st>>>(d, a);
  }
  CKL();
  /* the whole flag block: the signal speed and the primitive pass's failure bookkeeping */
  DevFlags f;
  CK(cudaMemcpyAsync(&f, fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  uint64_t bits = f.amax_bits;
  std::memcpy(amax, &bits, 8);
  if (counters) {
    std::memset(counters, 0, sizeof(*counters));
    counters->nprimfail = f.nprimfail;
    counters->nvacuum = f.nvacuum;
    if (f.rep != (unsigned long long)REP_NONE) {
      counters->primfail_index = (int64_t)(f.rep >> 8);
      counters->primfail_reason = (int32_t)(f.rep & 0xff);
    } else {
      counters->primfail_index = -1;
    }
    counters->primfail_resnorm = fx::nan_();
    counters->amax = *amax;
  }
  return FIVO_OK;
}

/* ------------------------------------------------------------------------
 * Batches of events (event-by-event hydro: many independent events, uneven
 * grids). Each event is a context with its own stream; a pool of host threads
 * drives them, so the kernels of different events run on the GPU at the same
 * time and the latency-bound passes of one event overlap the work of others.
 * Events share the model parameters; each has its own grid, dt and control
 * flow, exactly as separate run_sim_2d! calls.
 * ---------------------------------------------------------------------- */
struct Lockstep;
int ls_destroy(Lockstep* L);

struct fivo_batch {
  std::vector<fivo_ctx*> ev;
  int nworkers = 1;
  int device = 0;
  Lockstep* ls = nullptr;     /* lockstep mode (fivo_batch_set_lockstep) */
  bool lockstep = false;
};

int fivo_batch_create(const fivo_params* p, int nevents, const int* nx, const int* ny, const double* xmax,
                      const double* ymax, int nghost, int nworkers, fivo_batch** out) {
  if (!p || !nx || !ny || !xmax || !ymax || !out) return fail(FIVO_ERR_ARG, "null argument");
  *out = nullptr;
  if (nevents < 1) return fail(FIVO_ERR_ARG, "fivo_batch_create: nevents must be >= 1");
  fivo_batch* b = new fivo_batch();
  if (cudaGetDevice(&b->device) != cudaSuccess) { delete b; return fail(FIVO_ERR_CUDA, "no CUDA device"); }
  b->nworkers = nworkers > 0 ? std::min(nworkers, nevents) : std::min(nevents, 32);
  for (int k = 0; k < nevents; ++k) {
    fivo_ctx* c = nullptr;
    int rc = fivo_ctx_create(p, nx[k], ny[k], nghost, xmax[k], ymax[k], &c);
    if (rc == FIVO_OK && cudaEventCreateWithFlags(&c->ev_sync, cudaEventBlockingSync | cudaEventDisableTiming) !=
                             cudaSuccess)
      rc = fail(FIVO_ERR_CUDA, "event creation failed");
    if (rc != FIVO_OK) {
      std::string msg = "event " + std::to_string(k) + ": " + g_err;
      if (c) fivo_ctx_destroy(c);
      fivo_batch_destroy(b);
      return fail(rc, msg);
    }
    b->ev.push_back(c);
  }
  *out = b;
  return FIVO_OK;
}

int fivo_batch_destroy(fivo_batch* b) {
  if (!b) return FIVO_OK;
  ls_destroy(b->ls);
  for (fivo_ctx* c : b->ev) fivo_ctx_destroy(c);
  delete b;
  return FIVO_OK;
}

int fivo_batch_event(fivo_batch* b, int k, fivo_ctx** ctx) {
  if (!b || !ctx) return fail(FIVO_ERR_ARG, "null argument");
  if (k < 0 || k >= (int)b->ev.size()) return fail(FIVO_ERR_ARG, "fivo_batch_event: index out of range");
  *ctx = b->ev[k];
  return FIVO_OK;
}

namespace {
/* run fn(k) for every event on the batch's worker threads; per-event status
 * and message; returns the first failing event's status */
template <class F>
int batch_for_each(fivo_batch* b, int* status, F fn) {
  const int n = (int)b->ev.size();
  std::vector<int> st(n, FIVO_OK);
  std::vector<std::string> msg(n);
  std::atomic<int> next{0};
  auto worker = [&]() {
    if (cudaSetDevice(b->device) != cudaSuccess) return;
    for (;;) {
      int k = next.fetch_add(1);
      if (k >= n) break;
      st[k] = fn(k);
      if (st[k] != FIVO_OK) msg[k] = g_err;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < b->nworkers; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  int first = -1;
  for (int k = 0; k < n; ++k) {
    if (status) status[k] = st[k];
    if (st[k] != FIVO_OK && first < 0) first = k;
  }
  if (next.load() < n) return fail(FIVO_ERR_CUDA, "fivo_batch: a worker could not select the device");
  if (first >= 0) return fail(st[first], "event " + std::to_string(first) + ": " + msg[first]);
  return FIVO_OK;
}
}  // namespace

/* ------------------------------------------------------------------------
 * Lockstep batches (fivo_batch_set_lockstep): the events' steps taken together,
 * each kernel of a step launched once over every event's blocks (batch.cuh).
 * The launch sequences:
 *   STEP  the optimistic SSPRK step of every active event: k_snapshot (when
 *         due), the warm-start save and copy_state, then per stage the ghost
 *         fill, flag reset, fast recovery, deferred recoveries, faces, update,
 *         admissibility inversions and the output's ghost fill; the flag blocks
 *         of all events gathered and read back at once.
 *   POST  update_primitives_2d! and relax_dissipative_2d! (+ project_shear!) on
 *         the events whose step was accepted, then the flags again.
 *   FULL  STEP then POST in one sequence (one host read per step), POST on the
 *         roles an accepted step takes; the step's first kernel also copies the
 *         history planes POST overwrites.
 * After the read the host settles, per event, what advance_loop settles after
 * step2/step3: an event with an inadmissible cell is undone (roles, warm
 * starts, and after FULL the history planes and, for step2, the state from its
 * copy) and stepped by step2_rest/step3_rest on its own stream, exactly as a
 * separate run would after its optimistic pass, and then gets its own POST. So
 * every event sees the same kernels on the same inputs in the same order as in
 * fivo_run, and its results are bitwise those of a separate run.
 * ---------------------------------------------------------------------- */
/* the launch sequences: the optimistic step; the post-step pass; both in one (the
 * post-step pass speculating that the step is accepted, undone where it is not) */
enum { LS_STEP = 0, LS_POST = 1, LS_FULL = 2 };

struct Lockstep {
  int flags = 0;
  cudaStream_t st = nullptr;                 /* the lockstep's own stream */
  cudaStream_t run_st = nullptr;             /* where the sequences run: st, or a single context's stream */
  int64_t kernels = 0;                       /* kernels launched (graph nodes replayed included) */
  int last_nk = 0;                           /* kernels of the sequence built last */
  cudaEvent_t done = nullptr;                /* the end of a sequence; one host thread waits on it */
  bool prepared = false;                     /* the learned kernels' shared-memory attributes are set */
  cudaEvent_t ta = nullptr, tb = nullptr;    /* device time of a launch sequence */
  int nev = 0, nsm = 148;
  DevParams d0;                              /* the shared model; grid fields come from Geo */
  bt::Geo* geo_d[2] = {nullptr, nullptr};    /* per block order */
  unsigned short* eob_d[2][bt::NSHAPE] = {};
  int nblocks[bt::NSHAPE] = {};
  bt::Ev* tab_d = nullptr;
  bt::Ev* tab_h = nullptr;                   /* pinned; copied in by each launch sequence */
  unsigned int* pre_d = nullptr;
  bt::Ctl* ctl_d = nullptr;
  DevFlags* flg_d = nullptr;
  DevFlags* flg_h = nullptr;                 /* pinned */
  DevFlags* flg2_d = nullptr;                /* the post-step flags of a LS_FULL sequence */
  DevFlags* flg2_h = nullptr;                /* pinned */
  bool speculate = true;                     /* LS_FULL where a post-step pass exists */
  struct Cand { int order, slow, fused; };   /* block order, deferred-pass blocks per SM, face pass in one launch */
  std::vector<Cand> cands;
  std::vector<double> cand_ms;
  int chosen = -1;
  int tuned_steps = 0;
  /* (sequence, integrator and boundary condition, candidate, precision, recovery, the learned guess's weights) */
  std::map<std::tuple<int, int, int, int, int, std::string>, std::pair<cudaGraphExec_t, int>> graphs;
  int64_t steps = 0, fallbacks = 0;
  double ms_step = 0.0, ms_post = 0.0;
};

constexpr int LS_TUNE_ROUNDS = 2;

int ls_destroy(Lockstep* L) {
  if (!L) return FIVO_OK;
  if (L->st) cudaStreamSynchronize(L->st);
  for (auto& g : L->graphs) cudaGraphExecDestroy(g.second.first);
  for (int o = 0; o < 2; ++o) {
    cudaFree(L->geo_d[o]);
    for (int s = 0; s < bt::NSHAPE; ++s) cudaFree(L->eob_d[o][s]);
  }
  cudaFree(L->tab_d); cudaFree(L->pre_d); cudaFree(L->ctl_d); cudaFree(L->flg_d); cudaFree(L->flg2_d);
  if (L->tab_h) cudaFreeHost(L->tab_h);
  if (L->flg_h) cudaFreeHost(L->flg_h);
  if (L->flg2_h) cudaFreeHost(L->flg2_h);
  if (L->done) cudaEventDestroy(L->done);
  if (L->ta) cudaEventDestroy(L->ta);
  if (L->tb) cudaEventDestroy(L->tb);
  if (L->st) cudaStreamDestroy(L->st);
  delete L;
  return FIVO_OK;
}

namespace {

/* the units of each launch shape for one event */
void ls_units(const DevParams& d, long long u[bt::NSHAPE]) {
  u[bt::SH_CELL] = d.Ntot;
  u[bt::SH_FRAME] = d.Ntot - (long long)d.Nx * d.Ny;
  u[bt::SH_FACEX] = 2LL * (d.Nxtot - 1) * d.Nytot;
  u[bt::SH_FACEY] = 2LL * d.Nxtot * (d.Nytot - 1);
  u[bt::SH_FACEXY] = u[bt::SH_FACEX] + u[bt::SH_FACEY];   /* (blocks: those of x plus those of y) */
  u[bt::SH_INT] = (long long)d.Nx * d.Ny;
}

int ls_create(fivo_batch* b, int flags, Lockstep** out) {
  const int n = (int)b->ev.size();
  if (n > 65535) return fail(FIVO_ERR_ARG, "fivo_batch_set_lockstep: at most 65535 events");
  Lockstep* L = new Lockstep();
  auto cleanup = [&](int code) { ls_destroy(L); return code; };
  L->flags = flags;
  L->nev = n;
  L->d0 = b->ev[0]->dp;
  L->nsm = b->ev[0]->nsm;
  if (cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&L->done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&L->ta) != cudaSuccess || cudaEventCreate(&L->tb) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_CUDA, "fivo_batch_set_lockstep: stream or event creation failed"));
  L->run_st = L->st;
  for (int order = 0; order < 2; ++order) {
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    if (order == 1)
      std::stable_sort(perm.begin(), perm.end(),
                       [&](int a, int c) { return b->ev[a]->dp.Ntot > b->ev[c]->dp.Ntot; });
    std::vector<bt::Geo> geo(n);
    std::vector<unsigned short> eob[bt::NSHAPE];
    long long cnt[bt::NSHAPE] = {0, 0, 0, 0, 0, 0};
    for (int e : perm) {
      const DevParams& d = b->ev[e]->dp;
      bt::Geo& g = geo[e];
      std::memset(&g, 0, sizeof(g));
      g.Nx = d.Nx; g.Ny = d.Ny; g.Nxtot = d.Nxtot; g.Nytot = d.Nytot; g.Ntot = d.Ntot;
      g.dx = d.dx; g.dy = d.dy; g.xmin = d.xmin; g.ymin = d.ymin;
      long long u[bt::NSHAPE];
      ls_units(d, u);
      g.nbx = (int)((u[bt::SH_FACEX] + 127) / 128);
      for (int s = 0; s < bt::NSHAPE; ++s) {
        const long long nb = s == bt::SH_FACEXY ? g.nbx + (u[bt::SH_FACEY] + 127) / 128 : (u[s] + 127) / 128;
        g.b0[s] = (int)cnt[s];
        eob[s].insert(eob[s].end(), (size_t)nb, (unsigned short)e);
        cnt[s] += nb;
      }
    }
    for (int s = 0; s < bt::NSHAPE; ++s) {
      if (cnt[s] >= 0x7fffffffLL) return cleanup(fail(FIVO_ERR_ARG, "fivo_batch_set_lockstep: batch too large"));
      L->nblocks[s] = (int)cnt[s];
      if (cudaMalloc(&L->eob_d[order][s], std::max<size_t>(1, eob[s].size()) * sizeof(unsigned short)) != cudaSuccess)
        return cleanup(fail(FIVO_ERR_NOMEM, "fivo_batch_set_lockstep: device allocation failed"));
      if (!eob[s].empty())
        CK(cudaMemcpy(L->eob_d[order][s], eob[s].data(), eob[s].size() * sizeof(unsigned short),
                      cudaMemcpyHostToDevice));
    }
    if (cudaMalloc(&L->geo_d[order], n * sizeof(bt::Geo)) != cudaSuccess)
      return cleanup(fail(FIVO_ERR_NOMEM, "fivo_batch_set_lockstep: device allocation failed"));
    CK(cudaMemcpy(L->geo_d[order], geo.data(), n * sizeof(bt::Geo), cudaMemcpyHostToDevice));
  }
  if (cudaMalloc(&L->tab_d, n * sizeof(bt::Ev)) != cudaSuccess ||
      cudaMalloc(&L->pre_d, (n + 1) * sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&L->ctl_d, sizeof(bt::Ctl)) != cudaSuccess ||
      cudaMalloc(&L->flg_d, n * sizeof(DevFlags)) != cudaSuccess ||
      cudaMalloc(&L->flg2_d, n * sizeof(DevFlags)) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_NOMEM, "fivo_batch_set_lockstep: device allocation failed"));
  if (cudaMallocHost(&L->tab_h, n * sizeof(bt::Ev)) != cudaSuccess ||
      cudaMallocHost(&L->flg_h, n * sizeof(DevFlags)) != cudaSuccess ||
      cudaMallocHost(&L->flg2_h, n * sizeof(DevFlags)) != cudaSuccess)
    return cleanup(fail(FIVO_ERR_NOMEM, "fivo_batch_set_lockstep: pinned allocation failed"));
  std::memset(L->tab_h, 0, n * sizeof(bt::Ev));
  for (int order = 0; order < 2; ++order)
    for (int slow : {2, 4})
      for (int fused = 0; fused < 2; ++fused) L->cands.push_back({order, slow, fused});
  L->cand_ms.assign(L->cands.size(), 0.0);
  /* untuned: batch order, 2 blocks per SM (the single-event deferred pass's grid), the
   * face directions in two launches (as the single-event path) */
  L->chosen = (flags & FIVO_LOCKSTEP_TUNE) ? -1 : 0;
  *out = L;
  return FIVO_OK;
}

/* the buffers of event c in its record (everything but the per-pass arguments) */
void ls_fill_common(fivo_ctx* c, bt::Ev& e) {
  const DevParams& d = c->dp;
  std::memset(&e, 0, sizeof(e));
  e.w = c->w; e.h = c->h; e.fl = c->fl;
  e.qp = c->queues; e.qa = c->queues + d.Ntot; e.qq = c->queues + 2 * d.Ntot;
  e.fhx = c->fh; e.fhy = c->fh + (size_t)d.nv * d.Ntot;
  e.fhx32 = c->fh32; e.fhy32 = c->fh32 ? c->fh32 + (size_t)d.nv * d.Ntot : nullptr;
  e.x0save = c->x0save;
  e.hsave = c->hsave;
}

/* the optimistic step of step2/step3 on the context's current roles */
void ls_fill_step(fivo_ctx* c, bt::Ev& e, int integrator, double tau, double D, bool snap) {
  ls_fill_common(c, e);
  e.active = 1;
  e.snap = snap ? 1 : 0;
  const int U = c->iU, U1 = c->iU1, U2 = c->iU2, T = c->iT;
  e.cp_dst = c->S[U2]; e.cp_src = c->S[U];
  auto stage = [&](int k, int ub, int uo, double t, double ts, double wold, double wnew, int mode) {
    StageArgs& a = e.st[k];
    a.Ub = c->S[ub]; a.Uold = c->S[U2]; a.Uout = c->S[uo]; a.w = c->w; a.ffo = nullptr; a.bad = c->masks;
    a.dU = nullptr; a.tau = t; a.tau_state = ts; a.dt = D; a.wold = wold; a.wnew = wnew; a.mode = mode;
    a.fl = c->fl;
    e.pU[k] = c->S[ub];
    e.ptau[k] = t;
  };
  if (integrator == FIVO_SSPRK3) {
    stage(0, U, U1, tau, tau + D, 1.0, 0.0, COMB_EULER);
    stage(1, U1, T, tau + D, tau + D, 0.75, 0.25, COMB_BLEND);
    /* step3 swaps U1 and T here: the third stage reads the second's output */
    stage(2, T, U1, tau + (0.5 * D), tau + D, 0.0, 0.0, COMB_THIRD);
  } else {
    stage(0, U, U1, tau, tau + D, 1.0, 0.0, COMB_EULER);
    stage(1, U1, T, tau + D, tau + D, 0.5, 0.5, COMB_BLEND);
  }
}

/* the post-step pass's arguments: update_prims + relax_project on state buffer u
 * (scratch buffer t) at time tau after a step of length used */
void ls_set_post(fivo_ctx* c, bt::Ev& e, int u, int t, double tau, double used, int do_relax, int do_project) {
  e.pU[3] = c->S[u];
  e.ptau[3] = tau;
  e.rq = c->S[u]; e.ro = c->S[t];
  e.rtau = tau; e.rD = used;
  e.do_relax = do_relax; e.do_project = do_project;
}

/* update_prims + relax_project after an accepted step (state U at time tau) */
void ls_fill_post(fivo_ctx* c, bt::Ev& e, double tau, double used, int do_relax, int do_project) {
  ls_fill_common(c, e);
  e.active = 1;
  ls_set_post(c, e, c->iU, c->iT, tau, used, do_relax, do_project);
}

/* the post-step pass in the step's own sequence, on the roles the step takes when it
 * is accepted (step3: U <- U1, T <- U; step2: U <- T, T <- U) */
void ls_fill_spec(fivo_ctx* c, bt::Ev& e, int integrator, double tau_post, double used, int do_relax,
                  int do_project) {
  e.spec = 1;
  ls_set_post(c, e, integrator == FIVO_SSPRK3 ? c->iU1 : c->iT, c->iU, tau_post, used, do_relax, do_project);
}

/* the history planes the post-step pass overwrote, back from the copies taken
 * before the step (an undone speculative step) */
int restore_hist(fivo_ctx* c) {
  const size_t N = (size_t)c->dp.Ntot;
  CK(cudaMemcpyAsync(c->h.ux_prev, c->hsave, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemcpyAsync(c->h.nux_prev, c->hsave + 2 * N, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  return FIVO_OK;
}

#define LS_GRID(s) L.nblocks[s] ? L.nblocks[s] : 1
#define LS_K() \
  do {         \
    CKL();     \
    ++nk;      \
  } while (0)
constexpr int LS_LEARNED_DYN = LEARNED_SMEM - (int)sizeof(guess::FwdSmem) - 1024;
constexpr int LS_RETRY_DYN = LEARNED_SMEM - (int)sizeof(guess::FwdSmem) - 128;

/* enqueue one launch sequence on L.run_st (recorded into a graph or run directly) */
template <int EOS, bool NCH>
int ls_launch_t(fivo_batch* b, int seq, int integrator, int bc, int cand, int prec, bool any_sector, bool relax_on) {
  Lockstep& L = *b->ls;
  const int n = L.nev;
  const int order = L.cands[cand].order;
  const unsigned slow_blocks = (unsigned)(L.cands[cand].slow * L.nsm);
  const bool fused = L.cands[cand].fused != 0;
  const bt::Geo* geo = L.geo_d[order];
  unsigned short* const* eob = L.eob_d[order];
  const DevParams& d0 = L.d0;
  cudaStream_t st = L.run_st;
  const bool f32 = prec != FIVO_PRECISION_FP64;
  const unsigned gr = nblk(n, 256);
  int nk = 0;   /* kernels of this sequence */
  CK(cudaMemcpyAsync(L.tab_d, L.tab_h, n * sizeof(bt::Ev), cudaMemcpyHostToDevice, st));
  /* _primitive_pass!: as launch_primitive_t, with or without the learned guess */
  const fivo_ctx* c0 = b->ev[0];
  auto prim_pass = [&](int which) -> int {
    if (c0->learned && c0->guess_mode == FIVO_GUESS_EVERY_CELL) {
      bt::kb_prim_learned<EOS, NCH><<<LS_GRID(bt::SH_CELL), 128, LS_LEARNED_DYN, st>>>(d0, geo, L.tab_d,
                                                                                     eob[bt::SH_CELL], which, c0->gnet);
      LS_K();
    } else {
      bt::kb_prim_fast<EOS, NCH><<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_CELL], which);
      LS_K();
    }
    int left = 0;
    if (c0->learned && c0->guess_mode == FIVO_GUESS_DEFERRED) {
      /* the network's guess for the deferred cells of every event, then the full
       * recovery of what it leaves */
      bt::kb_scan<<<1, 1024, 0, st>>>(L.tab_d, n, 3, L.pre_d, L.ctl_d);
      LS_K();
      bt::kb_prim_learned_retry<EOS, NCH><<<LS_GRID(bt::SH_CELL), 128, LS_RETRY_DYN, st>>>(
          d0, geo, L.tab_d, L.pre_d, n, L.ctl_d, which, c0->gnet);
      LS_K();
      left = 1;
    }
    bt::kb_scan<<<1, 1024, 0, st>>>(L.tab_d, n, left ? 2 : 0, L.pre_d, L.ctl_d);
    LS_K();
    bt::kb_prim_slow<EOS, NCH><<<slow_blocks, 128, 0, st>>>(d0, geo, L.tab_d, L.pre_d, n, L.ctl_d, which, left);
    LS_K();
    return FIVO_OK;
  };
  auto gather = [&](DevFlags* dev, DevFlags* host) -> int {
    bt::kb_gather_flags<<<nblk((long long)n * (sizeof(DevFlags) / 8), 256), 256, 0, st>>>(L.tab_d, n, dev);
    LS_K();
    CK(cudaMemcpyAsync(host, dev, n * sizeof(DevFlags), cudaMemcpyDeviceToHost, st));
    return FIVO_OK;
  };
  int rc;
  if (seq == LS_STEP || seq == LS_FULL) {
    bt::kb_pre_step<<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_CELL]);
    LS_K();
    const int nst = integrator == FIVO_SSPRK3 ? 3 : 2;
    const bool full = d0.hasNu && d0.hasPi && d0.hasShear;
    for (int k = 0; k < nst; ++k) {
      if (k == 0) {
        bt::kb_bc<<<LS_GRID(bt::SH_FRAME), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FRAME], 0, bc);
        LS_K();
      }
      bt::kb_reset<<<gr, 256, 0, st>>>(L.tab_d, n, k == 0 ? (1 | 2 | 64) : (1 | 2));
      LS_K();
      if ((rc = prim_pass(k))) return rc;
      if (fused) {
        if (f32) bt::kb_faces_xy<EOS, true><<<LS_GRID(bt::SH_FACEXY), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEXY], k);
        else bt::kb_faces_xy<EOS, false><<<LS_GRID(bt::SH_FACEXY), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEXY], k);
        LS_K();
      }
      if (f32) {
        if (!fused) {
          bt::kb_faces<EOS, true, true><<<LS_GRID(bt::SH_FACEX), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEX], k);
          LS_K();
          bt::kb_faces<EOS, false, true><<<LS_GRID(bt::SH_FACEY), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEY], k);
          LS_K();
        }
        if (full) bt::kb_update<EOS, NCH, float, true><<<LS_GRID(bt::SH_INT), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_INT], k);
        else bt::kb_update<EOS, NCH, float, false><<<LS_GRID(bt::SH_INT), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_INT], k);
        LS_K();
      } else {
        if (!fused) {
          bt::kb_faces<EOS, true, false><<<LS_GRID(bt::SH_FACEX), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEX], k);
          LS_K();
          bt::kb_faces<EOS, false, false><<<LS_GRID(bt::SH_FACEY), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FACEY], k);
          LS_K();
        }
        if (full) bt::kb_update<EOS, NCH, double, true><<<LS_GRID(bt::SH_INT), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_INT], k);
        else bt::kb_update<EOS, NCH, double, false><<<LS_GRID(bt::SH_INT), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_INT], k);
        LS_K();
      }
      bt::kb_scan<<<1, 1024, 0, st>>>(L.tab_d, n, 1, L.pre_d, L.ctl_d);
      LS_K();
      bt::kb_adm_slow<EOS, NCH><<<(unsigned)L.nsm, 128, 0, st>>>(d0, geo, L.tab_d, L.pre_d, n, L.ctl_d, k);
      LS_K();
      bt::kb_bc<<<LS_GRID(bt::SH_FRAME), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_FRAME], k + 1, bc);
      LS_K();
    }
    /* the step's flags, before the post-step pass resets them */
    if (seq == LS_FULL && (rc = gather(L.flg_d, L.flg_h))) return rc;
  }
  if (seq == LS_POST || seq == LS_FULL) {
    if (any_sector) {
      bt::kb_reset<<<gr, 256, 0, st>>>(L.tab_d, n, 1 | 64);
      LS_K();
      if ((rc = prim_pass(3))) return rc;
    }
    if (relax_on) {
      bt::kb_reset<<<gr, 256, 0, st>>>(L.tab_d, n, 4);
      LS_K();
      if (prec == FIVO_PRECISION_FP32 && any_sector)
        bt::kb_relax<EOS, false, true><<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_CELL]);
      else if (d0.hasM2)
        bt::kb_relax<EOS, true, false><<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_CELL]);
      else
        bt::kb_relax<EOS, false, false><<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(d0, geo, L.tab_d, eob[bt::SH_CELL]);
      LS_K();
      bt::kb_post_hist<<<LS_GRID(bt::SH_CELL), 128, 0, st>>>(geo, L.tab_d, eob[bt::SH_CELL]);
      LS_K();
    }
  }
  if (seq == LS_FULL) rc = gather(L.flg2_d, L.flg2_h);
  else rc = gather(L.flg_d, L.flg_h);
  if (rc) return rc;
  L.last_nk = nk;
  return FIVO_OK;
}

/* dynamic shared memory of the learned kernels: with their static part, at most 4 CTAs
 * per SM (4 x 128 tensor-memory columns), as the single-event launches reserve */
template <int EOS, bool NCH>
int ls_prepare_t() {
  CK(cudaFuncSetAttribute(bt::kb_prim_learned<EOS, NCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, LS_LEARNED_DYN));
  CK(cudaFuncSetAttribute(bt::kb_prim_learned_retry<EOS, NCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          LS_RETRY_DYN));
  return FIVO_OK;
}

int ls_prepare(const DevParams& d) {
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG) return ls_prepare_t<FIVO_EOS_LATTICE_HRG, true>();
  if (d.ncharge) return ls_prepare_t<FIVO_EOS_CONFORMAL_HQ, true>();
  return ls_prepare_t<FIVO_EOS_CONFORMAL_HQ, false>();
}

int ls_launch(fivo_batch* b, int seq, int integrator, int bc, int cand, int prec, bool any_sector, bool relax_on) {
  const DevParams& d = b->ls->d0;
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG)
    return ls_launch_t<FIVO_EOS_LATTICE_HRG, true>(b, seq, integrator, bc, cand, prec, any_sector, relax_on);
  if (d.ncharge) return ls_launch_t<FIVO_EOS_CONFORMAL_HQ, true>(b, seq, integrator, bc, cand, prec, any_sector, relax_on);
  return ls_launch_t<FIVO_EOS_CONFORMAL_HQ, false>(b, seq, integrator, bc, cand, prec, any_sector, relax_on);
}

/* run one launch sequence (replaying its graph when graphs are on) and wait for it */
int ls_exec(fivo_batch* b, int seq, int integrator, int bc, int cand, int prec, bool any_sector, bool relax_on,
            float* ms) {
  Lockstep& L = *b->ls;
  if (!L.prepared) {
    const int rc0 = ls_prepare(L.d0);
    if (rc0) return rc0;
    L.prepared = true;
  }
  CK(cudaEventRecord(L.ta, L.run_st));
  if (L.flags & FIVO_LOCKSTEP_GRAPHS) {
    const fivo_ctx* c0 = b->ev[0];
    /* the guess's weights and normalisation are kernel arguments: a graph per attached network */
    const std::string net = c0->learned ? std::string((const char*)&c0->gnet, sizeof(c0->gnet)) : std::string();
    const auto key = std::make_tuple(seq, integrator * 16 + bc, cand, prec, c0->learned ? 1 + c0->guess_mode : 0, net);
    auto it = L.graphs.find(key);
    if (it == L.graphs.end()) {
      CK(cudaStreamBeginCapture(L.run_st, cudaStreamCaptureModeThreadLocal));
      const int rc = ls_launch(b, seq, integrator, bc, cand, prec, any_sector, relax_on);
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(L.run_st, &g);
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (ec != cudaSuccess) return fail(FIVO_ERR_CUDA, std::string("lockstep graph capture: ") + cudaGetErrorString(ec));
      cudaGraphExec_t x = nullptr;
      const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) return fail(FIVO_ERR_CUDA, std::string("lockstep graph instantiation: ") + cudaGetErrorString(ei));
      it = L.graphs.emplace(key, std::make_pair(x, L.last_nk)).first;
    }
    CK(cudaGraphLaunch(it->second.first, L.run_st));
    L.kernels += it->second.second;
  } else {
    const int rc = ls_launch(b, seq, integrator, bc, cand, prec, any_sector, relax_on);
    if (rc) return rc;
    L.kernels += L.last_nk;
  }
  CK(cudaEventRecord(L.tb, L.run_st));
  CK(cudaEventRecord(L.done, L.run_st));
  CK(cudaEventSynchronize(L.done));
  CK(cudaEventElapsedTime(ms, L.ta, L.tb));
  return FIVO_OK;
}

/* fn(k) for the listed events on the batch's worker threads (a thread that cannot
 * select the device still runs fn: its CUDA calls then fail into the event's status) */
template <class F>
void ls_parallel(fivo_batch* b, const std::vector<int>& ks, F fn) {
  std::atomic<int> next{0};
  auto worker = [&]() {
    cudaSetDevice(b->device);
    for (;;) {
      const int j = next.fetch_add(1);
      if (j >= (int)ks.size()) break;
      fn(ks[j]);
    }
  };
  const int nw = std::min<int>(b->nworkers, (int)ks.size());
  std::vector<std::thread> pool;
  for (int t = 1; t < nw; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
}

/* advance_loop (run_sim_2d!'s while loop, main2D.jl:436-513) for every event of
 * the batch in lockstep; tau[k] is event k's time, advanced in place */
int ls_loop(fivo_batch* b, std::vector<double>& tau, double taufinal, double cfl, double cfltau, int integrator,
            int bc, int64_t max_steps, fivo_run_result* out, std::vector<int>& st, std::vector<std::string>& msg) {
  Lockstep& L = *b->ls;
  const int n = L.nev;
  const DevParams& d = L.d0;
  const fivo_params& p = d.p;
  const bool any_sector = p.enable_shear || p.enable_bulk || p.enable_diff;
  const bool relax_on = d.nv > 4 && (any_sector || d.hasShear);
  const bool post = any_sector || d.hasShear;
  const int prec = b->ev[0]->precision;
  const fivo_ctx* c0 = b->ev[0];
  /* the post-step pass speculates in the step's sequence (one host read per step) */
  const bool spec = L.speculate && post;
  const int do_relax = any_sector ? 1 : 0, do_project = any_sector ? d.hasShear : 1;
  for (fivo_ctx* c : b->ev) {
    if (c->learned != c0->learned || (c->learned && (c->guess_mode != c0->guess_mode || c->gnet.img != c0->gnet.img)))
      return fail(FIVO_ERR_CONFIG, "lockstep batch: every event must use the same recovery (one learned guess, one mode, or none)");
    if (c->precision != prec) return fail(FIVO_ERR_CONFIG, "lockstep batch: every event must use the same precision");
    if (!c->x0save) {
      if (cudaMalloc(&c->x0save, 4 * (size_t)c->dp.Ntot * sizeof(double)) != cudaSuccess) {
        c->x0save = nullptr;
        return fail(FIVO_ERR_NOMEM, "device allocation failed");
      }
    }
    if (spec && !c->hsave) {
      if (cudaMalloc(&c->hsave, 4 * (size_t)c->dp.Ntot * sizeof(double)) != cudaSuccess) {
        c->hsave = nullptr;
        return fail(FIVO_ERR_NOMEM, "device allocation failed");
      }
    }
    /* the sequences' stream reads what the contexts' streams wrote (one host thread
     * waits here, so it spins rather than sleeps as the batch workers do) */
    CK(cudaStreamSynchronize(c->st));
    prof_flush(c);
  }
  std::vector<char> done(n, 0), stepped(n, 0), posted(n, 0);
  std::vector<double> D(n, 0.0), used(n, 0.0), msr(n, 0.0);
  std::vector<int64_t> nsteps(n, 0), npf(n, 0), nvac(n, 0);
  for (int k = 0; k < n; ++k) out[k].ok = 1;
  while (true) {
    int nact = 0;
    for (int k = 0; k < n; ++k) {
      fivo_ctx* c = b->ev[k];
      bt::Ev& e = L.tab_h[k];
      e.active = 0;
      stepped[k] = 0;
      posted[k] = 0;
      if (done[k] || st[k] != FIVO_OK) continue;
      if (!(tau[k] < taufinal && nsteps[k] < max_steps)) { done[k] = 1; continue; }
      double Dk;
      fivo_compute_dt(c, tau[k], cfl, cfltau, &Dk);
      Dk = jmin(Dk, taufinal - tau[k]);
      if (Dk <= 0) { done[k] = 1; continue; }
      const bool snap = c->hist_valid || c->nsteps_run > 0;
      if (snap) c->hist_valid = true;
      c->cnt.nmood = 0; c->cnt.nhalve = 0;
      ls_fill_step(c, e, integrator, tau[k], Dk, snap);
      if (spec) ls_fill_spec(c, e, integrator, tau[k] + Dk, Dk, do_relax, do_project);
      D[k] = Dk;
      ++nact;
    }
    if (!nact) break;
    /* the schedule: the chosen candidate, or the next one to time */
    int cand = L.chosen;
    const bool tuning = cand < 0;
    if (tuning) cand = L.tuned_steps % (int)L.cands.size();
    float ms = 0.f;
    int rc = ls_exec(b, spec ? LS_FULL : LS_STEP, integrator, bc, cand, prec, any_sector, relax_on, &ms);
    if (rc) return rc;
    L.ms_step += ms;
    L.steps += 1;
    if (tuning) {
      double& best = L.cand_ms[cand];
      if (best == 0.0 || ms < best) best = ms;
      if (++L.tuned_steps >= LS_TUNE_ROUNDS * (int)L.cands.size())
        L.chosen = (int)(std::min_element(L.cand_ms.begin(), L.cand_ms.end()) - L.cand_ms.begin());
    }
    std::vector<int> redo;
    for (int k = 0; k < n; ++k) {
      if (!L.tab_h[k].active) continue;
      fivo_ctx* c = b->ev[k];
      *c->flh = L.flg_h[k];
      if ((rc = parse_flags(c, true))) { st[k] = rc; msg[k] = g_err; continue; }
      const long long nbad = c->flh->nbad;
      if (integrator == FIVO_SSPRK3) { std::swap(c->iU1, c->iT); std::swap(c->iU, c->iT); }
      if (nbad == 0) {
        if (integrator != FIVO_SSPRK3) std::swap(c->iU, c->iT);
        used[k] = D[k];
        stepped[k] = 1;
        posted[k] = spec ? 1 : 0;
      } else {
        if (integrator == FIVO_SSPRK3) std::swap(c->iU, c->iU2);   /* the state before the step */
        redo.push_back(k);
      }
    }
    /* events whose optimistic step found an inadmissible cell: the rest of step2/step3 */
    if (!redo.empty()) {
      L.fallbacks += (int64_t)redo.size();
      ls_parallel(b, redo, [&](int k) {
        fivo_ctx* c = b->ev[k];
        int ok = 0, r = restore_warm(c);
        /* a speculative post-step pass also wrote the history planes and, for step2,
         * the relaxed rows into U itself (its scratch role); U2 holds U's copy */
        if (!r && spec) r = restore_hist(c);
        if (!r && spec && integrator != FIVO_SSPRK3) r = copy_state(c, c->iU, c->iU2);
        if (!r) {
          r = integrator == FIVO_SSPRK3 ? step3_rest(c, tau[k], D[k], 12, bc, &used[k], &ok)
                                        : step2_rest(c, tau[k], D[k], 12, 2, bc, &used[k], &ok);
        }
        if (!r && ctx_sync(c) != cudaSuccess) r = fail(FIVO_ERR_CUDA, "lockstep batch: stream synchronisation failed");
        if (r) { st[k] = r; msg[k] = g_err; return; }
        if (!ok) { out[k].ok = 0; done[k] = 1; return; }
        stepped[k] = 1;
      });
    }
    int npost = 0;
    for (int k = 0; k < n; ++k) {
      L.tab_h[k].active = 0;
      if (!stepped[k]) continue;
      fivo_ctx* c = b->ev[k];
      tau[k] += used[k];
      nsteps[k] += 1;
      c->nsteps_run += 1;
      if (post && !posted[k]) {
        ls_fill_post(c, L.tab_h[k], tau[k], used[k], do_relax, do_project);
        ++npost;
      }
    }
    if (npost) {
      if ((rc = ls_exec(b, LS_POST, integrator, bc, L.chosen < 0 ? 0 : L.chosen, prec, any_sector, relax_on, &ms)))
        return rc;
      L.ms_post += ms;
    }
    for (int k = 0; k < n; ++k) {
      if (!stepped[k]) continue;
      fivo_ctx* c = b->ev[k];
      if (post) {
        if (relax_on)   /* relax_project: U's dissipative planes are now the scratch state's */
          for (int a = 4; a < d.nv; ++a) std::swap(c->S[c->iU].f[a], c->S[c->iT].f[a]);
        *c->flh = posted[k] ? L.flg2_h[k] : L.flg_h[k];
        if (any_sector && (rc = parse_flags(c, false))) { st[k] = rc; msg[k] = g_err; continue; }
        if (d.hasShear) {
          uint64_t bits = c->flh->shear_max_bits;
          double r;
          std::memcpy(&r, &bits, 8);
          msr[k] = jmax(msr[k], r);
        }
      }
      npf[k] += c->cnt.nprimfail;
      nvac[k] += c->cnt.nvacuum;
    }
  }
  for (int k = 0; k < n; ++k) {
    out[k].tau = tau[k]; out[k].nsteps = nsteps[k]; out[k].nprimfail = npf[k]; out[k].nvacuum = nvac[k];
    out[k].max_shear_res = msr[k];
  }
  return FIVO_OK;
}

/* per-event statuses and messages of a lockstep call into the batch's convention */
int ls_status(const std::vector<int>& st, const std::vector<std::string>& msg, int* status) {
  int first = -1;
  for (size_t k = 0; k < st.size(); ++k) {
    if (status) status[k] = st[k];
    if (st[k] != FIVO_OK && first < 0) first = (int)k;
  }
  if (first >= 0) return fail(st[first], "event " + std::to_string(first) + ": " + msg[first]);
  return FIVO_OK;
}

void ls_info(const Lockstep& L, bool enabled, fivo_lockstep_info* out) {
  out->enabled = enabled ? 1 : 0;
  out->flags = L.flags;
  out->ncand = std::min<int>((int)L.cands.size(), FIVO_LOCKSTEP_MAXCAND);
  out->chosen = L.chosen;
  for (int i = 0; i < out->ncand; ++i) {
    out->cand_order[i] = L.cands[i].order;
    out->cand_slow[i] = L.cands[i].slow;
    out->cand_fused[i] = L.cands[i].fused;
    out->cand_ms[i] = L.cand_ms[i];
  }
  out->steps = L.steps;
  out->fallbacks = L.fallbacks;
  out->ms_step = L.ms_step;
  out->ms_post = L.ms_post;
  out->kernels = L.kernels;
}
}  // namespace

int fivo_batch_set_lockstep(fivo_batch* b, int enable, int flags) {
  if (!b) return fail(FIVO_ERR_ARG, "null argument");
  if (flags & ~(FIVO_LOCKSTEP_GRAPHS | FIVO_LOCKSTEP_TUNE)) return fail(FIVO_ERR_ARG, "fivo_batch_set_lockstep: unknown flags");
  if (!enable) { b->lockstep = false; return FIVO_OK; }
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(FIVO_ERR_CUDA, "cudaSetDevice failed");
  if (b->ls && b->ls->flags != flags) { ls_destroy(b->ls); b->ls = nullptr; }
  if (!b->ls) {
    int rc = ls_create(b, flags, &b->ls);
    if (rc) { b->ls = nullptr; return rc; }
  }
  b->lockstep = true;
  return FIVO_OK;
}

int fivo_batch_lockstep_info(fivo_batch* b, fivo_lockstep_info* out) {
  if (!b || !out) return fail(FIVO_ERR_ARG, "null argument");
  std::memset(out, 0, sizeof(*out));
  out->enabled = b->lockstep ? 1 : 0;
  out->chosen = -1;
  if (!b->ls) return FIVO_OK;
  ls_info(*b->ls, b->lockstep, out);
  return FIVO_OK;
}

int fivo_batch_run(fivo_batch* b, double tau0, double taufinal, double cfl, double cfltau, int integrator, int bc,
                   int64_t max_steps, int reset_hist, fivo_run_result* results, int* status) {
  if (!b || !results) return fail(FIVO_ERR_ARG, "null argument");
  if (integrator != FIVO_SSPRK2 && integrator != FIVO_SSPRK3)
    return fail(FIVO_ERR_ARG, "integrator must be FIVO_SSPRK2 or FIVO_SSPRK3");
  if (b->lockstep) {
    const int n = (int)b->ev.size();
    std::vector<double> Qin(n, 0.0), tau(n, tau0);
    int rc = batch_for_each(b, status, [&](int k) {
      std::memset(&results[k], 0, sizeof(results[k]));
      return run_begin(b->ev[k], tau0, bc, reset_hist, &Qin[k]);
    });
    if (rc) return rc;
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(FIVO_ERR_CUDA, "cudaSetDevice failed");
    std::vector<int> st(n, FIVO_OK);
    std::vector<std::string> msg(n);
    if ((rc = ls_loop(b, tau, taufinal, cfl, cfltau, integrator, bc, max_steps, results, st, msg))) return rc;
    if ((rc = ls_status(st, msg, status))) return rc;
    return batch_for_each(b, status, [&](int k) { return run_end(b->ev[k], Qin[k], &results[k]); });
  }
  return batch_for_each(b, status, [&](int k) {
    return fivo_run(b->ev[k], tau0, taufinal, cfl, cfltau, integrator, bc, max_steps, reset_hist, &results[k]);
  });
}

int fivo_batch_advance(fivo_batch* b, const double* tau, double taufinal, double cfl, double cfltau, int integrator,
                       int bc, int64_t max_steps, fivo_run_result* results, int* status) {
  if (!b || !tau || !results) return fail(FIVO_ERR_ARG, "null argument");
  if (integrator != FIVO_SSPRK2 && integrator != FIVO_SSPRK3)
    return fail(FIVO_ERR_ARG, "integrator must be FIVO_SSPRK2 or FIVO_SSPRK3");
  if (b->lockstep) {
    const int n = (int)b->ev.size();
    std::vector<double> t(tau, tau + n);
    for (int k = 0; k < n; ++k) std::memset(&results[k], 0, sizeof(results[k]));
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(FIVO_ERR_CUDA, "cudaSetDevice failed");
    std::vector<int> st(n, FIVO_OK);
    std::vector<std::string> msg(n);
    int rc = ls_loop(b, t, taufinal, cfl, cfltau, integrator, bc, max_steps, results, st, msg);
    if (rc) return rc;
    return ls_status(st, msg, status);
  }
  return batch_for_each(b, status, [&](int k) {
    return fivo_advance(b->ev[k], tau[k], taufinal, cfl, cfltau, integrator, bc, max_steps, &results[k]);
  });
}

/* ------------------------------------------------------------------------
 * One context through the lockstep launch sequences (fivo_ctx_set_graphs): a
 * batch of this one context, whose STEP and POST sequences run on the context's
 * stream as captured CUDA graphs (two graph launches and two host reads per
 * step instead of ~32 launches), with the lockstep's default schedule. The
 * kernels and their inputs are those of the single-context path, so results are
 * the same bits; the face pass is the global-load one.
 * ---------------------------------------------------------------------- */
void solo_destroy(fivo_batch* b) {
  if (!b) return;
  ls_destroy(b->ls);
  delete b;   /* the batch does not own its one context */
}

int solo_advance(fivo_ctx* c, double tau, double taufinal, double cfl, double cfltau, int integrator, int bc,
                 int64_t max_steps, fivo_run_result* out) {
  const int want = c->graphs == 2 ? 0 : FIVO_LOCKSTEP_GRAPHS;
  if (c->solo && c->solo->ls->flags != want) {
    solo_destroy(c->solo);
    c->solo = nullptr;
  }
  if (!c->solo) {
    fivo_batch* b = new fivo_batch();
    b->ev.push_back(c);
    b->nworkers = 1;
    b->device = c->device;
    int rc = ls_create(b, want, &b->ls);
    if (rc) { b->ls = nullptr; delete b; return rc; }
    b->lockstep = true;
    c->solo = b;
  }
  fivo_batch* b = c->solo;
  b->ls->run_st = c->st;   /* the caller's stream (fivo_ctx_set_stream) orders the work */
  std::vector<double> t(1, tau);
  std::vector<int> st(1, FIVO_OK);
  std::vector<std::string> msg(1);
  int rc = ls_loop(b, t, taufinal, cfl, cfltau, integrator, bc, max_steps, out, st, msg);
  if (rc) return rc;
  if (st[0] != FIVO_OK) return fail(st[0], msg[0]);
  return FIVO_OK;
}

int fivo_ctx_set_graphs(fivo_ctx* c, int mode) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (mode < 0 || mode > 2) return fail(FIVO_ERR_ARG, "fivo_ctx_set_graphs: mode must be 0, 1 or 2");
  c->graphs = mode;
  return FIVO_OK;
}


int fivo_ctx_lockstep_info(fivo_ctx* c, fivo_lockstep_info* out) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  std::memset(out, 0, sizeof(*out));
  out->enabled = c->graphs ? 1 : 0;
  out->chosen = -1;
  if (c->solo) ls_info(*c->solo->ls, c->graphs != 0, out);
  return FIVO_OK;
}

/* ------------------------------------------------ the learned recovery guess */

struct fivo_guess {
  int device = 0;
  cudaStream_t st = nullptr;
  float* params = nullptr;          /* NPARAM FP32 master weights */
  float* adam = nullptr;            /* m | v */
  uint8_t* img = nullptr;           /* BF16 operand images */
  guess::Norm norm{};
  int64_t adam_t = 0;
  float* samples = nullptr;         /* the sample store, cap x NSAMP floats */
  int64_t cap = 0;
  unsigned long long* count = nullptr;
  float* part = nullptr;            /* per-CTA partial gradients of a step */
  int part_ctas = 0;
  float* loss_part = nullptr;
  float* grad = nullptr;
  int* err = nullptr;
};

namespace {

guess::Net net_of(const fivo_guess* g) { return guess::Net{g->img, g->params, g->norm}; }

int guess_pack(fivo_guess* g) {
  guess::k_pack<<<(guess::PACK_ELEMS + 255) / 256, 256, 0, g->st>>>(g->params, g->img);
  CKL();
  return FIVO_OK;
}

int guess_parts(fivo_guess* g, int ctas) {
  if (ctas <= g->part_ctas) return FIVO_OK;
  cudaFree(g->part); cudaFree(g->loss_part);
  g->part = nullptr; g->loss_part = nullptr; g->part_ctas = 0;
  CK(cudaMalloc(&g->part, (size_t)ctas * guess::NPARAM * sizeof(float)));
  CK(cudaMalloc(&g->loss_part, (size_t)ctas * sizeof(float)));
  g->part_ctas = ctas;
  return FIVO_OK;
}

/* one forward + backward over ctas x 128 samples, the partials summed by k_adam
 * (lr = 0: the summed gradient only, into grad_out) */
int guess_step(fivo_guess* g, const float* smp, long long n, unsigned long long seed, int ctas, float lr,
               float* grad_out) {
  int rc = guess_parts(g, ctas);
  if (rc) return rc;
  CK(cudaFuncSetAttribute(guess::k_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)sizeof(guess::TrainSmem)));
  guess::k_train<<<ctas, 128, sizeof(guess::TrainSmem), g->st>>>(net_of(g), smp, n, seed, 0,
                                                                 1.0f / (128.0f * (float)ctas), g->part,
                                                                 g->loss_part, g->err);
  CKL();
  float c1 = 1.0f, c2 = 1.0f;
  if (lr != 0.0f) {
    g->adam_t += 1;
    c1 = 1.0f - std::pow(0.9f, (float)g->adam_t);
    c2 = 1.0f - std::pow(0.999f, (float)g->adam_t);
  }
  guess::k_adam<<<(guess::NPARAM + 255) / 256, 256, 0, g->st>>>(g->params, g->adam, g->adam + guess::NPARAM,
                                                               g->part, ctas, lr, 0.9f, 0.999f, 1e-8f, c1, c2,
                                                               grad_out);
  CKL();
  if (lr != 0.0f) return guess_pack(g);
  return FIVO_OK;
}

int guess_loss(fivo_guess* g, int ctas, double* loss) {
  std::vector<float> lp(ctas);
  CK(cudaMemcpyAsync(lp.data(), g->loss_part, ctas * sizeof(float), cudaMemcpyDeviceToHost, g->st));
  CK(cudaStreamSynchronize(g->st));
  int e = 0;
  CK(cudaMemcpy(&e, g->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(FIVO_ERR_DEVICE, "guess training: a tensor-core wait gave up");
  double s = 0.0;
  for (int b = 0; b < ctas; ++b) s += lp[b];
  *loss = s / (128.0 * ctas);
  return FIVO_OK;
}

}  // namespace

int fivo_guess_create(fivo_ctx* c, uint64_t seed, fivo_guess** out) {
  if (!out) return fail(FIVO_ERR_ARG, "null argument");
  *out = nullptr;
  fivo_guess* g = new fivo_guess();
  g->device = c ? c->device : 0;
  if (!c) cudaGetDevice(&g->device);
  auto bad = [&](int rc) { fivo_guess_destroy(g); return rc; };
  if (cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&g->params, guess::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&g->adam, 2 * guess::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&g->img, guess::IMG_BYTES) != cudaSuccess || cudaMalloc(&g->err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&g->count, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&g->grad, guess::NPARAM * sizeof(float)) != cudaSuccess)
    return bad(fail(FIVO_ERR_NOMEM, "fivo_guess_create: device allocation failed"));
  if (cudaMemset(g->count, 0, sizeof(unsigned long long)) != cudaSuccess)
    return bad(fail(FIVO_ERR_CUDA, "fivo_guess_create: memset failed"));
  /* uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights from a splitmix64 stream, zero biases */
  std::vector<float> P(guess::NPARAM, 0.0f);
  uint64_t st = seed;
  auto uni = [&]() { st += 1; return (double)(guess::mix64(st) >> 11) * (1.0 / 9007199254740992.0); };
  for (int j = 0; j < guess::NH; ++j)
    for (int k = 0; k < guess::NIN; ++k) P[guess::P_W1 + j * guess::K0 + k] = (float)((2 * uni() - 1) / std::sqrt(8.0));
  for (int j = 0; j < guess::NH; ++j)
    for (int k = 0; k < guess::NH; ++k) P[guess::P_W2 + j * guess::NH + k] = (float)((2 * uni() - 1) / 8.0);
  for (int o = 0; o < guess::NOUT; ++o)
    for (int k = 0; k < guess::NH; ++k) P[guess::P_W3 + o * guess::NH + k] = (float)((2 * uni() - 1) / 8.0);
  float nm[FIVO_GUESS_NNORM];
  for (int q = 0; q < 8; ++q) { nm[q] = 0.0f; nm[8 + q] = 1.0f; }
  for (int o = 0; o < 3; ++o) { nm[16 + o] = 0.0f; nm[19 + o] = 1.0f; }
  int rc = fivo_guess_set_params(g, P.data(), nm);
  if (rc) return bad(rc);
  *out = g;
  return FIVO_OK;
}

int fivo_guess_destroy(fivo_guess* g) {
  if (!g) return FIVO_OK;
  if (g->st) cudaStreamSynchronize(g->st);
  cudaFree(g->params); cudaFree(g->adam); cudaFree(g->img); cudaFree(g->samples); cudaFree(g->count);
  cudaFree(g->part); cudaFree(g->loss_part); cudaFree(g->grad); cudaFree(g->err);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
  return FIVO_OK;
}

int fivo_guess_set_params(fivo_guess* g, const float* params, const float* norm) {
  if (!g) return fail(FIVO_ERR_ARG, "null guess");
  if (params) {
    CK(cudaMemcpyAsync(g->params, params, guess::NPARAM * sizeof(float), cudaMemcpyHostToDevice, g->st));
    CK(cudaMemsetAsync(g->adam, 0, 2 * guess::NPARAM * sizeof(float), g->st));
    g->adam_t = 0;
    int rc = guess_pack(g);
    if (rc) return rc;
  }
  if (norm) {
    for (int q = 0; q < 8; ++q) { g->norm.in_mean[q] = norm[q]; g->norm.in_istd[q] = norm[8 + q]; }
    for (int o = 0; o < 3; ++o) { g->norm.out_mean[o] = norm[16 + o]; g->norm.out_std[o] = norm[19 + o]; }
  }
  CK(cudaMemsetAsync(g->err, 0, sizeof(int), g->st));
  CK(cudaStreamSynchronize(g->st));
  return FIVO_OK;
}

int fivo_guess_get_params(fivo_guess* g, float* params, float* norm) {
  if (!g) return fail(FIVO_ERR_ARG, "null guess");
  if (params) {
    CK(cudaMemcpyAsync(params, g->params, guess::NPARAM * sizeof(float), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
  }
  if (norm) {
    for (int q = 0; q < 8; ++q) { norm[q] = g->norm.in_mean[q]; norm[8 + q] = g->norm.in_istd[q]; }
    for (int o = 0; o < 3; ++o) { norm[16 + o] = g->norm.out_mean[o]; norm[19 + o] = g->norm.out_std[o]; }
  }
  return FIVO_OK;
}

int fivo_guess_reserve(fivo_guess* g, int64_t capacity) {
  if (!g || capacity < 0) return fail(FIVO_ERR_ARG, "bad argument");
  CK(cudaStreamSynchronize(g->st));
  cudaFree(g->samples);
  g->samples = nullptr;
  g->cap = 0;
  if (capacity > 0 && cudaMalloc(&g->samples, (size_t)capacity * guess::NSAMP * sizeof(float)) != cudaSuccess)
    return fail(FIVO_ERR_NOMEM, "fivo_guess_reserve: device allocation failed");
  g->cap = capacity;
  CK(cudaMemset(g->count, 0, sizeof(unsigned long long)));
  return FIVO_OK;
}

int fivo_guess_nsamples(fivo_guess* g, int64_t* n) {
  if (!g || !n) return fail(FIVO_ERR_ARG, "null argument");
  unsigned long long k = 0;
  CK(cudaStreamSynchronize(g->st));
  CK(cudaMemcpy(&k, g->count, sizeof(k), cudaMemcpyDeviceToHost));
  *n = (int64_t)std::min<unsigned long long>(k, (unsigned long long)g->cap);
  return FIVO_OK;
}

int fivo_guess_set_samples(fivo_guess* g, const float* samples, int64_t n) {
  if (!g || (!samples && n > 0) || n < 0) return fail(FIVO_ERR_ARG, "bad argument");
  if (n > g->cap) { int rc = fivo_guess_reserve(g, n); if (rc) return rc; }
  if (n > 0) CK(cudaMemcpy(g->samples, samples, (size_t)n * guess::NSAMP * sizeof(float), cudaMemcpyHostToDevice));
  unsigned long long k = (unsigned long long)n;
  CK(cudaMemcpy(g->count, &k, sizeof(k), cudaMemcpyHostToDevice));
  return FIVO_OK;
}

int fivo_guess_get_samples(fivo_guess* g, float* samples, int64_t n) {
  int64_t have = 0;
  int rc = fivo_guess_nsamples(g, &have);
  if (rc) return rc;
  if (!samples || n < 0 || n > have) return fail(FIVO_ERR_ARG, "bad argument");
  if (n > 0) CK(cudaMemcpy(samples, g->samples, (size_t)n * guess::NSAMP * sizeof(float), cudaMemcpyDeviceToHost));
  return FIVO_OK;
}

int fivo_guess_harvest(fivo_ctx* c, fivo_guess* g, double tau, int stride, int phase) {
  if (!c || !g || stride < 1 || phase < 0) return fail(FIVO_ERR_ARG, "bad argument");
  if (g->cap <= 0) return fail(FIVO_ERR_ARG, "fivo_guess_harvest: no sample store (fivo_guess_reserve)");
  if (g->device != c->device) return fail(FIVO_ERR_ARG, "fivo_guess_harvest: the guess lives on another device");
  CK(ctx_sync(c));
  const DevParams& d = c->dp;
  if (d.p.eos_kind == FIVO_EOS_LATTICE_HRG)
    k_guess_harvest<FIVO_EOS_LATTICE_HRG><<<nblk(d.Ntot, 256), 256, 0, c->st>>>(
        d, c->S[c->iU], c->w, tau, g->samples, (unsigned long long)g->cap, g->count, stride, phase);
  else
    k_guess_harvest<FIVO_EOS_CONFORMAL_HQ><<<nblk(d.Ntot, 256), 256, 0, c->st>>>(
        d, c->S[c->iU], c->w, tau, g->samples, (unsigned long long)g->cap, g->count, stride, phase);
  CKL();
  CK(ctx_sync(c));
  return FIVO_OK;
}

int fivo_guess_fit_norm(fivo_guess* g) {
  int64_t n = 0;
  int rc = fivo_guess_nsamples(g, &n);
  if (rc) return rc;
  if (n < 2) return fail(FIVO_ERR_ARG, "fivo_guess_fit_norm: fewer than 2 samples");
  const int nb = 256;
  double* part = nullptr;
  CK(cudaMalloc(&part, (size_t)nb * 2 * guess::NSAMP * sizeof(double)));
  guess::k_moments<<<nb, 256, 0, g->st>>>(g->samples, n, part);
  std::vector<double> hp((size_t)nb * 2 * guess::NSAMP);
  cudaError_t e1 = cudaGetLastError();
  cudaError_t e2 = cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, g->st);
  cudaError_t e3 = cudaStreamSynchronize(g->st);
  cudaFree(part);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
    return fail(FIVO_ERR_CUDA, "fivo_guess_fit_norm: moments failed");
  double sum[guess::NSAMP] = {}, sq[guess::NSAMP] = {};
  for (int b = 0; b < nb; ++b)
    for (int q = 0; q < guess::NSAMP; ++q) {
      sum[q] += hp[(size_t)b * 2 * guess::NSAMP + q];
      sq[q] += hp[(size_t)b * 2 * guess::NSAMP + guess::NSAMP + q];
    }
  for (int q = 0; q < guess::NSAMP; ++q) {
    const double m = sum[q] / n;
    const double sd = std::sqrt(std::max(sq[q] / n - m * m, 0.0));
    const double s = std::max(sd, 1e-6);
    if (q < guess::NIN) { g->norm.in_mean[q] = (float)m; g->norm.in_istd[q] = (float)(1.0 / s); }
    else { g->norm.out_mean[q - guess::NIN] = (float)m; g->norm.out_std[q - guess::NIN] = (float)s; }
  }
  return FIVO_OK;
}

int fivo_guess_train(fivo_guess* g, int steps, int ctas, float lr, uint64_t seed, double* loss_out) {
  if (!g || steps < 1 || ctas < 1 || !(lr > 0.0f)) return fail(FIVO_ERR_ARG, "bad argument");
  int64_t n = 0;
  int rc = fivo_guess_nsamples(g, &n);
  if (rc) return rc;
  if (n < 1) return fail(FIVO_ERR_ARG, "fivo_guess_train: no samples");
  CK(cudaMemsetAsync(g->err, 0, sizeof(int), g->st));
  for (int s = 0; s < steps; ++s) {
    const unsigned long long sd = guess::mix64(seed + (uint64_t)s) | 1ULL;
    if ((rc = guess_step(g, g->samples, n, sd, ctas, lr, nullptr))) return rc;
    if (loss_out && (s == 0 || s == steps - 1)) {
      double l = 0.0;
      if ((rc = guess_loss(g, ctas, &l))) return rc;
      loss_out[s == 0 ? 0 : 1] = l;
      if (steps == 1) loss_out[1] = l;
    }
  }
  CK(cudaStreamSynchronize(g->st));
  return FIVO_OK;
}

int fivo_guess_grad(fivo_guess* g, const float* samples, int64_t n, float* grad, double* loss) {
  if (!g || !samples || !grad || n < 128 || n % 128) return fail(FIVO_ERR_ARG, "bad argument");
  float* ds = nullptr;
  CK(cudaMalloc(&ds, (size_t)n * guess::NSAMP * sizeof(float)));
  int rc = FIVO_OK;
  if (cudaMemcpy(ds, samples, (size_t)n * guess::NSAMP * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(FIVO_ERR_CUDA, "fivo_guess_grad: upload failed");
  if (!rc) { cudaMemsetAsync(g->err, 0, sizeof(int), g->st); rc = guess_step(g, ds, n, 0ULL, (int)(n / 128), 0.0f, g->grad); }
  double l = 0.0;
  if (!rc) rc = guess_loss(g, (int)(n / 128), &l);
  if (!rc && cudaMemcpy(grad, g->grad, guess::NPARAM * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(FIVO_ERR_CUDA, "fivo_guess_grad: download failed");
  cudaFree(ds);
  if (!rc && loss) *loss = l;
  return rc;
}

int fivo_guess_forward(fivo_guess* g, const float* raw, int64_t n, float* out) {
  if (!g || !raw || !out || n < 1) return fail(FIVO_ERR_ARG, "bad argument");
  float *dr = nullptr, *dout = nullptr;
  CK(cudaMalloc(&dr, (size_t)n * guess::NIN * sizeof(float)));
  if (cudaMalloc(&dout, (size_t)n * guess::NOUT * sizeof(float)) != cudaSuccess) {
    cudaFree(dr);
    return fail(FIVO_ERR_NOMEM, "fivo_guess_forward: device allocation failed");
  }
  int rc = FIVO_OK;
  const int dyn = LEARNED_SMEM - (int)sizeof(guess::FwdSmem);
  if (cudaMemcpy(dr, raw, (size_t)n * guess::NIN * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(g->err, 0, sizeof(int)) != cudaSuccess ||
      cudaFuncSetAttribute(guess::k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess)
    rc = fail(FIVO_ERR_CUDA, "fivo_guess_forward: setup failed");
  if (!rc) {
    guess::k_infer<<<(unsigned)((n + 127) / 128), 128, dyn, g->st>>>(net_of(g), dr, n, dout, g->err);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(g->st) != cudaSuccess)
      rc = fail(FIVO_ERR_CUDA, "fivo_guess_forward: kernel failed");
  }
  int e = 0;
  if (!rc && cudaMemcpy(&e, g->err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && e)
    rc = fail(FIVO_ERR_DEVICE, "fivo_guess_forward: a tensor-core wait gave up");
  if (!rc && cudaMemcpy(out, dout, (size_t)n * guess::NOUT * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(FIVO_ERR_CUDA, "fivo_guess_forward: download failed");
  cudaFree(dr);
  cudaFree(dout);
  return rc;
}

int fivo_ctx_set_guess(fivo_ctx* c, fivo_guess* g) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (g && g->device != c->device) return fail(FIVO_ERR_ARG, "fivo_ctx_set_guess: the guess lives on another device");
  CK(ctx_sync(c));
  if (g) CK(cudaStreamSynchronize(g->st));
  c->learned = g != nullptr;
  c->gnet = g ? net_of(g) : guess::Net{};
  return FIVO_OK;
}

int fivo_ctx_set_guess_mode(fivo_ctx* c, int mode) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (mode != FIVO_GUESS_EVERY_CELL && mode != FIVO_GUESS_DEFERRED)
    return fail(FIVO_ERR_ARG, "fivo_ctx_set_guess_mode: unknown mode");
  CK(ctx_sync(c));
  c->guess_mode = mode;
  return FIVO_OK;
}

int fivo_newton_stats_read(fivo_ctx* c, fivo_newton_stats* out, int reset) {
  if (!c || !out) return fail(FIVO_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(c->flh, c->fl, sizeof(DevFlags), cudaMemcpyDeviceToHost, c->st));
  CK(ctx_sync(c));
  const DevFlags& f = *c->flh;
  out->it_fast = f.it_fast; out->n_fast = f.n_fast; out->it_learn = f.it_learn; out->n_learn = f.n_learn;
  out->ok_learn = f.ok_learn; out->it_fb = f.it_fb; out->n_fb = f.n_fb;
  out->deferred = f.tot_p - (uint64_t)c->stats_base_p;
  if (reset) {
    k_reset_flags<<<1, 32, 0, c->st>>>(c->fl, 32, 0ULL);
    CKL();
    c->stats_base_p = (int64_t)f.tot_p;
    CK(ctx_sync(c));
  }
  return FIVO_OK;
}

/* ------------------------------------------------ freeze-out surface and Cooper-Frye */

struct fivo_fo {
  int device = 0;
  cudaStream_t st = nullptr;
  int nx = 0, ny = 0;
  double dx = 0.0, T_fo = 0.0;
  double tau_prev = 0.0;
  bool have_prev = false;
  double* planes = nullptr;               /* tau_fo | uxf | uyf | Tprev */
  uint8_t* above = nullptr;
  unsigned long long* refroze = nullptr;
  double* part = nullptr;
  long long part_n = 0;
};

namespace {
fo::Surf surf_of(fivo_fo* f) {
  const size_t n = (size_t)f->nx * f->ny;
  return fo::Surf{f->planes, f->planes + n, f->planes + 2 * n, f->planes + 3 * n, f->above, f->refroze, f->nx, f->ny};
}
}  // namespace

void fivo_cf_params_default(fivo_cf_params* p) {
  if (!p) return;
  p->T_fo = 0.156; p->m = 0.138; p->pt_lo = 0.1; p->pt_hi = 5.0; p->eta_max = 6.0; p->f_yield = 2.0 * 2.5;
  p->n_eta = 40; p->n_pt = 40; p->n_phi = 24; p->pad = 0;
}

int fivo_fo_create(fivo_ctx* c, double T_fo, fivo_fo** out) {
  if (!c || !out || !(T_fo > 0.0)) return fail(FIVO_ERR_ARG, "bad argument");
  *out = nullptr;
  fivo_fo* f = new fivo_fo();
  f->device = c->device; f->nx = c->dp.Nx; f->ny = c->dp.Ny; f->dx = c->dp.dx; f->T_fo = T_fo;
  if (c->dp.dx != c->dp.dy) { delete f; return fail(FIVO_ERR_ARG, "fivo_fo_create: the surface needs dx == dy"); }
  const size_t n = (size_t)f->nx * f->ny;
  if (cudaStreamCreateWithFlags(&f->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&f->planes, 4 * n * sizeof(double)) != cudaSuccess || cudaMalloc(&f->above, n) != cudaSuccess ||
      cudaMalloc(&f->refroze, sizeof(unsigned long long)) != cudaSuccess) {
    fivo_fo_destroy(f);
    return fail(FIVO_ERR_NOMEM, "fivo_fo_create: device allocation failed");
  }
  int rc = fivo_fo_reset(f);
  if (rc) { fivo_fo_destroy(f); return rc; }
  *out = f;
  return FIVO_OK;
}

int fivo_fo_reset(fivo_fo* f) {
  if (!f) return fail(FIVO_ERR_ARG, "null surface");
  const size_t n = (size_t)f->nx * f->ny;
  k_fill_nan<<<nblk((long long)n, 256), 256, 0, f->st>>>(f->planes, (long long)n);             /* tau_fo */
  CKL();
  CK(cudaMemsetAsync(f->planes + n, 0, 2 * n * sizeof(double), f->st));                     /* uxf, uyf */
  k_fill_nan<<<nblk((long long)n, 256), 256, 0, f->st>>>(f->planes + 3 * n, (long long)n);  /* Tprev */
  CKL();
  CK(cudaMemsetAsync(f->above, 0, n, f->st));
  CK(cudaMemsetAsync(f->refroze, 0, sizeof(unsigned long long), f->st));
  CK(cudaStreamSynchronize(f->st));
  f->have_prev = false;
  return FIVO_OK;
}

int fivo_fo_destroy(fivo_fo* f) {
  if (!f) return FIVO_OK;
  if (f->st) cudaStreamSynchronize(f->st);
  cudaFree(f->planes); cudaFree(f->above); cudaFree(f->refroze); cudaFree(f->part);
  if (f->st) cudaStreamDestroy(f->st);
  delete f;
  return FIVO_OK;
}

int fivo_fo_record(fivo_fo* f, fivo_ctx* c, double tau) {
  if (!f || !c) return fail(FIVO_ERR_ARG, "null argument");
  if (c->dp.Nx != f->nx || c->dp.Ny != f->ny) return fail(FIVO_ERR_ARG, "fivo_fo_record: grid mismatch");
  if (c->device != f->device) return fail(FIVO_ERR_ARG, "fivo_fo_record: the surface lives on another device");
  const double tp = f->have_prev ? f->tau_prev : tau;
  const long long n = (long long)f->nx * f->ny;
  fo::k_record<<<nblk(n, 256), 256, 0, c->st>>>(c->dp, c->w, tau, tp, f->T_fo, surf_of(f));
  CKL();
  CK(ctx_sync(c));
  f->tau_prev = tau;
  f->have_prev = true;
  return FIVO_OK;
}

int fivo_fo_surface(fivo_fo* f, double* tau_fo, double* uxf, double* uyf, int64_t* counts) {
  if (!f) return fail(FIVO_ERR_ARG, "null surface");
  const size_t n = (size_t)f->nx * f->ny;
  std::vector<double> t(n);
  std::vector<uint8_t> ab(n);
  unsigned long long rf = 0;
  CK(cudaMemcpyAsync(t.data(), f->planes, n * sizeof(double), cudaMemcpyDeviceToHost, f->st));
  if (uxf) CK(cudaMemcpyAsync(uxf, f->planes + n, n * sizeof(double), cudaMemcpyDeviceToHost, f->st));
  if (uyf) CK(cudaMemcpyAsync(uyf, f->planes + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, f->st));
  CK(cudaMemcpyAsync(ab.data(), f->above, n, cudaMemcpyDeviceToHost, f->st));
  CK(cudaMemcpyAsync(&rf, f->refroze, sizeof(rf), cudaMemcpyDeviceToHost, f->st));
  CK(cudaStreamSynchronize(f->st));
  if (tau_fo) std::memcpy(tau_fo, t.data(), n * sizeof(double));
  if (counts) {
    int64_t hot = 0, froze = 0;
    for (size_t k = 0; k < n; ++k) { hot += ab[k] != 0; froze += !std::isnan(t[k]); }
    counts[0] = hot; counts[1] = froze; counts[2] = (int64_t)rf;
  }
  return FIVO_OK;
}

int fivo_fo_set_surface(fivo_fo* f, const double* tau_fo, const double* uxf, const double* uyf) {
  if (!f || !tau_fo || !uxf || !uyf) return fail(FIVO_ERR_ARG, "null argument");
  const size_t n = (size_t)f->nx * f->ny;
  CK(cudaMemcpyAsync(f->planes, tau_fo, n * sizeof(double), cudaMemcpyHostToDevice, f->st));
  CK(cudaMemcpyAsync(f->planes + n, uxf, n * sizeof(double), cudaMemcpyHostToDevice, f->st));
  CK(cudaMemcpyAsync(f->planes + 2 * n, uyf, n * sizeof(double), cudaMemcpyHostToDevice, f->st));
  CK(cudaStreamSynchronize(f->st));
  return FIVO_OK;
}

int fivo_cooper_frye(fivo_fo* f, const fivo_cf_params* p, double* out) {
  if (!f || !p || !out) return fail(FIVO_ERR_ARG, "null argument");
  if (p->n_eta < 2 || p->n_pt < 2 || p->n_phi < 1 || !(p->T_fo > 0.0))
    return fail(FIVO_ERR_ARG, "fivo_cooper_frye: bad grid");
  const long long total = (long long)f->nx * f->ny * p->n_pt * p->n_phi;
  const long long nb = nblk(total, 256);
  if (nb > f->part_n) {
    cudaFree(f->part);
    f->part = nullptr;
    f->part_n = 0;
    CK(cudaMalloc(&f->part, (size_t)nb * 4 * sizeof(double)));
    f->part_n = nb;
  }
  const fo::CF cf{p->T_fo, p->m, p->pt_lo, p->pt_hi, p->eta_max, p->n_eta, p->n_pt, p->n_phi};
  fo::k_cooper_frye<<<(unsigned)nb, 256, 0, f->st>>>(surf_of(f), f->dx, cf, f->part);
  CKL();
  std::vector<double> h((size_t)nb * 4);
  CK(cudaMemcpyAsync(h.data(), f->part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, f->st));
  CK(cudaStreamSynchronize(f->st));
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long b = 0; b < nb; ++b)
    for (int q = 0; q < 4; ++q) s[q] += h[(size_t)b * 4 + q];
  const double hc = 0.1973269804;
  const double pref = p->f_yield / std::pow((2.0 * M_PI) * hc, 3);
  out[0] = pref * s[0];
  out[1] = pref * s[1];
  out[2] = s[2] / std::max(s[3] + s[2], 1e-30);
  return FIVO_OK;
}

/* ------------------------------------------------ mixed precision */

int fivo_ctx_set_face_pass(fivo_ctx* c, int x_cfg, int y_cfg) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  const int cfg[2] = {x_cfg, y_cfg};
  for (int dir = 0; dir < 2; ++dir) {
    if (cfg[dir] < -2 || cfg[dir] >= FT_NSHAPES)
      return fail(FIVO_ERR_ARG, "fivo_ctx_set_face_pass: configuration out of range");
    if (cfg[dir] >= 0 && !(c->dp.Nytot % 2 == 0 && ft_encode(c, dir, cfg[dir])))
      return fail(FIVO_ERR_ARG, "fivo_ctx_set_face_pass: the tiled face pass needs an even Ny + 6");
  }
  CK(ctx_sync(c));
  c->ft_cfg[0] = x_cfg;
  c->ft_cfg[1] = y_cfg;
  if (x_cfg == -2 || y_cfg == -2) c->ft_cfg[0] = c->ft_cfg[1] = -2;
  return FIVO_OK;
}

int fivo_ctx_face_pass(fivo_ctx* c, int* x_cfg, int* y_cfg) {
  if (!c || !x_cfg || !y_cfg) return fail(FIVO_ERR_ARG, "null argument");
  *x_cfg = c->ft_cfg[0];
  *y_cfg = c->ft_cfg[1];
  return FIVO_OK;
}

int fivo_ctx_set_precision(fivo_ctx* c, int mode) {
  if (!c) return fail(FIVO_ERR_ARG, "null context");
  if (mode != FIVO_PRECISION_FP64 && mode != FIVO_PRECISION_FP32_FACES && mode != FIVO_PRECISION_FP32)
    return fail(FIVO_ERR_ARG, "fivo_ctx_set_precision: unknown mode");
  if (mode == FIVO_PRECISION_FP32 && c->dp.hasM2)
    return fail(FIVO_ERR_CONFIG, "fivo_ctx_set_precision: the FP32 relaxation sources do not cover consistent_m2");
  CK(ctx_sync(c));
  if (mode != FIVO_PRECISION_FP64 && !c->fh32) {
    if (cudaMalloc(&c->fh32, 2 * (size_t)c->dp.nv * c->dp.Ntot * sizeof(float)) != cudaSuccess) {
      c->fh32 = nullptr;
      return fail(FIVO_ERR_NOMEM, "fivo_ctx_set_precision: device allocation failed");
    }
  }
  c->precision = mode;
  return FIVO_OK;
}
