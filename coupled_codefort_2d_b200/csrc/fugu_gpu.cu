// fugu_gpu.cu -- host orchestration and C ABI of the B200 FUGU-2D hot path.
//
// A context owns every device buffer of one case in the uniform padded layout
// (fugu_internal.cuh) and one CUDA stream.  The step, the Krylov solvers and
// the PCD preconditioner are sequences of the kernels in kernels.cuh,
// persistent.cuh and scalars.cuh; Krylov scalars stay on the device, and the
// host only polls the `active` flag once per Krylov iteration.
//
// Compiled for sm_100a with --fmad=false (see build.py): the FP64 plain form
// then rounds every operation as the CPU oracle does.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "fugu_gpu.h"
#include "adjoint.cuh"
#include "fgmres.cuh"
#include "kernels.cuh"
#include "pcg_cluster.cuh"
#include "persistent.cuh"
#include "scalars.cuh"
#include "step_vjp.cuh"

using namespace fugu;

namespace {

struct CudaError {
  cudaError_t e;
  const char* what;
};
#define CK(x)                                     \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) throw CudaError{e_, #x}; \
  } while (0)
// every kernel launch site is followed by CKL: it checks the launch and
// counts it (c is the context in scope at each site)
#define CKL(what)                                          \
  do {                                                     \
    cudaError_t e_ = cudaGetLastError();                   \
    if (e_ != cudaSuccess) throw CudaError{e_, what};      \
    ++c->launches;                                         \
  } while (0)

// NVTX range over a host scope: the phases of a step and each Krylov
// iteration show as named ranges in a timeline profiler (no-ops otherwise)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct ApiError {
  int code;
  std::string msg;
};

template <typename T>
struct Trip {
  T* base = nullptr;
  T* u = nullptr;
  T* v = nullptr;
  T* p = nullptr;
};

template <typename T>
struct PcgWork {
  T *cx = nullptr, *cy = nullptr, *dinv = nullptr, *r = nullptr, *z = nullptr, *pb0 = nullptr,
    *pb1 = nullptr, *ap = nullptr;
  T *w1 = nullptr, *pv = nullptr;  // the FP32 single-reduction grid-wide PCG's two more vectors
};

template <typename T>
struct PcdWork {
  T *phi = nullptr, *zuw = nullptr, *zvw = nullptr, *tmp = nullptr;
};

// coefficient fields of the coupled operator in one precision
template <typename T>
struct CoefBufs {
  T *u_adv = nullptr, *v_adv = nullptr, *rho_c = nullptr, *rho_u = nullptr, *rho_v = nullptr,
    *kappa = nullptr, *zeta = nullptr, *eta = nullptr, *pen_u = nullptr, *pen_v = nullptr,
    *mdu = nullptr, *mdv = nullptr;
};

// which optional coefficient fields a solve uses
struct SolveOpt {
  bool pen = false;
  bool amp = false;
};

template <typename T>
struct KrylovWork {
  Trip<T> t[13];  // bh, r, rt, uu, vv, ww, ss, tt, z, q + refine r, d, ax
  PcdWork<T> pcd;
  PcgWork<T> pcg;
  CoefBufs<T> cf;  // converted coefficients (FP32 only; FP64 points at the originals)
};

// flexible GMRES basis: V_0..V_m and Z_0..Z_{m-1}, contiguous triples
template <typename T>
struct FgWork {
  T* V = nullptr;
  T* Z = nullptr;
  double* st = nullptr;  // FgLayout scalars
  int cap = 0;           // m the buffers hold
};

// buffers of the step's vector-Jacobian product (allocated on first use)
struct VjpWork {
  bool ready = false;
  // the state before the step: C^n, u^n, v^n, u^(n-1), v^(n-1)
  double *c0 = nullptr, *u0 = nullptr, *v0 = nullptr, *up0 = nullptr, *vp0 = nullptr;
  // adjoints after the step (inputs; b_c1 also collects C^(n+1)'s whole adjoint)
  double *b_u1 = nullptr, *b_v1 = nullptr, *b_c1 = nullptr, *b_up1 = nullptr, *b_vp1 = nullptr;
  // adjoints before the step (outputs) and of C_smooth
  double *b_c0 = nullptr, *b_u0 = nullptr, *b_v0 = nullptr, *b_up0 = nullptr, *b_vp0 = nullptr;
  double *b_cs = nullptr, *t1 = nullptr, *t2 = nullptr;
  Trip<double> g, lam, resid;
  int* svof_it = nullptr;
  // duals: VOF stage (C^n, u^n, v^n -> C^(n+1))
  ad::Dual *dc0 = nullptr, *du0 = nullptr, *dv0 = nullptr, *dc1o = nullptr;
  // duals: inputs and intermediates of the solve's stage
  ad::Dual *dc1 = nullptr, *dcs = nullptr, *dun = nullptr, *dvn = nullptr, *dunm1 = nullptr, *dvnm1 = nullptr;
  ad::Dual *drc = nullptr, *dru = nullptr, *drv = nullptr, *dka = nullptr, *dze = nullptr, *det = nullptr;
  ad::Dual *dkc = nullptr, *dfu = nullptr, *dfv = nullptr, *dua = nullptr, *dva = nullptr;
  ad::Dual *dB[3] = {}, *dX[3] = {}, *dY[3] = {};
  // duals: the final wall BCs of the step (owned velocity -> every entry)
  ad::Dual *dgu = nullptr, *dgv = nullptr;
};

}  // namespace

struct fugu_ctx {
  fugu_params prm{};
  Geo g{};
  int device = 0;
  int nsm = 148;
  cudaStream_t s = nullptr;
  long n = 0;  // elements per buffer
  std::vector<void*> allocs;
  double* f[FUGU_NUM_FIELDS] = {};
  // step temporaries
  double *u_nm1 = nullptr, *v_nm1 = nullptr, *u_adv = nullptr, *v_adv = nullptr, *c_new = nullptr,
         *c_s = nullptr, *svof_w = nullptr, *fcx = nullptr, *fcy = nullptr, *mdu = nullptr,
         *mdv = nullptr, *pen_u = nullptr, *pen_v = nullptr;
  Trip<double> B;
  Trip<double> Xstate;  // u_vel, v_vel, p_field (contiguous)
  KrylovWork<double> w64;
  KrylovWork<float> w32;
  bool w32_ready = false;
  FgWork<double> fg64;
  FgWork<float> fg32;
  int pcg_cap_cur = 0;    // PCG cap of the PCD during an adaptive solve (0: pcg_max_iter)
  int pcg_cap_state = 0;  // cap the last adaptive solve ended with (carried to the next)
  int pcd_sweeps_cur = 0;    // PCD Jacobi sweeps during an adaptive solve (0: pcd_sweeps)
  int pcd_sweeps_state = 0;  // sweeps the last adaptive solve ended with
  // adjoint: the probed stencil of the coupled operator; while adj_on, the
  // solvers' operator is S A^T S instead of A
  double* adj_val = nullptr;
  unsigned int* adj_err = nullptr;
  bool adj_on = false;
  VjpWork vjp;
  // routine-level scratch
  double* scratch[20] = {};
  // device scalars / state
  double* sc = nullptr;
  KState* ks = nullptr;
  double* part = nullptr;
  long part_len = 0;
  GridSync* gs = nullptr;
  PcgOut* pcg_out = nullptr;
  int* svof_iters = nullptr;
  int* svof_status = nullptr;
  // pinned host mirrors
  KState* h_ks = nullptr;
  double* h_sc = nullptr;
  PcgOut* h_pcg = nullptr;
  int* h_int = nullptr;
  int pcg_grid = 0;
  int svof_grid = 0;
  int dot_grid = 0;
  // failure-detection test hook: > 0 arms the next grid-wide PCG launch to
  // wait for one CTA too many and give up after this many polls
  unsigned int test_spin_limit = 0;
  // limits for concurrent use (a batch lowers them so many cases fit at once)
  int max_cluster = 16;  // CTAs of the cluster-resident PCG
  int max_coop = 1 << 30;  // CTAs of a grid-wide cooperative kernel
  bool coop_as_cluster = false;  // launch those as one cluster (max_coop <= 8)
  // Krylov iterations whose PCG is the grid-wide kernel are captured into
  // graphs as cooperative kernel nodes; cleared (for good) if a capture or an
  // instantiation with such a node fails, and those iterations run eagerly
  bool coop_graphs = true;
  bool capture_coop = false;  // the capture in progress holds a grid-wide launch
  // cluster-resident PCG plan per precision (index 0 FP64, 1 FP32)
  struct ClusterPlan {
    bool ok = false;
    int C = 0, rows_per = 0, cpt = 0;
    size_t smem = 0;
  } pcgc[2];
  // CUDA graphs of the flexible-GMRES Arnoldi steps (graphs = 1), per
  // precision (0 FP64, 1 FP32) and step index j
  struct StepGraph {
    std::vector<unsigned char> key;  // everything the captured launches depend on
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;  // kernel launches in one replay
    // around its PCG launches (profiling): one pair per launch in the body
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    size_t ev_used = 0;
    bool timed = false;  // its PCG launches are timed (profiling)
  };
  std::vector<StepGraph> fg_graphs[2];
  // one BiCGStab (index 0) / BiCGStab(2) (index 1) iteration per precision,
  // its iteration index on the device (KState::kiter)
  StepGraph kr_graphs[2][2];
  StepGraph* capturing = nullptr;     // the step graph being captured
  StepGraph* pcg_timed = nullptr;     // replayed with PCG events, not yet read
  // measurement: launch count, CUDA-event timing of the persistent kernels
  unsigned long long launches = 0;
  int prof = 0;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pcg;
  double prof_pcg_ms = 0.0;
  unsigned long long prof_pcg_launches = 0, prof_pcg_iters = 0, prof_pcg_cells = 0, prof_pcg_iters_timed = 0;
  std::string err;
};

namespace {

constexpr int PCG_TPB = 512;
constexpr int DOT_TPB = 256;

template <typename T>
T* dalloc(fugu_ctx* c, long n) {
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * n) != cudaSuccess) throw ApiError{FUGU_ENOMEM, "cudaMalloc failed"};
  c->allocs.push_back(p);
  CK(cudaMemsetAsync(p, 0, sizeof(T) * n, c->s));
  return (T*)p;
}
template <typename T>
Trip<T> talloc(fugu_ctx* c) {
  Trip<T> t;
  t.base = dalloc<T>(c, 3 * c->n);
  t.u = t.base;
  t.v = t.base + c->n;
  t.p = t.base + 2 * c->n;
  return t;
}

Geo make_geo(const fugu_params& p) {
  Geo g{};
  g.nx = p.nx;
  g.ny = p.ny;
  g.P = ((p.nx + 5 + 15) / 16) * 16;
  g.R = p.ny + 5;
  g.dx = p.dx;
  g.dy = p.dy;
  g.idx = 1.0 / p.dx;
  g.idy = 1.0 / p.dy;
  g.idx2 = 1.0 / (p.dx * p.dx);
  g.idy2 = 1.0 / (p.dy * p.dy);
  g.px = p.periodic_x ? 1 : 0;
  g.py = p.periodic_y ? 1 : 0;
  g.fsx = p.free_slip_x ? 1 : 0;
  return g;
}

int kind_of_field(int f) {
  switch (f) {
    case FUGU_F_U_VEL: case FUGU_F_U_PREV: case FUGU_F_RHO_U: case FUGU_F_F_SIGMA_U: case FUGU_F_PHI_S_U:
      return K_U;
    case FUGU_F_V_VEL: case FUGU_F_V_PREV: case FUGU_F_RHO_V: case FUGU_F_F_SIGMA_V: case FUGU_F_PHI_S_V:
      return K_V;
    case FUGU_F_ZETA: case FUGU_F_ETA:
      return K_VERT;
    default:
      return K_CELL;
  }
}

// Fortran-layout host array <-> uniform device box (strided 2-D copies)
void copy_kind(fugu_ctx* c, double* dev, const double* host, int kind, bool h2d, double* hostw = nullptr) {
  const Geo& g = c->g;
  int i0, i1, j0, j1;
  g.extent(kind, i0, i1, j0, j1);
  const size_t w = (size_t)(i1 - i0 + 1), h = (size_t)(j1 - j0 + 1);
  double* d = dev + g.at(i0, j0);
  if (h2d)
    CK(cudaMemcpy2DAsync(d, sizeof(double) * g.P, host, sizeof(double) * w, sizeof(double) * w, h,
                         cudaMemcpyHostToDevice, c->s));
  else
    CK(cudaMemcpy2DAsync(hostw, sizeof(double) * w, d, sizeof(double) * g.P, sizeof(double) * w, h,
                         cudaMemcpyDeviceToHost, c->s));
}
void up(fugu_ctx* c, double* dev, const double* host, int kind) {
  if (!host) throw ApiError{FUGU_EINVAL, "NULL host array"};
  copy_kind(c, dev, host, kind, true);
}
void down(fugu_ctx* c, double* host, const double* dev, int kind) {
  if (!host) throw ApiError{FUGU_EINVAL, "NULL host array"};
  copy_kind(c, (double*)dev, nullptr, kind, false, host);
}
void sync(fugu_ctx* c) { CK(cudaStreamSynchronize(c->s)); }

int grid1d(fugu_ctx* c, long n) {
  long b = (n + 255) / 256;
  long cap = (long)c->nsm * 8;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// ------------------------------------------------------------------ launches
template <typename T>
void halo(fugu_ctx* c, T* a, int kind, const int* active = nullptr) {
  if (!c->g.px && !c->g.py) return;
  k_halo<T><<<1, 1024, 0, c->s>>>(c->g, a, kind, active);
  CKL("k_halo");
}
template <typename T>
void vbcs(fugu_ctx* c, T* u, T* v, double lid, const int* active = nullptr) {
  if (c->g.px && c->g.py) return;
  k_velocity_bcs<T><<<1, 1024, 0, c->s>>>(c->g, u, v, T(lid), active);
  CKL("k_velocity_bcs");
}

template <typename T>
Coefs<T> coefs_of(const CoefBufs<T>& b, const SolveOpt& o) {
  Coefs<T> cf;
  cf.u_adv = b.u_adv; cf.v_adv = b.v_adv; cf.rho_c = b.rho_c; cf.rho_u = b.rho_u; cf.rho_v = b.rho_v;
  cf.kappa = b.kappa; cf.zeta = b.zeta; cf.eta = b.eta;
  cf.pen_u = o.pen ? b.pen_u : nullptr;
  cf.pen_v = o.pen ? b.pen_v : nullptr;
  cf.mdot_u = o.amp ? b.mdu : nullptr;
  cf.mdot_v = o.amp ? b.mdv : nullptr;
  return cf;
}

template <typename T>
void matvec(fugu_ctx* c, const CoefBufs<T>& cb, const SolveOpt& o, Trip<T> X, Trip<T> Y, double dt,
            const int* active) {
  if (c->adj_on) {  // adjoint solve: the sign-conjugated transpose from the probed stencil
    if constexpr (std::is_same<T, double>::value) {
      Box b = box_launch(c->g);
      k_adj_apply_t<<<b.grid, b.block, 0, c->s>>>(c->g, c->n, c->adj_val, X.base, Y.base, -1.0, active,
                                                   &c->ks->matvecs);
      CKL("k_adj_apply_t");
      return;
    } else {
      throw ApiError{FUGU_EINVAL, "the adjoint solve runs in FP64"};
    }
  }
  halo(c, X.u, K_U, active);
  halo(c, X.v, K_V, active);
  halo(c, X.p, K_CELL, active);
  // staged tiles of MT_TX x TY outputs (rows per tile: 16 in FP32, 8 in FP64)
  constexpr int TY = sizeof(T) == 4 ? 16 : 8;
  const dim3 grid((c->g.P + MT_TX - 1) / MT_TX, (c->g.R + TY - 1) / TY);
  k_matvec_tile<T, TY><<<grid, MT_TPB, mt_matvec_smem<T, TY>(), c->s>>>(c->g, coefs_of(cb, o), X.u, X.v, X.p, Y.u, Y.v,
                                                                        Y.p, T(dt), 1, active, &c->ks->matvecs);
  CKL("k_matvec_tile");
}

template <typename T>
void lin(fugu_ctx* c, Trip<T> y, Trip<T> x, double s1 = 0, const double* c1 = nullptr, Trip<T> z1 = {},
         double s2 = 0, const double* c2 = nullptr, Trip<T> z2 = {}, double s3 = 0,
         const double* c3 = nullptr, Trip<T> z3 = {}, const int* active = nullptr) {
  Lin<T> L;
  L.x = x.base; L.z1 = z1.base; L.z2 = z2.base; L.z3 = z3.base;
  L.c1 = c1; L.c2 = c2; L.c3 = c3;
  L.s1 = s1; L.s2 = s2; L.s3 = s3;
  const long n3 = 3 * c->n;
  k_lin<T><<<grid1d(c, n3), 256, 0, c->s>>>(n3, y.base, L, active);
  CKL("k_lin");
}

template <typename T>
void dot_op(fugu_ctx* c, std::initializer_list<std::pair<Trip<T>, Trip<T>>> pairs, OpArgs op,
            bool check_active) {
  DotArgs<T> d;
  d.g = c->g;
  d.n = c->n;
  int k = 0;
  for (auto& pr : pairs) {
    d.a[k] = pr.first.base;
    d.b[k] = pr.second.base;
    ++k;
  }
  for (; k < 5; ++k) { d.a[k] = nullptr; d.b[k] = nullptr; }
  d.npairs = (int)pairs.size();
  d.vol = c->g.dx * c->g.dy;
  d.part = c->part;
  d.sc = c->sc;
  d.ks = c->ks;
  d.op = op;
  d.check_active = check_active ? 1 : 0;
  k_dot_op<T><<<c->dot_grid, DOT_TPB, 0, c->s>>>(d);
  CKL("k_dot_op");
}
void scalar_op(fugu_ctx* c, OpArgs op, bool check_active) {
  k_scalar_op<<<1, 1, 0, c->s>>>(op, c->sc, c->ks, check_active ? 1 : 0);
  CKL("k_scalar_op");
}

// cluster-resident PCG: kernel for a cells-per-thread count
template <typename T>
const void* pcgc_fn(int cpt) {
  switch (cpt) {
    case 1: return (const void*)k_pcg_cluster<T, 1>;
    case 2: return (const void*)k_pcg_cluster<T, 2>;
    case 4: return (const void*)k_pcg_cluster<T, 4>;
    case 8: return (const void*)k_pcg_cluster<T, 8>;
    case 16: return (const void*)k_pcg_cluster<T, 16>;
    case 32:
      if constexpr (sizeof(T) == 4) return (const void*)k_pcg_cluster<T, 32>;
      break;
  }
  return nullptr;
}
template <typename T>
cudaLaunchConfig_t pcgc_cfg(int C, size_t smem, cudaStream_t s, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(PCGC_TPB, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}
template <typename T>
cudaError_t launch_pcg_cluster(PcgClusterArgs<T> a, int C, int cpt, size_t smem, cudaStream_t s) {
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = pcgc_cfg<T>(C, smem, s, at);
  void* args[] = {&a};
  return cudaLaunchKernelExC(&cfg, pcgc_fn<T>(cpt), args);
}
// Plan the cluster-resident PCG for precision T: up to 16 CTAs of PCGC_TPB
// threads, every CTA's rows must fit the shared memory and the register
// arrays (cpt <= 8 in FP64, <= 32 in FP32 with the lean variant above 16),
// and the device must be able to co-schedule such a cluster.
template <typename T>
void plan_pcg_cluster(fugu_ctx* c, fugu_ctx::ClusterPlan& pl) {
  pl = fugu_ctx::ClusterPlan{};
  const char* env = std::getenv("FUGU_PCG");
  if (env && std::strcmp(env, "grid") == 0) return;
  const int nx = c->prm.nx, ny = c->prm.ny;
  const int cmax = ny < c->max_cluster ? ny : c->max_cluster;
  const int rows_per = (ny + cmax - 1) / cmax;
  const int C = (ny + rows_per - 1) / rows_per;
  // every thread owns one column and a strip of cpt rows: nx * strips <= TPB
  if (nx > PCGC_TPB) return;
  int cpt = 1;
  while ((long)nx * ((rows_per + cpt - 1) / cpt) > PCGC_TPB) cpt *= 2;
  const int cpt_max = sizeof(T) == 8 ? 8 : 32;
  if (cpt > cpt_max) return;
  const void* fn = pcgc_fn<T>(cpt);
  // The dynamic shared-memory limit is a property of the kernel, shared by
  // every context in the process, so it is always raised to the device's
  // maximum (never to one case's need, which would shrink it for another).
  int optin = 0;
  cudaFuncAttributes fa;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, fn) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const size_t smem = sizeof(T) * (size_t)pcgc_smem_elems<T>(nx, rows_per, cpt);
  const size_t smem_cap = (size_t)optin - fa.sharedSizeBytes;
  if (smem > smem_cap) return;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap) != cudaSuccess ||
      cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = pcgc_cfg<T>(C, smem, c->s, at);
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess || nclusters < 1) {
    cudaGetLastError();
    return;
  }
  pl.ok = true;
  pl.C = C;
  pl.rows_per = rows_per;
  pl.cpt = cpt;
  pl.smem = smem;
}

// Launch a persistent kernel whose CTAs wait on one another at grid
// barriers.  A context alone uses a cooperative launch, which makes all CTAs
// co-resident.  In a batch, many cases' kernels share the device and two
// partly resident cooperative grids could each wait for CTAs the other's
// occupy (until the bounded barrier gives up), so there the grid is launched
// as one thread-block cluster (at most 8 CTAs), whose CTAs the hardware
// schedules together or not at all.  Both forms are launch attributes, so a
// stream capture records them as attributes of the kernel node.
void launch_coop(fugu_ctx* c, const void* fn, int grid, void** args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(PCG_TPB);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->s;
  cudaLaunchAttribute at[1];
  if (c->coop_as_cluster) {
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = grid;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
  } else {
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
  }
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (c->capturing) c->capture_coop = true;
  CK(cudaLaunchKernelExC(&cfg, fn, args));
}

cudaEvent_t ev_get(fugu_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}
// fold the recorded PCG launch intervals into the profile (stream synced)
void prof_drain(fugu_ctx* c) {
  for (auto& pr : c->ev_pcg) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
    c->prof_pcg_ms += ms;
    c->prof_pcg_launches += 1;
    c->ev_pool.push_back(pr.first);
    c->ev_pool.push_back(pr.second);
  }
  c->ev_pcg.clear();
}

// persistent PCG (solve_poisson_pressure)
template <typename T>
void pcg(fugu_ctx* c, PcgWork<T>& w, T* phi, const T* rhs, double tol, int max_iter, bool phi_zero,
         const int* active) {
  PcgArgs<T> a{};
  a.g = c->g;
  a.rhs = rhs; a.cx = w.cx; a.cy = w.cy; a.dinv = w.dinv;
  a.phi = phi; a.r = w.r; a.z = w.z; a.pb0 = w.pb0; a.pb1 = w.pb1; a.ap = w.ap;
  a.part = c->part; a.gs = c->gs; a.out = c->pcg_out; a.active = active;
  a.tol = tol; a.max_iter = max_iter; a.phi_zero = phi_zero ? 1 : 0;
  const fugu_ctx::ClusterPlan& cp = c->pcgc[sizeof(T) == 8 ? 0 : 1];
  // timed: profiling, and not inside a captured step that is not sampled
  const bool rec = c->prof && (!c->capturing || c->capturing->timed);
  a.timed = rec ? 1 : 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rec) {
    if (c->capturing) {  // a captured step records its own pairs, as graph nodes
      fugu_ctx::StepGraph& sg = *c->capturing;
      if (sg.ev_used >= sg.ev.size()) throw ApiError{FUGU_EINVAL, "captured step: too many PCG launches"};
      e0 = sg.ev[sg.ev_used].first;
      e1 = sg.ev[sg.ev_used].second;
      ++sg.ev_used;
      CK(cudaEventRecordWithFlags(e0, c->s, cudaEventRecordExternal));
    } else {
      e0 = ev_get(c);
      e1 = ev_get(c);
      CK(cudaEventRecord(e0, c->s));
    }
  }
  // an armed failure-detection test takes the grid-wide kernel (the one with
  // software waits) for this launch only; never inside a capture
  const bool armed = c->test_spin_limit > 0 && !c->capturing;
  if (armed) {
    a.spin_limit = c->test_spin_limit;
    a.extra_arrivals = 1;
    c->test_spin_limit = 0;
  }
  if (cp.ok && !armed) {
    PcgClusterArgs<T> ca;
    ca.g = c->g;
    ca.rhs = rhs; ca.cx = w.cx; ca.cy = w.cy; ca.dinv = w.dinv; ca.phi = phi;
    ca.out = c->pcg_out; ca.active = active; ca.tol = tol; ca.max_iter = max_iter;
    ca.phi_zero = phi_zero ? 1 : 0; ca.rows_per = cp.rows_per; ca.timed = a.timed;
    CK(launch_pcg_cluster<T>(ca, cp.C, cp.cpt, cp.smem, c->s));
  } else {
    CK(cudaMemsetAsync(c->gs, 0, sizeof(GridSync), c->s));
    void* args[] = {&a};
    if constexpr (sizeof(T) == 4) {
      // the FP32 inner solve: one grid barrier per iteration
      a.w1 = w.w1;
      a.pv = w.pv;
      launch_coop(c, (const void*)k_pcg1<T>, c->pcg_grid, args);
    } else {
      launch_coop(c, (const void*)k_pcg<T>, c->pcg_grid, args);
    }
  }
  ++c->launches;
  if (rec) {
    if (c->capturing) {
      CK(cudaEventRecordWithFlags(e1, c->s, cudaEventRecordExternal));
    } else {
      CK(cudaEventRecord(e1, c->s));
      c->ev_pcg.push_back({e0, e1});
    }
  }
}

template <typename T>
void poisson_coefs(fugu_ctx* c, PcgWork<T>& w, const double* rho_u, const double* rho_v) {
  Box b = box_launch(c->g);
  k_poisson_coefs<T><<<b.grid, b.block, 0, c->s>>>(c->g, rho_u, rho_v, w.cx, w.cy, w.dinv);
  CKL("k_poisson_coefs");
}

// The vectorised row kernels (VW elements of a row per thread, kernels.cuh)
// run when fugu_params.vec_rows is 1, or 0 with a box of at least auto_min
// points, and every array they touch is 16-byte aligned.  Same bits as the
// one-thread-per-element kernels.  The size rule, from CUDA-event timings on
// a B200 (FP32, us per launch): the PCD steps and single sweeps gain from
// 1024^2 up (k_pcd_zwork 8.2 -> 6.2, one Jacobi sweep 12.3 -> 10.2) and lose
// below (a sweep at 512^2 4.7 -> 5.7); against the staged multi-sweep kernel
// of wall-bounded cases, six vector sweeps lose at 1024^2 (61 against 55)
// and win at 2048^2 (154 against 187), hence the larger bound there.
constexpr long VEC_ROWS_AUTO = 1L << 20;
constexpr long VEC_ROWS_AUTO_WALL_SWEEPS = 1L << 21;
bool vec_rows_on(const fugu_ctx* c, std::initializer_list<const void*> ps, long auto_min = VEC_ROWS_AUTO) {
  const int m = c->prm.vec_rows;
  if (m < 0 || (m == 0 && c->n < auto_min)) return false;
  for (const void* p : ps)
    if (reinterpret_cast<uintptr_t>(p) & 15u) return false;
  return true;
}
template <typename T>
dim3 vec_grid(const Geo& g) {
  constexpr int cols = VEC_TX * VecW<T>::value;
  return dim3((g.P + cols - 1) / cols, (g.R + VEC_TY - 1) / VEC_TY);
}

// damped-Jacobi smoother: n sweeps of solve_helmholtz_{u,v} in place on sol
template <typename T>
void helmholtz(fugu_ctx* c, bool is_u, T* sol, T* tmp, const T* rhs, const CoefBufs<T>& cb,
               const SolveOpt& o, double dt, int n_sweeps, const int* active) {
  Box b = box_launch(c->g);
  T* cur = sol;
  T* nxt = tmp;
  const T* pen = o.pen ? (is_u ? cb.pen_u : cb.pen_v) : nullptr;
  if (c->prm.pcd_smoother == 1 && !c->g.px && !c->g.py) {
    // red-black SOR, both colours of a sweep in one launch, alternating
    // between sol and tmp (extension)
    const dim3 grid((c->g.P + RB_TX - 1) / RB_TX, (c->g.R + RB_TY - 1) / RB_TY);
    for (int s = 0; s < n_sweeps; ++s) {
      k_rbsor_sweep<T><<<grid, RB_TPB, 0, c->s>>>(c->g, is_u ? 0 : 1, cur, nxt, rhs, is_u ? cb.rho_u : cb.rho_v,
                                                  cb.kappa, cb.zeta, cb.eta, pen, T(dt), T(c->prm.pcd_sor_omega),
                                                  active);
      CKL("k_rbsor_sweep");
      std::swap(cur, nxt);
    }
    if (cur != sol) CK(cudaMemcpyAsync(sol, cur, sizeof(T) * c->n, cudaMemcpyDeviceToDevice, c->s));
    return;
  }
  if (c->prm.pcd_smoother == 1) {  // red-black SOR in place, one launch per colour (periodic cases)
    for (int s = 0; s < n_sweeps; ++s)
      for (int col = 0; col < 2; ++col) {
        halo(c, sol, is_u ? K_U : K_V, active);
        if (is_u)
          k_rbsor_u<T><<<b.grid, b.block, 0, c->s>>>(c->g, sol, rhs, cb.rho_u, cb.kappa, cb.zeta, cb.eta, pen,
                                                     T(dt), T(c->prm.pcd_sor_omega), col, active);
        else
          k_rbsor_v<T><<<b.grid, b.block, 0, c->s>>>(c->g, sol, rhs, cb.rho_v, cb.kappa, cb.zeta, cb.eta, pen,
                                                     T(dt), T(c->prm.pcd_sor_omega), col, active);
        CKL("k_rbsor");
      }
    return;
  }
  const T* rho = is_u ? cb.rho_u : cb.rho_v;
  const bool walls = !c->g.px && !c->g.py;
  if (vec_rows_on(c, {sol, tmp, rhs, rho, cb.kappa, cb.zeta, cb.eta, pen},
                  walls ? VEC_ROWS_AUTO_WALL_SWEEPS : VEC_ROWS_AUTO)) {
    // one sweep per launch, VW faces per thread, alternating buffers
    const dim3 grid = vec_grid<T>(c->g);
    for (int s = 0; s < n_sweeps; ++s) {
      halo(c, cur, is_u ? K_U : K_V, active);
      k_jacobi_vec<T><<<grid, dim3(VEC_TX, VEC_TY), 0, c->s>>>(c->g, is_u ? 0 : 1, cur, nxt, rhs, rho, cb.kappa,
                                                               cb.zeta, cb.eta, pen, T(dt), T(c->prm.jacobi_omega),
                                                               active);
      CKL("k_jacobi_vec");
      std::swap(cur, nxt);
    }
    if (cur != sol) CK(cudaMemcpyAsync(sol, cur, sizeof(T) * c->n, cudaMemcpyDeviceToDevice, c->s));
    return;
  }
  if (!c->g.px && !c->g.py) {
    // up to JM_K sweeps per launch on staged tiles, alternating between sol
    // and tmp
    const dim3 grid((c->g.P + JM_TX - 1) / JM_TX, (c->g.R + JM_TY - 1) / JM_TY);
    for (int s = 0; s < n_sweeps; s += JM_K) {
      const int k = std::min(JM_K, n_sweeps - s);
      k_jacobi_multi<T><<<grid, JM_TPB, sizeof(JmSmem<T>), c->s>>>(
          c->g, is_u ? 0 : 1, k, cur, nxt, rhs, is_u ? cb.rho_u : cb.rho_v, cb.kappa, cb.zeta, cb.eta, pen, T(dt),
          T(c->prm.jacobi_omega), active);
      CKL("k_jacobi_multi");
      std::swap(cur, nxt);
    }
    if (cur != sol) CK(cudaMemcpyAsync(sol, cur, sizeof(T) * c->n, cudaMemcpyDeviceToDevice, c->s));
    return;
  }
  for (int s = 0; s < n_sweeps; ++s) {
    halo(c, cur, is_u ? K_U : K_V, active);
    if (is_u)
      k_jacobi_u<T><<<b.grid, b.block, 0, c->s>>>(c->g, cur, nxt, rhs, cb.rho_u, cb.kappa, cb.zeta, cb.eta, pen,
                                                  T(dt), T(c->prm.jacobi_omega), active);
    else
      k_jacobi_v<T><<<b.grid, b.block, 0, c->s>>>(c->g, cur, nxt, rhs, cb.rho_v, cb.kappa, cb.zeta, cb.eta, pen,
                                                  T(dt), T(c->prm.jacobi_omega), active);
    CKL("k_jacobi");
    std::swap(cur, nxt);
  }
  if (cur != sol) CK(cudaMemcpyAsync(sol, cur, sizeof(T) * c->n, cudaMemcpyDeviceToDevice, c->s));
}

// apply_pcd_precond, mod_pcd_precond.f90:14-104: z -> r
template <typename T>
void pcd(fugu_ctx* c, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o, Trip<T> z, Trip<T> r,
         double dt, const int* active) {
  PcdWork<T>& pw = w.pcd;
  Box b = box_launch(c->g);
  // r = zero; phi_p = zero (mod_pcd_precond.f90:44-47).  Plain memsets run
  // even after an exit; the output of an exited iteration is never read.
  CK(cudaMemsetAsync(r.base, 0, sizeof(T) * 3 * c->n, c->s));
  CK(cudaMemsetAsync(pw.phi, 0, sizeof(T) * c->n, c->s));
  pcg<T>(c, w.pcg, pw.phi, z.p, c->prm.pcg_tol, c->pcg_cap_cur > 0 ? c->pcg_cap_cur : c->prm.pcg_max_iter, true,
         active);
  halo(c, pw.phi, K_CELL, active);
  const bool vec = vec_rows_on(c, {pw.phi, cb.u_adv, cb.v_adv, r.p, cb.kappa, z.p, z.u, z.v, pw.zuw, pw.zvw,
                                   cb.eta, r.v});
  const dim3 vg = vec_grid<T>(c->g), vb(VEC_TX, VEC_TY);
  if (vec)
    k_pcd_schur_vec<T><<<vg, vb, 0, c->s>>>(c->g, pw.phi, cb.u_adv, cb.v_adv, r.p, T(1.0 / dt), cb.kappa, z.p,
                                            T(c->prm.pcd_visc_scale), active);
  else
    k_pcd_schur<T><<<b.grid, b.block, 0, c->s>>>(c->g, pw.phi, cb.u_adv, cb.v_adv, r.p, T(1.0 / dt), cb.kappa, z.p,
                                                  T(c->prm.pcd_visc_scale), active);
  CKL("k_pcd_schur");
  halo(c, r.p, K_CELL, active);
  if (vec)
    k_pcd_zwork_vec<T><<<vg, vb, 0, c->s>>>(c->g, z.u, z.v, r.p, pw.zuw, pw.zvw, active);
  else
    k_pcd_zwork<T><<<b.grid, b.block, 0, c->s>>>(c->g, z.u, z.v, r.p, pw.zuw, pw.zvw, active);
  CKL("k_pcd_zwork");
  const int sweeps = c->pcd_sweeps_cur > 0 ? c->pcd_sweeps_cur : c->prm.pcd_sweeps;
  helmholtz<T>(c, false, r.v, pw.tmp, pw.zvw, cb, o, dt, sweeps, active);
  halo(c, r.v, K_V, active);
  if (vec)
    k_pcd_cross_vec<T><<<vg, vb, 0, c->s>>>(c->g, cb.eta, r.v, pw.zuw, active);
  else
    k_pcd_cross<T><<<b.grid, b.block, 0, c->s>>>(c->g, cb.eta, r.v, pw.zuw, active);
  CKL("k_pcd_cross");
  helmholtz<T>(c, true, r.u, pw.tmp, pw.zuw, cb, o, dt, sweeps, active);
  halo(c, r.u, K_U, active);
}

template <typename T>
void zero_trip(fugu_ctx* c, Trip<T> t) {
  CK(cudaMemsetAsync(t.base, 0, sizeof(T) * 3 * c->n, c->s));
}

// restart the Krylov flags (the matvec counter survives; it is per step)
void reset_ks(fugu_ctx* c) {
  static const KState k0 = {1, 0, 0, 0u, 1, 0ull};
  CK(cudaMemcpyAsync(c->ks, &k0, offsetof(KState, matvecs), cudaMemcpyHostToDevice, c->s));
}
// poll the device Krylov state (one round trip)
KState read_ks(fugu_ctx* c) {
  CK(cudaMemcpyAsync(c->h_ks, c->ks, sizeof(KState), cudaMemcpyDeviceToHost, c->s));
  sync(c);
  return *c->h_ks;
}
double read_slot(fugu_ctx* c, int slot) {
  CK(cudaMemcpyAsync(c->h_sc, c->sc + slot, sizeof(double), cudaMemcpyDeviceToHost, c->s));
  sync(c);
  return c->h_sc[0];
}

struct KrylovResult {
  int iter = 0;
  double res = 0.0;
  int status = FUGU_CONVERGED;
};

void graph_prof_read(fugu_ctx* c);

// Krylov iterations of precision pi (0 FP64, 1 FP32) replay from graphs
bool graphs_on(const fugu_ctx* c, int pi) { return c->prm.graphs == 1 && (c->pcgc[pi].ok || c->coop_graphs); }

// Run body() on the context's stream from a CUDA graph: the captured graph
// is replayed while key (every value its launches depend on) is unchanged;
// otherwise body() is captured again and the executable graph updated in
// place (or instantiated anew when its topology changed).  Capture is
// thread-local, so other host threads (a batch) keep launching meanwhile.
template <typename F>
void run_graphed(fugu_ctx* c, fugu_ctx::StepGraph& sg, std::vector<unsigned char>&& key, bool timed, F body) {
  if (!sg.exec || sg.key != key) {
    // event pairs for the PCG launches of a timed body (at most 4: BiCGStab(2)
    // applies PCD four times per iteration), created before the capture
    sg.timed = timed;
    while (timed && sg.ev.size() < 4) {
      cudaEvent_t a, b;
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      sg.ev.push_back({a, b});
    }
    sg.ev_used = 0;
    cudaGraph_t graph = nullptr;
    const unsigned long long l0 = c->launches;
    // a capture or an instantiation that fails with a grid-wide kernel in it:
    // no more such graphs in this context, and this body runs eagerly (the
    // failed capture launched nothing)
    auto coop_fallback = [&]() {
      if (!c->capture_coop || !c->coop_graphs) return false;
      c->coop_graphs = false;
      c->capture_coop = false;
      cudaGetLastError();
      sg.timed = false;
      body();
      return true;
    };
    c->capture_coop = false;
    CK(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
    c->capturing = &sg;
    try {
      body();
    } catch (...) {
      c->capturing = nullptr;
      c->launches = l0;
      cudaStreamEndCapture(c->s, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      if (coop_fallback()) return;
      throw;
    }
    c->capturing = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->s, &graph);
    sg.launches = c->launches - l0;
    c->launches = l0;
    if (ec != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (coop_fallback()) return;
      throw CudaError{ec, "cudaStreamEndCapture"};
    }
    bool updated = false;
    if (sg.exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(sg.exec, graph, &info) == cudaSuccess) {
        updated = true;
      } else {
        cudaGetLastError();
        cudaGraphExecDestroy(sg.exec);
        sg.exec = nullptr;
      }
    }
    if (!updated) {
      const cudaError_t e = cudaGraphInstantiate(&sg.exec, graph, 0);
      if (e != cudaSuccess) {
        sg.exec = nullptr;
        cudaGraphDestroy(graph);
        if (coop_fallback()) return;
        throw CudaError{e, "cudaGraphInstantiate"};
      }
    }
    cudaGraphDestroy(graph);
    sg.key = std::move(key);
  }
  // the PCG intervals of the step replayed before this one are read while
  // this one runs (its events completed at the step's synchronisation), or
  // before the launch when this replay is about to record the same events
  if (c->pcg_timed == &sg) graph_prof_read(c);
  CK(cudaGraphLaunch(sg.exec, c->s));
  c->launches += sg.launches;
  graph_prof_read(c);
  if (sg.timed) c->pcg_timed = &sg;
}

// fold the PCG intervals of the last replayed step graph into the profile
// (once the stream passed it, before a replay of it records them again)
void graph_prof_read(fugu_ctx* c) {
  if (!c->pcg_timed) return;
  for (size_t i = 0; i < c->pcg_timed->ev_used; ++i) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->pcg_timed->ev[i].first, c->pcg_timed->ev[i].second));
    c->prof_pcg_ms += ms;
    c->prof_pcg_launches += 1;
  }
  c->pcg_timed = nullptr;
}

template <typename V>
void key_put(std::vector<unsigned char>& k, const V& v) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), b, b + sizeof(V));
}

// what a captured BiCGStab(l) iteration depends on
template <typename T>
std::vector<unsigned char> krylov_key(fugu_ctx* c, const KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o,
                                      Trip<T> X, double dt, double tol) {
  std::vector<unsigned char> key;
  key_put(key, w.t[0].base); key_put(key, cb); key_put(key, o); key_put(key, X.base); key_put(key, dt);
  key_put(key, tol); key_put(key, c->pcg_cap_cur); key_put(key, c->pcd_sweeps_cur); key_put(key, c->adj_on);
  key_put(key, c->prm); key_put(key, c->prof);
  return key;
}

// bicgstab_solve, mod_bicgstab2.f90:77-264
template <typename T>
KrylovResult bicgstab1(fugu_ctx* c, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o, Trip<T> X,
                       Trip<T> B, double dt, double tol, int max_iter, bool has_lid, double lid) {
  Trip<T>&bh = w.t[0], &r = w.t[1], &r0 = w.t[2], &p = w.t[3], &v = w.t[4], &s = w.t[5], &t = w.t[6],
  &z = w.t[7];
  const int* act = &c->ks->active;
  double* sc = c->sc;
  reset_ks(c);
  vbcs(c, X.u, X.v, 0.0);
  pcd<T>(c, w, cb, o, B, bh, dt, nullptr);
  dot_op<T>(c, {{bh, bh}}, OpArgs{OP_NORMB, 0, tol}, false);
  matvec<T>(c, cb, o, X, z, dt, nullptr);
  pcd<T>(c, w, cb, o, z, v, dt, nullptr);
  lin<T>(c, r, bh, -1.0, sc + S_ONE, v);
  CK(cudaMemcpyAsync(r0.base, r.base, sizeof(T) * 3 * c->n, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(p.base, r.base, sizeof(T) * 3 * c->n, cudaMemcpyDeviceToDevice, c->s));
  dot_op<T>(c, {{r0, r}, {r, r}}, OpArgs{OP_B1_INIT, 1, tol}, false);
  KState ks = read_ks(c);
  // graphs = 1: one captured iteration, replayed for every k (k on the device)
  const int pi = sizeof(T) == 8 ? 0 : 1;
  const bool graphed = graphs_on(c, pi);
  int k = 1;
  for (; k <= max_iter && ks.active; ++k) {
    NvtxRange r_it("bicgstab_iteration");
    const int kk = graphed ? -1 : k;
    auto iteration = [&] {
      vbcs(c, p.u, p.v, 0.0, act);
      matvec<T>(c, cb, o, p, z, dt, act);
      pcd<T>(c, w, cb, o, z, v, dt, act);
      vbcs(c, v.u, v.v, 0.0, act);
      dot_op<T>(c, {{r0, v}}, OpArgs{OP_B1_ALPHA, kk, tol}, true);
      lin<T>(c, s, r, -1.0, sc + S_ALPHA, v, 0, nullptr, {}, 0, nullptr, {}, act);
      vbcs(c, s.u, s.v, 0.0, act);
      matvec<T>(c, cb, o, s, z, dt, act);
      pcd<T>(c, w, cb, o, z, t, dt, act);
      vbcs(c, t.u, t.v, 0.0, act);
      dot_op<T>(c, {{t, t}, {t, s}}, OpArgs{OP_B1_OMEGA, kk, tol}, true);
      lin<T>(c, X, X, 1.0, sc + S_ALPHA, p, 1.0, sc + S_OMEGA, s, 0, nullptr, {}, act);
      lin<T>(c, r, s, -1.0, sc + S_OMEGA, t, 0, nullptr, {}, 0, nullptr, {}, act);
      dot_op<T>(c, {{r, r}, {r0, r}}, OpArgs{OP_B1_END, kk, tol}, true);
      k_pupdate<T><<<grid1d(c, 3 * c->n), 256, 0, c->s>>>(3 * c->n, p.base, r.base, v.base, sc + S_BETA,
                                                            sc + S_OMEGA, act);
      CKL("k_pupdate");
      vbcs(c, X.u, X.v, 0.0, act);
    };
    if (graphed)
      run_graphed(c, c->kr_graphs[pi][0], krylov_key(c, w, cb, o, X, dt, tol), c->prof != 0, iteration);
    else
      iteration();
    ks = read_ks(c);
  }
  graph_prof_read(c);
  if (has_lid) vbcs(c, X.u, X.v, lid);
  ks = read_ks(c);
  KrylovResult res;
  res.iter = ks.active ? max_iter : (ks.exit_iter < max_iter ? ks.exit_iter : max_iter);
  res.res = read_slot(c, S_REL);
  res.status = ks.nan ? FUGU_NAN : (ks.active ? FUGU_MAXITER : (res.res < tol ? FUGU_CONVERGED : FUGU_BREAKDOWN));
  return res;
}

// bicgstab2_solve, mod_bicgstab2.f90:270-570
template <typename T>
KrylovResult bicgstab2(fugu_ctx* c, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o, Trip<T> X,
                       Trip<T> B, double dt, double tol, int max_iter, bool has_lid, double lid) {
  Trip<T>&bh = w.t[0], &r = w.t[1], &rt = w.t[2], &uu = w.t[3], &vv = w.t[4], &ww = w.t[5], &ss = w.t[6],
  &tt = w.t[7], &z = w.t[8], &q = w.t[9];
  const int* act = &c->ks->active;
  double* sc = c->sc;
  reset_ks(c);
  vbcs(c, X.u, X.v, 0.0);
  pcd<T>(c, w, cb, o, B, bh, dt, nullptr);
  dot_op<T>(c, {{bh, bh}}, OpArgs{OP_NORMB, 0, tol}, false);
  matvec<T>(c, cb, o, X, z, dt, nullptr);
  pcd<T>(c, w, cb, o, z, q, dt, nullptr);
  lin<T>(c, r, bh, -1.0, sc + S_ONE, q);
  CK(cudaMemcpyAsync(rt.base, r.base, sizeof(T) * 3 * c->n, cudaMemcpyDeviceToDevice, c->s));
  zero_trip(c, uu);
  zero_trip(c, vv);
  dot_op<T>(c, {{r, r}}, OpArgs{OP_B2_INIT, 1, tol}, false);
  KState ks = read_ks(c);
  // graphs = 1: one captured iteration, replayed for every k (k on the device)
  const int pi = sizeof(T) == 8 ? 0 : 1;
  const bool graphed = graphs_on(c, pi);
  int k = 1;
  for (; k <= max_iter && ks.active; ++k) {
    NvtxRange r_it("bicgstab2_iteration");
    const int kk = graphed ? -1 : k;
    auto iteration = [&] {
      // even half
      dot_op<T>(c, {{rt, r}}, OpArgs{OP_B2_XI_EVEN, kk, tol}, true);
      lin<T>(c, uu, r, -1.0, sc + S_BETA, uu, 0, nullptr, {}, 0, nullptr, {}, act);
      vbcs(c, uu.u, uu.v, 0.0, act);
      matvec<T>(c, cb, o, uu, z, dt, act);
      pcd<T>(c, w, cb, o, z, vv, dt, act);
      vbcs(c, vv.u, vv.v, 0.0, act);
      dot_op<T>(c, {{rt, vv}}, OpArgs{OP_B2_GAMMA, kk, tol}, true);
      lin<T>(c, r, r, -1.0, sc + S_ALPHA, vv, 0, nullptr, {}, 0, nullptr, {}, act);
      if (c->prm.krylov_bc_fix) vbcs(c, r.u, r.v, 0.0, act);
      matvec<T>(c, cb, o, r, z, dt, act);
      pcd<T>(c, w, cb, o, z, ss, dt, act);
      vbcs(c, ss.u, ss.v, 0.0, act);
      lin<T>(c, X, X, 1.0, sc + S_ALPHA, uu, 0, nullptr, {}, 0, nullptr, {}, act);
      // odd half
      dot_op<T>(c, {{rt, ss}}, OpArgs{OP_B2_XI_ODD, kk, tol}, true);
      lin<T>(c, vv, ss, -1.0, sc + S_BETA, vv, 0, nullptr, {}, 0, nullptr, {}, act);
      vbcs(c, vv.u, vv.v, 0.0, act);
      matvec<T>(c, cb, o, vv, z, dt, act);
      pcd<T>(c, w, cb, o, z, ww, dt, act);
      vbcs(c, ww.u, ww.v, 0.0, act);
      dot_op<T>(c, {{rt, ww}}, OpArgs{OP_B2_GAMMA, kk, tol}, true);
      lin<T>(c, uu, r, -1.0, sc + S_BETA, uu, 0, nullptr, {}, 0, nullptr, {}, act);
      lin<T>(c, r, r, -1.0, sc + S_ALPHA, vv, 0, nullptr, {}, 0, nullptr, {}, act);
      lin<T>(c, ss, ss, -1.0, sc + S_ALPHA, ww, 0, nullptr, {}, 0, nullptr, {}, act);
      matvec<T>(c, cb, o, ss, z, dt, act);
      pcd<T>(c, w, cb, o, z, tt, dt, act);
      vbcs(c, tt.u, tt.v, 0.0, act);
      // GCR(2)
      dot_op<T>(c, {{r, ss}, {ss, ss}, {ss, tt}, {tt, tt}, {r, tt}}, OpArgs{OP_B2_GCR, kk, tol}, true);
      lin<T>(c, X, X, 1.0, sc + S_OM1, r, 1.0, sc + S_OM2, ss, 1.0, sc + S_ALPHA, uu, act);
      lin<T>(c, r, r, -1.0, sc + S_OM1, ss, -1.0, sc + S_OM2, tt, 0, nullptr, {}, act);
      lin<T>(c, uu, uu, -1.0, sc + S_OM1, vv, -1.0, sc + S_OM2, ww, 0, nullptr, {}, act);
      dot_op<T>(c, {{r, r}}, OpArgs{OP_B2_REL, kk, tol}, true);
      vbcs(c, X.u, X.v, 0.0, act);
      scalar_op(c, OpArgs{OP_TOPCHECK, graphed ? -1 : k + 1, tol}, true);
    };
    if (graphed)
      run_graphed(c, c->kr_graphs[pi][1], krylov_key(c, w, cb, o, X, dt, tol), c->prof != 0, iteration);
    else
      iteration();
    ks = read_ks(c);
  }
  graph_prof_read(c);
  if (has_lid) vbcs(c, X.u, X.v, lid);
  ks = read_ks(c);
  KrylovResult res;
  res.iter = ks.active ? max_iter : (ks.exit_iter < max_iter ? ks.exit_iter : max_iter);
  res.res = read_slot(c, S_REL);
  res.status = ks.nan ? FUGU_NAN : (ks.active ? FUGU_MAXITER : (res.res < tol ? FUGU_CONVERGED : FUGU_BREAKDOWN));
  return res;
}

template <typename T>
FgWork<T>& fg_work(fugu_ctx* c);
template <>
FgWork<double>& fg_work<double>(fugu_ctx* c) { return c->fg64; }
template <>
FgWork<float>& fg_work<float>(fugu_ctx* c) { return c->fg32; }

template <typename T>
FgWork<T>& ensure_fg(fugu_ctx* c, int m) {
  FgWork<T>& f = fg_work<T>(c);
  if (f.cap < m) {
    f.V = dalloc<T>(c, (long)(m + 1) * 3 * c->n);
    f.Z = dalloc<T>(c, (long)m * 3 * c->n);
    f.st = dalloc<double>(c, FgLayout{m}.size());
    f.cap = m;
  }
  return f;
}

template <typename T>
Trip<T> trip_at(T* base, int i, long n) {
  Trip<T> t;
  t.base = base + (long)i * 3 * n;
  t.u = t.base;
  t.v = t.base + n;
  t.p = t.base + 2 * n;
  return t;
}

template <typename T>
void mdot(fugu_ctx* c, const T* w, const T* V0, int nvec, int op, int j, double tol, FgLayout L, double* st) {
  MdotArgs<T> a;
  a.g = c->g;
  a.n = c->n;
  a.w = w;
  a.V0 = V0;
  a.stride = 3 * c->n;
  a.nvec = nvec;
  a.vol = c->g.dx * c->g.dy;
  a.part = c->part;
  a.st = st;
  a.ks = c->ks;
  a.L = L;
  a.op = op;
  a.j = j;
  a.tol = tol;
  // about four CTAs per SM over all vectors (enough loads in flight when the
  // vectors stream from HBM), each with a work item per warp
  const long per_cta = MDOT_TPB / 32;
  long G = (4L * c->nsm + nvec - 1) / nvec;
  const long gmax = (mdot_items(c->g) + per_cta - 1) / per_cta;
  if (G > gmax) G = gmax;
  if (G < 1) G = 1;
  if (nvec > MDOT_MAXV || 2L * nvec * G > c->part_len) throw ApiError{FUGU_EINVAL, "k_mdot: too many vectors"};
  k_mdot<T><<<dim3((unsigned)G, (unsigned)nvec), MDOT_TPB, 0, c->s>>>(a);
  CKL("k_mdot");
}

// flexible GMRES(m), right PCD preconditioning, one cycle from X = 0
// (extension; the inner solve of refine_solve when refine = 2)
template <typename T>
KrylovResult fgmres(fugu_ctx* c, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o, Trip<T> X, Trip<T> B,
                    double dt, double tol, int m) {
  FgWork<T>& f = ensure_fg<T>(c, m);
  const FgLayout L{m};
  const long n3 = 3 * c->n;
  const int g1 = grid1d(c, n3);
  Trip<T>& wv = w.t[0];
  const int* act = &c->ks->active;
  reset_ks(c);
  CK(cudaMemsetAsync(f.st, 0, sizeof(double) * L.size(), c->s));
  mdot<T>(c, B.base, B.base, 1, FG_BETA, 0, tol, L, f.st);
  k_fg_scale<T><<<g1, 256, 0, c->s>>>(n3, f.V, B.base, f.st + L.inv(), act);
  CKL("k_fg_scale");
  KState ks = read_ks(c);
  // graphs = 1: each Arnoldi step is replayed from a CUDA graph; while
  // profiling, the graph records the PCG interval on its own event pair,
  // read after each step
  const int pi = sizeof(T) == 8 ? 0 : 1;
  const bool graphed = graphs_on(c, pi);
  if (graphed && (int)c->fg_graphs[pi].size() < m) {
    // a solve that ended in an error may have left a sample pending in the
    // vector that is about to move
    if (c->pcg_timed && c->pcg_timed >= c->fg_graphs[pi].data() &&
        c->pcg_timed < c->fg_graphs[pi].data() + c->fg_graphs[pi].size())
      c->pcg_timed = nullptr;
    c->fg_graphs[pi].resize(m);
  }
  auto arnoldi_step_j = [&](int j) {
    Trip<T> Vj = trip_at(f.V, j, c->n), Zj = trip_at(f.Z, j, c->n);
    pcd<T>(c, w, cb, o, Vj, Zj, dt, act);
    vbcs(c, Zj.u, Zj.v, 0.0, act);
    matvec<T>(c, cb, o, Zj, wv, dt, act);
    // classical Gram-Schmidt, twice
    mdot<T>(c, wv.base, f.V, j + 1, FG_PROJ1, j, tol, L, f.st);
    k_maxpy<T><<<g1, 256, 0, c->s>>>(n3, wv.base, f.V, n3, f.st + L.h(), j + 1, -1.0, act);
    CKL("k_maxpy");
    mdot<T>(c, wv.base, f.V, j + 1, FG_PROJ2, j, tol, L, f.st);
    k_maxpy<T><<<g1, 256, 0, c->s>>>(n3, wv.base, f.V, n3, f.st + L.h(), j + 1, -1.0, act);
    CKL("k_maxpy");
    mdot<T>(c, wv.base, wv.base, 1, FG_ROTATE, j, tol, L, f.st);
    k_fg_scale<T><<<g1, 256, 0, c->s>>>(n3, f.V + (long)(j + 1) * n3, wv.base, f.st + L.inv(), act);
    CKL("k_fg_scale");
  };
  for (int j = 0; j < m && ks.active; ++j) {
    NvtxRange r_it("arnoldi_step");
    auto arnoldi_step = [&] { arnoldi_step_j(j); };
    if (graphed) {
      std::vector<unsigned char> key;
      key_put(key, j); key_put(key, m); key_put(key, f.V); key_put(key, f.Z); key_put(key, f.st);
      key_put(key, wv.base); key_put(key, cb); key_put(key, o); key_put(key, dt); key_put(key, tol);
      key_put(key, c->pcg_cap_cur); key_put(key, c->pcd_sweeps_cur); key_put(key, c->adj_on);
      // profiling samples the PCG of the first Arnoldi step of each cycle:
      // event-record nodes split a graph's launch sequence, so timing every
      // step would slow the replay it measures
      const bool timed = c->prof && j == 0;
      key_put(key, c->prm); key_put(key, timed);
      run_graphed(c, c->fg_graphs[pi][j], std::move(key), timed, arnoldi_step);
    } else {
      arnoldi_step();
    }
    ks = read_ks(c);
  }
  graph_prof_read(c);
  const int k = ks.active ? m : ks.exit_iter;
  KrylovResult res;
  if (k > 0) {
    k_fg_solve<<<1, 32, 0, c->s>>>(f.st, L, k);
    CKL("k_fg_solve");
    k_maxpy<T><<<g1, 256, 0, c->s>>>(n3, X.base, f.Z, n3, f.st + L.y(), k, 1.0, nullptr);
    CKL("k_maxpy");
  }
  CK(cudaMemcpyAsync(c->h_sc, f.st + L.rel(), sizeof(double), cudaMemcpyDeviceToHost, c->s));
  sync(c);
  res.iter = k;
  res.res = c->h_sc[0];
  res.status = ks.nan ? FUGU_NAN : (res.res < tol ? FUGU_CONVERGED : FUGU_MAXITER);
  return res;
}

template <typename T>
KrylovResult krylov_inner(fugu_ctx* c, int solver, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o,
                          Trip<T> X, Trip<T> B, double dt, double tol, int max_iter, bool has_lid, double lid) {
  if (solver == 2) return bicgstab2<T>(c, w, cb, o, X, B, dt, tol, max_iter, has_lid, lid);
  return bicgstab1<T>(c, w, cb, o, X, B, dt, tol, max_iter, has_lid, lid);
}

// inner solve of the defect correction: flexible GMRES when refine = 2,
// else the step's BiCGStab(l)
template <typename T>
KrylovResult refine_inner(fugu_ctx* c, int solver, KrylovWork<T>& w, const CoefBufs<T>& cb, const SolveOpt& o,
                          Trip<T> X, Trip<T> B, double dt) {
  if (c->prm.refine == 2) return fgmres<T>(c, w, cb, o, X, B, dt, c->prm.refine_inner_tol, c->prm.refine_max_inner);
  return krylov_inner<T>(c, solver, w, cb, o, X, B, dt, c->prm.refine_inner_tol, c->prm.refine_max_inner, false, 0.0);
}

void ensure_w32(fugu_ctx* c) {
  if (c->w32_ready) return;
  KrylovWork<float>& w = c->w32;
  for (auto& t : w.t) t = talloc<float>(c);
  w.pcd.phi = dalloc<float>(c, c->n); w.pcd.zuw = dalloc<float>(c, c->n);
  w.pcd.zvw = dalloc<float>(c, c->n); w.pcd.tmp = dalloc<float>(c, c->n);
  PcgWork<float>& p = w.pcg;
  p.cx = dalloc<float>(c, c->n); p.cy = dalloc<float>(c, c->n); p.dinv = dalloc<float>(c, c->n);
  p.r = dalloc<float>(c, c->n); p.z = dalloc<float>(c, c->n); p.pb0 = dalloc<float>(c, c->n);
  p.pb1 = dalloc<float>(c, c->n); p.ap = dalloc<float>(c, c->n);
  p.w1 = dalloc<float>(c, c->n); p.pv = dalloc<float>(c, c->n);
  CoefBufs<float>& f = w.cf;
  f.u_adv = dalloc<float>(c, c->n); f.v_adv = dalloc<float>(c, c->n); f.rho_c = dalloc<float>(c, c->n);
  f.rho_u = dalloc<float>(c, c->n); f.rho_v = dalloc<float>(c, c->n); f.kappa = dalloc<float>(c, c->n);
  f.zeta = dalloc<float>(c, c->n); f.eta = dalloc<float>(c, c->n); f.pen_u = dalloc<float>(c, c->n);
  f.pen_v = dalloc<float>(c, c->n); f.mdu = dalloc<float>(c, c->n); f.mdv = dalloc<float>(c, c->n);
  c->w32_ready = true;
}

void cvt(fugu_ctx* c, float* dst, const double* src) {
  if (!src) return;
  k_convert<float><<<grid1d(c, c->n), 256, 0, c->s>>>(c->n, dst, src, 1.0);
  CKL("k_convert");
}

// FP64 defect correction (extension): X += inner(B - A X) until the true
// relative residual |B - A X| / |B| < tol (coupled_dot norm).
KrylovResult refine_solve(fugu_ctx* c, int solver, const CoefBufs<double>& cb64, const SolveOpt& o,
                          Trip<double> X, Trip<double> B, double dt, double tol, bool has_lid, double lid,
                          int* outer_out) {
  KrylovWork<double>& w = c->w64;
  Trip<double>&r = w.t[10], &d = w.t[11], &ax = w.t[12];
  const bool mixed = c->prm.precision == FUGU_MIXED;
  if (mixed) {
    ensure_w32(c);
    CoefBufs<float>& f = c->w32.cf;
    cvt(c, f.u_adv, cb64.u_adv); cvt(c, f.v_adv, cb64.v_adv); cvt(c, f.rho_c, cb64.rho_c);
    cvt(c, f.rho_u, cb64.rho_u); cvt(c, f.rho_v, cb64.rho_v); cvt(c, f.kappa, cb64.kappa);
    cvt(c, f.zeta, cb64.zeta); cvt(c, f.eta, cb64.eta);
    if (o.pen) { cvt(c, f.pen_u, cb64.pen_u); cvt(c, f.pen_v, cb64.pen_v); }
    if (o.amp) { cvt(c, f.mdu, cb64.mdu); cvt(c, f.mdv, cb64.mdv); }
    poisson_coefs<float>(c, c->w32.pcg, cb64.rho_u, cb64.rho_v);
  }
  reset_ks(c);
  vbcs(c, X.u, X.v, 0.0);
  dot_op<double>(c, {{B, B}}, OpArgs{OP_REF_NORMB, 0, tol}, false);
  KrylovResult res;
  int outer = 0, inner_total = 0;
  double rel = 0.0;
  // adaptive PCG cap of the PCD (refine = 2 with pcg_cap_start > 0): start
  // from the cap the previous solve ended with (at least pcg_cap_start),
  // double it after a pass whose inner solve missed its tolerance; the guard
  // restores the fixed cap however the solve ends
  const bool adapt = c->prm.refine == 2 && c->prm.pcg_cap_start > 0;
  // likewise the PCD's Jacobi sweeps once the cap cannot grow
  const bool adapt_sw = c->prm.refine == 2 && c->prm.pcd_sweeps_max > c->prm.pcd_sweeps;
  struct CapGuard {
    fugu_ctx* c;
    ~CapGuard() {
      c->pcg_cap_cur = 0;
      c->pcd_sweeps_cur = 0;
    }
  } cap_guard{c};
  if (adapt)
    c->pcg_cap_cur = std::min(std::max(c->prm.pcg_cap_start, c->pcg_cap_state), c->prm.pcg_max_iter);
  if (adapt_sw)
    c->pcd_sweeps_cur = std::min(std::max(c->prm.pcd_sweeps, c->pcd_sweeps_state), c->prm.pcd_sweeps_max);
  for (;; ++outer) {
    NvtxRange r_pass("defect_correction_pass");
    matvec<double>(c, cb64, o, X, ax, dt, nullptr);
    lin<double>(c, r, B, -1.0, c->sc + S_ONE, ax);
    dot_op<double>(c, {{r, r}}, OpArgs{OP_REF_REL, 0, tol}, false);
    rel = read_slot(c, S_TRUEREL);
    KState ks = read_ks(c);
    if (ks.nan || std::isnan(rel)) { res.status = FUGU_NAN; break; }
    if (rel < tol) { res.status = FUGU_CONVERGED; break; }
    if (outer >= c->prm.refine_max_outer) { res.status = FUGU_MAXITER; break; }
    KrylovResult ir;
    if (mixed) {
      // the defect is scaled to unit norm before the FP32 solve (range safety)
      KrylovWork<float>& w32 = c->w32;
      Trip<float> r32 = w32.t[10], d32 = w32.t[11];
      const long n3 = 3 * c->n;
      k_convert_scaled<float><<<grid1d(c, n3), 256, 0, c->s>>>(n3, r32.base, r.base, c->sc + S_INVRNORM);
      CKL("k_convert_scaled");
      zero_trip(c, d32);
      ir = refine_inner<float>(c, solver, w32, w32.cf, o, d32, r32, dt);
      k_accumulate<float><<<grid1d(c, n3), 256, 0, c->s>>>(n3, X.base, d32.base, c->sc + S_RNORM);
      CKL("k_accumulate");
    } else {
      zero_trip(c, d);
      ir = refine_inner<double>(c, solver, w, cb64, o, d, r, dt);
      lin<double>(c, X, X, 1.0, c->sc + S_ONE, d);
    }
    inner_total += ir.iter;
    if (!(ir.res < c->prm.refine_inner_tol)) {
      if (adapt && c->pcg_cap_cur < c->prm.pcg_max_iter)
        c->pcg_cap_cur = std::min(2 * c->pcg_cap_cur, c->prm.pcg_max_iter);
      else if (adapt_sw && c->pcd_sweeps_cur < c->prm.pcd_sweeps_max)
        c->pcd_sweeps_cur = std::min(2 * c->pcd_sweeps_cur, c->prm.pcd_sweeps_max);
    }
    reset_ks(c);
    vbcs(c, X.u, X.v, 0.0);
  }
  if (has_lid) vbcs(c, X.u, X.v, lid);
  if (adapt) c->pcg_cap_state = c->pcg_cap_cur;
  if (adapt_sw) c->pcd_sweeps_state = c->pcd_sweeps_cur;
  res.iter = inner_total;
  res.res = rel;
  if (outer_out) *outer_out = outer;
  return res;
}

}  // namespace

// ===================================================================== step
namespace {

Mix mix_of(const fugu_params& p) { return Mix{p.rho1, p.rho2, p.mu1, p.mu2}; }

void properties(fugu_ctx* c, const double* cf, double* rho_c, double* rho_u, double* rho_v, double* kappa,
                double* zeta, double* eta) {
  Box b = box_launch(c->g);
  k_properties<<<b.grid, b.block, 0, c->s>>>(c->g, mix_of(c->prm), cf, rho_c, rho_u, rho_v, kappa, zeta, eta);
  CKL("k_properties");
}

// vof_advection_tvd (mod_vof.f90:38-140)
void vof(fugu_ctx* c, const double* cin, double* cout, const double* u, const double* v, double dt, double* fx,
         double* fy) {
  Box b = box_launch(c->g);
  k_vof_update<<<b.grid, b.block, 0, c->s>>>(c->g, c->prm.limiter, cin, u, v, dt, cout);
  CKL("k_vof_update");
  if (fx && fy) {
    k_vof_fluxes<<<b.grid, b.block, 0, c->s>>>(c->g, c->prm.limiter, cin, u, v, dt, fx, fy);
    CKL("k_vof_fluxes");
    halo(c, fx, K_U);
    halo(c, fy, K_V);
  }
  halo(c, cout, K_CELL);
}

// svof_helmholtz_filter (mod_vof.f90:145-194); returns nothing, adds the
// iteration count to c->svof_iters
void svof(fugu_ctx* c, const double* craw, double* cs, double* work, double delta, int max_iter, double tol) {
  SvofArgs a;
  a.g = c->g;
  a.craw = craw;
  a.out = cs;
  a.work = work;
  a.cx = (delta / c->g.dx) * (delta / c->g.dx);
  a.cy = (delta / c->g.dy) * (delta / c->g.dy);
  a.diag = 1.0 + 2.0 * (a.cx + a.cy);
  a.max_iter = max_iter;
  a.tol = tol;
  a.part = c->part;
  a.gs = c->gs;
  a.iters = c->svof_iters;
  a.status = c->svof_status;
  CK(cudaMemsetAsync(c->gs, 0, sizeof(GridSync), c->s));
  void* args[] = {&a};
  launch_coop(c, (const void*)k_svof, c->svof_grid, args);
  ++c->launches;
}

void curvature(fugu_ctx* c, const double* cs, double* kc) {
  Box b = box_launch(c->g);
  k_curvature<<<b.grid, b.block, 0, c->s>>>(c->g, cs, kc);
  CKL("k_curvature");
}
void csf(fugu_ctx* c, const double* cf, const double* kc, double* fu, double* fv) {
  Box b = box_launch(c->g);
  k_csf<<<b.grid, b.block, 0, c->s>>>(c->g, c->prm.sigma, cf, kc, fu, fv);
  CKL("k_csf");
}

void reset_counters(fugu_ctx* c) {
  CK(cudaMemsetAsync(&c->ks->matvecs, 0, sizeof(unsigned long long), c->s));
  CK(cudaMemsetAsync(c->pcg_out, 0, sizeof(PcgOut), c->s));
  CK(cudaMemsetAsync(c->svof_iters, 0, sizeof(int), c->s));
  CK(cudaMemsetAsync(c->svof_status, 0, sizeof(int), c->s));
  // a barrier that gave up in an earlier call left its flag set; a call that
  // takes the cluster PCG never clears it otherwise
  CK(cudaMemsetAsync(c->gs, 0, sizeof(GridSync), c->s));
}
// read statistics and the device-wait status; a barrier timeout is an error
void collect(fugu_ctx* c, fugu_stats* st) {
  CK(cudaMemcpyAsync(c->h_pcg, c->pcg_out, sizeof(PcgOut), cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(c->h_int, c->svof_iters, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(c->h_int + 1, c->svof_status, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(c->h_int + 2, &c->gs->error, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  sync(c);
  if (c->h_int[1] || c->h_int[2] || c->h_pcg->status)
    throw ApiError{FUGU_ETIMEOUT, "a persistent kernel's grid barrier gave up waiting"};
  if (st) {
    st->pcg_iters = (long long)c->h_pcg->total_iters;
    st->pcg_calls = (int)c->h_pcg->calls;
    st->svof_iters = c->h_int[0];
  }
  if (c->prof) {
    prof_drain(c);
    c->prof_pcg_iters += c->h_pcg->total_iters;
    c->prof_pcg_iters_timed += c->h_pcg->timed_iters;
    c->prof_pcg_cells = (unsigned long long)c->prm.nx * c->prm.ny;
  }
}

CoefBufs<double> coef64(fugu_ctx* c, const double* u_adv, const double* v_adv) {
  CoefBufs<double> b;
  b.u_adv = (double*)u_adv;
  b.v_adv = (double*)v_adv;
  b.rho_c = c->f[FUGU_F_RHO_C];
  b.rho_u = c->f[FUGU_F_RHO_U];
  b.rho_v = c->f[FUGU_F_RHO_V];
  b.kappa = c->f[FUGU_F_KAPPA];
  b.zeta = c->f[FUGU_F_ZETA];
  b.eta = c->f[FUGU_F_ETA];
  b.pen_u = c->pen_u;
  b.pen_v = c->pen_v;
  b.mdu = c->mdu;
  b.mdv = c->mdv;
  return b;
}

// the solve used by the step and by fugu_krylov_solve
KrylovResult solve(fugu_ctx* c, int solver, const CoefBufs<double>& cb, const SolveOpt& o, Trip<double> X,
                   Trip<double> B, double dt, double tol, int max_iter, bool has_lid, double lid, int* outer) {
  poisson_coefs<double>(c, c->w64.pcg, cb.rho_u, cb.rho_v);
  if (c->prm.refine) return refine_solve(c, solver, cb, o, X, B, dt, tol, has_lid, lid, outer);
  if (outer) *outer = 0;
  return krylov_inner<double>(c, solver, c->w64, cb, o, X, B, dt, tol, max_iter, has_lid, lid);
}

// the settings of one step that its stages share
struct StepSetup {
  bool amp, pen, bdf2;
  double tol, lid, dt_eff;
  int max_it;
};
StepSetup step_setup(const fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o) {
  const fugu_params& p = c->prm;
  StepSetup s;
  s.amp = o->consistent_amp != 0;
  s.pen = o->has_penalty != 0;
  s.tol = o->has_tol ? o->tol : p.tol_bicgstab2;
  s.max_it = o->has_max_iter ? o->max_iter : p.max_iter_bicgstab2;
  s.lid = o->has_lid ? o->u_top_lid : 0.0;
  s.bdf2 = (p.time_order == 2 && step_idx >= 2);
  s.dt_eff = s.bdf2 ? dt / 1.5 : dt;
  return s;
}

// advance_coupled_step, mod_solver_coupled.f90:137-380, before the solve:
// the explicit stages 1-6 up to the right-hand side
void step_pre(fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o) {
  const fugu_params& p = c->prm;
  double** f = c->f;
  const long n = c->n;
  const StepSetup su = step_setup(c, dt, step_idx, o);
  const bool amp = su.amp, pen = su.pen, bdf2 = su.bdf2;
  const double lid = su.lid;
  reset_counters(c);
  // 1. AB extrapolation u_adv = 2u^n - u^(n-1); u_prev <- u^n (u_prev then holds u^n)
  k_extrapolate<<<grid1d(c, n), 256, 0, c->s>>>(n, f[FUGU_F_U_VEL], f[FUGU_F_U_PREV], c->u_nm1, c->u_adv,
                                                 step_idx <= 1);
  k_extrapolate<<<grid1d(c, n), 256, 0, c->s>>>(n, f[FUGU_F_V_VEL], f[FUGU_F_V_PREV], c->v_nm1, c->v_adv,
                                                 step_idx <= 1);
  CKL("k_extrapolate");
  const double* u_n = f[FUGU_F_U_PREV];
  const double* v_n = f[FUGU_F_V_PREV];
  // 2. VOF transport with u^n (+ AMP mass fluxes)
  {
  NvtxRange r_vof("vof_transport");
  vof(c, f[FUGU_F_C_FIELD], c->c_new, u_n, v_n, dt, amp ? c->fcx : nullptr, amp ? c->fcy : nullptr);
  if (amp) {
    k_axpby<<<grid1d(c, n), 256, 0, c->s>>>(n, c->mdu, p.rho1 - p.rho2, c->fcx, p.rho2, c->u_adv);
    k_axpby<<<grid1d(c, n), 256, 0, c->s>>>(n, c->mdv, p.rho1 - p.rho2, c->fcy, p.rho2, c->v_adv);
    CKL("k_axpby");
  }
  CK(cudaMemcpyAsync(f[FUGU_F_C_FIELD], c->c_new, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->s));
  }
  // 3. properties at t^(n+1)
  properties(c, f[FUGU_F_C_FIELD], f[FUGU_F_RHO_C], f[FUGU_F_RHO_U], f[FUGU_F_RHO_V], f[FUGU_F_KAPPA],
             f[FUGU_F_ZETA], f[FUGU_F_ETA]);
  // 4. SVOF + curvature + CSF
  if (p.sigma > 1.0e-14) {
    NvtxRange r_st("svof_curvature_csf");
    const double delta = p.svof_delta_h * (c->g.dx < c->g.dy ? c->g.dx : c->g.dy);
    svof(c, f[FUGU_F_C_FIELD], c->c_s, c->svof_w, delta, p.svof_max_iter, p.svof_tol);
    curvature(c, c->c_s, f[FUGU_F_KAPPA_CURV]);
    csf(c, f[FUGU_F_C_FIELD], f[FUGU_F_KAPPA_CURV], f[FUGU_F_F_SIGMA_U], f[FUGU_F_F_SIGMA_V]);
  } else {
    CK(cudaMemsetAsync(f[FUGU_F_KAPPA_CURV], 0, sizeof(double) * n, c->s));
    CK(cudaMemsetAsync(f[FUGU_F_F_SIGMA_U], 0, sizeof(double) * n, c->s));
    CK(cudaMemsetAsync(f[FUGU_F_F_SIGMA_V], 0, sizeof(double) * n, c->s));
  }
  // 5. Darcy penalty
  if (pen) {
    k_axpby<<<grid1d(c, n), 256, 0, c->s>>>(n, c->pen_u, p.alpha_penalty, f[FUGU_F_PHI_S_U], 0.0, nullptr);
    k_axpby<<<grid1d(c, n), 256, 0, c->s>>>(n, c->pen_v, p.alpha_penalty, f[FUGU_F_PHI_S_V], 0.0, nullptr);
    CKL("k_axpby");
  }
  // 6. right-hand side
  RhsArgs ra;
  ra.rho_u = f[FUGU_F_RHO_U]; ra.rho_v = f[FUGU_F_RHO_V];
  ra.u_n = u_n; ra.u_nm1 = c->u_nm1; ra.v_n = v_n; ra.v_nm1 = c->v_nm1;
  ra.fsu = f[FUGU_F_F_SIGMA_U]; ra.fsv = f[FUGU_F_F_SIGMA_V];
  ra.pen_u = pen ? c->pen_u : nullptr; ra.pen_v = pen ? c->pen_v : nullptr;
  ra.zeta = f[FUGU_F_ZETA]; ra.eta = f[FUGU_F_ETA];
  ra.dt = dt; ra.gx = p.gx; ra.gy = p.gy;
  ra.u_sol = o->has_u_solid ? o->u_solid : 0.0;
  ra.v_sol = o->has_v_solid ? o->v_solid : 0.0;
  ra.u_lid = lid;
  ra.bdf2 = bdf2 ? 1 : 0;
  ra.has_lid = o->has_lid ? 1 : 0;
  Box b = box_launch(c->g);
  k_rhs<<<b.grid, b.block, 0, c->s>>>(c->g, ra, c->B.u, c->B.v, c->B.p);
  CKL("k_rhs");
}

// after the solve: 8. final halos and BCs, then the step's statistics
void step_post(fugu_ctx* c, const StepSetup& su, const KrylovResult& kr, int outer, fugu_stats* st) {
  Trip<double> Xc = c->Xstate;
  halo(c, Xc.u, K_U);
  halo(c, Xc.v, K_V);
  halo(c, Xc.p, K_CELL);
  vbcs(c, Xc.u, Xc.v, su.lid);
  collect(c, st);
  if (st) {
    st->iter = kr.iter;
    st->res = kr.res;
    st->outer = outer;
    st->status = kr.status;
    KState ks = read_ks(c);
    st->matvecs = (int)ks.matvecs;
  }
}

// advance_coupled_step, mod_solver_coupled.f90:137-380, on the device state
void step(fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o, fugu_stats* st) {
  NvtxRange r_step("fugu_step");
  const StepSetup su = step_setup(c, dt, step_idx, o);
  step_pre(c, dt, step_idx, o);
  // 7. monolithic solve (u_top_lid is always present in this call); the
  // state u_vel, v_vel, p_field is one contiguous coupled triple
  SolveOpt so;
  so.pen = su.pen;
  so.amp = su.amp;
  CoefBufs<double> cb = coef64(c, c->u_adv, c->v_adv);
  KrylovResult kr;
  int outer = 0;
  {
    NvtxRange r_solve("coupled_solve");
    kr = solve(c, o->use_bicgstab2 ? 2 : 1, cb, so, c->Xstate, c->B, su.dt_eff, su.tol, su.max_it, true, su.lid,
               &outer);
  }
  step_post(c, su, kr, outer, st);
}

}  // namespace

// ================================================================= context
namespace {

int check_params(const fugu_params* p) {
  if (!p) return FUGU_EINVAL;
  if (p->nx < 4 || p->ny < 4 || p->nx > 65536 || p->ny > 65536) return FUGU_EINVAL;
  if (!(p->dx > 0.0) || !(p->dy > 0.0)) return FUGU_EINVAL;
  if (p->pcg_max_iter < 0 || p->pcd_sweeps < 0 || p->svof_max_iter < 0 || p->pcg_cap_start < 0) return FUGU_EINVAL;
  if (p->pcd_sweeps_max < 0 || p->pcd_sweeps_max > 1024) return FUGU_EINVAL;
  // the sweeps double from pcd_sweeps, which must be > 0 for that
  if (p->refine == 2 && p->pcd_sweeps_max > p->pcd_sweeps && p->pcd_sweeps < 1) return FUGU_EINVAL;
  if (p->precision == FUGU_MIXED && !p->refine) return FUGU_EINVAL;
  if (p->refine < 0 || p->refine > 2) return FUGU_EINVAL;
  // flexible GMRES keeps one projection per basis vector in shared memory
  if (p->refine == 2 && (p->refine_max_inner < 1 || p->refine_max_inner > 127)) return FUGU_EINVAL;
  if (p->precision != FUGU_FP64 && p->precision != FUGU_MIXED) return FUGU_EINVAL;
  if (p->pcd_smoother < 0 || p->pcd_smoother > 1) return FUGU_EINVAL;
  if (p->graphs < 0 || p->graphs > 1) return FUGU_EINVAL;
  if (!(p->pcd_visc_scale >= 0.0 && p->pcd_visc_scale < 1.0e6)) return FUGU_EINVAL;
  if (p->vec_rows < -1 || p->vec_rows > 1) return FUGU_EINVAL;
  if (p->pcd_smoother == 1 && !(p->pcd_sor_omega > 0.0 && p->pcd_sor_omega < 2.0)) return FUGU_EINVAL;
  return FUGU_OK;
}

int coop_grid(const void* fn, int tpb, int nsm, long work, int max_ctas) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, tpb, 0) != cudaSuccess || occ < 1) return 0;
  long want = (work + tpb - 1) / tpb;
  long cap = (long)nsm * occ;
  if (cap > nsm) cap = nsm;  // one CTA per SM keeps the barrier short
  if (cap > max_ctas) cap = max_ctas;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

void create(fugu_ctx* c) {
  CK(cudaSetDevice(c->device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, c->device));
  if (!prop.cooperativeLaunch) throw ApiError{FUGU_ECUDA, "device lacks cooperative launch"};
  c->nsm = prop.multiProcessorCount;
  CK(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
  c->g = make_geo(c->prm);
  c->n = c->g.n();
  c->Xstate = talloc<double>(c);
  for (int i = 0; i < FUGU_NUM_FIELDS; ++i) c->f[i] = dalloc<double>(c, c->n);
  c->f[FUGU_F_U_VEL] = c->Xstate.u;
  c->f[FUGU_F_V_VEL] = c->Xstate.v;
  c->f[FUGU_F_P_FIELD] = c->Xstate.p;
  c->u_nm1 = dalloc<double>(c, c->n); c->v_nm1 = dalloc<double>(c, c->n);
  c->u_adv = dalloc<double>(c, c->n); c->v_adv = dalloc<double>(c, c->n);
  c->c_new = dalloc<double>(c, c->n); c->c_s = dalloc<double>(c, c->n); c->svof_w = dalloc<double>(c, c->n);
  c->fcx = dalloc<double>(c, c->n); c->fcy = dalloc<double>(c, c->n);
  c->mdu = dalloc<double>(c, c->n); c->mdv = dalloc<double>(c, c->n);
  c->pen_u = dalloc<double>(c, c->n); c->pen_v = dalloc<double>(c, c->n);
  c->B = talloc<double>(c);
  KrylovWork<double>& w = c->w64;
  for (auto& t : w.t) t = talloc<double>(c);
  w.pcd.phi = dalloc<double>(c, c->n); w.pcd.zuw = dalloc<double>(c, c->n);
  w.pcd.zvw = dalloc<double>(c, c->n); w.pcd.tmp = dalloc<double>(c, c->n);
  PcgWork<double>& p = w.pcg;
  p.cx = dalloc<double>(c, c->n); p.cy = dalloc<double>(c, c->n); p.dinv = dalloc<double>(c, c->n);
  p.r = dalloc<double>(c, c->n); p.z = dalloc<double>(c, c->n); p.pb0 = dalloc<double>(c, c->n);
  p.pb1 = dalloc<double>(c, c->n); p.ap = dalloc<double>(c, c->n);
  // routine-level scratch (c->scratch) is allocated on first use
  c->sc = dalloc<double>(c, NSLOTS);
  c->ks = dalloc<KState>(c, 1);
  const long ncell = (long)c->prm.nx * c->prm.ny;
  c->pcg_grid = coop_grid((const void*)k_pcg<double>, PCG_TPB, c->nsm, ncell, c->max_coop);
  int g32 = coop_grid((const void*)k_pcg<float>, PCG_TPB, c->nsm, ncell, c->max_coop);
  if (g32 < c->pcg_grid) c->pcg_grid = g32;
  g32 = coop_grid((const void*)k_pcg1<float>, PCG_TPB, c->nsm, ncell, c->max_coop);
  if (g32 < c->pcg_grid) c->pcg_grid = g32;
  c->svof_grid = coop_grid((const void*)k_svof, PCG_TPB, c->nsm, ncell, c->max_coop);
  if (c->pcg_grid < 1 || c->svof_grid < 1) throw ApiError{FUGU_ECUDA, "no co-resident grid for persistent kernels"};
  plan_pcg_cluster<double>(c, c->pcgc[0]);
  plan_pcg_cluster<float>(c, c->pcgc[1]);
  // the multi-sweep Jacobi tiles of FP64 need more than the default 48 KB
  CK(cudaFuncSetAttribute((const void*)k_jacobi_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)sizeof(JmSmem<double>)));
  CK(cudaFuncSetAttribute((const void*)k_jacobi_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)sizeof(JmSmem<float>)));
  const char* env = std::getenv("FUGU_PCG");
  if (env && std::strcmp(env, "cluster") == 0 && !(c->pcgc[0].ok && c->pcgc[1].ok))
    throw ApiError{FUGU_EINVAL, "FUGU_PCG=cluster but this grid does not fit a thread-block cluster"};
  c->dot_grid = c->nsm * 2;
  // CTA partials: the reductions' 8 per CTA, or k_mdot's 2 per vector and CTA
  c->part_len = std::max(8L * (c->nsm * 8 + 64), 2L * MDOT_MAXV * c->nsm);
  c->part = dalloc<double>(c, c->part_len);
  c->gs = dalloc<GridSync>(c, 1);
  c->pcg_out = dalloc<PcgOut>(c, 1);
  c->svof_iters = dalloc<int>(c, 1);
  c->svof_status = dalloc<int>(c, 1);
  CK(cudaMallocHost(&c->h_ks, sizeof(KState)));
  CK(cudaMallocHost(&c->h_sc, sizeof(double) * NSLOTS));
  CK(cudaMallocHost(&c->h_pcg, sizeof(PcgOut)));
  CK(cudaMallocHost(&c->h_int, sizeof(int) * 8));
  const double one = 1.0;
  CK(cudaMemcpyAsync(c->sc + S_ONE, &one, sizeof(double), cudaMemcpyHostToDevice, c->s));
  sync(c);
}

void destroy(fugu_ctx* c) {
  if (!c) return;
  if (c->s) cudaStreamSynchronize(c->s);
  for (auto& pr : c->ev_pcg) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  auto drop = [](fugu_ctx::StepGraph& sg) {
    if (sg.exec) cudaGraphExecDestroy(sg.exec);
    for (auto& pr : sg.ev) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  };
  for (auto& v : c->fg_graphs)
    for (auto& sg : v) drop(sg);
  for (auto& pr : c->kr_graphs)
    for (auto& sg : pr) drop(sg);
  for (void* p : c->allocs) cudaFree(p);
  if (c->h_ks) cudaFreeHost(c->h_ks);
  if (c->h_sc) cudaFreeHost(c->h_sc);
  if (c->h_pcg) cudaFreeHost(c->h_pcg);
  if (c->h_int) cudaFreeHost(c->h_int);
  if (c->s) cudaStreamDestroy(c->s);
  delete c;
}

// run fn, translating exceptions into an ABI status and a message
template <typename F>
int guard(fugu_ctx* c, F fn) {
  if (!c) return FUGU_EINVAL;
  try {
    cudaSetDevice(c->device);
    fn();
    return FUGU_OK;
  } catch (const CudaError& e) {
    c->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);
    return FUGU_ECUDA;
  } catch (const ApiError& e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return FUGU_ECUDA;
  }
}

// routine-level helpers: scratch buffer k (single component) / triple view
double* S(fugu_ctx* c, int k) {
  if (!c->scratch[k]) c->scratch[k] = dalloc<double>(c, 3 * c->n);
  return c->scratch[k];
}
Trip<double> ST(fugu_ctx* c, int k) {
  Trip<double> t;
  t.base = S(c, k);
  t.u = t.base;
  t.v = t.base + c->n;
  t.p = t.base + 2 * c->n;
  return t;
}
double* upk(fugu_ctx* c, int k, const double* h, int kind) {
  if (!h) return nullptr;
  up(c, S(c, k), h, kind);
  return S(c, k);
}

}  // namespace

// ================================================================== C ABI
extern "C" {

void fugu_params_default(fugu_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->nx = 64; p->ny = 64; p->dx = 1.0 / 64; p->dy = 1.0 / 64;
  p->rho1 = 1000.0; p->rho2 = 1.0; p->mu1 = 1.0; p->mu2 = 0.01;
  p->sigma = 0.0; p->gx = 0.0; p->gy = -9.81;
  p->cfl_target = 0.5; p->alpha_penalty = 1.0e12; p->time_order = 1;
  p->tol_bicgstab2 = 1.0e-6; p->max_iter_bicgstab2 = 500;
  p->pcg_tol = 1.0e-5; p->pcg_max_iter = 150; p->pcd_sweeps = 3; p->jacobi_omega = 0.8;
  p->svof_delta_h = 1.5; p->svof_max_iter = 150; p->svof_tol = 1.0e-7;
  p->refine_inner_tol = 1.0e-2; p->refine_max_inner = 20; p->refine_max_outer = 30;
  p->precision = FUGU_FP64;
  p->pcd_smoother = 0; p->pcd_sor_omega = 1.0; p->graphs = 0; p->pcd_visc_scale = 0.0; p->vec_rows = 0;
}

const char* fugu_version(void) { return "fugu-b200 1 (sm_100a)"; }

int fugu_create(const fugu_params* p, int device, fugu_ctx** out) {
  if (!out) return FUGU_EINVAL;
  *out = nullptr;
  int rc = check_params(p);
  if (rc) return rc;
  fugu_ctx* c = new fugu_ctx();
  c->prm = *p;
  c->device = device;
  rc = guard(c, [&] { create(c); });
  if (rc) {
    fprintf(stderr, "fugu_create: %s\n", c->err.c_str());
    destroy(c);
    return rc;
  }
  *out = c;
  return FUGU_OK;
}

void fugu_destroy(fugu_ctx* ctx) { destroy(ctx); }

int fugu_set_params(fugu_ctx* c, const fugu_params* p) {
  int rc = check_params(p);
  if (rc || !c) return rc ? rc : FUGU_EINVAL;
  if (p->nx != c->prm.nx || p->ny != c->prm.ny) {
    c->err = "fugu_set_params: the grid size of a context is fixed";
    return FUGU_EINVAL;
  }
  c->prm = *p;
  c->g = make_geo(*p);
  c->pcg_cap_state = 0;  // the adaptive PCG cap and sweeps restart from their starts
  c->pcd_sweeps_state = 0;
  return FUGU_OK;
}

const char* fugu_last_error(const fugu_ctx* c) { return c ? c->err.c_str() : "NULL context"; }

int fugu_get_stream(fugu_ctx* c, void** stream) {
  if (!c || !stream) return FUGU_EINVAL;
  *stream = (void*)c->s;
  return FUGU_OK;
}

int fugu_profile(fugu_ctx* c, int enable, fugu_profile_stats* out) {
  return guard(c, [&] {
    sync(c);
    prof_drain(c);
    graph_prof_read(c);
    if (out) {
      out->kernel_launches = c->launches;
      out->pcg_ms = c->prof_pcg_ms;
      out->pcg_launches = c->prof_pcg_launches;
      out->pcg_iters = c->prof_pcg_iters;
      out->pcg_cells = c->prof_pcg_cells;
      out->pcg_grid = c->pcg_grid;
      out->svof_grid = c->svof_grid;
      out->pcg_cluster_fp64 = c->pcgc[0].ok ? c->pcgc[0].C : 0;
      out->pcg_cluster_fp32 = c->pcgc[1].ok ? c->pcgc[1].C : 0;
      out->pcg_iters_timed = c->prof_pcg_iters_timed;
    }
    if (enable >= 0) {
      c->prof = enable;
      c->launches = 0;
      c->prof_pcg_ms = 0.0;
      c->prof_pcg_launches = c->prof_pcg_iters = c->prof_pcg_iters_timed = 0;
    }
  });
}

int fugu_upload(fugu_ctx* c, int field, const double* host) {
  return guard(c, [&] {
    if (field < 0 || field >= FUGU_NUM_FIELDS) throw ApiError{FUGU_EINVAL, "bad field id"};
    up(c, c->f[field], host, kind_of_field(field));
    sync(c);
  });
}
int fugu_download(fugu_ctx* c, int field, double* host) {
  return guard(c, [&] {
    if (field < 0 || field >= FUGU_NUM_FIELDS) throw ApiError{FUGU_EINVAL, "bad field id"};
    down(c, host, c->f[field], kind_of_field(field));
    sync(c);
  });
}

int fugu_step(fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o, fugu_stats* st) {
  return guard(c, [&] {
    if (!o) throw ApiError{FUGU_EINVAL, "NULL options"};
    if (st) std::memset(st, 0, sizeof(*st));
    step(c, dt, step_idx, o, st);
  });
}

int fugu_advance_coupled_step(fugu_ctx* c, double* u_vel, double* v_vel, double* p_field, double* c_field,
                              double* u_prev, double* v_prev, double* rho_c, double* rho_u, double* rho_v,
                              double* kappa, double* zeta, double* eta, double* kappa_curv, double* f_sigma_u,
                              double* f_sigma_v, const double* phi_s_u, const double* phi_s_v, double dt,
                              int step_idx, const fugu_step_opts* o, fugu_stats* st) {
  return guard(c, [&] {
    if (!o) throw ApiError{FUGU_EINVAL, "NULL options"};
    if (o->has_penalty && (!phi_s_u || !phi_s_v)) throw ApiError{FUGU_EINVAL, "penalty without mask"};
    double* in[] = {u_vel, v_vel, p_field, c_field, u_prev, v_prev, rho_c, rho_u, rho_v,
                    kappa, zeta, eta, kappa_curv, f_sigma_u, f_sigma_v};
    for (int i = 0; i < 15; ++i) up(c, c->f[i], in[i], kind_of_field(i));
    if (o->has_penalty) {
      up(c, c->f[FUGU_F_PHI_S_U], phi_s_u, K_U);
      up(c, c->f[FUGU_F_PHI_S_V], phi_s_v, K_V);
    }
    if (st) std::memset(st, 0, sizeof(*st));
    step(c, dt, step_idx, o, st);
    for (int i = 0; i < 15; ++i) down(c, in[i], c->f[i], kind_of_field(i));
    sync(c);
  });
}

int fugu_compute_adaptive_dt(fugu_ctx* c, const double* u_vel, const double* v_vel, double dt_max,
                             double* dt_out) {
  return guard(c, [&] {
    if (!dt_out) throw ApiError{FUGU_EINVAL, "NULL dt_out"};
    double* u = upk(c, 0, u_vel, K_U);
    double* v = upk(c, 1, v_vel, K_V);
    const int nb = c->nsm;
    k_maxvel<<<nb, 256, 0, c->s>>>(c->g, u, v, c->part);
    CKL("k_maxvel");
    std::vector<double> part(2 * nb);
    CK(cudaMemcpyAsync(part.data(), c->part, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, c->s));
    sync(c);
    double um = 0.0, vm = 0.0;
    for (int b = 0; b < nb; ++b) {
      um = part[2 * b] > um ? part[2 * b] : um;
      vm = part[2 * b + 1] > vm ? part[2 * b + 1] : vm;
    }
    // scalar tail of compute_adaptive_dt (mod_solver_coupled.f90:68-90)
    const fugu_params& p = c->prm;
    const double h = p.dx < p.dy ? p.dx : p.dy;
    const double pi = 3.141592653589793238462643383279502884197;
    double dcfl = (um / p.dx + vm / p.dy > 1.0e-12) ? p.cfl_target / (um / p.dx + vm / p.dy) : dt_max;
    double dtl = dt_max < dcfl ? dt_max : dcfl;
    if (p.sigma > 1.0e-14) {
      const double dcap = 0.5 * std::sqrt((p.rho1 + p.rho2) * (h * h * h) / (4.0 * pi * p.sigma));
      dtl = dtl < dcap ? dtl : dcap;
    }
    const double gm = std::sqrt(p.gx * p.gx + p.gy * p.gy);
    if (gm > 1.0e-14) {
      const double dg = 0.5 * std::sqrt(h / gm);
      dtl = dtl < dg ? dtl : dg;
    }
    *dt_out = dtl;
  });
}

int fugu_build_cylinder_mask(fugu_ctx* c, double xc, double yc, double rad, double* phi_s_u, double* phi_s_v) {
  return guard(c, [&] {
    Box b = box_launch(c->g);
    k_cylinder<<<b.grid, b.block, 0, c->s>>>(c->g, xc, yc, rad, S(c, 0), S(c, 1));
    CKL("k_cylinder");
    halo(c, S(c, 0), K_U);
    halo(c, S(c, 1), K_V);
    down(c, phi_s_u, S(c, 0), K_U);
    down(c, phi_s_v, S(c, 1), K_V);
    sync(c);
  });
}

int fugu_halo_scalar(fugu_ctx* c, double* phi) {
  return guard(c, [&] { upk(c, 0, phi, K_CELL); halo(c, S(c, 0), K_CELL); down(c, phi, S(c, 0), K_CELL); sync(c); });
}
int fugu_halo_u(fugu_ctx* c, double* u) {
  return guard(c, [&] { upk(c, 0, u, K_U); halo(c, S(c, 0), K_U); down(c, u, S(c, 0), K_U); sync(c); });
}
int fugu_halo_v(fugu_ctx* c, double* v) {
  return guard(c, [&] { upk(c, 0, v, K_V); halo(c, S(c, 0), K_V); down(c, v, S(c, 0), K_V); sync(c); });
}

int fugu_compute_mixture_densities(fugu_ctx* c, const double* cf, double* rho_c, double* rho_u, double* rho_v) {
  return guard(c, [&] {
    double* cc = upk(c, 0, cf, K_CELL);
    properties(c, cc, S(c, 1), S(c, 2), S(c, 3), S(c, 4), S(c, 5), S(c, 6));
    down(c, rho_c, S(c, 1), K_CELL);
    down(c, rho_u, S(c, 2), K_U);
    down(c, rho_v, S(c, 3), K_V);
    sync(c);
  });
}
int fugu_compute_mixture_viscosities(fugu_ctx* c, const double* cf, double* kappa, double* zeta, double* eta) {
  return guard(c, [&] {
    double* cc = upk(c, 0, cf, K_CELL);
    properties(c, cc, S(c, 1), S(c, 2), S(c, 3), S(c, 4), S(c, 5), S(c, 6));
    down(c, kappa, S(c, 4), K_CELL);
    down(c, zeta, S(c, 5), K_VERT);
    down(c, eta, S(c, 6), K_VERT);
    sync(c);
  });
}

int fugu_op_divergence(fugu_ctx* c, const double* u, const double* v, double* div) {
  return guard(c, [&] {
    double* du = upk(c, 0, u, K_U);
    double* dv = upk(c, 1, v, K_V);
    Box b = box_launch(c->g);
    k_op_divergence<<<b.grid, b.block, 0, c->s>>>(c->g, du, dv, S(c, 2));
    CKL("k_op_divergence");
    down(c, div, S(c, 2), K_CELL);
    sync(c);
  });
}
int fugu_op_grad_pressure(fugu_ctx* c, const double* p, double* gu, double* gv) {
  return guard(c, [&] {
    double* dp = upk(c, 0, p, K_CELL);
    Box b = box_launch(c->g);
    k_op_grad<<<b.grid, b.block, 0, c->s>>>(c->g, dp, S(c, 1), S(c, 2));
    CKL("k_op_grad");
    down(c, gu, S(c, 1), K_U);
    down(c, gv, S(c, 2), K_V);
    sync(c);
  });
}
int fugu_op_viscous_stress(fugu_ctx* c, const double* u, const double* v, const double* kappa, const double* zeta,
                           const double* eta, double* vu, double* vv) {
  return guard(c, [&] {
    double *du = upk(c, 0, u, K_U), *dv = upk(c, 1, v, K_V), *dk = upk(c, 2, kappa, K_CELL);
    double *dz = upk(c, 3, zeta, K_VERT), *de = upk(c, 4, eta, K_VERT);
    Box b = box_launch(c->g);
    k_op_visc<<<b.grid, b.block, 0, c->s>>>(c->g, du, dv, dk, dz, de, S(c, 5), S(c, 6));
    CKL("k_op_visc");
    down(c, vu, S(c, 5), K_U);
    down(c, vv, S(c, 6), K_V);
    sync(c);
  });
}
int fugu_op_advection(fugu_ctx* c, const double* u_adv, const double* v_adv, const double* rho_c,
                      const double* rho_u, const double* rho_v, const double* u, const double* v, double* adv_u,
                      double* adv_v, const double* mdot_u, const double* mdot_v) {
  return guard(c, [&] {
    Coefs<double> cf{};
    cf.u_adv = upk(c, 0, u_adv, K_U);
    cf.v_adv = upk(c, 1, v_adv, K_V);
    cf.rho_c = upk(c, 2, rho_c, K_CELL);
    cf.rho_u = upk(c, 3, rho_u, K_U);
    cf.rho_v = upk(c, 4, rho_v, K_V);
    const bool cons = mdot_u && mdot_v;
    cf.mdot_u = cons ? upk(c, 5, mdot_u, K_U) : nullptr;
    cf.mdot_v = cons ? upk(c, 6, mdot_v, K_V) : nullptr;
    double *du = upk(c, 7, u, K_U), *dv = upk(c, 8, v, K_V);
    Box b = box_launch(c->g);
    k_op_adv<<<b.grid, b.block, 0, c->s>>>(c->g, cf, du, dv, S(c, 9), S(c, 10));
    CKL("k_op_adv");
    down(c, adv_u, S(c, 9), K_U);
    down(c, adv_v, S(c, 10), K_V);
    sync(c);
  });
}
int fugu_apply_velocity_bcs(fugu_ctx* c, double* u, double* v, int has_lid, double u_lid) {
  return guard(c, [&] {
    upk(c, 0, u, K_U);
    upk(c, 1, v, K_V);
    vbcs(c, S(c, 0), S(c, 1), has_lid ? u_lid : 0.0);
    down(c, u, S(c, 0), K_U);
    down(c, v, S(c, 1), K_V);
    sync(c);
  });
}

}  // extern "C"

namespace {
// coefficient set of a routine-level call: uploads into scratch 4..15
CoefBufs<double> up_coefs(fugu_ctx* c, const double* u_adv, const double* v_adv, const double* rho_c,
                          const double* rho_u, const double* rho_v, const double* kappa, const double* zeta,
                          const double* eta, const double* pen_u, const double* pen_v, const double* mdu,
                          const double* mdv) {
  CoefBufs<double> b;
  b.u_adv = upk(c, 4, u_adv, K_U);
  b.v_adv = upk(c, 5, v_adv, K_V);
  b.rho_c = upk(c, 6, rho_c, K_CELL);
  b.rho_u = upk(c, 7, rho_u, K_U);
  b.rho_v = upk(c, 8, rho_v, K_V);
  b.kappa = upk(c, 9, kappa, K_CELL);
  b.zeta = upk(c, 10, zeta, K_VERT);
  b.eta = upk(c, 11, eta, K_VERT);
  b.pen_u = upk(c, 12, pen_u, K_U);
  b.pen_v = upk(c, 13, pen_v, K_V);
  b.mdu = upk(c, 14, mdu, K_U);
  b.mdv = upk(c, 15, mdv, K_V);
  return b;
}
void up_trip(fugu_ctx* c, Trip<double> t, const double* u, const double* v, const double* p) {
  up(c, t.u, u, K_U);
  up(c, t.v, v, K_V);
  up(c, t.p, p, K_CELL);
}
void down_trip(fugu_ctx* c, Trip<double> t, double* u, double* v, double* p) {
  if (u) down(c, u, t.u, K_U);
  if (v) down(c, v, t.v, K_V);
  if (p) down(c, p, t.p, K_CELL);
}

// colour period of the stencil probe along one direction: 5 on a wall-bounded
// extent; on a periodic one the smallest divisor >= 5 of the extent, so
// colours stay 5 apart across the wrap
int probe_period(int len, bool periodic) {
  if (!periodic) return 5;
  if (len < 5) throw ApiError{FUGU_EINVAL, "the adjoint needs at least 5 cells along a periodic direction"};
  for (int q = 5; q < len; ++q)
    if (len % q == 0) return q;
  return len;
}

// Probe the coupled operator x_owned -> (A . BC(x))_owned (BC: the homogeneous
// wall BCs the Krylov solvers apply before each product) with coloured unit
// vectors and store its stencil in c->adj_val.
void adj_assemble(fugu_ctx* c, const CoefBufs<double>& cb, const SolveOpt& o, double dt) {
  if (!c->adj_val) {
    c->adj_val = dalloc<double>(c, (long)ADJ_SLOTS * c->n);
    c->adj_err = dalloc<unsigned int>(c, 1);
  }
  CK(cudaMemsetAsync(c->adj_val, 0, sizeof(double) * ADJ_SLOTS * c->n, c->s));
  CK(cudaMemsetAsync(c->adj_err, 0, sizeof(unsigned int), c->s));
  const int qx = probe_period(c->g.nx, c->g.px), qy = probe_period(c->g.ny, c->g.py);
  Trip<double> X = ST(c, 16), Y = ST(c, 17);
  Box b = box_launch(c->g);
  const bool was_on = c->adj_on;
  c->adj_on = false;
  for (int cc = 0; cc < 3; ++cc)
    for (int a = 0; a < qx; ++a)
      for (int bb = 0; bb < qy; ++bb) {
        CK(cudaMemsetAsync(X.base, 0, sizeof(double) * 3 * c->n, c->s));
        k_adj_probe_set<<<b.grid, b.block, 0, c->s>>>(c->g, X.base, c->n, cc, qx, qy, a, bb);
        CKL("k_adj_probe_set");
        vbcs(c, X.u, X.v, 0.0);
        matvec<double>(c, cb, o, X, Y, dt, nullptr);
        k_adj_probe_collect<<<b.grid, b.block, 0, c->s>>>(c->g, Y.base, c->n, cc, qx, qy, a, bb, c->adj_val,
                                                          c->adj_err);
        CKL("k_adj_probe_collect");
      }
  c->adj_on = was_on;
  unsigned int err = 0;
  CK(cudaMemcpyAsync(&err, c->adj_err, sizeof(err), cudaMemcpyDeviceToHost, c->s));
  sync(c);
  if (err) throw ApiError{FUGU_ECUDA, "adjoint stencil probe: " + std::to_string(err) +
                                          " operator entries beyond a 2-cell reach"};
}

// Solve A^T X = B on the device: the FP64 defect correction around flexible
// GMRES on S A^T S (S flips the pressure block), then X = S X.  B is
// overwritten.  The context's parameters and its adaptive PCG cap and sweeps
// come back as they were, so the forward steps that follow are unaffected.
KrylovResult adjoint_solve_dev(fugu_ctx* c, const CoefBufs<double>& cb, const SolveOpt& o, double dt, double tol,
                               Trip<double> B, Trip<double> X, int* outer) {
  struct Restore {
    fugu_ctx* c;
    fugu_params prm;
    int cap, sweeps;
    ~Restore() {
      c->prm = prm;
      c->adj_on = false;
      c->pcg_cap_state = cap;
      c->pcd_sweeps_state = sweeps;
    }
  } restore{c, c->prm, c->pcg_cap_state, c->pcd_sweeps_state};
  adj_assemble(c, cb, o, dt);
  zero_trip(c, X);
  const int g1 = grid1d(c, c->n);
  k_adj_flip_p<<<g1, 256, 0, c->s>>>(c->n, B.base);  // S g
  CKL("k_adj_flip_p");
  // inner solve: flexible GMRES, or BiCGStab(2) (the reference's solver on
  // the transposed system) when the context's refine is 1; the defect
  // correction around it in FP64 either way
  c->prm.refine = c->prm.refine == 1 ? 1 : 2;
  c->prm.precision = FUGU_FP64;
  if (c->prm.refine_max_inner < 1 || c->prm.refine_max_inner > 127) c->prm.refine_max_inner = 30;
  c->adj_on = true;
  reset_counters(c);
  KrylovResult kr = solve(c, 2, cb, o, X, B, dt, tol, 0, false, 0.0, outer);
  c->adj_on = false;
  k_adj_flip_p<<<g1, 256, 0, c->s>>>(c->n, X.base);  // lambda = S mu
  CKL("k_adj_flip_p");
  return kr;
}

// ------------------------------------------------ vector-Jacobian product of one step
// Reach (cells, in i and j) of each local stage, which fixes the colour
// period 2R + 1 of its probes: the VOF update reads C two cells away; the
// solve's stage reads C_smooth three cells away (curvature then CSF) and the
// coefficients two; the wall BCs mirror up to four cells (u(-2) = -u(2)).
constexpr int VJP_RA = 2, VJP_RB = 4, VJP_RG = 4;

void vjp_alloc(fugu_ctx* c) {
  VjpWork& w = c->vjp;
  if (w.ready) return;
  auto F = [&] { return dalloc<double>(c, c->n); };
  auto D = [&] { return dalloc<ad::Dual>(c, c->n); };
  w.c0 = F(); w.u0 = F(); w.v0 = F(); w.up0 = F(); w.vp0 = F();
  w.b_u1 = F(); w.b_v1 = F(); w.b_c1 = F(); w.b_up1 = F(); w.b_vp1 = F();
  w.b_c0 = F(); w.b_u0 = F(); w.b_v0 = F(); w.b_up0 = F(); w.b_vp0 = F();
  w.b_cs = F(); w.t1 = F(); w.t2 = F();
  w.g = talloc<double>(c); w.lam = talloc<double>(c); w.resid = talloc<double>(c);
  w.svof_it = dalloc<int>(c, 1);
  w.dc0 = D(); w.du0 = D(); w.dv0 = D(); w.dc1o = D();
  w.dc1 = D(); w.dcs = D(); w.dun = D(); w.dvn = D(); w.dunm1 = D(); w.dvnm1 = D();
  w.drc = D(); w.dru = D(); w.drv = D(); w.dka = D(); w.dze = D(); w.det = D();
  w.dkc = D(); w.dfu = D(); w.dfv = D(); w.dua = D(); w.dva = D();
  for (int q = 0; q < 3; ++q) { w.dB[q] = D(); w.dX[q] = D(); w.dY[q] = D(); }
  w.dgu = D(); w.dgv = D();
  w.ready = true;
}

void vjp_pack(fugu_ctx* c, const double* x, ad::Dual* out, int mask, bool seeded, int s, int a, int b) {
  Box bx = box_launch(c->g);
  k_dual_pack<<<bx.grid, bx.block, 0, c->s>>>(c->g, x, out, mask, seeded ? 1 : 0, s, a, b);
  CKL("k_dual_pack");
}

void vjp_gather(fugu_ctx* c, const VjpOut& o, int mask, int s, int a, int b, int R, double* xbar) {
  const int ti = (c->g.P - a + s - 1) / s, tj = (c->g.R - b + s - 1) / s;
  if (ti <= 0 || tj <= 0) return;
  const dim3 blk(32, 4), grd((ti + 31) / 32, (tj + 3) / 4);
  k_vjp_gather<<<grd, blk, 0, c->s>>>(c->g, o, mask, s, a, b, R, xbar);
  CKL("k_vjp_gather");
}

// one input field of a probed stage: its values, its dual buffer, the
// entries that are inputs, and where its adjoint accumulates
struct VjpIn {
  const double* x;
  ad::Dual* d;
  int mask;
  double* bar;
};

// x_bar += J^T y_bar for every input of a stage: each input field in turn is
// seeded colour by colour while the others carry zero derivatives
template <typename Stage>
void vjp_probe(fugu_ctx* c, VjpIn* in, int nin, const VjpOut& out, int R, Stage&& stage) {
  const int s = 2 * R + 1;
  for (int e = 0; e < nin; ++e) vjp_pack(c, in[e].x, in[e].d, in[e].mask, false, s, 0, 0);
  for (int f = 0; f < nin; ++f) {
    for (int a = 0; a < s; ++a)
      for (int b = 0; b < s; ++b) {
        vjp_pack(c, in[f].x, in[f].d, in[f].mask, true, s, a, b);
        stage();
        vjp_gather(c, out, in[f].mask, s, a, b, R, in[f].bar);
      }
    vjp_pack(c, in[f].x, in[f].d, in[f].mask, false, s, 0, 0);
  }
}

// the VOF stage on duals: C^n, u^n, v^n -> C^(n+1) (vof() without AMP fluxes)
void vjp_stage_vof(fugu_ctx* c, double dt) {
  VjpWork& w = c->vjp;
  Box bx = box_launch(c->g);
  k_vof_update<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(c->g, c->prm.limiter, w.dc0, w.du0, w.dv0, dt, w.dc1o);
  CKL("k_vof_update<Dual>");
  halo(c, w.dc1o, K_CELL);
}

// the solve's stage on duals: C^(n+1), C_smooth, u^n, v^n, u^(n-1), v^(n-1)
// and the parameters -> B and A X with X fixed at the step's solution
// (properties, curvature, CSF, AB extrapolation, right-hand side, matvec)
void vjp_stage_solve(fugu_ctx* c, double dt, double dt_eff, bool bdf2, bool first, const fugu_step_opts* o,
                     const MixT<ad::Dual>& m, ad::Dual sigma) {
  VjpWork& w = c->vjp;
  const Geo& g = c->g;
  const fugu_params& p = c->prm;
  Box bx = box_launch(g);
  k_properties<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, m, w.dc1, w.drc, w.dru, w.drv, w.dka, w.dze, w.det);
  CKL("k_properties<Dual>");
  if (p.sigma > 1.0e-14) {
    k_fill_ghost_neumann<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, w.dcs);
    k_curvature<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, w.dcs, w.dkc);
    k_csf<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, sigma, w.dc1, w.dkc, w.dfu, w.dfv);
    CKL("k_csf<Dual>");
  } else {
    vjp_pack(c, nullptr, w.dfu, VM_U, false, 1, 0, 0);
    vjp_pack(c, nullptr, w.dfv, VM_V, false, 1, 0, 0);
  }
  const int g1 = grid1d(c, c->n);
  k_adv_dual<<<g1, 256, 0, c->s>>>(c->n, w.dun, w.dunm1, w.dua, first ? 1 : 0);
  k_adv_dual<<<g1, 256, 0, c->s>>>(c->n, w.dvn, w.dvnm1, w.dva, first ? 1 : 0);
  CKL("k_adv_dual");
  RhsArgsT<ad::Dual> ra{};
  ra.rho_u = w.dru; ra.rho_v = w.drv;
  ra.u_n = w.dun; ra.u_nm1 = w.dunm1; ra.v_n = w.dvn; ra.v_nm1 = w.dvnm1;
  ra.fsu = w.dfu; ra.fsv = w.dfv;
  ra.pen_u = nullptr; ra.pen_v = nullptr;
  ra.zeta = w.dze; ra.eta = w.det;
  ra.dt = dt; ra.gx = p.gx; ra.gy = p.gy;
  ra.u_sol = o->has_u_solid ? o->u_solid : 0.0;
  ra.v_sol = o->has_v_solid ? o->v_solid : 0.0;
  ra.u_lid = o->has_lid ? o->u_top_lid : 0.0;
  ra.bdf2 = bdf2 ? 1 : 0;
  ra.has_lid = o->has_lid ? 1 : 0;
  k_rhs<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, ra, w.dB[0], w.dB[1], w.dB[2]);
  CKL("k_rhs<Dual>");
  Coefs<ad::Dual> cf{};
  cf.u_adv = w.dua; cf.v_adv = w.dva; cf.rho_c = w.drc; cf.rho_u = w.dru; cf.rho_v = w.drv;
  cf.kappa = w.dka; cf.zeta = w.dze; cf.eta = w.det;
  k_matvec<ad::Dual><<<bx.grid, bx.block, 0, c->s>>>(g, cf, w.dX[0], w.dX[1], w.dX[2], w.dY[0], w.dY[1], w.dY[2],
                                                     ad::Dual(dt_eff), 1, nullptr, nullptr);
  CKL("k_matvec<Dual>");
}

// the step's final BCs on duals: owned velocity -> every velocity entry
void vjp_stage_bc(fugu_ctx* c) {
  VjpWork& w = c->vjp;
  halo(c, w.dgu, K_U);
  halo(c, w.dgv, K_V);
  vbcs(c, w.dgu, w.dgv, 0.0);
}

MixT<ad::Dual> vjp_mix(const fugu_params& p, int seed) {
  // seed: 1 sigma (not here), 2 mu1, 3 mu2, 4 rho1, 5 rho2
  return MixT<ad::Dual>{ad::Dual(p.rho1, seed == 4 ? 1.0 : 0.0), ad::Dual(p.rho2, seed == 5 ? 1.0 : 0.0),
                        ad::Dual(p.mu1, seed == 2 ? 1.0 : 0.0), ad::Dual(p.mu2, seed == 3 ? 1.0 : 0.0)};
}

// The step as a map of the state (u, v, C, u_prev, v_prev) -> (u', v', C',
// u_prev' = u, v_prev' = v) and its transpose applied to the adjoints of the
// state after the step.  The context holds the state before the step and is
// left holding the state after it.
void step_vjp(fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o, const double* const* bar_out,
              double* const* bar_in, double* bar_theta, fugu_stats* st_out) {
  const fugu_params& p = c->prm;
  const Geo& g = c->g;
  if (g.px || g.py) throw ApiError{FUGU_EINVAL, "the step VJP supports wall-bounded boxes only"};
  if (o->consistent_amp) throw ApiError{FUGU_EINVAL, "the step VJP does not support consistent_amp"};
  if (o->has_penalty) throw ApiError{FUGU_EINVAL, "the step VJP does not support the Darcy penalty"};
  for (int q = 0; q < 5; ++q)
    if (!bar_out[q] || !bar_in[q]) throw ApiError{FUGU_EINVAL, "NULL adjoint array"};
  vjp_alloc(c);
  VjpWork& w = c->vjp;
  double** f = c->f;
  const long n = c->n;
  const size_t nb = sizeof(double) * n;
  CK(cudaMemcpyAsync(w.c0, f[FUGU_F_C_FIELD], nb, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(w.u0, f[FUGU_F_U_VEL], nb, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(w.v0, f[FUGU_F_V_VEL], nb, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(w.up0, f[FUGU_F_U_PREV], nb, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(w.vp0, f[FUGU_F_V_PREV], nb, cudaMemcpyDeviceToDevice, c->s));
  // the forward step
  fugu_stats fst;
  std::memset(&fst, 0, sizeof(fst));
  step(c, dt, step_idx, o, &fst);
  const bool bdf2 = (p.time_order == 2 && step_idx >= 2);
  const double dt_eff = bdf2 ? dt / 1.5 : dt;
  const bool first = step_idx <= 1;
  // adjoints after the step
  double* accs[] = {w.b_u1, w.b_v1, w.b_c1, w.b_up1, w.b_vp1, w.b_c0, w.b_u0, w.b_v0, w.b_up0, w.b_vp0, w.b_cs};
  for (double* a : accs) CK(cudaMemsetAsync(a, 0, nb, c->s));
  up(c, w.b_u1, bar_out[0], K_U);
  up(c, w.b_v1, bar_out[1], K_V);
  up(c, w.b_c1, bar_out[2], K_CELL);
  up(c, w.b_up1, bar_out[3], K_U);
  up(c, w.b_vp1, bar_out[4], K_V);
  // 1. the final BCs: fold the adjoints of u', v' onto the owned unknowns
  zero_trip(c, w.g);
  {
    VjpIn in[2] = {{nullptr, w.dgu, VM_OWNED_U, w.g.u}, {nullptr, w.dgv, VM_OWNED_V, w.g.v}};
    VjpOut out{};
    out.y[0] = w.dgu; out.ybar[0] = w.b_u1;
    out.y[1] = w.dgv; out.ybar[1] = w.b_v1;
    out.n = 2;
    vjp_probe(c, in, 2, out, VJP_RG, [&] { vjp_stage_bc(c); });
  }
  // 2. lambda = A^-T g (the step's operator at its coefficients and dt_eff)
  SolveOpt so;
  const double tol = o->has_tol ? o->tol : p.tol_bicgstab2;
  int aouter = 0;
  KrylovResult ak = adjoint_solve_dev(c, coef64(c, c->u_adv, c->v_adv), so, dt_eff, tol, w.g, w.lam, &aouter);
  {
    Box bx = box_launch(g);
    k_keep_owned<<<bx.grid, bx.block, 0, c->s>>>(g, w.lam.base, n);
    CKL("k_keep_owned");
  }
  // 3. the solve's stage: x_bar += (dB/dx - (dA/dx) X)^T lambda
  vjp_pack(c, c->Xstate.u, w.dX[0], VM_U, false, 1, 0, 0);
  vjp_pack(c, c->Xstate.v, w.dX[1], VM_V, false, 1, 0, 0);
  vjp_pack(c, c->Xstate.p, w.dX[2], VM_CELL, false, 1, 0, 0);
  const MixT<ad::Dual> m0 = vjp_mix(p, 0);
  const ad::Dual sig0(p.sigma);
  VjpOut out{};
  for (int q = 0; q < 3; ++q) {
    out.y[q] = w.dB[q];
    out.ysub[q] = w.dY[q];
  }
  out.ybar[0] = w.lam.u; out.ybar[1] = w.lam.v; out.ybar[2] = w.lam.p;
  out.n = 3;
  {
    VjpIn in[6] = {{f[FUGU_F_C_FIELD], w.dc1, VM_CELL, w.b_c1}, {c->c_s, w.dcs, VM_INTERIOR, w.b_cs},
                   {w.u0, w.dun, VM_U, w.b_u0},                 {w.v0, w.dvn, VM_V, w.b_v0},
                   {w.up0, w.dunm1, VM_U, w.b_up0},             {w.vp0, w.dvnm1, VM_V, w.b_vp0}};
    vjp_probe(c, in, 6, out, VJP_RB,
              [&] { vjp_stage_solve(c, dt, dt_eff, bdf2, first, o, m0, sig0); });
    // parameters: theta_bar += (dB/dtheta - (dA/dtheta) X) . lambda
    const double vol = g.dx * g.dy;
    for (int q = 0; q < 5; ++q) {
      const int seed = q + 1;
      vjp_stage_solve(c, dt, dt_eff, bdf2, first, o, vjp_mix(p, seed), ad::Dual(p.sigma, seed == 1 ? 1.0 : 0.0));
      Box bx = box_launch(g);
      k_dual_resid<<<bx.grid, bx.block, 0, c->s>>>(g, w.dB[0], w.dB[1], w.dB[2], w.dY[0], w.dY[1], w.dY[2],
                                                    w.resid.base, n);
      CKL("k_dual_resid");
      dot_op<double>(c, {{w.resid, w.lam}}, OpArgs{OP_STORE, 0, 0.0}, false);
      if (bar_theta) bar_theta[q] += read_slot(c, S_D0) / vol;
    }
  }
  // 4. SVOF: C_smooth = L C^(n+1) with L a polynomial of the symmetric Jacobi
  // iteration matrix (K sweeps), so L^T = L: the same sweeps on C_smooth's adjoint
  if (p.sigma > 1.0e-14 && fst.svof_iters > 0) {
    const double delta = p.svof_delta_h * (g.dx < g.dy ? g.dx : g.dy);
    SvofArgs a;
    a.g = g;
    a.craw = w.b_cs;
    a.out = w.t1;
    a.work = w.t2;
    a.cx = (delta / g.dx) * (delta / g.dx);
    a.cy = (delta / g.dy) * (delta / g.dy);
    a.diag = 1.0 + 2.0 * (a.cx + a.cy);
    a.max_iter = fst.svof_iters;
    a.tol = -1.0;  // no early exit: exactly the forward's sweeps
    a.part = c->part;
    a.gs = c->gs;
    a.iters = w.svof_it;
    a.status = c->svof_status;
    CK(cudaMemsetAsync(c->gs, 0, sizeof(GridSync), c->s));
    void* args[] = {&a};
    launch_coop(c, (const void*)k_svof, c->svof_grid, args);
    ++c->launches;
    Box bx = box_launch(g);
    k_add_interior<<<bx.grid, bx.block, 0, c->s>>>(g, w.t1, w.b_c1);
    CKL("k_add_interior");
  }
  // 5. the VOF stage: C^(n+1)'s whole adjoint back to C^n, u^n, v^n
  {
    VjpIn in[3] = {{w.c0, w.dc0, VM_CELL, w.b_c0}, {w.u0, w.du0, VM_U, w.b_u0}, {w.v0, w.dv0, VM_V, w.b_v0}};
    VjpOut vo{};
    vo.y[0] = w.dc1o;
    vo.ybar[0] = w.b_c1;
    vo.n = 1;
    vjp_probe(c, in, 3, vo, VJP_RA, [&] { vjp_stage_vof(c, dt); });
  }
  // 6. u_prev' = u^n and v_prev' = v^n pass their adjoints through
  const int g1 = grid1d(c, n);
  k_axpby<<<g1, 256, 0, c->s>>>(n, w.b_u0, 1.0, w.b_u0, 1.0, w.b_up1);
  k_axpby<<<g1, 256, 0, c->s>>>(n, w.b_v0, 1.0, w.b_v0, 1.0, w.b_vp1);
  CKL("k_axpby");
  down(c, bar_in[0], w.b_u0, K_U);
  down(c, bar_in[1], w.b_v0, K_V);
  down(c, bar_in[2], w.b_c0, K_CELL);
  down(c, bar_in[3], w.b_up0, K_U);
  down(c, bar_in[4], w.b_vp0, K_V);
  collect(c, nullptr);  // the adjoint SVOF's barrier status
  sync(c);
  if (st_out) {
    *st_out = fst;
    // a converged forward step reports the adjoint solve's outcome
    if (fst.status == FUGU_CONVERGED) st_out->status = ak.status;
    st_out->outer = aouter;
  }
}

}  // namespace

extern "C" {

int fugu_matvec_coupled(fugu_ctx* c, double* Xu, double* Xv, double* Xp, double* Yu, double* Yv, double* Yp,
                        const double* u_adv, const double* v_adv, const double* rho_c, const double* rho_u,
                        const double* rho_v, const double* kappa, const double* zeta, const double* eta,
                        double dt, int include_advection, const double* pen_u, const double* pen_v,
                        const double* mdot_u, const double* mdot_v) {
  return guard(c, [&] {
    CoefBufs<double> cb = up_coefs(c, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta, pen_u, pen_v,
                                   mdot_u, mdot_v);
    SolveOpt o;
    o.pen = pen_u && pen_v;
    o.amp = mdot_u && mdot_v;
    Trip<double> X = ST(c, 0), Y = ST(c, 1);
    up_trip(c, X, Xu, Xv, Xp);
    halo(c, X.u, K_U);
    halo(c, X.v, K_V);
    halo(c, X.p, K_CELL);
    Box b = box_launch(c->g);
    k_matvec<double><<<b.grid, b.block, 0, c->s>>>(c->g, coefs_of(cb, o), X.u, X.v, X.p, Y.u, Y.v, Y.p, dt,
                                                    include_advection ? 1 : 0, nullptr, nullptr);
    CKL("k_matvec");
    down_trip(c, X, Xu, Xv, Xp);
    down_trip(c, Y, Yu, Yv, Yp);
    sync(c);
  });
}

int fugu_solve_poisson_pressure(fugu_ctx* c, double* phi, const double* rhs, const double* rho_u,
                                const double* rho_v, double tol, int max_iter, int* iter_out, double* res_out) {
  return guard(c, [&] {
    double* dphi = upk(c, 0, phi, K_CELL);
    double* drhs = upk(c, 1, rhs, K_CELL);
    double* dru = upk(c, 2, rho_u, K_U);
    double* drv = upk(c, 3, rho_v, K_V);
    reset_counters(c);
    poisson_coefs<double>(c, c->w64.pcg, dru, drv);
    pcg<double>(c, c->w64.pcg, dphi, drhs, tol, max_iter, false, nullptr);
    collect(c, nullptr);
    down(c, phi, dphi, K_CELL);
    CK(cudaMemcpyAsync(c->h_pcg, c->pcg_out, sizeof(PcgOut), cudaMemcpyDeviceToHost, c->s));
    sync(c);
    if (iter_out) *iter_out = c->h_pcg->iters;
    if (res_out) *res_out = c->h_pcg->res;
  });
}

}  // extern "C"

namespace {
int helm_entry(fugu_ctx* c, bool is_u, double* sol, const double* rhs, const double* rho,
                      const double* kappa, const double* zeta, const double* eta, double dt, int n_sweeps,
                      const double* pen) {
  return guard(c, [&] {
    const int kind = is_u ? K_U : K_V;
    double* ds = upk(c, 0, sol, kind);
    double* dr = upk(c, 1, rhs, kind);
    CoefBufs<double> cb;
    if (is_u) cb.rho_u = upk(c, 2, rho, K_U);
    else cb.rho_v = upk(c, 2, rho, K_V);
    cb.kappa = upk(c, 3, kappa, K_CELL);
    cb.zeta = upk(c, 4, zeta, K_VERT);
    cb.eta = upk(c, 5, eta, K_VERT);
    if (is_u) cb.pen_u = upk(c, 6, pen, K_U);
    else cb.pen_v = upk(c, 6, pen, K_V);
    SolveOpt o;
    o.pen = pen != nullptr;
    helmholtz<double>(c, is_u, ds, S(c, 7), dr, cb, o, dt, n_sweeps, nullptr);
    down(c, sol, ds, kind);
    sync(c);
  });
}
}  // namespace

extern "C" {

int fugu_solve_helmholtz_u(fugu_ctx* c, double* u_sol, const double* rhs_u, const double* rho_u,
                           const double* kappa, const double* zeta, const double* eta, double dt, int n_sweeps,
                           const double* penalty_u) {
  return helm_entry(c, true, u_sol, rhs_u, rho_u, kappa, zeta, eta, dt, n_sweeps, penalty_u);
}
int fugu_solve_helmholtz_v(fugu_ctx* c, double* v_sol, const double* rhs_v, const double* rho_v,
                           const double* kappa, const double* zeta, const double* eta, double dt, int n_sweeps,
                           const double* penalty_v) {
  return helm_entry(c, false, v_sol, rhs_v, rho_v, kappa, zeta, eta, dt, n_sweeps, penalty_v);
}

int fugu_apply_pcd_precond(fugu_ctx* c, const double* z_u, const double* z_v, const double* z_p, double* r_u,
                           double* r_v, double* r_p, const double* u_adv, const double* v_adv,
                           const double* rho_u, const double* rho_v, const double* kappa, const double* zeta,
                           const double* eta, double dt, const double* penalty_u, const double* penalty_v) {
  return guard(c, [&] {
    CoefBufs<double> cb = up_coefs(c, u_adv, v_adv, nullptr, rho_u, rho_v, kappa, zeta, eta, penalty_u,
                                   penalty_v, nullptr, nullptr);
    SolveOpt o;
    o.pen = penalty_u && penalty_v;
    Trip<double> Z = ST(c, 0), R = ST(c, 1);
    up_trip(c, Z, z_u, z_v, z_p);
    reset_counters(c);
    poisson_coefs<double>(c, c->w64.pcg, cb.rho_u, cb.rho_v);
    pcd<double>(c, c->w64, cb, o, Z, R, dt, nullptr);
    collect(c, nullptr);
    down_trip(c, R, r_u, r_v, r_p);
    sync(c);
  });
}

int fugu_coupled_dot(fugu_ctx* c, const double* u1, const double* v1, const double* p1, const double* u2,
                     const double* v2, const double* p2, double* out) {
  return guard(c, [&] {
    if (!out) throw ApiError{FUGU_EINVAL, "NULL out"};
    Trip<double> A = ST(c, 0), B = ST(c, 1);
    up_trip(c, A, u1, v1, p1);
    up_trip(c, B, u2, v2, p2);
    dot_op<double>(c, {{A, B}}, OpArgs{OP_STORE, 0, 0.0}, false);
    *out = read_slot(c, S_D0);
  });
}

int fugu_krylov_solve(fugu_ctx* c, int solver, double* X_u, double* X_v, double* X_p, const double* B_u,
                      const double* B_v, const double* B_p, const double* u_adv, const double* v_adv,
                      const double* rho_c, const double* rho_u, const double* rho_v, const double* kappa,
                      const double* zeta, const double* eta, double dt, double tol, int max_iter, int has_lid,
                      double u_lid, const double* penalty_u, const double* penalty_v, const double* mdot_u,
                      const double* mdot_v, fugu_stats* st) {
  return guard(c, [&] {
    if (solver != 1 && solver != 2) throw ApiError{FUGU_EINVAL, "solver must be 1 or 2"};
    CoefBufs<double> cb = up_coefs(c, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta, penalty_u,
                                   penalty_v, mdot_u, mdot_v);
    SolveOpt o;
    o.pen = penalty_u && penalty_v;
    o.amp = mdot_u && mdot_v;
    Trip<double> X = ST(c, 0), B = ST(c, 1);
    up_trip(c, X, X_u, X_v, X_p);
    up_trip(c, B, B_u, B_v, B_p);
    reset_counters(c);
    int outer = 0;
    KrylovResult kr = solve(c, solver, cb, o, X, B, dt, tol, max_iter, has_lid != 0, u_lid, &outer);
    if (st) std::memset(st, 0, sizeof(*st));
    collect(c, st);
    if (st) {
      st->iter = kr.iter;
      st->res = kr.res;
      st->outer = outer;
      st->status = kr.status;
      KState ks = read_ks(c);
      st->matvecs = (int)ks.matvecs;
    }
    down_trip(c, X, X_u, X_v, X_p);
    sync(c);
  });
}

int fugu_matvec_coupled_t(fugu_ctx* c, const double* Y_u, const double* Y_v, const double* Y_p, double* X_u,
                          double* X_v, double* X_p, const double* u_adv, const double* v_adv, const double* rho_c,
                          const double* rho_u, const double* rho_v, const double* kappa, const double* zeta,
                          const double* eta, double dt, const double* penalty_u, const double* penalty_v,
                          const double* mdot_u, const double* mdot_v) {
  return guard(c, [&] {
    CoefBufs<double> cb = up_coefs(c, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta, penalty_u,
                                   penalty_v, mdot_u, mdot_v);
    SolveOpt o;
    o.pen = penalty_u && penalty_v;
    o.amp = mdot_u && mdot_v;
    adj_assemble(c, cb, o, dt);
    Trip<double> Y = ST(c, 0), X = ST(c, 1);
    up_trip(c, Y, Y_u, Y_v, Y_p);
    Box b = box_launch(c->g);
    k_adj_apply_t<<<b.grid, b.block, 0, c->s>>>(c->g, c->n, c->adj_val, Y.base, X.base, 1.0, nullptr, nullptr);
    CKL("k_adj_apply_t");
    down_trip(c, X, X_u, X_v, X_p);
    sync(c);
  });
}

int fugu_adjoint_solve(fugu_ctx* c, const double* g_u, const double* g_v, const double* g_p, double* lam_u,
                       double* lam_v, double* lam_p, const double* u_adv, const double* v_adv, const double* rho_c,
                       const double* rho_u, const double* rho_v, const double* kappa, const double* zeta,
                       const double* eta, double dt, double tol, const double* penalty_u, const double* penalty_v,
                       const double* mdot_u, const double* mdot_v, fugu_stats* st) {
  return guard(c, [&] {
    CoefBufs<double> cb = up_coefs(c, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta, penalty_u,
                                   penalty_v, mdot_u, mdot_v);
    SolveOpt o;
    o.pen = penalty_u && penalty_v;
    o.amp = mdot_u && mdot_v;
    Trip<double> X = ST(c, 0), B = ST(c, 1);
    up_trip(c, B, g_u, g_v, g_p);
    int outer = 0;
    KrylovResult kr = adjoint_solve_dev(c, cb, o, dt, tol, B, X, &outer);
    if (st) std::memset(st, 0, sizeof(*st));
    collect(c, st);
    if (st) {
      st->iter = kr.iter;
      st->res = kr.res;
      st->outer = outer;
      st->status = kr.status;
    }
    down_trip(c, X, lam_u, lam_v, lam_p);
    sync(c);
  });
}

int fugu_step_vjp(fugu_ctx* c, double dt, int step_idx, const fugu_step_opts* o, const double* bar_u_out,
                  const double* bar_v_out, const double* bar_c_out, const double* bar_uprev_out,
                  const double* bar_vprev_out, double* bar_u_in, double* bar_v_in, double* bar_c_in,
                  double* bar_uprev_in, double* bar_vprev_in, double* bar_theta, fugu_stats* st) {
  return guard(c, [&] {
    if (!o) throw ApiError{FUGU_EINVAL, "NULL step options"};
    const double* bo[5] = {bar_u_out, bar_v_out, bar_c_out, bar_uprev_out, bar_vprev_out};
    double* bi[5] = {bar_u_in, bar_v_in, bar_c_in, bar_uprev_in, bar_vprev_in};
    step_vjp(c, dt, step_idx, o, bo, bi, bar_theta, st);
  });
}

int fugu_vof_advection_tvd(fugu_ctx* c, const double* c_in, double* c_out, const double* u, const double* v,
                           double dt, double* flux_x, double* flux_y) {
  return guard(c, [&] {
    double* ci = upk(c, 0, c_in, K_CELL);
    double* du = upk(c, 1, u, K_U);
    double* dv = upk(c, 2, v, K_V);
    const bool fl = flux_x && flux_y;
    vof(c, ci, S(c, 3), du, dv, dt, fl ? S(c, 4) : nullptr, fl ? S(c, 5) : nullptr);
    down(c, c_out, S(c, 3), K_CELL);
    if (fl) {
      down(c, flux_x, S(c, 4), K_U);
      down(c, flux_y, S(c, 5), K_V);
    }
    sync(c);
  });
}

int fugu_svof_helmholtz_filter(fugu_ctx* c, const double* c_raw, double* c_smooth, double delta, int max_iter,
                               double tol, int* iters_out) {
  return guard(c, [&] {
    double* cr = upk(c, 0, c_raw, K_CELL);
    reset_counters(c);
    svof(c, cr, S(c, 1), S(c, 2), delta, max_iter, tol);
    fugu_stats st{};
    collect(c, &st);
    if (iters_out) *iters_out = st.svof_iters;
    down(c, c_smooth, S(c, 1), K_CELL);
    sync(c);
  });
}

int fugu_compute_interface_curvature(fugu_ctx* c, const double* c_smooth, double* kappa_curv) {
  return guard(c, [&] {
    double* cs = upk(c, 0, c_smooth, K_CELL);
    curvature(c, cs, S(c, 1));
    down(c, kappa_curv, S(c, 1), K_CELL);
    sync(c);
  });
}

int fugu_compute_csf_force(fugu_ctx* c, const double* c_raw, const double* kappa_curv, double* f_sigma_u,
                           double* f_sigma_v) {
  return guard(c, [&] {
    double* cr = upk(c, 0, c_raw, K_CELL);
    double* kc = upk(c, 1, kappa_curv, K_CELL);
    csf(c, cr, kc, S(c, 2), S(c, 3));
    down(c, f_sigma_u, S(c, 2), K_U);
    down(c, f_sigma_v, S(c, 3), K_V);
    sync(c);
  });
}

// mod_io.f90:169-225 byte format
int fugu_write_checkpoint(fugu_ctx* c, const char* path, int step_no, double t) {
  return guard(c, [&] {
    if (!path) throw ApiError{FUGU_EINVAL, "NULL path"};
    const int nx = c->prm.nx, ny = c->prm.ny;
    const size_t nu = (size_t)(nx + 5) * (ny + 4), nv = (size_t)(nx + 4) * (ny + 5), nc = (size_t)(nx + 4) * (ny + 4);
    std::vector<double> buf(2 * nu + 2 * nv + 2 * nc);
    double* b = buf.data();
    down(c, b, c->f[FUGU_F_U_VEL], K_U); b += nu;
    down(c, b, c->f[FUGU_F_V_VEL], K_V); b += nv;
    down(c, b, c->f[FUGU_F_U_PREV], K_U); b += nu;
    down(c, b, c->f[FUGU_F_V_PREV], K_V); b += nv;
    down(c, b, c->f[FUGU_F_P_FIELD], K_CELL); b += nc;
    down(c, b, c->f[FUGU_F_C_FIELD], K_CELL);
    sync(c);
    FILE* fp = fopen(path, "wb");
    if (!fp) throw ApiError{FUGU_EIO, std::string("cannot open ") + path};
    const int hdr[3] = {nx, ny, 2};
    bool ok = fwrite(&step_no, sizeof(int), 1, fp) == 1 && fwrite(&t, sizeof(double), 1, fp) == 1 &&
              fwrite(hdr, sizeof(int), 3, fp) == 3 && fwrite(buf.data(), sizeof(double), buf.size(), fp) == buf.size();
    ok = (fclose(fp) == 0) && ok;
    if (!ok) throw ApiError{FUGU_EIO, "checkpoint write failed"};
  });
}

int fugu_read_checkpoint(fugu_ctx* c, const char* path, int* step_no, double* t) {
  return guard(c, [&] {
    if (!path || !step_no || !t) throw ApiError{FUGU_EINVAL, "NULL argument"};
    const int nx = c->prm.nx, ny = c->prm.ny;
    FILE* fp = fopen(path, "rb");
    if (!fp) throw ApiError{FUGU_EIO, std::string("cannot open ") + path};
    int hdr[3];
    if (fread(step_no, sizeof(int), 1, fp) != 1 || fread(t, sizeof(double), 1, fp) != 1 ||
        fread(hdr, sizeof(int), 3, fp) != 3 || hdr[0] != nx || hdr[1] != ny || hdr[2] != 2) {
      fclose(fp);
      throw ApiError{FUGU_EIO, "checkpoint header does not match the context (nx, ny, nh)"};
    }
    const size_t nu = (size_t)(nx + 5) * (ny + 4), nv = (size_t)(nx + 4) * (ny + 5), nc = (size_t)(nx + 4) * (ny + 4);
    std::vector<double> buf(2 * nu + 2 * nv + 2 * nc);
    const bool ok = fread(buf.data(), sizeof(double), buf.size(), fp) == buf.size();
    fclose(fp);
    if (!ok) throw ApiError{FUGU_EIO, "checkpoint body truncated"};
    const double* b = buf.data();
    up(c, c->f[FUGU_F_U_VEL], b, K_U); b += nu;
    up(c, c->f[FUGU_F_V_VEL], b, K_V); b += nv;
    up(c, c->f[FUGU_F_U_PREV], b, K_U); b += nu;
    up(c, c->f[FUGU_F_V_PREV], b, K_V); b += nv;
    up(c, c->f[FUGU_F_P_FIELD], b, K_CELL); b += nc;
    up(c, c->f[FUGU_F_C_FIELD], b, K_CELL);
    sync(c);
  });
}

}  // extern "C"

// ================================================================ batched form
//
// Many independent cases on one GPU.  Each case is a full context (state,
// Krylov work space, stream); a pool of host threads steps them, so the
// device runs as many cases' kernels at once as its SMs hold.  Cases are
// handed out largest first (longest-processing-time order) from one atomic
// counter.  The cluster size of each case's PCG comes from a measured
// autotune: per distinct (grid, boundary, precision), every feasible size is
// timed on the case's own coefficients and the one with the least SM time
// per iteration (CTAs x microseconds) wins, because a full GPU is limited by
// SM time, not by one case's latency.
//
// With fugu_batch_opts.lockstep the coupled solves of all cases run in
// lockstep instead: one launch per kernel family serves every running case
// (lockstep.cuh, lockstep_host.cuh), and the host threads only issue each
// case's explicit stages and final BCs.
#include "lockstep_host.cuh"

struct fugu_batch {
  int device = 0;
  int nthreads = 1;
  std::vector<fugu_ctx*> cases;
  std::vector<int> order;
  std::string err;
  // the lockstep solvers (lockstep = 1): one per group of cases, a group
  // being cases of one PCG grid class (at most lockstep_group of them), each
  // group advanced by its own host thread on its own stream
  std::vector<LockstepBase*> groups;
  std::vector<std::vector<int>> group_ids;  // the batch indices of each group's cases
  std::vector<cudaEvent_t> ev_group;        // per group: its ended solves' final BCs are queued
  // the batch stream: a run starts after the work queued on it before the
  // run and ends before the work queued on it after
  cudaStream_t s = nullptr;
  cudaEvent_t ev_start = nullptr;
  std::vector<cudaEvent_t> ev_case;  // per case: its stage of the run is done
};

namespace {

template <typename T>
PcgWork<T>& pcg_work(fugu_ctx* c);
template <>
PcgWork<double>& pcg_work<double>(fugu_ctx* c) { return c->w64.pcg; }
template <>
PcgWork<float>& pcg_work<float>(fugu_ctx* c) { return c->w32.pcg; }

// time one PCG launch of `iters` iterations (tol 0: never converges) on the
// context's current cluster plan; returns microseconds per iteration
template <typename T>
double time_pcg_iter(fugu_ctx* c, PcgWork<T>& w, T* phi, const T* rhs, int iters) {
  cudaEvent_t e0 = ev_get(c), e1 = ev_get(c);
  CK(cudaMemsetAsync(phi, 0, sizeof(T) * c->n, c->s));
  pcg<T>(c, w, phi, rhs, 0.0, iters, false, nullptr);  // warm-up
  CK(cudaMemsetAsync(phi, 0, sizeof(T) * c->n, c->s));
  CK(cudaEventRecord(e0, c->s));
  pcg<T>(c, w, phi, rhs, 0.0, iters, false, nullptr);
  CK(cudaEventRecord(e1, c->s));
  sync(c);
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  c->ev_pool.push_back(e0);
  c->ev_pool.push_back(e1);
  return 1e3 * ms / iters;
}

// Autotune the PCG cluster size of context c for precision T: candidates
// 2, 4, 8, 16 CTAs (those the planner accepts).  The Poisson coefficients
// are those of uniform unit density, the right-hand side a smooth mode; the
// iteration cost does not depend on the values.  Returns the chosen size
// (0 when no cluster plan fits: the grid-wide kernel is used).
template <typename T>
int tune_cluster(fugu_ctx* c) {
  const int idx = sizeof(T) == 8 ? 0 : 1;
  PcgWork<T>& w = pcg_work<T>(c);
  const Geo& g = c->g;
  // scratch: unit density (double), then phi and rhs of type T
  std::vector<double> host((size_t)c->n, 1.0);
  double* ones = S(c, 0);
  T* phi = (T*)S(c, 1);
  T* rhs = (T*)S(c, 2);
  CK(cudaMemcpyAsync(ones, host.data(), sizeof(double) * c->n, cudaMemcpyHostToDevice, c->s));
  poisson_coefs<T>(c, w, ones, ones);
  std::vector<T> hr((size_t)c->n, T(0));
  for (int j = 1; j <= g.ny; ++j)
    for (int i = 1; i <= g.nx; ++i)
      hr[(size_t)g.at(i, j)] = T(std::sin(6.283185307179586 * i / g.nx) * std::cos(3.141592653589793 * j / g.ny));
  CK(cudaMemcpyAsync(rhs, hr.data(), sizeof(T) * c->n, cudaMemcpyHostToDevice, c->s));
  sync(c);  // the host vectors go out of scope
  int best = 0;
  double best_cost = 0.0;
  for (int C = 2; C <= 16; C *= 2) {
    c->max_cluster = C;
    plan_pcg_cluster<T>(c, c->pcgc[idx]);
    if (!c->pcgc[idx].ok || c->pcgc[idx].C != C) continue;
    const double cost = C * time_pcg_iter<T>(c, w, phi, rhs, 64);
    if (!best || cost < best_cost) {
      best = C;
      best_cost = cost;
    }
  }
  c->max_cluster = best ? best : 16;
  plan_pcg_cluster<T>(c, c->pcgc[idx]);
  sync(c);
  return best;
}

// accumulate one step's statistics into a run's totals (sums of the counts,
// the largest residual, the first error)
void add_stats(fugu_stats& t, const fugu_stats& s) {
  t.iter += s.iter;
  t.outer += s.outer;
  t.pcg_iters += s.pcg_iters;
  t.pcg_calls += s.pcg_calls;
  t.matvecs += s.matvecs;
  t.svof_iters += s.svof_iters;
  if (s.res > t.res || std::isnan(s.res)) t.res = s.res;
  if (t.status == FUGU_CONVERGED && s.status != FUGU_CONVERGED) t.status = s.status;
}

struct BatchRun {
  int nsteps;
  const double* dt;
  const int* step0;
  const fugu_step_opts* opts;
  fugu_stats* last;
  double* max_res;
  int* status;
  fugu_stats* total;
  std::atomic<int> next{0};
};

void batch_worker(fugu_batch* b, BatchRun* r) {
  const int nc = (int)b->cases.size();
  for (;;) {
    const int k = r->next.fetch_add(1);
    if (k >= nc) return;
    const int i = b->order[k];
    fugu_ctx* c = b->cases[i];
    double mres = 0.0;
    fugu_stats st{}, tot{};
    tot.status = FUGU_CONVERGED;
    const int rc = guard(c, [&] {
      for (int s = 0; s < r->nsteps; ++s) {
        std::memset(&st, 0, sizeof st);
        step(c, r->dt[i], r->step0[i] + s, &r->opts[i], &st);
        if (st.res > mres || std::isnan(st.res)) mres = st.res;
        add_stats(tot, st);
      }
    });
    if (r->last) r->last[i] = st;
    if (r->total) r->total[i] = tot;
    if (r->max_res) r->max_res[i] = mres;
    if (r->status) r->status[i] = rc;
  }
}

// Lockstep set-up: every case runs the flexible-GMRES defect correction
// (refine = 2) in one precision with one smoother and cycle length, and its
// PCG fits a thread-block cluster.  The cases are grouped by their PCG's
// cluster plan (one PCG launch per Arnoldi step and group), in groups of at
// most group_max cases (0: no limit) in the order of the batch.
int lockstep_create(fugu_batch* b, int group_max) {
  const int nc = (int)b->cases.size();
  const fugu_params& p0 = b->cases[0]->prm;
  const int pi = p0.precision == FUGU_MIXED ? 1 : 0;
  std::map<std::array<long, 4>, std::vector<int>> by_class;
  std::vector<std::array<long, 4>> class_order;
  for (int i = 0; i < nc; ++i) {
    const fugu_ctx* c = b->cases[i];
    const fugu_params& p = c->prm;
    std::string why;
    if (p.refine != 2) why = "refine must be 2 (flexible GMRES inside the defect correction)";
    else if (p.precision != p0.precision) why = "every case needs the same precision";
    else if (p.refine_max_inner != p0.refine_max_inner) why = "every case needs the same refine_max_inner";
    else if (p.pcd_smoother != p0.pcd_smoother) why = "every case needs the same pcd_smoother";
    else if (!c->pcgc[pi].ok) why = "the PCG of the case does not fit a thread-block cluster";
    if (!why.empty()) {
      b->err = "lockstep batch, case " + std::to_string(i) + ": " + why;
      return FUGU_EINVAL;
    }
    const fugu_ctx::ClusterPlan& pl = c->pcgc[pi];
    const std::array<long, 4> key = {pl.C, pl.cpt, pl.rows_per, (long)pl.smem};
    auto it = by_class.find(key);
    if (it == by_class.end()) {
      class_order.push_back(key);
      it = by_class.emplace(key, std::vector<int>{}).first;
    }
    it->second.push_back(i);
  }
  const int gmax = group_max > 0 ? std::min(group_max, LS_MAX) : LS_MAX;
  for (const auto& key : class_order) {
    const std::vector<int>& ids = by_class[key];
    for (size_t k = 0; k < ids.size(); k += gmax)
      b->group_ids.emplace_back(ids.begin() + k, ids.begin() + std::min(ids.size(), k + (size_t)gmax));
  }
  try {
    CK(cudaSetDevice(b->device));
    for (const std::vector<int>& ids : b->group_ids) {
      std::vector<fugu_ctx*> cs;
      for (int i : ids) cs.push_back(b->cases[i]);
      if (p0.precision == FUGU_MIXED) {
        Lockstep<float>* ls = new Lockstep<float>();
        b->groups.push_back(ls);
        ls->create(cs);
      } else {
        Lockstep<double>* ls = new Lockstep<double>();
        b->groups.push_back(ls);
        ls->create(cs);
      }
      cudaEvent_t e;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->ev_group.push_back(e);
    }
  } catch (const CudaError& e) {
    b->err = std::string("lockstep batch: ") + e.what + ": " + cudaGetErrorString(e.e);
    return FUGU_ECUDA;
  } catch (const ApiError& e) {
    b->err = "lockstep batch: " + e.msg;
    return e.code;
  }
  return FUGU_OK;
}

// the batch stream and its events (created with the batch)
void batch_streams(fugu_batch* b) {
  CK(cudaSetDevice(b->device));
  CK(cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming));
  b->ev_case.resize(b->cases.size(), nullptr);
  for (auto& e : b->ev_case) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}
// every case stream and lockstep stream waits for the work queued on the
// batch stream so far
void batch_begin(fugu_batch* b) {
  CK(cudaSetDevice(b->device));
  CK(cudaEventRecord(b->ev_start, b->s));
  for (fugu_ctx* c : b->cases) CK(cudaStreamWaitEvent(c->s, b->ev_start, 0));
  for (LockstepBase* ls : b->groups) CK(cudaStreamWaitEvent(ls->stream(), b->ev_start, 0));
}
// the batch stream waits for every case stream's and lockstep stream's work
// of the run
void batch_end(fugu_batch* b) {
  CK(cudaSetDevice(b->device));
  for (size_t i = 0; i < b->cases.size(); ++i) {
    CK(cudaEventRecord(b->ev_case[i], b->cases[i]->s));
    CK(cudaStreamWaitEvent(b->s, b->ev_case[i], 0));
  }
  for (size_t g = 0; g < b->groups.size(); ++g) {
    CK(cudaEventRecord(b->ev_group[g], b->groups[g]->stream()));
    CK(cudaStreamWaitEvent(b->s, b->ev_group[g], 0));
  }
}

// run fn(i) for the cases ids (in that order) from up to nthreads host
// threads (0: the batch's); returns a status per case of the batch
template <typename F>
std::vector<int> for_ids(fugu_batch* b, const std::vector<int>& ids, F fn, int nthreads = 0) {
  std::vector<int> st(b->cases.size(), FUGU_OK);
  const int n = (int)ids.size();
  std::atomic<int> next{0};
  auto work = [&] {
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) return;
      const int i = ids[k];
      st[i] = guard(b->cases[i], [&] { fn(i); });
    }
  };
  const int nt = std::min(nthreads > 0 ? nthreads : b->nthreads, n);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  return st;
}
// the same for every case (largest first)
template <typename F>
std::vector<int> for_cases(fugu_batch* b, F fn) {
  return for_ids(b, b->order, fn);
}

// The lockstep batch run (continuous batching, lockstep_host.cuh).  Each
// group of cases is advanced by its own host thread: every case goes
// through nsteps steps; a case whose solve ends at a pass goes through its
// final BCs and statistics and its next step's explicit stages on its own
// stream while the group's other cases' next cycle runs, and joins the
// lockstep solve again at the following pass.  The groups do not wait for
// one another.
int lockstep_run(fugu_batch* b, int nsteps, const double* dt, const int* step0, const fugu_step_opts* opts,
                 fugu_stats* last, double* max_res, int* status, fugu_stats* total) {
  const int nc = (int)b->cases.size();
  std::vector<double> mres(nc, 0.0);
  std::vector<int> cst(nc, FUGU_OK);
  std::vector<fugu_stats> lst(nc), tot(nc);
  for (auto& t : tot) {
    std::memset(&t, 0, sizeof t);
    t.status = FUGU_CONVERGED;
  }
  std::atomic<int> rc{FUGU_OK};
  std::mutex err_mu;
  auto fail = [&](int code, const std::string& msg) {
    std::lock_guard<std::mutex> lk(err_mu);
    if (rc.load() == FUGU_OK) {
      rc = code;
      b->err = msg;
    }
  };
  try {
    for (LockstepBase* ls : b->groups) ls->reset();
    batch_begin(b);
  } catch (const CudaError& e) {
    b->err = std::string("batch stream: ") + e.what + ": " + cudaGetErrorString(e.e);
    return FUGU_ECUDA;
  }
  std::vector<int> done(nc, 0);  // steps completed per case
  const int ng = (int)b->groups.size();
  const int nt = std::max(1, b->nthreads / ng);  // host threads of a group's per-case work
  auto run_group = [&](int g) {
    LockstepBase* ls = b->groups[g];
    const std::vector<int>& ids = b->group_ids[g];  // local index k: batch case ids[k]
    const int n = (int)ids.size();
    cudaStream_t ls_s = ls->stream();
    std::vector<StepSetup> su(n);
    std::vector<KrylovResult> kr(n);
    std::vector<int> outer(n, 0);
    std::vector<int> loc(nc, -1);
    for (int k = 0; k < n; ++k) loc[ids[k]] = k;
    auto take = [&](const std::vector<int>& st, const std::vector<int>& bids) {
      for (int i : bids)
        if (st[i] != FUGU_OK) {
          cst[i] = st[i];
          fail(st[i], "case " + std::to_string(i) + ": " + b->cases[i]->err);
        }
    };
    // explicit stages of case i's next step on its own stream
    auto pre = [&](int i) {
      fugu_ctx* c = b->cases[i];
      su[loc[i]] = step_setup(c, dt[i], step0[i] + done[i], &opts[i]);
      step_pre(c, dt[i], step0[i] + done[i], &opts[i]);
      CK(cudaEventRecord(b->ev_case[i], c->s));
    };
    std::vector<int> joining;  // batch ids
    if (nsteps > 0) {
      take(for_ids(b, ids, pre, nt), ids);
      joining = ids;
    }
    try {
      CK(cudaSetDevice(b->device));
      while (rc.load() == FUGU_OK) {
        if (!joining.empty()) {
          std::vector<int> lj;
          for (int i : joining) {
            CK(cudaStreamWaitEvent(ls_s, b->ev_case[i], 0));
            lj.push_back(loc[i]);
          }
          ls->join(lj, su);
          joining.clear();
        }
        const std::vector<int> ended_l = ls->defect();
        std::vector<int> ended;
        for (int k : ended_l) ended.push_back(ids[k]);
        if (!ended.empty()) {
          ls->finish(ended_l, kr, outer);
          CK(cudaEventRecord(b->ev_group[g], ls_s));
        }
        const bool cycling = ls->cycle_launch();
        if (!ended.empty()) {
          // meanwhile on the host threads: the ended steps' final BCs and
          // statistics, and the next steps' explicit stages
          std::vector<int> st = for_ids(b, ended, [&](int i) {
            fugu_ctx* c = b->cases[i];
            const int k = loc[i];
            CK(cudaStreamWaitEvent(c->s, b->ev_group[g], 0));
            std::memset(&lst[i], 0, sizeof(fugu_stats));
            step_post(c, su[k], kr[k], outer[k], &lst[i]);
            if (lst[i].res > mres[i] || std::isnan(lst[i].res)) mres[i] = lst[i].res;
            add_stats(tot[i], lst[i]);
            if (++done[i] < nsteps) pre(i);
          }, nt);
          take(st, ended);
          for (int i : ended)
            if (done[i] < nsteps) joining.push_back(i);
        }
        if (cycling) ls->cycle_finish();
        if (!cycling && joining.empty()) break;
      }
    } catch (const CudaError& e) {
      fail(FUGU_ECUDA, std::string("lockstep solve: ") + e.what + ": " + cudaGetErrorString(e.e));
    } catch (const ApiError& e) {
      fail(e.code, "lockstep solve: " + e.msg);
    }
  };
  std::vector<std::thread> pool;
  for (int g = 1; g < ng; ++g) pool.emplace_back(run_group, g);
  if (ng > 0) run_group(0);
  for (auto& th : pool) th.join();
  int code = rc.load();
  if (code != FUGU_OK) {
    for (int i = 0; i < nc; ++i)
      if (cst[i] == FUGU_OK) cst[i] = code;
  } else {
    try {
      batch_end(b);
    } catch (const CudaError& e) {
      b->err = std::string("batch stream: ") + e.what + ": " + cudaGetErrorString(e.e);
      code = FUGU_ECUDA;
    }
  }
  for (int i = 0; i < nc; ++i) {
    if (last) last[i] = lst[i];
    if (max_res) max_res[i] = mres[i];
    if (status) status[i] = cst[i];
    if (total) total[i] = tot[i];
  }
  return code;
}

}  // namespace

extern "C" {

int fugu_batch_create(const fugu_params* params, int ncases, int device, const fugu_batch_opts* opts,
                      fugu_batch** out) {
  if (!out) return FUGU_EINVAL;
  *out = nullptr;
  if (!params || ncases < 1) return FUGU_EINVAL;
  for (int i = 0; i < ncases; ++i)
    if (check_params(&params[i]) != FUGU_OK) return FUGU_EINVAL;
  fugu_batch_opts o{};
  if (opts) o = *opts;
  if (o.nthreads < 0 || o.max_cluster < 0 || o.max_cluster > 16 || o.max_coop < 0 || o.lockstep < 0 ||
      o.lockstep > 1)
    return FUGU_EINVAL;
  fugu_batch* b = new fugu_batch();
  b->device = device;
  const int hw = (int)std::thread::hardware_concurrency();
  b->nthreads = o.nthreads ? o.nthreads : (hw > 0 ? hw : 8);
  if (b->nthreads > ncases) b->nthreads = ncases;
  // autotune decisions shared by cases of the same grid, boundaries and precision
  std::map<std::array<int, 5>, int> tuned;
  for (int i = 0; i < ncases; ++i) {
    fugu_ctx* c = new fugu_ctx();
    c->prm = params[i];
    c->device = device;
    c->max_coop = o.max_coop ? std::min(o.max_coop, 8) : 8;
    c->coop_as_cluster = true;
    c->max_cluster = o.max_cluster ? o.max_cluster : 16;
    b->cases.push_back(c);
    const int rc = guard(c, [&] {
      create(c);
      if (c->prm.precision == FUGU_MIXED) ensure_w32(c);
      if (o.max_cluster) return;
      const std::array<int, 5> key = {c->prm.nx, c->prm.ny, c->prm.periodic_x, c->prm.periodic_y,
                                      c->prm.precision};
      auto it = tuned.find(key);
      if (it == tuned.end()) {
        const int C = c->prm.precision == FUGU_MIXED ? tune_cluster<float>(c) : tune_cluster<double>(c);
        it = tuned.emplace(key, C ? C : 16).first;
      }
      c->max_cluster = it->second;
      plan_pcg_cluster<double>(c, c->pcgc[0]);
      plan_pcg_cluster<float>(c, c->pcgc[1]);
    });
    if (rc) {
      b->err = "case " + std::to_string(i) + ": " + c->err;
      fprintf(stderr, "fugu_batch_create: %s\n", b->err.c_str());
      for (fugu_ctx* x : b->cases) destroy(x);
      delete b;
      return rc;
    }
  }
  if (o.lockstep) {
    const int rc = lockstep_create(b, o.lockstep_group);
    if (rc) {
      fprintf(stderr, "fugu_batch_create: %s\n", b->err.c_str());
      fugu_batch_destroy(b);
      return rc;
    }
  }
  try {
    batch_streams(b);
  } catch (const CudaError& e) {
    b->err = std::string("batch stream: ") + e.what + ": " + cudaGetErrorString(e.e);
    fprintf(stderr, "fugu_batch_create: %s\n", b->err.c_str());
    fugu_batch_destroy(b);
    return FUGU_ECUDA;
  }
  b->order.resize(ncases);
  for (int i = 0; i < ncases; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int z) {
    return (long)params[a].nx * params[a].ny > (long)params[z].nx * params[z].ny;
  });
  *out = b;
  return FUGU_OK;
}

void fugu_batch_destroy(fugu_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  for (cudaEvent_t e : b->ev_case) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_group) cudaEventDestroy(e);
  if (b->ev_start) cudaEventDestroy(b->ev_start);
  if (b->s) {
    cudaStreamSynchronize(b->s);
    cudaStreamDestroy(b->s);
  }
  for (LockstepBase* ls : b->groups) delete ls;
  for (fugu_ctx* c : b->cases) destroy(c);
  delete b;
}

const char* fugu_batch_last_error(const fugu_batch* b) { return b ? b->err.c_str() : "NULL batch"; }

int fugu_batch_size(const fugu_batch* b) { return b ? (int)b->cases.size() : 0; }

int fugu_batch_case(fugu_batch* b, int i, fugu_ctx** ctx) {
  if (!b || !ctx || i < 0 || i >= (int)b->cases.size()) return FUGU_EINVAL;
  *ctx = b->cases[i];
  return FUGU_OK;
}

int fugu_batch_run(fugu_batch* b, int nsteps, const double* dt, const int* step0, const fugu_step_opts* opts,
                   fugu_stats* last, double* max_res, int* status, fugu_stats* total) {
  if (!b) return FUGU_EINVAL;
  if (nsteps < 0 || !dt || !step0 || !opts) {
    b->err = "fugu_batch_run: NULL dt/step0/opts or nsteps < 0";
    return FUGU_EINVAL;
  }
  if (!b->groups.empty()) return lockstep_run(b, nsteps, dt, step0, opts, last, max_res, status, total);
  try {
    batch_begin(b);
  } catch (const CudaError& e) {
    b->err = std::string("batch stream: ") + e.what + ": " + cudaGetErrorString(e.e);
    return FUGU_ECUDA;
  }
  BatchRun r;
  r.nsteps = nsteps;
  r.dt = dt;
  r.step0 = step0;
  r.opts = opts;
  r.last = last;
  r.max_res = max_res;
  r.total = total;
  std::vector<int> st(b->cases.size(), FUGU_OK);
  r.status = st.data();
  std::vector<std::thread> pool;
  for (int t = 1; t < b->nthreads; ++t) pool.emplace_back(batch_worker, b, &r);
  batch_worker(b, &r);
  for (auto& th : pool) th.join();
  if (status) std::memcpy(status, st.data(), sizeof(int) * st.size());
  for (size_t i = 0; i < st.size(); ++i)
    if (st[i] != FUGU_OK) {
      b->err = "case " + std::to_string(i) + ": " + b->cases[i]->err;
      return st[i];
    }
  try {
    batch_end(b);
  } catch (const CudaError& e) {
    b->err = std::string("batch stream: ") + e.what + ": " + cudaGetErrorString(e.e);
    return FUGU_ECUDA;
  }
  return FUGU_OK;
}

int fugu_batch_get_stream(fugu_batch* b, void** stream) {
  if (!b || !stream) return FUGU_EINVAL;
  *stream = (void*)b->s;
  return FUGU_OK;
}

unsigned long long fugu_batch_launches(const fugu_batch* b) {
  if (!b) return 0;
  unsigned long long n = 0;
  for (const LockstepBase* ls : b->groups) n += ls->launch_count();
  for (const fugu_ctx* c : b->cases) n += c->launches;
  return n;
}

}  // extern "C"

// ============================================== allocation-free Poisson solve
//
// fugu_solve_poisson_pressure_noalloc runs solve_poisson_pressure
// (mod_subsolvers.f90:32-246) with the grid-wide PCG kernel k_pcg<double>,
// but every byte of its working memory comes from na_scratch, one file-scope
// device array, instead of from a context.  The call allocates nothing: no
// cudaMalloc, cudaFree, cudaMallocHost or library routine that allocates.
//
// na_scratch layout (offsets in doubles, every region 256-byte aligned):
//   [0, 32)               GridSync at 0, PcgOut at 16
//   [32, 32 + 12*256)     CTA partial sums of k_pcg (12 per CTA, <= 256 CTAs)
//   [NA_FIELD0, ...)      12 fields of NA_MAX_POINTS each in the padded
//                         device layout: phi, rhs, rho_u, rho_v, cx, cy,
//                         dinv, r, z, pb0, pb1, ap
namespace {

constexpr long NA_MAX_POINTS = FUGU_NOALLOC_MAX_POINTS;  // padded points per field
constexpr int NA_MAX_CTAS = 256;
constexpr long NA_PART = 32;
constexpr long NA_FIELD0 = NA_PART + 12L * NA_MAX_CTAS;
constexpr int NA_NFIELDS = 12;
constexpr long NA_TOTAL = NA_FIELD0 + NA_NFIELDS * NA_MAX_POINTS;
constexpr int NA_MAX_DEVICES = 64;
static_assert((NA_FIELD0 * sizeof(double)) % 256 == 0, "field region alignment");
static_assert((NA_MAX_POINTS * sizeof(double)) % 256 == 0, "field stride alignment");
static_assert(sizeof(GridSync) <= 16 * sizeof(double) && sizeof(PcgOut) <= 16 * sizeof(double), "header");

static __device__ __align__(256) double na_scratch[NA_TOTAL];

// Per-device set-up, done by the first call with that device current and
// redone whenever the device's current CUDA context has changed since (after
// cudaDeviceReset the library's module, and with it na_scratch, is loaded
// again, possibly at another address).
struct NaDevice {
  bool ready = false;
  void* cu_ctx = nullptr;  // the CUDA context the address below belongs to
  double* base = nullptr;  // device address of na_scratch in that context
  int max_ctas = 0;        // co-resident CTAs of k_pcg<double>, one per SM at most
};
std::mutex na_mu;
NaDevice na_dev[NA_MAX_DEVICES];
// failure-detection test hook for this entry (fugu_test_arm_barrier_timeout
// with a NULL context): > 0 arms the next call's PCG launch
std::atomic<unsigned int> na_test_spin_limit{0};

// the calling thread's current CUDA context (driver cuCtxGetCurrent, found
// through the runtime so the library does not link the driver library)
cudaError_t na_current_context(void** out) {
  using GetCurrent = int (*)(void**);
  static GetCurrent fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !f) return cudaErrorSymbolNotFound;
    fn = (GetCurrent)f;
  }
  return fn(out) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// message into the caller's buffer (no heap use on any path of the entry)
int na_fail(char* err, int err_len, int code, const char* what, const char* detail = "") {
  if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s%s", what, detail);
  return code;
}

}  // namespace

extern "C" int fugu_solve_poisson_pressure_noalloc(const fugu_params* p, void* stream, double* phi,
                                                   const double* rhs, const double* rho_u, const double* rho_v,
                                                   double tol, int max_iter, int* iter_out, double* res_out,
                                                   char* err, int err_len) {
  if (err && err_len > 0) err[0] = '\0';
  if (check_params(p) != FUGU_OK) return na_fail(err, err_len, FUGU_EINVAL, "invalid fugu_params");
  if (!phi || !rhs || !rho_u || !rho_v) return na_fail(err, err_len, FUGU_EINVAL, "NULL array argument");
  if (max_iter < 0) return na_fail(err, err_len, FUGU_EINVAL, "max_iter < 0");
  const Geo g = make_geo(*p);
  if (g.n() > NA_MAX_POINTS) {
    char m[256];
    std::snprintf(m, sizeof m,
                  "grid %d x %d needs %ld padded points per field; the allocation-free solve holds at most "
                  "%ld (round_up(nx+5,16)*(ny+5); every grid up to 256 x 256 fits)",
                  p->nx, p->ny, g.n(), NA_MAX_POINTS);
    return na_fail(err, err_len, FUGU_EINVAL, m);
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "cudaGetDevice: ", cudaGetErrorString(e));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return na_fail(err, err_len, FUGU_EINVAL, "device ordinal out of range");
  void* cu_ctx = nullptr;
  e = na_current_context(&cu_ctx);
  if (e == cudaSuccess && !cu_ctx) {
    // no context is current yet: cudaSetDevice makes the device's primary
    // context current (it allocates no device memory)
    e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = na_current_context(&cu_ctx);
  }
  if (e == cudaSuccess && !cu_ctx) e = cudaErrorDeviceUninitialized;
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "current CUDA context: ", cudaGetErrorString(e));
  NaDevice d;
  {
    std::lock_guard<std::mutex> lk(na_mu);
    NaDevice& nd = na_dev[dev];
    if (!nd.ready || nd.cu_ctx != cu_ctx) {
      nd.ready = false;
      double* ptr = nullptr;
      e = cudaGetSymbolAddress((void**)&ptr, na_scratch);
      if (e != cudaSuccess)
        return na_fail(err, err_len, FUGU_ECUDA, "cudaGetSymbolAddress: ", cudaGetErrorString(e));
      int nsm = 0, occ = 0;
      e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k_pcg<double>, PCG_TPB, 0);
      if (e != cudaSuccess || nsm < 1 || occ < 1)
        return na_fail(err, err_len, FUGU_ECUDA, "no co-resident grid for the PCG kernel on this device");
      nd.cu_ctx = cu_ctx;
      nd.base = ptr;
      nd.max_ctas = nsm < NA_MAX_CTAS ? nsm : NA_MAX_CTAS;
      nd.ready = true;
    }
    d = nd;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long n = g.n();
  GridSync* gs = (GridSync*)d.base;
  PcgOut* out = (PcgOut*)(d.base + 16);
  double* part = d.base + NA_PART;
  double* f[NA_NFIELDS];
  for (int k = 0; k < NA_NFIELDS; ++k) f[k] = d.base + NA_FIELD0 + k * NA_MAX_POINTS;
  // caller's array (reference layout, host or device memory) <-> padded field
  auto copy = [&](double* dst_f, const double* src, double* dst, const double* src_f, int kind) {
    int i0, i1, j0, j1;
    g.extent(kind, i0, i1, j0, j1);
    const size_t w = (size_t)(i1 - i0 + 1), h = (size_t)(j1 - j0 + 1);
    if (dst_f)
      return cudaMemcpy2DAsync(dst_f + g.at(i0, j0), sizeof(double) * g.P, src, sizeof(double) * w,
                               sizeof(double) * w, h, cudaMemcpyDefault, s);
    return cudaMemcpy2DAsync(dst, sizeof(double) * w, src_f + g.at(i0, j0), sizeof(double) * g.P,
                             sizeof(double) * w, h, cudaMemcpyDefault, s);
  };
  // the barrier counters, the result record and every field start at zero
  e = cudaMemsetAsync(d.base, 0, sizeof(double) * (size_t)(NA_FIELD0 + (NA_NFIELDS - 1) * NA_MAX_POINTS + n), s);
  if (e == cudaSuccess) e = copy(f[0], phi, nullptr, nullptr, K_CELL);
  if (e == cudaSuccess) e = copy(f[1], rhs, nullptr, nullptr, K_CELL);
  if (e == cudaSuccess) e = copy(f[2], rho_u, nullptr, nullptr, K_U);
  if (e == cudaSuccess) e = copy(f[3], rho_v, nullptr, nullptr, K_V);
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "copy in: ", cudaGetErrorString(e));
  Box b = box_launch(g);
  k_poisson_coefs<double><<<b.grid, b.block, 0, s>>>(g, f[2], f[3], f[4], f[5], f[6]);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "k_poisson_coefs: ", cudaGetErrorString(e));
  PcgArgs<double> a{};
  a.g = g;
  a.rhs = f[1]; a.cx = f[4]; a.cy = f[5]; a.dinv = f[6];
  a.phi = f[0]; a.r = f[7]; a.z = f[8]; a.pb0 = f[9]; a.pb1 = f[10]; a.ap = f[11];
  a.part = part; a.gs = gs; a.out = out; a.active = nullptr;
  a.tol = tol; a.max_iter = max_iter; a.phi_zero = 0; a.timed = 0;
  const unsigned int test_lim = na_test_spin_limit.exchange(0u);
  if (test_lim > 0) {
    a.spin_limit = test_lim;
    a.extra_arrivals = 1;
  }
  long want = ((long)p->nx * p->ny + PCG_TPB - 1) / PCG_TPB;
  const int grid = (int)(want < d.max_ctas ? (want < 1 ? 1 : want) : d.max_ctas);
  void* args[] = {&a};
  e = cudaLaunchCooperativeKernel((void*)k_pcg<double>, dim3(grid), dim3(PCG_TPB), args, 0, s);
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "k_pcg: ", cudaGetErrorString(e));
  e = copy(nullptr, nullptr, phi, f[0], K_CELL);
  // the barrier record and the result record (one 256-byte header) together
  double hdr[NA_PART];
  if (e == cudaSuccess) e = cudaMemcpyAsync(hdr, d.base, sizeof hdr, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return na_fail(err, err_len, FUGU_ECUDA, "copy out: ", cudaGetErrorString(e));
  GridSync hg;
  PcgOut h;
  std::memcpy(&hg, hdr, sizeof hg);
  std::memcpy(&h, hdr + 16, sizeof h);
  if (hg.error != 0 || h.status != 0)
    return na_fail(err, err_len, FUGU_ETIMEOUT,
                   "k_pcg: a grid barrier wait gave up; phi holds a partial result");
  if (iter_out) *iter_out = h.iters;
  if (res_out) *res_out = h.res;
  return FUGU_OK;
}

extern "C" int fugu_test_arm_barrier_timeout(fugu_ctx* ctx, unsigned int spin_limit) {
  if (spin_limit == 0) return FUGU_EINVAL;
  if (ctx) ctx->test_spin_limit = spin_limit;
  else na_test_spin_limit.store(spin_limit);
  return FUGU_OK;
}
