// lockstep_host.cuh -- host side of the fused batched form (lockstep.cuh).
// Included by fugu_gpu.cu after the context, the step and the solvers.
//
// A batch run advances every case through its steps; a case's step is
//   1. its explicit stages (AB extrapolation, VOF, properties, SVOF,
//      curvature, CSF, right-hand side) on the case's own stream, issued by
//      the batch's host threads (step_pre);
//   2. its coupled solve, in lockstep with the other running cases on the
//      lockstep stream: the FP64 defect correction around flexible GMRES +
//      PCD (refine_solve and fgmres in fugu_gpu.cu), every phase one launch
//      per kernel family for all running cases; each flexible-GMRES cycle is
//      one CUDA graph whose Arnoldi steps sit in conditional nodes armed on
//      the device;
//   3. its final halos, wall BCs and statistics (step_post).
// The cases do not wait for one another between steps: a case whose solve
// ends at a defect-correction pass goes through 3 and 1 of its next step
// while the others' next cycle runs, and joins the lockstep solve again at
// the following pass (continuous batching).  So the batch's time follows the
// sum of the work rather than the slowest case of every step.  The host
// synchronises twice per defect-correction pass for the whole batch (the
// single-case form does so per Arnoldi step and per case).
#pragma once

#include "lockstep.cuh"

namespace {

// check a launch of the lockstep solver and count it
#define LSCKL(what)                                        \
  do {                                                     \
    cudaError_t e_ = cudaGetLastError();                   \
    if (e_ != cudaSuccess) throw CudaError{e_, what};      \
    ++launches;                                            \
  } while (0)

struct LsClass {
  int C = 0, cpt = 0, rows_per = 0;
  size_t smem = 0;
  std::vector<int> cases;
  int* d_list = nullptr;
};

// per-case bookkeeping of one solve
struct LsCaseRun {
  bool adapt = false, adapt_sw = false;
  int cap = 0, sweeps = 0;     // current adaptive values (0: fixed)
  int outer = 0, inner_total = 0;
  double rel = 0.0, tol = 0.0;
  int status = FUGU_CONVERGED;
  bool done = false;
};

struct LockstepBase {
  virtual ~LockstepBase() {}
  // a run starts: no case is in the solve (after a run that ended in an
  // error too)
  virtual void reset() = 0;
  // the solves of cases ids start (their explicit stages are done before the
  // lockstep stream's current position)
  virtual void join(const std::vector<int>& ids, const std::vector<StepSetup>& su) = 0;
  // a defect pass of the running cases; returns the cases whose solve ended
  virtual std::vector<int> defect() = 0;
  // end the solves of ids: the final wall BCs with the lid, their results
  // and the adaptive PCG cap and sweeps back to their contexts
  virtual void finish(const std::vector<int>& ids, std::vector<KrylovResult>& kr, std::vector<int>& outer) = 0;
  // queue one flexible-GMRES cycle of the running cases (false: none runs)
  virtual bool cycle_launch() = 0;
  // wait for it, adapt the cases' PCG caps and sweeps, set up the next pass
  virtual void cycle_finish() = 0;
  virtual cudaStream_t stream() const = 0;
  virtual unsigned long long launch_count() const = 0;
};

template <typename T>
struct Lockstep : LockstepBase {
  std::vector<fugu_ctx*> cases;
  int ncase = 0, m = 0, smoother = 0, device = 0, nsm = 148;
  bool any_periodic = false;
  cudaStream_t s = nullptr;   // the lockstep stream
  cudaStream_t q = nullptr;   // the stream launches are issued on (s, or s2 while a body is captured)
  cudaStream_t s2 = nullptr;  // captures the bodies of the cycle graph's conditional nodes
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  LsCase<T>* d_cases = nullptr;
  LsDyn* d_dyn = nullptr;
  LsDyn* h_dyn = nullptr;   // the host's copy, uploaded through h_ring
  // pinned snapshots of h_dyn, one per upload since the lockstep stream last
  // synchronised (a pinned copy is read when the stream reaches it, so a
  // buffer the host changes again cannot be its source)
  static constexpr int RING = 8;
  LsDyn* h_ring = nullptr;
  int ring_next = 0;
  LsPlan* d_plan = nullptr;
  LsRead* d_read = nullptr;
  LsRead* h_read = nullptr;
  int* h_nact = nullptr;
  std::vector<LsClass> classes;
  std::map<const void*, int> grids;  // persistent grid per family kernel
  // virtual blocks of each family with every case of the group running
  long cap_box = 0, cap_e1 = 0, cap_dot = 0, cap_mdot = 0, cap_tile = 0;
  unsigned long long launches = 0;   // kernel launches issued, replays included
  // per Arnoldi step, one graph (the host checks between steps)
  struct Graph {
    int max_sweeps = -1;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;  // kernel launches of one replay
  };
  std::vector<Graph> graphs;
  // one whole flexible-GMRES cycle as one graph (a conditional IF node per
  // Arnoldi step), one per largest sweep count of the running cases
  struct Cycle {
    cudaGraphExec_t exec = nullptr;
    unsigned long long head = 0, body = 0;  // launches outside the steps, per executed step
  };
  std::map<int, Cycle> cycles;
  bool use_cycle_graph = true;
  std::vector<void*> allocs;
  // the continuous run: per case its solve's bookkeeping and whether it runs
  std::vector<LsCaseRun> cr;
  std::vector<char> running;

  cudaStream_t stream() const override { return s; }
  unsigned long long launch_count() const override { return launches; }

  ~Lockstep() override {
    if (s) cudaStreamSynchronize(s);
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& kv : cycles)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto& c : classes)
      if (c.d_list) cudaFree(c.d_list);
    for (void* p : allocs) cudaFree(p);
    if (h_dyn) cudaFreeHost(h_dyn);
    if (h_ring) cudaFreeHost(h_ring);
    if (h_read) cudaFreeHost(h_read);
    if (h_nact) cudaFreeHost(h_nact);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto e : ev_join) cudaEventDestroy(e);
    for (auto x : side) cudaStreamDestroy(x);
    if (s2) cudaStreamDestroy(s2);
    if (s) cudaStreamDestroy(s);
  }

  template <typename U>
  U* dal(long n) {
    U* p = nullptr;
    CK(cudaMalloc(&p, sizeof(U) * (size_t)n));
    allocs.push_back(p);
    return p;
  }

  // --------------------------------------------------------- set-up
  void create(const std::vector<fugu_ctx*>& cs) {
    cases = cs;
    ncase = (int)cs.size();
    fugu_ctx* c0 = cs[0];
    device = c0->device;
    nsm = c0->nsm;
    m = c0->prm.refine_max_inner;
    smoother = c0->prm.pcd_smoother;
    const int pi = sizeof(T) == 8 ? 0 : 1;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    q = s;
    std::vector<LsCase<T>> rec(ncase);
    std::map<std::array<long, 4>, int> cls_of;
    for (int i = 0; i < ncase; ++i) {
      fugu_ctx* c = cs[i];
      if (c->g.px || c->g.py) any_periodic = true;
      LsCase<T>& r = rec[i];
      std::memset(&r, 0, sizeof r);
      r.g = c->g;
      r.n = c->n;
      r.dot_grid = c->dot_grid;
      r.nsm = c->nsm;
      r.mdot_gmax = (mdot_items(c->g) + MDOT_TPB / 32 - 1) / (MDOT_TPB / 32);
      r.X = c->Xstate.base;
      r.B = c->B.base;
      r.r64 = c->w64.t[10].base;
      r.ax = c->w64.t[12].base;
      const CoefBufs<double> cb = coef64(c, c->u_adv, c->v_adv);
      r.c64.u_adv = cb.u_adv; r.c64.v_adv = cb.v_adv; r.c64.rho_c = cb.rho_c; r.c64.rho_u = cb.rho_u;
      r.c64.rho_v = cb.rho_v; r.c64.kappa = cb.kappa; r.c64.zeta = cb.zeta; r.c64.eta = cb.eta;
      r.c64.pen_u = cb.pen_u; r.c64.pen_v = cb.pen_v; r.c64.mdot_u = cb.mdu; r.c64.mdot_v = cb.mdv;
      r.sc = c->sc;
      r.part = c->part;
      r.ks = c->ks;
      r.pcg_out = c->pcg_out;
      FgWork<T>& f = ensure_fg<T>(c, m);
      r.V = f.V;
      r.Z = f.Z;
      r.st = f.st;
      if constexpr (sizeof(T) == 8) {
        KrylovWork<double>& w = c->w64;
        r.ri = w.t[10].base;
        r.di = w.t[11].base;
        r.w = w.t[0].base;
        r.cf = r.c64;
        r.cx = w.pcg.cx; r.cy = w.pcg.cy; r.dinv = w.pcg.dinv;
        r.phi = w.pcd.phi; r.zuw = w.pcd.zuw; r.zvw = w.pcd.zvw; r.tmp = w.pcd.tmp;
      } else {
        ensure_w32(c);
        KrylovWork<float>& w = c->w32;
        r.ri = w.t[10].base;
        r.di = w.t[11].base;
        r.w = w.t[0].base;
        const CoefBufs<float>& qf = w.cf;
        r.cf.u_adv = qf.u_adv; r.cf.v_adv = qf.v_adv; r.cf.rho_c = qf.rho_c; r.cf.rho_u = qf.rho_u;
        r.cf.rho_v = qf.rho_v; r.cf.kappa = qf.kappa; r.cf.zeta = qf.zeta; r.cf.eta = qf.eta;
        r.cf.pen_u = qf.pen_u; r.cf.pen_v = qf.pen_v; r.cf.mdot_u = qf.mdu; r.cf.mdot_v = qf.mdv;
        r.cx = w.pcg.cx; r.cy = w.pcg.cy; r.dinv = w.pcg.dinv;
        r.phi = w.pcd.phi; r.zuw = w.pcd.zuw; r.zvw = w.pcd.zvw; r.tmp = w.pcd.tmp;
      }
      r.pcg_tol = c->prm.pcg_tol;
      r.inner_tol = c->prm.refine_inner_tol;
      r.jac_omega = c->prm.jacobi_omega;
      r.sor_omega = c->prm.pcd_sor_omega;
      r.visc = c->prm.pcd_visc_scale;
      // PCG grid class: the cluster plan of the case's inner precision
      const fugu_ctx::ClusterPlan& pl = c->pcgc[pi];
      const std::array<long, 4> key = {pl.C, pl.cpt, pl.rows_per, (long)pl.smem};
      auto it = cls_of.find(key);
      if (it == cls_of.end()) {
        LsClass k;
        k.C = pl.C;
        k.cpt = pl.cpt;
        k.rows_per = pl.rows_per;
        k.smem = pl.smem;
        classes.push_back(k);
        it = cls_of.emplace(key, (int)classes.size() - 1).first;
      }
      classes[it->second].cases.push_back(i);
    }
    for (const LsCase<T>& r : rec) {
      cap_box += ls_box_blocks(r.g);
      cap_e1 += ls_e1_blocks(3 * r.n);
      cap_dot += r.dot_grid;
      cap_tile += ls_tile_blocks(r.g);
    }
    for (int nvec = 1; nvec <= m + 1; ++nvec) {
      long t = 0;
      for (const LsCase<T>& r : rec) t += (long)ls_mdot_g(r.nsm, r.mdot_gmax, nvec) * nvec;
      cap_mdot = std::max(cap_mdot, t);
    }
    d_cases = dal<LsCase<T>>(ncase);
    CK(cudaMemcpy(d_cases, rec.data(), sizeof(LsCase<T>) * ncase, cudaMemcpyHostToDevice));
    d_dyn = dal<LsDyn>(ncase);
    d_plan = dal<LsPlan>(1);
    d_read = dal<LsRead>(ncase);
    CK(cudaMallocHost(&h_dyn, sizeof(LsDyn) * ncase));
    CK(cudaMallocHost(&h_ring, sizeof(LsDyn) * ncase * RING));
    cr.assign(ncase, LsCaseRun{});
    running.assign(ncase, 0);
    CK(cudaMallocHost(&h_read, sizeof(LsRead) * ncase));
    CK(cudaMallocHost(&h_nact, sizeof(int)));
    std::memset(h_dyn, 0, sizeof(LsDyn) * ncase);
    for (auto& k : classes) {
      CK(cudaMalloc(&k.d_list, sizeof(int) * k.cases.size()));
      CK(cudaMemcpy(k.d_list, k.cases.data(), sizeof(int) * k.cases.size(), cudaMemcpyHostToDevice));
      const void* fn = pcg_fn(k.cpt);
      int optin = 0;
      CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
      cudaFuncAttributes fa;
      CK(cudaFuncGetAttributes(&fa, fn));
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    for (size_t k = 1; k < classes.size(); ++k) {
      cudaStream_t x;
      CK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
      side.push_back(x);
    }
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    for (size_t k = 0; k < classes.size(); ++k) {
      cudaEvent_t e;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev_join.push_back(e);
    }
    graphs.resize(m);
    warm_grids();
  }

  const void* pcg_fn(int cpt) {
    switch (cpt) {
      case 1: return (const void*)k_ls_pcg<T, 1>;
      case 2: return (const void*)k_ls_pcg<T, 2>;
      case 4: return (const void*)k_ls_pcg<T, 4>;
      case 8: return (const void*)k_ls_pcg<T, 8>;
      case 16: return (const void*)k_ls_pcg<T, 16>;
      case 32:
        if constexpr (sizeof(T) == 4) return (const void*)k_ls_pcg<T, 32>;
        break;
    }
    throw ApiError{FUGU_EINVAL, "lockstep batch: no PCG kernel for this cluster plan"};
  }

  // co-resident CTAs of a family kernel (its persistent grid)
  // (capped at the most virtual blocks the family can have: a larger grid
  // would only launch CTAs without work, which a small group pays for on
  // every launch)
  int grid_of(const void* fn, int tpb, long cap, size_t smem = 0) {
    auto it = grids.find(fn);
    if (it != grids.end()) return it->second;
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, tpb, smem));
    const int g = (int)std::max(1L, std::min((long)nsm * (occ > 0 ? occ : 1), cap));
    grids.emplace(fn, g);
    return g;
  }
  // the persistent grid of every family kernel, taken before any capture
  template <class F>
  void warm_box() { grid_of((const void*)k_ls_box<T, F>, LS_TPB, cap_box); }
  template <class F>
  void warm_e1() { grid_of((const void*)k_ls_e1<T, F>, LS_TPB, cap_e1); }
  void warm_grids() {
    warm_box<LsMatvecOuter<T>>(); warm_box<LsPoissonCoefs<T>>();
    warm_box<LsSchur<T>>(); warm_box<LsZwork<T>>(); warm_box<LsCross<T>>(); warm_box<LsRbsor<T>>();
    warm_box<LsJacobi<T>>();
    warm_e1<LsCvtCoefs<T>>(); warm_e1<LsDefect<T>>(); warm_e1<LsUpdate64<T>>(); warm_e1<LsScaleDefect<T>>();
    warm_e1<LsZeroCorrection<T>>(); warm_e1<LsAccumulate<T>>(); warm_e1<LsFgScale<T>>(); warm_e1<LsZeroPcd<T>>();
    warm_e1<LsJacobiCopy<T>>();
    grid_of((const void*)k_ls_dot<T>, DOT_TPB, cap_dot);
    grid_of((const void*)k_ls_mdot<T>, MDOT_TPB, cap_mdot);
    grid_of((const void*)k_ls_maxpy<T>, LS_TPB, cap_e1);
    grid_of((const void*)k_ls_rbsor<T>, RB_TPB, cap_tile);
    CK(cudaFuncSetAttribute((const void*)k_ls_matvec<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            mt_matvec_smem<T, RB_TY>()));
    grid_of((const void*)k_ls_matvec<T>, MT_TPB, cap_tile, mt_matvec_smem<T, RB_TY>());
  }

  // ------------------------------------------------------- launches
  template <class F>
  void box(F f) {
    const void* fn = (const void*)k_ls_box<T, F>;
    k_ls_box<T, F><<<grid_of(fn, LS_TPB, cap_box), LS_TPB, 0, q>>>(d_cases, d_dyn, d_plan, f);
    LSCKL("k_ls_box");
  }
  template <class F>
  void e1(F f) {
    const void* fn = (const void*)k_ls_e1<T, F>;
    k_ls_e1<T, F><<<grid_of(fn, LS_TPB, cap_e1), LS_TPB, 0, q>>>(d_cases, d_dyn, d_plan, f);
    LSCKL("k_ls_e1");
  }
  template <class F>
  void one(F f) {
    k_ls_one<T, F><<<ncase, 1024, 0, q>>>(d_cases, d_dyn, d_plan, f);
    LSCKL("k_ls_one");
  }
  template <class F>
  void all(F f) {
    k_ls_all<T, F><<<ncase, 128, 0, q>>>(d_cases, d_dyn, ncase, f);
    LSCKL("k_ls_all");
  }
  void plan(int src, int nvec) {
    k_ls_plan<T><<<1, LS_MAX, 0, q>>>(d_cases, d_dyn, ncase, src, nvec, d_plan);
    LSCKL("k_ls_plan");
  }
  void dot(int which, int op) {
    const void* fn = (const void*)k_ls_dot<T>;
    k_ls_dot<T><<<grid_of(fn, DOT_TPB, cap_dot), DOT_TPB, 0, q>>>(d_cases, d_plan, which, OpArgs{op, 0, 0.0});
    LSCKL("k_ls_dot");
  }
  void mdot(int which, int nvec, int op, int j) {
    const void* fn = (const void*)k_ls_mdot<T>;
    k_ls_mdot<T><<<grid_of(fn, MDOT_TPB, cap_mdot), MDOT_TPB, 0, q>>>(d_cases, d_plan, which, nvec, op, j, m);
    LSCKL("k_ls_mdot");
  }
  void maxpy(int which, int nvec) {
    const void* fn = (const void*)k_ls_maxpy<T>;
    k_ls_maxpy<T><<<grid_of(fn, LS_TPB, cap_e1), LS_TPB, 0, q>>>(d_cases, d_plan, which, nvec, m);
    LSCKL("k_ls_maxpy");
  }
  // the PCD's PCG of every grid class, the classes side by side
  void pcg(int j) {
    if (classes.size() > 1) CK(cudaEventRecord(ev_fork, q));
    for (size_t k = 0; k < classes.size(); ++k) {
      const LsClass& cl = classes[k];
      cudaStream_t st = k == 0 ? q : side[k - 1];
      if (k > 0) CK(cudaStreamWaitEvent(st, ev_fork, 0));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(cl.C * cl.cases.size()), 1, 1);
      cfg.blockDim = dim3(PCGC_TPB, 1, 1);
      cfg.dynamicSmemBytes = cl.smem;
      cfg.stream = st;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = cl.C;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      const LsCase<T>* a0 = d_cases;
      const LsDyn* a1 = d_dyn;
      const int* a2 = cl.d_list;
      int a3 = cl.rows_per, a4 = j;
      void* args[] = {&a0, &a1, &a2, &a3, &a4};
      CK(cudaLaunchKernelExC(&cfg, pcg_fn(cl.cpt), args));
      ++launches;
      if (k > 0) {
        CK(cudaEventRecord(ev_join[k], st));
        CK(cudaStreamWaitEvent(q, ev_join[k], 0));
      }
    }
  }
  void sync() {
    CK(cudaStreamSynchronize(s));
    ring_next = 0;  // every queued upload has been read
  }
  void upload_dyn() {
    if (ring_next == RING) sync();
    LsDyn* src = h_ring + (size_t)ring_next++ * ncase;
    std::memcpy(src, h_dyn, sizeof(LsDyn) * ncase);
    CK(cudaMemcpyAsync(d_dyn, src, sizeof(LsDyn) * ncase, cudaMemcpyHostToDevice, s));
  }
  // run flags: the running cases (or only the cases in ids)
  void set_run(const std::vector<int>* ids = nullptr) {
    for (int i = 0; i < ncase; ++i) h_dyn[i].run = ids ? 0 : running[i];
    if (ids)
      for (int i : *ids) h_dyn[i].run = 1;
  }
  void readback() {
    all(LsReadback<T>{d_read, m});
    CK(cudaMemcpyAsync(h_read, d_read, sizeof(LsRead) * ncase, cudaMemcpyDeviceToHost, s));
    sync();
  }

  // ----------------------------------------------- one Arnoldi step j
  // (pcd, wall BCs, matvec, CGS2, new basis vector: fgmres() in fugu_gpu.cu),
  // then the plan of step j + 1
  void helmholtz(int j, int comp, int max_sw) {
    if (smoother == 1 && !any_periodic) {  // both colours of a sweep in one launch
      const void* fn = (const void*)k_ls_rbsor<T>;
      for (int sw = 0; sw < max_sw; ++sw) {
        k_ls_rbsor<T><<<grid_of(fn, RB_TPB, cap_tile), RB_TPB, 0, q>>>(d_cases, d_dyn, d_plan, j, comp, sw);
        LSCKL("k_ls_rbsor");
      }
      e1(LsJacobiCopy<T>{j, comp});
      return;
    }
    if (smoother == 1) {
      for (int sw = 0; sw < max_sw; ++sw)
        for (int col = 0; col < 2; ++col) {
          if (any_periodic) one(LsHalo<T>{LB_ZJ, comp, j, sw});
          box(LsRbsor<T>{j, comp, sw, col});
        }
      return;
    }
    for (int sw = 0; sw < max_sw; ++sw) {
      if (any_periodic) one(LsHalo<T>{LB_JTMP, comp, j, sw});
      box(LsJacobi<T>{j, comp, sw});
    }
    e1(LsJacobiCopy<T>{j, comp});
  }
  void arnoldi_step(int j, int max_sw, bool count_to_host) {
    const FgLayout L{m};
    e1(LsZeroPcd<T>{j});
    pcg(j);
    if (any_periodic) one(LsHalo<T>{LB_PHI, 2, j, -1});
    box(LsSchur<T>{j});
    if (any_periodic) one(LsHalo<T>{LB_ZJ, 2, j, -1});
    box(LsZwork<T>{j});
    helmholtz(j, 1, max_sw);
    if (any_periodic) one(LsHalo<T>{LB_ZJ, 1, j, -1});
    box(LsCross<T>{j});
    helmholtz(j, 0, max_sw);
    if (any_periodic) one(LsHalo<T>{LB_ZJ, 0, j, -1});
    one(LsVbcs<T>{LB_ZJ, j, 0});
    if (any_periodic)
      for (int comp = 0; comp < 3; ++comp) one(LsHalo<T>{LB_ZJ, comp, j, -1});
    {
      const void* fn = (const void*)k_ls_matvec<T>;
      k_ls_matvec<T><<<grid_of(fn, MT_TPB, cap_tile), MT_TPB, mt_matvec_smem<T, RB_TY>(), q>>>(d_cases, d_dyn, d_plan, j);
      LSCKL("k_ls_matvec");
    }
    mdot(1, j + 1, FG_PROJ1, j);
    maxpy(0, j + 1);
    mdot(1, j + 1, FG_PROJ2, j);
    maxpy(0, j + 1);
    mdot(2, 1, FG_ROTATE, j);
    e1(LsFgScale<T>{j + 1, L.inv()});
    plan(1, j + 2);
    if (count_to_host) CK(cudaMemcpyAsync(h_nact, &d_plan->n, sizeof(int), cudaMemcpyDeviceToHost, q));
  }
  void run_step_graph(int j, int max_sw) {
    Graph& g = graphs[j];
    if (!g.exec || g.max_sweeps != max_sw) {
      cudaGraph_t graph;
      const unsigned long long before = launches;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        arnoldi_step(j, max_sw, true);
        g.launches = launches - before;
        launches = before;
      } catch (...) {
        launches = before;
        cudaGraph_t junk;
        cudaStreamEndCapture(s, &junk);
        if (junk) cudaGraphDestroy(junk);
        throw;
      }
      CK(cudaStreamEndCapture(s, &graph));
      if (g.exec) CK(cudaGraphExecDestroy(g.exec));
      g.exec = nullptr;
      const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      CK(e);
      g.max_sweeps = max_sw;
    }
    CK(cudaGraphLaunch(g.exec, s));
    launches += g.launches;
  }

  // The whole cycle as one graph: the cycle's set-up, then per Arnoldi step j
  // a one-thread kernel that arms a conditional IF node with "some case is
  // still active" and the IF node whose body is step j (ending with the plan
  // of step j + 1), then the back substitution and the update.  A step whose
  // node is not armed is skipped on the device, and so is every later one.
  void build_cycle(int max_sw) {
    const FgLayout L{m};
    Cycle& cyc = cycles[max_sw];
    if (cyc.exec) CK(cudaGraphExecDestroy(cyc.exec));
    cyc.exec = nullptr;
    const unsigned long long before = launches;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    bool body_open = false;
    try {
      q = s;
      all(LsResetKs{});
      plan(0, 1);
      one(LsZeroSt<T>{L.size()});
      mdot(0, 1, FG_BETA, 0);
      e1(LsFgScale<T>{0, L.inv()});
      plan(1, 1);
      const unsigned long long head0 = launches - before;
      unsigned long long body = 0;
      for (int j = 0; j < m; ++j) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
        cudaGraphConditionalHandle h;
        CK(cudaGraphConditionalHandleCreate(&h, cg, 0, 0));
        k_ls_cond<<<1, 32, 0, s>>>(d_plan, h);
        LSCKL("k_ls_cond");
        CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, cg, deps, nd, &cp));
        CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t bg = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(s2, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        body_open = true;
        q = s2;
        const unsigned long long b0 = launches;
        arnoldi_step(j, max_sw, false);
        body = launches - b0;
        q = s;
        cudaGraph_t bout = nullptr;
        body_open = false;
        CK(cudaStreamEndCapture(s2, &bout));
      }
      const unsigned long long t0 = launches;
      plan(0, 1);
      one(LsFgSolve<T>{m});
      maxpy(1, 0);
      cyc.head = head0 + (unsigned long long)m + (launches - t0);
      cyc.body = body;
    } catch (...) {
      q = s;
      launches = before;
      if (body_open) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(s2, &junk);
      }
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(s, &junk);
      if (junk) cudaGraphDestroy(junk);
      throw;
    }
    launches = before;
    CK(cudaStreamEndCapture(s, &graph));
    const cudaError_t e = cudaGraphInstantiate(&cyc.exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(e);
  }

  // one flexible-GMRES(m) cycle of every running case from a zero correction
  void fgmres_cycle(int max_sw) {
    if (use_cycle_graph && !cycles[max_sw].exec) {
      try {
        build_cycle(max_sw);
      } catch (const CudaError&) {
        // a runtime that cannot build the conditional graph: launch the
        // steps one graph at a time, with a host check between them
        cudaGetLastError();
        use_cycle_graph = false;
      }
    }
    if (use_cycle_graph) {
      const Cycle& cyc = cycles[max_sw];
      CK(cudaGraphLaunch(cyc.exec, s));
      launches += cyc.head;  // the executed steps' launches are added after the cycle
      cyc_body = cyc.body;
      return;
    }
    const FgLayout L{m};
    all(LsResetKs{});
    plan(0, 1);
    one(LsZeroSt<T>{L.size()});
    mdot(0, 1, FG_BETA, 0);
    e1(LsFgScale<T>{0, L.inv()});
    plan(1, 1);
    CK(cudaMemcpyAsync(h_nact, &d_plan->n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int j = 0; j < m && *h_nact > 0; ++j) {
      NvtxRange r_it("lockstep_arnoldi_step");
      run_step_graph(j, max_sw);
      CK(cudaStreamSynchronize(s));
    }
    plan(0, 1);
    one(LsFgSolve<T>{m});
    maxpy(1, 0);
  }

  // ------------------------------------------------ the lockstep solve
  // refine_solve (fugu_gpu.cu) for every running case at once, split at its
  // host checks so that cases can join and leave at every pass
  unsigned long long cyc_body = 0;  // launches of one executed Arnoldi step of the last cycle

  void reset() override {
    CK(cudaSetDevice(device));
    sync();
    running.assign(ncase, 0);
  }

  void join(const std::vector<int>& ids, const std::vector<StepSetup>& su) override {
    CK(cudaSetDevice(device));
    q = s;
    for (int i : ids) {
      fugu_ctx* c = cases[i];
      const fugu_params& p = c->prm;
      LsCaseRun& r = cr[i];
      r = LsCaseRun{};
      r.adapt = p.pcg_cap_start > 0;
      r.adapt_sw = p.pcd_sweeps_max > p.pcd_sweeps;
      if (r.adapt) r.cap = std::min(std::max(p.pcg_cap_start, c->pcg_cap_state), p.pcg_max_iter);
      if (r.adapt_sw) r.sweeps = std::min(std::max(p.pcd_sweeps, c->pcd_sweeps_state), p.pcd_sweeps_max);
      r.tol = su[i].tol;
      LsDyn& d = h_dyn[i];
      d.pcg_cap = r.cap > 0 ? r.cap : p.pcg_max_iter;
      d.sweeps = r.sweeps > 0 ? r.sweeps : p.pcd_sweeps;
      d.pen = su[i].pen ? 1 : 0;
      d.amp = su[i].amp ? 1 : 0;
      d.has_lid = 1;  // the step always passes its lid (zero when absent)
      d.dt = su[i].dt_eff;
      d.lid = su[i].lid;
    }
    set_run(&ids);
    upload_dyn();
    plan(0, 1);
    if constexpr (sizeof(T) == 4) e1(LsCvtCoefs<T>{});
    box(LsPoissonCoefs<T>{});
    all(LsResetKs{});
    one(LsVbcs<T>{LB_X, 0, 0});
    dot(0, OP_REF_NORMB);
    for (int i : ids) running[i] = 1;
  }

  std::vector<int> defect() override {
    NvtxRange r_pass("lockstep_defect_correction_pass");
    q = s;
    set_run();
    upload_dyn();
    plan(0, 1);
    if (any_periodic)
      for (int comp = 0; comp < 3; ++comp) one(LsHalo<T>{LB_X, comp, 0, -1});
    box(LsMatvecOuter<T>{});
    e1(LsDefect<T>{});
    dot(1, OP_REF_REL);
    readback();
    std::vector<int> ended;
    for (int i = 0; i < ncase; ++i) {
      if (!running[i]) continue;
      LsCaseRun& r = cr[i];
      const double rel = h_read[i].true_rel;
      r.rel = rel;
      if (h_read[i].nan || std::isnan(rel)) r.status = FUGU_NAN;
      else if (rel < r.tol) r.status = FUGU_CONVERGED;
      else if (r.outer >= cases[i]->prm.refine_max_outer) r.status = FUGU_MAXITER;
      else continue;
      r.done = true;
      ended.push_back(i);
    }
    return ended;
  }

  void finish(const std::vector<int>& ids, std::vector<KrylovResult>& kr, std::vector<int>& outer) override {
    q = s;
    for (int i : ids) running[i] = 0;
    if (ids.empty()) return;
    // the lid (refine_solve's final vbcs with has_lid)
    set_run(&ids);
    upload_dyn();
    plan(0, 1);
    one(LsVbcs<T>{LB_X, 0, 1});
    for (int i : ids) {
      fugu_ctx* c = cases[i];
      const LsCaseRun& r = cr[i];
      if (r.adapt) c->pcg_cap_state = r.cap;
      if (r.adapt_sw) c->pcd_sweeps_state = r.sweeps;
      kr[i].iter = r.inner_total;
      kr[i].res = r.rel;
      kr[i].status = r.status;
      outer[i] = r.outer;
    }
  }

  bool cycle_launch() override {
    q = s;
    int max_sw = 0;
    bool any = false;
    for (int i = 0; i < ncase; ++i)
      if (running[i]) {
        any = true;
        max_sw = std::max(max_sw, h_dyn[i].sweeps);
      }
    if (!any) return false;
    set_run();
    upload_dyn();
    plan(0, 1);
    if constexpr (sizeof(T) == 4) e1(LsScaleDefect<T>{});
    else e1(LsZeroCorrection<T>{});
    fgmres_cycle(max_sw);
    plan(0, 1);
    if constexpr (sizeof(T) == 4) e1(LsAccumulate<T>{});
    else e1(LsUpdate64<T>{});
    return true;
  }

  void cycle_finish() override {
    readback();
    int steps_run = 0;
    for (int i = 0; i < ncase; ++i)
      if (running[i]) steps_run = std::max(steps_run, h_read[i].active ? m : h_read[i].exit_iter);
    if (use_cycle_graph) launches += cyc_body * (unsigned long long)steps_run;
    for (int i = 0; i < ncase; ++i) {
      if (!running[i]) continue;
      LsCaseRun& r = cr[i];
      const fugu_params& p = cases[i]->prm;
      const LsRead& rd = h_read[i];
      r.inner_total += rd.active ? m : rd.exit_iter;
      const double ir = rd.inner_rel;
      LsDyn& d = h_dyn[i];
      if (!(ir < p.refine_inner_tol)) {
        if (r.adapt && r.cap < p.pcg_max_iter) {
          r.cap = std::min(2 * r.cap, p.pcg_max_iter);
          d.pcg_cap = r.cap;
        } else if (r.adapt_sw && r.sweeps < p.pcd_sweeps_max) {
          r.sweeps = std::min(2 * r.sweeps, p.pcd_sweeps_max);
          d.sweeps = r.sweeps;
        }
      }
      ++r.outer;
    }
    set_run();
    upload_dyn();
    plan(0, 1);
    all(LsResetKs{});
    one(LsVbcs<T>{LB_X, 0, 0});
  }
};

}  // namespace
