// rowbench.cu -- kernel timing on synthetic fields of the padded box: the
// damped-Jacobi sweep, the PCD's Schur, residual and cross steps (one thread
// per element against the vectorised row kernels, and the staged six-sweep
// kernel), the Gram-Schmidt multi-axpy k_maxpy (16-byte path against the
// one-element path) and a device copy, at n x n for n = 256 ... 4096, FP32
// and FP64.  Each kernel is timed with CUDA events over back-to-back
// launches that rotate through four sets of fields (together far larger
// than L2 from 1024^2 up); GB/s = the kernel's algorithmic bytes (each
// distinct array read once and written once over the n x n interior) per
// launch time.  Before timing, every vectorised kernel's output is compared
// with the scalar kernel's bit for bit on the same inputs.
//
// Build and run (one GPU):
//   python -m coupled_codefort_2d_b200.build --rowbench
//   coupled_codefort_2d_b200/rowbench [peak GB/s]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <random>
#include "fgmres.cuh"
#include "kernels.cuh"
using namespace fugu;

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { printf("CUDA %s at %d\n", cudaGetErrorString(e_), __LINE__); exit(1); } } while (0)

template <typename T>
struct Set {
  T *uo, *un, *rhs, *rho, *kap, *zeta, *eta, *phi, *ua, *va, *rp, *zp, *zu, *zv, *zuw, *zvw, *rv;
};

template <typename T>
__global__ void k_fill(T* p, long n, unsigned seed, double lo, double hi) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    unsigned long long x = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed * 0xBF58476D1CE4E5B9ull;
    x ^= x >> 31; x *= 0x94D049BB133111EBull; x ^= x >> 29;
    p[i] = T(lo + (hi - lo) * double(x >> 11) * (1.0 / 9007199254740992.0));
  }
}
template <typename T>
T* dev_rand(long n, std::mt19937& r, double lo, double hi) {
  T* p;
  CK(cudaMalloc(&p, sizeof(T) * n));
  k_fill<T><<<1184, 256>>>(p, n, (unsigned)r(), lo, hi);
  CK(cudaGetLastError());
  return p;
}

// plain per-element restatement of k_maxpy's updates (the order of the
// FGMRES projection: x = w; x = s_i v_i + x for i = 0 .. nvec-1)
template <typename T>
__global__ void k_maxpy_ref(long n3, T* w, const T* V0, long stride, const double* coef, int nvec, double sign) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n3; q += (long)gridDim.x * blockDim.x) {
    T x = w[q];
    for (int i = 0; i < nvec; ++i) x = madd(T(sign * coef[i]), V0[i * stride + q], x);
    w[q] = x;
  }
}

template <typename T>
bool same(const T* a, const T* b, long n) {
  std::vector<T> x(n), y(n);
  CK(cudaMemcpy(x.data(), a, sizeof(T) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(y.data(), b, sizeof(T) * n, cudaMemcpyDeviceToHost));
  return memcmp(x.data(), y.data(), sizeof(T) * n) == 0;
}

template <typename T, typename F>
float time_it(F f, int reps) {
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  for (int i = 0; i < 3; ++i) f(i);
  CK(cudaDeviceSynchronize());
  CK(cudaEventRecord(a));
  for (int i = 0; i < reps; ++i) f(i);
  CK(cudaEventRecord(b));
  CK(cudaEventSynchronize(b));
  float ms;
  CK(cudaEventElapsedTime(&ms, a, b));
  CK(cudaGetLastError());
  return 1000.f * ms / reps;
}

template <typename T>
void run(int nx, double peak) {
  Geo g{};
  g.nx = nx; g.ny = nx; g.P = ((nx + 5 + 15) / 16) * 16; g.R = nx + 5;
  g.dx = g.dy = 1.0 / nx; g.idx = g.idy = nx; g.idx2 = g.idy2 = double(nx) * nx;
  const long n = g.n();
  std::mt19937 r(7);
  const int NS = 4;
  Set<T> s[NS];
  for (int k = 0; k < NS; ++k) {
    s[k].uo = dev_rand<T>(n, r, -1, 1); s[k].un = dev_rand<T>(n, r, -1, 1); s[k].rhs = dev_rand<T>(n, r, -1, 1);
    s[k].rho = dev_rand<T>(n, r, 0.1, 1); s[k].kap = dev_rand<T>(n, r, 0.01, 1); s[k].zeta = dev_rand<T>(n, r, 0.01, 1);
    s[k].eta = dev_rand<T>(n, r, 0.001, 0.005); s[k].phi = dev_rand<T>(n, r, -1, 1); s[k].ua = dev_rand<T>(n, r, -1, 1);
    s[k].va = dev_rand<T>(n, r, -1, 1); s[k].rp = dev_rand<T>(n, r, -1, 1); s[k].zp = dev_rand<T>(n, r, -1, 1);
    s[k].zu = dev_rand<T>(n, r, -1, 1); s[k].zv = dev_rand<T>(n, r, -1, 1); s[k].zuw = dev_rand<T>(n, r, -1, 1);
    s[k].zvw = dev_rand<T>(n, r, -1, 1); s[k].rv = dev_rand<T>(n, r, -1, 1);
  }
  T* chk = dev_rand<T>(n, r, 0, 1);
  T* chk2 = dev_rand<T>(n, r, 0, 1);
  Box b = box_launch(g);
  constexpr int W = VecW<T>::value;
  const dim3 vg((g.P + VEC_TX * W - 1) / (VEC_TX * W), (g.R + VEC_TY - 1) / VEC_TY), vb(VEC_TX, VEC_TY);
  const dim3 mg((g.P + JM_TX - 1) / JM_TX, (g.R + JM_TY - 1) / JM_TY);
  CK(cudaFuncSetAttribute((const void*)k_jacobi_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(JmSmem<T>)));
  const T dt = T(1e-3), om = T(0.8);
  const double cells = double(nx) * nx, B = sizeof(T);
  const int reps = nx >= 2048 ? 40 : 200;
  const char* tn = sizeof(T) == 4 ? "f32" : "f64";
  // bitwise checks
  for (int comp = 0; comp < 2; ++comp) {
    Set<T>& a = s[0];
    if (comp == 0) k_jacobi_u<T><<<b.grid, b.block>>>(g, a.uo, chk, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr);
    else k_jacobi_v<T><<<b.grid, b.block>>>(g, a.uo, chk, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr);
    k_jacobi_vec<T><<<vg, vb>>>(g, comp, a.uo, chk2, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr);
    CK(cudaDeviceSynchronize());
    printf("check %s n=%d jacobi comp %d: %s\n", tn, nx, comp, same(chk, chk2, n) ? "same" : "DIFFER");
  }
  {
    Set<T>& a = s[0];
    k_pcd_schur<T><<<b.grid, b.block>>>(g, a.phi, a.ua, a.va, chk, T(1000), a.kap, a.zp, T(1), nullptr);
    k_pcd_schur_vec<T><<<vg, vb>>>(g, a.phi, a.ua, a.va, chk2, T(1000), a.kap, a.zp, T(1), nullptr);
    CK(cudaDeviceSynchronize());
    printf("check %s n=%d schur: %s\n", tn, nx, same(chk, chk2, n) ? "same" : "DIFFER");
    k_pcd_zwork<T><<<b.grid, b.block>>>(g, a.zu, a.zv, a.rp, chk, a.zvw, nullptr);
    k_pcd_zwork_vec<T><<<vg, vb>>>(g, a.zu, a.zv, a.rp, chk2, a.zuw, nullptr);
    CK(cudaDeviceSynchronize());
    printf("check %s n=%d zwork: %s %s\n", tn, nx, same(chk, chk2, n) ? "same" : "DIFFER", same(a.zvw, a.zuw, n) ? "same" : "DIFFER");
    CK(cudaMemcpy(chk2, chk, sizeof(T) * n, cudaMemcpyDeviceToDevice));
    k_pcd_cross<T><<<b.grid, b.block>>>(g, a.eta, a.rv, chk, nullptr);
    k_pcd_cross_vec<T><<<vg, vb>>>(g, a.eta, a.rv, chk2, nullptr);
    CK(cudaDeviceSynchronize());
    printf("check %s n=%d cross: %s\n", tn, nx, same(chk, chk2, n) ? "same" : "DIFFER");
  }
  auto rep = [&](const char* name, float us, double vals) {
    const double gbs = vals * B * cells / (us * 1e3);
    printf("%s n=%d %-22s %9.2f us  %7.1f GB/s  %.3f of %.0f\n", tn, nx, name, us, gbs, gbs / peak, peak);
  };
  rep("k_jacobi_u", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_jacobi_u<T><<<b.grid, b.block>>>(g, a.uo, a.un, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr); }, reps), 7);
  rep("k_jacobi_v", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_jacobi_v<T><<<b.grid, b.block>>>(g, a.uo, a.un, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr); }, reps), 7);
  rep("k_jacobi_vec u", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_jacobi_vec<T><<<vg, vb>>>(g, 0, a.uo, a.un, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr); }, reps), 7);
  rep("k_jacobi_vec v", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_jacobi_vec<T><<<vg, vb>>>(g, 1, a.uo, a.un, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr); }, reps), 7);
  rep("k_jacobi_multi u x6", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_jacobi_multi<T><<<mg, JM_TPB, sizeof(JmSmem<T>)>>>(g, 0, 6, a.uo, a.un, a.rhs, a.rho, a.kap, a.zeta, a.eta, nullptr, dt, om, nullptr); }, reps), 7);
  rep("k_pcd_schur", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_schur<T><<<b.grid, b.block>>>(g, a.phi, a.ua, a.va, a.rp, T(1000), a.kap, a.zp, T(0), nullptr); }, reps), 4);
  rep("k_pcd_schur_vec", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_schur_vec<T><<<vg, vb>>>(g, a.phi, a.ua, a.va, a.rp, T(1000), a.kap, a.zp, T(0), nullptr); }, reps), 4);
  rep("k_pcd_zwork", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_zwork<T><<<b.grid, b.block>>>(g, a.zu, a.zv, a.rp, a.zuw, a.zvw, nullptr); }, reps), 5);
  rep("k_pcd_zwork_vec", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_zwork_vec<T><<<vg, vb>>>(g, a.zu, a.zv, a.rp, a.zuw, a.zvw, nullptr); }, reps), 5);
  rep("k_pcd_cross", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_cross<T><<<b.grid, b.block>>>(g, a.eta, a.rv, a.zuw, nullptr); }, reps), 4);
  rep("k_pcd_cross_vec", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    k_pcd_cross_vec<T><<<vg, vb>>>(g, a.eta, a.rv, a.zuw, nullptr); }, reps), 4);
  {
    // k_maxpy over nvec basis vectors of the coupled triple (3 boxes): the
    // 16-byte path (aligned) against the one-element path (the same call
    // shifted by one element, which the alignment test sends there); bits
    // checked against a plain per-element evaluation of the same updates
    const long n3 = 3 * n;
    const int NV = 16;
    T* V = dev_rand<T>(n3 * NV + 16, r, -1, 1);
    T* w0 = dev_rand<T>(n3 + 16, r, -1, 1);
    T* wa = dev_rand<T>(n3 + 16, r, -1, 1);
    T* wb = dev_rand<T>(n3 + 16, r, -1, 1);
    double* coef;
    CK(cudaMalloc(&coef, sizeof(double) * NV));
    k_fill<double><<<1, 32>>>(coef, NV, 99u, -0.5, 0.5);
    const int g1 = (int)std::min<long>((n3 + 255) / 256, 148L * 8);
    for (int nv : {1, 4, 8, 15}) {
      CK(cudaMemcpy(wa, w0, sizeof(T) * (n3 + 16), cudaMemcpyDeviceToDevice));
      CK(cudaMemcpy(wb, w0, sizeof(T) * (n3 + 16), cudaMemcpyDeviceToDevice));
      k_maxpy<T><<<g1, 256>>>(n3, wa, V, n3, coef, nv, -1.0, nullptr);
      k_maxpy_ref<T><<<g1, 256>>>(n3, wb, V, n3, coef, nv, -1.0);
      CK(cudaDeviceSynchronize());
      printf("check %s n=%d maxpy k=%d: %s\n", tn, nx, nv, same(wa, wb, n3) ? "same" : "DIFFER");
      char nm[64];
      snprintf(nm, sizeof nm, "k_maxpy k=%d vec", nv);
      rep(nm, time_it<T>([&](int) { k_maxpy<T><<<g1, 256>>>(n3, wa, V, n3, coef, nv, -1.0, nullptr); }, reps),
          3.0 * (nv + 2) * n / cells);
      snprintf(nm, sizeof nm, "k_maxpy k=%d scalar", nv);
      rep(nm, time_it<T>([&](int) { k_maxpy<T><<<g1, 256>>>(n3 - 1, wa + 1, V + 1, n3, coef, nv, -1.0, nullptr); },
                         reps),
          3.0 * (nv + 2) * n / cells);
    }
    CK(cudaFree(V)); CK(cudaFree(w0)); CK(cudaFree(wa)); CK(cudaFree(wb)); CK(cudaFree(coef));
  }
  rep("copy (1R+1W)", time_it<T>([&](int i) { Set<T>& a = s[i % NS];
    CK(cudaMemcpyAsync(a.un, a.uo, sizeof(T) * n, cudaMemcpyDeviceToDevice)); }, reps), 2);
  for (int k = 0; k < NS; ++k) {
    T** p = (T**)&s[k];
    for (size_t q = 0; q < sizeof(Set<T>) / sizeof(T*); ++q) CK(cudaFree(p[q]));
  }
  CK(cudaFree(chk));
  CK(cudaFree(chk2));
}

int main(int argc, char** argv) {
  const double peak = argc > 1 ? atof(argv[1]) : 6560.6;
  for (int nx : {256, 512, 1024, 2048, 4096}) {
    run<float>(nx, peak);
    run<double>(nx, peak);
  }
  return 0;
}
