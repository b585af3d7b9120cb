// fm_flowmap.cu -- flow-map transport kernels and their C ABI (sm_100a).
//
// Gather kernels (one thread per output node, B-spline taps read through the
// read-only path; the 128^3 working set sits in the 126 MB L2) for:
//   advect_u_grid / advect_scalar_grid   (3D/flowmap.py:202-320)
//   RK_grid / RK_grid_only_psi           (3D/flowmap.py:85-179)
//   advect_u / advect_scalar (pullback)  (3D/flowmap.py:51-79), BFECC epilogues
//   accumulate_init / accumulate_init_new(3D/flowmap.py:485-545)
//   calculate_nabla_u_w / _scalar_adjoint(3D/flowmap.py:359-403)
//   reset_to_identity, add_fields
#include "fm_common.cuh"
#include "fm_internal.h"
#include "fm_q2.cuh"

#include <mutex>
#include <unordered_map>

namespace fm {

constexpr int kThreads = 256;

// CTAs per SM the march kernel is compiled for: 3 in FP32 (80 registers; 0.697
// vs 0.723 ms per 128^3 RK4 launch at 2 CTAs / 128 registers; 4 CTAs force 64
// registers with spills and measure no faster), 2 in FP64 (80 registers would
// spill over 1 KB per thread there).
template <typename T>
constexpr int march_min_blocks() {
  return sizeof(T) == 4 ? 3 : 2;
}

// Midpoint (RK2) / RK4 backtrace from X through u0 (3D/flowmap.py:210-219, :257-262).
template <typename T, int D, int RK>
__device__ __forceinline__ void backtrace(const Mac<T>& u0, const fm_grid& g, const Q2Lim<T>& lim, const T* X,
                                          T inv_dx, T dt, T* p) {
  T v[3], vs[3], q[3] = {0, 0, 0};
  q2_mac_val<T, D>(u0, g, lim, X, inv_dx, v);
#pragma unroll
  for (int a = 0; a < D; ++a) q[a] = X[a] - v[a] * dt * (T)0.5;
  if constexpr (RK == 2) {
    q2_mac_val<T, D>(u0, g, lim, q, inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = X[a] - v[a] * dt;
  } else {
    // v1 + 2 v2 + 2 v3 + v4 accumulated left to right as the stages complete
#pragma unroll
    for (int a = 0; a < D; ++a) vs[a] = v[a];
    q2_mac_val<T, D>(u0, g, lim, q, inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) { vs[a] = vs[a] + (T)2 * v[a]; q[a] = X[a] - v[a] * dt * (T)0.5; }
    q2_mac_val<T, D>(u0, g, lim, q, inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) { vs[a] = vs[a] + (T)2 * v[a]; q[a] = X[a] - v[a] * dt; }
    q2_mac_val<T, D>(u0, g, lim, q, inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = X[a] - (vs[a] + v[a]) / (T)6.0 * dt;
  }
}

// u2 = u1 sampled at the foot of the backtrace through u0; with u1b/u2b set,
// a second field is sampled at the same foot (the adjoint advects adj_u and u
// along the same midpoint velocity, 3D/lfm_midpoint_diff_simulator.py:488-499).
template <typename T, int D, int RK>
__global__ void __launch_bounds__(kThreads) k_advect_u_grid(fm_grid g, T dx, T dt, Mac<T> u0, Mac<T> u1,
                                                            MacW<T> u2, Mac<T> u1b, MacW<T> u2b) {
  const int c = blockIdx.y;
  const Shape s = face_shape(g, c);
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= s.size()) return;
  int i, j, k;
  unflatten(s, q, i, j, k);
  T X[3] = {0, 0, 0}, p[3] = {0, 0, 0};
  node_pos<T, D>(c, i, j, k, dx, X);
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  backtrace<T, D, RK>(u0, g, lim, X, inv_dx, dt, p);
  CompStencil<T, D> st;
  st.setup(lim, c, p, inv_dx);
  pick(u2, c)[q] = st.eval(pick(u1, c), s);
  if (u1b.c[0] != nullptr) pick(u2b, c)[q] = st.eval(pick(u1b, c), s);
}

template <typename T, int D, int RK>
__global__ void __launch_bounds__(kThreads) k_advect_scalar_grid(fm_grid g, T dx, T dt, Mac<T> u0,
                                                                 const T* __restrict__ s1, T* __restrict__ s2,
                                                                 const T* __restrict__ s1b, T* __restrict__ s2b) {
  const Shape s = cell_shape(g);
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= s.size()) return;
  int i, j, k;
  unflatten(s, q, i, j, k);
  T X[3] = {0, 0, 0}, p[3] = {0, 0, 0};
  node_pos<T, D>(-1, i, j, k, dx, X);
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  backtrace<T, D, RK>(u0, g, lim, X, inv_dx, dt, p);
  Q2<T, false> ax, ay, az;
  ax.setup(p[0] * inv_dx, (T)0.5, lim.h5[0]);
  ay.setup(p[1] * inv_dx, (T)0.5, lim.h5[1]);
  if (D == 3) az.setup(p[2] * inv_dx, (T)0.5, lim.h5[2]);
  s2[q] = q2_val<T, D, false>(s1, s, ax, ay, az);
  if (s1b != nullptr) s2b[q] = q2_val<T, D, false>(s1b, s, ax, ay, az);
}

// One march job: a flow map psi (D planes) on grid `face` (-1 = centre),
// optionally with its Jacobian rows T (D planes).
template <typename T>
struct MarchJob {
  T* psi;
  T* Tm;
  int face;
};
template <typename T>
struct MarchJobs {
  MarchJob<T> j[4];
};

// One RK stage: velocity k = u(pos) and, with the Jacobian, d = (grad u)(pos) . t.
template <typename T, int D, bool WT>
__device__ __forceinline__ void march_eval(const Mac<T>& u, const fm_grid& g, const Q2Lim<T>& lim, const T* pos,
                                           const T* t, T inv_dx, T* k, T* d) {
  if constexpr (WT) q2_mac_grad_dot<T, D>(u, g, lim, pos, inv_dx, t, k, d);
  else q2_mac_val<T, D>(u, g, lim, pos, inv_dx, k);
}

// RK2_grid / RK4_grid (WT) and RK*_grid_only_psi (!WT) for one node, in place.
// The RK4 sums (k1 + 2 k2 + 2 k3 + k4) are accumulated as the stages complete,
// in the reference's left-to-right order.
template <typename T, int D, int RK, bool WT>
__device__ __forceinline__ void march_node(const Mac<T>& u, const fm_grid& g, T dx, T dt, T* psi, T* Tm, long N,
                                           long q) {
  T P[3] = {0, 0, 0}, Tv[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    P[a] = psi[a * N + q];
    if constexpr (WT) Tv[a] = Tm[a * N + q];
  }
  const T neg_dt = -dt;
  const T h = (T)0.5 * neg_dt;
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  T k[3], d[3] = {0, 0, 0}, pos[3] = {0, 0, 0}, tt[3] = {0, 0, 0};
  march_eval<T, D, WT>(u, g, lim, P, Tv, inv_dx, k, d);
  if constexpr (RK == 2) {
#pragma unroll
    for (int a = 0; a < D; ++a) { pos[a] = P[a] + h * k[a]; tt[a] = Tv[a] + h * d[a]; }
    march_eval<T, D, WT>(u, g, lim, pos, tt, inv_dx, k, d);
#pragma unroll
    for (int a = 0; a < D; ++a) {
      psi[a * N + q] = P[a] + neg_dt * k[a];
      if constexpr (WT) Tm[a * N + q] = Tv[a] + neg_dt * d[a];
    }
  } else {
    T ks[3], ds[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
      ks[a] = k[a];
      ds[a] = d[a];
      pos[a] = P[a] + h * k[a];
      tt[a] = Tv[a] + h * d[a];
    }
    march_eval<T, D, WT>(u, g, lim, pos, tt, inv_dx, k, d);  // stage 2
#pragma unroll
    for (int a = 0; a < D; ++a) {
      ks[a] = ks[a] + (T)2 * k[a];
      ds[a] = ds[a] + (T)2 * d[a];
      pos[a] = P[a] + h * k[a];
      tt[a] = Tv[a] + h * d[a];
    }
    march_eval<T, D, WT>(u, g, lim, pos, tt, inv_dx, k, d);  // stage 3
#pragma unroll
    for (int a = 0; a < D; ++a) {
      ks[a] = ks[a] + (T)2 * k[a];
      ds[a] = ds[a] + (T)2 * d[a];
      pos[a] = P[a] + (T)1.0 * neg_dt * k[a];
      tt[a] = Tv[a] + (T)1.0 * neg_dt * d[a];
    }
    march_eval<T, D, WT>(u, g, lim, pos, tt, inv_dx, k, d);  // stage 4
    const T c6 = neg_dt * (T)1 / (T)6;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      psi[a * N + q] = P[a] + c6 * (ks[a] + k[a]);
      if constexpr (WT) Tm[a * N + q] = Tv[a] + c6 * (ds[a] + d[a]);
    }
  }
}

template <typename T>
__device__ __forceinline__ MarchJob<T> pick_job(const MarchJobs<T>& jobs, int y) {
  return y == 0 ? jobs.j[0] : (y == 1 ? jobs.j[1] : (y == 2 ? jobs.j[2] : jobs.j[3]));
}

// RK2_grid / RK4_grid (with T) and RK*_grid_only_psi (without); blockIdx.y
// selects the job (face grids and/or the centre map of one march).
template <typename T, int D, int RK>
__global__ void __launch_bounds__(kThreads, march_min_blocks<T>()) k_march(fm_grid g, T dx, T dt, MarchJobs<T> jobs, Mac<T> u) {
  const MarchJob<T> job = pick_job(jobs, blockIdx.y);
  const Shape s = job.face >= 0 ? face_shape(g, job.face) : cell_shape(g);
  const long N = s.size();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  if (job.Tm != nullptr) march_node<T, D, RK, true>(u, g, dx, dt, job.psi, job.Tm, N, q);
  else march_node<T, D, RK, false>(u, g, dx, dt, job.psi, nullptr, N, q);
}

// out_c = alpha * (T_c . u0(psi_c) + beta * base_c)
template <typename T, int D>
__global__ void __launch_bounds__(kThreads) k_pullback_u(fm_grid g, T dx, Mac<T> u0, MacW<T> out, Mac<T> Tm,
                                                         Mac<T> psi, T alpha, T beta, Mac<T> base) {
  const int c = blockIdx.y;
  const Shape s = face_shape(g, c);
  const long N = s.size();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const T* psi_c = pick(psi, c);
  const T* T_c = pick(Tm, c);
  T p[3] = {0, 0, 0}, v[3];
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = psi_c[a * N + q];
  q2_mac_val<T, D>(u0, g, Q2Lim<T>(g), p, (T)1 / dx, v);
  T acc = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) acc += T_c[a * N + q] * v[a];
  if (beta != (T)0) acc = acc + beta * pick(base, c)[q];
  pick(out, c)[q] = alpha * acc;
}

template <typename T, int D>
__global__ void __launch_bounds__(kThreads) k_pullback_scalar(fm_grid g, T dx, const T* __restrict__ s0,
                                                              T* out, const T* __restrict__ psi, T alpha, T beta,
                                                              const T* base) {
  const Shape s = cell_shape(g);
  const long N = s.size();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  T p[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = psi[a * N + q];
  T acc = q2_scalar<T, D>(s0, g, Q2Lim<T>(g), p, (T)1 / dx);
  if (beta != (T)0) acc = acc + beta * base[q];
  out[q] = alpha * acc;
}

// With TWO, a second field f2 is accumulated afterwards with coefficient dt2 and
// no history, from the same positions and rows (the adjoint's passive-scalar
// source, 3D/lfm_midpoint_diff_simulator.py:519-523): the same operations as a
// second plain launch on the first one's result.
template <typename T, int D, bool AB3, bool TWO = false>
__global__ void __launch_bounds__(kThreads) k_accumulate(fm_grid g, T dx, T dt, int ind, Mac<T> f, MacW<T> init,
                                                         Mac<T> F, Mac<T> phi, MacW<T> Hp, MacW<T> Hpp,
                                                         Mac<T> f2 = Mac<T>{}, T dt2 = 0) {
  const int c = blockIdx.y;
  const Shape s = face_shape(g, c);
  const long N = s.size();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const T* phi_c = pick(phi, c);
  const T* F_c = pick(F, c);
  T p[3] = {0, 0, 0}, v[3], v2[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = phi_c[a * N + q];
  {
    MacStencil<T, D, false> st;
    st.setup(Q2Lim<T>(g), p, (T)1 / dx);
#pragma unroll
    for (int b = 0; b < D; ++b) {
      v[b] = q2_val<T, D, false>(f.c[b], face_shape(g, b), st.ax(b, 0), st.ax(b, 1), st.ax(b, 2 % D));
      if constexpr (TWO) v2[b] = q2_val<T, D, false>(f2.c[b], face_shape(g, b), st.ax(b, 0), st.ax(b, 1), st.ax(b, 2 % D));
    }
  }
  T Fv = 0, Fv23 = 0, Fv16 = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const T Fa = F_c[a * N + q];
    Fv += Fa * v[a];
    if (AB3) { Fv23 += ((T)23 * Fa) * v[a]; Fv16 += ((T)16 * Fa) * v[a]; }
  }
  T* init_c = pick(init, c);
  T acc = init_c[q];
  if (!AB3 || ind == 0) {
    acc += Fv * dt;
  } else {
    const T hp = pick(Hp, c)[q];
    if (ind == 1) acc += (Fv23 - Fv16 + (T)5 * hp) / (T)12 * dt;
    else acc += (Fv23 - (T)16 * hp + (T)5 * pick(Hpp, c)[q]) / (T)12 * dt;
  }
  if (AB3) {  // history shifts on every call, ind == 0 included
    T* hp_c = pick(Hp, c);
    pick(Hpp, c)[q] = hp_c[q];
    hp_c[q] = Fv;
  }
  if constexpr (TWO) {
    T Fv2 = 0;
#pragma unroll
    for (int a = 0; a < D; ++a) Fv2 += F_c[a * N + q] * v2[a];
    acc += Fv2 * dt2;
  }
  init_c[q] = acc;
}

template <typename T, int D>
__global__ void k_reset_identity(fm_grid g, T dx, MarchJobs<T> jobs) {
  const MarchJob<T> job = pick_job(jobs, blockIdx.y);
  if (!job.psi && !job.Tm) return;
  const Shape s = job.face >= 0 ? face_shape(g, job.face) : cell_shape(g);
  const long N = s.size();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  int i, j, k;
  unflatten(s, q, i, j, k);
  T X[3] = {0, 0, 0};
  node_pos<T, D>(job.face, i, j, k, dx, X);
#pragma unroll
  for (int a = 0; a < D; ++a) {
    if (job.psi) job.psi[a * N + q] = X[a];
    if (job.Tm) job.Tm[a * N + q] = (a == job.face) ? (T)1 : (T)0;
  }
}

template <typename T>
__global__ void k_add_fields(long n, const T* f1, const T* f2, T* dest, T m) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    dest[q] = f1[q] + m * f2[q];
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------
static inline long max_face(const fm_grid& g) {
  long m = 0;
  for (int c = 0; c < g.dim; ++c) m = face_shape(g, c).size() > m ? face_shape(g, c).size() : m;
  return m;
}
static inline dim3 grid_for(long n, int ycount, int threads = kThreads) {
  return dim3((unsigned)((n + threads - 1) / threads), (unsigned)ycount, 1);
}

// Block sizes picked by the autotuner (fm_tune_set), per kernel class and grid
// shape; 256 when none was set.  Every kernel here computes each node
// independently, so the block size changes only the speed, never a result.
struct TuneKey {
  int kind, dim, n0, n1, n2;
  bool operator==(const TuneKey& o) const {
    return kind == o.kind && dim == o.dim && n0 == o.n0 && n1 == o.n1 && n2 == o.n2;
  }
};
struct TuneHash {
  size_t operator()(const TuneKey& k) const {
    return ((((size_t)k.kind * 31 + k.dim) * 1000003 + k.n0) * 1000003 + k.n1) * 1000003 + k.n2;
  }
};
static std::mutex g_tune_mu;
static std::unordered_map<TuneKey, int, TuneHash> g_tune;

int tuned_value(int kind, const fm_grid& g, int dflt) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(TuneKey{kind, g.dim, g.n[0], g.n[1], g.n[2]});
  return it == g_tune.end() ? dflt : it->second;
}

static inline int tuned_threads(int kind, const fm_grid& g) { return tuned_value(kind, g, kThreads); }

template <typename T>
static Mac<T> mac(const void* x, const void* y, const void* z) {
  Mac<T> m;
  m.c[0] = (const T*)x; m.c[1] = (const T*)y; m.c[2] = (const T*)z;
  return m;
}
template <typename T>
static MacW<T> macw(void* x, void* y, void* z) {
  MacW<T> m;
  m.c[0] = (T*)x; m.c[1] = (T*)y; m.c[2] = (T*)z;
  return m;
}
static inline bool mac_ok(const fm_grid& g, const void* x, const void* y, const void* z) {
  return x && y && (g.dim == 2 || z);
}

#define FM_DISPATCH_D(g, ...)                 \
  do {                                        \
    if ((g).dim == 3) { constexpr int D = 3; __VA_ARGS__; } \
    else { constexpr int D = 2; __VA_ARGS__; } \
  } while (0)

template <typename T>
static int advect_u_grid_t(const fm_grid& g, int rk, double dx, double dt, Mac<T> u0, Mac<T> u1, MacW<T> u2,
                           Mac<T> u1b, MacW<T> u2b, cudaStream_t st) {
  const int th = tuned_threads(FM_TUNE_ADVECT_U, g);
  dim3 grid = grid_for(max_face(g), g.dim, th);
  FM_DISPATCH_D(g, if (rk == 2) k_advect_u_grid<T, D, 2><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, u0, u1, u2, u1b,
                                                                               u2b);
                else k_advect_u_grid<T, D, 4><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, u0, u1, u2, u1b, u2b));
  return check_launch();
}

template <typename T>
static int advect_scalar_grid_t(const fm_grid& g, int rk, double dx, double dt, Mac<T> u0, const T* s1, T* s2,
                                const T* s1b, T* s2b, cudaStream_t st) {
  const int th = tuned_threads(FM_TUNE_ADVECT_SCALAR, g);
  dim3 grid = grid_for(cell_shape(g).size(), 1, th);
  FM_DISPATCH_D(g, if (rk == 2) k_advect_scalar_grid<T, D, 2><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, u0, s1, s2,
                                                                                   s1b, s2b);
                else k_advect_scalar_grid<T, D, 4><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, u0, s1, s2, s1b, s2b));
  return check_launch();
}

template <typename T>
static int march_t(const fm_grid& g, int rk, double dx, double dt, const MarchJobs<T>& jobs, int njobs, Mac<T> u,
                   cudaStream_t st) {
  if (njobs == 0) return FM_OK;
  long n = cell_shape(g).size();
  for (int i = 0; i < njobs; ++i) {
    long m = jobs.j[i].face >= 0 ? face_shape(g, jobs.j[i].face).size() : cell_shape(g).size();
    n = m > n ? m : n;
  }
  const int th = tuned_threads(FM_TUNE_MARCH, g);
  dim3 grid = grid_for(n, njobs, th);
  FM_DISPATCH_D(g, if (rk == 2) k_march<T, D, 2><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, jobs, u);
                else k_march<T, D, 4><<<grid, th, 0, st>>>(g, (T)dx, (T)dt, jobs, u));
  return check_launch();
}

template <typename T>
static int accumulate_t(const fm_grid& g, double dx, double dt, int ab3, int ind, Mac<T> f, MacW<T> in, Mac<T> F,
                        Mac<T> ph, MacW<T> hp, MacW<T> hpp, Mac<T> f2, double dt2, cudaStream_t s) {
  const int th = tuned_threads(FM_TUNE_ACCUMULATE, g);
  dim3 grid = grid_for(max_face(g), g.dim, th);
  const bool two = f2.c[0] != nullptr;
#define FM_ACC(AB, TW) \
  k_accumulate<T, D, AB, TW><<<grid, th, 0, s>>>(g, (T)dx, (T)dt, ind, f, in, F, ph, hp, hpp, f2, (T)dt2)
  FM_DISPATCH_D(g, if (ab3) { if (two) FM_ACC(true, true); else FM_ACC(true, false); }
                   else { if (two) FM_ACC(false, true); else FM_ACC(false, false); });
#undef FM_ACC
  return check_launch();
}

}  // namespace fm

using namespace fm;

#define FM_STREAM(s) ((cudaStream_t)(s))

extern "C" {

int fm_advect_u_grid(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x, const void* u0y,
                     const void* u0z, const void* u1x, const void* u1y, const void* u1z, void* u2x, void* u2y,
                     void* u2z, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_ok(*g, u0x, u0y, u0z) || !mac_ok(*g, u1x, u1y, u1z) || !mac_ok(*g, u2x, u2y, u2z))
    return FM_ERR_ARG;
  if (dtype == FM_F32)
    return advect_u_grid_t<float>(*g, rk, dx, dt, mac<float>(u0x, u0y, u0z), mac<float>(u1x, u1y, u1z),
                                  macw<float>(u2x, u2y, u2z), mac<float>(nullptr, nullptr, nullptr),
                                  macw<float>(nullptr, nullptr, nullptr), FM_STREAM(stream));
  return advect_u_grid_t<double>(*g, rk, dx, dt, mac<double>(u0x, u0y, u0z), mac<double>(u1x, u1y, u1z),
                                 macw<double>(u2x, u2y, u2z), mac<double>(nullptr, nullptr, nullptr),
                                 macw<double>(nullptr, nullptr, nullptr), FM_STREAM(stream));
}

int fm_advect_u_grid_pair(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x,
                          const void* u0y, const void* u0z, const void* u1x, const void* u1y, const void* u1z,
                          void* u2x, void* u2y, void* u2z, const void* v1x, const void* v1y, const void* v1z,
                          void* v2x, void* v2y, void* v2z, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_ok(*g, u0x, u0y, u0z) || !mac_ok(*g, u1x, u1y, u1z) ||
      !mac_ok(*g, u2x, u2y, u2z) || !mac_ok(*g, v1x, v1y, v1z) || !mac_ok(*g, v2x, v2y, v2z))
    return FM_ERR_ARG;
  if (dtype == FM_F32)
    return advect_u_grid_t<float>(*g, rk, dx, dt, mac<float>(u0x, u0y, u0z), mac<float>(u1x, u1y, u1z),
                                  macw<float>(u2x, u2y, u2z), mac<float>(v1x, v1y, v1z),
                                  macw<float>(v2x, v2y, v2z), FM_STREAM(stream));
  return advect_u_grid_t<double>(*g, rk, dx, dt, mac<double>(u0x, u0y, u0z), mac<double>(u1x, u1y, u1z),
                                 macw<double>(u2x, u2y, u2z), mac<double>(v1x, v1y, v1z),
                                 macw<double>(v2x, v2y, v2z), FM_STREAM(stream));
}

int fm_advect_scalar_grid(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x,
                          const void* u0y, const void* u0z, const void* s1, void* s2, void* stream) {
  return fm_advect_scalar_grid_pair(g, dtype, rk, dx, dt, u0x, u0y, u0z, s1, s2, nullptr, nullptr, stream);
}

int fm_advect_scalar_grid_pair(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x,
                               const void* u0y, const void* u0z, const void* s1, void* s2, const void* t1, void* t2,
                               void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_ok(*g, u0x, u0y, u0z) || !s1 || !s2 || (!t1 != !t2)) return FM_ERR_ARG;
  if (dtype == FM_F32)
    return advect_scalar_grid_t<float>(*g, rk, dx, dt, mac<float>(u0x, u0y, u0z), (const float*)s1, (float*)s2,
                                       (const float*)t1, (float*)t2, FM_STREAM(stream));
  return advect_scalar_grid_t<double>(*g, rk, dx, dt, mac<double>(u0x, u0y, u0z), (const double*)s1, (double*)s2,
                                      (const double*)t1, (double*)t2, FM_STREAM(stream));
}

int fm_rk_grid(const fm_grid* g, int dtype, int rk, double dx, double dt, int face, void* psi, void* T,
               const void* ux, const void* uy, const void* uz, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !psi || face < -1 || face >= g->dim || (face == -1 && T) || !mac_ok(*g, ux, uy, uz))
    return FM_ERR_ARG;
  if (dtype == FM_F32) {
    MarchJobs<float> jobs{};
    jobs.j[0] = MarchJob<float>{(float*)psi, (float*)T, face};
    return march_t<float>(*g, rk, dx, dt, jobs, 1, mac<float>(ux, uy, uz), FM_STREAM(stream));
  }
  MarchJobs<double> jobs{};
  jobs.j[0] = MarchJob<double>{(double*)psi, (double*)T, face};
  return march_t<double>(*g, rk, dx, dt, jobs, 1, mac<double>(ux, uy, uz), FM_STREAM(stream));
}

int fm_march_map(const fm_grid* g, int dtype, int rk, double dx, double dt, void* psi_c, void* psi_x, void* T_x,
                 void* psi_y, void* T_y, void* psi_z, void* T_z, const void* ux, const void* uy, const void* uz,
                 void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_ok(*g, ux, uy, uz)) return FM_ERR_ARG;
  void* ps[3] = {psi_x, psi_y, psi_z};
  void* ts[3] = {T_x, T_y, T_z};
  for (int c = 0; c < g->dim; ++c)
    if (!ps[c] || !ts[c]) return FM_ERR_ARG;
  if (dtype == FM_F32) {
    MarchJobs<float> jobs{};
    int n = 0;
    for (int c = 0; c < g->dim; ++c) jobs.j[n++] = MarchJob<float>{(float*)ps[c], (float*)ts[c], c};
    if (psi_c) jobs.j[n++] = MarchJob<float>{(float*)psi_c, nullptr, -1};
    return march_t<float>(*g, rk, dx, dt, jobs, n, mac<float>(ux, uy, uz), FM_STREAM(stream));
  }
  MarchJobs<double> jobs{};
  int n = 0;
  for (int c = 0; c < g->dim; ++c) jobs.j[n++] = MarchJob<double>{(double*)ps[c], (double*)ts[c], c};
  if (psi_c) jobs.j[n++] = MarchJob<double>{(double*)psi_c, nullptr, -1};
  return march_t<double>(*g, rk, dx, dt, jobs, n, mac<double>(ux, uy, uz), FM_STREAM(stream));
}

int fm_pullback_u(const fm_grid* g, int dtype, double dx, const void* u0x, const void* u0y, const void* u0z,
                  void* outx, void* outy, void* outz, const void* Tx, const void* Ty, const void* Tz,
                  const void* psix, const void* psiy, const void* psiz, double alpha, double beta,
                  const void* basex, const void* basey, const void* basez, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!mac_ok(*g, u0x, u0y, u0z) || !mac_ok(*g, outx, outy, outz) || !mac_ok(*g, Tx, Ty, Tz) ||
      !mac_ok(*g, psix, psiy, psiz) || (beta != 0.0 && !mac_ok(*g, basex, basey, basez)))
    return FM_ERR_ARG;
  const int th = tuned_threads(FM_TUNE_PULLBACK_U, *g);
  dim3 grid = grid_for(max_face(*g), g->dim, th);
  cudaStream_t s = FM_STREAM(stream);
  if (dtype == FM_F32) {
    FM_DISPATCH_D(*g, k_pullback_u<float, D><<<grid, th, 0, s>>>(
                          *g, (float)dx, mac<float>(u0x, u0y, u0z), macw<float>(outx, outy, outz),
                          mac<float>(Tx, Ty, Tz), mac<float>(psix, psiy, psiz), (float)alpha, (float)beta,
                          mac<float>(basex, basey, basez)));
  } else {
    FM_DISPATCH_D(*g, k_pullback_u<double, D><<<grid, th, 0, s>>>(
                          *g, dx, mac<double>(u0x, u0y, u0z), macw<double>(outx, outy, outz),
                          mac<double>(Tx, Ty, Tz), mac<double>(psix, psiy, psiz), alpha, beta,
                          mac<double>(basex, basey, basez)));
  }
  return check_launch();
}

int fm_pullback_scalar(const fm_grid* g, int dtype, double dx, const void* s0, void* out, const void* psi,
                       double alpha, double beta, const void* base, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!s0 || !out || !psi || (beta != 0.0 && !base)) return FM_ERR_ARG;
  const int th = tuned_threads(FM_TUNE_PULLBACK_SCALAR, *g);
  dim3 grid = grid_for(cell_shape(*g).size(), 1, th);
  cudaStream_t s = FM_STREAM(stream);
  if (dtype == FM_F32) {
    FM_DISPATCH_D(*g, k_pullback_scalar<float, D><<<grid, th, 0, s>>>(
                          *g, (float)dx, (const float*)s0, (float*)out, (const float*)psi, (float)alpha,
                          (float)beta, (const float*)base));
  } else {
    FM_DISPATCH_D(*g, k_pullback_scalar<double, D><<<grid, th, 0, s>>>(
                          *g, dx, (const double*)s0, (double*)out, (const double*)psi, alpha, beta,
                          (const double*)base));
  }
  return check_launch();
}

static int accumulate_entry(const fm_grid* g, int dtype, double dx, double dt, int ab3, int ind, const void* fx,
                            const void* fy, const void* fz, void* initx, void* inity, void* initz, const void* Fx,
                            const void* Fy, const void* Fz, const void* phix, const void* phiy, const void* phiz,
                            void* Hpx, void* Hppx, void* Hpy, void* Hppy, void* Hpz, void* Hppz, const void* f2x,
                            const void* f2y, const void* f2z, double dt2, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!mac_ok(*g, fx, fy, fz) || !mac_ok(*g, initx, inity, initz) || !mac_ok(*g, Fx, Fy, Fz) ||
      !mac_ok(*g, phix, phiy, phiz) || ind < 0)
    return FM_ERR_ARG;
  if (ab3 && (!mac_ok(*g, Hpx, Hpy, Hpz) || !mac_ok(*g, Hppx, Hppy, Hppz))) return FM_ERR_ARG;
  if ((f2x || f2y || f2z) && !mac_ok(*g, f2x, f2y, f2z)) return FM_ERR_ARG;
  cudaStream_t s = FM_STREAM(stream);
  if (dtype == FM_F32)
    return accumulate_t<float>(*g, dx, dt, ab3, ind, mac<float>(fx, fy, fz), macw<float>(initx, inity, initz),
                               mac<float>(Fx, Fy, Fz), mac<float>(phix, phiy, phiz), macw<float>(Hpx, Hpy, Hpz),
                               macw<float>(Hppx, Hppy, Hppz), mac<float>(f2x, f2y, f2z), dt2, s);
  return accumulate_t<double>(*g, dx, dt, ab3, ind, mac<double>(fx, fy, fz), macw<double>(initx, inity, initz),
                              mac<double>(Fx, Fy, Fz), mac<double>(phix, phiy, phiz), macw<double>(Hpx, Hpy, Hpz),
                              macw<double>(Hppx, Hppy, Hppz), mac<double>(f2x, f2y, f2z), dt2, s);
}

int fm_accumulate_init(const fm_grid* g, int dtype, double dx, double dt, int ab3, int ind, const void* fx,
                       const void* fy, const void* fz, void* initx, void* inity, void* initz, const void* Fx,
                       const void* Fy, const void* Fz, const void* phix, const void* phiy, const void* phiz,
                       void* Hpx, void* Hppx, void* Hpy, void* Hppy, void* Hpz, void* Hppz, void* stream) {
  return accumulate_entry(g, dtype, dx, dt, ab3, ind, fx, fy, fz, initx, inity, initz, Fx, Fy, Fz, phix, phiy, phiz,
                          Hpx, Hppx, Hpy, Hppy, Hpz, Hppz, nullptr, nullptr, nullptr, 0.0, stream);
}

int fm_accumulate_init_pair(const fm_grid* g, int dtype, double dx, double dt, int ab3, int ind, const void* fx,
                            const void* fy, const void* fz, void* initx, void* inity, void* initz, const void* Fx,
                            const void* Fy, const void* Fz, const void* phix, const void* phiy, const void* phiz,
                            void* Hpx, void* Hppx, void* Hpy, void* Hppy, void* Hpz, void* Hppz, const void* f2x,
                            const void* f2y, const void* f2z, double dt2, void* stream) {
  if (!f2x) return FM_ERR_ARG;
  return accumulate_entry(g, dtype, dx, dt, ab3, ind, fx, fy, fz, initx, inity, initz, Fx, Fy, Fz, phix, phiy, phiz,
                          Hpx, Hppx, Hpy, Hppy, Hpz, Hppz, f2x, f2y, f2z, dt2, stream);
}

int fm_reset_to_identity(const fm_grid* g, int dtype, double dx, void* psi_c, void* psi_x, void* psi_y, void* psi_z,
                         void* T_x, void* T_y, void* T_z, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  void* ps[3] = {psi_x, psi_y, psi_z};
  void* ts[3] = {T_x, T_y, T_z};
  long n = cell_shape(*g).size();
  for (int c = 0; c < g->dim; ++c) n = face_shape(*g, c).size() > n ? face_shape(*g, c).size() : n;
  dim3 grid = grid_for(n, g->dim + 1);
  cudaStream_t s = FM_STREAM(stream);
  if (dtype == FM_F32) {
    MarchJobs<float> jobs{};
    for (int c = 0; c < g->dim; ++c) jobs.j[c] = MarchJob<float>{(float*)ps[c], (float*)ts[c], c};
    jobs.j[g->dim] = MarchJob<float>{(float*)psi_c, nullptr, -1};
    FM_DISPATCH_D(*g, k_reset_identity<float, D><<<grid, kThreads, 0, s>>>(*g, (float)dx, jobs));
  } else {
    MarchJobs<double> jobs{};
    for (int c = 0; c < g->dim; ++c) jobs.j[c] = MarchJob<double>{(double*)ps[c], (double*)ts[c], c};
    jobs.j[g->dim] = MarchJob<double>{(double*)psi_c, nullptr, -1};
    FM_DISPATCH_D(*g, k_reset_identity<double, D><<<grid, kThreads, 0, s>>>(*g, dx, jobs));
  }
  return check_launch();
}

int fm_add_fields(int dtype, long n, const void* f1, const void* f2, void* dest, double m, void* stream) {
  if (dtype != FM_F32 && dtype != FM_F64) return FM_ERR_DTYPE;
  if (n < 0 || (n > 0 && (!f1 || !f2 || !dest))) return FM_ERR_ARG;
  if (n == 0) return FM_OK;
  long blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t s = FM_STREAM(stream);
  if (dtype == FM_F32)
    k_add_fields<float><<<(unsigned)blocks, kThreads, 0, s>>>(n, (const float*)f1, (const float*)f2, (float*)dest,
                                                              (float)m);
  else
    k_add_fields<double><<<(unsigned)blocks, kThreads, 0, s>>>(n, (const double*)f1, (const double*)f2,
                                                               (double*)dest, m);
  return check_launch();
}

}  // extern "C"

// Autotuner table (see tuned_value): per kernel class and grid shape, the threads
// per block of the gather kernels (32..256 in multiples of 32) or the adjoint-
// source stencil's tile height (4 or 8 in 3D, 8 or 16 in 2D); 0 restores the default.
int fm_tune_set(int kind, const fm_grid* g, int threads) {
  using namespace fm;
  if (!g || kind < 0 || kind >= FM_TUNE_KINDS) return FM_ERR_ARG;
  if (kind == FM_TUNE_ADJ_SOURCE_TILE) {
    const bool ok = threads == 0 || (g->dim == 3 ? (threads == 4 || threads == 8) : (threads == 8 || threads == 16));
    if (!ok) return FM_ERR_ARG;
  } else if (threads != 0 && (threads < 32 || threads > kThreads || threads % 32 != 0)) {
    return FM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const TuneKey k{kind, g->dim, g->n[0], g->n[1], g->n[2]};
  if (threads == 0) g_tune.erase(k);
  else g_tune[k] = threads;
  return FM_OK;
}

int fm_tune_get(int kind, const fm_grid* g) {
  using namespace fm;
  if (!g || kind < 0 || kind >= FM_TUNE_KINDS) return -FM_ERR_ARG;
  if (kind == FM_TUNE_ADJ_SOURCE_TILE) return tuned_value(kind, *g, g->dim == 3 ? 8 : 16);
  return tuned_threads(kind, *g);
}
