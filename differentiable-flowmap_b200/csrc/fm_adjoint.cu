// fm_adjoint.cu -- discrete adjoints of the gather kernels (sm_100a): the
// backward passes of the per-kernel torch.autograd Functions for
//   advect_scalar_grid / advect_u_grid   (3D/flowmap.py:202-320)
//   advect_scalar / advect_u pullbacks   (3D/flowmap.py:51-79, the alpha/beta
//                                         form of the BFECC epilogues)
//
// Each kernel is the exact transpose of its forward kernel's linearisation.
// A quadratic B-spline sample f(p) = sum_taps w_tap(p) f[tap] is linear in f:
// its transpose scatters lambda * w_tap into the gradient of f.  In p it is
// piecewise smooth: d f / d p_a = inv_dx * sum_taps dw_tap/ds_a f[tap], and
// zero on an axis where the reference's clamp of s = p/dx - BL to
// [1, len-2-1e-6] is active (the weights are then constant in p).  The RK
// backtraces of the grid advections are differentiated stage by stage in
// reverse from recomputed stage positions.
//
// The field gradients are accumulated with atomic adds into caller-zeroed
// buffers (several nodes sample overlapping taps), so their last bits depend
// on the order in which the adds land; the per-node gradients (T, psi, base)
// are plain read-modify-writes of the node's own entries.
#include "fm_common.cuh"
#include "fm_internal.h"
#include "fm_q2.cuh"

namespace fm {
namespace {

constexpr int kAdjThreads = 128;

// One axis of a sample's stencil and whether the position clamp is inactive
// there (live = 1: s follows p; live = 0: s is pinned to a clamp bound).
template <typename T>
struct AxisAdj {
  Q2<T, true> q;
  T live;
  __device__ __forceinline__ void setup(T ps, T bl, T hi) {
    q.setup(ps, bl, hi);
    const T u = ps - bl;
    live = (u > (T)1 && u < hi) ? (T)1 : (T)0;
  }
};

// The stencil of one staggered field at p: `own` is the axis the field is
// staggered on (BL = 0, extent n+1), -1 for the cell grid (BL = 0.5 everywhere).
template <typename T, int D>
struct PointAdj {
  AxisAdj<T> ax[3];
  __device__ __forceinline__ void setup(const Q2Lim<T>& lim, int own, const T* p, T inv_dx) {
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const bool st = a == own;
      ax[a].setup(p[a] * inv_dx, st ? (T)0 : (T)0.5, st ? lim.h0[a] : lim.h5[a]);
    }
  }
};

// f[taps] += val * w(p)
template <typename T, int D>
__device__ __forceinline__ void scatter(T* f, const Shape& s, const PointAdj<T, D>& P, T val) {
  const Q2<T, true>& x = P.ax[0].q;
  const Q2<T, true>& y = P.ax[1].q;
  const T wx[3] = {x.w0, x.w1, x.w2}, wy[3] = {y.w0, y.w1, y.w2};
  if constexpr (D == 3) {
    const Q2<T, true>& z = P.ax[2].q;
    const T wz[3] = {z.w0, z.w1, z.w2};
    const unsigned sj = s.s2, si = (unsigned)s.s1 * s.s2;
    const unsigned b = ((unsigned)x.i0 * s.s1 + y.i0) * s.s2 + z.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T vi = val * wx[i];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T vij = vi * wy[j];
        T* row = f + b + i * si + j * sj;
#pragma unroll
        for (int k = 0; k < 3; ++k) atomicAdd(row + k, vij * wz[k]);
      }
    }
  } else {
    const unsigned si = s.s1;
    const unsigned b = (unsigned)x.i0 * s.s1 + y.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T vi = val * wx[i];
#pragma unroll
      for (int j = 0; j < 3; ++j) atomicAdd(f + b + i * si + j, vi * wy[j]);
    }
  }
}

// v = f(p) and gp = d f(p) / d p (the clamp-aware position gradient)
template <typename T, int D>
__device__ __forceinline__ void val_grad(const T* __restrict__ f, const Shape& s, const PointAdj<T, D>& P, T inv_dx,
                                         T& v, T* gp) {
  T gr[3] = {0, 0, 0};
  q2_grad<T, D>(f, s, P.ax[0].q, P.ax[1].q, P.ax[D == 3 ? 2 : 0].q, v, gr);
#pragma unroll
  for (int a = 0; a < D; ++a) gp[a] = gr[a] * inv_dx * P.ax[a].live;
}

// One RK stage of a backtrace in reverse: the stage sampled u0 at q, its
// adjoint vbar scatters into gu0 (when wanted) and qbar = (d u0(q) / d q)^T vbar.
template <typename T, int D>
__device__ __forceinline__ void stage_adj(const Mac<T>& u0, const MacW<T>& gu0, const fm_grid& g,
                                          const Q2Lim<T>& lim, const T* q, T inv_dx, const T* vbar, bool want_q,
                                          T* qbar) {
#pragma unroll
  for (int b = 0; b < D; ++b) qbar[b] = 0;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    PointAdj<T, D> P;
    P.setup(lim, c, q, inv_dx);
    const Shape s = face_shape(g, c);
    scatter<T, D>(gu0.c[c], s, P, vbar[c]);
    if (want_q) {
      T v, gp[3];
      val_grad<T, D>(u0.c[c], s, P, inv_dx, v, gp);
#pragma unroll
      for (int b = 0; b < D; ++b) qbar[b] += vbar[c] * gp[b];
    }
  }
}

// Forward backtrace with its stage positions kept (the same operations as the
// forward kernels' backtrace, so the recomputed foot equals theirs):
// RK2 stages at q[0] = X, q[1]; RK4 at q[0] = X, q[1], q[2], q[3].
template <typename T, int D, int RK>
__device__ __forceinline__ void backtrace_stages(const Mac<T>& u0, const fm_grid& g, const Q2Lim<T>& lim,
                                                 const T* X, T inv_dx, T dt, T q[4][3], T* p) {
  T v[3], vs[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) q[0][a] = X[a], q[1][a] = 0, q[2][a] = 0, q[3][a] = 0;
  q2_mac_val<T, D>(u0, g, lim, X, inv_dx, v);
#pragma unroll
  for (int a = 0; a < D; ++a) q[1][a] = X[a] - v[a] * dt * (T)0.5;
  if constexpr (RK == 2) {
    q2_mac_val<T, D>(u0, g, lim, q[1], inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = X[a] - v[a] * dt;
  } else {
#pragma unroll
    for (int a = 0; a < D; ++a) vs[a] = v[a];
    q2_mac_val<T, D>(u0, g, lim, q[1], inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) { vs[a] = vs[a] + (T)2 * v[a]; q[2][a] = X[a] - v[a] * dt * (T)0.5; }
    q2_mac_val<T, D>(u0, g, lim, q[2], inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) { vs[a] = vs[a] + (T)2 * v[a]; q[3][a] = X[a] - v[a] * dt; }
    q2_mac_val<T, D>(u0, g, lim, q[3], inv_dx, v);
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = X[a] - (vs[a] + v[a]) / (T)6.0 * dt;
  }
}

// Reverse of the backtrace given pbar = dL/dp at the foot: scatters every
// stage's velocity adjoint into gu0.
//   RK2: p = X - dt v2, q1 = X - dt/2 v1
//   RK4: p = X - dt/6 (v1 + 2 v2 + 2 v3 + v4), q1 = X - dt/2 v1, q2 = X - dt/2 v2,
//        q3 = X - dt v3
template <typename T, int D, int RK>
__device__ __forceinline__ void backtrace_adj(const Mac<T>& u0, const MacW<T>& gu0, const fm_grid& g,
                                              const Q2Lim<T>& lim, T q[4][3], T inv_dx, T dt, const T* pbar) {
  T vbar[3] = {0, 0, 0}, qbar[3] = {0, 0, 0};
  if constexpr (RK == 2) {
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = -dt * pbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[1], inv_dx, vbar, true, qbar);
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = (T)-0.5 * dt * qbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[0], inv_dx, vbar, false, qbar);
  } else {
    const T w16 = -dt / (T)6, w13 = -dt / (T)3;
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = w16 * pbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[3], inv_dx, vbar, true, qbar);  // v4 at q3
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = w13 * pbar[a] - dt * qbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[2], inv_dx, vbar, true, qbar);  // v3 at q2
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = w13 * pbar[a] + (T)-0.5 * dt * qbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[1], inv_dx, vbar, true, qbar);  // v2 at q1
#pragma unroll
    for (int a = 0; a < D; ++a) vbar[a] = w16 * pbar[a] + (T)-0.5 * dt * qbar[a];
    stage_adj<T, D>(u0, gu0, g, lim, q[0], inv_dx, vbar, false, qbar);  // v1 at X
  }
}

// Adjoint of advect_scalar_grid (field < 0: s1 on the cell grid) and of
// advect_u_grid (blockIdx.y = face component c: u2_c = u1_c(foot)).
// f1 / gout / gf1 hold the sampled field, dL/d(output) and dL/d(f1) (component
// c in slot c; the scalar in slot 0).
template <typename T, int D, int RK>
__global__ void __launch_bounds__(kAdjThreads) k_advect_grid_adj(fm_grid g, T dx, T dt, int scalar, Mac<T> u0,
                                                                 Mac<T> f1, Mac<T> gout, MacW<T> gu0,
                                                                 MacW<T> gf1) {
  const int c = scalar ? -1 : (int)blockIdx.y;
  const Shape s = c < 0 ? cell_shape(g) : face_shape(g, c);
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= s.size()) return;
  const int slot = c < 0 ? 0 : c;
  const T lam = pick(gout, slot)[n];
  if (lam == (T)0) return;  // a zero adjoint contributes nothing to either gradient
  int i, j, k;
  unflatten(s, n, i, j, k);
  T X[3] = {0, 0, 0}, p[3] = {0, 0, 0}, q[4][3];
  node_pos<T, D>(c, i, j, k, dx, X);
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  backtrace_stages<T, D, RK>(u0, g, lim, X, inv_dx, dt, q, p);
  PointAdj<T, D> P;
  P.setup(lim, c, p, inv_dx);
  T* gf = pick(gf1, slot);
  if (gf != nullptr) scatter<T, D>(gf, s, P, lam);
  if (gu0.c[0] == nullptr) return;
  T v, gp[3] = {0, 0, 0}, pbar[3] = {0, 0, 0};
  val_grad<T, D>(pick(f1, slot), s, P, inv_dx, v, gp);
#pragma unroll
  for (int a = 0; a < D; ++a) pbar[a] = lam * gp[a];
  backtrace_adj<T, D, RK>(u0, gu0, g, lim, q, inv_dx, dt, pbar);
}

// Adjoint of out_c = alpha (T_c . u0(psi_c) + beta base_c) on face grid
// c = blockIdx.y.  Any of gu0 / gT / gpsi / gbase may be absent (c[0] NULL).
template <typename T, int D>
__global__ void __launch_bounds__(kAdjThreads) k_pullback_u_adj(fm_grid g, T dx, Mac<T> u0, Mac<T> Tm, Mac<T> psi,
                                                                T alpha, T beta, Mac<T> gout, MacW<T> gu0,
                                                                MacW<T> gT, MacW<T> gpsi, MacW<T> gbase) {
  const int c = blockIdx.y;
  const Shape s = face_shape(g, c);
  const long N = s.size();
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const T al = alpha * pick(gout, c)[n];
  if (gbase.c[0] != nullptr) pick(gbase, c)[n] += al * beta;
  if (al == (T)0) return;
  const T* psi_c = pick(psi, c);
  const T* T_c = pick(Tm, c);
  T p[3] = {0, 0, 0}, t[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = psi_c[a * N + n], t[a] = T_c[a * N + n];
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  T pbar[3] = {0, 0, 0};
  const bool want_v = gT.c[0] != nullptr || gpsi.c[0] != nullptr;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    PointAdj<T, D> P;
    P.setup(lim, a, p, inv_dx);
    const Shape sa = face_shape(g, a);
    if (gu0.c[0] != nullptr) scatter<T, D>(gu0.c[a], sa, P, al * t[a]);
    if (want_v) {
      T v, gp[3] = {0, 0, 0};
      val_grad<T, D>(u0.c[a], sa, P, inv_dx, v, gp);
      if (gT.c[0] != nullptr) pick(gT, c)[a * N + n] += al * v;
#pragma unroll
      for (int b = 0; b < D; ++b) pbar[b] += al * t[a] * gp[b];
    }
  }
  if (gpsi.c[0] != nullptr) {
    T* gp_c = pick(gpsi, c);
#pragma unroll
    for (int b = 0; b < D; ++b) gp_c[b * N + n] += pbar[b];
  }
}

// Adjoint of out = alpha (s0(psi) + beta base) on the cell grid.
template <typename T, int D>
__global__ void __launch_bounds__(kAdjThreads) k_pullback_scalar_adj(fm_grid g, T dx, const T* __restrict__ s0,
                                                                     const T* __restrict__ psi, T alpha, T beta,
                                                                     const T* __restrict__ gout, T* gs0, T* gpsi,
                                                                     T* gbase) {
  const Shape s = cell_shape(g);
  const long N = s.size();
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const T al = alpha * gout[n];
  if (gbase != nullptr) gbase[n] += al * beta;
  if (al == (T)0) return;
  T p[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = psi[a * N + n];
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  PointAdj<T, D> P;
  P.setup(lim, -1, p, inv_dx);
  if (gs0 != nullptr) scatter<T, D>(gs0, s, P, al);
  if (gpsi != nullptr) {
    T v, gp[3] = {0, 0, 0};
    val_grad<T, D>(s0, s, P, inv_dx, v, gp);
#pragma unroll
    for (int b = 0; b < D; ++b) gpsi[b * N + n] += al * gp[b];
  }
}

// ---------------------------------------------------------------------------
// RK_grid (flow map psi and Jacobian row T marched through u): the stage
// k = u(pos), d = (grad u)(pos) t in reverse.  Besides the first derivatives
// this needs the Hessian of the sample: the quadratic B-spline's second
// derivative is 1, -2, 1 on the three taps of an axis (0 where the clamp is
// active).
// ---------------------------------------------------------------------------

// At the stencil P: v = f, g = d f / d p (clamp-aware), graw = the gradient
// the forward march uses in d = graw . t (the B-spline derivative at the
// clamped position, scaled by 1/dx, not masked), Ht = d (graw . t) / d p.
template <typename T, int D>
__device__ __forceinline__ void val_grad_hess(const T* __restrict__ f, const Shape& s, const PointAdj<T, D>& P,
                                              T inv_dx, const T* t, T& v, T* g, T* graw, T* Ht) {
  T w[3][3], d[3][3], dd[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const Q2<T, true>& q = P.ax[a < D ? a : 0].q;
    w[a][0] = q.w0, w[a][1] = q.w1, w[a][2] = q.w2;
    d[a][0] = q.d0, d[a][1] = q.d1, d[a][2] = q.d2;
    dd[a][0] = (T)1, dd[a][1] = (T)-2, dd[a][2] = (T)1;
  }
  T acc_v = 0, G[3] = {0, 0, 0}, H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if constexpr (D == 3) {
    const unsigned sj = s.s2, si = (unsigned)s.s1 * s.s2;
    const unsigned b = ((unsigned)P.ax[0].q.i0 * s.s1 + P.ax[1].q.i0) * s.s2 + P.ax[2].q.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const T x = ldg(f + b + i * si + j * sj + k);
          acc_v += x * w[0][i] * w[1][j] * w[2][k];
          G[0] += x * d[0][i] * w[1][j] * w[2][k];
          G[1] += x * w[0][i] * d[1][j] * w[2][k];
          G[2] += x * w[0][i] * w[1][j] * d[2][k];
          H[0][0] += x * dd[0][i] * w[1][j] * w[2][k];
          H[1][1] += x * w[0][i] * dd[1][j] * w[2][k];
          H[2][2] += x * w[0][i] * w[1][j] * dd[2][k];
          H[0][1] += x * d[0][i] * d[1][j] * w[2][k];
          H[0][2] += x * d[0][i] * w[1][j] * d[2][k];
          H[1][2] += x * w[0][i] * d[1][j] * d[2][k];
        }
  } else {
    const unsigned si = s.s1;
    const unsigned b = (unsigned)P.ax[0].q.i0 * s.s1 + P.ax[1].q.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T x = ldg(f + b + i * si + j);
        acc_v += x * w[0][i] * w[1][j];
        G[0] += x * d[0][i] * w[1][j];
        G[1] += x * w[0][i] * d[1][j];
        H[0][0] += x * dd[0][i] * w[1][j];
        H[1][1] += x * w[0][i] * dd[1][j];
        H[0][1] += x * d[0][i] * d[1][j];
      }
  }
  H[1][0] = H[0][1], H[2][0] = H[0][2], H[2][1] = H[1][2];
  v = acc_v;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    graw[a] = G[a] * inv_dx;
    g[a] = graw[a] * P.ax[a].live;
    T h = 0;
#pragma unroll
    for (int b2 = 0; b2 < D; ++b2) h += H[a][b2] * inv_dx * t[b2];
    Ht[a] = h * inv_dx * P.ax[a].live;
  }
}

// f[taps] += kv * w + kd * (grad w . t)   (value and directional-derivative
// adjoints; the derivative weights unmasked, as the forward's d uses them)
template <typename T, int D>
__device__ __forceinline__ void scatter_vd(T* f, const Shape& s, const PointAdj<T, D>& P, T inv_dx, T kv, T kd,
                                           const T* t) {
  T w[3][3], e[3][3];  // e = derivative weight * t_a / dx
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const Q2<T, true>& q = P.ax[a < D ? a : 0].q;
    const T sa = a < D ? inv_dx * t[a] : (T)0;
    w[a][0] = q.w0, w[a][1] = q.w1, w[a][2] = q.w2;
    e[a][0] = q.d0 * sa, e[a][1] = q.d1 * sa, e[a][2] = q.d2 * sa;
  }
  if constexpr (D == 3) {
    const unsigned sj = s.s2, si = (unsigned)s.s1 * s.s2;
    const unsigned b = ((unsigned)P.ax[0].q.i0 * s.s1 + P.ax[1].q.i0) * s.s2 + P.ax[2].q.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const T wv = w[0][i] * w[1][j] * w[2][k];
          const T wd = e[0][i] * w[1][j] * w[2][k] + w[0][i] * e[1][j] * w[2][k] + w[0][i] * w[1][j] * e[2][k];
          atomicAdd(f + b + i * si + j * sj + k, kv * wv + kd * wd);
        }
  } else {
    const unsigned si = s.s1;
    const unsigned b = (unsigned)P.ax[0].q.i0 * s.s1 + P.ax[1].q.i0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T wv = w[0][i] * w[1][j];
        const T wd = e[0][i] * w[1][j] + w[0][i] * e[1][j];
        atomicAdd(f + b + i * si + j, kv * wv + kd * wd);
      }
  }
}

// One march stage in reverse: k = u(pos), d = (grad u)(pos) t with adjoints
// kbar, dbar (dbar unused when !WT) -> posbar, tbar; u's gradient scattered.
template <typename T, int D, bool WT>
__device__ __forceinline__ void march_stage_adj(const Mac<T>& u, const MacW<T>& gu, const fm_grid& g,
                                                const Q2Lim<T>& lim, const T* pos, const T* t, T inv_dx,
                                                const T* kbar, const T* dbar, T* posbar, T* tbar) {
#pragma unroll
  for (int a = 0; a < 3; ++a) posbar[a] = 0, tbar[a] = 0;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    PointAdj<T, D> P;
    P.setup(lim, c, pos, inv_dx);
    const Shape s = face_shape(g, c);
    T v, gr[3] = {0, 0, 0}, graw[3] = {0, 0, 0}, Ht[3] = {0, 0, 0};
    if constexpr (WT) {
      val_grad_hess<T, D>(u.c[c], s, P, inv_dx, t, v, gr, graw, Ht);
#pragma unroll
      for (int a = 0; a < D; ++a) {
        posbar[a] += kbar[c] * gr[a] + dbar[c] * Ht[a];
        tbar[a] += dbar[c] * graw[a];
      }
      if (gu.c[0] != nullptr) scatter_vd<T, D>(gu.c[c], s, P, inv_dx, kbar[c], dbar[c], t);
    } else {
      val_grad<T, D>(u.c[c], s, P, inv_dx, v, gr);
#pragma unroll
      for (int a = 0; a < D; ++a) posbar[a] += kbar[c] * gr[a];
      if (gu.c[0] != nullptr) scatter<T, D>(gu.c[c], s, P, kbar[c]);
    }
  }
}

// Adjoint of RK2/RK4_grid (WT) or RK*_grid_only_psi for one node: recomputes
// the stage states (the same operations as the forward march), then
//   RK2: psi' = P + (-dt) k2,  stage 2 at (P + h k1, T + h d1), h = -dt/2
//   RK4: psi' = P + c6 (k1 + 2 k2 + 2 k3 + k4), c6 = -dt/6, stages at
//        (P, T), (P + h k1, T + h d1), (P + h k2, T + h d2), (P - dt k3, T - dt d3)
// and T' likewise with d.  g_psi / g_T receive dL/dpsi, dL/dT of the inputs.
template <typename T, int D, int RK, bool WT>
__global__ void __launch_bounds__(kAdjThreads) k_march_adj(fm_grid g, T dx, T dt, int face, Mac<T> u,
                                                           const T* __restrict__ psi, const T* __restrict__ Tm,
                                                           const T* __restrict__ g_psi_out,
                                                           const T* __restrict__ g_T_out, MacW<T> gu, T* g_psi,
                                                           T* g_T) {
  const Shape s = face >= 0 ? face_shape(g, face) : cell_shape(g);
  const long N = s.size();
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  constexpr int S = RK == 2 ? 2 : 4;
  T P0[3] = {0, 0, 0}, T0[3] = {0, 0, 0}, Pb[3] = {0, 0, 0}, Tb[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    P0[a] = psi[a * N + n];
    Pb[a] = g_psi_out[a * N + n];
    if constexpr (WT) {
      T0[a] = Tm[a * N + n];
      Tb[a] = g_T_out[a * N + n];
    }
  }
  const T neg_dt = -dt;
  const T h = (T)0.5 * neg_dt;
  const T inv_dx = (T)1 / dx;
  const Q2Lim<T> lim(g);
  // forward stage states
  T pos[S][3], tt[S][3], k[3], d[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < 3; ++a) pos[0][a] = P0[a], tt[0][a] = T0[a];
#pragma unroll
  for (int st = 1; st < S; ++st) {
    if constexpr (WT) q2_mac_grad_dot<T, D>(u, g, lim, pos[st - 1], inv_dx, tt[st - 1], k, d);
    else q2_mac_val<T, D>(u, g, lim, pos[st - 1], inv_dx, k);
    const T hs = (RK == 4 && st == 3) ? (T)1.0 * neg_dt : h;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pos[st][a] = a < D ? P0[a] + hs * k[a] : (T)0;
      tt[st][a] = (WT && a < D) ? T0[a] + hs * d[a] : (T)0;
    }
  }
  // reverse sweep
  T kb[3], db[3] = {0, 0, 0}, pb[3], tb[3];
  if constexpr (RK == 2) {
#pragma unroll
    for (int a = 0; a < 3; ++a) kb[a] = neg_dt * Pb[a], db[a] = neg_dt * Tb[a];
    march_stage_adj<T, D, WT>(u, gu, g, lim, pos[1], tt[1], inv_dx, kb, db, pb, tb);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      kb[a] = h * pb[a], db[a] = h * tb[a];
      Pb[a] += pb[a], Tb[a] += tb[a];
    }
    march_stage_adj<T, D, WT>(u, gu, g, lim, pos[0], tt[0], inv_dx, kb, db, pb, tb);
  } else {
    const T c6 = neg_dt * (T)1 / (T)6;
    const T Po[3] = {Pb[0], Pb[1], Pb[2]}, To[3] = {Tb[0], Tb[1], Tb[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) kb[a] = c6 * Po[a], db[a] = c6 * To[a];
#pragma unroll
    for (int st = 3; st >= 1; --st) {
      march_stage_adj<T, D, WT>(u, gu, g, lim, pos[st], tt[st], inv_dx, kb, db, pb, tb);
      const T hs = st == 3 ? neg_dt : h;        // how stage st's state depends on the previous stage's k, d
      const T wprev = st == 1 ? c6 : (T)2 * c6;  // weight of the previous stage's k, d in the update
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Pb[a] += pb[a], Tb[a] += tb[a];
        kb[a] = wprev * Po[a] + hs * pb[a];
        db[a] = wprev * To[a] + hs * tb[a];
      }
    }
    march_stage_adj<T, D, WT>(u, gu, g, lim, pos[0], tt[0], inv_dx, kb, db, pb, tb);
  }
#pragma unroll
  for (int a = 0; a < D; ++a) {
    Pb[a] += pb[a];
    if (g_psi != nullptr) g_psi[a * N + n] += Pb[a];
    if constexpr (WT) {
      Tb[a] += tb[a];
      if (g_T != nullptr) g_T[a * N + n] += Tb[a];
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <typename T>
Mac<T> cmac(const void* x, const void* y, const void* z) {
  Mac<T> m;
  m.c[0] = (const T*)x; m.c[1] = (const T*)y; m.c[2] = (const T*)z;
  return m;
}
template <typename T>
MacW<T> wmac(void* x, void* y, void* z) {
  MacW<T> m;
  m.c[0] = (T*)x; m.c[1] = (T*)y; m.c[2] = (T*)z;
  return m;
}
// all D components present, or (when `optional`) all absent
inline bool mac_args(const fm_grid& g, const void* x, const void* y, const void* z, bool optional) {
  const bool all = x && y && (g.dim == 2 || z);
  const bool none = !x && !y && !z;
  return all || (optional && none);
}
inline long max_face_size(const fm_grid& g) {
  long m = 0;
  for (int c = 0; c < g.dim; ++c) m = face_shape(g, c).size() > m ? face_shape(g, c).size() : m;
  return m;
}
inline dim3 blocks(long n, int y) { return dim3((unsigned)((n + kAdjThreads - 1) / kAdjThreads), (unsigned)y, 1); }

template <typename T>
int advect_grid_adj_t(const fm_grid& g, int rk, double dx, double dt, int scalar, Mac<T> u0, Mac<T> f1,
                      Mac<T> gout, MacW<T> gu0, MacW<T> gf1, cudaStream_t st) {
  const dim3 grid = scalar ? blocks(cell_shape(g).size(), 1) : blocks(max_face_size(g), g.dim);
#define FM_ADJ_LAUNCH(D, RK) \
  k_advect_grid_adj<T, D, RK><<<grid, kAdjThreads, 0, st>>>(g, (T)dx, (T)dt, scalar, u0, f1, gout, gu0, gf1)
  if (g.dim == 3) {
    if (rk == 2) FM_ADJ_LAUNCH(3, 2);
    else FM_ADJ_LAUNCH(3, 4);
  } else {
    if (rk == 2) FM_ADJ_LAUNCH(2, 2);
    else FM_ADJ_LAUNCH(2, 4);
  }
#undef FM_ADJ_LAUNCH
  return check_launch();
}

}  // namespace
}  // namespace fm

using namespace fm;

extern "C" {

int fm_advect_scalar_grid_adj(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x,
                              const void* u0y, const void* u0z, const void* s1, const void* g_s2, void* g_u0x,
                              void* g_u0y, void* g_u0z, void* g_s1, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_args(*g, u0x, u0y, u0z, false) || !s1 || !g_s2 ||
      !mac_args(*g, g_u0x, g_u0y, g_u0z, true))
    return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32)
    return advect_grid_adj_t<float>(*g, rk, dx, dt, 1, cmac<float>(u0x, u0y, u0z), cmac<float>(s1, nullptr, nullptr),
                                    cmac<float>(g_s2, nullptr, nullptr), wmac<float>(g_u0x, g_u0y, g_u0z),
                                    wmac<float>(g_s1, nullptr, nullptr), s);
  return advect_grid_adj_t<double>(*g, rk, dx, dt, 1, cmac<double>(u0x, u0y, u0z),
                                   cmac<double>(s1, nullptr, nullptr), cmac<double>(g_s2, nullptr, nullptr),
                                   wmac<double>(g_u0x, g_u0y, g_u0z), wmac<double>(g_s1, nullptr, nullptr), s);
}

int fm_advect_u_grid_adj(const fm_grid* g, int dtype, int rk, double dx, double dt, const void* u0x,
                         const void* u0y, const void* u0z, const void* u1x, const void* u1y, const void* u1z,
                         const void* g_u2x, const void* g_u2y, const void* g_u2z, void* g_u0x, void* g_u0y,
                         void* g_u0z, void* g_u1x, void* g_u1y, void* g_u1z, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || !mac_args(*g, u0x, u0y, u0z, false) || !mac_args(*g, u1x, u1y, u1z, false) ||
      !mac_args(*g, g_u2x, g_u2y, g_u2z, false) || !mac_args(*g, g_u0x, g_u0y, g_u0z, true) ||
      !mac_args(*g, g_u1x, g_u1y, g_u1z, true))
    return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32)
    return advect_grid_adj_t<float>(*g, rk, dx, dt, 0, cmac<float>(u0x, u0y, u0z), cmac<float>(u1x, u1y, u1z),
                                    cmac<float>(g_u2x, g_u2y, g_u2z), wmac<float>(g_u0x, g_u0y, g_u0z),
                                    wmac<float>(g_u1x, g_u1y, g_u1z), s);
  return advect_grid_adj_t<double>(*g, rk, dx, dt, 0, cmac<double>(u0x, u0y, u0z), cmac<double>(u1x, u1y, u1z),
                                   cmac<double>(g_u2x, g_u2y, g_u2z), wmac<double>(g_u0x, g_u0y, g_u0z),
                                   wmac<double>(g_u1x, g_u1y, g_u1z), s);
}

int fm_pullback_u_adj(const fm_grid* g, int dtype, double dx, const void* u0x, const void* u0y, const void* u0z,
                      const void* Tx, const void* Ty, const void* Tz, const void* psix, const void* psiy,
                      const void* psiz, double alpha, double beta, const void* g_outx, const void* g_outy,
                      const void* g_outz, void* g_u0x, void* g_u0y, void* g_u0z, void* g_Tx, void* g_Ty,
                      void* g_Tz, void* g_psix, void* g_psiy, void* g_psiz, void* g_basex, void* g_basey,
                      void* g_basez, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!mac_args(*g, u0x, u0y, u0z, false) || !mac_args(*g, Tx, Ty, Tz, false) ||
      !mac_args(*g, psix, psiy, psiz, false) || !mac_args(*g, g_outx, g_outy, g_outz, false) ||
      !mac_args(*g, g_u0x, g_u0y, g_u0z, true) || !mac_args(*g, g_Tx, g_Ty, g_Tz, true) ||
      !mac_args(*g, g_psix, g_psiy, g_psiz, true) || !mac_args(*g, g_basex, g_basey, g_basez, true))
    return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const dim3 grid = blocks(max_face_size(*g), g->dim);
#define FM_PB_LAUNCH(T, D)                                                                                          \
  k_pullback_u_adj<T, D><<<grid, kAdjThreads, 0, s>>>(                                                              \
      *g, (T)dx, cmac<T>(u0x, u0y, u0z), cmac<T>(Tx, Ty, Tz), cmac<T>(psix, psiy, psiz), (T)alpha, (T)beta,         \
      cmac<T>(g_outx, g_outy, g_outz), wmac<T>(g_u0x, g_u0y, g_u0z), wmac<T>(g_Tx, g_Ty, g_Tz),                     \
      wmac<T>(g_psix, g_psiy, g_psiz), wmac<T>(g_basex, g_basey, g_basez))
  if (dtype == FM_F32) {
    if (g->dim == 3) FM_PB_LAUNCH(float, 3);
    else FM_PB_LAUNCH(float, 2);
  } else {
    if (g->dim == 3) FM_PB_LAUNCH(double, 3);
    else FM_PB_LAUNCH(double, 2);
  }
#undef FM_PB_LAUNCH
  return check_launch();
}

int fm_pullback_scalar_adj(const fm_grid* g, int dtype, double dx, const void* s0, const void* psi, double alpha,
                           double beta, const void* g_out, void* g_s0, void* g_psi, void* g_base, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!s0 || !psi || !g_out) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const dim3 grid = blocks(cell_shape(*g).size(), 1);
#define FM_PS_LAUNCH(T, D)                                                                                      \
  k_pullback_scalar_adj<T, D><<<grid, kAdjThreads, 0, s>>>(*g, (T)dx, (const T*)s0, (const T*)psi, (T)alpha,    \
                                                           (T)beta, (const T*)g_out, (T*)g_s0, (T*)g_psi,       \
                                                           (T*)g_base)
  if (dtype == FM_F32) {
    if (g->dim == 3) FM_PS_LAUNCH(float, 3);
    else FM_PS_LAUNCH(float, 2);
  } else {
    if (g->dim == 3) FM_PS_LAUNCH(double, 3);
    else FM_PS_LAUNCH(double, 2);
  }
#undef FM_PS_LAUNCH
  return check_launch();
}

int fm_rk_grid_adj(const fm_grid* g, int dtype, int rk, double dx, double dt, int face, const void* psi,
                   const void* T, const void* ux, const void* uy, const void* uz, const void* g_psi_out,
                   const void* g_T_out, void* g_psi, void* g_T, void* g_ux, void* g_uy, void* g_uz, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if ((rk != 2 && rk != 4) || face < -1 || face >= g->dim || !psi || !g_psi_out || (face == -1 && T) ||
      (!T != !g_T_out) || (!T && g_T) || !mac_args(*g, ux, uy, uz, false) || !mac_args(*g, g_ux, g_uy, g_uz, true))
    return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const long n = face >= 0 ? face_shape(*g, face).size() : cell_shape(*g).size();
  const dim3 grid = blocks(n, 1);
#define FM_MA_LAUNCH(Tp, D, RK, WT)                                                                             \
  k_march_adj<Tp, D, RK, WT><<<grid, kAdjThreads, 0, s>>>(*g, (Tp)dx, (Tp)dt, face, cmac<Tp>(ux, uy, uz),        \
                                                          (const Tp*)psi, (const Tp*)T, (const Tp*)g_psi_out,   \
                                                          (const Tp*)g_T_out, wmac<Tp>(g_ux, g_uy, g_uz),       \
                                                          (Tp*)g_psi, (Tp*)g_T)
#define FM_MA_WT(Tp, D, RK)              \
  if (T) FM_MA_LAUNCH(Tp, D, RK, true);  \
  else FM_MA_LAUNCH(Tp, D, RK, false)
#define FM_MA_RK(Tp, D)          \
  if (rk == 2) { FM_MA_WT(Tp, D, 2); } \
  else { FM_MA_WT(Tp, D, 4); }
  if (dtype == FM_F32) {
    if (g->dim == 3) { FM_MA_RK(float, 3) }
    else { FM_MA_RK(float, 2) }
  } else {
    if (g->dim == 3) { FM_MA_RK(double, 3) }
    else { FM_MA_RK(double, 2) }
  }
#undef FM_MA_RK
#undef FM_MA_WT
#undef FM_MA_LAUNCH
  return check_launch();
}

}  // extern "C"
