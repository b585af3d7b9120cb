// fm_force.cu -- Gaussian control forces and their parameter adjoint.
//
// Force (apply_gausion_force_kernel, 3D/lfm_midpoint_simulator.py:309-344,
// 2D/shape/lfm_midpoint_simulator.py:283-299): on every MAC face X of
// component c,
//     f_c(X) = sum over I < n with q_I(X) < 5 of exp(-q_I(X)) s_I[c],
//     q_I(X) = |X - c_I|^2 r_I   (|.| = sqrt of the sum of squares, squared),
// summed in ascending I as the reference's per-face loop does; r_I is the
// inverse squared radius.
//
// Adjoint (calculate_adj_gausion_force_kernel,
// 3D/lfm_midpoint_diff_simulator.py:63-110): for every Gaussian the sums over
// the faces of its support of
//     adj_strength[c] += e a_c            adj_center += s_c e 2 (X - c) r a_c
//     pen_strength[c] += 2 f e            pen_center += 2 f s_c e 2 (X - c) r
// with e = exp(-q), f = e s_c and a the adjoint velocity, in the reference's
// operation order per face, accumulated in FP64.
//
// B200 mapping.  3000 Gaussians against every face is compute work, so both
// kernels cull by support first:
//  * k_gauss_force: one CTA per tile of cells (16x16 in 2D, 8x8x8 in 3D).  The
//    CTA walks the Gaussians in chunks of 256, keeps those whose support ball
//    (radius sqrt(5/r), widened) reaches the tile's box, compacted in
//    ascending order into shared memory (ballot + popc prefix), and every
//    thread accumulates its faces over that list.  The cull is a superset of
//    the exact per-face test, which decides inclusion with the reference's
//    rounding (no FMA contraction), so culling never changes a sum.
//  * k_gauss_grad: one CTA per Gaussian over the face-index box of its
//    support; fixed-order warp-shuffle + shared-memory reduction, so the
//    result is deterministic (the reference's atomics are not).
#include <math.h>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

constexpr int kGfThreads = 256;
constexpr int kGfWarps = kGfThreads / 32;
constexpr int kGfMaxN = 1 << 24;

template <int D> struct GfTile;
template <> struct GfTile<2> { static constexpr int B0 = 16, B1 = 16, B2 = 1, F = 2; };  // 17*16 faces <= 2*256
template <> struct GfTile<3> { static constexpr int B0 = 8, B1 = 8, B2 = 8, F = 3; };    // 9*8*8 faces <= 3*256

// Relative widening of the support radius used by the culls; far above the
// few ulps by which the exact test's rounding can move the boundary.
constexpr double kGfMargin = 1e-4;

// The exact inclusion test and weight at one face, with the reference's
// rounding: d = sqrt(sum (X - c)^2), q = (d d) r, included iff q < 5, e = exp(-q).
// The pre-test rejects, without the square root, faces whose s2 r exceeds 5 by
// more than the rounding of the exact path can account for.
template <typename T, int D>
__device__ __forceinline__ bool gf_weight(const T* p, const T* c, T r, T* dp, T& e, T& q) {
#pragma unroll
  for (int a = 0; a < D; ++a) dp[a] = rn_sub(p[a], c[a]);
  T s2 = rn_mul(dp[0], dp[0]);
#pragma unroll
  for (int a = 1; a < D; ++a) s2 = rn_add(s2, rn_mul(dp[a], dp[a]));
  if (r > (T)0 && rn_mul(s2, r) > (T)(5.0 * (1.0 + kGfMargin))) return false;
  const T d = sqrt(s2);
  q = rn_mul(rn_mul(d, d), r);
  if (!(q < (T)5)) return false;
  e = exp(-q);
  return true;
}

// Tile cull: does Gaussian (c, r) possibly reach a face inside [lo, hi]?
template <typename T, int D>
__device__ __forceinline__ bool gf_touches(const T* c, T r, const double* lo, const double* hi) {
  if (r != r) return false;          // NaN radius: the exact test excludes every face
  if (!(r > (T)0)) return true;      // r <= 0: q <= 0 everywhere (left to the exact test)
  double d2 = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double x = (double)c[a];
    const double t = x < lo[a] ? lo[a] - x : (x > hi[a] ? x - hi[a] : 0.0);
    d2 += t * t;
  }
  return d2 <= 5.0 / (double)r * (1.0 + kGfMargin);
}

template <typename T, int D>
__global__ void __launch_bounds__(kGfThreads) k_gauss_force(fm_grid g, T dx, int n, const T* __restrict__ cen,
                                                            const T* __restrict__ ir, const T* __restrict__ str,
                                                            T* __restrict__ f0, T* __restrict__ f1,
                                                            T* __restrict__ f2) {
  using Tl = GfTile<D>;
  constexpr int F = Tl::F;
  __shared__ T s_c[D][kGfThreads], s_s[D][kGfThreads], s_r[kGfThreads];
  __shared__ int s_cnt[kGfWarps];

  const int nt1 = (g.n[1] + Tl::B1 - 1) / Tl::B1, nt2 = (g.n[2] + Tl::B2 - 1) / Tl::B2;
  int t = blockIdx.x;
  const int t2 = t % nt2;
  t /= nt2;
  const int t1 = t % nt1, t0 = t / nt1;
  const int lo[3] = {t0 * Tl::B0, t1 * Tl::B1, t2 * Tl::B2};
  const int hc[3] = {min(lo[0] + Tl::B0, g.n[0]), min(lo[1] + Tl::B1, g.n[1]), min(lo[2] + Tl::B2, g.n[2])};
  // the tile's box: faces at i dx (the last tile along an axis also owns the
  // face at n dx), centres at (i + 1/2) dx, widened by a hundredth of a cell
  double blo[3], bhi[3];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    blo[a] = ((double)lo[a] - 0.01) * (double)dx;
    bhi[a] = ((double)hc[a] + 1.01) * (double)dx;
  }

  T acc[D][F];
#pragma unroll
  for (int c = 0; c < D; ++c)
#pragma unroll
    for (int m = 0; m < F; ++m) acc[c][m] = (T)0;

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < n; base += kGfThreads) {
    const int I = base + threadIdx.x;
    T c[D], s[D], r = (T)0;
    bool hit = false;
    if (I < n) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        c[a] = cen[(long)I * D + a];
        s[a] = str[(long)I * D + a];
      }
      r = ir[I];
      hit = gf_touches<T, D>(c, r, blo, bhi);
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_cnt[w] = __popc(m);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int k = 0; k < kGfWarps; ++k) {
      const int v = s_cnt[k];
      off += k < w ? v : 0;
      tot += v;
    }
    if (hit) {
      const int slot = off + __popc(m & ((1u << lane) - 1u));
#pragma unroll
      for (int a = 0; a < D; ++a) {
        s_c[a][slot] = c[a];
        s_s[a][slot] = s[a];
      }
      s_r[slot] = r;
    }
    __syncthreads();
    if (tot > 0) {
#pragma unroll
      for (int cc = 0; cc < D; ++cc) {
        const int e0 = hc[0] + (cc == 0 && hc[0] == g.n[0]) - lo[0];
        const int e1 = hc[1] + (cc == 1 && hc[1] == g.n[1]) - lo[1];
        const int e2 = hc[2] + (cc == 2 && hc[2] == g.n[2]) - lo[2];
#pragma unroll
        for (int fm_ = 0; fm_ < F; ++fm_) {
          const int q = threadIdx.x + fm_ * kGfThreads;
          if (q >= e0 * e1 * e2) continue;
          const int k = q % e2, ij = q / e2, j = ij % e1, i = ij / e1;
          T p[D];
          node_pos<T, D>(cc, lo[0] + i, lo[1] + j, lo[2] + k, dx, p);
          T a = acc[cc][fm_];
          for (int l = 0; l < tot; ++l) {
            T cl[D], dp[D], e, qq;
#pragma unroll
            for (int b = 0; b < D; ++b) cl[b] = s_c[b][l];
            if (gf_weight<T, D>(p, cl, s_r[l], dp, e, qq)) a = rn_add(a, rn_mul(e, s_s[cc][l]));
          }
          acc[cc][fm_] = a;
        }
      }
    }
    __syncthreads();  // the next chunk overwrites the list and the counts
  }

#pragma unroll
  for (int cc = 0; cc < D; ++cc) {
    const Shape fs = face_shape(g, cc);
    const int e0 = hc[0] + (cc == 0 && hc[0] == g.n[0]) - lo[0];
    const int e1 = hc[1] + (cc == 1 && hc[1] == g.n[1]) - lo[1];
    const int e2 = hc[2] + (cc == 2 && hc[2] == g.n[2]) - lo[2];
#pragma unroll
    for (int fm_ = 0; fm_ < F; ++fm_) {
      const int q = threadIdx.x + fm_ * kGfThreads;
      if (q >= e0 * e1 * e2) continue;
      const int k = q % e2, ij = q / e2, j = ij % e1, i = ij / e1;
      T* const o = cc == 0 ? f0 : (cc == 1 ? f1 : f2);
      o[fs.idx(lo[0] + i, lo[1] + j, lo[2] + k)] = acc[cc][fm_];
    }
  }
}

// Face-index range along axis `a` of component-`c` faces within the support
// of a Gaussian at x with widened radius R (R < 0: the whole axis).
__device__ __forceinline__ void gf_axis_range(double x, double R, double dx, bool face_axis, int len, int& i0,
                                              int& i1) {
  if (R < 0) {
    i0 = 0;
    i1 = len - 1;
    return;
  }
  const double off = face_axis ? 0.0 : 0.5;
  double a = ceil((x - R) / dx - off) - 1.0, b = floor((x + R) / dx - off) + 1.0;
  a = fmax(a, 0.0);
  b = fmin(b, (double)(len - 1));
  if (!(a <= b)) {
    i0 = 1;
    i1 = 0;
    return;
  }
  i0 = (int)a;
  i1 = (int)b;
}

template <typename T, int D>
__global__ void __launch_bounds__(kGfThreads) k_gauss_grad(fm_grid g, T dx, const T* __restrict__ cen,
                                                           const T* __restrict__ ir, const T* __restrict__ str,
                                                           const T* __restrict__ a0, const T* __restrict__ a1,
                                                           const T* __restrict__ a2, double* __restrict__ adj_c,
                                                           double* __restrict__ adj_s, double* __restrict__ pen_c,
                                                           double* __restrict__ pen_s) {
  constexpr int NV = 4 * D;  // adj_strength, adj_center, pen_strength, pen_center
  __shared__ double s_red[kGfWarps][NV];
  const int I = blockIdx.x;
  T c[D], s[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    c[a] = cen[(long)I * D + a];
    s[a] = str[(long)I * D + a];
  }
  const T r = ir[I];
  // support radius (widened) or -1 for "every face"; NaN r or a non-finite
  // centre with r > 0 reaches no face
  double R = -1.0;
  bool none = r != r;
  if (r > (T)0) {
    R = sqrt(5.0 / (double)r) * (1.0 + kGfMargin) + 0.01 * (double)dx;
#pragma unroll
    for (int a = 0; a < D; ++a) none = none || !isfinite((double)c[a]);
  }
  const T* const adj[3] = {a0, a1, a2};
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;

  if (!none) {
#pragma unroll
    for (int cc = 0; cc < D; ++cc) {
      const Shape fs = face_shape(g, cc);
      int i0[3] = {0, 0, 0}, i1[3] = {0, 0, 0};
#pragma unroll
      for (int a = 0; a < D; ++a) gf_axis_range((double)c[a], R, (double)dx, a == cc, axis_len(fs, a), i0[a], i1[a]);
      const int e0 = i1[0] - i0[0] + 1, e1 = i1[1] - i0[1] + 1, e2 = i1[2] - i0[2] + 1;
      if (e0 <= 0 || e1 <= 0 || e2 <= 0) continue;
      // a face grid holds fewer than 2^32 entries (validate_grid): 32-bit decode
      const unsigned cnt = (unsigned)e0 * (unsigned)e1 * (unsigned)e2;
      const T sc = s[cc];
      for (unsigned q = threadIdx.x; q < cnt; q += kGfThreads) {
        const unsigned ij = q / (unsigned)e2;
        const int k = (int)(q - ij * (unsigned)e2);
        const unsigned ii = ij / (unsigned)e1;
        const int j = (int)(ij - ii * (unsigned)e1), i = (int)ii;
        T p[D], dp[D], e, qq;
        node_pos<T, D>(cc, i0[0] + i, i0[1] + j, i0[2] + k, dx, p);
        if (!gf_weight<T, D>(p, c, r, dp, e, qq)) continue;
        const T av = adj[cc][fs.idx(i0[0] + i, i0[1] + j, i0[2] + k)];
        const T f = rn_mul(e, sc);
        v[cc] += (double)rn_mul(e, av);                       // adj_strength[c]
        v[2 * D + cc] += (double)rn_mul(rn_mul((T)2, f), e);  // pen_strength[c]
        const T ga = rn_mul(rn_mul(sc, e), (T)2);             // s e 2
        const T gp = rn_mul(rn_mul(rn_mul(rn_mul((T)2, f), sc), e), (T)2);  // 2 f s e 2
#pragma unroll
        for (int a = 0; a < D; ++a) {
          v[D + a] += (double)rn_mul(rn_mul(rn_mul(ga, dp[a]), r), av);  // adj_center
          v[3 * D + a] += (double)rn_mul(rn_mul(gp, dp[a]), r);          // pen_center
        }
      }
    }
  }
  // fixed-order reduction: butterfly within each warp, then warps in order
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    v[k] = x;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) s_red[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0.0;
#pragma unroll
    for (int k = 0; k < kGfWarps; ++k) x += s_red[k][threadIdx.x];
    const int which = threadIdx.x / D, a = threadIdx.x % D;
    double* const o = which == 0 ? adj_s : (which == 1 ? adj_c : (which == 2 ? pen_s : pen_c));
    o[(long)I * D + a] = x;
  }
}

template <typename T>
int gauss_force(const fm_grid& g, double dx, int n, const void* cen, const void* ir, const void* str, void* fx,
                void* fy, void* fz, cudaStream_t s) {
  const T tdx = (T)dx;
  if (g.dim == 2) {
    using Tl = GfTile<2>;
    const unsigned tiles = (unsigned)(((g.n[0] + Tl::B0 - 1) / Tl::B0) * ((g.n[1] + Tl::B1 - 1) / Tl::B1));
    launch(k_gauss_force<T, 2>, tiles, kGfThreads, 0, s, g, tdx, n, (const T*)cen, (const T*)ir, (const T*)str,
           (T*)fx, (T*)fy, (T*)nullptr);
  } else {
    using Tl = GfTile<3>;
    const unsigned tiles = (unsigned)((long)((g.n[0] + Tl::B0 - 1) / Tl::B0) * ((g.n[1] + Tl::B1 - 1) / Tl::B1) *
                                      ((g.n[2] + Tl::B2 - 1) / Tl::B2));
    launch(k_gauss_force<T, 3>, tiles, kGfThreads, 0, s, g, tdx, n, (const T*)cen, (const T*)ir, (const T*)str,
           (T*)fx, (T*)fy, (T*)fz);
  }
  return check_cuda();
}

template <typename T>
int gauss_grad(const fm_grid& g, double dx, int n, const void* cen, const void* ir, const void* str, const void* ax,
               const void* ay, const void* az, double* adj_c, double* adj_s, double* pen_c, double* pen_s,
               cudaStream_t s) {
  if (n == 0) return FM_OK;
  if (g.dim == 2)
    launch(k_gauss_grad<T, 2>, (unsigned)n, kGfThreads, 0, s, g, (T)dx, (const T*)cen, (const T*)ir, (const T*)str,
           (const T*)ax, (const T*)ay, (const T*)nullptr, adj_c, adj_s, pen_c, pen_s);
  else
    launch(k_gauss_grad<T, 3>, (unsigned)n, kGfThreads, 0, s, g, (T)dx, (const T*)cen, (const T*)ir, (const T*)str,
           (const T*)ax, (const T*)ay, (const T*)az, adj_c, adj_s, pen_c, pen_s);
  return check_cuda();
}

}  // namespace fm

extern "C" {

int fm_gaussian_force(const fm_grid* g, int dtype, double dx, int n, const void* center, const void* inv_radius,
                      const void* strength, void* f_x, void* f_y, void* f_z, void* stream) {
  using namespace fm;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (n < 0 || n > kGfMaxN || !(dx > 0)) return FM_ERR_ARG;
  if (n > 0 && (!center || !inv_radius || !strength)) return FM_ERR_ARG;
  if (!f_x || !f_y || (g->dim == 3 && !f_z)) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32) return gauss_force<float>(*g, dx, n, center, inv_radius, strength, f_x, f_y, f_z, s);
  return gauss_force<double>(*g, dx, n, center, inv_radius, strength, f_x, f_y, f_z, s);
}

int fm_gaussian_force_grad(const fm_grid* g, int dtype, double dx, int n, const void* center, const void* inv_radius,
                           const void* strength, const void* adj_x, const void* adj_y, const void* adj_z,
                           double* adj_center, double* adj_strength, double* penalty_center,
                           double* penalty_strength, void* stream) {
  using namespace fm;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (n < 0 || n > kGfMaxN || !(dx > 0)) return FM_ERR_ARG;
  if (n > 0 && (!center || !inv_radius || !strength || !adj_center || !adj_strength || !penalty_center ||
                !penalty_strength))
    return FM_ERR_ARG;
  if (!adj_x || !adj_y || (g->dim == 3 && !adj_z)) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32)
    return gauss_grad<float>(*g, dx, n, center, inv_radius, strength, adj_x, adj_y, adj_z, adj_center, adj_strength,
                             penalty_center, penalty_strength, s);
  return gauss_grad<double>(*g, dx, n, center, inv_radius, strength, adj_x, adj_y, adj_z, adj_center, adj_strength,
                            penalty_center, penalty_strength, s);
}

}  // extern "C"
