// fm_stencil.cu -- the adjoint source terms as tiled separable stencils.
//
//   calculate_nabla_u_w           r_c = sum_a (d_c u_a)(X_c) w_a(X_c)   (3D/flowmap.py:359-380,
//                                                                        2D/vortex/flowmap.py:361-377)
//   calculate_nabla_scalar_adjoint r_c = (d_c s)(X_c) adj_s(X_c)        (3D/flowmap.py:382-403)
//
// Both interpolate with cubic (3D) / quartic (2D) B-splines at the face nodes
// X_c themselves.  The stencil along an axis (first tap, weights) depends only
// on the node's index along that axis, so the 3D sum factorises across a tile
// of nodes: one CTA loads the tile's input footprint into shared memory once
// and contracts it along k, then j, then i -- O(taps) work per node and each
// input value read from HBM about once, instead of a (taps)^3 gather per node.
// Weights, first taps and the clamp band follow the reference exactly
// (s = clamp(X/dx - BL, 1, len-2-eps), taps iu+lo+t, sample() index clamp);
// only the summation order differs.
#include <cmath>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

// 3D tile: TI x TJ x TK output nodes (k contiguous); 2D: TI x TJ (j contiguous)
constexpr int kTJ3 = 8, kTK3 = 32;  // the tile height along i is a template parameter (4 or 8)
constexpr int kTJ2 = 64;  // the tile height along i is a template parameter (8, 12 or 16)
constexpr int kStThreads = 256;

template <typename T>
struct StTerm {
  const T* f;  // differentiated along the output face axis
  const T* h;  // interpolated
  int s0, s1, s2;
  T bl0, bl1, bl2;
};
template <typename T>
struct StTerms {
  StTerm<T> t[3];
  int n;
};

template <typename T>
__device__ __forceinline__ StTerm<T> pick_term(const StTerms<T>& ts, int a) {
  return a == 0 ? ts.t[0] : (a == 1 ? ts.t[1] : ts.t[2]);
}

// Per-axis stencil of one output node: unclamped first tap, weights and
// derivative weights of the ORDER+1 taps that can be non-zero.
template <typename T, int ORDER>
__device__ __forceinline__ void axis_stencil(T pos, T dx, T bl, int len, int& base, T* w, T* dw) {
  constexpr int NZ = Taps<ORDER>::nz;
  T u = pos / dx;
  u = u - bl;
  const T hi = (T)((double)len - 2.0 - 1e-6);
  T s = u < hi ? u : hi;
  s = s > (T)1 ? s : (T)1;
  const T iu = floor(s);
  const T f = s - iu;
  int t0;
  if (ORDER == 3) t0 = 1;
  else if (ORDER == 2) t0 = f >= (T)0.5 ? 1 : 0;
  else t0 = f >= (T)0.5 ? 2 : 1;
  base = (int)iu + Taps<ORDER>::lo + t0;
#pragma unroll
  for (int t = 0; t < NZ; ++t) {
    const T x = s - (iu + (T)(Taps<ORDER>::lo + t0 + t));
    bs_eval<T, ORDER>(x, w[t], dw[t]);
  }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename T, int ORDER, int M, int TI3>
__global__ void __launch_bounds__(kStThreads) k_fixed_grad_dot3(fm_grid g, T dx, int c, StTerms<T> terms,
                                                                  T* __restrict__ out) {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int TI = TI3, TJ = kTJ3, TK = kTK3;
  // footprint: taps from the tile's first base - M (see fixed3_smem)
  constexpr int FI = TI + NZ - 1 + 2 * M, FJ = TJ + NZ - 1 + 2 * M, FK = TK + NZ - 1 + 2 * M;
  constexpr int NOUT = TI * TJ * TK / kStThreads;
  // dynamic shared: [F | H] footprints, then [Af | Ah] after the k pass; the
  // j pass reuses the footprint region for [Bf | Bh]
  extern __shared__ __align__(16) unsigned char st_smem[];
  T* sF = reinterpret_cast<T*>(st_smem);
  T* sA = sF + 2 * FI * FJ * FK;
  __shared__ T wI[TI][NZ], dI[TI][NZ], wJ[TJ][NZ], dJ[TJ][NZ], wK[TK][NZ], dK[TK][NZ];
  __shared__ int bI[TI], bJ[TJ], bK[TK];

  const Shape so = face_shape(g, c);
  const int i0 = blockIdx.z * TI, j0 = blockIdx.y * TJ, k0 = blockIdx.x * TK;
  const T inv_dx = (T)1 / dx;
  T acc[NOUT];
#pragma unroll
  for (int e = 0; e < NOUT; ++e) acc[e] = 0;

  for (int a = 0; a < terms.n; ++a) {
    const StTerm<T> tm = pick_term(terms, a);
    __syncthreads();
    // axis tables (node positions: face axis at i*dx, others at (i+0.5)*dx)
    for (int e = threadIdx.x; e < TI + TJ + TK; e += blockDim.x) {
      int ax, loc, len;
      T bl;
      if (e < TI) { ax = 0; loc = e; len = tm.s0; bl = tm.bl0; }
      else if (e < TI + TJ) { ax = 1; loc = e - TI; len = tm.s1; bl = tm.bl1; }
      else { ax = 2; loc = e - TI - TJ; len = tm.s2; bl = tm.bl2; }
      const int node = (ax == 0 ? i0 : (ax == 1 ? j0 : k0)) + loc;
      T fi = (T)node;
      if (ax != c) fi = fi + (T)0.5;
      const T pos = fi * dx;
      int base;
      T w[NZ], dw[NZ];
      axis_stencil<T, ORDER>(pos, dx, bl, len, base, w, dw);
      int* bt = ax == 0 ? bI : (ax == 1 ? bJ : bK);
      T* wt = ax == 0 ? &wI[0][0] : (ax == 1 ? &wJ[0][0] : &wK[0][0]);
      T* dt = ax == 0 ? &dI[0][0] : (ax == 1 ? &dJ[0][0] : &dK[0][0]);
      bt[loc] = base;
#pragma unroll
      for (int t = 0; t < NZ; ++t) { wt[loc * NZ + t] = w[t]; dt[loc * NZ + t] = dw[t]; }
    }
    __syncthreads();
    const int li = bI[0] - M, lj = bJ[0] - M, lk = bK[0] - M;
    // footprint (clamped indices: sample())
    for (int e = threadIdx.x; e < FI * FJ * FK; e += blockDim.x) {
      const int kk = e % FK, jj = (e / FK) % FJ, ii = e / (FK * FJ);
      const int gi = clampi(li + ii, 0, tm.s0 - 1), gj = clampi(lj + jj, 0, tm.s1 - 1),
                gk = clampi(lk + kk, 0, tm.s2 - 1);
      const long q = ((long)gi * tm.s1 + gj) * tm.s2 + gk;
      sF[e] = ldg(tm.f + q);
      sF[FI * FJ * FK + e] = ldg(tm.h + q);
    }
    __syncthreads();
    // k pass
    for (int e = threadIdx.x; e < FI * FJ * TK; e += blockDim.x) {
      const int k = e % TK, row = e / TK;
      const int off = bK[k] - lk;
      const T* Fr = sF + row * FK + off;
      const T* Hr = sF + FI * FJ * FK + row * FK + off;
      const T* wf = c == 2 ? &dK[k][0] : &wK[k][0];
      T af = 0, ah = 0;
#pragma unroll
      for (int t = 0; t < NZ; ++t) { af += Fr[t] * wf[t]; ah += Hr[t] * wK[k][t]; }
      sA[e] = af;
      sA[FI * FJ * TK + e] = ah;
    }
    __syncthreads();
    // j pass into the footprint region
    T* sB = sF;
    for (int e = threadIdx.x; e < FI * TJ * TK; e += blockDim.x) {
      const int k = e % TK, j = (e / TK) % TJ, ii = e / (TK * TJ);
      const int off = bJ[j] - lj;
      const T* wf = c == 1 ? &dJ[j][0] : &wJ[j][0];
      T bf = 0, bh = 0;
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        const int src = (ii * FJ + off + t) * TK + k;
        bf += sA[src] * wf[t];
        bh += sA[FI * FJ * TK + src] * wJ[j][t];
      }
      sB[e] = bf;
      sB[FI * TJ * TK + e] = bh;
    }
    __syncthreads();
    // i pass and product, NOUT outputs per thread
#pragma unroll
    for (int r = 0; r < NOUT; ++r) {
      const int e = threadIdx.x + r * kStThreads;
      const int k = e % TK, j = (e / TK) % TJ, i = e / (TK * TJ);
      const int off = bI[i] - li;
      const T* wf = c == 0 ? &dI[i][0] : &wI[i][0];
      T gf = 0, hh = 0;
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        const int src = ((off + t) * TJ + j) * TK + k;
        gf += sB[src] * wf[t];
        hh += sB[FI * TJ * TK + src] * wI[i][t];
      }
      acc[r] += (gf * inv_dx) * hh;
    }
  }
#pragma unroll
  for (int r = 0; r < NOUT; ++r) {
    const int e = threadIdx.x + r * kStThreads;
    const int k = k0 + e % TK, j = j0 + (e / TK) % TJ, i = i0 + e / (TK * TJ);
    if (i < so.s0 && j < so.s1 && k < so.s2) out[so.idx(i, j, k)] = acc[r];
  }
}

template <typename T, int ORDER, int M, int TI2>
__global__ void __launch_bounds__(kStThreads) k_fixed_grad_dot2(fm_grid g, T dx, int c, StTerms<T> terms,
                                                                  T* __restrict__ out) {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int TI = TI2, TJ = kTJ2;
  constexpr int FI = TI + NZ - 1 + 2 * M, FJ = TJ + NZ - 1 + 2 * M;  // taps from the first base - M (fixed3_smem)
  constexpr int NOUT = TI * TJ / kStThreads;
  __shared__ T sF[2 * FI * FJ];
  __shared__ T sA[2 * FI * TJ];
  __shared__ T wI[TI][NZ], dI[TI][NZ], wJ[TJ][NZ], dJ[TJ][NZ];
  __shared__ int bI[TI], bJ[TJ];

  const Shape so = face_shape(g, c);
  const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
  const T inv_dx = (T)1 / dx;
  T acc[NOUT];
#pragma unroll
  for (int e = 0; e < NOUT; ++e) acc[e] = 0;

  for (int a = 0; a < terms.n; ++a) {
    const StTerm<T> tm = pick_term(terms, a);
    __syncthreads();
    for (int e = threadIdx.x; e < TI + TJ; e += blockDim.x) {
      const int ax = e < TI ? 0 : 1, loc = e < TI ? e : e - TI;
      const int len = ax == 0 ? tm.s0 : tm.s1;
      const T bl = ax == 0 ? tm.bl0 : tm.bl1;
      const int node = (ax == 0 ? i0 : j0) + loc;
      T fi = (T)node;
      if (ax != c) fi = fi + (T)0.5;
      int base;
      T w[NZ], dw[NZ];
      axis_stencil<T, ORDER>(fi * dx, dx, bl, len, base, w, dw);
      (ax == 0 ? bI : bJ)[loc] = base;
      T* wt = ax == 0 ? &wI[0][0] : &wJ[0][0];
      T* dt = ax == 0 ? &dI[0][0] : &dJ[0][0];
#pragma unroll
      for (int t = 0; t < NZ; ++t) { wt[loc * NZ + t] = w[t]; dt[loc * NZ + t] = dw[t]; }
    }
    __syncthreads();
    const int li = bI[0] - M, lj = bJ[0] - M;
    for (int e = threadIdx.x; e < FI * FJ; e += blockDim.x) {
      const int jj = e % FJ, ii = e / FJ;
      const long q = (long)clampi(li + ii, 0, tm.s0 - 1) * tm.s1 + clampi(lj + jj, 0, tm.s1 - 1);
      sF[e] = ldg(tm.f + q);
      sF[FI * FJ + e] = ldg(tm.h + q);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < FI * TJ; e += blockDim.x) {
      const int j = e % TJ, ii = e / TJ;
      const int off = bJ[j] - lj;
      const T* wf = c == 1 ? &dJ[j][0] : &wJ[j][0];
      T af = 0, ah = 0;
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        af += sF[ii * FJ + off + t] * wf[t];
        ah += sF[FI * FJ + ii * FJ + off + t] * wJ[j][t];
      }
      sA[e] = af;
      sA[FI * TJ + e] = ah;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NOUT; ++r) {
      const int e = threadIdx.x + r * kStThreads;
      const int j = e % TJ, i = e / TJ;
      const int off = bI[i] - li;
      const T* wf = c == 0 ? &dI[i][0] : &wI[i][0];
      T gf = 0, hh = 0;
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        gf += sA[(off + t) * TJ + j] * wf[t];
        hh += sA[FI * TJ + (off + t) * TJ + j] * wI[i][t];
      }
      acc[r] += (gf * inv_dx) * hh;
    }
  }
#pragma unroll
  for (int r = 0; r < NOUT; ++r) {
    const int e = threadIdx.x + r * kStThreads;
    const int j = j0 + e % TJ, i = i0 + e / TJ;
    if (i < so.s0 && j < so.s1) out[so.idx(i, j, 0)] = acc[r];
  }
}

// A node's first tap is floor(node position / dx - BL) plus a constant.  With a
// power-of-two dx the quotient is exact and the first taps of a tile of n nodes
// lie within [b0, b0 + n - 1] of the first node's b0 (M = 0).  Otherwise the
// quotient carries a rounding error and they lie within [b0 - 1, b0 + n]: the
// footprints then hold n + NZ + 1 taps from b0 - 1 (M = 1).
template <typename T, int ORDER, int M, int TI>
static size_t fixed3_smem() {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int FI = TI + NZ - 1 + 2 * M, FJ = kTJ3 + NZ - 1 + 2 * M, FK = kTK3 + NZ - 1 + 2 * M;
  return sizeof(T) * (2 * FI * FJ * FK + 2 * FI * FJ * kTK3);
}

static bool power_of_two(double x) {
  int e;
  return x > 0 && std::frexp(x, &e) == 0.5;
}

template <typename T, int ORDER, int M, int TI>
static void launch_fixed3(const fm_grid& g, T dx, int c, const StTerms<T>& terms, T* out, cudaStream_t s) {
  const Shape so = face_shape(g, c);
  const size_t smem = fixed3_smem<T, ORDER, M, TI>();
  if (!raise_smem_limit(k_fixed_grad_dot3<T, ORDER, M, TI>, smem)) return;
  dim3 grid((so.s2 + kTK3 - 1) / kTK3, (so.s1 + kTJ3 - 1) / kTJ3, (so.s0 + TI - 1) / TI);
  launch(k_fixed_grad_dot3<T, ORDER, M, TI>, grid, kStThreads, smem, s, g, dx, c, terms, out);
}

template <typename T, int ORDER>
static void launch_fixed(const fm_grid& g, T dx, int c, const StTerms<T>& terms, T* out, cudaStream_t s) {
  const Shape so = face_shape(g, c);
  // tile height along i: the autotuner's choice (fm_tune_set, FM_TUNE_ADJ_SOURCE_TILE),
  // else 8 in 3D and 16 in 2D; the tile changes only the speed, never a result
  const int ti = tuned_value(FM_TUNE_ADJ_SOURCE_TILE, g, g.dim == 3 ? 8 : 16);
  const bool exact = power_of_two((double)dx);
  if (g.dim == 3) {
    if (exact) {
      if (ti == 4) launch_fixed3<T, ORDER, 0, 4>(g, dx, c, terms, out, s);
      else launch_fixed3<T, ORDER, 0, 8>(g, dx, c, terms, out, s);
    } else {
      if (ti == 4) launch_fixed3<T, ORDER, 1, 4>(g, dx, c, terms, out, s);
      else launch_fixed3<T, ORDER, 1, 8>(g, dx, c, terms, out, s);
    }
  } else {
    // with margins a 16-row FP64 quartic tile would exceed 48 KB of static shared memory: 12 rows
    if (ti == 8) {
      dim3 grid((so.s1 + kTJ2 - 1) / kTJ2, (so.s0 + 7) / 8, 1);
      if (exact) launch(k_fixed_grad_dot2<T, ORDER, 0, 8>, grid, kStThreads, 0, s, g, dx, c, terms, out);
      else launch(k_fixed_grad_dot2<T, ORDER, 1, 8>, grid, kStThreads, 0, s, g, dx, c, terms, out);
    } else if (exact) {
      dim3 grid((so.s1 + kTJ2 - 1) / kTJ2, (so.s0 + 15) / 16, 1);
      launch(k_fixed_grad_dot2<T, ORDER, 0, 16>, grid, kStThreads, 0, s, g, dx, c, terms, out);
    } else {
      dim3 grid((so.s1 + kTJ2 - 1) / kTJ2, (so.s0 + 11) / 12, 1);
      launch(k_fixed_grad_dot2<T, ORDER, 1, 12>, grid, kStThreads, 0, s, g, dx, c, terms, out);
    }
  }
}

template <typename T>
static int fixed_grad_dot(const fm_grid& g, int order, double dx, int c, const StTerms<T>& terms, T* out,
                          cudaStream_t s) {
  if (order == 2) launch_fixed<T, 2>(g, (T)dx, c, terms, out, s);
  else if (order == 3) launch_fixed<T, 3>(g, (T)dx, c, terms, out, s);
  else launch_fixed<T, 4>(g, (T)dx, c, terms, out, s);
  return check_cuda();
}

template <typename T>
static int nabla_u_w_t(const fm_grid& g, int order, double dx, const void* const* u, const void* const* w,
                       void* const* r, cudaStream_t s) {
  StTerms<T> terms{};
  terms.n = g.dim;
  for (int a = 0; a < g.dim; ++a) {
    const Shape sa = face_shape(g, a);
    terms.t[a] = StTerm<T>{(const T*)u[a], (const T*)w[a], sa.s0, sa.s1, sa.s2,
                           a == 0 ? (T)0 : (T)0.5, a == 1 ? (T)0 : (T)0.5, a == 2 ? (T)0 : (T)0.5};
  }
  for (int c = 0; c < g.dim; ++c) {
    int st = fixed_grad_dot<T>(g, order, dx, c, terms, (T*)r[c], s);
    if (st) return st;
  }
  return FM_OK;
}

template <typename T>
static int nabla_scalar_t(const fm_grid& g, double dx, const void* sc, const void* adj, void* const* r,
                          cudaStream_t s) {
  StTerms<T> terms{};
  terms.n = 1;
  const Shape cs = cell_shape(g);
  terms.t[0] = StTerm<T>{(const T*)sc, (const T*)adj, cs.s0, cs.s1, cs.s2, (T)0.5, (T)0.5, (T)0.5};
  for (int c = 0; c < g.dim; ++c) {
    int st = fixed_grad_dot<T>(g, 3, dx, c, terms, (T*)r[c], s);
    if (st) return st;
  }
  return FM_OK;
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_nabla_u_w(const fm_grid* g, int dtype, int order, double dx, const void* ux, const void* uy, const void* uz,
                 const void* wx, const void* wy, const void* wz, void* rx, void* ry, void* rz, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  const void* u[3] = {ux, uy, uz};
  const void* w[3] = {wx, wy, wz};
  void* r[3] = {rx, ry, rz};
  if (order != 2 && order != 3 && order != 4) return FM_ERR_ARG;
  for (int c = 0; c < g->dim; ++c)
    if (!u[c] || !w[c] || !r[c]) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32) return nabla_u_w_t<float>(*g, order, dx, u, w, r, s);
  return nabla_u_w_t<double>(*g, order, dx, u, w, r, s);
}

int fm_nabla_scalar_adjoint(const fm_grid* g, int dtype, double dx, const void* sc, const void* adj, void* rx,
                            void* ry, void* rz, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  void* r[3] = {rx, ry, rz};
  if (!sc || !adj) return FM_ERR_ARG;
  for (int c = 0; c < g->dim; ++c)
    if (!r[c]) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32) return nabla_scalar_t<float>(*g, dx, sc, adj, r, s);
  return nabla_scalar_t<double>(*g, dx, sc, adj, r, s);
}

}  // extern "C"
