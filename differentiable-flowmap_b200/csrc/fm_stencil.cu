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
#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

// 3D tile: TI x TJ x TK output nodes (k contiguous); 2D: TI x TJ (j contiguous)
constexpr int kTI3 = 8, kTJ3 = 8, kTK3 = 32;
constexpr int kTI2 = 16, kTJ2 = 64;
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

template <typename T, int ORDER>
__global__ void __launch_bounds__(kStThreads) k_fixed_grad_dot3(fm_grid g, T dx, int c, StTerms<T> terms,
                                                                  T* __restrict__ out) {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int TI = kTI3, TJ = kTJ3, TK = kTK3;
  constexpr int FI = TI + NZ - 1, FJ = TJ + NZ - 1, FK = TK + NZ - 1;
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
    const int li = bI[0], lj = bJ[0], lk = bK[0];
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

template <typename T, int ORDER>
__global__ void __launch_bounds__(kStThreads) k_fixed_grad_dot2(fm_grid g, T dx, int c, StTerms<T> terms,
                                                                  T* __restrict__ out) {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int TI = kTI2, TJ = kTJ2;
  constexpr int FI = TI + NZ - 1, FJ = TJ + NZ - 1;
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
    const int li = bI[0], lj = bJ[0];
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

// ---------------------------------------------------------------------------
// 3D: plane-streaming form.  A CTA owns a kSJ x kSK tile of output nodes in
// (j, k) and walks an i-chunk of kSI outputs plane by plane.  For every input
// plane it loads the (j, k) footprint of every term's two fields once, contracts
// it along k (a sliding register window where the tile's stencils advance one
// tap per node) and then along j, and keeps the last NZ+1 contracted planes in
// registers; an output node is finished by the i contraction from that ring as
// soon as its last plane has been read.  Each input value is read from memory
// once per i-chunk (plus the chunk's NZ-1 halo planes), and all three terms of
// nabla_u_w share one pass.  Stencil tables, the clamp band and sample()'s
// index clamp are those of k_fixed_grad_dot3; only the summation order differs.
// ---------------------------------------------------------------------------
constexpr int kSJ = 16, kSK = 32, kSI = 16;
constexpr int kSThreads = 256;  // 32 k-lanes x 8 j-pairs

template <typename T, int ORDER, int NT>
struct StreamSmem {
  static constexpr int NZ = Taps<ORDER>::nz;
  static constexpr int FJ = kSJ + NZ - 1, FK = kSK + NZ - 1;
  static constexpr size_t plane = (size_t)NT * 2 * FJ * FK;   // footprints [a][f][jj][kk]
  static constexpr size_t kpass = (size_t)NT * 2 * FJ * kSK;  // after the k pass [a][f][jj][k]
  static constexpr size_t bytes = sizeof(T) * (plane + kpass);
};

template <typename T, int ORDER, int NT>
__global__ void __launch_bounds__(kSThreads) k_src_stream3(fm_grid g, T dx, int c, StTerms<T> terms,
                                                           T* __restrict__ out) {
  using SM = StreamSmem<T, ORDER, NT>;
  constexpr int NZ = SM::NZ, FJ = SM::FJ, FK = SM::FK, NR = NZ + 1;
  extern __shared__ __align__(16) unsigned char ss_raw[];
  T* sP = reinterpret_cast<T*>(ss_raw);
  T* sA = sP + SM::plane;
  __shared__ int bI[NT][kSI], bJ[NT][kSJ], bK[NT][kSK];
  __shared__ T wI[NT][2][kSI][NZ], wJ[NT][2][kSJ][NZ], wK[NT][2][kSK][NZ];
  __shared__ int fastJ[NT], fastK[NT];

  const Shape so = face_shape(g, c);
  const int i0 = blockIdx.z * kSI, j0 = blockIdx.y * kSJ, k0 = blockIdx.x * kSK;
  const int iend = min(i0 + kSI, so.s0);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const T inv_dx = (T)1 / dx;

  // per-term axis tables: first tap and weights of every node of the tile / chunk
  // (field f: derivative weights along the output face axis c, value weights
  // elsewhere; field h: value weights)
  for (int e = threadIdx.x; e < NT * (kSI + kSJ + kSK); e += blockDim.x) {
    const int a = e / (kSI + kSJ + kSK), r = e % (kSI + kSJ + kSK);
    const StTerm<T> tm = pick_term(terms, a);
    int ax, loc, len;
    T bl;
    if (r < kSI) { ax = 0; loc = r; len = tm.s0; bl = tm.bl0; }
    else if (r < kSI + kSJ) { ax = 1; loc = r - kSI; len = tm.s1; bl = tm.bl1; }
    else { ax = 2; loc = r - kSI - kSJ; len = tm.s2; bl = tm.bl2; }
    const int node = (ax == 0 ? i0 : (ax == 1 ? j0 : k0)) + loc;
    T fi = (T)node;
    if (ax != c) fi = fi + (T)0.5;
    int base;
    T w[NZ], dw[NZ];
    axis_stencil<T, ORDER>(fi * dx, dx, bl, len, base, w, dw);
    int* bt = ax == 0 ? &bI[a][loc] : (ax == 1 ? &bJ[a][loc] : &bK[a][loc]);
    T* wf = ax == 0 ? &wI[a][0][loc][0] : (ax == 1 ? &wJ[a][0][loc][0] : &wK[a][0][loc][0]);
    T* wh = ax == 0 ? &wI[a][1][loc][0] : (ax == 1 ? &wJ[a][1][loc][0] : &wK[a][1][loc][0]);
    *bt = base;
#pragma unroll
    for (int t = 0; t < NZ; ++t) {
      wf[t] = ax == c ? dw[t] : w[t];
      wh[t] = w[t];
    }
  }
  __syncthreads();
  // fast paths: the stencils of the whole tile advance one tap per node (no clamp
  // band inside the tile), so all nodes share one set of weights
  if (threadIdx.x < 2 * NT) {
    const int a = threadIdx.x >> 1;
    const bool alongK = threadIdx.x & 1;
    const int n = alongK ? kSK : kSJ;
    const int* b = alongK ? &bK[a][0] : &bJ[a][0];
    bool ok = true;
    for (int q = 1; q < n; ++q) ok = ok && b[q] == b[0] + q;
    if (alongK) fastK[a] = ok; else fastJ[a] = ok;
  }
  __syncthreads();

  // planes the chunk reads, over all terms
  int pmin = bI[0][0], pmax = bI[0][iend - 1 - i0];
#pragma unroll
  for (int a = 1; a < NT; ++a) {
    pmin = min(pmin, bI[a][0]);
    pmax = max(pmax, bI[a][iend - 1 - i0]);
  }
  pmax += NZ - 1;

  T ring[NT][2][2][NR];  // [term][field][j of the pair][plane p - slot]
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int f = 0; f < 2; ++f)
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int q = 0; q < NR; ++q) ring[a][f][m][q] = (T)0;
  int inext = i0;

  for (int p = pmin; p <= pmax; ++p) {
    // 1. footprints of plane p: rows of FK values, a warp per row (sample()'s index clamp)
    for (int row = ty; row < NT * 2 * FJ; row += kSThreads / 32) {
      const int a = row / (2 * FJ), f = (row / FJ) & 1, jj = row % FJ;
      const StTerm<T> tm = pick_term(terms, a);
      const T* src = f == 0 ? tm.f : tm.h;
      const int gi = clampi(p, 0, tm.s0 - 1), gj = clampi(bJ[a][0] + jj, 0, tm.s1 - 1);
      const long rb = ((long)gi * tm.s1 + gj) * tm.s2;
      T* dst = sP + (size_t)row * FK;
      for (int kk = tx; kk < FK; kk += 32) dst[kk] = ldg(src + rb + clampi(bK[a][0] + kk, 0, tm.s2 - 1));
    }
    __syncthreads();
    // 2. k pass: segments of 4 outputs of one row
    for (int task = threadIdx.x; task < NT * 2 * FJ * (kSK / 4); task += kSThreads) {
      const int row = task / (kSK / 4), seg = task % (kSK / 4);
      const int a = row / (2 * FJ), f = (row / FJ) & 1;
      const T* src = sP + (size_t)row * FK;
      T* dst = sA + (size_t)row * kSK + seg * 4;
      const int kb = seg * 4;
      if (fastK[a]) {
        const int o = bK[a][kb] - bK[a][0];
        T v[NZ + 3], w[NZ];
#pragma unroll
        for (int q = 0; q < NZ + 3; ++q) v[q] = src[o + q];
#pragma unroll
        for (int t = 0; t < NZ; ++t) w[t] = wK[a][f][kb][t];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          T acc = 0;
#pragma unroll
          for (int t = 0; t < NZ; ++t) acc += v[m + t] * w[t];
          dst[m] = acc;
        }
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int o = bK[a][kb + m] - bK[a][0];
          T acc = 0;
#pragma unroll
          for (int t = 0; t < NZ; ++t) acc += src[o + t] * wK[a][f][kb + m][t];
          dst[m] = acc;
        }
      }
    }
    __syncthreads();
    // 3. j pass for this thread's nodes (j = 2 ty, 2 ty + 1; k = tx), into the ring
    const int ja = 2 * ty;
#pragma unroll
    for (int a = 0; a < NT; ++a) {
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const T* col = sA + (size_t)(a * 2 + f) * FJ * kSK + tx;
        T r0 = 0, r1 = 0;
        if (fastJ[a]) {
          const int o = bJ[a][ja] - bJ[a][0];
          T v[NZ + 1];
#pragma unroll
          for (int q = 0; q < NZ + 1; ++q) v[q] = col[(o + q) * kSK];
#pragma unroll
          for (int t = 0; t < NZ; ++t) {
            const T w = wJ[a][f][ja][t];
            r0 += v[t] * w;
            r1 += v[t + 1] * w;
          }
        } else {
          const int o0 = bJ[a][ja] - bJ[a][0], o1 = bJ[a][ja + 1] - bJ[a][0];
#pragma unroll
          for (int t = 0; t < NZ; ++t) {
            r0 += col[(o0 + t) * kSK] * wJ[a][f][ja][t];
            r1 += col[(o1 + t) * kSK] * wJ[a][f][ja + 1][t];
          }
        }
#pragma unroll
        for (int q = NR - 1; q > 0; --q) {
          ring[a][f][0][q] = ring[a][f][0][q - 1];
          ring[a][f][1][q] = ring[a][f][1][q - 1];
        }
        ring[a][f][0][0] = r0;
        ring[a][f][1][0] = r1;
      }
    }
    // 4. finish every output whose last plane (over all terms) is p
    while (inext < iend) {
      const int li = inext - i0;
      int e = bI[0][li];
#pragma unroll
      for (int a = 1; a < NT; ++a) e = max(e, bI[a][li]);
      if (e + NZ - 1 != p) break;
      T acc0 = 0, acc1 = 0;
#pragma unroll
      for (int a = 0; a < NT; ++a) {
        const int d = e - bI[a][li];  // 0 or 1: this term's window ended one plane earlier
        T gf0 = 0, gf1 = 0, hh0 = 0, hh1 = 0;
#pragma unroll
        for (int t = 0; t < NZ; ++t) {
          const int slot = NZ - 1 - t;  // plane bI + t sits at ring slot d + NZ - 1 - t
          const T f0 = d ? ring[a][0][0][slot + 1] : ring[a][0][0][slot];
          const T f1 = d ? ring[a][0][1][slot + 1] : ring[a][0][1][slot];
          const T h0 = d ? ring[a][1][0][slot + 1] : ring[a][1][0][slot];
          const T h1 = d ? ring[a][1][1][slot + 1] : ring[a][1][1][slot];
          const T wf = wI[a][0][li][t], wh = wI[a][1][li][t];
          gf0 += f0 * wf;
          gf1 += f1 * wf;
          hh0 += h0 * wh;
          hh1 += h1 * wh;
        }
        acc0 += (gf0 * inv_dx) * hh0;
        acc1 += (gf1 * inv_dx) * hh1;
      }
      const int k = k0 + tx;
      if (k < so.s2) {
        if (j0 + ja < so.s1) out[so.idx(inext, j0 + ja, k)] = acc0;
        if (j0 + ja + 1 < so.s1) out[so.idx(inext, j0 + ja + 1, k)] = acc1;
      }
      ++inext;
    }
    __syncthreads();
  }
}

template <typename T, int ORDER>
static size_t fixed3_smem() {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int FI = kTI3 + NZ - 1, FJ = kTJ3 + NZ - 1, FK = kTK3 + NZ - 1;
  return sizeof(T) * (2 * FI * FJ * FK + 2 * FI * FJ * kTK3);
}

template <typename T, int ORDER>
static void launch_fixed(const fm_grid& g, T dx, int c, const StTerms<T>& terms, T* out, cudaStream_t s) {
  const Shape so = face_shape(g, c);
  if (g.dim == 3) {
    dim3 grid((so.s2 + kSK - 1) / kSK, (so.s1 + kSJ - 1) / kSJ, (so.s0 + kSI - 1) / kSI);
    if (terms.n == 3) {
      const size_t smem = StreamSmem<T, ORDER, 3>::bytes;
      static bool attr_set = false;  // per instantiation, set once
      if (!attr_set && smem > 48 * 1024) {
        cudaFuncSetAttribute(k_src_stream3<T, ORDER, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
      }
      launch(k_src_stream3<T, ORDER, 3>, grid, kSThreads, smem, s, g, dx, c, terms, out);
    } else {
      const size_t smem = StreamSmem<T, ORDER, 1>::bytes;
      static bool attr_set = false;
      if (!attr_set && smem > 48 * 1024) {
        cudaFuncSetAttribute(k_src_stream3<T, ORDER, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
      }
      launch(k_src_stream3<T, ORDER, 1>, grid, kSThreads, smem, s, g, dx, c, terms, out);
    }
  } else {
    dim3 grid((so.s1 + kTJ2 - 1) / kTJ2, (so.s0 + kTI2 - 1) / kTI2, 1);
    launch(k_fixed_grad_dot2<T, ORDER>, grid, kStThreads, 0, s, g, dx, c, terms, out);
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
