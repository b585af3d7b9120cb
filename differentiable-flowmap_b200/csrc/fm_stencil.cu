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

// 2D tile: TI x TJ output nodes (j contiguous)
constexpr int kTI2 = 12, kTJ2 = 64;
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
__global__ void __launch_bounds__(kStThreads) k_fixed_grad_dot2(fm_grid g, T dx, int c, StTerms<T> terms,
                                                                  T* __restrict__ out) {
  constexpr int NZ = Taps<ORDER>::nz;
  constexpr int TI = kTI2, TJ = kTJ2;
  constexpr int FI = TI + NZ + 2, FJ = TJ + NZ + 2;  // one tap of margin on each side (see below)
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
    const int li = bI[0] - 1, lj = bJ[0] - 1;
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
// (j, k) and an i-chunk of kSI outputs.  For each term it walks the input
// planes the chunk needs: the plane's (j, k) footprint of the term's two fields
// is staged in shared memory (the next plane's values are already loaded into
// registers while this one is contracted), contracted along k (a sliding
// register window where the tile's stencils advance one tap per node) and then
// along j; the last NZ+1 contracted planes stay in registers, and an output
// node takes its term from them by the i contraction as soon as its last plane
// has been read, accumulating the terms in shared memory.  Each input value is
// read from memory once per i-chunk (plus the chunk's halo planes).  Stencil
// tables, the clamp band and sample()'s index clamp are the reference's; only
// the summation order differs from the gather form.
//
// Footprint widths: a stencil's first tap is floor(node position / dx - BL)
// plus a constant; with a dx that is not a power of two the quotient carries a
// rounding error, so over a tile of n nodes the first taps spread over up to n
// (not n - 1) cells: the footprints hold n + NZ values.
// ---------------------------------------------------------------------------
constexpr int kSJ = 16, kSK = 32, kSI = 4;
constexpr int kSThreads = 256;  // 32 k-lanes x 8 j-pairs

template <typename T, int ORDER>
struct StreamSmem {
  static constexpr int NZ = Taps<ORDER>::nz;
  static constexpr int FJ = kSJ + NZ + 2, FK = kSK + NZ + 2;  // one tap of margin on each side
  static constexpr int ROWS = 2 * FJ;                          // footprint rows of the two fields
  static constexpr int RPW = (ROWS + kSThreads / 32 - 1) / (kSThreads / 32);  // rows per warp
  static constexpr size_t plane = (size_t)ROWS * FK;           // [f][jj][kk]
  static constexpr size_t kpass = (size_t)ROWS * kSK;          // [f][jj][k]
  static constexpr size_t outs = (size_t)kSI * kSJ * kSK;      // the chunk's outputs
  static constexpr size_t bytes = sizeof(T) * (plane + kpass + outs);
};

template <typename T, int ORDER, int NT>
__global__ void __launch_bounds__(kSThreads, 3) k_src_stream3(fm_grid g, T dx, int c, StTerms<T> terms,
                                                           T* __restrict__ out) {
  using SM = StreamSmem<T, ORDER>;
  constexpr int NZ = SM::NZ, FJ = SM::FJ, FK = SM::FK, NR = NZ + 1, RPW = SM::RPW;
  extern __shared__ __align__(16) unsigned char ss_raw[];
  T* sP = reinterpret_cast<T*>(ss_raw);
  T* sA = sP + SM::plane;
  T* sO = sA + SM::kpass;
  __shared__ int bI[NT][kSI], bJ[NT][kSJ], bK[NT][kSK];
  __shared__ T wI[NT][2][kSI][NZ], wJ[NT][2][kSJ][NZ], wK[NT][2][kSK][NZ];
  __shared__ int fastJ[NT], fastK[NT];

  const Shape so = face_shape(g, c);
  const int i0 = blockIdx.z * kSI, j0 = blockIdx.y * kSJ, k0 = blockIdx.x * kSK;
  const int iend = min(i0 + kSI, so.s0);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int ja = 2 * ty;  // this thread's output nodes: (j0 + ja + m, k0 + tx), m = 0, 1
  const T inv_dx = (T)1 / dx;

  // per-term axis tables: first tap and weights of every node of the tile and
  // chunk (field f: derivative weights along the output face axis c, value
  // weights elsewhere; field h: value weights)
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
  for (int e = threadIdx.x; e < kSI * kSJ * kSK; e += blockDim.x) sO[e] = (T)0;
  __syncthreads();
  // fast paths: the stencils of the whole tile advance one tap per node (no clamp
  // band, no rounding step inside the tile), so all its nodes share one weight set
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

  for (int a = 0; a < NT; ++a) {
    const StTerm<T> tm = pick_term(terms, a);
    int pmin = bI[a][0], pmax = bI[a][0];
    for (int q = 1; q < iend - i0; ++q) {
      pmin = min(pmin, bI[a][q]);
      pmax = max(pmax, bI[a][q]);
    }
    pmax += NZ - 1;
    const int lj = bJ[a][0] - 1, lk = bK[a][0] - 1;
    // this lane's footprint columns (sample()'s index clamp) and rows
    const int gk0 = clampi(lk + tx, 0, tm.s2 - 1), gk1 = clampi(lk + tx + 32, 0, tm.s2 - 1);
    const bool col1 = tx + 32 < FK;
    auto load_plane = [&](int p, T (&v)[RPW][2]) {
      const long gi = clampi(p, 0, tm.s0 - 1);
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        const int row = ty + q * (kSThreads / 32);
        if (row < SM::ROWS) {
          const int f = row / FJ, jj = row % FJ;
          const T* src = f == 0 ? tm.f : tm.h;
          const long rb = (gi * tm.s1 + clampi(lj + jj, 0, tm.s1 - 1)) * tm.s2;
          v[q][0] = ldg(src + rb + gk0);
          if (col1) v[q][1] = ldg(src + rb + gk1);
        }
      }
    };
    T nxt[RPW][2];
    load_plane(pmin, nxt);
    T ring[2][2][NR];  // [field][node m][plane p - slot]
#pragma unroll
    for (int f = 0; f < 2; ++f)
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int q = 0; q < NR; ++q) ring[f][m][q] = (T)0;
    int inext = i0;
    for (int p = pmin; p <= pmax; ++p) {
      // 1. stage plane p; start loading plane p + 1
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        const int row = ty + q * (kSThreads / 32);
        if (row < SM::ROWS) {
          sP[row * FK + tx] = nxt[q][0];
          if (col1) sP[row * FK + tx + 32] = nxt[q][1];
        }
      }
      __syncthreads();
      if (p < pmax) load_plane(p + 1, nxt);
      // 2. k pass: segments of 4 outputs of one row
      for (int task = threadIdx.x; task < SM::ROWS * (kSK / 4); task += kSThreads) {
        const int row = task / (kSK / 4), seg = task % (kSK / 4);
        const int f = row / FJ;
        const T* src = sP + row * FK;
        T* dst = sA + row * kSK + seg * 4;
        const int kb = seg * 4;
        if (fastK[a]) {
          T v[NZ + 3], w[NZ];
#pragma unroll
          for (int q = 0; q < NZ + 3; ++q) v[q] = src[kb + 1 + q];
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
            const int o = bK[a][kb + m] - lk;
            T acc = 0;
#pragma unroll
            for (int t = 0; t < NZ; ++t) acc += src[o + t] * wK[a][f][kb + m][t];
            dst[m] = acc;
          }
        }
      }
      __syncthreads();
      // 3. j pass for this thread's two nodes, into the ring
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const T* col = sA + f * FJ * kSK + tx;
        T r0 = 0, r1 = 0;
        if (fastJ[a]) {
          T v[NZ + 1];
#pragma unroll
          for (int q = 0; q < NZ + 1; ++q) v[q] = col[(ja + 1 + q) * kSK];
#pragma unroll
          for (int t = 0; t < NZ; ++t) {
            const T w = wJ[a][f][ja][t];
            r0 += v[t] * w;
            r1 += v[t + 1] * w;
          }
        } else {
          const int o0 = bJ[a][ja] - lj, o1 = bJ[a][ja + 1] - lj;
#pragma unroll
          for (int t = 0; t < NZ; ++t) {
            r0 += col[(o0 + t) * kSK] * wJ[a][f][ja][t];
            r1 += col[(o1 + t) * kSK] * wJ[a][f][ja + 1][t];
          }
        }
#pragma unroll
        for (int q = NR - 1; q > 0; --q) {
          ring[f][0][q] = ring[f][0][q - 1];
          ring[f][1][q] = ring[f][1][q - 1];
        }
        ring[f][0][0] = r0;
        ring[f][1][0] = r1;
      }
      // 4. this term of every output whose last plane is p (or p - 1 where the
      // first taps step back by one: plane bI + t then sits at ring slot
      // d + NZ - 1 - t with d = p - (bI + NZ - 1))
      while (inext < iend && bI[a][inext - i0] + NZ - 1 <= p) {
        const int li = inext - i0;
        const bool d = bI[a][li] + NZ - 1 < p;
        T gf0 = 0, gf1 = 0, hh0 = 0, hh1 = 0;
#pragma unroll
        for (int t = 0; t < NZ; ++t) {
          const T wf = wI[a][0][li][t], wh = wI[a][1][li][t];
          const int sl = NZ - 1 - t;
          gf0 += (d ? ring[0][0][sl + 1] : ring[0][0][sl]) * wf;
          gf1 += (d ? ring[0][1][sl + 1] : ring[0][1][sl]) * wf;
          hh0 += (d ? ring[1][0][sl + 1] : ring[1][0][sl]) * wh;
          hh1 += (d ? ring[1][1][sl + 1] : ring[1][1][sl]) * wh;
        }
        T* o = sO + (li * kSJ + ja) * kSK + tx;
        o[0] += (gf0 * inv_dx) * hh0;
        o[kSK] += (gf1 * inv_dx) * hh1;
        ++inext;
      }
      __syncthreads();
    }
  }
  // write the chunk's outputs (each thread its own nodes: no barrier needed)
  for (int li = 0; li < iend - i0; ++li) {
    const int k = k0 + tx;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int j = j0 + ja + m;
      if (k < so.s2 && j < so.s1) out[so.idx(i0 + li, j, k)] = sO[(li * kSJ + ja + m) * kSK + tx];
    }
  }
}

template <typename T, int ORDER>
static void launch_fixed(const fm_grid& g, T dx, int c, const StTerms<T>& terms, T* out, cudaStream_t s) {
  const Shape so = face_shape(g, c);
  if (g.dim == 3) {
    dim3 grid((so.s2 + kSK - 1) / kSK, (so.s1 + kSJ - 1) / kSJ, (so.s0 + kSI - 1) / kSI);
    // dynamic plus static shared memory exceeds the default 48 KB window: the
    // dynamic limit is raised whatever the dynamic part alone needs
    const size_t smem = StreamSmem<T, ORDER>::bytes;
    if (terms.n == 3) {
      if (!raise_smem_limit(k_src_stream3<T, ORDER, 3>, smem)) return;
      launch(k_src_stream3<T, ORDER, 3>, grid, kSThreads, smem, s, g, dx, c, terms, out);
    } else {
      if (!raise_smem_limit(k_src_stream3<T, ORDER, 1>, smem)) return;
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
