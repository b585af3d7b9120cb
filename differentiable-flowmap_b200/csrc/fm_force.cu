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
// with e = exp(-q), f = e s_c and a the adjoint velocity.
//
// Inclusion is decided exactly as the reference rounds it: s2 = sum (X - c)^2
// (left to right, no FMA contraction), d = sqrt(s2), q = (d d) r, q < 5.
// Off the boundary (s2 r outside 5 (1 -+ 1e-4)) the decision cannot depend on
// the rounding of d d and is taken without the square root (against
// 5 (1 -+ 1e-4) / r - s2_other, for the faces of a column).  The weight uses
// the Gaussian's separability, exp(-r s2) = exp(-r s2_other) exp(-r dz^2),
// which differs from exp(-q) by a few ulps.
//
// B200 mapping.  3000 Gaussians against every face is compute work.  Both
// kernels give each thread a column of faces along the fastest axis (k in 3D,
// j in 2D), tabulate per Gaussian the squared offsets and the factors
// exp(-r dx_a^2) in shared memory (every axis in the force kernel, the column
// axis in the adjoint), and combine the other axes once per (column,
// Gaussian); a face then costs two shared loads, a compare and an FMA.
//  * k_gauss_force: one CTA per tile of cells (16x16 in 2D, 8x8x8 in 3D).  The
//    CTA walks the Gaussians in chunks of 256 and appends those whose support
//    ball (radius sqrt(5/r), widened) reaches the tile's box to a list in
//    shared memory, in ascending order (ballot + popc prefix); once the list
//    could not take another chunk, or at the end, it tabulates the listed
//    Gaussians a sub-chunk at a time and every thread accumulates its column
//    segment over them in list order.  The cull is a superset of the exact test.
//  * k_gauss_grad: one CTA per Gaussian over the columns of its support box;
//    each column's faces are summed in registers of the run's type and
//    flushed to FP64 per column; fixed-order warp-shuffle + shared-memory
//    reduction, so the result is deterministic (the reference's atomics are
//    not).  Gaussians with r <= 0 or a support wider than the table take a
//    per-face path in the reference's operation order.
#include <math.h>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

constexpr int kGfThreads = 256;
constexpr int kGfWarps = kGfThreads / 32;
constexpr int kGfMaxN = 1 << 24;
constexpr int kGfTab = 256;   // column-table capacity of the adjoint kernel (faces)

// Tiles of the force kernel; the column axis is D-1.  SEG: faces per thread
// along it (one segment per thread: 3D 9*8 + 8*9 + 8*8 = 208, 2D 17*4 + 16*5 = 148).
template <int D> struct GfTile;
template <> struct GfTile<2> { static constexpr int B0 = 16, B1 = 16, B2 = 1, BC = 16, SEG = 4; };
template <> struct GfTile<3> { static constexpr int B0 = 8, B1 = 8, B2 = 8, BC = 8, SEG = 9; };

// Relative widening of the support radius used by the culls and by the
// square-root-free decisions; far above the few ulps by which the rounding of
// the exact test can move the boundary.
constexpr double kGfMargin = 1e-4;

// Position of index i along an axis: face grids at i dx on their own axis,
// (i + 1/2) dx elsewhere (node_pos, 3D/taichi_utils.py:95-128).
template <typename T>
__device__ __forceinline__ T gf_pos(int i, bool face, T dx) {
  T f = (T)i;
  if (!face) f = f + (T)0.5;
  return f * dx;
}

// Inclusion of a face with squared distance s2 (rounded as the reference
// rounds it) for inverse radius r.
template <typename T>
__device__ __forceinline__ bool gf_inside(T s2, T r) {
  const T t = rn_mul(s2, r);
  if (t < (T)(5.0 * (1.0 - kGfMargin))) return true;   // r <= 0 lands here too
  if (t > (T)(5.0 * (1.0 + kGfMargin))) return false;
  const T d = sqrt(s2);                                   // near the boundary: the exact test
  return rn_mul(rn_mul(d, d), r) < (T)5;                  // NaN excluded
}

// The per-face path: exact test and weight at one face.
template <typename T, int D>
__device__ __forceinline__ bool gf_weight(const T* p, const T* c, T r, T* dp, T& e) {
#pragma unroll
  for (int a = 0; a < D; ++a) dp[a] = rn_sub(p[a], c[a]);
  T s2 = rn_mul(dp[0], dp[0]);
#pragma unroll
  for (int a = 1; a < D; ++a) s2 = rn_add(s2, rn_mul(dp[a], dp[a]));
  if (!gf_inside(s2, r)) return false;
  e = exp(-rn_mul(s2, r));
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
  constexpr int CA = D - 1, SEG = Tl::SEG;
  constexpr int BM = (Tl::B0 > Tl::BC ? Tl::B0 : Tl::BC) + 1;        // table entries per axis and variant
  constexpr int SUB = sizeof(T) == 4 ? 64 : 32;                       // Gaussians tabulated at a time
  constexpr int TS = D * 2 * BM;                                      // table entries per Gaussian
  constexpr int CAP = sizeof(T) == 4 ? 2 * kGfThreads : kGfThreads;  // culled-list capacity
  __shared__ T s_c[D][CAP], s_s[D][CAP], s_r[CAP];
  // per tabulated Gaussian l, axis a, variant v (0 cell, 1 face), index q - lo[a]:
  // squared offset and exp(-r offset^2)
  __shared__ T t_sq[SUB][D][2][BM], t_ex[SUB][D][2][BM];
  __shared__ T t_lo[SUB], t_hi[SUB];  // 5 (1 -+ m) / r, or +inf for r <= 0
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

  // this thread's segment: component cc, tile-local other-axis indices io[],
  // tile-local column indices [k0, k0 + len)
  int cc = -1, io[2] = {0, 0}, k0 = 0, len = 0;
  {
    int q = threadIdx.x;
#pragma unroll
    for (int comp = 0; comp < D; ++comp) {
      if (cc < 0) {
        int e[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) e[a] = hc[a] + (comp == a && hc[a] == g.n[a]) - lo[a];
        const int nseg = (e[CA] + SEG - 1) / SEG;
        const int cnt = (D == 3 ? e[0] * e[1] : e[0]) * nseg;
        if (q < cnt) {
          cc = comp;
          const int sg = q % nseg, o = q / nseg;
          if (D == 3) {
            io[0] = o / e[1];
            io[1] = o % e[1];
          } else {
            io[0] = o;
          }
          k0 = sg * SEG;
          len = min(SEG, e[CA] - sg * SEG);
        } else {
          q -= cnt;
        }
      }
    }
  }
  const int v0 = cc == 0 ? 1 : 0, v1 = cc == 1 ? 1 : 0, vc = cc == CA ? 1 : 0;

  T acc[SEG];
#pragma unroll
  for (int m = 0; m < SEG; ++m) acc[m] = (T)0;

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int listed = 0;  // culled Gaussians waiting in the list (uniform across the CTA)
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
    int off = 0, got = 0;
#pragma unroll
    for (int k = 0; k < kGfWarps; ++k) {
      const int v = s_cnt[k];
      off += k < w ? v : 0;
      got += v;
    }
    if (hit) {  // appended in ascending order after the Gaussians already listed
      const int slot = listed + off + __popc(m & ((1u << lane) - 1u));
#pragma unroll
      for (int a = 0; a < D; ++a) {
        s_c[a][slot] = c[a];
        s_s[a][slot] = s[a];
      }
      s_r[slot] = r;
    }
    __syncthreads();
    listed += got;
    // evaluate once the list could not take another chunk, or at the end
    if (listed > CAP - kGfThreads || base + kGfThreads >= n) {
      const int tot = listed;
      listed = 0;
      for (int sub = 0; sub < tot; sub += SUB) {
        const int cnt = min(SUB, tot - sub);
        for (int x = threadIdx.x; x < cnt * TS; x += kGfThreads) {
          const int l = x / TS, rem = x - l * TS, a = rem / (2 * BM), rv = rem - a * 2 * BM, v = rv / BM,
                    q = rv - v * BM;
          const T rr = s_r[sub + l];
          const T d = rn_sub(gf_pos<T>(lo[a] + q, v == 1, dx), s_c[a][sub + l]);
          const T sq = rn_mul(d, d);
          t_sq[l][a][v][q] = sq;
          t_ex[l][a][v][q] = exp(-rn_mul(sq, rr));
          if (rem == 0) {
            const bool pos = rr > (T)0;
            t_lo[l] = pos ? (T)(5.0 * (1.0 - kGfMargin)) / rr : (T)INFINITY;
            t_hi[l] = pos ? (T)(5.0 * (1.0 + kGfMargin)) / rr : (T)INFINITY;
          }
        }
        __syncthreads();
        if (cc >= 0) {
          for (int l = 0; l < cnt; ++l) {
            // the other axes once per (column, Gaussian)
            T sxy = t_sq[l][0][v0][io[0]], exy = t_ex[l][0][v0][io[0]];
            if (D == 3) {
              sxy = rn_add(sxy, t_sq[l][1][v1][io[1]]);
              exy = exy * t_ex[l][1][v1][io[1]];
            }
            // dz^2 < A: inside off the boundary; dz^2 > B: outside; between: the exact test
            const T B = t_hi[l] - sxy;
            if (B < (T)0) continue;  // the column misses the support
            const T A = t_lo[l] - sxy, rr = s_r[sub + l];
            const T ev = exy * s_s[cc][sub + l];
#pragma unroll
            for (int q = 0; q < SEG; ++q) {
              if (q < len) {
                const T sq = t_sq[l][CA][vc][k0 + q];
                bool in = sq < A;
                if (!in && sq <= B) {
                  const T d = sqrt(rn_add(sxy, sq));
                  in = rn_mul(rn_mul(d, d), rr) < (T)5;
                }
                if (in) acc[q] += ev * t_ex[l][CA][vc][k0 + q];
              }
            }
          }
        }
        __syncthreads();  // the next tables / list entries overwrite what was read
      }
    }
  }

  if (cc >= 0) {
    const Shape fs = face_shape(g, cc);
    T* const o = cc == 0 ? f0 : (cc == 1 ? f1 : f2);
    const long b = D == 3 ? fs.idx(lo[0] + io[0], lo[1] + io[1], lo[2] + k0) : fs.idx(lo[0] + io[0], lo[1] + k0, 0);
    const long st = D == 3 ? 1 : fs.s2;  // the column axis is contiguous (3D: k; 2D: j with s2 == 1)
#pragma unroll
    for (int q = 0; q < SEG; ++q)
      if (q < len) o[b + q * st] = acc[q];
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

// Per-Gaussian sums v[c] adj_strength, v[D+a] adj_center, v[2D+c]
// pen_strength, v[3D+a] pen_center (FP64).
template <typename T, int D>
__global__ void __launch_bounds__(kGfThreads, 4) k_gauss_grad(fm_grid g, T dx, const T* __restrict__ cen,
                                                              const T* __restrict__ ir, const T* __restrict__ str,
                                                              const T* __restrict__ a0, const T* __restrict__ a1,
                                                              const T* __restrict__ a2, double* __restrict__ adj_c,
                                                              double* __restrict__ adj_s, double* __restrict__ pen_c,
                                                              double* __restrict__ pen_s) {
  constexpr int NV = 4 * D;
  constexpr int CA = D - 1;
  __shared__ double s_red[kGfWarps][NV];
  __shared__ T t_dp[kGfTab], t_ex[kGfTab];
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
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;

  if (!none) {
#pragma unroll
    for (int cc = 0; cc < D; ++cc) {
      const Shape fs = face_shape(g, cc);
      const T* const adj = cc == 0 ? a0 : (cc == 1 ? a1 : a2);
      int i0[3] = {0, 0, 0}, i1[3] = {0, 0, 0};
#pragma unroll
      for (int a = 0; a < D; ++a) gf_axis_range((double)c[a], R, (double)dx, a == cc, axis_len(fs, a), i0[a], i1[a]);
      const int e0 = i1[0] - i0[0] + 1, e1 = i1[1] - i0[1] + 1, e2 = i1[2] - i0[2] + 1;
      if (e0 <= 0 || e1 <= 0 || e2 <= 0) continue;
      const int ecol = CA == 2 ? e2 : e1;
      const T sc = s[cc];
      if (r > (T)0 && ecol <= kGfTab) {
        // column path: the column axis tabulated, the other axes per column
        __syncthreads();  // the previous component's columns are done with the table
        for (int q = threadIdx.x; q < ecol; q += kGfThreads) {
          const T dz = rn_sub(gf_pos<T>(i0[CA] + q, cc == CA, dx), c[CA]);
          t_dp[q] = dz;
          t_ex[q] = exp(-rn_mul(rn_mul(dz, dz), r));
        }
        __syncthreads();
        const double k1 = 2.0 * (double)sc * (double)r, k2 = 4.0 * (double)sc * (double)sc * (double)r,
                     k3 = 2.0 * (double)sc;
        const double rcap = 5.0 * (1.0 + kGfMargin) / (double)r, off = cc == CA ? 0.0 : 0.5;
        const T tlo = (T)(5.0 * (1.0 - kGfMargin)) / r, thi = (T)(5.0 * (1.0 + kGfMargin)) / r;
        const int ncol = D == 3 ? e0 * e1 : e0;
        for (int col = threadIdx.x; col < ncol; col += kGfThreads) {
          int io[2] = {0, 0};
          if (D == 3) {
            io[0] = i0[0] + col / e1;
            io[1] = i0[1] + col % e1;
          } else {
            io[0] = i0[0] + col;
          }
          T dpo[2] = {(T)0, (T)0}, sxy = (T)0;
#pragma unroll
          for (int a = 0; a < CA; ++a) {
            dpo[a] = rn_sub(gf_pos<T>(io[a], a == cc, dx), c[a]);
            sxy = a == 0 ? rn_mul(dpo[a], dpo[a]) : rn_add(sxy, rn_mul(dpo[a], dpo[a]));
          }
          // dz^2 < A: inside off the boundary; dz^2 > B: outside; between: the exact test
          const T A = tlo - sxy, B = thi - sxy;
          if (B < (T)0) continue;  // the column misses the support
          // the column's included faces lie within |dz| <= sqrt(5 (1 + m) / r - sxy)
          const double half = sqrt(fmax(rcap - (double)sxy, 0.0)) + 0.01 * (double)dx;
          const int qa = max(0, (int)ceil(((double)c[CA] - half) / (double)dx - off) - 1 - i0[CA]);
          const int qb = min(ecol - 1, (int)floor(((double)c[CA] + half) / (double)dx - off) + 1 - i0[CA]);
          const T exy = exp(-rn_mul(sxy, r));
          // the column axis is contiguous in memory (3D: k; 2D: j, where s2 == 1)
          const T* row = adj + (D == 3 ? fs.idx(io[0], io[1], i0[2]) : fs.idx(io[0], i0[1], 0));
          T sea = (T)0, seaz = (T)0, se2 = (T)0, se2z = (T)0;
          // straight-line body (weights selected to 0 outside): the loads pipeline
#pragma unroll 4
          for (int q = qa; q <= qb; ++q) {
            const T dz = t_dp[q], sq = rn_mul(dz, dz);
            bool in = sq < A;
            if (!in && sq <= B) {  // rare: a face within the margin of the cutoff
              const T d = sqrt(rn_add(sxy, sq));
              in = rn_mul(rn_mul(d, d), r) < (T)5;
            }
            const T e = exy * t_ex[q], av = __ldg(row + q);
            const T ea = in ? e * av : (T)0, e2 = in ? e * e : (T)0;  // selects: a NaN outside stays out
            sea += ea;
            seaz += ea * dz;
            se2 += e2;
            se2z += e2 * dz;
          }
          v[cc] += (double)sea;
          v[2 * D + cc] += k3 * (double)se2;
#pragma unroll
          for (int a = 0; a < CA; ++a) {
            v[D + a] += k1 * (double)dpo[a] * (double)sea;
            v[3 * D + a] += k2 * (double)dpo[a] * (double)se2;
          }
          v[D + CA] += k1 * (double)seaz;
          v[3 * D + CA] += k2 * (double)se2z;
        }
      } else {
        // per-face path (r <= 0, or a support wider than the table), in the
        // reference's operation order per face
        const unsigned cnt = (unsigned)e0 * (unsigned)e1 * (unsigned)e2;  // < 2^32 (validate_grid)
        for (unsigned q = threadIdx.x; q < cnt; q += kGfThreads) {
          const unsigned ij = q / (unsigned)e2;
          const int k = (int)(q - ij * (unsigned)e2);
          const unsigned ii = ij / (unsigned)e1;
          const int j = (int)(ij - ii * (unsigned)e1), i = (int)ii;
          T p[D], dp[D], e;
          node_pos<T, D>(cc, i0[0] + i, i0[1] + j, i0[2] + k, dx, p);
          if (!gf_weight<T, D>(p, c, r, dp, e)) continue;
          const T av = adj[fs.idx(i0[0] + i, i0[1] + j, i0[2] + k)];
          const T f = rn_mul(e, sc);
          v[cc] += (double)rn_mul(e, av);
          v[2 * D + cc] += (double)rn_mul(rn_mul((T)2, f), e);
          const T ga = rn_mul(rn_mul(sc, e), (T)2);
          const T gp = rn_mul(rn_mul(rn_mul(rn_mul((T)2, f), sc), e), (T)2);
#pragma unroll
          for (int a = 0; a < D; ++a) {
            v[D + a] += (double)rn_mul(rn_mul(rn_mul(ga, dp[a]), r), av);
            v[3 * D + a] += (double)rn_mul(rn_mul(gp, dp[a]), r);
          }
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
