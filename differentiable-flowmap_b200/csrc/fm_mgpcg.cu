// fm_mgpcg.cu -- MGPCG pressure projection for sm_100a.
//
// Restates the reference solver (3D/mgpcg.py:12-439; 2D/vortex/mgpcg_solid.py
// with an empty obstacle mask): all-Neumann 5/7-point Laplacian, red-black
// Gauss-Seidel V-cycle (2 pre + 2 post sweeps, piecewise-constant prolongation,
// restriction summing fine residuals into I//2 scaled 1/(dim-1), bottom RBGS),
// recentring of r, PCG with absolute (and optional relative) rTr tolerance.
//
// B200 design:
//  * alpha/beta/convergence live on the device (FP64), so an iteration issues
//    no host read; the host only polls the `done` word every check_every
//    iterations (the reference syncs three times per iteration).
//  * inner products use fixed-grid block partials reduced in a fixed order
//    (deterministic, FP64 accumulation).
//  * restriction is a gather over the 2^dim children (no atomics, no zero-fill);
//    the first red sweep of every level fuses the zero-fill of z (and, on the
//    fine level, the recentring of r); the last fine sweep fuses z.r.
//  * the coarsest level is smoothed by one CTA in shared memory (the reference
//    issues 2*bottom launches there).
//  * one PCG iteration (~40 launches) is captured once into a CUDA graph.
#include <cuda_bf16.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

std::atomic<long long> g_launch_count{0};
std::atomic<int> g_last_cuda_error{0};
std::atomic<int> g_pdl{1};

constexpr int kRedBlocks = 148 * 4;  // fixed reduction grid: 4 CTAs per SM
constexpr int kRedThreads = 256;
constexpr int kMaxLevels = 16;
// single-CTA bottom solve: 512 threads x up to 8 cells each
constexpr int kBottomThreads = 512;
constexpr int kBottomCellsPerThread = 8;
constexpr int kBottomMaxCells = kBottomThreads * kBottomCellsPerThread;

struct DevState {
  double zTr_old, tol, rTr, alpha, beta, mean, pAp;
  int it;        // completed PCG iterations (reference `it`)
  int done;      // converged, max_iters reached or non-finite
  int conv;
  int nonfinite;
  int result_it;
  int max_it_seen;
  // cumulative over all solves since create / the last stats reset
  long long solves, iters_total, not_converged, nonfinite_count;
  long long bodies;  // while-loop bodies executed (device mode), for the launch count
  // outer defect correction (fm_mgpcg_solve_dc): mean of b, |b - mean|^2, |r|^2,
  // and an rTr floor for the inner solves (0 outside a defect correction)
  double dc_mean, dc_b2, dc_r2, dc_tol;
  // device-side defect correction (fm_project_dc): set once |r| <= rel_tol |b|;
  // every later correction, and the inner solves inside them, skip their work
  int dc_done;
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

template <int D>
__device__ __forceinline__ int parity(int i, int j, int k) {
  return (i + j + (D == 3 ? k : 0)) & 1;
}

// neighbor_sum / num_fluid_neighbors (3D/mgpcg.py:97-120), all-Neumann walls.
template <typename T, int D>
__device__ __forceinline__ T nb_sum(const T* __restrict__ x, const Shape& s, int i, int j, int k, T& diag) {
  T acc = 0;
  int nd = 2 * D;
  const long q = s.idx(i, j, k);
  if (i < s.s0 - 1) acc += x[q + (long)s.s1 * s.s2]; else --nd;
  if (i > 0) acc += x[q - (long)s.s1 * s.s2]; else --nd;
  if (j < s.s1 - 1) acc += x[q + s.s2]; else --nd;
  if (j > 0) acc += x[q - s.s2]; else --nd;
  if (D == 3) {
    if (k < s.s2 - 1) acc += x[q + 1]; else --nd;
    if (k > 0) acc += x[q - 1]; else --nd;
  }
  diag = (T)nd;
  return acc;
}

// Storage of MG levels: the compute type T, or BF16 for the levels between the
// finest and the cluster-resident ones when coarse_bf16 is set (FP32 solvers).
__device__ __forceinline__ float to_c(float v) { return v; }
__device__ __forceinline__ double to_c(double v) { return v; }
__device__ __forceinline__ float to_c(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename S, typename T>
__device__ __forceinline__ S to_s(T v) {
  if constexpr (std::is_same<S, __nv_bfloat16>::value) return __float2bfloat16_rn((float)v);
  else return (S)v;
}

// nb_sum over a stored level (values converted to the compute type T)
template <typename T, int D, typename S>
__device__ __forceinline__ T nb_sum_s(const S* __restrict__ x, const Shape& s, int i, int j, int k, T& diag) {
  T acc = 0;
  int nd = 2 * D;
  const long q = s.idx(i, j, k);
  if (i < s.s0 - 1) acc += (T)to_c(x[q + (long)s.s1 * s.s2]); else --nd;
  if (i > 0) acc += (T)to_c(x[q - (long)s.s1 * s.s2]); else --nd;
  if (j < s.s1 - 1) acc += (T)to_c(x[q + s.s2]); else --nd;
  if (j > 0) acc += (T)to_c(x[q - s.s2]); else --nd;
  if (D == 3) {
    if (k < s.s2 - 1) acc += (T)to_c(x[q + 1]); else --nd;
    if (k > 0) acc += (T)to_c(x[q - 1]); else --nd;
  }
  diag = (T)nd;
  return acc;
}

template <int D>
__device__ __forceinline__ int diag_of(const Shape& s, int i, int j, int k) {
  int nd = 2 * D;
  nd -= (i == 0) + (i == s.s0 - 1) + (j == 0) + (j == s.s1 - 1);
  if (D == 3) nd -= (k == 0) + (k == s.s2 - 1);
  return nd;
}

__device__ __forceinline__ void block_reduce2(double a, double b, double* out2) {
  __shared__ double sa[32], sb[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (w == 0) {
    a = lane < nw ? sa[lane] : 0.0;
    b = lane < nw ? sb[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (lane == 0) { out2[0] = a; out2[1] = b; }
  }
}

// Sum the fixed-grid partials in a fixed order (one CTA of 256 threads).
__device__ __forceinline__ void sum_partials(const double* __restrict__ part, double& a, double& b) {
  double x = 0, y = 0;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) { x += part[2 * i]; y += part[2 * i + 1]; }
  __shared__ double res[2];
  block_reduce2(x, y, res);
  __syncthreads();
  a = res[0];
  b = res[1];
}

#define FM_GRID_STRIDE(q, n) for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < (n); q += (long)gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------
// projection front/back end
// ---------------------------------------------------------------------------
// apply_bc + divergence + init(r = -div) + x = 0, with partial sums of r for
// the recentring (3D/mgpcg.py:368-399, :76-84, :179-185).
// Each thread takes kDivUnroll cells of its grid-stride sequence at a time and
// issues all their face loads before any store, so 6 x kDivUnroll loads are in
// flight (a plain grid-stride loop waits one memory latency per cell).  The
// hoisting is safe: the only faces written are domain-wall faces, and every
// cell that reads one replaces the loaded value by 0.  The per-thread sum runs
// over the same cells in the same order as the plain loop.
constexpr int kDivUnroll = 2;

template <typename T, int D>
__global__ void __launch_bounds__(kRedThreads, 4) k_div_bc(fm_grid g, MacW<T> u, T* __restrict__ r,
                                                           T* __restrict__ x, double* __restrict__ part) {
  pdl_begin();
  const Shape cs = cell_shape(g);
  const unsigned n = (unsigned)cs.size();  // every field has fewer than 2^32 entries
  const unsigned stride = gridDim.x * blockDim.x;
  unsigned fstep[3];  // face offset of the high face of a cell, per component
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const Shape fs = face_shape(g, c);
    fstep[c] = c == 0 ? (unsigned)fs.s1 * fs.s2 : (c == 1 ? (unsigned)fs.s2 : 1u);
  }
  double sum = 0;
  for (unsigned base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kDivUnroll * stride) {
    T vl[kDivUnroll][3], vr[kDivUnroll][3];
    unsigned qf[kDivUnroll][3];
    int I[kDivUnroll][3];
#pragma unroll
    for (int m = 0; m < kDivUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      unflatten(cs, q, I[m][0], I[m][1], I[m][2]);
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const Shape fs = face_shape(g, c);
        const unsigned ql = ((unsigned)I[m][0] * fs.s1 + I[m][1]) * fs.s2 + I[m][2];
        qf[m][c] = ql;
        vl[m][c] = u.c[c][ql];
        vr[m][c] = u.c[c][ql + fstep[c]];
      }
    }
#pragma unroll
    for (int m = 0; m < kDivUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      T acc = 0;
#pragma unroll
      for (int c = 0; c < D; ++c) {
        T a = vl[m][c], b = vr[m][c];
        if (I[m][c] == 0) { a = 0; u.c[c][qf[m][c]] = 0; }
        if (I[m][c] == axis_len(cs, c) - 1) { b = 0; u.c[c][qf[m][c] + fstep[c]] = 0; }
        if (c == 0) acc = b - a;
        else { acc = acc + b; acc = acc - a; }
      }
      const T bq = acc * (T)-1;
      r[q] = bq;
      x[q] = 0;
      sum += (double)bq;
    }
  }
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

// rhs given directly (fm_mgpcg_solve)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_load_rhs(long n, const T* __restrict__ b, T* __restrict__ r,
                                                          T* __restrict__ x, double* __restrict__ part) {
  pdl_begin();
  double sum = 0;
  FM_GRID_STRIDE(q, n) {
    const T v = b[q];
    r[q] = v;
    x[q] = 0;
    sum += (double)v;
  }
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

// ---------------------------------------------------------------------------
// outer defect correction in FP64 around FP32 MGPCG solves (fm_mgpcg_solve_dc)
// ---------------------------------------------------------------------------
template <typename TB>
__global__ void __launch_bounds__(kRedThreads) k_dc_sum(long n, const TB* __restrict__ b, double* __restrict__ part) {
  pdl_begin();
  double sum = 0;
  FM_GRID_STRIDE(q, n) sum += (double)b[q];
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

// which = 0: dc_mean = sum / n;  1: dc_b2 = dc_r2 = sum of squares;  2: dc_r2 = sum of squares
__global__ void k_dc_fin(DevState* st, const double* part, double n, int which) {
  pdl_begin();
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    if (which == 0) st->dc_mean = a / n;
    else {
      st->dc_r2 = b;
      if (which == 1) st->dc_b2 = b;
    }
  }
}

// work = (b - mean) - A x in FP64, partial sums of work^2 (second slot).
template <typename TB, int D>
__global__ void __launch_bounds__(kRedThreads) k_dc_residual(Shape s, const TB* __restrict__ b,
                                                             const double* __restrict__ x, double* __restrict__ work,
                                                             double* __restrict__ part, const DevState* st) {
  pdl_begin();
  const double mean = st->dc_mean;
  double acc = 0;
  FM_GRID_STRIDE(q, s.size()) {
    int i, j, k;
    unflatten(s, q, i, j, k);
    double diag;
    const double nb = nb_sum<double, D>(x, s, i, j, k, diag);
    const double r = ((double)b[q] - mean) - (diag * x[q] - nb);
    work[q] = r;
    acc += r * r;
  }
  block_reduce2(0.0, acc, part + 2 * blockIdx.x);
}

// Inner right-hand side r32 = work / |work| (unit norm keeps FP32 away from
// underflow as the residual shrinks), x32 = 0, partial sums of r32 for the
// recentring of the inner solve.
__global__ void __launch_bounds__(kRedThreads) k_dc_load(long n, const double* __restrict__ work,
                                                         float* __restrict__ r, float* __restrict__ x,
                                                         double* __restrict__ part, const DevState* st) {
  pdl_begin();
  const double inv = 1.0 / sqrt(st->dc_r2);
  double sum = 0;
  FM_GRID_STRIDE(q, n) {
    const float v = (float)(work[q] * inv);
    r[q] = v;
    x[q] = 0.f;
    sum += (double)v;
  }
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

// rTr floor of the next inner solve (unit-norm right-hand side): a correction
// only has to bring |r| down to rel_tol |b|, with a factor 2 margin; 0 clears it.
__global__ void k_dc_set_tol(DevState* st, double rel_tol, int clear) {
  pdl_begin();
  const double t = clear ? 0.0 : 0.5 * rel_tol * sqrt(st->dc_b2 / st->dc_r2);
  st->dc_tol = t * t;
}

// x += |r| * e
__global__ void k_dc_update(long n, double* __restrict__ x, const float* __restrict__ e, const DevState* st) {
  pdl_begin();
  const double s = sqrt(st->dc_r2);
  FM_GRID_STRIDE(q, n) x[q] += s * (double)e[q];
}

// fm_project_dc: b = -div(u) of the FP32 velocity formed in FP64 (apply_bc
// zeroes the wall faces, as k_div_bc does), x = 0, partial sums of b.
template <int D>
__global__ void __launch_bounds__(kRedThreads) k_dc_div(fm_grid g, MacW<float> u, double* __restrict__ b,
                                                        double* __restrict__ x, double* __restrict__ part) {
  pdl_begin();
  const Shape cs = cell_shape(g);
  double sum = 0;
  FM_GRID_STRIDE(q, cs.size()) {
    int I[3];
    unflatten(cs, q, I[0], I[1], I[2]);
    double acc = 0;
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const Shape fs = face_shape(g, c);
      const long step = c == 0 ? (long)fs.s1 * fs.s2 : (c == 1 ? (long)fs.s2 : 1);
      const long ql = fs.idx(I[0], I[1], I[2]);
      double a = (double)u.c[c][ql], bb = (double)u.c[c][ql + step];
      if (I[c] == 0) { a = 0; u.c[c][ql] = 0.f; }
      if (I[c] == axis_len(cs, c) - 1) { bb = 0; u.c[c][ql + step] = 0.f; }
      acc += bb - a;
    }
    b[q] = -acc;
    x[q] = 0;
    sum += -acc;
  }
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

// fm_project_dc: after a residual, |r|^2 (which = 1 also |b|^2) and the stop
// test |r| <= rel_tol |b|; nothing once the correction loop is done.
__global__ void k_dc_check(DevState* st, const double* part, double rel_tol, int which) {
  pdl_begin();
  if (st->dc_done) return;
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    st->dc_r2 = b;
    if (which == 1) st->dc_b2 = b;
    if (!isfinite(b)) { st->dc_done = 1; st->nonfinite_count += 1; }
    else if (st->dc_b2 == 0.0 || b <= rel_tol * rel_tol * st->dc_b2) st->dc_done = 1;
  }
}

// The correction-loop versions of k_dc_residual / k_dc_load / k_dc_set_tol /
// k_dc_update: each returns at once when the loop is done.
template <int D>
__global__ void __launch_bounds__(kRedThreads) k_dc_residual_g(Shape s, const double* __restrict__ b,
                                                               const double* __restrict__ x, double* __restrict__ w,
                                                               double* __restrict__ part, const DevState* st) {
  pdl_begin();
  if (st->dc_done) return;
  const double mean = st->dc_mean;
  double acc = 0;
  FM_GRID_STRIDE(q, s.size()) {
    int i, j, k;
    unflatten(s, q, i, j, k);
    double diag;
    const double nb = nb_sum<double, D>(x, s, i, j, k, diag);
    const double r = (b[q] - mean) - (diag * x[q] - nb);
    w[q] = r;
    acc += r * r;
  }
  block_reduce2(0.0, acc, part + 2 * blockIdx.x);
}

__global__ void __launch_bounds__(kRedThreads) k_dc_load_g(long n, const double* __restrict__ w,
                                                           float* __restrict__ r, float* __restrict__ x,
                                                           double* __restrict__ part, const DevState* st) {
  pdl_begin();
  if (st->dc_done) return;
  const double inv = 1.0 / sqrt(st->dc_r2);
  double sum = 0;
  FM_GRID_STRIDE(q, n) {
    const float v = (float)(w[q] * inv);
    r[q] = v;
    x[q] = 0.f;
    sum += (double)v;
  }
  block_reduce2(sum, 0.0, part + 2 * blockIdx.x);
}

__global__ void k_dc_set_tol_g(DevState* st, double rel_tol) {
  pdl_begin();
  if (st->dc_done) return;
  const double t = 0.5 * rel_tol * sqrt(st->dc_b2 / st->dc_r2);
  st->dc_tol = t * t;
}

__global__ void k_dc_update_g(long n, double* __restrict__ x, const float* __restrict__ e, const DevState* st) {
  pdl_begin();
  if (st->dc_done) return;
  const double sc = sqrt(st->dc_r2);
  FM_GRID_STRIDE(q, n) x[q] += sc * (double)e[q];
}

// u -= grad x in FP64, rounded to FP32 (apply_bc: wall faces zero)
template <int D>
__global__ void k_dc_subgrad(fm_grid g, const double* __restrict__ x, MacW<float> u) {
  pdl_begin();
  const int c = blockIdx.y;
  const Shape fs = face_shape(g, c);
  const Shape cs = cell_shape(g);
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= fs.size()) return;
  int I[3];
  unflatten(fs, q, I[0], I[1], I[2]);
  if (I[c] == 0 || I[c] == axis_len(cs, c)) { u.c[c][q] = 0.f; return; }
  const long pc = cs.idx(I[0], I[1], I[2]);
  const long step = c == 0 ? (long)cs.s1 * cs.s2 : (c == 1 ? cs.s2 : 1);
  u.c[c][q] = (float)((double)u.c[c][q] - (x[pc] - x[pc - step]));
}

// End of fm_project_dc: an unconverged loop counts as a not-converged solve;
// the state returns to plain solves (no floor, not done).
__global__ void k_dc_finish(DevState* st) {
  pdl_begin();
  if (!st->dc_done) st->not_converged += 1;
  st->dc_done = 0;
  st->dc_tol = 0.0;
}

// subtract_grad_p + apply_bc (3D/mgpcg.py:401-427)
template <typename T, int D>
__global__ void k_subgrad_bc(fm_grid g, const T* __restrict__ p, MacW<T> u) {
  pdl_begin();
  const int c = blockIdx.y;
  const Shape fs = face_shape(g, c);
  const Shape cs = cell_shape(g);
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= fs.size()) return;
  int I[3];
  unflatten(fs, q, I[0], I[1], I[2]);
  if (I[c] == 0 || I[c] == axis_len(cs, c)) { u.c[c][q] = 0; return; }
  const long pc = cs.idx(I[0], I[1], I[2]);
  const long step = c == 0 ? (long)cs.s1 * cs.s2 : (c == 1 ? cs.s2 : 1);
  u.c[c][q] -= p[pc] - p[pc - step];
}

// ---------------------------------------------------------------------------
// scalar finalizers (one CTA)
// ---------------------------------------------------------------------------
__global__ void k_fin_mean(DevState* st, const double* part, double n) {
  pdl_begin();
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    st->mean = a / n;
    st->done = st->dc_done;  // 0 outside fm_project_dc
    st->conv = 0; st->nonfinite = 0; st->it = 0; st->result_it = 0;
    st->beta = 0; st->alpha = 0;
  }
}

__global__ void k_fin_alpha(DevState* st, const double* part, double eps) {
  pdl_begin();
  if (st->done) return;
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    st->pAp = a;
    st->alpha = st->zTr_old / (a + eps);
  }
}

// Called by thread 0 when a solve ends: fold it into the cumulative counters.
__device__ __forceinline__ void finish_solve(DevState* st) {
  st->done = 1;
  st->result_it = st->it;
  st->solves += 1;
  st->iters_total += st->it;
  if (st->it > st->max_it_seen) st->max_it_seen = st->it;
  if (st->nonfinite) st->nonfinite_count += 1;
  else if (!st->conv) st->not_converged += 1;
}

__global__ void k_fin_conv(DevState* st, const double* part, double n) {
  pdl_begin();
  if (st->done) return;
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    st->rTr = a;
    st->mean = b / n;
    if (!isfinite(a)) { st->nonfinite = 1; finish_solve(st); }
    else if (a < st->tol) { st->conv = 1; finish_solve(st); }
  }
}

// Node before a while loop: skip the loop when the solve is already done at
// its start (an inner solve of a finished defect correction, a non-finite
// start), instead of running one body of early-returning kernels.
__global__ void k_loop_init(cudaGraphConditionalHandle h, const DevState* st) {
  cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

// Last node of the while-loop body: keep iterating until the solve is done.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, DevState* st) {
  pdl_begin();
  st->bodies += 1;
  cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

__global__ void k_fin_beta(DevState* st, const double* part, double eps, double abs_tol, double rel_tol,
                           int max_iters, int first) {
  pdl_begin();
  if (st->done) return;
  double a, b;
  sum_partials(part, a, b);
  if (threadIdx.x == 0) {
    if (first) {
      st->zTr_old = a;
      double tol = abs_tol;
      if (rel_tol > 0 && a * rel_tol > tol) tol = a * rel_tol;
      if (st->dc_tol > tol) tol = st->dc_tol;
      st->tol = tol;
      st->beta = 0;
      if (!isfinite(a)) { st->nonfinite = 1; finish_solve(st); }
      // z.r = 0 means r = 0 (the preconditioner is SPD on mean-zero fields): the
      // zero start is the solution.  Stopping here keeps alpha = 0 / (0 + eps)
      // from becoming NaN when eps = 0.
      else if (a == 0.0) { st->conv = 1; finish_solve(st); }
    } else {
      st->beta = a / (st->zTr_old + eps);
      st->zTr_old = a;
      st->it += 1;
      if (st->it >= max_iters) finish_solve(st);
    }
  }
}

// ---------------------------------------------------------------------------
// PCG vector kernels
// ---------------------------------------------------------------------------
// Neighbour values of cell (i, j, k) at 32-bit index q in the reference's
// summation order (+i, -i, +j, -j, +k, -k), 0 where the neighbour is outside.
// Summing all six (or four) from +0.0 gives the skipping sum bit for bit: a
// round-to-nearest sum that starts at +0.0 is never -0.0, so adding +0.0
// changes nothing.
template <typename T, int D>
__device__ __forceinline__ void nb_load(const T* x, const Shape& s, unsigned q, int i, int j, int k, T* v) {
  const unsigned si = (unsigned)s.s1 * s.s2, sj = s.s2;
  v[0] = i < s.s0 - 1 ? x[q + si] : (T)0;
  v[1] = i > 0 ? x[q - si] : (T)0;
  v[2] = j < s.s1 - 1 ? x[q + sj] : (T)0;
  v[3] = j > 0 ? x[q - sj] : (T)0;
  if (D == 3) {
    v[4] = k < s.s2 - 1 ? x[q + 1] : (T)0;
    v[5] = k > 0 ? x[q - 1] : (T)0;
  }
}
template <typename T, int D>
__device__ __forceinline__ T nb_add(const T* v) {
  T acc = 0;
#pragma unroll
  for (int m = 0; m < 2 * D; ++m) acc += v[m];
  return acc;
}

// The grid-stride vector kernels below take kVecUnroll cells of a thread's
// sequence at a time and issue all their loads before any store (memory-level
// parallelism); the per-thread partial sums keep the cell order of a plain
// grid-stride loop.
constexpr int kVecUnroll = 2;

template <typename T, int D>
__global__ void __launch_bounds__(kRedThreads) k_Ap_dot(Shape s, const T* __restrict__ p, T* __restrict__ Ap,
                                                        double* __restrict__ part, const DevState* st) {
  pdl_begin();
  if (st->done) return;
  const unsigned n = (unsigned)s.size(), stride = gridDim.x * blockDim.x;
  double acc = 0;
  for (unsigned base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kVecUnroll * stride) {
    T v[kVecUnroll][6], pv[kVecUnroll];
    int nd[kVecUnroll];
#pragma unroll
    for (int m = 0; m < kVecUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      int i, j, k;
      unflatten(s, q, i, j, k);
      nb_load<T, D>(p, s, q, i, j, k, v[m]);
      pv[m] = p[q];
      nd[m] = diag_of<D>(s, i, j, k);
    }
#pragma unroll
    for (int m = 0; m < kVecUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      const T a = rn_sub(rn_mul((T)nd[m], pv[m]), nb_add<T, D>(v[m]));
      Ap[q] = a;
      acc += (double)pv[m] * (double)a;
    }
  }
  block_reduce2(acc, 0.0, part + 2 * blockIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_update_xr(long n, T* __restrict__ x, T* __restrict__ r,
                                                           const T* __restrict__ p, const T* __restrict__ Ap,
                                                           double* __restrict__ part, const DevState* st) {
  pdl_begin();
  if (st->done) return;
  const T alpha = (T)st->alpha;
  double rr = 0, rs = 0;
  FM_GRID_STRIDE(q, n) {
    x[q] = rn_add(x[q], rn_mul(alpha, p[q]));
    const T rv = rn_sub(r[q], rn_mul(alpha, Ap[q]));
    r[q] = rv;
    rr += (double)rv * (double)rv;
    rs += (double)rv;
  }
  block_reduce2(rr, rs, part + 2 * blockIdx.x);
}

template <typename T>
__global__ void k_update_p(long n, T* __restrict__ p, const T* __restrict__ z, const DevState* st, int first) {
  pdl_begin();
  if (st->done) return;
  const T beta = (T)st->beta;
  FM_GRID_STRIDE(q, n) p[q] = first ? z[q] : rn_add(z[q], rn_mul(beta, p[q]));
}

// ---------------------------------------------------------------------------
// V-cycle kernels
// ---------------------------------------------------------------------------
// First red sweep from z == 0 (fuses z.fill(0)); optionally recentres r.
template <typename T, int D>
__global__ void k_smooth_first(Shape s, T* __restrict__ r, T* __restrict__ z, const DevState* st, int recenter) {
  pdl_begin();
  if (st->done) return;
  const T mean = recenter ? (T)st->mean : (T)0;
  FM_GRID_STRIDE(q, s.size()) {
    int i, j, k;
    unflatten(s, q, i, j, k);
    T rv = r[q];
    if (recenter) { rv = rv - mean; r[q] = rv; }
    z[q] = parity<D>(i, j, k) == 0 ? div_nd(rv, diag_of<D>(s, i, j, k)) : (T)0;
  }
}

// Pair-per-thread RBGS sweeps for the levels above the cluster kernel.  A
// thread owns cells (.., 2m) and (.., 2m+1) along the innermost axis (k in 3D,
// j in 2D), one red and one black, so every lane updates a cell in every
// half-sweep.  Launch: block (32, 8); 3D grid (pairs/32, n1/8, n0) over
// (pair, j, i), 2D grid (pairs/32, n0/8) over (pair, i).
constexpr int kPairBX = 32, kPairBY = 8;

template <int D>
__device__ __forceinline__ bool pair_coords(const Shape& s, int& i, int& j, int& k0) {
  const int m = blockIdx.x * kPairBX + threadIdx.x;
  if (D == 3) {
    i = blockIdx.z;
    j = blockIdx.y * kPairBY + threadIdx.y;
    k0 = 2 * m;
    return j < s.s1 && k0 < s.s2;
  }
  i = blockIdx.y * kPairBY + threadIdx.y;
  j = 2 * m;
  k0 = 0;
  return i < s.s0 && j < s.s1;
}

// Neighbour sum (reference order +i, -i, +j, -j, +k, -k) and neighbour count
// of cell (i, j, k) at 32-bit index q.
template <typename T, int D, typename S>
__device__ __forceinline__ T nb_sum32(const S* __restrict__ x, const Shape& s, unsigned q, int i, int j, int k,
                                      int& nd) {
  const unsigned si = (unsigned)s.s1 * s.s2, sj = s.s2;
  T acc = 0;
  nd = 0;
  if (i < s.s0 - 1) { acc += (T)to_c(x[q + si]); ++nd; }
  if (i > 0) { acc += (T)to_c(x[q - si]); ++nd; }
  if (j < s.s1 - 1) { acc += (T)to_c(x[q + sj]); ++nd; }
  if (j > 0) { acc += (T)to_c(x[q - sj]); ++nd; }
  if (D == 3) {
    if (k < s.s2 - 1) { acc += (T)to_c(x[q + 1]); ++nd; }
    if (k > 0) { acc += (T)to_c(x[q - 1]); ++nd; }
  }
  return acc;
}

// smooth(l, phase) over pairs: only the cell of colour `phase` is updated.
// S: storage type of the level (T, or BF16 with coarse_bf16).
template <typename T, int D, typename S = T>
__global__ void __launch_bounds__(kPairBX* kPairBY) k_smooth_pair(Shape s, const S* __restrict__ r, S* z, int phase,
                                                                 const DevState* st) {
  pdl_begin();
  if (st->done) return;
  int i, j, k;
  if (!pair_coords<D>(s, i, j, k)) return;
  // the colour-`phase` cell of the pair: parity(i, j, k0) is (i + j) & 1 in 3D, i & 1 in 2D
  const int shift = ((D == 3 ? i + j : i) + phase) & 1;
  if (D == 3) k += shift; else j += shift;
  if ((D == 3 ? k : j) >= (D == 3 ? s.s2 : s.s1)) return;
  const unsigned q = ((unsigned)i * s.s1 + j) * s.s2 + k;
  int nd;
  const T nb = nb_sum32<T, D, S>(z, s, q, i, j, k, nd);
  z[q] = to_s<S>(div_nd((T)to_c(r[q]) + nb, nd));
}

// First red sweep from z == 0 over pairs (fuses z.fill(0)); optionally recentres r.
template <typename T, int D, typename S = T>
__global__ void __launch_bounds__(kPairBX* kPairBY) k_smooth_first_pair(Shape s, S* __restrict__ r, S* __restrict__ z,
                                                                       const DevState* st, int recenter) {
  pdl_begin();
  if (st->done) return;
  int i, j, k;
  if (!pair_coords<D>(s, i, j, k)) return;
  const T mean = recenter ? (T)st->mean : (T)0;
  const int red_second = (D == 3 ? i + j : i) & 1;  // the pair's second cell is red
  const unsigned q0 = ((unsigned)i * s.s1 + j) * s.s2 + k;
  const bool has2 = (D == 3 ? k : j) + 1 < (D == 3 ? s.s2 : s.s1);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    if (c == 1 && !has2) break;
    const unsigned q = q0 + c;
    T rv = (T)to_c(r[q]);
    if (recenter) { rv = rv - mean; r[q] = to_s<S>(rv); }
    if (c == red_second) {
      const int ci = i, cj = D == 3 ? j : j + c, ck = D == 3 ? k + c : 0;
      z[q] = to_s<S>(div_nd(rv, diag_of<D>(s, ci, cj, ck)));
    } else {
      z[q] = to_s<S>((T)0);
    }
  }
}

// smooth(l, phase) (3D/mgpcg.py:170-177); with part != nullptr also z.r over all cells.
// A half-sweep reads only cells of the other colour and writes only cells of
// colour `phase`, so the hoisted loads never see a value written in this launch.
template <typename T, int D, bool DOT>
__global__ void __launch_bounds__(kRedThreads) k_smooth(Shape s, const T* __restrict__ r, T* z, int phase,
                                                        double* __restrict__ part, const DevState* st) {
  pdl_begin();
  if (st->done) return;
  const unsigned n = (unsigned)s.size(), stride = gridDim.x * blockDim.x;
  double acc = 0;
  for (unsigned base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kVecUnroll * stride) {
    T v[kVecUnroll][6], rv[kVecUnroll], zo[kVecUnroll];
    int nd[kVecUnroll];
    bool upd[kVecUnroll];
#pragma unroll
    for (int m = 0; m < kVecUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      int i, j, k;
      unflatten(s, q, i, j, k);
      upd[m] = parity<D>(i, j, k) == phase;
      rv[m] = r[q];
      if (upd[m]) {
        nb_load<T, D>(z, s, q, i, j, k, v[m]);
        nd[m] = diag_of<D>(s, i, j, k);
      } else {
        zo[m] = z[q];
      }
    }
#pragma unroll
    for (int m = 0; m < kVecUnroll; ++m) {
      const unsigned q = base + m * stride;
      if (q >= n) break;
      T zv;
      if (upd[m]) {
        zv = div_nd(rv[m] + nb_add<T, D>(v[m]), nd[m]);
        z[q] = zv;
      } else {
        zv = zo[m];
      }
      if (DOT) acc += (double)zv * (double)rv[m];
    }
  }
  if (DOT) block_reduce2(acc, 0.0, part + 2 * blockIdx.x);
}

// restrict(l) (3D/mgpcg.py:157-163) as a gather over the 2^D children.
// SF / SC: storage types of the fine and the coarse level.
template <typename T, int D, typename SF = T, typename SC = T>
__global__ void k_restrict(Shape sf, Shape sc, const SF* __restrict__ rf, const SF* __restrict__ zf,
                           SC* __restrict__ rc, const DevState* st) {
  pdl_begin();
  if (st->done) return;
  const T scale = (T)1.0 / (T)(D - 1.0);
  FM_GRID_STRIDE(q, sc.size()) {
    int I, J, K;
    unflatten(sc, q, I, J, K);
    T acc = 0;
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int dk = 0; dk < (D == 3 ? 2 : 1); ++dk) {
          const int i = 2 * I + di, j = 2 * J + dj, k = D == 3 ? 2 * K + dk : 0;
          const long f = sf.idx(i, j, k);
          T diag;
          const T nb = nb_sum_s<T, D, SF>(zf, sf, i, j, k, diag);
          const T res = rn_sub((T)to_c(rf[f]), rn_sub(rn_mul(diag, (T)to_c(zf[f])), nb));
          acc = rn_add(acc, rn_mul(res, scale));
        }
    rc[q] = to_s<SC>(acc);
  }
}

// prolongate(l) (3D/mgpcg.py:165-168)
template <typename T, int D, typename SF = T, typename SC = T>
__global__ void k_prolong(Shape sf, Shape sc, SF* __restrict__ zf, const SC* __restrict__ zc, const DevState* st) {
  pdl_begin();
  if (st->done) return;
  FM_GRID_STRIDE(q, sf.size()) {
    int i, j, k;
    unflatten(sf, q, i, j, k);
    zf[q] = to_s<SF>((T)to_c(zf[q]) + (T)to_c(zc[sc.idx(i >> 1, j >> 1, D == 3 ? (k >> 1) : 0)]));
  }
}

// Bottom smoothing on the coarsest level by one CTA in shared memory.
// z starts at zero (the reference zero-fills before restricting).
template <typename T, int D>
__global__ void k_bottom(Shape s, const T* __restrict__ r, T* __restrict__ z, int bottom, int mode,
                         const DevState* st) {
  pdl_begin();
  if (st->done) return;
  extern __shared__ unsigned char smem_raw[];
  T* zs = reinterpret_cast<T*>(smem_raw);
  T* rs = zs + s.size();
  const int n = (int)s.size();
  for (int q = threadIdx.x; q < n; q += blockDim.x) { zs[q] = 0; rs[q] = r[q]; }
  // per-thread cells (n <= kBottomMaxCells = 8 * blockDim): index, parity,
  // in-domain neighbour mask and diagonal computed once, outside the sweeps
  int cq[kBottomCellsPerThread], cinfo[kBottomCellsPerThread];
  const int si = s.s1 * s.s2, sj = s.s2;
#pragma unroll
  for (int m = 0; m < kBottomCellsPerThread; ++m) {
    const int q = threadIdx.x + m * blockDim.x;
    cq[m] = q;
    cinfo[m] = -1;
    if (q < n) {
      int i, j, k;
      unflatten(s, q, i, j, k);
      int mask = 0;
      mask |= (i < s.s0 - 1) << 0;
      mask |= (i > 0) << 1;
      mask |= (j < s.s1 - 1) << 2;
      mask |= (j > 0) << 3;
      if (D == 3) { mask |= (k < s.s2 - 1) << 4; mask |= (k > 0) << 5; }
      cinfo[m] = mask | (parity<D>(i, j, k) << 6);
    }
  }
  __syncthreads();
  auto sweep = [&](int phase) {
#pragma unroll
    for (int m = 0; m < kBottomCellsPerThread; ++m) {
      const int info = cinfo[m];
      if (info >= 0 && (info >> 6) == phase) {
        const int q = cq[m];
        T nb = 0;
        if (info & 1) nb += zs[q + si];
        if (info & 2) nb += zs[q - si];
        if (info & 4) nb += zs[q + sj];
        if (info & 8) nb += zs[q - sj];
        if (D == 3) {
          if (info & 16) nb += zs[q + 1];
          if (info & 32) nb += zs[q - 1];
        }
        zs[q] = div_nd(rs[q] + nb, __popc(info & 63));
      }
    }
    __syncthreads();
  };
  if (mode == 0) {
    for (int it = 0; it < bottom; ++it) { sweep(0); sweep(1); }
  } else {
    for (int it = 0; it < bottom / 2; ++it) { sweep(0); sweep(1); }
    for (int it = 0; it < bottom / 2; ++it) { sweep(1); sweep(0); }
  }
  for (long q = threadIdx.x; q < n; q += blockDim.x) z[q] = zs[q];
}

template <typename T, int D>
__global__ void k_laplacian(Shape s, const T* __restrict__ p, T* __restrict__ Ap) {
  pdl_begin();
  FM_GRID_STRIDE(q, s.size()) {
    int i, j, k;
    unflatten(s, q, i, j, k);
    T diag;
    const T nb = nb_sum<T, D>(p, s, i, j, k, diag);
    Ap[q] = rn_sub(rn_mul(diag, p[q]), nb);
  }
}

}  // namespace fm

#include "fm_mg_cluster.cuh"

using namespace fm;

struct fm_mgpcg {
  fm_grid g;
  int dtype;
  fm_mg_params P;
  int L;
  Shape lv[kMaxLevels];
  void* r[kMaxLevels];
  void* z[kMaxLevels];
  void* x;
  void* p;
  void* Ap;
  double* part;
  DevState* st;
  DevState* h_st;  // pinned
  cudaStream_t cap;
  cudaGraphExec_t prologue;    // recentring, first V-cycle, p = z, zTr
  long long prologue_kernels;
  cudaGraphExec_t chunk;       // host-checked mode: check_every iterations
  long long chunk_kernels;
  cudaGraphExec_t loop;        // device mode: conditional WHILE node around one iteration
  long long loop_kernels;      // kernels per loop iteration
  size_t bottom_smem;
  int lc;                      // levels lc .. L-1 run as one cluster launch (<= 0: per-level launches)
  int nc;                      // CTAs in that cluster
  size_t coarse_smem;
  int bf16_hi;                 // levels 1 .. bf16_hi-1 stored in BF16 (0: none)
};

namespace fm {

// (red, black) cell pairs along the innermost axis of `planes` planes of level s.
static long coarse_pairs(const Shape& s, int dim, int planes) {
  const long nin = dim == 3 ? s.s2 : s.s1;
  return (long)planes * (dim == 3 ? s.s1 : 1) * ((nin + 1) / 2);
}
static long coarse_ring(const Shape& s, int dim, int planes) {
  return (long)planes * (s.s1 + 2) * (dim == 3 ? s.s2 + 2 : 1);
}

// Picks the finest level lc >= 1 from which the rest of the V-cycle fits one
// cluster launch: level lc split into nc <= 8 slabs of an even number of
// planes, every slab and every deeper level at most kCoarsePPT cell pairs per
// thread, all of it (zero-ringed z, compact r) within 200 KB of shared memory
// per CTA.  lc = -1 when no level qualifies (the V-cycle launches per level).
static void plan_coarse(fm_mgpcg* S, size_t es) {
  S->lc = -1;
  S->nc = 0;
  S->coarse_smem = 0;
  const int dim = S->g.dim;
  const long max_pairs = (long)kCoarsePPT * kCoarseThreads;
  for (int l = 1; l < S->L - 1; ++l) {
    const Shape t = S->lv[l];
    int nc = kCoarseMaxNC;
    while (nc > 1 && t.s0 % (2 * nc) != 0) nc >>= 1;
    if (t.s0 % (2 * nc) != 0) continue;
    const int P = t.s0 / nc;
    if (coarse_pairs(t, dim, P) > max_pairs) continue;
    long cells = coarse_ring(t, dim, P + 2) + (long)P * t.s1 * t.s2;
    bool fits = true;
    for (int m = l + 1; m < S->L; ++m) {
      const Shape d = S->lv[m];
      fits = fits && coarse_pairs(d, dim, d.s0) <= max_pairs;
      cells += d.size() + coarse_ring(d, dim, d.s0 + 2);
    }
    const size_t smem = es * (size_t)cells;
    if (!fits || smem > 200 * 1024) continue;
    S->lc = l;
    S->nc = nc;
    S->coarse_smem = smem;
    return;
  }
}

template <typename T, int D>
static bool enable_coarse_kernel(size_t smem) {
  return raise_smem_limit(k_mg_coarse<T, D>, smem);
}

static inline unsigned blocks_for(long n, int threads, long cap) {
  long b = (n + threads - 1) / threads;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// Levels lc .. L-1 of the V-cycle as one cluster launch (fm_mg_cluster.cuh).
template <typename T, int D>
static void launch_coarse(fm_mgpcg* S, cudaStream_t s) {
  CoarseArgs a;
  int off = 0;  // deep levels in CTA 0: compact r, then zero-ringed z
  for (int l = 0; l < kMaxLevels; ++l) {
    a.lv[l] = S->lv[l];
    a.roff[l] = a.zoff[l] = off;
    if (l > S->lc && l < S->L) {
      a.zoff[l] = off + (int)S->lv[l].size();
      off = a.zoff[l] + (int)coarse_ring(S->lv[l], S->g.dim, S->lv[l].s0 + 2);
    }
  }
  a.lc = S->lc;
  a.L = S->L;
  a.pre_post = S->P.pre_post;
  a.bottom = S->P.bottom;
  a.bottom_mode = S->P.bottom_mode;
  a.r_top = S->r[S->lc];
  a.z_top = S->z[S->lc];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)S->nc, 1, 1);
  cfg.blockDim = dim3(kCoarseThreads, 1, 1);
  cfg.dynamicSmemBytes = S->coarse_smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)S->nc;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = g_pdl.load(std::memory_order_relaxed) ? 2 : 1;
  const DevState* st = S->st;
  cudaLaunchKernelEx(&cfg, k_mg_coarse<T, D>, a, st);
  count_launch(1);
}

// One V-cycle (apply_preconditioner, 3D/mgpcg.py:187-205) on r[0] -> z[0].
// recenter: subtract st->mean from r[0] first (fused into the first sweep);
// dot_last: the last fine sweep also writes z.r block partials.
template <typename T, int D>
static void launch_vcycle(fm_mgpcg* S, cudaStream_t s, bool dot_last, bool recenter = true) {
  const int L = S->L;
  const fm_mg_params& P = S->P;
  T** r = (T**)S->r;
  T** z = (T**)S->z;
  const long cap = 148L * 16;
  const int lc = S->lc > 0 ? S->lc : L - 1;  // first level not smoothed by per-level launches
  const dim3 pblk(kPairBX, kPairBY, 1);
  auto pair_grid = [](const Shape& sh) {
    if (D == 3)
      return dim3((unsigned)((sh.s2 + 1) / 2 + kPairBX - 1) / kPairBX, (unsigned)(sh.s1 + kPairBY - 1) / kPairBY,
                  (unsigned)sh.s0);
    return dim3((unsigned)((sh.s1 + 1) / 2 + kPairBX - 1) / kPairBX, (unsigned)(sh.s0 + kPairBY - 1) / kPairBY, 1);
  };
  // level storage: T, or BF16 for levels 1 .. bf16_hi-1 (FP32 solvers with coarse_bf16)
  using BF = __nv_bfloat16;
  auto bf = [&](int l) { return std::is_same<T, float>::value && l >= 1 && l < S->bf16_hi; };
  auto sweep = [&](int l, int phase) {
    const Shape sh = S->lv[l];
    if (bf(l)) launch_pdl(k_smooth_pair<T, D, BF>, pair_grid(sh), pblk, 0, s, sh, (const BF*)S->r[l], (BF*)S->z[l], phase, S->st);
    else launch_pdl(k_smooth_pair<T, D>, pair_grid(sh), pblk, 0, s, sh, (const T*)r[l], z[l], phase, S->st);
  };
  for (int l = 0; l < lc; ++l) {
    const Shape sh = S->lv[l];
    const dim3 pg = pair_grid(sh);
    for (int it = 0; it < P.pre_post; ++it) {
      if (it == 0) {
        if (bf(l)) launch_pdl(k_smooth_first_pair<T, D, BF>, pg, pblk, 0, s, sh, (BF*)S->r[l], (BF*)S->z[l], S->st, 0);
        else launch_pdl(k_smooth_first_pair<T, D>, pg, pblk, 0, s, sh, r[l], z[l], S->st, l == 0 && recenter ? 1 : 0);
      } else {
        sweep(l, 0);
      }
      sweep(l, 1);
    }
    const Shape sc = S->lv[l + 1];
    const unsigned rb = blocks_for(sc.size(), 256, cap);
    if (bf(l) && bf(l + 1))
      launch_pdl(k_restrict<T, D, BF, BF>, rb, 256, 0, s, sh, sc, (const BF*)S->r[l], (const BF*)S->z[l], (BF*)S->r[l + 1], S->st);
    else if (bf(l))
      launch_pdl(k_restrict<T, D, BF, T>, rb, 256, 0, s, sh, sc, (const BF*)S->r[l], (const BF*)S->z[l], r[l + 1], S->st);
    else if (bf(l + 1))
      launch_pdl(k_restrict<T, D, T, BF>, rb, 256, 0, s, sh, sc, (const T*)r[l], (const T*)z[l], (BF*)S->r[l + 1], S->st);
    else
      launch_pdl(k_restrict<T, D>, rb, 256, 0, s, sh, sc, (const T*)r[l], (const T*)z[l], r[l + 1], S->st);
  }
  const Shape sb = S->lv[L - 1];
  if (S->lc > 0) {
    launch_coarse<T, D>(S, s);
  } else if (S->bottom_smem) {
    launch_pdl(k_bottom<T, D>, 1, kBottomThreads, S->bottom_smem, s, sb, r[L - 1], z[L - 1], P.bottom, P.bottom_mode,
           S->st);
  } else {
    // large coarsest level: per-sweep launches (z zero-filled by the first sweep)
    const unsigned nb = blocks_for(sb.size(), 256, cap);
    int first = 1;
    auto pair = [&](int a, int b) {
      if (first && a == 0) launch_pdl(k_smooth_first<T, D>, nb, 256, 0, s, sb, r[L - 1], z[L - 1], S->st, L == 1 ? 1 : 0);
      else {
        if (first) cudaMemsetAsync(z[L - 1], 0, sizeof(T) * sb.size(), s);
        launch_pdl(k_smooth<T, D, false>, nb, 256, 0, s, sb, r[L - 1], z[L - 1], a, nullptr, S->st);
      }
      first = 0;
      launch_pdl(k_smooth<T, D, false>, nb, 256, 0, s, sb, r[L - 1], z[L - 1], b, nullptr, S->st);
    };
    if (P.bottom_mode == 0) for (int i = 0; i < P.bottom; ++i) pair(0, 1);
    else {
      for (int i = 0; i < P.bottom / 2; ++i) pair(0, 1);
      for (int i = 0; i < P.bottom / 2; ++i) pair(1, 0);
    }
    if (first) cudaMemsetAsync(z[L - 1], 0, sizeof(T) * sb.size(), s);  // no bottom sweeps
  }
  for (int l = lc - 1; l >= 0; --l) {
    const Shape sh = S->lv[l];
    const Shape sc = S->lv[l + 1];
    const unsigned nb = blocks_for(sh.size(), 256, cap);
    if (bf(l) && bf(l + 1))
      launch_pdl(k_prolong<T, D, BF, BF>, nb, 256, 0, s, sh, sc, (BF*)S->z[l], (const BF*)S->z[l + 1], S->st);
    else if (bf(l))
      launch_pdl(k_prolong<T, D, BF, T>, nb, 256, 0, s, sh, sc, (BF*)S->z[l], (const T*)z[l + 1], S->st);
    else if (bf(l + 1))
      launch_pdl(k_prolong<T, D, T, BF>, nb, 256, 0, s, sh, sc, z[l], (const BF*)S->z[l + 1], S->st);
    else
      launch_pdl(k_prolong<T, D>, nb, 256, 0, s, sh, sc, z[l], (const T*)z[l + 1], S->st);
    for (int it = 0; it < P.pre_post; ++it) {
      sweep(l, 1);
      const bool last = dot_last && l == 0 && it == P.pre_post - 1;
      if (last) launch_pdl(k_smooth<T, D, true>, kRedBlocks, kRedThreads, 0, s, sh, r[l], z[l], 0, S->part, S->st);
      else sweep(l, 0);
    }
  }
  if (dot_last && L == 1) {
    // single-level: z.r over the bottom result
    launch_pdl(k_smooth<T, D, true>, kRedBlocks, kRedThreads, 0, s, sb, r[0], z[0], 2 /* no update */, S->part, S->st);
  }
}

// x += alpha p, r -= alpha A p and the convergence test: the second half of a
// PCG iteration (3D/mgpcg.py:240-260).
template <typename T, int D>
static void launch_step(fm_mgpcg* S, cudaStream_t s) {
  const Shape s0 = S->lv[0];
  const long n = s0.size();
  launch_pdl(k_Ap_dot<T, D>, kRedBlocks, kRedThreads, 0, s, s0, (T*)S->p, (T*)S->Ap, S->part, S->st);
  launch_pdl(k_fin_alpha, 1, 256, 0, s, S->st, S->part, S->P.eps);
  launch_pdl(k_update_xr<T>, kRedBlocks, kRedThreads, 0, s, n, (T*)S->x, (T*)S->r[0], (T*)S->p, (T*)S->Ap,
             S->part, S->st);
  launch_pdl(k_fin_conv, 1, 256, 0, s, S->st, S->part, (double)n);
}

// One PCG iteration (3D/mgpcg.py:240-284) as a fixed launch sequence, rotated
// so that the convergence test ends it: z = M r, beta, p = z + beta p, then the
// next x / r update and its test.  A solve that converges stops right after
// its test, with no V-cycle of early-returning kernels behind it; the kernels
// run in the same order as the unrotated loop, so results are unchanged.
template <typename T, int D>
static void launch_iteration(fm_mgpcg* S, cudaStream_t s) {
  const long n = S->lv[0].size();
  launch_vcycle<T, D>(S, s, true);
  launch_pdl(k_fin_beta, 1, 256, 0, s, S->st, S->part, S->P.eps, S->P.abs_tol, S->P.rel_tol, S->P.max_iters, 0);
  launch_pdl(k_update_p<T>, blocks_for(n, 256, 148L * 16), 256, 0, s, n, (T*)S->p, (T*)S->z[0], S->st, 0);
  launch_step<T, D>(S, s);
}

// Prologue after r0 = b and partial sums of b: recentre, V-cycle, p = z, zTr,
// and the first x / r update with its convergence test.
template <typename T, int D>
static void launch_prologue(fm_mgpcg* S, cudaStream_t s) {
  const long n = S->lv[0].size();
  launch_pdl(k_fin_mean, 1, 256, 0, s, S->st, S->part, (double)n);
  launch_vcycle<T, D>(S, s, true);
  launch_pdl(k_fin_beta, 1, 256, 0, s, S->st, S->part, S->P.eps, S->P.abs_tol, S->P.rel_tol, S->P.max_iters, 1);
  launch_pdl(k_update_p<T>, blocks_for(n, 256, 148L * 16), 256, 0, s, n, (T*)S->p, (T*)S->z[0], S->st, 1);
  launch_step<T, D>(S, s);
}

// Device mode: one graph holding a conditional WHILE node whose body is one PCG
// iteration followed by k_loop_cond.  The solve then needs no host round trip.
template <typename T>
static int build_loop_graph(fm_mgpcg* S) {
  const int D = S->g.dim;
  cudaGraph_t graph = nullptr;
  if (cudaGraphCreate(&graph, 0) != cudaSuccess) return FM_ERR_CUDA;
  int status = FM_ERR_CUDA;
  do {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
    cudaKernelNodeParams kp = {};
    DevState* st_arg = S->st;
    void* kargs[2] = {&h, &st_arg};
    kp.func = (void*)k_loop_init;
    kp.gridDim = dim3(1, 1, 1);
    kp.blockDim = dim3(1, 1, 1);
    kp.kernelParams = kargs;
    cudaGraphNode_t init;
    if (cudaGraphAddKernelNode(&init, graph, nullptr, 0, &kp) != cudaSuccess) break;
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, graph, &init, 1, &cp) != cudaSuccess) break;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(S->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
      break;
    const long long before = g_launch_count.load();
    if (D == 3) launch_iteration<T, 3>(S, S->cap); else launch_iteration<T, 2>(S, S->cap);
    launch_pdl(k_loop_cond, 1, 1, 0, S->cap, h, S->st);
    S->loop_kernels = g_launch_count.load() - before;
    g_launch_count.fetch_sub(S->loop_kernels);
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(S->cap, &captured) != cudaSuccess) break;
    if (cudaGraphInstantiate(&S->loop, graph, 0) != cudaSuccess) { S->loop = nullptr; break; }
    status = FM_OK;
  } while (0);
  cudaGraphDestroy(graph);
  cudaGetLastError();
  return status;
}

// The prologue (~45 kernels, internal buffers only) captured once into a graph.
template <typename T>
static int build_prologue_graph(fm_mgpcg* S) {
  cudaGraph_t graph;
  if (cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FM_ERR_CUDA;
  const long long before = g_launch_count.load();
  if (S->g.dim == 3) launch_prologue<T, 3>(S, S->cap); else launch_prologue<T, 2>(S, S->cap);
  S->prologue_kernels = g_launch_count.load() - before;
  g_launch_count.fetch_sub(S->prologue_kernels);  // captured, not executed
  if (cudaStreamEndCapture(S->cap, &graph) != cudaSuccess) return FM_ERR_CUDA;
  const cudaError_t e = cudaGraphInstantiate(&S->prologue, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { S->prologue = nullptr; return FM_ERR_CUDA; }
  return FM_OK;
}

// True while `s` records into a CUDA graph (a caller capturing a whole
// gradient); the solver then adds its work to that graph instead of launching
// its own executable graphs.
static bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return false;
  return cs == cudaStreamCaptureStatusActive;
}

// A device-mode solve recorded into the graph being captured on `s`: the
// prologue's kernels go onto `s`, and the PCG loop becomes a conditional WHILE
// node appended to the captured graph (after the prologue), its body one PCG
// iteration and k_loop_cond recorded from S->cap.  Every solve recorded this
// way owns its own node and condition handle.
template <typename T>
static int capture_solve(fm_mgpcg* S, cudaStream_t s) {
  const int D = S->g.dim;
  if (D == 3) launch_prologue<T, 3>(S, s); else launch_prologue<T, 2>(S, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e);
  cudaStreamCaptureStatus cs;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  if ((e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps)) != cudaSuccess) return cuda_fail(e);
  if (cs != cudaStreamCaptureStatusActive) return cuda_fail(cudaErrorStreamCaptureInvalidated);
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return cuda_fail(e);
  k_loop_init<<<1, 1, 0, s>>>(h, S->st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps)) != cudaSuccess) return cuda_fail(e);
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return cuda_fail(e);
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(S->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return cuda_fail(e);
  const long long before = g_launch_count.load();
  if (D == 3) launch_iteration<T, 3>(S, S->cap); else launch_iteration<T, 2>(S, S->cap);
  launch_pdl(k_loop_cond, 1, 1, 0, S->cap, h, S->st);
  g_launch_count.fetch_sub(g_launch_count.load() - before);  // the loop body runs a data-dependent number of times
  cudaGraph_t captured = nullptr;
  if ((e = cudaStreamEndCapture(S->cap, &captured)) != cudaSuccess) return cuda_fail(e);
  return FM_OK;
}

template <typename T>
static int run_solve(fm_mgpcg* S, cudaStream_t s, int* iters, double* rtr) {
  const int D = S->g.dim;
  if (stream_capturing(s)) {
    // recorded, not run: no host read of the outcome, no host-checked loop
    if (iters || rtr || S->P.check_every != 0) return FM_ERR_ARG;
    return capture_solve<T>(S, s);
  }
  if (!S->prologue) {
    const int e = build_prologue_graph<T>(S);
    if (e) return e;
  }
  if (cudaGraphLaunch(S->prologue, s) != cudaSuccess) return FM_ERR_CUDA;
  count_launch(S->prologue_kernels);
  if (S->P.check_every == 0) {
    if (!S->loop) {
      int e = build_loop_graph<T>(S);
      if (e) return e;
    }
    if (cudaGraphLaunch(S->loop, s) != cudaSuccess) return FM_ERR_CUDA;
    if (!iters && !rtr) return FM_OK;  // asynchronous: outcome via fm_mgpcg_stats
    if (cudaMemcpyAsync(S->h_st, S->st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    if (iters) *iters = S->h_st->result_it;
    if (rtr) *rtr = S->h_st->rTr;
    if (S->h_st->nonfinite) return FM_ERR_NONFINITE;
    if (!S->h_st->conv) return FM_ERR_NOT_CONVERGED;
    return FM_OK;
  }
  if (!S->chunk) {
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FM_ERR_CUDA;
    const long long before = g_launch_count.load();
    for (int i = 0; i < S->P.check_every; ++i) {
      if (D == 3) launch_iteration<T, 3>(S, S->cap); else launch_iteration<T, 2>(S, S->cap);
    }
    // captured, not executed: count them per graph launch instead
    S->chunk_kernels = g_launch_count.load() - before;
    g_launch_count.fetch_sub(S->chunk_kernels);
    if (cudaStreamEndCapture(S->cap, &graph) != cudaSuccess) return FM_ERR_CUDA;
    cudaError_t e = cudaGraphInstantiate(&S->chunk, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { S->chunk = nullptr; return FM_ERR_CUDA; }
  }
  long launched = 0;
  const long limit = (long)S->P.max_iters + S->P.check_every;
  for (;;) {
    if (cudaGraphLaunch(S->chunk, s) != cudaSuccess) return FM_ERR_CUDA;
    count_launch(S->chunk_kernels);
    launched += S->P.check_every;
    if (cudaMemcpyAsync(S->h_st, S->st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    if (S->h_st->done || launched >= limit) break;
  }
  if (iters) *iters = S->h_st->result_it;
  if (rtr) *rtr = S->h_st->rTr;
  if (S->h_st->nonfinite) return FM_ERR_NONFINITE;
  if (!S->h_st->conv) return FM_ERR_NOT_CONVERGED;
  return FM_OK;
}

}  // namespace fm

extern "C" {

int fm_mgpcg_create(const fm_grid* g, int dtype, const fm_mg_params* params, fm_mgpcg** out) {
  if (!out || !params) return FM_ERR_ARG;
  *out = nullptr;
  int st = validate_grid(g, dtype);
  if (st) return st;
  const fm_mg_params& P = *params;
  if (P.levels < 2 || P.levels > kMaxLevels || P.pre_post < 1 || P.bottom < 0 || P.max_iters < 1 ||
      P.check_every < 0 || (P.bottom_mode != 0 && P.bottom_mode != 1))
    return FM_ERR_ARG;
  if (P.coarse_bf16 && dtype != FM_F32) return FM_ERR_ARG;
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] % (1 << (P.levels - 1)) != 0 || (g->n[a] >> (P.levels - 1)) < 1) return FM_ERR_SHAPE;
  fm_mgpcg* S = (fm_mgpcg*)calloc(1, sizeof(fm_mgpcg));
  if (!S) return FM_ERR_ARG;
  S->g = *g;
  S->dtype = dtype;
  S->P = P;
  S->L = P.levels;
  const size_t es = dtype == FM_F32 ? sizeof(float) : sizeof(double);
  bool ok = true;
  for (int l = 0; l < S->L; ++l) {
    Shape sh{1, 1, 1};
    sh.s0 = g->n[0] >> l;
    sh.s1 = g->n[1] >> l;
    sh.s2 = g->dim == 3 ? (g->n[2] >> l) : 1;
    S->lv[l] = sh;
  }
  // coarse levels in one cluster launch where they fit
  plan_coarse(S, es);
  if (S->lc > 0) {
    const bool en = dtype == FM_F32 ? (g->dim == 3 ? enable_coarse_kernel<float, 3>(S->coarse_smem)
                                                   : enable_coarse_kernel<float, 2>(S->coarse_smem))
                                    : (g->dim == 3 ? enable_coarse_kernel<double, 3>(S->coarse_smem)
                                                   : enable_coarse_kernel<double, 2>(S->coarse_smem));
    if (!en) {
      cudaGetLastError();
      S->lc = -1;
    }
  }
  // BF16 storage for the per-level coarse levels 1 .. lc-1 (needs the cluster path)
  S->bf16_hi = (P.coarse_bf16 && S->lc > 1) ? S->lc : 0;
  for (int l = 0; l < S->L; ++l) {
    const size_t e = (l >= 1 && l < S->bf16_hi) ? sizeof(__nv_bfloat16) : es;
    ok = ok && cudaMalloc(&S->r[l], e * S->lv[l].size()) == cudaSuccess;
    ok = ok && cudaMalloc(&S->z[l], e * S->lv[l].size()) == cudaSuccess;
  }
  const long n0 = S->lv[0].size();
  ok = ok && cudaMalloc(&S->x, es * n0) == cudaSuccess;
  ok = ok && cudaMalloc(&S->p, es * n0) == cudaSuccess;
  ok = ok && cudaMalloc(&S->Ap, es * n0) == cudaSuccess;
  ok = ok && cudaMalloc(&S->part, sizeof(double) * 2 * kRedBlocks) == cudaSuccess;
  ok = ok && cudaMalloc(&S->st, sizeof(DevState)) == cudaSuccess;
  ok = ok && cudaMallocHost(&S->h_st, sizeof(DevState)) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking) == cudaSuccess;
  if (ok) ok = cudaMemset(S->st, 0, sizeof(DevState)) == cudaSuccess;
  const long nb = S->lv[S->L - 1].size();
  const size_t smem = 2 * es * nb;
  if (ok && smem <= 200 * 1024 && nb <= kBottomMaxCells) {
    S->bottom_smem = smem;
    if (smem > 48 * 1024) {
      bool e;
      if (dtype == FM_F32)
        e = g->dim == 3 ? raise_smem_limit(k_bottom<float, 3>, smem) : raise_smem_limit(k_bottom<float, 2>, smem);
      else
        e = g->dim == 3 ? raise_smem_limit(k_bottom<double, 3>, smem) : raise_smem_limit(k_bottom<double, 2>, smem);
      if (!e) {
        cudaGetLastError();
        S->bottom_smem = 0;
      }
    }
  }
  if (!ok) {
    fm_mgpcg_destroy(S);
    return FM_ERR_CUDA;
  }
  *out = S;
  return FM_OK;
}

int fm_mgpcg_destroy(fm_mgpcg* S) {
  if (!S) return FM_OK;
  for (int l = 0; l < kMaxLevels; ++l) {
    if (S->r[l]) cudaFree(S->r[l]);
    if (S->z[l]) cudaFree(S->z[l]);
  }
  if (S->x) cudaFree(S->x);
  if (S->p) cudaFree(S->p);
  if (S->Ap) cudaFree(S->Ap);
  if (S->part) cudaFree(S->part);
  if (S->st) cudaFree(S->st);
  if (S->h_st) cudaFreeHost(S->h_st);
  if (S->chunk) cudaGraphExecDestroy(S->chunk);
  if (S->prologue) cudaGraphExecDestroy(S->prologue);
  if (S->loop) cudaGraphExecDestroy(S->loop);
  if (S->cap) cudaStreamDestroy(S->cap);
  free(S);
  return FM_OK;
}

int fm_project(fm_mgpcg* S, void* ux, void* uy, void* uz, void* p_out, void* stream, int* iters, double* rtr) {
  if (!S || !ux || !uy || (S->g.dim == 3 && !uz)) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const fm_grid g = S->g;
  const long n = S->lv[0].size();
  int status;
  long maxf = 0;
  for (int c = 0; c < g.dim; ++c) maxf = face_shape(g, c).size() > maxf ? face_shape(g, c).size() : maxf;
  dim3 fgrid((unsigned)((maxf + 255) / 256), (unsigned)g.dim, 1);
  if (S->dtype == FM_F32) {
    MacW<float> u{{(float*)ux, (float*)uy, (float*)uz}};
    if (g.dim == 3) launch_pdl(k_div_bc<float, 3>, kRedBlocks, kRedThreads, 0, s, g, u, (float*)S->r[0], (float*)S->x, S->part);
    else launch_pdl(k_div_bc<float, 2>, kRedBlocks, kRedThreads, 0, s, g, u, (float*)S->r[0], (float*)S->x, S->part);
    status = run_solve<float>(S, s, iters, rtr);
    if (status == FM_ERR_CUDA) return status;
    if (g.dim == 3) launch_pdl(k_subgrad_bc<float, 3>, fgrid, 256, 0, s, g, (const float*)S->x, u);
    else launch_pdl(k_subgrad_bc<float, 2>, fgrid, 256, 0, s, g, (const float*)S->x, u);
  } else {
    MacW<double> u{{(double*)ux, (double*)uy, (double*)uz}};
    if (g.dim == 3) launch_pdl(k_div_bc<double, 3>, kRedBlocks, kRedThreads, 0, s, g, u, (double*)S->r[0], (double*)S->x, S->part);
    else launch_pdl(k_div_bc<double, 2>, kRedBlocks, kRedThreads, 0, s, g, u, (double*)S->r[0], (double*)S->x, S->part);
    status = run_solve<double>(S, s, iters, rtr);
    if (status == FM_ERR_CUDA) return status;
    if (g.dim == 3) launch_pdl(k_subgrad_bc<double, 3>, fgrid, 256, 0, s, g, (const double*)S->x, u);
    else launch_pdl(k_subgrad_bc<double, 2>, fgrid, 256, 0, s, g, (const double*)S->x, u);
  }
  if (p_out) cudaMemcpyAsync(p_out, S->x, (S->dtype == FM_F32 ? 4 : 8) * n, cudaMemcpyDeviceToDevice, s);
  if (check_cuda()) return FM_ERR_CUDA;
  return status;
}

int fm_mgpcg_solve(fm_mgpcg* S, const void* b, void* x, void* stream, int* iters, double* rtr) {
  if (!S || !b || !x) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const long n = S->lv[0].size();
  int status;
  if (S->dtype == FM_F32) {
    launch_pdl(k_load_rhs<float>, kRedBlocks, kRedThreads, 0, s, n, (const float*)b, (float*)S->r[0], (float*)S->x, S->part);
    status = run_solve<float>(S, s, iters, rtr);
  } else {
    launch_pdl(k_load_rhs<double>, kRedBlocks, kRedThreads, 0, s, n, (const double*)b, (double*)S->r[0], (double*)S->x, S->part);
    status = run_solve<double>(S, s, iters, rtr);
  }
  if (status == FM_ERR_CUDA) return status;
  cudaMemcpyAsync(x, S->x, (S->dtype == FM_F32 ? 4 : 8) * n, cudaMemcpyDeviceToDevice, s);
  if (check_cuda()) return FM_ERR_CUDA;
  return status;
}

int fm_mg_vcycle(fm_mgpcg* S, const void* r, void* z, void* stream) {
  if (!S || !r || !z) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (S->dtype == FM_F32 ? 4 : 8) * (size_t)S->lv[0].size();
  if (cudaMemcpyAsync(S->r[0], r, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return FM_ERR_CUDA;
  // every V-cycle kernel is gated on the solver's `done` word
  if (cudaMemsetAsync(&S->st->done, 0, sizeof(int), s) != cudaSuccess) return FM_ERR_CUDA;
  if (S->dtype == FM_F32) {
    if (S->g.dim == 3) launch_vcycle<float, 3>(S, s, false, false);
    else launch_vcycle<float, 2>(S, s, false, false);
  } else {
    if (S->g.dim == 3) launch_vcycle<double, 3>(S, s, false, false);
    else launch_vcycle<double, 2>(S, s, false, false);
  }
  if (cudaMemcpyAsync(z, S->z[0], bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return FM_ERR_CUDA;
  return check_cuda();
}

int fm_mgpcg_solve_dc(fm_mgpcg* S, int b_dtype, const void* b, double* x, double* work, double rel_tol,
                      int max_outer, void* stream, int* outer_iters, int* inner_iters, double* rel_res) {
  if (!S || !b || !x || !work || max_outer < 0 || !(rel_tol >= 0.0)) return FM_ERR_ARG;
  if (S->dtype != FM_F32 || (b_dtype != FM_F32 && b_dtype != FM_F64)) return FM_ERR_DTYPE;
  cudaStream_t s = (cudaStream_t)stream;
  const Shape s0 = S->lv[0];
  const long n = s0.size();
  const int D = S->g.dim;
  const unsigned nb = blocks_for(n, 256, 148L * 16);
  if (b_dtype == FM_F32) launch_pdl(k_dc_sum<float>, kRedBlocks, kRedThreads, 0, s, n, (const float*)b, S->part);
  else launch_pdl(k_dc_sum<double>, kRedBlocks, kRedThreads, 0, s, n, (const double*)b, S->part);
  launch_pdl(k_dc_fin, 1, 256, 0, s, S->st, S->part, (double)n, 0);
  if (cudaMemsetAsync(x, 0, sizeof(double) * n, s) != cudaSuccess) return FM_ERR_CUDA;
  auto residual = [&](int which) {
    if (b_dtype == FM_F32) {
      if (D == 3) launch_pdl(k_dc_residual<float, 3>, kRedBlocks, kRedThreads, 0, s, s0, (const float*)b, x, work, S->part, S->st);
      else launch_pdl(k_dc_residual<float, 2>, kRedBlocks, kRedThreads, 0, s, s0, (const float*)b, x, work, S->part, S->st);
    } else {
      if (D == 3) launch_pdl(k_dc_residual<double, 3>, kRedBlocks, kRedThreads, 0, s, s0, (const double*)b, x, work, S->part, S->st);
      else launch_pdl(k_dc_residual<double, 2>, kRedBlocks, kRedThreads, 0, s, s0, (const double*)b, x, work, S->part, S->st);
    }
    launch_pdl(k_dc_fin, 1, 256, 0, s, S->st, S->part, (double)n, which);
  };
  residual(1);
  int outer = 0, inner = 0, status = FM_OK;
  double rel = 0;
  for (;;) {
    if (cudaMemcpyAsync(S->h_st, S->st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    const double b2 = S->h_st->dc_b2, r2 = S->h_st->dc_r2;
    rel = b2 > 0 ? sqrt(r2 / b2) : 0.0;
    if (!isfinite(rel)) { status = FM_ERR_NONFINITE; break; }
    if (rel <= rel_tol || r2 == 0.0) break;
    if (outer >= max_outer) { status = FM_ERR_NOT_CONVERGED; break; }
    launch_pdl(k_dc_load, kRedBlocks, kRedThreads, 0, s, n, (const double*)work, (float*)S->r[0], (float*)S->x, S->part,
           (const DevState*)S->st);
    launch_pdl(k_dc_set_tol, 1, 1, 0, s, S->st, rel_tol, 0);
    int it = 0;
    double rtr = 0;
    const int st = run_solve<float>(S, s, &it, &rtr);  // reaching max_iters is fine: the outer loop corrects
    inner += it;
    if (st == FM_ERR_CUDA || st == FM_ERR_NONFINITE) { status = st; break; }
    launch_pdl(k_dc_update, nb, 256, 0, s, n, x, (const float*)S->x, (const DevState*)S->st);
    ++outer;
    residual(2);
  }
  launch_pdl(k_dc_set_tol, 1, 1, 0, s, S->st, 0.0, 1);
  if (outer_iters) *outer_iters = outer;
  if (inner_iters) *inner_iters = inner;
  if (rel_res) *rel_res = rel;
  if (check_cuda()) return FM_ERR_CUDA;
  return status;
}

int fm_project_dc(fm_mgpcg* S, void* ux, void* uy, void* uz, double* work, double rel_tol, int max_outer,
                  double* p_out, void* stream) {
  if (!S || !ux || !uy || (S->g.dim == 3 && !uz) || !work || max_outer < 1 || max_outer > 16 ||
      !(rel_tol > 0.0))
    return FM_ERR_ARG;
  if (S->dtype != FM_F32) return FM_ERR_DTYPE;
  if (S->P.check_every != 0) return FM_ERR_ARG;  // device-side loops only
  cudaStream_t s = (cudaStream_t)stream;
  const fm_grid g = S->g;
  const Shape s0 = S->lv[0];
  const long n = s0.size();
  const int D = g.dim;
  double* b = work;
  double* x = work + n;
  double* w = work + 2 * n;
  MacW<float> u{{(float*)ux, (float*)uy, (float*)uz}};
  const unsigned nb = blocks_for(n, 256, 148L * 16);
  if (D == 3) launch_pdl(k_dc_div<3>, kRedBlocks, kRedThreads, 0, s, g, u, b, x, S->part);
  else launch_pdl(k_dc_div<2>, kRedBlocks, kRedThreads, 0, s, g, u, b, x, S->part);
  launch_pdl(k_dc_fin, 1, 256, 0, s, S->st, S->part, (double)n, 0);  // dc_mean
  auto residual = [&](int which) {
    if (D == 3) launch_pdl(k_dc_residual_g<3>, kRedBlocks, kRedThreads, 0, s, s0, (const double*)b, (const double*)x, w, S->part, (const DevState*)S->st);
    else launch_pdl(k_dc_residual_g<2>, kRedBlocks, kRedThreads, 0, s, s0, (const double*)b, (const double*)x, w, S->part, (const DevState*)S->st);
    launch_pdl(k_dc_check, 1, 256, 0, s, S->st, S->part, rel_tol, which);
  };
  residual(1);
  for (int o = 0; o < max_outer; ++o) {
    launch_pdl(k_dc_load_g, kRedBlocks, kRedThreads, 0, s, n, (const double*)w, (float*)S->r[0], (float*)S->x,
               S->part, (const DevState*)S->st);
    launch_pdl(k_dc_set_tol_g, 1, 1, 0, s, S->st, rel_tol);
    const int st = run_solve<float>(S, s, nullptr, nullptr);
    if (st) return st;
    launch_pdl(k_dc_update_g, nb, 256, 0, s, n, x, (const float*)S->x, (const DevState*)S->st);
    residual(2);
  }
  long maxf = 0;
  for (int c = 0; c < D; ++c) maxf = face_shape(g, c).size() > maxf ? face_shape(g, c).size() : maxf;
  dim3 fgrid((unsigned)((maxf + 255) / 256), (unsigned)D, 1);
  if (D == 3) launch_pdl(k_dc_subgrad<3>, fgrid, 256, 0, s, g, (const double*)x, u);
  else launch_pdl(k_dc_subgrad<2>, fgrid, 256, 0, s, g, (const double*)x, u);
  launch_pdl(k_dc_finish, 1, 1, 0, s, S->st);
  if (p_out) cudaMemcpyAsync(p_out, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  if (check_cuda()) return FM_ERR_CUDA;
  return FM_OK;
}

int fm_mgpcg_stats(fm_mgpcg* S, void* stream, int reset, fm_mg_stats* out) {
  if (!S || !out) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(S->h_st, S->st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
  const DevState& h = *S->h_st;
  out->solves = h.solves;
  out->iterations = h.iters_total;
  out->not_converged = h.not_converged;
  out->nonfinite = h.nonfinite_count;
  out->last_iters = h.result_it;
  out->max_iters_seen = h.max_it_seen;
  out->last_rtr = h.rTr;
  // kernels run inside device-mode while loops since the last call
  count_launch(h.bodies * S->loop_kernels);
  long long zero_bodies = 0;
  if (cudaMemcpyAsync(&S->st->bodies, &zero_bodies, sizeof(long long), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return FM_ERR_CUDA;
  if (reset) {
    DevState z = h;
    z.solves = z.iters_total = z.not_converged = z.nonfinite_count = 0;
    z.max_it_seen = 0;
    z.bodies = 0;
    if (cudaMemcpyAsync(S->st, &z, sizeof(DevState), cudaMemcpyHostToDevice, s) != cudaSuccess) return FM_ERR_CUDA;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
  return FM_OK;
}

int fm_laplacian(const fm_grid* g, int dtype, const void* p, void* Ap, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!p || !Ap) return FM_ERR_ARG;
  Shape s = cell_shape(*g);
  cudaStream_t cs = (cudaStream_t)stream;
  unsigned nb = blocks_for(s.size(), 256, 148L * 16);
  if (dtype == FM_F32) {
    if (g->dim == 3) launch_pdl(k_laplacian<float, 3>, nb, 256, 0, cs, s, (const float*)p, (float*)Ap);
    else launch_pdl(k_laplacian<float, 2>, nb, 256, 0, cs, s, (const float*)p, (float*)Ap);
  } else {
    if (g->dim == 3) launch_pdl(k_laplacian<double, 3>, nb, 256, 0, cs, s, (const double*)p, (double*)Ap);
    else launch_pdl(k_laplacian<double, 2>, nb, 256, 0, cs, s, (const double*)p, (double*)Ap);
  }
  return check_cuda();
}

int fm_abi_version(void) { return 1; }

long long fm_launch_count(int reset) {
  if (reset) return g_launch_count.exchange(0);
  return g_launch_count.load();
}

int fm_set_pdl(int enable) {
  return g_pdl.exchange(enable ? 1 : 0);
}

int fm_last_cuda_error(char* buf, int len) {
  const int e = g_last_cuda_error.load();
  if (buf && len > 0) {
    const char* name = e ? cudaGetErrorName((cudaError_t)e) : "cudaSuccess";
    int i = 0;
    for (; name && name[i] && i < len - 1; ++i) buf[i] = name[i];
    buf[i] = 0;
  }
  return e;
}

const char* fm_status_string(int status) {
  switch (status) {
    case FM_OK: return "ok";
    case FM_ERR_SHAPE: return "unsupported grid shape";
    case FM_ERR_ARG: return "invalid argument";
    case FM_ERR_NOT_CONVERGED: return "MGPCG did not converge within max_iters";
    case FM_ERR_NONFINITE: return "non-finite residual in MGPCG";
    case FM_ERR_TIMEOUT: return "bounded device wait timed out";
    case FM_ERR_CUDA: return "CUDA runtime error";
    case FM_ERR_DTYPE: return "unsupported dtype";
    case FM_ERR_CAPACITY: return "grid too large for the static scratch of fm_project_noalloc";
    default: return "unknown status";
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// fm_project_noalloc: the projection without any allocation.
//
// Its MG hierarchy, PCG vectors, reduction partials and solver state are carved
// out of one file-scope __device__ array (kNoAllocScratchBytes), which every
// GPU that loads this library holds until the process exits.  Host code cannot
// use the array's name as a device address (it names a host-side shadow), so
// the address is fetched with cudaGetSymbolAddress once per device, with that
// device current, on the first call made on it; that first call should
// therefore come before any stream capture.  Under CUDA's lazy module loading
// (the default) that first call is also when the array and this library's
// kernels receive their device memory, so it must come before another runtime
// claims the device's memory (or the process sets CUDA_MODULE_LOADING=EAGER,
// which places them when the library loads).  Kernels are launched directly (no
// CUDA graph, whose instantiation may allocate) and convergence is polled
// through a host stack variable (no pinned buffer).
// ---------------------------------------------------------------------------
namespace fm {

constexpr size_t kNoAllocScratchBytes = size_t(48) << 20;  // 48 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static void* g_noalloc_base[kMaxDevices];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FM_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();  // leave no pending error for an unrelated later check
      return FM_ERR_CUDA;
    }
    g_noalloc_base[dev] = p;
  }
  *out = g_noalloc_base[dev];
  return FM_OK;
}

// Lays the solver's buffers out from `base` (nullptr: size only); returns bytes.
static size_t noalloc_layout(const fm_grid& g, int dtype, int levels, fm_mgpcg* S, unsigned char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> void* {
    off = (off + 255) & ~size_t(255);
    void* p = base ? (void*)(base + off) : nullptr;
    off += bytes;
    return p;
  };
  const size_t es = dtype == FM_F32 ? sizeof(float) : sizeof(double);
  for (int l = 0; l < levels; ++l) {
    Shape sh{g.n[0] >> l, g.n[1] >> l, g.dim == 3 ? (g.n[2] >> l) : 1};
    S->lv[l] = sh;
    S->r[l] = take(es * sh.size());
    S->z[l] = take(es * sh.size());
  }
  const long n0 = S->lv[0].size();
  S->x = take(es * n0);
  S->p = take(es * n0);
  S->Ap = take(es * n0);
  S->part = (double*)take(sizeof(double) * 2 * kRedBlocks);
  S->st = (DevState*)take(sizeof(DevState));
  return off;
}

// Host-checked solve with direct launches (no graph).
template <typename T>
static int run_solve_direct(fm_mgpcg* S, cudaStream_t s, int* iters, double* rtr) {
  const int D = S->g.dim;
  const int every = S->P.check_every > 0 ? S->P.check_every : 4;
  if (D == 3) launch_prologue<T, 3>(S, s); else launch_prologue<T, 2>(S, s);
  DevState h;
  long launched = 0;
  const long limit = (long)S->P.max_iters + every;
  for (;;) {
    for (int i = 0; i < every; ++i) {
      if (D == 3) launch_iteration<T, 3>(S, s); else launch_iteration<T, 2>(S, s);
    }
    launched += every;
    if (cudaMemcpyAsync(&h, S->st, sizeof(DevState), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    if (h.done || launched >= limit) break;
  }
  if (iters) *iters = h.result_it;
  if (rtr) *rtr = h.rTr;
  if (h.nonfinite) return FM_ERR_NONFINITE;
  if (!h.conv) return FM_ERR_NOT_CONVERGED;
  return FM_OK;
}

}  // namespace fm

extern "C" int fm_project_noalloc(const fm_grid* g, int dtype, const fm_mg_params* params, void* ux, void* uy,
                                  void* uz, void* stream, int* iters, double* rtr) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (!params) return FM_ERR_ARG;
  const fm_mg_params& P = *params;
  if (P.levels < 2 || P.levels > kMaxLevels || P.pre_post < 1 || P.bottom < 0 || P.max_iters < 1 ||
      P.check_every < 0 || (P.bottom_mode != 0 && P.bottom_mode != 1) || P.coarse_bf16)
    return FM_ERR_ARG;
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] % (1 << (P.levels - 1)) != 0) return FM_ERR_SHAPE;
  fm_mgpcg S;
  memset(&S, 0, sizeof(S));
  S.g = *g;
  S.dtype = dtype;
  S.P = P;
  S.L = P.levels;
  // capacity before the field pointers: a caller can ask whether a grid fits without passing any
  if (noalloc_layout(*g, dtype, P.levels, &S, nullptr) > kNoAllocScratchBytes) return FM_ERR_CAPACITY;
  if (!ux || !uy || (g->dim == 3 && !uz)) return FM_ERR_ARG;
  void* base = nullptr;
  if ((st = noalloc_scratch(&base))) return st;
  noalloc_layout(*g, dtype, P.levels, &S, (unsigned char*)base);
  const size_t es = dtype == FM_F32 ? sizeof(float) : sizeof(double);
  const size_t smem = 2 * es * S.lv[S.L - 1].size();
  // larger coarsest levels: per-sweep launches
  S.bottom_smem = (smem <= 48 * 1024 && S.lv[S.L - 1].size() <= kBottomMaxCells) ? smem : 0;
  cudaStream_t s = (cudaStream_t)stream;
  // the scratch keeps the previous call's contents: the solver state must start at zero
  if (cudaMemsetAsync(S.st, 0, sizeof(DevState), s) != cudaSuccess) return FM_ERR_CUDA;
  long maxf = 0;
  for (int c = 0; c < g->dim; ++c) maxf = face_shape(*g, c).size() > maxf ? face_shape(*g, c).size() : maxf;
  dim3 fgrid((unsigned)((maxf + 255) / 256), (unsigned)g->dim, 1);
  const fm_grid gg = *g;
  int status;
  if (dtype == FM_F32) {
    MacW<float> u{{(float*)ux, (float*)uy, (float*)uz}};
    if (gg.dim == 3) launch_pdl(k_div_bc<float, 3>, kRedBlocks, kRedThreads, 0, s, gg, u, (float*)S.r[0], (float*)S.x, S.part);
    else launch_pdl(k_div_bc<float, 2>, kRedBlocks, kRedThreads, 0, s, gg, u, (float*)S.r[0], (float*)S.x, S.part);
    status = run_solve_direct<float>(&S, s, iters, rtr);
    if (status == FM_ERR_CUDA) return status;
    if (gg.dim == 3) launch_pdl(k_subgrad_bc<float, 3>, fgrid, 256, 0, s, gg, (const float*)S.x, u);
    else launch_pdl(k_subgrad_bc<float, 2>, fgrid, 256, 0, s, gg, (const float*)S.x, u);
  } else {
    MacW<double> u{{(double*)ux, (double*)uy, (double*)uz}};
    if (gg.dim == 3) launch_pdl(k_div_bc<double, 3>, kRedBlocks, kRedThreads, 0, s, gg, u, (double*)S.r[0], (double*)S.x, S.part);
    else launch_pdl(k_div_bc<double, 2>, kRedBlocks, kRedThreads, 0, s, gg, u, (double*)S.r[0], (double*)S.x, S.part);
    status = run_solve_direct<double>(&S, s, iters, rtr);
    if (status == FM_ERR_CUDA) return status;
    if (gg.dim == 3) launch_pdl(k_subgrad_bc<double, 3>, fgrid, 256, 0, s, gg, (const double*)S.x, u);
    else launch_pdl(k_subgrad_bc<double, 2>, fgrid, 256, 0, s, gg, (const double*)S.x, u);
  }
  if (check_cuda()) return FM_ERR_CUDA;
  return status;
}
