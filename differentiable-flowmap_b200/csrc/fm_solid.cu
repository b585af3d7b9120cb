// fm_solid.cu -- the obstacle path: MGPCG with a boundary mask and the mask
// kernels.
//
// Solver (2D/vortex/mgpcg_solid.py:14-458, MGPCG_2_solid; dimension-generic):
// cells with mask > 0 are solid.  Coarse masks follow downsample_bm (a coarse
// cell is solid only when all its children are, :114-127).  The operator,
// the red-black Gauss-Seidel smoother, the residual restriction and the PCG
// updates act on fluid cells only, with neighbour counts and sums over
// in-domain fluid neighbours, each axis adding its right then its left
// neighbour (:141-172); the restricted residual is scaled by 1/(dim-1)
// (:225); prolongation adds to every cell (:228-231); recentring subtracts the
// mean over all cells, solid ones included (:241-247).  Every smoother,
// restriction and prolongation step rounds as the reference writes it (no FMA
// contraction, IEEE division), and a coarse cell sums its children's
// residuals in lexicographic order (the reference scatters them with
// atomics), so the V-cycle equals the oracle's bit for bit.  PCG inner
// products are fixed-grid FP64 reductions.
//
// B200 mapping.  The hierarchy is small next to the flow-map state (256^2:
// 0.5 MB per level), so the levels are plain global arrays and every step is a
// grid-stride kernel; the coarsest levels that fit 96 KB of shared memory
// (down-sweeps, bottom, up-sweeps) run in one CTA out of shared memory.  The PCG loop keeps its
// scalars (alpha, beta, the inner products, a done flag) on the device: every
// kernel of an iteration returns at once after convergence, so the host only
// polls the flag every check_every iterations (a chunk of iterations captured
// once as a CUDA graph and replayed), and the result equals stopping at the
// exact iteration.
//
// Mask kernels (2D/vortex/init_conditions.py:549-583, 3D/init_conditions.py:
// 536-578): mask >= 1 is solid there.  mask_velocity writes the boundary
// velocity on the faces of solid cells; where two adjacent solid cells would
// write one face with different velocities (the reference races) the cell on
// the face's high side wins.  mask_passive gives a solid cell the mean of its
// fluid 3^dim neighbours (lexicographic offset order) or 0.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {
namespace solid {

constexpr int kThreads = 256;
constexpr int kRedBlocks = 148 * 4;
constexpr int kBottomThreads = 1024;
constexpr size_t kCoarseSmem = 96 * 1024;  // shared memory for the single-CTA coarse levels

struct State {
  double old_zr, tol, rtr, pAp, new_zr, sum_r;
  double alpha, beta, mean;
  int done, iters, converged, max_iters;
  double abs_tol, rel_tol, eps;
  int loops;  // device-side loop bodies run in this solve (a hard bound on the WHILE node)
};

// Outcome of every solve, accumulated on the device (fm_solid_stats).
struct Stats {
  long long solves, iterations, not_converged, nonfinite, bodies;
  int last_iters, max_iters_seen;
  double last_rtr;
};

// The solve's scalars from the parameters (replaces a host copy, so that a
// recorded graph does not depend on host memory).
__global__ void k_state_init(State* st, int max_iters, double abs_tol, double rel_tol, double eps) {
  State h{};
  h.max_iters = max_iters;
  h.abs_tol = abs_tol;
  h.rel_tol = rel_tol;
  h.eps = eps;
  *st = h;
}

// Device mode: the WHILE node runs the next PCG iteration while the solve is
// not done; the body count is bounded by max_iters + 1 whatever the flags say.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, State* st, Stats* stats) {
  st->loops += 1;
  stats->bodies += 1;
  cudaGraphSetConditional(h, (!st->done && st->loops <= st->max_iters) ? 1u : 0u);
}

// Before the WHILE node: skip the loop when the prologue's test already ended
// the solve.
__global__ void k_loop_init(cudaGraphConditionalHandle h, const State* st) {
  cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

__global__ void k_stats(const State* st, Stats* out) {
  const bool nf = !isfinite(st->rtr);
  out->solves += 1;
  out->iterations += st->iters;
  out->nonfinite += nf ? 1 : 0;
  out->not_converged += (!nf && !st->converged) ? 1 : 0;
  out->last_iters = st->iters;
  if (st->iters > out->max_iters_seen) out->max_iters_seen = st->iters;
  out->last_rtr = st->rtr;
}

__device__ __forceinline__ void idx3(const Shape& s, long q, int* I) {
  int i, j, k;
  unflatten(s, q, i, j, k);
  I[0] = i;
  I[1] = j;
  I[2] = k;
}

__device__ __forceinline__ long stride_of(const Shape& s, int a) {
  return a == 0 ? (long)s.s1 * s.s2 : (a == 1 ? (long)s.s2 : 1L);
}

// (count, sum) over in-domain fluid neighbours: per axis the right, then the
// left neighbour (neighbor_sum2 / num_fluid_neighbors2, :141-172)
template <typename T, int D>
__device__ __forceinline__ int fluid_nbrs(const T* __restrict__ x, const uint8_t* __restrict__ fl, const Shape& s,
                                          const int* I, long q, T& sum) {
  int n = 0;
  sum = (T)0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const long st = stride_of(s, a);
    if (I[a] < axis_len(s, a) - 1 && fl[q + st]) {
      sum = rn_add(sum, x[q + st]);
      ++n;
    }
    if (I[a] > 0 && fl[q - st]) {
      sum = rn_add(sum, x[q - st]);
      ++n;
    }
  }
  return n;
}

__global__ void k_mask0(long n, const float* __restrict__ mask, uint8_t* __restrict__ fl) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    fl[q] = mask[q] > 0.f ? 0 : 1;
}

template <int D>
__global__ void k_downsample(Shape sf, const uint8_t* __restrict__ ff, Shape sc, uint8_t* __restrict__ fc) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < sc.size(); q += (long)gridDim.x * blockDim.x) {
    int I[3];
    idx3(sc, q, I);
    uint8_t any = 0;
    for (int d0 = 0; d0 < 2; ++d0)
      for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < (D == 3 ? 2 : 1); ++d2) any |= ff[sf.idx(2 * I[0] + d0, 2 * I[1] + d1, D == 3 ? 2 * I[2] + d2 : 0)];
    fc[q] = any;
  }
}

// z = (r + sum) / n with div_nd (rounded as the IEEE quotient)
template <typename T, int D>
__device__ __forceinline__ void smooth_at(const Shape& s, T* z, const T* r, const uint8_t* fl, const int* I, long q) {
  if (!fl[q]) return;
  T sum;
  const int n = fluid_nbrs<T, D>(z, fl, s, I, q, sum);
  z[q] = div_nd(rn_add(r[q], sum), n);
}

template <typename T, int D>
__device__ __forceinline__ void smooth_cell(const Shape& s, T* z, const T* r, const uint8_t* fl, long q, int phase) {
  int I[3];
  idx3(s, q, I);
  if (((I[0] + I[1] + I[2]) & 1) != phase) return;
  smooth_at<T, D>(s, z, r, fl, I, q);
}

// grid-wide half-sweep: one thread per cell of the colour (row = blockIdx.y
// (and .z in 3D), the fastest axis holding every other cell)
template <typename T, int D>
__global__ void k_smooth(Shape s, T* __restrict__ z, const T* __restrict__ r, const uint8_t* __restrict__ fl,
                         int phase, const State* __restrict__ st) {
  if (st && st->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int I[3];
  if (D == 3) {
    I[0] = blockIdx.z;
    I[1] = blockIdx.y;
    I[2] = 2 * t + ((I[0] + I[1] + phase) & 1);
    if (I[2] >= s.s2) return;
  } else {
    I[0] = blockIdx.y;
    I[1] = 2 * t + ((I[0] + phase) & 1);
    I[2] = 0;
    if (I[1] >= s.s1) return;
  }
  smooth_at<T, D>(s, z, r, fl, I, s.idx(I[0], I[1], I[2]));
}

// launch shape of k_smooth for a level
inline void smooth_grid(const Shape& s, int dim, dim3& grid, dim3& block) {
  const int row = dim == 3 ? s.s2 : s.s1, half = (row + 1) / 2;
  block = dim3(half >= 128 ? 128 : 32 * ((half + 31) / 32));
  grid = dim3((half + block.x - 1) / block.x, dim == 3 ? s.s1 : s.s0, dim == 3 ? s.s0 : 1);
}

template <typename T, int D>
__device__ __forceinline__ void restrict_cell(const Shape& sf, const T* z, const T* r, const uint8_t* fl,
                                              const Shape& sc, T* rc, T* zc, long qc) {
  const T scale = (T)(1.0 / (D - 1.0));
  int C[3];
  idx3(sc, qc, C);
  T acc = (T)0;
  for (int d0 = 0; d0 < 2; ++d0)
    for (int d1 = 0; d1 < 2; ++d1)
      for (int d2 = 0; d2 < (D == 3 ? 2 : 1); ++d2) {
        int I[3] = {2 * C[0] + d0, 2 * C[1] + d1, D == 3 ? 2 * C[2] + d2 : 0};
        const long q = sf.idx(I[0], I[1], I[2]);
        if (!fl[q]) continue;
        T sum;
        const T n = (T)fluid_nbrs<T, D>(z, fl, sf, I, q, sum);
        const T res = rn_sub(r[q], rn_sub(rn_mul(n, z[q]), sum));
        acc = rn_add(acc, rn_mul(res, scale));
      }
  rc[qc] = acc;
  zc[qc] = (T)0;
}

// The levels lc..L-1 of a V-cycle in one CTA, staged in shared memory: the
// residual of level lc and every level's fluid flags are loaded, the
// down-sweeps (with restriction), the bottom sweeps and the up-sweeps (with
// prolongation) run on shared arrays with block barriers between dependent
// steps, and z of level lc is written back for the prolongation into lc - 1.
// z[lc] starts at zero.  The same operations in the same order as the
// grid-wide kernels, so the V-cycle is unchanged bit for bit.
struct CoarseLevels {
  int lc, L, pre_post, bottom, mode;
  Shape sh[16];
  const void* r_lc;
  void* z_lc;
  const uint8_t* fl[16];
};

template <typename T>
constexpr size_t coarse_cell_bytes() { return 2 * sizeof(T) + 1; }

template <typename T, int D>
__device__ __forceinline__ void sweep_block(const Shape& s, T* z, const T* r, const uint8_t* fl, int phase) {
  for (long q = threadIdx.x; q < s.size(); q += blockDim.x) smooth_cell<T, D>(s, z, r, fl, q, phase);
  __syncthreads();
}

template <typename T, int D>
__global__ void __launch_bounds__(kBottomThreads) k_coarse(CoarseLevels c, const State* __restrict__ st) {
  if (st && st->done) return;
  extern __shared__ __align__(16) unsigned char smem[];
  T* zs[16];
  T* rs[16];
  uint8_t* fs[16];
  {
    T* p = (T*)smem;
    for (int l = c.lc; l < c.L; ++l) {
      zs[l] = p;
      p += c.sh[l].size();
      rs[l] = p;
      p += c.sh[l].size();
    }
    uint8_t* f = (uint8_t*)p;
    for (int l = c.lc; l < c.L; ++l) {
      fs[l] = f;
      f += c.sh[l].size();
    }
  }
  for (int l = c.lc; l < c.L; ++l)
    for (long q = threadIdx.x; q < c.sh[l].size(); q += blockDim.x) fs[l][q] = c.fl[l][q];
  for (long q = threadIdx.x; q < c.sh[c.lc].size(); q += blockDim.x) {
    rs[c.lc][q] = ((const T*)c.r_lc)[q];
    zs[c.lc][q] = (T)0;
  }
  __syncthreads();
  for (int l = c.lc; l < c.L - 1; ++l) {
    for (int i = 0; i < c.pre_post; ++i)
      for (int ph = 0; ph < 2; ++ph) sweep_block<T, D>(c.sh[l], zs[l], rs[l], fs[l], ph);
    for (long q = threadIdx.x; q < c.sh[l + 1].size(); q += blockDim.x)
      restrict_cell<T, D>(c.sh[l], zs[l], rs[l], fs[l], c.sh[l + 1], rs[l + 1], zs[l + 1], q);
    __syncthreads();
  }
  const int b = c.L - 1;
  const int pairs = c.mode == 1 ? c.bottom / 2 : c.bottom;
  for (int pass = 0; pass < (c.mode == 1 ? 2 : 1); ++pass)
    for (int it = 0; it < pairs; ++it)
      for (int h = 0; h < 2; ++h) sweep_block<T, D>(c.sh[b], zs[b], rs[b], fs[b], pass == 0 ? h : 1 - h);
  for (int l = c.L - 2; l >= c.lc; --l) {
    const Shape s = c.sh[l], sc = c.sh[l + 1];
    for (long q = threadIdx.x; q < s.size(); q += blockDim.x) {
      int I[3];
      idx3(s, q, I);
      zs[l][q] = rn_add(zs[l][q], zs[l + 1][sc.idx(I[0] / 2, I[1] / 2, D == 3 ? I[2] / 2 : 0)]);
    }
    __syncthreads();
    for (int i = 0; i < c.pre_post; ++i)
      for (int ph = 1; ph >= 0; --ph) sweep_block<T, D>(s, zs[l], rs[l], fs[l], ph);
  }
  for (long q = threadIdx.x; q < c.sh[c.lc].size(); q += blockDim.x) ((T*)c.z_lc)[q] = zs[c.lc][q];
}

// r_c = sum over fluid children (lexicographic) of (r - (n z - sum)) / (dim - 1); z_c = 0
template <typename T, int D>
__global__ void k_restrict(Shape sf, const T* __restrict__ z, const T* __restrict__ r, const uint8_t* __restrict__ fl,
                           Shape sc, T* __restrict__ rc, T* __restrict__ zc, const State* __restrict__ st) {
  if (st && st->done) return;
  for (long qc = (long)blockIdx.x * blockDim.x + threadIdx.x; qc < sc.size(); qc += (long)gridDim.x * blockDim.x)
    restrict_cell<T, D>(sf, z, r, fl, sc, rc, zc, qc);
}

template <typename T, int D>
__global__ void k_prolong(Shape s, T* __restrict__ z, Shape sc, const T* __restrict__ zc, const State* __restrict__ st) {
  if (st && st->done) return;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < s.size(); q += (long)gridDim.x * blockDim.x) {
    int I[3];
    idx3(s, q, I);
    z[q] = rn_add(z[q], zc[sc.idx(I[0] / 2, I[1] / 2, D == 3 ? I[2] / 2 : 0)]);
  }
}

template <typename T>
__global__ void k_fill(long n, T* __restrict__ x, const State* __restrict__ st) {
  if (st && st->done) return;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) x[q] = (T)0;
}

// ----------------------------------------------------------------- PCG pieces
template <typename T>
__device__ __forceinline__ void block_sum_to(double acc, double* part) {
  __shared__ double red[kThreads];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// part = sum a b over fluid cells (fl == nullptr: over all cells, b unused)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dot(long n, const T* __restrict__ a, const T* __restrict__ b,
                                                  const uint8_t* __restrict__ fl, double* __restrict__ part,
                                                  const State* __restrict__ st) {
  if (st->done) return;
  double acc = 0.0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    if (fl == nullptr) acc += (double)a[q];
    else if (fl[q]) acc += (double)a[q] * (double)b[q];
  }
  block_sum_to<T>(acc, part);
}

constexpr int kFinThreads = 256;

// which: 0 initial zTr (tolerance), 1 alpha, 2 rTr (convergence), 3 mean of r,
// 4 beta (and the iteration count).  The partials are summed in a fixed order
// (strided per thread, then a tree), so the result is deterministic.
__global__ void __launch_bounds__(kFinThreads) k_fin(int which, const double* __restrict__ part,
                                                     State* __restrict__ st, long ncells) {
  if (st->done) return;
  __shared__ double red[kFinThreads];
  double a = 0.0;
  for (int b = threadIdx.x; b < kRedBlocks; b += kFinThreads) a += part[b];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int h = kFinThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double s = red[0];
  if (which == 0) {
    st->old_zr = s;
    st->tol = fmax(st->abs_tol, s * st->rel_tol);
    if (s == 0.0) {  // r = 0: the zero start is the solution (and alpha would be 0 / 0 with eps = 0)
      st->done = 1;
      st->converged = 1;
    }
  } else if (which == 1) {
    st->pAp = s;
    st->alpha = st->old_zr / (s + st->eps);
  } else if (which == 2) {
    st->rtr = s;
    if (!isfinite(s)) {
      st->done = 1;
    } else if (s < st->tol) {
      st->done = 1;
      st->converged = 1;
    }
  } else if (which == 3) {
    st->mean = s / (double)ncells;
  } else {
    st->new_zr = s;
    st->beta = s / (st->old_zr + st->eps);
    st->old_zr = s;
    st->iters += 1;
    if (st->iters >= st->max_iters) st->done = 1;
  }
}

template <typename T>
__global__ void k_recenter(long n, T* __restrict__ r, const State* __restrict__ st) {
  if (st->done) return;
  const T m = (T)st->mean;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) r[q] = r[q] - m;
}

template <typename T, int D>
__global__ void k_Ap(Shape s, const T* __restrict__ p, const uint8_t* __restrict__ fl, T* __restrict__ Ap,
                     const State* __restrict__ st) {
  if (st->done) return;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < s.size(); q += (long)gridDim.x * blockDim.x) {
    if (!fl[q]) {
      Ap[q] = (T)0;
      continue;
    }
    int I[3];
    idx3(s, q, I);
    T sum;
    const T n = (T)fluid_nbrs<T, D>(p, fl, s, I, q, sum);
    Ap[q] = rn_sub(rn_mul(n, p[q]), sum);
  }
}

template <typename T>
__global__ void k_update_xr(long n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                            const T* __restrict__ Ap, const uint8_t* __restrict__ fl, const State* __restrict__ st) {
  if (st->done) return;
  const T alpha = (T)st->alpha;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    if (!fl[q]) continue;
    x[q] = rn_add(x[q], rn_mul(alpha, p[q]));
    r[q] = rn_sub(r[q], rn_mul(alpha, Ap[q]));
  }
}

template <typename T>
__global__ void k_update_p(long n, T* __restrict__ p, const T* __restrict__ z, const uint8_t* __restrict__ fl,
                           const State* __restrict__ st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    if (fl[q]) p[q] = rn_add(z[q], rn_mul(beta, p[q]));
}

template <typename T>
__global__ void k_init(long n, const T* __restrict__ b, T k, T* __restrict__ r, T* __restrict__ x, T* __restrict__ p) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    r[q] = b[q] * k;
    x[q] = (T)0;
    p[q] = (T)0;
  }
}

// ----------------------------------------------------------------- projection
// zero the domain walls and the faces of solid cells
template <typename T, int D>
__global__ void k_bc(fm_grid g, int c, T* __restrict__ u, const uint8_t* __restrict__ fl) {
  const Shape fs = face_shape(g, c), cs = cell_shape(g);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < fs.size(); q += (long)gridDim.x * blockDim.x) {
    int I[3];
    idx3(fs, q, I);
    bool zero = I[c] == 0 || I[c] == axis_len(fs, c) - 1;
    if (!zero && I[c] < axis_len(cs, c) && !fl[cs.idx(I[0], I[1], I[2])]) zero = true;
    if (!zero && I[c] >= 1) {
      int J[3] = {I[0], I[1], I[2]};
      J[c] -= 1;
      if (!fl[cs.idx(J[0], J[1], J[2])]) zero = true;
    }
    if (zero) u[q] = (T)0;
  }
}

template <typename T, int D>
__global__ void k_div(fm_grid g, const T* __restrict__ ux, const T* __restrict__ uy, const T* __restrict__ uz,
                      const uint8_t* __restrict__ fl, T* __restrict__ div) {
  const Shape cs = cell_shape(g);
  const T* u[3] = {ux, uy, uz};
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < cs.size(); q += (long)gridDim.x * blockDim.x) {
    if (!fl[q]) {
      div[q] = (T)0;
      continue;
    }
    int I[3];
    idx3(cs, q, I);
    T acc = (T)0;
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const Shape fs = face_shape(g, c);
      int J[3] = {I[0], I[1], I[2]};
      const T vl = u[c][fs.idx(J[0], J[1], J[2])];
      J[c] += 1;
      const T vr = u[c][fs.idx(J[0], J[1], J[2])];
      acc = c == 0 ? rn_sub(vr, vl) : rn_sub(rn_add(acc, vr), vl);
    }
    div[q] = acc;
  }
}

// u -= p(I) - p(I - e_c), p = 0 outside (the walls are zeroed by the next k_bc)
template <typename T, int D>
__global__ void k_grad(fm_grid g, int c, T* __restrict__ u, const T* __restrict__ p) {
  const Shape fs = face_shape(g, c), cs = cell_shape(g);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < fs.size(); q += (long)gridDim.x * blockDim.x) {
    int I[3];
    idx3(fs, q, I);
    T pr = (T)0, pl = (T)0;
    if (I[c] < axis_len(cs, c)) pr = p[cs.idx(I[0], I[1], I[2])];
    if (I[c] >= 1) {
      I[c] -= 1;
      pl = p[cs.idx(I[0], I[1], I[2])];
    }
    u[q] = rn_sub(u[q], rn_sub(pr, pl));
  }
}

// ----------------------------------------------------------------- mask kernels
template <typename T, int D>
__global__ void k_mask_velocity(fm_grid g, int c, const float* __restrict__ mask, const T* __restrict__ bvel,
                                T* __restrict__ u) {
  const Shape fs = face_shape(g, c), cs = cell_shape(g);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < fs.size(); q += (long)gridDim.x * blockDim.x) {
    int I[3];
    idx3(fs, q, I);
    long cell = -1;
    if (I[c] < axis_len(cs, c) && mask[cs.idx(I[0], I[1], I[2])] >= 1.f) {
      cell = cs.idx(I[0], I[1], I[2]);  // the cell on the face's high side
    } else if (I[c] >= 1) {
      int J[3] = {I[0], I[1], I[2]};
      J[c] -= 1;
      if (mask[cs.idx(J[0], J[1], J[2])] >= 1.f) cell = cs.idx(J[0], J[1], J[2]);
    }
    if (cell >= 0) u[q] = bvel ? bvel[(long)c * cs.size() + cell] : (T)0;
  }
}

template <typename T, int D>
__global__ void k_mask_passive(fm_grid g, const float* __restrict__ mask, T* __restrict__ s, int adjoint) {
  const Shape cs = cell_shape(g);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < cs.size(); q += (long)gridDim.x * blockDim.x) {
    if (!(mask[q] >= 1.f)) continue;
    if (adjoint) {
      s[q] = (T)0;
      continue;
    }
    int I[3];
    idx3(cs, q, I);
    T acc = (T)0, w = (T)0;
    for (int d0 = -1; d0 <= 1; ++d0)
      for (int d1 = -1; d1 <= 1; ++d1)
        for (int d2 = (D == 3 ? -1 : 0); d2 <= (D == 3 ? 1 : 0); ++d2) {
          const int a = I[0] + d0, b = I[1] + d1, k = I[2] + d2;
          if (a < 0 || b < 0 || k < 0 || a >= cs.s0 || b >= cs.s1 || k >= cs.s2) continue;
          const long nq = cs.idx(a, b, k);
          if (mask[nq] <= 0.f) {  // fluid neighbours are never written here
            acc = rn_add(acc, s[nq]);
            w = w + (T)1;
          }
        }
    s[q] = w > (T)0 ? acc / w : acc;
  }
}

}  // namespace solid
}  // namespace fm

// ----------------------------------------------------------------- handle
struct fm_solid {
  fm_grid g;
  int dtype, dim, levels;
  fm_mg_params P;
  fm::Shape sh[16];
  void* r[16];
  void* z[16];
  uint8_t* fl[16];
  void *x, *p, *Ap, *div;
  double* part;
  fm::solid::State* st;
  fm::solid::State* st_host;  // pinned
  fm::solid::Stats* stats;
  fm::solid::Stats* stats_host;  // pinned
  // check_every PCG iterations captured once as a graph (replayed per poll)
  cudaStream_t cap;
  cudaGraphExec_t chunk;
  size_t chunk_nodes;
  // device mode (check_every == 0): a graph with a conditional WHILE node
  cudaGraphExec_t loop;
  long long loop_kernels;  // kernels per loop body
};

namespace fm {
namespace solid {

inline unsigned blocks_for(long n) {
  long b = (n + kThreads - 1) / kThreads;
  if (b > 148L * 16) b = 148L * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

template <typename T, int D>
inline void launch_smooth(const Shape& sh, cudaStream_t s, T* z, const T* r, const uint8_t* fl, int phase,
                          const State* st) {
  dim3 grid, block;
  smooth_grid(sh, D, grid, block);
  launch(k_smooth<T, D>, grid, block, 0, s, sh, z, r, fl, phase, st);
}

// first level from which the remaining levels fit the coarse kernel's shared
// memory (L when not even the coarsest one does)
template <typename T>
int coarse_start(const fm_solid* S, size_t* bytes) {
  size_t acc = 0;
  int lc = S->levels;
  for (int l = S->levels - 1; l >= 0; --l) {
    const size_t need = acc + (size_t)S->sh[l].size() * coarse_cell_bytes<T>();
    if (need > kCoarseSmem) break;
    acc = need;
    lc = l;
  }
  *bytes = acc;
  return lc;
}

template <typename T, int D>
void vcycle(fm_solid* S, cudaStream_t s, const State* st) {
  size_t smem = 0;
  const int L = S->levels, lc = coarse_start<T>(S, &smem);
  launch(k_fill<T>, blocks_for(S->sh[0].size()), kThreads, 0, s, S->sh[0].size(), (T*)S->z[0], st);
  const int down = lc < L ? lc : L - 1;  // levels smoothed and restricted by grid-wide launches
  for (int l = 0; l < down; ++l) {
    for (int i = 0; i < S->P.pre_post; ++i)
      for (int ph = 0; ph < 2; ++ph)
        launch_smooth<T, D>(S->sh[l], s, (T*)S->z[l], (const T*)S->r[l],
               (const uint8_t*)S->fl[l], ph, st);
    launch(k_restrict<T, D>, blocks_for(S->sh[l + 1].size()), kThreads, 0, s, S->sh[l], (const T*)S->z[l],
           (const T*)S->r[l], (const uint8_t*)S->fl[l], S->sh[l + 1], (T*)S->r[l + 1], (T*)S->z[l + 1], st);
  }
  if (lc < L) {
    CoarseLevels c;
    c.lc = lc;
    c.L = L;
    c.pre_post = S->P.pre_post;
    c.bottom = S->P.bottom;
    c.mode = S->P.bottom_mode;
    c.r_lc = S->r[lc];
    c.z_lc = S->z[lc];
    for (int l = 0; l < L; ++l) {
      c.sh[l] = S->sh[l];
      c.fl[l] = S->fl[l];
    }
    launch(k_coarse<T, D>, 1, kBottomThreads, smem, s, c, st);
  } else {
    // even the coarsest level is large: its bottom sweeps as grid-wide launches
    const int b = L - 1;
    const int pairs = S->P.bottom_mode == 1 ? S->P.bottom / 2 : S->P.bottom;
    for (int pass = 0; pass < (S->P.bottom_mode == 1 ? 2 : 1); ++pass)
      for (int it = 0; it < pairs; ++it)
        for (int h = 0; h < 2; ++h)
          launch_smooth<T, D>(S->sh[b], s, (T*)S->z[b], (const T*)S->r[b],
                 (const uint8_t*)S->fl[b], pass == 0 ? h : 1 - h, st);
  }
  for (int l = down - 1; l >= 0; --l) {
    launch(k_prolong<T, D>, blocks_for(S->sh[l].size()), kThreads, 0, s, S->sh[l], (T*)S->z[l], S->sh[l + 1],
           (const T*)S->z[l + 1], st);
    for (int i = 0; i < S->P.pre_post; ++i)
      for (int ph = 1; ph >= 0; --ph)
        launch_smooth<T, D>(S->sh[l], s, (T*)S->z[l], (const T*)S->r[l],
               (const uint8_t*)S->fl[l], ph, st);
  }
}

// The second half of a PCG iteration (2D/vortex/mgpcg_solid.py solve(), :318-363):
// x += alpha p, r -= alpha A p and the convergence test; every kernel frozen once
// st->done is set.
template <typename T, int D>
void step(fm_solid* S, cudaStream_t s) {
  const long n = S->sh[0].size();
  const unsigned nb = blocks_for(n);
  State* st = S->st;
  T* r = (T*)S->r[0];
  T* p = (T*)S->p;
  T* Ap = (T*)S->Ap;
  const uint8_t* fl = S->fl[0];
  launch(k_Ap<T, D>, nb, kThreads, 0, s, S->sh[0], (const T*)p, fl, Ap, (const State*)st);
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)p, (const T*)Ap, fl, S->part, (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 1, (const double*)S->part, st, n);
  launch(k_update_xr<T>, nb, kThreads, 0, s, n, (T*)S->x, r, (const T*)p, (const T*)Ap, fl, (const State*)st);
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)r, (const T*)r, fl, S->part, (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 2, (const double*)S->part, st, n);
}

// One PCG iteration, rotated so that the convergence test ends it: recentre r,
// z = M r, beta, p = z + beta p, then the next x / r update and its test (step).
// A converged solve leaves the loop right after its test; the kernels run in
// the order of the unrotated loop, so results are unchanged.
template <typename T, int D>
void iteration(fm_solid* S, cudaStream_t s) {
  const long n = S->sh[0].size();
  const unsigned nb = blocks_for(n);
  State* st = S->st;
  T* r = (T*)S->r[0];
  T* p = (T*)S->p;
  const uint8_t* fl = S->fl[0];
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)r, (const T*)nullptr, (const uint8_t*)nullptr, S->part,
         (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 3, (const double*)S->part, st, n);
  launch(k_recenter<T>, nb, kThreads, 0, s, n, r, (const State*)st);
  vcycle<T, D>(S, s, st);
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)S->z[0], (const T*)r, fl, S->part, (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 4, (const double*)S->part, st, n);
  launch(k_update_p<T>, nb, kThreads, 0, s, n, p, (const T*)S->z[0], fl, (const State*)st);
  step<T, D>(S, s);
}

// The PCG loop as a conditional WHILE node appended to `graph` after `deps`
// (the body, one iteration and k_loop_cond, recorded from S->cap), preceded by
// k_loop_init; *node_out receives the node.  `capturing`: the caller's stream
// when `graph` is the graph it is recording (k_loop_init is then recorded from
// that stream and the node follows the stream's current dependencies).
template <typename T, int D>
int add_loop_node(fm_solid* S, cudaGraph_t graph, const cudaGraphNode_t* deps, size_t ndeps, cudaGraphNode_t* node_out,
                  cudaStream_t capturing) {
  cudaGraphConditionalHandle h;
  cudaError_t e;
  if ((e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return cuda_fail(e);
  // k_loop_init ahead of the node: recorded from the capturing stream inside a
  // caller's capture, else added as a kernel node
  cudaGraphNode_t init;
  if (capturing) {
    k_loop_init<<<1, 1, 0, capturing>>>(h, S->st);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e);
    cudaStreamCaptureStatus cs;
    if ((e = cudaStreamGetCaptureInfo(capturing, &cs, nullptr, &graph, &deps, &ndeps)) != cudaSuccess)
      return cuda_fail(e);
    if (cs != cudaStreamCaptureStatusActive) return cuda_fail(cudaErrorStreamCaptureInvalidated);
  } else {
    cudaKernelNodeParams kp = {};
    State* st_arg = S->st;
    void* kargs[2] = {&h, &st_arg};
    kp.func = (void*)k_loop_init;
    kp.gridDim = dim3(1, 1, 1);
    kp.blockDim = dim3(1, 1, 1);
    kp.kernelParams = kargs;
    if ((e = cudaGraphAddKernelNode(&init, graph, deps, ndeps, &kp)) != cudaSuccess) return cuda_fail(e);
    deps = &init;
    ndeps = 1;
  }
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if ((e = cudaGraphAddNode(node_out, graph, deps, ndeps, &cp)) != cudaSuccess) return cuda_fail(e);
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(S->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return cuda_fail(e);
  const long long before = g_launch_count.load();
  iteration<T, D>(S, S->cap);
  launch(k_loop_cond, 1, 1, 0, S->cap, h, S->st, S->stats);
  S->loop_kernels = g_launch_count.load() - before;
  g_launch_count.fetch_sub(S->loop_kernels);  // counted per body run (fm_solid_stats)
  cudaGraph_t captured = nullptr;
  if ((e = cudaStreamEndCapture(S->cap, &captured)) != cudaSuccess) return cuda_fail(e);
  return FM_OK;
}

// Device mode: the PCG loop without host polling.  Outside a capture it is one
// launch of a graph built once; inside a caller's capture the WHILE node is
// appended to the graph being recorded.
template <typename T, int D>
int device_loop(fm_solid* S, cudaStream_t s, bool capturing) {
  if (capturing) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e;
    if ((e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps)) != cudaSuccess) return cuda_fail(e);
    cudaGraphNode_t node;
    const int st = add_loop_node<T, D>(S, graph, deps, ndeps, &node, s);
    if (st) return st;
    if ((e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
      return cuda_fail(e);
    return FM_OK;
  }
  if (!S->loop) {
    cudaGraph_t graph = nullptr;
    cudaError_t e;
    if ((e = cudaGraphCreate(&graph, 0)) != cudaSuccess) return cuda_fail(e);
    cudaGraphNode_t node;
    int st = add_loop_node<T, D>(S, graph, nullptr, 0, &node, nullptr);
    if (!st && (e = cudaGraphInstantiate(&S->loop, graph, 0)) != cudaSuccess) {
      S->loop = nullptr;
      st = cuda_fail(e);
    }
    cudaGraphDestroy(graph);
    if (st) return st;
  }
  cudaError_t e;
  if ((e = cudaGraphLaunch(S->loop, s)) != cudaSuccess) return cuda_fail(e);
  return FM_OK;
}

template <typename T, int D>
int solve(fm_solid* S, const void* b, double k, void* x, cudaStream_t s, int* iters, double* rtr) {
  // check_every == 0: device-side loop (capturable into a caller's graph when
  // no outcome is read back); otherwise the host polls every check_every
  // iterations, which cannot be recorded
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return FM_ERR_CUDA;
  const bool capturing = cs != cudaStreamCaptureStatusNone;
  const bool device = S->P.check_every == 0;
  if (capturing && (!device || iters || rtr)) return FM_ERR_ARG;
  const long n = S->sh[0].size();
  launch(k_state_init, 1, 1, 0, s, S->st, S->P.max_iters, S->P.abs_tol, S->P.rel_tol, S->P.eps);
  State* st = S->st;
  T* r = (T*)S->r[0];
  T* z = (T*)S->z[0];
  T* p = (T*)S->p;
  T* xs = (T*)S->x;
  const uint8_t* fl = S->fl[0];
  const unsigned nb = blocks_for(n);
  launch(k_init<T>, nb, kThreads, 0, s, n, (const T*)b, (T)k, r, xs, p);
  // recenter, precondition, p = z, zTr
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)r, (const T*)nullptr, (const uint8_t*)nullptr, S->part,
         (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 3, (const double*)S->part, st, n);
  launch(k_recenter<T>, nb, kThreads, 0, s, n, r, (const State*)st);
  vcycle<T, D>(S, s, st);
  launch(k_update_p<T>, nb, kThreads, 0, s, n, p, (const T*)z, fl, (const State*)st);
  launch(k_dot<T>, kRedBlocks, kThreads, 0, s, n, (const T*)z, (const T*)r, fl, S->part, (const State*)st);
  launch(k_fin, 1, kFinThreads, 0, s, 0, (const double*)S->part, st, n);
  step<T, D>(S, s);  // the first x / r update and its convergence test
  if (device) {
    const int dl = device_loop<T, D>(S, s, capturing);
    if (dl) return dl;
    launch(k_stats, 1, 1, 0, s, (const State*)st, S->stats);
    if (x != nullptr && x != S->x) cudaMemcpyAsync(x, S->x, n * sizeof(T), cudaMemcpyDeviceToDevice, s);
    if (!iters && !rtr) return check_cuda();  // asynchronous: the outcome goes to fm_solid_stats
    if (cudaMemcpyAsync(S->st_host, st, sizeof(State), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    if (iters) *iters = S->st_host->iters;
    if (rtr) *rtr = S->st_host->rtr;
    const int cst = check_cuda();
    if (cst) return cst;
    if (!isfinite(S->st_host->rtr)) return FM_ERR_NONFINITE;
    return S->st_host->converged ? FM_OK : FM_ERR_NOT_CONVERGED;
  }
  const int every = S->P.check_every;
  if (!S->chunk) {
    // capture check_every iterations once; the captured kernels are counted per replay
    const long long before = g_launch_count.load();
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FM_ERR_CUDA;
    for (int i = 0; i < every; ++i) iteration<T, D>(S, S->cap);
    if (cudaStreamEndCapture(S->cap, &graph) != cudaSuccess) return FM_ERR_CUDA;
    g_launch_count.store(before);
    if (cudaGraphGetNodes(graph, nullptr, &S->chunk_nodes) != cudaSuccess ||
        cudaGraphInstantiate(&S->chunk, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      return FM_ERR_CUDA;
    }
    cudaGraphDestroy(graph);
  }
  for (int it = 0; it < S->P.max_iters; it += every) {
    if (cudaGraphLaunch(S->chunk, s) != cudaSuccess) return FM_ERR_CUDA;
    count_launch((long long)S->chunk_nodes);
    if (cudaMemcpyAsync(S->st_host, st, sizeof(State), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
    if (S->st_host->done) break;
  }
  launch(k_stats, 1, 1, 0, s, (const State*)st, S->stats);
  if (cudaMemcpyAsync(S->st_host, st, sizeof(State), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FM_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
  if (x != nullptr && x != S->x) cudaMemcpyAsync(x, S->x, n * sizeof(T), cudaMemcpyDeviceToDevice, s);
  if (iters) *iters = S->st_host->iters;
  if (rtr) *rtr = S->st_host->rtr;
  const int cst = check_cuda();
  if (cst) return cst;
  if (!isfinite(S->st_host->rtr)) return FM_ERR_NONFINITE;
  return S->st_host->converged ? FM_OK : FM_ERR_NOT_CONVERGED;
}

template <typename T, int D>
int project(fm_solid* S, void* const* u, void* p_out, cudaStream_t s, int* iters, double* rtr) {
  const fm_grid& g = S->g;
  for (int c = 0; c < D; ++c)
    launch(k_bc<T, D>, blocks_for(face_shape(g, c).size()), kThreads, 0, s, g, c, (T*)u[c], (const uint8_t*)S->fl[0]);
  launch(k_div<T, D>, blocks_for(S->sh[0].size()), kThreads, 0, s, g, (const T*)u[0], (const T*)u[1],
         (const T*)(D == 3 ? u[2] : nullptr), (const uint8_t*)S->fl[0], (T*)S->div);
  const int st = solve<T, D>(S, S->div, -1.0, nullptr, s, iters, rtr);
  if (st != FM_OK && st != FM_ERR_NOT_CONVERGED && st != FM_ERR_NONFINITE) return st;
  for (int c = 0; c < D; ++c) {
    launch(k_grad<T, D>, blocks_for(face_shape(g, c).size()), kThreads, 0, s, g, c, (T*)u[c], (const T*)S->x);
    launch(k_bc<T, D>, blocks_for(face_shape(g, c).size()), kThreads, 0, s, g, c, (T*)u[c], (const uint8_t*)S->fl[0]);
  }
  if (p_out) cudaMemcpyAsync(p_out, S->x, S->sh[0].size() * sizeof(T), cudaMemcpyDeviceToDevice, s);
  const int cst = check_cuda();
  return cst ? cst : st;
}

}  // namespace solid
}  // namespace fm

extern "C" {

int fm_solid_destroy(fm_solid* S) {
  if (!S) return FM_OK;
  for (int l = 0; l < S->levels; ++l) {
    cudaFree(S->r[l]);
    cudaFree(S->z[l]);
    cudaFree(S->fl[l]);
  }
  cudaFree(S->x);
  cudaFree(S->p);
  cudaFree(S->Ap);
  cudaFree(S->div);
  cudaFree(S->part);
  cudaFree(S->st);
  cudaFree(S->stats);
  if (S->st_host) cudaFreeHost(S->st_host);
  if (S->stats_host) cudaFreeHost(S->stats_host);
  if (S->chunk) cudaGraphExecDestroy(S->chunk);
  if (S->loop) cudaGraphExecDestroy(S->loop);
  if (S->cap) cudaStreamDestroy(S->cap);
  free(S);
  return FM_OK;
}

int fm_solid_set_mask(fm_solid* S, const float* mask, void* stream) {
  using namespace fm::solid;
  if (!S || !mask) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  fm::launch(k_mask0, blocks_for(S->sh[0].size()), kThreads, 0, s, S->sh[0].size(), mask, S->fl[0]);
  for (int l = 1; l < S->levels; ++l) {
    if (S->dim == 2)
      fm::launch(k_downsample<2>, blocks_for(S->sh[l].size()), kThreads, 0, s, S->sh[l - 1], (const uint8_t*)S->fl[l - 1],
                 S->sh[l], S->fl[l]);
    else
      fm::launch(k_downsample<3>, blocks_for(S->sh[l].size()), kThreads, 0, s, S->sh[l - 1], (const uint8_t*)S->fl[l - 1],
                 S->sh[l], S->fl[l]);
  }
  return fm::check_cuda();
}

int fm_solid_create(const fm_grid* g, int dtype, const fm_mg_params* params, const float* mask, fm_solid** out) {
  using namespace fm;
  if (!out || !params) return FM_ERR_ARG;
  *out = nullptr;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  const fm_mg_params& P = *params;
  if (P.levels < 1 || P.levels > 16 || P.pre_post < 0 || P.bottom < 0 || P.max_iters < 1 || P.check_every < 0 ||
      (P.bottom_mode != 0 && P.bottom_mode != 1) || P.coarse_bf16)
    return FM_ERR_ARG;
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] % (1 << (P.levels - 1)) != 0) return FM_ERR_SHAPE;
  fm_solid* S = (fm_solid*)calloc(1, sizeof(fm_solid));
  if (!S) return FM_ERR_CUDA;
  S->g = *g;
  S->dtype = dtype;
  S->dim = g->dim;
  S->levels = P.levels;
  S->P = P;
  const size_t es = dtype == FM_F32 ? 4 : 8;
  bool ok = true;
  for (int l = 0; l < P.levels; ++l) {
    Shape sh{g->n[0] >> l, g->n[1] >> l, g->dim == 3 ? g->n[2] >> l : 1};
    S->sh[l] = sh;
    ok = ok && cudaMalloc(&S->r[l], sh.size() * es) == cudaSuccess;
    ok = ok && cudaMalloc(&S->z[l], sh.size() * es) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&S->fl[l], sh.size()) == cudaSuccess;
  }
  const long n = S->sh[0].size();
  ok = ok && cudaMalloc(&S->x, n * es) == cudaSuccess && cudaMalloc(&S->p, n * es) == cudaSuccess &&
       cudaMalloc(&S->Ap, n * es) == cudaSuccess && cudaMalloc(&S->div, n * es) == cudaSuccess &&
       cudaMalloc((void**)&S->part, solid::kRedBlocks * sizeof(double)) == cudaSuccess &&
       cudaMalloc((void**)&S->st, sizeof(solid::State)) == cudaSuccess &&
       cudaMallocHost((void**)&S->st_host, sizeof(solid::State)) == cudaSuccess &&
       cudaMalloc((void**)&S->stats, sizeof(solid::Stats)) == cudaSuccess &&
       cudaMallocHost((void**)&S->stats_host, sizeof(solid::Stats)) == cudaSuccess &&
       cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking) == cudaSuccess;
  if (ok) ok = cudaMemset(S->stats, 0, sizeof(solid::Stats)) == cudaSuccess;
  if (!ok) {
    fm_solid_destroy(S);
    return FM_ERR_CUDA;
  }
  // the coarse-levels kernel may use more than the default 48 KB of shared memory
  if (dtype == FM_F32)
    cudaFuncSetAttribute(g->dim == 2 ? solid::k_coarse<float, 2> : solid::k_coarse<float, 3>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solid::kCoarseSmem);
  else
    cudaFuncSetAttribute(g->dim == 2 ? solid::k_coarse<double, 2> : solid::k_coarse<double, 3>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solid::kCoarseSmem);
  if (mask) {
    const int ms = fm_solid_set_mask(S, mask, nullptr);
    if (ms == FM_OK) cudaDeviceSynchronize();
    if (ms != FM_OK) {
      fm_solid_destroy(S);
      return ms;
    }
  } else {
    for (int l = 0; l < P.levels; ++l) cudaMemset(S->fl[l], 1, S->sh[l].size());
  }
  *out = S;
  return check_cuda();
}

int fm_solid_stats(fm_solid* S, void* stream, int reset, fm_mg_stats* out) {
  using namespace fm::solid;
  if (!S || !out) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(S->stats_host, S->stats, sizeof(Stats), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return FM_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
  const Stats h = *S->stats_host;
  out->solves = h.solves;
  out->iterations = h.iterations;
  out->not_converged = h.not_converged;
  out->nonfinite = h.nonfinite;
  out->last_iters = h.last_iters;
  out->max_iters_seen = h.max_iters_seen;
  out->last_rtr = h.last_rtr;
  fm::count_launch(h.bodies * S->loop_kernels);  // kernels run inside device-mode loops since the last read
  Stats z = h;
  z.bodies = 0;
  if (reset) {
    z.solves = z.iterations = z.not_converged = z.nonfinite = 0;
    z.last_iters = z.max_iters_seen = 0;
    z.last_rtr = 0.0;
  }
  *S->stats_host = z;
  if (cudaMemcpyAsync(S->stats, S->stats_host, sizeof(Stats), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return FM_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FM_ERR_CUDA;
  return fm::check_cuda();
}

int fm_solid_vcycle(fm_solid* S, const void* r, void* z, void* stream) {
  using namespace fm::solid;
  if (!S || !r || !z) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = S->sh[0].size() * (S->dtype == FM_F32 ? 4 : 8);
  cudaMemcpyAsync(S->r[0], r, bytes, cudaMemcpyDeviceToDevice, s);
  if (S->dtype == FM_F32) {
    if (S->dim == 2) vcycle<float, 2>(S, s, nullptr);
    else vcycle<float, 3>(S, s, nullptr);
  } else {
    if (S->dim == 2) vcycle<double, 2>(S, s, nullptr);
    else vcycle<double, 3>(S, s, nullptr);
  }
  cudaMemcpyAsync(z, S->z[0], bytes, cudaMemcpyDeviceToDevice, s);
  return fm::check_cuda();
}

int fm_solid_solve(fm_solid* S, const void* b, void* x, void* stream, int* iters, double* rtr) {
  using namespace fm::solid;
  if (!S || !b || !x) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (S->dtype == FM_F32)
    return S->dim == 2 ? solve<float, 2>(S, b, 1.0, x, s, iters, rtr) : solve<float, 3>(S, b, 1.0, x, s, iters, rtr);
  return S->dim == 2 ? solve<double, 2>(S, b, 1.0, x, s, iters, rtr) : solve<double, 3>(S, b, 1.0, x, s, iters, rtr);
}

int fm_solid_project(fm_solid* S, void* ux, void* uy, void* uz, void* p_out, void* stream, int* iters, double* rtr) {
  using namespace fm::solid;
  if (!S || !ux || !uy || (S->dim == 3 && !uz)) return FM_ERR_ARG;
  void* u[3] = {ux, uy, uz};
  cudaStream_t s = (cudaStream_t)stream;
  if (S->dtype == FM_F32)
    return S->dim == 2 ? project<float, 2>(S, u, p_out, s, iters, rtr) : project<float, 3>(S, u, p_out, s, iters, rtr);
  return S->dim == 2 ? project<double, 2>(S, u, p_out, s, iters, rtr) : project<double, 3>(S, u, p_out, s, iters, rtr);
}

int fm_mask_velocity(const fm_grid* g, int dtype, const float* mask, const void* bvel, void* ux, void* uy, void* uz,
                     void* stream) {
  using namespace fm;
  using namespace fm::solid;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (!mask || !ux || !uy || (g->dim == 3 && !uz)) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  void* u[3] = {ux, uy, uz};
  for (int c = 0; c < g->dim; ++c) {
    const unsigned nb = blocks_for(face_shape(*g, c).size());
    if (dtype == FM_F32) {
      if (g->dim == 2) launch(k_mask_velocity<float, 2>, nb, kThreads, 0, s, *g, c, mask, (const float*)bvel, (float*)u[c]);
      else launch(k_mask_velocity<float, 3>, nb, kThreads, 0, s, *g, c, mask, (const float*)bvel, (float*)u[c]);
    } else {
      if (g->dim == 2) launch(k_mask_velocity<double, 2>, nb, kThreads, 0, s, *g, c, mask, (const double*)bvel, (double*)u[c]);
      else launch(k_mask_velocity<double, 3>, nb, kThreads, 0, s, *g, c, mask, (const double*)bvel, (double*)u[c]);
    }
  }
  return check_cuda();
}

int fm_mask_passive(const fm_grid* g, int dtype, const float* mask, void* s_field, int adjoint, void* stream) {
  using namespace fm;
  using namespace fm::solid;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (!mask || !s_field) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb = blocks_for(cell_shape(*g).size());
  if (dtype == FM_F32) {
    if (g->dim == 2) launch(k_mask_passive<float, 2>, nb, kThreads, 0, s, *g, mask, (float*)s_field, adjoint);
    else launch(k_mask_passive<float, 3>, nb, kThreads, 0, s, *g, mask, (float*)s_field, adjoint);
  } else {
    if (g->dim == 2) launch(k_mask_passive<double, 2>, nb, kThreads, 0, s, *g, mask, (double*)s_field, adjoint);
    else launch(k_mask_passive<double, 3>, nb, kThreads, 0, s, *g, mask, (double*)s_field, adjoint);
  }
  return check_cuda();
}

}  // extern "C"
