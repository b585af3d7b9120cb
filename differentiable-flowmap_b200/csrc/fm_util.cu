// fm_util.cu -- elementwise storage conversion for the trajectory stores.
//
// The mixed-precision form keeps every step's midpoint velocity and passive
// scalar in BF16 (round to nearest even) and widens them back to FP32 when the
// adjoint reads them.  bf16 -> f32 is exact, so a stored value is read back as
// exactly the BF16-rounded FP32 value.
#include <cuda_bf16.h>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

template <typename S, typename D>
__device__ __forceinline__ D cvt(S v) {
  return (D)v;
}
template <>
__device__ __forceinline__ __nv_bfloat16 cvt<float, __nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ float cvt<__nv_bfloat16, float>(__nv_bfloat16 v) {
  return __bfloat162float(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 cvt<double, __nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
template <>
__device__ __forceinline__ double cvt<__nv_bfloat16, double>(__nv_bfloat16 v) {
  return (double)__bfloat162float(v);
}

template <typename S, typename D>
__global__ void k_convert(long n, const S* __restrict__ src, D* __restrict__ dst) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    dst[q] = cvt<S, D>(src[q]);
}

template <typename S>
static int convert_from(long n, const void* src, int dst_dtype, void* dst, cudaStream_t s, unsigned blocks) {
  if (dst_dtype == FM_F32) k_convert<S, float><<<blocks, 256, 0, s>>>(n, (const S*)src, (float*)dst);
  else if (dst_dtype == FM_F64) k_convert<S, double><<<blocks, 256, 0, s>>>(n, (const S*)src, (double*)dst);
  else if (dst_dtype == FM_BF16)
    k_convert<S, __nv_bfloat16><<<blocks, 256, 0, s>>>(n, (const S*)src, (__nv_bfloat16*)dst);
  else return FM_ERR_DTYPE;
  return check_launch();
}

}  // namespace fm

using namespace fm;

extern "C" int fm_convert(long n, int src_dtype, const void* src, int dst_dtype, void* dst, void* stream) {
  if (n < 0 || (n > 0 && (!src || !dst))) return FM_ERR_ARG;
  if (n == 0) return FM_OK;
  long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t s = (cudaStream_t)stream;
  if (src_dtype == FM_F32) return convert_from<float>(n, src, dst_dtype, dst, s, (unsigned)blocks);
  if (src_dtype == FM_F64) return convert_from<double>(n, src, dst_dtype, dst, s, (unsigned)blocks);
  if (src_dtype == FM_BF16) return convert_from<__nv_bfloat16>(n, src, dst_dtype, dst, s, (unsigned)blocks);
  return FM_ERR_DTYPE;
}

// ---------------------------------------------------------------------------
// BFECC clamp: dst = clamp(src, min, max of ref over the 2*dim axis neighbours),
// neighbours sampled with the index clamp of sample() (clamp_u,
// 3D/flowmap.py:324-334, 2D/vortex/flowmap.py:333-341).  The centre value of
// ref is not part of the bounds, as in the reference.
// ---------------------------------------------------------------------------
namespace fm {

template <typename T, int D>
__global__ void k_clamp_extrema(Shape s, const T* __restrict__ src, const T* __restrict__ ref, T* __restrict__ dst) {
  const long n = s.size();
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    unflatten(s, q, i, j, k);
    const int im = i > 0 ? i - 1 : 0, ip = i < s.s0 - 1 ? i + 1 : s.s0 - 1;
    const int jm = j > 0 ? j - 1 : 0, jp = j < s.s1 - 1 ? j + 1 : s.s1 - 1;
    T mx = ref[s.idx(im, j, k)], mn = mx, v;
    v = ref[s.idx(ip, j, k)]; mx = fmax(mx, v); mn = fmin(mn, v);
    v = ref[s.idx(i, jm, k)]; mx = fmax(mx, v); mn = fmin(mn, v);
    v = ref[s.idx(i, jp, k)]; mx = fmax(mx, v); mn = fmin(mn, v);
    if (D == 3) {
      const int km = k > 0 ? k - 1 : 0, kp = k < s.s2 - 1 ? k + 1 : s.s2 - 1;
      v = ref[s.idx(i, j, km)]; mx = fmax(mx, v); mn = fmin(mn, v);
      v = ref[s.idx(i, j, kp)]; mx = fmax(mx, v); mn = fmin(mn, v);
    }
    dst[q] = fmin(fmax(src[q], mn), mx);
  }
}

}  // namespace fm

extern "C" int fm_clamp_extrema(const fm_grid* g, int dtype, int face, const void* src, const void* ref, void* dst,
                                void* stream) {
  using namespace fm;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (face < -1 || face >= g->dim) return FM_ERR_ARG;
  if (!src || !ref || !dst) return FM_ERR_ARG;
  const Shape s = face >= 0 ? face_shape(*g, face) : cell_shape(*g);
  long b = (s.size() + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  cudaStream_t cs = (cudaStream_t)stream;
  if (dtype == FM_F32) {
    if (g->dim == 3) launch(k_clamp_extrema<float, 3>, (unsigned)b, 256, 0, cs, s, (const float*)src, (const float*)ref, (float*)dst);
    else launch(k_clamp_extrema<float, 2>, (unsigned)b, 256, 0, cs, s, (const float*)src, (const float*)ref, (float*)dst);
  } else {
    if (g->dim == 3) launch(k_clamp_extrema<double, 3>, (unsigned)b, 256, 0, cs, s, (const double*)src, (const double*)ref, (double*)dst);
    else launch(k_clamp_extrema<double, 2>, (unsigned)b, 256, 0, cs, s, (const double*)src, (const double*)ref, (double*)dst);
  }
  return check_cuda();
}

// ---------------------------------------------------------------------------
// 2D viscous force (calculate_viscous_force, 2D/vortex/flowmap.py:4-17): on
// each face grid, vis = nu * (s(i+1,j) + s(i-1,j) + s(i,j+1) + s(i,j-1)
// - 4 s(i,j)) / dx / dx with sample()'s index clamp, rounded as the reference
// writes it (no FMA contraction).  With an adjoint velocity it also adds
// sum adj . vis / nu over both face grids to *dot (calculate_viscous_force_adj,
// 2D/vortex/flowmap.py:20-35; the reference skips the sum when nu == 0), by a
// fixed-grid FP64 reduction into `part` and an ordered final sum.
// ---------------------------------------------------------------------------
namespace fm {

constexpr int kVisBlocks = 148 * 4;
constexpr int kVisThreads = 256;

template <typename T>
__device__ __forceinline__ T vis_at(const T* __restrict__ u, int n0, int n1, int i, int j, T nu, T dx) {
  const int im = i > 0 ? i - 1 : 0, ip = i < n0 - 1 ? i + 1 : n0 - 1;
  const int jm = j > 0 ? j - 1 : 0, jp = j < n1 - 1 ? j + 1 : n1 - 1;
  const T s = rn_add(rn_add(rn_add(u[(long)ip * n1 + j], u[(long)im * n1 + j]), u[(long)i * n1 + jp]),
                     u[(long)i * n1 + jm]);
  const T lap = rn_sub(s, rn_mul((T)4, u[(long)i * n1 + j]));
  return rn_mul(nu, lap) / dx / dx;
}

template <typename T>
__global__ void __launch_bounds__(kVisThreads) k_viscous_force(int n0, int n1, T nu, T dx, const T* __restrict__ ux,
                                                               const T* __restrict__ uy, T* __restrict__ vx,
                                                               T* __restrict__ vy, const T* __restrict__ ax,
                                                               const T* __restrict__ ay, double* __restrict__ part) {
  const long nx = (long)(n0 + 1) * n1, ny = (long)n0 * (n1 + 1);
  double acc = 0.0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < nx + ny; q += (long)gridDim.x * blockDim.x) {
    if (q < nx) {
      const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
      const T v = vis_at(ux, n0 + 1, n1, i, j, nu, dx);
      vx[q] = v;
      if (ax) acc += (double)(ax[q] * v / nu);
    } else {
      const long r = q - nx;
      const int i = (int)(r / (n1 + 1)), j = (int)(r - (long)i * (n1 + 1));
      const T v = vis_at(uy, n0, n1 + 1, i, j, nu, dx);
      vy[r] = v;
      if (ax) acc += (double)(ay[r] * v / nu);
    }
  }
  if (!part) return;
  __shared__ double red[kVisThreads];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kVisThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_viscous_dot_fin(int nblocks, const double* __restrict__ part, double* __restrict__ dot) {
  if (threadIdx.x == 0) {
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[b];
    *dot += s;
  }
}

}  // namespace fm

extern "C" int fm_viscous_force_2d(const fm_grid* g, int dtype, double nu, double dx, const void* ux, const void* uy,
                                   void* vis_x, void* vis_y, const void* adj_x, const void* adj_y, double* part,
                                   double* dot, void* stream) {
  using namespace fm;
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (g->dim != 2) return FM_ERR_SHAPE;
  if (!ux || !uy || !vis_x || !vis_y || !(dx > 0)) return FM_ERR_ARG;
  const bool with_dot = adj_x || adj_y;
  if (with_dot && (!adj_x || !adj_y || !part || !dot)) return FM_ERR_ARG;
  const bool sum = with_dot && nu != 0.0;  // the reference adds nothing when nu == 0
  cudaStream_t s = (cudaStream_t)stream;
  const int n0 = g->n[0], n1 = g->n[1];
  if (dtype == FM_F32)
    launch(k_viscous_force<float>, kVisBlocks, kVisThreads, 0, s, n0, n1, (float)nu, (float)dx, (const float*)ux,
           (const float*)uy, (float*)vis_x, (float*)vis_y, sum ? (const float*)adj_x : nullptr,
           sum ? (const float*)adj_y : nullptr, sum ? part : nullptr);
  else
    launch(k_viscous_force<double>, kVisBlocks, kVisThreads, 0, s, n0, n1, nu, dx, (const double*)ux,
           (const double*)uy, (double*)vis_x, (double*)vis_y, sum ? (const double*)adj_x : nullptr,
           sum ? (const double*)adj_y : nullptr, sum ? part : nullptr);
  if (sum) launch(k_viscous_dot_fin, 1, 32, 0, s, kVisBlocks, (const double*)part, dot);
  return check_cuda();
}

// ---------------------------------------------------------------------------
// FP32 FMA throughput probe (the denominator of the gather kernels' roofline).
// Every thread runs 16 independent FMA chains of `iters` steps -- 16 scalar
// fmaf chains, or 8 chains of paired __ffma2_rn (two FMAs per instruction) --
// and writes their sum, so no chain is optimised away.  x <- x * a + b with
// |a| < 1 keeps every value finite.  FLOPs = blocks * 256 * iters * 32.
// ---------------------------------------------------------------------------
namespace fm {

constexpr int kProbeThreads = 256;

template <bool PAIRED>
__global__ void __launch_bounds__(kProbeThreads) k_fma_probe(int iters, float a, float b, float* __restrict__ out) {
  const int gid = blockIdx.x * kProbeThreads + threadIdx.x;
  float acc = 0.f;
  if constexpr (PAIRED) {
    float2 x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = make_float2(1e-3f * threadIdx.x + i, 2e-3f * threadIdx.x - i);
    const float2 A = make_float2(a, a), B = make_float2(b, b);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = __ffma2_rn(x[i], A, B);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) acc += x[i].x + x[i].y;
  } else {
    float x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = 1e-3f * threadIdx.x + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int i = 0; i < 16; ++i) x[i] = fmaf(x[i], a, b);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) acc += x[i];
  }
  out[gid] = acc;
}

}  // namespace fm

extern "C" int fm_fp32_fma_probe(int paired, int blocks, int iters, float* out, void* stream) {
  using namespace fm;
  if (blocks < 1 || iters < 1 || !out) return FM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (paired) launch(k_fma_probe<true>, blocks, kProbeThreads, 0, s, iters, 0.9999999f, 1e-7f, out);
  else launch(k_fma_probe<false>, blocks, kProbeThreads, 0, s, iters, 0.9999999f, 1e-7f, out);
  return check_cuda();
}
