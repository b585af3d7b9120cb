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
