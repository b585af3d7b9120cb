// fm_util.cu -- elementwise storage conversion for the trajectory stores.
//
// The mixed-precision form keeps every step's midpoint velocity and passive
// scalar in BF16 (round to nearest even) and widens them back to FP32 when the
// adjoint reads them.  bf16 -> f32 is exact, so a stored value is read back as
// exactly the BF16-rounded FP32 value.
#include <cuda_bf16.h>

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
