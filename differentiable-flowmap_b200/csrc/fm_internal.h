// fm_internal.h -- argument validation and error mapping shared by the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <unordered_map>
#include <utility>

#include "../../include/flowmap_sm100.h"

namespace fm {

inline int validate_grid(const fm_grid* g, int dtype) {
  if (dtype != FM_F32 && dtype != FM_F64) return FM_ERR_DTYPE;
  if (!g) return FM_ERR_ARG;
  if (g->dim != 2 && g->dim != 3) return FM_ERR_SHAPE;
  for (int a = 0; a < 3; ++a)
    if (g->n[a] < 1) return FM_ERR_SHAPE;
  if (g->dim == 2 && g->n[2] != 1) return FM_ERR_SHAPE;
  // the B-spline stencils clamp to [1, n-2]: at least 4 cells per axis
  for (int a = 0; a < g->dim; ++a)
    if (g->n[a] < 4) return FM_ERR_SHAPE;
  // kernels decompose flat indices with 32-bit arithmetic: every grid (faces
  // included) must hold fewer than 2^32 entries
  if ((long long)(g->n[0] + 1) * (g->n[1] + 1) * (g->n[2] + 1) >= (1LL << 32)) return FM_ERR_SHAPE;
  return FM_OK;
}

// Host-side count of kernels this library has launched (graph launches add
// the number of kernel nodes they contain); read by fm_launch_count().
extern std::atomic<long long> g_launch_count;
// The autotuner's value for kernel class `kind` on grid g (fm_tune_set), else dflt.
int tuned_value(int kind, const fm_grid& g, int dflt);

inline void count_launch(long long n = 1) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

// The CUDA error behind the most recent FM_ERR_CUDA (fm_last_cuda_error()).
extern std::atomic<int> g_last_cuda_error;
inline int cuda_fail(cudaError_t e) {
  g_last_cuda_error.store((int)e, std::memory_order_relaxed);
  return FM_ERR_CUDA;
}

inline int check_cuda() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FM_OK : cuda_fail(e);
}

// After an entry point's single kernel launch.
inline int check_launch() {
  count_launch();
  return check_cuda();
}

// Raise-only setting of a kernel's dynamic shared-memory limit.  The attribute
// is per kernel and process-wide, while solvers of different sizes need
// different amounts: setting it to each new solver's need would lower it under
// what an earlier, larger solver launches (its later launches, and any launch
// recorded into a graph after that, would fail).  Thread-safe.
template <typename... KArgs>
inline bool raise_smem_limit(void (*k)(KArgs...), size_t smem) {
  static std::mutex mu;
  static std::unordered_map<const void*, size_t> limit;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limit[(const void*)k];
  if (smem <= cur) return true;
  if (cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return false;
  cur = smem;
  return true;
}

// Launches through launch_pdl use programmatic dependent launch unless it is
// switched off (fm_set_pdl); their kernels start with pdl_begin().
extern std::atomic<int> g_pdl;

// Launch helper that counts the launch.
template <typename... KArgs, typename... Args>
inline void launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  k<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
  count_launch();
}

// As launch(), with the programmatic-serialization attribute: the kernel's CTAs
// may be scheduled before its stream predecessor finishes and wait for it in
// pdl_begin().  Only for kernels whose first statement is pdl_begin().
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  if (!g_pdl.load(std::memory_order_relaxed)) {
    launch(k, grid, block, smem, s, std::forward<Args>(args)...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
  count_launch();
}

}  // namespace fm
