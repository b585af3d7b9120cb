// fm_vortex.cu -- the 2D vortex problem's initial-condition map and vorticity
// loss, with their adjoints (the 256^2 vortex optimisation workload: gradient
// of a final-vorticity loss with respect to the vortex parameters).
//
//  * velocity law: a sum of Gaussian-core point vortices evaluated at the cell
//    centres, u_c = sum_k f(|p_k|) w_k (-p_k.y, p_k.x), p_k = X - c_k,
//    f(r) = angular_vel_func(r, 0.02, -0.01) (2D/vortex/init_conditions.py:
//    142-145, 386-414), then split to the MAC faces with clamped samples
//    (split_central_vector, 2D/vortex/taichi_utils.py:158-167).
//    theta = [w_0..w_{K-1}, cx_0..cx_{K-1}, cy_0..cy_{K-1}].
//  * vorticity: omega = curl of the face-averaged centre velocity with clamped
//    samples (get_central_vector / curl, 2D/vortex/taichi_utils.py:153-156,
//    199-205).
//  * adjoints: both maps are linear in u (vorticity) or smooth in theta
//    (velocity); their transposes are written as gathers (no atomics), the
//    theta gradient as a deterministic fixed-grid FP64 reduction.
#include <math.h>

#include "fm_common.cuh"
#include "fm_internal.h"

namespace fm {

constexpr int kVortexMax = 64;
constexpr int kVxBlocks = 148 * 4;
constexpr int kVxThreads = 256;

struct VortexParams {
  int nv;
  double th[3 * kVortexMax];
};

// angular_vel_func(r, rad, strength) (2D/vortex/init_conditions.py:142-145) in T
template <typename T>
__device__ __forceinline__ T angular_vel(T r, T rad, T strength) {
  r = r + (T)1e-6;
  const T linear_vel = strength * ((T)1. / r) * ((T)1. - exp(-(r * r) / (rad * rad)));
  return ((T)1. / r) * linear_vel;
}

// derivative of angular_vel with respect to r (analytic, for the theta gradient)
template <typename T>
__device__ __forceinline__ T angular_vel_dr(T r, T rad, T strength) {
  const T rr = r + (T)1e-6;
  const T a2 = rad * rad;
  const T e = exp(-(rr * rr) / a2);
  return (T)2 * strength * (e / (a2 * rr) - ((T)1 - e) / (rr * rr * rr));
}

constexpr double kVortexCore = 0.02, kVortexStrength = -0.01;

// velocity at cell (i, j): four_vortex_vel_func_with_coef's per-vortex sum
template <typename T>
__device__ __forceinline__ void vortex_cell(const VortexParams& P, T dx, int i, int j, T& vx, T& vy) {
  const T X = ((T)i + (T)0.5) * dx, Y = ((T)j + (T)0.5) * dx;
  vx = 0;
  vy = 0;
  for (int k = 0; k < P.nv; ++k) {
    const T w = (T)P.th[k], cx = (T)P.th[P.nv + k], cy = (T)P.th[2 * P.nv + k];
    const T px = X - cx, py = Y - cy;
    const T r = sqrt(px * px + py * py);
    const T fw = angular_vel(r, (T)kVortexCore, (T)kVortexStrength) * w;
    vx += fw * -py;
    vy += fw * px;
  }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// face velocities: u_x[i, j] = 0.5 (c(i, j).x + c(i-1, j).x), u_y likewise (clamped)
template <typename T>
__global__ void k_vortex_velocity(int n0, int n1, T dx, VortexParams P, T* __restrict__ ux, T* __restrict__ uy) {
  const long nx = (long)(n0 + 1) * n1, ny = (long)n0 * (n1 + 1);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < nx + ny; q += (long)gridDim.x * blockDim.x) {
    T ax, ay, bx, by;
    if (q < nx) {
      const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
      vortex_cell<T>(P, dx, clampi(i, 0, n0 - 1), j, ax, ay);
      vortex_cell<T>(P, dx, clampi(i - 1, 0, n0 - 1), j, bx, by);
      ux[q] = (T)0.5 * (ax + bx);
    } else {
      const long t = q - nx;
      const int i = (int)(t / (n1 + 1)), j = (int)(t - (long)i * (n1 + 1));
      vortex_cell<T>(P, dx, i, clampi(j, 0, n1 - 1), ax, ay);
      vortex_cell<T>(P, dx, i, clampi(j - 1, 0, n1 - 1), bx, by);
      uy[t] = (T)0.5 * (ay + by);
    }
  }
}

// Adjoint of split_central_vector at cell (i, j): the face cotangents gathered
// onto the centre (a face takes half of each of its two clamped samples).
template <typename T>
__device__ __forceinline__ void split_adjoint(const T* __restrict__ lx, const T* __restrict__ ly, int n0, int n1, int i,
                                              int j, double& gx, double& gy) {
  gx = 0.5 * ((double)lx[(long)i * n1 + j] + (double)lx[(long)(i + 1) * n1 + j]);
  if (i == 0) gx += 0.5 * (double)lx[j];
  if (i == n0 - 1) gx += 0.5 * (double)lx[(long)n0 * n1 + j];
  gy = 0.5 * ((double)ly[(long)i * (n1 + 1) + j] + (double)ly[(long)i * (n1 + 1) + j + 1]);
  if (j == 0) gy += 0.5 * (double)ly[(long)i * (n1 + 1)];
  if (j == n1 - 1) gy += 0.5 * (double)ly[(long)i * (n1 + 1) + n1];
}

// dL/dtheta = sum over cells of (split^T lambda) . d u_c / d theta, FP64
template <typename T>
__global__ void __launch_bounds__(kVxThreads) k_vortex_grad(int n0, int n1, double dx, VortexParams P,
                                                            const T* __restrict__ lx, const T* __restrict__ ly,
                                                            double* __restrict__ part) {
  double acc[3 * kVortexMax];
  const int m = 3 * P.nv;
  for (int a = 0; a < m; ++a) acc[a] = 0;
  const long n = (long)n0 * n1;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
    double gx, gy;
    split_adjoint<T>(lx, ly, n0, n1, i, j, gx, gy);
    const double X = (i + 0.5) * dx, Y = (j + 0.5) * dx;
    for (int k = 0; k < P.nv; ++k) {
      const double w = P.th[k], px = X - P.th[P.nv + k], py = Y - P.th[2 * P.nv + k];
      const double r = sqrt(px * px + py * py);
      const double f = angular_vel<double>(r, kVortexCore, kVortexStrength);
      const double fr = r > 0 ? angular_vel_dr<double>(r, kVortexCore, kVortexStrength) / r : 0.0;
      // v = w f (-py, px); dv/dpx = w (fr px (-py, px) + f (0, 1)); dv/dpy = w (fr py (-py, px) + f (-1, 0))
      const double dot_rot = gx * -py + gy * px;
      acc[k] += f * dot_rot;                                    // d/dw
      acc[P.nv + k] -= w * (fr * px * dot_rot + f * gy);        // d/dcx = -d/dpx
      acc[2 * P.nv + k] -= w * (fr * py * dot_rot - f * gx);    // d/dcy = -d/dpy
    }
  }
  // block reduction of the m accumulators, in a fixed order
  __shared__ double red[kVxThreads];
  for (int a = 0; a < m; ++a) {
    red[threadIdx.x] = acc[a];
    __syncthreads();
    for (int s = kVxThreads / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(long)blockIdx.x * m + a] = red[0];
    __syncthreads();
  }
}

__global__ void k_vortex_grad_fin(int m, int nblocks, const double* __restrict__ part, double* __restrict__ out) {
  const int a = threadIdx.x;
  if (a >= m) return;
  double s = 0;
  for (int b = 0; b < nblocks; ++b) s += part[(long)b * m + a];
  out[a] = s;
}

// centre velocity with clamped samples (get_central_vector on sample(...))
template <typename T>
__device__ __forceinline__ void centre(const T* __restrict__ ux, const T* __restrict__ uy, int n0, int n1, int i, int j,
                                       T& cx, T& cy) {
  i = clampi(i, 0, n0 - 1);
  j = clampi(j, 0, n1 - 1);
  cx = (T)0.5 * (ux[(long)(i + 1) * n1 + j] + ux[(long)i * n1 + j]);
  cy = (T)0.5 * (uy[(long)i * (n1 + 1) + j + 1] + uy[(long)i * (n1 + 1) + j]);
}

template <typename T>
__device__ __forceinline__ T vorticity_at(const T* ux, const T* uy, int n0, int n1, T dx, int i, int j) {
  T lx, ly, rx, ry, bx, by, tx, ty;
  centre<T>(ux, uy, n0, n1, i - 1, j, lx, ly);
  centre<T>(ux, uy, n0, n1, i + 1, j, rx, ry);
  centre<T>(ux, uy, n0, n1, i, j - 1, bx, by);
  centre<T>(ux, uy, n0, n1, i, j + 1, tx, ty);
  return (ry - ly - tx + bx) / ((T)2 * dx);
}

template <typename T>
__global__ void k_vorticity(int n0, int n1, T dx, const T* __restrict__ ux, const T* __restrict__ uy,
                            T* __restrict__ om) {
  const long n = (long)n0 * n1;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
    om[q] = vorticity_at<T>(ux, uy, n0, n1, dx, i, j);
  }
}

// g = 2 (omega - omega*) into `work`, partial sums of (omega - omega*)^2
template <typename T>
__global__ void __launch_bounds__(kVxThreads) k_vort_loss(int n0, int n1, T dx, const T* __restrict__ ux,
                                                          const T* __restrict__ uy, const T* __restrict__ target,
                                                          T* __restrict__ work, double* __restrict__ part) {
  const long n = (long)n0 * n1;
  double acc = 0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
    const T d = vorticity_at<T>(ux, uy, n0, n1, dx, i, j) - target[q];
    work[q] = (T)2 * d;
    acc += (double)d * (double)d;
  }
  __shared__ double red[kVxThreads];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kVxThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_vort_loss_fin(int nblocks, const double* __restrict__ part, double* __restrict__ loss) {
  if (threadIdx.x == 0) {
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[b];
    *loss = s;
  }
}

// Cotangent of the clamped centre sample c(a, b) seen from centre cell (i, j):
// the omega cells whose +-1 samples land on (i, j) along each axis.
// gcx(i, j) = sum over cells (i, b) with B(b) = j of g/(2dx) - with T(b) = j;
// gcy(i, j) = sum over cells (a, j) with R(a) = i of g/(2dx) - with L(a) = i.
template <typename T>
__device__ __forceinline__ void centre_cotangent(const T* __restrict__ g, int n0, int n1, T dx, int i, int j, T& gcx,
                                                 T& gcy) {
  const T h = (T)1 / ((T)2 * dx);
  T sx = 0, sy = 0;
  // T(b) = clamp(b+1) = j: b = j-1 (j >= 1), and b = n1-1 when j = n1-1
  if (j >= 1) sx -= g[(long)i * n1 + j - 1];
  if (j == n1 - 1) sx -= g[(long)i * n1 + n1 - 1];
  // B(b) = clamp(b-1) = j: b = j+1 (j <= n1-2), and b = 0 when j = 0
  if (j <= n1 - 2) sx += g[(long)i * n1 + j + 1];
  if (j == 0) sx += g[(long)i * n1];
  // R(a) = clamp(a+1) = i: a = i-1 (i >= 1), and a = n0-1 when i = n0-1
  if (i >= 1) sy += g[(long)(i - 1) * n1 + j];
  if (i == n0 - 1) sy += g[(long)(n0 - 1) * n1 + j];
  // L(a) = clamp(a-1) = i: a = i+1 (i <= n0-2), and a = 0 when i = 0
  if (i <= n0 - 2) sy -= g[(long)(i + 1) * n1 + j];
  if (i == 0) sy -= g[j];
  gcx = sx * h;
  gcy = sy * h;
}

// lambda on the faces = (d omega / d u)^T g (the centre average's transpose)
template <typename T>
__global__ void k_vort_adjoint(int n0, int n1, T dx, const T* __restrict__ g, T* __restrict__ lx, T* __restrict__ ly) {
  const long nx = (long)(n0 + 1) * n1, ny = (long)n0 * (n1 + 1);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < nx + ny; q += (long)gridDim.x * blockDim.x) {
    T s = 0, cx, cy;
    if (q < nx) {
      const int i = (int)(q / n1), j = (int)(q - (long)i * n1);
      // face i is the right sample of centre i-1 and the left of centre i
      if (i >= 1) { centre_cotangent<T>(g, n0, n1, dx, i - 1, j, cx, cy); s += (T)0.5 * cx; }
      if (i <= n0 - 1) { centre_cotangent<T>(g, n0, n1, dx, i, j, cx, cy); s += (T)0.5 * cx; }
      lx[q] = s;
    } else {
      const long t = q - nx;
      const int i = (int)(t / (n1 + 1)), j = (int)(t - (long)i * (n1 + 1));
      if (j >= 1) { centre_cotangent<T>(g, n0, n1, dx, i, j - 1, cx, cy); s += (T)0.5 * cy; }
      if (j <= n1 - 1) { centre_cotangent<T>(g, n0, n1, dx, i, j, cx, cy); s += (T)0.5 * cy; }
      ly[t] = s;
    }
  }
}

static int vortex_check(const fm_grid* g, int dtype, int nv) {
  const int st = validate_grid(g, dtype);
  if (st) return st;
  if (g->dim != 2) return FM_ERR_SHAPE;
  if (nv < 1 || nv > kVortexMax) return FM_ERR_ARG;
  return FM_OK;
}

static unsigned grid_for(long n) {
  long b = (n + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_vortex_velocity_2d(const fm_grid* g, int dtype, double dx, int nv, const double* theta, void* ux, void* uy,
                          void* stream) {
  int st = vortex_check(g, dtype, nv);
  if (st) return st;
  if (!theta || !ux || !uy) return FM_ERR_ARG;
  VortexParams P{};
  P.nv = nv;
  for (int a = 0; a < 3 * nv; ++a) P.th[a] = theta[a];
  const int n0 = g->n[0], n1 = g->n[1];
  const unsigned nb = grid_for((long)(n0 + 1) * n1 + (long)n0 * (n1 + 1));
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32) launch(k_vortex_velocity<float>, nb, 256, 0, s, n0, n1, (float)dx, P, (float*)ux, (float*)uy);
  else launch(k_vortex_velocity<double>, nb, 256, 0, s, n0, n1, dx, P, (double*)ux, (double*)uy);
  return check_cuda();
}

int fm_vortex_velocity_grad_2d(const fm_grid* g, int dtype, double dx, int nv, const double* theta, const void* lam_x,
                               const void* lam_y, double* work, double* grad, void* stream) {
  int st = vortex_check(g, dtype, nv);
  if (st) return st;
  if (!theta || !lam_x || !lam_y || !work || !grad) return FM_ERR_ARG;
  VortexParams P{};
  P.nv = nv;
  for (int a = 0; a < 3 * nv; ++a) P.th[a] = theta[a];
  const int n0 = g->n[0], n1 = g->n[1];
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FM_F32)
    launch(k_vortex_grad<float>, kVxBlocks, kVxThreads, 0, s, n0, n1, dx, P, (const float*)lam_x, (const float*)lam_y, work);
  else
    launch(k_vortex_grad<double>, kVxBlocks, kVxThreads, 0, s, n0, n1, dx, P, (const double*)lam_x,
           (const double*)lam_y, work);
  launch(k_vortex_grad_fin, 1, 3 * kVortexMax, 0, s, 3 * nv, kVxBlocks, (const double*)work, grad);
  return check_cuda();
}

int fm_vorticity_2d(const fm_grid* g, int dtype, double dx, const void* ux, const void* uy, void* omega, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (g->dim != 2) return FM_ERR_SHAPE;
  if (!ux || !uy || !omega) return FM_ERR_ARG;
  const int n0 = g->n[0], n1 = g->n[1];
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb = grid_for((long)n0 * n1);
  if (dtype == FM_F32)
    launch(k_vorticity<float>, nb, 256, 0, s, n0, n1, (float)dx, (const float*)ux, (const float*)uy, (float*)omega);
  else
    launch(k_vorticity<double>, nb, 256, 0, s, n0, n1, dx, (const double*)ux, (const double*)uy, (double*)omega);
  return check_cuda();
}

int fm_vorticity_loss_2d(const fm_grid* g, int dtype, double dx, const void* ux, const void* uy, const void* omega_target,
                         void* work, double* part, void* lam_x, void* lam_y, double* loss, void* stream) {
  int st = validate_grid(g, dtype);
  if (st) return st;
  if (g->dim != 2) return FM_ERR_SHAPE;
  if (!ux || !uy || !omega_target || !work || !part || !lam_x || !lam_y || !loss) return FM_ERR_ARG;
  const int n0 = g->n[0], n1 = g->n[1];
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nf = grid_for((long)(n0 + 1) * n1 + (long)n0 * (n1 + 1));
  if (dtype == FM_F32) {
    launch(k_vort_loss<float>, kVxBlocks, kVxThreads, 0, s, n0, n1, (float)dx, (const float*)ux, (const float*)uy,
           (const float*)omega_target, (float*)work, part);
    launch(k_vort_adjoint<float>, nf, 256, 0, s, n0, n1, (float)dx, (const float*)work, (float*)lam_x, (float*)lam_y);
  } else {
    launch(k_vort_loss<double>, kVxBlocks, kVxThreads, 0, s, n0, n1, dx, (const double*)ux, (const double*)uy,
           (const double*)omega_target, (double*)work, part);
    launch(k_vort_adjoint<double>, nf, 256, 0, s, n0, n1, dx, (const double*)work, (double*)lam_x, (double*)lam_y);
  }
  launch(k_vort_loss_fin, 1, 32, 0, s, kVxBlocks, (const double*)part, loss);
  return check_cuda();
}

}  // extern "C"
