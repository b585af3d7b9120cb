// fm_q2.cuh -- quadratic B-spline interpolation specialised for the flow-map
// transport kernels (advect_u_grid, RK_grid, advect_u, accumulate_init,
// advect_scalar_grid): interp_grad_2 / interp_2_scalar / interp_u_MAC_grad of
// 3D/taichi_utils.py:433-466, 567-601.
//
// Per axis the reference evaluates 4 taps at iu-1..iu+2 with
// s = clamp(p/dx - BL, 1, len-2-eps), iu = floor(s), weight N2(s - tap).
// With f = s - iu and t0 = (f >= 0.5), t = f - t0 in [-0.5, 0.5), the three
// taps that can be non-zero start at i0 = iu - 1 + t0 and sit at x = t+1, t,
// t-1, where the reference's branches reduce to
//   N2:  0.5 (0.5 - t)^2,   0.75 - t^2,   0.5 (0.5 + t)^2
//   dN2: t - 0.5,           -2 t,          t + 0.5
// Every intermediate (s - iu, t, 0.5 -+ t, 2x - 3) is exact in floating point,
// so these are bit-identical to the reference's N_2 / dN_2 values.
// The taps i0..i0+2 never leave [0, len-1] (iu >= 1, and iu = len-2 forces
// f = 0), so sample()'s clamp is never active: the three taps of an axis are
// contiguous and one row offset serves a whole k-triple.
// Positions are scaled by 1/dx (exact for the power-of-two dx of the
// benchmark grids; within one ulp of the reference's p/dx otherwise).
//
// Issue economy (these kernels are instruction-issue bound): field offsets are
// 32-bit (every field has fewer than 2^32 entries), the clamp bounds are
// computed once per thread (Q2Lim), and in FP32 the two rows i0 and i0+1 of a
// 3D stencil are contracted together with paired FMAs (__ffma2_rn: two IEEE
// fused multiply-adds in one instruction), each lane performing exactly the
// operation sequence of the scalar row.
#pragma once
#include <type_traits>

#include "fm_common.cuh"

namespace fm {

// Clamp bounds len - 2 - 1e-6 per axis for the face-staggered extent (n+1,
// BL = 0) and the cell-centred extent (n, BL = 0.5).
template <typename T>
struct Q2Lim {
  T h0[3], h5[3];
  __device__ __forceinline__ explicit Q2Lim(const fm_grid& g) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      h0[a] = (T)((double)(g.n[a] + 1) - 2.0 - 1e-6);
      h5[a] = (T)((double)g.n[a] - 2.0 - 1e-6);
    }
  }
};

// floor(s) as a float and as an int for 1 <= s < 2^23: the integer is read
// from the mantissa of floor(s) + 2^23 instead of a float->int conversion (an
// XU-pipe instruction).  Exact: the same values as floor() and (int) floor().
__device__ __forceinline__ float floor_pos(float s, int& i) {
  const float f = floorf(s);
  i = __float_as_int(__fadd_rn(f, 8388608.0f)) - 0x4B000000;  // exact: f is an integer below 2^23
  return f;
}
__device__ __forceinline__ double floor_pos(double s, int& i) {
  const double f = floor(s);
  i = (int)f;
  return f;
}

template <typename T, bool GRAD>
struct Q2 {
  int i0;
  T w0, w1, w2;
  T d0, d1, d2;
  __device__ __forceinline__ void setup(T pos_scaled, T bl, T hi) {
    const T u = pos_scaled - bl;
    T s = u < hi ? u : hi;
    s = s > (T)1 ? s : (T)1;
    int ii;
    const T iu = floor_pos(s, ii);  // s >= 1 after the clamp
    const T f = s - iu;
    const bool up = f >= (T)0.5;
    const T t = up ? f - (T)1 : f;
    i0 = ii - 1 + (up ? 1 : 0);
    const T a = (T)0.5 - t, b = (T)0.5 + t;
    w0 = (T)0.5 * (a * a);
    w1 = (T)0.75 - t * t;
    w2 = (T)0.5 * (b * b);
    if (GRAD) {
      d0 = t - (T)0.5;
      d1 = (T)-2 * t;
      d2 = b;
    }
  }
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// sum_k f[r + k] w_k for k = 0..2, as (f0 w0 + f1 w1) + f2 w2
template <typename T>
__device__ __forceinline__ T row3(const T* __restrict__ f, unsigned r, T w0, T w1, T w2) {
  return ldg(f + r) * w0 + ldg(f + r + 1) * w1 + ldg(f + r + 2) * w2;
}
// the same for rows r and r' in the two lanes
__device__ __forceinline__ float2 row3x2(const float* __restrict__ f, unsigned r, unsigned r2, float2 w0, float2 w1,
                                         float2 w2) {
  float2 a = __fmul2_rn(f2(ldg(f + r), ldg(f + r2)), w0);
  a = __ffma2_rn(f2(ldg(f + r + 1), ldg(f + r2 + 1)), w1, a);
  return __ffma2_rn(f2(ldg(f + r + 2), ldg(f + r2 + 2)), w2, a);
}

// value of one staggered field with shape s at the stencil (ax, ay, az)
template <typename T, int D, bool G>
__device__ __forceinline__ T q2_val(const T* __restrict__ f, const Shape& s, const Q2<T, G>& ax, const Q2<T, G>& ay,
                                    const Q2<T, G>& az) {
  if constexpr (D == 3) {
    const unsigned sj = s.s2, si = (unsigned)s.s1 * s.s2;
    const unsigned b = ((unsigned)ax.i0 * s.s1 + ay.i0) * s.s2 + az.i0;
    const T wy[3] = {ay.w0, ay.w1, ay.w2};
    if constexpr (std::is_same<T, float>::value) {
      const float2 W0 = f2(az.w0), W1 = f2(az.w1), W2 = f2(az.w2);
      float2 v01 = f2(0.f);
      float v2 = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const unsigned r0 = b + j * sj;
        v01 = __ffma2_rn(row3x2(f, r0, r0 + si, W0, W1, W2), f2(wy[j]), v01);
        v2 += row3(f, r0 + 2 * si, az.w0, az.w1, az.w2) * wy[j];
      }
      float v = 0.f;
      v += v01.x * ax.w0;
      v += v01.y * ax.w1;
      v += v2 * ax.w2;
      return v;
    } else {
      const T wx[3] = {ax.w0, ax.w1, ax.w2};
      T v = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        T vi = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) vi += row3(f, b + i * si + j * sj, az.w0, az.w1, az.w2) * wy[j];
        v += vi * wx[i];
      }
      return v;
    }
  } else {
    const unsigned si = s.s1;
    const unsigned b = (unsigned)ax.i0 * s.s1 + ay.i0;
    const T wx[3] = {ax.w0, ax.w1, ax.w2};
    T v = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) v += row3(f, b + i * si, ay.w0, ay.w1, ay.w2) * wx[i];
    return v;
  }
}

// value and gradient (unscaled by 1/dx) of one staggered field
template <typename T, int D>
__device__ __forceinline__ void q2_grad(const T* __restrict__ f, const Shape& s, const Q2<T, true>& ax,
                                        const Q2<T, true>& ay, const Q2<T, true>& az, T& v, T* g) {
  const T wx[3] = {ax.w0, ax.w1, ax.w2}, dx_[3] = {ax.d0, ax.d1, ax.d2};
  const T wy[3] = {ay.w0, ay.w1, ay.w2}, dy_[3] = {ay.d0, ay.d1, ay.d2};
  if constexpr (D == 3) {
    const unsigned sj = s.s2, si = (unsigned)s.s1 * s.s2;
    const unsigned b = ((unsigned)ax.i0 * s.s1 + ay.i0) * s.s2 + az.i0;
    T A[3], B[3], Cc[3];
    if constexpr (std::is_same<T, float>::value) {
      // rows i = 0, 1 in the two lanes, row i = 2 scalar
      const float2 W0 = f2(az.w0), W1 = f2(az.w1), W2 = f2(az.w2);
      const float2 E0 = f2(az.d0), E1 = f2(az.d1), E2 = f2(az.d2);
      float2 A01 = f2(0.f), B01 = f2(0.f), C01 = f2(0.f);
      float A2 = 0.f, B2 = 0.f, C2 = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const unsigned r0 = b + j * sj, r1 = r0 + si, r2 = r1 + si;
        const float2 x0 = f2(ldg(f + r0), ldg(f + r1));
        const float2 x1 = f2(ldg(f + r0 + 1), ldg(f + r1 + 1));
        const float2 x2 = f2(ldg(f + r0 + 2), ldg(f + r1 + 2));
        const float2 a = __ffma2_rn(x2, W2, __ffma2_rn(x1, W1, __fmul2_rn(x0, W0)));
        const float2 bb = __ffma2_rn(x2, E2, __ffma2_rn(x1, E1, __fmul2_rn(x0, E0)));
        A01 = __ffma2_rn(a, f2(wy[j]), A01);
        B01 = __ffma2_rn(a, f2(dy_[j]), B01);
        C01 = __ffma2_rn(bb, f2(wy[j]), C01);
        const float g0 = ldg(f + r2), g1 = ldg(f + r2 + 1), g2 = ldg(f + r2 + 2);
        const float a2 = g0 * az.w0 + g1 * az.w1 + g2 * az.w2;
        const float b2 = g0 * az.d0 + g1 * az.d1 + g2 * az.d2;
        A2 += a2 * wy[j];
        B2 += a2 * dy_[j];
        C2 += b2 * wy[j];
      }
      A[0] = A01.x; A[1] = A01.y; A[2] = A2;
      B[0] = B01.x; B[1] = B01.y; B[2] = B2;
      Cc[0] = C01.x; Cc[1] = C01.y; Cc[2] = C2;
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        A[i] = 0; B[i] = 0; Cc[i] = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const unsigned r = b + i * si + j * sj;
          const T f0 = ldg(f + r), f1 = ldg(f + r + 1), f2_ = ldg(f + r + 2);
          const T a = f0 * az.w0 + f1 * az.w1 + f2_ * az.w2;
          const T bb = f0 * az.d0 + f1 * az.d1 + f2_ * az.d2;
          A[i] += a * wy[j];
          B[i] += a * dy_[j];
          Cc[i] += bb * wy[j];
        }
      }
    }
    T vv = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      vv += A[i] * wx[i];
      gx += A[i] * dx_[i];
      gy += B[i] * wx[i];
      gz += Cc[i] * wx[i];
    }
    v = vv;
    g[0] = gx;
    g[1] = gy;
    g[2] = gz;
  } else {
    const unsigned si = s.s1;
    const unsigned b = (unsigned)ax.i0 * s.s1 + ay.i0;
    T vv = 0, gx = 0, gy = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const unsigned r = b + i * si;
      const T f0 = ldg(f + r), f1 = ldg(f + r + 1), f2_ = ldg(f + r + 2);
      const T a = f0 * ay.w0 + f1 * ay.w1 + f2_ * ay.w2;
      const T bb = f0 * ay.d0 + f1 * ay.d1 + f2_ * ay.d2;
      vv += a * wx[i];
      gx += a * dx_[i];
      gy += bb * wx[i];
    }
    v = vv;
    g[0] = gx;
    g[1] = gy;
  }
}

// Stencils of a MAC sample point: per axis one setup for the component
// staggered on that axis (BL = 0, extent n+1) and one shared by the others
// (BL = 0.5, extent n).
template <typename T, int D, bool G>
struct MacStencil {
  Q2<T, G> s0[3];  // BL = 0
  Q2<T, G> s5[3];  // BL = 0.5
  __device__ __forceinline__ void setup(const Q2Lim<T>& lim, const T* p, T inv_dx) {
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const T ps = p[a] * inv_dx;
      s0[a].setup(ps, (T)0, lim.h0[a]);
      s5[a].setup(ps, (T)0.5, lim.h5[a]);
    }
  }
  __device__ __forceinline__ const Q2<T, G>& ax(int c, int a) const { return a == c ? s0[a] : s5[a]; }
};

// interp_u_MAC (value only), all components
template <typename T, int D>
__device__ __forceinline__ void q2_mac_val(const Mac<T>& u, const fm_grid& g, const Q2Lim<T>& lim, const T* p,
                                           T inv_dx, T* v) {
  MacStencil<T, D, false> st;
  st.setup(lim, p, inv_dx);
#pragma unroll
  for (int c = 0; c < D; ++c) v[c] = q2_val<T, D, false>(u.c[c], face_shape(g, c), st.ax(c, 0), st.ax(c, 1), st.ax(c, 2 % D));
}

// Stencil of face component c (runtime) at p.
template <typename T, int D>
struct CompStencil {
  Q2<T, false> ax, ay, az;
  __device__ __forceinline__ void setup(const Q2Lim<T>& lim, int c, const T* p, T inv_dx) {
    ax.setup(p[0] * inv_dx, c == 0 ? (T)0 : (T)0.5, c == 0 ? lim.h0[0] : lim.h5[0]);
    ay.setup(p[1] * inv_dx, c == 1 ? (T)0 : (T)0.5, c == 1 ? lim.h0[1] : lim.h5[1]);
    if (D == 3) az.setup(p[2] * inv_dx, c == 2 ? (T)0 : (T)0.5, c == 2 ? lim.h0[2] : lim.h5[2]);
  }
  __device__ __forceinline__ T eval(const T* f, const Shape& s) const { return q2_val<T, D, false>(f, s, ax, ay, az); }
};

// value v = u(p) and d = (grad u)(p) . t (RK_grid's Jacobian update)
template <typename T, int D>
__device__ __forceinline__ void q2_mac_grad_dot(const Mac<T>& u, const fm_grid& g, const Q2Lim<T>& lim, const T* p,
                                                T inv_dx, const T* t, T* v, T* d) {
  MacStencil<T, D, true> st;
  st.setup(lim, p, inv_dx);
#pragma unroll
  for (int c = 0; c < D; ++c) {
    T gr[3];
    q2_grad<T, D>(u.c[c], face_shape(g, c), st.ax(c, 0), st.ax(c, 1), st.ax(c, 2 % D), v[c], gr);
    T acc = 0;
#pragma unroll
    for (int b = 0; b < D; ++b) acc += (gr[b] * inv_dx) * t[b];
    d[c] = acc;
  }
}

// interp_2_scalar on the cell grid (BL = 0.5 on every axis)
template <typename T, int D>
__device__ __forceinline__ T q2_scalar(const T* __restrict__ f, const fm_grid& g, const Q2Lim<T>& lim, const T* p,
                                       T inv_dx) {
  Q2<T, false> ax, ay, az;
  ax.setup(p[0] * inv_dx, (T)0.5, lim.h5[0]);
  ay.setup(p[1] * inv_dx, (T)0.5, lim.h5[1]);
  if (D == 3) az.setup(p[2] * inv_dx, (T)0.5, lim.h5[2]);
  return q2_val<T, D, false>(f, cell_shape(g), ax, ay, az);
}

}  // namespace fm
