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
// contiguous and one row pointer serves a whole k-triple.
// Positions are scaled by 1/dx (exact for the power-of-two dx of the
// benchmark grids; within one ulp of the reference's p/dx otherwise).
#pragma once
#include "fm_common.cuh"

namespace fm {

template <typename T, bool GRAD>
struct Q2 {
  int i0;
  T w0, w1, w2;
  T d0, d1, d2;
  __device__ __forceinline__ void setup(T pos_scaled, T bl, int len) {
    const T u = pos_scaled - bl;
    const T hi = (T)((double)len - 2.0 - 1e-6);
    T s = u < hi ? u : hi;
    s = s > (T)1 ? s : (T)1;
    const T iu = floor(s);
    const T f = s - iu;
    const bool up = f >= (T)0.5;
    const T t = up ? f - (T)1 : f;
    i0 = (int)iu - 1 + (up ? 1 : 0);
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

// value of one staggered field with shape s at the stencil (ax, ay, az)
template <typename T, int D, bool G>
__device__ __forceinline__ T q2_val(const T* __restrict__ f, const Shape& s, const Q2<T, G>& ax, const Q2<T, G>& ay,
                                    const Q2<T, G>& az) {
  if (D == 3) {
    const long sj = s.s2, si = (long)s.s1 * s.s2;
    const T* p = f + ((long)ax.i0 * s.s1 + ay.i0) * s.s2 + az.i0;
    const T wy[3] = {ay.w0, ay.w1, ay.w2};
    const T wx[3] = {ax.w0, ax.w1, ax.w2};
    T v = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T vi = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T* r = p + i * si + j * sj;
        const T a = ldg(r) * az.w0 + ldg(r + 1) * az.w1 + ldg(r + 2) * az.w2;
        vi += a * wy[j];
      }
      v += vi * wx[i];
    }
    return v;
  } else {
    const long si = s.s1;
    const T* p = f + (long)ax.i0 * s.s1 + ay.i0;
    const T wx[3] = {ax.w0, ax.w1, ax.w2};
    T v = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T* r = p + i * si;
      v += (ldg(r) * ay.w0 + ldg(r + 1) * ay.w1 + ldg(r + 2) * ay.w2) * wx[i];
    }
    return v;
  }
}

// value and gradient (unscaled by 1/dx) of one staggered field
template <typename T, int D>
__device__ __forceinline__ void q2_grad(const T* __restrict__ f, const Shape& s, const Q2<T, true>& ax,
                                        const Q2<T, true>& ay, const Q2<T, true>& az, T& v, T* g) {
  const T wx[3] = {ax.w0, ax.w1, ax.w2}, dx_[3] = {ax.d0, ax.d1, ax.d2};
  const T wy[3] = {ay.w0, ay.w1, ay.w2}, dy_[3] = {ay.d0, ay.d1, ay.d2};
  if (D == 3) {
    const long sj = s.s2, si = (long)s.s1 * s.s2;
    const T* p = f + ((long)ax.i0 * s.s1 + ay.i0) * s.s2 + az.i0;
    T vv = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T A = 0, B = 0, Cc = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T* r = p + i * si + j * sj;
        const T f0 = ldg(r), f1 = ldg(r + 1), f2 = ldg(r + 2);
        const T a = f0 * az.w0 + f1 * az.w1 + f2 * az.w2;
        const T b = f0 * az.d0 + f1 * az.d1 + f2 * az.d2;
        A += a * wy[j];
        B += a * dy_[j];
        Cc += b * wy[j];
      }
      vv += A * wx[i];
      gx += A * dx_[i];
      gy += B * wx[i];
      gz += Cc * wx[i];
    }
    v = vv;
    g[0] = gx;
    g[1] = gy;
    g[2] = gz;
  } else {
    const long si = s.s1;
    const T* p = f + (long)ax.i0 * s.s1 + ay.i0;
    T vv = 0, gx = 0, gy = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T* r = p + i * si;
      const T f0 = ldg(r), f1 = ldg(r + 1), f2 = ldg(r + 2);
      const T a = f0 * ay.w0 + f1 * ay.w1 + f2 * ay.w2;
      const T b = f0 * ay.d0 + f1 * ay.d1 + f2 * ay.d2;
      vv += a * wx[i];
      gx += a * dx_[i];
      gy += b * wx[i];
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
  __device__ __forceinline__ void setup(const fm_grid& g, const T* p, T inv_dx) {
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const T ps = p[a] * inv_dx;
      s0[a].setup(ps, (T)0, g.n[a] + 1);
      s5[a].setup(ps, (T)0.5, g.n[a]);
    }
  }
  __device__ __forceinline__ const Q2<T, G>& ax(int c, int a) const { return a == c ? s0[a] : s5[a]; }
};

// interp_u_MAC (value only), all components
template <typename T, int D>
__device__ __forceinline__ void q2_mac_val(const Mac<T>& u, const fm_grid& g, const T* p, T inv_dx, T* v) {
  MacStencil<T, D, false> st;
  st.setup(g, p, inv_dx);
#pragma unroll
  for (int c = 0; c < D; ++c) v[c] = q2_val<T, D, false>(u.c[c], face_shape(g, c), st.ax(c, 0), st.ax(c, 1), st.ax(c, 2 % D));
}

// Stencil of face component c (runtime) at p.
template <typename T, int D>
struct CompStencil {
  Q2<T, false> ax, ay, az;
  __device__ __forceinline__ void setup(const fm_grid& g, int c, const T* p, T inv_dx) {
    ax.setup(p[0] * inv_dx, c == 0 ? (T)0 : (T)0.5, g.n[0] + (c == 0));
    ay.setup(p[1] * inv_dx, c == 1 ? (T)0 : (T)0.5, g.n[1] + (c == 1));
    if (D == 3) az.setup(p[2] * inv_dx, c == 2 ? (T)0 : (T)0.5, g.n[2] + (c == 2));
  }
  __device__ __forceinline__ T eval(const T* f, const Shape& s) const { return q2_val<T, D, false>(f, s, ax, ay, az); }
};

// one component c (runtime) of the MAC velocity
template <typename T, int D>
__device__ __forceinline__ T q2_mac_comp(const Mac<T>& u, const fm_grid& g, int c, const T* p, T inv_dx) {
  CompStencil<T, D> st;
  st.setup(g, c, p, inv_dx);
  return st.eval(pick(u, c), face_shape(g, c));
}

// value v = u(p) and d = (grad u)(p) . t (RK_grid's Jacobian update)
template <typename T, int D>
__device__ __forceinline__ void q2_mac_grad_dot(const Mac<T>& u, const fm_grid& g, const T* p, T inv_dx,
                                                const T* t, T* v, T* d) {
  MacStencil<T, D, true> st;
  st.setup(g, p, inv_dx);
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
__device__ __forceinline__ T q2_scalar(const T* __restrict__ f, const fm_grid& g, const T* p, T inv_dx) {
  Q2<T, false> ax, ay, az;
  ax.setup(p[0] * inv_dx, (T)0.5, g.n[0]);
  ay.setup(p[1] * inv_dx, (T)0.5, g.n[1]);
  if (D == 3) az.setup(p[2] * inv_dx, (T)0.5, g.n[2]);
  return q2_val<T, D, false>(f, cell_shape(g), ax, ay, az);
}

}  // namespace fm
