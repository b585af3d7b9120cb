// fm_common.cuh -- grid indexing and B-spline interpolation for the flow-map
// kernels (sm_100a).  Everything is templated on the arithmetic type T
// (float = the reference's ti.f32 drop-in; double = the FP64 run used to state
// errors) and on the dimension D (2 or 3).
//
// Layout (shared with include/flowmap_sm100.h): scalar fields are C-order
// [i][j][k] with k fastest; 2D grids use n[2] == 1.  MAC face grid c has
// extent n[c]+1 on axis c.  Vector fields on a grid (psi, T, phi, F) are SoA:
// D consecutive planes of the grid's size.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/flowmap_sm100.h"

namespace fm {

struct Shape {
  int s0, s1, s2;
  __host__ __device__ __forceinline__ long size() const { return (long)s0 * s1 * s2; }
  __host__ __device__ __forceinline__ long idx(int i, int j, int k) const {
    return ((long)i * s1 + j) * s2 + k;
  }
};

__host__ __device__ __forceinline__ Shape cell_shape(const fm_grid& g) {
  return Shape{g.n[0], g.n[1], g.n[2]};
}
__host__ __device__ __forceinline__ Shape face_shape(const fm_grid& g, int c) {
  Shape s{g.n[0], g.n[1], g.n[2]};
  if (c == 0) s.s0 += 1;
  else if (c == 1) s.s1 += 1;
  else if (c == 2) s.s2 += 1;
  return s;
}
__host__ __device__ __forceinline__ int axis_len(const Shape& s, int a) {
  return a == 0 ? s.s0 : (a == 1 ? s.s1 : s.s2);
}

__device__ __forceinline__ void unflatten(const Shape& s, long q, int& i, int& j, int& k) {
  k = (int)(q % s.s2);
  long r = q / s.s2;
  j = (int)(r % s.s1);
  i = (int)(r / s.s1);
}

// Node coordinates: center (I+0.5)*dx; face c: axis c at i*dx, others
// (i+0.5)*dx.  Reference 3D/taichi_utils.py:95-128 (same FP32 ops).
template <typename T, int D>
__device__ __forceinline__ void node_pos(int c, int i, int j, int k, T dx, T* p) {
  int I[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    T fa = (T)I[a];
    if (c < 0 || a != c) fa = fa + (T)0.5;
    p[a] = fa * dx;
  }
}

// --------------------------------------------------------------------------
// B-spline kernels (reference 3D/taichi_utils.py:354-431)
// --------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T bs_N2(T x) {
  T a = fabs(x), r = 0;
  if (a < (T)0.5) r = (T)0.75 - a * a;
  else if (a < (T)1.5) { T t = (T)1.5 - a; r = (T)0.5 * (t * t); }
  return r;
}
template <typename T> __device__ __forceinline__ T bs_dN2(T x) {
  T a = fabs(x), r = 0;
  if (a < (T)0.5) r = (T)-2 * a;
  else if (a < (T)1.5) r = (T)0.5 * ((T)2 * a - (T)3);
  return x < (T)0 ? -r : r;
}
template <typename T> __device__ __forceinline__ T bs_N3(T x) {
  T a = fabs(x), r = 0;
  if (a < (T)1) r = (T)0.5 * (a * a * a) - a * a + (T)(2.0 / 3.0);
  else if (a < (T)2) { T t = (T)2 - a; r = (T)(1.0 / 6.0) * (t * t * t); }
  return r;
}
template <typename T> __device__ __forceinline__ T bs_dN3(T x) {
  T a = fabs(x), r = 0;
  if (a < (T)1) r = (T)1.5 * (a * a) - (T)2 * a;
  else if (a < (T)2) { T t = (T)2 - a; r = (T)-0.5 * (t * t); }
  return x < (T)0 ? -r : r;
}
template <typename T> __device__ __forceinline__ T bs_N4(T x) {
  T a = fabs(x), r = 0;
  T a2 = a * a, a3 = a2 * a, a4 = a2 * a2;
  if (a < (T)0.5) r = (T)(115.0 / 192) - ((T)5 * a2) / (T)8 + a4 / (T)4;
  else if (a < (T)1.5)
    r = (T)(55.0 / 96) + ((T)5 * a) / (T)24 - (T)5 * a2 / (T)4 + ((T)5 * a3) / (T)6 - a4 / (T)6;
  else if (a < (T)2.5)
    r = (T)(625.0 / 384) - ((T)125 * a) / (T)48 + ((T)25 * a2) / (T)16 - ((T)5 * a3) / (T)12 + a4 / (T)24;
  return r;
}
template <typename T> __device__ __forceinline__ T bs_dN4(T x) {
  T a = fabs(x), r = 0;
  T a2 = a * a, a3 = a2 * a;
  if (a < (T)0.5) r = (T)(-5.0 / 4) * a + a3;
  else if (a < (T)1.5) r = (T)(5.0 / 24) - (T)(5.0 / 2) * a + (T)(5.0 / 2) * a2 - (T)(2.0 / 3) * a3;
  else if (a < (T)2.5) r = (T)(-125.0 / 48) + (T)(25.0 / 8) * a - (T)(5.0 / 4) * a2 + (T)(1.0 / 6) * a3;
  return x < (T)0 ? -r : r;
}

template <int ORDER> struct Taps;
template <> struct Taps<2> { static constexpr int lo = -1, n = 4; };
template <> struct Taps<3> { static constexpr int lo = -2, n = 6; };
template <> struct Taps<4> { static constexpr int lo = -3, n = 8; };

template <typename T, int ORDER>
__device__ __forceinline__ void bs_eval(T x, T& w, T& dw) {
  if (ORDER == 2) { w = bs_N2(x); dw = bs_dN2(x); }
  else if (ORDER == 3) { w = bs_N3(x); dw = bs_dN3(x); }
  else { w = bs_N4(x); dw = bs_dN4(x); }
}
template <typename T, int ORDER>
__device__ __forceinline__ T bs_val(T x) {
  if (ORDER == 2) return bs_N2(x);
  else if (ORDER == 3) return bs_N3(x);
  else return bs_N4(x);
}

// Per-axis stencil setup, exactly as the reference: u = p/dx - BL,
// s = max(1, min(u, len-2-eps)), iu = floor(s), tap t at iu+lo+t with
// weight N(s - (iu+lo+t)); tap index clamped to [0, len-1] (sample()).
// The upper bound is computed in double and rounded to T, as Taichi folds
// the Python constant `u_dim - 2 - eps`.
template <typename T, int ORDER, bool GRAD>
struct Axis {
  T w[Taps<ORDER>::n];
  T dw[GRAD ? Taps<ORDER>::n : 1];
  int id[Taps<ORDER>::n];
  __device__ __forceinline__ void setup(T p, T dx, T bl, int len) {
    T u = p / dx;
    u = u - bl;
    const T hi = (T)((double)len - 2.0 - 1e-6);
    T s = u < hi ? u : hi;
    s = s > (T)1 ? s : (T)1;
    T iu = floor(s);
    int iiu = (int)iu;
#pragma unroll
    for (int t = 0; t < Taps<ORDER>::n; ++t) {
      T x = s - (iu + (T)(Taps<ORDER>::lo + t));
      if (GRAD) bs_eval<T, ORDER>(x, w[t], dw[t]);
      else w[t] = bs_val<T, ORDER>(x);
      int ii = iiu + Taps<ORDER>::lo + t;
      id[t] = ii < 0 ? 0 : (ii > len - 1 ? len - 1 : ii);
    }
  }
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Value-only interpolation of one staggered scalar field (sum-factorised:
// contract k, then j, then i).
template <typename T, int D, int ORDER>
__device__ __forceinline__ T interp_val(const T* __restrict__ f, const Shape& s, const T* p, T dx,
                                        T bl0, T bl1, T bl2) {
  constexpr int NT = Taps<ORDER>::n;
  Axis<T, ORDER, false> ax, ay;
  ax.setup(p[0], dx, bl0, s.s0);
  ay.setup(p[1], dx, bl1, s.s1);
  T v = 0;
  if (D == 3) {
    Axis<T, ORDER, false> az;
    az.setup(p[2], dx, bl2, s.s2);
#pragma unroll
    for (int ti = 0; ti < NT; ++ti) {
      T vi = 0;
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) {
        const T* row = f + ((long)ax.id[ti] * s.s1 + ay.id[tj]) * s.s2;
        T vj = 0;
#pragma unroll
        for (int tk = 0; tk < NT; ++tk) vj += ldg(row + az.id[tk]) * az.w[tk];
        vi += vj * ay.w[tj];
      }
      v += vi * ax.w[ti];
    }
  } else {
#pragma unroll
    for (int ti = 0; ti < NT; ++ti) {
      T vi = 0;
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) vi += ldg(f + (long)ax.id[ti] * s.s1 + ay.id[tj]) * ay.w[tj];
      v += vi * ax.w[ti];
    }
  }
  return v;
}

// Value + gradient (interp_grad_2/3/4, reference 3D/taichi_utils.py:433-536).
template <typename T, int D, int ORDER>
__device__ __forceinline__ void interp_grad(const T* __restrict__ f, const Shape& s, const T* p, T dx,
                                            T bl0, T bl1, T bl2, T& val, T* grad) {
  constexpr int NT = Taps<ORDER>::n;
  const T inv_dx = (T)1 / dx;
  Axis<T, ORDER, true> ax, ay;
  ax.setup(p[0], dx, bl0, s.s0);
  ay.setup(p[1], dx, bl1, s.s1);
  if (D == 3) {
    Axis<T, ORDER, true> az;
    az.setup(p[2], dx, bl2, s.s2);
    T v = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int ti = 0; ti < NT; ++ti) {
      T A = 0, B = 0, Cc = 0;  // sum_j wy*a, sum_j dwy*a, sum_j wy*b
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) {
        const T* row = f + ((long)ax.id[ti] * s.s1 + ay.id[tj]) * s.s2;
        T a = 0, b = 0;
#pragma unroll
        for (int tk = 0; tk < NT; ++tk) {
          T fv = ldg(row + az.id[tk]);
          a += fv * az.w[tk];
          b += fv * az.dw[tk];
        }
        A += a * ay.w[tj];
        B += a * ay.dw[tj];
        Cc += b * ay.w[tj];
      }
      v += A * ax.w[ti];
      gx += A * ax.dw[ti];
      gy += B * ax.w[ti];
      gz += Cc * ax.w[ti];
    }
    val = v;
    grad[0] = gx * inv_dx;
    grad[1] = gy * inv_dx;
    grad[2] = gz * inv_dx;
  } else {
    T v = 0, gx = 0, gy = 0;
#pragma unroll
    for (int ti = 0; ti < NT; ++ti) {
      T a = 0, b = 0;
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) {
        T fv = ldg(f + (long)ax.id[ti] * s.s1 + ay.id[tj]);
        a += fv * ay.w[tj];
        b += fv * ay.dw[tj];
      }
      v += a * ax.w[ti];
      gx += a * ax.dw[ti];
      gy += b * ax.w[ti];
    }
    val = v;
    grad[0] = gx * inv_dx;
    grad[1] = gy * inv_dx;
  }
}

// MAC velocity (D component pointers) on grid g.
template <typename T>
struct Mac {
  const T* c[3];
};
template <typename T>
struct MacW {
  T* c[3];
};

// interp_u_MAC (value only) of all components at p.
template <typename T, int D>
__device__ __forceinline__ void interp_mac_val(const Mac<T>& u, const fm_grid& g, const T* p, T dx, T* v) {
#pragma unroll
  for (int c = 0; c < D; ++c) {
    Shape s = face_shape(g, c);
    v[c] = interp_val<T, D, 2>(u.c[c], s, p, dx, c == 0 ? (T)0 : (T)0.5, c == 1 ? (T)0 : (T)0.5,
                               c == 2 ? (T)0 : (T)0.5);
  }
}

// interp_u_MAC_grad: values and G[a][b] = d u_a / d x_b.
template <typename T, int D, int ORDER>
__device__ __forceinline__ void interp_mac_grad(const Mac<T>& u, const fm_grid& g, const T* p, T dx, T* v,
                                                T G[3][3]) {
#pragma unroll
  for (int c = 0; c < D; ++c) {
    Shape s = face_shape(g, c);
    interp_grad<T, D, ORDER>(u.c[c], s, p, dx, c == 0 ? (T)0 : (T)0.5, c == 1 ? (T)0 : (T)0.5,
                             c == 2 ? (T)0 : (T)0.5, v[c], G[c]);
  }
}

// One component c of the MAC velocity at p.
template <typename T, int D>
__device__ __forceinline__ T interp_mac_comp(const Mac<T>& u, const fm_grid& g, int c, const T* p, T dx) {
  Shape s = face_shape(g, c);
  return interp_val<T, D, 2>(u.c[c], s, p, dx, c == 0 ? (T)0 : (T)0.5, c == 1 ? (T)0 : (T)0.5,
                             c == 2 ? (T)0 : (T)0.5);
}

}  // namespace fm
