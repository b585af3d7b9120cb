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

// Programmatic dependent launch (sm_90+).  A kernel launched with the
// programmatic-serialization attribute may become resident while its
// predecessor in the stream still runs; griddepcontrol.wait blocks until that
// predecessor has completed and its writes are visible, and
// launch_dependents lets the next kernel's CTAs be scheduled.  Both are no-ops
// for an ordinary launch.  Called first thing in a kernel, before any global
// memory access, this hides only launch latency: no access ever overlaps the
// predecessor.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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

// Round-to-nearest arithmetic that the compiler may not fuse into FMAs, for
// code that must round exactly as the reference's separate multiplies and
// adds do (the MG operators, the Gaussian-force support test).
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }

// x / nd for the RBGS updates, nd = number of in-domain (fluid) neighbours
// (0..6), rounded exactly as the IEEE division.  FP32: nd = s * d with s a power of
// two (exact scaling) and d in {1, 3, 5}; q0 = y * RN(1/d), e = y - q0 * d
// (exact by FMA), q = q0 + e * RN(1/d).  Checked against the IEEE quotient for
// all 2^32 float inputs and every nd: equal bit for bit whenever
// 2^-100 <= |x| <= 2^100; outside that range (zeros, tiny, huge, non-finite)
// and for nd = 0 the IEEE division is used.  It replaces a division whose
// latency doubled the time of a coarse-level half-sweep.
__device__ __forceinline__ float div_nd(float x, int nd) {
  const float ax = fabsf(x);
  if (ax >= 0x1p-100f && ax <= 0x1p100f && nd > 0) {
    const float s = (nd == 2 || nd == 6) ? 0.5f : (nd == 4 ? 0.25f : 1.0f);
    const float d = (nd == 3 || nd == 6) ? 3.0f : (nd == 5 ? 5.0f : 1.0f);
    const float rd = (nd == 3 || nd == 6) ? (1.0f / 3.0f) : (nd == 5 ? (1.0f / 5.0f) : 1.0f);
    const float y = __fmul_rn(x, s);
    const float q0 = __fmul_rn(y, rd);
    const float e = __fmaf_rn(-q0, d, y);
    return __fmaf_rn(e, rd, q0);
  }
  return x / (float)nd;
}
__device__ __forceinline__ double div_nd(double x, int nd) { return x / (double)nd; }

// Flat index -> (i, j, k).  Grids stay below 2^32 entries (validate_grid), so
// 32-bit unsigned division suffices; 64-bit division would cost ~5x more.
__device__ __forceinline__ void unflatten(const Shape& s, long q, int& i, int& j, int& k) {
  const unsigned uq = (unsigned)q;
  const unsigned r = uq / (unsigned)s.s2;
  k = (int)(uq - r * (unsigned)s.s2);
  const unsigned ii = r / (unsigned)s.s1;
  j = (int)(r - ii * (unsigned)s.s1);
  i = (int)ii;
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

// The reference loops over a window of n taps starting at iu+lo
// (3D/taichi_utils.py:454, :489, :524).  A B-spline of degree ORDER is
// non-zero on |x| < (ORDER+1)/2, so only nz = ORDER+1 consecutive taps of that
// window can carry weight; the others have N = dN = 0 exactly (see
// Axis::setup).  The kernels visit just those nz taps: 27 instead of 64 taps
// per 3D quadratic sample, 64 instead of 216 cubic, 125 instead of 512 quartic.
template <int ORDER> struct Taps;
template <> struct Taps<2> { static constexpr int lo = -1, n = 4, nz = 3; };
template <> struct Taps<3> { static constexpr int lo = -2, n = 6, nz = 4; };
template <> struct Taps<4> { static constexpr int lo = -3, n = 8, nz = 5; };

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
//
// Non-zero window: with f = s - iu in [0,1) (exact in floating point), tap t of
// the reference window sits at x_t = f - lo - t, which is exact as well, and is
// non-zero iff |x_t| < (ORDER+1)/2.  Quadratic: taps 0..2 when f < 0.5, else
// 1..3; cubic: taps 1..4; quartic: 1..5 when f < 0.5, else 2..6.
template <typename T, int ORDER, bool GRAD>
struct Axis {
  static constexpr int NZ = Taps<ORDER>::nz;
  T w[NZ];
  T dw[GRAD ? NZ : 1];
  int id[NZ];
  __device__ __forceinline__ void setup(T p, T dx, T bl, int len) {
    T u = p / dx;
    u = u - bl;
    const T hi = (T)((double)len - 2.0 - 1e-6);
    T s = u < hi ? u : hi;
    s = s > (T)1 ? s : (T)1;
    const T iu = floor(s);
    const int iiu = (int)iu;
    const T f = s - iu;
    int t0;
    if (ORDER == 3) t0 = 1;
    else if (ORDER == 2) t0 = f >= (T)0.5 ? 1 : 0;
    else t0 = f >= (T)0.5 ? 2 : 1;
#pragma unroll
    for (int t = 0; t < NZ; ++t) {
      const int off = Taps<ORDER>::lo + t0 + t;
      const T x = s - (iu + (T)off);
      if (GRAD) bs_eval<T, ORDER>(x, w[t], dw[t]);
      else w[t] = bs_val<T, ORDER>(x);
      const int ii = iiu + off;
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
  constexpr int NT = Taps<ORDER>::nz;
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
  constexpr int NT = Taps<ORDER>::nz;
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

// Gradient of f and value of h, two fields on the same staggered grid sampled
// at the same position: one stencil setup, both fields gathered in one pass
// (calculate_nabla_u_w interpolates u and w at the same node, 3D/flowmap.py:368-369).
template <typename T, int D, int ORDER>
__device__ __forceinline__ void interp_grad_val2(const T* __restrict__ f, const T* __restrict__ h, const Shape& s,
                                                 const T* p, T dx, T bl0, T bl1, T bl2, T* grad, T& hval) {
  constexpr int NT = Taps<ORDER>::nz;
  const T inv_dx = (T)1 / dx;
  Axis<T, ORDER, true> ax, ay;
  ax.setup(p[0], dx, bl0, s.s0);
  ay.setup(p[1], dx, bl1, s.s1);
  if (D == 3) {
    Axis<T, ORDER, true> az;
    az.setup(p[2], dx, bl2, s.s2);
    T gx = 0, gy = 0, gz = 0, hv = 0;
#pragma unroll 1
    for (int ti = 0; ti < NT; ++ti) {
      T A = 0, B = 0, Cc = 0, H = 0;
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) {
        const long row = ((long)ax.id[ti] * s.s1 + ay.id[tj]) * s.s2;
        T a = 0, b = 0, hh = 0;
#pragma unroll
        for (int tk = 0; tk < NT; ++tk) {
          const T fv = ldg(f + row + az.id[tk]);
          const T hv2 = ldg(h + row + az.id[tk]);
          a += fv * az.w[tk];
          b += fv * az.dw[tk];
          hh += hv2 * az.w[tk];
        }
        A += a * ay.w[tj];
        B += a * ay.dw[tj];
        Cc += b * ay.w[tj];
        H += hh * ay.w[tj];
      }
      gx += A * ax.dw[ti];
      gy += B * ax.w[ti];
      gz += Cc * ax.w[ti];
      hv += H * ax.w[ti];
    }
    grad[0] = gx * inv_dx;
    grad[1] = gy * inv_dx;
    grad[2] = gz * inv_dx;
    hval = hv;
  } else {
    T gx = 0, gy = 0, hv = 0;
#pragma unroll
    for (int ti = 0; ti < NT; ++ti) {
      T a = 0, b = 0, hh = 0;
#pragma unroll
      for (int tj = 0; tj < NT; ++tj) {
        const long idx = (long)ax.id[ti] * s.s1 + ay.id[tj];
        const T fv = ldg(f + idx);
        a += fv * ay.w[tj];
        b += fv * ay.dw[tj];
        hh += ldg(h + idx) * ay.w[tj];
      }
      gx += a * ax.dw[ti];
      gy += b * ax.w[ti];
      hv += hh * ax.w[ti];
    }
    grad[0] = gx * inv_dx;
    grad[1] = gy * inv_dx;
    hval = hv;
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

// Select element c (a runtime value such as blockIdx.y) without indexing the
// by-value kernel parameter dynamically (which would copy it to local memory).
template <typename P>
__device__ __forceinline__ P pick3(const P& a, const P& b, const P& c2, int c) {
  return c == 0 ? a : (c == 1 ? b : c2);
}
template <typename T>
__device__ __forceinline__ const T* pick(const Mac<T>& m, int c) { return pick3(m.c[0], m.c[1], m.c[2], c); }
template <typename T>
__device__ __forceinline__ T* pick(const MacW<T>& m, int c) { return pick3(m.c[0], m.c[1], m.c[2], c); }

// One component c of the MAC velocity at p.
template <typename T, int D>
__device__ __forceinline__ T interp_mac_comp(const Mac<T>& u, const fm_grid& g, int c, const T* p, T dx) {
  Shape s = face_shape(g, c);
  return interp_val<T, D, 2>(pick(u, c), s, p, dx, c == 0 ? (T)0 : (T)0.5, c == 1 ? (T)0 : (T)0.5,
                             c == 2 ? (T)0 : (T)0.5);
}

// Velocity v = u(p) and the Jacobian-row update d = (grad u)(p) . t, without
// materialising the 3x3 gradient (RK_grid's dT/dt = grad_u @ T,
// 3D/flowmap.py:95).
template <typename T, int D>
__device__ __forceinline__ void interp_mac_grad_dot(const Mac<T>& u, const fm_grid& g, const T* p, T dx,
                                                    const T* t, T* v, T* d) {
#pragma unroll
  for (int c = 0; c < D; ++c) {
    Shape s = face_shape(g, c);
    T gr[3];
    interp_grad<T, D, 2>(u.c[c], s, p, dx, c == 0 ? (T)0 : (T)0.5, c == 1 ? (T)0 : (T)0.5,
                         c == 2 ? (T)0 : (T)0.5, v[c], gr);
    T acc = 0;
#pragma unroll
    for (int b = 0; b < D; ++b) acc += gr[b] * t[b];
    d[c] = acc;
  }
}

}  // namespace fm
