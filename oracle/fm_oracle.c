/*
 * fm_oracle.c -- CPU restatement of the reference's flow-map kernels and MGPCG
 * Poisson solver.  TEST INFRASTRUCTURE ONLY: this file is the parity checker for
 * the CUDA library and is never linked into, called by, or shipped with the
 * product path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.
 *
 * Compiled twice (see oracle/Makefile):
 *   REAL=double -> liboracle_f64.so : the FP64 reference algorithm
 *   REAL=float  -> liboracle_f32.so : FP32, same operation order as the Taichi
 *                                     source (default_fp=ti.f32)
 *
 * Parity status: the reference (Taichi + an unvendored CUDA Poisson solver) has
 * no tests or golden vectors for this path and cannot run in this container, so
 * this restatement is "parity unpinned": it is pinned only by known-answer
 * tests derived from the mathematics (B-spline partition of unity, exactness on
 * polynomials, adjoint identities) in tests/test_oracle_kat.py.
 *
 * Layout: every scalar field is C-order [i][j][k] (k fastest), FP `REAL`.
 * 2D grids use nz == 1 and dim == 2.  MAC face grid c has extent n[c]+1 on
 * axis c.  Vector fields on a grid (psi, T, phi, F) are SoA: `dim` consecutive
 * planes of the grid's size.
 *
 * Every function cites the reference file:line it restates.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

typedef struct {
    int dim;        /* 2 or 3 */
    int n[3];       /* cell counts nx, ny, nz (nz == 1 in 2D) */
} fmo_grid;

/* ------------------------------------------------------------------------ */
/* index helpers                                                             */
/* ------------------------------------------------------------------------ */
static inline long lin(const int *s, int i, int j, int k) {
    return ((long)i * s[1] + j) * s[2] + k;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline long gsize(const int *s) { return (long)s[0] * s[1] * s[2]; }

/* face grid extents for MAC component c (c < dim) */
static inline void face_shape(const fmo_grid *g, int c, int *s) {
    s[0] = g->n[0]; s[1] = g->n[1]; s[2] = g->n[2];
    s[c] += 1;
}
static inline void cell_shape(const fmo_grid *g, int *s) {
    s[0] = g->n[0]; s[1] = g->n[1]; s[2] = g->n[2];
}

/* node coordinates.  Reference: 3D/taichi_utils.py:95-128 (center, x_coords_func,
 * y_coords_func, z_coords_func) and 2D/vortex/taichi_utils.py:137-150.
 * center: (I+0.5)*dx ; face c: axis c at i*dx, other axes (i+0.5)*dx. */
static inline void node_pos(int dim, int c, int i, int j, int k, real dx, real *p) {
    int I[3] = {i, j, k};
    for (int a = 0; a < dim; ++a) {
        real fa = (real)I[a];
        if (c < 0 || a != c) fa = fa + (real)0.5;
        p[a] = fa * dx;
    }
    if (dim == 2) p[2] = 0;
}

/* ------------------------------------------------------------------------ */
/* B-spline kernels.  Reference: 3D/taichi_utils.py:354-431                  */
/* ------------------------------------------------------------------------ */
static inline real N2(real x) {
    real a = fabs(x), r = 0;
    if (a < (real)0.5) r = (real)0.75 - a * a;
    else if (a < (real)1.5) { real t = (real)1.5 - a; r = (real)0.5 * (t * t); }
    return r;
}
static inline real dN2(real x) {
    real a = fabs(x), r = 0;
    if (a < (real)0.5) r = (real)-2 * a;
    else if (a < (real)1.5) r = (real)0.5 * ((real)2 * a - (real)3);
    if (x < 0) r = -r;
    return r;
}
static inline real N3(real x) {
    real a = fabs(x), r = 0;
    if (a < 1) r = (real)0.5 * (a * a * a) - a * a + (real)(2.0 / 3.0);
    else if (a < 2) { real t = 2 - a; r = (real)(1.0 / 6.0) * (t * t * t); }
    return r;
}
static inline real dN3(real x) {
    real a = fabs(x), r = 0;
    if (a < 1) r = (real)1.5 * (a * a) - 2 * a;
    else if (a < 2) { real t = 2 - a; r = (real)-0.5 * (t * t); }
    if (x < 0) r = -r;
    return r;
}
static inline real N4(real x) {
    real a = fabs(x), r = 0;
    real a2 = a * a, a3 = a2 * a, a4 = a2 * a2;
    if (a < (real)0.5)
        r = (real)(115.0 / 192) - ((real)5 * a2) / 8 + a4 / 4;
    else if (a < (real)1.5)
        r = (real)(55.0 / 96) + ((real)5 * a) / 24 - (real)5 * a2 / 4 + ((real)5 * a3) / 6 - a4 / 6;
    else if (a < (real)2.5)
        r = (real)(625.0 / 384) - ((real)125 * a) / 48 + ((real)25 * a2) / 16 - ((real)5 * a3) / 12 + a4 / 24;
    return r;
}
static inline real dN4(real x) {
    real a = fabs(x), r = 0;
    real a2 = a * a, a3 = a2 * a;
    if (a < (real)0.5)
        r = (real)(-5.0 / 4) * a + a3;
    else if (a < (real)1.5)
        r = (real)(5.0 / 24) - (real)(5.0 / 2) * a + (real)(5.0 / 2) * a2 - (real)(2.0 / 3) * a3;
    else if (a < (real)2.5)
        r = (real)(-125.0 / 48) + (real)(25.0 / 8) * a - (real)(5.0 / 4) * a2 + (real)(1.0 / 6) * a3;
    if (x < 0) r = -r;
    return r;
}

/* ------------------------------------------------------------------------ */
/* interp_grad_{2,3,4}: B-spline value and gradient of a staggered scalar     */
/* field at an arbitrary position.                                            */
/* Reference: 3D/taichi_utils.py:433-536 (interp_grad_2/3/4),                 */
/*            2D/vortex/taichi_utils.py:413-520, sample() 3D :130-136.        */
/* order 2 -> taps [-1,3), order 3 -> [-2,4), order 4 -> [-3,5).              */
/* ------------------------------------------------------------------------ */
static void interp_grad(int dim, int order, const real *f, const int *s, const real *p,
                        real dx, const real *BL, real *val, real *grad /* may be NULL */) {
    int lo = order == 2 ? -1 : (order == 3 ? -2 : -3);
    int nt = order == 2 ? 4 : (order == 3 ? 6 : 8);
    real w[3][8], dw[3][8];
    int id[3][8];
    int ntap[3] = {1, 1, 1};
    real inv_dx = (real)1 / dx;
    for (int a = 0; a < 3; ++a) { w[a][0] = 1; dw[a][0] = 0; id[a][0] = 0; }
    for (int a = 0; a < dim; ++a) {
        real u = p[a] / dx;
        u = u - BL[a];
        real hi = (real)((double)s[a] - 2.0 - 1e-6);
        real sa = u < hi ? u : hi;
        sa = sa > (real)1 ? sa : (real)1;
        real iu = floor(sa);
        ntap[a] = nt;
        for (int t = 0; t < nt; ++t) {
            real x = sa - (iu + (real)(lo + t));
            if (order == 2) { w[a][t] = N2(x); dw[a][t] = dN2(x); }
            else if (order == 3) { w[a][t] = N3(x); dw[a][t] = dN3(x); }
            else { w[a][t] = N4(x); dw[a][t] = dN4(x); }
            id[a][t] = clampi((int)(iu + (real)(lo + t)), 0, s[a] - 1);
        }
    }
    real v = 0, gx = 0, gy = 0, gz = 0;
    for (int ti = 0; ti < ntap[0]; ++ti)
        for (int tj = 0; tj < ntap[1]; ++tj)
            for (int tk = 0; tk < ntap[2]; ++tk) {
                real value = f[lin(s, id[0][ti], id[1][tj], id[2][tk])];
                gx += inv_dx * (value * dw[0][ti] * w[1][tj] * w[2][tk]);
                gy += inv_dx * (value * w[0][ti] * dw[1][tj] * w[2][tk]);
                if (dim == 3) gz += inv_dx * (value * w[0][ti] * w[1][tj] * dw[2][tk]);
                v += value * w[0][ti] * w[1][tj] * w[2][tk];
            }
    *val = v;
    if (grad) { grad[0] = gx; grad[1] = gy; grad[2] = gz; }
}

typedef struct { const real *c[3]; } mac_c;  /* const MAC velocity */
typedef struct { real *c[3]; } mac_m;        /* mutable MAC velocity */

/* interp_u_MAC_grad (order 2) / interp_u_MAC_grad3 (order 3 in 3D, 4 in 2D).
 * Reference: 3D/taichi_utils.py:596-608, 2D/vortex/taichi_utils.py:636-646.
 * G[a][b] = d u_a / d x_b (rows = gradient of each component). */
static void interp_mac(const fmo_grid *g, int order, mac_c u, const real *p, real dx,
                       real *val, real G[3][3]) {
    for (int c = 0; c < g->dim; ++c) {
        int s[3]; face_shape(g, c, s);
        real BL[3] = {0.5, 0.5, 0.5};
        BL[c] = 0;
        real gr[3];
        interp_grad(g->dim, order, u.c[c], s, p, dx, BL, &val[c], G ? gr : NULL);
        if (G) { G[c][0] = gr[0]; G[c][1] = gr[1]; G[c][2] = gr[2]; }
    }
}

/* interp_2_scalar on a cell-centred field.  Reference: 3D/taichi_utils.py:567-594 */
static real interp_scalar(const fmo_grid *g, const real *f, const real *p, real dx) {
    int s[3]; cell_shape(g, s);
    real BL[3] = {0.5, 0.5, 0.5};
    real v;
    interp_grad(g->dim, 2, f, s, p, dx, BL, &v, NULL);
    return v;
}

/* ------------------------------------------------------------------------ */
/* exported point queries (used by the known-answer tests)                   */
/* ------------------------------------------------------------------------ */
void fmo_interp_grad(int dim, int order, const real *f, const int *shape, const real *p,
                     real dx, const real *BL, real *out4) {
    real v, gr[3];
    interp_grad(dim, order, f, shape, p, dx, BL, &v, gr);
    out4[0] = v; out4[1] = gr[0]; out4[2] = gr[1]; out4[3] = gr[2];
}
void fmo_bspline(int order, int deriv, const real *x, real *y, long n) {
    for (long i = 0; i < n; ++i) {
        real r;
        if (order == 2) r = deriv ? dN2(x[i]) : N2(x[i]);
        else if (order == 3) r = deriv ? dN3(x[i]) : N3(x[i]);
        else r = deriv ? dN4(x[i]) : N4(x[i]);
        y[i] = r;
    }
}

/* ------------------------------------------------------------------------ */
/* RK_grid: flow map + Jacobian march on a face grid (in place).             */
/* Reference: 3D/flowmap.py:85-137 (RK4_grid, RK2_grid),                      */
/*            2D/vortex/flowmap.py:125-175.                                   */
/* psi, T: dim planes each on face grid `face` (face = -1 -> centre grid and  */
/* T must be NULL: RK_grid_only_psi, 3D/flowmap.py:139-179).                  */
/* ------------------------------------------------------------------------ */
void fmo_rk_grid(const fmo_grid *g, int rk, real dx, real dt, int face, real *psi, real *T,
                 const real *ux, const real *uy, const real *uz) {
    int s[3];
    if (face >= 0) face_shape(g, face, s); else cell_shape(g, s);
    long N = gsize(s);
    int d = g->dim;
    mac_c u = {{ux, uy, uz}};
    real neg_dt = -1 * dt;
    #pragma omp parallel for schedule(static)
    for (long q = 0; q < N; ++q) {
        real P[3] = {0, 0, 0}, Tv[3] = {0, 0, 0};
        for (int a = 0; a < d; ++a) { P[a] = psi[a * N + q]; if (T) Tv[a] = T[a * N + q]; }
        real u1[3] = {0}, u2[3] = {0}, u3[3] = {0}, u4[3] = {0};
        real G[3][3];
        real dT1[3] = {0}, dT2[3] = {0}, dT3[3] = {0}, dT4[3] = {0};
        real p1[3] = {0}, p2[3] = {0}, p3[3] = {0}, T1[3] = {0}, T2[3] = {0}, T3[3] = {0};
        real h = (real)0.5 * neg_dt;
#define MATVEC(out, Gm, v) for (int aa = 0; aa < d; ++aa) { real acc = 0; for (int bb = 0; bb < d; ++bb) acc += Gm[aa][bb] * v[bb]; out[aa] = acc; }
        interp_mac(g, 2, u, P, dx, u1, G);
        if (T) { MATVEC(dT1, G, Tv); }
        for (int a = 0; a < d; ++a) { p1[a] = P[a] + h * u1[a]; T1[a] = Tv[a] + h * dT1[a]; }
        interp_mac(g, 2, u, p1, dx, u2, G);
        if (T) { MATVEC(dT2, G, T1); }
        if (rk == 2) {
            for (int a = 0; a < d; ++a) {
                psi[a * N + q] = P[a] + neg_dt * u2[a];
                if (T) T[a * N + q] = Tv[a] + neg_dt * dT2[a];
            }
            continue;
        }
        for (int a = 0; a < d; ++a) { p2[a] = P[a] + h * u2[a]; T2[a] = Tv[a] + h * dT2[a]; }
        interp_mac(g, 2, u, p2, dx, u3, G);
        if (T) { MATVEC(dT3, G, T2); }
        for (int a = 0; a < d; ++a) { p3[a] = P[a] + (real)1.0 * neg_dt * u3[a]; T3[a] = Tv[a] + (real)1.0 * neg_dt * dT3[a]; }
        interp_mac(g, 2, u, p3, dx, u4, G);
        if (T) { MATVEC(dT4, G, T3); }
#undef MATVEC
        real c6 = neg_dt * (real)1 / (real)6;
        for (int a = 0; a < d; ++a) {
            psi[a * N + q] = P[a] + c6 * (u1[a] + 2 * u2[a] + 2 * u3[a] + u4[a]);
            if (T) T[a * N + q] = Tv[a] + c6 * (dT1[a] + 2 * dT2[a] + 2 * dT3[a] + dT4[a]);
        }
    }
}

/* midpoint / RK4 backtrace used by advect_u_grid and advect_scalar_grid.
 * Reference: 3D/flowmap.py:202-320 */
static void backtrace(const fmo_grid *g, int rk, mac_c u0, const real *X, real dx, real dt, real *p) {
    int d = g->dim;
    real v1[3] = {0}, v2[3] = {0}, v3[3] = {0}, v4[3] = {0};
    real p2[3] = {0}, p3[3] = {0}, p4[3] = {0};
    interp_mac(g, 2, u0, X, dx, v1, NULL);
    for (int a = 0; a < d; ++a) p2[a] = X[a] - v1[a] * dt * (real)0.5;
    interp_mac(g, 2, u0, p2, dx, v2, NULL);
    if (rk == 2) {
        for (int a = 0; a < d; ++a) p[a] = X[a] - v2[a] * dt;
        return;
    }
    for (int a = 0; a < d; ++a) p3[a] = X[a] - v2[a] * dt * (real)0.5;
    interp_mac(g, 2, u0, p3, dx, v3, NULL);
    for (int a = 0; a < d; ++a) p4[a] = X[a] - v3[a] * dt;
    interp_mac(g, 2, u0, p4, dx, v4, NULL);
    for (int a = 0; a < d; ++a) p[a] = X[a] - (v1[a] + 2 * v2[a] + 2 * v3[a] + v4[a]) / (real)6.0 * dt;
}

/* advect_u_grid (RK2/RK4): semi-Lagrangian advection of u1 by u0 sampled at the
 * backtraced face nodes.  Reference: 3D/flowmap.py:202-282, 2D/vortex/flowmap.py:233-291.
 * Output must not alias the inputs. */
void fmo_advect_u_grid(const fmo_grid *g, int rk, real dx, real dt,
                       const real *u0x, const real *u0y, const real *u0z,
                       const real *u1x, const real *u1y, const real *u1z,
                       real *u2x, real *u2y, real *u2z) {
    mac_c u0 = {{u0x, u0y, u0z}}, u1 = {{u1x, u1y, u1z}};
    real *out[3] = {u2x, u2y, u2z};
    for (int c = 0; c < g->dim; ++c) {
        int s[3]; face_shape(g, c, s);
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    real X[3], p[3], v5[3];
                    node_pos(g->dim, c, i, j, k, dx, X);
                    backtrace(g, rk, u0, X, dx, dt, p);
                    if (g->dim == 2) p[2] = 0;
                    interp_mac(g, 2, u1, p, dx, v5, NULL);
                    out[c][lin(s, i, j, k)] = v5[c];
                }
    }
}

/* advect_scalar_grid.  Reference: 3D/flowmap.py:284-320 */
void fmo_advect_scalar_grid(const fmo_grid *g, int rk, real dx, real dt,
                            const real *u0x, const real *u0y, const real *u0z,
                            const real *s1, real *s2) {
    mac_c u0 = {{u0x, u0y, u0z}};
    int s[3]; cell_shape(g, s);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < s[0]; ++i)
        for (int j = 0; j < s[1]; ++j)
            for (int k = 0; k < s[2]; ++k) {
                real X[3], p[3];
                node_pos(g->dim, -1, i, j, k, dx, X);
                backtrace(g, rk, u0, X, dx, dt, p);
                if (g->dim == 2) p[2] = 0;
                s2[lin(s, i, j, k)] = interp_scalar(g, s1, p, dx);
            }
}

/* advect_u: impulse pullback u1_c = T_c . u0(psi_c).  Reference: 3D/flowmap.py:51-69 */
void fmo_pullback_u(const fmo_grid *g, real dx,
                    const real *u0x, const real *u0y, const real *u0z,
                    real *u1x, real *u1y, real *u1z,
                    const real *Tx, const real *Ty, const real *Tz,
                    const real *px, const real *py, const real *pz) {
    mac_c u0 = {{u0x, u0y, u0z}};
    real *out[3] = {u1x, u1y, u1z};
    const real *T[3] = {Tx, Ty, Tz}, *P[3] = {px, py, pz};
    int d = g->dim;
    for (int c = 0; c < d; ++c) {
        int s[3]; face_shape(g, c, s);
        long N = gsize(s);
        #pragma omp parallel for schedule(static)
        for (long q = 0; q < N; ++q) {
            real p[3] = {0, 0, 0}, v[3] = {0, 0, 0};
            for (int a = 0; a < d; ++a) p[a] = P[c][a * N + q];
            interp_mac(g, 2, u0, p, dx, v, NULL);
            real acc = 0;
            for (int a = 0; a < d; ++a) acc += T[c][a * N + q] * v[a];
            out[c][q] = acc;
        }
    }
}

/* advect_scalar: s1 = s0(psi).  Reference: 3D/flowmap.py:71-79 */
void fmo_pullback_scalar(const fmo_grid *g, real dx, const real *s0, real *s1, const real *psi) {
    int s[3]; cell_shape(g, s);
    long N = gsize(s);
    int d = g->dim;
    #pragma omp parallel for schedule(static)
    for (long q = 0; q < N; ++q) {
        real p[3] = {0, 0, 0};
        for (int a = 0; a < d; ++a) p[a] = psi[a * N + q];
        s1[q] = interp_scalar(g, s0, p, dx);
    }
}

/* accumulate_init (ab3 = 0) and accumulate_init_new (ab3 = 1, AB3 history).
 * Reference: 3D/flowmap.py:485-545, 2D/vortex/flowmap.py:508-553.
 * The ind == 1 branch keeps the reference's (23 Fv - 16 Fv + 5 H_prev)/12. */
void fmo_accumulate_init(const fmo_grid *g, real dx, real dt, int ab3, int ind,
                         const real *fx, const real *fy, const real *fz,
                         real *ix, real *iy, real *iz,
                         const real *Fx, const real *Fy, const real *Fz,
                         const real *px, const real *py, const real *pz,
                         real *Hpx, real *Hppx, real *Hpy, real *Hppy, real *Hpz, real *Hppz) {
    mac_c f = {{fx, fy, fz}};
    real *init[3] = {ix, iy, iz};
    const real *F[3] = {Fx, Fy, Fz}, *P[3] = {px, py, pz};
    real *Hp[3] = {Hpx, Hpy, Hpz}, *Hpp[3] = {Hppx, Hppy, Hppz};
    int d = g->dim;
    for (int c = 0; c < d; ++c) {
        int s[3]; face_shape(g, c, s);
        long N = gsize(s);
        #pragma omp parallel for schedule(static)
        for (long q = 0; q < N; ++q) {
            real p[3] = {0, 0, 0}, v[3] = {0, 0, 0};
            for (int a = 0; a < d; ++a) p[a] = P[c][a * N + q];
            interp_mac(g, 2, f, p, dx, v, NULL);
            real Fv = 0, Fv23 = 0, Fv16 = 0;
            for (int a = 0; a < d; ++a) {
                real Fa = F[c][a * N + q];
                Fv += Fa * v[a];
                Fv23 += ((real)23 * Fa) * v[a];
                Fv16 += ((real)16 * Fa) * v[a];
            }
            if (!ab3 || ind == 0) {
                init[c][q] += Fv * dt;
            } else if (ind == 1) {
                init[c][q] += (Fv23 - Fv16 + (real)5 * Hp[c][q]) / (real)12 * dt;
            } else {
                init[c][q] += (Fv23 - (real)16 * Hp[c][q] + (real)5 * Hpp[c][q]) / (real)12 * dt;
            }
            if (ab3) {
                Hpp[c][q] = Hp[c][q];
                Hp[c][q] = Fv;
            }
        }
    }
}

/* calculate_nabla_u_w: r_c = ((grad u)^T w)_c at face nodes, interpolating u
 * and w with interp_u_MAC_grad3 at the grid nodes.  The reference uses the
 * cubic kernel in 3D (3D/flowmap.py:359-380, 3D/taichi_utils.py:603-608) and
 * the quartic kernel in 2D (2D/vortex/flowmap.py:361-377,
 * 2D/vortex/taichi_utils.py:642-646).  `order` selects it. */
void fmo_nabla_u_w(const fmo_grid *g, int order, real dx,
                   const real *ux, const real *uy, const real *uz,
                   const real *wx, const real *wy, const real *wz,
                   real *rx, real *ry, real *rz) {
    mac_c u = {{ux, uy, uz}}, w = {{wx, wy, wz}};
    real *out[3] = {rx, ry, rz};
    int d = g->dim;
    for (int c = 0; c < d; ++c) {
        int s[3]; face_shape(g, c, s);
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    real X[3], uv[3] = {0}, wv[3] = {0}, G[3][3];
                    node_pos(d, c, i, j, k, dx, X);
                    interp_mac(g, order, u, X, dx, uv, G);
                    interp_mac(g, order, w, X, dx, wv, NULL);
                    real acc = 0;
                    for (int a = 0; a < d; ++a) acc += G[a][c] * wv[a];
                    out[c][lin(s, i, j, k)] = acc;
                }
    }
}

/* calculate_nabla_scalar_adjoint: r_c = (d_c s) * adj_s at face nodes, cubic.
 * Reference: 3D/flowmap.py:382-403, 2D/vortex/flowmap.py:379-395 */
void fmo_nabla_scalar_adjoint(const fmo_grid *g, real dx, const real *sc, const real *adj,
                              real *rx, real *ry, real *rz) {
    real *out[3] = {rx, ry, rz};
    int d = g->dim;
    int cs[3]; cell_shape(g, cs);
    real BL[3] = {0.5, 0.5, 0.5};
    for (int c = 0; c < d; ++c) {
        int s[3]; face_shape(g, c, s);
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    real X[3], v, gr[3], av;
                    node_pos(d, c, i, j, k, dx, X);
                    interp_grad(d, 3, sc, cs, X, dx, BL, &v, gr);
                    interp_grad(d, 3, adj, cs, X, dx, BL, &av, NULL);
                    out[c][lin(s, i, j, k)] = gr[c] * av;
                }
    }
}

/* reset_to_identity.  Reference: 3D/flowmap.py:336-356 */
void fmo_reset_to_identity(const fmo_grid *g, real dx, real *psi,
                           real *px, real *py, real *pz, real *Tx, real *Ty, real *Tz) {
    int d = g->dim;
    real *P[3] = {px, py, pz}, *T[3] = {Tx, Ty, Tz};
    for (int c = -1; c < d; ++c) {
        int s[3];
        if (c >= 0) face_shape(g, c, s); else cell_shape(g, s);
        long N = gsize(s);
        real *dst = c >= 0 ? P[c] : psi;
        if (!dst) continue;
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    real X[3];
                    node_pos(d, c, i, j, k, dx, X);
                    long q = lin(s, i, j, k);
                    for (int a = 0; a < d; ++a) {
                        dst[a * N + q] = X[a];
                        if (c >= 0 && T[c]) T[c][a * N + q] = (a == c) ? 1 : 0;
                    }
                }
    }
}

/* ------------------------------------------------------------------------ */
/* Pressure projection.                                                       */
/* apply_bc / divergence / subtract_grad_p: 3D/mgpcg.py:368-427,               */
/* 3D/fast_mgpcg.py:37-119,199-239; 2D/shape/mgpcg.py:301-344.                  */
/* ------------------------------------------------------------------------ */
void fmo_apply_bc(const fmo_grid *g, real *ux, real *uy, real *uz) {
    real *u[3] = {ux, uy, uz};
    for (int c = 0; c < g->dim; ++c) {
        int s[3]; face_shape(g, c, s);
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    int I[3] = {i, j, k};
                    if (I[c] == 0 || I[c] == s[c] - 1) u[c][lin(s, i, j, k)] = 0;
                }
    }
}

void fmo_divergence(const fmo_grid *g, const real *ux, const real *uy, const real *uz, real *div) {
    int cs[3]; cell_shape(g, cs);
    const real *u[3] = {ux, uy, uz};
    int d = g->dim;
    for (int i = 0; i < cs[0]; ++i)
        for (int j = 0; j < cs[1]; ++j)
            for (int k = 0; k < cs[2]; ++k) {
                real acc = 0;
                for (int c = 0; c < d; ++c) {
                    int s[3]; face_shape(g, c, s);
                    int I[3] = {i, j, k};
                    real vl = u[c][lin(s, I[0], I[1], I[2])];
                    I[c] += 1;
                    real vr = u[c][lin(s, I[0], I[1], I[2])];
                    /* vr - vl + vt - vb + vc - va, evaluated left to right */
                    if (c == 0) acc = vr - vl;
                    else { acc = acc + vr; acc = acc - vl; }
                }
                div[lin(cs, i, j, k)] = acc;
            }
}

/* subtract_grad_p with the plain-solver wall rule (p outside = 0).  Walls are
 * zeroed by the following apply_bc, so the solid variant's rule
 * (2D/vortex/mgpcg_solid.py:419-445) gives identical results. */
void fmo_subtract_grad_p(const fmo_grid *g, const real *p, real *ux, real *uy, real *uz) {
    int cs[3]; cell_shape(g, cs);
    real *u[3] = {ux, uy, uz};
    for (int c = 0; c < g->dim; ++c) {
        int s[3]; face_shape(g, c, s);
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k) {
                    int I[3] = {i, j, k};
                    real pr = 0, pl = 0;
                    if (I[c] < cs[c]) pr = p[lin(cs, I[0], I[1], I[2])];
                    if (I[c] >= 1) { I[c] -= 1; pl = p[lin(cs, I[0], I[1], I[2])]; }
                    u[c][lin(s, i, j, k)] -= pr - pl;
                }
    }
}

/* ------------------------------------------------------------------------ */
/* MGPCG.  Reference: 3D/mgpcg.py:12-290 (plain), 2D/vortex/mgpcg_solid.py:14-367  */
/* (solid-aware; with an empty obstacle mask its operator equals the plain one). */
/* All-Neumann 5/7-point Laplacian: diag = number of in-domain neighbours.     */
/* ------------------------------------------------------------------------ */
typedef struct {
    int levels;          /* number of MG levels */
    int pre_post;        /* RBGS pre/post sweeps per level (reference: 2) */
    int bottom;          /* bottom smoothing count */
    int bottom_mode;     /* 0: bottom x (R,B)  [3D/mgpcg.py:197-199]
                            1: bottom/2 x (R,B) + bottom/2 x (B,R)  [mgpcg_solid.py:263-268] */
    int max_iters;
    double abs_tol;      /* converged when rTr < max(abs_tol, rel_tol * zTr0) */
    double rel_tol;
    double eps;          /* added to denominators (reference: 1e-12) */
} fmo_mg_params;

typedef struct { int n[3]; } lvl_t;

static real neighbor_sum(int dim, const real *x, const int *s, int i, int j, int k) {
    real ret = 0;
    int I[3] = {i, j, k};
    for (int a = 0; a < dim; ++a) {
        if (I[a] < s[a] - 1) { int J[3] = {i, j, k}; J[a] += 1; ret += x[lin(s, J[0], J[1], J[2])]; }
        if (I[a] > 0) { int J[3] = {i, j, k}; J[a] -= 1; ret += x[lin(s, J[0], J[1], J[2])]; }
    }
    return ret;
}
static real num_nb(int dim, const int *s, int i, int j, int k) {
    real num = (real)(2 * dim);
    int I[3] = {i, j, k};
    for (int a = 0; a < dim; ++a) {
        if (I[a] <= 0) num -= 1;
        if (I[a] >= s[a] - 1) num -= 1;
    }
    return num;
}

static void mg_smooth(int dim, const int *s, real *z, const real *r, int phase) {
    #pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < s[0]; ++i)
        for (int j = 0; j < s[1]; ++j)
            for (int k = 0; k < s[2]; ++k)
                if (((i + j + k) & 1) == phase) {
                    real m = num_nb(dim, s, i, j, k);
                    z[lin(s, i, j, k)] = (r[lin(s, i, j, k)] + neighbor_sum(dim, z, s, i, j, k)) / m;
                }
}

static void mg_restrict(int dim, const int *s, const int *sc, const real *z, const real *r, real *rc) {
    long Nc = gsize(sc);
    memset(rc, 0, sizeof(real) * Nc);
    real scale = (real)1.0 / (real)(dim - 1.0);
    for (int i = 0; i < s[0]; ++i)
        for (int j = 0; j < s[1]; ++j)
            for (int k = 0; k < s[2]; ++k) {
                real m = num_nb(dim, s, i, j, k);
                real res = r[lin(s, i, j, k)] - (m * z[lin(s, i, j, k)] - neighbor_sum(dim, z, s, i, j, k));
                int kc = dim == 3 ? k / 2 : 0;
                rc[lin(sc, i / 2, j / 2, kc)] += res * scale;
            }
}

static void mg_prolongate(int dim, const int *s, const int *sc, real *z, const real *zc) {
    for (int i = 0; i < s[0]; ++i)
        for (int j = 0; j < s[1]; ++j)
            for (int k = 0; k < s[2]; ++k) {
                int kc = dim == 3 ? k / 2 : 0;
                z[lin(s, i, j, k)] += zc[lin(sc, i / 2, j / 2, kc)];
            }
}

static double dotp(const real *a, const real *b, long n) {
    double acc = 0;
    for (long i = 0; i < n; ++i) acc += (double)a[i] * (double)b[i];
    return acc;
}

static void recenter(real *r, long n) {
    double m = 0;
    for (long i = 0; i < n; ++i) m += (double)(r[i] / (real)n);
    real rm = (real)m;
    for (long i = 0; i < n; ++i) r[i] -= rm;
}

static void v_cycle(int dim, const fmo_mg_params *P, lvl_t *L, real **r, real **z) {
    long N0 = gsize(L[0].n);
    memset(z[0], 0, sizeof(real) * N0);
    int nl = P->levels;
    for (int l = 0; l < nl - 1; ++l) {
        for (int i = 0; i < P->pre_post; ++i) {
            mg_smooth(dim, L[l].n, z[l], r[l], 0);
            mg_smooth(dim, L[l].n, z[l], r[l], 1);
        }
        memset(z[l + 1], 0, sizeof(real) * gsize(L[l + 1].n));
        mg_restrict(dim, L[l].n, L[l + 1].n, z[l], r[l], r[l + 1]);
    }
    int b = nl - 1;
    if (P->bottom_mode == 0) {
        for (int i = 0; i < P->bottom; ++i) {
            mg_smooth(dim, L[b].n, z[b], r[b], 0);
            mg_smooth(dim, L[b].n, z[b], r[b], 1);
        }
    } else {
        for (int i = 0; i < P->bottom / 2; ++i) {
            mg_smooth(dim, L[b].n, z[b], r[b], 0);
            mg_smooth(dim, L[b].n, z[b], r[b], 1);
        }
        for (int i = 0; i < P->bottom / 2; ++i) {
            mg_smooth(dim, L[b].n, z[b], r[b], 1);
            mg_smooth(dim, L[b].n, z[b], r[b], 0);
        }
    }
    for (int l = nl - 2; l >= 0; --l) {
        mg_prolongate(dim, L[l].n, L[l + 1].n, z[l], z[l + 1]);
        for (int i = 0; i < P->pre_post; ++i) {
            mg_smooth(dim, L[l].n, z[l], r[l], 1);
            mg_smooth(dim, L[l].n, z[l], r[l], 0);
        }
    }
}

/* Solve A x = b (A = Neumann Laplacian, b = rhs) with MG-preconditioned CG.
 * Reference: 3D/mgpcg.py:207-289 and 2D/vortex/mgpcg_solid.py:276-367.
 * x: output.  Returns the iteration count (reference `it`); *rtr_out gets the
 * last rTr, *conv whether the tolerance was met. */
int fmo_mgpcg_solve(const fmo_grid *g, const fmo_mg_params *P, const real *b, real *x,
                    double *rtr_out, int *conv) {
    int dim = g->dim, nl = P->levels;
    lvl_t L[16];
    real *r[16], *z[16];
    for (int l = 0; l < nl; ++l) {
        for (int a = 0; a < 3; ++a) L[l].n[a] = (a < dim) ? (g->n[a] >> l) : 1;
        long n = gsize(L[l].n);
        r[l] = (real *)calloc(n, sizeof(real));
        z[l] = (real *)calloc(n, sizeof(real));
    }
    long N = gsize(L[0].n);
    real *p = (real *)calloc(N, sizeof(real)), *Ap = (real *)calloc(N, sizeof(real));
    memcpy(r[0], b, sizeof(real) * N);
    memset(x, 0, sizeof(real) * N);
    recenter(r[0], N);
    v_cycle(dim, P, L, r, z);
    /* update_p with beta = 0 (field initialised to 0) */
    for (long i = 0; i < N; ++i) p[i] = z[0][i];
    real old_zTr = (real)dotp(z[0], r[0], N);
    double tol = P->abs_tol;
    if (P->rel_tol > 0 && (double)old_zTr * P->rel_tol > tol) tol = (double)old_zTr * P->rel_tol;
    int it = 0;
    real rTr = 0;
    int converged = 0;
    while (P->max_iters < 0 || it < P->max_iters) {
        const int *s = L[0].n;
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < s[0]; ++i)
            for (int j = 0; j < s[1]; ++j)
                for (int k = 0; k < s[2]; ++k)
                    Ap[lin(s, i, j, k)] = num_nb(dim, s, i, j, k) * p[lin(s, i, j, k)] - neighbor_sum(dim, p, s, i, j, k);
        real pAp = (real)dotp(p, Ap, N);
        /* the reference divides host-side in double and stores to an f32 field */
        real alpha = (real)((double)old_zTr / ((double)pAp + P->eps));
        for (long i = 0; i < N; ++i) x[i] += alpha * p[i];
        for (long i = 0; i < N; ++i) r[0][i] -= alpha * Ap[i];
        rTr = (real)dotp(r[0], r[0], N);
        if ((double)rTr < tol) { converged = 1; break; }
        recenter(r[0], N);
        v_cycle(dim, P, L, r, z);
        real new_zTr = (real)dotp(z[0], r[0], N);
        real beta = (real)((double)new_zTr / ((double)old_zTr + P->eps));
        for (long i = 0; i < N; ++i) p[i] = z[0][i] + beta * p[i];
        old_zTr = new_zTr;
        it++;
    }
    for (int l = 0; l < nl; ++l) { free(r[l]); free(z[l]); }
    free(p); free(Ap);
    if (rtr_out) *rtr_out = (double)rTr;
    if (conv) *conv = converged;
    return it;
}

/* One V-cycle application z = M^-1 r (for preconditioner tests). */
void fmo_mg_vcycle(const fmo_grid *g, const fmo_mg_params *P, const real *rin, real *zout) {
    int dim = g->dim, nl = P->levels;
    lvl_t L[16];
    real *r[16], *z[16];
    for (int l = 0; l < nl; ++l) {
        for (int a = 0; a < 3; ++a) L[l].n[a] = (a < dim) ? (g->n[a] >> l) : 1;
        long n = gsize(L[l].n);
        r[l] = (real *)calloc(n, sizeof(real));
        z[l] = (real *)calloc(n, sizeof(real));
    }
    long N = gsize(L[0].n);
    memcpy(r[0], rin, sizeof(real) * N);
    v_cycle(dim, P, L, r, z);
    memcpy(zout, z[0], sizeof(real) * N);
    for (int l = 0; l < nl; ++l) { free(r[l]); free(z[l]); }
}

/* Apply the Laplacian (for tests). */
void fmo_laplacian(const fmo_grid *g, const real *p, real *Ap) {
    int s[3]; cell_shape(g, s);
    for (int i = 0; i < s[0]; ++i)
        for (int j = 0; j < s[1]; ++j)
            for (int k = 0; k < s[2]; ++k)
                Ap[lin(s, i, j, k)] = num_nb(g->dim, s, i, j, k) * p[lin(s, i, j, k)] - neighbor_sum(g->dim, p, s, i, j, k);
}

/* Poisson(u): apply_bc, divergence, solve A p = -div, subtract grad p, apply_bc.
 * Reference: 3D/mgpcg.py:429-439, 2D/vortex/mgpcg_solid.py:447-458.
 * p_out (cell grid) receives the pressure when non-NULL. */
int fmo_project(const fmo_grid *g, const fmo_mg_params *P, real *ux, real *uy, real *uz,
                real *p_out, double *rtr_out, int *conv) {
    int cs[3]; cell_shape(g, cs);
    long N = gsize(cs);
    real *div = (real *)calloc(N, sizeof(real));
    real *p = (real *)calloc(N, sizeof(real));
    fmo_apply_bc(g, ux, uy, uz);
    fmo_divergence(g, ux, uy, uz, div);
    for (long i = 0; i < N; ++i) div[i] = div[i] * (real)-1;
    int it = fmo_mgpcg_solve(g, P, div, p, rtr_out, conv);
    fmo_subtract_grad_p(g, p, ux, uy, uz);
    fmo_apply_bc(g, ux, uy, uz);
    if (p_out) memcpy(p_out, p, sizeof(real) * N);
    free(div); free(p);
    return it;
}

/* elementwise helpers: dest = f1 + m * f2 (add_fields, 3D/taichi_utils.py:86-89) */
void fmo_add_fields(const real *f1, const real *f2, real *dest, real m, long n) {
    for (long i = 0; i < n; ++i) dest[i] = f1[i] + m * f2[i];
}
