/*
 * flowmap_sm100.h -- C ABI of libflowmap_sm100.so, the B200 (sm_100a) kernels
 * for the leapfrog flow-map fluid step, its adjoint and the MGPCG pressure
 * projection of pearseven/differentiable-flowmap.
 *
 * Every entry point takes raw device pointers, an explicit grid descriptor, a
 * dtype selector (FM_F32: the reference's ti.f32 arithmetic; FM_F64: the FP64
 * run used to state errors) and a cudaStream_t passed as `void *`.  Work is
 * stream-ordered; nothing synchronises the host except fm_project /
 * fm_mgpcg_solve in host-checked mode (see fm_mg_params.check_every).
 * No entry point allocates memory except fm_mgpcg_create.
 *
 * Layout: scalar fields are C-order [i][j][k], k fastest.  2D grids use
 * dim = 2 and n[2] = 1.  MAC face grid c has extent n[c]+1 on axis c.
 * Vector fields on a grid (psi, T, phi, F) are SoA: dim consecutive planes of
 * that grid's size.  For 2D calls the *_z pointers must be NULL.
 *
 * Return value: FM_OK or one of the FM_ERR_* codes below.
 */
#ifndef FLOWMAP_SM100_H
#define FLOWMAP_SM100_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int dim;   /* 2 or 3 */
    int n[3];  /* cell counts; n[2] == 1 when dim == 2 */
} fm_grid;

enum { FM_F32 = 0, FM_F64 = 1, FM_BF16 = 2 /* storage only: fm_convert */ };

enum {
    FM_OK = 0,
    FM_ERR_SHAPE = 1,          /* bad grid / unsupported size */
    FM_ERR_ARG = 2,            /* NULL pointer, bad rk/order/flag */
    FM_ERR_NOT_CONVERGED = 3,  /* MGPCG hit max_iters without meeting the tolerance */
    FM_ERR_NONFINITE = 4,      /* NaN/Inf residual in MGPCG */
    FM_ERR_TIMEOUT = 5,        /* a bounded device wait gave up */
    FM_ERR_CUDA = 6,           /* CUDA runtime error (launch/alloc) */
    FM_ERR_DTYPE = 7,          /* dtype not FM_F32/FM_F64 */
    FM_ERR_CAPACITY = 8        /* grid too large for fm_project_noalloc's static scratch */
};

int fm_abi_version(void);
const char *fm_status_string(int status);

/* Number of kernels this library has launched on any stream since load (or
 * the last reset); a CUDA-graph launch adds the kernels it contains.  Used by
 * the benchmark to report its launch count.  reset != 0 returns the count and
 * zeroes it. */
long long fm_launch_count(int reset);

/* The CUDA runtime error code (cudaError_t) behind the most recent
 * FM_ERR_CUDA returned by any entry point (0 if none), with its name written
 * to buf (at most len bytes, NUL-terminated) when buf is not NULL. */
int fm_last_cuda_error(char *buf, int len);

/* Programmatic dependent launch for the pressure solver's kernels (on by
 * default): each kernel's CTAs may be scheduled while its stream predecessor
 * finishes, and wait for it before their first memory access, hiding launch
 * latency in the solver's chain of small kernels.  Results do not depend on
 * it.  enable = 0 switches it off for later launches; returns the previous
 * setting. */
int fm_set_pdl(int enable);

/* FP32 FMA throughput probe (no reference counterpart; measures the FP32 peak
 * the gather kernels are reported against): `blocks` CTAs of 256 threads each
 * run 16 independent FMA chains of `iters` steps -- scalar fmaf, or paired
 * two-lane FMAs when paired != 0 -- and write one float per thread to `out`
 * (blocks * 256 floats).  FLOPs per launch = blocks * 256 * iters * 32. */
int fm_fp32_fma_probe(int paired, int blocks, int iters, float *out, void *stream);

/* advect_u_grid: semi-Lagrangian advection, RK2 (midpoint) or RK4 backtrace
 * of the face nodes through u0, then u2_c = (u1 sampled at the foot)_c.
 * Replaces RK2_advect_u_grid / RK4_advect_u_grid (3D/flowmap.py:202-282,
 * dispatch 3D/flowmap.py:27-37; 2D/vortex/flowmap.py:233-291).
 * u2 must not alias u0 or u1. */
int fm_advect_u_grid(const fm_grid *g, int dtype, int rk, double dx, double dt,
                     const void *u0x, const void *u0y, const void *u0z,
                     const void *u1x, const void *u1y, const void *u1z,
                     void *u2x, void *u2y, void *u2z, void *stream);

/* Two advect_u_grid calls that share u0, rk and dt, in one pass: the foot of
 * each face node's backtrace is computed once and both u1 (-> u2) and v1
 * (-> v2) are sampled there.  The adjoint advects adj_u and u backwards along
 * the same midpoint velocity (3D/lfm_midpoint_diff_simulator.py:488-499);
 * results equal two fm_advect_u_grid calls. */
int fm_advect_u_grid_pair(const fm_grid *g, int dtype, int rk, double dx, double dt,
                          const void *u0x, const void *u0y, const void *u0z,
                          const void *u1x, const void *u1y, const void *u1z,
                          void *u2x, void *u2y, void *u2z,
                          const void *v1x, const void *v1y, const void *v1z,
                          void *v2x, void *v2y, void *v2z, void *stream);

/* advect_scalar_grid: the same backtrace from cell centres, quadratic sample
 * of s1.  Replaces RK2/RK4_advect_scalar_grid (3D/flowmap.py:284-320,
 * dispatch :39-49).  s2 must not alias s1. */
int fm_advect_scalar_grid(const fm_grid *g, int dtype, int rk, double dx, double dt,
                          const void *u0x, const void *u0y, const void *u0z,
                          const void *s1, void *s2, void *stream);

/* Two scalars along the same backtrace (passive and adj_passive in the
 * adjoint, 3D/lfm_midpoint_diff_simulator.py:494, :506).  t1/t2 may both be
 * NULL (then equal to fm_advect_scalar_grid). */
int fm_advect_scalar_grid_pair(const fm_grid *g, int dtype, int rk, double dx, double dt,
                               const void *u0x, const void *u0y, const void *u0z,
                               const void *s1, void *s2, const void *t1, void *t2, void *stream);

/* RK_grid / RK_grid_only_psi: in-place march of a flow map (psi, dim planes)
 * and, when T != NULL, its Jacobian rows (T, dim planes) with neg_dt = -dt.
 * face = 0..dim-1 selects face grid c, face = -1 the cell-centre grid
 * (T must then be NULL).  Replaces RK2_grid/RK4_grid (3D/flowmap.py:85-137)
 * and RK*_grid_only_psi (3D/flowmap.py:139-179), dispatch :6-25. */
int fm_rk_grid(const fm_grid *g, int dtype, int rk, double dx, double dt, int face,
               void *psi, void *T, const void *ux, const void *uy, const void *uz, void *stream);

/* March the centre map and all face maps with their Jacobians in one launch:
 * march_phi_grid / march_psi_grid / march_no_neural
 * (3D/lfm_midpoint_simulator.py:357-381, 3D/lfm_midpoint_diff_simulator.py:384-388).
 * psi_c may be NULL (no centre map). */
int fm_march_map(const fm_grid *g, int dtype, int rk, double dx, double dt,
                 void *psi_c, void *psi_x, void *T_x, void *psi_y, void *T_y, void *psi_z, void *T_z,
                 const void *ux, const void *uy, const void *uz, void *stream);

/* advect_u (impulse pullback) with a fused epilogue:
 *   out_c = alpha * (T_c . u0(psi_c) + beta * base_c)
 * alpha=1, beta=0 is the reference's advect_u (3D/flowmap.py:51-69); the two
 * other BFECC passes (3D/flowmap.py:405-434) are alpha=0.5, beta=-1,
 * base=init and alpha=-1, beta=-1, base=u (in place).  base may be NULL when
 * beta == 0 and may alias out; out must not alias u0. */
int fm_pullback_u(const fm_grid *g, int dtype, double dx,
                  const void *u0x, const void *u0y, const void *u0z,
                  void *outx, void *outy, void *outz,
                  const void *Tx, const void *Ty, const void *Tz,
                  const void *psix, const void *psiy, const void *psiz,
                  double alpha, double beta,
                  const void *basex, const void *basey, const void *basez, void *stream);

/* advect_scalar with the same epilogue: out = alpha*(s0(psi) + beta*base).
 * Replaces advect_scalar (3D/flowmap.py:71-79) and the BFECC_scalar passes
 * (3D/flowmap.py:436-452). */
int fm_pullback_scalar(const fm_grid *g, int dtype, double dx, const void *s0, void *out,
                       const void *psi, double alpha, double beta, const void *base, void *stream);

/* accumulate_init (ab3 = 0) / accumulate_init_new (ab3 = 1): pull a face
 * force back to the reinit frame, init_c += F_c . f(phi_c) * dt, with the
 * reference's Adams-Bashforth-3 history (including its ind == 1 formula).
 * Replaces 3D/flowmap.py:485-545 / 2D/vortex/flowmap.py:508-553.
 * Hp/Hpp (3 pointers each) are read and updated when ab3 = 1. */
int fm_accumulate_init(const fm_grid *g, int dtype, double dx, double dt, int ab3, int ind,
                       const void *fx, const void *fy, const void *fz,
                       void *initx, void *inity, void *initz,
                       const void *Fx, const void *Fy, const void *Fz,
                       const void *phix, const void *phiy, const void *phiz,
                       void *Hpx, void *Hppx, void *Hpy, void *Hppy, void *Hpz, void *Hppz,
                       void *stream);

/* fm_accumulate_init followed by a plain accumulate_init of a second face
 * field f2 with coefficient dt2 through the same phi and F, in one pass (the
 * adjoint step's two accumulations, 3D/lfm_midpoint_diff_simulator.py:513-523):
 * the same result as the two calls, with the positions, rows and stencils
 * loaded once.  f2 is required. */
int fm_accumulate_init_pair(const fm_grid *g, int dtype, double dx, double dt, int ab3, int ind,
                            const void *fx, const void *fy, const void *fz,
                            void *initx, void *inity, void *initz,
                            const void *Fx, const void *Fy, const void *Fz,
                            const void *phix, const void *phiy, const void *phiz,
                            void *Hpx, void *Hppx, void *Hpy, void *Hppy, void *Hpz, void *Hppz,
                            const void *f2x, const void *f2y, const void *f2z, double dt2, void *stream);

/* calculate_nabla_u_w: r_c = ((grad u)^T w)_c at face nodes, B-spline of
 * `order` (3 = cubic, as 3D/flowmap.py:359-380; 4 = quartic, as
 * 2D/vortex/flowmap.py:361-377). */
int fm_nabla_u_w(const fm_grid *g, int dtype, int order, double dx,
                 const void *ux, const void *uy, const void *uz,
                 const void *wx, const void *wy, const void *wz,
                 void *rx, void *ry, void *rz, void *stream);

/* calculate_nabla_scalar_adjoint: r_c = (d_c s) * adj_s at face nodes, cubic.
 * Replaces 3D/flowmap.py:382-403. */
int fm_nabla_scalar_adjoint(const fm_grid *g, int dtype, double dx, const void *s, const void *adj,
                            void *rx, void *ry, void *rz, void *stream);

/* reset_to_identity (3D/flowmap.py:336-356).  Any pointer may be NULL. */
int fm_reset_to_identity(const fm_grid *g, int dtype, double dx, void *psi_c,
                         void *psi_x, void *psi_y, void *psi_z, void *T_x, void *T_y, void *T_z,
                         void *stream);

/* add_fields: dest = f1 + m * f2 over n elements (3D/taichi_utils.py:86-89).
 * dest may alias f1 or f2. */
int fm_add_fields(int dtype, long n, const void *f1, const void *f2, void *dest, double m, void *stream);

/* Elementwise conversion between FM_F32 / FM_F64 / FM_BF16 (round to nearest
 * even) for the trajectory stores that replace RW_Cache
 * (3D/lfm_midpoint_simulator.py:46-165): the mixed-precision form stores each
 * step's midpoint velocity and passive scalar in BF16.  src and dst must not
 * overlap. */
int fm_convert(long n, int src_dtype, const void *src, int dst_dtype, void *dst, void *stream);

/* ------------------------------------------------------------------------
 * Discrete adjoints of the gather kernels (the backward passes of the
 * per-kernel torch.autograd Functions).  Each is the exact transpose of its
 * forward kernel's linearisation at the given inputs: the sampled field
 * enters linearly (its gradient is a scatter of the B-spline weights), the
 * sample position through the B-spline derivative weights (zero on an axis
 * where the forward's position clamp is active), and an RK backtrace stage by
 * stage in reverse.  Gradients are ADDED to the g_* buffers, which the caller
 * zeroes; field gradients use atomic adds (their last bits depend on the
 * order of the adds).  A g_* MAC argument is either complete or all NULL (not
 * wanted).  The reference has no counterpart: its adjoint is the continuous
 * one of 3D/lfm_midpoint_diff_simulator.py:390-594 (fm_nabla_* above).
 * ------------------------------------------------------------------------ */
/* Transpose of fm_advect_scalar_grid: g_s2 = dL/ds2 (cell grid) ->
 * g_u0 += dL/du0, g_s1 += dL/ds1 (either may be NULL). */
int fm_advect_scalar_grid_adj(const fm_grid *g, int dtype, int rk, double dx, double dt,
                              const void *u0x, const void *u0y, const void *u0z, const void *s1,
                              const void *g_s2, void *g_u0x, void *g_u0y, void *g_u0z, void *g_s1,
                              void *stream);
/* Transpose of fm_advect_u_grid: g_u2 = dL/du2 -> g_u0 += dL/du0 (through
 * the backtrace), g_u1 += dL/du1 (the sampled field).  For self-advection
 * (u1 == u0) the caller adds the two. */
int fm_advect_u_grid_adj(const fm_grid *g, int dtype, int rk, double dx, double dt,
                         const void *u0x, const void *u0y, const void *u0z,
                         const void *u1x, const void *u1y, const void *u1z,
                         const void *g_u2x, const void *g_u2y, const void *g_u2z,
                         void *g_u0x, void *g_u0y, void *g_u0z, void *g_u1x, void *g_u1y, void *g_u1z,
                         void *stream);
/* Transpose of fm_pullback_u (out_c = alpha (T_c . u0(psi_c) + beta base_c)):
 * g_out -> g_u0, g_T (D planes per face grid), g_psi (D planes), g_base. */
int fm_pullback_u_adj(const fm_grid *g, int dtype, double dx,
                      const void *u0x, const void *u0y, const void *u0z,
                      const void *Tx, const void *Ty, const void *Tz,
                      const void *psix, const void *psiy, const void *psiz,
                      double alpha, double beta,
                      const void *g_outx, const void *g_outy, const void *g_outz,
                      void *g_u0x, void *g_u0y, void *g_u0z, void *g_Tx, void *g_Ty, void *g_Tz,
                      void *g_psix, void *g_psiy, void *g_psiz, void *g_basex, void *g_basey, void *g_basez,
                      void *stream);
/* Transpose of fm_pullback_scalar (out = alpha (s0(psi) + beta base)):
 * g_out -> g_s0, g_psi (D planes), g_base (each may be NULL). */
int fm_pullback_scalar_adj(const fm_grid *g, int dtype, double dx, const void *s0, const void *psi, double alpha,
                           double beta, const void *g_out, void *g_s0, void *g_psi, void *g_base, void *stream);
/* Transpose of fm_rk_grid (one flow map psi, with its Jacobian row T when T is
 * not NULL, marched through u): psi, T are the march's INPUTS; g_psi_out,
 * g_T_out = dL/d(psi', T') of its outputs -> g_psi, g_T += dL/d(psi, T),
 * g_u += dL/du.  The Jacobian update d = (grad u)(pos) . t is differentiated
 * through the B-spline's second derivative.  g_T_out is required with T;
 * g_psi, g_T, g_u may be NULL. */
int fm_rk_grid_adj(const fm_grid *g, int dtype, int rk, double dx, double dt, int face,
                   const void *psi, const void *T, const void *ux, const void *uy, const void *uz,
                   const void *g_psi_out, const void *g_T_out, void *g_psi, void *g_T,
                   void *g_ux, void *g_uy, void *g_uz, void *stream);

/* ------------------------------------------------------------------------
 * MGPCG pressure projection.  Replaces MGPCG_3 / MGPCG_2 / MGPCG_2_solid
 * (3D/mgpcg.py:12-439, 2D/shape/mgpcg.py, 2D/vortex/mgpcg_solid.py) and the
 * 3D fast_mgpcg wrapper (3D/fast_mgpcg.py:241-323), empty obstacle mask.
 * ------------------------------------------------------------------------ */
typedef struct {
    int levels;        /* MG levels (reference: log2(min n) - base_level + 1) */
    int pre_post;      /* RBGS sweeps per level down and up (reference: 2) */
    int bottom;        /* bottom smoothing count */
    int bottom_mode;   /* 0: bottom x (R,B) [3D/mgpcg.py:197-199];
                          1: bottom/2 x (R,B) + bottom/2 x (B,R) [mgpcg_solid.py:263-268] */
    int max_iters;     /* reference: 400 */
    double abs_tol;    /* converged when rTr < max(abs_tol, rel_tol * zTr0) */
    double rel_tol;
    double eps;        /* added to alpha/beta denominators (reference: 1e-12) */
    int check_every;   /* 0: device mode -- the PCG loop is a CUDA-graph conditional
                          WHILE node, the solve never synchronises the host, and
                          its outcome is read with fm_mgpcg_stats;
                          k >= 1: host-checked mode, the host polls convergence
                          every k iterations */
    int coarse_bf16;   /* 1: store levels >= 1 in BF16 (FM_F32 only) */
} fm_mg_params;

typedef struct fm_mgpcg fm_mgpcg;

/* Allocates the MG hierarchy for one grid shape.  The only allocating call. */
int fm_mgpcg_create(const fm_grid *g, int dtype, const fm_mg_params *params, fm_mgpcg **out);
int fm_mgpcg_destroy(fm_mgpcg *solver);

/* Poisson(u): apply_bc, divergence, solve A p = -div, u -= grad p, apply_bc,
 * in place on the MAC velocity (3D/mgpcg.py:434-439).  Used for both
 * Poisson and Poisson_adj (3D/fast_mgpcg.py:241-323, which differ only in
 * name).  iters (reference `it`) and rtr (last r.r) may be NULL.
 * p_out (cell grid) receives the pressure when not NULL.
 * Returns FM_ERR_NOT_CONVERGED when max_iters was reached (the reference
 * continues silently; the host decides). */
int fm_project(fm_mgpcg *solver, void *ux, void *uy, void *uz, void *p_out, void *stream,
               int *iters, double *rtr);

/* Solve A x = b (b cell grid, recentred internally as the reference does).
 * In device mode (check_every = 0) fm_project and fm_mgpcg_solve return as
 * soon as the work is enqueued when iters and rtr are both NULL; passing
 * either synchronises the stream and reports the outcome. */
int fm_mgpcg_solve(fm_mgpcg *solver, const void *b, void *x, void *stream, int *iters, double *rtr);

/* One application of the MG preconditioner, z = M^-1 r (apply_preconditioner,
 * 3D/mgpcg.py:187-205): z = 0, per level pre_post x (red, black) sweeps and a
 * restriction, bottom smoothing, then per level prolongation and pre_post x
 * (black, red) sweeps.  r is not recentred.  r and z are cell-grid arrays of
 * the solver's dtype; the solver's level-0 buffers are overwritten. */
int fm_mg_vcycle(fm_mgpcg *solver, const void *r, void *z, void *stream);

/* Mixed-precision solve of A x = b to a relative FP64 residual: FP32 MGPCG
 * inner solves on `solver` (an FM_F32 handle; its tolerances set the inner
 * accuracy) inside an FP64 outer defect correction.  The solver itself and its
 * RBGS V-cycle are those of 3D/mgpcg.py:12-289; the outer loop has no
 * reference counterpart (the reference solves in FP32 only).
 *   b (b_dtype FM_F32 or FM_F64, cell grid) is recentred to mean zero in FP64;
 *   x (FP64, cell grid) receives the solution, starting from 0;
 *   work (FP64, cell grid) is caller-provided scratch.
 * Loop: r = (b - mean b) - A x in FP64; stop when |r| <= rel_tol |b - mean b|;
 * else solve A e = r/|r| in FP32 and x += |r| e.  At most max_outer
 * corrections (FM_ERR_NOT_CONVERGED beyond).  outer_iters, inner_iters (total
 * PCG iterations) and rel_res (final |r|/|b - mean b|) may be NULL.
 * Synchronises `stream` once per correction. */
int fm_mgpcg_solve_dc(fm_mgpcg *solver, int b_dtype, const void *b, double *x, double *work, double rel_tol,
                      int max_outer, void *stream, int *outer_iters, int *inner_iters, double *rel_res);

/* Poisson(u) (3D/mgpcg.py:207-289 with apply_bc, divergence and
 * subtract_grad_p, :368-427) with an FP64 outer defect correction around the
 * FP32 MGPCG of `solver` (an FM_F32 handle in device mode, check_every == 0).
 * The correction loop has no reference counterpart (the reference solves in
 * FP32 only): b = -div u and every residual b - mean(b) - A x are formed in
 * FP64; each correction solves A e = r/|r| with the FP32 MGPCG (its own
 * tolerances, floored at what the outer target needs) and adds |r| e to x in
 * FP64; the loop stops when |r| <= rel_tol |b - mean b| or after max_outer
 * (1..16) corrections (counted as a not-converged solve in fm_mgpcg_stats);
 * then u -= grad x in FP64, rounded to FP32.  Every stop decision is taken on
 * the device: no host synchronisation, and on a capturing stream the whole
 * projection is recorded (each inner solve a conditional while node).
 * work: 3 x cells doubles of caller-owned scratch (b, x, r).  p_out (FP64 cell
 * grid, may be NULL) receives x. */
int fm_project_dc(fm_mgpcg *solver, void *ux, void *uy, void *uz, double *work, double rel_tol, int max_outer,
                  double *p_out, void *stream);

/* Cumulative solver outcome (synchronises `stream`).  reset != 0 zeroes the
 * counters afterwards.  The reference reports non-convergence only with a
 * print (3D/mgpcg.py:286-289); here it is counted. */
typedef struct {
    long long solves;         /* completed solves */
    long long iterations;     /* sum of PCG iterations */
    long long not_converged;  /* solves that hit max_iters */
    long long nonfinite;      /* solves stopped by a NaN/Inf residual */
    int last_iters;           /* iterations of the last solve */
    int max_iters_seen;       /* largest iteration count */
    double last_rtr;          /* last r.r */
} fm_mg_stats;
int fm_mgpcg_stats(fm_mgpcg *solver, void *stream, int reset, fm_mg_stats *out);

/* Allocation-free Poisson(u).  This entry point has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory: code
 * running inside another runtime's preallocated pool (Taichi claims its device
 * memory at ti.init), under a fixed memory budget, or where a cudaMalloc would
 * synchronise the device at a bad moment.  It does what fm_mgpcg_create +
 * fm_project + fm_mgpcg_destroy do, with every scratch buffer carved out of
 * one static 48 MiB array inside the library: FP32 grids up to about 2.4 M
 * cells (128^3, 1024^2), FP64 up to about 1.2 M.  Larger grids return
 * FM_ERR_CAPACITY.  It calls no cudaMalloc, cudaFree or allocating library
 * routine.  The array is one per GPU and shared by all calls: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) and should come before any stream capture.
 * Under CUDA's lazy module loading (the default) that first call is also when
 * the array and this library's kernels get their device memory: make it before
 * another runtime claims the device's memory (e.g. right after loading the
 * library, before ti.init), or run with CUDA_MODULE_LOADING=EAGER.  The
 * capacity check comes before the field-pointer check, so a call with NULL
 * fields tells whether a grid fits (FM_ERR_CAPACITY if not, FM_ERR_ARG if so).
 * Every call synchronises `stream` to poll convergence (params->check_every
 * iterations per poll; 0 means 4).  Result and status as fm_project. */
int fm_project_noalloc(const fm_grid *g, int dtype, const fm_mg_params *params, void *ux, void *uy, void *uz,
                       void *stream, int *iters, double *rtr);

/* Apply the Neumann Laplacian: Ap = A p (for tests and defect correction). */
int fm_laplacian(const fm_grid *g, int dtype, const void *p, void *Ap, void *stream);

/* BFECC clamp (clamp_u, 3D/flowmap.py:324-334; 2D/vortex/flowmap.py:333-341):
 * dst = clamp(src, min, max of ref over the 2*dim axis neighbours), neighbours
 * sampled with sample()'s index clamp, on grid `face` (0..dim-1 a face grid,
 * -1 the cell grid).  dst may not alias ref. */
int fm_clamp_extrema(const fm_grid *g, int dtype, int face, const void *src, const void *ref, void *dst, void *stream);

/* 2D viscous force (calculate_viscous_force, 2D/vortex/flowmap.py:4-17):
 * vis = nu (s(i+1,j) + s(i-1,j) + s(i,j+1) + s(i,j-1) - 4 s(i,j)) / dx / dx on
 * each face grid, samples index-clamped.  With adj_x/adj_y (both or neither)
 * it also adds sum adj . vis / nu over both grids to *dot (device FP64;
 * calculate_viscous_force_adj, 2D/vortex/flowmap.py:20-35), nothing when
 * nu == 0; part: device FP64 scratch of 592 entries. */
int fm_viscous_force_2d(const fm_grid *g, int dtype, double nu, double dx, const void *ux, const void *uy, void *vis_x,
                        void *vis_y, const void *adj_x, const void *adj_y, double *part, double *dot, void *stream);

/* ------------------------------------------------------------------------
 * Launch tuning (no reference counterpart: the reference's kernels are
 * scheduled by Taichi).  The gather kernels compute every node independently,
 * so their block size changes only the speed; the autotuner (tune.py) times
 * the candidates on one grid shape and stores the fastest here.
 * ------------------------------------------------------------------------ */
enum {
    FM_TUNE_ADVECT_U = 0,        /* fm_advect_u_grid(_pair) */
    FM_TUNE_ADVECT_SCALAR = 1,   /* fm_advect_scalar_grid(_pair) */
    FM_TUNE_MARCH = 2,           /* fm_march_map, fm_rk_grid */
    FM_TUNE_PULLBACK_U = 3,      /* fm_pullback_u */
    FM_TUNE_PULLBACK_SCALAR = 4, /* fm_pullback_scalar */
    FM_TUNE_ACCUMULATE = 5,      /* fm_accumulate_init */
    FM_TUNE_ADJ_SOURCE_TILE = 6, /* fm_nabla_u_w, fm_nabla_scalar_adjoint: output tile height along i */
    FM_TUNE_KINDS = 7
};
/* Kernel classes 0-5: threads per block on grid g, 32..256 in multiples of 32
 * (default 256).  FM_TUNE_ADJ_SOURCE_TILE: the adjoint-source stencil's tile
 * height along i, 4 or 8 output nodes in 3D (default 8), 8 or 16 in 2D
 * (default 16; with a dx that is not a power of two, 16 runs as 12).  0
 * restores the default.  Neither changes a result.  Thread-safe; applies to
 * later launches. */
int fm_tune_set(int kind, const fm_grid *g, int threads);
/* The value launches of `kind` on g use; -FM_ERR_ARG on a bad kind. */
int fm_tune_get(int kind, const fm_grid *g);

/* ------------------------------------------------------------------------
 * Obstacles: MGPCG with a boundary mask and the mask kernels.
 * mask: device float32 array on the cell grid; the solver treats cells with
 * mask > 0 as solid (mgpcg_solid.py), the mask kernels cells with mask >= 1
 * (init_conditions.py), as the reference does.
 * ------------------------------------------------------------------------ */
typedef struct fm_solid fm_solid;

/* Allocates a solid-aware MG hierarchy (2D/vortex/mgpcg_solid.py:24-79,
 * MGPCG_2_solid :370-382; dimension-generic) and, when mask is not NULL,
 * downsamples it (downsample_bm, :114-127: a coarse cell is solid only when
 * all its children are).  params as for fm_mgpcg_create: check_every >= 1 is
 * the host polling interval; 0 runs the PCG loop on the device (a graph
 * conditional WHILE node: no host synchronisation, and a solve on a capturing
 * stream is recorded into the caller's graph); coarse_bf16 must be 0.  The
 * only allocating call. */
int fm_solid_create(const fm_grid *g, int dtype, const fm_mg_params *params, const float *mask, fm_solid **out);
int fm_solid_destroy(fm_solid *solver);
/* Cumulative outcome of the solver's solves (as fm_mgpcg_stats; synchronises
 * `stream`).  With check_every == 0 and iters/rtr NULL, fm_solid_solve and
 * fm_solid_project return before the solve ends and report only here. */
int fm_solid_stats(fm_solid *solver, void *stream, int reset, fm_mg_stats *out);
/* Re-derives the level masks from a (new) mask; the reference downsamples
 * before every solve (:270-272). */
int fm_solid_set_mask(fm_solid *solver, const float *mask, void *stream);
/* apply_preconditioner (:249-268) on the fluid cells: z = V-cycle(r). */
int fm_solid_vcycle(fm_solid *solver, const void *r, void *z, void *stream);
/* solve (:270-367) of A x = b with recentring; *iters, *rtr as fm_mgpcg_solve. */
int fm_solid_solve(fm_solid *solver, const void *b, void *x, void *stream, int *iters, double *rtr);
/* MGPCG_2_solid.Poisson (:447-458): apply_bc (walls and the faces of solid
 * cells zeroed), divergence (0 in solid cells), solve with k = -1,
 * u -= grad p, apply_bc; p_out (cell grid) may be NULL. */
int fm_solid_project(fm_solid *solver, void *ux, void *uy, void *uz, void *p_out, void *stream, int *iters,
                     double *rtr);
/* mask_velocity_by_boundary (2D/vortex/init_conditions.py:549-556,
 * 3D/init_conditions.py:536-544): the faces of solid cells take the boundary
 * velocity bvel (dim planes on the cell grid, the dtype), or 0 when bvel is
 * NULL (mask_adj_velocity_by_boundary).  Where two solid cells share a face
 * the cell on its high side wins (the reference's parallel writes race). */
int fm_mask_velocity(const fm_grid *g, int dtype, const float *mask, const void *bvel, void *ux, void *uy, void *uz,
                     void *stream);
/* mask_passive_by_boundary (:558-571 / :547-561): a solid cell takes the mean
 * of its fluid 3^dim neighbours, or 0; adjoint != 0: the solid cells are
 * zeroed (mask_adj_passive_by_boundary). */
int fm_mask_passive(const fm_grid *g, int dtype, const float *mask, void *s, int adjoint, void *stream);

/* ------------------------------------------------------------------------
 * Gaussian control forces.  n Gaussians, device arrays of the dtype:
 * center n x dim (row-major), inv_radius n (r = 1/radius^2), strength n x dim.
 * ------------------------------------------------------------------------ */
/* f_c(X) = sum over I with q_I(X) = |X - c_I|^2 r_I < 5 of exp(-q_I(X)) strength_I[c]
 * on every face of component c, summed in ascending I (apply_gausion_force_kernel,
 * 3D/lfm_midpoint_simulator.py:309-344; 2D/shape/lfm_midpoint_simulator.py:283-299).
 * Every face is written (0 where no Gaussian reaches it).  0 <= n <= 2^24. */
int fm_gaussian_force(const fm_grid *g, int dtype, double dx, int n, const void *center, const void *inv_radius,
                      const void *strength, void *f_x, void *f_y, void *f_z, void *stream);
/* Per-Gaussian sums over the faces of its support (calculate_adj_gausion_force_kernel,
 * 3D/lfm_midpoint_diff_simulator.py:63-110; 2D/shape/lfm_midpoint_diff_simulator.py:75-103):
 * adj_strength[I][c] = sum e a_c, adj_center[I] = sum_c sum s_c e 2 (X - c_I) r a_c,
 * penalty_strength[I][c] = sum 2 f e, penalty_center[I] = sum_c sum 2 f s_c e 2 (X - c_I) r,
 * e = exp(-q), f = e s_c, a = adj_{x,y,z}.  Outputs: device FP64, n x dim each,
 * overwritten (the reference zero-fills them first); deterministic summation. */
int fm_gaussian_force_grad(const fm_grid *g, int dtype, double dx, int n, const void *center, const void *inv_radius,
                           const void *strength, const void *adj_x, const void *adj_y, const void *adj_z,
                           double *adj_center, double *adj_strength, double *penalty_center, double *penalty_strength,
                           void *stream);

/* ------------------------------------------------------------------------
 * 2D vortex problem (the vortex optimisation's control map and loss).
 * theta = [w_0..w_{K-1}, cx_0..cx_{K-1}, cy_0..cy_{K-1}], K <= 64, host array.
 * ------------------------------------------------------------------------ */
/* Face velocity of K Gaussian-core point vortices: at every cell centre X the
 * sum of angular_vel_func(|X-c_k|, 0.02, -0.01) w_k (-(X-c_k).y, (X-c_k).x)
 * (2D/vortex/init_conditions.py:142-145, 386-414), split to the faces with
 * clamped samples (split_central_vector, 2D/vortex/taichi_utils.py:158-167). */
int fm_vortex_velocity_2d(const fm_grid *g, int dtype, double dx, int nv, const double *theta, void *ux, void *uy,
                          void *stream);
/* grad[3K] (device, FP64) = sum over faces of lambda . d u / d theta, the
 * analytic form of the reference's finite-difference calculate_dtheta_ind
 * (2D/vortex/optimize_vortex.py:193-220).  work: device FP64 scratch of
 * 592 * 3K entries. */
int fm_vortex_velocity_grad_2d(const fm_grid *g, int dtype, double dx, int nv, const double *theta, const void *lam_x,
                               const void *lam_y, double *work, double *grad, void *stream);
/* omega (cell grid) = curl of the face-averaged centre velocity with clamped
 * samples (get_central_vector, curl: 2D/vortex/taichi_utils.py:153-156, 199-205). */
int fm_vorticity_2d(const fm_grid *g, int dtype, double dx, const void *ux, const void *uy, void *omega, void *stream);
/* Final-vorticity loss and adjoint seed: *loss (device FP64) = sum (omega - omega*)^2,
 * lam = (d omega / d u)^T 2 (omega - omega*) on the faces.  work: cell-grid
 * scratch of the dtype; part: device FP64 scratch of 592 entries.  The
 * vorticity loss has no reference counterpart (the reference's vortex loss is
 * on passive scalars, 2D/vortex/lfm_midpoint_diff_simulator.py:165-174). */
int fm_vorticity_loss_2d(const fm_grid *g, int dtype, double dx, const void *ux, const void *uy, const void *omega_target,
                         void *work, double *part, void *lam_x, void *lam_y, double *loss, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FLOWMAP_SM100_H */
