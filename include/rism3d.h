/*
  rism3d.h -- C ABI of the B200-native 3D-RISM solute solver.

  This is the drop-in boundary for the hot path of bgy3d's
  ``runbgy.scm energy --hnc``: the hnc3d.c fixed-point / Newton loop.
  Every entry point takes plain pointers and sizes; no PETSc, Guile or
  torch types cross it.  All entry points return 0 on success and a
  negative RISM3D_ERR_* code on failure (the reference longjmps through
  scm_misc_error instead, bgy3d-snes.c:338-345).

  Units are the reference's: Angstrom, kcal/mol, elementary charges,
  beta in mol/kcal (bgy3d.h:120-145, units.f90).

  Array layouts:
    real grid field    [m][N2][N1][N0], N0 (x) fastest -- the DMDA order of
                       bgy3d-fftw3.c:295-339; grid point (i0,i1,i2) sits at
                       r = i*h - L/2 (vec_rmap3, bgy3d-vec.h:578-607).
    solvent chi(k)     [m][m][nrad] on k_p = (p + 1/2) * pi / rmax -- the
                       buffer rism_solvent() fills (rism.f90:57-102) and
                       hnc3d_solute_solve() consumes (hnc3d.c:1442-1560).
*/
#ifndef RISM3D_H
#define RISM3D_H

#ifdef __cplusplus
extern "C" {
#endif

/* Closures, numbered as ClosureEnum (bgy3d.h:211-223). */
enum {
  RISM3D_HNC = 0, RISM3D_KH = 1, RISM3D_PY = 2,
  RISM3D_PSE0 = 3, RISM3D_PSE1, RISM3D_PSE2, RISM3D_PSE3,
  RISM3D_PSE4, RISM3D_PSE5, RISM3D_PSE6, RISM3D_PSE7
};

/* Non-linear solvers, as --snes-solver (bgy3d-snes.c:16-35). */
enum { RISM3D_NEWTON = 0, RISM3D_PICARD = 1, RISM3D_TRIAL = 2, RISM3D_JAGER = 3 };

/* Arithmetic of the solve. */
enum {
  RISM3D_FP64 = 0,   /* plain form: every F, J.v and Krylov vector in FP64 */
  RISM3D_MIXED = 1   /* FP32 bulk Newton, then FP64 residual + FP32 J.v
                        iterative refinement to the same tolerance */
};

/* Status codes. */
enum {
  RISM3D_OK = 0,
  RISM3D_ERR_ARG = -1,        /* bad argument (size, NULL, layout)        */
  RISM3D_ERR_CUDA = -2,       /* CUDA runtime error                       */
  RISM3D_ERR_NOMEM = -3,      /* device allocation failed                 */
  RISM3D_ERR_TABLE = -4,      /* |k| of the grid beyond the chi table     */
  RISM3D_ERR_NOT_CONVERGED = -5, /* max_iter reached (SNES reason <= 0)   */
  RISM3D_ERR_NAN = -6,        /* residual became NaN/Inf                  */
  RISM3D_ERR_UNSUPPORTED = -7 /* e.g. PY closure has no Jacobian          */
};

/* Mirrors ``Site`` (bgy3d-solutes.h:9-16) without the SCM handle. */
typedef struct rism3d_site {
  char name[8];
  double x[3];        /* Angstrom */
  double sigma;       /* LJ sigma, Angstrom */
  double epsilon;     /* LJ epsilon, kcal/mol */
  double charge;      /* e */
} rism3d_site;

/* Mirrors ``ProblemData`` (bgy3d.h:228-256) plus the flags the reference
   reads through bgy3d_getopt_* (hnc3d.c:1782-1784, 1613-1627;
   bgy3d-snes.c:20). */
typedef struct rism3d_problem {
  int N[3];           /* grid points; each 2^a 3^b, even, 8..512 */
  double L[3];        /* FULL box edges (the reference's PD->L = 2 * --L,
                         bgy3d-guile.c:284-288) */
  double beta;        /* inverse temperature, mol/kcal */
  double rho;         /* solvent site density, 1/A^3 */
  double rmax;        /* radial extent of chi (1D grid), A */
  int nrad;           /* radial points of chi */
  int closure;        /* RISM3D_HNC ... RISM3D_PSE7 */
  int max_iter;       /* Newton iterations (PD->max_iter) */
  double norm_tol;    /* stop when ||F(t)||_inf < norm_tol */
  double lambda;      /* Picard mixing (PD->lambda) */
  int solver;         /* RISM3D_NEWTON / _PICARD / _TRIAL / _JAGER (bgy3d-snes.c:19-31) */
  int renorm;         /* 1: default; 0: --no-renorm (hnc3d.c:1607-1615) */
  int precision;      /* RISM3D_FP64 or RISM3D_MIXED */
  int verbosity;      /* 0 silent; 1 one line per Newton step on stderr */
  /* Krylov solver of the Newton steps.  krylov_restart 30, ew_forcing 0 and
     coarse_h 0 are the reference's settings: GMRES(30) without
     preconditioner at a fixed KSP rtol of 1e-3 (bgy3d-snes.c:262-306).
     rism3d_problem_defaults() selects 30 / 1 / 0.75 / 16. */
  int krylov_restart; /* GMRES restart length (0: 30) */
  int ew_forcing;     /* 1: Eisenstat-Walker forcing terms, floored at 1e-3;
                         0: fixed rtol 1e-3 */
  double coarse_h;    /* two-grid preconditioner (then flexible GMRES):
                         coarse grid spacing in A -- per axis the smallest
                         even 2^a 3^b point count n with L / n <= coarse_h,
                         used when n <= N/2 on every axis; otherwise the
                         grid of max(coarse_h, 1 A) spacing if it is coarser
                         than N on every axis; off when 0 or neither fits */
  int coarse_steps;   /* GMRES steps of each coarse solve (0: 16; defaults: 16) */
} rism3d_problem;

/* What hnc3d_solute_solve conses onto its result alist
   (hnc3d.c:2230-2267) plus solver diagnostics. */
typedef struct rism3d_result {
  double mu;          /* free-energy: functional of the native closure */
  double mu_hnc, mu_kh, mu_gf; /* print_chempot, hnc3d.c:668-687 */
  double pmv_factor;  /* partial-molar-volume-factor, 1 - rho int c */
  double resid_inf;   /* ||F(t)||_inf at exit (vec_norm, bgy3d-vec.h:301) */
  double resid_2;     /* ||F(t)||_2 at exit (SNES norm) */
  int status;         /* RISM3D_OK or RISM3D_ERR_* */
  int newton_iters;
  int f_evals;        /* F evaluations (iterate_t1), all precisions */
  int jv_evals;       /* J.v products (jacobian_t1), all precisions */
  int f_evals_fp32, jv_evals_fp32;
  int jv_evals_coarse; /* J.v products on the coarse grid (preconditioner) */
  double seconds;     /* device time of the non-linear solve */
  long long launches; /* kernels this library launched for the solve (a
                         replayed CUDA graph counts its kernel nodes) */
} rism3d_result;

/* Defaults of bgy3d-guile.c:243-386 / guile/bgy3d.scm:323-340 for a cubic
   box: half edge ``L_half`` (the --L flag), N points per edge. */
void rism3d_problem_defaults(rism3d_problem *pd, double L_half, int N);

/*
  One complete solute solve.  Replaces hnc3d_solute_solve()
  (hnc3d.h:13-21, hnc3d.c:1762-2350) with the 1D-RISM chi supplied by the
  caller (the chi_fft_buf != NULL branch, hnc3d.c:1449-1469).

    chi      [m][m][nrad] solvent susceptibility chi = omega + rho h
             (NOT offset by one), host memory, borrowed.
    t_inout  host [m][N2][N1][N0] or NULL.  If non-NULL it is the initial
             guess on entry and the converged t on exit -- the Restart
             token of hnc3d.c:1830-1845, 2301-2316.
    g_out    host [m][N2][N1][N0] or NULL: g = h + 1 (hnc3d.c:2320, 2341).
    out      results; out->status repeats the return code.

  The device context of a finished call (grids, chi tables, the
  preconditioner's coarse problem, Krylov buffers) is kept for the next
  call on the same device with equal problem settings, solvent sites and
  chi contents, which then only rebinds the solute -- the PES loop of
  guile/bgy3d.scm:819-880 calling this repeatedly pays the set-up once.
  At most RISM3D_CTX_CACHE contexts (environment, read once; default 1,
  0 turns the cache off) stay allocated between calls; concurrent calls
  never share one.
*/
int rism3d_solute_solve(const rism3d_problem *pd,
                        int m, const rism3d_site *solvent,
                        int n, const rism3d_site *solute,
                        const double *chi,
                        double *t_inout, double *g_out,
                        rism3d_result *out);

/* Frees the contexts rism3d_solute_solve keeps between calls (no
   counterpart in the reference, which builds its context on every call). */
void rism3d_cache_clear(void);

/* Derivatives of the free energy mu (the closure's native functional) with
   respect to the solute's site parameters, and diagnostics of the adjoint
   solve that yields them.  Arrays are host, caller-owned; a NULL array is
   skipped.  Units: kcal/mol per e, per A (sigma, x), per kcal/mol (eps). */
typedef struct rism3d_grad {
  double *dq;         /* [n] dmu/dq_u */
  double *dsigma;     /* [n] dmu/dsigma_u */
  double *depsilon;   /* [n] dmu/depsilon_u */
  double *dx;         /* [n][3] dmu/dx_u: minus the solvation force on site u */
  int adjoint_jv;     /* J.v products of the adjoint solve */
  double adjoint_resid; /* ||J^T lambda - dmu/dt||_2 / ||dmu/dt||_2 */
  double seconds;     /* device time of the gradient */
  double *dx_reference; /* [n][3] or NULL: the reference's own
                         free-energy-gradient, rho h^3 sum_i <g_i, dv_i/dx_u>
                         (see rism3d_free_energy_gradient) */
} rism3d_grad;

/*
  Solve, then dmu/d(solute q, sigma, eps, x).  Replaces the `derivatives`
  branch of hnc3d_solute_solve (gradients / energy1 / field1,
  hnc3d.c:1665-1742, bgy3d-solutes.c:381-468), which takes
  dmu/dx = rho h^3 sum_i <g_i, dv_i/dx> (bgy3d-force.c forces), by the
  adjoint of the converged fixed point instead: J^T lambda = dmu/dt, then
  dmu/dp = d mu/dp|_t - lambda . dF/dp|_t, exact for any closure's
  functional and for the renormalised long-range term.  Arguments as
  rism3d_solute_solve (t_inout may be NULL).  Renormalised form only
  (RISM3D_ERR_UNSUPPORTED with renorm = 0).  With grad->dx_reference set it
  also receives the reference's own formula (rism3d_free_energy_gradient).
*/
int rism3d_solute_grad(const rism3d_problem *pd,
                       int m, const rism3d_site *solvent,
                       int n, const rism3d_site *solute,
                       const double *chi, double *t_inout,
                       rism3d_result *out, rism3d_grad *grad);

/* One solute of a batch: the arguments of rism3d_solute_solve for that
   solute (its own problem -- grid, box, closure, precision -- and chi
   table) and its result. */
typedef struct rism3d_job {
  rism3d_problem pd;
  int n;                      /* solute sites */
  const rism3d_site *solute;  /* host, borrowed */
  const double *chi;          /* [m][m][pd.nrad] host, borrowed (may be shared) */
  double *t_inout;            /* host [m][N2][N1][N0] or NULL, as above */
  double *g_out;              /* host [m][N2][N1][N0] or NULL */
  rism3d_result result;       /* out; result.status is the job's code */
} rism3d_job;

/*
  Many independent solute solves in one solvent, of uneven site counts and
  grid sizes (a set of solutes or the points of a PES scan: the loops over
  hnc3d_solute_solve calls in guile/bgy3d.scm:819-880, 943-975), solved
  concurrently on the current device: `workers` host threads (0: 8), each
  issuing on its own CUDA stream, take the jobs largest grid first; device
  memory comes from the stream-ordered pool, so no job's setup or teardown
  synchronises the device.  Returns RISM3D_OK when every job converged,
  otherwise the code of the first failing job in job order (every job still
  runs; see jobs[i].result.status).
*/
int rism3d_solve_batch(int m, const rism3d_site *solvent, int njobs, rism3d_job *jobs, int workers);

/* ---- device-resident context: the inner plug points ------------------ */

typedef struct rism3d_ctx rism3d_ctx;

/* Builds everything hnc3d_solute_solve sets up before SNES
   (hnc3d.c:1790-1966): the solute field v_short (bgy3d_solute_field /
   field0, bgy3d-solutes.c:343-377, 845-969), chi - 1 and the renormalised
   long-range kernel tau as radial tables (solvent_kernel_rism,
   hnc3d.c:1442-1560; rism_solvent_renorm, rism.f90:141-208) and the
   centred electric form factor (bgy3d_solute_form, bgy3d-solutes.c:633-698).
   The context owns its device memory; it is bound to the current device. */
int rism3d_ctx_create(const rism3d_problem *pd,
                      int m, const rism3d_site *solvent,
                      int n, const rism3d_site *solute,
                      const double *chi, rism3d_ctx **ctx);
void rism3d_ctx_destroy(rism3d_ctx *ctx);

/* Number of reals in one long vector T: m * N0 * N1 * N2. */
long long rism3d_ctx_size(const rism3d_ctx *ctx);

/* F(T) = (chi-1) * c(T) - beta/eps0 tau - T: the VecFunc1 iterate_t1
   (hnc3d.c:1183-1285).  T, dT: device pointers, FP64, [m][N2][N1][N0].
   resid (optional, host, 2 doubles) receives ||dT||_inf and ||dT||_2. */
int rism3d_iterate_t1(rism3d_ctx *ctx, const double *T, double *dT, double *resid);

/* J(T) dT = (chi-1) * (c'(T) dT) - dT: the VecFunc2 jacobian_t1
   (hnc3d.c:1289-1362).  Device pointers, FP64. */
int rism3d_jacobian_t1(rism3d_ctx *ctx, const double *T, const double *dT, double *JdT);

/* FP32 forms of the two above (device pointers to float). */
int rism3d_iterate_t1_f32(rism3d_ctx *ctx, const float *T, float *dT, double *resid);
int rism3d_jacobian_t1_f32(rism3d_ctx *ctx, const float *T, const float *dT, float *JdT);

/* Solve F(T) = 0 in place (T on the device, FP64): the bgy3d_snes_default
   call of hnc3d.c:1967 with the solver/precision of the problem. */
int rism3d_solve(rism3d_ctx *ctx, double *T, rism3d_result *out);

/* Post-processing of a converged T (hnc3d.c:2148-2269): mu by the native,
   HNC, KH and GF functionals, PMV factor; g = h + 1 into g (device, FP64,
   optional). */
int rism3d_observables(rism3d_ctx *ctx, const double *T, double *g, rism3d_result *out);

/* Copies an internal real field to a device buffer of [m][N] (which = 0:
   v_short, 1: long-range Coulomb uc (one field, [N])). */
int rism3d_get_field(rism3d_ctx *ctx, int which, double *dst);

/* Last CUDA error string of this thread (diagnostics). */
const char *rism3d_last_error(void);

/* The two-grid preconditioner of the Newton-Krylov solver at state T
   (diagnostics and tests; the reference's GMRES has no preconditioner, so
   this has no counterpart there): z = M^-1 v with
   M^-1 v = P (J_H^-1 + I) R v - v, where R / P are the band-limited
   transfers to / from the coarse grid, J_H the coarse Jacobian built from
   the restricted closure slope R c'(T), and J_H^-1 a coarse_steps-step
   FP32 GMRES from zero.  Device pointers, FP64 [m][N2][N1][N0].  Returns
   RISM3D_ERR_UNSUPPORTED when the context has no coarse grid. */
int rism3d_precondition(rism3d_ctx *ctx, const double *T, const double *v, double *z);

/* The same preconditioner in FP32, as the mixed-precision solve applies it
   (FP32 device pointers [m][N2][N1][N0]); its x-axis grid transfers run on
   the tensor cores where the (fine, coarse) pair has a kernel. */
int rism3d_precondition_f32(rism3d_ctx *ctx, const float *T, const float *v, float *z);

/* Rebinds the context to another solute of the same solvent and grid (a
   new geometry, charges or LJ parameters): recomputes the solute's
   short-range field and long-range term only, keeping every buffer, the
   chi tables and the preconditioner's coarse problem, so that consecutive
   solves of a PES scan or a geometry optimisation (the restart loop of
   guile/bgy3d.scm:819-880 with hnc3d.c:1830-1845) pay no setup and can
   start from the previous t.  n may differ from the creating call's. */
int rism3d_ctx_set_solute(rism3d_ctx *ctx, int n, const rism3d_site *solute);

/* The transposed Jacobian at T (the adjoint operator of the gradient):
   JT = J^T dT = c'(T) . ((chi - 1) * dT) - dT.  FP64 device pointers. */
int rism3d_jacobian_transpose_t1(rism3d_ctx *ctx, const double *T, const double *dT, double *JT);

/* dmu/d(solute parameters) at a converged T (FP64 device pointer); see
   rism3d_solute_grad. */
int rism3d_gradient(rism3d_ctx *ctx, const double *T, rism3d_grad *grad);

/* The `derivatives` output of hnc3d_solute_solve, consed as
   "free-energy-gradient" (gradients / energy1, hnc3d.c:1665-1742, 2270-2289):
   de[u][a] = rho h^3 sum_i sum_r g_i(r) dv_i(r)/dx_{u,a}, g = c(T) + T + 1
   and dv the derivative of the solute field for a unit displacement of site
   u (field1, bgy3d-solutes.c:381-468: LJ and the FULL capped Coulomb; 0 at
   a grid point on the site).  The formula takes mu as stationary in t and
   the Coulomb derivative in real space; rism3d_gradient differentiates the
   renormalised, periodic functional exactly, and the two differ by about
   1 % of the largest component (0.8-0.9 % on the test solutes).  T:
   converged FP64 device pointer; de: host [n][3].  Any solute context
   (renormalised or not, radial or 3D chi). */
int rism3d_free_energy_gradient(rism3d_ctx *ctx, const double *T, double *de);

/* Linear-response derivatives dmu/dx_u[n][3] at a converged T (FP64
   device pointer), as the `response` branch of hnc3d_solute_solve computes
   them ("free-energy-response", hnc3d.c:1969-2135 with response_t1,
   1366-1421): for each unit displacement of one site, dv = field1 (the LJ
   and FULL capped Coulomb derivative, bgy3d-solutes.c:381-468), the linear
   solve J dT = beta (chi - 1) * ((c' + 1) dv) from zero, and the
   differential of the free-energy density (chempot1, hnc3d.c:627-650,
   form1, closures.f90:615-653) with the long-range correlation held fixed.
   Writes grad->dx only (dq, dsigma, depsilon are left alone);
   grad->adjoint_jv = J.v products of all 3n solves, grad->adjoint_resid =
   the largest ||beta K((c'+1)dv) - J dT||_2 / ||beta K((c'+1)dv)||_2, grad->
   seconds = device time.  PY has no closure differential: RISM3D_ERR_UNSUPPORTED. */
int rism3d_response(rism3d_ctx *ctx, const double *T, rism3d_grad *grad);

/* The pass schedule the context runs, written to out[10]: x rows, y and z
   columns per CTA of the runtime-length passes for FP64 (out[0..2]) and
   FP32 (out[3..5]), whether the shape-specialised passes run (out[6]
   FP64, out[7] FP32) and the z-column width of their z pass (out[8],
   out[9]; negative when that pass runs from persistent double-buffered
   CTAs).  Chosen when the context is created by timing the
   candidates on its own buffers, once per grid shape and process
   (RISM3D_AUTOTUNE=0: a register / occupancy rule instead). */
int rism3d_tile_shapes(rism3d_ctx *ctx, int *out);

/* Points per axis of the two-grid preconditioner's coarse grid, written to
   n[3] (zeros when the preconditioner is off). */
int rism3d_coarse_grid(rism3d_ctx *ctx, int *n);

/* How the last coarse solve of the preconditioner ran (diagnostics; no
   counterpart in the reference): 2 = one persistent cooperative kernel
   (cubic coarse grids of 48, 64, 72, 96 or 128 points, m <= 3, coarse_steps
   <= 16, one solve per process at a time), 1 = a replayed CUDA graph of the
   step-by-step kernels, 0 = host-driven GMRES, -1 = none yet.
   RISM3D_COARSE_PERSIST=0 / RISM3D_COARSE_GRAPH=0 (environment, read when
   a context first solves) turn the first two off. */
int rism3d_coarse_driver(rism3d_ctx *ctx);

/* Per-pass CUDA-event timing (diagnostics): on != 0 enables it (it
   synchronises after every pass, so it is for measurement only).  The
   totals accumulated since the last call are returned in ms[12] /
   launches[12] (either may be NULL) and reset; bucket = pass + 6 * p with
   pass 0..5 = x-forward, y, z, x-inverse, vector ops, two-grid
   preconditioner (grid transfers and the whole coarse solve) and p = 0
   for FP64, 1 for FP32.  Launches are counted even when timing is off. */
int rism3d_profile(rism3d_ctx *ctx, int on, double *ms, long long *launches);

/* Jacobian product J dT = (chi - 1) * (d . dT) - dT for a caller-supplied
   closure slope d = dc/dt at the current t ([m][N2][N1][N0], device, FP64),
   computed by the same passes as rism3d_jacobian_t1 -- but allocating no
   device memory.  It has no counterpart in the reference: it exists for
   callers that cannot call cudaMalloc (solver loops where an allocation
   would synchronise the device or is forbidden by the host framework, or
   code that owns every device buffer itself).  Its scratch lives in a
   32 MiB file-scope device array held by every device that loads the
   library until exit; grids whose scratch exceeds it return RISM3D_ERR_ARG
   (m = 3 fits up to 96^3).  chi is the host [m][m][nrad] table as for
   rism3d_ctx_create; d, dT, JdT are device pointers.  The work runs on the
   calling host thread's per-thread default stream (cudaStreamPerThread; the
   library is built with per-thread default streams), so d and dT must be
   complete with respect to that stream; the call returns after the result
   is complete, without waiting for other streams.  The first call on a
   device looks up the array's device address (make it before any stream
   capture).  All calls share the array: calls that overlap on the GPU
   race.  Failures leave a message for rism3d_last_error(). */
int rism3d_jacobian_apply_noalloc(const rism3d_problem *pd, int m, const double *chi,
                                  const double *d, const double *dT, double *JdT);

/* ---- post-processing observables --------------------------------------- */

/* What print_info writes after a solute solve (info(), bgy3d-potential.c:
   245-493): moments of the solute's Gaussian charge density rho_u (cores(),
   bgy3d-solutes.c:555-577) and of the solvent charge density rho_v = rho
   sum_i q_i g_i (bgy3d_solvent_field), and three electrostatic energies with
   the solvent's Poisson potential v_e (bgy3d_poisson, bgy3d-poisson.c:
   103-183; no metallic cage).  Moments as bgy3d_moments (bgy3d-vec.c:
   576-593): q = h^3 sum f, d_a = h^3 h_a sum f x_a, Q_ab = h^3 h_a h_b sum
   f x_a x_b with x_a the grid index minus N_a / 2. */
typedef struct rism3d_info_result {
  double q_u, d_u[3], Q_u[3][3];  /* solute charge density */
  double q_v, d_v[3], Q_v[3][3];  /* solvent charge density */
  double d_n[3];                  /* dipole sum q x of the solute's point charges */
  double U_v_rho_N;               /* sum_u q_u v_e(x_u), trigonometric interpolation (bgy3d_pot_interp) */
  double U_v_rho_N_trilinear;     /* the same with trilinear interpolation (bgy3d_interp,
                                     bgy3d-interp.c:37-136; the value the regression outputs hold) */
  double U_v_rho_u;               /* h^3 sum v_e rho_u */
  double rho_v_U_u;               /* h^3 sum u_c rho_v, u_c the solute's long-range Coulomb */
  double seconds;
} rism3d_info_result;

/* The observables at a converged T (FP64 device pointer) of a solute
   context; site_potential (host [n] or NULL) receives v_e at the solute
   sites (trigonometric, print_table's column). */
int rism3d_info(rism3d_ctx *ctx, const double *T, rism3d_info_result *out, double *site_potential);

/* Moments of 1 - g for `fields` distributions g (device, [fields][N2][N1]
   [N0] on the context's grid): the `moments` command of the regression
   summaries (guile/bgy3d.scm:1136-1155).  out: host [fields][13] = q, d[3],
   Q[3][3] per field. */
int rism3d_moments(rism3d_ctx *ctx, const double *g, int fields, double *out);

/* ---- 3D solvent susceptibility (the --solvent-3d path) ---------------- */

/* Results of the pure-solvent solve. */
typedef struct rism3d_solvent_result {
  double mu;          /* excess chemical potential, the closure's functional, kcal/mol */
  double mu_hnc, mu_kh, mu_gf; /* the HNC, KH and GF functionals (print_chempot, hnc3d.c:674-694) */
  double a;           /* rho c(k=0) / 2 beta, kcal/mol (print_kappa, hnc3d.c:738-760) */
  double kappa;       /* isothermal compressibility beta / (rho (1 - rho c(k=0))), A^3/kcal */
  double resid_inf, resid_2;
  int status, newton_iters, f_evals, jv_evals;
  double seconds;     /* device time of the solve and post-processing */
} rism3d_solvent_result;

/*
  3D RISM of the pure solvent: replaces hnc3d_solvent_solve (hnc3d.c:
  803-1073).  The unknowns are the m(m+1)/2 site-site indirect correlations
  t_ij, i >= j, packed as pair p = i(i+1)/2 + j (vec_aliases_create2,
  bgy3d-vec.h:739-758), each a field [N2][N1][N0] centred on the box; the
  per-k molecular OZ equation h = (1 - rho W C)^-1 W C W with the
  intramolecular W = sinc(k r_ij) and the site-site potentials of
  bgy3d_pair_potential (bgy3d-force.c:123-147).  Newton-GMRES with the OZ
  equation's exact Jacobian (the reference differences F instead).  Uses
  pd->N, L (a cubic box), beta, rho, closure (not PY), norm_tol, max_iter,
  krylov_restart, ew_forcing; m <= 4.
    t_in     host [m(m+1)/2][N2][N1][N0] initial guess, or NULL for the 1D
             RISM t(r) on the upscaled radial grid (rmax = 2 max(L), nrad =
             16 max(N); hnc3d.c:776-851);
    t_out    host, the converged pair fields, or NULL;
    chi_out  host complex [m(m+1)/2][N2][N1][N0/2+1] (re, im pairs), or NULL:
             chi - 1 = rho h(k) + omega - 1 at the grid corner, the content of
             the reference's x%d%d-fft.bin (hnc3d.c:1011-1047), as the chi3
             input of rism3d_solute_solve_chi3;
    g_out    host [m(m+1)/2][N2][N1][N0] g = 1 + h, or NULL. */
int rism3d_solvent_solve(const rism3d_problem *pd, int m, const rism3d_site *solvent,
                         const double *t_in, double *t_out, double *chi_out, double *g_out,
                         rism3d_solvent_result *out);

/* A context on the pure solvent's pair fields: rism3d_iterate_t1 /
   rism3d_jacobian_t1 then evaluate iterate_t2 (hnc3d.c:353-456) and its
   Jacobian (FP64); the solute-only entry points return
   RISM3D_ERR_UNSUPPORTED. */
int rism3d_solvent_ctx_create(const rism3d_problem *pd, int m, const rism3d_site *solvent,
                              rism3d_ctx **ctx);

/* The solute solve on a 3D solvent kernel: chi3 = chi - 1 on the k grid
   (host complex [m(m+1)/2][N2][N1][N0/2+1], as rism3d_solvent_solve writes
   it) replaces the radial chi table -- the `solvent-3d` branch of
   solvent_kernel (hnc3d.c:1575-1587), which also selects the no-renorm
   long-range form.  Other arguments as rism3d_solute_solve; pd->rmax,
   nrad, renorm and coarse_h are ignored (no two-grid preconditioner). */
int rism3d_ctx_create_chi3(const rism3d_problem *pd, int m, const rism3d_site *solvent,
                           int n, const rism3d_site *solute, const double *chi3, rism3d_ctx **ctx);
int rism3d_solute_solve_chi3(const rism3d_problem *pd, int m, const rism3d_site *solvent,
                             int n, const rism3d_site *solute, const double *chi3,
                             double *t_inout, double *g_out, rism3d_result *out);

/* ---- solvent susceptibility (setup, CPU) ------------------------------ */

/* 1D RISM / DRISM of the pure solvent: replaces rism_solvent()
   (rism.f90:57-102, rism_vv 310-583).  Uses pd->beta, rho, rmax, nrad
   (2^a 3^b), closure, norm_tol (on r t(r)) and max_iter.
     dielectric  target epsilon of the DRISM correction (--dielectric), or 0
                 for plain RISM;
     chi         out, [m][m][nrad]: chi = omega + rho h -- the chi_fft_buf of
                 hnc3d_solute_solve and of rism3d_solute_solve above;
     t           optional, [m][m][nrad]: initial guess on entry, t(r) on exit;
     mu          optional, out: the solvent's excess chemical potential. */
int rism1d_solvent_chi(const rism3d_problem *pd, double dielectric, int m,
                       const rism3d_site *solvent, double *chi, double *t,
                       double *mu);

#ifdef __cplusplus
}
#endif
#endif /* RISM3D_H */
