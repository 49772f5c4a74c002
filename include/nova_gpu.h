/*
 * nova_gpu.h -- C ABI of the B200 explicit time advance for NOVA.
 *
 * Plain C types only: opaque handles, pointers and sizes.  Every entry point
 * returns a nova_status; nova_last_error(ctx) gives the message of the last
 * failure on that context.  A context owns one CUDA stream (or uses the one
 * given to nova_set_stream) and all device memory it allocates; calls are
 * synchronous at the ABI unless documented otherwise.  A context is not
 * thread-safe, like the reference's one-thread-per-rank model.
 *
 * Reference interfaces replaced (paths inside the NOVA source tree):
 *   Mesh(std::string, Time&)                  src/Mesh/Mesh.cpp:24-179   -> nova_create
 *   Field<T>(Mesh&, const T&, std::string)    src/Field/Field.hxx:84-101 -> nova_field_create
 *   Field<T>::ptr() data / correctBoundaryConditions()
 *                                             src/Field/Field.h:98-101, Field.hxx:310-401
 *                                                        -> nova_field_upload / nova_field_download
 *   ex::grad(const Field<scalar>&)            src/ex/grad/grad.h:37-40     -> nova_grad_s
 *   ex::grad(const Field<vector>&)            src/ex/grad/grad.h:43-46     -> nova_grad_v
 *   ex::div(const Field<vector>&)             src/ex/div/div.h (div.hxx:22-81)  -> nova_div_v
 *   ex::div(const Field<vector>&, const Field<T>&)
 *                                             src/ex/div/div.h (div.hxx:84-172) -> nova_div_vf
 *   ex::curl(const Field<vector>&)            src/ex/curl/curl.h:35-43     -> nova_curl
 *   ex::laplacian(const scalar&, const Field<T>&)
 *                                             src/ex/laplacian/laplacian.h (laplacian.hxx:130-191)
 *                                                        -> nova_laplacian
 *   poisson::rhs(...) + poisson::solve()      src/poisson/poisson.h:111-113 -> nova_poisson_solve
 *   tools::maximum(shared_ptr<Field<T>>)      src/Tools/Tools.h:19-36      -> nova_field_maxabs
 *   the loop bodies app/TG_Piosson/RKLoop.H:1-54, app/OT_Poisson/UEqn.H:1-54,
 *   app/OT_Poisson/BEqn.H:1-110 and app/shearLayer/UEqn.H:1-54 (one time step each),
 *   with the per-step diagnostics of app/OT_Poisson/OT.cpp:132-176 and
 *   tools::CFL (src/Tools/Tools.cpp:9-41)                     -> nova_advance
 *   ex::div(tensor / symmTensor / scalar, tensor), ex::laplacian(Field nu, .)
 *                                             src/ex/div/div.hxx:173-285, laplacian.hxx:64-127
 *                                                        -> nova_div_t, nova_div_st, nova_laplacian_f
 *   im::laplacian, fdMatrix<scalar> and its operators, relax, setReference, residual, solve
 *                                             src/im/laplacian/laplacian.hxx:24-68,
 *                                             src/im/fdMatrix/fdMatrix.hxx:19-413
 *                                                        -> nova_im_laplacian, nova_fdm_*
 *   Field<T>::write / read, Mesh::write (EnSight Gold)
 *                                             src/Field/Field.hxx:404-516, src/Mesh/Mesh.cpp:224-369
 *                                                        -> nova_ensight_*
 */
#ifndef NOVA_GPU_H
#define NOVA_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NOVA_OK = 0,
    NOVA_E_INVALID = 1,     /* bad argument (sizes, null pointers, mismatched fields) */
    NOVA_E_CUDA = 2,        /* a CUDA or cuFFT call failed */
    NOVA_E_OOM = 3,         /* device allocation failed */
    NOVA_E_NONFINITE = 4,   /* a diagnostic reduction saw NaN/Inf in the state */
    NOVA_E_TIMEOUT = 5,     /* a bounded device wait (the stage pipeline's mbarriers) gave up */
    NOVA_E_UNSUPPORTED = 6  /* valid request this build does not implement */
} nova_status;

typedef enum {
    NOVA_F64 = 0,       /* FP64 storage and arithmetic */
    NOVA_F32SPLIT = 1   /* FP32 stencils/storage, state kept as a (hi, lo) float pair */
} nova_precision;

typedef enum { NOVA_BC_PERIODIC = 0, NOVA_BC_NEUMANN = 1, NOVA_BC_DIRICHLET = 2 } nova_bc_type;

/* Face order of the reference's BC files (src/BC/BCenums.h:8). */
typedef enum { NOVA_NORTH = 0, NOVA_SOUTH, NOVA_EAST, NOVA_WEST, NOVA_TOP, NOVA_BOTTOM } nova_face;

typedef struct nova_ctx nova_ctx;
typedef struct nova_field nova_field;

/* Mesh file contents (src/Mesh/Mesh.cpp:38-62) plus settings::m_. */
typedef struct {
    int N[3];            /* "N:"  intervals per axis (global; one GPU holds all of them) */
    double L[3];         /* "L:"  domain lengths */
    double origin[3];    /* "origin:" */
    int m;               /* stencil order 2, 4, 6 or 8 (settings::m_, default 6) */
    int hyperbolic_z;    /* "hypz:" present */
    double s1, s2;       /* "hypz:" arguments */
    int walls[3];        /* 0 = periodic axis (default); 1 = bounded by walls (Neumann/Dirichlet
                            faces, N+1 nodes stored).  This build supports walls in y only. */
} nova_mesh_desc;

/* BC lines "<face> <type> <val> <comp>" (src/Field/Field.hxx:519-547), index face + 6*comp. */
typedef struct {
    int type[18];
    double val[18];
} nova_bc;

typedef enum { NOVA_MODEL_NS = 0, NOVA_MODEL_MHD = 1 } nova_model;
/* LITERAL: app/TG_Piosson/RKLoop.H and app/OT_Poisson/UEqn.H as written (U not refreshed
 * between stages); CLASSICAL: the same loop with the stage state refreshed (RK4);
 * SHEARLAYER: app/shearLayer/UEqn.H:14-38 -- per stage rk, U* = UOld + RK4[rk] dt F(U)
 * with RK4 = {1/6, 1/3, 1/3, 1/6}, then a projection with rhs div(U*)/dt/RK4c[rk] and
 * U = U* - RK4c[rk] dt grad(p), so U is refreshed by a projected stage value (for MHD
 * the U loop runs with the Lorentz terms of a frozen B, and B is not advanced, as in
 * that app, whose BEqn.H is not included). */
typedef enum { NOVA_RK_LITERAL = 0, NOVA_RK_CLASSICAL = 1, NOVA_RK_SHEARLAYER = 2 } nova_rk_mode;
/* Pressure solve on a mesh with y walls.  FFT: the reference's poisson::solve on the N
 * unique y nodes as if y were periodic (what app/shearLayer does).  DCT: the inverse
 * consistent with the node-based walls -- the even extension in y (a DCT-I), so that
 * div(U) vanishes on the interior nodes after the projection. */
typedef enum { NOVA_POISSON_FFT = 0, NOVA_POISSON_DCT = 1 } nova_poisson_mode;

/* One nova_advance call = nsteps of the reference's per-step loop body. */
typedef struct {
    int model;        /* nova_model: NS = app/TG_Piosson, MHD = app/OT_Poisson */
    int rk_mode;      /* nova_rk_mode: LITERAL keeps the reference's stage loop as written
                         (U not refreshed between stages), CLASSICAL refreshes it (RK4) */
    int precision;    /* nova_precision of the state fields */
    int diag_every;   /* diagnostics row every diag_every steps (0 = none) */
    double dt, nu, eta;
    double t0;        /* time of the state on entry (only reported in the history) */
    int poisson;      /* nova_poisson_mode (meshes with y walls; periodic meshes ignore it) */
    int reserved;
} nova_run_desc;

/* Fields advanced by nova_advance.  U (3 comps) and p (1) always; B, pB for MHD. */
typedef struct {
    nova_field *U, *p, *B, *pB;
} nova_state;

/* One history row (the diagnostics the apps compute after each step):
 *   0 step, 1 t, 2 Ek = <1/2|U|^2>, 3 Em = <1/2|B|^2>, 4 max|div U|, 5 max|div B|
 *     (tools::maximum of ex::div, app/TG_Piosson/RKLoop.H:42-51, app/OT_Poisson/BEqn.H:46-54),
 *   6 omega = <|ex::curl(U)|>, 7 Jav = <|ex::curl(B)|>, 8 Jmax = max|ex::curl(B)|,
 *   9 epsilon = -nu omega^2 - eta Jav^2, 10 Umax = max|U|   (app/OT_Poisson/OT.cpp:132-176),
 *   11-13 cfl_x, cfl_y, cfl_z of tools::CFL (src/Tools/Tools.cpp:9-41, as written: signed
 *     velocities, and cfl_y, cfl_z compared against cfl_x at the loop's last node only),
 *   14 1/2 <|curl U|^2>, 15 1/2 <|curl B|^2> with the central 6th-order curl (the enstrophy;
 *     ex::curl is the reference's Q1 stencil of ex::grad(vector), which 6-8 keep).
 * <.> and the maxima of 8 and 10 run over the unique nodes, the divergence maxima and
 * cfl_x over every stored node.  nova_advance_wc fills the columns of U (0-2, 4, 6, 9-14;
 * epsilon with its mu). */
#define NOVA_HIST_COLS 16

/* ---- context ---- */
nova_status nova_create(const nova_mesh_desc *mesh, nova_ctx **out);
nova_status nova_destroy(nova_ctx *ctx);
const char *nova_last_error(const nova_ctx *ctx);
nova_status nova_set_stream(nova_ctx *ctx, void *cuda_stream);   /* cudaStream_t; NULL = own stream */
nova_status nova_synchronize(nova_ctx *ctx);
/* local ghosted sizes N+1+m of the reference Field layout */
nova_status nova_mesh_local_n(const nova_ctx *ctx, int local_n[3]);
/* Mesh::dzdxi_ / d2zdxi2_ (length local_n[2]), as the reference computes them */
nova_status nova_mesh_metrics(const nova_ctx *ctx, double *dzdxi, double *d2zdxi2);

/* ---- fields ---- */
nova_status nova_field_create(nova_ctx *ctx, int ncomp, int precision, nova_field **out);
nova_status nova_field_destroy(nova_ctx *ctx, nova_field *f);
/* Field<T>::setBC (src/Field/Field.hxx:519-547): the field's boundary conditions, used for
 * its ghosts in every stencil and for the wall-node overwrites of nova_advance.  Periodic
 * axes need periodic faces; wall axes need Neumann or Dirichlet faces.  Default: periodic,
 * Neumann 0 on wall faces. */
nova_status nova_field_set_bc(nova_ctx *ctx, nova_field *f, const nova_bc *bc);
nova_status nova_field_get_bc(nova_ctx *ctx, const nova_field *f, nova_bc *bc);
/* Reference Field<T>::ptr() layout: ghosted, AoS, z fastest, local_n = N+1+m per axis.
 * Upload reads the N0*N1*N2 unique interior nodes; download writes the interior
 * (incl. the duplicate node) and fills the ghosts per `bc` (NULL = all periodic). */
nova_status nova_field_upload(nova_ctx *ctx, nova_field *f, const double *host_aos, const int local_n[3]);
nova_status nova_field_download(nova_ctx *ctx, const nova_field *f, double *host_aos, const int local_n[3],
                                const nova_bc *bc);
/* Device-native layout: component-major, z fastest: [c][i][j][k], float64, over the
 * stored nodes (N per periodic axis, N+1 per wall axis). */
nova_status nova_field_upload_soa(nova_ctx *ctx, nova_field *f, const double *host_soa);
nova_status nova_field_download_soa(nova_ctx *ctx, const nova_field *f, double *host_soa);
/* Same, from/to device memory the caller owns (e.g. a torch tensor). */
nova_status nova_field_copy_from_device(nova_ctx *ctx, nova_field *f, const double *dev_soa);
nova_status nova_field_copy_to_device(nova_ctx *ctx, const nova_field *f, double *dev_soa);

/* ---- ex:: operators (one call each; out must have the right ncomp) ---- */
nova_status nova_grad_s(nova_ctx *ctx, const nova_field *s, nova_field *out);          /* 1 -> 3 */
nova_status nova_grad_v(nova_ctx *ctx, const nova_field *U, nova_field *out);          /* 3 -> 9 */
nova_status nova_curl(nova_ctx *ctx, const nova_field *U, nova_field *out);            /* 3 -> 3 */
nova_status nova_div_v(nova_ctx *ctx, const nova_field *U, nova_field *out);           /* 3 -> 1 */
nova_status nova_div_vf(nova_ctx *ctx, const nova_field *U, const nova_field *f, nova_field *out);
nova_status nova_laplacian(nova_ctx *ctx, double nu, const nova_field *f, nova_field *out);
/* poisson::rhs(rhs); poisson::solve(): p = L^-1 rhs on the unique nodes (mean mode 0) */
nova_status nova_poisson_solve(nova_ctx *ctx, const nova_field *rhs, nova_field *p);
/* ex:: variants no app's time advance calls (FP64):
 *   ex::div(Field<tensor>)              src/ex/div/div.hxx:258-285  -> nova_div_t (9 -> 3)
 *   ex::div(Field<symmTensor>)          div.hxx:222-255             -> nova_div_t (6 -> 3; xx xy xz yy yz zz)
 *   ex::div(Field<scalar>, Field<tensor>) div.hxx:173-207            -> nova_div_st (1 x 9 -> 3)
 *   ex::laplacian(Field<scalar>, Field<T>) src/ex/laplacian/laplacian.hxx:64-127 -> nova_laplacian_f
 * The tensor divergences carry no z metric, as in the reference. */
nova_status nova_div_t(nova_ctx *ctx, const nova_field *T, nova_field *out);
nova_status nova_div_st(nova_ctx *ctx, const nova_field *s, const nova_field *T, nova_field *out);
nova_status nova_laplacian_f(nova_ctx *ctx, const nova_field *nu, const nova_field *f, nova_field *out);
nova_status nova_field_maxabs(nova_ctx *ctx, const nova_field *s, double *out);
/* Allocation-free max|s|: the same result as nova_field_maxabs, which keeps its
 * per-block partials in memory the context allocates on first use (no
 * counterpart in the reference).  Here the partials live in a fixed 64 KiB
 * scratch in the library image (a static device array, one per device that
 * loads the library, held until the process exits), so the call never invokes
 * cudaMalloc/cudaFree or any pool allocator.  For callers that cannot allocate
 * device memory when they check a field: a solver whose HBM is all handed out
 * (fields sized to fill the device, or a framework's caching allocator holding
 * the rest), or a monitor that must not add an allocation's implicit
 * synchronisation to the running time steps.
 * Limit: at most NOVA_MAXABS_NOALLOC_MAX_NODES stored nodes (N0*N1*N2, with y
 * walls N0*(N1+1)*N2); larger fields return NOVA_E_INVALID (use
 * nova_field_maxabs).  The scratch needs no zeroing: each call writes every
 * slot before it reads it.  Each call looks up the scratch address with the
 * caller's device current (cudaGetSymbolAddress); the first call on a device
 * may load the library's device code, so make it before any stream capture.
 * Calls that overlap in time on one device (two streams, threads or contexts)
 * share the scratch and race: serialise them. */
#define NOVA_MAXABS_NOALLOC_MAX_NODES (1LL << 27)
nova_status nova_field_maxabs_noalloc(nova_ctx *ctx, const nova_field *s, double *out);

/* ---- fused time advance ---- */
/* hist: nsteps x NOVA_HIST_COLS doubles (rows of steps without diagnostics are zero); may be NULL */
nova_status nova_advance(nova_ctx *ctx, const nova_run_desc *run, nova_state *state, int nsteps, double *hist);

/* ---- discrete adjoint (no counterpart in the reference: added capability) ---- */
/* NOVA_OBJ_EKIN_FINAL:         J = Ek(N), Ek = mean(1/2 |U|^2) over the unique nodes
 * NOVA_OBJ_DISSIPATION_WINDOW: J = sum over steps n0+1..N of eps_n dt, eps_n = -(E(n) - E(n-1))/dt
 *                              the dissipation rate the apps print (app/TG/TG.cpp:113-115),
 *                              i.e. J = E(n0) - E(N), n0 = window_start; E = Ek (Navier-Stokes)
 *                              or Ek + Em (MHD; the apps print Ek, Em and their rates, app/OT_Poisson/OT.cpp:135-180)
 * NOVA_OBJ_ETOT_FINAL:         J = Ek(N) + Em(N), Em = mean(1/2 |B|^2) (MHD only)
 * NOVA_OBJ_LINEAR_FINAL:       J = <w, U(N)> / (N0 N1 N2), w = the weight field (Navier-Stokes,
 *                              FP64): the gradient is the adjoint of the linearised N-step map
 *                              applied to w / (N0 N1 N2), for the dot-product test
 *                              <D Phi v, w> = <v, D Phi^T w> */
typedef enum {
    NOVA_OBJ_EKIN_FINAL = 0,
    NOVA_OBJ_DISSIPATION_WINDOW = 1,
    NOVA_OBJ_ETOT_FINAL = 2,
    NOVA_OBJ_LINEAR_FINAL = 3
} nova_objective;
typedef struct {
    nova_run_desc run;     /* forward run: NS or MHD, classical RK4, FP64 or FP32-split, periodic uniform mesh */
    int nsteps;            /* steps of the forward solve */
    int checkpoint_every;  /* K: states kept every K steps, segments recomputed in reverse */
    int objective;         /* nova_objective */
    int window_start;      /* n0 of NOVA_OBJ_DISSIPATION_WINDOW, 0 <= n0 < nsteps */
    const nova_field *weight;  /* w of NOVA_OBJ_LINEAR_FINAL (3 comps, FP64); else ignored */
} nova_adj_desc;
/* Gradient of J with respect to the initial fields by the hand-written
 * discrete adjoint of the fused stages, the RK4 loops and the (self-adjoint)
 * projection.  init is not modified (its fields in the run's precision; for
 * FP32-split the trajectory is the split path's and the adjoint stages run in
 * FP32 with the adjoint state in FP64); gradU receives dJ/dU0 (FP64, 3 comps);
 * for MHD (run.model NOVA_MODEL_MHD, the U loop then the B loop of each step
 * as nova_advance runs them) gradB receives dJ/dB0 (FP64, 3 comps; required);
 * for Navier-Stokes gradB must be NULL.  *objective receives J. */
nova_status nova_adjoint_grad(nova_ctx *ctx, const nova_adj_desc *adj, const nova_state *init, nova_field *gradU,
                              nova_field *gradB, double *objective);

/* ---- implicit operators (src/im) ----
 * nova_fdm is the reference's fdMatrix<scalar> (src/im/fdMatrix/fdMatrix.h:33-77)
 * on a periodic uniform mesh: per-node coefficients al[0..5] of the neighbours
 * j+1, j-1, i+1, i-1, k+1, k-1 (N, S, E, W, T, B), the centre ap and the
 * source b, for A x = b with (A x)_n = ap x_n + sum_l al_l x_{n+l}, and the
 * transported FP64 scalar field x it solves for (kept by pointer, as the
 * reference keeps its shared_ptr). */
typedef struct nova_fdm nova_fdm;
/* im::laplacian(mu, x) (src/im/laplacian/laplacian.hxx:24-58): al = mu/d^2,
 * ap = -2 mu sum 1/d^2, b = -ex::laplacian(mu, x) + A x (the deferred
 * correction, src/im/fdMatrix/fdMatrix.hxx:201-225) */
nova_status nova_im_laplacian(nova_ctx *ctx, double mu, nova_field *x, nova_fdm **out);
/* a += alpha b, coefficients and source (operator+= / -=, fdMatrix.hxx:311-339; operator+ / binary operator-, 359-369, 383-393) */
nova_status nova_fdm_add(nova_ctx *ctx, nova_fdm *a, double alpha, const nova_fdm *b);
/* a *= b node by node, coefficients and source (operator*=, fdMatrix.hxx:341-354) */
nova_status nova_fdm_mul(nova_ctx *ctx, nova_fdm *a, const nova_fdm *b);
/* coefficients and source times s (s = -1: the unary operator-, fdMatrix.hxx:395-413) */
nova_status nova_fdm_scale(nova_ctx *ctx, nova_fdm *a, double s);
/* b += alpha f (operator== with alpha = 1, fdMatrix.hxx:371-381); f: FP64 scalar */
nova_status nova_fdm_add_source(nova_ctx *ctx, nova_fdm *a, double alpha, const nova_field *f);
/* ap += d (Field arithmetic on fdMatrix::ap()) */
nova_status nova_fdm_add_diagonal(nova_ctx *ctx, nova_fdm *a, double d);
/* fdMatrix::relax(urf) (fdMatrix.hxx:227-232): b += (1 - urf)/urf ap x, ap /= urf; urf > 0 */
nova_status nova_fdm_relax(nova_ctx *ctx, nova_fdm *a, double urf);
/* fdMatrix::setReference (fdMatrix.hxx:235-246) at the unique node (i, j, k): b += 1e15 val, ap *= 1e15 */
nova_status nova_fdm_set_reference(nova_ctx *ctx, nova_fdm *a, int i, int j, int k, double val);
/* fdMatrix::residual (fdMatrix.hxx:249-290): the RMS of b - A x over the
 * (N0+1)(N1+1)(N2+1) nodes the reference counts (the duplicate periodic
 * nodes included) */
nova_status nova_fdm_residual(nova_ctx *ctx, const nova_fdm *a, double *res);
/* fdMatrix::solve(tol, max_its) (fdMatrix.hxx:59-198): per iteration the
 * residual check (stop when not above tol), then line sweeps along j, i and k
 * on x.  Every line of a sweep is solved at once as a periodic tridiagonal
 * system with the neighbours off the line taken at the sweep's start, where
 * the reference solves the lines one after another (Gauss-Seidel across
 * lines), each as a Dirichlet problem whose ghost and duplicate end nodes keep
 * their values from the last ghost refresh (once per iteration): a different
 * iteration with the same fixed point.  its, res (the last residual checked)
 * may be NULL.  The first call allocates the solve's device storage, kept
 * until nova_fdm_destroy: a second x buffer and the factors of the three
 * line directions, 13 N0 N1 N2 doubles plus two per line; the factors are
 * recomputed only after a call that changes the coefficients. */
nova_status nova_fdm_solve(nova_ctx *ctx, nova_fdm *a, double tol, int max_its, int *its, double *res);
/* the eight fields to the host, SoA over the unique nodes: al0..al5, ap, b (8 x N0 N1 N2 doubles) */
nova_status nova_fdm_download(nova_ctx *ctx, const nova_fdm *a, double *host);
nova_status nova_fdm_destroy(nova_fdm *a);

/* ---- weakly-compressible time advance ----
 * One call = nsteps of the compressible loop bodies on a periodic mesh, FP64:
 *   NOVA_WC_TG:    app/TG/TG.cpp:73-75          rhoEqn.H, pEqn.H (p = K (rho rho), K = 50), UEqn.H
 *   NOVA_WC_SHEAR: app/shearLayerWC/shearLayer.cpp:197-200
 *                  UEqn.H (buoyancy -(rho T) g), rhoEqn.H, pEqn.H (p = (K rho) rho,
 *                  K = c^2/(2 rho0)), TEqn.H
 * Each loop is the reference's classical RK4 on rho*U, rho, rho*T.
 * hist: nsteps x NOVA_HIST_COLS rows (the columns of U; B's are zero) or NULL. */
typedef enum { NOVA_WC_TG = 0, NOVA_WC_SHEAR = 1 } nova_wc_case;
typedef struct {
    int wc_case;      /* nova_wc_case */
    int diag_every;   /* diagnostics row every n steps (0: none) */
    double dt;
    double mu;        /* laplacian(mu, U) */
    double ka;        /* laplacian(ka, T) (shear case) */
    double eos_k;     /* K of the EOS */
    double g[3];      /* gravity of the buoyancy term (shear case) */
    double t0;        /* time before the first step (for the hist rows) */
} nova_wc_desc;
typedef struct {
    nova_field *U, *rho, *p, *T;  /* T may be NULL for NOVA_WC_TG */
} nova_wc_state;
nova_status nova_advance_wc(nova_ctx *ctx, const nova_wc_desc *wd, nova_wc_state *st, int nsteps, double *hist);
/* The initialisation of app/shearLayerWC/shearLayer.cpp:114-150: p = (K rho0) rho0 plus the column
 * integral of T dz g_z rho0 from the top node down (hydrostaticP.H:1-38), rho = (p/K)^(1/2). */
nova_status nova_wc_hydrostatic(nova_ctx *ctx, const nova_wc_desc *wd, double rho0, const nova_field *T,
                                nova_field *p, nova_field *rho);

/* ---- restart checkpoints ----
 * Lossless FP64 restart of a state (the reference restarts from its EnSight
 * float output, src/Field/Field.hxx:404-516; this file keeps every bit).
 * Layout, host byte order:
 *   "NOVACKP1"; mesh: int32 N[3], m, walls[3], hyperbolic_z; double L[3],
 *   origin[3], s1, s2; double t; int64 step; int32 nfields, reserved;
 *   per field present (slot 0 U, 1 p, 2 B, 3 pB): int32 slot, ncomp, precision,
 *   reserved; nova_bc (int32 type[18], double val[18]); ncomp * N0*N1*N2
 *   doubles, component-major [c][i][j][k] over the stored nodes (N1 + 1 rows
 *   with y walls); FP32-split fields as hi + lo.
 * nova_checkpoint_write writes the fields of st that are non-NULL.
 * nova_checkpoint_read refuses a file of another mesh (NOVA_E_INVALID), fills
 * the non-NULL fields of st that the file holds (values and BCs; FP32-split
 * targets get the FP64 values split into hi + lo) and leaves the others as
 * they are; t and step may be NULL. */
nova_status nova_checkpoint_write(nova_ctx *ctx, const char *path, const nova_state *st, double t, long long step);
nova_status nova_checkpoint_read(nova_ctx *ctx, const char *path, nova_state *st, double *t, long long *step);

/* ---- EnSight Gold output (and input) in the reference's layout ----
 * The files the reference writes for post-processing (one rank, processor 0000):
 *   <dir>/geom.p0000.geo          block rectilinear, N+1 nodes per axis, float32
 *                                 coordinates (src/Mesh/Mesh.cpp:224-300)
 *   <dir>/fd.p0000.case, <dir>/restart.p.0000.case   the case file with the
 *                                 reference's variable list and the output times
 *                                 (Mesh.cpp:302-355)
 *   <dir>/<name>.0000.<num:05>.dat  float32 values over nodes 0..N of every axis
 *                                 (periodic duplicate included), i fastest,
 *                                 component by component (src/Field/Field.hxx:404-453)
 * The host functions need no GPU: soa is the stored-node layout [c][i][j][k] of
 * nova_field_download_soa.  nova_ensight_read_* is Field<T>::read
 * (Field.hxx:456-485): it restores float32 values.  Errors: NOVA_E_INVALID. */
nova_status nova_ensight_write_geometry(const nova_mesh_desc *md, const char *dir);
nova_status nova_ensight_write_case(const char *dir, int ntimes, const double *times);
nova_status nova_ensight_write_host(const nova_mesh_desc *md, const double *soa, int ncomp, const char *dir,
                                    const char *name, int num);
nova_status nova_ensight_read_host(const nova_mesh_desc *md, double *soa, int ncomp, const char *dir,
                                   const char *name, int num);
nova_status nova_ensight_write_field(nova_ctx *ctx, const nova_field *f, const char *dir, const char *name, int num);
nova_status nova_ensight_read_field(nova_ctx *ctx, nova_field *f, const char *dir, const char *name, int num);

/* ---- instrumentation: per-kernel CUDA-event timing of nova_advance ---- */
typedef enum { NOVA_K_STAGE = 0, NOVA_K_DIV = 1, NOVA_K_FFT = 2, NOVA_K_CORRECT = 3, NOVA_K_DIAG = 4, NOVA_K_ADJ = 5,
               NOVA_K_COUNT = 6 } nova_kernel_class;
nova_status nova_profile_enable(nova_ctx *ctx, int on);
/* total milliseconds and launch count per class since the last reset */
nova_status nova_profile_read(nova_ctx *ctx, int kernel_class, double *total_ms, long *launches, int reset);
/* number of kernels this library launched since the last reset */
nova_status nova_launch_count(nova_ctx *ctx, long *launches, int reset);

#ifdef __cplusplus
}
#endif
#endif
