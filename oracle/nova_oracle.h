/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the explicit time advance.
 *
 * A plain-C restatement of the reference's hot path: the 6th-order (or 2/4/8)
 * central operators of src/ex, the ghost fills of src/BC, the FFT projection
 * of src/poisson and the Runge-Kutta loop bodies of app/TG_Piosson and
 * app/OT_Poisson.  Every loop keeps the reference's loop nesting and the
 * association order of its floating-point expressions, so that (compiled with
 * -ffp-contract=off) it reproduces the reference bit for bit; the recipe in
 * oracle/Makefile builds the reference itself into oracle/_ref to check that.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker / reported CPU baseline.
 *
 * Data layout is the reference's Field<T> layout: ghosted, array-of-structs,
 * z fastest: element (i,j,k,c) at ((i*n1 + j)*n2 + k)*nc + c with
 * n = N + 1 + m per axis (src/Field/Field.h:82-85, src/Mesh/Mesh.cpp:89-138).
 */
#ifndef NOVA_ORACLE_H
#define NOVA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mesh orc_mesh;

enum { ORC_PERIODIC = 0, ORC_NEUMANN = 1, ORC_DIRICHLET = 2 };
/* face order of src/BC/BCenums.h:8: north(+j) south(-j) east(-i) west(+i) top(+k) bottom(-k) */
enum { ORC_NORTH = 0, ORC_SOUTH, ORC_EAST, ORC_WEST, ORC_TOP, ORC_BOTTOM };

orc_mesh *orc_mesh_new(const int N[3], const double L[3], const double origin[3], int m,
                       int hyperbolic_z, double s1, double s2);
void orc_mesh_free(orc_mesh *mesh);
void orc_mesh_dims(const orc_mesh *mesh, int n[3]);
void orc_mesh_metrics(const orc_mesh *mesh, double *dzdxi, double *d2zdxi2);

/* Ghost fill for a field with nc components; type/val indexed dir + 6*comp. */
void orc_bc_apply(const orc_mesh *mesh, double *f, int nc, const int *type, const double *val);

/* Operators: `out` is fully overwritten (zeros outside the interior loop range). */
void orc_grad_s(const orc_mesh *mesh, const double *f, double *out);            /* 1 -> 3 */
void orc_grad_v(const orc_mesh *mesh, const double *U, double *out);            /* 3 -> 9 */
void orc_curl(const orc_mesh *mesh, const double *U, double *out);              /* 3 -> 3 */
void orc_div_v(const orc_mesh *mesh, const double *U, double *out);             /* 3 -> 1 */
void orc_div_vf(const orc_mesh *mesh, const double *U, const double *f, int nc, double *out);
void orc_lap(const orc_mesh *mesh, double nu, const double *f, int nc, double *out);
void orc_div_t(const orc_mesh *mesh, const double *T, int symm, double *out);
void orc_div_sT(const orc_mesh *mesh, const double *s, const double *T, double *out);
void orc_lap_f(const orc_mesh *mesh, const double *nu, const double *f, int nc, double *out);
double orc_maximum(const orc_mesh *mesh, const double *f);                     /* scalar field */

/* poisson::rhs + poisson::solve: p's N0*N1*N2 unique interior nodes are written. */
void orc_poisson_solve(const orc_mesh *mesh, const double *rhs, double *p);
/* modified-wavenumber table k2[i + N0*(j + N1*k)] (poisson.cpp:337-396) */
void orc_poisson_k2(const orc_mesh *mesh, double *k2);

typedef struct {
    int model;      /* 0 = incompressible NS (TG_Piosson), 1 = incompressible MHD (OT_Poisson) */
    int rk_mode;    /* 0 = literal reference loop, 1 = classical RK4 (U refreshed per stage),
                       2 = app/shearLayer/UEqn.H (RK4 weights as stage coefficients, a projection
                       per stage; with model 1 the B terms enter the U loop and B stays frozen) */
    int nsteps;
    int diag_every; /* write a history row every diag_every steps (0 = never) */
    double dt, nu, eta;
    int bcU_type[18];
    double bcU_val[18];
    int bcp_type[6];
    double bcp_val[6];
    int bcB_type[18];
    double bcB_val[18];
    int bcpB_type[6];
    double bcpB_val[6];
} orc_run_desc;

/* History row: 0 step, 1 t, 2 Ek, 3 Em, 4 max|div U|, 5 max|div B|, 6 omega = mean|ex::curl(U)|,
 * 7 Jav = mean|ex::curl(B)|, 8 Jmax, 9 epsilon = -nu omega^2 - eta Jav^2, 10 Umax,
 * 11-13 tools::CFL x, y, z, 14 1/2<|curl U|^2>, 15 1/2<|curl B|^2> (central curl) */
#define ORC_HIST_COLS 16

/* Advance U (and B) by nsteps; p/pB hold the last pressures. hist: nsteps rows. */
int orc_run(const orc_mesh *mesh, const orc_run_desc *rd, double *U, double *B,
            double *p, double *pB, double *hist);
/* one history row of the state (U, B ghost-filled; B NULL for model 0) after step+1 steps at time t */
void orc_diag_row(const orc_mesh *mesh, const orc_run_desc *rd, int step, double t, const double *U,
                  const double *B, double *row);

#ifdef __cplusplus
}
#endif
#endif
