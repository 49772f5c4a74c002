/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the explicit time advance.
 * See nova_oracle.h.  Each function names the reference lines it restates.
 * Build with -ffp-contract=off: the expressions below keep the reference's
 * association order so the result matches the reference bit for bit.
 *
 * With OpenMP the node loops are split across threads by i (inside each `l`
 * pass where the reference sweeps l outermost), so every node still receives
 * its terms in the reference's order and the result does not depend on the
 * thread count; the reductions of the diagnostics stay serial.
 */
#include "nova_oracle.h"
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_mesh {
    int m;          /* settings::m_ */
    int h;          /* m/2 ghost layers */
    int N[3];
    int n[3];       /* N + 1 + m */
    double d[3];    /* dx_, dy_, dz_ */
    double L[3];
    double origin[3];
    int hyper;
    double s1, s2;
    double *dzdxi;
    double *d2zdxi2;
    double coef[4];
};

/* settings::coef_ (src/settings/settings.cpp:25-31) */
static const double COEF[4][4] = {
    {1.0, 0.0, 0.0, 0.0},
    {4.0 / 3.0, -1.0 / 3.0, 0.0, 0.0},
    {6.0 / 4.0, -12.0 / 20.0, 1.0 / 10.0, 0.0},
    {8.0 / 5.0, -4.0 / 5.0, 24.0 / 105.0, -8.0 / 280.0},
};

/* settings::RK4a_ (src/settings/settings.cpp:44-50) */
static const double RK4A[4][4] = {
    {0.5, 0, 0, 0},
    {0, 0.5, 0, 0},
    {0, 0, 1.0, 0},
    {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0},
};

#define IDX(M, i, j, k) ((((long)(i) * (M)->n[1] + (j)) * (M)->n[2]) + (k))

static long npts(const orc_mesh *M) { return (long)M->n[0] * M->n[1] * M->n[2]; }

/* Mesh::z (src/Mesh/Mesh.cpp:373-407); single rank, so localStart_ == (ptrdiff_t)origin. */
static double mesh_z(const orc_mesh *M, int k)
{
    if (M->hyper) {
        double A = pow(M->s1 / M->s2, 0.5);
        int globK = k - M->h + (int)(long)M->origin[2];
        int globN = M->N[2] + 1;
        double R = (double)globK / (double)(globN - 1) - 0.5;
        double b = 1.0;
        for (int i = 1; i < 10000; i++)
            b = asinh(b / ((globN - 1) * pow(M->s1 * M->s2, 0.5)));
        double U = 1.0 + tanh(b * R) / tanh(b / 2.0);
        return U / (2.0 * A + (1 - A) * U) * M->L[2];
    }
    return (k - M->h) * M->d[2] + M->origin[2];
}

/* Mesh::Mesh (src/Mesh/Mesh.cpp:64-179), one rank. */
orc_mesh *orc_mesh_new(const int N[3], const double L[3], const double origin[3], int m,
                       int hyperbolic_z, double s1, double s2)
{
    if (m != 2 && m != 4 && m != 6 && m != 8) return NULL;
    orc_mesh *M = (orc_mesh *)calloc(1, sizeof(orc_mesh));
    M->m = m;
    M->h = m / 2;
    for (int a = 0; a < 3; a++) {
        M->N[a] = N[a];
        M->L[a] = L[a];
        M->origin[a] = origin[a];
        M->d[a] = L[a] / N[a];
        M->n[a] = N[a] / 1 + 1 + m;
    }
    M->hyper = hyperbolic_z;
    M->s1 = s1;
    M->s2 = s2;
    for (int l = 0; l < 4; l++) M->coef[l] = COEF[(m - 2) / 2][l];
    const int nk = M->n[2];
    M->dzdxi = (double *)calloc(nk, sizeof(double));
    M->d2zdxi2 = (double *)calloc(nk, sizeof(double));
    const double dz = M->d[2];
    for (int k = M->h; k < nk - M->h; k++) {
        M->dzdxi[k] = 0;
        for (int l = 0; l < M->h; l++) {
            M->dzdxi[k] += (M->coef[l] / 2.0 / (l + 1) / dz * mesh_z(M, k + 1 + l)
                            - M->coef[l] / 2.0 / (l + 1) / dz * mesh_z(M, k - 1 - l));
        }
    }
    for (int k = M->h; k < nk - M->h; k++) {
        M->d2zdxi2[k] = 0;
        for (int l = 0; l < M->h; l++) {
            M->d2zdxi2[k] += (M->coef[l] / pow((l + 1) * dz, 2) * mesh_z(M, k + 1 + l)
                              + M->coef[l] / pow((l + 1) * dz, 2) * mesh_z(M, k - 1 - l)
                              + (-2.0 * M->coef[l] / pow((l + 1) * dz, 2)) * mesh_z(M, k));
        }
    }
    return M;
}

void orc_mesh_free(orc_mesh *M)
{
    if (!M) return;
    free(M->dzdxi);
    free(M->d2zdxi2);
    free(M);
}

void orc_mesh_dims(const orc_mesh *M, int n[3])
{
    for (int a = 0; a < 3; a++) n[a] = M->n[a];
}

void orc_mesh_metrics(const orc_mesh *M, double *dzdxi, double *d2zdxi2)
{
    memcpy(dzdxi, M->dzdxi, sizeof(double) * M->n[2]);
    memcpy(d2zdxi2, M->d2zdxi2, sizeof(double) * M->n[2]);
}

/* ------------------------------------------------------------------ BCs -- */

/* periodicBC::update (src/BC/periodicBC.hxx:1-66): copies whole T; active on east/south/bottom. */
static void bc_periodic(const orc_mesh *M, double *f, int nc, int dir)
{
    const int ni = M->n[0], nj = M->n[1], nk = M->n[2], m = M->m, h = M->h;
    if (dir == ORC_EAST) {
        for (int k = 0; k < nk; k++)
            for (int j = 0; j < nj; j++) {
                for (int i = 0; i < h; i++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i + ni - m - 1, j, k) * nc + c];
                for (int i = ni - h - 1; i < ni; i++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i - ni + m + 1, j, k) * nc + c];
            }
    }
    if (dir == ORC_SOUTH) {
        for (int k = 0; k < nk; k++)
            for (int i = 0; i < ni; i++) {
                for (int j = 0; j < h; j++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i, j + nj - m - 1, k) * nc + c];
                for (int j = nj - h - 1; j < nj; j++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i, j - nj + m + 1, k) * nc + c];
            }
    }
    if (dir == ORC_BOTTOM) {
        for (int i = 0; i < ni; i++)
            for (int j = 0; j < nj; j++) {
                for (int k = 0; k < h; k++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i, j, k + nk - m - 1) * nc + c];
                for (int k = nk - h - 1; k < nk; k++)
                    for (int c = 0; c < nc; c++)
                        f[IDX(M, i, j, k) * nc + c] = f[IDX(M, i, j, k - nk + m + 1) * nc + c];
            }
    }
}

/* neumannBC::update (src/BC/neumannBC.hxx:1-134) and dirichletBC::update
 * (src/BC/dirichletBC.hxx:1-127).  `lo` faces: east(i), south(j), bottom(k). */
static void bc_wall(const orc_mesh *M, double *f, int nc, int dir, int comp, int type, double val)
{
    const int h = M->h;
    int ax, lo;
    switch (dir) {
    case ORC_EAST: ax = 0; lo = 1; break;
    case ORC_WEST: ax = 0; lo = 0; break;
    case ORC_SOUTH: ax = 1; lo = 1; break;
    case ORC_NORTH: ax = 1; lo = 0; break;
    case ORC_BOTTOM: ax = 2; lo = 1; break;
    default: ax = 2; lo = 0; break;
    }
    const double del = M->d[ax];
    const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
    const int wall = lo ? h : M->n[ax] - h - 1;
    const int s = lo ? 1 : -1; /* step into the domain */
    for (int p = 0; p < M->n[a1]; p++)
        for (int q = 0; q < M->n[a2]; q++) {
            int ijk[3];
            ijk[a1] = p;
            ijk[a2] = q;
#define AT(off) (f[IDX(M, (ax == 0 ? wall + (off) : ijk[0]), (ax == 1 ? wall + (off) : ijk[1]), \
                        (ax == 2 ? wall + (off) : ijk[2])) * nc + comp])
            if (type == ORC_NEUMANN) {
                if (lo)
                    AT(0) = AT(1) - val * del;
                else
                    AT(0) = AT(-1) + val * del;
                for (int l = 0; l < h; l++)
                    AT(-s * (l + 1)) = AT(s * (l + 1)) - 2.0 * (l + 1) * val * del;
            } else {
                AT(0) = val;
                for (int l = 0; l < h; l++)
                    AT(-s * (l + 1)) = 2.0 * (l + 1) * val - AT(s * (l + 1));
            }
#undef AT
        }
}

/* Field<T>::correctBoundaryConditions (src/Field/Field.hxx:310-322): bc index d = dir + 6*comp. */
void orc_bc_apply(const orc_mesh *M, double *f, int nc, const int *type, const double *val)
{
    for (int d = 0; d < 6 * nc; d++) {
        int dir = d % 6, comp = d / 6;
        if (type[d] == ORC_PERIODIC)
            bc_periodic(M, f, nc, dir);
        else
            bc_wall(M, f, nc, dir, comp, type[d], val[d]);
    }
}

/* ------------------------------------------------------------ operators -- */

/* ex::grad(Field<scalar>) (src/ex/grad/grad.cpp:25-62) */
void orc_grad_s(const orc_mesh *M, const double *f, double *g)
{
    const int h = M->h;
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(g, 0, sizeof(double) * 3 * npts(M));
    for (int l = 0; l < h; l++)
#pragma omp parallel for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++)
                for (int k = h; k < M->n[2] - h; k++) {
                    double *gp = g + IDX(M, i, j, k) * 3;
                    double gx = co[l] / 2.0 / (l + 1) / dx * f[IDX(M, i + 1 + l, j, k)]
                              - co[l] / 2.0 / (l + 1) / dx * f[IDX(M, i - 1 - l, j, k)];
                    double gy = co[l] / 2.0 / (l + 1) / dy * f[IDX(M, i, j + 1 + l, k)]
                              - co[l] / 2.0 / (l + 1) / dy * f[IDX(M, i, j - 1 - l, k)];
                    double gz = co[l] / 2.0 / (l + 1) / dz * f[IDX(M, i, j, k + 1 + l)] / M->dzdxi[k]
                              - co[l] / 2.0 / (l + 1) / dz * f[IDX(M, i, j, k - 1 - l)] / M->dzdxi[k];
                    gp[0] += gx;
                    gp[1] += gy;
                    gp[2] += gz;
                }
}

/* ex::grad(Field<vector>) -> tensor, row = component, column = direction
 * (src/ex/grad/grad.cpp:65-102).  Keeps the reference stencil f(i+l)-f(i-1-l). */
void orc_grad_v(const orc_mesh *M, const double *U, double *T)
{
    const int h = M->h;
    const double *co = M->coef;
    memset(T, 0, sizeof(double) * 9 * npts(M));
#pragma omp parallel for schedule(static)
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                double *t = T + IDX(M, i, j, k) * 9;
                for (int q = 0; q < 9; q++) t[q] = 0.0;
                for (int l = 0; l < h; l++) {
                    double dx = co[l] / (l + 1) / M->d[0];
                    double dy = co[l] / (l + 1) / M->d[1];
                    double dz = co[l] / (l + 1) / M->d[2] / M->dzdxi[k];
                    for (int c = 0; c < 3; c++) {
                        t[3 * c + 0] += dx * (U[IDX(M, i + l, j, k) * 3 + c] - U[IDX(M, i - 1 - l, j, k) * 3 + c]);
                        t[3 * c + 1] += dy * (U[IDX(M, i, j + l, k) * 3 + c] - U[IDX(M, i, j - 1 - l, k) * 3 + c]);
                        t[3 * c + 2] += dz * (U[IDX(M, i, j, k + l) * 3 + c] - U[IDX(M, i, j, k - 1 - l) * 3 + c]);
                    }
                }
            }
}

/* ex::curl (src/ex/curl/curl.cpp:25-57): antisymmetric part of grad(vector). */
void orc_curl(const orc_mesh *M, const double *U, double *out)
{
    const int h = M->h;
    double *T = (double *)malloc(sizeof(double) * 9 * npts(M));
    orc_grad_v(M, U, T);
    memset(out, 0, sizeof(double) * 3 * npts(M));
#pragma omp parallel for schedule(static)
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                const double *t = T + IDX(M, i, j, k) * 9;
                double *o = out + IDX(M, i, j, k) * 3;
                o[0] = t[7] - t[5]; /* zy - yz */
                o[1] = t[2] - t[6]; /* xz - zx */
                o[2] = t[3] - t[1]; /* yx - xy */
            }
    free(T);
}

/* ex::div(Field<vector>) (src/ex/div/div.hxx:22-81) */
void orc_div_v(const orc_mesh *M, const double *U, double *out)
{
    const int h = M->h, nk = M->n[2];
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * npts(M));
#pragma omp parallel
    {
    double *Up = (double *)malloc(sizeof(double) * 6 * nk);
    double *Um = Up + nk, *Vp = Up + 2 * nk, *Vm = Up + 3 * nk, *Wp = Up + 4 * nk, *Wm = Up + 5 * nk;
    for (int l = 0; l < h; l++)
#pragma omp for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *dp = out + IDX(M, i, j, 0);
                for (int k = h; k < nk - h; k++) {
                    Vp[k] = U[IDX(M, i, j + 1 + l, k) * 3 + 1];
                    Vm[k] = U[IDX(M, i, j - 1 - l, k) * 3 + 1];
                    Up[k] = U[IDX(M, i + 1 + l, j, k) * 3 + 0];
                    Um[k] = U[IDX(M, i - 1 - l, j, k) * 3 + 0];
                    Wp[k] = U[IDX(M, i, j, k + 1 + l) * 3 + 2];
                    Wm[k] = U[IDX(M, i, j, k - 1 - l) * 3 + 2];
                }
                for (int k = h; k < nk - h; k++)
                    dp[k] += (co[l] / 2.0 / (l + 1) / dy * Vp[k]
                              - co[l] / 2.0 / (l + 1) / dy * Vm[k]
                              + co[l] / 2.0 / (l + 1) / dx * Up[k]);
                for (int k = h; k < nk - h; k++)
                    dp[k] += (-co[l] / 2.0 / (l + 1) / dx * Um[k]
                              + co[l] / 2.0 / (l + 1) / dz * Wp[k] / M->dzdxi[k]
                              - co[l] / 2.0 / (l + 1) / dz * Wm[k] / M->dzdxi[k]);
            }
    free(Up);
    }
}

/* ex::div(Field<vector> U, Field<T> f): skew-symmetric advective form
 * (src/ex/div/div.hxx:84-172); T has nc components, each updated with the same
 * scalar factors the vector algebra of src/Types/vector/vector.cpp applies. */
void orc_div_vf(const orc_mesh *M, const double *U, const double *f, int nc, double *out)
{
    const int h = M->h, nk = M->n[2];
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * nc * npts(M));
#define F(i, j, k, c) f[IDX(M, i, j, k) * nc + (c)]
#pragma omp parallel
    {
    double *Up = (double *)malloc(sizeof(double) * 6 * nk);
    double *Um = Up + nk, *Vp = Up + 2 * nk, *Vm = Up + 3 * nk, *Wp = Up + 4 * nk, *Wm = Up + 5 * nk;
    for (int l = 0; l < h; l++)
#pragma omp for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *dp = out + IDX(M, i, j, 0) * nc;
                for (int k = h; k < nk - h; k++) {
                    Vp[k] = U[IDX(M, i, j + 1 + l, k) * 3 + 1];
                    Vm[k] = U[IDX(M, i, j - 1 - l, k) * 3 + 1];
                    Up[k] = U[IDX(M, i + 1 + l, j, k) * 3 + 0];
                    Um[k] = U[IDX(M, i - 1 - l, j, k) * 3 + 0];
                    Wp[k] = U[IDX(M, i, j, k + 1 + l) * 3 + 2];
                    Wm[k] = U[IDX(M, i, j, k - 1 - l) * 3 + 2];
                }
                for (int k = h; k < nk - h; k++)
                    for (int c = 0; c < nc; c++)
                        dp[k * nc + c] += (0.5 * co[l] / 2.0 / (l + 1) / dy * F(i, j + 1 + l, k, c) * Vp[k]
                                           - 0.5 * co[l] / 2.0 / (l + 1) / dy * F(i, j - 1 - l, k, c) * Vm[k]
                                           + 0.5 * co[l] / 2.0 / (l + 1) / dx * F(i + 1 + l, j, k, c) * Up[k]);
                for (int k = h; k < nk - h; k++)
                    for (int c = 0; c < nc; c++)
                        dp[k * nc + c] += (-0.5 * co[l] / 2.0 / (l + 1) / dx * F(i - 1 - l, j, k, c) * Um[k]
                                           + 0.5 * co[l] / 2.0 / (l + 1) / dz * F(i, j, k + 1 + l, c) * Wp[k] / M->dzdxi[k]
                                           - 0.5 * co[l] / 2.0 / (l + 1) / dz * F(i, j, k - 1 - l, c) * Wm[k] / M->dzdxi[k]);
                for (int k = h; k < nk - h; k++) {
                    const double *u0 = U + IDX(M, i, j, k) * 3;
                    for (int c = 0; c < nc; c++)
                        dp[k * nc + c] += (0.5 * u0[1] * co[l] / 2.0 / (l + 1) / dy * F(i, j + 1 + l, k, c)
                                           - 0.5 * u0[1] * co[l] / 2.0 / (l + 1) / dy * F(i, j - 1 - l, k, c)
                                           + 0.5 * u0[0] * co[l] / 2.0 / (l + 1) / dx * F(i + 1 + l, j, k, c)
                                           - 0.5 * u0[0] * co[l] / 2.0 / (l + 1) / dx * F(i - 1 - l, j, k, c)
                                           + 0.5 * u0[2] * co[l] / 2.0 / (l + 1) / dz * F(i, j, k + 1 + l, c) / M->dzdxi[k]
                                           - 0.5 * u0[2] * co[l] / 2.0 / (l + 1) / dz * F(i, j, k - 1 - l, c) / M->dzdxi[k]);
                }
                for (int k = h; k < nk - h; k++)
                    for (int c = 0; c < nc; c++) {
                        double f0 = 0.5 * F(i, j, k, c);
                        dp[k * nc + c] += (f0 * (co[l] / 2.0 / (l + 1) / dy * Vp[k])
                                           - f0 * (co[l] / 2.0 / (l + 1) / dy * Vm[k])
                                           + f0 * (co[l] / 2.0 / (l + 1) / dx * Up[k])
                                           - f0 * (co[l] / 2.0 / (l + 1) / dx * Um[k])
                                           + f0 * (co[l] / 2.0 / (l + 1) / dz * Wp[k]) / M->dzdxi[k]
                                           - f0 * (co[l] / 2.0 / (l + 1) / dz * Wm[k]) / M->dzdxi[k]);
                    }
            }
    free(Up);
    }
#undef F
}

/* ex::laplacian(scalar nu, Field<T>) incl. the stretched-z correction
 * (src/ex/laplacian/laplacian.hxx:130-191). */
void orc_lap(const orc_mesh *M, double nu, const double *f, int nc, double *out)
{
    const int h = M->h;
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * nc * npts(M));
#define F(i, j, k, c) f[IDX(M, i, j, k) * nc + (c)]
    for (int l = 0; l < h; l++)
#pragma omp parallel for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *lp = out + IDX(M, i, j, 0) * nc;
                for (int k = h; k < M->n[2] - h; k++) {
                    const double zz = pow(M->dzdxi[k], 2);
                    for (int c = 0; c < nc; c++)
                        lp[k * nc + c] += (nu * co[l] / pow((l + 1) * dy, 2) * F(i, j + 1 + l, k, c)
                                           + nu * co[l] / pow((l + 1) * dy, 2) * F(i, j - 1 - l, k, c)
                                           + nu * co[l] / pow((l + 1) * dx, 2) * F(i + 1 + l, j, k, c)
                                           + nu * co[l] / pow((l + 1) * dx, 2) * F(i - 1 - l, j, k, c)
                                           + nu * co[l] / pow((l + 1) * dz, 2) * F(i, j, k + 1 + l, c) / zz
                                           + nu * co[l] / pow((l + 1) * dz, 2) * F(i, j, k - 1 - l, c) / zz
                                           + (-(nu + nu) * co[l] / pow((l + 1) * dx, 2)
                                              - (nu + nu) * co[l] / pow((l + 1) * dy, 2)
                                              - (nu + nu) * co[l] / pow((l + 1) * dz, 2) / zz) * F(i, j, k, c));
                }
            }
    for (int l = 0; l < h; l++)
#pragma omp parallel for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *lp = out + IDX(M, i, j, 0) * nc;
                for (int k = h; k < M->n[2] - h; k++) {
                    const double z3 = pow(M->dzdxi[k], 3);
                    for (int c = 0; c < nc; c++)
                        lp[k * nc + c] -= (co[l] / 2.0 / (l + 1) / dz * F(i, j, k + 1 + l, c)
                                           - co[l] / 2.0 / (l + 1) / dz * F(i, j, k - 1 - l, c))
                                          * nu * M->d2zdxi2[k] / z3;
                }
            }
#undef F
}

/* ex::div(Field<tensor>) (src/ex/div/div.hxx:258-285) and ex::div(Field<symmTensor>)
 * (div.hxx:222-255, tensor(symm) of src/Types/tensor/tensor.cpp:43-46 with the
 * storage xx xy xz yy yz zz): out_c = sum_l N - S + E - W + T - B of component
 * [c*3 + d], no z metric.  T holds 9 (symm = 0) or 6 (symm = 1) components. */
static double tens(const double *T, long p, int symm, int r)
{
    static const int S[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    return symm ? T[p * 6 + S[r]] : T[p * 9 + r];
}

void orc_div_t(const orc_mesh *M, const double *T, int symm, double *out)
{
    const int h = M->h;
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * 3 * npts(M));
#pragma omp parallel for schedule(static)
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                double *o = out + IDX(M, i, j, k) * 3;
                for (int l = 0; l < h; l++)
                    for (int c = 0; c < 3; c++) {
                        o[c] += co[l] / 2.0 / (l + 1) / dy * tens(T, IDX(M, i, j + 1 + l, k), symm, c * 3 + 1);
                        o[c] += -co[l] / 2.0 / (l + 1) / dy * tens(T, IDX(M, i, j - 1 - l, k), symm, c * 3 + 1);
                        o[c] += co[l] / 2.0 / (l + 1) / dx * tens(T, IDX(M, i + 1 + l, j, k), symm, c * 3);
                        o[c] += -co[l] / 2.0 / (l + 1) / dx * tens(T, IDX(M, i - 1 - l, j, k), symm, c * 3);
                        o[c] += co[l] / 2.0 / (l + 1) / dz * tens(T, IDX(M, i, j, k + 1 + l), symm, c * 3 + 2);
                        o[c] += -co[l] / 2.0 / (l + 1) / dz * tens(T, IDX(M, i, j, k - 1 - l), symm, c * 3 + 2);
                    }
            }
}

/* ex::div(Field<scalar> s, Field<tensor> T) (div.hxx:173-207): the same sums of s*T */
void orc_div_sT(const orc_mesh *M, const double *s, const double *T, double *out)
{
    const int h = M->h;
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * 3 * npts(M));
#define SV(i, j, k) s[IDX(M, i, j, k)]
#define TV(i, j, k, r) T[IDX(M, i, j, k) * 9 + (r)]
#pragma omp parallel for schedule(static)
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                double *o = out + IDX(M, i, j, k) * 3;
                for (int l = 0; l < h; l++)
                    for (int c = 0; c < 3; c++) {
                        o[c] += co[l] / 2.0 / (l + 1) / dy * SV(i, j + 1 + l, k) * TV(i, j + 1 + l, k, c * 3 + 1);
                        o[c] += -co[l] / 2.0 / (l + 1) / dy * SV(i, j - 1 - l, k) * TV(i, j - 1 - l, k, c * 3 + 1);
                        o[c] += co[l] / 2.0 / (l + 1) / dx * SV(i + 1 + l, j, k) * TV(i + 1 + l, j, k, c * 3);
                        o[c] += -co[l] / 2.0 / (l + 1) / dx * SV(i - 1 - l, j, k) * TV(i - 1 - l, j, k, c * 3);
                        o[c] += co[l] / 2.0 / (l + 1) / dz * SV(i, j, k + 1 + l) * TV(i, j, k + 1 + l, c * 3 + 2);
                        o[c] += -co[l] / 2.0 / (l + 1) / dz * SV(i, j, k - 1 - l) * TV(i, j, k - 1 - l, c * 3 + 2);
                    }
            }
#undef SV
#undef TV
}

/* ex::laplacian(Field<scalar> nu, Field<T>) (src/ex/laplacian/laplacian.hxx:64-127):
 * the + neighbour weighted by nu at offset l, the - neighbour by nu at -1-l */
void orc_lap_f(const orc_mesh *M, const double *nu, const double *f, int nc, double *out)
{
    const int h = M->h;
    const double dx = M->d[0], dy = M->d[1], dz = M->d[2];
    const double *co = M->coef;
    memset(out, 0, sizeof(double) * nc * npts(M));
#define F(i, j, k, c) f[IDX(M, i, j, k) * nc + (c)]
#define NU(i, j, k) nu[IDX(M, i, j, k)]
    for (int l = 0; l < h; l++)
#pragma omp parallel for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *lp = out + IDX(M, i, j, 0) * nc;
                for (int k = h; k < M->n[2] - h; k++) {
                    const double zz = pow(M->dzdxi[k], 2);
                    const double nN = NU(i, j + l, k), nS = NU(i, j - 1 - l, k), nE = NU(i + l, j, k),
                                 nW = NU(i - 1 - l, j, k), nT = NU(i, j, k + l), nB = NU(i, j, k - 1 - l);
                    for (int c = 0; c < nc; c++)
                        lp[k * nc + c] += (nN * co[l] / pow((l + 1) * dy, 2) * F(i, j + 1 + l, k, c)
                                           + nS * co[l] / pow((l + 1) * dy, 2) * F(i, j - 1 - l, k, c)
                                           + nE * co[l] / pow((l + 1) * dx, 2) * F(i + 1 + l, j, k, c)
                                           + nW * co[l] / pow((l + 1) * dx, 2) * F(i - 1 - l, j, k, c)
                                           + nT * co[l] / pow((l + 1) * dz, 2) * F(i, j, k + 1 + l, c) / zz
                                           + nB * co[l] / pow((l + 1) * dz, 2) * F(i, j, k - 1 - l, c) / zz
                                           + (-(nE + nW) * co[l] / pow((l + 1) * dx, 2)
                                              - (nN + nS) * co[l] / pow((l + 1) * dy, 2)
                                              - (nT + nB) * co[l] / pow((l + 1) * dz, 2) / zz) * F(i, j, k, c));
                }
            }
    for (int l = 0; l < h; l++)
#pragma omp parallel for schedule(static)
        for (int i = h; i < M->n[0] - h; i++)
            for (int j = h; j < M->n[1] - h; j++) {
                double *lp = out + IDX(M, i, j, 0) * nc;
                for (int k = h; k < M->n[2] - h; k++) {
                    const double z3 = pow(M->dzdxi[k], 3);
                    for (int c = 0; c < nc; c++)
                        lp[k * nc + c] -= (co[l] / 2.0 / (l + 1) / dz * F(i, j, k + 1 + l, c)
                                           - co[l] / 2.0 / (l + 1) / dz * F(i, j, k - 1 - l, c))
                                          * NU(i, j, k) * M->d2zdxi2[k] / z3;
                }
            }
#undef F
#undef NU
}

/* tools::maximum (src/Tools/Tools.h:19-36) for a scalar field */
double orc_maximum(const orc_mesh *M, const double *f)
{
    const int h = M->h;
    double mx = 0.0;
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                double a = fabs(f[IDX(M, i, j, k)]);
                mx = a > mx ? a : mx; /* std::max(|f|, max) returns max unless |f| > max */
            }
    return mx;
}

/* -------------------------------------------------------------- poisson -- */

/* poisson::wavenumbersFFT_ (src/poisson/poisson.cpp:337-396), one rank (localStart = 0). */
void orc_poisson_k2(const orc_mesh *M, double *k2)
{
    const int ni = M->N[0], nj = M->N[1], nk = M->N[2];
    const double eps = 1.0e-16, pi = M_PI;
    const double *co = M->coef;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++)
            for (int i = 0; i < ni; i++) {
                const long l = ((long)k * nj + j) * ni + i;
                double kx, ky, kz;
                if (2 * (i) < M->N[0])
                    kx = 2.0 * pi * (i) / M->L[0];
                else
                    kx = 2.0 * pi * (M->N[0] - i) / M->L[0];
                if (2 * (j) < M->N[1])
                    ky = 2.0 * pi * (j) / M->L[1];
                else
                    ky = 2.0 * pi * (M->N[1] - j) / M->L[1];
                kz = 2.0 * pi * (k) / M->L[2];
                double kpx = 0.0, kpy = 0.0, kpz = 0.0;
                if (kx > eps)
                    for (int ll = 0; ll < M->h; ll++)
                        kpx += kx * co[ll] / (ll + 1) * sin((ll + 1) * kx * M->d[0]) / (kx * M->d[0]);
                if (ky > eps)
                    for (int ll = 0; ll < M->h; ll++)
                        kpy += ky * co[ll] / (ll + 1) * sin((ll + 1) * ky * M->d[1]) / (ky * M->d[1]);
                if (kz > eps)
                    for (int ll = 0; ll < M->h; ll++)
                        kpz += kz * co[ll] / (ll + 1) * sin((ll + 1) * kz * M->d[2]) / (kz * M->d[2]);
                k2[l] = kpx * kpx + kpy * kpy + kpz * kpz;
            }
}

/* poisson::rhs + poisson::solve (src/poisson/poisson.cpp:167-181, 223-265) */
void orc_poisson_solve(const orc_mesh *M, const double *rhs, double *p)
{
    const int h = M->h;
    const int N0 = M->N[0], N1 = M->N[1], N2 = M->N[2];
    const long tot = (long)N0 * N1 * N2;
    orc_cplx *phi = (orc_cplx *)malloc(sizeof(orc_cplx) * tot);
    double *k2 = (double *)malloc(sizeof(double) * tot);
    orc_poisson_k2(M, k2);
    long l = 0;
    for (int k = h; k < M->n[2] - 1 - h; k++)
        for (int j = h; j < M->n[1] - 1 - h; j++)
            for (int i = h; i < M->n[0] - 1 - h; i++) {
                phi[l].re = rhs[IDX(M, i, j, k)];
                phi[l].im = 0.0;
                l++;
            }
    orc_fft3d(M->N, phi, -1);
    const double eps = 1.0e-16;
#pragma omp parallel for schedule(static)
    for (l = 0; l < tot; l++) {
        if (k2[l] < eps) {
            phi[l].re = 0.0;
            phi[l].im = 0.0;
        } else {
            double re = -phi[l].re / k2[l];
            double im = -phi[l].im / k2[l];
            phi[l].re = re;
            phi[l].im = im;
        }
    }
    orc_fft3d(M->N, phi, +1);
    l = 0;
    const double scale = (double)((long)N0 * N1 * N2);
    for (int k = h; k < M->n[2] - 1 - h; k++)
        for (int j = h; j < M->n[1] - 1 - h; j++)
            for (int i = h; i < M->n[0] - 1 - h; i++) {
                p[IDX(M, i, j, k)] = phi[l].re / scale;
                l++;
            }
    free(phi);
    free(k2);
}

/* -------------------------------------------------------- time advance -- */

/* one component of a vector field as a scalar field, ghosts included */
static void component(const orc_mesh *M, const double *U, int c, double *out)
{
    const long n = npts(M);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n; q++) out[q] = U[3 * q + c];
}

/* the central curl of U from grad(scalar) of its components (src/ex/grad/grad.cpp:25-62
 * applied to U.x, U.y, U.z); g: 9*npts scratch (grad of component c at 3*c) */
static void central_curl(const orc_mesh *M, const double *U, double *s, double *g, double *w)
{
    const long n = npts(M);
    for (int c = 0; c < 3; c++) {
        component(M, U, c, s);
        orc_grad_s(M, s, g + 3 * n * c);
    }
    const double *gu = g, *gv = g + 3 * n, *gw = g + 6 * n;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n; q++) {
        w[3 * q + 0] = gw[3 * q + 1] - gv[3 * q + 2]; /* dw/dy - dv/dz */
        w[3 * q + 1] = gu[3 * q + 2] - gw[3 * q + 0]; /* du/dz - dw/dx */
        w[3 * q + 2] = gv[3 * q + 0] - gu[3 * q + 1]; /* dv/dx - du/dy */
    }
}

/* mean of 1/2 |w|^2 over the unique nodes, summed in the order of the apps' energy loops */
static double half_sq_mean(const orc_mesh *M, const double *w)
{
    const int h = M->h;
    double e = 0.0;
    int n = 0;
    for (int i = h; i < M->n[0] - h - 1; i++)
        for (int j = h; j < M->n[1] - h - 1; j++)
            for (int k = h; k < M->n[2] - h - 1; k++) {
                const double *v = w + IDX(M, i, j, k) * 3;
                e += 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                n++;
            }
    return e / n;
}

/* One history row: the diagnostics of app/OT_Poisson/OT.cpp:132-176 (Ek, Em,
 * Jav, Jmax, omega, epsilon and Umax over the unique nodes, in its loop
 * order; J = ex::curl(B), omega from ex::curl(U) -- the Q1 stencil of
 * grad(vector) -- and epsilon = -mu omega^2 - eta Jav^2 from the means),
 * tools::CFL (src/Tools/Tools.cpp:9-41: cfl_y and cfl_z take std::max with
 * cfl_x, and keep only the last node's value), tools::maximum of div U and
 * div B (app/TG_Piosson/RKLoop.H:42-51, app/OT_Poisson/BEqn.H:46-54), plus
 * 1/2 <|curl U|^2> and 1/2 <|curl B|^2> with the central 6th-order curl. */
static void diag_row(const orc_mesh *M, const orc_run_desc *rd, int step, double t, const double *U,
                     const double *B, double *row, double *w1, double *w2, double *g9, double *s)
{
    const int h = M->h;
    const int mhd = rd->model == 1;
    const double mu = rd->nu, eta = mhd ? rd->eta : 0.0;
    row[0] = step + 1;
    row[1] = t;
    orc_curl(M, U, w1); /* omegav = ex::curl(U) */
    if (mhd) orc_curl(M, B, w2); else memset(w2, 0, sizeof(double) * 3 * npts(M)); /* J = ex::curl(B) */
    double Ek = 0.0, Em = 0.0, Jmax = 0.0, Umax = 0.0, Jav = 0.0, omega = 0.0;
    int n = 0;
    for (int i = h; i < M->n[0] - h - 1; i++)
        for (int j = h; j < M->n[1] - h - 1; j++)
            for (int k = h; k < M->n[2] - h - 1; k++) {
                const long p = IDX(M, i, j, k) * 3;
                const double *u = U + p, *J = w2 + p, *o = w1 + p;
                Ek += 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                if (mhd) {
                    const double *b = B + p;
                    Em += 0.5 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
                }
                const double jm = sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]);
                Jmax = Jmax < jm ? jm : Jmax; /* std::max(Jmax, .) */
                const double um = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                Umax = Umax < um ? um : Umax;
                omega += sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
                Jav += sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]);
                n++;
            }
    Ek /= n;
    Em /= n;
    Jav /= n;
    omega /= n;
    row[2] = Ek;
    row[3] = Em;
    row[6] = omega;
    row[7] = Jav;
    row[8] = Jmax;
    row[9] = -mu * (omega * omega) - eta * (Jav * Jav);
    row[10] = Umax;
    /* tools::CFL over [m/2, n - m/2) (duplicate nodes included) */
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for (int i = h; i < M->n[0] - h; i++)
        for (int j = h; j < M->n[1] - h; j++)
            for (int k = h; k < M->n[2] - h; k++) {
                const double *u = U + IDX(M, i, j, k) * 3;
                const double vx = u[0] * rd->dt / M->d[0], vy = u[1] * rd->dt / M->d[1], vz = u[2] * rd->dt / M->d[2];
                cx = cx < vx ? vx : cx;
                cy = cx < vy ? vy : cx;
                cz = cx < vz ? vz : cx;
            }
    row[11] = cx;
    row[12] = cy;
    row[13] = cz;
    orc_div_v(M, U, s);
    row[4] = orc_maximum(M, s);
    if (mhd) {
        orc_div_v(M, B, s);
        row[5] = orc_maximum(M, s);
    } else {
        row[5] = 0.0;
    }
    central_curl(M, U, s, g9, w1);
    row[14] = half_sq_mean(M, w1);
    if (mhd) {
        central_curl(M, B, s, g9, w1);
        row[15] = half_sq_mean(M, w1);
    } else {
        row[15] = 0.0;
    }
}

void orc_diag_row(const orc_mesh *M, const orc_run_desc *rd, int step, double t, const double *U, const double *B,
                  double *row)
{
    const long n = npts(M);
    double *mem = (double *)calloc((size_t)(n * 16), sizeof(double));
    if (!mem) return;
    diag_row(M, rd, step, t, U, B, row, mem, mem + 3 * n, mem + 6 * n, mem + 15 * n);
    free(mem);
}

/* one evaluation of dt*(RHS) of app/TG_Piosson/RKLoop.H:17-22 (model 0) or
 * app/OT_Poisson/UEqn.H:16-23 (model 1), with every Field operator of
 * src/Field/Field.hxx:617-1150 applied over all points in its order. */
static void u_rhs(const orc_mesh *M, const orc_run_desc *rd, const double *U, const double *B,
                  double *dU, double *t1, double *t2, double *s1, double *s2)
{
    const long n = npts(M);
    orc_div_vf(M, U, U, 3, t1);                               /* ex::div(U,U) */
    orc_lap(M, rd->nu, U, 3, t2);                             /* ex::laplacian(mu,U) */
#pragma omp parallel for schedule(static)
    for (long q = 0; q < 3 * n; q++) dU[q] = -t1[q] + t2[q];  /* -a + b */
    if (rd->model == 1) {
        orc_div_vf(M, B, B, 3, t1);                           /* + ex::div(B,B) */
#pragma omp parallel for schedule(static)
        for (long q = 0; q < 3 * n; q++) dU[q] = dU[q] + t1[q];
#pragma omp parallel for schedule(static)
        for (long p = 0; p < n; p++) {                        /* 0.5*(B&B) */
            const double *b = B + 3 * p;
            s1[p] = (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) * 0.5;
        }
        orc_grad_s(M, s1, t1);                                /* - ex::grad(...) */
#pragma omp parallel for schedule(static)
        for (long q = 0; q < 3 * n; q++) dU[q] = dU[q] - t1[q];
    }
    (void)s2;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < 3 * n; q++) dU[q] = dU[q] * rd->dt; /* time.dt() * (...) */
}

/* app/OT_Poisson/BEqn.H:72-78: dt*(-div(U,B) + div(B,U) + laplacian(eta,B)) */
static void b_rhs(const orc_mesh *M, const orc_run_desc *rd, const double *U, const double *B,
                  double *dB, double *t1, double *t2)
{
    const long n = npts(M);
    orc_div_vf(M, U, B, 3, t1);
    orc_div_vf(M, B, U, 3, t2);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < 3 * n; q++) dB[q] = -t1[q] + t2[q];
    orc_lap(M, rd->eta, B, 3, t1);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < 3 * n; q++) dB[q] = (dB[q] + t1[q]) * rd->dt;
}

/* x[q] = x[q] + y[q] * a */
static void axpy_(long n, double *x, const double *y, double a)
{
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n; q++) x[q] = x[q] + y[q] * a;
}

/* app/shearLayer/UEqn.H:14-38: RK4 weights used as stage coefficients,
 * Ustar = UOld + RK4[rk]*dU with the stage state U refreshed by a projection
 * after every stage (rhs div(Ustar)/dt/RK4c[rk], correction RK4c[rk]*dt*grad p) */
static const double RK4W[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0}; /* shearLayer.cpp:164 */
static const double RK4C[4] = {0.5, 0.5, 1.0, 1.0};                         /* settings::RK4c_ */

int orc_run(const orc_mesh *M, const orc_run_desc *rd, double *U, double *B, double *p,
            double *pB, double *hist)
{
    const long n = npts(M);
    const long v = 3 * n;
    double *mem = (double *)calloc((size_t)(v * 12 + n * 4), sizeof(double));
    if (!mem) return -1;
    double *UOld = mem, *Ustar = mem + v, *t1 = mem + 2 * v, *t2 = mem + 3 * v;
    double *dU[4] = {mem + 4 * v, mem + 5 * v, mem + 6 * v, mem + 7 * v};
    double *Bold = mem + 8 * v, *Bstar = mem + 9 * v, *t3 = mem + 10 * v, *t4 = mem + 11 * v;
    double *s1 = mem + 12 * v, *s2 = s1 + n, *s3 = s1 + 2 * n, *s4 = s1 + 3 * n;
    (void)t4;
    double t = 0.0;
    for (int step = 0; step < rd->nsteps; step++) {
        t += rd->dt;
        if (rd->rk_mode == 2) {
            /* ---- U equation: app/shearLayer/UEqn.H:1-54 (B frozen, BEqn.H not included) ---- */
            memcpy(UOld, U, sizeof(double) * v);
            for (int rk = 0; rk < 4; rk++) {
                u_rhs(M, rd, U, B, dU[0], t1, t2, s1, s2);
                memcpy(Ustar, UOld, sizeof(double) * v);
                axpy_(v, Ustar, dU[0], RK4W[rk]);
                orc_bc_apply(M, Ustar, 3, rd->bcU_type, rd->bcU_val);
                orc_div_v(M, Ustar, s3);
#pragma omp parallel for schedule(static)
                for (long q = 0; q < n; q++) s3[q] = s3[q] / rd->dt / RK4C[rk];
                orc_poisson_solve(M, s3, p);
                orc_bc_apply(M, p, 1, rd->bcp_type, rd->bcp_val);
                orc_grad_s(M, p, t1);
                const double cs = RK4C[rk] * rd->dt;
#pragma omp parallel for schedule(static)
                for (long q = 0; q < v; q++) U[q] = Ustar[q] - cs * t1[q];
                orc_bc_apply(M, U, 3, rd->bcU_type, rd->bcU_val);
            }
        } else {
        /* ---- U equation: app/TG_Piosson/RKLoop.H:1-38, app/OT_Poisson/UEqn.H:1-39 ---- */
        memcpy(UOld, U, sizeof(double) * v);
        for (int rk = 0; rk < 4; rk++) {
            u_rhs(M, rd, U, B, dU[rk], t1, t2, s1, s2);
            memcpy(Ustar, UOld, sizeof(double) * v);
            for (int j = 0; j <= rk; j++) axpy_(v, Ustar, dU[j], RK4A[rk][j]);
            if (rd->rk_mode == 1) {
                /* classical RK4: the stage state is refreshed, as the reference's own B loop does */
                memcpy(U, Ustar, sizeof(double) * v);
                orc_bc_apply(M, U, 3, rd->bcU_type, rd->bcU_val);
            }
        }
        orc_bc_apply(M, Ustar, 3, rd->bcU_type, rd->bcU_val);
        orc_div_v(M, Ustar, s3);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < n; q++) s3[q] = s3[q] / rd->dt;
        orc_poisson_solve(M, s3, p);
        orc_bc_apply(M, p, 1, rd->bcp_type, rd->bcp_val);
        orc_grad_s(M, p, t1);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < v; q++) U[q] = Ustar[q] - t1[q] * rd->dt;
        orc_bc_apply(M, U, 3, rd->bcU_type, rd->bcU_val);

        /* ---- B equation: app/OT_Poisson/BEqn.H:1-98 ---- */
        if (rd->model == 1) {
            memcpy(Bold, B, sizeof(double) * v);
            for (int rk = 0; rk < 4; rk++) {
                b_rhs(M, rd, U, B, dU[rk], t1, t2);
                memcpy(Bstar, Bold, sizeof(double) * v);
                for (int j = 0; j <= rk; j++) axpy_(v, Bstar, dU[j], RK4A[rk][j]);
                memcpy(B, Bstar, sizeof(double) * v);
                orc_bc_apply(M, B, 3, rd->bcB_type, rd->bcB_val);
            }
            orc_div_v(M, B, s3);
            orc_poisson_solve(M, s3, pB);
            orc_bc_apply(M, pB, 1, rd->bcpB_type, rd->bcpB_val);
            orc_grad_s(M, pB, t3);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < v; q++) B[q] -= t3[q];
            orc_bc_apply(M, B, 3, rd->bcB_type, rd->bcB_val);
        }
        }

        if (hist && rd->diag_every > 0 && ((step + 1) % rd->diag_every == 0 || step + 1 == rd->nsteps)) {
            /* dU[0..3] (4 vector fields, 12 npts) and s4 serve as the row's scratch */
            diag_row(M, rd, step, t, U, (rd->model == 1) ? B : NULL, hist + (long)step * ORC_HIST_COLS, dU[0], dU[1],
                     dU[2], s4);
        }
    }
    free(mem);
    return 0;
}
