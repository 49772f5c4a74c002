// Launchers of nova_ops.cu (projection, diagnostics, operators, layout).
#pragma once

#include "nova_internal.cuh"

namespace nova {

enum OpKind {
    OP_GRAD_S = 0, OP_GRAD_V = 1, OP_DIV_V = 2, OP_DIV_VF = 3, OP_LAP = 4, OP_CURL = 5,
    OP_DIV_T = 6,   // div(tensor) (a: 9 comps) or div(symmTensor) (a: 6 comps)
    OP_DIV_ST = 7,  // div(scalar a, tensor b)
    OP_LAP_F = 8    // laplacian(Field nu = a, f = b with nc comps)
};

// wall-node overwrite per component: type 1 = Neumann, 2 = Dirichlet (0 = none)
struct WallFix {
    int on, nc;
    double dy;
    int type[2][9];   // [side: 0 south, 1 north][comp]
    double val[2][9];
};

// ex: with a non-null error word (ex.err) the TMA-pipelined kernels of
// nova_proj_tma.cu run where the mesh fits them (proj_tma_fits: N2 % 32 == 0,
// N1 >= 32 and, with periodic y, N1 % 16 == 0; walls in y when the field's
// ghost BCs are on) and StageExec::impl is not STAGE_MARCH; otherwise the
// tiled march kernels.  Returns
// cudaErrorInvalidValue when a tensor map cannot be encoded.
cudaError_t launch_div_proj(int h, const Geo &g, const Walls<double> &wl, const Coef<double> &co, const double *ia,
                            const double *U64, const float *hi, const float *lo, double divisor, double *rhs,
                            cudaStream_t st, const StageExec &ex = StageExec{STAGE_MARCH, nullptr});
// ny: y extent of the spectrum (the unique y nodes of the transform)
void launch_scale(const Geo &g, int ny, void *spec, const double *kx2, const double *ky2, const double *kz2,
                  double invN3, cudaStream_t st);
// the i direction of the periodic spectral solve fused with the scale
// (nova_pois_i.cu): in place on the half spectrum [i][j][kz] of the 2-D
// (j, k) transforms; twN = W_N0^m, m = 0..N0-1 (interleaved re, im)
bool pois_i_fits(const Geo &g);
// the (j, k) plane transforms in one pass each (nova_fft2d.cu, clusters of
// eight CTAs): periodic y, N1 = N2 = 256, and the device can hold a cluster;
// x real [i][j][k] <-> spec [i][j][kz] (kz < 129), unnormalised like cuFFT's
// batched 2-D D2Z / Z2D; tw256 = W_256^m (interleaved re, im)
bool fft2_fits(const Geo &g);
void launch_fft2_fwd(const Geo &g, const double *x, void *spec, const double *tw256, cudaStream_t st);
void launch_fft2_inv(const Geo &g, const void *spec, double *x, const double *tw256, cudaStream_t st);
// the wall Poisson's y direction in DCT mode (nova_pois_dct.cu): in place on
// the half spectrum [i][j][kz] (j = 0..256) of the batched 2-D (i, k) D2Z of
// the stored rows, per (i, kz) column DCT-I along j, the scale
// -invN3 / (kx'^2 + ky'^2 + kz'^2) (ky2e: the even extension's table) and
// DCT-I back; walls in y with N[1] = 256, N2 % 16 == 0, N0 % 8 == 0.
// tw256 = W_256^m, t512 = W_512^n (n < 256), interleaved (re, im)
bool pois_dct_fits(const Geo &g, int ny);
void launch_pois_dct(const Geo &g, void *spec, const double *tw256, const double *t512, const double *kx2,
                     const double *ky2e, const double *kz2, double invN3, cudaStream_t st);

// err: the pipeline's error word (a bounded wait that gives up raises it);
// null runs the register kernel k_pois_i, else N0 = 256 meshes with
// N2 % 16 == 0 and N1 % 8 == 0 run the TMA-fed k_pois_tma
void launch_pois_i(const Geo &g, int ny, void *spec, const double *twN, const double *kx2, const double *ky2,
                   const double *kz2, double invN3, int *err, cudaStream_t st);
cudaError_t launch_correct(int h, const Geo &g, const Walls<double> &pw, const Coef<double> &co, const double *ia,
                           const double *p, double s, const double *Us64, double *U64, const float *Ushi,
                           const float *Uslo, float *hi, float *lo, cudaStream_t st,
                           const StageExec &ex = StageExec{STAGE_MARCH, nullptr});
bool proj_tma_fits(const Geo &g, bool wl_on);
cudaError_t launch_div_tma(const Geo &g, const Coef<double> &co, const Walls<double> &wl, const double *ia,
                           const double *U64, const float *hi, const float *lo, double divisor, double *rhs, int *err,
                           cudaStream_t st);
cudaError_t launch_correct_tma(const Geo &g, const Coef<double> &co, const Walls<double> &pw, const double *ia,
                               const double *p, double s, const double *Us64, double *U64, const float *Ushi,
                               const float *Uslo, float *hi, float *lo, int *err, cudaStream_t st);
int diag_blocks(const Geo &g);
// implicit operators (nova_im.cu): coef = 8 FP64 fields [al0..al5 | ap | b]
void launch_fdm_laplacian(const Geo &g, const Coef<double> &co, const double *ia, const double *corr2, int h,
                          double mu, double dx, double dy, double dz, const double *x, double *hoa, double *coef,
                          cudaStream_t st);
// mode 0: a += alpha b, 1: a *= b, 2: a *= alpha (all eight fields)
void launch_fdm_algebra(const Geo &g, int mode, double alpha, double *a, const double *b, cudaStream_t st);
// mode 0: b += v f, 1: ap += v, 2: relax with urf = v (f = x)
void launch_fdm_point(const Geo &g, int mode, double v, double *coef, const double *f, cudaStream_t st);
void launch_fdm_setref(const Geo &g, double *coef, long long n, double val, cudaStream_t st);
void launch_fdm_residual(const Geo &g, const double *coef, const double *x, double *part, int nb, double *out,
                         cudaStream_t st);
// the factors of the periodic tridiagonal line systems along axis: fac 4 N3
// doubles, ls 2 x (lines along axis) doubles
void launch_fdm_factor(int axis, const Geo &g, const double *coef, double *fac, double *ls, cudaStream_t st);
// one sweep of line solves along axis with those factors, xin -> xout (distinct)
void launch_fdm_line(int axis, const Geo &g, const double *coef, const double *fac, const double *ls,
                     const double *xin, double *xout, cudaStream_t st);
// the history row from nb blocks of partials (kDiagParts per block)
void launch_diag_final(const double *part, int nb, const DiagFinal &fin, double *row, int *flag, cudaStream_t st);
// the physical parameters of a history row (epsilon, tools::CFL); zeros where
// only the energies are wanted
struct DiagPhys {
    double nu, eta, dt, dx, dy, dz;
};
// the DiagFinal of a row of the state (U64 or Uhi/Ulo) on mesh g
DiagFinal diag_final_of(const Geo &g, const DiagPhys &ph, double step, double time, const double *U64,
                        const float *Uhi, const float *Ulo);
// the history row of the state U (and B where hasB) by the tiled diagnostics kernel
void launch_diag(int h, const Geo &g, const Walls<double> &wl, const Coef<double> &co, const double *ia,
                 const double *U64, const float *Uhi, const float *Ulo, const double *B64, const float *Bhi,
                 const float *Blo, int hasB, double *part, double step, double time, double *row, int *flag,
                 cudaStream_t st, const DiagPhys &ph = DiagPhys{0, 0, 0, 1, 1, 1});
void launch_maxabs(const Geo &g, const double *s, double *part, double *out, cudaStream_t st);
void launch_op(int op, int h, const Geo &g, const Walls<double> &wa, const Walls<double> &wb, const Coef<double> &co,
               const double *ia, const double *corr2, const double *a, const double *b, int nc, double nu, double *out,
               cudaStream_t st);
void launch_aos_to_soa(const Geo &g, int h, const int n[3], int nc, const double *aos, double *d64, float *hi,
                       float *lo, cudaStream_t st);
void launch_soa_to_aos(const Geo &g, const Walls<double> &wl, int h, const int n[3], int nc, const double *d64,
                       const float *hi, const float *lo, double *aos, cudaStream_t st);
void launch_wall_fix64(const Geo &g, const WallFix &wf, double *f, cudaStream_t st);
void launch_wall_fix32(const Geo &g, const WallFix &wf, float *f, cudaStream_t st);
void launch_wall_fix_split(const Geo &g, const WallFix &wf, float *hi, float *lo, cudaStream_t st);
void launch_even_extend(const Geo &g, int ny, const double *rhs, double *ext, cudaStream_t st);
void launch_restrict_rows(const Geo &g, int ny, const double *ext, double *p, cudaStream_t st);
// allocation-free max|s|: one block per kMaxabsChunk nodes, one partial each
constexpr int kMaxabsChunk = 16384;
constexpr int kMaxabsStaticParts = 8192;
// address of this device's static scratch (kMaxabsStaticParts partials + the result)
cudaError_t maxabs_noalloc_scratch(double **scratch);
void launch_maxabs_noalloc(long long n, const double *s, double *scratch, cudaStream_t st);
void launch_split(long long n, const double *x, float *hi, float *lo, cudaStream_t st);
void launch_join(long long n, const float *hi, const float *lo, double *x, cudaStream_t st);

}  // namespace nova
