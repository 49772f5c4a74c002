// Launchers of the weakly-compressible loops (nova_wc.cu).
#pragma once

#include "nova_gpu.h"
#include "nova_internal.cuh"

namespace nova {

enum WcLoop { WC_LOOP_U = 0, WC_LOOP_RHO = 1, WC_LOOP_T = 2 };

struct WcArgs {
    const double *Y;    // halo'd stage state of the loop's quantity (U: 3 components)
    const double *U;    // U, frozen during the rho and T loops
    const double *rho;  // rho, frozen during the U and T loops
    const double *T;    // T of the buoyancy term (U loop, shear case)
    const double *Q0;   // the loop's value at the start of the step (stages 1-3)
    double *acc;        // RK accumulator of rho*q (rho itself in the rho loop)
    double *Ynext;      // next stage state, or the updated field after stage 3
    double *p;          // read (halo'd) by the U loop, written from the EOS by the last rho stage
    double dt, visc, eos_k;
    double g[3];
};

void launch_wc_stage(int loop, int stage, int wc_case, bool stretch, const Geo &g, const Coef<double> &co,
                     const double *ia, const double *corr2, const WcArgs &a, cudaStream_t st);
void launch_wc_hydrostatic(const Geo &g, double dz, double gz, double rho0, double K, const double *T, double *p,
                           double *rho, cudaStream_t st);

}  // namespace nova
