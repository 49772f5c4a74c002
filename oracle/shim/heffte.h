/* TEST INFRASTRUCTURE ONLY: single-rank stand-in for the heFFTe API names the
 * reference's src/poisson/poisson.cpp uses (box3d, fft3d<backend::fftw>,
 * forward/backward unscaled, size_inbox/outbox/workspace, nullify_executor).
 * The transforms run the oracle's own FFT (oracle/orc_fft.c) on the full box,
 * first index fastest.  fft3d<backend::fftw_cos1> exists so poisson.cpp
 * compiles; its transforms are never used by the reference's apps and abort. */
#ifndef ORC_SHIM_HEFFTE_H
#define ORC_SHIM_HEFFTE_H
#include <array>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "mpi.h"
#include "../orc_fft.h"

inline void fftw_free(void *) {}

namespace heffte {
template <typename index = int> struct box3d {
    std::array<index, 3> low, high;
    box3d(std::array<index, 3> lo, std::array<index, 3> hi) : low(lo), high(hi) {}
    index size(int a) const { return high[a] - low[a] + 1; }
    long count() const { return (long)size(0) * size(1) * size(2); }
};
namespace backend {
struct fftw {};
struct fftw_cos1 {};
}

template <typename tag, typename index = int> class fft3d {
    box3d<index> in_;
    bool active_[3] = {true, true, true};
    void run(orc_cplx *d, int sign) const
    {
        int n[3] = {(int)in_.size(0), (int)in_.size(1), (int)in_.size(2)};
        if (active_[0] && active_[1] && active_[2]) {
            orc_fft3d(n, d, sign);
            return;
        }
        const long n0 = n[0], n1 = n[1], n2 = n[2];
        if (active_[0])
            for (long k = 0; k < n2; k++)
                for (long j = 0; j < n1; j++) orc_fft1d(n[0], d + n0 * (j + n1 * k), 1, sign);
        if (active_[1])
            for (long k = 0; k < n2; k++)
                for (long i = 0; i < n0; i++) orc_fft1d(n[1], d + i + n0 * n1 * k, n0, sign);
        if (active_[2])
            for (long j = 0; j < n1; j++)
                for (long i = 0; i < n0; i++) orc_fft1d(n[2], d + i + n0 * j, n0 * n1, sign);
    }
public:
    fft3d(box3d<index> inbox, box3d<index>, MPI_Comm) : in_(inbox) {}
    long size_inbox() const { return in_.count(); }
    long size_outbox() const { return in_.count(); }
    long size_workspace() const { return in_.count(); }
    void nullify_executor(int axis) { active_[axis] = false; }
    void forward(const double *in, std::complex<double> *out) const
    {
        long n = in_.count();
        std::vector<orc_cplx> d(n);
        for (long q = 0; q < n; q++) { d[q].re = in[q]; d[q].im = 0.0; }
        run(d.data(), -1);
        std::memcpy((void *)out, d.data(), sizeof(orc_cplx) * n);
    }
    void forward(const std::complex<double> *in, std::complex<double> *out) const
    {
        long n = in_.count();
        std::vector<orc_cplx> d(n);
        std::memcpy(d.data(), (const void *)in, sizeof(orc_cplx) * n);
        run(d.data(), -1);
        std::memcpy((void *)out, d.data(), sizeof(orc_cplx) * n);
    }
    void backward(const std::complex<double> *in, double *out) const
    {
        long n = in_.count();
        std::vector<orc_cplx> d(n);
        std::memcpy(d.data(), (const void *)in, sizeof(orc_cplx) * n);
        run(d.data(), +1);
        for (long q = 0; q < n; q++) out[q] = d[q].re;
    }
    void backward(const std::complex<double> *in, std::complex<double> *out) const
    {
        long n = in_.count();
        std::vector<orc_cplx> d(n);
        std::memcpy(d.data(), (const void *)in, sizeof(orc_cplx) * n);
        run(d.data(), +1);
        std::memcpy((void *)out, d.data(), sizeof(orc_cplx) * n);
    }
    /* real-to-real overloads of the cosine backend: unused by every app */
    void forward(const double *, double *) const { std::abort(); }
    void backward(const double *, double *, double *) const { std::abort(); }
    void backward(const double *, double *) const { std::abort(); }
};
} // namespace heffte
#endif
