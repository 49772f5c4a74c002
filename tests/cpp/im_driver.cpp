// C++ caller of the implicit operators through include/nova/nova.hpp, written
// the way a reference app uses src/im: an implicit Helmholtz step
// (im::laplacian(mu, x) - c) == f, then solve on x.
//
//   im_driver <case-dir> <mu> <c> <x.bin> <f.bin> <tol> <maxits> <out.bin>
//
// x.bin and f.bin hold Field<scalar> values in the reference layout
// (ghosted, float64); out.bin receives x after the solve in the same layout.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>

#include "nova/nova.hpp"

static bool read_field(const std::string &path, nova::Field<nova::scalar> &f)
{
    std::ifstream in(path, std::ios::binary);
    const size_t n = (size_t)f.ni() * f.nj() * f.nk();
    in.read(reinterpret_cast<char *>(f.ptr()), (std::streamsize)(n * sizeof(double)));
    return (size_t)in.gcount() == n * sizeof(double);
}

int main(int argc, char **argv)
{
    if (argc < 9) {
        std::fprintf(stderr, "usage: im_driver <case> <mu> <c> <x> <f> <tol> <maxits> <out>\n");
        return 2;
    }
    const std::string zone = argv[1];
    const double mu = std::atof(argv[2]), c = std::atof(argv[3]), tol = std::atof(argv[6]);
    const int maxits = std::atoi(argv[7]);
    try {
        nova::Mesh mesh(zone + "/mesh");
        auto x = std::make_shared<nova::Field<nova::scalar>>(mesh);
        auto f = std::make_shared<nova::Field<nova::scalar>>(mesh);
        if (!read_field(argv[4], *x) || !read_field(argv[5], *f)) {
            std::fprintf(stderr, "short read of x or f\n");
            return 1;
        }
        x->correctBoundaryConditions();
        auto M = nova::im::laplacian(mu, x);
        M->ap() -= c;
        auto S = (M == f);
        S->solve(tol, maxits);
        std::printf("%.17g\n", S->residual());
        std::ofstream out(argv[8], std::ios::binary);
        out.write(reinterpret_cast<const char *>(x->ptr()),
                  (std::streamsize)((size_t)x->ni() * x->nj() * x->nk() * sizeof(double)));
    } catch (const nova::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
