// C++ caller of the adapter in include/nova/nova.hpp, written the way the
// reference's app/TG_Piosson/TG.cpp is: read a mesh file, set the
// Taylor-Green field on the interior nodes, correct the boundary conditions,
// then advance.  The whole RKLoop.H body runs as one nova::Advance call.
//
//   tg_driver <case-dir> <nsteps> <dt> <nu> <literal|classical> <out.bin>
//
// Writes U in the reference Field<vector> layout (float64) to out.bin and the
// diagnostics history to out.bin.hist.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "nova/nova.hpp"

int main(int argc, char **argv)
{
    if (argc < 7) {
        std::fprintf(stderr, "usage: tg_driver <case> <nsteps> <dt> <nu> <literal|classical> <out>\n");
        return 2;
    }
    const std::string zone = argv[1];
    const int nsteps = std::atoi(argv[2]);
    const double dt = std::atof(argv[3]);
    const double nu = std::atof(argv[4]);
    const bool classical = std::string(argv[5]) == "classical";
    try {
        nova::Mesh mesh(zone + "/mesh");
        nova::Field<nova::vector> U(mesh);
        const int h = mesh.m() / 2;
        for (int i = h; i < mesh.ni() - h; i++)
            for (int j = h; j < mesh.nj() - h; j++)
                for (int k = h; k < mesh.nk() - h; k++) {
                    const double x = (i - h) * mesh.dx(), y = (j - h) * mesh.dy(), z = (k - h) * mesh.dz();
                    U(i, j, k) = nova::vector(std::sin(x) * std::cos(y) * std::cos(z),
                                              -std::cos(x) * std::sin(y) * std::cos(z), 0.0);
                }
        U.correctBoundaryConditions();
        nova_run_desc rd{};
        rd.model = NOVA_MODEL_NS;
        rd.rk_mode = classical ? NOVA_RK_CLASSICAL : NOVA_RK_LITERAL;
        rd.precision = NOVA_F64;
        rd.diag_every = 1;
        rd.dt = dt;
        rd.nu = nu;
        nova::Advance adv(mesh, rd);
        adv.setU(U);
        std::vector<double> hist = adv.run(nsteps);
        adv.getU(U);
        FILE *fp = std::fopen(argv[6], "wb");
        std::fwrite(U.ptr(), sizeof(nova::vector), (size_t)mesh.ni() * mesh.nj() * mesh.nk(), fp);
        std::fclose(fp);
        fp = std::fopen((std::string(argv[6]) + ".hist").c_str(), "wb");
        std::fwrite(hist.data(), sizeof(double), hist.size(), fp);
        std::fclose(fp);
        // operator-level drop-in: max|div U| through ex::div + tools::maximum
        std::printf("maxdivU %.17g\n", nova::tools::maximum(nova::ex::div(U)));
    } catch (const nova::Error &e) {
        std::fprintf(stderr, "nova error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    return 0;
}
