/*
 * TEST INFRASTRUCTURE ONLY -- driver for the reference compiled in place
 * (oracle/Makefile, target _ref/nova_ref).  It builds the reference's Mesh,
 * Field, poisson objects exactly as app/TG_Piosson/TG.cpp and
 * app/OT_Poisson/OT.cpp do, then runs the reference's own loop bodies
 * (app/TG_Piosson/RKLoop.H, app/OT_Poisson/UEqn.H + BEqn.H) for the literal
 * mode, the same loop with the stage state refreshed for the classical RK4
 * mode, or app/shearLayer/UEqn.H (shear mode).  Each step's history row is
 * the diagnostics of app/OT_Poisson/OT.cpp:132-176 and tools::CFL.  I/O is raw little-endian float64 in the Field<T> layout; the wall
 * time of each step's loop body goes to <out>_time.txt, one line per step.
 *
 *   nova_ref run <case> <ns|mhd> <literal|classical|shear> <nsteps> <dt> <nu> <eta> <U.bin> <B.bin|-> <out>
 *   nova_ref ops <case> <nu> <U.bin> <s.bin> <out>
 *   nova_ref wc <case> <tg|shear> <nsteps> <dt> <mu> <ka> <c> <rho0> <gz> <U.bin> <rho.bin> <p.bin> <T.bin|-> <out>
 *   nova_ref wcinit <case> <c> <rho0> <gz> <T.bin> <out>
 *   nova_ref ensight <case> <nsteps> <dt> <U.bin> <p.bin> <dir>
 *   nova_ref ops2 <case> <T.bin> <S.bin> <s.bin> <nu.bin> <U.bin> <out>
 *   nova_ref im <case> <mu> <c> <x.bin> <f.bin> <tol> <maxits> <out>
 *   (any may end with the reference's `-m <order>` option)
 *
 * `wc` runs the compressible loop bodies: app/TG (rhoEqn.H, pEqn.H, UEqn.H in
 * the order of app/TG/TG.cpp:73-75) or app/shearLayerWC (UEqn.H, rhoEqn.H,
 * pEqn.H, TEqn.H in the order of shearLayer.cpp:197-200).  `wcinit` runs the
 * weakly-compressible initialisation of shearLayer.cpp:114-155 (pEqn.H on
 * rho = rho0, hydrostaticP.H, rho from the EOS) for a given T.
 *
 * <case> holds `mesh` and the BC files (UBC, pBC, BBC, pBBC, rhoBC, TBC).
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "Field/Field.h"
#include "BC/BC.h"
#include "Time/Time.h"
#include "Tools/Tools.h"
#include "Types/vector/vector.h"
#include "ex/curl/curl.h"
#include "ex/div/div.h"
#include "ex/grad/grad.h"
#include "ex/laplacian/laplacian.h"
#include "im/laplacian/laplacian.h" /* after ex/laplacian, which it uses */
#include "parallelCom/parallelCom.h"
#include "poisson/poisson.h"
#include "settings/settings.h"

template <class T> static void load(Field<T> &f, const std::string &path)
{
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
    size_t n = (size_t)f.ni() * f.nj() * f.nk();
    if (std::fread(f.ptr(), sizeof(T), n, fp) != n) { std::fprintf(stderr, "short read %s\n", path.c_str()); std::exit(2); }
    std::fclose(fp);
}

template <class T> static void save(const Field<T> &f, const std::string &path)
{
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(2); }
    size_t n = (size_t)f.ni() * f.nj() * f.nk();
    std::fwrite(f.ptr(), sizeof(T), n, fp);
    std::fclose(fp);
}

/* tools::CFL (src/Tools/Tools.cpp:9-41) prints its three values; run it with
 * std::cout redirected and at full precision, and read them back */
static void cfl_of(const Field<vector> &U, const Mesh &mesh, double out[3])
{
    std::ostringstream os;
    os.precision(17);
    std::streambuf *old = std::cout.rdbuf(os.rdbuf());
    const std::streamsize prec = std::cout.precision(17);
    tools::CFL(U, mesh);
    std::cout.precision(prec);
    std::cout.rdbuf(old);
    const std::string txt = os.str();
    const char *keys[3] = {"CFL x:", "CFL y:", "CFL z:"};
    for (int a = 0; a < 3; a++) {
        const size_t at = txt.find(keys[a]);
        out[a] = at == std::string::npos ? std::nan("") : std::strtod(txt.c_str() + at + 6, nullptr);
    }
}

/* 1/2 <|curl V|^2> over the unique nodes with the central curl built from the
 * reference's ex::grad of each component (the ghosts of V copied along) */
static double central_enstrophy(Mesh &mesh, const Field<vector> &V)
{
    std::shared_ptr<Field<vector> > g[3];
    for (int c = 0; c < 3; c++) {
        Field<scalar> s(mesh, 0, "p");
        for (int i = 0; i < mesh.ni(); i++)
            for (int j = 0; j < mesh.nj(); j++)
                for (int k = 0; k < mesh.nk(); k++) s(i, j, k) = V(i, j, k)[c];
        g[c] = ex::grad(s);
    }
    scalar e = 0.0;
    int n = 0;
    for (int i = settings::m() / 2; i < mesh.ni() - settings::m() / 2 - 1; i++)
        for (int j = settings::m() / 2; j < mesh.nj() - settings::m() / 2 - 1; j++)
            for (int k = settings::m() / 2; k < mesh.nk() - settings::m() / 2 - 1; k++) {
                const scalar wx = (*g[2])(i, j, k).y() - (*g[1])(i, j, k).z();
                const scalar wy = (*g[0])(i, j, k).z() - (*g[2])(i, j, k).x();
                const scalar wz = (*g[1])(i, j, k).x() - (*g[0])(i, j, k).y();
                e += 0.5 * (wx * wx + wy * wy + wz * wz);
                n++;
            }
    return e / n;
}

/* The history row of a step: the diagnostics loop of app/OT_Poisson/OT.cpp:132-176
 * (omegav = ex::curl(U), J = ex::curl(B)), tools::CFL, tools::maximum of the
 * divergences, and the central-curl enstrophies.  Columns as ORC_HIST_COLS. */
static void hist_row(Mesh &mesh, const Time &time, int step, bool mhd, scalar mu, scalar eta,
                     Field<vector> &U, Field<vector> &B, double row[16])
{
    for (int q = 0; q < 16; q++) row[q] = 0.0;
    row[0] = double(step + 1);
    row[1] = time.curTime();
    auto omegav = ex::curl(U);
    auto Jp = ex::curl(B);
    const Field<vector> &J = *Jp;
    scalar Ek = 0.0, Em = 0.0, Jmax = 0.0, Umax = 0.0, Jav = 0.0, omega = 0.0;
    int n = 0;
    for (int i = settings::m() / 2; i < mesh.ni() - settings::m() / 2 - 1; i++)
        for (int j = settings::m() / 2; j < mesh.nj() - settings::m() / 2 - 1; j++)
            for (int k = settings::m() / 2; k < mesh.nk() - settings::m() / 2 - 1; k++) {
                Ek += 0.5 * (U(i, j, k).x() * U(i, j, k).x() + U(i, j, k).y() * U(i, j, k).y() + U(i, j, k).z() * U(i, j, k).z());
                Em += 0.5 * (B(i, j, k).x() * B(i, j, k).x() + B(i, j, k).y() * B(i, j, k).y() + B(i, j, k).z() * B(i, j, k).z());
                Jmax = std::max(Jmax, sqrt(J(i, j, k).x() * J(i, j, k).x() + J(i, j, k).y() * J(i, j, k).y() + J(i, j, k).z() * J(i, j, k).z()));
                Umax = std::max(Umax, sqrt(U(i, j, k).x() * U(i, j, k).x() + U(i, j, k).y() * U(i, j, k).y() + U(i, j, k).z() * U(i, j, k).z()));
                omega += sqrt((*omegav)(i, j, k).x() * (*omegav)(i, j, k).x() + (*omegav)(i, j, k).y() * (*omegav)(i, j, k).y()
                              + (*omegav)(i, j, k).z() * (*omegav)(i, j, k).z());
                Jav += sqrt(J(i, j, k).x() * J(i, j, k).x() + J(i, j, k).y() * J(i, j, k).y() + J(i, j, k).z() * J(i, j, k).z());
                n++;
            }
    Ek /= n;
    Em /= n;
    Jav /= n;
    omega /= n;
    row[2] = Ek;
    row[3] = mhd ? Em : 0.0;
    row[6] = omega;
    row[7] = Jav;
    row[8] = Jmax;
    row[9] = -mu * (omega * omega) - (mhd ? eta : 0.0) * (Jav * Jav);
    row[10] = Umax;
    cfl_of(U, mesh, row + 11);
    {
        auto d = ex::div(U);
        row[4] = tools::maximum(d);
    }
    if (mhd) {
        auto d = ex::div(B);
        row[5] = tools::maximum(d);
    }
    row[14] = central_enstrophy(mesh, U);
    if (mhd) row[15] = central_enstrophy(mesh, B);
}

/* app/TG_Piosson/TG.cpp:148-166 */
static double ek_mean(const Mesh &mesh, const Field<vector> &U)
{
    scalar Ek = 0.0;
    int n = 0;
    for (int i = settings::m() / 2; i < mesh.ni() - settings::m() / 2 - 1; i++)
        for (int j = settings::m() / 2; j < mesh.nj() - settings::m() / 2 - 1; j++)
            for (int k = settings::m() / 2; k < mesh.nk() - settings::m() / 2 - 1; k++) {
                Ek += 0.5 * (U(i, j, k).x() * U(i, j, k).x() + U(i, j, k).y() * U(i, j, k).y()
                             + U(i, j, k).z() * U(i, j, k).z());
                n++;
            }
    return Ek / n;
}

static int run(int argc, char **argv)
{
    if (argc < 12) { std::fprintf(stderr, "usage: run <case> <ns|mhd> <literal|classical|shear> <nsteps> <dt> <nu> <eta> <U> <B|-> <out>\n"); return 2; }
    settings::zoneName() = argv[2];
    const bool mhd = std::string(argv[3]) == "mhd";
    const bool classical = std::string(argv[4]) == "classical";
    const bool shear = std::string(argv[4]) == "shear";
    scalar RK4[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0}; /* app/shearLayer/shearLayer.cpp:164 */
    const int nsteps = std::atoi(argv[5]);
    const double dt = std::atof(argv[6]);
    const scalar mu = std::atof(argv[7]);
    const scalar eta = std::atof(argv[8]);
    const std::string inU = argv[9], inB = argv[10], out = argv[11];

    Time time(dt, dt * (nsteps + 0.5), 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);

    Field<vector> U(mesh, vector(0, 0, 0), "U");
    Field<vector> Ustar(mesh, vector(0, 0, 0), "U");
    Field<vector> B(mesh, vector(0, 0, 0), "B");
    Field<vector> Bstar(mesh, vector(0, 0, 0), "B");
    Field<vector> J(mesh, vector(0, 0, 0), "B");
    std::shared_ptr<Field<scalar> > p_ptr(std::make_shared<Field<scalar> >(mesh, 0, "p"));
    auto &p = (*p_ptr);
    std::shared_ptr<Field<scalar> > pB_ptr(std::make_shared<Field<scalar> >(mesh, 0, "pB"));
    auto &pB = (*pB_ptr);
    /* never destroyed: poisson::~poisson frees memory it does not own */
    poisson &pEqn = *new poisson(p_ptr);
    poisson &pBEqn = *new poisson(pB_ptr);

    load(U, inU);
    U.correctBoundaryConditions();
    p.correctBoundaryConditions();
    if (mhd) {
        load(B, inB);
        B.correctBoundaryConditions();
        pB.correctBoundaryConditions();
    }

    std::vector<double> hist, step_s;
    for (int step = 0; step < nsteps; step++) {
        const auto t0 = std::chrono::steady_clock::now();
        time++;
        if (shear) {
            /* app/shearLayer: the U loop only (BEqn.H is not included there), B frozen; with
             * the ns model B stays zero and its terms add zeros */
#include "shearLayer/UEqn.H"
        } else if (!mhd && !classical) {
#include "TG_Piosson/RKLoop.H"
        } else if (mhd && !classical) {
#include "OT_Poisson/UEqn.H"
#include "OT_Poisson/BEqn.H"
        } else {
            /* RKLoop.H / UEqn.H with U = Ustar refreshed per stage (the pattern of OT_Poisson/BEqn.H:86-87) */
            std::array<std::shared_ptr<Field<vector> >, 4> dU;
            for (int i = 0; i < 4; i++) {
                reuseTmp<vector> dUt(mesh);
                dU[i] = dUt();
            }
            reuseTmp<vector> UOldt(mesh);
            std::shared_ptr<Field<vector> > UOld(UOldt());
            *UOld = U;
            for (int rk = 0; rk < 4; rk++) {
                if (mhd)
                    dU[rk] = time.dt() * (-ex::div(U, U) + ex::laplacian(mu, U) + ex::div(B, B) - ex::grad(0.5 * (B & B)));
                else
                    dU[rk] = time.dt() * (-ex::div(U, U) + ex::laplacian(mu, U));
                Ustar = UOld;
                for (int j = 0; j <= rk; j++) Ustar = Ustar + settings::RK4a()[rk][j] * dU[j];
                U = Ustar;
                U.correctBoundaryConditions();
            }
            Ustar.correctBoundaryConditions();
            pEqn.rhs(ex::div(Ustar) / time.dt());
            pEqn.solve();
            p.correctBoundaryConditions();
            U = Ustar - time.dt() * ex::grad(p);
            U.correctBoundaryConditions();
            if (mhd) {
#include "OT_Poisson/BEqn.H"
            }
        }
        step_s.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        double row[16];
        hist_row(mesh, time, step, mhd, mu, eta, U, B, row);
        hist.insert(hist.end(), row, row + 16);
    }

    save(U, out + "_U.bin");
    save(p, out + "_p.bin");
    if (mhd) {
        save(B, out + "_B.bin");
        save(pB, out + "_pB.bin");
    }
    FILE *fp = std::fopen((out + "_hist.bin").c_str(), "wb");
    std::fwrite(hist.data(), sizeof(double), hist.size(), fp);
    std::fclose(fp);
    /* wall time of each time-step loop body (diagnostics and I/O excluded) */
    fp = std::fopen((out + "_time.txt").c_str(), "w");
    for (double t : step_s) std::fprintf(fp, "%.9f\n", t);
    std::fclose(fp);
    return 0;
}

static int ops(int argc, char **argv)
{
    if (argc < 7) { std::fprintf(stderr, "usage: ops <case> <nu> <U> <s> <out>\n"); return 2; }
    settings::zoneName() = argv[2];
    const scalar nu = std::atof(argv[3]);
    const std::string out = argv[6];
    Time time(0.01, 1.0, 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    Field<vector> U(mesh, vector(0, 0, 0), "U");
    std::shared_ptr<Field<scalar> > s_ptr(std::make_shared<Field<scalar> >(mesh, 0, "p"));
    auto &s = *s_ptr;
    std::shared_ptr<Field<scalar> > p_ptr(std::make_shared<Field<scalar> >(mesh, 0, "p"));
    poisson &pEqn = *new poisson(p_ptr);
    load(U, argv[4]);
    load(s, argv[5]);

    save(*ex::grad(s), out + "_grad_s.bin");
    save(*ex::div(U), out + "_div_v.bin");
    save(*ex::div(U, U), out + "_div_vv.bin");
    save(*ex::div(U, s), out + "_div_vs.bin");
    save(*ex::laplacian(nu, U), out + "_lap_v.bin");
    save(*ex::laplacian(nu, s), out + "_lap_s.bin");
    save(*ex::curl(U), out + "_curl.bin");
    pEqn.rhs(s_ptr);
    pEqn.solve();
    save(*p_ptr, out + "_poisson.bin");
    return 0;
}

/* app/TG/TG.cpp:91-109 and the reference's max|div U| */
static void wc_hist(std::vector<double> &hist, int step, const Mesh &mesh, const Time &time, Field<vector> &U)
{
    double row[6] = {double(step + 1), time.curTime(), ek_mean(mesh, U), 0.0, 0.0, 0.0};
    auto d = ex::div(U);
    row[4] = tools::maximum(d);
    hist.insert(hist.end(), row, row + 6);
}

static int wc(int argc, char **argv)
{
    if (argc < 16) {
        std::fprintf(stderr, "usage: wc <case> <tg|shear> <nsteps> <dt> <mu> <ka> <c> <rho0> <gz> <U> <rho> <p> <T|-> <out>\n");
        return 2;
    }
    settings::zoneName() = argv[2];
    const bool tg = std::string(argv[3]) == "tg";
    const int nsteps = std::atoi(argv[4]);
    const double dt = std::atof(argv[5]);
    const scalar mu = std::atof(argv[6]);
    const scalar ka = std::atof(argv[7]);
    const scalar c = std::atof(argv[8]);
    const scalar rho0 = std::atof(argv[9]);
    vector g(0, 0, std::atof(argv[10]));
    const std::string inT = argv[14], out = argv[15];
    scalar RK4[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

    Time time(dt, dt * (nsteps + 0.5), 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    Field<vector> U(mesh, vector(0, 0, 0), "U");
    Field<scalar> rho(mesh, rho0, "rho");
    Field<scalar> p(mesh, 0, "p");
    Field<scalar> T(mesh, 0, "T");
    load(U, argv[11]);
    load(rho, argv[12]);
    load(p, argv[13]);
    if (inT != "-") load(T, inT);
    U.correctBoundaryConditions();
    p.correctBoundaryConditions();
    rho.correctBoundaryConditions();
    T.correctBoundaryConditions();

    std::vector<double> hist;
    for (int step = 0; step < nsteps; step++) {
        time++;
        if (tg) {
#include "TG/rhoEqn.H"
#include "TG/pEqn.H"
#include "TG/UEqn.H"
        } else {
#include "shearLayerWC/UEqn.H"
#include "shearLayerWC/rhoEqn.H"
#include "shearLayerWC/pEqn.H"
#include "shearLayerWC/TEqn.H"
        }
        wc_hist(hist, step, mesh, time, U);
    }
    save(U, out + "_U.bin");
    save(rho, out + "_rho.bin");
    save(p, out + "_p.bin");
    save(T, out + "_T.bin");
    FILE *fp = std::fopen((out + "_hist.bin").c_str(), "wb");
    std::fwrite(hist.data(), sizeof(double), hist.size(), fp);
    std::fclose(fp);
    return 0;
}

static int wcinit(int argc, char **argv)
{
    if (argc < 8) { std::fprintf(stderr, "usage: wcinit <case> <c> <rho0> <gz> <T> <out>\n"); return 2; }
    settings::zoneName() = argv[2];
    const scalar c = std::atof(argv[3]);
    const scalar rho0 = std::atof(argv[4]);
    vector g(0, 0, std::atof(argv[5]));
    const std::string out = argv[7];
    Time time(0.01, 1.0, 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    Field<scalar> T(mesh, 0, "T");
    Field<scalar> p(mesh, 0, "p");
    Field<scalar> pHyd(mesh, 0, "pHyd");
    Field<scalar> rho(mesh, rho0, "rho");
    load(T, argv[6]);
    T.correctBoundaryConditions();
#include "shearLayerWC/pEqn.H"
#include "shearLayerWC/hydrostaticP.H"
    for (int i = settings::m() / 2; i < mesh.ni() - settings::m() / 2; i++)
        for (int j = settings::m() / 2; j < mesh.nj() - settings::m() / 2; j++)
            for (int k = settings::m() / 2; k < mesh.nk() - settings::m() / 2; k++)
                rho(i, j, k) = std::pow(p(i, j, k) / (c * c / 2.0 / rho0), 0.5); /* shearLayer.cpp:141-150 */
    p.correctBoundaryConditions();
    rho.correctBoundaryConditions();
    save(p, out + "_p.bin");
    save(rho, out + "_rho.bin");
    return 0;
}

/* the ex:: variants no app of the time advance uses: div(tensor), div(symmTensor),
 * div(scalar, tensor), laplacian(Field nu, vector / scalar); inputs are ghosted as given */
static int ops2(int argc, char **argv)
{
    if (argc < 9) { std::fprintf(stderr, "usage: ops2 <case> <T> <S> <s> <nu> <U> <out>\n"); return 2; }
    settings::zoneName() = argv[2];
    const std::string out = argv[8];
    Time time(0.01, 1.0, 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    Field<tensor> T(mesh, tensor(0.0), "Tt");
    Field<symmTensor> S(mesh, symmTensor(0.0), "Ss");
    Field<scalar> s(mesh, 0, "ss");
    Field<scalar> nu(mesh, 0, "nu");
    Field<vector> U(mesh, vector(0, 0, 0), "Uu");
    load(T, argv[3]);
    load(S, argv[4]);
    load(s, argv[5]);
    load(nu, argv[6]);
    load(U, argv[7]);
    auto Tp = std::make_shared<Field<tensor> >(T);
    save(*ex::div(T), out + "_div_t.bin");
    save(*ex::div(S), out + "_div_st.bin");
    save(*ex::div(s, Tp), out + "_div_sT.bin");
    save(*ex::laplacian(nu, U), out + "_lap_f_v.bin");
    save(*ex::laplacian(nu, s), out + "_lap_f_s.bin");
    return 0;
}

/* the implicit Laplacian (src/im): M = im::laplacian(mu, x) (7-point coefficients and the
 * deferred correction against ex::laplacian), M.ap() -= c, then (M == f).solve(tol, maxits)
 * on x (the reference's line relaxation, fdMatrix.hxx:59-198); saves the coefficients and the
 * source as built, x after the solve, the residual and the solve's wall time */
static int im_solve(int argc, char **argv)
{
    if (argc < 10) { std::fprintf(stderr, "usage: im <case> <mu> <c> <x> <f> <tol> <maxits> <out>\n"); return 2; }
    settings::zoneName() = argv[2];
    const double mu = std::atof(argv[3]), c = std::atof(argv[4]), tol = std::atof(argv[7]);
    const int maxits = std::atoi(argv[8]);
    const std::string out = argv[9];
    Time time(0.01, 1.0, 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    auto x = std::make_shared<Field<scalar> >(mesh, 0, "p");  // the scalar BCs of the case (pBC)
    auto f = std::make_shared<Field<scalar> >(mesh, 0, "p");
    load(*x, argv[5]);
    load(*f, argv[6]);
    x->correctBoundaryConditions();
    auto M = im::laplacian(mu, x);
    for (int l = 0; l < 6; l++) save(M->al(l), out + "_al" + std::to_string(l) + ".bin");
    save(M->ap(), out + "_ap.bin");
    save(*dynamic_cast<Field<scalar> *>(M.get()), out + "_src.bin");
    M->ap() -= c;
    auto S = (M == f);
    const auto t0 = std::chrono::steady_clock::now();
    S->solve(tol, maxits);
    const double solve_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    save(*x, out + "_x.bin");
    const scalar res = S->residual();
    std::FILE *fp = std::fopen((out + "_res.txt").c_str(), "w");
    std::fprintf(fp, "%.17g\n", res);
    std::fclose(fp);
    fp = std::fopen((out + "_time.txt").c_str(), "w");  /* wall seconds of the solve call */
    std::fprintf(fp, "%.9g\n", solve_s);
    std::fclose(fp);
    return 0;
}

/* the apps' output after each step: Mesh::write (geometry, case, restart) and Field<T>::write */
static int ensight(int argc, char **argv)
{
    if (argc < 8) { std::fprintf(stderr, "usage: ensight <case> <nsteps> <dt> <U> <p> <dir>\n"); return 2; }
    settings::zoneName() = argv[2];
    const int nsteps = std::atoi(argv[3]);
    const double dt = std::atof(argv[4]);
    const std::string dir = argv[7];
    Time time(dt, dt * (nsteps + 0.5), 1);
    parallelCom::decompose(settings::zoneName() + "/" + "mesh");
    Mesh mesh(settings::zoneName() + "/" + "mesh", time);
    Field<vector> U(mesh, vector(0, 0, 0), "U");
    Field<scalar> p(mesh, 0, "p");
    load(U, argv[5]);
    load(p, argv[6]);
    U.correctBoundaryConditions();
    p.correctBoundaryConditions();
    for (int step = 0; step < nsteps; step++) {
        time++;
        mesh.write(dir);
        U.write(dir, "U");
        p.write(dir, "p");
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 2) { std::fprintf(stderr, "usage: nova_ref run|ops|wc|wcinit|ensight|ops2|im ... [-m order]\n"); return 2; }
    settings::process(argc, argv); /* the reference's own -m option (settings.cpp:53-78) */
    std::string mode = argv[1];
    if (mode == "run") return run(argc, argv);
    if (mode == "ops") return ops(argc, argv);
    if (mode == "wc") return wc(argc, argv);
    if (mode == "wcinit") return wcinit(argc, argv);
    if (mode == "ensight") return ensight(argc, argv);
    if (mode == "ops2") return ops2(argc, argv);
    if (mode == "im") return im_solve(argc, argv);
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
