// nova.hpp -- header-only C++ adapter over include/nova_gpu.h that keeps the
// reference's host API: Mesh(file), Field<scalar>/Field<vector> with the
// ghosted array-of-structs storage of src/Field/Field.h:56-157,
// correctBoundaryConditions(), ex::grad/div/curl/laplacian returning
// std::shared_ptr<Field<T>> (src/ex/*/ *.h), poisson(p).rhs(f).solve()
// (src/poisson/poisson.h:36-115), tools::maximum (src/Tools/Tools.h:19-36) and
// im::laplacian with its fdMatrix (src/im).
// Each call runs on the GPU through the C ABI; host Fields are the caller's
// buffers in the reference layout, uploaded and downloaded per call.  The
// fused path replaces a whole loop body (RKLoop.H / UEqn.H + BEqn.H) with
// nova::Advance, which keeps the state resident on the device.
#pragma once

#include <array>
#include <cmath>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "nova_gpu.h"

namespace nova {

typedef double scalar;

// layout-compatible with the reference's vector (scalar v_[3], src/Types/vector/vector.h:24)
struct vector {
    scalar v_[3];
    vector() : v_{0, 0, 0} {}
    vector(scalar a, scalar b, scalar c) : v_{a, b, c} {}
    scalar &x() { return v_[0]; }
    scalar &y() { return v_[1]; }
    scalar &z() { return v_[2]; }
    scalar x() const { return v_[0]; }
    scalar y() const { return v_[1]; }
    scalar z() const { return v_[2]; }
    scalar &operator[](int d) { return v_[d]; }
};

// layout-compatible with the reference's tensor (scalar v_[9], xx xy xz yx ..., src/Types/tensor/tensor.h:25)
// and symmTensor (scalar v_[6], xx xy xz yy yz zz, src/Types/symmTensor/symmTensor.h:19)
struct tensor {
    scalar v_[9];
    tensor() : v_{0, 0, 0, 0, 0, 0, 0, 0, 0} {}
    scalar &operator[](int c) { return v_[c]; }
};
struct symmTensor {
    scalar v_[6];
    symmTensor() : v_{0, 0, 0, 0, 0, 0} {}
    scalar &operator[](int c) { return v_[c]; }
};

template <class T> struct nComp;
template <> struct nComp<scalar> { static constexpr int value = 1; };
template <> struct nComp<vector> { static constexpr int value = 3; };
template <> struct nComp<symmTensor> { static constexpr int value = 6; };
template <> struct nComp<tensor> { static constexpr int value = 9; };

class Error : public std::runtime_error {
public:
    nova_status status;
    Error(nova_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(nova_ctx *ctx, nova_status s, const char *what)
{
    if (s != NOVA_OK) throw Error(s, std::string(what) + ": " + (ctx ? nova_last_error(ctx) : "no context"));
}

// Mesh(std::string file): reads "origin:", "N:", "L:", "hypz:" (src/Mesh/Mesh.cpp:38-62)
class Mesh {
    std::shared_ptr<nova_ctx> ctx_;
    nova_mesh_desc d_{};
    int n_[3] = {0, 0, 0};

public:
    explicit Mesh(const nova_mesh_desc &d) : d_(d) { init(); }
    Mesh(const std::string &file, int m = 6)
    {
        std::ifstream fin(file);
        if (!fin) throw Error(NOVA_E_INVALID, "cannot open mesh file " + file);
        std::string line;
        d_.m = m;
        while (std::getline(fin, line)) {
            std::stringstream sp(line);
            std::string key;
            sp >> key;
            if (key == "origin:") sp >> d_.origin[0] >> d_.origin[1] >> d_.origin[2];
            else if (key == "N:") sp >> d_.N[0] >> d_.N[1] >> d_.N[2];
            else if (key == "L:") sp >> d_.L[0] >> d_.L[1] >> d_.L[2];
            else if (key == "hypz:") { d_.hyperbolic_z = 1; sp >> d_.s1 >> d_.s2; }
        }
        init();
    }
    void init()
    {
        nova_ctx *c = nullptr;
        check(nullptr, nova_create(&d_, &c), "nova_create");
        ctx_.reset(c, [](nova_ctx *p) { nova_destroy(p); });
        check(c, nova_mesh_local_n(c, n_), "nova_mesh_local_n");
    }
    nova_ctx *ctx() const { return ctx_.get(); }
    int ni() const { return n_[0]; }
    int nj() const { return n_[1]; }
    int nk() const { return n_[2]; }
    const int *local_n() const { return n_; }
    scalar dx() const { return d_.L[0] / d_.N[0]; }
    scalar dy() const { return d_.L[1] / d_.N[1]; }
    scalar dz() const { return d_.L[2] / d_.N[2]; }
    int m() const { return d_.m; }
    const nova_mesh_desc &desc() const { return d_; }
};

// Host field in the reference layout plus its device mirror.
template <class T> class Field {
    Mesh mesh_;
    std::vector<T> v_;
    std::shared_ptr<nova_field> dev_;

public:
    explicit Field(const Mesh &m, const T &val = T()) : mesh_(m), v_((size_t)m.ni() * m.nj() * m.nk(), val)
    {
        nova_field *f = nullptr;
        check(mesh_.ctx(), nova_field_create(mesh_.ctx(), nComp<T>::value, NOVA_F64, &f), "nova_field_create");
        Mesh keep = mesh_;
        dev_.reset(f, [keep](nova_field *p) { nova_field_destroy(keep.ctx(), p); });
    }
    int index(int i, int j, int k) const { return k + j * mesh_.nk() + i * (mesh_.nk() * mesh_.nj()); }
    T &operator()(int i, int j, int k) { return v_[index(i, j, k)]; }
    const T &operator()(int i, int j, int k) const { return v_[index(i, j, k)]; }
    T *ptr() { return v_.data(); }
    const T *ptr() const { return v_.data(); }
    const Mesh &mesh() const { return mesh_; }
    int ni() const { return mesh_.ni(); }
    int nj() const { return mesh_.nj(); }
    int nk() const { return mesh_.nk(); }
    nova_field *dev() const { return dev_.get(); }

    void toDevice() const
    {
        check(mesh_.ctx(), nova_field_upload(mesh_.ctx(), dev_.get(), (const double *)v_.data(), mesh_.local_n()),
              "nova_field_upload");
    }
    // device -> host, ghosts and the duplicate periodic node filled (periodic)
    void fromDevice()
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), dev_.get(), (double *)v_.data(), mesh_.local_n(), nullptr),
              "nova_field_download");
    }
    // periodicBC::update on every face: a round trip through the device ghost synthesis
    void correctBoundaryConditions()
    {
        toDevice();
        fromDevice();
    }
};

namespace ex {

inline std::shared_ptr<Field<vector>> grad(const Field<scalar> &f)
{
    auto out = std::make_shared<Field<vector>>(f.mesh());
    f.toDevice();
    check(f.mesh().ctx(), nova_grad_s(f.mesh().ctx(), f.dev(), out->dev()), "nova_grad_s");
    out->fromDevice();
    return out;
}

// ex::grad(const Field<vector>&) (src/ex/grad/grad.h:43-46, the Q1 stencil of grad.cpp:65-102)
inline std::shared_ptr<Field<tensor>> grad(const Field<vector> &U)
{
    auto out = std::make_shared<Field<tensor>>(U.mesh());
    U.toDevice();
    check(U.mesh().ctx(), nova_grad_v(U.mesh().ctx(), U.dev(), out->dev()), "nova_grad_v");
    out->fromDevice();
    return out;
}

// ex::div(const Field<tensor>&), ex::div(const Field<symmTensor>&) (src/ex/div/div.hxx:222-285)
template <class T>
typename std::enable_if<std::is_same<T, tensor>::value || std::is_same<T, symmTensor>::value,
                        std::shared_ptr<Field<vector>>>::type
div(const Field<T> &t)
{
    auto out = std::make_shared<Field<vector>>(t.mesh());
    t.toDevice();
    check(t.mesh().ctx(), nova_div_t(t.mesh().ctx(), t.dev(), out->dev()), "nova_div_t");
    out->fromDevice();
    return out;
}

// ex::div(const Field<scalar>&, std::shared_ptr<Field<tensor>>) (src/ex/div/div.hxx:173-207)
inline std::shared_ptr<Field<vector>> div(const Field<scalar> &s, const std::shared_ptr<Field<tensor>> &t)
{
    auto out = std::make_shared<Field<vector>>(s.mesh());
    s.toDevice();
    t->toDevice();
    check(s.mesh().ctx(), nova_div_st(s.mesh().ctx(), s.dev(), t->dev(), out->dev()), "nova_div_st");
    out->fromDevice();
    return out;
}

inline std::shared_ptr<Field<scalar>> div(const Field<vector> &U)
{
    auto out = std::make_shared<Field<scalar>>(U.mesh());
    U.toDevice();
    check(U.mesh().ctx(), nova_div_v(U.mesh().ctx(), U.dev(), out->dev()), "nova_div_v");
    out->fromDevice();
    return out;
}

template <class T> std::shared_ptr<Field<T>> div(const Field<vector> &U, const Field<T> &f)
{
    auto out = std::make_shared<Field<T>>(U.mesh());
    U.toDevice();
    f.toDevice();
    check(U.mesh().ctx(), nova_div_vf(U.mesh().ctx(), U.dev(), f.dev(), out->dev()), "nova_div_vf");
    out->fromDevice();
    return out;
}

inline std::shared_ptr<Field<vector>> curl(const Field<vector> &U)
{
    auto out = std::make_shared<Field<vector>>(U.mesh());
    U.toDevice();
    check(U.mesh().ctx(), nova_curl(U.mesh().ctx(), U.dev(), out->dev()), "nova_curl");
    out->fromDevice();
    return out;
}

template <class T> std::shared_ptr<Field<T>> laplacian(const scalar &nu, const Field<T> &f)
{
    auto out = std::make_shared<Field<T>>(f.mesh());
    f.toDevice();
    check(f.mesh().ctx(), nova_laplacian(f.mesh().ctx(), nu, f.dev(), out->dev()), "nova_laplacian");
    out->fromDevice();
    return out;
}

// ex::laplacian(const Field<scalar>& nu, const Field<T>&) (src/ex/laplacian/laplacian.hxx:64-127)
template <class T> std::shared_ptr<Field<T>> laplacian(const Field<scalar> &nu, const Field<T> &f)
{
    auto out = std::make_shared<Field<T>>(f.mesh());
    nu.toDevice();
    f.toDevice();
    check(f.mesh().ctx(), nova_laplacian_f(f.mesh().ctx(), nu.dev(), f.dev(), out->dev()), "nova_laplacian_f");
    out->fromDevice();
    return out;
}

}  // namespace ex

// poisson(p): rhs(f); solve() writes p's unique nodes (src/poisson/poisson.cpp:167-265)
class poisson {
    std::shared_ptr<Field<scalar>> p_;
    std::shared_ptr<Field<scalar>> rhs_;

public:
    explicit poisson(std::shared_ptr<Field<scalar>> p) : p_(std::move(p)) {}
    void rhs(std::shared_ptr<Field<scalar>> f) { rhs_ = std::move(f); }
    void solve()
    {
        rhs_->toDevice();
        check(p_->mesh().ctx(), nova_poisson_solve(p_->mesh().ctx(), rhs_->dev(), p_->dev()), "nova_poisson_solve");
        p_->fromDevice();
    }
};

namespace tools {
inline scalar maximum(const std::shared_ptr<Field<scalar>> &f)
{
    f->toDevice();
    double v = 0.0;
    check(f->mesh().ctx(), nova_field_maxabs(f->mesh().ctx(), f->dev(), &v), "nova_field_maxabs");
    return v;
}
}  // namespace tools

// fdMatrix<scalar> (src/im/fdMatrix/fdMatrix.h:33-77): the matrix lives on the
// device (nova_fdm); the transported field stays the caller's Field<scalar>,
// uploaded before every call that reads it and downloaded after solve().
// Like the reference's operators, these change the matrix in place.
template <class T> class fdMatrix {
    static_assert(std::is_same<T, scalar>::value, "the implicit operators are built for scalar fields");
    std::shared_ptr<Field<T>> x_;
    std::shared_ptr<nova_fdm> m_;
    nova_ctx *ctx() const { return x_->mesh().ctx(); }

public:
    fdMatrix(std::shared_ptr<Field<T>> x, nova_fdm *m) : x_(std::move(x)), m_(m, nova_fdm_destroy) {}
    nova_fdm *dev() const { return m_.get(); }

    // ap() += d / ap() -= d, the Field arithmetic apps apply to fdMatrix::ap()
    class Diagonal {
        fdMatrix &a_;

    public:
        explicit Diagonal(fdMatrix &a) : a_(a) {}
        Diagonal &operator+=(scalar d)
        {
            check(a_.ctx(), nova_fdm_add_diagonal(a_.ctx(), a_.dev(), d), "nova_fdm_add_diagonal");
            return *this;
        }
        Diagonal &operator-=(scalar d) { return *this += -d; }
    };
    Diagonal ap() { return Diagonal(*this); }

    // fdMatrix::solve (fdMatrix.hxx:59-198): x is the initial guess and the result
    void solve(scalar tol, int maxIts)
    {
        x_->toDevice();
        check(ctx(), nova_fdm_solve(ctx(), dev(), tol, maxIts, nullptr, nullptr), "nova_fdm_solve");
        x_->fromDevice();
    }
    T residual()
    {
        x_->toDevice();
        double r = 0.0;
        check(ctx(), nova_fdm_residual(ctx(), dev(), &r), "nova_fdm_residual");
        return r;
    }
    void relax(const scalar &urf)
    {
        x_->toDevice();
        check(ctx(), nova_fdm_relax(ctx(), dev(), urf), "nova_fdm_relax");
    }
    // (i, j, k) index the ghosted field as in the reference (m/2 ghost nodes
    // first); the node is taken modulo the periodic length, so the duplicate
    // end node N is node 0
    void setReference(int i, int j, int k, scalar val)
    {
        const nova_mesh_desc &d = x_->mesh().desc();
        const int h = d.m / 2, idx[3] = {i, j, k};
        int u[3];
        for (int a = 0; a < 3; a++) u[a] = ((idx[a] - h) % d.N[a] + d.N[a]) % d.N[a];
        check(ctx(), nova_fdm_set_reference(ctx(), dev(), u[0], u[1], u[2], val), "nova_fdm_set_reference");
    }
    fdMatrix &operator+=(const fdMatrix &r)
    {
        check(ctx(), nova_fdm_add(ctx(), dev(), 1.0, r.dev()), "nova_fdm_add");
        return *this;
    }
    fdMatrix &operator-=(const fdMatrix &r)
    {
        check(ctx(), nova_fdm_add(ctx(), dev(), -1.0, r.dev()), "nova_fdm_add");
        return *this;
    }
    fdMatrix &operator*=(const fdMatrix &r)
    {
        check(ctx(), nova_fdm_mul(ctx(), dev(), r.dev()), "nova_fdm_mul");
        return *this;
    }
    // the source += f
    void operator==(const Field<T> &f)
    {
        f.toDevice();
        check(ctx(), nova_fdm_add_source(ctx(), dev(), 1.0, f.dev()), "nova_fdm_add_source");
    }
    void negate() { check(ctx(), nova_fdm_scale(ctx(), dev(), -1.0), "nova_fdm_scale"); }
};

// the global operators of fdMatrix.hxx:359-413: the left operand, changed in place
template <class T>
std::shared_ptr<fdMatrix<T>> operator+(std::shared_ptr<fdMatrix<T>> a, const std::shared_ptr<fdMatrix<T>> &b)
{
    *a += *b;
    return a;
}
template <class T>
std::shared_ptr<fdMatrix<T>> operator-(std::shared_ptr<fdMatrix<T>> a, const std::shared_ptr<fdMatrix<T>> &b)
{
    *a -= *b;
    return a;
}
template <class T> std::shared_ptr<fdMatrix<T>> operator-(std::shared_ptr<fdMatrix<T>> a)
{
    a->negate();
    return a;
}
template <class T>
std::shared_ptr<fdMatrix<T>> operator==(std::shared_ptr<fdMatrix<T>> a, const std::shared_ptr<Field<T>> &f)
{
    *a == *f;
    return a;
}

namespace im {
// im::laplacian(mu, x) (src/im/laplacian/laplacian.hxx:24-58)
template <class T> std::shared_ptr<fdMatrix<T>> laplacian(const scalar mu, std::shared_ptr<Field<T>> x)
{
    static_assert(std::is_same<T, scalar>::value, "the implicit operators are built for scalar fields");
    x->toDevice();
    nova_fdm *m = nullptr;
    check(x->mesh().ctx(), nova_im_laplacian(x->mesh().ctx(), mu, x->dev(), &m), "nova_im_laplacian");
    return std::make_shared<fdMatrix<T>>(std::move(x), m);
}
// im::laplacian(x) = im::laplacian(1, x) (laplacian.hxx:61-68)
template <class T> std::shared_ptr<fdMatrix<T>> laplacian(std::shared_ptr<Field<T>> x)
{
    return laplacian(scalar(1.0), std::move(x));
}
}  // namespace im

// The fused loop body: state resident on the device between calls.
class Advance {
    Mesh mesh_;
    nova_run_desc rd_{};
    std::shared_ptr<nova_field> U_, p_, B_, pB_;

    std::shared_ptr<nova_field> make(int nc, int prec)
    {
        nova_field *f = nullptr;
        check(mesh_.ctx(), nova_field_create(mesh_.ctx(), nc, prec, &f), "nova_field_create");
        Mesh keep = mesh_;
        return std::shared_ptr<nova_field>(f, [keep](nova_field *p) { nova_field_destroy(keep.ctx(), p); });
    }

public:
    Advance(const Mesh &m, const nova_run_desc &rd) : mesh_(m), rd_(rd)
    {
        U_ = make(3, rd.precision);
        p_ = make(1, NOVA_F64);
        if (rd.model == NOVA_MODEL_MHD) {
            B_ = make(3, rd.precision);
            pB_ = make(1, NOVA_F64);
        }
    }
    // aos: the reference's Field<vector>::ptr() (ghosted array-of-structs, 3 doubles per node)
    void setU(const void *aos)
    {
        check(mesh_.ctx(), nova_field_upload(mesh_.ctx(), U_.get(), (const double *)aos, mesh_.local_n()), "upload U");
    }
    void setB(const void *aos)
    {
        check(mesh_.ctx(), nova_field_upload(mesh_.ctx(), B_.get(), (const double *)aos, mesh_.local_n()), "upload B");
    }
    void getU(void *aos) const
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), U_.get(), (double *)aos, mesh_.local_n(), nullptr),
              "download U");
    }
    void getB(void *aos) const
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), B_.get(), (double *)aos, mesh_.local_n(), nullptr),
              "download B");
    }
    void setU(const Field<vector> &U)
    {
        check(mesh_.ctx(), nova_field_upload(mesh_.ctx(), U_.get(), (const double *)U.ptr(), mesh_.local_n()), "upload U");
    }
    void setB(const Field<vector> &B)
    {
        check(mesh_.ctx(), nova_field_upload(mesh_.ctx(), B_.get(), (const double *)B.ptr(), mesh_.local_n()), "upload B");
    }
    // run nsteps; returns the diagnostics history (nsteps rows of NOVA_HIST_COLS)
    std::vector<double> run(int nsteps)
    {
        std::vector<double> hist((size_t)nsteps * NOVA_HIST_COLS, 0.0);
        nova_state st{U_.get(), p_.get(), B_.get(), pB_.get()};
        check(mesh_.ctx(), nova_advance(mesh_.ctx(), &rd_, &st, nsteps, hist.data()), "nova_advance");
        rd_.t0 += nsteps * rd_.dt;
        return hist;
    }
    void getU(Field<vector> &U) const
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), U_.get(), (double *)U.ptr(), mesh_.local_n(), nullptr),
              "download U");
    }
    void getB(Field<vector> &B) const
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), B_.get(), (double *)B.ptr(), mesh_.local_n(), nullptr),
              "download B");
    }
    void getp(Field<scalar> &p) const
    {
        check(mesh_.ctx(), nova_field_download(mesh_.ctx(), p_.get(), (double *)p.ptr(), mesh_.local_n(), nullptr),
              "download p");
    }
};

}  // namespace nova
