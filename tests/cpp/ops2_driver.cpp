// C++ caller of the operators no app's time advance uses, through
// include/nova/nova.hpp with the reference's types and spelling:
// ex::grad(Field<vector>), ex::div(Field<tensor>), ex::div(Field<symmTensor>),
// ex::div(Field<scalar>, shared_ptr<Field<tensor>>), ex::laplacian(Field<scalar> nu, Field<T>).
//
//   ops2_driver <case-dir> <in-prefix> <out-prefix>
//
// Reads <in-prefix>{T,S,s,nu,U}.bin and writes <out-prefix>{grad_v,div_t,div_st,
// div_sT,lap_f_v,lap_f_s}.bin, all Field<T> values in the reference layout
// (ghosted, float64).
#include <cstdio>
#include <fstream>
#include <memory>
#include <string>

#include "nova/nova.hpp"

template <class T> static bool read_field(const std::string &path, nova::Field<T> &f)
{
    std::ifstream in(path, std::ios::binary);
    const size_t n = (size_t)f.ni() * f.nj() * f.nk() * sizeof(T);
    in.read(reinterpret_cast<char *>(f.ptr()), (std::streamsize)n);
    return (size_t)in.gcount() == n;
}

template <class T> static void write_field(const std::string &path, const nova::Field<T> &f)
{
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char *>(f.ptr()), (std::streamsize)((size_t)f.ni() * f.nj() * f.nk() * sizeof(T)));
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: ops2_driver <case> <in-prefix> <out-prefix>\n");
        return 2;
    }
    const std::string zone = argv[1], in = argv[2], out = argv[3];
    try {
        nova::Mesh mesh(zone + "/mesh");
        auto T = std::make_shared<nova::Field<nova::tensor>>(mesh);
        nova::Field<nova::symmTensor> S(mesh);
        nova::Field<nova::scalar> s(mesh), nu(mesh);
        nova::Field<nova::vector> U(mesh);
        if (!read_field(in + "T.bin", *T) || !read_field(in + "S.bin", S) || !read_field(in + "s.bin", s) ||
            !read_field(in + "nu.bin", nu) || !read_field(in + "U.bin", U)) {
            std::fprintf(stderr, "short read\n");
            return 1;
        }
        write_field(out + "grad_v.bin", *nova::ex::grad(U));
        write_field(out + "div_t.bin", *nova::ex::div(*T));
        write_field(out + "div_st.bin", *nova::ex::div(S));
        write_field(out + "div_sT.bin", *nova::ex::div(s, T));
        write_field(out + "lap_f_v.bin", *nova::ex::laplacian(nu, U));
        write_field(out + "lap_f_s.bin", *nova::ex::laplacian(nu, s));
    } catch (const nova::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
