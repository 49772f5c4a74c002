// EnSight Gold output and input in the layout the reference writes for its
// post-processing and restarts, for one rank (processor number 0000):
//   geometry   <dir>/geom.p0000.geo        src/Mesh/Mesh.cpp:224-300
//   case       <dir>/fd.p0000.case         src/Mesh/Mesh.cpp:302-338
//              <dir>/restart.p.0000.case   src/Mesh/Mesh.cpp:340-355
//   field data <dir>/<name>.0000.<num>.dat src/Field/Field.hxx:404-453 (read: 456-485)
// Host code only: these entry points need no GPU.  The reference writes each
// 80-byte header line from a string whose resize acts on a temporary copy, so
// its bytes after the terminating NUL are unspecified; these writers pad with
// NULs, and readers (EnSight's and the reference's) use the text up to the NUL.
#include "nova_gpu.h"
#include "nova_mesh.cuh"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace nova {

namespace {

struct Out {
    std::FILE *fp = nullptr;
    bool ok = true;
    explicit Out(const std::string &path) : fp(std::fopen(path.c_str(), "wb")) { ok = fp != nullptr; }
    ~Out()
    {
        if (fp) std::fclose(fp);
    }
    void raw(const void *p, size_t n) { ok = ok && std::fwrite(p, 1, n, fp) == n; }
    void line(const char *text)  // one 80-byte header line
    {
        char b[80] = {0};
        std::strncpy(b, text, 79);
        raw(b, 80);
    }
    void i32(int v)
    {
        const int32_t x = v;
        raw(&x, 4);
    }
    void f32(float v) { raw(&v, 4); }
    bool close()
    {
        const bool c = fp && std::fclose(fp) == 0;
        fp = nullptr;
        return ok && c;
    }
};

bool valid_mesh(const nova_mesh_desc *md)
{
    if (!md || md->m < 2 || md->m > 8 || md->m % 2) return false;
    for (int a = 0; a < 3; a++)
        if (md->N[a] < 1 || !(md->L[a] > 0.0) || (md->walls[a] != 0 && md->walls[a] != 1)) return false;
    return true;
}

// stored nodes per axis: N (periodic) or N + 1 (walls)
int stored(const nova_mesh_desc *md, int a) { return md->N[a] + md->walls[a]; }

std::string data_name(const char *dir, const char *name, int num)
{
    char b[32];
    std::snprintf(b, sizeof b, ".0000.%05d.dat", num);  // Field.hxx:412 with processor 0
    return std::string(dir) + "/" + name + b;
}

}  // namespace

}  // namespace nova

using namespace nova;

extern "C" nova_status nova_ensight_write_geometry(const nova_mesh_desc *md, const char *dir)
{
    if (!valid_mesh(md) || !dir) return NOVA_E_INVALID;
    Out f(std::string(dir) + "/geom.p0000.geo");
    if (!f.ok) return NOVA_E_INVALID;
    for (const char *t : {"C Binary", "desc1", "desc2", "node id assign", "element id assign", "part"}) f.line(t);
    f.i32(1);
    f.line("part desc");
    f.line("block rectilinear");
    // the reference's ni - m nodes per axis: the N + 1 interior nodes
    const int n[3] = {md->N[0] + 1, md->N[1] + 1, md->N[2] + 1};
    for (int a = 0; a < 3; a++) f.i32(n[a]);
    const double dx = md->L[0] / md->N[0], dy = md->L[1] / md->N[1];
    for (int i = 0; i < n[0]; i++) f.f32((float)(md->origin[0] + dx * i));
    for (int j = 0; j < n[1]; j++) f.f32((float)(md->origin[1] + dy * j));
    const int h = md->m / 2;
    const double b = mesh_hyp_b(*md);
    for (int k = 0; k < n[2]; k++) f.f32((float)mesh_z(*md, h, b, k + h));
    return f.close() ? NOVA_OK : NOVA_E_INVALID;
}

extern "C" nova_status nova_ensight_write_case(const char *dir, int ntimes, const double *times)
{
    if (!dir || ntimes < 0 || (ntimes > 0 && !times)) return NOVA_E_INVALID;
    {
        std::ofstream c(std::string(dir) + "/fd.p0000.case");
        if (!c) return NOVA_E_INVALID;
        c << "FORMAT" << std::endl << "type: ensight gold" << std::endl;
        c << "GEOMETRY" << std::endl << "model: geom.p0000.geo" << std::endl;
        c << "VARIABLE" << std::endl;
        c << "vector per node: velocity U.0000.*****.dat" << std::endl;
        c << "vector per node: Uprime Uprime.0000.*****.dat" << std::endl;
        c << "vector per node: Udash Udash.0000.*****.dat" << std::endl;
        c << "scalar per node: p  p.0000.*****.dat" << std::endl;
        c << "scalar per node: T  T.0000.*****.dat" << std::endl;
        c << "vector per node: B B.0000.*****.dat" << std::endl;
        c << "vector per node: J J.0000.*****.dat" << std::endl;
        c << "TIME" << std::endl << "time set: 1" << std::endl;
        c << "number of steps: " << ntimes << std::endl;
        c << "filename start number: 00001" << std::endl << "filename increment: 1" << std::endl;
        c << "time values: ";
        for (int i = 0; i < ntimes; i++) c << times[i] << std::endl;
        c << std::endl;
        if (!c) return NOVA_E_INVALID;
    }
    std::ofstream r(std::string(dir) + "/restart.p.0000.case");
    if (!r) return NOVA_E_INVALID;
    r << ntimes << std::endl;
    for (int i = 0; i < ntimes; i++) r << times[i] << std::endl;
    return r ? NOVA_OK : NOVA_E_INVALID;
}

extern "C" nova_status nova_ensight_write_host(const nova_mesh_desc *md, const double *soa, int ncomp, const char *dir,
                                               const char *name, int num)
{
    if (!valid_mesh(md) || !soa || (ncomp != 1 && ncomp != 3) || !dir || !name || num < 0 || num > 99999)
        return NOVA_E_INVALID;
    const int s0 = stored(md, 0), s1 = stored(md, 1), s2 = stored(md, 2);
    const long long n3 = (long long)s0 * s1 * s2;
    Out f(data_name(dir, name, num));
    if (!f.ok) return NOVA_E_INVALID;
    f.line("description");
    f.line("part");
    f.i32(1);
    f.line("point");
    // nodes 0..N per axis, i fastest; on a periodic axis node N is node 0
    std::vector<float> row(md->N[0] + 1);
    for (int c = 0; c < ncomp; c++)
        for (int k = 0; k <= md->N[2]; k++)
            for (int j = 0; j <= md->N[1]; j++) {
                const int kk = k % s2, jj = j % s1;
                for (int i = 0; i <= md->N[0]; i++)
                    row[i] = (float)soa[c * n3 + ((long long)(i % s0) * s1 + jj) * s2 + kk];
                f.raw(row.data(), sizeof(float) * row.size());
            }
    return f.close() ? NOVA_OK : NOVA_E_INVALID;
}

extern "C" nova_status nova_ensight_read_host(const nova_mesh_desc *md, double *soa, int ncomp, const char *dir,
                                              const char *name, int num)
{
    if (!valid_mesh(md) || !soa || (ncomp != 1 && ncomp != 3) || !dir || !name || num < 0 || num > 99999)
        return NOVA_E_INVALID;
    const int s0 = stored(md, 0), s1 = stored(md, 1), s2 = stored(md, 2);
    const long long n3 = (long long)s0 * s1 * s2;
    std::FILE *fp = std::fopen(data_name(dir, name, num).c_str(), "rb");
    if (!fp) return NOVA_E_INVALID;
    bool ok = std::fseek(fp, 240 + sizeof(int32_t), SEEK_SET) == 0;  // Field.hxx:465
    std::vector<float> row(md->N[0] + 1);
    for (int c = 0; c < ncomp && ok; c++)
        for (int k = 0; k <= md->N[2] && ok; k++)
            for (int j = 0; j <= md->N[1] && ok; j++) {
                ok = std::fread(row.data(), sizeof(float), row.size(), fp) == row.size();
                // the stored nodes take the values of their own (first) occurrence
                if (!ok || k >= s2 || j >= s1) continue;
                for (int i = 0; i < s0; i++) soa[c * n3 + ((long long)i * s1 + j) * s2 + k] = (double)row[i];
            }
    std::fclose(fp);
    return ok ? NOVA_OK : NOVA_E_INVALID;
}
