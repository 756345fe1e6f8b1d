// host_io.cpp -- PLOT3D grid and solution files in the reference's format.
//
// The reference writes Fortran unformatted sequential files: every WRITE
// statement is one record, framed by a 4-byte record length before and
// after it, and every real is a default real (4 bytes).  mesh.x
// (gridder.f90:150-212) holds the cell-centre coordinates; NNNN.q
// (filer.f90:161-187) holds pre, uc, vc, wc and ETA, appended to the file
// when it exists (position='append'); reading_variables
// (reading_data.f90:62-90) restarts from such a file.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ntcfd_host.h"

namespace {

bool put_record(FILE* f, const void* data, uint32_t bytes) {
    return fwrite(&bytes, 4, 1, f) == 1 && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes) &&
           fwrite(&bytes, 4, 1, f) == 1;
}

bool get_record(FILE* f, std::vector<unsigned char>& out) {
    uint32_t a = 0, b = 0;
    if (fread(&a, 4, 1, f) != 1) return false;
    out.resize(a);
    if (a && fread(out.data(), 1, a, f) != a) return false;
    if (fread(&b, 4, 1, f) != 1) return false;
    return a == b;
}

}  // namespace

extern "C" int ntcfd_write_plot3d_x(const char* path, int nx, int ny, int nz, const double* X, const double* Y,
                                    const double* Z) {
    if (!path || !X || !Y || !Z || nx < 1 || ny < 1 || nz < 1) return -1;
    const size_t n = (size_t)nx * ny * nz;
    if (3 * n * 4 > 0xffffffffu) return -1;
    // cell centres Xs(i) = (X(i+1) + X(i)) / 2 in real*8, stored as default reals
    // (gridder.f90:174-196); X[q] holds X(q - 1)
    std::vector<float> xyz(3 * n);
    size_t q = 0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) xyz[q++] = (float)((X[i + 2] + X[i + 1]) / 2.0);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) xyz[q++] = (float)((Y[j + 2] + Y[j + 1]) / 2.0);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) xyz[q++] = (float)((Z[k + 2] + Z[k + 1]) / 2.0);
    FILE* f = fopen(path, "wb");
    if (!f) return -2;
    const int32_t nb = 1, dims[3] = {nx, ny, nz};
    const bool ok = put_record(f, &nb, 4) && put_record(f, dims, 12) &&
                    put_record(f, xyz.data(), (uint32_t)(xyz.size() * 4));
    return (fclose(f) == 0 && ok) ? 0 : -2;
}

extern "C" int ntcfd_write_plot3d_q(const char* path, int nx, int ny, int nz, const double* pre, const double* uc,
                                    const double* vc, const double* wc, const double* eta, int append) {
    if (!path || !pre || !uc || !vc || !wc || !eta || nx < 1 || ny < 1 || nz < 1) return -1;
    const size_t n = (size_t)nx * ny * nz;
    if (5 * n * 4 > 0xffffffffu) return -1;
    std::vector<float> q(5 * n);
    const double* src[4] = {pre, uc, vc, wc};
    for (int h = 0; h < 4; ++h)
        for (size_t c = 0; c < n; ++c) q[h * n + c] = (float)src[h][c];
    // ETA(i,j,k) of the halo array (index -1..n+2 in each direction)
    const size_t ex = (size_t)nx + 4, ey = (size_t)ny + 4;
    size_t c = 4 * n;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) q[c++] = (float)eta[(i + 1) + ex * ((j + 1) + ey * (k + 1))];
    FILE* f = fopen(path, append ? "ab" : "wb");
    if (!f) return -2;
    const int32_t nb = 1, dims[3] = {nx, ny, nz};
    const float temp[4] = {1.0f, 1.0f, 1.0f, 1.0f};   // mach, alpha, reyn, time: all 1.0
    const bool ok = put_record(f, &nb, 4) && put_record(f, dims, 12) && put_record(f, temp, 16) &&
                    put_record(f, q.data(), (uint32_t)(q.size() * 4));
    return (fclose(f) == 0 && ok) ? 0 : -2;
}

extern "C" int ntcfd_read_plot3d_q(const char* path, int nx, int ny, int nz, double* u, double* v, double* w,
                                   double* p) {
    if (!path || !u || !v || !w || !p || nx < 1 || ny < 1 || nz < 1) return -1;
    FILE* f = fopen(path, "rb");
    if (!f) return -2;
    std::vector<unsigned char> r0, r1, r2, r3;
    const bool ok = get_record(f, r0) && get_record(f, r1) && get_record(f, r2) && get_record(f, r3);
    fclose(f);
    const size_t n = (size_t)nx * ny * nz;
    if (!ok || r3.size() != 5 * n * 4) return -3;
    std::vector<float> Q(5 * n);
    std::memcpy(Q.data(), r3.data(), r3.size());
    const size_t ex = (size_t)nx + 4, ey = (size_t)ny + 4;
    auto H = [&](int i, int j, int k) { return (i + 1) + ex * ((j + 1) + ey * (k + 1)); };
    auto QI = [&](int i, int j, int k, int h) {
        return Q[(size_t)h * n + (size_t)(i - 1) + (size_t)nx * ((j - 1) + (size_t)ny * (k - 1))];
    };
    // face velocities from the centred ones on 1..n-1 in every direction, in default-real
    // arithmetic (Qout and the literal 0.5 are default reals), and p = pre
    // (reading_data.f90:71-85); every other entry of u, v, w, p is left as it was
    for (int k = 1; k <= nz - 1; ++k)
        for (int j = 1; j <= ny - 1; ++j)
            for (int i = 1; i <= nx - 1; ++i) {
                u[H(i, j, k)] = (double)(0.5f * (QI(i, j, k, 1) + QI(i + 1, j, k, 1)));
                v[H(i, j, k)] = (double)(0.5f * (QI(i, j, k, 2) + QI(i, j + 1, k, 2)));
                w[H(i, j, k)] = (double)(0.5f * (QI(i, j, k, 3) + QI(i, j, k + 1, 3)));
            }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) p[H(i, j, k)] = (double)QI(i, j, k, 0);
    return 0;
}
