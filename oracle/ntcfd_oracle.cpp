// ntcfd_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the CUDA
// time step.  Serial restatement of the NTUSTCFD Fortran routines on the
// hot path with nproc = 1 (istart = 1, iend = nz); see ntcfd_oracle.h for
// the parity status.  Compiled with -ffp-contract=off and without fast-math
// so that every expression is evaluated left to right as written, like the
// Fortran source.  Not linked into the product library.
#include "ntcfd_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Fortran array with lower bound lo_ in every dimension, column-major.
struct F3 {
    int lo = 0, n0 = 0, n1 = 0, n2 = 0;
    std::vector<double> d;
    void init(int lo_, int hi0, int hi1, int hi2) {
        lo = lo_;
        n0 = hi0 - lo_ + 1; n1 = hi1 - lo_ + 1; n2 = hi2 - lo_ + 1;
        d.assign((size_t)n0 * n1 * n2, 0.0);
    }
    inline double& operator()(int i, int j, int k) {
        return d[(size_t)(i - lo) + (size_t)n0 * ((size_t)(j - lo) + (size_t)n1 * (size_t)(k - lo))];
    }
    size_t size() const { return d.size(); }
};

struct F1 {
    int lo = 0;
    std::vector<double> d;
    void init(int lo_, int hi) { lo = lo_; d.assign((size_t)(hi - lo_ + 1), 0.0); }
    inline double& operator()(int i) { return d[(size_t)(i - lo)]; }
};

struct F2 {  // (1:n0, 1:n1)
    int n0 = 0, n1 = 0;
    std::vector<double> d;
    void init(int a, int b) { n0 = a; n1 = b; d.assign((size_t)a * b, 0.0); }
    inline double& operator()(int i, int j) { return d[(size_t)(i - 1) + (size_t)n0 * (size_t)(j - 1)]; }
};

}  // namespace

struct orc {
    ntcfd_params prm;
    int nx, ny, nz;
    double nu, dt, time = 0.0;
    int nthreads = 1;
    // grid (variables_module.f90:292-323)
    F1 X, Y, Z, iDx, Dxs, iDy, Dys, iDz, Dzs;
    // fields (variables_module.f90:159,215-225,337-347)
    F3 u, v, w, p, u1, v1, w1, u2, v2, w2, us, vs, ws, FX, FY, FZ, ETA;
    F3 pre, uc, vc, wc, Viseff;  // (1:n) stored with lo=1
    F2 FXz, FYz;
    std::vector<double> FXy, FYy;  // 1:nx
};

namespace {

inline bool par(const orc* o) { return o->nthreads > 1; }

// ---------------------------------------------------------------- BCs ----
// boundary_conditions.f90:13-301 (velocity), 305-324 (copies), 329-374 (p).
// Walls are applied in the reference order W, E, S, N, B, F; later walls
// overwrite edge and corner ghosts written by earlier ones.
void bc_velocity(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    F3 &u = o->u, &v = o->v, &w = o->w;
    const auto& bc = o->prm.bc;
    const auto& bv = o->prm.bc_value;
    // West (boundary_conditions.f90:13-57)
    for (int k = -1; k <= nz + 2; ++k)
        for (int j = -1; j <= ny + 2; ++j) {
            switch (bc[NTCFD_WEST][0]) {
                case NTCFD_BC_NOSLIP: u(0, j, k) = 0.0; break;
                case NTCFD_BC_NEUMANN: u(0, j, k) = u(1, j, k); break;
                case NTCFD_BC_DIRICHLET: u(0, j, k) = bv[NTCFD_WEST][0]; break;
                case NTCFD_BC_PERIODIC: u(0, j, k) = u(nx, j, k); break;
            }
            if (bc[NTCFD_WEST][0] == NTCFD_BC_PERIODIC) u(-1, j, k) = u(nx - 1, j, k);
            else u(-1, j, k) = u(0, j, k);
            F3* cc[2] = {&v, &w};
            for (int c = 1; c <= 2; ++c) {
                F3& f = *cc[c - 1];
                switch (bc[NTCFD_WEST][c]) {
                    case NTCFD_BC_NOSLIP: f(0, j, k) = 2 * 0 - f(1, j, k); break;
                    case NTCFD_BC_NEUMANN: f(0, j, k) = f(1, j, k); break;
                    case NTCFD_BC_DIRICHLET: f(0, j, k) = 2 * bv[NTCFD_WEST][c] - f(1, j, k); break;
                    case NTCFD_BC_PERIODIC: f(0, j, k) = f(nx, j, k); break;
                }
                if (bc[NTCFD_WEST][c] == NTCFD_BC_PERIODIC) f(-1, j, k) = f(nx - 1, j, k);
                else f(-1, j, k) = f(0, j, k);
            }
        }
    // East (boundary_conditions.f90:59-105)
    for (int k = -1; k <= nz + 2; ++k)
        for (int j = -1; j <= ny + 2; ++j) {
            if (bc[NTCFD_EAST][0] == NTCFD_BC_PERIODIC) {
                u(nx + 1, j, k) = u(1, j, k);
                u(nx + 2, j, k) = u(2, j, k);
            } else {
                switch (bc[NTCFD_EAST][0]) {
                    case NTCFD_BC_NOSLIP: u(nx, j, k) = 0.0; break;
                    case NTCFD_BC_NEUMANN: u(nx, j, k) = u(nx - 1, j, k); break;
                    case NTCFD_BC_DIRICHLET: u(nx, j, k) = bv[NTCFD_EAST][0]; break;
                }
                u(nx + 1, j, k) = u(nx, j, k);
                u(nx + 2, j, k) = u(nx + 1, j, k);
            }
            F3* cc[2] = {&v, &w};
            for (int c = 1; c <= 2; ++c) {
                F3& f = *cc[c - 1];
                if (bc[NTCFD_EAST][c] == NTCFD_BC_PERIODIC) {
                    f(nx + 1, j, k) = f(1, j, k);
                    f(nx + 2, j, k) = f(2, j, k);
                } else {
                    switch (bc[NTCFD_EAST][c]) {
                        case NTCFD_BC_NOSLIP: f(nx + 1, j, k) = 2 * 0 - f(nx, j, k); break;
                        case NTCFD_BC_NEUMANN: f(nx + 1, j, k) = f(nx, j, k); break;
                        case NTCFD_BC_DIRICHLET: f(nx + 1, j, k) = 2 * bv[NTCFD_EAST][c] - f(nx, j, k); break;
                    }
                    f(nx + 2, j, k) = f(nx + 1, j, k);
                }
            }
        }
    // South (boundary_conditions.f90:107-153)
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nx + 2; ++i) {
            F3* tang[2] = {&u, &w};
            const int tc[2] = {0, 2};
            for (int t = 0; t < 2; ++t) {
                F3& f = *tang[t];
                const int c = tc[t];
                switch (bc[NTCFD_SOUTH][c]) {
                    case NTCFD_BC_NOSLIP: f(i, 0, k) = 2 * 0 - f(i, 1, k); break;
                    case NTCFD_BC_NEUMANN: f(i, 0, k) = f(i, 1, k); break;
                    case NTCFD_BC_DIRICHLET: f(i, 0, k) = 2 * bv[NTCFD_SOUTH][c] - f(i, 1, k); break;
                    case NTCFD_BC_PERIODIC: f(i, 0, k) = f(i, ny, k); break;
                }
                if (bc[NTCFD_SOUTH][c] == NTCFD_BC_PERIODIC) f(i, -1, k) = f(i, ny - 1, k);
                else f(i, -1, k) = f(i, 0, k);
                if (t == 0) {
                    // v after u, as in the reference (u, v, w order)
                    switch (bc[NTCFD_SOUTH][1]) {
                        case NTCFD_BC_NOSLIP: v(i, 0, k) = 0.0; break;
                        case NTCFD_BC_NEUMANN: v(i, 0, k) = v(i, 1, k); break;
                        case NTCFD_BC_DIRICHLET: v(i, 0, k) = bv[NTCFD_SOUTH][1]; break;
                        case NTCFD_BC_PERIODIC: v(i, 0, k) = v(i, ny, k); break;
                    }
                    if (bc[NTCFD_SOUTH][1] == NTCFD_BC_PERIODIC) v(i, -1, k) = v(i, ny - 1, k);
                    else v(i, -1, k) = v(i, 0, k);
                }
            }
        }
    // North (boundary_conditions.f90:155-202)
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nx + 2; ++i) {
            // u
            if (bc[NTCFD_NORTH][0] == NTCFD_BC_PERIODIC) {
                u(i, ny + 1, k) = u(i, 1, k); u(i, ny + 2, k) = u(i, 2, k);
            } else {
                switch (bc[NTCFD_NORTH][0]) {
                    case NTCFD_BC_NOSLIP: u(i, ny + 1, k) = 2 * 0 - u(i, ny, k); break;
                    case NTCFD_BC_NEUMANN: u(i, ny + 1, k) = u(i, ny, k); break;
                    case NTCFD_BC_DIRICHLET: u(i, ny + 1, k) = 2 * bv[NTCFD_NORTH][0] - u(i, ny, k); break;
                }
                u(i, ny + 2, k) = u(i, ny + 1, k);
            }
            // v (normal)
            if (bc[NTCFD_NORTH][1] == NTCFD_BC_PERIODIC) {
                v(i, ny + 1, k) = v(i, 1, k); v(i, ny + 2, k) = v(i, 2, k);
            } else {
                switch (bc[NTCFD_NORTH][1]) {
                    case NTCFD_BC_NOSLIP: v(i, ny, k) = 0.0; break;
                    case NTCFD_BC_NEUMANN: v(i, ny, k) = v(i, ny - 1, k); break;
                    case NTCFD_BC_DIRICHLET: v(i, ny, k) = bv[NTCFD_NORTH][1]; break;
                }
                v(i, ny + 1, k) = v(i, ny, k);
                v(i, ny + 2, k) = v(i, ny + 1, k);
            }
            // w
            if (bc[NTCFD_NORTH][2] == NTCFD_BC_PERIODIC) {
                w(i, ny + 1, k) = w(i, 1, k); w(i, ny + 2, k) = w(i, 2, k);
            } else {
                switch (bc[NTCFD_NORTH][2]) {
                    case NTCFD_BC_NOSLIP: w(i, ny + 1, k) = 2 * 0 - w(i, ny, k); break;
                    case NTCFD_BC_NEUMANN: w(i, ny + 1, k) = w(i, ny, k); break;
                    case NTCFD_BC_DIRICHLET: w(i, ny + 1, k) = 2 * bv[NTCFD_NORTH][2] - w(i, ny, k); break;
                }
                w(i, ny + 2, k) = w(i, ny + 1, k);
            }
        }
    // Back (boundary_conditions.f90:205-252)
    for (int j = -1; j <= ny + 2; ++j)
        for (int i = -1; i <= nx + 2; ++i) {
            F3* tang[2] = {&u, &v};
            for (int c = 0; c < 2; ++c) {
                F3& f = *tang[c];
                switch (bc[NTCFD_BACK][c]) {
                    case NTCFD_BC_NOSLIP: f(i, j, 0) = 2 * 0 - f(i, j, 1); break;
                    case NTCFD_BC_NEUMANN:
                        // BackWall_v 'Neumann' is a no-op in the reference
                        // (v(i,j,0) = v(i,j,0), boundary_conditions.f90:228).
                        if (c == 0) f(i, j, 0) = f(i, j, 1);
                        break;
                    case NTCFD_BC_DIRICHLET: f(i, j, 0) = 2 * bv[NTCFD_BACK][c] - f(i, j, 1); break;
                    case NTCFD_BC_PERIODIC: f(i, j, 0) = f(i, j, nz); break;
                }
                if (bc[NTCFD_BACK][c] == NTCFD_BC_PERIODIC) f(i, j, -1) = f(i, j, nz - 1);
                else f(i, j, -1) = f(i, j, 0);
            }
            switch (bc[NTCFD_BACK][2]) {
                case NTCFD_BC_NOSLIP: w(i, j, 0) = 0.0; break;
                case NTCFD_BC_NEUMANN: w(i, j, 0) = w(i, j, 1); break;
                case NTCFD_BC_DIRICHLET: w(i, j, 0) = bv[NTCFD_BACK][2]; break;
                case NTCFD_BC_PERIODIC: w(i, j, 0) = w(i, j, nz); break;
            }
            if (bc[NTCFD_BACK][2] == NTCFD_BC_PERIODIC) w(i, j, -1) = w(i, j, nz - 1);
            else w(i, j, -1) = w(i, j, 0);
        }
    // Front (boundary_conditions.f90:255-301)
    for (int j = -1; j <= ny + 2; ++j)
        for (int i = -1; i <= nx + 2; ++i) {
            F3* tang[2] = {&u, &v};
            for (int c = 0; c < 2; ++c) {
                F3& f = *tang[c];
                if (bc[NTCFD_FRONT][c] == NTCFD_BC_PERIODIC) {
                    f(i, j, nz + 1) = f(i, j, 1); f(i, j, nz + 2) = f(i, j, 2);
                    continue;
                }
                switch (bc[NTCFD_FRONT][c]) {
                    case NTCFD_BC_NOSLIP: f(i, j, nz + 1) = 2 * 0 - f(i, j, nz); break;
                    case NTCFD_BC_NEUMANN: f(i, j, nz + 1) = f(i, j, nz); break;
                    case NTCFD_BC_DIRICHLET: f(i, j, nz + 1) = 2 * bv[NTCFD_FRONT][c] - f(i, j, nz); break;
                }
                f(i, j, nz + 2) = f(i, j, nz + 1);
            }
            if (bc[NTCFD_FRONT][2] == NTCFD_BC_PERIODIC) {
                w(i, j, nz + 1) = w(i, j, 1); w(i, j, nz + 2) = w(i, j, 2);
            } else {
                switch (bc[NTCFD_FRONT][2]) {
                    case NTCFD_BC_NOSLIP: w(i, j, nz) = 0.0; break;
                    case NTCFD_BC_NEUMANN: w(i, j, nz) = w(i, j, nz - 1); break;
                    case NTCFD_BC_DIRICHLET: w(i, j, nz) = bv[NTCFD_FRONT][2]; break;
                }
                w(i, j, nz + 1) = w(i, j, nz);
                w(i, j, nz + 2) = w(i, j, nz + 1);
            }
        }
}

void bc_copies_and_pressure(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    // boundary_conditions.f90:305-324: u1 = u2 = u_star = u over the whole halo array
    o->u1.d = o->u.d; o->v1.d = o->v.d; o->w1.d = o->w.d;
    o->u2.d = o->u.d; o->v2.d = o->v.d; o->w2.d = o->w.d;
    o->us.d = o->u.d; o->vs.d = o->v.d; o->ws.d = o->w.d;
    F3& p = o->p;
    const auto& bc = o->prm.bc;
    const bool perx = bc[NTCFD_WEST][0] == NTCFD_BC_PERIODIC;
    const bool pery = bc[NTCFD_SOUTH][1] == NTCFD_BC_PERIODIC;
    const bool perz = bc[NTCFD_BACK][2] == NTCFD_BC_PERIODIC;
    // boundary_conditions.f90:329-374 (zero-gradient; periodic copies when periodic)
    for (int k = -1; k <= nz + 2; ++k)
        for (int j = -1; j <= ny + 2; ++j) {
            if (perx) { p(0, j, k) = p(nx, j, k); p(-1, j, k) = p(nx - 1, j, k); }
            else { p(0, j, k) = p(1, j, k); p(-1, j, k) = p(0, j, k); }
        }
    for (int k = -1; k <= nz + 2; ++k)
        for (int j = -1; j <= ny + 2; ++j) {
            if (perx) { p(nx + 1, j, k) = p(1, j, k); p(nx + 2, j, k) = p(2, j, k); }
            else { p(nx + 1, j, k) = p(nx, j, k); p(nx + 2, j, k) = p(nx + 1, j, k); }
        }
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nx + 2; ++i) {
            if (pery) { p(i, 0, k) = p(i, ny, k); p(i, -1, k) = p(i, ny - 1, k); }
            else { p(i, 0, k) = p(i, 1, k); p(i, -1, k) = p(i, 0, k); }
        }
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nx + 2; ++i) {
            if (pery) { p(i, ny + 1, k) = p(i, 1, k); p(i, ny + 2, k) = p(i, 2, k); }
            else { p(i, ny + 1, k) = p(i, ny, k); p(i, ny + 2, k) = p(i, ny + 1, k); }
        }
    for (int j = -1; j <= ny + 2; ++j)
        for (int i = -1; i <= nx + 2; ++i) {
            if (perz) { p(i, j, 0) = p(i, j, nz); p(i, j, -1) = p(i, j, nz - 1); }
            else { p(i, j, 0) = p(i, j, 1); p(i, j, -1) = p(i, j, 0); }
        }
    for (int j = -1; j <= ny + 2; ++j)
        for (int i = -1; i <= nx + 2; ++i) {
            if (perz) { p(i, j, nz + 1) = p(i, j, 1); p(i, j, nz + 2) = p(i, j, 2); }
            else { p(i, j, nz + 1) = p(i, j, nz); p(i, j, nz + 2) = p(i, j, nz + 1); }
        }
}

// ------------------------------------------------------- Smagorinsky ----
// smagorinsky.f90:42-87, GradientPhiGauss.  In REF_ALIASED mode the dummy
// Phi(nx,ny,nz) is associated with the halo array u(-1:nx+2,...) by storage
// sequence (smagorinsky.f90:6-8,46): Phi(i,j,k) is storage element
// (i-1) + (j-1)*nx + (k-1)*nx*ny counted from u(-1,-1,-1).  Elements before
// the array (negative offsets, met on the k = 1 plane) read as 0.
struct PhiRef {
    F3* f; int nx, ny; bool aliased;
    inline double operator()(int i, int j, int k) const {
        if (!aliased) return (*f)(i, j, k);
        const long long off = (long long)(i - 1) + (long long)(j - 1) * nx + (long long)(k - 1) * nx * ny;
        if (off < 0 || off >= (long long)f->size()) return 0.0;
        return f->d[(size_t)off];
    }
};

inline void gradient_phi_gauss(const PhiRef& Phi, F1& Dxm, F1& Dym, F1& Dzm, int i, int j, int k,
                               double g[3]) {
    const double Phiface_e = 0.5 * (Phi(i + 1, j, k) + Phi(i, j, k));
    const double Phiface_w = 0.5 * (Phi(i - 1, j, k) + Phi(i, j, k));
    const double Phiface_n = 0.5 * (Phi(i, j + 1, k) + Phi(i, j, k));
    const double Phiface_s = 0.5 * (Phi(i, j - 1, k) + Phi(i, j, k));
    const double Phiface_f = 0.5 * (Phi(i, j, k + 1) + Phi(i, j, k));
    const double Phiface_b = 0.5 * (Phi(i, j, k - 1) + Phi(i, j, k));
    double d1 = Phiface_w * (-1) * (Dym(j) * Dzm(k)) + Phiface_e * (1) * (Dym(j) * Dzm(k));
    double d2 = Phiface_s * (-1) * (Dxm(i) * Dzm(k)) + Phiface_n * (1) * (Dxm(i) * Dzm(k));
    double d3 = Phiface_b * (-1) * (Dxm(i) * Dym(j)) + Phiface_f * (1) * (Dxm(i) * Dym(j));
    const double fact = 1.0 / (Dxm(i) * Dym(j) * Dzm(k));
    g[0] = fact * d1; g[1] = fact * d2; g[2] = fact * d3;
}

}  // namespace

extern "C" {

orc* orc_create(const ntcfd_params* p) {
    if (!p || p->nx < 2 || p->ny < 2 || p->nz < 2) return nullptr;
    orc* o = new orc();
    o->prm = *p;
    o->nx = p->nx; o->ny = p->ny; o->nz = p->nz;
    o->dt = p->dt;
    o->nu = 1. / p->Re;  // reading_data.f90:38
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    o->X.init(-1, nx + 3); o->Y.init(-1, ny + 3); o->Z.init(-1, nz + 3);
    o->iDx.init(-1, nx + 2); o->Dxs.init(-1, nx + 2);
    o->iDy.init(-1, ny + 2); o->Dys.init(-1, ny + 2);
    o->iDz.init(-1, nz + 2); o->Dzs.init(-1, nz + 2);
    F3* halo[] = {&o->u, &o->v, &o->w, &o->p, &o->u1, &o->v1, &o->w1, &o->u2, &o->v2, &o->w2,
                  &o->us, &o->vs, &o->ws, &o->FX, &o->FY, &o->FZ, &o->ETA};
    for (F3* a : halo) a->init(-1, nx + 2, ny + 2, nz + 2);
    F3* inner[] = {&o->pre, &o->uc, &o->vc, &o->wc, &o->Viseff};
    for (F3* a : inner) a->init(1, nx, ny, nz);
    o->FXz.init(nx, ny); o->FYz.init(nx, ny);
    o->FXy.assign(nx, 0.0); o->FYy.assign(nx, 0.0);
    return o;
}

void orc_destroy(orc* o) { delete o; }

void orc_set_threads(orc* o, int n) {
    o->nthreads = n < 1 ? 1 : n;
#ifdef _OPENMP
    omp_set_num_threads(o->nthreads);
#endif
}

int orc_set_metrics(orc* o, const double* iDx, const double* Dxs, const double* iDy,
                    const double* Dys, const double* iDz, const double* Dzs) {
    std::memcpy(o->iDx.d.data(), iDx, sizeof(double) * (o->nx + 4));
    std::memcpy(o->Dxs.d.data(), Dxs, sizeof(double) * (o->nx + 4));
    std::memcpy(o->iDy.d.data(), iDy, sizeof(double) * (o->ny + 4));
    std::memcpy(o->Dys.d.data(), Dys, sizeof(double) * (o->ny + 4));
    std::memcpy(o->iDz.d.data(), iDz, sizeof(double) * (o->nz + 4));
    std::memcpy(o->Dzs.d.data(), Dzs, sizeof(double) * (o->nz + 4));
    return 0;
}

int orc_set_coords(orc* o, const double* X, const double* Y, const double* Z) {
    std::memcpy(o->X.d.data(), X, sizeof(double) * (o->nx + 5));
    std::memcpy(o->Y.d.data(), Y, sizeof(double) * (o->ny + 5));
    std::memcpy(o->Z.d.data(), Z, sizeof(double) * (o->nz + 5));
    return 0;
}

int orc_get_coords(orc* o, double* X, double* Y, double* Z) {
    std::memcpy(X, o->X.d.data(), sizeof(double) * (o->nx + 5));
    std::memcpy(Y, o->Y.d.data(), sizeof(double) * (o->ny + 5));
    std::memcpy(Z, o->Z.d.data(), sizeof(double) * (o->nz + 5));
    return 0;
}

static std::vector<double>* field_by_name(orc* o, const char* name) {
    const std::string n(name);
    if (n == "u") return &o->u.d;
    if (n == "v") return &o->v.d;
    if (n == "w") return &o->w.d;
    if (n == "p") return &o->p.d;
    if (n == "u1") return &o->u1.d;
    if (n == "v1") return &o->v1.d;
    if (n == "w1") return &o->w1.d;
    if (n == "u2") return &o->u2.d;
    if (n == "v2") return &o->v2.d;
    if (n == "w2") return &o->w2.d;
    if (n == "u_star") return &o->us.d;
    if (n == "v_star") return &o->vs.d;
    if (n == "w_star") return &o->ws.d;
    if (n == "FX") return &o->FX.d;
    if (n == "FY") return &o->FY.d;
    if (n == "FZ") return &o->FZ.d;
    if (n == "ETA") return &o->ETA.d;
    if (n == "pre") return &o->pre.d;
    if (n == "uc") return &o->uc.d;
    if (n == "vc") return &o->vc.d;
    if (n == "wc") return &o->wc.d;
    if (n == "Viseff") return &o->Viseff.d;
    if (n == "FXz") return &o->FXz.d;
    if (n == "FYz") return &o->FYz.d;
    if (n == "FXy") return &o->FXy;
    if (n == "FYy") return &o->FYy;
    return nullptr;
}

int orc_set_field(orc* o, const char* name, const double* src) {
    auto* f = field_by_name(o, name);
    if (!f) return -1;
    std::memcpy(f->data(), src, sizeof(double) * f->size());
    return 0;
}

int orc_get_field(orc* o, const char* name, double* dst) {
    auto* f = field_by_name(o, name);
    if (!f) return -1;
    std::memcpy(dst, f->data(), sizeof(double) * f->size());
    return 0;
}

long orc_field_size(orc* o, const char* name) {
    auto* f = field_by_name(o, name);
    return f ? (long)f->size() : -1;
}

// initial_conditions.f90:9-29 -- every field zero.
void orc_initial_conditions(orc* o) {
    F3* halo[] = {&o->u, &o->v, &o->w, &o->p, &o->u1, &o->v1, &o->w1, &o->u2, &o->v2, &o->w2,
                  &o->us, &o->vs, &o->ws, &o->ETA};
    for (F3* a : halo) std::fill(a->d.begin(), a->d.end(), 0.0);
}

void orc_boundary_conditions(orc* o) {
    bc_velocity(o);
    bc_copies_and_pressure(o);
}

// smagorinsky.f90:1-37 -- CalculateSmagorinskyViscosity.
void orc_smagorinsky(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    const bool aliased = o->prm.smag_mode == NTCFD_SMAG_REF_ALIASED;
    const PhiRef U{&o->u, nx, ny, aliased}, V{&o->v, nx, ny, aliased}, W{&o->w, nx, ny, aliased};
    const double Cs = o->prm.Cs;
    const double third = (double)(1.f / 3.f);  // 1./3. is a default-real literal
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double dudx[3], dvdx[3], dwdx[3];
                gradient_phi_gauss(U, o->Dxs, o->iDy, o->iDz, i, j, k, dudx);
                gradient_phi_gauss(V, o->iDx, o->Dys, o->iDz, i, j, k, dvdx);
                gradient_phi_gauss(W, o->iDx, o->iDy, o->Dzs, i, j, k, dwdx);
                double mutsgs = std::fabs(2 * (dudx[0] * dudx[0]) + 2 * (dvdx[1] * dvdx[1]) +
                                          2 * (dwdx[2] * dwdx[2]) +
                                          (dudx[1] + dvdx[0]) * (dudx[1] + dvdx[0]) +
                                          (dudx[2] + dwdx[0]) * (dudx[2] + dwdx[0]) +
                                          (dvdx[2] + dwdx[1]) * (dvdx[2] + dwdx[1]));
                const double delta = std::pow(o->iDx(i) * o->iDy(j) * o->iDz(k), third);
                mutsgs = (Cs * delta) * (Cs * delta) * std::sqrt(mutsgs);
                o->Viseff(i, j, k) = mutsgs;
            }
    }
}

// discretisation_QUICK_centre.f90:1-345.
static void predictor_quick_centre(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    F3 &u = o->u, &v = o->v, &w = o->w;
    F1 &iDx = o->iDx, &Dxs = o->Dxs, &iDy = o->iDy, &Dys = o->Dys, &iDz = o->iDz, &Dzs = o->Dzs;
    const double dt = o->dt, nu = o->nu;
    const int LES = o->prm.LES;
    // u_star (discretisation_QUICK_centre.f90:7-117)
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double u_tilde_x1 = 0.5 * (u(i + 1, j, k) + u(i, j, k));
                const double u_tilde_x2 = 0.5 * (u(i - 1, j, k) + u(i, j, k));
                const double v_tilde_x1 = 0.5 * (v(i, j, k) + v(i + 1, j, k));
                const double v_tilde_x2 = 0.5 * (v(i, j - 1, k) + v(i + 1, j - 1, k));
                const double w_tilde_x1 = 0.5 * (w(i + 1, j, k) + w(i, j, k));
                const double w_tilde_x2 = 0.5 * (w(i, j, k - 1) + w(i + 1, j, k - 1));
                double ue, uw, un, us, uf, ub;
                if (u_tilde_x1 > 0)
                    ue = 0.5 * (u(i, j, k) + u(i + 1, j, k)) - 0.125 * iDx(i + 1) * iDx(i + 1) / Dxs(i) *
                         ((u(i + 1, j, k) - u(i, j, k)) / iDx(i + 1) - (u(i, j, k) - u(i - 1, j, k)) / iDx(i));
                else
                    ue = 0.5 * (u(i, j, k) + u(i + 1, j, k)) - 0.125 * iDx(i + 1) * iDx(i + 1) / Dxs(i + 1) *
                         ((u(i + 2, j, k) - u(i + 1, j, k)) / iDx(i + 2) - (u(i + 1, j, k) - u(i, j, k)) / iDx(i + 1));
                if (u_tilde_x2 > 0)
                    uw = 0.5 * (u(i - 1, j, k) + u(i, j, k)) - 0.125 * iDx(i) * iDx(i) / Dxs(i - 1) *
                         ((u(i, j, k) - u(i - 1, j, k)) / iDx(i) - (u(i - 1, j, k) - u(i - 2, j, k)) / iDx(i - 1));
                else
                    uw = 0.5 * (u(i - 1, j, k) + u(i, j, k)) - 0.125 * iDx(i) * iDx(i) / Dxs(i) *
                         ((u(i + 1, j, k) - u(i, j, k)) / iDx(i + 1) - (u(i, j, k) - u(i - 1, j, k)) / iDx(i));
                if (v_tilde_x1 > 0)
                    un = 0.5 * (u(i, j, k) + u(i, j + 1, k)) - 0.125 * Dys(j) * Dys(j) / iDy(j) *
                         ((u(i, j + 1, k) - u(i, j, k)) / Dys(j) - (u(i, j, k) - u(i, j - 1, k)) / Dys(j - 1));
                else
                    un = 0.5 * (u(i, j, k) + u(i, j + 1, k)) - 0.125 * Dys(j) * Dys(j) / iDy(j + 1) *
                         ((u(i, j + 2, k) - u(i, j + 1, k)) / Dys(j + 1) - (u(i, j + 1, k) - u(i, j, k)) / Dys(j));
                if (v_tilde_x2 > 0)
                    us = 0.5 * (u(i, j - 1, k) + u(i, j, k)) - 0.125 * Dys(j - 1) * Dys(j - 1) / iDy(j - 1) *
                         ((u(i, j, k) - u(i, j - 1, k)) / Dys(j - 1) - (u(i, j - 1, k) - u(i, j - 2, k)) / Dys(j - 2));
                else
                    us = 0.5 * (u(i, j - 1, k) + u(i, j, k)) - 0.125 * Dys(j - 1) * Dys(j - 1) / iDy(j) *
                         ((u(i, j + 1, k) - u(i, j, k)) / Dys(j) - (u(i, j, k) - u(i, j - 1, k)) / Dys(j - 1));
                if (w_tilde_x1 > 0)
                    uf = 0.5 * (u(i, j, k) + u(i, j, k + 1)) - 0.125 * Dzs(k) * Dzs(k) / iDz(k) *
                         ((u(i, j, k + 1) - u(i, j, k)) / Dzs(k) - (u(i, j, k) - u(i, j, k - 1)) / Dzs(k - 1));
                else
                    uf = 0.5 * (u(i, j, k) + u(i, j, k + 1)) - 0.125 * Dzs(k) * Dzs(k) / iDz(k + 1) *
                         ((u(i, j, k + 2) - u(i, j, k + 1)) / Dzs(k + 1) - (u(i, j, k + 1) - u(i, j, k)) / Dzs(k));
                if (w_tilde_x2 > 0)
                    ub = 0.5 * (u(i, j, k - 1) + u(i, j, k)) - 0.125 * Dzs(k - 1) * Dzs(k - 1) / iDz(k - 1) *
                         ((u(i, j, k) - u(i, j, k - 1)) / Dzs(k - 1) - (u(i, j, k - 1) - u(i, j, k - 2)) / Dzs(k - 2));
                else
                    ub = 0.5 * (u(i, j, k - 1) + u(i, j, k)) - 0.125 * Dzs(k - 1) * Dzs(k - 1) / iDz(k) *
                         ((u(i, j, k + 1) - u(i, j, k)) / Dzs(k) - (u(i, j, k) - u(i, j, k - 1)) / Dzs(k - 1));
                const double nut = o->Viseff(i, j, k);
                const double nue = nu + nut * LES;
                o->us(i, j, k) = u(i, j, k) - dt * (u_tilde_x1 * ue - u_tilde_x2 * uw) / Dxs(i)
                                 - dt * (v_tilde_x1 * un - v_tilde_x2 * us) / iDy(j)
                                 - dt * (w_tilde_x1 * uf - w_tilde_x2 * ub) / iDz(k)
                                 + nue * dt * ((u(i + 1, j, k) - u(i, j, k)) / iDx(i + 1) - (u(i, j, k) - u(i - 1, j, k)) / iDx(i)) / Dxs(i)
                                 + nue * dt * ((u(i, j + 1, k) - u(i, j, k)) / Dys(j) - (u(i, j, k) - u(i, j - 1, k)) / Dys(j - 1)) / iDy(j)
                                 + nue * dt * ((u(i, j, k + 1) - u(i, j, k)) / Dzs(k) - (u(i, j, k) - u(i, j, k - 1)) / Dzs(k - 1)) / iDz(k);
            }
    }
    // v_star (discretisation_QUICK_centre.f90:123-230)
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double u_tilde_y1 = 0.5 * (u(i, j, k) + u(i, j + 1, k));
                const double u_tilde_y2 = 0.5 * (u(i - 1, j, k) + u(i - 1, j + 1, k));
                const double v_tilde_y1 = 0.5 * (v(i, j, k) + v(i, j + 1, k));
                const double v_tilde_y2 = 0.5 * (v(i, j - 1, k) + v(i, j, k));
                const double w_tilde_y1 = 0.5 * (w(i, j, k) + w(i, j + 1, k));
                const double w_tilde_y2 = 0.5 * (w(i, j, k - 1) + w(i, j + 1, k - 1));
                double ve, vw, vn, vs, vf, vb;
                if (u_tilde_y1 > 0)
                    ve = 0.5 * (v(i, j, k) + v(i + 1, j, k)) - 0.125 * Dxs(i) * Dxs(i) / iDx(i) *
                         ((v(i + 1, j, k) - v(i, j, k)) / Dxs(i) - (v(i, j, k) - v(i - 1, j, k)) / Dxs(i - 1));
                else
                    ve = 0.5 * (v(i, j, k) + v(i + 1, j, k)) - 0.125 * Dxs(i) * Dxs(i) / iDx(i + 1) *
                         ((v(i + 2, j, k) - v(i + 1, j, k)) / Dxs(i + 1) - (v(i + 1, j, k) - v(i, j, k)) / Dxs(i));
                if (u_tilde_y2 > 0)
                    vw = 0.5 * (v(i - 1, j, k) + v(i, j, k)) - 0.125 * Dxs(i - 1) * Dxs(i - 1) / iDx(i - 1) *
                         ((v(i, j, k) - v(i - 1, j, k)) / Dxs(i - 1) - (v(i - 1, j, k) - v(i - 2, j, k)) / Dxs(i - 2));
                else
                    vw = 0.5 * (v(i - 1, j, k) + v(i, j, k)) - 0.125 * Dxs(i - 1) * Dxs(i - 1) / iDx(i) *
                         ((v(i + 1, j, k) - v(i, j, k)) / Dxs(i) - (v(i, j, k) - v(i - 1, j, k)) / Dxs(i - 1));
                if (v_tilde_y1 > 0)
                    vn = 0.5 * (v(i, j, k) + v(i, j + 1, k)) - 0.125 * iDy(j + 1) * iDy(j + 1) / Dys(j) *
                         ((v(i, j + 1, k) - v(i, j, k)) / iDy(j + 1) - (v(i, j, k) - v(i, j - 1, k)) / iDy(j));
                else
                    vn = 0.5 * (v(i, j, k) + v(i, j + 1, k)) - 0.125 * iDy(j + 1) * iDy(j + 1) / Dys(j + 1) *
                         ((v(i, j + 2, k) - v(i, j + 1, k)) / iDy(j + 2) - (v(i, j + 1, k) - v(i, j, k)) / iDy(j + 1));
                if (v_tilde_y2 > 0)
                    vs = 0.5 * (v(i, j - 1, k) + v(i, j, k)) - 0.125 * iDy(j) * iDy(j) / Dys(j - 1) *
                         ((v(i, j, k) - v(i, j - 1, k)) / iDy(j) - (v(i, j - 1, k) - v(i, j - 2, k)) / iDy(j - 1));
                else
                    vs = 0.5 * (v(i, j - 1, k) + v(i, j, k)) - 0.125 * iDy(j) * iDy(j) / Dys(j) *
                         ((v(i, j + 1, k) - v(i, j, k)) / iDy(j + 1) - (v(i, j, k) - v(i, j - 1, k)) / iDy(j));
                if (w_tilde_y1 > 0)
                    vf = 0.5 * (v(i, j, k) + v(i, j, k + 1)) - 0.125 * Dzs(k) * Dzs(k) / iDz(k) *
                         ((v(i, j, k + 1) - v(i, j, k)) / Dzs(k) - (v(i, j, k) - v(i, j, k - 1)) / Dzs(k - 1));
                else
                    vf = 0.5 * (v(i, j, k) + v(i, j, k + 1)) - 0.125 * Dzs(k) * Dzs(k) / iDz(k + 1) *
                         ((v(i, j, k + 2) - v(i, j, k + 1)) / Dzs(k + 1) - (v(i, j, k + 1) - v(i, j, k)) / Dzs(k));
                if (w_tilde_y2 > 0)
                    vb = 0.5 * (v(i, j, k - 1) + v(i, j, k)) - 0.125 * Dzs(k - 1) * Dzs(k - 1) / iDz(k - 1) *
                         ((v(i, j, k) - v(i, j, k - 1)) / Dzs(k - 1) - (v(i, j, k - 1) - v(i, j, k - 2)) / Dzs(k - 2));
                else
                    vb = 0.5 * (v(i, j, k - 1) + v(i, j, k)) - 0.125 * Dzs(k - 1) * Dzs(k - 1) / iDz(k) *
                         ((v(i, j, k + 1) - v(i, j, k)) / Dzs(k) - (v(i, j, k) - v(i, j, k - 1)) / Dzs(k - 1));
                const double nut = o->Viseff(i, j, k);
                const double nue = nu + nut * LES;
                o->vs(i, j, k) = v(i, j, k) - dt * (u_tilde_y1 * ve - u_tilde_y2 * vw) / iDx(i)
                                 - dt * (v_tilde_y1 * vn - v_tilde_y2 * vs) / Dys(j)
                                 - dt * (w_tilde_y1 * vf - w_tilde_y2 * vb) / iDz(k)
                                 + nue * dt * ((v(i + 1, j, k) - v(i, j, k)) / Dxs(i) - (v(i, j, k) - v(i - 1, j, k)) / Dxs(i - 1)) / iDx(i)
                                 + nue * dt * ((v(i, j + 1, k) - v(i, j, k)) / iDy(j + 1) - (v(i, j, k) - v(i, j - 1, k)) / iDy(j)) / Dys(j)
                                 + nue * dt * ((v(i, j, k + 1) - v(i, j, k)) / Dzs(k) - (v(i, j, k) - v(i, j, k - 1)) / Dzs(k - 1)) / iDz(k);
            }
    }
    // w_star (discretisation_QUICK_centre.f90:236-342)
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double u_tilde_z1 = 0.5 * (u(i, j, k + 1) + u(i, j, k));
                const double u_tilde_z2 = 0.5 * (u(i - 1, j, k + 1) + u(i - 1, j, k));
                const double v_tilde_z1 = 0.5 * (v(i, j, k) + v(i, j, k + 1));
                const double v_tilde_z2 = 0.5 * (v(i, j - 1, k + 1) + v(i, j - 1, k));
                const double w_tilde_z1 = 0.5 * (w(i, j, k + 1) + w(i, j, k));
                const double w_tilde_z2 = 0.5 * (w(i, j, k) + w(i, j, k - 1));
                double we, ww, wn, ws, wf, wb;
                if (u_tilde_z1 > 0)
                    we = 0.5 * (w(i, j, k) + w(i + 1, j, k)) - 0.125 * Dxs(i) * Dxs(i) / iDx(i) *
                         ((w(i + 1, j, k) - w(i, j, k)) / Dxs(i) - (w(i, j, k) - w(i - 1, j, k)) / Dxs(i - 1));
                else
                    we = 0.5 * (w(i, j, k) + w(i + 1, j, k)) - 0.125 * Dxs(i) * Dxs(i) / iDx(i + 1) *
                         ((w(i + 2, j, k) - w(i + 1, j, k)) / Dxs(i + 1) - (w(i + 1, j, k) - w(i, j, k)) / Dxs(i));
                if (u_tilde_z2 > 0)
                    ww = 0.5 * (w(i - 1, j, k) + w(i, j, k)) - 0.125 * Dxs(i - 1) * Dxs(i - 1) / iDx(i - 1) *
                         ((w(i, j, k) - w(i - 1, j, k)) / Dxs(i - 1) - (w(i - 1, j, k) - w(i - 2, j, k)) / Dxs(i - 2));
                else
                    ww = 0.5 * (w(i - 1, j, k) + w(i, j, k)) - 0.125 * Dxs(i - 1) * Dxs(i - 1) / iDx(i) *
                         ((w(i + 1, j, k) - w(i, j, k)) / Dxs(i) - (w(i, j, k) - w(i - 1, j, k)) / Dxs(i - 1));
                if (v_tilde_z1 > 0)
                    wn = 0.5 * (w(i, j, k) + w(i, j + 1, k)) - 0.125 * Dys(j) * Dys(j) / iDy(j) *
                         ((w(i, j + 1, k) - w(i, j, k)) / Dys(j) - (w(i, j, k) - w(i, j - 1, k)) / Dys(j - 1));
                else
                    wn = 0.5 * (w(i, j, k) + w(i, j + 1, k)) - 0.125 * Dys(j) * Dys(j) / iDy(j + 1) *
                         ((w(i, j + 2, k) - w(i, j + 1, k)) / Dys(j + 1) - (w(i, j + 1, k) - w(i, j, k)) / Dys(j));
                if (v_tilde_z2 > 0)
                    ws = 0.5 * (w(i, j - 1, k) + w(i, j, k)) - 0.125 * Dys(j - 1) * Dys(j - 1) / iDy(j - 1) *
                         ((w(i, j, k) - w(i, j - 1, k)) / Dys(j - 1) - (w(i, j - 1, k) - w(i, j - 2, k)) / Dys(j - 2));
                else
                    ws = 0.5 * (w(i, j - 1, k) + w(i, j, k)) - 0.125 * Dys(j - 1) * Dys(j - 1) / iDy(j) *
                         ((w(i, j + 1, k) - w(i, j, k)) / Dys(j) - (w(i, j, k) - w(i, j - 1, k)) / Dys(j - 1));
                if (w_tilde_z1 > 0)
                    wf = 0.5 * (w(i, j, k) + w(i, j, k + 1)) - 0.125 * iDz(k + 1) * iDz(k + 1) / Dzs(k) *
                         ((w(i, j, k + 1) - w(i, j, k)) / iDz(k + 1) - (w(i, j, k) - w(i, j, k - 1)) / iDz(k));
                else
                    wf = 0.5 * (w(i, j, k) + w(i, j, k + 1)) - 0.125 * iDz(k + 1) * iDz(k + 1) / Dzs(k + 1) *
                         ((w(i, j, k + 2) - w(i, j, k + 1)) / iDz(k + 2) - (w(i, j, k + 1) - w(i, j, k)) / iDz(k + 1));
                if (w_tilde_z2 > 0)
                    wb = 0.5 * (w(i, j, k - 1) + w(i, j, k)) - 0.125 * iDz(k) * iDz(k) / Dzs(k - 1) *
                         ((w(i, j, k) - w(i, j, k - 1)) / iDz(k) - (w(i, j, k - 1) - w(i, j, k - 2)) / iDz(k - 1));
                else
                    wb = 0.5 * (w(i, j, k - 1) + w(i, j, k)) - 0.125 * iDz(k) * iDz(k) / Dzs(k) *
                         ((w(i, j, k + 1) - w(i, j, k)) / iDz(k + 1) - (w(i, j, k) - w(i, j, k - 1)) / iDz(k));
                const double nut = o->Viseff(i, j, k);
                const double nue = nu + nut * LES;
                o->ws(i, j, k) = w(i, j, k) - dt * (u_tilde_z1 * we - u_tilde_z2 * ww) / iDx(i)
                                 - dt * (v_tilde_z1 * wn - v_tilde_z2 * ws) / iDy(j)
                                 - dt * (w_tilde_z1 * wf - w_tilde_z2 * wb) / Dzs(k)
                                 + nue * dt * ((w(i + 1, j, k) - w(i, j, k)) / Dxs(i) - (w(i, j, k) - w(i - 1, j, k)) / Dxs(i - 1)) / iDx(i)
                                 + nue * dt * ((w(i, j + 1, k) - w(i, j, k)) / Dys(j) - (w(i, j, k) - w(i, j - 1, k)) / Dys(j - 1)) / iDy(j)
                                 + nue * dt * ((w(i, j, k + 1) - w(i, j, k)) / iDz(k + 1) - (w(i, j, k) - w(i, j, k - 1)) / iDz(k)) / Dzs(k);
            }
    }
}

}  // extern "C"

namespace {

// ----------------------------------------------- uncalled K2 schemes ----
// discretisation_QUICK.f90:1-415, discretisation_upwind.f90:1-275 and
// discretisation_centre.f90:1-134.  The reference never calls them and
// cannot compile them (their flag Q1 is undeclared under implicit none);
// here Q1 is prm.LES.  u* on i = 1..nx-1, v* on j = 1..ny-1, w* on
// k = 1..nz-1; the wall faces keep the u -> u_star copy of the last
// boundary_conditions call.  Every expression keeps the reference's operand
// order; x**0.5 is evaluated as sqrt(x).

// QUICK face value between nodes a and a+1 of the line f(.).  stag: the line
// runs along the component's own axis (node spacing iD, the factor
// 0.125 iD(a+1)^2 / Ds), else across it (node spacing Ds, factor
// 0.125 Ds(a)^2 / iD); pos selects the upstream stencil of the positive
// branch (discretisation_QUICK.f90:11-33 and their siblings).
template <class Fn>
double quick_face_ref(bool pos, bool stag, const Fn& f, int a, F1& iD, F1& Ds) {
    const double mid = 0.5 * (f(a) + f(a + 1));
    if (stag) {
        if (pos)
            return mid - 0.125 * iD(a + 1) * iD(a + 1) / Ds(a) * ((f(a + 1) - f(a)) / iD(a + 1) - (f(a) - f(a - 1)) / iD(a));
        return mid - 0.125 * iD(a + 1) * iD(a + 1) / Ds(a + 1) *
                     ((f(a + 2) - f(a + 1)) / iD(a + 2) - (f(a + 1) - f(a)) / iD(a + 1));
    }
    if (pos) return mid - 0.125 * Ds(a) * Ds(a) / iD(a) * ((f(a + 1) - f(a)) / Ds(a) - (f(a) - f(a - 1)) / Ds(a - 1));
    return mid - 0.125 * Ds(a) * Ds(a) / iD(a + 1) * ((f(a + 2) - f(a + 1)) / Ds(a + 1) - (f(a + 1) - f(a)) / Ds(a));
}

inline double p2(double x) { return x * x; }

// The Q1 = 1 blocks (discretisation_upwind.f90:66-80, 156-170, 245-259; the
// same text in the other two files): eddy viscosity at the u, v, w points.
double nut_u_ref(orc* o, int i, int j, int k) {
    F3 &u = o->u, &v = o->v, &w = o->w;
    F1 &Dxs = o->Dxs, &iDy = o->iDy, &iDz = o->iDz;
    const double Cs = o->prm.Cs;
    const double delta = std::pow(Dxs(i) * iDy(j) * iDz(k), (double)(1.f / 3.f));
    const double s =
        0.5 * (1 / Dxs(i) / Dxs(i)) * p2((u(i + 1, j, k) + u(i, j, k)) - (u(i, j, k) + u(i - 1, j, k))) +
        0.5 * (1 / iDy(j) / iDy(j)) * p2((v(i + 1, j, k) + v(i, j, k)) - (v(i + 1, j - 1, k) + v(i, j - 1, k))) +
        0.5 * (1 / iDz(k) / iDz(k)) * p2((w(i + 1, j, k) + w(i, j, k)) - (w(i + 1, j, k - 1) + w(i, j, k - 1))) +
        p2(0.5 * (1 / iDy(j)) * ((u(i, j + 1, k) + u(i, j, k)) - (u(i, j, k) + u(i, j - 1, k))) +
           0.5 * (1 / Dxs(i)) * ((v(i + 1, j, k) + v(i + 1, j - 1, k)) - (v(i, j, k) + v(i, j - 1, k)))) +
        p2(0.5 * (1 / iDz(k)) * ((u(i, j, k + 1) + u(i, j, k)) - (u(i, j, k) + u(i, j, k - 1))) +
           0.5 * (1 / Dxs(i)) * ((w(i + 1, j, k) + w(i + 1, j, k - 1)) - (w(i, j, k) + w(i, j, k - 1)))) +
        p2(0.5 * (1 / iDz(k)) * ((v(i + 1, j, k + 1) + v(i, j - 1, k)) - (v(i + 1, j, k - 1) + v(i, j - 1, k))) +
           0.5 * (1 / iDy(j)) * ((w(i + 1, j + 1, k) + w(i, j, k - 1)) - (w(i + 1, j - 1, k) + w(i, j, k - 1))));
    return p2(Cs * delta) * std::sqrt(s);
}

double nut_v_ref(orc* o, int i, int j, int k) {
    F3 &u = o->u, &v = o->v, &w = o->w;
    F1 &iDx = o->iDx, &Dys = o->Dys, &iDz = o->iDz;
    const double Cs = o->prm.Cs;
    const double delta = std::pow(iDx(i) * Dys(j) * iDz(k), (double)(1.f / 3.f));
    const double s =
        0.5 * (1 / iDx(i) / iDx(i)) * p2((u(i, j + 1, k) + u(i, j, k)) - (u(i - 1, j + 1, k) + u(i - 1, j, k))) +
        0.5 * (1 / Dys(j) / Dys(j)) * p2((v(i, j + 1, k) + v(i, j, k)) - (v(i, j, k) + v(i, j - 1, k))) +
        0.5 * (1 / iDz(k) / iDz(k)) * p2((w(i, j + 1, k) + w(i, j, k)) - (w(i, j + 1, k - 1) + w(i, j, k - 1))) +
        p2(0.5 * (1 / Dys(j)) * ((u(i, j + 1, k) + u(i - 1, j + 1, k)) - (u(i, j, k) + u(i - 1, j, k))) +
           0.5 * (1 / iDx(i)) * ((v(i + 1, j, k) + v(i, j, k)) - (v(i, j, k) + v(i - 1, j, k)))) +
        p2(0.5 * (1 / iDz(k)) * ((u(i, j + 1, k + 1) + u(i - 1, j, k)) - (u(i, j + 1, k - 1) + u(i - 1, j, k - 1))) +
           0.5 * (1 / iDx(i)) * ((w(i + 1, j + 1, k) + w(i, j, k - 1)) - (w(i - 1, j + 1, k) + w(i, j, k - 1)))) +
        p2(0.5 * (1 / iDz(k)) * ((v(i, j, k + 1) + v(i, j, k)) - (v(i, j, k - 1) + v(i, j, k))) +
           0.5 * (1 / Dys(j)) * ((w(i, j + 1, k) + w(i, j + 1, k - 1)) - (w(i, j, k) + w(i, j, k - 1))));
    return p2(Cs * delta) * std::sqrt(s);
}

double nut_w_ref(orc* o, int i, int j, int k) {
    F3 &u = o->u, &v = o->v, &w = o->w;
    F1 &iDx = o->iDx, &iDy = o->iDy, &Dzs = o->Dzs;
    const double Cs = o->prm.Cs;
    const double delta = std::pow(iDx(i) * iDy(j) * Dzs(k), (double)(1.f / 3.f));
    const double s =
        0.5 * (1 / iDx(i) / iDx(i)) * p2((u(i, j, k + 1) + u(i, j, k)) - (u(i - 1, j, k + 1) + u(i - 1, j, k))) +
        0.5 * (1 / iDy(j) / iDy(j)) * p2((v(i, j, k + 1) + v(i, j, k)) - (v(i, j - 1, k + 1) + v(i, j - 1, k))) +
        0.5 * (1 / Dzs(k) / Dzs(k)) * p2((w(i, j, k + 1) + w(i, j, k)) - (w(i, j, k) + w(i, j, k - 1))) +
        p2(0.5 * (1 / iDy(j)) * ((u(i, j + 1, k) + u(i, j, k)) - (u(i, j, k) + u(i, j - 1, k))) +
           0.5 * (1 / iDx(i)) * ((v(i + 1, j, k + 1) + v(i, j - 1, k)) - (v(i - 1, j, k + 1) + v(i, j - 1, k)))) +
        p2(0.5 * (1 / Dzs(k)) * ((u(i, j, k + 1) + u(i - 1, j, k + 1)) - (u(i, j, k) + u(i - 1, j, k))) +
           0.5 * (1 / iDx(i)) * ((w(i + 1, j, k) + w(i, j, k)) - (w(i - 1, j, k) + w(i, j, k)))) +
        p2(0.5 * (1 / Dzs(k)) * ((v(i, j, k + 1) + v(i, j - 1, k + 1)) - (v(i, j, k) + v(i, j - 1, k))) +
           0.5 * (1 / iDy(j)) * ((w(i, j + 1, k) + w(i, j, k)) - (w(i, j - 1, k) + w(i, j, k))));
    return p2(Cs * delta) * std::sqrt(s);
}

void predictor_scheme(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz, scheme = o->prm.scheme;
    F3 &u = o->u, &v = o->v, &w = o->w;
    F1 &iDx = o->iDx, &Dxs = o->Dxs, &iDy = o->iDy, &Dys = o->Dys, &iDz = o->iDz, &Dzs = o->Dzs;
    const double dt = o->dt, nu = o->nu;
    const int Q1 = o->prm.LES;
    const bool quick = scheme == NTCFD_QUICK, upwind = scheme == NTCFD_UPWIND;
    // upwind face value: the upstream node when the advecting velocity is >= 0
    auto upw = [](double adv, double up, double down) { return adv >= 0 ? up : down; };
    // u_star (discretisation_QUICK.f90:7-143, _upwind.f90:7-92, _centre.f90:7-39)
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx - 1; ++i) {
                double cx, cy, cz;
                if (quick) {
                    const bool pu = u(i, j, k) > 0, pv = v(i, j, k) > 0, pw = w(i, j, k) > 0;
                    auto ux = [&](int a) { return u(a, j, k); };
                    auto uy = [&](int a) { return u(i, a, k); };
                    auto uz = [&](int a) { return u(i, j, a); };
                    auto vx0 = [&](int a) { return v(a, j, k); };
                    auto vx1 = [&](int a) { return v(a, j - 1, k); };
                    auto wx0 = [&](int a) { return w(a, j, k); };
                    auto wx1 = [&](int a) { return w(a, j, k - 1); };
                    const double ue = quick_face_ref(pu, true, ux, i, iDx, Dxs);
                    const double uw = quick_face_ref(pu, true, ux, i - 1, iDx, Dxs);
                    const double vnu = quick_face_ref(pu, false, vx0, i, iDx, Dxs);
                    const double vsu = quick_face_ref(pu, false, vx1, i, iDx, Dxs);
                    const double wfu = quick_face_ref(pu, false, wx0, i, iDx, Dxs);
                    const double wbu = quick_face_ref(pu, false, wx1, i, iDx, Dxs);
                    const double un = quick_face_ref(pv, false, uy, j, iDy, Dys);
                    const double us = quick_face_ref(pv, false, uy, j - 1, iDy, Dys);
                    const double uf = quick_face_ref(pw, false, uz, k, iDz, Dzs);
                    const double ub = quick_face_ref(pw, false, uz, k - 1, iDz, Dzs);
                    cx = dt * (ue * ue - uw * uw) / Dxs(i);
                    cy = dt * (un * vnu - us * vsu) / iDy(j);
                    cz = dt * (uf * wfu - ub * wbu) / iDz(k);
                } else {
                    const double ut1 = 0.5 * (u(i, j, k) + u(i + 1, j, k));
                    const double ut2 = upwind ? 0.5 * (u(i - 1, j, k) + u(i, j, k)) : 0.5 * (u(i, j, k) + u(i - 1, j, k));
                    const double vt1 = 0.5 * (v(i, j, k) + v(i + 1, j, k));
                    const double vt2 = 0.5 * (v(i, j - 1, k) + v(i + 1, j - 1, k));
                    const double wt1 = 0.5 * (w(i + 1, j, k) + w(i, j, k));
                    const double wt2 = 0.5 * (w(i, j, k - 1) + w(i + 1, j, k - 1));
                    if (upwind) {
                        cx = dt * (ut1 * upw(ut1, u(i, j, k), u(i + 1, j, k)) - ut2 * upw(ut2, u(i - 1, j, k), u(i, j, k))) / Dxs(i);
                        cy = dt * (vt1 * upw(vt1, u(i, j, k), u(i, j + 1, k)) - vt2 * upw(vt2, u(i, j - 1, k), u(i, j, k))) / iDy(j);
                        cz = dt * (wt1 * upw(wt1, u(i, j, k), u(i, j, k + 1)) - wt2 * upw(wt2, u(i, j, k - 1), u(i, j, k))) / iDz(k);
                    } else {
                        cx = dt * 0.5 * (ut1 * (u(i, j, k) + u(i + 1, j, k)) - ut2 * (u(i, j, k) + u(i - 1, j, k))) / Dxs(i);
                        cy = dt * 0.5 * (vt1 * (u(i, j, k) + u(i, j + 1, k)) - vt2 * (u(i, j, k) + u(i, j - 1, k))) / iDy(j);
                        cz = dt * 0.5 * (wt1 * (u(i, j, k) + u(i, j, k + 1)) - wt2 * (u(i, j, k) + u(i, j, k - 1))) / iDz(k);
                    }
                }
                const double nut = Q1 == 1 ? nut_u_ref(o, i, j, k) : 0.0;
                const double nue = nu + nut * Q1;
                o->us(i, j, k) = u(i, j, k) - cx - cy - cz
                    + nue * dt * ((u(i + 1, j, k) - u(i, j, k)) / iDx(i + 1) - (u(i, j, k) - u(i - 1, j, k)) / iDx(i)) / Dxs(i)
                    + nue * dt * ((u(i, j + 1, k) - u(i, j, k)) / Dys(j) - (u(i, j, k) - u(i, j - 1, k)) / Dys(j - 1)) / iDy(j)
                    + nue * dt * ((u(i, j, k + 1) - u(i, j, k)) / Dzs(k) - (u(i, j, k) - u(i, j, k - 1)) / Dzs(k - 1)) / iDz(k);
            }
    }
    // v_star (discretisation_QUICK.f90:145-283, _upwind.f90:94-181, _centre.f90:41-84)
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny - 1; ++j)
            for (int i = 1; i <= nx; ++i) {
                double cx, cy, cz;
                if (quick) {
                    const bool pu = u(i, j, k) > 0, pv = v(i, j, k) > 0, pw = w(i, j, k) > 0;
                    auto vx = [&](int a) { return v(a, j, k); };
                    auto vy = [&](int a) { return v(i, a, k); };
                    auto vz = [&](int a) { return v(i, j, a); };
                    auto uy0 = [&](int a) { return u(i, a, k); };
                    auto uy1 = [&](int a) { return u(i - 1, a, k); };
                    auto wy0 = [&](int a) { return w(i, a, k); };
                    auto wy1 = [&](int a) { return w(i, a, k - 1); };
                    const double ve = quick_face_ref(pu, false, vx, i, iDx, Dxs);
                    const double vw = quick_face_ref(pu, false, vx, i - 1, iDx, Dxs);
                    const double uev = quick_face_ref(pv, false, uy0, j, iDy, Dys);
                    const double uwv = quick_face_ref(pv, false, uy1, j, iDy, Dys);
                    const double vn = quick_face_ref(pv, true, vy, j, iDy, Dys);
                    const double vs = quick_face_ref(pv, true, vy, j - 1, iDy, Dys);
                    const double wfv = quick_face_ref(pv, false, wy0, j, iDy, Dys);
                    const double wbv = quick_face_ref(pv, false, wy1, j, iDy, Dys);
                    const double vf = quick_face_ref(pw, false, vz, k, iDz, Dzs);
                    const double vb = quick_face_ref(pw, false, vz, k - 1, iDz, Dzs);
                    cx = dt * (uev * ve - uwv * vw) / iDx(i);
                    cy = dt * (vn * vn - vs * vs) / Dys(j);
                    cz = dt * (vf * wfv - vb * wbv) / iDz(k);
                } else {
                    const double ut1 = 0.5 * (u(i, j, k) + u(i, j + 1, k));
                    const double ut2 = 0.5 * (u(i - 1, j, k) + u(i - 1, j + 1, k));
                    const double vt1 = 0.5 * (v(i, j, k) + v(i, j + 1, k));
                    const double vt2 = 0.5 * (v(i, j - 1, k) + v(i, j, k));
                    const double wt1 = 0.5 * (w(i, j, k) + w(i, j + 1, k));
                    const double wt2 = 0.5 * (w(i, j, k - 1) + w(i, j + 1, k - 1));
                    if (upwind) {
                        cx = dt * (ut1 * upw(ut1, v(i, j, k), v(i + 1, j, k)) - ut2 * upw(ut2, v(i - 1, j, k), v(i, j, k))) / iDx(i);
                        cy = dt * (vt1 * upw(vt1, v(i, j, k), v(i, j + 1, k)) - vt2 * upw(vt2, v(i, j - 1, k), v(i, j, k))) / Dys(j);
                        cz = dt * (wt1 * upw(wt1, v(i, j, k), v(i, j, k + 1)) - wt2 * upw(wt2, v(i, j, k - 1), v(i, j, k))) / iDz(k);
                    } else {
                        cx = dt * 0.5 * (ut1 * (v(i, j, k) + v(i + 1, j, k)) - ut2 * (v(i, j, k) + v(i - 1, j, k))) / iDx(i);
                        cy = dt * 0.5 * (vt1 * (v(i, j, k) + v(i, j + 1, k)) - vt2 * (v(i, j, k) + v(i, j - 1, k))) / Dys(j);
                        cz = dt * 0.5 * (wt1 * (v(i, j, k) + v(i, j, k + 1)) - wt2 * (v(i, j, k) + v(i, j, k - 1))) / iDz(k);
                    }
                }
                const double nut = Q1 == 1 ? nut_v_ref(o, i, j, k) : 0.0;
                const double nue = nu + nut * Q1;
                o->vs(i, j, k) = v(i, j, k) - cx - cy - cz
                    + nue * dt * ((v(i + 1, j, k) - v(i, j, k)) / Dxs(i) - (v(i, j, k) - v(i - 1, j, k)) / Dxs(i - 1)) / iDx(i)
                    + nue * dt * ((v(i, j + 1, k) - v(i, j, k)) / iDy(j + 1) - (v(i, j, k) - v(i, j - 1, k)) / iDy(j)) / Dys(j)
                    + nue * dt * ((v(i, j, k + 1) - v(i, j, k)) / Dzs(k) - (v(i, j, k) - v(i, j, k - 1)) / Dzs(k - 1)) / iDz(k);
            }
    }
    // w_star (discretisation_QUICK.f90:285-413, _upwind.f90:183-273, _centre.f90:86-132)
    for (int k = 1; k <= nz - 1; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double cx, cy, cz;
                if (quick) {
                    const bool pu = u(i, j, k) > 0, pv = v(i, j, k) > 0, pw = w(i, j, k) > 0;
                    auto wx = [&](int a) { return w(a, j, k); };
                    auto wy = [&](int a) { return w(i, a, k); };
                    auto wz = [&](int a) { return w(i, j, a); };
                    auto uz0 = [&](int a) { return u(i, j, a); };
                    auto uz1 = [&](int a) { return u(i - 1, j, a); };
                    auto vz0 = [&](int a) { return v(i, j, a); };
                    auto vz1 = [&](int a) { return v(i, j - 1, a); };
                    const double we = quick_face_ref(pu, false, wx, i, iDx, Dxs);
                    const double ww = quick_face_ref(pu, false, wx, i - 1, iDx, Dxs);
                    const double wn = quick_face_ref(pv, false, wy, j, iDy, Dys);
                    const double ws = quick_face_ref(pv, false, wy, j - 1, iDy, Dys);
                    const double uew = quick_face_ref(pw, false, uz0, k, iDz, Dzs);
                    const double uww = quick_face_ref(pw, false, uz1, k, iDz, Dzs);
                    const double vnw = quick_face_ref(pw, false, vz0, k, iDz, Dzs);
                    const double vsw = quick_face_ref(pw, false, vz1, k, iDz, Dzs);
                    const double wf = quick_face_ref(pw, true, wz, k, iDz, Dzs);
                    const double wb = quick_face_ref(pw, true, wz, k - 1, iDz, Dzs);
                    cx = dt * (uew * we - uww * ww) / iDx(i);
                    cy = dt * (vnw * wn - vsw * ws) / iDy(j);
                    cz = dt * (wf * wf - wb * wb) / Dzs(k);
                } else {
                    const double ut1 = 0.5 * (u(i, j, k + 1) + u(i, j, k));
                    const double ut2 = 0.5 * (u(i - 1, j, k + 1) + u(i - 1, j, k));
                    // discretisation_upwind.f90:195 reads v(i+1,j,k+1); the centre file v(i,j,k+1)
                    const double vt1 = upwind ? 0.5 * (v(i, j, k) + v(i + 1, j, k + 1)) : 0.5 * (v(i, j, k) + v(i, j, k + 1));
                    const double vt2 = 0.5 * (v(i, j - 1, k + 1) + v(i, j - 1, k));
                    const double wt1 = 0.5 * (w(i, j, k + 1) + w(i, j, k));
                    const double wt2 = 0.5 * (w(i, j, k) + w(i, j, k - 1));
                    if (upwind) {
                        cx = dt * (ut1 * upw(ut1, w(i, j, k), w(i + 1, j, k)) - ut2 * upw(ut2, w(i - 1, j, k), w(i, j, k))) / iDx(i);
                        cy = dt * (vt1 * upw(vt1, w(i, j, k), w(i, j + 1, k)) - vt2 * upw(vt2, w(i, j - 1, k), w(i, j, k))) / iDy(j);
                        cz = dt * (wt1 * upw(wt1, w(i, j, k), w(i, j, k + 1)) - wt2 * upw(wt2, w(i, j, k - 1), w(i, j, k))) / Dzs(k);
                    } else {
                        cx = dt * 0.5 * (ut1 * (w(i, j, k) + w(i + 1, j, k)) - ut2 * (w(i, j, k) + w(i - 1, j, k))) / iDx(i);
                        cy = dt * 0.5 * (vt1 * (w(i, j, k) + w(i, j + 1, k)) - vt2 * (w(i, j, k) + w(i, j - 1, k))) / iDy(j);
                        cz = dt * 0.5 * (wt1 * (w(i, j, k) + w(i, j, k + 1)) - wt2 * (w(i, j, k) + w(i, j, k - 1))) / Dzs(k);
                    }
                }
                const double nut = Q1 == 1 ? nut_w_ref(o, i, j, k) : 0.0;
                const double nue = nu + nut * Q1;
                o->ws(i, j, k) = w(i, j, k) - cx - cy - cz
                    + nue * dt * ((w(i + 1, j, k) - w(i, j, k)) / Dxs(i) - (w(i, j, k) - w(i - 1, j, k)) / Dxs(i - 1)) / iDx(i)
                    + nue * dt * ((w(i, j + 1, k) - w(i, j, k)) / Dys(j) - (w(i, j, k) - w(i, j - 1, k)) / Dys(j - 1)) / iDy(j)
                    + nue * dt * ((w(i, j, k + 1) - w(i, j, k)) / iDz(k + 1) - (w(i, j, k) - w(i, j, k - 1)) / iDz(k)) / Dzs(k);
            }
    }
}

}  // namespace

extern "C" {

// K2 of the configured scheme.
void orc_predictor(orc* o) {
    if (o->prm.scheme == NTCFD_QUICK_CENTRE) predictor_quick_centre(o);
    else predictor_scheme(o);
}

// GS.f90:1-106 -- SOR pressure solve.  LEX follows the reference loop order
// (k, j, i); REDBLACK updates cells with (i+j+k) even first, then odd.  The
// ghost values of p are not refreshed during the solve (they were set by the
// previous boundary_conditions call).  The divergence (mChange) does not
// change between sweeps, so it is evaluated once per cell per sweep as the
// reference does, without changing any result.
int orc_gauss_seidel(orc* o, int forced, double* last_change, int* converged) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    F3 &p = o->p, &us = o->us, &vs = o->vs, &ws = o->ws;
    F1 &iDx = o->iDx, &Dxs = o->Dxs, &iDy = o->iDy, &Dys = o->Dys, &iDz = o->iDz, &Dzs = o->Dzs;
    const double dt = o->dt, omega = o->prm.omega, zeta = o->prm.zeta;
    const int itmax = o->prm.itmax;
    const int check_every = o->prm.check_every > 0 ? o->prm.check_every : 1;
    const bool lex = o->prm.sor_order == NTCFD_SOR_LEX;
    int ik = 0;
    double pChangeMax_ = 1.0;
    bool conv = false;
    auto cell = [&](int i, int j, int k) -> double {
        const double mChange = (us(i, j, k) - us(i - 1, j, k)) * iDy(j) * iDz(k)
                             + (vs(i, j, k) - vs(i, j - 1, k)) * iDx(i) * iDz(k)
                             + (ws(i, j, k) - ws(i, j, k - 1)) * iDx(i) * iDy(j);
        const double pNew = (-p(i + 1, j, k) * iDy(j) * iDz(k) / Dxs(i)
                             - p(i - 1, j, k) * iDy(j) * iDz(k) / Dxs(i - 1)
                             - p(i, j + 1, k) * iDx(i) * iDz(k) / Dys(j)
                             - p(i, j - 1, k) * iDx(i) * iDz(k) / Dys(j - 1)
                             - p(i, j, k + 1) * iDx(i) * iDy(j) / Dzs(k)
                             - p(i, j, k - 1) * iDx(i) * iDy(j) / Dzs(k - 1)
                             + mChange / dt) /
                            (-iDy(j) * iDz(k) / Dxs(i) - iDy(j) * iDz(k) / Dxs(i - 1)
                             - iDx(i) * iDz(k) / Dys(j) - iDx(i) * iDz(k) / Dys(j - 1)
                             - iDx(i) * iDy(j) / Dzs(k) - iDx(i) * iDy(j) / Dzs(k - 1));
        const double pChange = std::fabs(pNew - p(i, j, k));
        p(i, j, k) = p(i, j, k) + (omega * (pNew - p(i, j, k)));
        return pChange;
    };
    while (true) {
        if (forced >= 0) { if (ik >= forced) break; }
        else if (!(pChangeMax_ > zeta && ik < itmax)) break;
        ++ik;
        double pChangeMax = 0.0;
        if (lex) {
            for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static) reduction(max : pChangeMax)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const double c = cell(i, j, k);
                        if (c > pChangeMax) pChangeMax = c;
                    }
            }
        } else {
            for (int colour = 0; colour < 2; ++colour)
                for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static) reduction(max : pChangeMax)
                    for (int j = 1; j <= ny; ++j) {
                        const int i0 = 1 + ((colour + 1 + j + k) & 1);
                        for (int i = i0; i <= nx; i += 2) {
                            const double c = cell(i, j, k);
                            if (c > pChangeMax) pChangeMax = c;
                        }
                    }
                }
        }
        if (forced < 0 && (ik % check_every) != 0 && ik < itmax) {
            pChangeMax_ = 1.0 + zeta;  // no stop test on this sweep
            if (last_change) *last_change = pChangeMax;
            continue;
        }
        pChangeMax_ = pChangeMax;
        if (last_change) *last_change = pChangeMax;
        if (forced < 0 && !(pChangeMax_ > zeta)) conv = true;
    }
    // GS.f90:86-94
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) o->pre(i, j, k) = p(i, j, k);
    if (converged) *converged = conv ? 1 : 0;
    return ik;
}

// calcul_new_velocity.f90:1-181 -- projection, direct forcing, centring.
void orc_calcul_new_velocity(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    F3& p = o->p;
    const double dt = o->dt;
    const double usol = o->prm.u_solid[0], vsol = o->prm.u_solid[1], wsol = o->prm.u_solid[2];
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                o->u1(i, j, k) = o->us(i, j, k) - dt * (p(i + 1, j, k) - p(i, j, k)) / o->Dxs(i);
                o->v1(i, j, k) = o->vs(i, j, k) - dt * (p(i, j + 1, k) - p(i, j, k)) / o->Dys(j);
                o->w1(i, j, k) = o->ws(i, j, k) - dt * (p(i, j, k + 1) - p(i, j, k)) / o->Dzs(k);
            }
    }
    for (int k = 1; k <= nz; ++k) {
#pragma omp parallel for if (par(o)) schedule(static)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double eta = o->ETA(i, j, k);
                o->u2(i, j, k) = eta * usol + (1 - eta) * o->u1(i, j, k);
                o->FX(i, j, k) = (o->u2(i, j, k) - o->u1(i, j, k)) / dt;
                o->v2(i, j, k) = eta * vsol + (1 - eta) * o->v1(i, j, k);
                o->FY(i, j, k) = (o->v2(i, j, k) - o->v1(i, j, k)) / dt;
                o->w2(i, j, k) = eta * wsol + (1 - eta) * o->w1(i, j, k);
                o->FZ(i, j, k) = (o->w2(i, j, k) - o->w1(i, j, k)) / dt;
            }
    }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                o->uc(i, j, k) = 0.5 * (o->u2(i, j, k) + o->u2(i - 1, j, k));
                o->vc(i, j, k) = 0.5 * (o->v2(i, j, k) + o->v2(i, j - 1, k));
                o->wc(i, j, k) = 0.5 * (o->w2(i, j, k) + o->w2(i, j, k - 1));
            }
}

// virtualForceIntegrator.f90:3-85.  FXz(i,0), FXz(i,ny+1), FXy(0) and
// FXy(nx+1) lie outside their arrays in the reference; they read as 0 here.
void orc_force_integral(orc* o, double* cDrag, double* cLift) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    F3 &FY = o->FY, &FZ = o->FZ;
    F1 &Dxs = o->Dxs, &Dys = o->Dys, &Dzs = o->Dzs;
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double fx = 0.0, fy = 0.0;
            for (int k = 1; k <= nz; ++k) {
                fx = fx + (FZ(i, j, k - 1) * Dzs(k - 1) + 4.0 * FZ(i, j, k) * Dzs(k) + FZ(i, j, k + 1) * Dzs(k + 1)) / 6.0;
                fy = fy + (FY(i, j, k - 1) * Dzs(k - 1) + 4.0 * FY(i, j, k) * Dzs(k) + FY(i, j, k + 1) * Dzs(k + 1)) / 6.0;
            }
            o->FXz(i, j) = fx; o->FYz(i, j) = fy;
        }
    auto Fz = [&](F2& a, int i, int j) -> double { return (j < 1 || j > ny) ? 0.0 : a(i, j); };
    for (int i = 1; i <= nx; ++i) {
        double fx = 0.0, fy = 0.0;
        for (int j = 1; j <= ny; ++j) {
            if (o->FXz(i, j) != 0.0)
                fx = fx + (Fz(o->FXz, i, j - 1) * Dys(j - 1) + 4.0 * o->FXz(i, j) * Dys(j) + Fz(o->FXz, i, j + 1) * Dys(j + 1)) / 6.0;
            if (o->FYz(i, j) != 0.0)
                fy = fy + (Fz(o->FYz, i, j - 1) * Dys(j - 1) + 4.0 * o->FYz(i, j) * Dys(j) + Fz(o->FYz, i, j + 1) * Dys(j + 1)) / 6.0;
        }
        o->FXy[i - 1] = fx; o->FYy[i - 1] = fy;
    }
    auto Fy = [&](std::vector<double>& a, int i) -> double { return (i < 1 || i > nx) ? 0.0 : a[i - 1]; };
    double totalFX = 0.0, totalFY = 0.0;
    for (int i = 1; i <= nx; ++i) {
        if (o->FXy[i - 1] != 0.0)
            totalFX = totalFX + (Fy(o->FXy, i - 1) * Dxs(i - 1) + 4.0 * o->FXy[i - 1] * Dxs(i) + Fy(o->FXy, i + 1) * Dxs(i + 1)) / 6.0;
        if (o->FYy[i - 1] != 0.0)
            totalFY = totalFY + (Fy(o->FYy, i - 1) * Dxs(i - 1) + 4.0 * o->FYy[i - 1] * Dxs(i) + Fy(o->FYy, i + 1) * Dxs(i + 1)) / 6.0;
    }
    *cDrag = (-2.0) * totalFX / o->prm.lx;
    *cLift = (-2.0) * totalFY / o->prm.lx;
}

// calcul_new_velocity.f90:195-243.
void orc_updating_velocity(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                o->u(i, j, k) = o->u2(i, j, k);
                o->v(i, j, k) = o->v2(i, j, k);
                o->w(i, j, k) = o->w2(i, j, k);
            }
}

double orc_divergence_max(orc* o) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    double m = 0.0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double d = (o->u(i, j, k) - o->u(i - 1, j, k)) * o->iDy(j) * o->iDz(k)
                               + (o->v(i, j, k) - o->v(i, j - 1, k)) * o->iDx(i) * o->iDz(k)
                               + (o->w(i, j, k) - o->w(i, j, k - 1)) * o->iDx(i) * o->iDy(j);
                m = std::max(m, std::fabs(d));
            }
    return m;
}

// main.f90:209-271 with nproc = 1 (all halo exchanges and gathers vanish).
int orc_step(orc* o, int nsteps, ntcfd_step_info* info, const int* forced) {
    int total = 0;
    for (int s = 0; s < nsteps; ++s) {
        orc_smagorinsky(o);
        orc_predictor(o);
        double last = 0.0;
        int conv = 0;
        const int ik = orc_gauss_seidel(o, forced ? forced[s] : -1, &last, &conv);
        orc_calcul_new_velocity(o);
        double cD = 0.0, cL = 0.0;
        orc_force_integral(o, &cD, &cL);
        orc_updating_velocity(o);
        orc_boundary_conditions(o);
        o->time = o->time + o->dt;
        total += ik;
        if (info) {
            ntcfd_step_info& I = info[s];
            std::memset(&I, 0, sizeof(I));
            I.sor_iters = ik; I.converged = conv; I.sor_last_change = last;
            I.cDrag = cD; I.cLift = cL;
            I.div_max = o->prm.diag_divergence ? orc_divergence_max(o) : 0.0;
        }
    }
    return total;
}

double orc_time(orc* o) { return o->time; }

// ---------------------------------------------------------- gridders ----
// gridder_equal (gridder.f90:228-327) with reading_data's uniform branch
// (reading_data.f90:26-30).  Arrays: X(-1:n+3) -> X[i+1], iDx(-1:n+2) -> iDx[i+1].
static void metrics_from_nodes(int n, const double* X, double* iD, double* Ds) {
    auto x = [&](int i) { return X[i + 1]; };
    for (int i = 1; i <= n - 1; ++i) {
        iD[i + 1] = (x(i + 1) - x(i));
        Ds[i + 1] = (x(i + 2) - x(i)) / 2.0;
    }
    // gridder.f90:121-131 (ghost lengths)
    iD[0 + 1] = iD[1 + 1];
    iD[-1 + 1] = iD[1 + 1];
    iD[n + 1] = x(n + 1) - x(n);
    iD[n + 1 + 1] = iD[n + 1];
    iD[n + 2 + 1] = iD[n + 1];
    Ds[0 + 1] = Ds[1 + 1];
    Ds[-1 + 1] = Ds[1 + 1];
    Ds[n + 1] = Ds[n - 1 + 1];
    Ds[n + 1 + 1] = Ds[n - 1 + 1];
    Ds[n + 2 + 1] = Ds[n - 1 + 1];
}

static void uniform_nodes(int n, double d, double* X) {
    // gridder.f90:235-243
    for (int i = 1; i <= n + 3; ++i) {
        if (i == 1) {
            X[1 + 1] = 0.0;
            X[0 + 1] = X[1 + 1] - d;
            X[-1 + 1] = X[0 + 1] - d;
        } else {
            X[i + 1] = X[i - 1 + 1] + d;
        }
    }
}

void orc_gridder_equal(int nx, int ny, int nz, double lx, double ly, double lz,
                       double* X, double* Y, double* Z,
                       double* iDx, double* Dxs, double* iDy, double* Dys,
                       double* iDz, double* Dzs) {
    const double dx = lx / nx, dy = ly / ny, dz = lz / nz;
    uniform_nodes(nx, dx, X);
    uniform_nodes(ny, dy, Y);
    uniform_nodes(nz, dz, Z);
    metrics_from_nodes(nx, X, iDx, Dxs);
    metrics_from_nodes(ny, Y, iDy, Dys);
    metrics_from_nodes(nz, Z, iDz, Dzs);
}

// gridder_Unequal (gridder.f90:1-157) with reading_data's non-uniform branch
// (reading_data.f90:6-23).  Y(0), Y(-1), Y(ny+2), Y(ny+3) (and Z likewise)
// are never assigned by the reference; they are left 0 here.
void orc_gridder_unequal(int nx, int ny, int nz, double lx, double ly, double lz,
                         const double* band,
                         double* X, double* Y, double* Z,
                         double* iDx, double* Dxs, double* iDy, double* Dys,
                         double* iDz, double* Dzs) {
    const double GridderXc = band[0], GridderYc = band[1], GridderZc = band[2];
    const int nySml = (int)band[4], nyMid = (int)band[5];
    const int nzSml = (int)band[6], nzMid = (int)band[7];
    const double lxSml = band[8], lySml = band[9], lyMid = band[10], lzSml = band[11], lzMid = band[12];
    (void)GridderXc; (void)lxSml;
    const double dySml = lySml / nySml, dzSml = lzSml / nzSml;
    const double dyMid = (lyMid - lySml) / (nyMid - nySml);
    const double dzMid = (lzMid - lzSml) / (nzMid - nzSml);
    const double dy = (ly - lyMid) / (ny - nyMid);
    const double dz = (lz - lzMid) / (nz - nzMid);
    const double dx = lx / nx;  // reading_data.f90:23 overrides the banded dx
    const double ySBgn = GridderYc - lySml / 2.0, ySEnd = GridderYc + lySml / 2.0;
    const double zSBgn = GridderZc, zSEnd = GridderZc + lzSml;
    const double zMBgn = GridderZc, zMEnd = GridderZc + lzMid;
    const double yMBgn = GridderYc - lyMid / 2.0, yMEnd = GridderYc + lyMid / 2.0;
    for (int i = 0; i < nx + 5; ++i) X[i] = 0.0;
    for (int i = 0; i < ny + 5; ++i) Y[i] = 0.0;
    for (int i = 0; i < nz + 5; ++i) Z[i] = 0.0;
    uniform_nodes(nx, dx, X);
    auto band_axis = [](int n, double* A, double dL, double dM, double dS, double MBgn, double MEnd,
                        double SBgn, double SEnd) {
        for (int j = 1; j <= n + 1; ++j) {
            const double prev = A[j - 1 + 1];
            const double nextL = prev + dL, nextM = prev + dM, nextS = prev + dS;
            double val;
            if (j == 1) val = 0.0;
            else if (nextL > MBgn) {
                if (nextM > MEnd) val = nextL;
                else if (nextM > SBgn) val = (nextS > SEnd) ? nextM : nextS;
                else val = nextM;
            } else val = nextL;
            A[j + 1] = val;
        }
    };
    band_axis(ny, Y, dy, dyMid, dySml, yMBgn, yMEnd, ySBgn, ySEnd);
    band_axis(nz, Z, dz, dzMid, dzSml, zMBgn, zMEnd, zSBgn, zSEnd);
    metrics_from_nodes(nx, X, iDx, Dxs);
    metrics_from_nodes(ny, Y, iDy, Dys);
    metrics_from_nodes(nz, Z, iDz, Dzs);
}

// ------------------------------------------------------- ray casting ----
// RayCasting (airfoil.f90:580-915).  The polygon arrays are copied and
// transformed (airfoil.f90:601-611; ay uses the already rotated az).  The
// grid tie moves of airfoil.f90:700-702,731-733 are applied to the oracle's
// Y and Z exactly as the reference does (a global side effect) and counted.
int orc_raycasting(orc* o, const double* az_in, const double* ay_in, int poly,
                   double AOA, double zc, double yc) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    std::vector<double> az(az_in, az_in + poly), ay(ay_in, ay_in + poly);
    const double PI = 4.0 * std::atan(1.0);
    for (int i = 0; i < poly; ++i) {
        az[i] = az[i] - 0.25;
        az[i] = std::cos((-AOA) * PI / 180) * az[i] - std::sin((-AOA) * PI / 180) * ay[i];
        ay[i] = std::sin((-AOA) * PI / 180) * az[i] + std::cos((-AOA) * PI / 180) * ay[i];
        az[i] = az[i] + zc;
        ay[i] = ay[i] + yc;
        az[i] = az[i] + 0.25;
    }
    auto Y = [&](int j) -> double& { return o->Y(j); };
    auto Z = [&](int k) -> double& { return o->Z(k); };
    const double miny = *std::min_element(ay.begin(), ay.end());
    const double maxy = *std::max_element(ay.begin(), ay.end());
    const double minz = *std::min_element(az.begin(), az.end());
    const double maxz = *std::max_element(az.begin(), az.end());
    int A = 0, B = 0, C = 0, E = 0;  // module integers, zero until set
    for (int j = 1; j <= ny; ++j) if (Y(j) > miny) { A = j - 1; break; }
    for (int j = 1; j <= ny; ++j) if (Y(j) > maxy) { B = j; break; }
    for (int k = 1; k <= nz; ++k) if (Z(k) > minz) { C = k - 1; break; }
    for (int k = 1; k <= nz; ++k) if (Z(k) > maxz) { E = k; break; }
    // points(1:nz,1:ny), intersection(1:nz,1:ny)
    std::vector<int> points((size_t)nz * ny, 0), inter((size_t)nz * ny, 0);
    auto PT = [&](int k, int j) -> int& { return points[(size_t)(k - 1) + (size_t)nz * (j - 1)]; };
    auto IN = [&](int k, int j) -> int& { return inter[(size_t)(k - 1) + (size_t)nz * (j - 1)]; };
    for (int m = 0; m < poly; ++m)
        for (int k = C; k <= E - 1; ++k)
            if (az[m] >= Z(k) && az[m] < Z(k + 1))
                for (int j = A; j <= B - 1; ++j)
                    if (ay[m] >= Y(j) && ay[m] < Y(j + 1))
                        if (k >= 1 && k <= nz && j >= 1 && j <= ny) PT(k, j) = 1;
    int ties = 0;
    for (int m = 0; m < poly - 1; ++m)
        for (int j = 1; j <= ny; ++j) {
            if (ay[m] >= (Y(j) + Y(j + 1)) / 2.0 && ay[m + 1] <= (Y(j) + Y(j + 1)) / 2.0) {
                for (int k = 1; k <= nz; ++k) {
                    const double zcell = (Z(k) + Z(k + 1)) / 2.0;
                    if (zcell >= std::max(az[m], az[m + 1])) {
                    } else if (zcell < std::min(az[m], az[m + 1])) {
                        IN(k, j) += 1;
                    } else {
                        if (Y(j) == ay[m + 1] || Z(k) == az[m + 1]) { Y(j) = Y(j) + 0.01; Z(k) = Z(k) + 0.01; ++ties; }
                        const double m_pa = (Y(j) - ay[m + 1]) / (Z(k) - az[m + 1]);
                        const double m_ab = (ay[m] - ay[m + 1]) / (az[m] - az[m + 1]);
                        if (m_pa > m_ab) IN(k, j) += 1;
                    }
                }
            }
            if (ay[m] <= (Y(j) + Y(j + 1)) / 2.0 && ay[m + 1] >= (Y(j) + Y(j + 1)) / 2.0) {
                for (int k = 1; k <= nz; ++k) {
                    const double zcell = (Z(k) + Z(k + 1)) / 2.0;
                    if (zcell >= std::max(az[m], az[m + 1])) {
                    } else if (zcell < std::min(az[m], az[m + 1])) {
                        IN(k, j) += 1;
                    } else {
                        if (Y(j) == ay[m] || Z(k) == az[m]) { Y(j) = Y(j) + 0.01; Z(k) = Z(k) + 0.01; ++ties; }
                        const double m_pa = (Y(j) - ay[m]) / (Z(k) - az[m]);
                        const double m_ab = (ay[m + 1] - ay[m]) / (az[m + 1] - az[m]);
                        if (m_pa > m_ab) IN(k, j) += 1;
                    }
                }
            }
        }
    std::vector<double> eta1((size_t)nz * ny, 0.0);
    auto E1 = [&](int k, int j) -> double& { return eta1[(size_t)(k - 1) + (size_t)nz * (j - 1)]; };
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j) E1(k, j) = (IN(k, j) % 2 == 0) ? 0.0 : 1.0;
    // sub-grid (airfoil.f90:773-884)
    const int NS = 50;
    for (int k = C; k <= E - 1; ++k)
        for (int j = A; j <= B - 1; ++j) {
            if (k < 1 || k > nz || j < 1 || j > ny) continue;
            if (PT(k, j) <= 0) continue;
            std::vector<int> sub((size_t)NS * NS, 0);  // sub(n,l), n fastest
            double ZZ[NS + 1], YY[NS + 1];
            for (int l = 1; l <= NS + 1; ++l) {
                ZZ[l - 1] = Z(k) + (l - 1) * (Z(k + 1) - Z(k)) / (double)NS;
                YY[l - 1] = Y(j) + (l - 1) * (Y(j + 1) - Y(j)) / (double)NS;
            }
            for (int m = 0; m < poly - 1; ++m)
                for (int l = 1; l <= NS; ++l) {
                    const double ycell = (YY[l - 1] + YY[l]) / 2.0;
                    if (ay[m] >= ycell && ay[m + 1] <= ycell) {
                        for (int n = 1; n <= NS; ++n) {
                            const double zcell = (ZZ[n - 1] + ZZ[n]) / 2.0;
                            if (zcell > std::max(az[m], az[m + 1])) {
                            } else if (zcell < std::min(az[m], az[m + 1])) {
                                sub[(size_t)(n - 1) + NS * (l - 1)] += 1;
                            } else {
                                if (YY[l - 1] == ay[m + 1] || ZZ[n - 1] == az[m + 1]) {
                                    YY[l - 1] += 0.01; ZZ[n - 1] += 0.01; ++ties;
                                }
                                const double m_pa = (YY[l - 1] - ay[m + 1]) / (ZZ[n - 1] - az[m + 1]);
                                const double m_ab = (ay[m] - ay[m + 1]) / (az[m] - az[m + 1]);
                                if (m_pa > m_ab) sub[(size_t)(n - 1) + NS * (l - 1)] += 1;
                            }
                        }
                    }
                    const double ycell2 = (YY[l - 1] + YY[l]) / 2.0;
                    if (ay[m] <= ycell2 && ay[m + 1] >= ycell2) {
                        for (int n = 1; n <= NS; ++n) {
                            const double zcell = (ZZ[n - 1] + ZZ[n]) / 2.0;
                            if (zcell > std::max(az[m], az[m + 1])) {
                            } else if (zcell < std::min(az[m], az[m + 1])) {
                                sub[(size_t)(n - 1) + NS * (l - 1)] += 1;
                            } else {
                                if (YY[l - 1] == ay[m + 1] || ZZ[n - 1] == az[m + 1]) {
                                    YY[l - 1] += 0.01; ZZ[n - 1] += 0.01; ++ties;
                                }
                                const double m_pa = (YY[l - 1] - ay[m]) / (ZZ[n - 1] - az[m]);
                                const double m_ab = (ay[m + 1] - ay[m]) / (az[m + 1] - az[m]);
                                if (m_pa > m_ab) sub[(size_t)(n - 1) + NS * (l - 1)] += 1;
                            }
                        }
                    }
                }
            double total = 0;
            for (size_t q = 0; q < sub.size(); ++q) total += (sub[q] % 2 == 0) ? 0 : 1;
            E1(k, j) = total / (double)NS / (double)NS;
        }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) o->ETA(i, j, k) = E1(k, j);
    return ties;
}

// DFIB_Cylinder (DFIB.f90:74-145): single precision (real*4) distances and
// sub-cell coordinates; iBgnVOS..iEndVOS = 1..nx, likewise j and k.
void orc_cylinder(orc* o, double zc, double yc, double r) {
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    const int NS = 50;
    const int i = 1;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j) {
            // x**2.D0 is evaluated as x*x; real*4 + real*4 sums stay real*4.
            const float DIAGONAL = (float)(std::sqrt(o->iDx(i) * o->iDx(i) + o->iDy(j) * o->iDy(j) + o->iDz(k) * o->iDz(k)) / 2.0);
            const double dzc = ((o->Z(k) + o->Z(k + 1)) / 2.0) - zc;
            const double dyc = ((o->Y(j) + o->Y(j + 1)) / 2.0) - yc;
            const float DISTANCE = (float)std::sqrt(dzc * dzc + dyc * dyc);
            double eta;
            if (std::fabs((double)DISTANCE - r) < (double)DIAGONAL) {
                float xi = 0.0f;
                float SZ[NS + 1], SY[NS + 1];
                const float dzg = (float)(o->iDz(k) / NS);
                const float dyg = (float)(o->iDy(j) / NS);
                for (int n = 1; n <= NS + 1; ++n) {
                    SZ[n - 1] = (float)(o->Z(k) + (double)((float)(n - 1) * dzg));
                    SY[n - 1] = (float)(o->Y(j) + (double)((float)(n - 1) * dyg));
                }
                for (int m = 1; m <= NS; ++m)
                    for (int n = 1; n <= NS; ++n) {
                        const double sz = (double)(SZ[n - 1] + SZ[n]) / 2.0 - zc;
                        const double sy = (double)(SY[m - 1] + SY[m]) / 2.0 - yc;
                        const float SDIST = (float)std::sqrt(sz * sz + sy * sy);
                        if ((double)SDIST <= r) xi = xi + 1;
                    }
                eta = (double)(xi / (float)(NS * NS));
            } else if ((double)DISTANCE > r) {
                eta = 0.0;
            } else {
                eta = 1.0;
            }
            o->ETA(i, j, k) = eta;
        }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int ii = 2; ii <= nx; ++ii) o->ETA(ii, j, k) = o->ETA(1, j, k);
}

}  // extern "C"
