// k_project.cuh -- K4 projection + direct forcing + velocity update, K5 force
// integral, K6 boundary conditions, K8 centred output, step bookkeeping.
#pragma once

#include "ntcfd_common.cuh"

namespace ntcfd {

// ---------------------------------------------------------------- K4 ----
// calcul_new_velocity.f90:13-100 and Updating_velocity (195-243) fused:
//   u1 = u* - dt (p(i+1)-p(i))/Dxs(i)            (17, 31, 45)
//   u2 = ETA u_solid + (1-ETA) u1, F = (u2-u1)/dt (65-66, 80-81, 95-96)
//   u  = u2                                      (209, 222, 236)
// Each thread walks `kc` planes of one (i,j) column and adds FZ and FY with
// the Simpson weights of virtualForceIntegrator.f90:30-31 collected per
// plane: FZ(k) enters FXz(i,j) with Dzs(k) (4 + [k>1] + [k<nz]) / 6 because
// FZ(i,j,0) = FZ(i,j,nz+1) = 0.  One double per (chunk, j, i) is written.
struct ProjArgs {
    double *u, *v, *w;
    const double *us, *vs, *ws, *p, *eta;
    double* partZ;   // [nchunk][ny][nx]
    double* partY;
    double dt, usol, vsol, wsol;
    int kc;
};

__global__ void __launch_bounds__(128) k_project(Geom g, ProjArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int chunk = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const int k0 = chunk * a.kc + 1;
    const int k1 = min(g.nz, k0 + a.kc - 1);
    const double dt = a.dt;
    double fz = 0.0, fy = 0.0;
    for (int k = k0; k <= k1; ++k) {
        const long long c = nat(g, i, j, k);
        const double pc = a.p[c];
        const double u1 = a.us[c] - dt * (a.p[c + 1] - pc) * g.rDxs[i];
        const double v1 = a.vs[c] - dt * (a.p[c + g.px] - pc) * g.rDys[j];
        const double w1 = a.ws[c] - dt * (a.p[c + g.pz] - pc) * g.rDzs[k];
        const double eta = a.eta[c];
        const double u2 = eta * a.usol + (1 - eta) * u1;
        const double v2 = eta * a.vsol + (1 - eta) * v1;
        const double w2 = eta * a.wsol + (1 - eta) * w1;
        a.u[c] = u2;
        a.v[c] = v2;
        a.w[c] = w2;
        const double wz = g.Dzs[k] * (4.0 + (k > 1 ? 1.0 : 0.0) + (k < g.nz ? 1.0 : 0.0)) / 6.0;
        fz += ((w2 - w1) / dt) * wz;
        fy += ((v2 - v1) / dt) * wz;
    }
    const long long q = (long long)chunk * g.ny * g.nx + (long long)(j - 1) * g.nx + (i - 1);
    a.partZ[q] = fz;
    a.partY[q] = fy;
}

// ---------------------------------------------------------------- K5 ----
// virtualForceIntegrator.f90:22-81.  First the k-sums per column (fixed
// chunk order), then one block does the guarded j-sums per i and the
// guarded i-sum (entries whose centre value is exactly 0 are skipped,
// virtualForceIntegrator.f90:48,52,67,71; FXz(i,0), FXz(i,ny+1), FXy(0) and
// FXy(nx+1) read as 0).
__global__ void k_force_columns(Geom g, const double* partZ, const double* partY, int nchunk,
                                double* FXz, double* FYz) {
    const long long n = (long long)g.nx * g.ny;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        double sz = 0.0, sy = 0.0;
        for (int c = 0; c < nchunk; ++c) {
            sz += partZ[(long long)c * n + q];
            sy += partY[(long long)c * n + q];
        }
        FXz[q] = sz;
        FYz[q] = sy;
    }
}

// Guarded j-sums (virtualForceIntegrator.f90:45-57): one warp per i, lanes
// over j, fixed-order shuffle reduction; FXy(i), FYy(i) to global.  The last
// block to finish (counter in ctl) does the guarded i-sum (60-76) in one
// block with a fixed-order tree, then cDrag and cLift (80-81).
template <int NT>
__global__ void __launch_bounds__(NT) k_force_total(Geom g, const double* FXz, const double* FYz,
                                                    double* FXy, double* FYy, double lx, Ctl* ctl,
                                                    unsigned int* done, StepRec* rec) {
    const int nx = g.nx, ny = g.ny;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (NT / 32) + (threadIdx.x >> 5) + 1;
    if (i <= nx) {
        double ax = 0.0, ay = 0.0;
        for (int j = lane + 1; j <= ny; j += 32) {
            const long long q = (long long)(j - 1) * nx + (i - 1);
            const double cx = FXz[q], cy = FYz[q];
            const double xm = (j > 1) ? FXz[q - nx] : 0.0, xp = (j < ny) ? FXz[q + nx] : 0.0;
            const double ym = (j > 1) ? FYz[q - nx] : 0.0, yp = (j < ny) ? FYz[q + nx] : 0.0;
            if (cx != 0.0) ax += (xm * g.Dys[j - 1] + 4.0 * cx * g.Dys[j] + xp * g.Dys[j + 1]) / 6.0;
            if (cy != 0.0) ay += (ym * g.Dys[j - 1] + 4.0 * cy * g.Dys[j] + yp * g.Dys[j + 1]) / 6.0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
        }
        if (lane == 0) { FXy[i - 1] = ax; FYy[i - 1] = ay; }
    }
    // last block: the i-sum
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(done, 1u) + 1u == gridDim.x;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double sx[NT], sy[NT];
    double tx = 0.0, ty = 0.0;
    for (int ii = threadIdx.x + 1; ii <= nx; ii += NT) {
        const double c = __ldcg(FXy + ii - 1), cyv = __ldcg(FYy + ii - 1);
        const double l = ii > 1 ? __ldcg(FXy + ii - 2) : 0.0, r = ii < nx ? __ldcg(FXy + ii) : 0.0;
        const double ly = ii > 1 ? __ldcg(FYy + ii - 2) : 0.0, ry = ii < nx ? __ldcg(FYy + ii) : 0.0;
        if (c != 0.0) tx += (l * g.Dxs[ii - 1] + 4.0 * c * g.Dxs[ii] + r * g.Dxs[ii + 1]) / 6.0;
        if (cyv != 0.0) ty += (ly * g.Dxs[ii - 1] + 4.0 * cyv * g.Dxs[ii] + ry * g.Dxs[ii + 1]) / 6.0;
    }
    sx[threadIdx.x] = tx;
    sy[threadIdx.x] = ty;
    __syncthreads();
    for (int st = NT / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            sx[threadIdx.x] += sx[threadIdx.x + st];
            sy[threadIdx.x] += sy[threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *done = 0u;
        const int s = ctl->step;
        ctl->cdrag = (-2.0) * sx[0] / lx;
        ctl->clift = (-2.0) * sy[0] / lx;
        rec[s].cdrag = ctl->cdrag;
        rec[s].clift = ctl->clift;
    }
}

// ---------------------------------------------------------------- K6 ----
// boundary_conditions.f90:13-374.  The six walls run as three launches in
// the reference order (W|E, S|N, B|F); the two walls of one pair touch
// disjoint planes, so they run in the same launch.  Pressure ghosts
// (329-374) are set in the same launches.  Before a wall overwrites the
// normal-velocity face that the centred output uses (u(0), u(nx), v(0),
// v(ny), w(0), w(nz)), the old interior-range value is saved: the
// reference centres the velocity before the boundary conditions
// (calcul_new_velocity.f90:171-181).
struct BcArgs {
    double *u, *v, *w, *p;
    int bc[6][3];
    double val[6][3];
    double *faceW, *faceE;   // u(0,j,k), u(nx,j,k) before the BCs, [(k-1)*ny + j-1]
    double *faceS, *faceN;   // v(i,0,k), v(i,ny,k), [(k-1)*nx + i-1]
    double *faceB, *faceF;   // w(i,j,0), w(i,j,nz), [(j-1)*nx + i-1]
};

enum { BC_NOSLIP = 0, BC_NEUMANN = 1, BC_DIRICHLET = 2, BC_PERIODIC = 3, BC_INTERFACE = 4 };

// ghost of a tangential component on a wall: 2*val - interior, interior, value, periodic copy
__device__ __forceinline__ double tangential(int kind, double val, double inner, double periodic_src) {
    switch (kind) {
        case BC_NOSLIP: return 2 * 0 - inner;
        case BC_NEUMANN: return inner;
        case BC_DIRICHLET: return 2 * val - inner;
        default: return periodic_src;
    }
}

__device__ __forceinline__ void bc_x_at(const Geom& g, const BcArgs& a, int j, int k, int fld) {
    const int nx = g.nx;
    auto I = [&](int i) { return nat(g, i, j, k); };
    const bool inside = j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
    if (fld == 0 && inside) {
        const long long f = (long long)(k - 1) * g.ny + (j - 1);
        a.faceW[f] = a.u[I(0)];
        a.faceE[f] = a.u[I(nx)];
    }
    // West (boundary_conditions.f90:13-57)
    if (fld == 0) {
        const int ku = a.bc[0][0];
        double u0;
        if (ku == BC_NOSLIP) u0 = 0.0;
        else if (ku == BC_NEUMANN) u0 = a.u[I(1)];
        else if (ku == BC_DIRICHLET) u0 = a.val[0][0];
        else u0 = a.u[I(nx)];
        a.u[I(0)] = u0;
        a.u[I(-1)] = (ku == BC_PERIODIC) ? a.u[I(nx - 1)] : u0;
    } else if (fld <= 2) {
        double* f2[2] = {a.v, a.w};
        {
            const int c = fld;
            double* f = f2[c - 1];
            const int kd = a.bc[0][c];
            const double g0 = tangential(kd, a.val[0][c], f[I(1)], f[I(nx)]);
            f[I(0)] = g0;
            f[I(-1)] = (kd == BC_PERIODIC) ? f[I(nx - 1)] : g0;
        }
    }
    // East (boundary_conditions.f90:59-105)
    if (fld == 0) {
        const int ku = a.bc[1][0];
        if (ku == BC_PERIODIC) {
            a.u[I(nx + 1)] = a.u[I(1)];
            a.u[I(nx + 2)] = a.u[I(2)];
        } else {
            double un;
            if (ku == BC_NOSLIP) un = 0.0;
            else if (ku == BC_NEUMANN) un = a.u[I(nx - 1)];
            else un = a.val[1][0];
            a.u[I(nx)] = un;
            a.u[I(nx + 1)] = un;
            a.u[I(nx + 2)] = un;
        }
    } else if (fld <= 2) {
        double* f2[2] = {a.v, a.w};
        {
            const int c = fld;
            double* f = f2[c - 1];
            const int kd = a.bc[1][c];
            if (kd == BC_PERIODIC) {
                f[I(nx + 1)] = f[I(1)];
                f[I(nx + 2)] = f[I(2)];
            } else {
                const double g1 = tangential(kd, a.val[1][c], f[I(nx)], 0.0);
                f[I(nx + 1)] = g1;
                f[I(nx + 2)] = g1;
            }
        }
    }
    // pressure (boundary_conditions.f90:329-342)
    if (fld != 3) return;
    if (a.bc[0][0] == BC_PERIODIC) {
        a.p[I(0)] = a.p[I(nx)]; a.p[I(-1)] = a.p[I(nx - 1)];
        a.p[I(nx + 1)] = a.p[I(1)]; a.p[I(nx + 2)] = a.p[I(2)];
    } else {
        const double p1 = a.p[I(1)], pn = a.p[I(nx)];
        a.p[I(0)] = p1; a.p[I(-1)] = p1;
        a.p[I(nx + 1)] = pn; a.p[I(nx + 2)] = pn;
    }
}

__global__ void k_bc_x(Geom g, BcArgs a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y - 1;
    if (j > g.ny + 2 || k > g.nz + 2) return;
    bc_x_at(g, a, j, k, blockIdx.z);
}

__device__ __forceinline__ void bc_y_at(const Geom& g, const BcArgs& a, int i, int k, int fld) {
    const int ny = g.ny;
    auto J = [&](int j) { return nat(g, i, j, k); };
    if (fld == 1 && i >= 1 && i <= g.nx && k >= 1 && k <= g.nz) {
        const long long f = (long long)(k - 1) * g.nx + (i - 1);
        a.faceS[f] = a.v[J(0)];
        a.faceN[f] = a.v[J(ny)];
    }
    // South (boundary_conditions.f90:107-153): u, v, w
    if (fld == 0) {
        const int kd = a.bc[2][0];
        const double g0 = tangential(kd, a.val[2][0], a.u[J(1)], a.u[J(ny)]);
        a.u[J(0)] = g0;
        a.u[J(-1)] = (kd == BC_PERIODIC) ? a.u[J(ny - 1)] : g0;
    }
    if (fld == 1) {
        const int kv = a.bc[2][1];
        double v0;
        if (kv == BC_NOSLIP) v0 = 0.0;
        else if (kv == BC_NEUMANN) v0 = a.v[J(1)];
        else if (kv == BC_DIRICHLET) v0 = a.val[2][1];
        else v0 = a.v[J(ny)];
        a.v[J(0)] = v0;
        a.v[J(-1)] = (kv == BC_PERIODIC) ? a.v[J(ny - 1)] : v0;
    }
    if (fld == 2) {
        const int kd = a.bc[2][2];
        const double g0 = tangential(kd, a.val[2][2], a.w[J(1)], a.w[J(ny)]);
        a.w[J(0)] = g0;
        a.w[J(-1)] = (kd == BC_PERIODIC) ? a.w[J(ny - 1)] : g0;
    }
    // North (boundary_conditions.f90:155-202)
    if (fld == 0) {
        const int kd = a.bc[3][0];
        if (kd == BC_PERIODIC) { a.u[J(ny + 1)] = a.u[J(1)]; a.u[J(ny + 2)] = a.u[J(2)]; }
        else {
            const double g1 = tangential(kd, a.val[3][0], a.u[J(ny)], 0.0);
            a.u[J(ny + 1)] = g1; a.u[J(ny + 2)] = g1;
        }
    }
    if (fld == 1) {
        const int kv = a.bc[3][1];
        if (kv == BC_PERIODIC) { a.v[J(ny + 1)] = a.v[J(1)]; a.v[J(ny + 2)] = a.v[J(2)]; }
        else {
            double vn;
            if (kv == BC_NOSLIP) vn = 0.0;
            else if (kv == BC_NEUMANN) vn = a.v[J(ny - 1)];
            else vn = a.val[3][1];
            a.v[J(ny)] = vn; a.v[J(ny + 1)] = vn; a.v[J(ny + 2)] = vn;
        }
    }
    if (fld == 2) {
        const int kd = a.bc[3][2];
        if (kd == BC_PERIODIC) { a.w[J(ny + 1)] = a.w[J(1)]; a.w[J(ny + 2)] = a.w[J(2)]; }
        else {
            const double g1 = tangential(kd, a.val[3][2], a.w[J(ny)], 0.0);
            a.w[J(ny + 1)] = g1; a.w[J(ny + 2)] = g1;
        }
    }
    // pressure (boundary_conditions.f90:344-358)
    if (fld != 3) return;
    if (a.bc[2][1] == BC_PERIODIC) {
        a.p[J(0)] = a.p[J(ny)]; a.p[J(-1)] = a.p[J(ny - 1)];
        a.p[J(ny + 1)] = a.p[J(1)]; a.p[J(ny + 2)] = a.p[J(2)];
    } else {
        const double p1 = a.p[J(1)], pn = a.p[J(ny)];
        a.p[J(0)] = p1; a.p[J(-1)] = p1;
        a.p[J(ny + 1)] = pn; a.p[J(ny + 2)] = pn;
    }
}

__global__ void k_bc_y(Geom g, BcArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y - 1;
    if (i > g.nx + 2 || k > g.nz + 2) return;
    bc_y_at(g, a, i, k, blockIdx.z);
}

__device__ __forceinline__ void bc_z_at(const Geom& g, const BcArgs& a, int i, int j, int fld) {
    const int nz = g.nz;
    auto K = [&](int k) { return nat(g, i, j, k); };
    if (fld == 2 && i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
        const long long f = (long long)(j - 1) * g.nx + (i - 1);
        a.faceB[f] = a.w[K(0)];
        a.faceF[f] = a.w[K(nz)];
    }
    // Back (boundary_conditions.f90:205-252): u, v tangential, w normal.  A face
    // shared with the neighbouring z-slab keeps the planes the exchange wrote.
    if (a.bc[4][0] != BC_INTERFACE && fld <= 1) {
        double* f2[2] = {a.u, a.v};
        const int c = fld;
        double* f = f2[c];
        const int kd = a.bc[4][c];
        if (kd == BC_NEUMANN && c == 1) {
            // BackWall_v 'Neumann' assigns v(i,j,0) to itself (boundary_conditions.f90:228)
            f[K(-1)] = f[K(0)];
        } else {
            const double g0 = tangential(kd, a.val[4][c], f[K(1)], f[K(nz)]);
            f[K(0)] = g0;
            f[K(-1)] = (kd == BC_PERIODIC) ? f[K(nz - 1)] : g0;
        }
    }
    if (a.bc[4][0] != BC_INTERFACE && fld == 2) {
        const int kw = a.bc[4][2];
        double w0;
        if (kw == BC_NOSLIP) w0 = 0.0;
        else if (kw == BC_NEUMANN) w0 = a.w[K(1)];
        else if (kw == BC_DIRICHLET) w0 = a.val[4][2];
        else w0 = a.w[K(nz)];
        a.w[K(0)] = w0;
        a.w[K(-1)] = (kw == BC_PERIODIC) ? a.w[K(nz - 1)] : w0;
    }
    // Front (boundary_conditions.f90:255-301)
    if (a.bc[5][0] != BC_INTERFACE && fld <= 1) {
        double* f2[2] = {a.u, a.v};
        const int c = fld;
        double* f = f2[c];
        const int kd = a.bc[5][c];
        if (kd == BC_PERIODIC) { f[K(nz + 1)] = f[K(1)]; f[K(nz + 2)] = f[K(2)]; }
        else {
            const double g1 = tangential(kd, a.val[5][c], f[K(nz)], 0.0);
            f[K(nz + 1)] = g1; f[K(nz + 2)] = g1;
        }
    }
    if (a.bc[5][0] != BC_INTERFACE && fld == 2) {
        const int kw = a.bc[5][2];
        if (kw == BC_PERIODIC) { a.w[K(nz + 1)] = a.w[K(1)]; a.w[K(nz + 2)] = a.w[K(2)]; }
        else {
            double wn;
            if (kw == BC_NOSLIP) wn = 0.0;
            else if (kw == BC_NEUMANN) wn = a.w[K(nz - 1)];
            else wn = a.val[5][2];
            a.w[K(nz)] = wn; a.w[K(nz + 1)] = wn; a.w[K(nz + 2)] = wn;
        }
    }
    // pressure (boundary_conditions.f90:360-374)
    if (fld != 3) return;
    if (a.bc[4][2] == BC_PERIODIC) {
        a.p[K(0)] = a.p[K(nz)]; a.p[K(-1)] = a.p[K(nz - 1)];
        a.p[K(nz + 1)] = a.p[K(1)]; a.p[K(nz + 2)] = a.p[K(2)];
    } else {
        const double p1 = a.p[K(1)], pn = a.p[K(nz)];
        if (a.bc[4][2] != BC_INTERFACE) { a.p[K(0)] = p1; a.p[K(-1)] = p1; }
        if (a.bc[5][2] != BC_INTERFACE) { a.p[K(nz + 1)] = pn; a.p[K(nz + 2)] = pn; }
    }
}

__global__ void k_bc_z(Geom g, BcArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
    if (i > g.nx + 2 || j > g.ny + 2) return;
    bc_z_at(g, a, i, j, blockIdx.z);
}

// Launch grids of k_bc_x/y/z: 32 x 8 threads over the face's (ghost-inclusive)
// rows, one z layer per field (u, v, w, p).  The fields of a face are
// independent, so the four layers run side by side: each thread keeps one
// field's short load/store chain instead of all four in sequence.
inline dim3 bc_grid_x(const Geom& g) { return dim3((g.ny + 4 + 31) / 32, (g.nz + 4 + 7) / 8, 4); }
inline dim3 bc_grid_y(const Geom& g) { return dim3((g.nx + 4 + 31) / 32, (g.nz + 4 + 7) / 8, 4); }
inline dim3 bc_grid_z(const Geom& g) { return dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 7) / 8, 4); }

// ---------------------------------------------------------------- K8 ----
// Centred output (calcul_new_velocity.f90:171-181) and pre = p (GS.f90:86-94),
// into Fortran-order (nx,ny,nz) device arrays.
__global__ void k_centre(Geom g, const double* u, const double* v, const double* w, const double* p,
                         const double* faceW, const double* faceE, const double* faceS,
                         const double* faceN, const double* faceB, const double* faceF,
                         double* pre, double* uc, double* vc, double* wc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const long long o = (long long)(i - 1) + (long long)g.nx * ((j - 1) + (long long)g.ny * (k - 1));
    const double ui = (i == g.nx) ? faceE[(long long)(k - 1) * g.ny + (j - 1)] : u[c];
    const double um = (i == 1) ? faceW[(long long)(k - 1) * g.ny + (j - 1)] : u[c - 1];
    const double vj = (j == g.ny) ? faceN[(long long)(k - 1) * g.nx + (i - 1)] : v[c];
    const double vm = (j == 1) ? faceS[(long long)(k - 1) * g.nx + (i - 1)] : v[c - g.px];
    const double wk = (k == g.nz) ? faceF[(long long)(j - 1) * g.nx + (i - 1)] : w[c];
    const double wm = (k == 1) ? faceB[(long long)(j - 1) * g.nx + (i - 1)] : w[c - g.pz];
    pre[o] = p[c];
    uc[o] = 0.5 * (ui + um);
    vc[o] = 0.5 * (vj + vm);
    wc[o] = 0.5 * (wk + wm);
}

// max |div u| V over the interior (diagnostic, after the boundary conditions)
template <int NT>
__global__ void __launch_bounds__(NT) k_divmax(Geom g, const double* u, const double* v,
                                               const double* w, unsigned long long* slot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    double d = 0.0;
    if (i <= g.nx && j <= g.ny && k <= g.nz) {
        const long long c = nat(g, i, j, k);
        d = fabs((u[c] - u[c - 1]) * g.iDy[j] * g.iDz[k] + (v[c] - v[c - g.px]) * g.iDx[i] * g.iDz[k] +
                 (w[c] - w[c - g.pz]) * g.iDx[i] * g.iDy[j]);
    }
    block_max_atomic<NT>(d, slot);  // one slot: the diagnostic runs once per step
}

// Records the step; `fixed` kernels per step, per_cycle per correction cycle
// (cycles restarted inside the resident SOR kernel launch nothing) and
// per_body per inner loop body.
// With forces = 0 (ETA is 0 everywhere, the force kernels did not run) it also
// records the coefficients those kernels give for zero forces: -2 * 0 / lx.
__global__ void k_step_end(Ctl* ctl, StepRec* rec, unsigned long long* divslot, int diag,
                           int fixed, int per_cycle, int per_body, int forces, double lx) {
    const int s = ctl->step;
    if (!forces) {
        const double z = (-2.0) * 0.0 / lx;
        ctl->cdrag = z;
        ctl->clift = z;
        rec[s].cdrag = z;
        rec[s].clift = z;
    }
    rec[s].launches = fixed + per_cycle * (ctl->cycles - ctl->restarts) + ctl->bodies * per_body;
    rec[s].timeout = ctl->timeout;
    rec[s].sor_iters = ctl->ik;
    rec[s].converged = ctl->converged;
    rec[s].last_change = ctl->last_change;
    rec[s].cycles = ctl->cycles;
    rec[s].nonfinite = ctl->nonfinite;
    rec[s].divmax = diag ? __longlong_as_double((long long)*divslot) : 0.0;
    *divslot = 0ULL;
    ctl->step = s + 1;
}

}  // namespace ntcfd
