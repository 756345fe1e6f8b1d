// k_adjoint.cuh -- discrete adjoint of the time step (no counterpart in the
// reference).  Each kernel is the transpose of the linearisation of a
// forward kernel about the forward state of that step:
//   k_adj_bc_{z,y,x}   transpose of boundary_conditions (walls in reverse order)
//   k_adj_weights      d(cDrag)/dFZ and d(cLift)/dFY per cell (guard pattern fixed)
//   k_adj_project1/2   projection + direct forcing + update
//   k_adj_solve_rhs,
//   k_adj_after_solve  converged pressure solve: M z = V^-1 lambda_p, y = V z
//   k_adj_rhs          divergence right-hand side
//   k_adj_predictor    QUICK/central predictor (upwind branch fixed)
// Adjoint fields are natural-layout FP64 halo arrays; "lam*" is the adjoint
// of the corresponding forward field.
#pragma once

#include "k_predictor.cuh"
#include "k_pressure.cuh"
#include "k_project.cuh"
#include "ntcfd_common.cuh"

namespace ntcfd {

// ------------------------------------------------------------- predictor
// Reverse of quick_face: the face value is linear in (fm1, f0, f1, f2) with
// coefficients fixed by the upwind branch.
__device__ __forceinline__ void quick_face_adj(double qbar, double adv, double A, double B, double r0,
                                               double r1, double r2, double& gm1, double& g0,
                                               double& g1, double& g2) {
    if (adv > 0.0) {
        gm1 += qbar * (-A * r0);
        g0 += qbar * (0.5 + A * r1 + A * r0);
        g1 += qbar * (0.5 - A * r1);
    } else {
        g0 += qbar * (0.5 - B * r1);
        g1 += qbar * (0.5 + B * r2 + B * r1);
        g2 += qbar * (-B * r2);
    }
}

// One axis of one momentum component: flux = t1*QF(f-1,f0,f1,f2;t1) - t2*QF(f-2,f-1,f0,f1;t2)
// enters r with factor -dt*cA, diffusion ((f1-f0)*d1 - (f0-f-1)*d0) with nue*dt*cD.
// g[0..4] accumulate d/d f(-2..+2); t1bar, t2bar the advecting-velocity adjoints;
// nubar the eddy-viscosity adjoint.
struct AxisIn {
    double fm2, fm1, f0, f1, f2;   // transported component along the axis
    double t1, t2;                 // face-averaged advecting velocities
    double A1, B1, p0, p1, p2;     // QUICK factors of the + face
    double A2, B2, q0, q1, q2;     // QUICK factors of the - face
    double cA;                     // flux divisor reciprocal
    double d0, d1, cD;             // diffusion factors
};

__device__ __forceinline__ void axis_adj(const AxisIn& a, double rbar, double dt, double nue, double les,
                                         double g[5], double& t1bar, double& t2bar, double& nubar) {
    // forward face values
    const double q1 = quick_face<double>(a.fm1, a.f0, a.f1, a.f2, a.t1, a.A1, a.B1, a.p0, a.p1, a.p2);
    const double q2 = quick_face<double>(a.fm2, a.fm1, a.f0, a.f1, a.t2, a.A2, a.B2, a.q0, a.q1, a.q2);
    const double Tbar = -dt * a.cA * rbar;
    t1bar += Tbar * q1;
    t2bar -= Tbar * q2;
    const double q1bar = Tbar * a.t1, q2bar = -Tbar * a.t2;
    quick_face_adj(q1bar, a.t1, a.A1, a.B1, a.p0, a.p1, a.p2, g[1], g[2], g[3], g[4]);
    quick_face_adj(q2bar, a.t2, a.A2, a.B2, a.q0, a.q1, a.q2, g[0], g[1], g[2], g[3]);
    const double Dbar = nue * dt * a.cD * rbar;
    g[3] += Dbar * a.d1;
    g[2] -= Dbar * (a.d1 + a.d0);
    g[1] += Dbar * a.d0;
    nubar += les * dt * a.cD * ((a.f1 - a.f0) * a.d1 - (a.f0 - a.fm1) * a.d0) * rbar;
}

struct AdjPredArgs {
    const double *u, *v, *w, *nut;       // forward state of the step (and nu_t)
    const double *lus, *lvs, *lws;       // adjoints of u*, v*, w* (interior)
    double *lu, *lv, *lw;                // adjoints of u, v, w (accumulated, atomics)
    double* lnut;                        // adjoint of nu_t (LES), or null
    double* gf;                          // gradient of the body force (fu, fv, fw; N apart), or null
    long long fstride;                   // N
    double dt, nu;
    int les;
};

__global__ void __launch_bounds__(128) k_adj_predictor(Geom g, Tabs<double> tb, AdjPredArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const long long sx = 1, sy = g.px, sz = g.pz;
    const AxisTabs<double> X = tb.ax[0], Y = tb.ax[1], Z = tb.ax[2];
    const double dt = a.dt;
    const double les = (double)a.les;
    const double nue = a.les ? a.nu + a.nut[c] * les : a.nu;
    double nubar = 0.0;
    const double* u = a.u;
    const double* v = a.v;
    const double* w = a.w;
    auto add = [](double* p, double val) { if (val != 0.0) atomicAdd(p, val); };

    // ---------------- u* (discretisation_QUICK_centre.f90:11-112)
    {
        const double rbar = a.lus[c];
        if (a.gf) a.gf[c] += dt * rbar;
        if (rbar != 0.0) {
            double gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
            double tx1 = 0, tx2 = 0, ty1 = 0, ty2 = 0, tz1 = 0, tz2 = 0;
            AxisIn ax{u[c - 2 * sx], u[c - sx], u[c], u[c + sx], u[c + 2 * sx],
                      0.5 * (u[c + sx] + u[c]), 0.5 * (u[c - sx] + u[c]),
                      X.As[i], X.Bs[i], X.riD[i], X.riD[i + 1], X.riD[i + 2],
                      X.As[i - 1], X.Bs[i - 1], X.riD[i - 1], X.riD[i], X.riD[i + 1],
                      X.rDs[i], X.riD[i], X.riD[i + 1], X.rDs[i]};
            AxisIn ay{u[c - 2 * sy], u[c - sy], u[c], u[c + sy], u[c + 2 * sy],
                      0.5 * (v[c] + v[c + sx]), 0.5 * (v[c - sy] + v[c + sx - sy]),
                      Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1],
                      Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j],
                      Y.riD[j], Y.rDs[j - 1], Y.rDs[j], Y.riD[j]};
            AxisIn az{u[c - 2 * sz], u[c - sz], u[c], u[c + sz], u[c + 2 * sz],
                      0.5 * (w[c + sx] + w[c]), 0.5 * (w[c - sz] + w[c + sx - sz]),
                      Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1],
                      Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k],
                      Z.riD[k], Z.rDs[k - 1], Z.rDs[k], Z.riD[k]};
            axis_adj(ax, rbar, dt, nue, les, gx, tx1, tx2, nubar);
            axis_adj(ay, rbar, dt, nue, les, gy, ty1, ty2, nubar);
            axis_adj(az, rbar, dt, nue, les, gz, tz1, tz2, nubar);
            // x-advecting velocity is u itself: t1 = (u(i+1)+u(i))/2, t2 = (u(i-1)+u(i))/2
            gx[3] += 0.5 * tx1; gx[2] += 0.5 * tx1 + 0.5 * tx2; gx[1] += 0.5 * tx2;
            add(a.lu + c, rbar + gx[2] + gy[2] + gz[2]);
            add(a.lu + c - 2 * sx, gx[0]); add(a.lu + c - sx, gx[1]);
            add(a.lu + c + sx, gx[3]); add(a.lu + c + 2 * sx, gx[4]);
            add(a.lu + c - 2 * sy, gy[0]); add(a.lu + c - sy, gy[1]);
            add(a.lu + c + sy, gy[3]); add(a.lu + c + 2 * sy, gy[4]);
            add(a.lu + c - 2 * sz, gz[0]); add(a.lu + c - sz, gz[1]);
            add(a.lu + c + sz, gz[3]); add(a.lu + c + 2 * sz, gz[4]);
            add(a.lv + c, 0.5 * ty1); add(a.lv + c + sx, 0.5 * ty1);
            add(a.lv + c - sy, 0.5 * ty2); add(a.lv + c + sx - sy, 0.5 * ty2);
            add(a.lw + c + sx, 0.5 * tz1); add(a.lw + c, 0.5 * tz1);
            add(a.lw + c - sz, 0.5 * tz2); add(a.lw + c + sx - sz, 0.5 * tz2);
        }
    }
    // ---------------- v* (discretisation_QUICK_centre.f90:127-226)
    {
        const double rbar = a.lvs[c];
        if (a.gf) a.gf[a.fstride + c] += dt * rbar;
        if (rbar != 0.0) {
            double gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
            double tx1 = 0, tx2 = 0, ty1 = 0, ty2 = 0, tz1 = 0, tz2 = 0;
            AxisIn ax{v[c - 2 * sx], v[c - sx], v[c], v[c + sx], v[c + 2 * sx],
                      0.5 * (u[c] + u[c + sy]), 0.5 * (u[c - sx] + u[c + sy - sx]),
                      X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1],
                      X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i],
                      X.riD[i], X.rDs[i - 1], X.rDs[i], X.riD[i]};
            AxisIn ay{v[c - 2 * sy], v[c - sy], v[c], v[c + sy], v[c + 2 * sy],
                      0.5 * (v[c] + v[c + sy]), 0.5 * (v[c - sy] + v[c]),
                      Y.As[j], Y.Bs[j], Y.riD[j], Y.riD[j + 1], Y.riD[j + 2],
                      Y.As[j - 1], Y.Bs[j - 1], Y.riD[j - 1], Y.riD[j], Y.riD[j + 1],
                      Y.rDs[j], Y.riD[j], Y.riD[j + 1], Y.rDs[j]};
            AxisIn az{v[c - 2 * sz], v[c - sz], v[c], v[c + sz], v[c + 2 * sz],
                      0.5 * (w[c] + w[c + sy]), 0.5 * (w[c - sz] + w[c + sy - sz]),
                      Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1],
                      Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k],
                      Z.riD[k], Z.rDs[k - 1], Z.rDs[k], Z.riD[k]};
            axis_adj(ax, rbar, dt, nue, les, gx, tx1, tx2, nubar);
            axis_adj(ay, rbar, dt, nue, les, gy, ty1, ty2, nubar);
            axis_adj(az, rbar, dt, nue, les, gz, tz1, tz2, nubar);
            gy[3] += 0.5 * ty1; gy[2] += 0.5 * ty1 + 0.5 * ty2; gy[1] += 0.5 * ty2;
            add(a.lv + c, rbar + gx[2] + gy[2] + gz[2]);
            add(a.lv + c - 2 * sx, gx[0]); add(a.lv + c - sx, gx[1]);
            add(a.lv + c + sx, gx[3]); add(a.lv + c + 2 * sx, gx[4]);
            add(a.lv + c - 2 * sy, gy[0]); add(a.lv + c - sy, gy[1]);
            add(a.lv + c + sy, gy[3]); add(a.lv + c + 2 * sy, gy[4]);
            add(a.lv + c - 2 * sz, gz[0]); add(a.lv + c - sz, gz[1]);
            add(a.lv + c + sz, gz[3]); add(a.lv + c + 2 * sz, gz[4]);
            add(a.lu + c, 0.5 * tx1); add(a.lu + c + sy, 0.5 * tx1);
            add(a.lu + c - sx, 0.5 * tx2); add(a.lu + c + sy - sx, 0.5 * tx2);
            add(a.lw + c, 0.5 * tz1); add(a.lw + c + sy, 0.5 * tz1);
            add(a.lw + c - sz, 0.5 * tz2); add(a.lw + c + sy - sz, 0.5 * tz2);
        }
    }
    // ---------------- w* (discretisation_QUICK_centre.f90:240-339)
    {
        const double rbar = a.lws[c];
        if (a.gf) a.gf[2 * a.fstride + c] += dt * rbar;
        if (rbar != 0.0) {
            double gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
            double tx1 = 0, tx2 = 0, ty1 = 0, ty2 = 0, tz1 = 0, tz2 = 0;
            AxisIn ax{w[c - 2 * sx], w[c - sx], w[c], w[c + sx], w[c + 2 * sx],
                      0.5 * (u[c + sz] + u[c]), 0.5 * (u[c + sz - sx] + u[c - sx]),
                      X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1],
                      X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i],
                      X.riD[i], X.rDs[i - 1], X.rDs[i], X.riD[i]};
            AxisIn ay{w[c - 2 * sy], w[c - sy], w[c], w[c + sy], w[c + 2 * sy],
                      0.5 * (v[c] + v[c + sz]), 0.5 * (v[c + sz - sy] + v[c - sy]),
                      Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1],
                      Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j],
                      Y.riD[j], Y.rDs[j - 1], Y.rDs[j], Y.riD[j]};
            AxisIn az{w[c - 2 * sz], w[c - sz], w[c], w[c + sz], w[c + 2 * sz],
                      0.5 * (w[c + sz] + w[c]), 0.5 * (w[c] + w[c - sz]),
                      Z.As[k], Z.Bs[k], Z.riD[k], Z.riD[k + 1], Z.riD[k + 2],
                      Z.As[k - 1], Z.Bs[k - 1], Z.riD[k - 1], Z.riD[k], Z.riD[k + 1],
                      Z.rDs[k], Z.riD[k], Z.riD[k + 1], Z.rDs[k]};
            axis_adj(ax, rbar, dt, nue, les, gx, tx1, tx2, nubar);
            axis_adj(ay, rbar, dt, nue, les, gy, ty1, ty2, nubar);
            axis_adj(az, rbar, dt, nue, les, gz, tz1, tz2, nubar);
            gz[3] += 0.5 * tz1; gz[2] += 0.5 * tz1 + 0.5 * tz2; gz[1] += 0.5 * tz2;
            add(a.lw + c, rbar + gx[2] + gy[2] + gz[2]);
            add(a.lw + c - 2 * sx, gx[0]); add(a.lw + c - sx, gx[1]);
            add(a.lw + c + sx, gx[3]); add(a.lw + c + 2 * sx, gx[4]);
            add(a.lw + c - 2 * sy, gy[0]); add(a.lw + c - sy, gy[1]);
            add(a.lw + c + sy, gy[3]); add(a.lw + c + 2 * sy, gy[4]);
            add(a.lw + c - 2 * sz, gz[0]); add(a.lw + c - sz, gz[1]);
            add(a.lw + c + sz, gz[3]); add(a.lw + c + 2 * sz, gz[4]);
            add(a.lu + c + sz, 0.5 * tx1); add(a.lu + c, 0.5 * tx1);
            add(a.lu + c + sz - sx, 0.5 * tx2); add(a.lu + c - sx, 0.5 * tx2);
            add(a.lv + c, 0.5 * ty1); add(a.lv + c + sz, 0.5 * ty1);
            add(a.lv + c + sz - sy, 0.5 * ty2); add(a.lv + c - sy, 0.5 * ty2);
        }
    }
    if (a.lnut) a.lnut[c] += nubar;
}

// ------------------------------------------------------------- Smagorinsky
// Storage element that phi_read(i,j,k) reads, or -1 when it reads 0.
__device__ __forceinline__ long long phi_addr(const Geom& g, int i, int j, int k, bool aliased) {
    if (!aliased) return nat(g, i, j, k);
    const long long off = (long long)(i - 1) + (long long)(j - 1) * g.nx +
                          (long long)(k - 1) * g.nx * g.ny;
    const long long ax = g.nx + 4, ay = g.ny + 4;
    if (off < 0 || off >= ax * ay * (g.nz + 4)) return -1;
    const int a = (int)(off % ax);
    const long long t = off / ax;
    const int b = (int)(t % ay);
    const int cc = (int)(t / ay);
    return nat(g, a - 1, b - 1, cc - 1);
}

// Reverse of grad_gauss: out[d] = (f(+e_d) - f(-e_d)) * 0.5 * fact * (product of the other two
// metrics) -- the centre value cancels.
__device__ __forceinline__ void grad_gauss_adj(const Geom& g, double* lf, bool al, int i, int j, int k,
                                               const double* Dxm, const double* Dym, const double* Dzm,
                                               const double gb[3]) {
    const double fact = 1.0 / (Dxm[i] * Dym[j] * Dzm[k]);
    const double cx = 0.5 * fact * (Dym[j] * Dzm[k]) * gb[0];
    const double cy = 0.5 * fact * (Dxm[i] * Dzm[k]) * gb[1];
    const double cz = 0.5 * fact * (Dxm[i] * Dym[j]) * gb[2];
    auto put = [&](int a, int b, int c, double val) {
        if (val == 0.0) return;
        const long long q = phi_addr(g, a, b, c, al);
        if (q >= 0) atomicAdd(lf + q, val);
    };
    put(i + 1, j, k, cx); put(i - 1, j, k, -cx);
    put(i, j + 1, k, cy); put(i, j - 1, k, -cy);
    put(i, j, k + 1, cz); put(i, j, k - 1, -cz);
}

// nu_t = (Cs delta)^2 sqrt(S) (smagorinsky.f90:1-87); S = 0 gives a zero derivative.
__global__ void __launch_bounds__(128) k_adj_smagorinsky(Geom g, const double* u, const double* v,
                                                         const double* w, const double* lnut, double Cs,
                                                         int aliased, double* lu, double* lv, double* lw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const double nb = lnut[nat(g, i, j, k)];
    if (nb == 0.0) return;
    const bool al = aliased != 0;
    double du[3], dv[3], dw[3];
    grad_gauss(g, u, al, i, j, k, g.Dxs, g.iDy, g.iDz, du);
    grad_gauss(g, v, al, i, j, k, g.iDx, g.Dys, g.iDz, dv);
    grad_gauss(g, w, al, i, j, k, g.iDx, g.iDy, g.Dzs, dw);
    const double s01 = du[1] + dv[0], s02 = du[2] + dw[0], s12 = dv[2] + dw[1];
    const double S = 2 * (du[0] * du[0]) + 2 * (dv[1] * dv[1]) + 2 * (dw[2] * dw[2]) + s01 * s01 +
                     s02 * s02 + s12 * s12;
    if (!(S > 0.0)) return;
    const double delta = pow(g.iDx[i] * g.iDy[j] * g.iDz[k], (double)(1.f / 3.f));
    const double Sb = nb * (Cs * delta) * (Cs * delta) * 0.5 / sqrt(S);
    const double gu[3] = {4 * du[0] * Sb, 2 * s01 * Sb, 2 * s02 * Sb};
    const double gv[3] = {2 * s01 * Sb, 4 * dv[1] * Sb, 2 * s12 * Sb};
    const double gw[3] = {2 * s02 * Sb, 2 * s12 * Sb, 4 * dw[2] * Sb};
    grad_gauss_adj(g, lu, al, i, j, k, g.Dxs, g.iDy, g.iDz, gu);
    grad_gauss_adj(g, lv, al, i, j, k, g.iDx, g.Dys, g.iDz, gv);
    grad_gauss_adj(g, lw, al, i, j, k, g.iDx, g.iDy, g.Dzs, gw);
}

// ------------------------------------------------------------------ BCs
// Transposes of k_bc_x/y/z, statement by statement in reverse order.  A
// forward assignment dst = a*src + b*val becomes lam[src] += a*lam[dst],
// gval[wall][comp] += b*lam[dst], lam[dst] = 0.  gval collects the
// derivatives with respect to the Dirichlet values bc_value[wall][comp].
struct AdjBcArgs {
    double *lu, *lv, *lw, *lp;
    int bc[6][3];
    double* gval;   // [6][3], accumulated with atomics
};

__device__ __forceinline__ double take(double* a, long long q) {
    const double v = a[q];
    a[q] = 0.0;
    return v;
}

// reverse of a tangential ghost g = tangential(kind, val, f(inner), f(per)) written to
// both ghost layers d0 (first) and d1 (second; periodic: f(per2))
__device__ __forceinline__ void tang_adj(double* f, int kind, long long d0, long long d1, long long inner,
                                         long long per, long long per2, double* gv) {
    double A = take(f, d0);
    const double A1 = take(f, d1);
    if (kind == BC_PERIODIC) {
        f[per2] += A1;
        f[per] += A;
        return;
    }
    A += A1;
    if (kind == BC_NOSLIP) f[inner] -= A;
    else if (kind == BC_NEUMANN) f[inner] += A;
    else { *gv += 2.0 * A; f[inner] -= A; }
}

__global__ void k_adj_bc_x(Geom g, AdjBcArgs a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y - 1;
    double gv[6] = {0, 0, 0, 0, 0, 0};   // [W u,v,w; E u,v,w]
    if (j <= g.ny + 2 && k <= g.nz + 2) {
        const int nx = g.nx;
        auto I = [&](int i) { return nat(g, i, j, k); };
        // pressure (forward: p1, pn read first, then the ghosts written)
        if (a.bc[0][0] == BC_PERIODIC) {
            a.lp[I(nx)] += take(a.lp, I(0));
            a.lp[I(nx - 1)] += take(a.lp, I(-1));
            a.lp[I(1)] += take(a.lp, I(nx + 1));
            a.lp[I(2)] += take(a.lp, I(nx + 2));
        } else {
            const double A0 = take(a.lp, I(0)) + take(a.lp, I(-1));
            const double An = take(a.lp, I(nx + 1)) + take(a.lp, I(nx + 2));
            a.lp[I(1)] += A0;
            a.lp[I(nx)] += An;
        }
        // East w, v (tangential), then u
        double* f2[2] = {a.lv, a.lw};
        for (int c = 2; c >= 1; --c)
            tang_adj(f2[c - 1], a.bc[1][c], I(nx + 1), I(nx + 2), I(nx), I(1), I(2), &gv[3 + c]);
        {
            const int ku = a.bc[1][0];
            if (ku == BC_PERIODIC) {
                a.lu[I(2)] += take(a.lu, I(nx + 2));
                a.lu[I(1)] += take(a.lu, I(nx + 1));
            } else {
                const double A = take(a.lu, I(nx)) + take(a.lu, I(nx + 1)) + take(a.lu, I(nx + 2));
                if (ku == BC_NEUMANN) a.lu[I(nx - 1)] += A;
                else if (ku == BC_DIRICHLET) gv[3] += A;
            }
        }
        // West w, v (tangential), then u
        for (int c = 2; c >= 1; --c)
            tang_adj(f2[c - 1], a.bc[0][c], I(0), I(-1), I(1), I(nx), I(nx - 1), &gv[c]);
        {
            const int ku = a.bc[0][0];
            const double L1 = take(a.lu, I(-1));
            double A = take(a.lu, I(0));
            if (ku == BC_PERIODIC) a.lu[I(nx - 1)] += L1;
            else A += L1;
            if (ku == BC_NEUMANN) a.lu[I(1)] += A;
            else if (ku == BC_DIRICHLET) gv[0] += A;
            else if (ku == BC_PERIODIC) a.lu[I(nx)] += A;
        }
    }
    for (int q = 0; q < 6; ++q) {
        double v = gv[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (((threadIdx.x + threadIdx.y * blockDim.x) & 31) == 0 && v != 0.0) atomicAdd(&a.gval[(q / 3) * 3 + q % 3], v);
    }
}

__global__ void k_adj_bc_y(Geom g, AdjBcArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y - 1;
    double gv[6] = {0, 0, 0, 0, 0, 0};   // [S u,v,w; N u,v,w]
    if (i <= g.nx + 2 && k <= g.nz + 2) {
        const int ny = g.ny;
        auto J = [&](int j) { return nat(g, i, j, k); };
        if (a.bc[2][1] == BC_PERIODIC) {
            a.lp[J(ny)] += take(a.lp, J(0));
            a.lp[J(ny - 1)] += take(a.lp, J(-1));
            a.lp[J(1)] += take(a.lp, J(ny + 1));
            a.lp[J(2)] += take(a.lp, J(ny + 2));
        } else {
            const double A0 = take(a.lp, J(0)) + take(a.lp, J(-1));
            const double An = take(a.lp, J(ny + 1)) + take(a.lp, J(ny + 2));
            a.lp[J(1)] += A0;
            a.lp[J(ny)] += An;
        }
        // North w, v (normal), u
        tang_adj(a.lw, a.bc[3][2], J(ny + 1), J(ny + 2), J(ny), J(1), J(2), &gv[5]);
        {
            const int kv = a.bc[3][1];
            if (kv == BC_PERIODIC) {
                a.lv[J(2)] += take(a.lv, J(ny + 2));
                a.lv[J(1)] += take(a.lv, J(ny + 1));
            } else {
                const double A = take(a.lv, J(ny)) + take(a.lv, J(ny + 1)) + take(a.lv, J(ny + 2));
                if (kv == BC_NEUMANN) a.lv[J(ny - 1)] += A;
                else if (kv == BC_DIRICHLET) gv[4] += A;
            }
        }
        tang_adj(a.lu, a.bc[3][0], J(ny + 1), J(ny + 2), J(ny), J(1), J(2), &gv[3]);
        // South w, v (normal), u
        tang_adj(a.lw, a.bc[2][2], J(0), J(-1), J(1), J(ny), J(ny - 1), &gv[2]);
        {
            const int kv = a.bc[2][1];
            const double L1 = take(a.lv, J(-1));
            double A = take(a.lv, J(0));
            if (kv == BC_PERIODIC) a.lv[J(ny - 1)] += L1;
            else A += L1;
            if (kv == BC_NEUMANN) a.lv[J(1)] += A;
            else if (kv == BC_DIRICHLET) gv[1] += A;
            else if (kv == BC_PERIODIC) a.lv[J(ny)] += A;
        }
        tang_adj(a.lu, a.bc[2][0], J(0), J(-1), J(1), J(ny), J(ny - 1), &gv[0]);
    }
    for (int q = 0; q < 6; ++q) {
        double v = gv[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (((threadIdx.x + threadIdx.y * blockDim.x) & 31) == 0 && v != 0.0) atomicAdd(&a.gval[6 + q], v);
    }
}

__global__ void k_adj_bc_z(Geom g, AdjBcArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
    double gv[6] = {0, 0, 0, 0, 0, 0};   // [B u,v,w; F u,v,w]
    if (i <= g.nx + 2 && j <= g.ny + 2) {
        const int nz = g.nz;
        auto K = [&](int k) { return nat(g, i, j, k); };
        if (a.bc[4][2] == BC_PERIODIC) {
            a.lp[K(nz)] += take(a.lp, K(0));
            a.lp[K(nz - 1)] += take(a.lp, K(-1));
            a.lp[K(1)] += take(a.lp, K(nz + 1));
            a.lp[K(2)] += take(a.lp, K(nz + 2));
        } else {
            const double A0 = take(a.lp, K(0)) + take(a.lp, K(-1));
            const double An = take(a.lp, K(nz + 1)) + take(a.lp, K(nz + 2));
            a.lp[K(1)] += A0;
            a.lp[K(nz)] += An;
        }
        // Front: w (normal), then v, u
        {
            const int kw = a.bc[5][2];
            if (kw == BC_PERIODIC) {
                a.lw[K(2)] += take(a.lw, K(nz + 2));
                a.lw[K(1)] += take(a.lw, K(nz + 1));
            } else {
                const double A = take(a.lw, K(nz)) + take(a.lw, K(nz + 1)) + take(a.lw, K(nz + 2));
                if (kw == BC_NEUMANN) a.lw[K(nz - 1)] += A;
                else if (kw == BC_DIRICHLET) gv[5] += A;
            }
        }
        double* f2[2] = {a.lu, a.lv};
        for (int c = 1; c >= 0; --c)
            tang_adj(f2[c], a.bc[5][c], K(nz + 1), K(nz + 2), K(nz), K(1), K(2), &gv[3 + c]);
        // Back: w (normal), then v, u
        {
            const int kw = a.bc[4][2];
            const double L1 = take(a.lw, K(-1));
            double A = take(a.lw, K(0));
            if (kw == BC_PERIODIC) a.lw[K(nz - 1)] += L1;
            else A += L1;
            if (kw == BC_NEUMANN) a.lw[K(1)] += A;
            else if (kw == BC_DIRICHLET) gv[2] += A;
            else if (kw == BC_PERIODIC) a.lw[K(nz)] += A;
        }
        for (int c = 1; c >= 0; --c) {
            double* f = f2[c];
            const int kd = a.bc[4][c];
            if (kd == BC_NEUMANN && c == 1) {
                // forward: v(0) kept, v(-1) = v(0)
                f[K(0)] += take(f, K(-1));
                continue;
            }
            tang_adj(f, kd, K(0), K(-1), K(1), K(nz), K(nz - 1), &gv[c]);
        }
    }
    for (int q = 0; q < 6; ++q) {
        double v = gv[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (((threadIdx.x + threadIdx.y * blockDim.x) & 31) == 0 && v != 0.0) atomicAdd(&a.gval[12 + q], v);
    }
}

// ------------------------------------------------------------- objective
// d cDrag / d FZ(i,j,k) and d cLift / d FY(i,j,k) with the zero-guard
// pattern of the step held fixed (virtualForceIntegrator.f90:22-81):
//   (-2/lx) * ax(i) * ay(i,j) * wz(k),
//   ay = Dys(j)/6 ([FXz(i,j+1)!=0] + 4[FXz(i,j)!=0] + [FXz(i,j-1)!=0]),
//   ax = Dxs(i)/6 ([FXy(i+1)!=0] + 4[FXy(i)!=0] + [FXy(i-1)!=0]),
//   wz = Dzs(k) (4 + [k>1] + [k<nz]) / 6.
// The guards as bytes, per step: [nx*ny: FXz != 0][nx*ny: FYz != 0][nx: FXy != 0][nx: FYy != 0].
__global__ void k_pack_guards(Geom g, const double* FXz, const double* FYz, const double* FXy,
                              const double* FYy, unsigned char* out) {
    const long long n = (long long)g.nx * g.ny;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n + g.nx;
         q += (long long)gridDim.x * blockDim.x) {
        if (q < n) {
            out[q] = FXz[q] != 0.0;
            out[n + q] = FYz[q] != 0.0;
        } else {
            out[2 * n + (q - n)] = FXy[q - n] != 0.0;
            out[2 * n + g.nx + (q - n)] = FYy[q - n] != 0.0;
        }
    }
}

__global__ void k_adj_weights(Geom g, const unsigned char* guards, double scaleD, double scaleL,
                              double* wD, double* wL) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const int nx = g.nx, ny = g.ny;
    const long long n = (long long)nx * ny;
    const unsigned char* gXz = guards;
    const unsigned char* gYz = guards + n;
    const unsigned char* gXy = guards + 2 * n;
    const unsigned char* gYy = guards + 2 * n + nx;
    const long long q = (long long)(j - 1) * nx + (i - 1);
    const double ayD = g.Dys[j] / 6.0 * ((j < ny ? gXz[q + nx] : 0) + 4.0 * gXz[q] + (j > 1 ? gXz[q - nx] : 0));
    const double ayL = g.Dys[j] / 6.0 * ((j < ny ? gYz[q + nx] : 0) + 4.0 * gYz[q] + (j > 1 ? gYz[q - nx] : 0));
    const double axD = g.Dxs[i] / 6.0 * ((i < nx ? gXy[i] : 0) + 4.0 * gXy[i - 1] + (i > 1 ? gXy[i - 2] : 0));
    const double axL = g.Dxs[i] / 6.0 * ((i < nx ? gYy[i] : 0) + 4.0 * gYy[i - 1] + (i > 1 ? gYy[i - 2] : 0));
    const double wz = g.Dzs[k] * (4.0 + (k > 1 ? 1.0 : 0.0) + (k < g.nz ? 1.0 : 0.0)) / 6.0;
    const long long c = nat(g, i, j, k);
    wD[c] = scaleD * axD * ayD * wz;
    wL[c] = scaleL * axL * ayL * wz;
}

// ------------------------------------------------------------- projection
// u1 = u* - dt (p(i+1)-p(i))/Dxs(i), u2 = (1-eta) u1 + eta us, F = (u2-u1)/dt.
// lam_u2 = lu (after the boundary-condition transpose); the objective adds
// dJ/dFZ = wD (drag) and dJ/dFY = wL (lift).  FZ = eta (w_solid - w1) / dt.
__global__ void k_adj_project1(Geom g, double* lu, double* lv, double* lw, const double* eta,
                               const double* wD, const double* wL, double dt, double* lus, double* lvs,
                               double* lws) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double e = eta[c];
    lus[c] = (1 - e) * lu[c];
    lvs[c] = (1 - e) * lv[c] - e / dt * wL[c];
    lws[c] = (1 - e) * lw[c] - e / dt * wD[c];
    // the step overwrites the whole interior: from here lu, lv, lw collect the state before it
    lu[c] = 0.0;
    lv[c] = 0.0;
    lw[c] = 0.0;
}

// dJ/dETA of one step, accumulated into geta: ETA enters u2 = (1 - eta) u1 + eta us
// (likewise v, w) and the force integrands FY = eta (vs - v1)/dt, FZ = eta (ws - w1)/dt,
// with u1 = u* - dt (p(i+1) - p(i))/Dxs(i): p^{n+1} inside (pn), the frozen ghosts of
// p^n at i = nx+1, j = ny+1, k = nz+1 (po), as k_project reads them.  lu, lv, lw hold
// lam of u2 after the boundary-condition transpose, wD and wL dJ/dFZ and dJ/dFY.
__global__ void k_adj_eta(Geom g, const double* lu, const double* lv, const double* lw, const double* wD,
                          const double* wL, const double* us, const double* vs, const double* ws,
                          const double* pn, const double* po, double usol, double vsol, double wsol, double dt,
                          double* geta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double pc = pn[c];
    const double pe = (i == g.nx ? po : pn)[c + 1];
    const double pnn = (j == g.ny ? po : pn)[c + g.px];
    const double pf = (k == g.nz ? po : pn)[c + g.pz];
    const double u1 = us[c] - dt * (pe - pc) * g.rDxs[i];
    const double v1 = vs[c] - dt * (pnn - pc) * g.rDys[j];
    const double w1 = ws[c] - dt * (pf - pc) * g.rDzs[k];
    geta[c] += lu[c] * (usol - u1) + lv[c] * (vsol - v1) + lw[c] * (wsol - w1) +
               (wL[c] * (vsol - v1) + wD[c] * (wsol - w1)) / dt;
}

// Column sums over i of a natural-layout field into a (k,j) plane (k fastest).
__global__ void k_colsum_i(Geom g, const double* f, double* plane) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > g.nz || j > g.ny) return;
    double s = 0.0;
    for (int i = 1; i <= g.nx; ++i) s += f[nat(g, i, j, k)];
    plane[(long long)(k - 1) + (long long)g.nz * (j - 1)] = s;
}

// lam_p of p^{n+1} (interior, gathered) and of the frozen ghosts of p^n
// (i = nx+1, j = ny+1, k = nz+1) from lam_u1 = lus etc.
__global__ void k_adj_project2(Geom g, const double* lus, const double* lvs, const double* lws, double dt,
                               double* lp_new, double* lp_old) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    double s = g.rDxs[i] * lus[c] + g.rDys[j] * lvs[c] + g.rDzs[k] * lws[c];
    if (i > 1) s -= g.rDxs[i - 1] * lus[c - 1];
    if (j > 1) s -= g.rDys[j - 1] * lvs[c - g.px];
    if (k > 1) s -= g.rDzs[k - 1] * lws[c - g.pz];
    lp_new[c] += dt * s;
    if (i == g.nx) lp_old[c + 1] -= dt * g.rDxs[i] * lus[c];
    if (j == g.ny) lp_old[c + g.px] -= dt * g.rDys[j] * lvs[c];
    if (k == g.nz) lp_old[c + g.pz] -= dt * g.rDzs[k] * lws[c];
}

// ------------------------------------------------------------- pressure solve
// Right-hand side of M z = V^-1 lam_p, in the SOR's b' form: b_adj = -rd * lam_p / V
__global__ void k_adj_solve_rhs(Geom g, SorCoef<double> sc, const double* lp_new, double* badj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double V = g.iDx[i] * g.iDy[j] * g.iDz[k];
    badj[c] = -rdiag_of(sc, i, j, k) * lp_new[c] / V;
}

// y = V z; lam_b' = -y / rd; lam of the frozen ghosts of p^n += c_nb * y
__global__ void k_adj_after_solve(Geom g, SorCoef<double> sc, const double* z, double* lb, double* lp_old) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double y = g.iDx[i] * g.iDy[j] * g.iDz[k] * z[c];
    lb[c] = -y / rdiag_of(sc, i, j, k);
    if (i == 1) lp_old[c - 1] += sc.cW[i] * y;
    if (i == g.nx) lp_old[c + 1] += sc.cE[i] * y;
    if (j == 1) lp_old[c - g.px] += sc.cS[j] * y;
    if (j == g.ny) lp_old[c + g.px] += sc.cN[j] * y;
    if (k == 1) lp_old[c - g.pz] += sc.cB[k] * y;
    if (k == g.nz) lp_old[c + g.pz] += sc.cF[k] * y;
}

// ------------------------------------------------------------- divergence RHS
// b'(c) = rd(c)/dt [(u*(c)-u*(c-ex)) riDx + (v*(c)-v*(c-ey)) riDy + (w*(c)-w*(c-ez)) riDz],
// with u*(0,j,k) = u(0,j,k) etc.: gather onto u*, v*, w* and the state's ghosts.
__global__ void k_adj_rhs(Geom g, SorCoef<double> sc, const double* lb, double dt, double* lus,
                          double* lvs, double* lws, double* lu_old, double* lv_old, double* lw_old) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double f0 = rdiag_of(sc, i, j, k) / dt * lb[c];
    double gu = g.riDx[i] * f0, gv = g.riDy[j] * f0, gw = g.riDz[k] * f0;
    if (i < g.nx) gu -= g.riDx[i + 1] * rdiag_of(sc, i + 1, j, k) / dt * lb[c + 1];
    if (j < g.ny) gv -= g.riDy[j + 1] * rdiag_of(sc, i, j + 1, k) / dt * lb[c + g.px];
    if (k < g.nz) gw -= g.riDz[k + 1] * rdiag_of(sc, i, j, k + 1) / dt * lb[c + g.pz];
    lus[c] += gu;
    lvs[c] += gv;
    lws[c] += gw;
    if (i == 1) lu_old[c - 1] -= g.riDx[i] * f0;
    if (j == 1) lv_old[c - g.px] -= g.riDy[j] * f0;
    if (k == 1) lw_old[c - g.pz] -= g.riDz[k] * f0;
}

// Initial guess of the next adjoint solve by linear extrapolation in time:
// z <- 2 z - zprev, zprev <- old z (interior).
__global__ void k_extrapolate(Geom g, double* z, double* zprev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double z1 = z[c];
    z[c] = 2.0 * z1 - zprev[c];
    zprev[c] = z1;
}

// max |x| over the interior (the adjoint solve's tolerance is relative to it)
template <int NT>
__global__ void __launch_bounds__(NT) k_absmax(Geom g, const double* x, unsigned long long* slot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    double v = 0.0;
    if (i <= g.nx && j <= g.ny && k <= g.nz) v = x[nat(g, i, j, k)];
    block_max_atomic<NT>(v, slot);
}

// natural-layout interior <- contiguous (nx,ny,nz) Fortran-order array (ghosts untouched)
__global__ void k_interior_in(Geom g, const double* src, double* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    dst[nat(g, i, j, k)] = src[(i - 1) + (long long)g.nx * ((j - 1) + (long long)g.ny * (k - 1))];
}

__global__ void k_interior_out(Geom g, const double* src, double* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    dst[(i - 1) + (long long)g.nx * ((j - 1) + (long long)g.ny * (k - 1))] = src[nat(g, i, j, k)];
}

}  // namespace ntcfd
