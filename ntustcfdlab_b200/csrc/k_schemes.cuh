// k_schemes.cuh -- K2 alternatives to discretisation_QUICK_centre: the
// predictors of discretisation_QUICK.f90, discretisation_upwind.f90 and
// discretisation_centre.f90.
//
// The reference keeps these three files but never calls them (main.f90:213
// calls discretisation_QUICK_centre) and cannot compile them: they test a
// flag Q1 that variables_module.f90 does not declare under implicit none.
// Here Q1 is the LES switch of ntcfd_params, nu = 1/Re (reading_data.f90:38)
// and Cs comes from the parameters.  What the three share, and how they
// differ from QUICK_centre:
//  * u* is predicted on i = 1..nx-1, v* on j = 1..ny-1, w* on k = 1..nz-1;
//    the wall faces keep u*(nx) = u(nx) etc., which the reference gets from
//    the u -> u_star copies of boundary_conditions.f90:305-324.
//  * With Q1 = 1 the eddy viscosity is evaluated inline at the staggered
//    point of each component (the same three blocks in all three files,
//    e.g. discretisation_upwind.f90:66-80,156-170,245-259); nothing reads
//    the Viseff of smagorinsky.f90.
//  * The diffusion terms are those of QUICK_centre.
// Convection:
//  * QUICK: face values by the QUICK interpolation upwinded on the node
//    velocity (u(i,j,k) > 0 for every x-face, v for y, w for z) and fluxes
//    as products of two face values (ue*ue, un*vnu, ...),
//    discretisation_QUICK.f90:5-413.
//  * upwind: first-order upwind face values on the face-averaged velocity
//    (>= 0 picks the upstream node), fluxes u_tilde * face value,
//    discretisation_upwind.f90:7-273.
//  * centre: the arithmetic mean of the two nodes, fluxes
//    0.5 u_tilde (f(a) + f(a+1)), discretisation_centre.f90:7-132.
// The stencil reads and their index ranges are the reference's as written,
// including the v_tilde_z1 = 0.5 (v(i,j,k) + v(i+1,j,k+1)) of
// discretisation_upwind.f90:195.  Divisions by metrics are multiplications
// by tabulated reciprocals, as in k_predictor.
#pragma once

#include "k_predictor.cuh"

namespace ntcfd {

constexpr int kSchemeQuick = 1, kSchemeUpwind = 2, kSchemeCentre = 3;   // NTCFD_QUICK, _UPWIND, _CENTRE

// A field around the thread's cell c: f(di, dj, dk) = f(i+di, j+dj, k+dk).
struct Fld {
    const double* p;
    long long c, sy, sz;
    __device__ __forceinline__ double operator()(int di, int dj, int dk) const {
        return __ldg(p + c + di + dj * sy + dk * sz);
    }
};

__device__ __forceinline__ double sq(double x) { return x * x; }

// The reference's Q1 = 1 eddy viscosity at the u point (i+1/2, j, k):
//  nut = (Cs delta)^2 sqrt(S), delta = (Dxs(i) iDy(j) iDz(k))^(1./3.) with
//  the default-real exponent, S the six-term sum of the reference.

__device__ __forceinline__ double nut_u(const Geom& g, const Fld& u, const Fld& v, const Fld& w, int i, int j,
                                        int k, double Cs) {
    const double hx = g.Dxs[i], hy = g.iDy[j], hz = g.iDz[k];
    const double rx = g.rDxs[i], ry = g.riDy[j], rz = g.riDz[k];
    const double U0 = u(0, 0, 0);
    const double s = 0.5 * (rx * rx) * sq((u(1, 0, 0) + U0) - (U0 + u(-1, 0, 0))) +
                     0.5 * (ry * ry) * sq((v(1, 0, 0) + v(0, 0, 0)) - (v(1, -1, 0) + v(0, -1, 0))) +
                     0.5 * (rz * rz) * sq((w(1, 0, 0) + w(0, 0, 0)) - (w(1, 0, -1) + w(0, 0, -1))) +
                     sq(0.5 * ry * ((u(0, 1, 0) + U0) - (U0 + u(0, -1, 0))) +
                        0.5 * rx * ((v(1, 0, 0) + v(1, -1, 0)) - (v(0, 0, 0) + v(0, -1, 0)))) +
                     sq(0.5 * rz * ((u(0, 0, 1) + U0) - (U0 + u(0, 0, -1))) +
                        0.5 * rx * ((w(1, 0, 0) + w(1, 0, -1)) - (w(0, 0, 0) + w(0, 0, -1)))) +
                     sq(0.5 * rz * ((v(1, 0, 1) + v(0, -1, 0)) - (v(1, 0, -1) + v(0, -1, 0))) +
                        0.5 * ry * ((w(1, 1, 0) + w(0, 0, -1)) - (w(1, -1, 0) + w(0, 0, -1))));
    const double delta = pow(hx * hy * hz, (double)(1.f / 3.f));
    return sq(Cs * delta) * sqrt(s);
}

// ... at the v point (i, j+1/2, k): delta from iDx(i) Dys(j) iDz(k)
__device__ __forceinline__ double nut_v(const Geom& g, const Fld& u, const Fld& v, const Fld& w, int i, int j,
                                        int k, double Cs) {
    const double hx = g.iDx[i], hy = g.Dys[j], hz = g.iDz[k];
    const double rx = g.riDx[i], ry = g.rDys[j], rz = g.riDz[k];
    const double V0 = v(0, 0, 0);
    const double s = 0.5 * (rx * rx) * sq((u(0, 1, 0) + u(0, 0, 0)) - (u(-1, 1, 0) + u(-1, 0, 0))) +
                     0.5 * (ry * ry) * sq((v(0, 1, 0) + V0) - (V0 + v(0, -1, 0))) +
                     0.5 * (rz * rz) * sq((w(0, 1, 0) + w(0, 0, 0)) - (w(0, 1, -1) + w(0, 0, -1))) +
                     sq(0.5 * ry * ((u(0, 1, 0) + u(-1, 1, 0)) - (u(0, 0, 0) + u(-1, 0, 0))) +
                        0.5 * rx * ((v(1, 0, 0) + V0) - (V0 + v(-1, 0, 0)))) +
                     sq(0.5 * rz * ((u(0, 1, 1) + u(-1, 0, 0)) - (u(0, 1, -1) + u(-1, 0, -1))) +
                        0.5 * rx * ((w(1, 1, 0) + w(0, 0, -1)) - (w(-1, 1, 0) + w(0, 0, -1)))) +
                     sq(0.5 * rz * ((v(0, 0, 1) + V0) - (v(0, 0, -1) + V0)) +
                        0.5 * ry * ((w(0, 1, 0) + w(0, 1, -1)) - (w(0, 0, 0) + w(0, 0, -1))));
    const double delta = pow(hx * hy * hz, (double)(1.f / 3.f));
    return sq(Cs * delta) * sqrt(s);
}

// ... at the w point (i, j, k+1/2): delta from iDx(i) iDy(j) Dzs(k)
__device__ __forceinline__ double nut_w(const Geom& g, const Fld& u, const Fld& v, const Fld& w, int i, int j,
                                        int k, double Cs) {
    const double hx = g.iDx[i], hy = g.iDy[j], hz = g.Dzs[k];
    const double rx = g.riDx[i], ry = g.riDy[j], rz = g.rDzs[k];
    const double W0 = w(0, 0, 0);
    const double s = 0.5 * (rx * rx) * sq((u(0, 0, 1) + u(0, 0, 0)) - (u(-1, 0, 1) + u(-1, 0, 0))) +
                     0.5 * (ry * ry) * sq((v(0, 0, 1) + v(0, 0, 0)) - (v(0, -1, 1) + v(0, -1, 0))) +
                     0.5 * (rz * rz) * sq((w(0, 0, 1) + W0) - (W0 + w(0, 0, -1))) +
                     sq(0.5 * ry * ((u(0, 1, 0) + u(0, 0, 0)) - (u(0, 0, 0) + u(0, -1, 0))) +
                        0.5 * rx * ((v(1, 0, 1) + v(0, -1, 0)) - (v(-1, 0, 1) + v(0, -1, 0)))) +
                     sq(0.5 * rz * ((u(0, 0, 1) + u(-1, 0, 1)) - (u(0, 0, 0) + u(-1, 0, 0))) +
                        0.5 * rx * ((w(1, 0, 0) + W0) - (w(-1, 0, 0) + W0))) +
                     sq(0.5 * rz * ((v(0, 0, 1) + v(0, -1, 1)) - (v(0, 0, 0) + v(0, -1, 0))) +
                        0.5 * ry * ((w(0, 1, 0) + W0) - (w(0, -1, 0) + W0)));
    const double delta = pow(hx * hy * hz, (double)(1.f / 3.f));
    return sq(Cs * delta) * sqrt(s);
}

// First-order upwind face value: the upstream node when adv >= 0.
__device__ __forceinline__ double upw(double adv, double up, double down) { return adv >= 0 ? up : down; }

// One thread per cell; each thread predicts the three components of its
// cell (or copies the wall faces).  Body force: added at the predicted
// points.
template <int S>
__global__ void __launch_bounds__(256) k_predictor_scheme(Geom g, Tabs<double> tb, PredArgs a, double Cs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const Fld u{a.u, c, g.px, g.pz}, v{a.v, c, g.px, g.pz}, w{a.w, c, g.px, g.pz};
    const AxisTabs<double>&X = tb.ax[0], &Y = tb.ax[1], &Z = tb.ax[2];
    const double dt = a.dt;

    // ---------------- u* on i = 1..nx-1 (discretisation_*.f90, x component)
    if (i < g.nx) {
        const double U0 = u(0, 0, 0), U1 = u(1, 0, 0), Um1 = u(-1, 0, 0);
        const double Un1 = u(0, 1, 0), Us1 = u(0, -1, 0), Uf1 = u(0, 0, 1), Ub1 = u(0, 0, -1);
        double cx, cy, cz;
        if constexpr (S == kSchemeQuick) {
            const double U2 = u(2, 0, 0), Um2 = u(-2, 0, 0);
            const double au = U0, av = v(0, 0, 0), aw = w(0, 0, 0);
            const double ue = quick_face(Um1, U0, U1, U2, au, X.As[i], X.Bs[i], X.riD[i], X.riD[i + 1], X.riD[i + 2]);
            const double uw = quick_face(Um2, Um1, U0, U1, au, X.As[i - 1], X.Bs[i - 1], X.riD[i - 1], X.riD[i],
                                         X.riD[i + 1]);
            const double vnu = quick_face(v(-1, 0, 0), v(0, 0, 0), v(1, 0, 0), v(2, 0, 0), au, X.Ac[i], X.Bc[i],
                                          X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
            const double vsu = quick_face(v(-1, -1, 0), v(0, -1, 0), v(1, -1, 0), v(2, -1, 0), au, X.Ac[i], X.Bc[i],
                                          X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
            const double wfu = quick_face(w(-1, 0, 0), w(0, 0, 0), w(1, 0, 0), w(2, 0, 0), au, X.Ac[i], X.Bc[i],
                                          X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
            const double wbu = quick_face(w(-1, 0, -1), w(0, 0, -1), w(1, 0, -1), w(2, 0, -1), au, X.Ac[i], X.Bc[i],
                                          X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
            const double un = quick_face(Us1, U0, Un1, u(0, 2, 0), av, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j],
                                         Y.rDs[j + 1]);
            const double us = quick_face(u(0, -2, 0), Us1, U0, Un1, av, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2],
                                         Y.rDs[j - 1], Y.rDs[j]);
            const double uf = quick_face(Ub1, U0, Uf1, u(0, 0, 2), aw, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k],
                                         Z.rDs[k + 1]);
            const double ub = quick_face(u(0, 0, -2), Ub1, U0, Uf1, aw, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2],
                                         Z.rDs[k - 1], Z.rDs[k]);
            cx = dt * (ue * ue - uw * uw);
            cy = dt * (un * vnu - us * vsu);
            cz = dt * (uf * wfu - ub * wbu);
        } else {
            const double ut1 = 0.5 * (U0 + U1), ut2 = 0.5 * (Um1 + U0);
            const double vt1 = 0.5 * (v(0, 0, 0) + v(1, 0, 0)), vt2 = 0.5 * (v(0, -1, 0) + v(1, -1, 0));
            const double wt1 = 0.5 * (w(1, 0, 0) + w(0, 0, 0)), wt2 = 0.5 * (w(0, 0, -1) + w(1, 0, -1));
            if constexpr (S == kSchemeUpwind) {
                cx = dt * (ut1 * upw(ut1, U0, U1) - ut2 * upw(ut2, Um1, U0));
                cy = dt * (vt1 * upw(vt1, U0, Un1) - vt2 * upw(vt2, Us1, U0));
                cz = dt * (wt1 * upw(wt1, U0, Uf1) - wt2 * upw(wt2, Ub1, U0));
            } else {
                cx = dt * 0.5 * (ut1 * (U0 + U1) - ut2 * (U0 + Um1));
                cy = dt * 0.5 * (vt1 * (U0 + Un1) - vt2 * (U0 + Us1));
                cz = dt * 0.5 * (wt1 * (U0 + Uf1) - wt2 * (U0 + Ub1));
            }
        }
        const double nue = a.les ? a.nu + nut_u(g, u, v, w, i, j, k, Cs) : a.nu;
        const double r = U0 - cx * X.rDs[i] - cy * Y.riD[j] - cz * Z.riD[k]
                       + nue * dt * ((U1 - U0) * X.riD[i + 1] - (U0 - Um1) * X.riD[i]) * X.rDs[i]
                       + nue * dt * ((Un1 - U0) * Y.rDs[j] - (U0 - Us1) * Y.rDs[j - 1]) * Y.riD[j]
                       + nue * dt * ((Uf1 - U0) * Z.rDs[k] - (U0 - Ub1) * Z.rDs[k - 1]) * Z.riD[k];
        a.us[c] = a.fb ? r + dt * __ldg(a.fb + c) : r;
    } else {
        a.us[c] = u(0, 0, 0);
    }

    // ---------------- v* on j = 1..ny-1 (y component)
    if (j < g.ny) {
        const double V0 = v(0, 0, 0), V1 = v(1, 0, 0), Vm1 = v(-1, 0, 0);
        const double Vn1 = v(0, 1, 0), Vs1 = v(0, -1, 0), Vf1 = v(0, 0, 1), Vb1 = v(0, 0, -1);
        double cx, cy, cz;
        if constexpr (S == kSchemeQuick) {
            const double au = u(0, 0, 0), av = V0, aw = w(0, 0, 0);
            const double ve = quick_face(Vm1, V0, V1, v(2, 0, 0), au, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i],
                                         X.rDs[i + 1]);
            const double vw = quick_face(v(-2, 0, 0), Vm1, V0, V1, au, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2],
                                         X.rDs[i - 1], X.rDs[i]);
            const double uev = quick_face(u(0, -1, 0), u(0, 0, 0), u(0, 1, 0), u(0, 2, 0), av, Y.Ac[j], Y.Bc[j],
                                          Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
            const double uwv = quick_face(u(-1, -1, 0), u(-1, 0, 0), u(-1, 1, 0), u(-1, 2, 0), av, Y.Ac[j], Y.Bc[j],
                                          Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
            const double vn = quick_face(Vs1, V0, Vn1, v(0, 2, 0), av, Y.As[j], Y.Bs[j], Y.riD[j], Y.riD[j + 1],
                                         Y.riD[j + 2]);
            const double vs = quick_face(v(0, -2, 0), Vs1, V0, Vn1, av, Y.As[j - 1], Y.Bs[j - 1], Y.riD[j - 1],
                                         Y.riD[j], Y.riD[j + 1]);
            const double wfv = quick_face(w(0, -1, 0), w(0, 0, 0), w(0, 1, 0), w(0, 2, 0), av, Y.Ac[j], Y.Bc[j],
                                          Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
            const double wbv = quick_face(w(0, -1, -1), w(0, 0, -1), w(0, 1, -1), w(0, 2, -1), av, Y.Ac[j], Y.Bc[j],
                                          Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
            const double vf = quick_face(Vb1, V0, Vf1, v(0, 0, 2), aw, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k],
                                         Z.rDs[k + 1]);
            const double vb = quick_face(v(0, 0, -2), Vb1, V0, Vf1, aw, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2],
                                         Z.rDs[k - 1], Z.rDs[k]);
            cx = dt * (uev * ve - uwv * vw);
            cy = dt * (vn * vn - vs * vs);
            cz = dt * (vf * wfv - vb * wbv);
        } else {
            const double ut1 = 0.5 * (u(0, 0, 0) + u(0, 1, 0)), ut2 = 0.5 * (u(-1, 0, 0) + u(-1, 1, 0));
            const double vt1 = 0.5 * (V0 + Vn1), vt2 = 0.5 * (Vs1 + V0);
            const double wt1 = 0.5 * (w(0, 0, 0) + w(0, 1, 0)), wt2 = 0.5 * (w(0, 0, -1) + w(0, 1, -1));
            if constexpr (S == kSchemeUpwind) {
                cx = dt * (ut1 * upw(ut1, V0, V1) - ut2 * upw(ut2, Vm1, V0));
                cy = dt * (vt1 * upw(vt1, V0, Vn1) - vt2 * upw(vt2, Vs1, V0));
                cz = dt * (wt1 * upw(wt1, V0, Vf1) - wt2 * upw(wt2, Vb1, V0));
            } else {
                cx = dt * 0.5 * (ut1 * (V0 + V1) - ut2 * (V0 + Vm1));
                cy = dt * 0.5 * (vt1 * (V0 + Vn1) - vt2 * (V0 + Vs1));
                cz = dt * 0.5 * (wt1 * (V0 + Vf1) - wt2 * (V0 + Vb1));
            }
        }
        const double nue = a.les ? a.nu + nut_v(g, u, v, w, i, j, k, Cs) : a.nu;
        const double r = V0 - cx * X.riD[i] - cy * Y.rDs[j] - cz * Z.riD[k]
                       + nue * dt * ((V1 - V0) * X.rDs[i] - (V0 - Vm1) * X.rDs[i - 1]) * X.riD[i]
                       + nue * dt * ((Vn1 - V0) * Y.riD[j + 1] - (V0 - Vs1) * Y.riD[j]) * Y.rDs[j]
                       + nue * dt * ((Vf1 - V0) * Z.rDs[k] - (V0 - Vb1) * Z.rDs[k - 1]) * Z.riD[k];
        a.vs[c] = a.fb ? r + dt * __ldg(a.fb + a.fstride + c) : r;
    } else {
        a.vs[c] = v(0, 0, 0);
    }

    // ---------------- w* on k = 1..nz-1 (z component)
    if (k < g.nz) {
        const double W0 = w(0, 0, 0), W1 = w(1, 0, 0), Wm1 = w(-1, 0, 0);
        const double Wn1 = w(0, 1, 0), Ws1 = w(0, -1, 0), Wf1 = w(0, 0, 1), Wb1 = w(0, 0, -1);
        double cx, cy, cz;
        if constexpr (S == kSchemeQuick) {
            const double au = u(0, 0, 0), av = v(0, 0, 0), aw = W0;
            const double we = quick_face(Wm1, W0, W1, w(2, 0, 0), au, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i],
                                         X.rDs[i + 1]);
            const double ww = quick_face(w(-2, 0, 0), Wm1, W0, W1, au, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2],
                                         X.rDs[i - 1], X.rDs[i]);
            const double wn = quick_face(Ws1, W0, Wn1, w(0, 2, 0), av, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j],
                                         Y.rDs[j + 1]);
            const double ws = quick_face(w(0, -2, 0), Ws1, W0, Wn1, av, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2],
                                         Y.rDs[j - 1], Y.rDs[j]);
            const double uew = quick_face(u(0, 0, -1), u(0, 0, 0), u(0, 0, 1), u(0, 0, 2), aw, Z.Ac[k], Z.Bc[k],
                                          Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
            const double uww = quick_face(u(-1, 0, -1), u(-1, 0, 0), u(-1, 0, 1), u(-1, 0, 2), aw, Z.Ac[k], Z.Bc[k],
                                          Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
            const double vnw = quick_face(v(0, 0, -1), v(0, 0, 0), v(0, 0, 1), v(0, 0, 2), aw, Z.Ac[k], Z.Bc[k],
                                          Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
            const double vsw = quick_face(v(0, -1, -1), v(0, -1, 0), v(0, -1, 1), v(0, -1, 2), aw, Z.Ac[k], Z.Bc[k],
                                          Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
            const double wf = quick_face(Wb1, W0, Wf1, w(0, 0, 2), aw, Z.As[k], Z.Bs[k], Z.riD[k], Z.riD[k + 1],
                                         Z.riD[k + 2]);
            const double wb = quick_face(w(0, 0, -2), Wb1, W0, Wf1, aw, Z.As[k - 1], Z.Bs[k - 1], Z.riD[k - 1],
                                         Z.riD[k], Z.riD[k + 1]);
            cx = dt * (uew * we - uww * ww);
            cy = dt * (vnw * wn - vsw * ws);
            cz = dt * (wf * wf - wb * wb);
        } else {
            const double ut1 = 0.5 * (u(0, 0, 1) + u(0, 0, 0)), ut2 = 0.5 * (u(-1, 0, 1) + u(-1, 0, 0));
            // discretisation_upwind.f90:195 averages v(i,j,k) and v(i+1,j,k+1)
            const double vt1 = S == kSchemeUpwind ? 0.5 * (v(0, 0, 0) + v(1, 0, 1)) : 0.5 * (v(0, 0, 0) + v(0, 0, 1));
            const double vt2 = 0.5 * (v(0, -1, 1) + v(0, -1, 0));
            const double wt1 = 0.5 * (Wf1 + W0), wt2 = 0.5 * (W0 + Wb1);
            if constexpr (S == kSchemeUpwind) {
                cx = dt * (ut1 * upw(ut1, W0, W1) - ut2 * upw(ut2, Wm1, W0));
                cy = dt * (vt1 * upw(vt1, W0, Wn1) - vt2 * upw(vt2, Ws1, W0));
                cz = dt * (wt1 * upw(wt1, W0, Wf1) - wt2 * upw(wt2, Wb1, W0));
            } else {
                cx = dt * 0.5 * (ut1 * (W0 + W1) - ut2 * (W0 + Wm1));
                cy = dt * 0.5 * (vt1 * (W0 + Wn1) - vt2 * (W0 + Ws1));
                cz = dt * 0.5 * (wt1 * (W0 + Wf1) - wt2 * (W0 + Wb1));
            }
        }
        const double nue = a.les ? a.nu + nut_w(g, u, v, w, i, j, k, Cs) : a.nu;
        const double r = W0 - cx * X.riD[i] - cy * Y.riD[j] - cz * Z.rDs[k]
                       + nue * dt * ((W1 - W0) * X.rDs[i] - (W0 - Wm1) * X.rDs[i - 1]) * X.riD[i]
                       + nue * dt * ((Wn1 - W0) * Y.rDs[j] - (W0 - Ws1) * Y.rDs[j - 1]) * Y.riD[j]
                       + nue * dt * ((Wf1 - W0) * Z.riD[k + 1] - (W0 - Wb1) * Z.riD[k]) * Z.rDs[k];
        a.ws[c] = a.fb ? r + dt * __ldg(a.fb + 2 * a.fstride + c) : r;
    } else {
        a.ws[c] = w(0, 0, 0);
    }
}

}  // namespace ntcfd
