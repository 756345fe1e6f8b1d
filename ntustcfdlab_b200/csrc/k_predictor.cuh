// k_predictor.cuh -- K1 Smagorinsky nu_t and K2 QUICK/central predictor.
//
// K2 follows discretisation_QUICK_centre.f90:7-342 term by term.  Every
// division by a metric is a multiplication by a tabulated reciprocal, and
// the QUICK correction factors 0.125*h^2/H are tabulated per face; the
// algebra is the reference's, the rounding differs at the last bit.
#pragma once

#include "ntcfd_common.cuh"

namespace ntcfd {

// Per-axis tables (pointers pre-offset, valid for index -2..n+2).
//  riD = 1/iD, rDs = 1/Ds,
//  "staggered" faces (component along the axis):  As(a) = 0.125 iD(a+1)^2 / Ds(a),
//                                                 Bs(a) = 0.125 iD(a+1)^2 / Ds(a+1)
//  "centred" faces (component across the axis):   Ac(a) = 0.125 Ds(a)^2 / iD(a),
//                                                 Bc(a) = 0.125 Ds(a)^2 / iD(a+1)
template <class T>
struct AxisTabs {
    const T *riD, *rDs, *As, *Bs, *Ac, *Bc;
};
template <class T>
struct Tabs {
    AxisTabs<T> ax[3];
};

// QUICK face value between cells a and a+1 of a row f(.), upwinded on adv
// (discretisation_QUICK_centre.f90:18-30 and the 17 sibling blocks).
// fm1 = f(a-1), f0 = f(a), f1 = f(a+1), f2 = f(a+2); A/B the face factors,
// r0 = 1/h(a-1..a), r1 = 1/h(a..a+1), r2 = 1/h(a+1..a+2).
template <class T>
__device__ __forceinline__ T quick_face(T fm1, T f0, T f1, T f2, T adv, T A, T B, T r0, T r1,
                                        T r2) {
    const T mid = T(0.5) * (f0 + f1);
    return (adv > T(0)) ? mid - A * ((f1 - f0) * r1 - (f0 - fm1) * r0)
                        : mid - B * ((f2 - f1) * r2 - (f1 - f0) * r1);
}

struct PredArgs {
    const double* u;
    const double* v;
    const double* w;
    const double* nut;   // null when LES = 0
    double* us;
    double* vs;
    double* ws;
    double dt, nu;
    int les;
    const double* fb;    // body force (fu, fv, fw: three natural-layout arrays, N apart), or null
    long long fstride;   // N
};

// One thread per cell (i,j,k), i fastest, in blocks of kPredBX x kPredBY x
// kPredBZ.  Reads u,v,w (+-2 stencil) and writes u*, v*, w* on the interior
// 1..nx, 1..ny, 1..nz (wall faces included, as the reference does).  The
// block's slices of the six metric tables of each axis (indices base-2 ..
// base+extent+2) are staged in shared memory first.
constexpr int kPredBX = 32, kPredBY = 4, kPredBZ = 2;

template <class T>
__global__ void __launch_bounds__(kPredBX * kPredBY * kPredBZ) k_predictor(Geom g, Tabs<T> tb, PredArgs a) {
    constexpr int LX = kPredBX + 5, LY = kPredBY + 5, LZ = kPredBZ + 5;
    __shared__ T stx[6 * LX], sty[6 * LY], stz[6 * LZ];
    const int tid = threadIdx.x + kPredBX * (threadIdx.y + kPredBY * threadIdx.z);
    const int ib = blockIdx.x * kPredBX - 1, jb = blockIdx.y * kPredBY - 1, kb = blockIdx.z * kPredBZ - 1;
    {
        auto tab = [](const AxisTabs<T>& A, int t) {
            return t == 0 ? A.riD : t == 1 ? A.rDs : t == 2 ? A.As : t == 3 ? A.Bs : t == 4 ? A.Ac : A.Bc;
        };
        for (int q = tid; q < 6 * (LX + LY + LZ); q += kPredBX * kPredBY * kPredBZ) {
            if (q < 6 * LX) {
                const int t = q / LX, o = q - t * LX;
                if (ib + o <= g.nx + 2) stx[q] = tab(tb.ax[0], t)[ib + o];
            } else if (q < 6 * (LX + LY)) {
                const int r = q - 6 * LX, t = r / LY, o = r - t * LY;
                if (jb + o <= g.ny + 2) sty[r] = tab(tb.ax[1], t)[jb + o];
            } else {
                const int r = q - 6 * (LX + LY), t = r / LZ, o = r - t * LZ;
                if (kb + o <= g.nz + 2) stz[r] = tab(tb.ax[2], t)[kb + o];
            }
        }
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const long long sx = 1, sy = g.px, sz = g.pz;
    const double* __restrict__ u = a.u;
    const double* __restrict__ v = a.v;
    const double* __restrict__ w = a.w;
#define LD(p, o) ((T)__ldg((p) + c + (o)))
    // the staged tables, indexed like the global ones (valid for the block's range)
    const AxisTabs<T> X{stx - ib, stx + LX - ib, stx + 2 * LX - ib, stx + 3 * LX - ib, stx + 4 * LX - ib,
                        stx + 5 * LX - ib};
    const AxisTabs<T> Y{sty - jb, sty + LY - jb, sty + 2 * LY - jb, sty + 3 * LY - jb, sty + 4 * LY - jb,
                        sty + 5 * LY - jb};
    const AxisTabs<T> Z{stz - kb, stz + LZ - kb, stz + 2 * LZ - kb, stz + 3 * LZ - kb, stz + 4 * LZ - kb,
                        stz + 5 * LZ - kb};
    const T dt = (T)a.dt;
    const T nue = (T)(a.les ? a.nu + __ldg(a.nut + c) * (double)a.les : a.nu);

    // ---------------- u* (discretisation_QUICK_centre.f90:11-112)
    {
        const T U0 = LD(u, 0), U1 = LD(u, sx), U2 = LD(u, 2 * sx), Um1 = LD(u, -sx), Um2 = LD(u, -2 * sx);
        const T Un1 = LD(u, sy), Un2 = LD(u, 2 * sy), Us1 = LD(u, -sy), Us2 = LD(u, -2 * sy);
        const T Uf1 = LD(u, sz), Uf2 = LD(u, 2 * sz), Ub1 = LD(u, -sz), Ub2 = LD(u, -2 * sz);
        const T ut1 = T(0.5) * (U1 + U0);
        const T ut2 = T(0.5) * (Um1 + U0);
        const T vt1 = T(0.5) * (LD(v, 0) + LD(v, sx));
        const T vt2 = T(0.5) * (LD(v, -sy) + LD(v, sx - sy));
        const T wt1 = T(0.5) * (LD(w, sx) + LD(w, 0));
        const T wt2 = T(0.5) * (LD(w, -sz) + LD(w, sx - sz));
        const T ue = quick_face(Um1, U0, U1, U2, ut1, X.As[i], X.Bs[i], X.riD[i], X.riD[i + 1], X.riD[i + 2]);
        const T uw = quick_face(Um2, Um1, U0, U1, ut2, X.As[i - 1], X.Bs[i - 1], X.riD[i - 1], X.riD[i], X.riD[i + 1]);
        const T un = quick_face(Us1, U0, Un1, Un2, vt1, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
        const T us = quick_face(Us2, Us1, U0, Un1, vt2, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j]);
        const T uf = quick_face(Ub1, U0, Uf1, Uf2, wt1, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
        const T ub = quick_face(Ub2, Ub1, U0, Uf1, wt2, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k]);
        const T r = U0 - dt * (ut1 * ue - ut2 * uw) * X.rDs[i]
                  - dt * (vt1 * un - vt2 * us) * Y.riD[j]
                  - dt * (wt1 * uf - wt2 * ub) * Z.riD[k]
                  + nue * dt * ((U1 - U0) * X.riD[i + 1] - (U0 - Um1) * X.riD[i]) * X.rDs[i]
                  + nue * dt * ((Un1 - U0) * Y.rDs[j] - (U0 - Us1) * Y.rDs[j - 1]) * Y.riD[j]
                  + nue * dt * ((Uf1 - U0) * Z.rDs[k] - (U0 - Ub1) * Z.rDs[k - 1]) * Z.riD[k];
        a.us[c] = a.fb ? (double)r + a.dt * __ldg(a.fb + c) : (double)r;
    }
    // ---------------- v* (discretisation_QUICK_centre.f90:127-226)
    {
        const T V0 = LD(v, 0), V1 = LD(v, sx), V2 = LD(v, 2 * sx), Vm1 = LD(v, -sx), Vm2 = LD(v, -2 * sx);
        const T Vn1 = LD(v, sy), Vn2 = LD(v, 2 * sy), Vs1 = LD(v, -sy), Vs2 = LD(v, -2 * sy);
        const T Vf1 = LD(v, sz), Vf2 = LD(v, 2 * sz), Vb1 = LD(v, -sz), Vb2 = LD(v, -2 * sz);
        const T ut1 = T(0.5) * (LD(u, 0) + LD(u, sy));
        const T ut2 = T(0.5) * (LD(u, -sx) + LD(u, sy - sx));
        const T vt1 = T(0.5) * (V0 + Vn1);
        const T vt2 = T(0.5) * (Vs1 + V0);
        const T wt1 = T(0.5) * (LD(w, 0) + LD(w, sy));
        const T wt2 = T(0.5) * (LD(w, -sz) + LD(w, sy - sz));
        const T ve = quick_face(Vm1, V0, V1, V2, ut1, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
        const T vw = quick_face(Vm2, Vm1, V0, V1, ut2, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i]);
        const T vn = quick_face(Vs1, V0, Vn1, Vn2, vt1, Y.As[j], Y.Bs[j], Y.riD[j], Y.riD[j + 1], Y.riD[j + 2]);
        const T vs = quick_face(Vs2, Vs1, V0, Vn1, vt2, Y.As[j - 1], Y.Bs[j - 1], Y.riD[j - 1], Y.riD[j], Y.riD[j + 1]);
        const T vf = quick_face(Vb1, V0, Vf1, Vf2, wt1, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
        const T vb = quick_face(Vb2, Vb1, V0, Vf1, wt2, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k]);
        const T r = V0 - dt * (ut1 * ve - ut2 * vw) * X.riD[i]
                  - dt * (vt1 * vn - vt2 * vs) * Y.rDs[j]
                  - dt * (wt1 * vf - wt2 * vb) * Z.riD[k]
                  + nue * dt * ((V1 - V0) * X.rDs[i] - (V0 - Vm1) * X.rDs[i - 1]) * X.riD[i]
                  + nue * dt * ((Vn1 - V0) * Y.riD[j + 1] - (V0 - Vs1) * Y.riD[j]) * Y.rDs[j]
                  + nue * dt * ((Vf1 - V0) * Z.rDs[k] - (V0 - Vb1) * Z.rDs[k - 1]) * Z.riD[k];
        a.vs[c] = a.fb ? (double)r + a.dt * __ldg(a.fb + a.fstride + c) : (double)r;
    }
    // ---------------- w* (discretisation_QUICK_centre.f90:240-339)
    {
        const T W0 = LD(w, 0), W1 = LD(w, sx), W2 = LD(w, 2 * sx), Wm1 = LD(w, -sx), Wm2 = LD(w, -2 * sx);
        const T Wn1 = LD(w, sy), Wn2 = LD(w, 2 * sy), Ws1 = LD(w, -sy), Ws2 = LD(w, -2 * sy);
        const T Wf1 = LD(w, sz), Wf2 = LD(w, 2 * sz), Wb1 = LD(w, -sz), Wb2 = LD(w, -2 * sz);
        const T ut1 = T(0.5) * (LD(u, sz) + LD(u, 0));
        const T ut2 = T(0.5) * (LD(u, sz - sx) + LD(u, -sx));
        const T vt1 = T(0.5) * (LD(v, 0) + LD(v, sz));
        const T vt2 = T(0.5) * (LD(v, sz - sy) + LD(v, -sy));
        const T wt1 = T(0.5) * (Wf1 + W0);
        const T wt2 = T(0.5) * (W0 + Wb1);
        const T we = quick_face(Wm1, W0, W1, W2, ut1, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
        const T ww = quick_face(Wm2, Wm1, W0, W1, ut2, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i]);
        const T wn = quick_face(Ws1, W0, Wn1, Wn2, vt1, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
        const T ws = quick_face(Ws2, Ws1, W0, Wn1, vt2, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j]);
        const T wf = quick_face(Wb1, W0, Wf1, Wf2, wt1, Z.As[k], Z.Bs[k], Z.riD[k], Z.riD[k + 1], Z.riD[k + 2]);
        const T wb = quick_face(Wb2, Wb1, W0, Wf1, wt2, Z.As[k - 1], Z.Bs[k - 1], Z.riD[k - 1], Z.riD[k], Z.riD[k + 1]);
        const T r = W0 - dt * (ut1 * we - ut2 * ww) * X.riD[i]
                  - dt * (vt1 * wn - vt2 * ws) * Y.riD[j]
                  - dt * (wt1 * wf - wt2 * wb) * Z.rDs[k]
                  + nue * dt * ((W1 - W0) * X.rDs[i] - (W0 - Wm1) * X.rDs[i - 1]) * X.riD[i]
                  + nue * dt * ((Wn1 - W0) * Y.rDs[j] - (W0 - Ws1) * Y.rDs[j - 1]) * Y.riD[j]
                  + nue * dt * ((Wf1 - W0) * Z.riD[k + 1] - (W0 - Wb1) * Z.riD[k]) * Z.rDs[k];
        a.ws[c] = a.fb ? (double)r + a.dt * __ldg(a.fb + 2 * a.fstride + c) : (double)r;
    }
#undef LD
}

// ---------------------------------------------------------------- K1 ----
// smagorinsky.f90:1-87.  REF_ALIASED reproduces the reference's storage
// association of the halo array u(-1:nx+2,...) with the dummy Phi(nx,ny,nz):
// Phi(i,j,k) is storage element (i-1)+(j-1)nx+(k-1)nx*ny counted from
// u(-1,-1,-1); elements before the array read as 0.
__device__ __forceinline__ double phi_read(const Geom& g, const double* f, int i, int j, int k,
                                           bool aliased) {
    if (!aliased) return __ldg(f + nat(g, i, j, k));
    const long long off = (long long)(i - 1) + (long long)(j - 1) * g.nx +
                          (long long)(k - 1) * g.nx * g.ny;
    const long long ax = g.nx + 4, ay = g.ny + 4;
    if (off < 0 || off >= ax * ay * (g.nz + 4)) return 0.0;
    const int a = (int)(off % ax);
    const long long t = off / ax;
    const int b = (int)(t % ay);
    const int cc = (int)(t / ay);
    // storage element `off` counted from u(-1,-1,-1): Fortran index = position - 1
    return __ldg(f + nat(g, a - 1, b - 1, cc - 1));
}

__device__ __forceinline__ void grad_gauss(const Geom& g, const double* f, bool al, int i, int j, int k,
                                           const double* Dxm, const double* Dym, const double* Dzm,
                                           double out[3]) {
    const double P0 = phi_read(g, f, i, j, k, al);
    const double fe = 0.5 * (phi_read(g, f, i + 1, j, k, al) + P0);
    const double fw = 0.5 * (phi_read(g, f, i - 1, j, k, al) + P0);
    const double fn = 0.5 * (phi_read(g, f, i, j + 1, k, al) + P0);
    const double fs = 0.5 * (phi_read(g, f, i, j - 1, k, al) + P0);
    const double ff = 0.5 * (phi_read(g, f, i, j, k + 1, al) + P0);
    const double fb = 0.5 * (phi_read(g, f, i, j, k - 1, al) + P0);
    const double d1 = fw * (-1) * (Dym[j] * Dzm[k]) + fe * (1) * (Dym[j] * Dzm[k]);
    const double d2 = fs * (-1) * (Dxm[i] * Dzm[k]) + fn * (1) * (Dxm[i] * Dzm[k]);
    const double d3 = fb * (-1) * (Dxm[i] * Dym[j]) + ff * (1) * (Dxm[i] * Dym[j]);
    const double fact = 1.0 / (Dxm[i] * Dym[j] * Dzm[k]);
    out[0] = fact * d1; out[1] = fact * d2; out[2] = fact * d3;
}

// The seven storage positions that phi_read reads for Phi(i,j,k) and its
// six neighbours under REF_ALIASED, as natural-layout indices (-1: outside
// the halo array, read as 0).  Storage element `off` sits at (a, b, c) =
// (off mod ax, (off / ax) mod ay, off / (ax ay)) of the (nx+4) x (ny+4) x
// (nz+4) array; the centre's position takes one division pair, and the
// neighbours at off +- 1, +- nx, +- nx*ny follow by adding the offset's own
// radix digits with one carry per digit (nx < ax and nx*ny < ax*ay).  The
// halo array holds fewer than 2^32 elements.
struct AliasPos {
    long long q[7];   // P0, E (+1), W (-1), N (+nx), S (-nx), F (+nx ny), B (-nx ny)
};
__device__ __forceinline__ AliasPos alias_positions(const Geom& g, int i, int j, int k) {
    const unsigned ax = g.nx + 4, ay = g.ny + 4, cz = g.nz + 4;
    const unsigned nxny = (unsigned)g.nx * g.ny;
    const unsigned fa = nxny % ax, fb = nxny / ax;   // nx*ny = fb*ax + fa, fb < ay
    const unsigned off = (unsigned)(i - 1) + (unsigned)(j - 1) * g.nx + (unsigned)(k - 1) * nxny;
    const int a0 = (int)(off % ax);
    const unsigned t = off / ax;
    const int b0 = (int)(t % ay), c0 = (int)(t / ay);
    auto at = [&](int a, int b, int c) -> long long {
        return (c < 0 || c >= (int)cz) ? -1 : nat(g, a - 1, b - 1, c - 1);
    };
    auto plus = [&](int da, int db) {
        int a = a0 + da, b = b0 + db, c = c0;
        if (a >= (int)ax) { a -= ax; ++b; }
        if (b >= (int)ay) { b -= ay; ++c; }
        return at(a, b, c);
    };
    auto minus = [&](int da, int db) {
        int a = a0 - da, b = b0 - db, c = c0;
        if (a < 0) { a += ax; --b; }
        if (b < 0) { b += ay; --c; }
        return at(a, b, c);
    };
    AliasPos p;
    p.q[0] = at(a0, b0, c0);
    p.q[1] = plus(1, 0);
    p.q[2] = minus(1, 0);
    p.q[3] = plus(g.nx, 0);
    p.q[4] = minus(g.nx, 0);
    p.q[5] = plus((int)fa, (int)fb);
    p.q[6] = minus((int)fa, (int)fb);
    return p;
}

// grad_gauss with the REF_ALIASED reads at precomputed positions (the same
// values phi_read returns, the same arithmetic).
__device__ __forceinline__ void grad_gauss_at(const Geom& g, const double* f, const AliasPos& P, int i, int j,
                                              int k, const double* Dxm, const double* Dym, const double* Dzm,
                                              double out[3]) {
    auto rd = [&](int n) { return P.q[n] < 0 ? 0.0 : __ldg(f + P.q[n]); };
    const double P0 = rd(0);
    const double fe = 0.5 * (rd(1) + P0);
    const double fw = 0.5 * (rd(2) + P0);
    const double fn = 0.5 * (rd(3) + P0);
    const double fs = 0.5 * (rd(4) + P0);
    const double ff = 0.5 * (rd(5) + P0);
    const double fb = 0.5 * (rd(6) + P0);
    const double d1 = fw * (-1) * (Dym[j] * Dzm[k]) + fe * (1) * (Dym[j] * Dzm[k]);
    const double d2 = fs * (-1) * (Dxm[i] * Dzm[k]) + fn * (1) * (Dxm[i] * Dzm[k]);
    const double d3 = fb * (-1) * (Dxm[i] * Dym[j]) + ff * (1) * (Dxm[i] * Dym[j]);
    const double fact = 1.0 / (Dxm[i] * Dym[j] * Dzm[k]);
    out[0] = fact * d1; out[1] = fact * d2; out[2] = fact * d3;
}

__global__ void __launch_bounds__(256) k_smagorinsky(Geom g, const double* u, const double* v,
                                                     const double* w, double* nut, double Cs,
                                                     int aliased) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    double du[3], dv[3], dw[3];
    if (aliased) {
        const AliasPos P = alias_positions(g, i, j, k);
        grad_gauss_at(g, u, P, i, j, k, g.Dxs, g.iDy, g.iDz, du);
        grad_gauss_at(g, v, P, i, j, k, g.iDx, g.Dys, g.iDz, dv);
        grad_gauss_at(g, w, P, i, j, k, g.iDx, g.iDy, g.Dzs, dw);
    } else {
        grad_gauss(g, u, false, i, j, k, g.Dxs, g.iDy, g.iDz, du);
        grad_gauss(g, v, false, i, j, k, g.iDx, g.Dys, g.iDz, dv);
        grad_gauss(g, w, false, i, j, k, g.iDx, g.iDy, g.Dzs, dw);
    }
    double m = fabs(2 * (du[0] * du[0]) + 2 * (dv[1] * dv[1]) + 2 * (dw[2] * dw[2]) +
                    (du[1] + dv[0]) * (du[1] + dv[0]) + (du[2] + dw[0]) * (du[2] + dw[0]) +
                    (dv[2] + dw[1]) * (dv[2] + dw[1]));
    // delta = (iDx iDy iDz)**(1./3.) with the default-real literal 1./3.
    const double delta = pow(g.iDx[i] * g.iDy[j] * g.iDz[k], (double)(1.f / 3.f));
    nut[nat(g, i, j, k)] = (Cs * delta) * (Cs * delta) * sqrt(m);
}

}  // namespace ntcfd
