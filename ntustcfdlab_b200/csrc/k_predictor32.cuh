// k_predictor32.cuh -- K2 of the mixed-precision path: the QUICK/central
// predictor of discretisation_QUICK_centre.f90:7-342 with FP32 arithmetic.
//
// The state stays FP64.  A block of 32 x 8 threads owns a 32 x 8 column of
// cells and marches along k through a chunk of planes, keeping u, v and w
// of the planes k-2..k+2 (with a two-cell ring in i and j) in shared memory
// as FP32: every FP64 value is loaded and converted once per block, and the
// loads of plane k+3 are in flight while plane k is computed.  The predictor
// is written in increment form: the FP32 part is the change
//     du = - dt * (convection) + nu_eff * dt * (diffusion)
// of discretisation_QUICK_centre.f90:104-109 (and 218-223, 331-336), and
// u* = u + du is formed in FP64 from the cell's own FP64 value, so the
// rounding error of the FP32 arithmetic scales with the step's change, not
// with the velocity.  The term-by-term algebra is that of k_predictor.
#pragma once

#include "k_predictor.cuh"

namespace ntcfd {

constexpr int kP32BX = 32, kP32BY = 8;                   // cells of a block's column
constexpr int kP32TX = kP32BX + 4, kP32TY = kP32BY + 4;  // one staged plane, two-cell ring
constexpr int kP32Plane = kP32TX * kP32TY;
constexpr int kP32Ring = 5;                              // planes k-2..k+2
constexpr int kP32NT = kP32BX * kP32BY;
constexpr int kP32Loads = (3 * kP32Plane + kP32NT - 1) / kP32NT;   // per thread per plane

// Planes per block: the k range in chunks of kc planes, the count of chunks
// chosen so that whole waves of blocks fill the SMs.  A block computes kc
// planes and stages 4 more in its prologue (counted as 2); with `resident`
// blocks at once on the device the launch takes ceil(blocks / resident)
// waves, and kc minimises waves x (kc + 2).  (A grid of 2.16 waves, as a
// fixed four blocks per SM gave at 128^3, spends a third wave on a sixth of
// the blocks.)
inline int p32_chunk(int nx, int ny, int nz, int resident) {
    const long long cols = (long long)((nx + kP32BX - 1) / kP32BX) * ((ny + kP32BY - 1) / kP32BY);
    const long long res = resident > 0 ? resident : 1;
    int best_kc = nz;
    long long best = -1;
    for (int kc = 1; kc <= nz; ++kc) {
        const long long chunks = (nz + kc - 1) / kc;
        if (kc > 1 && (nz + kc - 2) / (kc - 1) == chunks) continue;   // same chunks, fewer planes
        const long long waves = (cols * chunks + res - 1) / res;
        const long long cost = waves * (kc + 2);
        if (best < 0 || cost < best) {
            best = cost;
            best_kc = kc;
        }
    }
    return best_kc;
}

__global__ void __launch_bounds__(kP32NT, 2) k_predictor32(Geom g, Tabs<float> tb, PredArgs a, int kc) {
    // ring[slot][field][plane element]
    __shared__ float ring[kP32Ring * 3 * kP32Plane];
    constexpr int LX = kP32BX + 5, LY = kP32BY + 5;
    __shared__ float stx[6 * LX], sty[6 * LY];
    extern __shared__ float stz[];                        // 6 x (kc + 5) z-table entries
    const int LZ = kc + 5;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + kP32BX * ty;
    const int i0 = blockIdx.x * kP32BX + 1, j0 = blockIdx.y * kP32BY + 1;
    const int k0 = blockIdx.z * kc + 1, k1 = min(g.nz, k0 + kc - 1);
    const int ib = i0 - 2, jb = j0 - 2, kb = k0 - 2;
    {
        auto tab = [](const AxisTabs<float>& A, int t) {
            return t == 0 ? A.riD : t == 1 ? A.rDs : t == 2 ? A.As : t == 3 ? A.Bs : t == 4 ? A.Ac : A.Bc;
        };
        for (int q = tid; q < 6 * (LX + LY + LZ); q += kP32NT) {
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
    // element e of a staged plane: field e / Plane at (i0-2 + x, j0-2 + y), r = e % Plane =
    // y * TX + x; indices past the halo array's last one are clamped to it (never used)
    int goff[kP32Loads];
    const double* gsrc[kP32Loads];
#pragma unroll
    for (int q = 0; q < kP32Loads; ++q) {
        const int e = min(tid + q * kP32NT, 3 * kP32Plane - 1);
        const int f = e / kP32Plane, r = e - f * kP32Plane;
        const int ey = r / kP32TX, ex = r - ey * kP32TX;
        const int ii = min(ib + ex, g.nx + 2), jj = min(jb + ey, g.ny + 2);
        goff[q] = (int)(nat(g, ii, jj, -1) - nat(g, 0, 0, -1));   // offset within a plane
        gsrc[q] = f == 0 ? a.u : f == 1 ? a.v : a.w;
    }
    auto load_plane = [&](int k, double (&v)[kP32Loads]) {
        const long long pk = nat(g, 0, 0, k);
#pragma unroll
        for (int q = 0; q < kP32Loads; ++q) v[q] = __ldg(gsrc[q] + pk + goff[q]);
    };
    auto store_plane = [&](int slot, const double (&v)[kP32Loads]) {
#pragma unroll
        for (int q = 0; q < kP32Loads; ++q) {
            const int e = tid + q * kP32NT;
            if (e < 3 * kP32Plane) ring[slot * 3 * kP32Plane + e] = (float)v[q];
        }
    };
    // prologue: planes k0-2 .. k0+2 (the halo array holds k = -1 .. nz+2)
    {
        double v[kP32Loads];
        for (int k = k0 - 2; k <= k0 + 2; ++k) {
            load_plane(min(k, g.nz + 2), v);
            store_plane(k - kb, v);
        }
    }
    const int i = i0 + tx, j = j0 + ty;
    const bool inside = i <= g.nx && j <= g.ny;
    const AxisTabs<float> X{stx - ib, stx + LX - ib, stx + 2 * LX - ib, stx + 3 * LX - ib, stx + 4 * LX - ib,
                            stx + 5 * LX - ib};
    const AxisTabs<float> Y{sty - jb, sty + LY - jb, sty + 2 * LY - jb, sty + 3 * LY - jb, sty + 4 * LY - jb,
                            sty + 5 * LY - jb};
    const AxisTabs<float> Z{stz - kb, stz + LZ - kb, stz + 2 * LZ - kb, stz + 3 * LZ - kb, stz + 4 * LZ - kb,
                            stz + 5 * LZ - kb};
    const float dt = (float)a.dt;
    const int o0 = (ty + 2) * kP32TX + (tx + 2);          // the cell in a staged plane
    constexpr int SX = 1, SY = kP32TX, FV = kP32Plane, FW = 2 * kP32Plane;
    __syncthreads();
    for (int k = k0; k <= k1; ++k) {
        // the loads of plane k+3 are in flight while plane k is computed
        double nv[kP32Loads];
        load_plane(min(k + 3, g.nz + 2), nv);
        if (inside) {
            // element offsets of the cell in the planes k-2 .. k+2 (u; v at +FV, w at +FW)
            const int q = k - k0;
            const int s0 = ((q) % kP32Ring) * 3 * kP32Plane + o0;
            const int s1 = ((q + 1) % kP32Ring) * 3 * kP32Plane + o0;
            const int s2 = ((q + 2) % kP32Ring) * 3 * kP32Plane + o0;
            const int s3 = ((q + 3) % kP32Ring) * 3 * kP32Plane + o0;
            const int s4 = ((q + 4) % kP32Ring) * 3 * kP32Plane + o0;
            const float* R = ring;
            const long long c = nat(g, i, j, k);
            const float nue = (float)(a.les ? a.nu + __ldg(a.nut + c) * (double)a.les : a.nu);
            // ---------------- u* (discretisation_QUICK_centre.f90:11-112)
            {
                const float U0 = R[s2], U1 = R[s2 + SX], U2 = R[s2 + 2 * SX], Um1 = R[s2 - SX], Um2 = R[s2 - 2 * SX];
                const float Un1 = R[s2 + SY], Un2 = R[s2 + 2 * SY], Us1 = R[s2 - SY], Us2 = R[s2 - 2 * SY];
                const float Uf1 = R[s3], Uf2 = R[s4], Ub1 = R[s1], Ub2 = R[s0];
                const float ut1 = 0.5f * (U1 + U0);
                const float ut2 = 0.5f * (Um1 + U0);
                const float vt1 = 0.5f * (R[s2 + FV] + R[s2 + FV + SX]);
                const float vt2 = 0.5f * (R[s2 + FV - SY] + R[s2 + FV + SX - SY]);
                const float wt1 = 0.5f * (R[s2 + FW + SX] + R[s2 + FW]);
                const float wt2 = 0.5f * (R[s1 + FW] + R[s1 + FW + SX]);
                const float ue = quick_face(Um1, U0, U1, U2, ut1, X.As[i], X.Bs[i], X.riD[i], X.riD[i + 1], X.riD[i + 2]);
                const float uw = quick_face(Um2, Um1, U0, U1, ut2, X.As[i - 1], X.Bs[i - 1], X.riD[i - 1], X.riD[i], X.riD[i + 1]);
                const float un = quick_face(Us1, U0, Un1, Un2, vt1, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
                const float us = quick_face(Us2, Us1, U0, Un1, vt2, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j]);
                const float uf = quick_face(Ub1, U0, Uf1, Uf2, wt1, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
                const float ub = quick_face(Ub2, Ub1, U0, Uf1, wt2, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k]);
                const float du = -dt * (ut1 * ue - ut2 * uw) * X.rDs[i]
                               - dt * (vt1 * un - vt2 * us) * Y.riD[j]
                               - dt * (wt1 * uf - wt2 * ub) * Z.riD[k]
                               + nue * dt * ((U1 - U0) * X.riD[i + 1] - (U0 - Um1) * X.riD[i]) * X.rDs[i]
                               + nue * dt * ((Un1 - U0) * Y.rDs[j] - (U0 - Us1) * Y.rDs[j - 1]) * Y.riD[j]
                               + nue * dt * ((Uf1 - U0) * Z.rDs[k] - (U0 - Ub1) * Z.rDs[k - 1]) * Z.riD[k];
                const double r = __ldg(a.u + c) + (double)du;
                a.us[c] = a.fb ? r + a.dt * __ldg(a.fb + c) : r;
            }
            // ---------------- v* (discretisation_QUICK_centre.f90:127-226)
            {
                const int t2 = s2 + FV;
                const float V0 = R[t2], V1 = R[t2 + SX], V2 = R[t2 + 2 * SX], Vm1 = R[t2 - SX], Vm2 = R[t2 - 2 * SX];
                const float Vn1 = R[t2 + SY], Vn2 = R[t2 + 2 * SY], Vs1 = R[t2 - SY], Vs2 = R[t2 - 2 * SY];
                const float Vf1 = R[s3 + FV], Vf2 = R[s4 + FV], Vb1 = R[s1 + FV], Vb2 = R[s0 + FV];
                const float ut1 = 0.5f * (R[s2] + R[s2 + SY]);
                const float ut2 = 0.5f * (R[s2 - SX] + R[s2 + SY - SX]);
                const float vt1 = 0.5f * (V0 + Vn1);
                const float vt2 = 0.5f * (Vs1 + V0);
                const float wt1 = 0.5f * (R[s2 + FW] + R[s2 + FW + SY]);
                const float wt2 = 0.5f * (R[s1 + FW] + R[s1 + FW + SY]);
                const float ve = quick_face(Vm1, V0, V1, V2, ut1, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
                const float vw = quick_face(Vm2, Vm1, V0, V1, ut2, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i]);
                const float vn = quick_face(Vs1, V0, Vn1, Vn2, vt1, Y.As[j], Y.Bs[j], Y.riD[j], Y.riD[j + 1], Y.riD[j + 2]);
                const float vs = quick_face(Vs2, Vs1, V0, Vn1, vt2, Y.As[j - 1], Y.Bs[j - 1], Y.riD[j - 1], Y.riD[j], Y.riD[j + 1]);
                const float vf = quick_face(Vb1, V0, Vf1, Vf2, wt1, Z.Ac[k], Z.Bc[k], Z.rDs[k - 1], Z.rDs[k], Z.rDs[k + 1]);
                const float vb = quick_face(Vb2, Vb1, V0, Vf1, wt2, Z.Ac[k - 1], Z.Bc[k - 1], Z.rDs[k - 2], Z.rDs[k - 1], Z.rDs[k]);
                const float dv = -dt * (ut1 * ve - ut2 * vw) * X.riD[i]
                               - dt * (vt1 * vn - vt2 * vs) * Y.rDs[j]
                               - dt * (wt1 * vf - wt2 * vb) * Z.riD[k]
                               + nue * dt * ((V1 - V0) * X.rDs[i] - (V0 - Vm1) * X.rDs[i - 1]) * X.riD[i]
                               + nue * dt * ((Vn1 - V0) * Y.riD[j + 1] - (V0 - Vs1) * Y.riD[j]) * Y.rDs[j]
                               + nue * dt * ((Vf1 - V0) * Z.rDs[k] - (V0 - Vb1) * Z.rDs[k - 1]) * Z.riD[k];
                const double r = __ldg(a.v + c) + (double)dv;
                a.vs[c] = a.fb ? r + a.dt * __ldg(a.fb + a.fstride + c) : r;
            }
            // ---------------- w* (discretisation_QUICK_centre.f90:240-339)
            {
                const int t2 = s2 + FW;
                const float W0 = R[t2], W1 = R[t2 + SX], W2 = R[t2 + 2 * SX], Wm1 = R[t2 - SX], Wm2 = R[t2 - 2 * SX];
                const float Wn1 = R[t2 + SY], Wn2 = R[t2 + 2 * SY], Ws1 = R[t2 - SY], Ws2 = R[t2 - 2 * SY];
                const float Wf1 = R[s3 + FW], Wf2 = R[s4 + FW], Wb1 = R[s1 + FW], Wb2 = R[s0 + FW];
                const float ut1 = 0.5f * (R[s3] + R[s2]);
                const float ut2 = 0.5f * (R[s3 - SX] + R[s2 - SX]);
                const float vt1 = 0.5f * (R[s2 + FV] + R[s3 + FV]);
                const float vt2 = 0.5f * (R[s3 + FV - SY] + R[s2 + FV - SY]);
                const float wt1 = 0.5f * (Wf1 + W0);
                const float wt2 = 0.5f * (W0 + Wb1);
                const float we = quick_face(Wm1, W0, W1, W2, ut1, X.Ac[i], X.Bc[i], X.rDs[i - 1], X.rDs[i], X.rDs[i + 1]);
                const float ww = quick_face(Wm2, Wm1, W0, W1, ut2, X.Ac[i - 1], X.Bc[i - 1], X.rDs[i - 2], X.rDs[i - 1], X.rDs[i]);
                const float wn = quick_face(Ws1, W0, Wn1, Wn2, vt1, Y.Ac[j], Y.Bc[j], Y.rDs[j - 1], Y.rDs[j], Y.rDs[j + 1]);
                const float ws = quick_face(Ws2, Ws1, W0, Wn1, vt2, Y.Ac[j - 1], Y.Bc[j - 1], Y.rDs[j - 2], Y.rDs[j - 1], Y.rDs[j]);
                const float wf = quick_face(Wb1, W0, Wf1, Wf2, wt1, Z.As[k], Z.Bs[k], Z.riD[k], Z.riD[k + 1], Z.riD[k + 2]);
                const float wb = quick_face(Wb2, Wb1, W0, Wf1, wt2, Z.As[k - 1], Z.Bs[k - 1], Z.riD[k - 1], Z.riD[k], Z.riD[k + 1]);
                const float dw = -dt * (ut1 * we - ut2 * ww) * X.riD[i]
                               - dt * (vt1 * wn - vt2 * ws) * Y.riD[j]
                               - dt * (wt1 * wf - wt2 * wb) * Z.rDs[k]
                               + nue * dt * ((W1 - W0) * X.rDs[i] - (W0 - Wm1) * X.rDs[i - 1]) * X.riD[i]
                               + nue * dt * ((Wn1 - W0) * Y.rDs[j] - (W0 - Ws1) * Y.rDs[j - 1]) * Y.riD[j]
                               + nue * dt * ((Wf1 - W0) * Z.riD[k + 1] - (W0 - Wb1) * Z.riD[k]) * Z.rDs[k];
                const double r = __ldg(a.w + c) + (double)dw;
                a.ws[c] = a.fb ? r + a.dt * __ldg(a.fb + 2 * a.fstride + c) : r;
            }
        }
        __syncthreads();                         // plane k-2 is no longer read: k+3 takes its slot
        store_plane((k + 3 - kb) % kP32Ring, nv);
        __syncthreads();
    }
}

}  // namespace ntcfd
