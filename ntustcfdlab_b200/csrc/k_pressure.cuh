// k_pressure.cuh -- K3 pressure Poisson solve (GS.f90:1-106) as red-black
// SOR on the correction e of a defect-correction loop.
//
// The reference sweep (GS.f90:39-53) is, after dividing numerator and
// denominator by the cell volume V = iDx iDy iDz,
//     pNew = rdiag * sum_nb c_nb p_nb - b',
//     rdiag = 1 / sum_nb c_nb,  b' = rdiag * mChange / (dt V),
// with c_E = 1/(iDx(i) Dxs(i)), c_W = 1/(iDx(i) Dxs(i-1)), etc.  The ghost
// values of p stay frozen during the solve (the reference refreshes them
// only in boundary_conditions).  For p = p0 + e the same sweep reads
//     eNew = rdiag * sum_nb c_nb e_nb + d,  d = rdiag * sum c p0_nb - b' - p0,
// with e = 0 on every ghost, and eNew - e equals pNew - p: the stop rule
// max|pNew - p| <= zeta (GS.f90:11,53) is evaluated unchanged.  The FP64
// path runs the sweeps with double e and d; the mixed path runs them in
// float and recovers p in double.
#pragma once

#include <type_traits>

#include "ntcfd_common.cuh"

namespace ntcfd {

template <class Tc>
struct SorCoef {
    const Tc *cE, *cW, *cN, *cS, *cF, *cB;
};

__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }

// 1 / sum of the six coefficients (correctly rounded reciprocal)
template <class Tc>
__device__ __forceinline__ Tc rdiag_of(const SorCoef<Tc>& s, int i, int j, int k) {
    return rcp_rn(((s.cE[i] + s.cW[i]) + (s.cN[j] + s.cS[j])) + (s.cF[k] + s.cB[k]));
}

// Explicitly rounded operations: every kernel that evaluates a sweep or a
// defect uses these, so the resident and streaming paths round alike
// whatever the compiler would contract.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// One SOR update of a cell of the correction e (GS.f90:43-53 in the form
// eNew = rdiag * sum_nb c_nb e_nb + d): returns eNew - e0 and the relaxed
// value e0 + omega (eNew - e0) in *e1.
template <class Tc>
__device__ __forceinline__ Tc sor_update(Tc cE, Tc oE, Tc cW, Tc oW, Tc cN, Tc oN, Tc cS, Tc oS, Tc cF,
                                         Tc oF, Tc cB, Tc oB, Tc rd, Tc d, Tc e0, Tc om, Tc* e1) {
    Tc s = mul_rn(cE, oE);
    s = fma_rn(cW, oW, s);
    s = fma_rn(cN, oN, s);
    s = fma_rn(cS, oS, s);
    s = fma_rn(cF, oF, s);
    s = fma_rn(cB, oB, s);
    const Tc diff = sub_rn(fma_rn(rd, s, d), e0);
    *e1 = fma_rn(om, diff, e0);
    return diff;
}

// FP64 defect of a cell, d = rdiag * sum_nb c_nb p_nb - b' - p (the reference
// sweep's fixed-point residual), rd = rdiag_of of the cell: the same sums as
// sor_update.
__device__ __forceinline__ double defect_value(double cE, double pe, double cW, double pw, double cN, double pn,
                                               double cS, double ps, double cF, double pf, double cB, double pb,
                                               double rd, double bv, double pc) {
    double s = mul_rn(cE, pe);
    s = fma_rn(cW, pw, s);
    s = fma_rn(cN, pn, s);
    s = fma_rn(cS, ps, s);
    s = fma_rn(cF, pf, s);
    s = fma_rn(cB, pb, s);
    return sub_rn(fma_rn(rd, s, -bv), pc);
}

// FP64 reciprocal of a coefficient sum (positive and finite): the hardware's
// approximate double reciprocal refined by two Newton-Raphson steps
// x' = x + x (1 - s x), each of which squares the relative error.
__device__ __forceinline__ double rdiag64(double s) {
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(s));
    double r = fma_rn(-s, x, 1.0);
    x = fma_rn(x, r, x);
    r = fma_rn(-s, x, 1.0);
    x = fma_rn(x, r, x);
    return x;
}

// The FP64 defect of p + e from the defect d of p and the correction e of a
// defect-correction cycle: since the operator is linear,
//     d' = rdiag sum c (p+e)_nb - b' - (p+e) = d + rdiag sum_nb c_nb e_nb - e,
// formed in FP64 with the FP64 coefficients from the cycle's (exact) Tc
// values of e; rdiag is rdiag64 of the FP64 coefficient sum.  Both SOR paths
// restart a cycle with it.
template <class Tc>
__device__ __forceinline__ double defect_update(double cE, Tc eE, double cW, Tc eW, double cN, Tc eN, double cS,
                                                Tc eS, double cF, Tc eF, double cB, Tc eB, Tc d, Tc e) {
    double s = mul_rn(cE, (double)eE);
    s = fma_rn(cW, (double)eW, s);
    s = fma_rn(cN, (double)eN, s);
    s = fma_rn(cS, (double)eS, s);
    s = fma_rn(cF, (double)eF, s);
    s = fma_rn(cB, (double)eB, s);
    const double x = rdiag64(((cE + cW) + (cN + cS)) + (cF + cB));
    return sub_rn(fma_rn(x, s, (double)d), (double)e);
}

// Column-walking kernel (k_rhs): a 32 x 8 block covers (i, j) and
// walks the planes of its chunk k0..k1 (chunk = blockIdx.z, chunks of
// ceil(nz / gridDim.z) planes), carrying the k-1 value in a register, so a
// cell costs one new load per field along k and the x/y neighbours hit L1.
constexpr int kWalkBX = 32, kWalkBY = 8, kWalkUnroll = 4;

__device__ __forceinline__ void walk_range(const Geom& g, int& k0, int& k1) {
    const int kc = (g.nz + (int)gridDim.z - 1) / (int)gridDim.z;
    k0 = (int)blockIdx.z * kc + 1;
    k1 = min(g.nz, k0 + kc - 1);
}

// K3a -- b' on the interior from the predicted velocity (GS.f90:39-41).
// u*(0,j,k), v*(i,0,k), w*(i,j,0) equal the state's ghosts (the reference
// copies u into u_star over the whole halo array in boundary_conditions.f90:317-319),
// except w*(i,j,0) of a z-slab whose Back face is shared (back_iface): that plane
// is the lower neighbour's last plane of w* (main.f90:220-226).
__global__ void __launch_bounds__(kWalkBX * kWalkBY) k_rhs(Geom g, SorCoef<double> sc, const double* u,
                                                          const double* v, const double* w, const double* us,
                                                          const double* vs, const double* ws, double* b,
                                                          double dt, int back_iface) {
    const int i = blockIdx.x * kWalkBX + threadIdx.x + 1;
    const int j = blockIdx.y * kWalkBY + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    int k0, k1;
    walk_range(g, k0, k1);
    if (k0 > k1) return;
    // rdiag_of's sum, in its order, with the i and j parts hoisted
    const double sew = sc.cE[i] + sc.cW[i], sns = sc.cN[j] + sc.cS[j];
    const double rx = g.riDx[i], ry = g.riDy[j];
    const long long cb = nat(g, i, j, k0);
    double wb = (k0 == 1 && !back_iface) ? w[cb - g.pz] : ws[cb - g.pz];
#pragma unroll kWalkUnroll
    for (int k = k0; k <= k1; ++k) {
        const long long c = cb + (long long)(k - k0) * g.pz;
        const double uw = (i == 1) ? u[c - 1] : us[c - 1];
        const double vs_ = (j == 1) ? v[c - g.px] : vs[c - g.px];
        const double wc = ws[c];
        const double divv = (us[c] - uw) * rx + (vs[c] - vs_) * ry + (wc - wb) * g.riDz[k];
        b[c] = rcp_rn((sew + sns) + (sc.cF[k] + sc.cB[k])) * divv / dt;
        wb = wc;
    }
}

// Defect d = rdiag*sum c p0_nb - b' - p0 in double, stored per colour in
// Tc; e reset to 0.  With incr = 1, from the solve's second correction cycle
// on (ctl->cycles > 0), d is instead updated from the last cycle's correction
// (defect_update) and e is left for k_clear_e.  Inside the step graph
// (in_graph = 1) it also arms the inner loop's condition.
// For the resident path (ring != null) it also clears the ring of sweep
// maxima and the grid barrier the next kernel uses, and with begin = 1 it
// starts the solve (the counters k_sor_begin resets).
template <class Tc>
__global__ void __launch_bounds__(256) k_defect(Geom g, SorCoef<double> sc, const double* p,
                                                const double* b, Tc* dR, Tc* dB, Tc* eR, Tc* eB,
                                                const Tc* rdR, const Tc* rdB, Ctl* ctl,
                                                cudaGraphConditionalHandle inner, int in_graph,
                                                unsigned long long* ring, unsigned int* bar, int begin, int incr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0 && threadIdx.z == 0) {
        if (begin) {
            ctl->ik = 0;
            ctl->cycles = 0;
            ctl->restarts = 0;
            ctl->bodies = 0;
            ctl->timeout = 0;
            ctl->converged = 0;
            ctl->nonfinite = 0;
            ctl->last_change = 0.0;
        }
        ctl->inner = 0;
        if (in_graph) cudaGraphSetConditional(inner, 1u);
        if (ring) { ring[0] = 0ULL; ring[1] = 0ULL; ring[2] = 0ULL; }
        if (bar) { bar[0] = 0u; bar[1] = 0u; bar[2] = 0u; }   // GridBar word and err
    }
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long q = spl(g, (i + 2) >> 1, j, k);
    const bool red = ((i + j + k) & 1) == 0;
    if (incr && ctl->cycles > 0) {
        // the neighbours (other colour) at m(i-1) = (i+1)>>1, m(i+1) = (i+3)>>1, rows +-1
        const Tc* O = red ? eB : eR;
        const long long r0 = q - ((i + 2) >> 1);
        const Tc dv = (red ? dR : dB)[q];
        const double dn = defect_update(sc.cE[i], O[r0 + ((i + 3) >> 1)], sc.cW[i], O[r0 + ((i + 1) >> 1)], sc.cN[j],
                                        O[q + g.mxp], sc.cS[j], O[q - g.mxp], sc.cF[k], O[q + g.mz], sc.cB[k],
                                        O[q - g.mz], dv, (red ? eR : eB)[q]);
        (red ? dR : dB)[q] = (Tc)dn;
        return;
    }
    const long long c = nat(g, i, j, k);
    const double d = defect_value(sc.cE[i], p[c + 1], sc.cW[i], p[c - 1], sc.cN[j], p[c + g.px], sc.cS[j],
                                  p[c - g.px], sc.cF[k], p[c + g.pz], sc.cB[k], p[c - g.pz], rdiag_of(sc, i, j, k),
                                  b[c], p[c]);
    if (red) { dR[q] = (Tc)d; eR[q] = Tc(0); }
    else { dB[q] = (Tc)d; eB[q] = Tc(0); }
}

// e = 0 on the interior cells of both colours (after an incremental defect).
template <class Tc>
__global__ void __launch_bounds__(256) k_clear_e(Geom g, Tc* eR, Tc* eB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long q = spl(g, (i + 2) >> 1, j, k);
    if (((i + j + k) & 1) == 0) eR[q] = Tc(0);
    else eB[q] = Tc(0);
}

// rd = 1 / sum of the six coefficients of every interior cell, per colour,
// in the sweeps' precision; it depends on the grid only and is made once.
template <class Tc>
__global__ void k_make_rd(Geom g, SorCoef<Tc> sc, Tc* rdR, Tc* rdB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long q = spl(g, (i + 2) >> 1, j, k);
    const Tc rd = rdiag_of(sc, i, j, k);
    if (((i + j + k) & 1) == 0) rdR[q] = rd;
    else rdB[q] = rd;
}

// One half-sweep over colour `colour` (0 = red, (i+j+k) even), column form
// (used for FP64 e).  Thread t of
// row (j,k) owns the cell i = 2t + 2 - r, m = t + 2 - r, r = ((j+k)^colour)&1,
// for KPT consecutive planes k; all loads of the KPT cells are issued before
// any arithmetic so that a warp keeps 9*KPT loads in flight.  Offsets are
// 32-bit (a grid holds fewer than 2^31 cells per colour array).  With
// guard = 1 (several sweeps per loop body, or loop bodies queued ahead of the
// host's decision) the sweep is skipped once the sweep budget (itmax, cycle
// length) is used up or the solve has stopped.  The block's max |change|
// goes to slot sub*kSpread + (block index mod kSpread).  It reads e as it is
// (a cycle starts with k_clear_e); the first_mode argument of the row form is
// not taken.
template <class Tc, int NT, int KPT>
__global__ void __launch_bounds__(NT) k_sweep_cols(Geom g, SorCoef<Tc> sc, Tc* __restrict__ eOwn,
                                              const Tc* __restrict__ eOth, const Tc* __restrict__ dOwn,
                                              const Tc* __restrict__ rdOwn, int colour, double omega,
                                              const Ctl* ctl, int sub, int itmax, int cycle_len,
                                              int guard, unsigned long long* slots, int /*first_mode*/) {
    if (guard) {
        const int ik = ctl->ik, inner = ctl->inner;
        if (ik + sub >= itmax || inner + sub >= cycle_len || ctl->converged || ctl->nonfinite) return;
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * KPT + 1;
    const Tc om = (Tc)omega;
    using B = decltype(abs_bits(Tc(0)));
    const bool jok = j <= g.ny;
    const int jj = jok ? j : g.ny;
    const int ys = g.mxp, zs = (int)g.mz;
    const int rowj = ys * (jj + 1);
    int q[KPT];
    bool ok[KPT];
    Tc nE[KPT], nW[KPT], nN[KPT], nS[KPT], nF[KPT], nB[KPT], dd[KPT], e0[KPT], rd[KPT];
#pragma unroll
    for (int kk = 0; kk < KPT; ++kk) {
        const int k = min(k0 + kk, g.nz);
        const int r = ((jj + k) ^ colour) & 1;
        const int i = 2 * t + 2 - r;
        ok[kk] = jok && (k0 + kk <= g.nz) && i <= g.nx;
        // an inactive lane reads a valid interior cell and discards it
        const int rr = ok[kk] ? r : 1;
        const int qq = (ok[kk] ? t + 2 - r : 1) + rowj + zs * (k + 1);
        q[kk] = qq;
        nE[kk] = eOth[qq + rr];
        nW[kk] = eOth[qq - 1 + rr];
        nN[kk] = eOth[qq + ys];
        nS[kk] = eOth[qq - ys];
        nF[kk] = eOth[qq + zs];
        nB[kk] = eOth[qq - zs];
        dd[kk] = dOwn[qq];
        e0[kk] = eOwn[qq];
        rd[kk] = rdOwn[qq];
    }
    const Tc cN = sc.cN[jj], cS = sc.cS[jj];
    B ch = B(0);   // max |change| as an order-preserving pattern (NaN stays on top)
#pragma unroll
    for (int kk = 0; kk < KPT; ++kk) {
        if (!ok[kk]) continue;
        const int k = k0 + kk;
        const int i = 2 * t + 2 - (((j + k) ^ colour) & 1);
        Tc e1;
        const Tc diff = sor_update(sc.cE[i], nE[kk], sc.cW[i], nW[kk], cN, nN[kk], cS, nS[kk], sc.cF[k], nF[kk],
                                   sc.cB[k], nB[kk], rd[kk], dd[kk], e0[kk], om, &e1);
        eOwn[q[kk]] = e1;
        const B db = abs_bits(diff);
        ch = db > ch ? db : ch;
    }
    const int blin = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_max_bits<NT>(ch, &slots[sub * kSpread + (blin & (kSpread - 1))]);
}

// One half-sweep over colour `colour` (0 = red, (i+j+k) even), row form (used
// for FP32 e).  A warp takes a row (j,k) at a time, striding over the rows
// (rows j-fastest, so that neighbouring warps share their j+-1 neighbour
// rows; the stride is split into its j and k parts once, so the next row
// needs no division).  The colour's cells of a row are contiguous in the
// colour-split arrays (m = t + 2 - r, r = ((j+k)^colour)&1, i = 2t + 2 - r),
// and lane t updates the cells t and t + 32 of each 64-cell chunk with every
// load issued before its stores.  The row parity r is a template argument of
// the chunk update, so each array is read through one lane address per row
// with immediate offsets (east/west neighbour, second cell); rows of at most
// 64 cells per colour keep their lanes' cE, cW of both parities in
// registers.  A lane past the row's last cell reads inside the padded arrays
// (a split row holds at least 2 + (nx+1)/2 entries, the tables nx + 5, and
// the ghost rows and planes follow the interior ones), stores nothing and
// leaves the change maximum alone.  With guard = 1 (several sweeps per loop
// body, or loop bodies queued ahead of the host's decision) the sweep is
// skipped once the sweep budget (itmax, cycle length) is used up or the solve
// has stopped.  The block's max |change| goes to slot
// sub*kSpread + (block index mod kSpread).  In a cycle's first sweep
// (first_mode) e is zero everywhere before it, so the red half reads no e at
// all and the black half none of its own.  rdOwn is not read: the diagonal
// is formed from the 1-D tables, the same bits as the rd arrays.
template <class Tc, int NT>
__global__ void __launch_bounds__(NT, 4) k_sweep_rows(Geom g, SorCoef<Tc> sc, Tc* __restrict__ eOwn,
                                              const Tc* __restrict__ eOth, const Tc* __restrict__ dOwn,
                                              const Tc* __restrict__ /*rdOwn*/, int colour, double omega,
                                              const Ctl* ctl, int sub, int itmax, int cycle_len,
                                              int guard, unsigned long long* slots, int first_mode) {
    if (guard) {
        const int ik = ctl->ik, inner = ctl->inner;
        if (ik + sub >= itmax || inner + sub >= cycle_len || ctl->converged || ctl->nonfinite) return;
    }
    const bool first = first_mode && ctl->inner + sub == 0;
    using B = decltype(abs_bits(Tc(0)));
    const int lane = threadIdx.x & 31;
    const int ny = g.ny, nrow = g.ny * g.nz;
    const int nwarp = (int)gridDim.x * (NT / 32);
    const int w0 = blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
    const int nx = g.nx;
    const int half = (nx + 1) / 2;
    const int nown0 = nx / 2, nown1 = (nx + 1) / 2;
    const long long ys = g.mxp, zs = g.mz;
    const Tc om = (Tc)omega;
    B ch = B(0);   // max |change| as an order-preserving pattern (NaN stays on top)
    // the lane's coefficients in a one-chunk row: cells t = lane + 32h of parity r at
    // i = 2t + 2 - r (past the row's end: other table entries, never used)
    Tc cEr[2][2], cWr[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = min(2 * (lane + 32 * h) + 2 - r, nx + 2);
            cEr[r][h] = sc.cE[i];
            cWr[r][h] = sc.cW[i];
        }

    // cells t0 + lane and t0 + lane + 32 of a row of parity R; MD 0: a plain sweep,
    // 1: own e zero before it, 2: e zero everywhere before it
    auto chunk = [&](auto rr, auto md, const Tc* __restrict__ oC, Tc* __restrict__ eC,
                     const Tc* __restrict__ dC, int t0, int nown, Tc eA, Tc wA, Tc eB, Tc wB, Tc cN, Tc cS,
                     Tc cF, Tc cB, Tc sNS, Tc sFB) {
        constexpr int R = decltype(rr)::value;
        constexpr int MD = decltype(md)::value;
        const int tA = t0 + lane;
        const int m = tA + 2 - R;
        const Tc* __restrict__ o = oC + m;
        Tc nEA = Tc(0), nWA = Tc(0), nNA = Tc(0), nSA = Tc(0), nFA = Tc(0), nBA = Tc(0);
        Tc nEB = Tc(0), nWB = Tc(0), nNB = Tc(0), nSB = Tc(0), nFB = Tc(0), nBB = Tc(0);
        if (MD != 2) {
            const Tc* __restrict__ oN = o + ys;
            const Tc* __restrict__ oS = o - ys;
            const Tc* __restrict__ oF = o + zs;
            const Tc* __restrict__ oB = o - zs;
            nEA = o[R]; nWA = o[R - 1]; nEB = o[32 + R]; nWB = o[31 + R];
            nNA = oN[0]; nNB = oN[32]; nSA = oS[0]; nSB = oS[32];
            nFA = oF[0]; nFB = oF[32]; nBA = oB[0]; nBB = oB[32];
        }
        const Tc* __restrict__ dd = dC + m;
        Tc* __restrict__ ee = eC + m;
        const Tc dA = dd[0], dB = dd[32];
        const Tc e0A = MD ? Tc(0) : ee[0], e0B = MD ? Tc(0) : ee[32];
        const Tc rdA = rcp_rn(((eA + wA) + sNS) + sFB);
        const Tc rdB = rcp_rn(((eB + wB) + sNS) + sFB);
        Tc e1A, e1B;
        const Tc diffA = sor_update(eA, nEA, wA, nWA, cN, nNA, cS, nSA, cF, nFA, cB, nBA, rdA, dA, e0A, om, &e1A);
        const Tc diffB = sor_update(eB, nEB, wB, nWB, cN, nNB, cS, nSB, cF, nFB, cB, nBB, rdB, dB, e0B, om, &e1B);
        if (tA < nown) {
            ee[0] = e1A;
            const B db = abs_bits(diffA);
            ch = db > ch ? db : ch;
        }
        if (tA + 32 < nown) {
            ee[32] = e1B;
            const B db = abs_bits(diffB);
            ch = db > ch ? db : ch;
        }
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    auto rows = [&](auto md) {
        if (w0 >= nrow) return;
        int j = w0 % ny + 1, k = w0 / ny + 1;
        const int dj = nwarp % ny, dk = nwarp / ny;
        for (int row = w0; row < nrow; row += nwarp) {
            const int r = ((j + k) ^ colour) & 1;
            const long long rb = ys * (j + 1) + zs * (k + 1);   // colour-split row, m = 0
            const Tc* __restrict__ oC = eOth + rb;
            Tc* __restrict__ eC = eOwn + rb;
            const Tc* __restrict__ dC = dOwn + rb;
            const Tc cN = sc.cN[j], cS = sc.cS[j], cF = sc.cF[k], cB = sc.cB[k];
            const Tc sNS = cN + cS, sFB = cF + cB;
            if (half <= 64) {
                if (r == 0) chunk(I0{}, md, oC, eC, dC, 0, nown0, cEr[0][0], cWr[0][0], cEr[0][1], cWr[0][1], cN, cS,
                                  cF, cB, sNS, sFB);
                else chunk(I1{}, md, oC, eC, dC, 0, nown1, cEr[1][0], cWr[1][0], cEr[1][1], cWr[1][1], cN, cS, cF,
                           cB, sNS, sFB);
            } else {
                const int nown = r ? nown1 : nown0;
                for (int t0 = 0; t0 < nown; t0 += 64) {
                    const int iA = min(2 * (t0 + lane) + 2 - r, nx + 2), iB = min(iA + 64, nx + 2);
                    const Tc eA = sc.cE[iA], wA = sc.cW[iA], eB = sc.cE[iB], wB = sc.cW[iB];
                    if (r == 0) chunk(I0{}, md, oC, eC, dC, t0, nown, eA, wA, eB, wB, cN, cS, cF, cB, sNS, sFB);
                    else chunk(I1{}, md, oC, eC, dC, t0, nown, eA, wA, eB, wB, cN, cS, cF, cB, sNS, sFB);
                }
            }
            j += dj;
            k += dk;
            if (j > ny) {
                j -= ny;
                ++k;
            }
        }
    };
    if (!first) rows(std::integral_constant<int, 0>{});
    else if (colour != 0) rows(std::integral_constant<int, 1>{});
    else rows(std::integral_constant<int, 2>{});
    block_max_bits<NT>(ch, &slots[sub * kSpread + (blockIdx.x & (kSpread - 1))]);
}

// Launch shape of the row kernels (k_sweep_rows, k_defect_rows): NT threads,
// warps striding over the rows, at most `resident` blocks (the count the SMs
// hold at once), so that every block runs from the start and a block's max
// reduction and start-up are paid once for many rows.
inline dim3 sweep_grid(const Geom& g, int nt, int resident) {
    const long long rows = (long long)g.ny * g.nz;
    const long long need = (rows + nt / 32 - 1) / (nt / 32);
    const long long cap = resident > 0 ? resident : 1;
    return dim3((unsigned)(need < cap ? need : cap));
}

// The restart of a correction cycle of the streaming path in row form (the
// layout of k_sweep_rows): a warp per row (j,k), both colours, rows stepped as
// in k_sweep_rows.  The first cycle of a solve (ctl->cycles == 0) takes d from
// p: defect_value, the FP64 defect of p, a cell per lane and step.  Later
// cycles update it from the last cycle's e (defect_update, the same values
// k_defect forms) and add that e to p in the same pass (p += e of a cycle:
// the sweeps never read p, and the last cycle's e goes to p in k_correct_last
// after the cycle loop); there lane t takes the cells t and t + 32 of each
// 64-cell chunk of a colour, the row parity a template argument as in
// k_sweep_rows, every load issued before the stores.  A lane past the row's
// last cell reads inside the padded arrays (the natural row of p holds nx + 10
// entries or more and ghost rows and planes follow the interior) and stores
// nothing.  e stays in place: the next sweep, a cycle's first, reads it as
// zero (first_mode).  Block 0 starts the cycle: inner sweep count and the
// inner loop's condition.
template <class Tc, int NT>
__global__ void __launch_bounds__(NT, 3) k_defect_rows(Geom g, SorCoef<double> sc, SorCoef<Tc> /*st*/, double* p,
                                                    const double* b, Tc* dR, Tc* dB, const Tc* eR, const Tc* eB,
                                                    Ctl* ctl, cudaGraphConditionalHandle inner, int in_graph) {
    const bool incr = ctl->cycles > 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->inner = 0;
        ctl->pad_stop = 0;
        if (in_graph) cudaGraphSetConditional(inner, 1u);
    }
    const int lane = threadIdx.x & 31;
    const int ny = g.ny, nrow = g.ny * g.nz;
    const int nwarp = (int)gridDim.x * (NT / 32);
    const int w0 = blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
    if (w0 >= nrow) return;
    const int nx = g.nx;
    const int half = (nx + 1) / 2;
    const int nown0 = nx / 2, nown1 = (nx + 1) / 2;
    const long long ys = g.mxp, zs = g.mz;

    // cells t0 + lane and t0 + lane + 32 of colour arrays O (other), E (own), D of a
    // row of parity R whose natural row of p starts at pr (i = 0)
    auto chunk = [&](auto rr, const Tc* __restrict__ O, const Tc* __restrict__ E, Tc* __restrict__ D,
                     double* __restrict__ pr, int t0, int nown, double cN, double cS, double cF, double cB) {
        constexpr int R = decltype(rr)::value;
        const int tA = t0 + lane;
        const int m = tA + 2 - R;
        const int iA = 2 * tA + 2 - R;
        const int iAc = min(iA, nx + 2), iBc = min(iA + 64, nx + 2);
        const Tc* __restrict__ o = O + m;
        const Tc* __restrict__ oN = o + ys;
        const Tc* __restrict__ oS = o - ys;
        const Tc* __restrict__ oF = o + zs;
        const Tc* __restrict__ oB = o - zs;
        const Tc nEA = o[R], nWA = o[R - 1], nEB = o[32 + R], nWB = o[31 + R];
        const Tc nNA = oN[0], nNB = oN[32], nSA = oS[0], nSB = oS[32];
        const Tc nFA = oF[0], nFB = oF[32], nBA = oB[0], nBB = oB[32];
        const Tc dA = D[m], dB_ = D[m + 32], eA = E[m], eB_ = E[m + 32];
        double* __restrict__ pp = pr + iA;
        const double pA = pp[0], pB = pp[64];
        const double cEA = sc.cE[iAc], cWA = sc.cW[iAc], cEB = sc.cE[iBc], cWB = sc.cW[iBc];
        const double dnA = defect_update(cEA, nEA, cWA, nWA, cN, nNA, cS, nSA, cF, nFA, cB, nBA, dA, eA);
        const double dnB = defect_update(cEB, nEB, cWB, nWB, cN, nNB, cS, nSB, cF, nFB, cB, nBB, dB_, eB_);
        if (tA < nown) {
            D[m] = (Tc)dnA;
            pp[0] = pA + (double)eA;
        }
        if (tA + 32 < nown) {
            D[m + 32] = (Tc)dnB;
            pp[64] = pB + (double)eB_;
        }
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    int j = w0 % ny + 1, k = w0 / ny + 1;
    const int dj = nwarp % ny, dk = nwarp / ny;
    for (int row = w0; row < nrow; row += nwarp) {
        const long long rb = ys * (j + 1) + zs * (k + 1);
        const double cN = sc.cN[j], cS = sc.cS[j], cF = sc.cF[k], cB = sc.cB[k];
        for (int colour = 0; colour < 2; ++colour) {
            const int r = ((j + k) ^ colour) & 1;
            const Tc* __restrict__ O = (colour ? eR : eB) + rb;
            const Tc* __restrict__ E = (colour ? eB : eR) + rb;
            Tc* __restrict__ D = (colour ? dB : dR) + rb;
            if (incr) {
                double* __restrict__ pr = p + nat(g, 0, j, k);
                const int nown = r ? nown1 : nown0;
                for (int t0 = 0; t0 < nown; t0 += 64) {
                    if (r == 0) chunk(I0{}, O, E, D, pr, t0, nown, cN, cS, cF, cB);
                    else chunk(I1{}, O, E, D, pr, t0, nown, cN, cS, cF, cB);
                }
            } else {
                for (int t = lane; t < half; t += 32) {
                    const int i = 2 * t + 2 - r;
                    if (i > nx) break;
                    const int m = t + 2 - r;
                    const long long c = nat(g, i, j, k);
                    const double dn = defect_value(sc.cE[i], p[c + 1], sc.cW[i], p[c - 1], cN, p[c + g.px], cS,
                                                   p[c - g.px], cF, p[c + g.pz], cB, p[c - g.pz],
                                                   rdiag_of(sc, i, j, k), b[c], p[c]);
                    D[m] = (Tc)dn;
                }
            }
        }
        j += dj;
        k += dk;
        if (j > ny) {
            j -= ny;
            ++k;
        }
    }
}

// One warp: the max over the kSpread slots of that sweep is its max|change|.
// Outside a graph (in_graph = 0) the host reads ctl and takes the decision.
// A test queued after the cycle's stop (bodies queued ahead of the host's
// decision; their sweeps skip) leaves everything as it is.
__global__ void k_sor_check(Ctl* ctl, unsigned long long* slots, int csweeps, int itmax,
                            int cycle_len, double zeta, cudaGraphConditionalHandle inner, int in_graph) {
    if (ctl->pad_stop) return;
    const int lane = threadIdx.x;
    const int ik = ctl->ik, in = ctl->inner;
    int ran = csweeps;
    if (itmax - ik < ran) ran = itmax - ik;
    if (cycle_len - in < ran) ran = cycle_len - in;
    if (ran < 0) ran = 0;
    unsigned long long bits = ran > 0 ? slots[(ran - 1) * kSpread + lane] : 0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t2 = __shfl_xor_sync(0xffffffffu, bits, o);
        bits = t2 > bits ? t2 : bits;
    }
    for (int s = 0; s < csweeps; ++s) slots[s * kSpread + lane] = 0ULL;
    if (lane != 0) return;
    const double change = __longlong_as_double((long long)bits);
    ctl->ik = ik + ran;
    ctl->inner = in + ran;
    ctl->bodies += 1;
    const bool nonfinite = bits >= kInfBits;
    const bool conv = !nonfinite && ran > 0 && !(change > zeta);
    if (ran > 0) ctl->last_change = change;
    if (nonfinite) ctl->nonfinite = 1;
    if (conv) ctl->converged = 1;
    const bool stop = conv || nonfinite || ctl->ik >= itmax || ctl->inner >= cycle_len || ran == 0;
    ctl->pad_stop = stop ? 1 : 0;
    if (in_graph) cudaGraphSetConditional(inner, stop ? 0u : 1u);
}

// p += e over the interior (natural <- colour-split).
template <class Tc>
__global__ void __launch_bounds__(256) k_correct(Geom g, double* p, const Tc* eR, const Tc* eB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long q = spl(g, (i + 2) >> 1, j, k);
    const Tc e = (((i + j + k) & 1) == 0) ? eR[q] : eB[q];
    p[nat(g, i, j, k)] += (double)e;
}

// The streaming solve's final p += e: the e of its last correction cycle
// (k_defect_rows adds the e of every earlier cycle); nothing when no cycle ran.
template <class Tc>
__global__ void __launch_bounds__(256) k_correct_last(Geom g, double* p, const Tc* eR, const Tc* eB, const Ctl* ctl) {
    if (ctl->cycles == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long q = spl(g, (i + 2) >> 1, j, k);
    const Tc e = (((i + j + k) & 1) == 0) ? eR[q] : eB[q];
    p[nat(g, i, j, k)] += (double)e;
}

// Start of a solve: counters reset, outer loop armed when itmax > 0.
__global__ void k_sor_begin(Ctl* ctl, int itmax, cudaGraphConditionalHandle outer, int in_graph) {
    ctl->ik = 0;
    ctl->inner = 0;
    ctl->pad_stop = 0;
    ctl->cycles = 0;
    ctl->restarts = 0;
    ctl->bodies = 0;
    ctl->timeout = 0;
    ctl->converged = 0;
    ctl->nonfinite = 0;
    ctl->last_change = 0.0;
    if (in_graph) cudaGraphSetConditional(outer, itmax > 0 ? 1u : 0u);
}

// End of a defect-correction cycle: another cycle only when the inner loop
// stopped on its cycle length.
__global__ void k_outer_check(Ctl* ctl, int itmax, cudaGraphConditionalHandle outer, int in_graph) {
    ctl->cycles += 1;
    const bool more = !ctl->converged && !ctl->nonfinite && !ctl->timeout && ctl->ik < itmax;
    ctl->pad_more = more ? 1 : 0;
    if (in_graph) cudaGraphSetConditional(outer, more ? 1u : 0u);
}

}  // namespace ntcfd
