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

#include "ntcfd_common.cuh"

namespace ntcfd {

template <class Tc>
struct SorCoef {
    const Tc *cE, *cW, *cN, *cS, *cF, *cB;
};

template <class Tc>
__device__ __forceinline__ Tc rdiag_of(const SorCoef<Tc>& s, int i, int j, int k) {
    return Tc(1) / (((s.cE[i] + s.cW[i]) + (s.cN[j] + s.cS[j])) + (s.cF[k] + s.cB[k]));
}

// K3a -- b' on the interior from the predicted velocity (GS.f90:39-41).
// u*(0,j,k), v*(i,0,k), w*(i,j,0) equal the state's ghosts (the reference
// copies u into u_star over the whole halo array in boundary_conditions.f90:317-319).
__global__ void __launch_bounds__(256) k_rhs(Geom g, SorCoef<double> sc, const double* u,
                                             const double* v, const double* w, const double* us,
                                             const double* vs, const double* ws, double* b,
                                             double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double uw = (i == 1) ? u[c - 1] : us[c - 1];
    const double vs_ = (j == 1) ? v[c - g.px] : vs[c - g.px];
    const double wb = (k == 1) ? w[c - g.pz] : ws[c - g.pz];
    const double divv = (us[c] - uw) * g.riDx[i] + (vs[c] - vs_) * g.riDy[j] + (ws[c] - wb) * g.riDz[k];
    b[c] = rdiag_of(sc, i, j, k) * divv / dt;
}

// Defect d = rdiag*sum c p0_nb - b' - p0 in double, stored per colour in
// Tc; e reset to 0.  Inside the step graph (in_graph = 1) it also arms the
// inner loop's condition.
template <class Tc>
__global__ void __launch_bounds__(256) k_defect(Geom g, SorCoef<double> sc, const double* p,
                                                const double* b, Tc* dR, Tc* dB, Tc* eR, Tc* eB,
                                                Ctl* ctl, cudaGraphConditionalHandle inner,
                                                int in_graph) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (in_graph && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0 && threadIdx.z == 0) {
        ctl->inner = 0;
        cudaGraphSetConditional(inner, 1u);
    }
    if (i > g.nx || j > g.ny || k > g.nz) return;
    const long long c = nat(g, i, j, k);
    const double s = sc.cE[i] * p[c + 1] + sc.cW[i] * p[c - 1] + sc.cN[j] * p[c + g.px] +
                     sc.cS[j] * p[c - g.px] + sc.cF[k] * p[c + g.pz] + sc.cB[k] * p[c - g.pz];
    const double d = rdiag_of(sc, i, j, k) * s - b[c] - p[c];
    const long long q = spl(g, (i + 2) >> 1, j, k);
    if (((i + j + k) & 1) == 0) { dR[q] = (Tc)d; eR[q] = Tc(0); }
    else { dB[q] = (Tc)d; eB[q] = Tc(0); }
}

// One half-sweep over colour `colour` (0 = red, (i+j+k) even).  Thread t of
// row (j,k) owns the cell i = 2t + 2 - r, m = t + 2 - r, r = ((j+k)^colour)&1.
// `sub` is the index of this sweep inside the loop body; the sweep is skipped
// once the sweep budget (itmax, cycle length) is used up.
template <class Tc, int NT>
__global__ void __launch_bounds__(NT) k_sweep(Geom g, SorCoef<Tc> sc, Tc* eOwn, const Tc* eOth,
                                              const Tc* dOwn, int colour, double omega, Ctl* ctl,
                                              int sub, int itmax, int cycle_len,
                                              unsigned long long* slots) {
    const int ik = ctl->ik, inner = ctl->inner;
    if (ik + sub >= itmax || inner + sub >= cycle_len) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    double ch = 0.0;
    if (j <= g.ny && k <= g.nz) {
        const int r = ((j + k) ^ colour) & 1;
        const int i = 2 * t + 2 - r;
        if (i >= 1 && i <= g.nx) {
            const int m = t + 2 - r;
            const long long q = spl(g, m, j, k);
            const Tc s = sc.cE[i] * eOth[q + r] + sc.cW[i] * eOth[q - 1 + r] +
                         sc.cN[j] * eOth[q + g.mxp] + sc.cS[j] * eOth[q - g.mxp] +
                         sc.cF[k] * eOth[q + g.mz] + sc.cB[k] * eOth[q - g.mz];
            const Tc eNew = rdiag_of(sc, i, j, k) * s + dOwn[q];
            const Tc e0 = eOwn[q];
            const Tc diff = eNew - e0;
            eOwn[q] = e0 + (Tc)omega * diff;
            ch = (double)fabs(diff);
        }
    }
    block_max_atomic<NT>(ch, &slots[sub]);
}

// Loop control after a group of `csweeps` sweeps (one WHILE body).
// Implements `do while (pChangeMax_ > zeta .and. ik < itmax)` (GS.f90:11)
// on the change of the last sweep that ran; a cycle of the mixed path also
// ends after cycle_len sweeps.
__global__ void k_sor_check(Ctl* ctl, unsigned long long* slots, int csweeps, int itmax,
                            int cycle_len, double zeta, cudaGraphConditionalHandle inner) {
    const int ik = ctl->ik, in = ctl->inner;
    int ran = csweeps;
    if (itmax - ik < ran) ran = itmax - ik;
    if (cycle_len - in < ran) ran = cycle_len - in;
    if (ran < 0) ran = 0;
    unsigned long long bits = ran > 0 ? slots[ran - 1] : 0ULL;
    for (int s = 0; s < csweeps; ++s) slots[s] = 0ULL;
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
    cudaGraphSetConditional(inner, stop ? 0u : 1u);
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

// Start of a solve: counters reset, outer loop armed when itmax > 0.
__global__ void k_sor_begin(Ctl* ctl, int itmax, cudaGraphConditionalHandle outer) {
    ctl->ik = 0;
    ctl->inner = 0;
    ctl->cycles = 0;
    ctl->bodies = 0;
    ctl->converged = 0;
    ctl->nonfinite = 0;
    ctl->last_change = 0.0;
    cudaGraphSetConditional(outer, itmax > 0 ? 1u : 0u);
}

// End of a defect-correction cycle: another cycle only when the inner loop
// stopped on its cycle length.
__global__ void k_outer_check(Ctl* ctl, int itmax, cudaGraphConditionalHandle outer) {
    ctl->cycles += 1;
    const bool more = !ctl->converged && !ctl->nonfinite && ctl->ik < itmax;
    cudaGraphSetConditional(outer, more ? 1u : 0u);
}

}  // namespace ntcfd
