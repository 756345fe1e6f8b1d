// k_resident.cuh -- the SOR sweeps of one defect-correction cycle in a single
// persistent cooperative kernel, with the correction e resident in shared
// memory.
//
// The interior rows (j,k) are split into nbj x nbk bricks of at most JB x KB
// rows; CTA b owns brick (b % nbj, b / nbj) and keeps e of both colours for
// its rows plus a one-row halo in shared memory (colour-split rows of mx
// entries, see ntcfd_common.cuh), and the defect d of its rows when it fits.
// A half-sweep updates the CTA's cells of one colour from shared memory,
// publishes the updated brick-boundary rows to the global e arrays, waits at
// a grid barrier and copies the neighbours' boundary rows of that colour
// into its halo.  The sweep count, the stop rule (GS.f90:11,53) and the
// final p += e run inside the kernel.
//
// The grid barrier spins with a bounded number of polls; a CTA that gives
// up sets bar->err, and every CTA leaves the sweep loop at the next barrier,
// so the kernel always ends.  The host reports NTCFD_ETIMEOUT.
#pragma once

#include "k_pressure.cuh"
#include "ntcfd_common.cuh"

namespace ntcfd {

struct GridBar {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
};

struct Brick {
    int nbj, nbk;    // bricks along j and k
    int JB, KB;      // rows per brick (the last brick may hold fewer)
    int mx;          // colour-split row length (compact index m = 0..mx-1)
    int cache_d;     // 1: d of the brick lives in shared memory too
    int cache_rd;    // 1: rd of the brick lives in shared memory too
};

// Dynamic shared memory of k_sor_resident for a brick plan.
template <class Tc>
inline size_t resident_smem(const Brick& b, int nx) {
    const size_t tile = (size_t)(b.JB + 2) * (b.KB + 2) * b.mx;
    const size_t brick = (size_t)b.JB * b.KB * b.mx;
    return sizeof(Tc) * (2 * tile + 2 * (size_t)(nx + 4) + 2 * (size_t)(b.JB + b.KB) +
                         (b.cache_d ? 2 * brick : 0) + (b.cache_rd ? 2 * brick : 0));
}

constexpr unsigned int kBarrierPolls = 20000000u;   // ~1-2 s of polling without sleep

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int atom_add_release(unsigned int* p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int vload(const unsigned int* p) {
    return *(const volatile unsigned int*)p;
}
__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

// Grid-wide barrier of one cooperative launch, split into arrive and wait so
// that a CTA can work between the two.  Thread 0 of each CTA arrives with a
// release add on the counter (after a CTA barrier, so the CTA's earlier
// global writes are published); the last arrival resets the counter and
// publishes the next generation with a release store.  Waiting polls the
// generation with acquire loads, checks the shared error flag every 1024
// polls and gives up after kBarrierPolls polls, setting the flag so that
// every CTA leaves at its next wait.  Returns false on failure.
__device__ __forceinline__ void grid_arrive(GridBar* b, unsigned int nblocks, unsigned int gen) {
    __syncthreads();
    if (threadIdx.x == 0) {
        if (atom_add_release(&b->count, 1u) + 1u == nblocks) {
            b->count = 0u;                       // ordered before the release store below
            st_release(&b->gen, gen + 1u);
        }
    }
}

__device__ __forceinline__ bool grid_wait(GridBar* b, unsigned int& gen, int* s_flag) {
    if (threadIdx.x == 0) {
        const unsigned int target = gen + 1u;
        int fail = 0;
        unsigned int polls = 0;
        while (ld_acquire(&b->gen) != target) {
            if ((++polls & 1023u) == 0u) {
                if (vload(&b->err) != 0) { fail = 1; break; }
                if (polls > kBarrierPolls) {
                    atomicExch(&b->err, 1);
                    fail = 1;
                    break;
                }
            }
        }
        *s_flag = fail;
    }
    __syncthreads();
    gen += 1u;
    return *s_flag == 0;
}

__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned int nblocks, unsigned int& gen,
                                          int* s_flag) {
    grid_arrive(b, nblocks, gen);
    return grid_wait(b, gen, s_flag);
}

template <class Tc, int NT>
__global__ void __launch_bounds__(NT, 1)
k_sor_resident(Geom g, SorCoef<Tc> sc, Brick br, double* __restrict__ p, Tc* __restrict__ eRg,
               Tc* __restrict__ eBg, const Tc* __restrict__ dRg, const Tc* __restrict__ dBg,
               const Tc* __restrict__ rdRg, const Tc* __restrict__ rdBg, Ctl* ctl, GridBar* bar,
               double omega, double zeta, int itmax, int cycle_len, int check_every,
               unsigned long long* ring) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using B = decltype(abs_bits(Tc(0)));
    __shared__ int s_flag;
    __shared__ unsigned int s_gen;
    __shared__ unsigned long long s_ring;
    __shared__ B s_red[NT / 32];
    const int JB = br.JB, KB = br.KB, mx = br.mx;
    const int RS = JB + 2;                    // rows per k-plane of the tile
    const int plane = RS * mx;
    const int tile = plane * (KB + 2);
    const int brick = JB * KB * mx;
    // shared memory: e red, e black (tile with halo), coefficients cE, cW (index
    // i+1, i = -1..nx+2), then d red/black and rd red/black of the brick when cached
    Tc* const S0 = reinterpret_cast<Tc*>(smem_raw);
    Tc* const S1 = S0 + tile;
    Tc* const cEs = S1 + tile + 1;
    Tc* const cWs = cEs + (g.nx + 4);
    Tc* const cNs = cEs + 2 * (g.nx + 4) - 1;   // cN, cS of the brick's rows j0..j0+JB-1
    Tc* const cSs = cNs + JB;
    Tc* const cFs = cSs + JB;                  // cF, cB of the brick's planes k0..k0+KB-1
    Tc* const cBs = cFs + KB;
    Tc* const D0 = cBs + KB;
    Tc* const D1 = D0 + brick;
    Tc* const R0 = br.cache_d ? D1 + brick : D0;
    Tc* const R1 = R0 + brick;
    constexpr int NWARP = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tid = threadIdx.x;

    const int bj = blockIdx.x % br.nbj, bk = blockIdx.x / br.nbj;
    const int j0 = 1 + bj * JB, k0 = 1 + bk * KB;
    const int nj = max(0, min(g.ny, j0 + JB - 1) - j0 + 1);
    const int nk = max(0, min(g.nz, k0 + KB - 1) - k0 + 1);
    const int half = (g.nx + 1) / 2;
    const int ys = g.mxp, zs = (int)g.mz;   // colour-split row and plane pitch

    for (int q = tid; q < 2 * tile; q += NT) S0[q] = Tc(0);
    for (int i = tid - 1; i <= g.nx + 2; i += NT) {
        cEs[i] = sc.cE[i];
        cWs[i] = sc.cW[i];
    }
    for (int q = tid; q < JB; q += NT) {
        const int j = min(j0 + q, g.ny);
        cNs[q] = sc.cN[j];
        cSs[q] = sc.cS[j];
    }
    for (int q = tid; q < KB; q += NT) {
        const int k = min(k0 + q, g.nz);
        cFs[q] = sc.cF[k];
        cBs[q] = sc.cB[k];
    }
    if (br.cache_d || br.cache_rd) {
        for (int q = tid; q < nj * nk * mx; q += NT) {
            const int m = q % mx;
            const int row = q / mx;
            const int jl = row % nj, kl = row / nj;
            const long long gq = spl(g, m, j0 + jl, k0 + kl);
            const int sq = (kl * JB + jl) * mx + m;
            if (br.cache_d) { D0[sq] = dRg[gq]; D1[sq] = dBg[gq]; }
            if (br.cache_rd) { R0[sq] = rdRg[gq]; R1[sq] = rdBg[gq]; }
        }
    }
    if (tid == 0) s_gen = vload(&bar->gen);
    __syncthreads();
    unsigned int gen = s_gen;
    const unsigned int nblocks = gridDim.x;
    const int ik0 = ctl->ik;
    const int nrows = nj * nk;
    const Tc om = (Tc)omega;
    int done = 0;
    bool conv = false, nonfinite = false, failed = false;
    double last = 0.0;

    for (int s = 0; ik0 + s < itmax && s < cycle_len; ++s) {
        if (blockIdx.x == 0 && tid == 0) ring[(s + 1) % 3] = 0ULL;
        B ch = B(0);
        for (int c = 0; c < 2 && !failed; ++c) {
            Tc* W = c ? S1 : S0;
            const Tc* O = c ? S0 : S1;
            Tc* Ec = c ? eBg : eRg;
            const Tc* Dg = c ? dBg : dRg;
            const Tc* Rg = c ? rdBg : rdRg;
            const Tc* Ds = c ? D1 : D0;
            const Tc* Rs = c ? R1 : R0;
            // Two passes over the rows (one warp per row, lanes along the row):
            // first the brick-edge rows, which the neighbours need, then arrive
            // at the grid barrier, then the interior rows, then wait.
            for (int pass = 0; pass < 2; ++pass) {
                int jl = nj > 0 ? warp % nj + 1 : 1, kl = nj > 0 ? warp / nj + 1 : 1;
                for (int row = warp; row < nrows; row += NWARP) {
                    const bool edge = (jl == 1 || jl == nj || kl == 1 || kl == nk);
                    if (edge == (pass == 0)) {
                        const int j = j0 + jl - 1, k = k0 + kl - 1;
                        const int r = ((j + k) ^ c) & 1;
                        const int sr = (kl * RS + jl) * mx;
                        const int dr = ((kl - 1) * JB + (jl - 1)) * mx;
                        const int gr = ys * (j + 1) + zs * (k + 1);
                        const Tc cN = cNs[jl - 1], cS = cSs[jl - 1], cF = cFs[kl - 1], cB = cBs[kl - 1];
                        for (int t = lane; t < half; t += 32) {
                            const int i = 2 * t + 2 - r;
                            if (i > g.nx) break;
                            const int m = t + 2 - r;
                            const int so = sr + m;
                            const Tc sum = cEs[i] * O[so + r] + cWs[i] * O[so - 1 + r] + cN * O[so + mx] +
                                           cS * O[so - mx] + cF * O[so + plane] + cB * O[so - plane];
                            const Tc rd = br.cache_rd ? Rs[dr + m] : __ldg(Rg + gr + m);
                            const Tc dv = br.cache_d ? Ds[dr + m] : __ldg(Dg + gr + m);
                            const Tc e0 = W[so];
                            const Tc diff = (rd * sum + dv) - e0;
                            const Tc e1 = e0 + om * diff;
                            W[so] = e1;
                            if (edge) Ec[gr + m] = e1;
                            const B db = abs_bits(diff);
                            ch = db > ch ? db : ch;
                        }
                    }
                    jl += NWARP;
                    while (jl > nj) { jl -= nj; ++kl; }
                }
                // red half: arrive once the edge rows are out, wait after the interior
                if (pass == 0 && c == 0) grid_arrive(bar, nblocks, gen);
            }
            if (c == 1) {
                // this CTA's max |change| over the sweep -> ring slot of sweep s
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const B t2 = __shfl_xor_sync(0xffffffffu, ch, o);
                    ch = t2 > ch ? t2 : ch;
                }
                if (lane == 0) s_red[warp] = ch;
                __syncthreads();
                if (tid < 32) {
                    B b2 = (tid < NWARP) ? s_red[tid] : B(0);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const B t2 = __shfl_xor_sync(0xffffffffu, b2, o);
                        b2 = t2 > b2 ? t2 : b2;
                    }
                    if (tid == 0 && b2 != B(0)) atomicMax(&ring[s % 3], widen_bits(b2));
                }
                // black half: a full barrier, so that every CTA's max (interior
                // rows included) is in the ring before anyone reads it
                if (!grid_sync(bar, nblocks, gen, &s_flag)) {
                    failed = true;
                    break;
                }
                if (tid == 0) s_ring = *(volatile unsigned long long*)&ring[s % 3];
            } else if (!grid_wait(bar, gen, &s_flag)) {
                failed = true;
                break;
            }
            // neighbours' boundary rows of colour c into the halo, one warp per row
            for (int h = warp; h < 2 * nk + 2 * nj; h += NWARP) {
                int jl, kl;
                if (h < 2 * nk) { kl = h % nk + 1; jl = (h < nk) ? 0 : nj + 1; }
                else { const int h2 = h - 2 * nk; jl = h2 % nj + 1; kl = (h2 < nj) ? 0 : nk + 1; }
                const int j = j0 + jl - 1, k = k0 + kl - 1;
                if (j < 1 || j > g.ny || k < 1 || k > g.nz) continue;   // domain ghosts stay 0
                const Tc* src = Ec + spl(g, 0, j, k);
                Tc* dst = W + (kl * RS + jl) * mx;
                // L2 reads (ld.global.cg): the rows were written by other CTAs this half-sweep
                for (int m = lane; m < mx; m += 32) dst[m] = __ldcg(src + m);
            }
            __syncthreads();
        }
        if (failed) break;
        done = s + 1;
        const int ik = ik0 + done;
        if (ik % check_every == 0 || ik >= itmax) {
            const unsigned long long bits = s_ring;
            last = __longlong_as_double((long long)bits);
            nonfinite = bits >= kInfBits;
            conv = !nonfinite && !(last > zeta);
            if (conv || nonfinite) break;
        }
    }
    // p += e over the brick (natural <- shared memory)
    for (int it = tid; it < nj * nk * g.nx; it += NT) {
        const int i = it % g.nx + 1;
        const int row = it / g.nx;
        const int jl = row % nj + 1, kl = row / nj + 1;
        const int j = j0 + jl - 1, k = k0 + kl - 1;
        const int col = (i + j + k) & 1;
        p[nat(g, i, j, k)] += (double)(col ? S1 : S0)[(kl * RS + jl) * mx + ((i + 2) >> 1)];
    }
    if (blockIdx.x == 0 && tid == 0) {
        ctl->ik = ik0 + done;
        ctl->inner = done;
        ctl->bodies += done;
        if (done > 0) ctl->last_change = last;
        if (conv) ctl->converged = 1;
        if (nonfinite) ctl->nonfinite = 1;
        if (failed) ctl->timeout = 1;
    }
}

}  // namespace ntcfd
