// k_resident.cuh -- the SOR sweeps of one defect-correction cycle in a single
// persistent cooperative kernel, with the correction e resident in shared
// memory.
//
// The interior rows (j,k) are split into nbj x nbk bricks of at most JB x KB
// rows; CTA b owns brick (b % nbj, b / nbj) and keeps e of both colours for
// its rows in shared memory (colour-split rows of mx entries, see
// ntcfd_common.cuh; the tile has a one-row ring that stays 0 and stands for
// the domain's ghost rows), and the defect d of its rows when it fits.
// A half-sweep updates the CTA's cells of one colour from shared memory,
// the brick-boundary rows first: they read the neighbour bricks' rows
// straight from the global e arrays (L2), where every CTA publishes its own
// boundary rows as it updates them; then the CTA arrives at a grid barrier,
// updates its interior rows from shared memory only and waits.  The sweep
// count, the stop rule (GS.f90:11,53), the count
// of correction cycles and the final p += e run inside the kernel, and so do
// the restarts of the
// defect correction: when a cycle ends on its length (cycle_len sweeps), the
// kernel adds e to p, zeroes e (its published boundary rows included),
// passes a grid barrier, recomputes the FP64 defect of its brick (the
// arithmetic of k_defect) and sweeps on from e = 0.
//
// The grid barrier spins with a bounded number of polls; a CTA that gives
// up sets bar->err, and every CTA leaves the sweep loop at the next barrier,
// so the kernel always ends.  The host reports NTCFD_ETIMEOUT.
#pragma once

#include "k_pressure.cuh"
#include "ntcfd_common.cuh"

namespace ntcfd {

struct GridBar {
    unsigned int count;   // arrivals (low bits) and phase (top bit), see grid_arrive
    unsigned int gen;     // unused
    int err;
    int pad;
};

struct Brick {
    int nbj, nbk;    // bricks along j and k
    int JB, KB;      // rows per brick (the last brick may hold fewer)
    int mx;          // colour-split row length (compact index m = 0..mx-1)
    int cache_d;     // 1: d of the brick lives in shared memory too
    int cache_rd;    // 1: rd of the brick lives in shared memory too
    int narrow;      // 1: the NARROW instance (narrow_rows(nx))
};

// Dynamic shared memory of k_sor_resident for a brick plan.
template <class Tc>
inline size_t resident_smem(const Brick& b, int nx) {
    const size_t tile = (size_t)(b.JB + 2) * (b.KB + 2) * b.mx;
    const size_t brick = (size_t)b.JB * b.KB * b.mx;
    const size_t arrays = sizeof(Tc) * (2 * tile + 2 * (size_t)(nx + 4) + 2 * (size_t)(b.JB + b.KB) +
                                        (b.cache_d ? 2 * brick : 0) + (b.cache_rd ? 2 * brick : 0));
    // + row table (int4 offsets and four coefficients per row)
    const size_t rows = (size_t)b.JB * b.KB;
    return ((arrays + 15) & ~size_t(15)) + rows * (16 + 4 * sizeof(Tc));
}

constexpr unsigned int kBarrierPolls = 20000000u;   // ~1-2 s of polling without sleep
// Rows of at most 32 cells of a colour: the kernel's NARROW instance.
__host__ __device__ inline bool narrow_rows(int nx) { return (nx + 1) / 2 <= 32; }

constexpr int kFill = 4;      // elements in flight per lane when a CTA walks its brick
constexpr int kDefect = 2;    // cells in flight per lane in the in-kernel defect

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
// that a CTA can work between the two.  One 32-bit word counts arrivals:
// thread 0 of CTA 0 adds 2^31 - (nblocks - 1), every other CTA adds 1 (each
// with a release add, after a CTA barrier, so the CTA's earlier global
// writes are published).  Whatever the order, the top bit of the word flips
// exactly when the last CTA arrives and the low bits return to their value,
// so the word needs no reset between barriers and no second store releases
// the waiters.  Waiting polls the word with acquire loads until its top bit
// differs from the one this CTA's add returned, checks the shared error flag
// every 1024 polls and gives up after kBarrierPolls polls, setting the flag
// so that every CTA leaves at its next wait.  Returns false on failure.
__device__ __forceinline__ void grid_arrive(GridBar* b, unsigned int nblocks, unsigned int& ticket) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int inc = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1u) : 1u;
        ticket = atom_add_release(&b->count, inc);
    }
}

// With src non-null, thread 0 also copies *src (read after the barrier) to *dst
// before the closing CTA barrier, so every thread sees the same value.
__device__ __forceinline__ bool grid_wait(GridBar* b, unsigned int ticket, int* s_flag,
                                          const unsigned long long* src = nullptr,
                                          unsigned long long* dst = nullptr) {
    if (threadIdx.x == 0) {
        int fail = 0;
        unsigned int polls = 0;
        while (((ld_acquire(&b->count) ^ ticket) & 0x80000000u) == 0u) {
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
        if (src) *dst = *(const volatile unsigned long long*)src;
    }
    __syncthreads();
    return *s_flag == 0;
}

__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned int nblocks, int* s_flag,
                                          const unsigned long long* src = nullptr,
                                          unsigned long long* dst = nullptr) {
    unsigned int ticket = 0;
    grid_arrive(b, nblocks, ticket);
    return grid_wait(b, ticket, s_flag, src, dst);
}

// Row e of a brick's edge ring (jl or kl on the brick boundary), for e < ne,
// or of its interior, for e >= ne; nj x nk rows, ni = interior rows.
__device__ __forceinline__ void brick_row(int e, int nj, int nk, int ni, int ne, int& jl, int& kl) {
    if (ni == 0) {                       // every row is an edge row
        jl = e % nj + 1;
        kl = e / nj + 1;
    } else if (e >= ne) {                // interior: (nj-2) x (nk-2) rows
        const int q = e - ne;
        jl = q % (nj - 2) + 2;
        kl = q / (nj - 2) + 2;
    } else if (e < 2 * nj) {             // first and last k-row of the brick
        jl = e % nj + 1;
        kl = e < nj ? 1 : nk;
    } else {                             // first and last j-row, inner k
        const int q = e - 2 * nj;
        kl = q % (nk - 2) + 2;
        jl = q < nk - 2 ? 1 : nj;
    }
}

template <class Tc, int NT, bool CD, bool CR, bool NARROW>
__global__ void __launch_bounds__(NT, 1)
k_sor_resident(Geom g, SorCoef<Tc> sc, Brick br, double* __restrict__ p, const double* __restrict__ b,
               Tc* __restrict__ eRg,
               Tc* __restrict__ eBg, Tc* __restrict__ dRg, Tc* __restrict__ dBg,
               const Tc* __restrict__ rdRg, const Tc* __restrict__ rdBg, Ctl* ctl, GridBar* bar,
               double omega, double zeta, int itmax, int cycle_len, int check_every,
               unsigned long long* ring) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using B = decltype(abs_bits(Tc(0)));
    __shared__ int s_flag;
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
    Tc* const R0 = CD ? D1 + brick : D0;
    Tc* const R1 = R0 + brick;
    Tc* const arrays_end = CR ? R1 + brick : (CD ? D1 + brick : D0);
    // row table: per row of the brick, in sweep order (edge rows first), the shared-memory
    // tile row, the brick row of d/rd, the global colour-split row, and (j+k)&1 plus
    // four bits (N, S, F, B) set where that neighbour row lies in another brick; and
    // the row's cN, cS, cF, cB
    const size_t toff = ((size_t)((unsigned char*)arrays_end - smem_raw) + 15) & ~size_t(15);
    int4* const rowT = reinterpret_cast<int4*>(smem_raw + toff);
    Tc* const rowC = reinterpret_cast<Tc*>(rowT + JB * KB);
    constexpr int NWARP = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tid = threadIdx.x;

    const int bj = blockIdx.x % br.nbj, bk = blockIdx.x / br.nbj;
    const int j0 = 1 + bj * JB, k0 = 1 + bk * KB;
    const int nj = max(0, min(g.ny, j0 + JB - 1) - j0 + 1);
    const int nk = max(0, min(g.nz, k0 + KB - 1) - k0 + 1);
    const int half = (g.nx + 1) / 2;
    // NARROW (the launch's rows have at most 32 cells of a colour, narrow_rows()): a
    // lane's two cells lie in two rows
    constexpr bool narrow = NARROW;
    const int rpw = narrow ? 2 : 1, tstep = narrow ? 32 : 64;
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
    {
        const int nr = nj * nk;
        const int nin = (nj > 2 && nk > 2) ? (nj - 2) * (nk - 2) : 0;
        for (int er = tid; er < nr; er += NT) {
            int jl, kl;
            brick_row(er, nj, nk, nin, nr - nin, jl, kl);
            const int j = j0 + jl - 1, k = k0 + kl - 1;
            const int far = (jl == nj && j < g.ny ? 2 : 0) | (jl == 1 && j > 1 ? 4 : 0) |
                            (kl == nk && k < g.nz ? 8 : 0) | (kl == 1 && k > 1 ? 16 : 0);
            rowT[er] = make_int4((kl * RS + jl) * mx, ((kl - 1) * JB + (jl - 1)) * mx,
                                 ys * (j + 1) + zs * (k + 1), ((j + k) & 1) | far);
            rowC[4 * er + 0] = sc.cN[j];
            rowC[4 * er + 1] = sc.cS[j];
            rowC[4 * er + 2] = sc.cF[k];
            rowC[4 * er + 3] = sc.cB[k];
        }
    }
    if (CD || CR) {
        // one warp per row, lanes along m, kFill elements of each array in flight per lane
        for (int row = warp; row < nj * nk; row += NT / 32) {
            const int jl = row % nj, kl = row / nj;
            const long long gq0 = spl(g, 0, j0 + jl, k0 + kl);
            const int sq0 = (kl * JB + jl) * mx;
            for (int m0 = 0; m0 < mx; m0 += 32 * kFill) {
                Tc a0[kFill], a1[kFill], a2[kFill], a3[kFill];
#pragma unroll
                for (int u = 0; u < kFill; ++u) {
                    const int m = m0 + lane + 32 * u;
                    if (m < mx) {
                        if (CD) { a0[u] = dRg[gq0 + m]; a1[u] = dBg[gq0 + m]; }
                        if (CR) { a2[u] = rdRg[gq0 + m]; a3[u] = rdBg[gq0 + m]; }
                    }
                }
#pragma unroll
                for (int u = 0; u < kFill; ++u) {
                    const int m = m0 + lane + 32 * u;
                    if (m < mx) {
                        if (CD) { D0[sq0 + m] = a0[u]; D1[sq0 + m] = a1[u]; }
                        if (CR) { R0[sq0 + m] = a2[u]; R1[sq0 + m] = a3[u]; }
                    }
                }
            }
        }
    }
    __syncthreads();
    unsigned int ticket = 0;   // thread 0: the barrier word before this CTA's last arrival
    const unsigned int nblocks = gridDim.x;
    const int ik0 = ctl->ik;
    const int nrows = nj * nk;
    const int ni = (nj > 2 && nk > 2) ? (nj - 2) * (nk - 2) : 0;   // interior rows
    const int ne = nrows - ni;                                       // edge rows
    const Tc om = (Tc)omega;
    int done = 0;        // sweeps of this launch
    int done_c = 0;      // sweeps of the current cycle
    int restarts = 0;
    bool conv = false, nonfinite = false, failed = false;
    double last = 0.0;
    // p += e over the brick (natural <- shared memory)
    // (one warp per row, lanes along i, kFill values of p in flight per lane)
    auto add_e_to_p = [&]() {
        for (int row = warp; row < nrows; row += NWARP) {
            const int jl = row % nj + 1, kl = row / nj + 1;
            const int j = j0 + jl - 1, k = k0 + kl - 1;
            const long long c0 = nat(g, 0, j, k);
            const int sr = (kl * RS + jl) * mx;
            for (int i0 = 1; i0 <= g.nx; i0 += 32 * kFill) {
                double pv[kFill];
#pragma unroll
                for (int u = 0; u < kFill; ++u) {
                    const int i = i0 + lane + 32 * u;
                    if (i <= g.nx) pv[u] = p[c0 + i];
                }
#pragma unroll
                for (int u = 0; u < kFill; ++u) {
                    const int i = i0 + lane + 32 * u;
                    if (i <= g.nx) p[c0 + i] = pv[u] + (double)(((i + j + k) & 1) ? S1 : S0)[sr + ((i + 2) >> 1)];
                }
            }
        }
    };

  for (;;) {
    done_c = 0;
    for (int s = 0; ik0 + done + s < itmax && s < cycle_len; ++s) {
        const int sg = done + s;   // sweep of this launch: ring slot
        if (blockIdx.x == 0 && tid == 0) ring[(sg + 1) % 3] = 0ULL;
        B ch = B(0);
        for (int c = 0; c < 2 && !failed; ++c) {
            Tc* W = c ? S1 : S0;
            const Tc* O = c ? S0 : S1;
            Tc* Ec = c ? eBg : eRg;
            const Tc* Og = c ? eRg : eBg;   // the other colour, as the neighbour bricks publish it
            const Tc* Dg = c ? dBg : dRg;
            const Tc* Rg = c ? rdBg : rdRg;
            const Tc* Ds = c ? D1 : D0;
            const Tc* Rs = c ? R1 : R0;
            // Two passes over the rows (lanes along a row): first the brick-edge
            // rows, which the neighbours need, then arrive at the grid barrier,
            // then the interior rows, then wait.  An edge row reads a neighbour
            // row that lies in another brick from the global array
            // (ld.global.cg: it was written by that brick's CTA before the last
            // barrier); all its other reads are shared memory.  A lane updates two
            // cells with every load issued before any store: t and t + 32 of one
            // row, or, in the NARROW instance, t of two rows (a warp then takes two
            // rows at a time).  The wide loop is kept apart so that it carries none
            // of the narrow loop's per-cell selects.
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const bool edge = pass == 0;
                const int e0r = edge ? 0 : ne, e1r = edge ? ne : nrows;
                if constexpr (!NARROW) {
                    for (int er = e0r + warp; er < e1r; er += NWARP) {
                        const int4 rt = rowT[er];
                        const int sr = rt.x, dr = rt.y, gr = rt.z, r = (rt.w ^ c) & 1;
                        const int far = edge ? rt.w : 0;
                        const Tc cN = rowC[4 * er], cS = rowC[4 * er + 1], cF = rowC[4 * er + 2],
                                 cB = rowC[4 * er + 3];
                        // two cells per lane (t and t + 32), every load issued before any store
                        for (int t0 = lane; t0 < half; t0 += 64) {
                            const int tB = t0 + 32;
                            const int iA = 2 * t0 + 2 - r, iB0 = 2 * tB + 2 - r;
                            if (iA > g.nx) break;
                            const bool okB = tB < half && iB0 <= g.nx;
                            const int mA = t0 + 2 - r, mB = okB ? tB + 2 - r : mA;
                            const int iB = okB ? iB0 : iA;
                            const int sA = sr + mA, sB = sr + mB;
                            const Tc eA = cEs[iA], wA = cWs[iA], eB = cEs[iB], wB = cWs[iB];
                            const Tc oEA = O[sA + r], oWA = O[sA - 1 + r];
                            const Tc oEB = O[sB + r], oWB = O[sB - 1 + r];
                            const Tc oNA = (far & 2) ? __ldcg(Og + gr + ys + mA) : O[sA + mx];
                            const Tc oNB = (far & 2) ? __ldcg(Og + gr + ys + mB) : O[sB + mx];
                            const Tc oSA = (far & 4) ? __ldcg(Og + gr - ys + mA) : O[sA - mx];
                            const Tc oSB = (far & 4) ? __ldcg(Og + gr - ys + mB) : O[sB - mx];
                            const Tc oFA = (far & 8) ? __ldcg(Og + gr + zs + mA) : O[sA + plane];
                            const Tc oFB = (far & 8) ? __ldcg(Og + gr + zs + mB) : O[sB + plane];
                            const Tc oBA = (far & 16) ? __ldcg(Og + gr - zs + mA) : O[sA - plane];
                            const Tc oBB = (far & 16) ? __ldcg(Og + gr - zs + mB) : O[sB - plane];
                            const Tc rdA = CR ? Rs[dr + mA] : __ldg(Rg + gr + mA);
                            const Tc rdB = CR ? Rs[dr + mB] : __ldg(Rg + gr + mB);
                            // d may be rewritten by a restart of this launch, by this CTA only:
                            // a plain (L1-coherent) load, not the read-only path
                            const Tc dvA = CD ? Ds[dr + mA] : __ldca(Dg + gr + mA);
                            const Tc dvB = CD ? Ds[dr + mB] : __ldca(Dg + gr + mB);
                            const Tc e0A = W[sA], e0B = W[sB];
                            const Tc sumA = eA * oEA + wA * oWA + cN * oNA + cS * oSA + cF * oFA + cB * oBA;
                            const Tc sumB = eB * oEB + wB * oWB + cN * oNB + cS * oSB + cF * oFB + cB * oBB;
                            const Tc diffA = (rdA * sumA + dvA) - e0A;
                            const Tc diffB = (rdB * sumB + dvB) - e0B;
                            const Tc e1A = e0A + om * diffA;
                            const Tc e1B = e0B + om * diffB;
                            W[sA] = e1A;
                            if (edge) Ec[gr + mA] = e1A;
                            const B dbA = abs_bits(diffA);
                            ch = dbA > ch ? dbA : ch;
                            if (okB) {
                                W[sB] = e1B;
                                if (edge) Ec[gr + mB] = e1B;
                                const B dbB = abs_bits(diffB);
                                ch = dbB > ch ? dbB : ch;
                            }
                        }
                    }
                } else {
                    for (int er = e0r + warp * rpw; er < e1r; er += NWARP * rpw) {
                        const int erB = narrow && er + 1 < e1r ? er + 1 : er;
                        const bool rowB = !narrow || er + 1 < e1r;
                        const int4 rt = rowT[er], rtB = rowT[erB];
                        const int sr = rt.x, dr = rt.y, gr = rt.z, r = (rt.w ^ c) & 1;
                        const int srB = rtB.x, drB = rtB.y, grB = rtB.z, rB = (rtB.w ^ c) & 1;
                        const int far = edge ? rt.w : 0, farB = edge ? rtB.w : 0;
                        const Tc cN = rowC[4 * er], cS = rowC[4 * er + 1], cF = rowC[4 * er + 2],
                                 cB = rowC[4 * er + 3];
                        const Tc cNB = rowC[4 * erB], cSB = rowC[4 * erB + 1], cFB = rowC[4 * erB + 2],
                                 cBB = rowC[4 * erB + 3];
                        for (int t0 = lane; t0 < half; t0 += tstep) {
                            const int tB = narrow ? t0 : t0 + 32;
                            const int iA0 = 2 * t0 + 2 - r, iB0 = 2 * tB + 2 - rB;
                            const bool okA = iA0 <= g.nx;
                            const bool okB = rowB && tB < half && iB0 <= g.nx;
                            if (!okA && !okB) break;
                            // an invalid cell reuses the other cell's (valid) addresses and is not stored
                            const int mA0 = t0 + 2 - r, mB0 = tB + 2 - rB;
                            const int mA = okA ? mA0 : mB0, mB = okB ? mB0 : mA0;
                            const int iA = okA ? iA0 : iB0, iB = okB ? iB0 : iA0;
                            const int rAc = okA ? r : rB, rBc = okB ? rB : r;
                            const int srA = okA ? sr : srB, srBc = okB ? srB : sr;
                            const int drA = okA ? dr : drB, drBc = okB ? drB : dr;
                            const int grA = okA ? gr : grB, grBc = okB ? grB : gr;
                            const int farA = okA ? far : farB, farBc = okB ? farB : far;
                            const Tc cNA = okA ? cN : cNB, cSA = okA ? cS : cSB, cFA = okA ? cF : cFB,
                                     cBA = okA ? cB : cBB;
                            const Tc cNb = okB ? cNB : cN, cSb = okB ? cSB : cS, cFb = okB ? cFB : cF,
                                     cBb = okB ? cBB : cB;
                            const int sA = srA + mA, sB = srBc + mB;
                            const Tc eA = cEs[iA], wA = cWs[iA], eB = cEs[iB], wB = cWs[iB];
                            const Tc oEA = O[sA + rAc], oWA = O[sA - 1 + rAc];
                            const Tc oEB = O[sB + rBc], oWB = O[sB - 1 + rBc];
                            const Tc oNA = (farA & 2) ? __ldcg(Og + grA + ys + mA) : O[sA + mx];
                            const Tc oNB = (farBc & 2) ? __ldcg(Og + grBc + ys + mB) : O[sB + mx];
                            const Tc oSA = (farA & 4) ? __ldcg(Og + grA - ys + mA) : O[sA - mx];
                            const Tc oSB = (farBc & 4) ? __ldcg(Og + grBc - ys + mB) : O[sB - mx];
                            const Tc oFA = (farA & 8) ? __ldcg(Og + grA + zs + mA) : O[sA + plane];
                            const Tc oFB = (farBc & 8) ? __ldcg(Og + grBc + zs + mB) : O[sB + plane];
                            const Tc oBA = (farA & 16) ? __ldcg(Og + grA - zs + mA) : O[sA - plane];
                            const Tc oBB = (farBc & 16) ? __ldcg(Og + grBc - zs + mB) : O[sB - plane];
                            const Tc rdA = CR ? Rs[drA + mA] : __ldg(Rg + grA + mA);
                            const Tc rdB = CR ? Rs[drBc + mB] : __ldg(Rg + grBc + mB);
                            // d may be rewritten by a restart of this launch, by this CTA only:
                            // a plain (L1-coherent) load, not the read-only path
                            const Tc dvA = CD ? Ds[drA + mA] : __ldca(Dg + grA + mA);
                            const Tc dvB = CD ? Ds[drBc + mB] : __ldca(Dg + grBc + mB);
                            const Tc e0A = W[sA], e0B = W[sB];
                            const Tc sumA = eA * oEA + wA * oWA + cNA * oNA + cSA * oSA + cFA * oFA + cBA * oBA;
                            const Tc sumB = eB * oEB + wB * oWB + cNb * oNB + cSb * oSB + cFb * oFB + cBb * oBB;
                            const Tc diffA = (rdA * sumA + dvA) - e0A;
                            const Tc diffB = (rdB * sumB + dvB) - e0B;
                            const Tc e1A = e0A + om * diffA;
                            const Tc e1B = e0B + om * diffB;
                            if (okA) {
                                W[sA] = e1A;
                                if (edge) Ec[grA + mA] = e1A;
                                const B dbA = abs_bits(diffA);
                                ch = dbA > ch ? dbA : ch;
                            }
                            if (okB) {
                                W[sB] = e1B;
                                if (edge) Ec[grBc + mB] = e1B;
                                const B dbB = abs_bits(diffB);
                                ch = dbB > ch ? dbB : ch;
                            }
                        }
                    }
                }
                // red half: arrive once the edge rows are out, wait after the interior
                if (pass == 0 && c == 0) grid_arrive(bar, nblocks, ticket);
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
                    if (tid == 0 && b2 != B(0)) atomicMax(&ring[sg % 3], widen_bits(b2));
                }
                // black half: a full barrier, so that every CTA's max (interior
                // rows included) is in the ring before anyone reads it
                if (!grid_sync(bar, nblocks, &s_flag, &ring[sg % 3], &s_ring)) {
                    failed = true;
                    break;
                }
            } else if (!grid_wait(bar, ticket, &s_flag)) {
                failed = true;
                break;
            }
        }
        if (failed) break;
        done_c = s + 1;
        const int ik = ik0 + done + done_c;
        if (ik % check_every == 0 || ik >= itmax) {
            const unsigned long long bits = s_ring;
            last = __longlong_as_double((long long)bits);
            nonfinite = bits >= kInfBits;
            conv = !nonfinite && !(last > zeta);
            if (conv || nonfinite) break;
        }
    }
    done += done_c;
    // another cycle only when this one ended on its length
    if (failed || conv || nonfinite || done_c < cycle_len || ik0 + done >= itmax) break;
    // restart: p += e, then the FP64 defect from the updated p, with e = 0
    add_e_to_p();
    __syncthreads();
    for (int q = tid; q < 2 * tile; q += NT) S0[q] = Tc(0);
    // the published boundary rows too: the neighbour bricks read them as this brick's e
    for (int q = tid; q < ne * mx; q += NT) {
        const int er = q / mx, m = q - er * mx;
        const int gr = rowT[er].z;
        eRg[gr + m] = Tc(0);
        eBg[gr + m] = Tc(0);
    }
    if (!grid_sync(bar, nblocks, &s_flag)) {
        failed = true;
        break;
    }
    {
        // one warp per row, lanes along i, kDefect cells in flight per lane; p of this
        // launch's other CTAs is read from L2
        const SorCoef<double> scd{g.cE, g.cW, g.cN, g.cS, g.cF, g.cB};
        for (int row = warp; row < nrows; row += NWARP) {
            const int jl = row % nj + 1, kl = row / nj + 1;
            const int j = j0 + jl - 1, k = k0 + kl - 1;
            const long long c0 = nat(g, 0, j, k);
            const int dr = ((kl - 1) * JB + (jl - 1)) * mx;
            const long long g0 = spl(g, 0, j, k);
            // the coefficients are loaded with p, not after it: a second round trip
            // per chunk would double the pass
            const double cN = scd.cN[j], cS = scd.cS[j], cF = scd.cF[k], cB = scd.cB[k];
            // rows of this brick (and the frozen ghosts) through L1: this CTA wrote them
            // itself (stores do not leave stale L1 lines on the writing SM); rows of the
            // neighbour bricks, written by other SMs, from L2 only
            const bool nL1 = jl < nj || j == g.ny, sL1 = jl > 1 || j == 1;
            const bool fL1 = kl < nk || k == g.nz, bL1 = kl > 1 || k == 1;
            for (int i0 = 1; i0 <= g.nx; i0 += 32 * kDefect) {
                double pe[kDefect], pw[kDefect], pn[kDefect], ps[kDefect], pf[kDefect], pb[kDefect],
                    pc[kDefect], bc[kDefect], ce[kDefect], cw[kDefect];
#pragma unroll
                for (int u = 0; u < kDefect; ++u) {
                    const int i = min(i0 + lane + 32 * u, g.nx);
                    const long long c = c0 + i;
                    ce[u] = scd.cE[i];
                    cw[u] = scd.cW[i];
                    pe[u] = __ldca(p + c + 1);
                    pw[u] = __ldca(p + c - 1);
                    pn[u] = nL1 ? __ldca(p + c + g.px) : __ldcg(p + c + g.px);
                    ps[u] = sL1 ? __ldca(p + c - g.px) : __ldcg(p + c - g.px);
                    pf[u] = fL1 ? __ldca(p + c + g.pz) : __ldcg(p + c + g.pz);
                    pb[u] = bL1 ? __ldca(p + c - g.pz) : __ldcg(p + c - g.pz);
                    pc[u] = __ldca(p + c);
                    bc[u] = __ldg(b + c);
                }
#pragma unroll
                for (int u = 0; u < kDefect; ++u) {
                    const int i = i0 + lane + 32 * u;
                    if (i > g.nx) continue;
                    const double sv = ce[u] * pe[u] + cw[u] * pw[u] + cN * pn[u] + cS * ps[u] + cF * pf[u] +
                                      cB * pb[u];
                    // rdiag_of's sum in its order
                    const double rd = rcp_rn(((ce[u] + cw[u]) + (cN + cS)) + (cF + cB));
                    const double dval = rd * sv - bc[u] - pc[u];
                    const int m = (i + 2) >> 1;
                    const bool red = ((i + j + k) & 1) == 0;
                    if (CD) (red ? D0 : D1)[dr + m] = (Tc)dval;
                    else (red ? dRg : dBg)[g0 + m] = (Tc)dval;
                }
            }
        }
    }
    // the next half-sweep reads d only of this CTA's own cells
    __syncthreads();
    ++restarts;
  }
    add_e_to_p();
    if (blockIdx.x == 0 && tid == 0) {
        ctl->ik = ik0 + done;
        ctl->inner = done_c;
        ctl->cycles += restarts + (itmax > 0 ? 1 : 0);   // the launch's cycles, the last included
        ctl->restarts += restarts;
        ctl->bodies += done;
        if (done > 0) ctl->last_change = last;
        if (conv) ctl->converged = 1;
        if (nonfinite) ctl->nonfinite = 1;
        if (failed) ctl->timeout = 1;
    }
}

}  // namespace ntcfd
