// k_resident.cuh -- a whole pressure solve (every defect-correction cycle)
// in one persistent cooperative kernel, with the correction e resident in
// shared memory.
//
// The interior rows (j,k) are split into nbj x nbk bricks of at most JB x KB
// rows; CTA b owns brick (b % nbj, b / nbj) and keeps e of both colours for
// its rows in shared memory (colour-split rows of mx entries, see
// ntcfd_common.cuh) with a one-row ring, and the defect d and 1/diag rd of its
// rows when they fit.  The ring rows of a domain boundary stay 0; the others
// hold the neighbour bricks' boundary rows, which every CTA publishes to the
// global e arrays as it updates them and copies into its ring ("fill") once
// per half-sweep.  A sweep runs
//     red:   [fill the black ring] -> interior rows -> edge rows -> arrive
//     black: interior rows (own red values only) -> wait -> fill the red ring
//            -> edge rows -> max |change| -> grid barrier,
// so the fill latency overlaps the red interior rows and the first barrier
// overlaps the black interior rows.  The sweep count, the stop rule
// (GS.f90:11,53), the count of correction cycles and the final p += e run
// inside the kernel, and so do the restarts of the defect correction: when a
// cycle ends on its length (cycle_len sweeps), the kernel refreshes the black
// ring, adds e to p and updates d to the FP64 defect of p + e
// (defect_update: d + rdiag sum c e_nb - e, in FP64, from the exact FP32
// values of e) without a grid barrier, then sweeps on from e = 0.  The first
// defect of the solve comes from k_defect.
//
// A lane updates two cells at a time with every load issued before any
// store: cells t and t + 32 of one row (rows of at most 64 cells per colour,
// or in 64-cell chunks for wider rows), or, in the NARROW instance (rows of
// at most 32 cells per colour), t of two rows.  The row's parity r is a
// template argument of the update, so the east/west neighbours and the second
// cell are immediate offsets of one address.  Loads always read inside the
// shared-memory allocation (or the padded global arrays); a lane past the
// row's last cell stores nothing and leaves the change maximum alone.
//
// The grid barrier spins with a bounded number of polls; a CTA that gives
// up sets bar->err, and every CTA leaves the sweep loop at the next barrier,
// so the kernel always ends.  The host reports NTCFD_ETIMEOUT.
#pragma once

#include <type_traits>

#include "k_gridbar.cuh"
#include "k_pressure.cuh"
#include "ntcfd_common.cuh"

namespace ntcfd {

// Row shapes of k_sor_resident (Brick::mode).
enum { kResNarrow = 0, kResWide1 = 1, kResWide = 2 };

struct Brick {
    int nbj, nbk;    // bricks along j and k
    int JB, KB;      // rows per brick (the last brick may hold fewer)
    int mx;          // colour-split row length (compact index m = 0..mx-1)
    int cache_d;     // 1: d of the brick lives in shared memory too
    int cache_rd;    // 1: rd of the brick lives in shared memory too
    int mode;        // kResNarrow, kResWide1 or kResWide (res_mode(nx))
};

// Cells of a colour in a row: (nx + r) / 2 for parity r; at most (nx + 1) / 2.
__host__ __device__ inline int res_mode(int nx) {
    const int most = (nx + 1) / 2;
    return most <= 32 ? kResNarrow : most <= 64 ? kResWide1 : kResWide;
}

// Dynamic shared memory of k_sor_resident for a brick plan.
template <class Tc>
inline size_t resident_smem(const Brick& b, int nx) {
    const size_t tile = (size_t)(b.JB + 2) * (b.KB + 2) * b.mx;
    const size_t brick = (size_t)b.JB * b.KB * b.mx;
    const size_t arrays = sizeof(Tc) * (2 * tile + 2 * (size_t)(nx + 4) + 2 * (size_t)(b.JB + b.KB) +
                                        (b.cache_d ? 2 * brick : 0) + (b.cache_rd ? 2 * brick : 0));
    // + row table (int4 offsets and four coefficients per row), + the face-ring list
    // (int2 per ring row), + slack: the loads of a lane past a row's last cell may
    // reach up to 64 elements beyond the tiles
    const size_t rows = (size_t)b.JB * b.KB;
    return ((arrays + 15) & ~size_t(15)) + rows * (16 + 4 * sizeof(Tc)) + 2 * (size_t)(b.JB + b.KB) * 8 +
           64 * sizeof(Tc);
}

// ring values a thread holds in flight while it updates interior rows (32 bytes)
template <class Tc>
constexpr int kFillOf = 32 / (int)sizeof(Tc);

constexpr unsigned int kNanFlag = 1u << 20;   // high-half flag of a CTA whose max |change| was not finite

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

// Everything one half-sweep needs to know about a row.
template <class Tc>
struct ResRow {
    const Tc* O;      // other colour, tile row start (shared)
    Tc* W;            // own colour, tile row start (shared)
    const Tc* D;      // d of the row: brick row start (shared) or global row start
    const Tc* R;      // rd of the row, likewise
    Tc cN, cS, cF, cB;
    int par;          // (j + k) & 1 of the row
    long long gr;     // global colour-split row start
};

// The loaded operands of one cell.
template <class Tc>
struct ResIn {
    Tc oE, oW, oN, oS, oF, oB, e0, d, rd;
};

// Loads of the cell at own index m (t + 2 - R) of a row of parity R, all from
// shared memory: the tile's face ring holds the neighbour bricks' rows of the
// other colour (fill_ring).  d may be rewritten inside the launch by this CTA
// only: a plain (L1-coherent) load when it is global.
template <class Tc, bool CD, bool CR, int R>
__device__ __forceinline__ ResIn<Tc> res_load(const ResRow<Tc>& w, int m, int mx, int plane) {
    ResIn<Tc> x;
    const Tc* o = w.O + m;
    x.oE = o[R];
    x.oW = o[R - 1];
    x.oN = o[mx];
    x.oS = o[-mx];
    x.oF = o[plane];
    x.oB = o[-plane];
    x.e0 = w.W[m];
    x.d = CD ? w.D[m] : __ldca(w.D + m);
    x.rd = CR ? w.R[m] : __ldg(w.R + m);
    return x;
}

// The update of a loaded cell; stores e (and publishes it for an EDGE row)
// and takes the change into the maximum only when ok.
template <class Tc, bool EDGE, class B>
__device__ __forceinline__ void res_finish(const ResIn<Tc>& x, const ResRow<Tc>& w, int m, Tc cE, Tc cW, Tc om,
                                           bool ok, Tc* Ec, B& ch) {
    Tc e1;
    const Tc diff = sor_update(cE, x.oE, cW, x.oW, w.cN, x.oN, w.cS, x.oS, w.cF, x.oF, w.cB, x.oB, x.rd, x.d,
                               x.e0, om, &e1);
    if (ok) {
        w.W[m] = e1;
        if (EDGE) Ec[w.gr + m] = e1;
        const B db = abs_bits(diff);
        ch = db > ch ? db : ch;
    }
}

template <class Tc, int NT, bool CD, bool CR, int MODE>
__global__ void __launch_bounds__(NT, 1)
k_sor_resident(Geom g, SorCoef<Tc> sc, Brick br, double* __restrict__ p, const double* __restrict__ b,
               Tc* __restrict__ eRg, Tc* __restrict__ eBg, Tc* __restrict__ dRg, Tc* __restrict__ dBg,
               const Tc* __restrict__ rdRg, const Tc* __restrict__ rdBg, Ctl* ctl, GridBar* bar,
               double omega, double zeta, int itmax, int cycle_len, int check_every,
               unsigned long long* ring) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using B = decltype(abs_bits(Tc(0)));
    constexpr int kFill = kFillOf<Tc>;
    __shared__ int s_flag;
    __shared__ unsigned int s_hi;
    __shared__ B s_red[NT / 32];
    const int JB = br.JB, KB = br.KB, mx = br.mx;
    const int RS = JB + 2;                    // rows per k-plane of the tile
    const int plane = RS * mx;
    const int tile = plane * (KB + 2);
    const int brick = JB * KB * mx;
    // shared memory: e red, e black (tile with halo), coefficients cE, cW (index
    // i+1, i = -1..nx+2), cN, cS of the brick's rows, cF, cB of its planes, then d
    // red/black and rd red/black of the brick when cached, then the row table
    Tc* const S0 = reinterpret_cast<Tc*>(smem_raw);
    Tc* const S1 = S0 + tile;
    Tc* const cEs = S1 + tile + 1;
    Tc* const cWs = cEs + (g.nx + 4);
    Tc* const cNs = cEs + 2 * (g.nx + 4) - 1;
    Tc* const cSs = cNs + JB;
    Tc* const cFs = cSs + JB;
    Tc* const cBs = cFs + KB;
    Tc* const D0 = cBs + KB;
    Tc* const D1 = D0 + brick;
    Tc* const R0 = CD ? D1 + brick : D0;
    Tc* const R1 = R0 + brick;
    Tc* const arrays_end = CR ? R1 + brick : (CD ? D1 + brick : D0);
    // row table: per row of the brick, in sweep order (edge rows first), the tile row
    // start, the brick row start of d/rd, the global colour-split row start and
    // (j+k)&1; and the row's cN, cS, cF, cB.  Then the face ring: per ring row of
    // the tile that stands for a row of a neighbour brick, its tile row start and
    // global colour-split row start (y = -1: a domain ghost row, kept at 0).
    const size_t toff = ((size_t)((unsigned char*)arrays_end - smem_raw) + 15) & ~size_t(15);
    int4* const rowT = reinterpret_cast<int4*>(smem_raw + toff);
    Tc* const rowC = reinterpret_cast<Tc*>(rowT + JB * KB);
    int2* const ringT = reinterpret_cast<int2*>(rowC + 4 * JB * KB);
    constexpr int NWARP = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tid = threadIdx.x;

    const int bj = blockIdx.x % br.nbj, bk = blockIdx.x / br.nbj;
    const int j0 = 1 + bj * JB, k0 = 1 + bk * KB;
    const int nj = max(0, min(g.ny, j0 + JB - 1) - j0 + 1);
    const int nk = max(0, min(g.nz, k0 + KB - 1) - k0 + 1);
    const int ys = g.mxp, zs = (int)g.mz;   // colour-split row and plane pitch
    // cells of a colour in a row of parity r
    const int nown0 = g.nx / 2, nown1 = (g.nx + 1) / 2;

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
    const int nrows = nj * nk;
    const int ni = (nj > 2 && nk > 2) ? (nj - 2) * (nk - 2) : 0;   // interior rows
    const int ne = nrows - ni;                                       // edge rows
    const int nring = 2 * (nj + nk);
    for (int q = tid; q < nring; q += NT) {
        // faces j-low, j-high (nk rows each), then k-low, k-high (nj rows each)
        int jl, kl;
        if (q < 2 * nk) {
            kl = q % nk + 1;
            jl = q < nk ? 0 : nj + 1;
        } else {
            const int r = q - 2 * nk;
            jl = r % nj + 1;
            kl = r < nj ? 0 : nk + 1;
        }
        const int j = j0 + jl - 1, k = k0 + kl - 1;
        const bool inner = j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
        ringT[q] = make_int2((kl * RS + jl) * mx, inner ? ys * (j + 1) + zs * (k + 1) : -1);
    }
    for (int er = tid; er < nrows; er += NT) {
        int jl, kl;
        brick_row(er, nj, nk, ni, ne, jl, kl);
        const int j = j0 + jl - 1, k = k0 + kl - 1;
        rowT[er] = make_int4((kl * RS + jl) * mx, ((kl - 1) * JB + (jl - 1)) * mx, ys * (j + 1) + zs * (k + 1),
                             (j + k) & 1);
        rowC[4 * er + 0] = sc.cN[j];
        rowC[4 * er + 1] = sc.cS[j];
        rowC[4 * er + 2] = sc.cF[k];
        rowC[4 * er + 3] = sc.cB[k];
    }
    if (CD || CR) {
        // d (the solve's first defect, from k_defect) and rd of the brick: one warp per
        // row, lanes along m
        for (int row = warp; row < nrows; row += NWARP) {
            const int jl = row % nj, kl = row / nj;
            const long long gq0 = spl(g, 0, j0 + jl, k0 + kl);
            const int sq0 = (kl * JB + jl) * mx;
            for (int m = lane; m < mx; m += 32) {
                if (CD) {
                    D0[sq0 + m] = dRg[gq0 + m];
                    D1[sq0 + m] = dBg[gq0 + m];
                }
                if (CR) {
                    R0[sq0 + m] = rdRg[gq0 + m];
                    R1[sq0 + m] = rdBg[gq0 + m];
                }
            }
        }
    }
    __syncthreads();
    // lane coefficients of the one- and two-row instances: the cells t = lane (and
    // t = lane + 32) of a row of parity r sit at i = 2t + 2 - r (past the row's end
    // they read other table entries, never used)
    Tc cEr[2][2], cWr[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * (lane + 32 * h) + 2 - r;
            cEr[r][h] = MODE == kResWide ? Tc(0) : cEs[min(i, g.nx + 2)];
            cWr[r][h] = MODE == kResWide ? Tc(0) : cWs[min(i, g.nx + 2)];
        }

    unsigned int nbar = 0;   // grid barriers of this launch passed so far
    unsigned int hi_prev = 0u;   // high half of the barrier word at the last closing barrier
    bool tested = false;         // a stop test ran in this launch
    const unsigned int nblocks = gridDim.x;
    const int ik0 = ctl->ik;
    const Tc om = (Tc)omega;
    int done = 0;        // sweeps of this launch
    int done_c = 0;      // sweeps of the current cycle
    int restarts = 0;
    bool conv = false, nonfinite = false, failed = false;
    double last = 0.0;

    // p += e over the brick (natural <- shared memory); one warp per pair of rows,
    // lanes along i, 8 values of p in flight per lane
    auto add_e_to_p = [&]() {
        constexpr int U = 4;
        for (int row = 2 * warp; row < nrows; row += 2 * NWARP) {
            for (int i0 = 1; i0 <= g.nx; i0 += 32 * U) {
                double pv[2][U];
                long long c0[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int rr = min(row + h, nrows - 1);
                    c0[h] = nat(g, 0, j0 + rr % nj, k0 + rr / nj);
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + lane + 32 * u;
                        if (i <= g.nx) pv[h][u] = p[c0[h] + i];
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (row + h >= nrows) continue;
                    const int jl = (row + h) % nj + 1, kl = (row + h) / nj + 1;
                    const int j = j0 + jl - 1, k = k0 + kl - 1;
                    const int sr = (kl * RS + jl) * mx;
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + lane + 32 * u;
                        if (i <= g.nx)
                            p[c0[h] + i] = pv[h][u] + (double)(((i + j + k) & 1) ? S1 : S0)[sr + ((i + 2) >> 1)];
                    }
                }
            }
        }
    };

    struct DefIn {
        Tc* D;          // d of the row: shared (CD) or global
        double* pr;     // natural row of p, i = 0
        int nown, mA, iA;
        Tc oEA, oWA, oNA, oSA, oFA, oBA, oEB, oWB, oNB, oSB, oFB, oBB, eA, eB, dA, dB;
        double cEA, cWA, cEB, cWB, cN, cS, cF, cB, pA, pB;
    };
    // every load of the cells t0 + lane and t0 + lane + 32 of task rc = 2 * row + colour
    auto def_load = [&](int rc, int t0) {
        DefIn x;
        const int row = rc >> 1, c = rc & 1;
        const int jl = row % nj + 1, kl = row / nj + 1;
        const int j = j0 + jl - 1, k = k0 + kl - 1;
        const int r = ((j + k) ^ c) & 1;
        x.nown = r ? nown1 : nown0;
        x.cN = g.cN[j]; x.cS = g.cS[j]; x.cF = g.cF[k]; x.cB = g.cB[k];
        const int sr = (kl * RS + jl) * mx, dr = ((kl - 1) * JB + (jl - 1)) * mx;
        const Tc* O = (c ? S0 : S1) + sr;         // the other colour's tile row
        const Tc* Wt = (c ? S1 : S0) + sr;        // this colour's
        x.D = CD ? (c ? D1 : D0) + dr : (c ? dBg : dRg) + spl(g, 0, j, k);
        x.pr = p + nat(g, 0, j, k);
        const int tA = t0 + lane;
        const int mA = tA + 2 - r, mB = mA + 32;
        x.mA = mA;
        x.iA = 2 * tA + 2 - r;
        const int iAc = min(x.iA, g.nx + 2), iBc = min(x.iA + 64, g.nx + 2);
        x.oEA = O[mA + r]; x.oWA = O[mA - 1 + r]; x.oNA = O[mx + mA]; x.oSA = O[mA - mx];
        x.oFA = O[plane + mA]; x.oBA = O[mA - plane];
        x.oEB = O[mB + r]; x.oWB = O[mB - 1 + r]; x.oNB = O[mx + mB]; x.oSB = O[mB - mx];
        x.oFB = O[plane + mB]; x.oBB = O[mB - plane];
        x.eA = Wt[mA]; x.eB = Wt[mB];
        x.dA = x.D[mA]; x.dB = x.D[mB];
        x.cEA = g.cE[iAc]; x.cWA = g.cW[iAc]; x.cEB = g.cE[iBc]; x.cWB = g.cW[iBc];
        x.pA = x.pr[x.iA]; x.pB = x.pr[x.iA + 64];
        return x;
    };
    auto def_finish = [&](const DefIn& x, int t0) {
        const double dnA = defect_update(x.cEA, x.oEA, x.cWA, x.oWA, x.cN, x.oNA, x.cS, x.oSA, x.cF, x.oFA, x.cB,
                                         x.oBA, x.dA, x.eA);
        const double dnB = defect_update(x.cEB, x.oEB, x.cWB, x.oWB, x.cN, x.oNB, x.cS, x.oSB, x.cF, x.oFB, x.cB,
                                         x.oBB, x.dB, x.eB);
        const int tA = t0 + lane;
        if (tA < x.nown) {
            x.D[x.mA] = (Tc)dnA;
            x.pr[x.iA] = x.pA + (double)x.eA;
        }
        if (tA + 32 < x.nown) {
            x.D[x.mA + 32] = (Tc)dnB;
            x.pr[x.iA + 64] = x.pB + (double)x.eB;
        }
    };
    // Restart of a correction cycle: d of every cell of the brick becomes the FP64
    // defect of p + e (defect_update), from the tiles (both rings current), and the
    // cycle's e goes to p in the same pass (add_e_to_p takes only the last cycle's);
    // a warp per row and colour ("task"), lane t takes the cells t and t + 32 of
    // each 64-cell chunk (consecutive m: each shared-memory load of the warp reads
    // one tile without bank conflicts).  FP32 rows of 33-64 cells per colour (the
    // kResWide1 instance) go two tasks at a time, every load of both (p from L2
    // among them) issued before the FP64 arithmetic of either.  A lane past the row's last cell reads inside the
    // shared allocation, the padded d arrays and the natural p array (ghost rows
    // and planes follow the brick's) and stores nothing.
    auto update_defect = [&]() {
        // (FP64, whose restarts are rare, and the other row shapes keep one task at a
        // time: the pair makes those instances spill)
        if (sizeof(Tc) == 4 && MODE == kResWide1) {
            for (int rc = warp; rc < 2 * nrows; rc += 2 * NWARP) {
                const bool two = rc + NWARP < 2 * nrows;
                const DefIn xa = def_load(rc, 0);
                const DefIn xb = def_load(two ? rc + NWARP : rc, 0);
                def_finish(xa, 0);
                if (two) def_finish(xb, 0);
            }
        } else {
            for (int rc = warp; rc < 2 * nrows; rc += NWARP) {
                const int row = rc >> 1;
                const int r = ((j0 + row % nj + k0 + row / nj) ^ (rc & 1)) & 1;
                const int nown = r ? nown1 : nown0;
                for (int t0 = 0; t0 < nown; t0 += 64) {
                    const DefIn xa = def_load(rc, t0);
                    def_finish(xa, t0);
                }
            }
        }
    };
    auto zero_tile = [&]() {
        for (int q = tid; q < 2 * tile; q += NT) S0[q] = Tc(0);
    };


    // ---- the face ring of the other colour's tile from the neighbour bricks' rows,
    // published before the last grid barrier: loads through L2 only (the rows change
    // between half-sweeps, and this SM's L1 may hold an older copy).  fill_issue puts
    // the first kFill per thread in flight into registers; fill_commit stores them,
    // moves any further ones and ends with a CTA barrier.  For the red half the ring
    // is the black one (c = 0), for the black half the red one.
    const unsigned int mMX = 0xffffffffu / (unsigned)mx + 1u;   // q / mx, exact for q * mx < 2^32 (mx >= 3)
    const int ring_tot = nring * mx;
    auto fill_issue = [&](int c, Tc (&v)[kFill]) {
        const Tc* const Og = c ? eRg : eBg;
#pragma unroll
        for (int u = 0; u < kFill; ++u) {
            const int q = min(tid + NT * u, ring_tot - 1);
            const unsigned int r = __umulhi((unsigned)q, mMX);
            const int2 rr = ringT[r];
            v[u] = __ldcg(Og + max(rr.y, 0) + (q - (int)r * mx));
        }
    };
    auto fill_commit = [&](int c, const Tc (&v)[kFill]) {
        Tc* const O = c ? S0 : S1;
        const Tc* const Og = c ? eRg : eBg;
#pragma unroll
        for (int u = 0; u < kFill; ++u) {
            const int q = tid + NT * u;
            if (q >= ring_tot) continue;
            const unsigned int r = __umulhi((unsigned)q, mMX);
            const int2 rr = ringT[r];
            if (rr.y >= 0) O[rr.x + (q - (int)r * mx)] = v[u];
        }
        for (int q0 = NT * kFill; q0 < ring_tot; q0 += NT * kFill) {
            Tc w[kFill];
            int dst[kFill];
#pragma unroll
            for (int u = 0; u < kFill; ++u) {
                const int q = min(q0 + tid + NT * u, ring_tot - 1);
                const unsigned int r = __umulhi((unsigned)q, mMX);
                const int m = q - (int)r * mx;
                const int2 rr = ringT[r];
                dst[u] = rr.y >= 0 && q0 + tid + NT * u < ring_tot ? rr.x + m : -1;
                w[u] = __ldcg(Og + max(rr.y, 0) + m);
            }
#pragma unroll
            for (int u = 0; u < kFill; ++u)
                if (dst[u] >= 0) O[dst[u]] = w[u];
        }
        __syncthreads();
    };

    // ---- one half-sweep of colour c over rows [e0r, e1r) (edge rows: EDGE)
    auto rows_pass = [&](auto edge_tag, int c, int e0r, int e1r, B& ch) {
        constexpr bool EDGE = decltype(edge_tag)::value;
        Tc* const W = c ? S1 : S0;
        const Tc* const O = c ? S0 : S1;
        Tc* const Ec = c ? eBg : eRg;
        const Tc* const Dg = c ? dBg : dRg;
        const Tc* const Rg = c ? rdBg : rdRg;
        const Tc* const Ds = c ? D1 : D0;
        const Tc* const Rs = c ? R1 : R0;
        auto row_of = [&](int er) {
            const int4 rt = rowT[er];
            ResRow<Tc> w;
            w.O = O + rt.x;
            w.W = W + rt.x;
            w.D = CD ? Ds + rt.y : Dg + rt.z;
            w.R = CR ? Rs + rt.y : Rg + rt.z;
            w.cN = rowC[4 * er];
            w.cS = rowC[4 * er + 1];
            w.cF = rowC[4 * er + 2];
            w.cB = rowC[4 * er + 3];
            w.par = rt.w;
            w.gr = rt.z;
            return w;
        };
        using I0 = std::integral_constant<int, 0>;
        using I1 = std::integral_constant<int, 1>;
        if constexpr (MODE == kResNarrow) {
            // two rows per warp, lane t in each
            for (int er = e0r + 2 * warp; er < e1r; er += 2 * NWARP) {
                const bool twoRows = er + 1 < e1r;
                const ResRow<Tc> wA = row_of(er), wB = row_of(twoRows ? er + 1 : er);
                const int rA = (wA.par ^ c) & 1, rB = (wB.par ^ c) & 1;
                const bool okA = lane < (rA ? nown1 : nown0);
                const bool okB = twoRows && lane < (rB ? nown1 : nown0);
                auto two = [&](auto ra, auto rb) {
                    constexpr int RA = decltype(ra)::value, RB = decltype(rb)::value;
                    const int mA = lane + 2 - RA, mB = lane + 2 - RB;
                    const ResIn<Tc> xA = res_load<Tc, CD, CR, RA>(wA, mA, mx, plane);
                    const ResIn<Tc> xB = res_load<Tc, CD, CR, RB>(wB, mB, mx, plane);
                    res_finish<Tc, EDGE>(xA, wA, mA, cEr[RA][0], cWr[RA][0], om, okA, Ec, ch);
                    res_finish<Tc, EDGE>(xB, wB, mB, cEr[RB][0], cWr[RB][0], om, okB, Ec, ch);
                };
                if (rA == 0) {
                    if (rB == 0) two(I0{}, I0{});
                    else two(I0{}, I1{});
                } else {
                    if (rB == 0) two(I1{}, I0{});
                    else two(I1{}, I1{});
                }
            }
        } else {
            for (int er = e0r + warp; er < e1r; er += NWARP) {
                const ResRow<Tc> w = row_of(er);
                const int r = (w.par ^ c) & 1;
                const int nown = r ? nown1 : nown0;
                auto one = [&](auto rr) {
                    constexpr int R = decltype(rr)::value;
                    if constexpr (MODE == kResWide1) {
                        // cells t = lane (always in the row: it holds more than 32) and lane + 32
                        const int mA = lane + 2 - R;
                        const ResIn<Tc> xA = res_load<Tc, CD, CR, R>(w, mA, mx, plane);
                        const ResIn<Tc> xB = res_load<Tc, CD, CR, R>(w, mA + 32, mx, plane);
                        res_finish<Tc, EDGE>(xA, w, mA, cEr[R][0], cWr[R][0], om, true, Ec, ch);
                        res_finish<Tc, EDGE>(xB, w, mA + 32, cEr[R][1], cWr[R][1], om, lane + 32 < nown, Ec, ch);
                    } else {
                        for (int t0 = 0; t0 < nown; t0 += 64) {
                            const int tA = t0 + lane;
                            const int mA = tA + 2 - R;
                            const ResIn<Tc> xA = res_load<Tc, CD, CR, R>(w, mA, mx, plane);
                            const ResIn<Tc> xB = res_load<Tc, CD, CR, R>(w, mA + 32, mx, plane);
                            const int iA = min(2 * tA + 2 - R, g.nx + 2), iB = min(iA + 64, g.nx + 2);
                            const Tc eA = cEs[iA], wA = cWs[iA], eB = cEs[iB], wB = cWs[iB];
                            res_finish<Tc, EDGE>(xA, w, mA, eA, wA, om, tA < nown, Ec, ch);
                            res_finish<Tc, EDGE>(xB, w, mA + 32, eB, wB, om, tA + 32 < nown, Ec, ch);
                        }
                    }
                };
                if (r == 0) one(I0{});
                else one(I1{});
            }
        }
    };
    using EdgeT = std::integral_constant<bool, true>;
    using InnerT = std::integral_constant<bool, false>;

  for (;;) {
    if (failed) break;
    done_c = 0;
    for (int s = 0; ik0 + done + s < itmax && s < cycle_len; ++s) {
        const int sg = done + s;   // sweep of this launch: ring slot
        if (blockIdx.x == 0 && tid == 0) ring[(sg + 1) % 3] = 0ULL;
        B ch = B(0);
        Tc fv[kFill];
        // red half: the black ring in flight (it is 0 in a cycle's first sweep), the
        // interior rows, the ring, the edge rows (published), arrive
        if (s > 0) fill_issue(0, fv);
        rows_pass(InnerT{}, 0, ne, nrows, ch);
        if (s > 0) fill_commit(0, fv);
        rows_pass(EdgeT{}, 0, 0, ne, ch);
        grid_arrive(bar, nbar);
        // black half: the interior rows (they read only this brick's red values) while
        // the barrier completes, wait, the red ring, the edge rows (published), then this
        // CTA's max |change| over the sweep into the ring slot of sweep sg and a full
        // barrier, so that every CTA's max is in the ring before anyone reads it
        rows_pass(InnerT{}, 1, ne, nrows, ch);
        if (!grid_wait(bar, nbar, nblocks, &s_flag)) {
            failed = true;
            break;
        }
        fill_issue(1, fv);
        fill_commit(1, fv);
        rows_pass(EdgeT{}, 1, 0, ne, ch);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const B t2 = __shfl_xor_sync(0xffffffffu, ch, o);
            ch = t2 > ch ? t2 : ch;
        }
        if (lane == 0) s_red[warp] = ch;
        __syncthreads();
        // the CTA's max: whether it is above zeta (or not finite) rides on this CTA's
        // arrival at the closing barrier; the value itself goes to the ring slot of
        // the sweep after the arrival, off the critical path (the solve's last one is
        // read after a final barrier)
        unsigned long long mybits = 0ull;
        unsigned int flags = 0u;
        if (tid == 0) {
            B b2 = B(0);
            for (int q = 0; q < NWARP; ++q) b2 = s_red[q] > b2 ? s_red[q] : b2;
            mybits = widen_bits(b2);
            flags = (mybits >= kInfBits ? kNanFlag : 0u) |
                    ((__longlong_as_double((long long)mybits) > zeta || mybits >= kInfBits) ? 1u : 0u);
        }
        grid_arrive(bar, nbar, flags);
        if (tid == 0 && mybits != 0ull) atomicMax(&ring[sg % 3], mybits);
        if (!grid_wait(bar, nbar, nblocks, &s_flag, &s_hi)) {
            failed = true;
            break;
        }
        const unsigned int over = s_hi - hi_prev;   // CTAs above zeta, + kNanFlag per non-finite one
        hi_prev = s_hi;
        done_c = s + 1;
        const int ik = ik0 + done + done_c;
        if (ik % check_every == 0 || ik >= itmax) {
            nonfinite = over >= kNanFlag;
            conv = over == 0u;
            tested = true;
            if (conv || nonfinite) break;
        }
    }
    done += done_c;
    // another cycle only when this one ended on its length
    if (failed || conv || nonfinite || done_c < cycle_len || ik0 + done >= itmax) break;
    // restart: the black ring again (the neighbours' final black rows; the red one is
    // current), d = the FP64 defect of p + e and p += e in one pass, e = 0.  No grid barrier: the
    // next cycle's first red half reads a zero black ring, and its black half reads
    // red rows published after the next barrier.
    {
        Tc fv[kFill];
        fill_issue(0, fv);
        fill_commit(0, fv);
    }
    update_defect();
    __syncthreads();
    zero_tile();
    __syncthreads();
    ++restarts;
  }
    add_e_to_p();
    // the max |change| of the last (tested) sweep, whose slot every CTA has reached
    // through the release of a later arrival
    if (!failed && tested && done > 0 && grid_sync(bar, nbar, nblocks, &s_flag) && tid == 0)
        last = __longlong_as_double((long long)*(const volatile unsigned long long*)&ring[(done - 1) % 3]);
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
