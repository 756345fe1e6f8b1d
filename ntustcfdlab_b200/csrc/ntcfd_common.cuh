// ntcfd_common.cuh -- device-side layout of the staggered grid.
//
// Natural layout (velocity, pressure, ETA, b, nu_t): the Fortran halo array
// (-1:nx+2, -1:ny+2, -1:nz+2), i fastest, with each i-row padded to a
// multiple of 8 elements and shifted so that i = 1 starts on a 64-byte
// boundary (double) / 32-byte boundary (float):
//     element (i,j,k) at  ioff + i + px*(j+1) + pz*(k+1),  ioff = 7,
// so that i = -1 sits at offset 6 and rows/planes start at j, k = -1.
//
// Colour-split layout (SOR correction e and defect d): red cells
// ((i+j+k) even) and black cells ((i+j+k) odd) are stored in two arrays so
// that a half-sweep reads and writes only whole sectors.  Cell (i,j,k) of
// colour c sits at compact index m = (i+2)/2 of its row:
//     element (m,j,k) at  m + mxp*(j+1) + mz*(k+1).
// For a cell of colour c in row (j,k) let r = ((j+k)^c)&1; then
// i + 2 = 2m + r, its west/east neighbours (other colour) are at m-1+r and
// m+r of the same row, and its j+-1 / k+-1 neighbours are at the same m.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ntcfd {

constexpr int kIoff = 7;

struct Geom {
    int nx, ny, nz;
    int px;           // natural row pitch (elements)
    int py;           // rows per plane = ny + 4
    long long pz;     // natural plane pitch = px * py
    int mxp;          // split row pitch
    long long mz;     // split plane pitch = mxp * py
    // 1-D metrics, pointers pre-offset so that a[i] is valid for i in -2..n+2
    const double *iDx, *Dxs, *iDy, *Dys, *iDz, *Dzs;
    // reciprocals of the metrics (same indexing)
    const double *riDx, *rDxs, *riDy, *rDys, *riDz, *rDzs;
    // SOR coefficients divided by the cell volume:
    //   cE(i) = 1/(iDx(i) Dxs(i)), cW(i) = 1/(iDx(i) Dxs(i-1)), likewise N/S, F/B
    const double *cE, *cW, *cN, *cS, *cF, *cB;
    const float *cEf, *cWf, *cNf, *cSf, *cFf, *cBf;
};

__host__ __device__ __forceinline__ long long nat(const Geom& g, int i, int j, int k) {
    return (long long)kIoff + i + (long long)g.px * (j + 1) + g.pz * (k + 1);
}
__host__ __device__ __forceinline__ long long spl(const Geom& g, int m, int j, int k) {
    return (long long)m + (long long)g.mxp * (j + 1) + g.mz * (k + 1);
}

// Control block of one context (device memory).
struct Ctl {
    unsigned long long slot;      // max |change| bits of the sweep being tested
    unsigned long long dslot;     // max |d| bits of the last defect pass
    int ik;                       // sweeps done in this step
    int step;                     // step index inside the current ntcfd_step call
    int converged;                // stop rule fired
    int nonfinite;                // NaN/Inf met in a change or defect
    int cycles;                   // defect-correction cycles in this step
    int inner;                    // sweeps done in the current cycle
    int bodies;                   // inner loop bodies run in this step
    int timeout;                  // a bounded device wait gave up
    int pad_stop, pad_more;       // the last loop decisions (read by the host in eager mode)
    int restarts;                 // correction cycles restarted inside the resident SOR kernel
    int halt;                     // a moving body's mask met a tie: the call's remaining steps do nothing
    int halt_ties;                // the ties of that mask
    int pad2;
    double last_change;           // value of the last tested sweep
    double cdrag, clift, divmax;
};

// Per-step record copied back to the host after ntcfd_step.
struct StepRec {
    int sor_iters, converged;
    double last_change, cdrag, clift, divmax;
    int cycles, nonfinite;
    int launches, timeout;
};

__device__ __forceinline__ unsigned long long dbits(double x) {
    return (unsigned long long)__double_as_longlong(x);
}

// Order-preserving bit patterns of |x|: for non-negative IEEE values the
// unsigned pattern orders like the value, and every NaN pattern lies above
// +Inf, so a max over patterns also detects non-finite values.
__device__ __forceinline__ unsigned long long abs_bits(double x) {
    return dbits(x) & 0x7fffffffffffffffULL;
}
__device__ __forceinline__ unsigned int abs_bits(float x) {
    return __float_as_uint(x) & 0x7fffffffu;
}
__device__ __forceinline__ unsigned long long widen_bits(unsigned long long b) { return b; }
__device__ __forceinline__ unsigned long long widen_bits(unsigned int b) {
    return dbits((double)__uint_as_float(b));   // float -> double keeps order, Inf and NaN
}

// Block-wide max of order-preserving patterns b (see abs_bits), then one
// atomicMax of the double pattern on *dst.  NT = threads per block;
// blockDim.x must be a multiple of 32.
template <int NT, class B>
__device__ __forceinline__ void block_max_bits(B b, unsigned long long* dst) {
    __shared__ B red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const B t = __shfl_xor_sync(0xffffffffu, b, o);
        b = t > b ? t : b;
    }
    const int lane = threadIdx.x & 31;
    const int warp = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
    if (lane == 0) red[warp] = b;
    __syncthreads();
    if (warp == 0) {
        b = (lane < NT / 32) ? red[lane] : B(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const B t = __shfl_xor_sync(0xffffffffu, b, o);
            b = t > b ? t : b;
        }
        if (lane == 0 && b != B(0)) atomicMax(dst, widen_bits(b));
    }
}

template <int NT, class T>
__device__ __forceinline__ void block_max_atomic(T v, unsigned long long* dst) {
    block_max_bits<NT>(abs_bits(v), dst);
}

// Per-sweep maxima are spread over kSpread slots (by block index) so that
// thousands of blocks do not serialise on one address.
constexpr int kSpread = 32;

constexpr unsigned long long kInfBits = 0x7ff0000000000000ULL;

}  // namespace ntcfd
