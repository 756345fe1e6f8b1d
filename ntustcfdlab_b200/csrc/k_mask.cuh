// k_mask.cuh -- K7 immersed-boundary volume fraction ETA.
//
// K7 follows RayCasting (airfoil.f90:580-915): even-odd ray crossings per
// (k,j) cell centre against the polygon edges (ray towards +z), then 50x50
// sub-cells on the cells that hold a polygon vertex, then extrusion along
// i.  The reference moves the grid by 0.01 when a vertex ties exactly with
// a node coordinate (airfoil.f90:700-702,731-733,804-807,834-837); the
// device kernels count such ties instead and the host rejects the mask.
// K7b follows DFIB_Cylinder (DFIB.f90:74-145) in real*4 arithmetic.
#pragma once

#include "ntcfd_common.cuh"

namespace ntcfd {

// ETA_1 from the crossing parity (airfoil.f90:685-764).
// Y, Z: node coordinates pre-offset (Y[j] valid for j in -1..n+3).
__global__ void k_ray_main(int ny, int nz, const double* Y, const double* Z, const double* az,
                           const double* ay, int poly, double* eta1, int* ties) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > nz || j > ny) return;
    const double Yj = Y[j], Zk = Z[k];
    const double ycell = (Y[j] + Y[j + 1]) / 2.0;
    const double zcell = (Z[k] + Z[k + 1]) / 2.0;
    int cnt = 0, tie = 0;
    for (int m = 0; m < poly - 1; ++m) {
        const double a0 = ay[m], a1 = ay[m + 1], z0 = az[m], z1 = az[m + 1];
        if (a0 >= ycell && a1 <= ycell) {
            if (zcell >= fmax(z0, z1)) {
            } else if (zcell < fmin(z0, z1)) {
                ++cnt;
            } else {
                if (Yj == a1 || Zk == z1) ++tie;
                const double m_pa = (Yj - a1) / (Zk - z1);
                const double m_ab = (a0 - a1) / (z0 - z1);
                if (m_pa > m_ab) ++cnt;
            }
        }
        if (a0 <= ycell && a1 >= ycell) {
            if (zcell >= fmax(z0, z1)) {
            } else if (zcell < fmin(z0, z1)) {
                ++cnt;
            } else {
                if (Yj == a0 || Zk == z0) ++tie;
                const double m_pa = (Yj - a0) / (Zk - z0);
                const double m_ab = (a1 - a0) / (z1 - z0);
                if (m_pa > m_ab) ++cnt;
            }
        }
    }
    eta1[(long long)(k - 1) + (long long)nz * (j - 1)] = (cnt % 2 == 0) ? 0.0 : 1.0;
    if (tie) atomicAdd(ties, tie);
}

// points(k,j) = 1 when a polygon vertex lies in [Z(k),Z(k+1)) x [Y(j),Y(j+1))
// for k in C..E-1, j in A..B-1 (airfoil.f90:661-674).
__global__ void k_ray_points(int ny, int nz, const double* Y, const double* Z, const double* az,
                             const double* ay, int poly, int A, int B, int C, int E, int* points) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= poly) return;
    for (int k = C; k <= E - 1; ++k) {
        if (!(az[m] >= Z[k] && az[m] < Z[k + 1])) continue;
        for (int j = A; j <= B - 1; ++j)
            if (ay[m] >= Y[j] && ay[m] < Y[j + 1] && k >= 1 && k <= nz && j >= 1 && j <= ny)
                points[(long long)(k - 1) + (long long)nz * (j - 1)] = 1;
    }
}

// Sub-grid volume fraction of cut cells (airfoil.f90:773-884): one block per
// listed cell, one thread per group of sub-cells, ETA_1 = odd sub-cells / 2500.
constexpr int kSub = 50;
template <int NT>
__global__ void __launch_bounds__(NT) k_ray_sub(int nz, const double* Y, const double* Z,
                                                const double* az, const double* ay, int poly,
                                                const int* cells, double* eta1, int* ties) {
    const int cell = cells[blockIdx.x];
    const int k = cell % nz + 1, j = cell / nz + 1;
    const double Yj = Y[j], Yj1 = Y[j + 1], Zk = Z[k], Zk1 = Z[k + 1];
    int odd = 0, tie = 0;
    for (int s = threadIdx.x; s < kSub * kSub; s += NT) {
        const int n = s % kSub + 1, l = s / kSub + 1;   // sub_intersection(n,l)
        const double YYl = Yj + (l - 1) * (Yj1 - Yj) / (double)kSub;
        const double YYl1 = Yj + (l) * (Yj1 - Yj) / (double)kSub;
        const double ZZn = Zk + (n - 1) * (Zk1 - Zk) / (double)kSub;
        const double ZZn1 = Zk + (n) * (Zk1 - Zk) / (double)kSub;
        const double ycell = (YYl + YYl1) / 2.0;
        const double zcell = (ZZn + ZZn1) / 2.0;
        int cnt = 0;
        for (int m = 0; m < poly - 1; ++m) {
            const double a0 = ay[m], a1 = ay[m + 1], z0 = az[m], z1 = az[m + 1];
            if (a0 >= ycell && a1 <= ycell) {
                if (zcell > fmax(z0, z1)) {
                } else if (zcell < fmin(z0, z1)) {
                    ++cnt;
                } else {
                    if (YYl == a1 || ZZn == z1) ++tie;
                    const double m_pa = (YYl - a1) / (ZZn - z1);
                    const double m_ab = (a0 - a1) / (z0 - z1);
                    if (m_pa > m_ab) ++cnt;
                }
            }
            if (a0 <= ycell && a1 >= ycell) {
                if (zcell > fmax(z0, z1)) {
                } else if (zcell < fmin(z0, z1)) {
                    ++cnt;
                } else {
                    if (YYl == a1 || ZZn == z1) ++tie;
                    const double m_pa = (YYl - a0) / (ZZn - z0);
                    const double m_ab = (a1 - a0) / (z1 - z0);
                    if (m_pa > m_ab) ++cnt;
                }
            }
        }
        odd += (cnt % 2 != 0) ? 1 : 0;
    }
    __shared__ int red[NT];
    red[threadIdx.x] = odd;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double total = (double)red[0];
        eta1[(long long)(k - 1) + (long long)nz * (j - 1)] = total / (double)kSub / (double)kSub;
    }
    if (tie) atomicAdd(ties, tie);
}

// ETA(i,j,k) = ETA_1(k,j) on the interior (airfoil.f90:889-891); ghosts 0.
__global__ void k_extrude(Geom g, const double* eta1, double* eta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z - 1;
    if (i > g.nx + 2 || j > g.ny + 2 || k > g.nz + 2) return;
    const bool in = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
    eta[nat(g, i, j, k)] = in ? eta1[(long long)(k - 1) + (long long)g.nz * (j - 1)] : 0.0;
}

// DFIB_Cylinder (DFIB.f90:90-131): axis along x, centre (zc, yc), radius r.
// DISTANCE, DIAGONAL, SZ, SY, xi are real*4 as declared in DFIB.f90:78-85.
__global__ void k_cylinder(int ny, int nz, const double* Y, const double* Z, const double* iDx,
                           const double* iDy, const double* iDz, double zc, double yc, double r,
                           double* eta1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > nz || j > ny) return;
    const int i = 1;
    // explicit _rn products and sums: no contraction into FMA, as in the
    // reference's separately rounded operations
    const float DIAGONAL = __double2float_rn(
        sqrt(__dadd_rn(__dadd_rn(__dmul_rn(iDx[i], iDx[i]), __dmul_rn(iDy[j], iDy[j])),
                       __dmul_rn(iDz[k], iDz[k]))) / 2.0);
    const double dzc = ((Z[k] + Z[k + 1]) / 2.0) - zc;
    const double dyc = ((Y[j] + Y[j + 1]) / 2.0) - yc;
    const float DISTANCE = __double2float_rn(sqrt(__dadd_rn(__dmul_rn(dzc, dzc), __dmul_rn(dyc, dyc))));
    double eta;
    if (fabs((double)DISTANCE - r) < (double)DIAGONAL) {
        float xi = 0.0f;
        const float dzg = __double2float_rn(iDz[k] / kSub);
        const float dyg = __double2float_rn(iDy[j] / kSub);
        for (int m = 1; m <= kSub; ++m) {
            const float SYm = __double2float_rn(Y[j] + (double)__fmul_rn((float)(m - 1), dyg));
            const float SYm1 = __double2float_rn(Y[j] + (double)__fmul_rn((float)(m), dyg));
            const double sy = (double)__fadd_rn(SYm, SYm1) / 2.0 - yc;
            for (int n = 1; n <= kSub; ++n) {
                const float SZn = __double2float_rn(Z[k] + (double)__fmul_rn((float)(n - 1), dzg));
                const float SZn1 = __double2float_rn(Z[k] + (double)__fmul_rn((float)(n), dzg));
                const double sz = (double)__fadd_rn(SZn, SZn1) / 2.0 - zc;
                const float SDIST = __double2float_rn(sqrt(__dadd_rn(__dmul_rn(sz, sz), __dmul_rn(sy, sy))));
                if ((double)SDIST <= r) xi = __fadd_rn(xi, 1.0f);
            }
        }
        eta = (double)__fdiv_rn(xi, (float)(kSub * kSub));
    } else if ((double)DISTANCE > r) {
        eta = 0.0;
    } else {
        eta = 1.0;
    }
    eta1[(long long)(k - 1) + (long long)nz * (j - 1)] = eta;
}

}  // namespace ntcfd
