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

// ETA_1 from the crossing parity (airfoil.f90:685-764) of cell (k,j).
// Y, Z: node coordinates pre-offset (Y[j] valid for j in -1..n+3).
__device__ __forceinline__ void ray_main_cell(int k, int j, int nz, const double* Y, const double* Z,
                                              const double* az, const double* ay, int poly, double* eta1,
                                              int* ties) {
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

__global__ void k_ray_main(int ny, int nz, const double* Y, const double* Z, const double* az,
                           const double* ay, int poly, double* eta1, int* ties) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > nz || j > ny) return;
    ray_main_cell(k, j, nz, Y, Z, az, ay, poly, eta1, ties);
}

// points(k,j) = 1 when a polygon vertex lies in [Z(k),Z(k+1)) x [Y(j),Y(j+1))
// for k in C..E-1, j in A..B-1 (airfoil.f90:661-674).
__device__ __forceinline__ void ray_point(int m, int ny, int nz, const double* Y, const double* Z,
                                          const double* az, const double* ay, int A, int B, int C, int E,
                                          int* points) {
    for (int k = C; k <= E - 1; ++k) {
        if (!(az[m] >= Z[k] && az[m] < Z[k + 1])) continue;
        for (int j = A; j <= B - 1; ++j)
            if (ay[m] >= Y[j] && ay[m] < Y[j + 1] && k >= 1 && k <= nz && j >= 1 && j <= ny)
                points[(long long)(k - 1) + (long long)nz * (j - 1)] = 1;
    }
}

__global__ void k_ray_points(int ny, int nz, const double* Y, const double* Z, const double* az,
                             const double* ay, int poly, int A, int B, int C, int E, int* points) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= poly) return;
    ray_point(m, ny, nz, Y, Z, az, ay, A, B, C, E, points);
}

// Sub-grid volume fraction of cut cell `cell` (airfoil.f90:773-884): the
// block's threads share the 50 x 50 sub-cells, ETA_1 = odd sub-cells / 2500.
constexpr int kSub = 50;
template <int NT>
__device__ __forceinline__ void ray_sub_cell(int cell, int nz, const double* Y, const double* Z, const double* az,
                                             const double* ay, int poly, double* eta1, int* ties, int* red) {
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
    __syncthreads();   // red is reused by the block's next cell
    if (tie) atomicAdd(ties, tie);
}

// One block per listed cell.
template <int NT>
__global__ void __launch_bounds__(NT) k_ray_sub(int nz, const double* Y, const double* Z,
                                                const double* az, const double* ay, int poly,
                                                const int* cells, double* eta1, int* ties) {
    __shared__ int red[NT];
    ray_sub_cell<NT>(cells[blockIdx.x], nz, Y, Z, az, ay, poly, eta1, ties, red);
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

// ---- A smoothed, differentiable mask (no counterpart in the reference): the
// polygon moved as the ray cast moves it, ETA_1 a C1 ramp of the signed
// distance d from the (y,z) cell centre to the polygon (negative inside):
//     tau = -d / width,  ETA_1 = 1 (tau >= 1), 0 (tau <= -1),
//     0.5 + 0.75 tau - 0.25 tau^3 between,
// and dETA_1/dalpha from the vertices' derivatives (dpz, dpy) with respect to
// the angle: d is the distance to the nearest point Q = A + t (B - A) of the
// nearest edge, so dd/dalpha = -s n.((1 - t) dA + t dB), n the unit vector
// from Q to the centre, s = -1 inside.  Inside/outside by crossing parity.
__global__ void k_smooth_mask(int ny, int nz, const double* Y, const double* Z, const double* pz,
                              const double* py, const double* dpz, const double* dpy, int npts, double width,
                              double* eta1, double* deta1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > nz || j > ny) return;
    const double yc = (Y[j] + Y[j + 1]) / 2.0, zc = (Z[k] + Z[k + 1]) / 2.0;
    double best = INFINITY, bt = 0.0;
    int bm = 0;
    bool inside = false;
    for (int m = 0; m < npts - 1; ++m) {
        const double az = pz[m], ay = py[m], bz = pz[m + 1], by = py[m + 1];
        const double abz = bz - az, aby = by - ay, apz = zc - az, apy = yc - ay;
        const double l2 = abz * abz + aby * aby;
        const double t = l2 > 0.0 ? fmin(fmax((apz * abz + apy * aby) / l2, 0.0), 1.0) : 0.0;
        const double qz = zc - (az + t * abz), qy = yc - (ay + t * aby);
        const double d2 = qz * qz + qy * qy;
        if (d2 < best) { best = d2; bt = t; bm = m; }
        if ((ay > yc) != (by > yc)) {
            const double zi = az + (yc - ay) * abz / aby;
            if (zc < zi) inside = !inside;
        }
    }
    const double du = sqrt(best), sgn = inside ? -1.0 : 1.0;
    const double tau = -sgn * du / width;
    double e, de = 0.0;
    if (tau >= 1.0) e = 1.0;
    else if (tau <= -1.0) e = 0.0;
    else {
        e = 0.5 + 0.75 * tau - 0.25 * tau * tau * tau;
        if (du > 0.0) {
            const double az = pz[bm], ay = py[bm];
            const double qz = az + bt * (pz[bm + 1] - az), qy = ay + bt * (py[bm + 1] - ay);
            const double nz_ = (zc - qz) / du, ny_ = (yc - qy) / du;
            const double dqz = (1.0 - bt) * dpz[bm] + bt * dpz[bm + 1];
            const double dqy = (1.0 - bt) * dpy[bm] + bt * dpy[bm + 1];
            const double ddu = -(nz_ * dqz + ny_ * dqy);
            de = 0.75 * (1.0 - tau * tau) * (-sgn * ddu / width);
        }
    }
    const long long q = (long long)(k - 1) + (long long)nz * (j - 1);
    eta1[q] = e;
    deta1[q] = de;
}

// ---- The mask of a moving body on the device, one step at a time inside the
// step graph (ntcfd_set_dynamic_aoa).  The host evaluates each step's angle
// (airfoil.f90:313-317) and its cosine and sine; k_dyn_rotate turns the body
// polygon by them (airfoil.f90:597-611) for the step the control block's step
// counter names.  After a step whose polygon meets an exact vertex/grid tie (the
// reference moves the grid instead) the control block's halt flag is set: the
// mask kernels and, through the graph's IF node, the step itself do nothing
// for the rest of the call.
struct DynMask {
    const double* base;   // body polygon: az[npts], then ay[npts]
    const double* trig;   // cos, sin of each step of the call
    double* poly;         // this step's polygon: az, then ay
    int npts;
    double zc, yc;
    int* flags;           // ny*nz: cells that hold a vertex (k fastest)
    int* list;            // ny*nz: those cells, compacted
    int* meta;            // A, B, C, E (airfoil.f90:615-654), listed cells, ties
    double* eta1;         // ETA_1(k,j)
};

// The step's polygon and its bounds A, B, C, E (airfoil.f90:615-654: A = the
// first j with Y(j) > min ay, less one, 0 when there is none; B = the first j
// with Y(j) > max ay; C, E likewise in z); the counters cleared.  One block.
// The rotation keeps the reference's order of operations (the new az enters
// the new ay) with every product and sum rounded on its own, as on the host.
template <int NT>
__global__ void __launch_bounds__(NT) k_dyn_rotate(int ny, int nz, const double* Y, const double* Z, DynMask m,
                                                   const Ctl* ctl) {
    if (ctl->halt) return;
    __shared__ double sd[4][NT];
    __shared__ int si[4][NT];
    const double c = m.trig[2 * ctl->step], sn = m.trig[2 * ctl->step + 1];
    const int t = threadIdx.x;
    double mny = INFINITY, mxy = -INFINITY, mnz = INFINITY, mxz = -INFINITY;
    for (int q = t; q < m.npts; q += NT) {
        const double z0 = __dsub_rn(m.base[q], 0.25), y0 = m.base[m.npts + q];
        const double z1 = __dsub_rn(__dmul_rn(c, z0), __dmul_rn(sn, y0));
        const double y1 = __dadd_rn(__dmul_rn(sn, z1), __dmul_rn(c, y0));
        const double az = __dadd_rn(__dadd_rn(z1, m.zc), 0.25), ay = __dadd_rn(y1, m.yc);
        m.poly[q] = az;
        m.poly[m.npts + q] = ay;
        mny = fmin(mny, ay); mxy = fmax(mxy, ay);
        mnz = fmin(mnz, az); mxz = fmax(mxz, az);
    }
    sd[0][t] = mny; sd[1][t] = mxy; sd[2][t] = mnz; sd[3][t] = mxz;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (t < s) {
            sd[0][t] = fmin(sd[0][t], sd[0][t + s]); sd[1][t] = fmax(sd[1][t], sd[1][t + s]);
            sd[2][t] = fmin(sd[2][t], sd[2][t + s]); sd[3][t] = fmax(sd[3][t], sd[3][t + s]);
        }
        __syncthreads();
    }
    mny = sd[0][0]; mxy = sd[1][0]; mnz = sd[2][0]; mxz = sd[3][0];
    const int none = 0x7fffffff;
    int fa = none, fb = none, fc = none, fe = none;
    for (int j = t + 1; j <= ny; j += NT) {
        if (Y[j] > mny) fa = min(fa, j);
        if (Y[j] > mxy) fb = min(fb, j);
    }
    for (int k = t + 1; k <= nz; k += NT) {
        if (Z[k] > mnz) fc = min(fc, k);
        if (Z[k] > mxz) fe = min(fe, k);
    }
    si[0][t] = fa; si[1][t] = fb; si[2][t] = fc; si[3][t] = fe;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (t < s)
            for (int q = 0; q < 4; ++q) si[q][t] = min(si[q][t], si[q][t + s]);
        __syncthreads();
    }
    if (t == 0) {
        m.meta[0] = si[0][0] == none ? 0 : si[0][0] - 1;
        m.meta[1] = si[1][0] == none ? 0 : si[1][0];
        m.meta[2] = si[2][0] == none ? 0 : si[2][0] - 1;
        m.meta[3] = si[3][0] == none ? 0 : si[3][0];
        m.meta[4] = 0;
        m.meta[5] = 0;
    }
}

// Crossing parity of every (k,j) cell; the cut-cell flags cleared.
__global__ void k_dyn_main(int ny, int nz, const double* Y, const double* Z, DynMask m, const Ctl* ctl) {
    if (ctl->halt) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (k > nz || j > ny) return;
    const double* az = m.poly;
    m.flags[(long long)(k - 1) + (long long)nz * (j - 1)] = 0;
    ray_main_cell(k, j, nz, Y, Z, az, az + m.npts, m.npts, m.eta1, &m.meta[5]);
}

// Flags of the cells that hold a vertex (within the bounds).
__global__ void k_dyn_points(int ny, int nz, const double* Y, const double* Z, DynMask m, const Ctl* ctl) {
    if (ctl->halt) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m.npts) return;
    const double* az = m.poly;
    ray_point(q, ny, nz, Y, Z, az, az + m.npts, m.meta[0], m.meta[1], m.meta[2], m.meta[3], m.flags);
}

// The flagged cells into the list (in any order: each is computed on its own).
__global__ void k_dyn_compact(int cells, DynMask m, const Ctl* ctl) {
    if (ctl->halt) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < cells && m.flags[q]) m.list[atomicAdd(&m.meta[4], 1)] = q;
}

// Sub-cell fractions of the listed cells; blocks stride over the list.
template <int NT>
__global__ void __launch_bounds__(NT) k_dyn_sub(int nz, const double* Y, const double* Z, DynMask m,
                                                const Ctl* ctl) {
    if (ctl->halt) return;
    __shared__ int red[NT];
    const double* az = m.poly;
    const int count = m.meta[4];
    for (int q = blockIdx.x; q < count; q += gridDim.x)
        ray_sub_cell<NT>(m.list[q], nz, Y, Z, az, az + m.npts, m.npts, m.eta1, &m.meta[5], red);
}

// ETA from ETA_1, as k_extrude.
__global__ void k_dyn_extrude(Geom g, const double* eta1, double* eta, const Ctl* ctl) {
    if (ctl->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
    const int k = blockIdx.z * blockDim.z + threadIdx.z - 1;
    if (i > g.nx + 2 || j > g.ny + 2 || k > g.nz + 2) return;
    const bool in = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
    eta[nat(g, i, j, k)] = in ? eta1[(long long)(k - 1) + (long long)g.nz * (j - 1)] : 0.0;
}

// The step runs (IF condition 1) unless this or an earlier step of the call met
// a tie; the first such step's tie count is kept in the control block.
__global__ void k_dyn_gate(DynMask m, Ctl* ctl, cudaGraphConditionalHandle h) {
    if (!ctl->halt && m.meta[5] > 0) {
        ctl->halt = 1;
        ctl->halt_ties = m.meta[5];
    }
    cudaGraphSetConditional(h, ctl->halt ? 0u : 1u);
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
