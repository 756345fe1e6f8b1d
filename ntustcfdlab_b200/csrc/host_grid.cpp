// host_grid.cpp -- host-side set-up: grid generation (reading_data.f90,
// gridder.f90) and analytic body polygons.  Plain C++, no device work.
#include <cmath>
#include <vector>

#include "../../include/ntcfd_host.h"

namespace {

// a(-1:n+3) or a(-1:n+2) stored from index 0
struct Axis {
    double* a;
    double& operator()(int i) { return a[i + 1]; }
};

// gridder.f90:97-157 -- cell widths iD(i) = X(i+1)-X(i) and centre spacings
// Ds(i) = (X(i+2)-X(i))/2 for i = 1..n-1, then the ghost values.
void metrics(int n, double* Xp, double* iDp, double* Dsp) {
    Axis X{Xp}, iD{iDp}, Ds{Dsp};
    for (int i = 1; i <= n - 1; ++i) {
        iD(i) = X(i + 1) - X(i);
        Ds(i) = (X(i + 2) - X(i)) / 2.0;
    }
    iD(0) = iD(1);
    iD(-1) = iD(1);
    iD(n) = X(n + 1) - X(n);
    iD(n + 1) = iD(n);
    iD(n + 2) = iD(n);
    Ds(0) = Ds(1);
    Ds(-1) = Ds(1);
    Ds(n) = Ds(n - 1);
    Ds(n + 1) = Ds(n - 1);
    Ds(n + 2) = Ds(n - 1);
}

// gridder.f90:235-263 -- X(1) = 0, X(0) = -d, X(-1) = -2d, X(i) = X(i-1) + d.
void uniform(int n, double d, double* Xp) {
    Axis X{Xp};
    X(1) = 0.0;
    X(0) = X(1) - d;
    X(-1) = X(0) - d;
    for (int i = 2; i <= n + 3; ++i) X(i) = X(i - 1) + d;
}

// gridder.f90:45-93 -- greedy three-band stretching: from Y(j-1), take the
// small step inside the fine band, the middle step inside the middle band
// and the large step elsewhere.  Only Y(1..n+1) are assigned.
void banded(int n, double* Yp, double dL, double dM, double dS, double MBgn, double MEnd,
            double SBgn, double SEnd) {
    Axis Y{Yp};
    for (int j = 1; j <= n + 1; ++j) {
        if (j == 1) {
            Y(j) = 0.0;
            continue;
        }
        const double L = Y(j - 1) + dL, M = Y(j - 1) + dM, S = Y(j - 1) + dS;
        if (L > MBgn) {
            if (M > MEnd) Y(j) = L;
            else if (M > SBgn) Y(j) = (S > SEnd) ? M : S;
            else Y(j) = M;
        } else {
            Y(j) = L;
        }
    }
}

}  // namespace

extern "C" void ntcfd_gridder_equal(int nx, int ny, int nz, double lx, double ly, double lz,
                                    double* X, double* Y, double* Z, double* iDx, double* Dxs,
                                    double* iDy, double* Dys, double* iDz, double* Dzs) {
    uniform(nx, lx / nx, X);
    uniform(ny, ly / ny, Y);
    uniform(nz, lz / nz, Z);
    metrics(nx, X, iDx, Dxs);
    metrics(ny, Y, iDy, Dys);
    metrics(nz, Z, iDz, Dzs);
}

extern "C" void ntcfd_gridder_unequal(int nx, int ny, int nz, double lx, double ly, double lz,
                                      const double* b, double* X, double* Y, double* Z,
                                      double* iDx, double* Dxs, double* iDy, double* Dys,
                                      double* iDz, double* Dzs) {
    const double Yc = b[1], Zc = b[2];
    const int nySml = (int)b[4], nyMid = (int)b[5], nzSml = (int)b[6], nzMid = (int)b[7];
    const double lySml = b[9], lyMid = b[10], lzSml = b[11], lzMid = b[12];
    // reading_data.f90:8-23
    const double dySml = lySml / nySml, dzSml = lzSml / nzSml;
    const double dyMid = (lyMid - lySml) / (nyMid - nySml);
    const double dzMid = (lzMid - lzSml) / (nzMid - nzSml);
    const double dy = (ly - lyMid) / (ny - nyMid);
    const double dz = (lz - lzMid) / (nz - nzMid);
    for (int q = 0; q < nx + 5; ++q) X[q] = 0.0;
    for (int q = 0; q < ny + 5; ++q) Y[q] = 0.0;
    for (int q = 0; q < nz + 5; ++q) Z[q] = 0.0;
    uniform(nx, lx / nx, X);
    // gridder.f90:6-18: band limits
    banded(ny, Y, dy, dyMid, dySml, Yc - lyMid / 2.0, Yc + lyMid / 2.0, Yc - lySml / 2.0,
           Yc + lySml / 2.0);
    banded(nz, Z, dz, dzMid, dzSml, Zc, Zc + lzMid, Zc, Zc + lzSml);
    metrics(nx, X, iDx, Dxs);
    metrics(ny, Y, iDy, Dys);
    metrics(nz, Z, iDz, Dzs);
}

extern "C" int ntcfd_naca4_polygon_te(double t, int npts, int closed_te, double* z, double* y) {
    if (npts < 2) return 0;
    const double PI = 4.0 * std::atan(1.0);
    // last coefficient of the 4-digit thickness polynomial: -0.1015 leaves the
    // trailing edge open (NACA0012.DAT follows it), -0.1036 closes it (NACA0015.DAT)
    const double a4 = closed_te ? -0.1036 : -0.1015;
    auto thick = [t, a4](double x) {
        return 5.0 * t * (0.2969 * std::sqrt(x) - 0.1260 * x - 0.3516 * x * x +
                          0.2843 * x * x * x + a4 * x * x * x * x);
    };
    int q = 0;
    for (int i = 0; i < npts; ++i) {           // leading edge -> trailing edge, upper
        const double x = 0.5 * (1.0 - std::cos(PI * i / (npts - 1)));
        z[q] = x;
        y[q] = thick(x);
        ++q;
    }
    for (int i = npts - 1; i >= 0; --i) {      // trailing edge -> leading edge, lower
        const double x = 0.5 * (1.0 - std::cos(PI * i / (npts - 1)));
        z[q] = x;
        y[q] = -thick(x);
        ++q;
    }
    // the leading edge point closes the polygon: thick(0) = 0 on both sides
    return q;
}

extern "C" int ntcfd_naca4_polygon(double t, int npts, double* z, double* y) {
    return ntcfd_naca4_polygon_te(t, npts, 0, z, y);
}

extern "C" int ntcfd_circle_polygon(double r, int npts, double* z, double* y) {
    if (npts < 3) return 0;
    const double PI = 4.0 * std::atan(1.0);
    for (int i = 0; i < npts; ++i) {
        const double a = 2.0 * PI * i / npts;
        z[i] = r * std::cos(a);
        y[i] = r * std::sin(a);
    }
    z[npts] = z[0];
    y[npts] = y[0];
    return npts + 1;
}
