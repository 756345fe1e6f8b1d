/*
 * ntcfd_host.h -- host-side set-up routines of the B200 time step.
 *
 * These are the host half of the drop-in: the work the Fortran driver does
 * before the time loop (reading_data, gridder_equal/gridder_Unequal) and the
 * analytic body polygons that replace the NACA .DAT input files.  They run on
 * the CPU, allocate nothing on the device and can be called without a GPU.
 *
 * Array conventions follow variables_module.f90:292-316: node coordinates
 * X(-1:nx+3) have nx+5 entries, metrics iDx/Dxs(-1:nx+2) have nx+4 entries.
 */
#ifndef NTCFD_HOST_H
#define NTCFD_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* reading_data (uniform branch, reading_data.f90:26-30) + gridder_equal
 * (gridder.f90:228-327): dx = lx/nx, cumulative nodes from X(1) = 0. */
void ntcfd_gridder_equal(int nx, int ny, int nz, double lx, double ly, double lz,
                         double* X, double* Y, double* Z,
                         double* iDx, double* Dxs, double* iDy, double* Dys,
                         double* iDz, double* Dzs);

/* reading_data (non-uniform branch, reading_data.f90:6-23) + gridder_Unequal
 * (gridder.f90:1-157).  band[13] = {GridderXc, GridderYc, GridderZc, nxSml,
 * nySml, nyMid, nzSml, nzMid, lxSml, lySml, lyMid, lzSml, lzMid}
 * (variables_module.f90:56-80).  x stays uniform (reading_data.f90:23). */
void ntcfd_gridder_unequal(int nx, int ny, int nz, double lx, double ly, double lz,
                           const double* band,
                           double* X, double* Y, double* Z,
                           double* iDx, double* Dxs, double* iDy, double* Dys,
                           double* iDz, double* Dzs);

/* Closed NACA 4-digit symmetric section of chord 1 and thickness t from the
 * analytic thickness formula, npts cosine-spaced points per surface,
 * ordered like NACA0012.DAT: leading edge -> upper surface -> trailing edge
 * -> lower surface -> leading edge, last point = first point.  Writes
 * 2*npts points (z = chordwise, y = thickness) and returns that count. */
int ntcfd_naca4_polygon(double t, int npts, double* z, double* y);

/* The same with a choice of trailing edge: closed_te = 0 uses the open
 * trailing-edge coefficient -0.1015 (as ntcfd_naca4_polygon; the points of
 * NACA0012.DAT, read by airfoil.f90:590, follow it), closed_te = 1 the closed
 * one, -0.1036 (the points of NACA0015.DAT follow it). */
int ntcfd_naca4_polygon_te(double t, int npts, int closed_te, double* z, double* y);

/* Closed circle of radius r centred at (0,0), npts distinct points
 * counter-clockwise from angle 0, last point = first point; returns npts+1. */
int ntcfd_circle_polygon(double r, int npts, double* z, double* y);

#ifdef __cplusplus
}
#endif

#endif /* NTCFD_HOST_H */
