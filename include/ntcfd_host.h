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

/* PLOT3D files in the reference's format: Fortran unformatted sequential
 * records (4-byte length before and after each), default reals (4 bytes),
 * one block.  Return 0, -1 for bad arguments, -2 for a file error, -3 for a
 * file whose records do not match nx, ny, nz.
 *
 * ntcfd_write_plot3d_x: mesh.x of gridder.f90:150-212 -- the cell-centre
 * coordinates (X(i) + X(i+1))/2 etc. from the node coordinates X, Y, Z (n+5
 * entries, index -1..n+3, as ntcfd_gridder_* returns them). */
int ntcfd_write_plot3d_x(const char* path, int nx, int ny, int nz,
                         const double* X, const double* Y, const double* Z);

/* NNNN.q of filereachtime (filer.f90:161-187): pre, uc, vc, wc ((nx,ny,nz),
 * as ntcfd_get_output returns them) and ETA (the halo array of
 * ntcfd_get_mask, interior taken), with the four header reals 1.0.
 * append = 1 adds the solution to the end of an existing file, as the
 * reference's position='append' does; 0 replaces the file. */
int ntcfd_write_plot3d_q(const char* path, int nx, int ny, int nz, const double* pre,
                         const double* uc, const double* vc, const double* wc,
                         const double* eta, int append);

/* reading_variables (reading_data.f90:62-90): restart from the first
 * solution of a .q file.  u, v, w, p are halo arrays ((n+4)^3); u(i,j,k) =
 * 0.5 (uc(i) + uc(i+1)) in default-real arithmetic for i, j, k = 1..n-1 (and
 * likewise v, w), p = pre on the interior; every other entry keeps the
 * value the caller put there. */
int ntcfd_read_plot3d_q(const char* path, int nx, int ny, int nz,
                        double* u, double* v, double* w, double* p);

#ifdef __cplusplus
}
#endif

#endif /* NTCFD_HOST_H */
