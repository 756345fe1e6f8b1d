/*
 * ntcfd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of NTUSTCFD's projection-method time step, used as the
 * checker for the CUDA path (tests, smoke check) and as the timed CPU
 * baseline.  Nothing in the product library links, loads or calls it.
 *
 * Parity status: the reference (Fortran 90 + MPI + OpenMP) ships no tests,
 * no golden vectors and no fixtures, and no Fortran compiler exists here, so
 * this restatement cannot be pinned against reference outputs: parity is
 * unpinned by the reference's own tests.  It follows the reference line by
 * line (file:line cited per routine) with nproc = 1 (istart = 1, iend = nz).
 *
 * Every array is a Fortran-order halo array as in variables_module.f90.
 */
#ifndef NTCFD_ORACLE_H
#define NTCFD_ORACLE_H

#include "../include/ntcfd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

orc* orc_create(const ntcfd_params* p);
void orc_destroy(orc* o);
/* 0 or 1: serial (parity mode); >1: the reference's OpenMP schedule
 * (serial k, parallel j) for timing.  Lexicographic SOR is then a racy
 * chaotic relaxation exactly like the reference's, so use it for timing only. */
void orc_set_threads(orc* o, int nthreads);

int  orc_set_metrics(orc* o, const double* iDx, const double* Dxs, const double* iDy,
                     const double* Dys, const double* iDz, const double* Dzs);
int  orc_set_coords(orc* o, const double* X, const double* Y, const double* Z);
int  orc_get_coords(orc* o, double* X, double* Y, double* Z);
/* names: u v w p u1 v1 w1 u2 v2 w2 u_star v_star w_star FX FY FZ ETA (halo);
 *        pre uc vc wc Viseff (nx,ny,nz); FXz FYz (nx,ny); FXy FYy (nx) */
int  orc_set_field(orc* o, const char* name, const double* src);
int  orc_get_field(orc* o, const char* name, double* dst);
long orc_field_size(orc* o, const char* name);

void orc_initial_conditions(orc* o);
void orc_boundary_conditions(orc* o);
void orc_smagorinsky(orc* o);
void orc_predictor(orc* o);
/* forced_sweeps >= 0: run exactly that many sweeps (no stop test). */
int  orc_gauss_seidel(orc* o, int forced_sweeps, double* last_change, int* converged);
void orc_calcul_new_velocity(orc* o);
void orc_force_integral(orc* o, double* cDrag, double* cLift);
void orc_updating_velocity(orc* o);
/* One full loop body (main.f90:209-271); forced (may be NULL) gives the
 * sweep count per step. Returns the summed sweep count. */
int  orc_step(orc* o, int nsteps, ntcfd_step_info* info, const int* forced);
double orc_time(orc* o);

/* Max |div u| * cell volume over the interior, using the same face
 * differences as the SOR right-hand side (GS.f90:39-41) applied to u. */
double orc_divergence_max(orc* o);

/* Grid generators: gridder_equal (gridder.f90:228-383) and
 * gridder_Unequal (gridder.f90:1-223) with reading_data (reading_data.f90:6-33).
 * X,Y,Z: n+5 entries (-1..n+3); metrics n+4 entries (-1..n+2).
 * band[13] = {GridderXc, GridderYc, GridderZc, nxSml, nySml, nyMid, nzSml,
 *             nzMid, lxSml, lySml, lyMid, lzSml, lzMid}. */
void orc_gridder_equal(int nx, int ny, int nz, double lx, double ly, double lz,
                       double* X, double* Y, double* Z,
                       double* iDx, double* Dxs, double* iDy, double* Dys,
                       double* iDz, double* Dzs);
void orc_gridder_unequal(int nx, int ny, int nz, double lx, double ly, double lz,
                         const double* band,
                         double* X, double* Y, double* Z,
                         double* iDx, double* Dxs, double* iDy, double* Dys,
                         double* iDz, double* Dzs);

/* RayCasting (airfoil.f90:580-915); returns the number of tie moves. */
int  orc_raycasting(orc* o, const double* az, const double* ay, int npoly,
                    double aoa_deg, double zc, double yc);
/* DFIB_Cylinder (DFIB.f90:74-145) with r and the centre as arguments. */
void orc_cylinder(orc* o, double zc, double yc, double r);

#ifdef __cplusplus
}
#endif
#endif
