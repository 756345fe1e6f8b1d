! ntcfd_iface.f90 -- ISO_C_BINDING interface of the B200 time step for the
! NTUSTCFD Fortran driver (main.f90).  The types mirror include/ntcfd.h
! field by field (C arrays [6][3] appear as (3,6)); every interface is the
! C entry point of the same name in include/ntcfd.h or include/ntcfd_host.h.
!
! Status: written against the C headers, not compiled here (no Fortran
! compiler in this environment).  The C side it binds is built and tested,
! and tests/test_fortran_iface.py checks this file's type sizes and entry
! point list against the headers and the library.
module ntcfd_iface
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: NTCFD_OK = 0, NTCFD_NOT_CONVERGED = 1
   integer(c_int), parameter :: NTCFD_EINVAL = -1, NTCFD_ECUDA = -2, NTCFD_ENOMEM = -3, &
                                NTCFD_ENONFINITE = -4, NTCFD_ESTATE = -5, NTCFD_ETIMEOUT = -6
   integer(c_int), parameter :: NTCFD_BC_NOSLIP = 0, NTCFD_BC_NEUMANN = 1, &
                                NTCFD_BC_DIRICHLET = 2, NTCFD_BC_PERIODIC = 3, &
                                NTCFD_BC_INTERFACE = 4
   integer(c_int), parameter :: NTCFD_FIELD_U = 0, NTCFD_FIELD_V = 1, NTCFD_FIELD_W = 2, &
                                NTCFD_FIELD_P = 3, NTCFD_FIELD_WSTAR = 4, NTCFD_FIELD_E_RED = 5, &
                                NTCFD_FIELD_E_BLACK = 6
   integer(c_int), parameter :: NTCFD_STAGE_PREDICT = 0, NTCFD_STAGE_RHS = 1, &
                                NTCFD_STAGE_HALFSWEEP = 2, NTCFD_STAGE_CORRECT = 3, &
                                NTCFD_STAGE_PROJECT = 4
   integer(c_int), parameter :: NTCFD_WEST = 0, NTCFD_EAST = 1, NTCFD_SOUTH = 2, &
                                NTCFD_NORTH = 3, NTCFD_BACK = 4, NTCFD_FRONT = 5
   integer(c_int), parameter :: NTCFD_FP64 = 0, NTCFD_MIXED = 1
   integer(c_int), parameter :: NTCFD_QUICK_CENTRE = 0, NTCFD_QUICK = 1, NTCFD_UPWIND = 2, NTCFD_CENTRE = 3
   integer(c_int), parameter :: NTCFD_SMAG_REF_ALIASED = 0, NTCFD_SMAG_STAGGERED = 1
   integer(c_int), parameter :: NTCFD_SOR_AUTO = 0, NTCFD_SOR_STREAMING = 1, NTCFD_SOR_RESIDENT = 2

   type, bind(C) :: ntcfd_params
      integer(c_int) :: nx, ny, nz
      real(c_double) :: Re, dt, omega, zeta
      integer(c_int) :: itmax, LES
      real(c_double) :: Cs
      integer(c_int) :: scheme, precision, sor_order, smag_mode, check_every
      integer(c_int) :: bc(3, 6)          ! C bc[6][3]: (component, wall)
      real(c_double) :: bc_value(3, 6)
      real(c_double) :: u_solid(3)
      real(c_double) :: lx
      integer(c_int) :: mixed_cycle, diag_divergence, device, sor_path, eager
      integer(c_int) :: reserved(3)
   end type ntcfd_params

   type, bind(C) :: ntcfd_step_info
      integer(c_int) :: sor_iters, converged
      real(c_double) :: sor_last_change, cDrag, cLift, div_max
      integer(c_int) :: dc_cycles, launches, sor_path, pad
      real(c_double) :: aoa
   end type ntcfd_step_info

   type, bind(C) :: ntcfd_kernel_times
      real(c_float) :: predictor_ms, rhs_ms, defect_ms, sweep_ms, project_ms, bc_ms
      real(c_float) :: resident_ms, resident_sweeps
   end type ntcfd_kernel_times

   type, bind(C) :: ntcfd_adj_spec
      integer(c_int) :: nsteps, checkpoint_every
      real(c_double) :: w_drag, w_lift, adj_zeta, adj_omega
      integer(c_int) :: adj_itmax, inflow_wall, inflow_normal, inflow_tangential
      integer(c_int) :: initial_bc
      integer(c_int) :: reserved(3)
   end type ntcfd_adj_spec

   type, bind(C) :: ntcfd_adj_result
      real(c_double) :: J
      real(c_double) :: dJ_dbc(3, 6)      ! C dJ_dbc[6][3]: (component, wall)
      real(c_double) :: dJ_dU, dJ_dtheta
      real(c_double) :: forward_ms, total_ms, recompute_ms, solve_ms
      integer(c_long_long) :: adj_sweeps
      integer(c_int) :: adj_unconverged, recomputed_steps, fwd_status, pad
      real(c_double) :: dJ_daoa_body
   end type ntcfd_adj_result

   interface
      subroutine ntcfd_default_params(p) bind(C, name="ntcfd_default_params")
         import :: ntcfd_params
         type(ntcfd_params), intent(out) :: p
      end subroutine

      integer(c_int) function ntcfd_create(p, ctx) bind(C, name="ntcfd_create")
         import :: c_int, c_ptr, ntcfd_params
         type(ntcfd_params), intent(in) :: p
         type(c_ptr), intent(out) :: ctx
      end function

      subroutine ntcfd_destroy(ctx) bind(C, name="ntcfd_destroy")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end subroutine

      type(c_ptr) function ntcfd_last_error(ctx) bind(C, name="ntcfd_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function ntcfd_set_metrics(ctx, iDx, Dxs, iDy, Dys, iDz, Dzs) &
            bind(C, name="ntcfd_set_metrics")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: iDx(*), Dxs(*), iDy(*), Dys(*), iDz(*), Dzs(*)
      end function

      integer(c_int) function ntcfd_set_coords(ctx, X, Y, Z) bind(C, name="ntcfd_set_coords")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: X(*), Y(*), Z(*)
      end function

      integer(c_int) function ntcfd_set_mask(ctx, eta) bind(C, name="ntcfd_set_mask")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: eta(*)
      end function

      integer(c_int) function ntcfd_get_mask(ctx, eta) bind(C, name="ntcfd_get_mask")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: eta(*)
      end function

      integer(c_int) function ntcfd_build_mask_polygon(ctx, az, ay, npts, aoa, zc, yc, ties) &
            bind(C, name="ntcfd_build_mask_polygon")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: az(*), ay(*)
         integer(c_int), value :: npts
         real(c_double), value :: aoa, zc, yc
         integer(c_int), intent(out) :: ties
      end function

      integer(c_int) function ntcfd_build_mask_polygon_noalloc(ctx, az, ay, npts, aoa, zc, yc, ties) &
            bind(C, name="ntcfd_build_mask_polygon_noalloc")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: az(*), ay(*)
         integer(c_int), value :: npts
         real(c_double), value :: aoa, zc, yc
         integer(c_int), intent(out) :: ties
      end function

      integer(c_int) function ntcfd_build_mask_smooth(ctx, az, ay, npts, aoa_deg, zc, yc, width) &
            bind(C, name="ntcfd_build_mask_smooth")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: az(*), ay(*)
         integer(c_int), value :: npts
         real(c_double), value :: aoa_deg, zc, yc, width
      end function

      integer(c_int) function ntcfd_build_mask_cylinder(ctx, zc, yc, r) &
            bind(C, name="ntcfd_build_mask_cylinder")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), value :: zc, yc, r
      end function

      integer(c_int) function ntcfd_set_state(ctx, u, v, w, p) bind(C, name="ntcfd_set_state")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: u(*), v(*), w(*), p(*)
      end function

      integer(c_int) function ntcfd_get_state(ctx, u, v, w, p) bind(C, name="ntcfd_get_state")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: u(*), v(*), w(*), p(*)
      end function

      integer(c_int) function ntcfd_apply_bc(ctx) bind(C, name="ntcfd_apply_bc")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function ntcfd_get_output(ctx, pre, uc, vc, wc) bind(C, name="ntcfd_get_output")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: pre(*), uc(*), vc(*), wc(*)
      end function

      integer(c_int) function ntcfd_step(ctx, nsteps, info) bind(C, name="ntcfd_step")
         import :: c_int, c_ptr, ntcfd_step_info
         type(c_ptr), value :: ctx
         integer(c_int), value :: nsteps
         type(ntcfd_step_info), intent(out) :: info(*)
      end function

      real(c_double) function ntcfd_time(ctx) bind(C, name="ntcfd_time")
         import :: c_double, c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function ntcfd_last_step_ms(ctx, ms) bind(C, name="ntcfd_last_step_ms")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: ctx
         real(c_float), intent(out) :: ms
      end function

      integer(c_int) function ntcfd_time_kernels(ctx, reps, times) bind(C, name="ntcfd_time_kernels")
         import :: c_int, c_ptr, ntcfd_kernel_times
         type(c_ptr), value :: ctx
         integer(c_int), value :: reps
         type(ntcfd_kernel_times), intent(out) :: times
      end function

      integer(c_int) function ntcfd_set_dynamic_aoa(ctx, az, ay, npts, aoa1, reduce_frequency, zc, yc, &
            start_step) bind(C, name="ntcfd_set_dynamic_aoa")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: az(*), ay(*)
         integer(c_int), value :: npts
         real(c_double), value :: aoa1, reduce_frequency, zc, yc
         integer(c_int), value :: start_step
      end function

      ! pre, uc, vc, wc are written after the call returns, until
      ! ntcfd_output_wait: hence ASYNCHRONOUS here and on the actual arrays
      integer(c_int) function ntcfd_output_async(ctx, pre, uc, vc, wc) bind(C, name="ntcfd_output_async")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), asynchronous :: pre(*), uc(*), vc(*), wc(*)
      end function

      integer(c_int) function ntcfd_output_wait(ctx) bind(C, name="ntcfd_output_wait")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      ! z-slab stages (one context per slab; the caller exchanges the planes)
      integer(c_int) function ntcfd_slab_stage(ctx, stage, colour) bind(C, name="ntcfd_slab_stage")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: stage, colour
      end function

      integer(c_int) function ntcfd_slab_change(ctx, max_change) bind(C, name="ntcfd_slab_change")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: max_change
      end function

      integer(c_long_long) function ntcfd_slab_plane_elems(ctx, field) bind(C, name="ntcfd_slab_plane_elems")
         import :: c_int, c_ptr, c_long_long
         type(c_ptr), value :: ctx
         integer(c_int), value :: field
      end function

      ! buf: count * ntcfd_slab_plane_elems doubles (host, or c_loc of device memory)
      integer(c_int) function ntcfd_slab_planes(ctx, field, k0, count, buf, put) bind(C, name="ntcfd_slab_planes")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, buf
         integer(c_int), value :: field, k0, count, put
      end function

      ! fu, fv, fw: c_loc of an (nx,ny,nz) array, or c_null_ptr for a zero component
      integer(c_int) function ntcfd_set_body_force(ctx, fu, fv, fw) bind(C, name="ntcfd_set_body_force")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         type(c_ptr), value :: fu, fv, fw     ! c_loc(array) or c_null_ptr
      end function

      integer(c_int) function ntcfd_adjoint(ctx, spec, result, dJ_dfu, dJ_dfv, dJ_dfw, info) &
            bind(C, name="ntcfd_adjoint")
         import :: c_int, c_ptr, ntcfd_adj_spec, ntcfd_adj_result
         type(c_ptr), value :: ctx
         type(ntcfd_adj_spec), intent(in) :: spec
         type(ntcfd_adj_result), intent(out) :: result
         type(c_ptr), value :: dJ_dfu, dJ_dfv, dJ_dfw, info   ! c_loc(array) or c_null_ptr
      end function

      ! include/ntcfd_host.h
      subroutine ntcfd_gridder_equal(nx, ny, nz, lx, ly, lz, X, Y, Z, iDx, Dxs, iDy, Dys, iDz, Dzs) &
            bind(C, name="ntcfd_gridder_equal")
         import :: c_int, c_double
         integer(c_int), value :: nx, ny, nz
         real(c_double), value :: lx, ly, lz
         real(c_double), intent(out) :: X(*), Y(*), Z(*), iDx(*), Dxs(*), iDy(*), Dys(*), iDz(*), Dzs(*)
      end subroutine

      subroutine ntcfd_gridder_unequal(nx, ny, nz, lx, ly, lz, band, X, Y, Z, iDx, Dxs, iDy, Dys, &
            iDz, Dzs) bind(C, name="ntcfd_gridder_unequal")
         import :: c_int, c_double
         integer(c_int), value :: nx, ny, nz
         real(c_double), value :: lx, ly, lz
         real(c_double), intent(in) :: band(13)
         real(c_double), intent(out) :: X(*), Y(*), Z(*), iDx(*), Dxs(*), iDy(*), Dys(*), iDz(*), Dzs(*)
      end subroutine

      integer(c_int) function ntcfd_naca4_polygon(t, npts, z, y) bind(C, name="ntcfd_naca4_polygon")
         import :: c_int, c_double
         real(c_double), value :: t
         integer(c_int), value :: npts
         real(c_double), intent(out) :: z(*), y(*)
      end function

      integer(c_int) function ntcfd_naca4_polygon_te(t, npts, closed_te, z, y) &
            bind(C, name="ntcfd_naca4_polygon_te")
         import :: c_int, c_double
         real(c_double), value :: t
         integer(c_int), value :: npts, closed_te
         real(c_double), intent(out) :: z(*), y(*)
      end function

      integer(c_int) function ntcfd_circle_polygon(r, npts, z, y) bind(C, name="ntcfd_circle_polygon")
         import :: c_int, c_double
         real(c_double), value :: r
         integer(c_int), value :: npts
         real(c_double), intent(out) :: z(*), y(*)
      end function

      integer(c_int) function ntcfd_write_plot3d_x(path, nx, ny, nz, X, Y, Z) &
            bind(C, name="ntcfd_write_plot3d_x")
         import :: c_int, c_double, c_char
         character(kind=c_char), intent(in) :: path(*)      ! NUL-terminated
         integer(c_int), value :: nx, ny, nz
         real(c_double), intent(in) :: X(*), Y(*), Z(*)
      end function

      integer(c_int) function ntcfd_write_plot3d_q(path, nx, ny, nz, pre, uc, vc, wc, eta, append) &
            bind(C, name="ntcfd_write_plot3d_q")
         import :: c_int, c_double, c_char
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int), value :: nx, ny, nz
         real(c_double), intent(in) :: pre(*), uc(*), vc(*), wc(*), eta(*)
         integer(c_int), value :: append
      end function

      integer(c_int) function ntcfd_read_plot3d_q(path, nx, ny, nz, u, v, w, p) &
            bind(C, name="ntcfd_read_plot3d_q")
         import :: c_int, c_double, c_char
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int), value :: nx, ny, nz
         real(c_double), intent(inout) :: u(*), v(*), w(*), p(*)
      end function
   end interface
end module ntcfd_iface
