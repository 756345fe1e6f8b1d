! ntcfd_iface.f90 -- ISO_C_BINDING interface of the B200 time step for the
! NTUSTCFD Fortran driver (main.f90).  The types mirror include/ntcfd.h
! field by field; every function is the C entry point of the same name.
!
! Status: written against the C header, not compiled here (no Fortran
! compiler in this environment).  The C side it binds is built and tested.
module ntcfd_iface
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: NTCFD_OK = 0, NTCFD_NOT_CONVERGED = 1
   integer(c_int), parameter :: NTCFD_BC_NOSLIP = 0, NTCFD_BC_NEUMANN = 1, &
                                NTCFD_BC_DIRICHLET = 2, NTCFD_BC_PERIODIC = 3
   integer(c_int), parameter :: NTCFD_FP64 = 0, NTCFD_MIXED = 1

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
      integer(c_int) :: mixed_cycle, diag_divergence, device
      integer(c_int) :: reserved(5)
   end type ntcfd_params

   type, bind(C) :: ntcfd_step_info
      integer(c_int) :: sor_iters, converged
      real(c_double) :: sor_last_change, cDrag, cLift, div_max
      integer(c_int) :: dc_cycles, launches
   end type ntcfd_step_info

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

      integer(c_int) function ntcfd_build_mask_polygon(ctx, az, ay, npts, aoa, zc, yc, ties) &
            bind(C, name="ntcfd_build_mask_polygon")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: az(*), ay(*)
         integer(c_int), value :: npts
         real(c_double), value :: aoa, zc, yc
         integer(c_int), intent(out) :: ties
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
   end interface
end module ntcfd_iface
