! zfmm_b200: Fortran interface module of the B200 complex-coordinate FMM
! library (libzfmm_b200.so, C ABI in include/zfmm.h).
!
! Two ways to call the library from Fortran:
!
!  1. Unchanged reference code.  The library exports the reference's
!     subroutines under the names gfortran gives them (zlfmm2d_, zhfmm2d_,
!     zlfmm3d_, zhfmm3d_, z[lh][23]devaldirect_), with the reference's argument
!     lists (zfmm2d/src/laplace/zlfmm2d.f:14-15, zfmm2d/src/helmholtz/zhfmm2d.f:14-15,
!     zfmm3d/src/laplace/zlfmm3d.f:14-15, zfmm3d/src/helmholtz/zhfmm3d.f:1-2 and
!     the direct sums zlfmm2d.f:600-601, zhfmm2d.f:773-774, zlfmm3d.f:628-629,
!     zhfmm3d.f:626-627).  A program written against the reference links
!     against the library without source changes (implicit interfaces).
!
!  2. Explicit interfaces (this module): `use zfmm_b200` declares the same
!     subroutines with bind(C) names, so the compiler checks every argument,
!     plus the status-returning C entry points (zfmm_* functions: 0 = ok,
!     1 bad argument, 2 CUDA error, 3 out of device memory, 4 internal,
!     5 no GPU) and zfmm_last_error() for the message of the last failure.
!
! Arrays are the reference's: complex*16, column-major, zsrc(d, ns),
! dipvec(d, ns), grad(d, nt).  The subroutines clamp out-of-range
! ifcharge/ifdipole/ifpgh in place as the reference does (zlfmm2d.f:58-68);
! on failure they leave pot and grad zero (the reason is available from
! zfmm_last_error()).
!
! Build: gfortran -c include/zfmm.f90   (produces zfmm_b200.mod)
!        gfortran prog.f90 -L<repo>/zfmm_b200 -lzfmm_b200 -Wl,-rpath,<repo>/zfmm_b200
module zfmm_b200
  use iso_c_binding
  implicit none

  interface

    ! ---- the reference's subroutines (drop-in) --------------------------------

    subroutine zlfmm2d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, &
                       nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zlfmm2d_")
      import :: c_int, c_double, c_double_complex
      real(c_double), intent(in) :: eps
      integer(c_int), intent(in) :: ns, nt, isep, ifprint
      integer(c_int), intent(inout) :: ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: zsrc(2, *), charge(*), dipstr(*), dipvec(2, *)
      complex(c_double_complex), intent(in) :: ztarg(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end subroutine

    subroutine zhfmm2d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, &
                       grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zhfmm2d_")
      import :: c_int, c_double, c_double_complex
      real(c_double), intent(in) :: eps
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), intent(in) :: ns, nt, isep, ifprint
      integer(c_int), intent(inout) :: ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: zsrc(2, *), charge(*), dipstr(*), dipvec(2, *)
      complex(c_double_complex), intent(in) :: ztarg(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end subroutine

    subroutine zlfmm3d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, &
                       nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zlfmm3d_")
      import :: c_int, c_double, c_double_complex
      real(c_double), intent(in) :: eps
      integer(c_int), intent(in) :: ns, nt, isep, ifprint
      integer(c_int), intent(inout) :: ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: zsrc(3, *), charge(*), dipstr(*), dipvec(3, *)
      complex(c_double_complex), intent(in) :: ztarg(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end subroutine

    subroutine zhfmm3d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, &
                       grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zhfmm3d_")
      import :: c_int, c_double, c_double_complex
      real(c_double), intent(in) :: eps
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), intent(in) :: ns, nt, isep, ifprint
      integer(c_int), intent(inout) :: ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: zsrc(3, *), charge(*), dipstr(*), dipvec(3, *)
      complex(c_double_complex), intent(in) :: ztarg(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end subroutine

    ! direct sums: ADD into pot / grad (2D unscaled, 3D with 1/(4 pi))
    subroutine zl2devaldirect(nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, &
                              grad, ifdipole, ifpgh) bind(C, name="zl2devaldirect_")
      import :: c_int, c_double_complex
      integer(c_int), intent(in) :: nt, ns, ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: ztarg(2, *), zsrc(2, *), charge(*), dipstr(*)
      complex(c_double_complex), intent(in) :: dipvec(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end subroutine

    subroutine zh2devaldirect(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, &
                              grad, ifdipole, ifpgh) bind(C, name="zh2devaldirect_")
      import :: c_int, c_double_complex
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), intent(in) :: nt, ns, ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: ztarg(2, *), zsrc(2, *), charge(*), dipstr(*)
      complex(c_double_complex), intent(in) :: dipvec(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end subroutine

    subroutine zl3devaldirect(nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, &
                              grad, ifdipole, ifpgh) bind(C, name="zl3devaldirect_")
      import :: c_int, c_double_complex
      integer(c_int), intent(in) :: nt, ns, ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: ztarg(3, *), zsrc(3, *), charge(*), dipstr(*)
      complex(c_double_complex), intent(in) :: dipvec(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end subroutine

    subroutine zh3devaldirect(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, &
                              grad, ifdipole, ifpgh) bind(C, name="zh3devaldirect_")
      import :: c_int, c_double_complex
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), intent(in) :: nt, ns, ifcharge, ifdipole, ifpgh
      complex(c_double_complex), intent(in) :: ztarg(3, *), zsrc(3, *), charge(*), dipstr(*)
      complex(c_double_complex), intent(in) :: dipvec(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end subroutine

    ! ---- status-returning C entry points (host arrays, arguments by value) ----

    integer(c_int) function zfmm_zlfmm2d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, &
        dipvec, pot, grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zfmm_zlfmm2d")
      import :: c_int, c_double, c_double_complex
      real(c_double), value :: eps
      integer(c_int), value :: ns, ifcharge, ifdipole, nt, ifpgh, isep, ifprint
      complex(c_double_complex), intent(in) :: zsrc(2, *), charge(*), dipstr(*), dipvec(2, *)
      complex(c_double_complex), intent(in) :: ztarg(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end function

    integer(c_int) function zfmm_zhfmm2d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, &
        dipstr, dipvec, pot, grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zfmm_zhfmm2d")
      import :: c_int, c_double, c_double_complex
      real(c_double), value :: eps
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), value :: ns, ifcharge, ifdipole, nt, ifpgh, isep, ifprint
      complex(c_double_complex), intent(in) :: zsrc(2, *), charge(*), dipstr(*), dipvec(2, *)
      complex(c_double_complex), intent(in) :: ztarg(2, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(2, *)
    end function

    integer(c_int) function zfmm_zlfmm3d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, &
        dipvec, pot, grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zfmm_zlfmm3d")
      import :: c_int, c_double, c_double_complex
      real(c_double), value :: eps
      integer(c_int), value :: ns, ifcharge, ifdipole, nt, ifpgh, isep, ifprint
      complex(c_double_complex), intent(in) :: zsrc(3, *), charge(*), dipstr(*), dipvec(3, *)
      complex(c_double_complex), intent(in) :: ztarg(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end function

    integer(c_int) function zfmm_zhfmm3d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, &
        dipstr, dipvec, pot, grad, nt, ztarg, ifpgh, isep, ifprint) bind(C, name="zfmm_zhfmm3d")
      import :: c_int, c_double, c_double_complex
      real(c_double), value :: eps
      complex(c_double_complex), intent(in) :: zk
      integer(c_int), value :: ns, ifcharge, ifdipole, nt, ifpgh, isep, ifprint
      complex(c_double_complex), intent(in) :: zsrc(3, *), charge(*), dipstr(*), dipvec(3, *)
      complex(c_double_complex), intent(in) :: ztarg(3, *)
      complex(c_double_complex), intent(inout) :: pot(*), grad(3, *)
    end function

    type(c_ptr) function zfmm_last_error_c() bind(C, name="zfmm_last_error")
      import :: c_ptr
    end function

  end interface

contains

  ! message of the last failed call on this thread, as a Fortran string
  function zfmm_last_error() result(msg)
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: n
    interface
      integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
        import :: c_ptr, c_size_t
        type(c_ptr), value :: s
      end function
    end interface
    type(c_ptr) :: cp
    cp = zfmm_last_error_c()
    n = int(c_strlen(cp))
    call c_f_pointer(cp, p, [n])
    allocate(character(len=n) :: msg)
    msg = transfer(p(1:n), msg)
  end function

end module zfmm_b200
