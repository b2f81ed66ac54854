! A Fortran caller of the library, through the explicit interfaces of
! include/zfmm.f90: zlfmm2d and zhfmm3d as the reference's drivers call them
! (zfmm2d/test/laplace/test5.f, zfmm3d/test/helmholtz), the status-returning
! form, and the in-place clamping of an out-of-range flag.  Prints the values
! the test compares with the Python binding.
program drop_in
  use zfmm_b200
  implicit none
  integer, parameter :: n = 2000
  complex(c_double_complex) :: zsrc(2, n), charge(n), dipstr(n), dipvec(2, n), pot(n), grad(2, n)
  complex(c_double_complex) :: z3(3, n), dv3(3, n), pot3(n), grad3(3, n), zk
  integer(c_int) :: ifcharge, ifdipole, ifpgh, i, st
  real(c_double) :: t
  do i = 1, n
    t = 6.283185307179586d0 * (i - 1) / n
    zsrc(1, i) = cmplx(cos(t), 0.05d0 * sin(3 * t), c_double_complex)
    zsrc(2, i) = cmplx(sin(t), 0.05d0 * cos(3 * t), c_double_complex)
    charge(i) = cmplx(cos(7 * t), sin(5 * t), c_double_complex)
    dipstr(i) = cmplx(sin(2 * t), 1.0d0, c_double_complex)
    dipvec(1, i) = cos(t); dipvec(2, i) = sin(t)
    z3(1, i) = zsrc(1, i); z3(2, i) = zsrc(2, i); z3(3, i) = cmplx(0.1d0 * i / n, 0, c_double_complex)
    dv3(:, i) = (1.0d0, 0.0d0)
  end do
  ifcharge = 1; ifdipole = 1; ifpgh = 2
  call zlfmm2d(1d-9, n, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, n, zsrc, &
               ifpgh, 1, 0)
  write(*, '(A,4ES24.16)') 'zlfmm2d ', pot(1), pot(n)
  zk = (10.0d0, 0.2d0)
  ifpgh = 7  ! out of range: clamped to 1 in place
  call zhfmm3d(1d-9, zk, n, z3, ifcharge, charge, ifdipole, dipstr, dv3, pot3, grad3, n, z3, &
               ifpgh, 1, 0)
  write(*, '(A,I3,4ES24.16)') 'zhfmm3d ', ifpgh, pot3(1), pot3(n)
  st = zfmm_zlfmm2d(1d-9, n, zsrc, 1, charge, 0, dipstr, dipvec, pot, grad, n, zsrc, 1, 0, 0)
  write(*, '(A,I3,A,A)') 'status ', st, ' ', zfmm_last_error()
end program
