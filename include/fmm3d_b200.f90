! Explicit Fortran interfaces (iso_c_binding) to libfmm3d_b200.so.
!
! The library exports the reference's own gfortran-mangled symbols, so existing
! callers of lfmm3dpart / hfmm3dpart link unchanged; this module gives new code
! checked interfaces to the same entry points.  Argument lists and meanings are
! those of FMMLIB3D:
!   lfmm3dpart      src/lfmm3dpart.f:36-80       lfmm3dpartself  src/lfmm3dpart.f:87-131
!   lfmm3dparttarg  src/lfmm3dpart.f:138-522     l3dpartdirect   src/lfmm3dpart.f:1391-1523
!   hfmm3dpart      src/hfmm3dpart.f:39-83       hfmm3dpartself  src/hfmm3dpart.f:90-131
!   hfmm3dparttarg  src/hfmm3dpart.f:141-539     h3dpartdirect   src/hfmm3dpart.f:1268-1401
! Every argument is passed by reference; complex*16 is complex(c_double_complex).
!
! Build (where a Fortran compiler exists):
!   gfortran -c fmm3d_b200.f90 && gfortran main.f90 fmm3d_b200.o -L<dir> -lfmm3d_b200 -lcudart
module fmm3d_b200
  use iso_c_binding
  implicit none
  interface

    subroutine lfmm3dpart(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld) bind(C, name="lfmm3dpart_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      real(c_double) :: source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine lfmm3dpartself(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld) bind(C, name="lfmm3dpartself_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      real(c_double) :: source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine lfmm3dparttarg(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="lfmm3dparttarg_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      real(c_double) :: source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine l3dpartdirect(nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="l3dpartdirect_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      real(c_double) :: source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine hfmm3dpart(ier, iprec, zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld) bind(C, name="hfmm3dpart_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      complex(c_double_complex) :: zk
      real(c_double) :: source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine hfmm3dpartself(ier, iprec, zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld) bind(C, name="hfmm3dpartself_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      complex(c_double_complex) :: zk
      real(c_double) :: source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine hfmm3dparttarg(ier, iprec, zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="hfmm3dparttarg_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      complex(c_double_complex) :: zk
      real(c_double) :: source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine h3dpartdirect(zk, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="h3dpartdirect_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      complex(c_double_complex) :: zk
      real(c_double) :: source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    ! Arithmetic form of later calls: 0 FP64 (default), 1 mixed precision for iprec <= 1.
    ! Layer potentials of flat triangles (lfmm3dtriatarg, lfmm3dtriaself, lfmm3dtria, l3dtriadirect)
    subroutine lfmm3dtriatarg(ier, iprec, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="lfmm3dtriatarg_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine lfmm3dtriaself(ier, iprec, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld) bind(C, name="lfmm3dtriaself_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine lfmm3dtria(ier, iprec, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld) bind(C, name="lfmm3dtria_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine l3dtriadirect(nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="l3dtriadirect_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine hfmm3dtriatarg(ier, iprec, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="hfmm3dtriatarg_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      complex(c_double_complex) :: zk
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    subroutine hfmm3dtriaself(ier, iprec, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld) bind(C, name="hfmm3dtriaself_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      complex(c_double_complex) :: zk
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine hfmm3dtria(ier, iprec, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, &
        dipstr, dipvec, ifpot, pot, iffld, fld) bind(C, name="hfmm3dtria_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld
      complex(c_double_complex) :: zk
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *)
    end subroutine

    subroutine h3dtriadirect(nqtri, zk, nsource, triaflat, trianorm, source, ifcharge, charge, ifdipole, dipstr, &
        dipvec, ifpot, pot, iffld, fld, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg) &
        bind(C, name="h3dtriadirect_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: nqtri, nsource, ifcharge, ifdipole, ifpot, iffld, ntarget, ifpottarg, iffldtarg
      complex(c_double_complex) :: zk
      real(c_double) :: triaflat(3, 3, *), trianorm(3, *), source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), pottarg(*), fldtarg(3, *)
    end subroutine

    ! Hessians: the reference's one-point evaluators, and lfmm3dparttarg with Hessian outputs
    ! (hess(6, n): dxx, dyy, dzz, dxy, dxz, dyz; no counterpart in the reference)
    subroutine l3dtaevalhess(rscale, center, local, nterms, ztarg, pot, iffld, fld, ifhess, hess, ier) &
        bind(C, name="l3dtaevalhess_")
      import :: c_int, c_double, c_double_complex
      real(c_double) :: rscale, center(3), ztarg(3)
      integer(c_int) :: nterms, iffld, ifhess, ier
      complex(c_double_complex) :: local(0:nterms, -nterms:nterms), pot, fld(3), hess(6)
    end subroutine

    subroutine l3dmpevalhess(rscale, center, mpole, nterms, ztarg, pot, iffld, fld, ifhess, hess, ier) &
        bind(C, name="l3dmpevalhess_")
      import :: c_int, c_double, c_double_complex
      real(c_double) :: rscale, center(3), ztarg(3)
      integer(c_int) :: nterms, iffld, ifhess, ier
      complex(c_double_complex) :: mpole(0:nterms, -nterms:nterms), pot, fld(3), hess(6)
    end subroutine

    subroutine lfmm3dparttarghess(ier, iprec, nsource, source, ifcharge, charge, ifdipole, dipstr, dipvec, &
        ifpot, pot, iffld, fld, ifhess, hess, ntarget, target, ifpottarg, pottarg, iffldtarg, fldtarg, &
        ifhesstarg, hesstarg) bind(C, name="lfmm3dparttarghess_")
      import :: c_int, c_double, c_double_complex
      integer(c_int) :: ier, iprec, nsource, ifcharge, ifdipole, ifpot, iffld, ifhess, ntarget, ifpottarg, &
          iffldtarg, ifhesstarg
      real(c_double) :: source(3, *), dipvec(3, *), target(3, *)
      complex(c_double_complex) :: charge(*), dipstr(*), pot(*), fld(3, *), hess(6, *), pottarg(*), &
          fldtarg(3, *), hesstarg(6, *)
    end subroutine

    integer(c_int) function fmm3d_set_precision(mode) bind(C, name="fmm3d_set_precision")
      import :: c_int
      integer(c_int), value :: mode
    end function

    ! The same for the calling thread only (-1: follow fmm3d_set_precision).
    integer(c_int) function fmm3d_set_precision_thread(mode) bind(C, name="fmm3d_set_precision_thread")
      import :: c_int
      integer(c_int), value :: mode
    end function

  end interface
end module fmm3d_b200
