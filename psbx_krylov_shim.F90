! psbx_krylov_shim.F90 -- routes PSBLAS 3.9's psb_krylov to libpsbx.so's
! device-resident solver (psbx_dkrylov) when the matrix, both vectors and
! the preconditioner's inverse diagonal already live on the GPU, and leaves
! every other case to the CPU code unchanged.
!
! Build: compile with the PSBLAS 3.9 module directory on the include path
! (the psb_base, psb_prec and psb_cuda modules), link with -lpsbx -lcudart.
!
! Routing: krylov/psb_dkrylov.f90 (psb_dkrylov_vect) calls the shim right
! before its `select case(psb_toupper(method))` (psb_dkrylov.f90:179):
!
!     use psbx_krylov_shim_mod
!     logical :: done
!     ...
!     call psbx_krylov_gpu(method,a,prec,b,x,eps,desc_a,info, &
!          & itmax,iter,err,irst,istop,done)
!     if (done) then
!       if (do_alloc_wrk) call prec%free_wrk(info)
!       call psb_erractionrestore(err_act)
!       return
!     end if
!
! Taken on the device: CG, FCG, CGS, BICG, BICGSTAB, BICGSTABL (L = irst,
! default 1) and RGMRES/GMRES (restart irst, default 10; stop criterion 2
! only), one process (np == 1: the device solver has no halo exchange),
! matrix of type psb_d_cuda_hlg_sparse_mat, psb_d_cuda_elg_sparse_mat or
! psb_d_cuda_csrg_sparse_mat, b and x of type psb_d_vect_cuda, and a DIAG
! preconditioner whose inverse diagonal is a psb_d_vect_cuda, or NONE.
! Everything else -- GCR, other formats, vectors on the host, other
! preconditioners, several processes -- returns done = .false. and the
! caller's CPU path runs as before.  itmax (default 1000) and istop
! (default 2) follow psb_dcg.F90:158-195; iter and err come back as from
! the CPU methods; itrace is not honoured (no host printing on the device
! path).
module psbx_krylov_shim_mod
  use iso_c_binding
  use psb_base_mod
  use psb_prec_mod, only : psb_dprec_type
  use psb_d_diagprec, only : psb_d_diag_prec_type
  use psb_d_nullprec, only : psb_d_null_prec_type
  use psb_d_cuda_vect_mod, only : psb_d_vect_cuda
  use psb_d_cuda_hlg_mat_mod, only : psb_d_cuda_hlg_sparse_mat
  use psb_d_cuda_elg_mat_mod, only : psb_d_cuda_elg_sparse_mat
  use psb_d_cuda_csrg_mat_mod, only : psb_d_cuda_csrg_sparse_mat
  implicit none
  private
  public :: psbx_krylov_gpu, psbx_solveroptions

  ! the layout of psbx_SolverOptions (include/psbx.h), as the reference's
  ! cbind/krylov/psb_base_krylov_cbind_mod.f90 solveroptions
  type, bind(c) :: psbx_solveroptions
    integer(c_int) :: iter, itmax, itrace, irst, istop
    real(c_double) :: eps, err
  end type psbx_solveroptions

  integer(c_int), parameter :: psbx_fmt_hll = 0, psbx_fmt_ell = 1, psbx_fmt_csr = 2

  interface
    function psbx_dkrylov(method, mat, fmt, dinv, b, x, opt) result(res) &
         & bind(c, name='psbx_dkrylov')
      import :: c_char, c_ptr, c_int, psbx_solveroptions
      character(kind=c_char), dimension(*) :: method
      type(c_ptr), value     :: mat
      integer(c_int), value  :: fmt
      type(c_ptr), value     :: dinv, b, x
      type(psbx_solveroptions) :: opt
      integer(c_int)         :: res
    end function psbx_dkrylov
  end interface

contains

  subroutine psbx_krylov_gpu(method, a, prec, b, x, eps, desc_a, info, &
       & itmax, iter, err, irst, istop, done)
    character(len=*), intent(in)               :: method
    type(psb_dspmat_type), intent(in), target  :: a
    type(psb_dprec_type), intent(inout)        :: prec
    type(psb_d_vect_type), intent(inout)       :: b, x
    real(psb_dpk_), intent(in)                 :: eps
    type(psb_desc_type), intent(in)            :: desc_a
    integer(psb_ipk_), intent(out)             :: info
    integer(psb_ipk_), optional, intent(in)    :: itmax, irst, istop
    integer(psb_ipk_), optional, intent(out)   :: iter
    real(psb_dpk_), optional, intent(out)      :: err
    logical, intent(out)                       :: done

    type(psbx_solveroptions) :: opt
    type(c_ptr)              :: mat, dinv, bp, xp
    integer(c_int)           :: fmt, res
    character(len=20)        :: meth
    type(psb_ctxt_type)      :: ctxt
    integer(psb_ipk_)        :: me, np

    done = .false.
    info = psb_success_
    ctxt = desc_a%get_context()
    call psb_info(ctxt, me, np)
    if (np /= 1) return

    meth = psb_toupper(method)
    opt%itmax  = 1000
    opt%itrace = 0
    opt%istop  = 2
    opt%irst   = 10
    opt%eps    = eps
    opt%iter   = 0
    opt%err    = 0.d0
    if (present(itmax)) opt%itmax = itmax
    if (present(istop)) opt%istop = istop
    select case (trim(meth))
    case ('CG', 'FCG', 'CGS', 'BICG', 'BICGSTAB')
    case ('BICGSTABL')
      opt%irst = 1
      if (present(irst)) opt%irst = irst
    case ('RGMRES', 'GMRES')
      if (present(irst)) opt%irst = irst
      if (opt%istop /= 2) return
    case default
      return
    end select
    if (opt%irst <= 0) return

    ! the matrix, made current on the device
    if (.not. allocated(a%a)) return
    select type (aa => a%a)
    type is (psb_d_cuda_hlg_sparse_mat)
      if (aa%is_host()) call aa%sync()
      mat = aa%deviceMat
      fmt = psbx_fmt_hll
    type is (psb_d_cuda_elg_sparse_mat)
      if (aa%is_host()) call aa%sync()
      mat = aa%deviceMat
      fmt = psbx_fmt_ell
    type is (psb_d_cuda_csrg_sparse_mat)
      if (aa%is_host()) call aa%sync()
      mat = c_loc(aa%deviceMat)          ! d_Cmat, a bind(c) struct holding Mat
      fmt = psbx_fmt_csr
    class default
      return
    end select
    if (.not. c_associated(mat)) return

    ! the preconditioner: DIAG (its inverse diagonal on the device) or NONE
    dinv = c_null_ptr
    if (.not. allocated(prec%prec)) return
    select type (pp => prec%prec)
    type is (psb_d_diag_prec_type)
      if (.not. allocated(pp%dv)) return
      if (.not. allocated(pp%dv%v)) return
      select type (dd => pp%dv%v)
      type is (psb_d_vect_cuda)
        if (dd%is_host()) call dd%sync()
        dinv = dd%deviceVect
      class default
        return
      end select
    type is (psb_d_null_prec_type)
      dinv = c_null_ptr
    class default
      return
    end select

    ! right-hand side and solution vectors
    if (.not. allocated(b%v)) return
    if (.not. allocated(x%v)) return
    select type (bb => b%v)
    type is (psb_d_vect_cuda)
      if (bb%is_host()) call bb%sync()
      bp = bb%deviceVect
    class default
      return
    end select
    select type (xx => x%v)
    type is (psb_d_vect_cuda)
      if (xx%is_host()) call xx%sync()
      xp = xx%deviceVect
    class default
      return
    end select

    res = psbx_dkrylov(trim(meth)//c_null_char, mat, fmt, dinv, bp, xp, opt)
    done = .true.
    if (res /= 0) then
      info = psb_err_from_subroutine_
      call psb_errpush(info, 'psbx_krylov_gpu', a_err='psbx_dkrylov')
      return
    end if
    select type (xx => x%v)
    type is (psb_d_vect_cuda)
      call xx%set_dev()                  ! the solution is on the device
    end select
    if (present(iter)) iter = opt%iter
    if (present(err))  err  = opt%err
  end subroutine psbx_krylov_gpu

end module psbx_krylov_shim_mod
