! spex_gpu.f90 - ISO_C_BINDING interfaces of libspexgpu (include/spexgpu.h) for
! the SPEX Fortran driver. Every routine returns an integer(c_int) status,
! 0 on success; spx_last_error gives the message of the last failure.
!
! Arrays are passed exactly as SPEX holds them: cprod(npair, nbas) and
! susceph(nbas*(nbas+1)/2, nfrqh) as complex(c_double_complex), column-major.
!
! This module is interface-only; it is not compiled in the build image (no
! Fortran compiler is installed there).
module spex_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SPX_OK = 0, SPX_EINVAL = -1, SPX_ENOMEM = -2, &
                               SPX_ECUDA = -3, SPX_ETIMEOUT = -4, SPX_ENOTSUP = -5, &
                               SPX_ENODEV = -6
  integer(c_int), parameter :: SPX_FP64 = 0, SPX_SPLIT = 1
  integer(c_int), parameter :: SPX_PRODUCTS_AUTO = 0, SPX_PRODUCTS_FP64 = 1, SPX_PRODUCTS_SPLIT = 2

  type, bind(c) :: spx_options
    integer(c_int32_t) :: struct_size = 40
    integer(c_int32_t) :: verbose = 0
    integer(c_int64_t) :: workspace_limit = 0
    integer(c_int64_t) :: pinned_limit = 0
    integer(c_int32_t) :: chunk_pairs = 0
    integer(c_int32_t) :: timeout_ms = 0
    integer(c_int32_t) :: split_variant = 0
    integer(c_int32_t) :: products = 0           ! SPX_PRODUCTS_AUTO / _FP64 / _SPLIT
  end type

  type, bind(c) :: spx_chi0_stats
    real(c_double)     :: ms_total, ms_gram, ms_prep, flops
    integer(c_int64_t) :: h2d_bytes, d2h_bytes
    integer(c_int32_t) :: kernel_launches, precision
  end type

  ! spx_mt_desc / spx_pw_desc: host descriptors of the product basis (c_loc of
  ! Fortran arrays); the coefficient and cprod pointers of the _dev calls are
  ! device addresses (e.g. from an OpenACC host_data or CUDA Fortran device array)
  type, bind(c) :: spx_mt_desc
    integer(c_int32_t) :: natom, lcut, nrad, lcutm, nradm, ld1
    type(c_ptr) :: gaunt, integral, cexp
  end type

  type, bind(c) :: spx_pw_desc
    integer(c_int32_t) :: ngpt1, ngpt2, ngptm, step_radius
    type(c_ptr) :: gpt1, gpt2, gptm
    integer(c_int32_t) :: gshift(3)
    integer(c_int32_t) :: nfft = 0               ! 0 explicit convolution, n: FFT branch
    type(c_ptr) :: cstep
    real(c_double) :: vol
  end type

  type, bind(c) :: spx_q_desc
    integer(c_int32_t) :: nbas, variant = 0
    integer(c_int64_t) :: npair
    integer(c_int32_t) :: slab_pairs = 0, reserved0 = 0
    type(c_ptr) :: cprod                         ! device, or c_null_ptr = generated
    integer(c_int64_t) :: ldc
    integer(c_int64_t) :: seed                   ! uint64 in C
    integer(c_int32_t) :: stream_id, reserved1 = 0
    real(c_double) :: m_scale
    type(c_ptr) :: ediff, wscale
    real(c_double) :: scale_all
    type(c_ptr) :: susceph
  end type

  integer(c_int), parameter :: SPX_BATCH_AUTOTUNE = 1, SPX_BATCH_NOGRAPH = 2

  interface
    integer(c_int) function spx_ctx_create(device, opt, ctx) bind(c, name='spx_ctx_create')
      import :: c_int, c_ptr, spx_options
      integer(c_int), value :: device
      type(spx_options), intent(in) :: opt
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function spx_ctx_destroy(ctx) bind(c, name='spx_ctx_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    type(c_ptr) function spx_last_error(ctx) bind(c, name='spx_last_error')
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function

    ! replaces src/susceptibility.f:950-975 (weights) and :1182-1240 (body loop)
    integer(c_int) function spx_chi0_accumulate(ctx, cprod, ldc, npair, nbas, ediff, wscale, &
                                                scale_all, nw, omega, precision, susceph, stats) &
                                                bind(c, name='spx_chi0_accumulate')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double, c_double_complex, spx_chi0_stats
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: cprod(*)
      integer(c_int64_t), value :: ldc, npair
      integer(c_int32_t), value :: nbas
      real(c_double), intent(in) :: ediff(*)
      type(c_ptr), value :: wscale                 ! c_loc(wscale) or c_null_ptr
      real(c_double), value :: scale_all
      integer(c_int32_t), value :: nw
      real(c_double), intent(in) :: omega(*)
      integer(c_int32_t), value :: precision
      complex(c_double_complex), intent(inout) :: susceph(*)
      type(spx_chi0_stats), intent(out) :: stats
    end function

    ! replaces wavefproducts2_mt, src/wavefproducts.f:95-431 (device arrays)
    integer(c_int) function spx_wfprod_mt_dev(ctx, mt, nk, nocc, nunocc, cmt_occ, cmt_unocc, &
                                              cprod, ldc, stream) bind(c, name='spx_wfprod_mt_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, spx_mt_desc
      type(c_ptr), value :: ctx
      type(spx_mt_desc), intent(in) :: mt
      integer(c_int32_t), value :: nk, nocc, nunocc
      type(c_ptr), value :: cmt_occ, cmt_unocc, cprod, stream
      integer(c_int64_t), value :: ldc
    end function

    ! replaces the explicit-convolution wavefproducts2_pw, src/wavefproducts.f:760-997
    integer(c_int) function spx_wfprod_pw_dev(ctx, pw, nk, nocc, nunocc, cpw_occ, cpw_unocc, &
                                              cprod, ldc, col0, stream) bind(c, name='spx_wfprod_pw_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, spx_pw_desc
      type(c_ptr), value :: ctx
      type(spx_pw_desc), intent(in) :: pw
      integer(c_int32_t), value :: nk, nocc, nunocc, col0
      type(c_ptr), value :: cpw_occ, cpw_unocc, cprod, stream
      integer(c_int64_t), value :: ldc
    end function

    ! the packet loop src/susceptibility.f:751-1276 from coefficients to chi0
    integer(c_int) function spx_chi0_from_coeffs_dev(ctx, mt, pw, nk, nocc, nunocc, cmt_occ, &
        cmt_unocc, cpw_occ, cpw_unocc, ediff, wscale, scale_all, nw, omega, precision, susceph, &
        stream, stats) bind(c, name='spx_chi0_from_coeffs_dev')
      import :: c_int, c_int32_t, c_ptr, c_double, spx_mt_desc, spx_pw_desc, spx_chi0_stats
      type(c_ptr), value :: ctx
      type(spx_mt_desc), intent(in) :: mt
      type(spx_pw_desc), intent(in) :: pw
      integer(c_int32_t), value :: nk, nocc, nunocc, nw, precision
      type(c_ptr), value :: cmt_occ, cmt_unocc, cpw_occ, cpw_unocc, ediff, wscale, omega, susceph
      real(c_double), value :: scale_all
      type(c_ptr), value :: stream
      type(spx_chi0_stats), intent(out) :: stats
    end function

    ! Hilbert-mesh weights, src/susceptibility.f:996-1078 + src/hilbert.f:193-300
    integer(c_int) function spx_weights_hilbert_dev(ctx, npair, nfrqs, wtetra, ldt, thr, nw, wghtSr, &
                                                    scale_all, w, ldw, stream) bind(c, name='spx_weights_hilbert_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: ctx, wtetra, wghtSr, w, stream
      integer(c_int64_t), value :: npair, ldt, ldw
      integer(c_int32_t), value :: nfrqs, nw
      real(c_double), value :: thr, scale_all
    end function

    integer(c_int) function spx_chi0_accumulate_w_dev(ctx, cprod, ldc, npair, nbas, w, ldw, nw, &
        precision, susceph, stream, stats) bind(c, name='spx_chi0_accumulate_w_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, spx_chi0_stats
      type(c_ptr), value :: ctx, cprod, w, susceph, stream
      integer(c_int64_t), value :: ldc, npair, ldw
      integer(c_int32_t), value :: nbas, nw, precision
      type(spx_chi0_stats), intent(out) :: stats
    end function

    ! q -> 0 head and wings, src/susceptibility.f:1092-1157 (device arrays)
    integer(c_int) function spx_headwings_dev(ctx, cprod, ldc, npair, dim, dcprod, ldd, w, ldw, nw, &
                                              head, wing, stream) bind(c, name='spx_headwings_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx, cprod, dcprod, w, head, wing, stream
      integer(c_int64_t), value :: ldc, npair, ldd, ldw
      integer(c_int32_t), value :: dim, nw
    end function

    ! dielectric matrix and inverse, src/correlation.f:614-636, 703-745 (device arrays)
    integer(c_int) function spx_dielec_dev(ctx, nbas, nw, susceph, coul, invert, head, wing, stream) &
                                           bind(c, name='spx_dielec_dev')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx, susceph, coul, head, wing, stream
      integer(c_int32_t), value :: nbas, nw, invert
    end function

    ! transform to the Coulomb eigenbasis, src/susceptibility.f:806-832 (device arrays)
    integer(c_int) function spx_trafo_dev(ctx, cprod, ldc, npair, nbas, ctrafo, ldt, dim, out, &
                                          ldo, stream) bind(c, name='spx_trafo_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx, cprod, ctrafo, out, stream
      integer(c_int64_t), value :: ldc, npair, ldt, ldo
      integer(c_int32_t), value :: nbas, dim
    end function

    ! device-pointer form of spx_chi0_accumulate (device arrays, caller stream)
    integer(c_int) function spx_chi0_accumulate_dev(ctx, cprod, ldc, npair, nbas, ediff, wscale, &
        scale_all, nw, omega, precision, susceph, stream, stats) &
        bind(c, name='spx_chi0_accumulate_dev')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double, spx_chi0_stats
      type(c_ptr), value :: ctx, cprod, ediff, wscale, omega, susceph, stream
      integer(c_int64_t), value :: ldc, npair
      integer(c_int32_t), value :: nbas, nw, precision
      real(c_double), value :: scale_all
      type(spx_chi0_stats), intent(out) :: stats
    end function

    ! allocation-free FP64 accumulation (no counterpart in the reference): for hosts
    ! whose device heap belongs to their offload runtime; no context, static scratch,
    ! nw <= 262144, nbas <= 46340, never inside a stream capture
    integer(c_int) function spx_chi0_accumulate_dev_noalloc(cprod, ldc, npair, nbas, ediff, &
        wscale, scale_all, nw, omega, susceph, stream) &
        bind(c, name='spx_chi0_accumulate_dev_noalloc')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: cprod, ediff, wscale, omega, susceph, stream
      integer(c_int64_t), value :: ldc, npair
      integer(c_int32_t), value :: nbas, nw
      real(c_double), value :: scale_all
    end function

    ! the q loop around susceptibility, src/correlation.f:293-339
    integer(c_int) function spx_chi0_batched(ctx, nq, q, nw, omega, precision, flags, stream, &
                                             stats) bind(c, name='spx_chi0_batched')
      import :: c_int, c_int32_t, c_ptr, spx_q_desc, spx_chi0_stats
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nq, nw, precision, flags
      type(spx_q_desc), intent(in) :: q(*)
      type(c_ptr), value :: omega, stream
      type(spx_chi0_stats), intent(out) :: stats
    end function
  end interface
end module spex_gpu
