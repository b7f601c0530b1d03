! Fortran binding of libasr_b200 (include/asr_b200.h) for the asr code base: a maintainer adds this module to asr's
! src/ and links asr_b200 and cudart.  Every interface mirrors one C prototype of the header argument for argument
! (value scalars, arrays by reference, opaque handles as type(c_ptr)).
module asr_b200
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: ASR_OK = 0, ASR_MODE_PLAIN = 0, ASR_MODE_EDC = 1
  integer(c_int), parameter :: ASR_TAIL_NONE = 0, ASR_TAIL_HULL = 1, ASR_TAIL_BP = 2, ASR_TAIL_AVG2 = 3
  integer(c_int), parameter :: ASR_FP64 = 0, ASR_FP32 = 1
  type, bind(c) :: asr_chain_group
    type(c_ptr) :: c, d, o, e, pa, pb          ! (9, nsp) real(dp) arrays, c_null_ptr for pa/pb in plain mode
    integer(c_int) :: frozen_sp, start_orb, nlev, reserved
  end type
  type, bind(c) :: asr_ed3_group
    type(c_ptr) :: g, d, dc, del, enu, o, p     ! h' of ed3_setup and the ed3_t arrays
    integer(c_int) :: central, start_orb, nlev, reserved
  end type
  interface
    integer(c_int) function asr_ctx_create(device, ctx) bind(c)
      import; integer(c_int), value :: device; type(c_ptr) :: ctx
    end function
    integer(c_int) function asr_op_build(ctx, nsite, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, nop, dmat, &
                                         start, maxlevel, maxrank, flippable, stype, block, nbs, ntb, block0, op) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsite, ncls, ldspc, nsp, nop, start, maxlevel, maxrank, nbs, ntb
      integer(c_int) :: nbr_ptr(*), nbr(*), nsc(*), spc(*), cls(*), perm(*)
      type(c_ptr), value :: flippable, stype          ! c_loc(int array) or c_null_ptr
      real(c_double) :: conc(*), dmat(*), block(*)
      type(c_ptr), value :: block0
      type(c_ptr) :: op
    end function
    integer(c_int) function asr_op_apply(op, x, y, nvec) bind(c)
      import; type(c_ptr), value :: op; real(c_double) :: x(*), y(*); integer(c_int), value :: nvec
    end function
    integer(c_int) function asr_chains_run(ctx, op, groups, ngroup, z, nz, mode, depth_tol, tail, precision, project, &
                                           g, a, b, mused) bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, mode, tail, precision, project
      real(c_double), value :: depth_tol
      complex(c_double_complex) :: z(*), g(*)
      type(c_ptr), value :: a, b, mused
    end function
    integer(c_int) function asr_op_build_targets(ctx, nsite, nbr_ptr, nbr, ncls, nsc, spc, ldspc, conc, nsp, cls, perm, &
                                                 nop, dmat, start, maxlevel, maxrank, flippable, stype, block, nbs, ntb, &
                                                 block0, tsite, ntarget, tnode, tgop, op) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsite, ncls, ldspc, nsp, nop, start, maxlevel, maxrank, nbs, ntb, ntarget
      integer(c_int) :: nbr_ptr(*), nbr(*), nsc(*), spc(*), cls(*), perm(*), tsite(*), tnode(*), tgop(*)
      type(c_ptr), value :: flippable, stype, block0
      real(c_double) :: conc(*), dmat(*), block(*)
      type(c_ptr) :: op
    end function
    integer(c_int) function asr_op_set_params(op, c, d, o, e) bind(c)
      import; type(c_ptr), value :: op; real(c_double) :: c(*), d(*), o(*), e(*)
    end function
    integer(c_int) function asr_op_freeze_site(op, site, sp) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: site, sp
    end function
    integer(c_int) function asr_op_freeze_any(op, site, sp, nfound) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: site, sp; integer(c_int) :: nfound
    end function
    integer(c_int) function asr_op_hp_c(op, x, y, nvec) bind(c)
      import; type(c_ptr), value :: op; complex(c_double_complex) :: x(*), y(*); integer(c_int), value :: nvec
    end function
    integer(c_int) function asr_dos_final(ctx, op, groups, ngroup, comp, spin, lorb, worb, ncomp, nspin, emin, emax, eta, &
                                          ndos, depth_tol, tail, precision, edos_e, edos) bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, ncomp, nspin, ndos, tail, precision
      integer(c_int) :: comp(*), spin(*), lorb(*)
      real(c_double) :: worb(*), edos_e(*), edos(*)
      real(c_double), value :: emin, emax, eta, depth_tol
    end function
    integer(c_int) function asr_ctx_kernel_stats_kind(ctx, kind, ms, launches, bytes, flops) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: kind; real(c_double) :: ms, bytes, flops
      integer(c_int64_t) :: launches
    end function
    integer(c_int) function asr_chains_run_lanes(ctx, op, groups, ngroup, lane_group, lane_z, nlane, depth_tol, tail, &
                                                 precision, project, g, mused) bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nlane, tail, precision, project
      integer(c_int) :: lane_group(*), mused(*)
      complex(c_double_complex) :: lane_z(*), g(*)
      real(c_double), value :: depth_tol
    end function
    integer(c_int) function asr_chains_run_lanes_dev(ctx, op, groups, ngroup, lane_group, lane_z_dev, nlane, depth_tol, &
                                                     tail, precision, project, g_dev) bind(c)
      import
      type(c_ptr), value :: ctx, op, lane_z_dev, g_dev
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nlane, tail, precision, project
      integer(c_int) :: lane_group(*)
      real(c_double), value :: depth_tol
    end function
    integer(c_int) function asr_op_unfreeze(op) bind(c)
      import; type(c_ptr), value :: op
    end function
    integer(c_int) function asr_op_set_start(op, l0) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: l0
    end function
    integer(c_int) function asr_op_set_chi(op, chi) bind(c)
      import; type(c_ptr), value :: op; real(c_double) :: chi(*)
    end function
    integer(c_int) function asr_op_set_class_conc(op, kap, conc) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: kap; real(c_double) :: conc(*)
    end function
    integer(c_int) function asr_op_free(op) bind(c)
      import; type(c_ptr), value :: op
    end function
    integer(c_int) function asr_chains_proj(ctx, op, groups, ngroup, z, nz, tail, precision, project, nt, tnode, tgop, tw, &
                                            g, gp, gp4, mused) bind(c)
      import
      type(c_ptr), value :: ctx, op, mused
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, tail, precision, project, nt
      integer(c_int) :: tnode(*), tgop(*)
      real(c_double) :: tw(*)
      complex(c_double_complex) :: z(*), g(*), gp(*), gp4(*)
    end function
    integer(c_int) function asr_epi_blocks(ctx, op, groups, v9, chi, ngroup, z, nz, tail, precision, project, x, mused) bind(c)
      import
      type(c_ptr), value :: ctx, op, mused
      type(asr_chain_group) :: groups(*)
      real(c_double) :: v9(*), chi(*)
      integer(c_int), value :: ngroup, nz, tail, precision, project
      complex(c_double_complex) :: z(*), x(*)
    end function
    integer(c_int) function asr_ed3_blocks(ctx, op, groups, ngroup, z, nz, depth_tol, tail, precision, project, bk, mused, &
                                           a, b, c) bind(c)
      import
      type(c_ptr), value :: ctx, op, mused, a, b, c
      type(asr_ed3_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, tail, precision, project
      real(c_double), value :: depth_tol
      complex(c_double_complex) :: z(*), bk(*)
    end function
    integer(c_int) function asr_cf_eval(ctx, a, b, m, ld, nchain, z, nz, tail, g, edges, nfall) bind(c)
      import
      type(c_ptr), value :: ctx, edges
      complex(c_double_complex) :: a(*), b(*), z(*), g(*)
      integer(c_int) :: m(*)
      integer(c_int), value :: ld, nchain, nz, tail
      integer(c_int64_t) :: nfall
    end function
    integer(c_int) function asr_contour_nodes(ebot, ef, n, eta_end, z, w) bind(c)
      import; real(c_double), value :: ebot, ef, eta_end; integer(c_int), value :: n
      complex(c_double_complex) :: z(*), w(*)
    end function
    integer(c_int) function asr_contour_moment(z, w, g, n, enu, k, m) bind(c)
      import; complex(c_double_complex) :: z(*), w(*), g(*); integer(c_int), value :: n, k
      real(c_double), value :: enu; real(c_double) :: m
    end function
    integer(c_int) function asr_ctx_destroy(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function asr_last_error(buf, n) bind(c)
      import; character(kind=c_char) :: buf(*); integer(c_size_t), value :: n
    end function
    integer(c_int) function asr_version() bind(c)
      import
    end function
    integer(c_int) function asr_ctx_sync(ctx) bind(c)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function asr_ctx_stats(ctx, nchain, nlev, nfall) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int64_t) :: nchain, nlev, nfall
    end function
    integer(c_int) function asr_ctx_set_stream(ctx, stream) bind(c)
      import; type(c_ptr), value :: ctx, stream
    end function
    integer(c_int) function asr_ctx_profile(ctx, on) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: on
    end function
    integer(c_int) function asr_ctx_hold_workspace(ctx, on) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: on
    end function
    integer(c_int) function asr_ctx_kernel_stats(ctx, ms, launches, bytes, flops) bind(c)
      import; type(c_ptr), value :: ctx; real(c_double) :: ms, bytes, flops; integer(c_int64_t) :: launches
    end function
    integer(c_int) function asr_ctx_launches(ctx, launches) bind(c)
      import; type(c_ptr), value :: ctx; integer(c_int64_t) :: launches
    end function
    integer(c_int) function asr_op_dims(op, dims) bind(c)
      import; type(c_ptr), value :: op; integer(c_int) :: dims(*)
    end function
    integer(c_int) function asr_op_export_tables(op, flipr, flipg, hopr, hopg, lst, site, ncl, level, norb, sq, stab_ptr, &
                                                 stab) bind(c)
      import; type(c_ptr), value :: op
      integer(c_int) :: flipr(*), flipg(*), hopr(*), hopg(*), lst(*), site(*), ncl(*), level(*), stab_ptr(*), stab(*)
      real(c_double) :: norb(*), sq(*)
    end function
    integer(c_int) function asr_op_rand_c(op, par, x, w, nvec) bind(c)
      import; type(c_ptr), value :: op; complex(c_double_complex) :: par(*), x(*), w(*); integer(c_int), value :: nvec
    end function
    integer(c_int) function asr_op_project_c(op, x, nvec) bind(c)
      import; type(c_ptr), value :: op; complex(c_double_complex) :: x(*); integer(c_int), value :: nvec
    end function
    integer(c_int) function asr_chains_run_dev(ctx, op, groups, ngroup, z_dev, nz, mode, depth_tol, tail, precision, project, &
                                               g_dev, a, b, mused) bind(c)
      import
      type(c_ptr), value :: ctx, op, z_dev, g_dev
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, mode, tail, precision, project
      real(c_double), value :: depth_tol
      complex(c_double_complex) :: a(*), b(*)
      integer(c_int) :: mused(*)
    end function
    integer(c_int) function asr_autotune(ctx, op, groups, ngroup, z, nz, precision, levels, tpb, npw, times) bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, precision, levels
      complex(c_double_complex) :: z(*)
      integer(c_int) :: tpb, npw
      real(c_double) :: times(*)
    end function
    integer(c_int) function asr_op_tuning(op, precision, tpb, npw, link, ms) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: precision; integer(c_int) :: tpb, npw, link
      real(c_double) :: ms(*)
    end function
    integer(c_int) function asr_op_set_tuning(op, precision, tpb, npw, link) bind(c)
      import; type(c_ptr), value :: op; integer(c_int), value :: precision, tpb, npw, link
    end function
    integer(c_int) function asr_chains_adjoint(ctx, op, groups, ngroup, z, nz, w, tail, precision, project, stride, g, grad) &
                                               bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, tail, precision, project, stride
      complex(c_double_complex) :: z(*), w(*), g(*), grad(*)
    end function
    integer(c_int) function asr_chains_adjoint_ext(ctx, op, groups, ngroup, z, nz, w, depth_tol, tail, precision, project, &
                                                   stride, g, mused, grad) bind(c)
      import
      type(c_ptr), value :: ctx, op
      type(asr_chain_group) :: groups(*)
      integer(c_int), value :: ngroup, nz, tail, precision, project, stride
      real(c_double), value :: depth_tol
      complex(c_double_complex) :: z(*), w(*), g(*), grad(*)
      integer(c_int) :: mused(*)
    end function
    integer(c_int) function asr_cf_eval_noalloc(ctx, a, b, m, ld, nchain, z, nz, tail, g, nfall) bind(c)
      import
      type(c_ptr), value :: ctx
      complex(c_double_complex) :: a(*), b(*), z(*), g(*)
      integer(c_int) :: m(*)
      integer(c_int), value :: ld, nchain, nz, tail
      integer(c_int64_t) :: nfall
    end function
    integer(c_int) function asr_cf_adjoint(a, b, m, zr, zi, tail, wr, wi, abar, bbar, g) bind(c)
      import
      complex(c_double_complex) :: a(*), b(*), abar(*), bbar(*), g
      integer(c_int), value :: m, tail
      real(c_double), value :: zr, zi, wr, wi
    end function
    integer(c_int) function asr_supercell_build(ctx, nsite, nslot, nbr, spc, nsp, c, d, o, e, block, block0, sc) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsite, nslot, nsp
      integer(c_int) :: nbr(*), spc(*)
      real(c_double) :: c(*), d(*), o(*), e(*), block(*), block0(*)
      type(c_ptr) :: sc
    end function
    integer(c_int) function asr_supercell_free(sc) bind(c)
      import; type(c_ptr), value :: sc
    end function
    integer(c_int) function asr_supercell_apply(sc, x, y, nvec) bind(c)
      import; type(c_ptr), value :: sc; real(c_double) :: x(*), y(*); integer(c_int), value :: nvec
    end function
    integer(c_int) function asr_kpm_moments(ctx, sc, cen, scl, nmom, v0, nvec, seed, precision, doubling, mu) bind(c)
      import
      type(c_ptr), value :: ctx, sc
      real(c_double), value :: cen, scl
      integer(c_int), value :: nmom, v0, nvec, precision, doubling
      integer(c_int64_t), value :: seed
      real(c_double) :: mu(*)
    end function
    integer(c_int) function asr_kpm_dos(mu, nmom, cen, scl, e, ne, rho) bind(c)
      import
      real(c_double) :: mu(*), e(*), rho(*)
      integer(c_int), value :: nmom, ne
      real(c_double), value :: cen, scl
    end function
    integer(c_int) function asr_sro_layout(nsite, z, nbr, ldnbr, nsp, conc, alpha, seed, sweeps, spc, alpha_out) bind(c)
      import
      integer(c_int), value :: nsite, z, ldnbr, nsp, sweeps
      integer(c_int) :: nbr(*), spc(*)
      real(c_double) :: conc(*), alpha(*), alpha_out(*)
      integer(c_int64_t), value :: seed
    end function
    integer(c_int) function asr_gauss_legendre(n, x, w) bind(c)
      import; integer(c_int), value :: n; real(c_double) :: x(*), w(*)
    end function
    integer(c_int) function asr_contour_nodes_closed(ebot, ef, eta, n_arc, n_vert, z, w) bind(c)
      import; real(c_double), value :: ebot, ef, eta; integer(c_int), value :: n_arc, n_vert
      complex(c_double_complex) :: z(*), w(*)
    end function
    integer(c_int) function asr_contour_nodes_fermi(ebot, mu, kt, npole, n_main, n_step, z, w) bind(c)
      import; real(c_double), value :: ebot, mu, kt; integer(c_int), value :: npole, n_main, n_step
      complex(c_double_complex) :: z(*), w(*)
    end function
  end interface
end module asr_b200
