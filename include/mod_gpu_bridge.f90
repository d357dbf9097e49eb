! ISO_C_BINDING interface of libamrvac_gpu.so (include/amrvac_gpu.h) for the
! MPI-AMRVAC Fortran host.  The host keeps its octree, regrid and I/O; it
! replaces the block loops of advect1 (src/mod_advance.t:611-666) and of
! getdt_courant (src/mod_dt.t:30-52) with one library call each, and maps a
! negative return code to mpistop and a positive status word to crash = .true.
! (src/amrvac.t:312-318).  Compile it with the host (gfortran -c
! mod_gpu_bridge.f90) and link libamrvac_gpu.so; no Fortran compiler exists in
! the build image, so this file is compiled by the host's build only.
module mod_gpu_bridge
  use iso_c_binding
  implicit none
  integer, parameter :: AMRVAC_MAX_NW = 16
  type, bind(c) :: amrvac_cfg
     integer(c_int)  :: ndim, ndir, physics, block_nx(3), nghostcells
     real(c_double)  :: gamma
     integer(c_int)  :: flux_scheme, limiter, typeboundspeed, typedivbfix
     real(c_double)  :: mhd_glm_alpha
     integer(c_int)  :: mhd_glm_extended
     real(c_double)  :: divbdiff, courantpar
     integer(c_int)  :: type_courant
     real(c_double)  :: cada3_radius, tvdlfeps
     integer(c_int)  :: fix_small_values, check_small_values, small_values_method
     real(c_double)  :: small_density, small_pressure
     integer(c_int)  :: time_stepper, ssprk_order
     real(c_double)  :: dtmin
     integer(c_int)  :: typeboundary(AMRVAC_MAX_NW, 6)   ! C [6][16] = Fortran (16,6)
     integer(c_int)  :: zchunk, precision, slowsteps, time_integrator, dimsplit
     real(c_double)  :: schmid_rad(3)
     integer(c_int)  :: schmid_global
     integer(c_int)  :: small_values_daverage
  end type
  interface
     subroutine amrvac_gpu_default_cfg(cfg) bind(c)
       import; type(amrvac_cfg) :: cfg
     end subroutine
     integer(c_int) function amrvac_gpu_create(cfg, ctx) bind(c)
       import; type(amrvac_cfg), intent(in) :: cfg; type(c_ptr) :: ctx
     end function
     integer(c_int) function amrvac_gpu_set_blocks(ctx, nblocks, dx, neighbor) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: nblocks
       real(c_double), intent(in) :: dx(*); integer(c_int), intent(in) :: neighbor(*)
     end function
     integer(c_int) function amrvac_gpu_upload(ctx, reg, first, n, w) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reg, first, n
       real(c_double), intent(in) :: w(*)
     end function
     integer(c_int) function amrvac_gpu_download(ctx, reg, first, n, w) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reg, first, n
       real(c_double) :: w(*)
     end function
     integer(c_int) function amrvac_gpu_getdt(ctx, reg, dt, cmax_global) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reg
       real(c_double) :: dt, cmax_global
     end function
     integer(c_int) function amrvac_gpu_advect1(ctx, reg_ct, reg_new, reg_base, a_base, b_in, &
                                                dtfactor, dt) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reg_ct, reg_new, reg_base
       real(c_double), value :: a_base, b_in, dtfactor, dt
     end function
     integer(c_int) function amrvac_gpu_advect1_dim(ctx, reg_ct, reg_new, reg_base, a_base, b_in, &
                                                    dtfactor, dt, idim) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reg_ct, reg_new, reg_base, idim
       real(c_double), value :: a_base, b_in, dtfactor, dt
     end function
     integer(c_int) function amrvac_gpu_status(ctx, flags) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int32_t) :: flags
     end function
     integer(c_int) function amrvac_gpu_set_amr_grid(ctx, nleaf, leaf, nbase, xprobmin, xprobmax) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: nleaf
       integer(c_int), intent(in) :: leaf(4, *), nbase(3)
       real(c_double), intent(in) :: xprobmin(3), xprobmax(3)
     end function
     integer(c_int) function amrvac_gpu_amr_resettree(ctx, weight, logflag, refine_max_level, &
                                                      refine_threshold, derefine_ratio, amr_wavefilter, &
                                                      changed) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: refine_max_level
       real(c_double), intent(in) :: weight(*), refine_threshold(*), derefine_ratio(*), amr_wavefilter(*)
       integer(c_int), intent(in) :: logflag(*); integer(c_int) :: changed
     end function
     integer(c_int) function amrvac_gpu_amr_leaves(ctx, leaf) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int) :: leaf(4, *)
     end function
     integer(c_int) function amrvac_gpu_destroy(ctx) bind(c)
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function amrvac_gpu_set_cmax_global(ctx, cmax_global) bind(c)
       import; type(c_ptr), value :: ctx; real(c_double), value :: cmax_global
     end function
     integer(c_int) function amrvac_gpu_set_time(ctx, global_time, time_max, dtsave) bind(c)
       import; type(c_ptr), value :: ctx; real(c_double), value :: global_time, time_max, dtsave
     end function
     integer(c_int) function amrvac_gpu_step(ctx) bind(c)
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function amrvac_gpu_run(ctx, nsteps) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: nsteps
     end function
     integer(c_int) function amrvac_gpu_get_time(ctx, dt, cmax_global, global_time) bind(c)
       import; type(c_ptr), value :: ctx; real(c_double) :: dt, cmax_global, global_time
     end function
     ! launch shape: time every stage-kernel variant and work distribution once
     ! after the upload, or set a cached choice
     integer(c_int) function amrvac_gpu_autotune(ctx, reps, best_zchunk, best_ms) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: reps
       integer(c_int) :: best_zchunk; real(c_double) :: best_ms
     end function
     integer(c_int) function amrvac_gpu_set_zchunk(ctx, zchunk) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: zchunk
     end function
     integer(c_int) function amrvac_gpu_set_stage_variant(ctx, var) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int), value :: var
     end function
     integer(c_int) function amrvac_gpu_stage_variant(ctx, var, nvar, threads, ctas_per_sm, async) bind(c)
       import; type(c_ptr), value :: ctx; integer(c_int) :: var, nvar, threads, ctas_per_sm, async
     end function
  end interface
end module mod_gpu_bridge
