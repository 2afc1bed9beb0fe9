!+++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++
!
!   glissade_velo_higher_pcg_gpu.F90
!
!   Drop-in replacements for the four native PCG solvers of
!   libglissade/glissade_velo_higher_pcg.F90 that run on a B200 through the
!   C ABI of libcismgpu.so (include/cismgpu.h).  Every subroutine keeps the
!   reference argument list, intents and meaning:
!     pcg_solver_standard_2d   (:67-823)     pcg_solver_standard_3d   (:827-1537)
!     pcg_solver_chrongear_2d  (:1541-2628)  pcg_solver_chrongear_3d  (:2632-3594)
!   and, for the steps around the solve in the Picard loop of
!   libglissade/glissade_velo_higher.F90 (module procedures there, so a caller
!   takes these with "use glissade_velo_higher_pcg_gpu, only: gpu_x => x"):
!     compute_residual_vector_2d   (:9502-9689)    compute_residual_vector_3d   (:9693-9894)
!     compute_residual_velocity_2d (:10188-10310)  compute_residual_velocity_3d (:10314-10446)
!     check_symmetry_assembled_matrix_2d (:10648-10850)
!     check_symmetry_assembled_matrix_3d (:10854-11117)
!     assemble_stiffness_matrix_3d (:5382-5643), assemble_stiffness_matrix_2d (:4961-5378, SSA)
!     dirichlet_boundary_conditions_3d (:9305-9498), dirichlet_boundary_conditions_2d (:9133-9301)
!     basal_sliding_bc_3d (:8815-9129), basal_sliding_bc_2d (:8281-8531), local form
!   A nonzero library status is reported the way the reference reports a failed
!   solve: write_log(message, GM_FATAL).
!
!   type(parallel_type) is not interoperable, so the fields the path reads
!   (libglimmer/parallel_mpi.F90:78-153) are copied into a bind(C) struct.
!   logical arrays are passed as the 4-byte Fortran default logical; the library
!   treats any nonzero value as .true.
!
!   Build: compile with the CISM sources and link libcismgpu.so, e.g. add
!   "-L<path>/cism_b200/_lib -lcismgpu" to CISM_EXTRA_LIBS
!   (builds/linux-gnu/linux-gnu-cmake:56).
!
!+++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++++

  module glissade_velo_higher_pcg_gpu

    use, intrinsic :: iso_c_binding
    use glimmer_global, only: dp
    use glimmer_log
    use cism_parallel, only: parallel_type

    implicit none
    private
    public :: pcg_solver_standard_2d, pcg_solver_standard_3d, &
              pcg_solver_chrongear_2d, pcg_solver_chrongear_3d, &
              compute_residual_vector_2d, compute_residual_vector_3d, &
              compute_residual_velocity_2d, compute_residual_velocity_3d, &
              check_symmetry_assembled_matrix_2d, check_symmetry_assembled_matrix_3d, &
              assemble_stiffness_matrix_2d, assemble_stiffness_matrix_3d, &
              dirichlet_boundary_conditions_2d, dirichlet_boundary_conditions_3d, &
              basal_sliding_bc_2d, basal_sliding_bc_3d, &
              cismgpu_use_mixed_precision, cismgpu_use_reference_sum_order

    type, bind(C) :: cismgpu_par_t
       integer(c_int32_t) :: staggered_ilo, staggered_ihi
       integer(c_int32_t) :: staggered_jlo, staggered_jhi
       integer(c_int32_t) :: periodic_bc, outflow_bc, no_ice_bc
       integer(c_int32_t) :: reprosum
       integer(c_int32_t) :: tasks_row, tasks_col
    end type cismgpu_par_t

    interface
       integer(c_int) function c_pcg_standard_3d(nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, &
            Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond, ncheck, tol, maxiters, err, niters,        &
            itest, jtest, rtest) bind(C, name="cismgpu_pcg_standard_3d")
         import :: c_int, c_double, c_int32_t, cismgpu_par_t
         integer(c_int), value :: nx, ny, nz
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), indxA_3d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
         real(c_double), intent(inout) :: xu(*), xv(*)
         integer(c_int), value :: precond, ncheck, maxiters, itest, jtest, rtest
         real(c_double), value :: tol
         real(c_double), intent(out) :: err
         integer(c_int), intent(out) :: niters
       end function c_pcg_standard_3d

       integer(c_int) function c_pcg_chrongear_3d(nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, &
            Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond, ncheck, tol, maxiters, err, niters,         &
            itest, jtest, rtest) bind(C, name="cismgpu_pcg_chrongear_3d")
         import :: c_int, c_double, c_int32_t, cismgpu_par_t
         integer(c_int), value :: nx, ny, nz
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), indxA_3d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
         real(c_double), intent(inout) :: xu(*), xv(*)
         integer(c_int), value :: precond, ncheck, maxiters, itest, jtest, rtest
         real(c_double), value :: tol
         real(c_double), intent(out) :: err
         integer(c_int), intent(out) :: niters
       end function c_pcg_chrongear_3d

       integer(c_int) function c_pcg_standard_2d(nx, ny, par, indxA_2d, active_vertex,               &
            Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond, ncheck, tol, maxiters, err, niters,        &
            itest, jtest, rtest) bind(C, name="cismgpu_pcg_standard_2d")
         import :: c_int, c_double, c_int32_t, cismgpu_par_t
         integer(c_int), value :: nx, ny
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
         real(c_double), intent(inout) :: xu(*), xv(*)
         integer(c_int), value :: precond, ncheck, maxiters, itest, jtest, rtest
         real(c_double), value :: tol
         real(c_double), intent(out) :: err
         integer(c_int), intent(out) :: niters
       end function c_pcg_standard_2d

       integer(c_int) function c_pcg_chrongear_2d(nx, ny, par, indxA_2d, active_vertex,              &
            Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond, ncheck, tol, maxiters, err, niters,        &
            itest, jtest, rtest) bind(C, name="cismgpu_pcg_chrongear_2d")
         import :: c_int, c_double, c_int32_t, cismgpu_par_t
         integer(c_int), value :: nx, ny
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
         real(c_double), intent(inout) :: xu(*), xv(*)
         integer(c_int), value :: precond, ncheck, maxiters, itest, jtest, rtest
         real(c_double), value :: tol
         real(c_double), intent(out) :: err
         integer(c_int), intent(out) :: niters
       end function c_pcg_chrongear_2d

       integer(c_int) function c_set_oneshot_algorithm(algorithm) &
            bind(C, name="cismgpu_set_oneshot_algorithm")
         import :: c_int
         integer(c_int), value :: algorithm
       end function c_set_oneshot_algorithm

       integer(c_int) function c_set_sum_order(order) bind(C, name="cismgpu_set_sum_order")
         import :: c_int
         integer(c_int), value :: order
       end function c_set_sum_order

       type(c_ptr) function c_last_error() bind(C, name="cismgpu_last_error")
         import :: c_ptr
       end function c_last_error

       integer(c_int) function c_resid_vector_3d(nx, ny, nz, par, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, &
            bu, bv, uvel, vvel, resid_u, resid_v, L2_norm, L2_norm_relative)                          &
            bind(C, name="cismgpu_compute_residual_vector_3d")
         import :: c_int, c_double, c_int32_t, c_ptr, cismgpu_par_t
         integer(c_int), value :: nx, ny, nz
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_3d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*), uvel(*), vvel(*)
         real(c_double), intent(out) :: resid_u(*), resid_v(*), L2_norm
         type(c_ptr), value :: L2_norm_relative
       end function c_resid_vector_3d

       integer(c_int) function c_resid_vector_2d(nx, ny, par, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, &
            bu, bv, uvel, vvel, resid_u, resid_v, L2_norm, L2_norm_relative)                      &
            bind(C, name="cismgpu_compute_residual_vector_2d")
         import :: c_int, c_double, c_int32_t, c_ptr, cismgpu_par_t
         integer(c_int), value :: nx, ny
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*), uvel(*), vvel(*)
         real(c_double), intent(out) :: resid_u(*), resid_v(*), L2_norm
         type(c_ptr), value :: L2_norm_relative
       end function c_resid_vector_2d

       integer(c_int) function c_resid_velocity_3d(whichresid, nx, ny, nz, par, uvel, vvel, usav, vsav, &
            resid_velo) bind(C, name="cismgpu_compute_residual_velocity_3d")
         import :: c_int, c_double, cismgpu_par_t
         integer(c_int), value :: whichresid, nx, ny, nz
         type(cismgpu_par_t), intent(in) :: par
         real(c_double), intent(in) :: uvel(*), vvel(*), usav(*), vsav(*)
         real(c_double), intent(out) :: resid_velo
       end function c_resid_velocity_3d

       integer(c_int) function c_resid_velocity_2d(whichresid, nx, ny, par, uvel, vvel, usav, vsav, &
            resid_velo) bind(C, name="cismgpu_compute_residual_velocity_2d")
         import :: c_int, c_double, cismgpu_par_t
         integer(c_int), value :: whichresid, nx, ny
         type(cismgpu_par_t), intent(in) :: par
         real(c_double), intent(in) :: uvel(*), vvel(*), usav(*), vsav(*)
         real(c_double), intent(out) :: resid_velo
       end function c_resid_velocity_2d

       integer(c_int) function c_check_symmetry_3d(nx, ny, nz, par, indxA_3d, active_vertex, Auu, Auv, Avu, &
            Avv, maxdiff, nwarn) bind(C, name="cismgpu_check_symmetry_assembled_matrix_3d")
         import :: c_int, c_double, c_int32_t, c_long_long, cismgpu_par_t
         integer(c_int), value :: nx, ny, nz
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_3d(*), active_vertex(*)
         real(c_double), intent(inout) :: Auu(*), Auv(*), Avu(*), Avv(*)
         real(c_double), intent(out) :: maxdiff
         integer(c_long_long), intent(out) :: nwarn
       end function c_check_symmetry_3d

       integer(c_int) function c_check_symmetry_2d(nx, ny, par, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, &
            maxdiff, nwarn) bind(C, name="cismgpu_check_symmetry_assembled_matrix_2d")
         import :: c_int, c_double, c_int32_t, c_long_long, cismgpu_par_t
         integer(c_int), value :: nx, ny
         type(cismgpu_par_t), intent(in) :: par
         integer(c_int32_t), intent(in) :: indxA_2d(*), active_vertex(*)
         real(c_double), intent(in) :: Auu(*), Auv(*), Avu(*), Avv(*)
         real(c_double), intent(out) :: maxdiff
         integer(c_long_long), intent(out) :: nwarn
       end function c_check_symmetry_2d

       integer(c_int) function c_assemble_3d(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel, vvel, &
            stagusrf, stagthck, flwafact, whichapprox, whichefvs, efvs_constant, effstrain_min, n_glen, indxA_3d, &
            efvs, Auu, Auv, Avu, Avv) bind(C, name="cismgpu_assemble_stiffness_matrix_3d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo, whichapprox, whichefvs
         real(c_double), intent(in) :: sigma(*), xVertex(*), yVertex(*), uvel(*), vvel(*), stagusrf(*), &
              stagthck(*), flwafact(*)
         integer(c_int32_t), intent(in) :: active_cell(*), indxA_3d(*)
         real(c_double), value :: efvs_constant, effstrain_min, n_glen
         real(c_double), intent(out) :: efvs(*), Auu(*), Auv(*), Avu(*), Avv(*)
       end function c_assemble_3d

       integer(c_int) function c_assemble_2d(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, &
            vvel_2d, stagthck, flwafact, whichefvs, efvs_constant, effstrain_min, n_glen, indxA_2d, efvs, Auu, Auv, &
            Avu, Avv) bind(C, name="cismgpu_assemble_stiffness_matrix_2d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo, whichefvs
         real(c_double), intent(in) :: sigma(*), xVertex(*), yVertex(*), uvel_2d(*), vvel_2d(*), stagthck(*), &
              flwafact(*)
         integer(c_int32_t), intent(in) :: active_cell(*), indxA_2d(*)
         real(c_double), value :: efvs_constant, effstrain_min, n_glen
         real(c_double), intent(out) :: efvs(*), Auu(*), Auv(*), Avu(*), Avv(*)
       end function c_assemble_2d

       integer(c_int) function c_assemble_2d_diva(nx, ny, nz, nhalo, sigma, stagsigma, active_cell, xVertex, &
            yVertex, uvel_2d, vvel_2d, stagthck, thck, btractx, btracty, dsfx, dsfy, flwafact, whichefvs, &
            efvs_constant, effstrain_min, n_glen, indxA_2d, efvs_qp_3d, efvs, omega_k, omega, Auu, Auv, Avu, Avv) &
            bind(C, name="cismgpu_assemble_stiffness_matrix_2d_diva")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo, whichefvs
         real(c_double), intent(in) :: sigma(*), stagsigma(*), xVertex(*), yVertex(*), uvel_2d(*), vvel_2d(*), &
              stagthck(*), thck(*), btractx(*), btracty(*), dsfx(*), dsfy(*), flwafact(*)
         integer(c_int32_t), intent(in) :: active_cell(*), indxA_2d(*)
         real(c_double), value :: efvs_constant, effstrain_min, n_glen
         real(c_double), intent(inout) :: efvs_qp_3d(*), omega_k(*), omega(*)
         real(c_double), intent(out) :: efvs(*), Auu(*), Auv(*), Avu(*), Avv(*)
       end function c_assemble_2d_diva

       integer(c_int) function c_assemble_2d_l1l2(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, &
            uvel_2d, vvel_2d, stagthck, dusrf_dx, dusrf_dy, flwa, flwafact, whichefvs, efvs_constant, &
            effstrain_min, n_glen, indxA_2d, efvs, Auu, Auv, Avu, Avv) &
            bind(C, name="cismgpu_assemble_stiffness_matrix_2d_l1l2")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo, whichefvs
         real(c_double), intent(in) :: sigma(*), xVertex(*), yVertex(*), uvel_2d(*), vvel_2d(*), stagthck(*), &
              dusrf_dx(*), dusrf_dy(*), flwa(*), flwafact(*)
         integer(c_int32_t), intent(in) :: active_cell(*), indxA_2d(*)
         real(c_double), value :: efvs_constant, effstrain_min, n_glen
         real(c_double), intent(out) :: efvs(*), Auu(*), Auv(*), Avu(*), Avv(*)
       end function c_assemble_2d_l1l2

       integer(c_int) function c_dirichlet_3d(nx, ny, nz, nhalo, active_vertex, umask, vmask, uvel, vvel, &
            indxA_3d, Auu, Auv, Avu, Avv, bu, bv) bind(C, name="cismgpu_dirichlet_boundary_conditions_3d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo
         integer(c_int32_t), intent(in) :: active_vertex(*), umask(*), vmask(*), indxA_3d(*)
         real(c_double), intent(in) :: uvel(*), vvel(*)
         real(c_double), intent(inout) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
       end function c_dirichlet_3d

       integer(c_int) function c_dirichlet_2d(nx, ny, nhalo, active_vertex, umask, vmask, uvel, vvel, &
            indxA_2d, Auu, Auv, Avu, Avv, bu, bv) bind(C, name="cismgpu_dirichlet_boundary_conditions_2d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nhalo
         integer(c_int32_t), intent(in) :: active_vertex(*), umask(*), vmask(*), indxA_2d(*)
         real(c_double), intent(in) :: uvel(*), vvel(*)
         real(c_double), intent(inout) :: Auu(*), Auv(*), Avu(*), Avv(*), bu(*), bv(*)
       end function c_dirichlet_2d

       integer(c_int) function c_basal_3d(nx, ny, nz, nhalo, dx, dy, active_cell, active_vertex, beta, lsrf, &
            xVertex, yVertex, whichassemble_beta, indxA_3d, Auu, Avv) bind(C, name="cismgpu_basal_sliding_bc_3d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nz, nhalo, whichassemble_beta
         real(c_double), value :: dx, dy
         integer(c_int32_t), intent(in) :: active_cell(*), active_vertex(*), indxA_3d(*)
         real(c_double), intent(in) :: beta(*), lsrf(*), xVertex(*), yVertex(*)
         real(c_double), intent(inout) :: Auu(*), Avv(*)
       end function c_basal_3d

       integer(c_int) function c_basal_2d(nx, ny, nhalo, dx, dy, active_cell, active_vertex, beta, xVertex, &
            yVertex, whichassemble_beta, indxA_2d, Auu, Avv) bind(C, name="cismgpu_basal_sliding_bc_2d")
         import :: c_int, c_double, c_int32_t
         integer(c_int), value :: nx, ny, nhalo, whichassemble_beta
         real(c_double), value :: dx, dy
         integer(c_int32_t), intent(in) :: active_cell(*), active_vertex(*), indxA_2d(*)
         real(c_double), intent(in) :: beta(*), xVertex(*), yVertex(*)
         real(c_double), intent(inout) :: Auu(*), Avv(*)
       end function c_basal_2d
    end interface

  contains

    !-----------------------------------------------------------------------
    ! .true.: all four solvers run the mixed-precision persistent
    ! Chronopoulos-Gear solver (FP32 recurrences, FP64 solution and residual
    ! checks); .false. (default): the reference algorithms in FP64.
    subroutine cismgpu_use_mixed_precision(on)
      logical, intent(in) :: on
      integer(c_int) :: prev
      if (on) then
         prev = c_set_oneshot_algorithm(2_c_int)
      else
         prev = c_set_oneshot_algorithm(-1_c_int)
      endif
    end subroutine cismgpu_use_mixed_precision

    !-----------------------------------------------------------------------
    ! .true.: without parallel%reprosum, the FP64 solvers' global sums run in
    ! the reference's own sequential order (parallel_global_sum_stagger's loop),
    ! so a solve reproduces the CPU run bit for bit (slower); .false.
    ! (default): the library's fixed reduction tree.
    subroutine cismgpu_use_reference_sum_order(on)
      logical, intent(in) :: on
      integer(c_int) :: prev
      prev = c_set_sum_order(merge(1_c_int, 0_c_int, on))
    end subroutine cismgpu_use_reference_sum_order

    function to_c(parallel) result(p)
      type(parallel_type), intent(in) :: parallel
      type(cismgpu_par_t) :: p
      p%staggered_ilo = parallel%staggered_ilo
      p%staggered_ihi = parallel%staggered_ihi
      p%staggered_jlo = parallel%staggered_jlo
      p%staggered_jhi = parallel%staggered_jhi
      p%periodic_bc = merge(1, 0, parallel%periodic_bc)
      p%outflow_bc  = merge(1, 0, parallel%outflow_bc)
      p%no_ice_bc   = merge(1, 0, parallel%no_ice_bc)
      p%reprosum    = merge(1, 0, parallel%reprosum)
      p%tasks_row   = parallel%tasks_row
      p%tasks_col   = parallel%tasks_col
    end function to_c

    subroutine check(status)
      integer(c_int), intent(in) :: status
      character(kind=c_char), pointer :: msg(:)
      character(len=256) :: text
      integer :: n
      if (status == 0) return
      call c_f_pointer(c_last_error(), msg, [256])
      text = ' '
      do n = 1, 256
         if (msg(n) == c_null_char) exit
         text(n:n) = msg(n)
      enddo
      call write_log('GPU PCG solver has failed: '//trim(text), GM_FATAL)
    end subroutine check

    !-----------------------------------------------------------------------
    subroutine pcg_solver_standard_3d(nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, &
                                      Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,             &
                                      linear_solve_ncheck, tolerance, maxiters, err, niters,   &
                                      itest, jtest, rtest)
      integer, intent(in) :: nx, ny, nz
      type(parallel_type), intent(in) :: parallel
      integer, dimension(-1:1,-1:1), intent(in) :: indxA_2d
      integer, dimension(-1:1,-1:1,-1:1), intent(in) :: indxA_3d
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(27,nz,nx-1,ny-1), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nz,nx-1,ny-1), intent(in) :: bu, bv
      real(dp), dimension(nz,nx-1,ny-1), intent(inout) :: xu, xv
      integer, intent(in) :: precond, linear_solve_ncheck, maxiters
      real(dp), intent(in) :: tolerance
      real(dp), intent(out) :: err
      integer, intent(out) :: niters
      integer, intent(in) :: itest, jtest, rtest
      integer(c_int32_t) :: act(nx-1,ny-1)
      act = merge(1, 0, active_vertex)
      call check(c_pcg_standard_3d(nx, ny, nz, to_c(parallel), indxA_2d, indxA_3d, act, Auu, Auv, Avu, Avv, &
                                   bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters,      &
                                   err, niters, itest, jtest, rtest))
    end subroutine pcg_solver_standard_3d

    !-----------------------------------------------------------------------
    subroutine pcg_solver_chrongear_3d(nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, &
                                       Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,             &
                                       linear_solve_ncheck, tolerance, maxiters, err, niters,   &
                                       itest, jtest, rtest)
      integer, intent(in) :: nx, ny, nz
      type(parallel_type), intent(in) :: parallel
      integer, dimension(-1:1,-1:1), intent(in) :: indxA_2d
      integer, dimension(-1:1,-1:1,-1:1), intent(in) :: indxA_3d
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(27,nz,nx-1,ny-1), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nz,nx-1,ny-1), intent(in) :: bu, bv
      real(dp), dimension(nz,nx-1,ny-1), intent(inout) :: xu, xv
      integer, intent(in) :: precond, linear_solve_ncheck, maxiters
      real(dp), intent(in) :: tolerance
      real(dp), intent(out) :: err
      integer, intent(out) :: niters
      integer, intent(in) :: itest, jtest, rtest
      integer(c_int32_t) :: act(nx-1,ny-1)
      act = merge(1, 0, active_vertex)
      call check(c_pcg_chrongear_3d(nx, ny, nz, to_c(parallel), indxA_2d, indxA_3d, act, Auu, Auv, Avu, Avv, &
                                    bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters,      &
                                    err, niters, itest, jtest, rtest))
    end subroutine pcg_solver_chrongear_3d

    !-----------------------------------------------------------------------
    subroutine pcg_solver_standard_2d(nx, ny, parallel, indxA_2d, active_vertex,            &
                                      Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,          &
                                      linear_solve_ncheck, tolerance, maxiters, err, niters, &
                                      itest, jtest, rtest)
      integer, intent(in) :: nx, ny
      type(parallel_type), intent(in) :: parallel
      integer, dimension(-1:1,-1:1), intent(in) :: indxA_2d
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1,9), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nx-1,ny-1), intent(in) :: bu, bv
      real(dp), dimension(nx-1,ny-1), intent(inout) :: xu, xv
      integer, intent(in) :: precond, linear_solve_ncheck, maxiters
      real(dp), intent(in) :: tolerance
      real(dp), intent(out) :: err
      integer, intent(out) :: niters
      integer, intent(in) :: itest, jtest, rtest
      integer(c_int32_t) :: act(nx-1,ny-1)
      act = merge(1, 0, active_vertex)
      call check(c_pcg_standard_2d(nx, ny, to_c(parallel), indxA_2d, act, Auu, Auv, Avu, Avv,            &
                                   bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, &
                                   err, niters, itest, jtest, rtest))
    end subroutine pcg_solver_standard_2d

    !-----------------------------------------------------------------------
    subroutine pcg_solver_chrongear_2d(nx, ny, parallel, indxA_2d, active_vertex,            &
                                       Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,          &
                                       linear_solve_ncheck, tolerance, maxiters, err, niters, &
                                       itest, jtest, rtest)
      integer, intent(in) :: nx, ny
      type(parallel_type), intent(in) :: parallel
      integer, dimension(-1:1,-1:1), intent(in) :: indxA_2d
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1,9), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nx-1,ny-1), intent(in) :: bu, bv
      real(dp), dimension(nx-1,ny-1), intent(inout) :: xu, xv
      integer, intent(in) :: precond, linear_solve_ncheck, maxiters
      real(dp), intent(in) :: tolerance
      real(dp), intent(out) :: err
      integer, intent(out) :: niters
      integer, intent(in) :: itest, jtest, rtest
      integer(c_int32_t) :: act(nx-1,ny-1)
      act = merge(1, 0, active_vertex)
      call check(c_pcg_chrongear_2d(nx, ny, to_c(parallel), indxA_2d, act, Auu, Auv, Avu, Avv,            &
                                    bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, &
                                    err, niters, itest, jtest, rtest))
    end subroutine pcg_solver_chrongear_2d

    !-----------------------------------------------------------------------
    ! indxA_3d(iA,jA,kA) = 1 + (iA+1) + 3*(jA+1) + 9*(kA+1) and indxA_2d(iA,jA) = 1 + (iA+1) + 3*(jA+1):
    ! the module maps of glissade_velo_higher (glissade_velo_higher.F90:608-640) these routines use.
    subroutine compute_residual_vector_3d(nx, ny, nz, parallel, itest, jtest, rtest, active_vertex, &
                                          Auu, Auv, Avu, Avv, bu, bv, uvel, vvel, resid_u, resid_v, &
                                          L2_norm, L2_norm_relative)
      integer, intent(in) :: nx, ny, nz
      type(parallel_type), intent(in) :: parallel
      integer, intent(in) :: itest, jtest, rtest
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(27,nz,nx-1,ny-1), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nz,nx-1,ny-1), intent(in) :: bu, bv, uvel, vvel
      real(dp), dimension(nz,nx-1,ny-1), intent(out) :: resid_u, resid_v
      real(dp), intent(out) :: L2_norm
      real(dp), intent(out), optional :: L2_norm_relative
      integer(c_int32_t) :: act(nx-1,ny-1), indx3(27)
      real(c_double), target :: rel
      integer :: m
      act = merge(1, 0, active_vertex)
      indx3 = [(m, m = 1, 27)]
      if (present(L2_norm_relative)) then
         call check(c_resid_vector_3d(nx, ny, nz, to_c(parallel), indx3, act, Auu, Auv, Avu, Avv, bu, bv, &
                                      uvel, vvel, resid_u, resid_v, L2_norm, c_loc(rel)))
         L2_norm_relative = rel
      else
         call check(c_resid_vector_3d(nx, ny, nz, to_c(parallel), indx3, act, Auu, Auv, Avu, Avv, bu, bv, &
                                      uvel, vvel, resid_u, resid_v, L2_norm, c_null_ptr))
      endif
    end subroutine compute_residual_vector_3d

    !-----------------------------------------------------------------------
    subroutine compute_residual_vector_2d(nx, ny, parallel, itest, jtest, rtest, active_vertex, &
                                          Auu, Auv, Avu, Avv, bu, bv, uvel, vvel, resid_u, resid_v, &
                                          L2_norm, L2_norm_relative)
      integer, intent(in) :: nx, ny
      type(parallel_type), intent(in) :: parallel
      integer, intent(in) :: itest, jtest, rtest
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1,9), intent(in) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nx-1,ny-1), intent(in) :: bu, bv, uvel, vvel
      real(dp), dimension(nx-1,ny-1), intent(out) :: resid_u, resid_v
      real(dp), intent(out) :: L2_norm
      real(dp), intent(out), optional :: L2_norm_relative
      integer(c_int32_t) :: act(nx-1,ny-1), indx2(9)
      real(c_double), target :: rel
      integer :: m
      act = merge(1, 0, active_vertex)
      indx2 = [(m, m = 1, 9)]
      if (present(L2_norm_relative)) then
         call check(c_resid_vector_2d(nx, ny, to_c(parallel), indx2, act, Auu, Auv, Avu, Avv, bu, bv, &
                                      uvel, vvel, resid_u, resid_v, L2_norm, c_loc(rel)))
         L2_norm_relative = rel
      else
         call check(c_resid_vector_2d(nx, ny, to_c(parallel), indx2, act, Auu, Auv, Avu, Avv, bu, bv, &
                                      uvel, vvel, resid_u, resid_v, L2_norm, c_null_ptr))
      endif
    end subroutine compute_residual_vector_2d

    !-----------------------------------------------------------------------
    ! The arrays are (nz, nx-1, ny-1) as everywhere on this path.
    subroutine compute_residual_velocity_3d(whichresid, parallel, uvel, vvel, usav, vsav, resid_velo)
      integer, intent(in) :: whichresid
      type(parallel_type), intent(in) :: parallel
      real(dp), dimension(:,:,:), intent(in) :: uvel, vvel, usav, vsav
      real(dp), intent(out) :: resid_velo
      call check(c_resid_velocity_3d(whichresid, size(uvel,2) + 1, size(uvel,3) + 1, size(uvel,1), &
                                     to_c(parallel), uvel, vvel, usav, vsav, resid_velo))
    end subroutine compute_residual_velocity_3d

    !-----------------------------------------------------------------------
    subroutine compute_residual_velocity_2d(whichresid, parallel, uvel, vvel, usav, vsav, resid_velo)
      integer, intent(in) :: whichresid
      type(parallel_type), intent(in) :: parallel
      real(dp), dimension(:,:), intent(in) :: uvel, vvel, usav, vsav
      real(dp), intent(out) :: resid_velo
      call check(c_resid_velocity_2d(whichresid, size(uvel,1) + 1, size(uvel,2) + 1, to_c(parallel), &
                                     uvel, vvel, usav, vsav, resid_velo))
    end subroutine compute_residual_velocity_2d

    !-----------------------------------------------------------------------
    ! The nearly symmetric pairs (|difference| < eps11 * |diagonal|) are averaged in place, as
    ! in the reference; the reference's per-entry warnings become one log line with their count
    ! and the largest asymmetry.
    subroutine check_symmetry_assembled_matrix_3d(nx, ny, nz, parallel, active_vertex, Auu, Auv, Avu, Avv)
      integer, intent(in) :: nx, ny, nz
      type(parallel_type), intent(in) :: parallel
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(27,nz,nx-1,ny-1), intent(inout) :: Auu, Auv, Avu, Avv
      integer(c_int32_t) :: act(nx-1,ny-1), indx3(27)
      real(c_double) :: maxdiff
      integer(c_long_long) :: nwarn
      character(len=160) :: text
      integer :: m
      act = merge(1, 0, active_vertex)
      indx3 = [(m, m = 1, 27)]
      call check(c_check_symmetry_3d(nx, ny, nz, to_c(parallel), indx3, act, Auu, Auv, Avu, Avv, maxdiff, nwarn))
      if (nwarn > 0) then
         write(text, '(a,i0,a,es12.5)') 'Assembled matrix is not symmetric: ', nwarn, &
              ' warnings, max asymmetry =', maxdiff
         call write_log(trim(text), GM_WARNING)
      endif
    end subroutine check_symmetry_assembled_matrix_3d

    !-----------------------------------------------------------------------
    subroutine check_symmetry_assembled_matrix_2d(nx, ny, parallel, active_vertex, Auu, Auv, Avu, Avv)
      integer, intent(in) :: nx, ny
      type(parallel_type), intent(in) :: parallel
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1,9), intent(inout) :: Auu, Auv, Avu, Avv
      integer(c_int32_t) :: act(nx-1,ny-1), indx2(9)
      real(c_double) :: maxdiff
      integer(c_long_long) :: nwarn
      character(len=160) :: text
      integer :: m
      act = merge(1, 0, active_vertex)
      indx2 = [(m, m = 1, 9)]
      call check(c_check_symmetry_2d(nx, ny, to_c(parallel), indx2, act, Auu, Auv, Avu, Avv, maxdiff, nwarn))
      if (nwarn > 0) then
         write(text, '(a,i0,a,es12.5)') 'Assembled matrix is not symmetric: ', nwarn, &
              ' warnings, max asymmetry =', maxdiff
         call write_log(trim(text), GM_WARNING)
      endif
    end subroutine check_symmetry_assembled_matrix_2d

    !-----------------------------------------------------------------------
    ! The reference's argument lists (the diagnostic indices are accepted and unused); n_glen
    ! is glimmer_physcon's.  The 2D form runs the SSA, L1L2 and DIVA branches.
    subroutine assemble_stiffness_matrix_3d(nx, ny, nz, sigma, nhalo, itest, jtest, rtest, active_cell, &
                                            xVertex, yVertex, uvel, vvel, stagusrf, stagthck, flwafact, &
                                            whichapprox, whichefvs, efvs, efvs_constant, effstrain_min, &
                                            Auu, Auv, Avu, Avv)
      use glimmer_physcon, only: n_glen
      integer, intent(in) :: nx, ny, nz, nhalo, itest, jtest, rtest, whichapprox, whichefvs
      real(dp), dimension(nz), intent(in) :: sigma
      logical, dimension(nx,ny), intent(in) :: active_cell
      real(dp), dimension(nx-1,ny-1), intent(in) :: xVertex, yVertex, stagusrf, stagthck
      real(dp), dimension(nz,nx-1,ny-1), intent(in) :: uvel, vvel
      real(dp), dimension(nz-1,nx,ny), intent(in) :: flwafact
      real(dp), dimension(nz-1,nx,ny), intent(out) :: efvs
      real(dp), intent(in) :: efvs_constant, effstrain_min
      real(dp), dimension(27,nz,nx-1,ny-1), intent(out) :: Auu, Auv, Avu, Avv
      integer(c_int32_t) :: act(nx,ny), indx3(27)
      integer :: m
      act = merge(1, 0, active_cell)
      indx3 = [(m, m = 1, 27)]
      call check(c_assemble_3d(nx, ny, nz, nhalo, sigma, act, xVertex, yVertex, uvel, vvel, stagusrf, stagthck, &
                               flwafact, whichapprox, whichefvs, efvs_constant, effstrain_min, n_glen, indx3, &
                               efvs, Auu, Auv, Avu, Avv))
    end subroutine assemble_stiffness_matrix_3d

    !-----------------------------------------------------------------------
    subroutine assemble_stiffness_matrix_2d(nx, ny, nz, sigma, stagsigma, nhalo, itest, jtest, rtest, parallel, &
                                            active_cell, xVertex, yVertex, uvel_2d, vvel_2d, stagusrf, stagthck, &
                                            flwa, flwafact, whichapprox, diva_slope_factor_x, diva_slope_factor_y, &
                                            whichefvs, efvs, efvs_constant, effstrain_min, Auu, Auv, Avu, Avv, &
                                            dusrf_dx, dusrf_dy, thck, btractx, btracty, omega_k, omega, efvs_qp_3d)
      use glimmer_physcon, only: n_glen
      use glide_types, only: HO_APPROX_SSA, HO_APPROX_DIVA, HO_APPROX_L1L2
      integer, intent(in) :: nx, ny, nz, nhalo, itest, jtest, rtest, whichapprox, whichefvs
      real(dp), dimension(nz), intent(in) :: sigma
      real(dp), dimension(nz-1), intent(in) :: stagsigma
      type(parallel_type), intent(in) :: parallel
      logical, dimension(nx,ny), intent(in) :: active_cell
      real(dp), dimension(nx-1,ny-1), intent(in) :: xVertex, yVertex, uvel_2d, vvel_2d, stagusrf, stagthck
      real(dp), dimension(nz-1,nx,ny), intent(in) :: flwa, flwafact
      real(dp), dimension(nx,ny), intent(in) :: diva_slope_factor_x, diva_slope_factor_y
      real(dp), dimension(nz-1,nx,ny), intent(out) :: efvs
      real(dp), intent(in) :: efvs_constant, effstrain_min
      real(dp), dimension(nx-1,ny-1,9), intent(out) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nx-1,ny-1), intent(in), optional :: dusrf_dx, dusrf_dy, btractx, btracty
      real(dp), dimension(nx,ny), intent(in), optional :: thck
      real(dp), dimension(nz,nx,ny), intent(out), optional :: omega_k
      real(dp), dimension(nx,ny), intent(out), optional :: omega
      real(dp), dimension(nz-1,4,nx,ny), intent(inout), optional :: efvs_qp_3d
      integer(c_int32_t) :: act(nx,ny), indx2(9)
      integer :: m
      act = merge(1, 0, active_cell)
      indx2 = [(m, m = 1, 9)]
      if (whichapprox == HO_APPROX_DIVA) then
         if (.not. (present(thck) .and. present(btractx) .and. present(btracty) .and. present(omega_k) .and. &
                    present(omega) .and. present(efvs_qp_3d))) then
            call write_log('GPU DIVA assembly: thck, btractx/y, omega_k, omega and efvs_qp_3d are needed', GM_FATAL)
         endif
         call check(c_assemble_2d_diva(nx, ny, nz, nhalo, sigma, stagsigma, act, xVertex, yVertex, uvel_2d, &
                                       vvel_2d, stagthck, thck, btractx, btracty, diva_slope_factor_x, &
                                       diva_slope_factor_y, flwafact, whichefvs, efvs_constant, effstrain_min, &
                                       n_glen, indx2, efvs_qp_3d, efvs, omega_k, omega, Auu, Auv, Avu, Avv))
      elseif (whichapprox == HO_APPROX_SSA) then
         call check(c_assemble_2d(nx, ny, nz, nhalo, sigma, act, xVertex, yVertex, uvel_2d, vvel_2d, stagthck, &
                                  flwafact, whichefvs, efvs_constant, effstrain_min, n_glen, indx2, efvs, &
                                  Auu, Auv, Avu, Avv))
      elseif (whichapprox == HO_APPROX_L1L2) then
         if (.not. (present(dusrf_dx) .and. present(dusrf_dy))) then
            call write_log('GPU L1L2 assembly: dusrf_dx and dusrf_dy are needed', GM_FATAL)
         endif
         call check(c_assemble_2d_l1l2(nx, ny, nz, nhalo, sigma, act, xVertex, yVertex, uvel_2d, vvel_2d, &
                                       stagthck, dusrf_dx, dusrf_dy, flwa, flwafact, whichefvs, efvs_constant, &
                                       effstrain_min, n_glen, indx2, efvs, Auu, Auv, Avu, Avv))
      else
         call write_log('GPU 2D assembly: whichapprox must be SSA, L1L2 or DIVA', GM_FATAL)
      endif
    end subroutine assemble_stiffness_matrix_2d

    !-----------------------------------------------------------------------
    ! The boundary routines with the reference's argument lists.  basal_sliding_bc_3d receives
    ! the bed slices Auu(:,nz,:,:), Avv(:,nz,:,:), which the library addresses as one-level
    ! blocks.
    subroutine dirichlet_boundary_conditions_3d(nx, ny, nz, nhalo, active_vertex, umask_dirichlet, &
                                                vmask_dirichlet, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv)
      integer, intent(in) :: nx, ny, nz, nhalo
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      integer, dimension(nz,nx-1,ny-1), intent(in) :: umask_dirichlet, vmask_dirichlet
      real(dp), dimension(nz,nx-1,ny-1), intent(in) :: uvel, vvel
      real(dp), dimension(27,nz,nx-1,ny-1), intent(inout) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nz,nx-1,ny-1), intent(inout) :: bu, bv
      integer(c_int32_t) :: act(nx-1,ny-1), um(nz,nx-1,ny-1), vm(nz,nx-1,ny-1), indx3(27)
      integer :: m
      act = merge(1, 0, active_vertex)
      um = umask_dirichlet
      vm = vmask_dirichlet
      indx3 = [(m, m = 1, 27)]
      call check(c_dirichlet_3d(nx, ny, nz, nhalo, act, um, vm, uvel, vvel, indx3, Auu, Auv, Avu, Avv, bu, bv))
    end subroutine dirichlet_boundary_conditions_3d

    !-----------------------------------------------------------------------
    subroutine dirichlet_boundary_conditions_2d(nx, ny, nhalo, active_vertex, umask_dirichlet, vmask_dirichlet, &
                                                uvel, vvel, Auu, Auv, Avu, Avv, bu, bv)
      integer, intent(in) :: nx, ny, nhalo
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      integer, dimension(nx-1,ny-1), intent(in) :: umask_dirichlet, vmask_dirichlet
      real(dp), dimension(nx-1,ny-1), intent(in) :: uvel, vvel
      real(dp), dimension(nx-1,ny-1,9), intent(inout) :: Auu, Auv, Avu, Avv
      real(dp), dimension(nx-1,ny-1), intent(inout) :: bu, bv
      integer(c_int32_t) :: act(nx-1,ny-1), um(nx-1,ny-1), vm(nx-1,ny-1), indx2(9)
      integer :: m
      act = merge(1, 0, active_vertex)
      um = umask_dirichlet
      vm = vmask_dirichlet
      indx2 = [(m, m = 1, 9)]
      call check(c_dirichlet_2d(nx, ny, nhalo, act, um, vm, uvel, vvel, indx2, Auu, Auv, Avu, Avv, bu, bv))
    end subroutine dirichlet_boundary_conditions_2d

    !-----------------------------------------------------------------------
    subroutine basal_sliding_bc_3d(nx, ny, nNeighbors, nhalo, parallel, dx, dy, itest, jtest, rtest, &
                                   active_cell, active_vertex, beta, lsrf, xVertex, yVertex, &
                                   whichassemble_beta, Auu, Avv)
      integer, intent(in) :: nx, ny, nNeighbors, nhalo, itest, jtest, rtest, whichassemble_beta
      type(parallel_type), intent(in) :: parallel
      real(dp), intent(in) :: dx, dy
      logical, dimension(nx,ny), intent(in) :: active_cell
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1), intent(in) :: beta, xVertex, yVertex
      real(dp), dimension(nx,ny), intent(in) :: lsrf
      real(dp), dimension(nNeighbors,nx-1,ny-1), intent(inout) :: Auu, Avv
      integer(c_int32_t) :: act(nx-1,ny-1), cell(nx,ny), indx3(27)
      integer :: m
      act = merge(1, 0, active_vertex)
      cell = merge(1, 0, active_cell)
      indx3 = [(m, m = 1, 27)]
      call check(c_basal_3d(nx, ny, 1, nhalo, dx, dy, cell, act, beta, lsrf, xVertex, yVertex, &
                            whichassemble_beta, indx3, Auu, Avv))
    end subroutine basal_sliding_bc_3d

    !-----------------------------------------------------------------------
    subroutine basal_sliding_bc_2d(nx, ny, nNeighbors, nhalo, parallel, dx, dy, itest, jtest, rtest, &
                                   active_cell, active_vertex, beta, lsrf, xVertex, yVertex, &
                                   whichassemble_beta, Auu, Avv)
      integer, intent(in) :: nx, ny, nNeighbors, nhalo, itest, jtest, rtest, whichassemble_beta
      type(parallel_type), intent(in) :: parallel
      real(dp), intent(in) :: dx, dy
      logical, dimension(nx,ny), intent(in) :: active_cell
      logical, dimension(nx-1,ny-1), intent(in) :: active_vertex
      real(dp), dimension(nx-1,ny-1), intent(in) :: beta, xVertex, yVertex
      real(dp), dimension(nx,ny), intent(in) :: lsrf
      real(dp), dimension(nx-1,ny-1,nNeighbors), intent(inout) :: Auu, Avv
      integer(c_int32_t) :: act(nx-1,ny-1), cell(nx,ny), indx2(9)
      integer :: m
      act = merge(1, 0, active_vertex)
      cell = merge(1, 0, active_cell)
      indx2 = [(m, m = 1, 9)]
      call check(c_basal_2d(nx, ny, nhalo, dx, dy, cell, act, beta, xVertex, yVertex, whichassemble_beta, &
                            indx2, Auu, Avv))
    end subroutine basal_sliding_bc_2d

  end module glissade_velo_higher_pcg_gpu
