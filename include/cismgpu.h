/*
 * cismgpu.h -- C ABI of the B200 (sm_100a) native structured PCG velocity solve.
 *
 * These entry points replace the four native PCG solvers of CISM's Glissade
 * higher-order velocity solver,
 *   libglissade/glissade_velo_higher_pcg.F90
 *     pcg_solver_standard_2d   (:67-823)
 *     pcg_solver_standard_3d   (:827-1537)
 *     pcg_solver_chrongear_2d  (:1541-2628)
 *     pcg_solver_chrongear_3d  (:2632-3594)
 * called from glissade_velo_higher_solve (libglissade/glissade_velo_higher.F90:3229-3322).
 *
 * Argument lists keep the Fortran order and meaning.  Arrays are Fortran
 * column-major, exactly as the Fortran caller holds them:
 *   3D blocks   A(27, nz, nx-1, ny-1): element (m,k,i,j) at (m-1)+27*((k-1)+nz*((i-1)+(nx-1)*(j-1)))
 *   3D vectors  b(nz, nx-1, ny-1)
 *   2D blocks   A(nx-1, ny-1, 9):      element (i,j,m) at (i-1)+(nx-1)*((j-1)+(ny-1)*(m-1))
 *   2D vectors  b(nx-1, ny-1)
 *   indxA_3d(-1:1,-1:1,-1:1) and indxA_2d(-1:1,-1:1) as 27 / 9 int32 (iA fastest)
 *   active_vertex(nx-1, ny-1) as Fortran default logical (4 bytes, nonzero = .true.)
 * nx, ny are the *cell* dimensions of the haloed local grid (velocity arrays are
 * (nx-1) x (ny-1) vertices), as in the reference.
 *
 * type(parallel_type) is not C-interoperable, so the Fortran wrapper copies the
 * fields the path reads (libglimmer/parallel_mpi.F90:78-153) into cismgpu_par_t.
 *
 * Return value: CISMGPU_OK (0) on success, INCLUDING non-convergence (the
 * reference returns niters = maxiters and the last err, :1514-1520).  Nonzero
 * codes stand for the cases where the reference calls write_log(..., GM_FATAL)
 * (NaN breakdown, :637-639,697-700,1331,1391,2196,2467,3263,3434) or where the
 * GPU path cannot run the call.  The Fortran wrapper maps nonzero to GM_FATAL.
 *
 * Every call is synchronous: on return xu/xv hold the solution (including the
 * halo values the reference leaves in them), err and niters are set, and the
 * library holds no pointer to caller memory.
 *
 * Global sums in the standard and Chronopoulos-Gear solvers: with par->reprosum == 0
 * every parallel_global_sum_stagger of the reference is the library's fixed double-double
 * reduction tree (launch-independent, reproducible run to run), or, after
 * cismgpu_set_sum_order(CISMGPU_SUM_SEQUENTIAL), the reference's own sequential order, which
 * reproduces the reference's one-rank solve bit for bit (slower: see cismgpu_set_sum_order).  With par->reprosum != 0
 * (the one-shot solvers and cismgpu_solver_create) each of them is the reference's
 * reproducible sum (cism_reprosum_calc, libglimmer/cism_reprosum_mod.F90:237-1818, as
 * parallel_global_sum_stagger's reprosum branch calls it, parallel_mpi.F90:6703-6738), two
 * fields summed independently where the reference passes nflds = 2 (:1921, :2181, :2447),
 * so a solve reproduces the reference's reprosum run on one rank bit for bit; the host
 * then drives the iteration, with two short stream synchronizations per sum.  Non-finite
 * summands, undefined in the reference, give their IEEE sum (NaN, +Inf or -Inf), so the
 * NaN breakdown tests behave as without reprosum.  The mixed-precision solver ignores the
 * flag (its sums are the fixed FP64 tree of its checks).
 */
#ifndef CISMGPU_H
#define CISMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CISMGPU_OK                0
#define CISMGPU_EBREAKDOWN_ETA1   1  /* eta1 = (r,z) is NaN   (reference :637, :1331)            */
#define CISMGPU_EBREAKDOWN_ALPHA  2  /* alpha is NaN           (reference :697, :1391, :2196, :2467, :3263, :3434) */
#define CISMGPU_EUNSUPPORTED      3  /* tasks_row*tasks_col > 1; mixed solver with 2D precond 2  */
#define CISMGPU_EINVAL            4  /* bad sizes, null pointers, inconsistent owned bounds     */
#define CISMGPU_ECUDA             5  /* CUDA runtime error (message via cismgpu_last_error)     */
#define CISMGPU_ETIMEOUT          6  /* a bounded device wait gave up                           */
#define CISMGPU_ENOMEM            7  /* device allocation failed or HBM budget exceeded         */
#define CISMGPU_ENODEV            8  /* no CUDA device / not an sm_100 device                   */
#define CISMGPU_EDIVZERO          9  /* tridiagonal precond setup met a zero pivot (reference
                                        GM_FATAL :4339, :4380, :4475, :4492); x is unchanged      */

/* preconditioner options, libglide/glide_types.F90:342-346 */
#define CISMGPU_PRECOND_NONE            0
#define CISMGPU_PRECOND_DIAG            1
#define CISMGPU_PRECOND_SIA             2
#define CISMGPU_PRECOND_TRIDIAG_LOCAL   3
#define CISMGPU_PRECOND_TRIDIAG_GLOBAL  4

/* Fields of type(parallel_type) read on this path (libglimmer/parallel_mpi.F90:78-153).
 * Indices are 1-based, as in Fortran.  On one rank: periodic/no_penetration and
 * no_ice have staggered_ilo = jlo = 3, outflow has 2; staggered_ihi = nx-2,
 * staggered_jhi = ny-2 (parallel_mpi.F90:2640-2653). */
typedef struct cismgpu_par {
    int32_t staggered_ilo, staggered_ihi;
    int32_t staggered_jlo, staggered_jhi;
    int32_t periodic_bc;   /* logical: doubly periodic (also no_penetration, parallel_mpi.F90:2498) */
    int32_t outflow_bc;    /* logical: zero beyond the global boundary                              */
    int32_t no_ice_bc;     /* logical: zero the halo and the last owned row                         */
    int32_t reprosum;      /* logical: reproducible sums (global sums, FP64 solvers' dot products)  */
    int32_t tasks_row;     /* tasks on this row    (must be 1: whole domain on one GPU)            */
    int32_t tasks_col;     /* tasks on this column (must be 1)                                      */
} cismgpu_par_t;

/* Replaces pcg_solver_standard_3d, glissade_velo_higher_pcg.F90:827-838 (decls :895-949). */
int cismgpu_pcg_standard_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                            const int32_t *indxA_2d, const int32_t *indxA_3d,
                            const int32_t *active_vertex,
                            const double *Auu, const double *Auv,
                            const double *Avu, const double *Avv,
                            const double *bu, const double *bv,
                            double *xu, double *xv,
                            int precond, int linear_solve_ncheck,
                            double tolerance, int maxiters,
                            double *err, int *niters,
                            int itest, int jtest, int rtest);

/* Replaces pcg_solver_chrongear_3d, glissade_velo_higher_pcg.F90:2632-2643 (decls :2751-2805). */
int cismgpu_pcg_chrongear_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                             const int32_t *indxA_2d, const int32_t *indxA_3d,
                             const int32_t *active_vertex,
                             const double *Auu, const double *Auv,
                             const double *Avu, const double *Avv,
                             const double *bu, const double *bv,
                             double *xu, double *xv,
                             int precond, int linear_solve_ncheck,
                             double tolerance, int maxiters,
                             double *err, int *niters,
                             int itest, int jtest, int rtest);

/* Replaces pcg_solver_standard_2d, glissade_velo_higher_pcg.F90:67-77 (decls :109-158). */
int cismgpu_pcg_standard_2d(int nx, int ny, const cismgpu_par_t *par,
                            const int32_t *indxA_2d, const int32_t *active_vertex,
                            const double *Auu, const double *Auv,
                            const double *Avu, const double *Avv,
                            const double *bu, const double *bv,
                            double *xu, double *xv,
                            int precond, int linear_solve_ncheck,
                            double tolerance, int maxiters,
                            double *err, int *niters,
                            int itest, int jtest, int rtest);

/* Replaces pcg_solver_chrongear_2d, glissade_velo_higher_pcg.F90:1541-1551 (decls :1581-1630). */
int cismgpu_pcg_chrongear_2d(int nx, int ny, const cismgpu_par_t *par,
                             const int32_t *indxA_2d, const int32_t *active_vertex,
                             const double *Auu, const double *Auv,
                             const double *Avu, const double *Avv,
                             const double *bu, const double *bv,
                             double *xu, double *xv,
                             int precond, int linear_solve_ncheck,
                             double tolerance, int maxiters,
                             double *err, int *niters,
                             int itest, int jtest, int rtest);

/* Replaces matvec_multiply_structured_3d, glissade_velo_higher_pcg.F90:5528-5652
 * (public in the reference module, :58).  y = A x on locally owned, active
 * vertices; 0 elsewhere.  Bit-identical to the reference loop order. */
int cismgpu_matvec_structured_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                                 const int32_t *indxA_3d, const int32_t *active_vertex,
                                 const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv,
                                 const double *xu, const double *xv,
                                 double *yu, double *yv);

/* Mirrors matvec_multiply_structured_2d, glissade_velo_higher_pcg.F90:5656-5773. */
int cismgpu_matvec_structured_2d(int nx, int ny, const cismgpu_par_t *par,
                                 const int32_t *indxA_2d, const int32_t *active_vertex,
                                 const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv,
                                 const double *xu, const double *xv,
                                 double *yu, double *yv);

/* Mirrors parallel_global_sum_stagger(arr1, parallel, arr2)
 * (libglimmer/parallel_mpi.F90: _real8_2d :6537-6658, _real8_3d :6663-6794) on one rank:
 * the sum over locally owned vertices of arr1 + arr2.  Host arrays in the caller's layout
 * (nz, nx-1, ny-1); nz = 1 for 2D fields.  With par->reprosum == 0 the sum uses the
 * library's fixed double-double reduction tree (the same one every solver uses): launch-
 * independent and reproducible, the correctly rounded exact sum except in rare near-tie
 * cases; or, after cismgpu_set_sum_order(CISMGPU_SUM_SEQUENTIAL), the reference's own
 * sequential order, bit for bit.  With par->reprosum != 0 it is the reference's reproducible
 * sum (parallel_reduce_reprosum -> cism_reprosum_calc, libglimmer/cism_reprosum_mod.F90:
 * 237-1818): the integer-vector fixed-point sum, its value independent of the order of the
 * summands, bit for bit the reference's on one rank; an owned summand arr1 + arr2 that is
 * not finite (undefined in the reference) makes the result the IEEE sum of the non-finite
 * summands (NaN, +Inf or -Inf).  tasks_row*tasks_col > 1 returns CISMGPU_EUNSUPPORTED.
 * *sum receives the result. */
int cismgpu_global_sum_stagger(int nx, int ny, int nz, const cismgpu_par_t *par,
                               const double *arr1, const double *arr2, double *sum);

/* No counterpart in the reference: the sum above for callers that cannot let a
 * library allocate device memory -- a host whose own allocator has reserved the
 * device, code that must not stall the device mid-step the way cudaMalloc/cudaFree
 * can, or code that only holds device pointers another component gave it.
 * arr1_dev, arr2_dev (layout (nz, nx-1, ny-1)) and sum_dev are pointers the current
 * device can read (its own memory, managed or mapped pinned memory; another GPU's memory
 * returns CISMGPU_EINVAL); the kernel is enqueued on cuda_stream (NULL: the default
 * stream) and *sum_dev is written asynchronously, identical to cismgpu_global_sum_stagger's
 * result in the same sum order (cismgpu_set_sum_order).  par->reprosum != 0 returns
 * CISMGPU_EUNSUPPORTED: the reproducible sum needs host steps this asynchronous call
 * cannot take; tasks_row*tasks_col > 1 returns CISMGPU_EUNSUPPORTED as everywhere.
 * It allocates nothing: its scratch is a fixed array in the library's device memory,
 * sized for at most CISMGPU_NOALLOC_MAX_COLUMNS vertex columns (nx-1)*(ny-1) (any nz);
 * larger grids return CISMGPU_EINVAL.  All calls on a device share that array: calls
 * whose kernels overlap on the GPU race and give wrong sums, so order them (one stream).
 * The first call on each device looks up the array's address (and may load the
 * library's kernels onto the device): make it before any stream capture begins. */
#define CISMGPU_NOALLOC_MAX_COLUMNS 4194304
int cismgpu_global_sum_stagger_noalloc(int nx, int ny, int nz, const cismgpu_par_t *par,
                                       const double *arr1_dev, const double *arr2_dev,
                                       double *sum_dev, void *cuda_stream);

/* ------------------------------------------------------------------------
 * Nonlinear-iteration diagnostics (glissade_velo_higher.F90), one-shot form.
 * ------------------------------------------------------------------------ */

/* whichresid of compute_residual_velocity (HO_RESID_*, libglide/glide_types.F90:321-325) */
#define CISMGPU_RESID_MAXU          0  /* max relative speed change, all levels                */
#define CISMGPU_RESID_MAXU_NO_UBAS  1  /* ... without the bed level (3D)                        */
#define CISMGPU_RESID_MEANU         2  /* mean relative speed change, without the bed level (3D) */

/* Replaces compute_residual_vector_3d (glissade_velo_higher.F90:9693-9894):
 * resid = A*uvel - b on owned active vertices (0 elsewhere, same matvec statements as
 * matvec_multiply_structured_3d), L2_norm = |resid| and, if L2_norm_relative is not NULL,
 * L2_norm/|b| over owned active vertices (0 when |b| = 0).  Sums use the global sums' fixed
 * tree.  Arrays in the caller's layout as for the solver calls; itest/jtest/rtest (diagnostic
 * prints only) are not taken. */
int cismgpu_compute_residual_vector_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                                       const int32_t *indxA_3d, const int32_t *active_vertex,
                                       const double *Auu, const double *Auv, const double *Avu,
                                       const double *Avv, const double *bu, const double *bv,
                                       const double *uvel, const double *vvel, double *resid_u,
                                       double *resid_v, double *L2_norm, double *L2_norm_relative);

/* Replaces compute_residual_vector_2d (glissade_velo_higher.F90:9502-9689). */
int cismgpu_compute_residual_vector_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                       const int32_t *active_vertex, const double *Auu, const double *Auv,
                                       const double *Avu, const double *Avv, const double *bu,
                                       const double *bv, const double *uvel, const double *vvel,
                                       double *resid_u, double *resid_v, double *L2_norm,
                                       double *L2_norm_relative);

/* Replaces compute_residual_velocity_3d (glissade_velo_higher.F90:10314-10446): over owned
 * vertices, the largest (or, for CISMGPU_RESID_MEANU, the mean) of |(|usav| - |u|)/|u|| where
 * |u| = sqrt(uvel**2 + vvel**2) /= 0.  Max modes are exact; the mean's sum uses the global
 * sums' fixed tree.  (The reference's location of the maximum is diagnostic output only.) */
int cismgpu_compute_residual_velocity_3d(int whichresid, int nx, int ny, int nz, const cismgpu_par_t *par,
                                         const double *uvel, const double *vvel, const double *usav,
                                         const double *vsav, double *resid_velo);

/* Replaces compute_residual_velocity_2d (glissade_velo_higher.F90:10188-10310). */
int cismgpu_compute_residual_velocity_2d(int whichresid, int nx, int ny, const cismgpu_par_t *par,
                                         const double *uvel, const double *vvel, const double *usav,
                                         const double *vsav, double *resid_velo);

/* Replace check_symmetry_assembled_matrix_3d (glissade_velo_higher.F90:10854-11117) and
 * check_symmetry_assembled_matrix_2d (:10648-10850), which glissade_velo_higher_solve calls on
 * the assembled blocks before the solve (:2923-2931, :2704-2711).  Every owned active row
 * compares each coefficient with its transpose partner (Auu with Auu^T, Auv with Avu^T, Avv
 * with Avv^T, Avu with Auv^T).  Where the two differ by less than eps11 = 1e-11
 * (glimmer_paramets.F90:77) times |diagonal| of the visited row's block, the 3D check replaces
 * both by their average, in place in the caller's arrays; larger differences are reported.
 * The 2D check reports only (its averaging is commented out in the reference) and leaves the
 * blocks unchanged.  maxdiff: the largest |difference| met (the reference's maxdiff);
 * nwarn: the number of asymmetry warnings the reference writes to its log.  indxA_3d /
 * indxA_2d: the reference's module index maps.  A partner outside the arrays (an owned row on
 * the array edge, where the reference would read outside its arrays) is not compared. */
int cismgpu_check_symmetry_assembled_matrix_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                                               const int32_t *indxA_3d, const int32_t *active_vertex, double *Auu,
                                               double *Auv, double *Avu, double *Avv, double *maxdiff,
                                               long long *nwarn);
int cismgpu_check_symmetry_assembled_matrix_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                               const int32_t *active_vertex, const double *Auu, const double *Auv,
                                               const double *Avu, const double *Avv, double *maxdiff,
                                               long long *nwarn);

/* Replaces assemble_stiffness_matrix_3d (glissade_velo_higher.F90:5382-5643): the four
 * Blatter-Pattyn (whichapprox 2; 1 SSA and 0 SIA forms too) stiffness blocks of the
 * trilinear hexahedral elements of every active cell j = nhalo+1..ny-nhalo+1,
 * i = nhalo+1..nx-nhalo+1, layers 1..nz-1, with 8-point Gauss quadrature and the effective
 * viscosity of whichefvs (0 constant efvs_constant, 1 flow factor, 2 nonlinear from uvel,
 * vvel with effstrain_min; glide_types.F90:240-242), computed on the GPU.  Arguments are the
 * reference's (itest, jtest, rtest dropped), in its layouts: sigma(nz), active_cell(nx,ny)
 * (nonzero = .true.), xVertex, yVertex, stagusrf, stagthck (nx-1,ny-1), uvel, vvel
 * (nz,nx-1,ny-1), flwafact and efvs (nz-1,nx,ny), A** (27,nz,nx-1,ny-1); n_glen is
 * glimmer_physcon's n_glen and indxA_3d the module's index map.  nhalo must be >= 2.
 * Every coefficient is the reference's sum, term for term and in the reference's element
 * order (so A is exactly symmetric); only the flow law's pow is CUDA's rather than the host
 * C library's.  A singular element Jacobian (the reference stops with GM_FATAL) returns
 * CISMGPU_EINVAL.  The basal and Dirichlet conditions and the load vector are not applied. */
int cismgpu_assemble_stiffness_matrix_3d(int nx, int ny, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel, const double *vvel, const double *stagusrf,
                                         const double *stagthck, const double *flwafact, int whichapprox,
                                         int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                         const int32_t *indxA_3d, double *efvs, double *Auu, double *Auv,
                                         double *Avu, double *Avv);

/* Replaces assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378) for the SSA
 * (whichapprox = HO_APPROX_SSA; DIVA: cismgpu_assemble_stiffness_matrix_2d_diva below; the L1L2
 * branch is not built): 4-node cells with
 * 4-point Gauss quadrature, the viscosity of whichefvs at the flow factor averaged over the nz-1
 * layers (glissade_vertical_average), weighted by the thickness at each point.  uvel_2d,
 * vvel_2d, xVertex, yVertex, stagthck (nx-1,ny-1); sigma(nz); flwafact and efvs (nz-1,nx,ny),
 * efvs holding the cell's mean viscosity in every layer; A** (nx-1,ny-1,9) through indxA_2d.
 * Same arithmetic, order and error behaviour as the 3D call above. */
int cismgpu_assemble_stiffness_matrix_2d(int nx, int ny, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                         const double *flwafact, int whichefvs, double efvs_constant,
                                         double effstrain_min, double n_glen, const int32_t *indxA_2d, double *efvs,
                                         double *Auu, double *Auv, double *Avu, double *Avv);

/* Replaces dirichlet_boundary_conditions_3d (glissade_velo_higher.F90:9305-9498): at every
 * active vertex j = nhalo..ny-nhalo+1, i = nhalo..nx-nhalo+1, level k, with umask_dirichlet = 1
 * (then likewise vmask_dirichlet), b = uvel (vvel), a unit diagonal, the row zeroed, and the
 * column moved into the right-hand side of each neighbour not prescribed in that component.
 * Masks (nz,nx-1,ny-1) int32; velocities and b (nz,nx-1,ny-1); A** (27,nz,nx-1,ny-1) through
 * indxA_3d.  Right-hand-side moves are summed in the reference's order of the prescribed nodes,
 * so the result is the reference's bit for bit. */
int cismgpu_dirichlet_boundary_conditions_3d(int nx, int ny, int nz, int nhalo, const int32_t *active_vertex,
                                             const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet,
                                             const double *uvel, const double *vvel, const int32_t *indxA_3d,
                                             double *Auu, double *Auv, double *Avu, double *Avv, double *bu,
                                             double *bv);

/* Replaces basal_sliding_bc_3d (glissade_velo_higher.F90:8815-9129).  whichassemble_beta = 1
 * (HO_ASSEMBLE_BETA_LOCAL, CISM's default): at every active vertex the bed diagonal (level nz)
 * of Auu and Avv gains dx*dy/vol0 * beta / cos(theta), theta the slope angle of the lower
 * surface lsrf(nx,ny) staggered to the vertices (glissade_stagger, glissade_slope_angle); atan
 * and cos are CUDA's.  whichassemble_beta = 0 (standard): per active cell, 4-point quadrature of
 * beta phi_r phi_c over the lower surface (the curved area factor,
 * get_area_scale_factor_curved_2d) added to the bed level's 9 horizontal couplings, point by
 * point in the reference's order (its sqrt is IEEE, so bit-exact); it reads the vertices of the
 * cells nhalo+1..n-nhalo+1, so it needs nhalo >= 2 (EINVAL otherwise, as in the 2D forms).
 * beta, xVertex, yVertex (nx-1,ny-1); active_cell (nx,ny); Auu, Avv (27,nz,nx-1,ny-1) (nz = 1
 * for the bed slices). */
int cismgpu_basal_sliding_bc_3d(int nx, int ny, int nz, int nhalo, double dx, double dy,
                                const int32_t *active_cell, const int32_t *active_vertex, const double *beta,
                                const double *lsrf, const double *xVertex, const double *yVertex,
                                int whichassemble_beta, const int32_t *indxA_3d, double *Auu, double *Avv);

/* Replaces dirichlet_boundary_conditions_2d (glissade_velo_higher.F90:9133-9301) and
 * basal_sliding_bc_2d (:8281-8531: local form, the diagonal of Auu and Avv at every active
 * vertex += (dx*dy/vol0) * beta; standard form, the 4-point quadrature with the flat Jacobian).  Masks, velocities, beta and b (nx-1,ny-1); A**
 * (nx-1,ny-1,9) through indxA_2d.  As in the reference's 2D routine, a u-prescribed vertex
 * gets unit diagonals in Auu, Auv and Avu (a v-prescribed one then zero Auv, Avu and unit Avv),
 * and the moves into b are summed in its order (offsets outermost).  Bit-exact. */
int cismgpu_dirichlet_boundary_conditions_2d(int nx, int ny, int nhalo, const int32_t *active_vertex,
                                             const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet,
                                             const double *uvel, const double *vvel, const int32_t *indxA_2d,
                                             double *Auu, double *Auv, double *Avu, double *Avv, double *bu,
                                             double *bv);
int cismgpu_basal_sliding_bc_2d(int nx, int ny, int nhalo, double dx, double dy, const int32_t *active_cell,
                                const int32_t *active_vertex, const double *beta, const double *xVertex,
                                const double *yVertex, int whichassemble_beta, const int32_t *indxA_2d, double *Auu,
                                double *Avv);

/* assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378) with whichapprox =
 * HO_APPROX_DIVA: per active cell and Gauss point, the layer viscosities of
 * compute_effective_viscosity_diva (:7730-7997, its iterative form; the cubic form is disabled
 * in the reference) from the previous ones in efvs_qp_3d (nz-1,4,nx,ny), read and updated, the
 * basal traction btractx, btracty (nx-1,ny-1) and the slope factors diva_slope_factor_x/_y
 * (nx,ny); their sigma-weighted average times the thickness in the element matrix; efvs
 * (nz-1,nx,ny) the mean over the points; compute_integrals_diva (:5649-5775) into omega_k
 * (nz,nx,ny) and omega (nx,ny) of the assembled cells (the rest unchanged).  thck (nx,ny) is
 * the cell thickness of the integrals; stagsigma (nz-1).  The flow law's pow is CUDA's. */
int cismgpu_assemble_stiffness_matrix_2d_diva(int nx, int ny, int nz, int nhalo, const double *sigma,
                                              const double *stagsigma, const int32_t *active_cell,
                                              const double *xVertex, const double *yVertex, const double *uvel_2d,
                                              const double *vvel_2d, const double *stagthck, const double *thck,
                                              const double *btractx, const double *btracty,
                                              const double *diva_slope_factor_x, const double *diva_slope_factor_y,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const int32_t *indxA_2d,
                                              double *efvs_qp_3d, double *efvs, double *omega_k, double *omega,
                                              double *Auu, double *Auv, double *Avu, double *Avv);

/* Replaces basal_sliding_bc_2d_diva (glissade_velo_higher.F90:8535-8811), the DIVA basal term
 * with slope correction (CISM's default for DIVA): beta_eff_x into Auu and beta_eff_y into Avv.
 * Local form (1): the diagonals gain (dx*dy/vol0)*beta_eff/cos(theta) with theta_x = atan|dz/dx|,
 * theta_y = atan|dz/dy| of the staggered lower surface lsrf(nx,ny) (atan, cos are CUDA's).
 * Standard form (0): 4-point quadrature with the curved area factor, bit-exact. */
int cismgpu_basal_sliding_bc_2d_diva(int nx, int ny, int nhalo, double dx, double dy, const int32_t *active_cell,
                                     const int32_t *active_vertex, const double *beta_eff_x, const double *beta_eff_y,
                                     const double *lsrf, const double *xVertex, const double *yVertex,
                                     int whichassemble_beta, const int32_t *indxA_2d, double *Auu, double *Avv);

/* assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378) with whichapprox =
 * HO_APPROX_L1L2: per Gauss point and layer the viscosity of compute_effective_viscosity_L1L2
 * (:7474-7726; the cubic for the parallel stress from the surface gradient dusrf_dx/_dy
 * (nx-1,ny-1) and flwa (nz-1,nx,ny)), its sigma-weighted average times the thickness in the
 * element matrix, efvs the mean over the points.  n_glen must be 1 or 3 for the nonlinear
 * viscosity (the reference's GM_FATAL otherwise: CISMGPU_EINVAL).  pow is CUDA's. */
int cismgpu_assemble_stiffness_matrix_2d_l1l2(int nx, int ny, int nz, int nhalo, const double *sigma,
                                              const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                              const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                              const double *dusrf_dx, const double *dusrf_dy, const double *flwa,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const int32_t *indxA_2d,
                                              double *efvs, double *Auu, double *Auv, double *Avu, double *Avv);

/* Replaces load_vector_gravity (glissade_velo_higher.F90:4228-4449): the gravitational driving
 * stress added into loadu, loadv (nz,nx-1,ny-1) (the reference's caller zeroes them first).
 * whichassemble_taud = 1 (local, CISM's default): per active vertex and level
 * -rhoi*grav*dx*dy*dz/vol0 * dusrf_dx with dz from stagwbndsigma (0:nz) and stagthck;
 * 0 (standard): 8-point quadrature over the hexahedra of the active cells (nhalo >= 2).
 * rhoi = 910, grav = 9.81 (glimmer_physcon.F90:67, :69).  Bit-exact. */
int cismgpu_load_vector_gravity(int nx, int ny, int nz, int nhalo, const double *sigma, const double *stagwbndsigma,
                                double dx, double dy, const int32_t *active_cell, const int32_t *active_vertex,
                                const double *xVertex, const double *yVertex, const double *stagusrf,
                                const double *stagthck, const double *dusrf_dx, const double *dusrf_dy,
                                int whichassemble_taud, double *loadu, double *loadv);

/* ------------------------------------------------------------------------
 * Device-resident solver handles (no reference counterpart: the reference
 * solvers are stateless calls).  A handle uploads A, b and x0 once and keeps
 * them, and all Krylov state, in HBM, so repeated solves (benchmarking, the
 * serving loop, batched ensembles) pay no host<->device traffic.  Each handle
 * owns its buffers and runs on the stream given at creation (NULL: a new
 * non-blocking stream), so handles on different streams run concurrently.
 * ------------------------------------------------------------------------ */
typedef struct cismgpu_solver cismgpu_solver_t;

/* algorithms */
#define CISMGPU_ALG_STANDARD        0  /* pcg_solver_standard_*  (FP64, reference statements)        */
#define CISMGPU_ALG_CHRONGEAR       1  /* pcg_solver_chrongear_* (FP64, reference statements)        */
#define CISMGPU_ALG_MIXED_CHRONGEAR 2  /* FP32 inner Chronopoulos-Gear + FP64 iterative refinement  */

/* dims = 3 (27-point blocks, indxA = indxA_3d) or 2 (9-point blocks, indxA = indxA_2d, nz = 1).
 * Array arguments as for the solver calls above; x0 may be NULL (zero initial guess).
 * 3D handles use the standard indxA_2d (m = 1 + (iA+1) + 3*(jA+1)) where the tridiagonal
 * preconditioners (3, 4) read the vertically summed couplings. */
int cismgpu_solver_create(cismgpu_solver_t **out, int dims, int nx, int ny, int nz,
                          const cismgpu_par_t *par, const int32_t *indxA, const int32_t *active_vertex,
                          const double *Auu, const double *Auv, const double *Avu, const double *Avv,
                          const double *bu, const double *bv, const double *xu0, const double *xv0,
                          void *cuda_stream);

/* Solve from the stored x0; err/niters as in the reference calls (for the mixed
 * algorithm: err is the FP64 true relative residual, niters the total inner
 * iterations).  Blocks until the solve has finished.  The mixed algorithm takes
 * precond 0, 1, 2 (3D) and the tridiagonal line preconditioners 3 and 4: their
 * setup is the FP64 one (a zero pivot returns CISMGPU_EDIVZERO, x unchanged), the
 * line solves run in FP32, and 2D solves run to maxiters (pcg_solver_chrongear_2d's
 * budget of 100 iterations for these preconditioners, which the FP64 algorithms keep,
 * counts FP64 iterations; the FP32 recurrences can need more). */
int cismgpu_solver_solve(cismgpu_solver_t *s, int algorithm, int precond, int linear_solve_ncheck,
                         double tolerance, int maxiters, double *err, int *niters);

/* Solve n independent systems (uneven sizes allowed) in ONE persistent cooperative
 * launch on cuda_stream (NULL: the first handle's stream).  algorithm must be
 * CISMGPU_ALG_MIXED_CHRONGEAR; all handles must have the same dims, and nz <= 32.
 * Every system's result is bit-identical to the same system batched alone
 * (batches use a dynamic persistent kernel with per-system tile heights, so
 * what else is in the batch never changes a result).  Per-system
 * err/niters/status arrays of length n; returns the first nonzero status. */
int cismgpu_solver_solve_batch(cismgpu_solver_t **solvers, int n, int algorithm, int precond,
                               int linear_solve_ncheck, double tolerance, int maxiters,
                               double *errs, int *niters, int *statuses, void *cuda_stream);

/* ------------------------------------------------------------------------
 * Graph-captured batches (no reference counterpart).  cismgpu_batch_create
 * prepares the mixed solver on every member (FP32 matrix, preconditioner,
 * per-member tile height), plans one persistent launch over all their tiles
 * and captures a whole batched solve -- resets to each member's x0, the launch,
 * the results -- into a CUDA graph.  cismgpu_batch_run replays it
 * (asynchronously, on the batch's stream); cismgpu_batch_wait synchronizes and
 * returns per-member err/niters/status.  Until cismgpu_batch_destroy the
 * members belong to the batch: cismgpu_solver_solve, _solve_batch, _destroy
 * and another batch_create on them return CISMGPU_EINVAL; cismgpu_solver_get_x
 * first waits for the batch's stream.  A changed matrix needs a new batch.
 * Results are bit-identical to cismgpu_solver_solve_batch and to each member
 * batched alone.  cuda_stream NULL: the batch creates its own stream.
 * ------------------------------------------------------------------------ */
typedef struct cismgpu_batch cismgpu_batch_t;
int cismgpu_batch_create(cismgpu_batch_t **out, cismgpu_solver_t **solvers, int n, int precond,
                         int linear_solve_ncheck, double tolerance, int maxiters, void *cuda_stream);
int cismgpu_batch_run(cismgpu_batch_t *b);
int cismgpu_batch_wait(cismgpu_batch_t *b, double *errs, int *niters, int *statuses);
int cismgpu_batch_destroy(cismgpu_batch_t *b);

/* ------------------------------------------------------------------------
 * Serving loop (no reference counterpart): continuous batching of independent
 * solves with the mixed-precision solver.  A host thread admits requests in
 * arrival order within an HBM budget (each admitted request holds its own
 * device-resident matrix and Krylov state), runs every admitted request in
 * epochs of at most epoch_steps steps of one persistent launch per kernel class
 * (2D, 3D nz <= 16, 3D nz <= 32), and between epochs retires finished requests
 * (x copied to the caller, device memory freed) and admits new ones, whose
 * upload overlaps the running epoch.  A request's result is bit-identical
 * whether it is served alone or in any mix.
 * The arrays a request points to must stay valid until it is done; xu/xv
 * receive the solution (caller's layout) when it completes.
 * ------------------------------------------------------------------------ */
typedef struct cismgpu_server cismgpu_server_t;
typedef struct cismgpu_request {
    int dims;                        /* 2 or 3                                  */
    int nx, ny, nz;                  /* nz ignored (1) for dims = 2             */
    const cismgpu_par_t *par;        /* copied at submit                        */
    const int32_t *indxA;            /* indxA_3d (27) or indxA_2d (9)           */
    const int32_t *active_vertex;
    const double *Auu, *Auv, *Avu, *Avv;
    const double *bu, *bv;
    const double *xu0, *xv0;         /* initial guess, NULL: zero               */
    double *xu, *xv;                 /* solution, written on completion         */
    int precond, linear_solve_ncheck;
    double tolerance;
    int maxiters;
} cismgpu_request_t;
int cismgpu_server_create(cismgpu_server_t **out, size_t hbm_budget_bytes, int epoch_steps);
int cismgpu_server_submit(cismgpu_server_t *s, const cismgpu_request_t *req, long long *id);
/* done: 1 once xu/xv hold the result; latency_ms: submit to completion (or to now);
 * queue_ms: submit to admission. */
int cismgpu_server_poll(cismgpu_server_t *s, long long id, int *done, double *err, int *niters, int *status,
                        double *latency_ms, double *queue_ms);
int cismgpu_server_drain(cismgpu_server_t *s);  /* wait until every submitted request is done and its
                                                   device memory released */
int cismgpu_server_stats(cismgpu_server_t *s, long long *epochs, size_t *bytes_in_use, int *active, int *queued);
/* Kernel launches of the serving loop so far (one per kernel class and epoch), and how many of
 * them held 2D and 3D requests together in one multi-class launch. */
int cismgpu_server_launch_stats(cismgpu_server_t *s, long long *launches, long long *multi_class_launches);
int cismgpu_server_destroy(cismgpu_server_t *s); /* finishes the queued requests first */

/* Copy the current solution (caller's Fortran layout, halo entries included) to host memory. */
int cismgpu_solver_get_x(cismgpu_solver_t *s, double *xu, double *xv);

/* The Picard loop on a handle, with A, b and x kept in HBM between nonlinear iterations:
 *  cismgpu_solver_set_system  new coefficients and right-hand side for the same geometry and
 *                             active vertices; with x0_from_solution != 0 and a solve done since
 *                             the last system, the next initial guess is that solution (on the
 *                             device: nothing crosses PCIe but A and b);
 *  cismgpu_solver_residual_vector   compute_residual_vector of the current velocity (the last
 *                             solution, or the stored initial guess if no solve ran since the
 *                             system was set) with the current A and b; resid_u/resid_v may be
 *                             NULL (norms only), L2_norm_relative may be NULL;
 *  cismgpu_solver_residual_velocity compute_residual_velocity between the last solution and
 *                             the initial guess that solve started from (EINVAL before a solve). */
int cismgpu_solver_set_system(cismgpu_solver_t *s, const double *Auu, const double *Auv, const double *Avu,
                              const double *Avv, const double *bu, const double *bv, int x0_from_solution);
int cismgpu_solver_residual_vector(cismgpu_solver_t *s, double *resid_u, double *resid_v, double *L2_norm,
                                   double *L2_norm_relative);
int cismgpu_solver_residual_velocity(cismgpu_solver_t *s, int whichresid, double *resid_velo);

/* The saved state of evaluate_accelerated_picard_{2d,3d} (glissade_velo_higher.F90:9898-10184)
 * on a handle: cismgpu_solver_save keeps a device copy of the current velocity and of A
 * ("uvel_sav = uvel; Auu_sav = Auu ..."; b is not saved, as there); cismgpu_solver_restore
 * brings them back ("uvel = uvel_sav; Auu = Auu_sav ...": the restored velocity becomes the
 * current one and the next solve's initial guess).  The scalar decision between extending,
 * accepting and restoring stays with the caller.  Restore without a save: CISMGPU_EINVAL. */
int cismgpu_solver_save(cismgpu_solver_t *s);
int cismgpu_solver_restore(cismgpu_solver_t *s);

/* check_symmetry_assembled_matrix_{3d,2d} (see above) on the handle's resident blocks: in 3D
 * the averages are written into the device copy that the next solve uses (the caller's host
 * arrays are not touched); in 2D nothing changes.  maxdiff and nwarn may be NULL. */
int cismgpu_solver_check_symmetry(cismgpu_solver_t *s, double *maxdiff, long long *nwarn);

/* cismgpu_assemble_stiffness_matrix_3d (see above) into a 3D handle's resident blocks: the
 * next solve, residual or check uses the assembled A without it crossing PCIe.  uvel = vvel =
 * NULL takes the handle's current velocity (the last solution, else the initial guess), so a
 * Picard loop uploads only the geometry and flow factor.  efvs may be NULL.  The right-hand
 * side and the boundary conditions are not touched (cismgpu_solver_set_system replaces all). */
int cismgpu_solver_assemble_stiffness_3d(cismgpu_solver_t *s, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel, const double *vvel, const double *stagusrf,
                                         const double *stagthck, const double *flwafact, int whichapprox,
                                         int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                         double *efvs);
/* One Picard iteration's 3D system on the device, as glissade_velo_higher_solve builds it
 * (glissade_velo_higher.F90:2829-2904): the stiffness blocks from the handle's current velocity,
 * the local basal term (beta, lsrf; both NULL for a no-slip bed), b = the load vector
 * (loadu, loadv), the Dirichlet conditions (masks NULL: none) with the current velocity as the
 * prescribed values, and the staggered halo of A and b.  Only the 2D fields, the flow factor,
 * the load and the masks cross PCIe; A is built in HBM. */
int cismgpu_solver_assemble_system_3d(cismgpu_solver_t *s, int nhalo, double dx, double dy, const double *sigma,
                                      const int32_t *active_cell, const int32_t *active_vertex,
                                      const double *xVertex, const double *yVertex, const double *stagusrf,
                                      const double *stagthck, const double *flwafact, int whichapprox,
                                      int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                      const double *beta, const double *lsrf, int whichassemble_beta,
                                      const double *loadu, const double *loadv, const int32_t *umask_dirichlet,
                                      const int32_t *vmask_dirichlet, double *efvs);

/* The 2D (SSA) counterpart (glissade_velo_higher.F90:2560-2666): stiffness from the handle's
 * current velocity, local basal term (beta NULL: none), b = load, Dirichlet (masks (nx-1,ny-1),
 * NULL: none), staggered halo of A and b.  nz: the sigma levels of flwafact. */
int cismgpu_solver_assemble_system_2d(cismgpu_solver_t *s, int nz, int nhalo, double dx, double dy,
                                      const double *sigma, const int32_t *active_cell, const int32_t *active_vertex,
                                      const double *xVertex, const double *yVertex, const double *stagthck,
                                      const double *flwafact, int whichefvs, double efvs_constant,
                                      double effstrain_min, double n_glen, const double *beta, int whichassemble_beta,
                                      const double *loadu, const double *loadv, const int32_t *umask_dirichlet,
                                      const int32_t *vmask_dirichlet, double *efvs);

/* The DIVA assembly into a 2D handle.  The layer viscosities per Gauss point stay in HBM
 * between calls (zero at first, as the reference's); efvs_qp_3d_in non-NULL replaces them
 * first.  uvel_2d = vvel_2d = NULL: the handle's current velocity.  efvs, omega_k, omega may be
 * NULL. */
int cismgpu_solver_assemble_stiffness_2d_diva(cismgpu_solver_t *s, int nz, int nhalo, const double *sigma,
                                              const double *stagsigma, const int32_t *active_cell,
                                              const double *xVertex, const double *yVertex, const double *uvel_2d,
                                              const double *vvel_2d, const double *stagthck, const double *thck,
                                              const double *btractx, const double *btracty,
                                              const double *diva_slope_factor_x, const double *diva_slope_factor_y,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const double *efvs_qp_3d_in,
                                              double *efvs, double *omega_k, double *omega);

/* The DIVA system of one Picard iteration on a 2D handle (:2560-2666 with whichapprox =
 * HO_APPROX_DIVA): the DIVA stiffness from the current velocity and the kept layer viscosities,
 * the DIVA basal term (beta_eff_x/_y, lsrf; NULL: none), b = load, Dirichlet, halo. */
int cismgpu_solver_assemble_system_2d_diva(
    cismgpu_solver_t *s, int nz, int nhalo, double dx, double dy, const double *sigma, const double *stagsigma,
    const int32_t *active_cell, const int32_t *active_vertex, const double *xVertex, const double *yVertex,
    const double *stagthck, const double *thck, const double *btractx, const double *btracty,
    const double *diva_slope_factor_x, const double *diva_slope_factor_y, const double *flwafact, int whichefvs,
    double efvs_constant, double effstrain_min, double n_glen, const double *beta_eff_x, const double *beta_eff_y,
    const double *lsrf, int whichassemble_beta, const double *loadu, const double *loadv,
    const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet, double *efvs, double *omega_k, double *omega);

/* The 2D (SSA) assembly into a 2D handle; nz: the number of sigma levels of flwafact. */
int cismgpu_solver_assemble_stiffness_2d(cismgpu_solver_t *s, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                         const double *flwafact, int whichefvs, double efvs_constant,
                                         double effstrain_min, double n_glen, double *efvs);

/* Per-kernel CUDA-event timing of the structured matvec launches (off by default).
 * read: total device milliseconds, launch count, and algorithmic bytes per launch
 * (active owned nodes x (4*NC*sizeof(A) + vector streams)). */
int cismgpu_solver_profile(cismgpu_solver_t *s, int enable);
int cismgpu_solver_profile_read(cismgpu_solver_t *s, double *total_ms, int *launches, double *bytes_per_launch);

/* Device bytes held by the handle. */
size_t cismgpu_solver_device_bytes(const cismgpu_solver_t *s);

int cismgpu_solver_destroy(cismgpu_solver_t *s);

/* Algorithm used by the four reference-signature calls above.  Default (-1): the
 * reference algorithm each call names, in FP64 (bit-reproducible, parity-tested).
 * CISMGPU_ALG_MIXED_CHRONGEAR: all four calls run the mixed-precision persistent
 * Chronopoulos-Gear solver instead (same system, same err definition, FP64 true
 * residual below the tolerance; x agrees with the FP64 solution to the accuracy the
 * tolerance implies).  No reference counterpart: a configuration switch of this
 * library.  Returns the previous setting. */
int cismgpu_set_oneshot_algorithm(int algorithm);

/* Order of the global sums when parallel%reprosum is off.
 * CISMGPU_SUM_TREE (default): the library's fixed double-double reduction tree, run by many
 *   CTAs: reproducible run to run and launch-independent, the correctly rounded exact sum
 *   except in rare near-tie cases.
 * CISMGPU_SUM_SEQUENTIAL: the reference's own order, parallel_global_sum_stagger's non-reprosum
 *   loop (libglimmer/parallel_mpi.F90:6770 3D, :6637 2D, nflds forms :7042, :6904):
 *   local_sum = local_sum + arr1 + arr2 over the owned vertices, j outer, then i, then k, each
 *   addition rounded in turn, the work arrays' products (worku = ru*zu, ...) rounded first.
 *   A solve then reproduces the reference's one-rank run bit for bit, whatever the conditioning
 *   of its trajectory.  The chain of additions runs on one GPU thread (the other threads of its
 *   CTA stage the summands), so each sum costs one pass at the latency of a dependent FP64 add
 *   per summand: a mode for parity and reproduction runs, not for speed.
 * Process-wide; read by the FP64 solvers at each solve (the four one-shot calls and
 * cismgpu_solver_solve with CISMGPU_ALG_STANDARD / _CHRONGEAR), by cismgpu_global_sum_stagger
 * and by cismgpu_global_sum_stagger_noalloc.  par->reprosum != 0 takes precedence, as in the
 * reference.  The mixed-precision solver ignores it.  Any other value selects
 * CISMGPU_SUM_TREE.  No reference counterpart (the reference has one order per build).
 * Returns the previous setting. */
#define CISMGPU_SUM_TREE        0
#define CISMGPU_SUM_SEQUENTIAL  1
int cismgpu_set_sum_order(int order);

/* Matrix layout of the mixed-precision solver's FP32 and FP64 copies (no reference counterpart).
 * CISMGPU_MIXED_LAYOUT_AUTO (default): a 3D matrix whose every lower coupling of an owned active
 *   row equals its transpose partner bit for bit (Auu with Auu, Auv with Avu, Avv with Avv at the
 *   neighbour node and the opposite offset; check_symmetry_assembled_matrix_3d, which the
 *   reference runs before every 3D solve, glissade_velo_higher.F90:2923-2931, makes it so) is
 *   stored as its symmetric half: the diagonal and the 13 upper couplings of each node (224 of
 *   432 FP32 bytes, 448 of 864 FP64), a lower coupling read from its partner.  The coefficients
 *   are the same numbers either way, so results are bit-identical to the full layout.  Any other
 *   matrix keeps all 27 couplings.
 * CISMGPU_MIXED_LAYOUT_FULL: all couplings always.
 * Process-wide, read whenever a handle builds its mixed copies (first mixed solve after an
 * upload or a new system).  Returns the previous setting. */
#define CISMGPU_MIXED_LAYOUT_AUTO 0
#define CISMGPU_MIXED_LAYOUT_FULL 1
int cismgpu_set_mixed_layout(int layout);

/* The mixed solver's tile heights (no reference counterpart).  The kernels cut a system's owned
 * vertices into 32 x TY tiles; a tuner times the candidate heights on the system itself the first
 * time it meets a key -- single solves: (dims, nz, layout, tile columns, height bucket); batches:
 * the least height per (dims, nz class), timed on a short launch of the first such batch -- and
 * keeps the winner for the process and in a cache file ($CISMGPU_TILE_CACHE, else
 * $HOME/.cache/cismgpu/tiles-<GPU name>.txt), so a system's tiling, and its rounding, depends on
 * the system alone.  The occupancy rule is the default and stays unless a candidate is more than
 * 3 % faster; CISMGPU_TILE_TUNING=0 turns timing off; the serving loop uses the table and never
 * times.  cismgpu_tile_table writes the table, one "key height [# timings]" line per key, into buf
 * (NUL-terminated, truncated to len) and returns the length it needs. */
size_t cismgpu_tile_table(char *buf, size_t len);

/* Whether the handle's mixed copies hold the symmetric half (1) or every coupling (0; also
 * before its first mixed solve). */
int cismgpu_solver_mixed_layout(const cismgpu_solver_t *s, int *symmetric_half);

/* Test hook for the bounded device waits of the mixed-precision kernels (single solves,
 * batches and serving epochs); no reference counterpart.  Every spin-wait of those kernels
 * gives up after wait_cycles SM clock cycles (<= 0: the default, 2^31, about 1 s), sets the
 * launch's abort word, and the launch ends with CISMGPU_ETIMEOUT for every solve it had not
 * finished; the context stays usable and the next solve starts from a clean state.
 * withhold_step != 0 makes tile 0 of every solve skip publishing its record of that step
 * (steps count from 1 in each solve), so the waits for that record run out: a wait on a flag
 * nothing sets, the way the tests exercise the timeout path without any fault.  (0, 0)
 * restores normal operation.  Applies to the current device, to launches made after the call. */
int cismgpu_test_set_device_waits(long long wait_cycles, unsigned int withhold_step);

/* Message for the last nonzero status on the calling thread ("" if none). */
const char *cismgpu_last_error(void);

/* Library version string. */
const char *cismgpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CISMGPU_H */
