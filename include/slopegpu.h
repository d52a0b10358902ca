/*
 * slopegpu.h -- C ABI of the B200 Newton-step hot path for SSR/LL continuation on P2
 * finite elements (drop-in for the native layer of Beremi/slope_stability_octave).
 *
 * Conventions
 *   - Every function returns SG_OK (0) or a negative SG_ERR_* code; sg_last_error()
 *     gives the message of the calling thread's last failure.  Nothing aborts.
 *   - Host-buffer entry points ("drop-in") take and return plain host arrays with the
 *     reference MEX layouts (Octave column-major == per-point AoS), copy to the device,
 *     compute, copy back and return when done.  Callers own every buffer.
 *   - *_dev entry points take device pointers and a cudaStream_t (as void*), enqueue
 *     work and return without synchronising.
 *   - Indices in the reference-facing arrays (scatter maps, pattern I/J) are 1-based
 *     like Octave's; everything internal to the device is 0-based.
 *   - Branch ids: 0 elastic, 1 smooth face, 2 left edge, 3 right edge, 4 apex.
 */
#ifndef SLOPEGPU_H
#define SLOPEGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SG_OK = 0,
    SG_ERR_ARG = -1,      /* invalid argument (null pointer, bad size, bad option) */
    SG_ERR_CUDA = -2,     /* CUDA runtime error (message has the CUDA error string) */
    SG_ERR_NOMEM = -3,    /* device or host allocation failed */
    SG_ERR_STATE = -4,    /* object used before the required set-up step */
    SG_ERR_NUMERIC = -5,  /* numerical breakdown (NaN/Inf, singular coarse matrix) */
    SG_ERR_NODEVICE = -6  /* no CUDA device visible */
};

int sg_abi_version(void);
const char *sg_last_error(void);
int sg_device_count(void);

/* ------------------------------------------------------------------------------
 * (a1, a2) Mohr-Coulomb return mapping + consistent tangent, 3D.
 * Replaces constitutive_problem_3D_SDS_mex / constitutive_problem_3D_S_mex
 * (+CONSTITUTIVE_PROBLEM/mex/constitutive_problem_3D_SDS_mex.c:29-64,
 *  constitutive_problem_3D_S_mex.c:29-59; per-point kernel constitutive_3D_kernel.h:101-410).
 *   E       6 x n_int  engineering strain (e11,e22,e33,g12,g23,g13), column-major
 *   c_bar, sin_phi, shear, bulk, lame   1 x n_int  (bulk is accepted and unused, as in the MEX)
 *   S       6 x n_int  out
 *   DS      36 x n_int out, column-major 6x6 per point (k = i + 6 j); NULL = stress only
 *   branch  n_int      out, optional (NULL)
 * ---------------------------------------------------------------------------- */
int sg_constitutive3d(const double *E, const double *c_bar, const double *sin_phi,
                      const double *shear, const double *bulk, const double *lame,
                      int64_t n_int, double *S, double *DS, uint8_t *branch);
int sg_constitutive3d_dev(const double *E, const double *c_bar, const double *sin_phi,
                          const double *shear, const double *bulk, const double *lame,
                          int64_t n_int, double *S, double *DS, uint8_t *branch, void *stream);

/* (a3) 2D plane-strain twin.  Replaces constitutive_problem_2D_{SDS,S}_mex
 * (+CONSTITUTIVE_PROBLEM/mex/constitutive_problem_2D_SDS_mex.c, kernel
 *  constitutive_2D_kernel.h:36-369).  E 3 x n_int, S 4 x n_int (s11,s22,s12,s33),
 *  DS 9 x n_int (3x3 column-major) or NULL. */
int sg_constitutive2d(const double *E, const double *c_bar, const double *sin_phi,
                      const double *shear, const double *bulk, const double *lame,
                      int64_t n_int, double *S, double *DS, uint8_t *branch);
int sg_constitutive2d_dev(const double *E, const double *c_bar, const double *sin_phi,
                          const double *shear, const double *bulk, const double *lame,
                          int64_t n_int, double *S, double *DS, uint8_t *branch, void *stream);

/* Allocation-free variant of sg_constitutive3d (no counterpart in the reference).  Same
 * arguments and outputs; stages through a fixed array in the library's device image instead
 * of cudaMalloc'd memory, on the legacy default stream, for callers that must not allocate
 * device memory after start-up.  At most SG_NOALLOC_MAX_POINTS points per call (larger n_int
 * returns SG_ERR_ARG with nothing launched).  The first call on a device sets up the array's
 * address and should come before any stream capture starts.  One array per device: calls
 * that overlap in time on the same device race on it and must be serialised by the caller. */
#define SG_NOALLOC_MAX_POINTS 16384
int sg_constitutive3d_noalloc(const double *E, const double *c_bar, const double *sin_phi,
                              const double *shear, const double *bulk, const double *lame,
                              int64_t n_int, double *S, double *DS, uint8_t *branch);

/* (a4) Davis strength reduction, +CONSTITUTIVE_PROBLEM/reduction.m:25-58 (types 'A','B','C';
 * type 'C' is applied point-wise).  Device pointers. */
int sg_reduction_dev(const double *c0, const double *phi, const double *psi, double lambda,
                     char davis_type, int64_t n, double *c_bar, double *sin_phi, void *stream);

/* Integrated elastoplastic potential sum_p WEIGHT_p * Psi(E_p), CONSTITUTIVE.potential_energy
 * (+CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m:363-387, Psi of potential_3D.m / potential_2D.m), the
 * energy of the SSR direct continuation (omega_SSR_direct_continuation.m:45-66).  E is the
 * strain (6 x n_int in 3D, 3 x n_int in 2D, engineering shears); device arrays; the sum is
 * returned to the host. */
int sg_potential_dev(int dim, const double *E, const double *c_bar, const double *sin_phi,
                     const double *shear, const double *bulk, const double *lame, const double *weight,
                     int64_t n_int, double *result, void *stream);

/* ------------------------------------------------------------------------------
 * (b3, b5) Element-level tangent assembly.  Replaces assemble_K_tangent_vals /
 * assemble_K_tangent_vals_2D (+ASSEMBLY/mex/assemble_K_tangent_vals.c:38-172,
 * assemble_K_tangent_vals_2D.c:31-165): V_tang[map-1] += (sum_q B_q'(w_q D_q)B_q)_loc.
 *   DPhi1..3  n_p x n_int (DPhi3 unused/NULL in 2D), DS (ns^2) x n_int, WEIGHT 1 x n_int
 *   scatter_map (dim*n_p)^2 x n_e int64, 1-based, 0 = skip (Dirichlet)
 *   V_tang nnz_out (zeroed and written by the call)
 * ---------------------------------------------------------------------------- */
int sg_assemble_ktangent3d(const double *DPhi1, const double *DPhi2, const double *DPhi3,
                           const double *DS, const double *WEIGHT, const int64_t *scatter_map,
                           int32_t n_p, int64_t n_int, int64_t n_e, int32_t n_q,
                           int64_t nnz_out, double *V_tang);
int sg_assemble_ktangent2d(const double *DPhi1, const double *DPhi2, const double *DS,
                           const double *WEIGHT, const int64_t *scatter_map, int32_t n_p,
                           int64_t n_int, int64_t n_e, int32_t n_q, int64_t nnz_out,
                           double *V_tang);
int sg_assemble_ktangent_dev(int dim, const double *DPhi1, const double *DPhi2, const double *DPhi3,
                             const double *DS, const double *WEIGHT, const int64_t *scatter_map,
                             int32_t n_p, int64_t n_e, int32_t n_q, int64_t nnz_out,
                             double *V_tang, void *stream);

/* ------------------------------------------------------------------------------
 * Device-resident mesh (set-up once per mesh).  Replaces the one-time part of the
 * CONSTITUTIVE object: set_element_data + init_K_r_pattern + build_scatter_map
 * (+CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m:393-464, 538-635).
 *   elem   n_p x n_e (column-major, 0-based node ids)
 *   DPhi*  n_p x n_int physical basis gradients, weight 1 x n_int (ASSEMBLY outputs)
 *   Q      dim x n_n free-DOF mask (column-major, 1 = free)
 * The stiffness lives in a node-adjacency block pattern (dim x dim blocks, all nodes);
 * Dirichlet DOFs carry identity rows/columns there.  The reference's scalar K(Q,Q)
 * pattern (Octave find() order) and its scatter map are produced on request.
 * ---------------------------------------------------------------------------- */
typedef struct sg_mesh sg_mesh;
typedef struct sg_bsr sg_bsr;

int sg_mesh_create(int dim, int32_t n_p, int32_t n_q, int64_t n_n, int64_t n_e, const int32_t *elem,
                   const double *DPhi1, const double *DPhi2, const double *DPhi3, const double *weight,
                   const uint8_t *Q, sg_mesh **out);
int sg_mesh_destroy(sg_mesh *mesh);
/* sizes[0..4] = n_dof (dim*n_n), n_Q, nnz of K(Q,Q), BSR blocks, n_int */
int sg_mesh_sizes(const sg_mesh *mesh, int64_t *sizes);
/* borrowed pointer to the mesh's block pattern (valid until sg_mesh_destroy) */
int sg_mesh_bsr(const sg_mesh *mesh, const sg_bsr **bsr);
/* (b1) ref_I, ref_J: 1-based pattern of K(Q,Q) in find() order; transpose_perm: 1-based
 * position of (J,I) for every (I,J) (CONSTITUTIVE.m:445-454).  Any pointer may be NULL. */
int sg_mesh_pattern(const sg_mesh *mesh, int64_t *ref_I, int64_t *ref_J, int64_t *transpose_perm);
/* (b2) the reference's element scatter map, (dim*n_p)^2 x n_e int64 (CONSTITUTIVE.m:582-635) */
int sg_mesh_scatter_map(const sg_mesh *mesh, int64_t *scatter_map);
/* 0-based DOF index of every free DOF, in order (Octave find(Q(:)) - 1) */
int sg_mesh_free_dofs(const sg_mesh *mesh, int64_t *q_flat);

/* (a5) E = B U: U dim x n_n (column-major), E n_strain x n_int (CONSTITUTIVE.m:218) */
int sg_strain_dev(const sg_mesh *mesh, const double *U, double *E, void *stream);
/* (a6) F = B' (w .* S(1:n_strain,:)): S has s_rows rows per point; F dim x n_n (CONSTITUTIVE.m:281) */
int sg_force_dev(const sg_mesh *mesh, const double *S, int32_t s_rows, double *F, void *stream);
/* (a5 + a1/a2 + a6 fused) stress-only residual of P2 tetrahedra: F = B'(w .* S(B U)) with
 * the reduced strength (c_bar, sin_phi) and the stress-only return mapping in between: the
 * chain sg_strain_dev -> sg_constitutive3d_dev(DS = NULL) -> sg_force_dev of
 * CONSTITUTIVE.build_F_reduced / build_F_all (CONSTITUTIVE.m:218-233, 268-285) in one kernel,
 * E and S never stored.  branch (n_int, optional) receives the branch ids; F (3 x n_n) is
 * zeroed and written.  3D, n_p = 10 only (SG_ERR_ARG otherwise). */
int sg_residual_dev(const sg_mesh *mesh, const double *U, const double *c_bar, const double *sin_phi,
                    const double *shear, const double *lame, uint8_t *branch, double *F, void *stream);
/* (b3) K_t = sum_e B'(w DS)B into the block pattern (values zeroed first) */
int sg_assemble_bsr_dev(const sg_mesh *mesh, const double *DS, double *K, void *stream);
/* DS_elast of CONSTITUTIVE.m:413-422 per point (n_strain^2 x n_int) */
int sg_elastic_ds_dev(const sg_mesh *mesh, const double *shear, const double *bulk, double *DS, void *stream);
/* Ks = (K + K')/2 on the block pattern */
int sg_symmetrize_bsr_dev(const sg_mesh *mesh, const double *K, double *Ks, void *stream);
/* (b4) K_r = sym(r K_el + (1-r) K_t) with Dirichlet identity (CONSTITUTIVE.m:515-532) */
int sg_kr_blend_dev(const sg_mesh *mesh, double r, const double *K_el, const double *K_t, double *K_r, void *stream);
/* (b3 + b4) K_r = r K_el + (1 - r) K_t with K_t assembled from DS in the same call (the
 * sequence build_K_tangent_QQ_vals + build_K_r_QQ_vals, CONSTITUTIVE.m:515-532 and
 * assemble_K_tangent_vals.c:77-171).  On P2 tetrahedra the assembly is deterministic (fixed
 * summation order, bitwise reproducible) and exactly symmetric, and K_t itself is not stored
 * (K_t_scratch may be NULL); other elements assemble into K_t_scratch, then blend. */
int sg_assemble_kr_dev(sg_mesh *mesh, const double *DS, double r, const double *K_el, double *K_t_scratch,
                       double *K_r, void *stream);
/* block-pattern values -> V in the reference's find() order (nnz of K(Q,Q)) */
int sg_bsr_to_ref_dev(sg_mesh *mesh, const double *K, double *V_ref, void *stream);

/* ------------------------------------------------------------------------------
 * Unconfined seepage (+SEEPAGE: seepage_problem_3D.m / seepage_problem_2D.m, newton_flow.m)
 * on the mechanical mesh.  The pore pressure is one value per node; its systems live in the
 * mesh's node adjacency with 1 x 1 blocks (sg_mesh_bsr_scalar), usable with sg_amg_create
 * (near-null space: the constant, nns = 1), sg_dfgmres_solve and sg_a_orthogonalize.
 *   hat      n_q x n_p basis values at the quadrature points (HatP transposed: point-major)
 *   conduct  n_int conductivity per point (heter_conduct.m); eps n_e penalty per element
 *            (penalty_parameters_3D.m / _2D.m); gy dim x n_int = Bw * y (the gradient of the
 *            vertical coordinate, q2 of seepage_problem_3D.m:43)
 *   mask     n_n, 1 free / 0 Dirichlet node (Q_w); NULL leaves K and F unmasked
 * ---------------------------------------------------------------------------- */
/* borrowed pointer to the node adjacency with 1 x 1 blocks (device arrays shared with
 * sg_mesh_bsr's pattern; valid until sg_mesh_destroy) */
int sg_mesh_bsr_scalar(sg_mesh *mesh, const sg_bsr **bsr);
/* K (n_blocks of the pattern, zeroed first, may be NULL) and F (n_n, zeroed first, may be
 * NULL) at the pressure pw:
 *   F = -Bw'(wc .* (Bw pw + grho kappa .* gy))      (newton_flow.m:120-123)
 *   K = K_D + Bw' E C, E = conduct .* perm_r' .* weight .* (grho gy)   (newton_flow.m:104-118)
 * kappa_mode 0: kappa = 0 and K = K_D (seepage_problem_2D.m initial right-hand side);
 * 1: kappa = 1, K = K_D (seepage_problem_3D.m:42-46); 2: kappa = perm_r(pw_int), Newton
 * tangent.  With mask, Dirichlet rows/columns of K become identity and F is zero there. */
int sg_seepage_system_dev(const sg_mesh *mesh, const double *hat, const double *pw, const double *conduct,
                          const double *eps, const double *gy, double grho, int32_t kappa_mode,
                          const double *mask, double *K, double *F, void *stream);
/* grad = Bw * field per integration point: field n_n, grad dim x n_int (point-major):
 * q2 = Bw y (seepage_problem_3D.m:43) and grad_p = Bw pw (:62) */
int sg_point_gradient_dev(const sg_mesh *mesh, const double *field, double *grad, void *stream);
/* per element: mean (n_e, may be NULL) = weighted mean of pw over its integration points,
 * sat (n_e, may be NULL) = mean >= 0.1 eps (seepage_problem_3D.m:63-74) */
int sg_seepage_saturation_dev(const sg_mesh *mesh, const double *hat, const double *pw, const double *eps,
                              double *mean, uint8_t *sat, void *stream);

/* ------------------------------------------------------------------------------
 * (c2) Block sparse matrix-vector product and reductions (device pointers).
 * ---------------------------------------------------------------------------- */
/* info[0..2] = block size, block rows, blocks */
int sg_bsr_info(const sg_bsr *A, int64_t *info);
int sg_bsr_spmv_dev(const sg_bsr *A, const double *vals, const double *x, double *y, void *stream);
/* *result = x'y (synchronises the stream) */
int sg_dot_dev(int64_t n, const double *x, const double *y, double *result, void *stream);
/* *result = sum mask .* (a - b).^2  (b, mask may be NULL; synchronises the stream) */
int sg_masked_diff_norm2_dev(int64_t n, const double *a, const double *b, const double *mask, double *result,
                             void *stream);
/* y = a x + b y */
int sg_axpby_dev(int64_t n, double a, const double *x, double b, double *y, void *stream);

/* ------------------------------------------------------------------------------
 * (d1, d2) AMG preconditioner.  Takes the role of the BoomerAMG instance of
 * +LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp (commands setup_ijv :1013-1146,
 * update_values :1151-1213, apply :751-796, clear): one V-cycle per apply, numeric
 * set-up redone on every value update.  Smoothed aggregation on the node blocks with a
 * near-null space (near_null_space_elasticity_3D.m: 6 rigid-body modes in 3D), Chebyshev
 * smoothing, FP64 or FP32 cycle.
 *   A_vals     device values of A used for the strength graph of every level (NULL: whole
 *              block graph); the numeric set-up runs during creation when given
 *   nullspace  (n_rows*b) x nns column-major host array; fixed: per-DOF 1 = Dirichlet (host)
 *   opts       [max_levels, coarse_size, cheb_degree, cheb_ratio, power_its, mixed(0/1),
 *               omega_scale, theta, fine_half(0/1), symmetric(0/1)]; entries <= 0 keep the
 *               defaults (10, 1200, 3, 10, 10, 0, 4/3, 0.02, 0, 0) except theta, where 0 selects
 *               the whole block graph.
 *               fine_half (mixed cycle, 3x3 blocks, theta > 0): the cycle's level-0 SpMVs read
 *               an FP16 copy of A scaled by a power of two (FP32 accumulation); the numeric
 *               set-up stays FP32.
 *               symmetric: the caller's A is symmetric (as K_r is), so each Galerkin matrix
 *               P'AP is formed on and above its diagonal only and mirrored below it (half the
 *               P'(AP) work, and A P only where those blocks read it); leave 0 for a
 *               non-symmetric A (the seepage tangent)
 * ---------------------------------------------------------------------------- */
typedef struct sg_amg sg_amg;
int sg_amg_create(const sg_bsr *A, const double *A_vals, const double *nullspace, int32_t nns,
                  const uint8_t *fixed, const double *opts, int32_t n_opts, sg_amg **out, void *stream);
int sg_amg_destroy(sg_amg *amg);
/* A second set of V-cycle vectors over the hierarchy of `amg` (no counterpart in the
 * reference): the clone shares every matrix, transfer operator and inverse and follows the
 * parent's updates, so sg_amg_apply on the parent and on the clone may run at the same time
 * on different streams (the two independent Krylov solves of a Newton step).  Only the parent
 * is updated (sg_amg_update on a clone is SG_ERR_ARG); destroy the clone before the parent;
 * no learned correction on a clone. */
int sg_amg_clone(const sg_amg *amg, sg_amg **clone);
/* numeric set-up from device values of A (kept by reference until the next update) */
int sg_amg_update(sg_amg *amg, const double *A_vals, void *stream);
/* z = V-cycle(r), device vectors of n_rows*b entries */
int sg_amg_apply(sg_amg *amg, const double *r, double *z, void *stream);
/* info[0] levels, info[1] coarsest dense size, then (block size, block rows, blocks) per level
 * (at most 10 levels); with cap > 32, info[32 + l] = blocks of level l's prolongator */
int sg_amg_info(const sg_amg *amg, int64_t *info, int32_t cap);
/* ------------------------------------------------------------------------------
 * (d1, d2) Preconditioner instances keyed by id over host COO triplets.  Replaces the
 * command set of hypre_boomeramg_mex (+LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp:
 * 'setup_ijv' :1013-1146, 'update_values' :1151-1213, 'apply' :751-796, 'clear' :798-829,
 * 'info' :830-853), as called by DFGMRES.setup_preconditioner_ijv /
 * update_preconditioner_values (+LINEAR_SOLVERS/DFGMRES.m:172-202) through the closures of
 * set_linear_solver.m:216-240.
 *   id        instance name (the reference's instance_id string)
 *   I, J, V   nnz triplets of the full n x n matrix, I and J 1-based, stored as doubles
 *             (Octave numeric arrays); duplicate (I, J) entries are summed
 *   Z         n x nns near-null space, column-major (nns 0: the translations)
 *   dof_func  length n, component index of every unknown in [0, num_functions) (NULL:
 *             (q - 1) mod num_functions, as set_linear_solver.m builds it); consecutive
 *             unknowns with increasing component form one node block
 *   opts      numeric AMG options as for sg_amg_create (may be NULL)
 *   force_rebuild  0: an existing id with the same nnz keeps its pattern and takes the new
 *             values only (the reference's fast path); 1: rebuild
 *   setup_seconds  out (optional): wall time of the call, as the reference's
 *             setup_time_seconds
 * The instance lives on the device that is current at its creation and is used from any
 * thread (calls are serialised by the library).  apply takes and returns host vectors of
 * length n and returns when done.  Unknown ids give SG_ERR_STATE, bad sizes SG_ERR_ARG.
 * ---------------------------------------------------------------------------- */
int sg_amg_setup_ijv(const char *id, const double *I, const double *J, const double *V, int64_t nnz,
                     int64_t n, const double *Z, int32_t nns, const double *dof_func,
                     int32_t num_functions, const double *opts, int32_t n_opts, int32_t force_rebuild,
                     double *setup_seconds);
int sg_amg_update_values(const char *id, const double *V, int64_t nnz, double *setup_seconds);
int sg_amg_apply_host(const char *id, const double *r, double *y, int64_t n);
/* id NULL clears every instance */
int sg_amg_clear(const char *id);
/* id NULL: info[0] = number of instances; else info = [n, nnz, num_functions, nns, nodes,
 * blocks, full builds, value updates] (up to cap entries) */
int sg_amg_ijv_info(const char *id, int64_t *info, int32_t cap);
/* host copies of level l's A pattern/values and P pattern/values (any pointer may be NULL);
 * values are those of the FP64 numeric set-up: for a mixed-precision hierarchy (opts[5] != 0),
 * whose value updates run in FP32, they are the values of its set-up in sg_amg_create */
int sg_amg_export(const sg_amg *amg, int32_t level, int32_t *A_rp, int32_t *A_col, double *A_vals,
                  int32_t *P_rp, int32_t *P_col, double *P_vals);

/* ------------------------------------------------------------------------------
 * (c1, c3) Deflated FGMRES and A-orthogonalisation.
 *   sg_dfgmres_solve     +LINEAR_SOLVERS/dfgmres_solver.m:1-181 (DFGMRES.solve, DFGMRES.m:134-147)
 *   sg_a_orthogonalize   +LINEAR_SOLVERS/A_orthogonalize.m:1-58 (DFGMRES.A_orthogonalize)
 * Device vectors of n entries; the deflation basis W is n x k column-major (device).
 * ---------------------------------------------------------------------------- */
typedef struct sg_krylov sg_krylov;
int sg_krylov_create(int64_t n, int32_t maxit, sg_krylov **out);
int sg_krylov_destroy(sg_krylov *ws);
/* AW = A W (optional, may be NULL): as produced by sg_a_orthogonalize; when given, the
 * projection w - W (W' (A w)) is evaluated as w - W ((A W)' w) (A symmetric), saving one
 * SpMV per iteration. */
int sg_dfgmres_solve(sg_krylov *ws, const sg_bsr *A, const double *A_vals, sg_amg *M, const double *W,
                     const double *AW, int32_t k, const double *b, double *x, double tol, int32_t maxit,
                     int32_t *iters, double *relres, double *res_hist, void *stream);
/* Solves run as one replayed CUDA graph per (matrix, preconditioner): start, the iteration
 * loop (a conditional WHILE node) and the least-squares solution stay on the device, with one
 * host synchronisation per solve (on = 1, the default); on = 0 selects the host-driven loop
 * (one synchronisation per iteration).  Both give the same iterates. */
int sg_krylov_set_graph(sg_krylov *ws, int32_t on);
/* How sg_a_orthogonalize forms the basis (replaces nothing in the reference: both modes are
 * A_orthogonalize.m's one-pass recurrence, +LINEAR_SOLVERS/A_orthogonalize.m:27-48).
 * mode 1 (default): G = S'(A S) for the input columns S, the recurrence on the k x k matrix
 * G (coefficients (T'G)(j,i), norms t'G(:,i)), then the kept columns U = S T and A U = (A S) T
 * by two tall-skinny products; mode 0: column-blocked Gram-Schmidt on the n-long vectors.
 * Same kept columns and the same basis up to rounding. */
int sg_krylov_set_aorth(sg_krylov *ws, int32_t mode);
/* AW (optional, may be NULL): receives A times the kept columns of W, in W's output order. */
int sg_a_orthogonalize(sg_krylov *ws, const sg_bsr *A, const double *A_vals, double *W, double *AW,
                       int32_t k, double eps_add, int32_t *k_out, void *stream);

/* ------------------------------------------------------------------------------
 * Learned node-wise correction of the V-cycle (no counterpart in the reference, whose
 * DFGMRES is preconditioned by one BoomerAMG V-cycle: hypre_boomeramg_mex.cpp:751-796).
 * With a correction set, the preconditioner inside sg_dfgmres_solve becomes
 *     z = V(r);   z += C (r - A z),   C_i = M_i G_i D_i^{-1}  (3 x 3 per node),
 * G_i = MLP(phi_i), a per-node network 16 -> 64 -> 64 -> 9 (ReLU) run on the tensor cores
 * (BF16 operands, FP32 accumulation) over node features phi from the matrix, the Newton
 * residual and the constitutive state; D_i the node's diagonal block, M_i its free-DOF mask.
 * Training minimises the residual norm |rz - A M G D^{-1} rz|^2 (or, as an option, the
 * energy norm of the error the corrected cycle leaves) over residual vectors rz = v - A V(v)
 * of the plain preconditioner, collected from the Newton system; the last layer starts at
 * zero, so the untrained correction is the plain V-cycle.
 * ---------------------------------------------------------------------------- */
#define SG_LEARNED_NPARAM 6288 /* W1[16][64] b1[64] W2[64][64] b2[64] W3[64][16] b3[16] (FP32) */
/* z += C (r - A z) after every V-cycle; C: device n_rows x 9 (row-major 3 x 3), copied;
 * NULL switches the correction off */
int sg_amg_set_correction(sg_amg *amg, const double *C, void *stream);
/* stateless network passes on device arrays: X is n_pad x 16 BF16 bit patterns (n_pad =
 * 128*ceil(n/128), padding rows zero), G and dG n_pad x 16 FP32 (columns 9..15 unused);
 * err: device int set to 1 when a tensor-core completion wait ran out (nothing then written) */
int sg_mlp_forward_dev(const float *params, const uint16_t *X, int64_t n, float *G, int *err, void *stream);
int64_t sg_mlp_part_size(int64_t n);
int sg_mlp_backward_dev(const float *params, const uint16_t *X, const float *dG, int64_t n, float *grad,
                        float *part, int *err, void *stream);

typedef struct sg_learned sg_learned;
/* coord: host 3 x n_n column-major node coordinates; max_vectors per slot; seed of the
 * initial weights (He-uniform, last layer zero) */
int sg_learned_create(const sg_mesh *mesh, const double *coord, int32_t max_vectors, uint64_t seed,
                      sg_learned **out);
int sg_learned_destroy(sg_learned *h);
/* host copy of the NPARAM parameters (set != 0 writes them and resets the optimiser) */
int sg_learned_params(sg_learned *h, float *host, int32_t set);
/* features and diagonal-block inverses for matrix values A_vals (device, mesh pattern), the
 * Newton residual res (device, dim*n_n), branch ids and reduced cohesion per integration
 * point (device; either may be NULL) */
int sg_learned_features(sg_learned *h, const double *A_vals, const double *res, const uint8_t *branch,
                        const double *c_bar, void *stream);
/* C from the current network; handed to amg when amg != NULL; copied to C_out when given */
int sg_learned_correction(sg_learned *h, sg_amg *amg, double *C_out, void *stream);
/* collect `count` residual vectors of the plain V-cycle on A x = b into slot 0 (training) or
 * 1 (held out), replacing (append = 0) or appending; switches amg's correction off */
int sg_learned_collect(sg_learned *h, sg_amg *amg, const sg_bsr *A, const double *A_vals, const double *b,
                       int32_t count, int32_t slot, int32_t append, void *stream);
/* training objective: 0 (default) the mean relative corrected residual |rz - A d|^2/|rz|^2;
 * 1 the mean change of the error's energy norm, (|e - d|_A^2 - |e|_A^2) / (rz' D^{-1} rz) with
 * A e = rz (0 for the plain cycle, negative when the correction helps) */
int sg_learned_set_loss(sg_learned *h, int32_t kind);
/* the training objective over a slot's vectors */
int sg_learned_loss(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t slot, double *loss,
                    void *stream);
/* gradient of that loss with respect to the parameters (host, NPARAM floats) */
int sg_learned_gradient(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t slot, float *grad,
                        double *loss, void *stream);
/* `steps` full-batch Adam steps on slot 0; loss_hist (host, may be NULL) gets the loss
 * before each step */
int sg_learned_train(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t steps, double lr,
                     double *loss_hist, void *stream);
/* host copy, for checks: what 0 features (n_pad x 16 BF16 bits), 1 last network output G
 * (n_pad x 16 FP32), 2 diagonal-block inverses (n_n x 9), 3 / 4 residual vector `index` of
 * slot 0 / 1 (dim*n_n), 5 the correction C (n_n x 9) */
int sg_learned_export(const sg_learned *h, int32_t what, int32_t index, void *host);
/* info: [NPARAM, vectors in slot 0, vectors in slot 1, padded node count, Adam steps taken] */
int sg_learned_info(const sg_learned *h, int64_t *info);

/* ------------------------------------------------------------------------------
 * Live kernel timing (no reference counterpart: profiling support in the spirit of the
 * reference's PROFILING.Profiler).  When enabled, every `sample`-th launch of each kind is
 * bracketed by CUDA events on its stream.  Kinds (capacity 12): 0 fine SpMV FP64 (FGMRES,
 * residuals), 1 fine SpMV FP32, 2 return mapping + tangent, 3 return mapping (stress),
 * 4 assembly, 5 AMG value update, 6 AMG V-cycle, 7 fine SpMV on the FP16 copy, 8 fine SpMV
 * FP64 inside sg_a_orthogonalize, 9 fused residual (sg_residual_dev), 10 fine SpMM FP64 of
 * sg_a_orthogonalize (several vectors per launch), 11 a whole sg_a_orthogonalize call (units:
 * basis columns).  sg_instr_read synchronises the device and resets the
 * counters.
 * ---------------------------------------------------------------------------- */
int sg_instr_enable(int on, int sample);
int sg_instr_read(double *ms, int64_t *timed, int64_t *launches, int32_t cap);
/* work units per kind since the last sg_instr_read (kind 10: vectors multiplied, kind 11:
 * basis columns) */
int sg_instr_units(int64_t *units, int32_t cap);
/* number of kernels the library launched since the last reset (reset != 0 clears it) */
int64_t sg_launch_count(int reset);
/* number of device allocations (cudaMalloc) the library made since the last reset (reset != 0
 * clears it); lets a caller check that a timed region allocated no device memory */
int64_t sg_device_alloc_count(int reset);
/* the library's device status word on the current device: bit 0 is set when the bulk-staged
 * element-block kernel of the P2-tetrahedron assembly gave up its bounded wait for a copy
 * (about one second; the K_t / K_r of that call is then incomplete).  Synchronises the device;
 * reset != 0 clears the word after reading it.  Returns SG_OK or an error code. */
int sg_device_status(int32_t reset, int32_t *status);

#ifdef __cplusplus
}
#endif
#endif /* SLOPEGPU_H */
