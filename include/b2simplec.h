/* b2simplec — the SIMPLEC outer iteration of an unstructured finite-volume solver, as
 * hand-written CUDA for NVIDIA B200 (sm_100a), behind a plain C ABI.
 *
 * Counterpart of FlowTrace's native kernel ABI (flowtrace/native/fvm_kernels.h:27-72, ABI 2)
 * and of the array code of flowtrace/unstructured/simple.py:500-703 that calls it. Differences
 * from the reference's ABI, all deliberate:
 *   - every pointer is a DEVICE pointer; each call takes the stream it is ordered on and
 *     never synchronises it (results that the host needs are written to device memory);
 *   - cell/face indices are int32 (the reference passes int64 face/cell indices);
 *   - every function returns an int status: B2S_OK, or a negative B2S_ERR_* code;
 *   - the library never allocates: callers pass work space, sized by the *_workspace_bytes
 *     queries (the reference's ft_bicgstab_jacobi takes its 7n-double work array the same way);
 *   - vector fields are component-major ("SoA"): a field with k components over n entities is
 *     k contiguous arrays of n values, component c at offset c*n.
 *
 * Entity order: cells in the mesh's device order (a reverse Cuthill-McKee permutation of the
 * reference's order), interior faces sorted by (owner, reference face index), boundary faces
 * sorted by (owner, reference boundary-face index). The host layer keeps the permutations
 * and converts to and from the reference's order.
 */
#ifndef B2SIMPLEC_H
#define B2SIMPLEC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2S_ABI_VERSION 5

#if defined(__GNUC__)
#define B2S_API __attribute__((visibility("default")))
#else
#define B2S_API
#endif

#define B2S_OK 0
#define B2S_ERR_ARG (-1)        /* invalid size, null pointer or unsupported option */
#define B2S_ERR_LAUNCH (-2)     /* a kernel launch failed (cudaGetLastError) */
#define B2S_ERR_WORKSPACE (-3)  /* work space smaller than the *_workspace_bytes query */
#define B2S_ERR_DEVICE (-4)     /* no usable device, or a device query failed */
#define B2S_ERR_TOO_LARGE (-5)  /* the problem exceeds a fixed capacity (b2s_bicgstab_jacobi_noalloc_d) */

typedef struct CUstream_st* b2s_stream_t; /* a cudaStream_t; NULL is the legacy default stream */

/* Finite-volume description of one mesh (device arrays). Counterpart of the arrays that
 * flowtrace/unstructured/fvmesh.py:61-230 precomputes. */
typedef struct b2s_mesh {
  int32_t nc, nf, nb, dim, nnz;
  /* interior faces: owner, neighbour, reference interior-face index */
  const int32_t* fP;
  const int32_t* fN;
  const int32_t* forig;
  const int32_t* own_ptr;  /* [nc+1]: the faces a cell owns are own_ptr[c] .. own_ptr[c+1]-1 */
  const int32_t* nei_ptr;  /* [nc+1] */
  const int32_t* nei_face; /* [nf]: faces whose neighbour is the cell, by reference face index */
  const int32_t* bP;       /* [nb] boundary-face owner */
  const int32_t* bptr;     /* [nc+1]: boundary faces of a cell */
  const double* w;         /* [nf] owner interpolation weight */
  const double* alpha;     /* [nf] S.S / S.d */
  const double* wl;        /* [nf] least-squares weight 1/|d|^2 */
  const double* S;         /* [dim][nf] area vector, owner -> neighbour */
  const double* d;         /* [dim][nf] x_N - x_P */
  const double* Tv;        /* [dim][nf] non-orthogonal part S - alpha d */
  const double* dxm;       /* [dim][nf] face centre minus its point on the P-N line */
  const double* dPf;       /* [dim][nf] owner centre -> face centre */
  const double* dNf;       /* [dim][nf] neighbour centre -> face centre */
  const double* alpha_b;   /* [nb] */
  const double* wlb;       /* [nb] */
  const double* Sb_mag;    /* [nb] */
  const double* Sb;        /* [dim][nb] outward area vector */
  const double* db;        /* [dim][nb] face centre minus owner centre */
  const double* nbv;       /* [dim][nb] unit outward normal */
  const double* dbt;       /* [dim][nb] tangential part of db */
  const double* vol;       /* [nc] */
  const double* Ginv;      /* [dim][dim][nc] inverse least-squares matrices */
  const int32_t* rowptr;   /* [nc+1] CSR pattern of cell-cell operators */
  const int32_t* col;      /* [nnz] (each row in the reference's column order) */
  const int32_t* slot_diag;/* [nc] */
  const int32_t* slot_PN;  /* [nf] CSR slot of (P, N) */
  const int32_t* slot_NP;  /* [nf] CSR slot of (N, P) */
  /* Optional tiling of the cells (NULL: none), for block-diagonal batches of independent cases:
   * tile t is cells tiles[t] .. tiles[t+1]-1, at most 256 cells, never two cases. With a tiling,
   * the stages that write per-block partial sums (momentum, pressure, correction and energy
   * assembly) give one partial per tile (b2s_mesh_part_blocks), so sums per case follow. */
  const int32_t* tiles;
  int32_t ntiles;
  int32_t pad_;
} b2s_mesh;

/* Boundary conditions as face masks (0/1 doubles, as flowtrace/unstructured/simple.py:228-240). */
typedef struct b2s_bc {
  const double* m_wall;
  const double* m_inlet;
  const double* m_pres;    /* outlet or pressure opening */
  const double* m_sym;
  const double* m_dirvel;  /* wall, inlet or symmetry: Dirichlet velocity */
  const double* ub_fixed;  /* [dim][nb] */
  const double* pb_fixed;  /* [nb] */
  const double* m_tfix;    /* [nb] fixed temperature */
  const double* m_tflux;   /* [nb] given heat flux */
  const double* m_out;     /* [nb] outlet (backflow takes tval) */
  const double* tval;      /* [nb] */
} b2s_bc;

/* ----------------------------------------------------------------------------------------- */
B2S_API int b2s_abi_version(void);
/* Number of multiprocessors of the current device (0 without a device). */
B2S_API int b2s_device_sm_count(void);

/* Device set-up of the finite-volume data from the raw mesh, in the reference's numbering and
 * operation order (replaces the host set-up of flowtrace/mesh/unstructured.py:171-261 and
 * flowtrace/unstructured/fvmesh.py:61-230). Points and vectors are row-major [n][dim].
 *
 * b2s_face_geometry_d: face centres fc and area vectors S of nf faces (face_ptr/face_nodes: the
 * nodes of face f are face_nodes[face_ptr[f] .. face_ptr[f+1]-1]); *bad counts faces with a
 * node count the dimension does not allow (2-D: 2; 3-D: 3..32).
 *
 * b2s_cell_geometry_d: cell volumes and centroids by the pyramid decomposition about the mean
 * of the face centres (ca), after turning every S to point away from its owner; own_ptr/own:
 * the faces each cell owns, nei_ptr/nei: the interior faces whose neighbour it is, each list in
 * increasing face index. counts[2]: faces turned, cells of non-positive volume.
 *
 * b2s_fv_faces_d: the interior-face quantities (if_idx: the interior faces in increasing index,
 * P/N their cells) d, w, alpha, wl = 1/|d|^2, T = S - alpha d, dPf, dNf, dxm, and the
 * boundary-face quantities (bf_idx, Pb) db, alpha_b, wlb, |Sb|, unit normal, tangential part of
 * db and wall distance |db.Sb|/|Sb|; *cos_min the smallest cosine between S and d.
 *
 * b2s_ls_matrices_d: the least-squares matrices G (the cell's interior faces as owner, as
 * neighbour and its boundary faces, summed family by family) and their inverses (LU with
 * partial pivoting); flag[c] = 1 where G is singular (|det| <= 1e-300) or the inverse not
 * finite: the caller substitutes the pseudo-inverse there, as the reference does. */
B2S_API int b2s_face_geometry_d(int32_t dim, int32_t nf, const double* nodes, const int32_t* face_ptr,
                                const int32_t* face_nodes, double* fc, double* S, int32_t* bad, b2s_stream_t s);
B2S_API int b2s_cell_geometry_d(int32_t dim, int32_t nc, int32_t nf, const int32_t* owner, const int32_t* neighbour,
                                const int32_t* own_ptr, const int32_t* own, const int32_t* nei_ptr, const int32_t* nei,
                                const double* fc, double* S, double* ca, double* vol, double* xc, int32_t* counts,
                                b2s_stream_t s);
B2S_API int b2s_fv_faces_d(int32_t dim, int32_t n_if, const int32_t* if_idx, const int32_t* P, const int32_t* N,
                           int32_t n_bf, const int32_t* bf_idx, const int32_t* Pb, const double* xc, const double* fc,
                           const double* S, double* d, double* w, double* alpha, double* wl, double* Tv, double* dPf,
                           double* dNf, double* dxm, double* db, double* alpha_b, double* wlb, double* Sb_mag,
                           double* nb, double* db_t, double* yb, double* cos_min, b2s_stream_t s);
/* Host counterpart of the two geometry calls above (the same per-face and per-cell code in host
 * loops; every pointer a HOST pointer): fc, S [nf][dim], xc [nc][dim], vol [nc]; repair != 0
 * turns area vectors away from their owners; counts[3]: faces of a node count the dimension does
 * not allow (nothing else is computed then), faces turned, cells of non-positive volume. */
B2S_API int b2s_host_face_geometry(int32_t dim, int32_t nf, const double* nodes, const int32_t* face_ptr,
                                   const int32_t* face_nodes, double* fc, double* S);
B2S_API int b2s_host_geometry(int32_t dim, int32_t nc, int32_t nf, const double* nodes, const int32_t* face_ptr,
                              const int32_t* face_nodes, const int32_t* owner, const int32_t* neighbour,
                              int32_t repair, double* fc, double* S, double* xc, double* vol, int32_t* counts);
B2S_API int b2s_ls_matrices_d(int32_t dim, int32_t nc, const int32_t* pi_ptr, const int32_t* pi,
                              const int32_t* ni_ptr, const int32_t* ni, const int32_t* pb_ptr, const int32_t* pb,
                              const double* d, const double* wl, const double* db, const double* wlb, double* G,
                              double* Ginv, int32_t* flag, b2s_stream_t s);

/* out[c][f] = w[f] phi[c][P] + (1 - w[f]) phi[c][N] for k components.
 * Replaces ft_face_interp (flowtrace/native/fvm_kernels.h:34-36). */
B2S_API int b2s_face_interp_d(const b2s_mesh* m, int k, const double* phi, double* out, b2s_stream_t s);

/* Least-squares cell gradients of nfield fields at once: phi [nfield][nc], phib [nfield][nb],
 * grad [nfield][dim][nc]. Replaces ft_ls_gradient (fvm_kernels.h:38-44). */
B2S_API int b2s_ls_gradient_d(const b2s_mesh* m, int nfield, const double* phi, const double* phib, double* grad,
                      b2s_stream_t s);

/* Green-Gauss gradient with the skewness correction from grad (NULL: none); out [dim][nc].
 * Replaces ft_gg_gradient (fvm_kernels.h:46-53). */
B2S_API int b2s_gg_gradient_d(const b2s_mesh* m, const double* phi, const double* phib, const double* grad, double* out,
                      b2s_stream_t s);

/* CSR values of a cell-cell operator from its diagonal and face coefficients (faces sharing a
 * cell pair are summed). Replaces ft_assemble (fvm_kernels.h:55-58). */
B2S_API int b2s_assemble_d(const b2s_mesh* m, const double* diag, const double* aPN, const double* aNP, double* val,
                   b2s_stream_t s);

/* y[c][i] = sum_j A[i,j] x[c][j] for k right-hand sides. Replaces ft_csr_spmm (fvm_kernels.h:30-32). */
B2S_API int b2s_spmv_d(int32_t n, int k, const int32_t* rowptr, const int32_t* col, const double* val, const double* x,
               double* y, b2s_stream_t s);

/* Outcome of a Krylov solve, per system, written to device memory. */
typedef struct b2s_solve_info {
  int32_t iterations;
  int32_t converged;
  double residual; /* final relative residual; NaN after a breakdown with a non-finite residual */
} b2s_solve_info;

/* Jacobi-preconditioned BiCGSTAB on nrhs (1..3) independent systems that share one matrix:
 * b, x, inv_diag are [nrhs][n] ([n] for inv_diag); x holds x0 on entry. Same algorithm and
 * stopping rules as flowtrace/linalg/krylov.py:68-121 with relative_to_initial, per system.
 * Replaces ft_bicgstab_jacobi (fvm_kernels.h:60-66); info is [nrhs] device structs. */
B2S_API int64_t b2s_bicgstab_workspace_bytes(int32_t n, int nrhs);
B2S_API int b2s_bicgstab_jacobi_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col, const double* val,
                          const double* b, const double* inv_diag, double* x, double tol, int maxiter,
                          int relative_to_initial, void* work, int64_t work_bytes, b2s_solve_info* info,
                          b2s_stream_t s);

/* The same Jacobi-BiCGSTAB for callers that cannot allocate device memory (a host code that
 * reaches the solver only through this C ABI and owns no CUDA allocator, or one whose device
 * memory is fully handed out before the solve): no work argument; the work space is a static
 * device array inside the library, sized for n * nrhs <= B2S_NOALLOC_MAX_UNKNOWNS (larger
 * problems return B2S_ERR_TOO_LARGE): 11,704,832 bytes, held by every GPU that loads the
 * library until exit. The first call in each CUDA context of a device looks the array's device
 * address up in that context (make it before any stream capture); calls that overlap on the
 * GPU share the array and race. No counterpart in the reference, whose ft_bicgstab_jacobi
 * always takes its work array from the caller. */
#define B2S_NOALLOC_MAX_UNKNOWNS 131072
B2S_API int b2s_bicgstab_jacobi_noalloc_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col,
                                          const double* val, const double* b, const double* inv_diag, double* x,
                                          double tol, int maxiter, int relative_to_initial, b2s_solve_info* info,
                                          b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* Fused stages of one SIMPLEC outer iteration (flowtrace/unstructured/simple.py:500-703).    */

typedef struct b2s_flow_params {
  double rho, mu, relax_u, relax_p;
  double body[3];          /* uniform body force per unit volume */
  int32_t simplec;         /* 1: SIMPLEC d-coefficients, 0: SIMPLE */
  int32_t second_order;    /* bounded second-order deferred correction in momentum */
  int32_t singular_p;      /* no pressure boundary: the pressure is fixed by its mean */
  int32_t pad;
  /* Batches (optional, NULL: the scalars above): per-cell under-relaxation and SIMPLEC flag, so
   * that each case of a batch keeps its own (its stability guard lowers them per case). */
  const double* relax_u_cell;
  const double* relax_p_cell;
  const int32_t* simplec_cell;
} b2s_flow_params;

/* Boundary values of p and U (simple.py:305-325) with lagged gradients: Up is [1+dim][nc]
 * (p, then the velocity components), gUp [1+dim][dim][nc] or NULL, gpf [dim][nc] (the
 * pressure gradient used by the reconstruction) or NULL; out [1+dim][nb]. */
B2S_API int b2s_flow_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const double* Up, const double* gUp, const double* gpf,
                     double* bUp, b2s_stream_t s);

/* Momentum system (simple.py:526-590): coefficients, right-hand sides, CSR values of the
 * under-relaxed matrix, Jacobi inverse, SIMPLEC d = V/(a_P/alpha_u - sum a_nb), the Fluent-
 * scaled residual partial sums, and b_r = b + (1-alpha_u)/alpha_u a_P u.
 *   in:  Up [1+dim][nc], gUp [1+dim][dim][nc], gp [dim][nc] (pressure force gradient),
 *        bUp [1+dim][nb], F [nf], Fb [nb], porosity [nc] or NULL (Brinkman alpha, adds
 *        alpha V to a_P), msrc [dim][nc] or NULL (momentum source already times V)
 *   out: val [nnz] (relaxed), diag [nc] (unrelaxed a_P), inv [nc], dP [nc], b [dim][nc],
 *        br [dim][nc], part [nblk][2*dim] block partials of sum|b - A u| and sum|a_P u|;
 *        *nblk receives the number of blocks used (at most b2s_part_blocks(nc)). */
B2S_API int b2s_part_blocks(int32_t n);
B2S_API int b2s_momentum_assemble_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Up,
                            const double* gUp, const double* gp, const double* bUp, const double* F,
                            const double* Fb, const double* porosity, const double* msrc, double* val,
                            double* diag, double* inv, double* dP, double* b, double* br, double* part,
                            b2s_stream_t s);

/* b2s_momentum_assemble_d with a viscosity per face and an extra per-cell source, as the
 * turbulence model supplies them (simple.py:545-548): mu_f [nf] (mu + mu_t), mu_b [nb] (walls:
 * the wall-function viscosity), tsrc [dim][nc] (the transpose stress, a cell total added after
 * msrc). prm->mu is not used. */
B2S_API int b2s_momentum_assemble_turb_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                         const double* Up, const double* gUp, const double* gp, const double* bUp,
                                         const double* F, const double* Fb, const double* porosity,
                                         const double* msrc, const double* mu_f, const double* mu_b,
                                         const double* tsrc, double* val, double* diag, double* inv, double* dP,
                                         double* b, double* br, double* part, b2s_stream_t s);

/* Rhie-Chow predictor fluxes and the pressure-correction system (simple.py:583-623):
 *   in:  Ustar [dim][nc], p [nc], gp [dim][nc], dP [nc]
 *   out: Fst [nf], cf [nf], Fbst [nb], cb [nb], val [nnz] (A_p), rhs [nc] (= -m*),
 *        part [nblk] block partials of sum|m*|. */
B2S_API int b2s_pressure_assemble_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Ustar,
                            const double* p, const double* gp, const double* dP, double* Fst, double* cf,
                            double* Fbst, double* cb, double* val, double* rhs, double* part, b2s_stream_t s);

/* Corrections (simple.py:638-646): F = F* + c_f (p'_P - p'_N), Fb = Fb* + c_b p'_P,
 * p_new = p + relax_p p', U_new = U* - d grad_LS(p'). Up_new is [1+dim][nc] (p, U).
 * part [nblk][3]: sum p_new, sum|F| (owned faces), sum|Fb|. The mean of p_new is removed by
 * b2s_remove_mean_d when the pressure is singular. */
B2S_API int b2s_correct_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Fst,
                  const double* cf, const double* Fbst, const double* cb, const double* pp, const double* p,
                  const double* Ustar, const double* dP, double* F, double* Fb, double* Up_new, double* part,
                  b2s_stream_t s);

/* x -= (sum of nblk partials at part[q], stride nq) / n. */
B2S_API int b2s_remove_mean_d(int32_t n, double* x, const double* part, int nblk, int nq, int q, b2s_stream_t s);

/* Sums column q of nblk x nq block partials into out[j] for the (q, j) pairs listed. */
B2S_API int b2s_sum_partials_d(const double* part, int nblk, int nq, int npairs, const int32_t* q_of, double* out,
                       b2s_stream_t s);

/* Energy (simple.py:778-813): boundary temperatures, gradient, assembly and the scaled
 * residual; T_b uses the lagged gradient gT (NULL on the first iteration).
 *   out: Tb [nb] */
B2S_API int b2s_energy_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const double* T, const double* gT, const double* Fb,
                       double* Tb, b2s_stream_t s);
/*   in:  T [nc], gT [dim][nc], Tb [nb], F, Fb, esrc [nc] or NULL (already times V/cp)
 *   out: val [nnz] (relaxed by relax_T), diag, inv, b, br [nc], part [nblk][2] */
B2S_API int b2s_energy_assemble_d(const b2s_mesh* m, const b2s_bc* bc, double gamma, double cp, double relax_T,
                          int second_order, const double* T, const double* gT, const double* Tb, const double* F,
                          const double* Fb, const double* esrc, double* val, double* diag, double* inv, double* b,
                          double* br, double* part, b2s_stream_t s);

/* b2s_energy_assemble_d with the diffusivity per face: gamma_f [nf], gamma_b [nb] (k/cp + mu_t/Pr_t,
 * walls k/cp; flowtrace/unstructured/turbulence.py:245-249). */
B2S_API int b2s_energy_assemble_turb_d(const b2s_mesh* m, const b2s_bc* bc, const double* gamma_f,
                                       const double* gamma_b, double cp, double relax_T, int second_order,
                                       const double* T, const double* gT, const double* Tb, const double* F,
                                       const double* Fb, const double* esrc, double* val, double* diag, double* inv,
                                       double* b, double* br, double* part, b2s_stream_t s);

/* Row residuals and scales of a system (flowtrace/unstructured/diagnostics.py:146-151):
 * r = b - A x, s = |b| + |A| |x|; with dval, row i's diagonal entry (slot_diag[i]) is dval[i]. */
B2S_API int b2s_row_residuals_d(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                                const int32_t* slot_diag, const double* dval, const double* b, const double* x,
                                double* r, double* s_out, b2s_stream_t s);
/* Cell mass imbalance (net outflow) and throughflow sum |F| of face fluxes (diagnostics.py:253-257). */
B2S_API int b2s_flux_balance_d(const b2s_mesh* m, const double* F, const double* Fb, double* mass, double* through,
                               b2s_stream_t s);
/* Properties of a cell-cell matrix on the mesh's CSR pattern that decide whether CG applies
 * (replaces the host check of flowtrace/unstructured/diagnostics.py:384-412):
 * out[0] = max |a_ij|, out[1] = max over faces |a_PN - a_NP| (the largest entry of |A - A^T|),
 * out[2] = the largest off-diagonal entry, out[3] = min over rows (a_ii - sum_j!=i |a_ij|) /
 * max(|a_ii|, 1e-300), out[4] = min a_ii. NaN entries make the affected outputs NaN. work holds
 * b2s_matrix_properties_workspace_bytes() bytes; out is device memory (5 doubles). */
B2S_API int64_t b2s_matrix_properties_workspace_bytes(void);
B2S_API int b2s_matrix_properties_d(const b2s_mesh* m, const double* val, double* work, int64_t work_bytes,
                                    double* out, b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* Smoothed-aggregation AMG (flowtrace/linalg/amg.py:80-146) with aggregates and sparsity
 * patterns fixed at set-up; every numeric quantity is rebuilt on the device. */

#define B2S_AMG_MAX_LEVELS 20

typedef struct b2s_amg_level {
  int32_t n, nnz;              /* rows and entries of A */
  int32_t nc;                  /* rows of the next level */
  int32_t p_nnz, w_nnz;
  const int32_t* rowptr;       /* A (level 0: the pressure-correction matrix) */
  const int32_t* col;
  double* val;                 /* level 0: the caller's matrix values; coarser: rebuilt */
  const int32_t* diag_slot;    /* [n] */
  double* dinv;                /* [n] */
  const int32_t* agg;          /* [n] aggregate of each row */
  const double* tval;          /* [nc] 1/sqrt(aggregate size) */
  const double* x0;            /* [n] start vector of the spectral-radius power iteration */
  const int32_t* p_rowptr;     /* P = (I - 4/(3 rho) D^-1 A) T, [n x nc], sorted columns */
  const int32_t* p_col;
  double* p_val;
  const int32_t* r_rowptr;     /* R = P^T, [nc x n] */
  const int32_t* r_col;
  const int32_t* r_from_p;     /* R entry -> P entry */
  double* r_val;
  const int32_t* w_rowptr;     /* W = A P, [n x nc], sorted columns */
  const int32_t* w_col;
  double* w_val;
  double* rho;                 /* [1] spectral radius estimate (device); batches: [ngroups] */
  const uint8_t* strong;       /* [nnz] strength of each entry at set-up (1: strong), or NULL */
  const int32_t* group_ptr;    /* batches: [ngroups+1] rows of each case on this level, or NULL */
  /* Optional term lists of the fixed-pattern products (NULL: the row-owned kernels locate each
   * term's slot by binary search). The terms of slot s are t in
   * [x_tptr[s], x_tptr[s+1]), listed in the order the row-owned kernels add them, so both give
   * the same values bit for bit:
   *   P slot s (row i):  sum_t (dinv_i a[p_tj[t]]) tval[col]       (A entries of row i)
   *   W slot s:          sum_t a[w_tj[t]] p[w_te[t]]               (A entry, P entry)
   *   A_c slot s:        sum_t r[c_te[t]] w[c_ts[t]]               (R entry, W entry) */
  const int32_t* p_tptr;       /* [p_nnz+1] */
  const int32_t* p_tj;         /* [nnz] */
  const int32_t* w_tptr;       /* [w_nnz+1] */
  const int32_t* w_tj;
  const int32_t* w_te;
  const int32_t* c_tptr;       /* [c_nnz+1], or NULL (the warp-per-row Galerkin kernel) */
  const int32_t* c_te;
  const int32_t* c_ts;
  int32_t c_nnz;               /* entries of the next level's matrix */
  int32_t pad_;
} b2s_amg_level;

typedef struct b2s_amg {
  int32_t nlevels;             /* levels with smoothing; the coarse level follows */
  int32_t coarse_n;
  int32_t singular;            /* shift the coarse matrix by 1e-10 mean|diag| */
  int32_t sweeps;              /* Jacobi sweeps before and after the coarse correction */
  double omega;                /* Jacobi damping */
  const int32_t* coarse_rowptr;/* coarse CSR (values are level nlevels-1's Galerkin product) */
  const int32_t* coarse_col;
  double* coarse_val;
  double* coarse_inv;          /* [coarse_n][coarse_n]; batches: one dense block per case */
  /* Batches of independent cases (ngroups > 0): every level is block diagonal with the rows of a
   * case contiguous (levels[l].group_ptr), the coarse inverse is stored per case (block g of
   * size n_g = coarse_group_ptr[g+1]-coarse_group_ptr[g] at coarse_inv + coarse_inv_off[g]) and
   * the singular shift applies per case (group_singular[g]). */
  int32_t ngroups;
  int32_t pad_;
  const int32_t* coarse_group_ptr;
  const int64_t* coarse_inv_off;
  const int32_t* group_singular;
  b2s_amg_level levels[B2S_AMG_MAX_LEVELS];
} b2s_amg;

/* Rebuild every numeric quantity of the hierarchy from level 0's matrix values. */
B2S_API int64_t b2s_amg_workspace_bytes(const b2s_amg* h);
B2S_API int b2s_amg_rebuild_d(const b2s_amg* h, void* work, int64_t work_bytes, b2s_stream_t s);

/* Preconditioned CG with one V-cycle per iteration (flowtrace/linalg/krylov.py:25-65 with
 * M = SmoothedAggregationAMG) on the operator A = (rowptr, col, val) of n rows; the hierarchy
 * keeps the matrices of its last rebuild, as the reference's preconditioner object does between
 * rebuilds. project != 0 removes the mean from the residual and the preconditioned residual
 * (singular pure-Neumann systems). x starts at zero. */
B2S_API int64_t b2s_pcg_workspace_bytes(const b2s_amg* h);
/* Launch shape of the AMG-PCG and V-cycle kernels (b2s_pcg_amg_d, b2s_pcg_amg_mixed_d,
 * b2s_amg_vcycle_d), for all later launches: cooperative launches made of thread-block clusters
 * of cluster_blocks blocks (2, 4, 8 or 16; 0: no clusters, the default), and the size below
 * which a level of the V-cycle runs on a subset of the grid instead of all of it: levels (and the
 * coarse solve) of at most sub_entries matrix entries run on the first cluster with cluster
 * barriers, or without clusters on block 0 with block barriers (defaults 32768 and 4096). Results
 * agree up to round-off (how many lanes share a row depends on the phase's thread count).
 * Returns B2S_OK or B2S_ERR_ARG. No counterpart in the reference (launch parameters of this
 * implementation). */
B2S_API int b2s_pcg_set_launch(int cluster_blocks, int sub_entries);
B2S_API int b2s_pcg_amg_d(const b2s_amg* h, int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                          const double* b, double* x, double tol, int maxiter, int project, void* work,
                          int64_t work_bytes, b2s_solve_info* info, b2s_stream_t s);

/* Number of matrix entries, over all levels with smoothing, whose strength of connection
 * |a_ij| >= theta sqrt(|a_ii a_jj|) differs from the set-up's (the levels' strong flags); the
 * reference re-aggregates at every rebuild, so a non-zero count means its aggregates changed.
 * *count (device int) is overwritten. */
B2S_API int b2s_amg_strength_changes_d(const b2s_amg* h, double theta, int32_t* count, b2s_stream_t s);
/* The same count per level: counts[l] (device ints, [nlevels]) for level l. */
B2S_API int b2s_amg_level_strength_changes_d(const b2s_amg* h, double theta, int32_t* counts, b2s_stream_t s);

/* Apply one V-cycle: x = M b (for tests of the preconditioner). */
B2S_API int b2s_amg_vcycle_d(const b2s_amg* h, const double* b, double* x, void* work, int64_t work_bytes, b2s_stream_t s);

/* Host set-up helper: the greedy three-pass aggregation of flowtrace/linalg/amg.py:25-57 on a
 * strength graph given as HOST CSR arrays; agg[n] (host) receives each node's aggregate and
 * the return value is the number of aggregates (-1 on invalid arguments). */
B2S_API int64_t b2s_host_aggregate(int64_t n, const int64_t* indptr, const int64_t* indices, int64_t* agg);

/* Device set-up of the hierarchy, level by level (replaces the host set-up of
 * flowtrace/linalg/amg.py:88-117 when the hierarchy is re-aggregated on the device).
 *
 * b2s_amg_strength_d: strong[e] = 1 where |a_e| >= theta sqrt(|a_ii a_jj|), col[e] != i
 * (amg.py:60-66), for every stored entry of the CSR matrix (rowptr, col, val) of n rows.
 *
 * b2s_csr_transpose_slots_d: for a structurally symmetric pattern, tslot[e] = the slot of the
 * transposed entry (col[e], row of e); sorted != 0 when every row's columns ascend (binary
 * search), else rows are scanned. *missing (device int) counts entries without a transpose
 * (their tslot is e itself).
 *
 * b2s_amg_aggregate_d: the greedy three-pass aggregation of amg.py:25-57 on the strength graph
 * S(i) = {col[e] : e in row i, strong[e]}, visiting nodes in the order prio (a permutation of
 * 0..n-1; rank_node its inverse), exactly the reference's result when prio is the reference's
 * numbering and each row's strong columns are that numbering's columns. agg[n] receives the
 * aggregates (numbered as the reference numbers them), counts[n] the size of each aggregate
 * (entries >= the number of aggregates are 0), info[4] (device ints): [0] the number of
 * aggregates, [1] an error code (0; 1: a poll limit of the pass-1 kernel ran out; 2: an
 * inconsistent pass-2 chain; 3: the conflict lists exceed the work space), [2] the aggregates of
 * pass 1, [3] the nodes of pass 3. The work space holds the nodes' conflict lists: at most
 * capacity = nnz + sum over rows of (row length)^2 entries always suffices
 * (b2s_amg_aggregate_workspace_bytes(n, capacity)). The pass-1 kernel is a cooperative launch
 * whose threads wait on each other's decisions with bounded polls.
 *
 * b2s_amg_level_rebuild_d: the numeric rebuild of one (single-case) level from its matrix
 * values (D^-1, rho, P, R, W) writing the next level's values cval on the pattern (crow, ccol);
 * b2s_amg_coarse_inverse_d: the coarse inverse of a complete hierarchy (its workspace is
 * b2s_amg_workspace_bytes). b2s_amg_rebuild_d is these applied to every level in turn. */
B2S_API int b2s_amg_strength_d(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                               const int32_t* diag_slot, double theta, uint8_t* strong, b2s_stream_t s);
B2S_API int b2s_csr_transpose_slots_d(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t sorted,
                                      int32_t* tslot, int32_t* missing, b2s_stream_t s);
B2S_API int64_t b2s_amg_aggregate_workspace_bytes(int32_t n, int64_t capacity);
B2S_API int b2s_amg_aggregate_d(int32_t n, const int32_t* rowptr, const int32_t* col, const uint8_t* strong,
                                const int32_t* tslot, const int32_t* prio, const int32_t* rank_node, int32_t* agg,
                                int32_t* counts, int32_t* info, void* work, int64_t work_bytes, b2s_stream_t s);
B2S_API int64_t b2s_amg_level_workspace_bytes(const b2s_amg_level* L);
B2S_API int b2s_amg_level_rebuild_d(const b2s_amg_level* L, const int32_t* crow, const int32_t* ccol, double* cval,
                                    void* work, int64_t work_bytes, b2s_stream_t s);
B2S_API int b2s_amg_coarse_inverse_d(const b2s_amg* h, void* work, int64_t work_bytes, b2s_stream_t s);

/* The patterns of P = A T and W = A P of one level, with the term lists of the row-owned rebuild
 * (b2s_amg_level): rp/cl the level's CSR in stored order, agg its aggregates, ncols their number
 * (one warp per row, with a counter per column in shared memory, when ncols is at most
 * b2s_amg_pattern_warp_cols - 2048 by default; else one thread per row).
 * Two passes each: pass 0 writes per-row counts (pcnt; wcnt = W entries, tcnt = W terms), which
 * the caller scans (b2s_scan_counts_d) into p_ptr (w_ptr, t_ptr) and allocates from; pass 1
 * fills p_idx, p_tptr, p_tj (w_idx, w_tptr, w_tj, w_te), never past p_cap/nnz (w_cap/t_cap).
 * *overflow (device int, not cleared): 1 where a row has more than 64 distinct P columns or 128
 * distinct W columns (one thread per row), 2 where the offsets disagree with the counts; the
 * caller then builds the level another way. */
B2S_API int b2s_amg_p_pattern_d(int32_t n, int32_t ncols, const int32_t* rp, const int32_t* cl, const int32_t* agg,
                                int32_t pass, int32_t* pcnt, const int32_t* p_ptr, int64_t p_cap, int32_t* p_idx,
                                int32_t* p_tptr, int32_t* p_tj, int64_t nnz, int32_t* overflow, b2s_stream_t s);
B2S_API int b2s_amg_w_pattern_d(int32_t n, int32_t ncols, const int32_t* rp, const int32_t* cl, const int32_t* p_ptr,
                                const int32_t* p_idx, int32_t pass, int32_t* wcnt, int32_t* tcnt, const int32_t* w_ptr,
                                const int32_t* t_ptr, int64_t w_cap, int64_t t_cap, int32_t* w_idx, int32_t* w_tptr,
                                int32_t* w_tj, int32_t* w_te, int32_t* overflow, b2s_stream_t s);
/* R = P^T (the transposes of amg.py:102,115): r_rowptr [na + 1], r_col [p_nnz] (fine rows,
 * ascending in each row) and r_from_p [p_nnz] (the P entry of each R entry), from P's pattern
 * (each row's columns ascending), with no host synchronisation; work space from
 * b2s_amg_r_workspace_bytes(na). *overflow: 1 where an R row has more than 256 entries. */
B2S_API int64_t b2s_amg_r_workspace_bytes(int32_t na);
B2S_API int b2s_amg_r_pattern_d(int32_t n, int32_t na, const int32_t* p_ptr, const int32_t* p_idx, int64_t p_nnz,
                                int32_t* r_rowptr, int32_t* r_col, int32_t* r_from_p, void* work, int64_t work_bytes,
                                int32_t* overflow, b2s_stream_t s);
/* The pattern of A_c = R W (the Galerkin product P^T A P, amg.py:102) with its term lists (one
 * warp per coarse row as for P and W, else one thread), in the two passes of the P and W builders: pass 0 writes ccnt (A_c
 * entries) and tcnt (terms) per row; pass 1 fills c_idx, c_diag [na] (the slot of each row's
 * diagonal), c_tptr [c_nnz + 1], c_te (R entries) and c_ts (W entries). *overflow: 1 where a row
 * has more than 128 distinct columns (one thread per row), 2 where the offsets disagree with the
 * counts. */
B2S_API int b2s_amg_c_pattern_d(int32_t na, const int32_t* r_rowptr, const int32_t* r_col, const int32_t* w_ptr,
                                const int32_t* w_idx, int32_t pass, int32_t* ccnt, int32_t* tcnt, const int32_t* c_ptr,
                                const int32_t* t_ptr, int64_t c_cap, int64_t t_cap, int32_t* c_idx, int32_t* c_diag,
                                int32_t* c_tptr, int32_t* c_te, int32_t* c_ts, int32_t* overflow, b2s_stream_t s);
/* The largest column count (aggregates) whose P, W and A_c builders run one warp per row:
 * default and maximum 2048, 0 for one thread per row always; ncols < 0 only queries. Returns the
 * previous value. Process-wide and not synchronised: set it before the builders run. */
B2S_API int b2s_amg_pattern_warp_cols(int32_t ncols);
/* Exclusive scan of n int32 counts into out[0..n], out[n] the total. */
B2S_API int64_t b2s_scan_workspace_bytes(int32_t n);
B2S_API int b2s_scan_counts_d(int32_t n, const int32_t* counts, int32_t* out, void* work, int64_t work_bytes,
                              b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* Mixed precision. No counterpart in the reference (its path is FP64 throughout): the linear    */
/* systems are stored and solved in float, while the nonlinear residuals, the continuity and     */
/* norm reductions, the iterative refinement of the pressure-correction solve and the AMG        */
/* coarsest-level solve stay double. Every linear system is solved in correction form           */
/* A_r dphi = b - A phi from dphi = 0, so a converged iteration is the double one's fixed point. */

/* Momentum assembly of b2s_momentum_assemble_d with the relaxed matrix values and the Jacobi
 * inverse written in float, and, instead of b / b_r, the double residual r = b - A U of the
 * unrelaxed system ([dim][nc], stored in float). part receives the same scaled-residual sums. */
B2S_API int b2s_momentum_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                          const double* Up, const double* gUp, const double* gp, const double* bUp,
                                          const double* F, const double* Fb, const double* porosity,
                                          const double* msrc, float* val, float* inv, double* dP, float* r,
                                          double* part, b2s_stream_t s);

/* Pressure-correction assembly of b2s_pressure_assemble_d with the matrix values in float. */
B2S_API int b2s_pressure_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                          const double* Ustar, const double* p, const double* gp, const double* dP,
                                          double* Fst, double* cf, double* Fbst, double* cb, float* val, double* rhs,
                                          double* part, b2s_stream_t s);

/* b2s_momentum_assemble_mixed_d with the turbulence model's face viscosities and transpose-stress
 * source (as b2s_momentum_assemble_turb_d). */
B2S_API int b2s_momentum_assemble_mixed_turb_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                               const double* Up, const double* gUp, const double* gp,
                                               const double* bUp, const double* F, const double* Fb,
                                               const double* porosity, const double* msrc, const double* mu_f,
                                               const double* mu_b, const double* tsrc, float* val, float* inv,
                                               double* dP, float* r, double* part, b2s_stream_t s);

/* Energy assembly of b2s_energy_assemble_d in the form of b2s_momentum_assemble_mixed_d. */
B2S_API int b2s_energy_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, double gamma, double cp,
                                        double relax_T, int second_order, const double* T, const double* gT,
                                        const double* Tb, const double* F, const double* Fb, const double* esrc,
                                        float* val, float* inv, float* r, double* part, b2s_stream_t s);

/* b2s_energy_assemble_mixed_d with the diffusivity per face (as b2s_energy_assemble_turb_d). */
B2S_API int b2s_energy_assemble_mixed_turb_d(const b2s_mesh* m, const b2s_bc* bc, const double* gamma_f,
                                             const double* gamma_b, double cp, double relax_T, int second_order,
                                             const double* T, const double* gT, const double* Tb, const double* F,
                                             const double* Fb, const double* esrc, float* val, float* inv, float* r,
                                             double* part, b2s_stream_t s);

/* Jacobi-BiCGSTAB of b2s_bicgstab_jacobi_d with float matrix values and vectors (reductions in
 * double). zero_x0 starts from x = 0 without reading x; out64/base64 (both or neither, [nrhs][n])
 * receive out64 = base64 + x in double at the end. */
B2S_API int64_t b2s_bicgstab_f32_workspace_bytes(int32_t n, int nrhs);
B2S_API int b2s_bicgstab_jacobi_f32_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col,
                                      const float* val, const float* b, const float* inv_diag, float* x, double tol,
                                      int maxiter, int relative_to_initial, int zero_x0, double* out64,
                                      const double* base64, void* work, int64_t work_bytes, b2s_solve_info* info,
                                      b2s_stream_t s);

/* Float copies of the hierarchy's per-level values (the V-cycle of the mixed solve reads these;
 * the coarse inverse stays double). Arrays are caller-allocated with the level sizes. */
typedef struct b2s_amg_f32 {
  float* val[B2S_AMG_MAX_LEVELS];
  float* dinv[B2S_AMG_MAX_LEVELS];
  float* p_val[B2S_AMG_MAX_LEVELS];
  float* r_val[B2S_AMG_MAX_LEVELS];
} b2s_amg_f32;
B2S_API int b2s_amg_to_f32_d(const b2s_amg* h, const b2s_amg_f32* h32, b2s_stream_t s);

/* Pressure-correction solve with iterative refinement: passes of the AMG-PCG in float (tolerance
 * tol / current relative residual, floored at min_inner_tol), each followed by x += correction
 * and the true residual r = b - A x in double, A applied from the double face coefficients
 * (A x)_c = sum_f cf_f (x_c - x_nb) + sum_b cb_b x_c of the mesh m. Stops when |r| / |b| < tol
 * (r projected when project != 0), after maxpass passes or maxiter float iterations in total.
 * (rowptr, col, val) is the float operator of the inner solve; x ([n], double) is overwritten.
 * info->iterations counts the float iterations, info->residual is the double one. */
B2S_API int64_t b2s_pcg_mixed_workspace_bytes(const b2s_amg* h);
B2S_API int b2s_pcg_amg_mixed_d(const b2s_amg* h, const b2s_amg_f32* h32, const b2s_mesh* m, const double* cf,
                                const double* cb, int32_t n, const int32_t* rowptr, const int32_t* col,
                                const float* val, const double* b, double* x, double tol, int maxiter, int project,
                                int maxpass, double min_inner_tol, void* work, int64_t work_bytes,
                                b2s_solve_info* info, b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* Batches of independent cases. No counterpart in the reference, which runs the cases of a     */
/* sweep one after another (flowtrace/runtime/batch.py:142-222): here they share one device      */
/* mesh, the disjoint union of their meshes with each case's cells contiguous, every stage runs */
/* once for all of them, and each Krylov solve keeps per-case scalars and stopping tests.        */

/* Partial-sum blocks of the stages of a mesh: its tile count when tiled, else b2s_part_blocks. */
B2S_API int b2s_mesh_part_blocks(const b2s_mesh* m);

/* out[g][q] = sum of part[q][t] over the tiles t = group_tiles[g] .. group_tiles[g+1]-1. */
B2S_API int b2s_group_sums_d(const double* part, int nblk, int nq, int ngroups, const int32_t* group_tiles,
                             double* out, b2s_stream_t s);

/* x -= the mean of x over every case g with singular[g] != 0, the sums taken from part[q][tiles
 * of the case] (as written by b2s_correct_d on the tiled mesh m); group_cells [ngroups+1]. */
B2S_API int b2s_remove_group_means_d(const b2s_mesh* m, double* x, const double* part, int nblk, int q,
                                     const int32_t* group_tiles, const int32_t* tile_group,
                                     const int32_t* group_cells, const int32_t* singular, b2s_stream_t s);

/* Jacobi-BiCGSTAB in float of every case's rows (group_ptr [ngroups+1]) as separate systems,
 * with the semantics of b2s_bicgstab_jacobi_f32_d per case; order [ngroups] is the processing
 * order (largest first); info is [ngroups][nrhs]. */
/* Shape of the team that solves one case of a batch: the blocks of one thread-block cluster.
 * NULL selects the default (4 blocks of 1024 threads, rows averaging 24 or more entries walked one
 * warp per row); the batch solver's autotuner times candidate shapes on the batch itself. */
typedef struct b2s_team_config {
  int32_t cluster_blocks;  /* blocks per team (1 .. 8) */
  int32_t block_threads;   /* threads per block: a multiple of 32, 64 .. 1024 */
  int32_t wide_row;        /* rows averaging at least this many entries go one warp per row (0: never) */
  int32_t pad_;
} b2s_team_config;

B2S_API int64_t b2s_bicgstab_groups_workspace_bytes(int32_t n, int nrhs, int single);
B2S_API int b2s_bicgstab_groups_f32_d(int ngroups, const int32_t* group_ptr, const int32_t* order, int32_t n, int nrhs,
                                      const int32_t* rowptr, const int32_t* col, const float* val, const float* b,
                                      const float* inv_diag, float* x, double tol, int maxiter,
                                      int relative_to_initial, int zero_x0, double* out64, const double* base64,
                                      void* work, int64_t work_bytes, b2s_solve_info* info,
                                      const b2s_team_config* team, b2s_stream_t s);

/* The refined pressure-correction solve of b2s_pcg_amg_mixed_d per case, on a batch hierarchy
 * (h->ngroups > 0); project [ngroups] marks the singular cases, info is [ngroups]. */
B2S_API int64_t b2s_pcg_groups_workspace_bytes(const b2s_amg* h);
B2S_API int b2s_pcg_groups_mixed_d(const b2s_amg* h, const b2s_amg_f32* h32, const int32_t* order,
                                   const int32_t* project, const b2s_mesh* m, const double* cf, const double* cb,
                                   int32_t n, const int32_t* rowptr, const int32_t* col, const float* val,
                                   const double* b, double* x, double tol, int maxiter, int maxpass,
                                   double min_inner_tol, void* work, int64_t work_bytes, b2s_solve_info* info,
                                   const b2s_team_config* team, b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* Discrete adjoint. No counterpart in the reference (it has no derivatives).                   */

/* Vector-Jacobian product of the steady residual R(x; theta) of the outer iteration with
 * upwind convection on a mesh without non-orthogonal terms, the unknowns being
 * x = (U [dim][nc], p [nc], g [dim][nc] the Green-Gauss pressure gradient, F [nf], Fb [nb]) and
 * theta = (porosity [nc], the fixed boundary velocities bc->ub_fixed):
 *   R_m = b - A U, R_c = Cdiff F + Cb Fb, R_g = g - GG(p, p_b), R_F = F - RhieChow(U, p, g, dP),
 *   R_Fb = Fb - (inlet flux + Rhie-Chow pressure-face flux), dP = V / (a_P / relax_u - sum a_nb)
 *   (simplec != 0) or V / (a_P / relax_u).
 * Given lambda = (lm [dim][nc], lc [nc], lg [dim][nc], lF [nf], lFb [nb]) it writes
 * (dR/dx)^T lambda into (oU, op, og, oF, oFb) and, when the pointers are set, (dR/dporosity)^T
 * lambda into opor [nc] and (dR/dub)^T lambda into oub [dim][nb]. work holds 4 nc doubles. */
B2S_API int b2s_residual_vjp_d(const b2s_mesh* m, const b2s_bc* bc, double rho, double mu, double relax_u,
                               int simplec, const double* U, const double* p, const double* g, const double* F,
                               const double* Fb, const double* porosity, const double* lm, const double* lc,
                               const double* lg, const double* lF, const double* lFb, double* work, double* oU,
                               double* op, double* og, double* oF, double* oFb, double* opor, double* oub,
                               b2s_stream_t s);

/* ----------------------------------------------------------------------------------------- */
/* k-omega SST (Menter, Kuntz & Langtry 2003; flowtrace/unstructured/turbulence.py:116-438).
 * The model's state is k and omega ([2][nc]: k then omega) and mu_t [nc]; per outer iteration:
 *   before the momentum assembly   b2s_sst_momentum_terms_d
 *   after the energy equation      b2s_sst_bvals_d, b2s_ls_gradient_d (2 fields),
 *                                  b2s_sst_sources_d, then for q = 0 (k) and q = 1 (omega):
 *                                  b2s_sst_transport_assemble_d, b2s_sst_transport_finish_d and a
 *                                  Jacobi-BiCGSTAB solve (tol 1e-3, 60 iterations, from the old
 *                                  field), and b2s_sst_update_d. */
typedef struct b2s_sst {
  double rho, mu, nu;       /* density, molecular viscosity, mu / rho */
  double k_min, w_min;      /* floors of k and omega */
  double relax_k, relax_w;  /* under-relaxation of the two transport solves */
  double k_over_cp;         /* energy: conductivity / cp (unused without energy) */
  double eb;                /* exp(-kappa B) of Spalding's law (kappa 0.41, B 5.2) */
  double cmu25;             /* Cmu^0.25 (Cmu 0.09) */
  double g1, g2;            /* gamma_1,2 = beta_1,2 / beta* - sigma_w1,2 kappa^2 / sqrt(beta*) */
  int32_t second_order;     /* bounded second-order convection of k and omega (else upwind) */
  int32_t pad_;
  const double* y;          /* [nc] wall distance (wall cells: normal distance to their wall face) */
  const double* y_wall;     /* [nc] wall cells: smallest normal distance to one of their wall faces; +inf elsewhere */
  const double* yb;         /* [nb] |db . n|, owner centre to face, normal */
  const double* kb_in;      /* [nb] k where the face is fixed (inlets, inflow at openings) */
  const double* wb_in;      /* [nb] omega there */
} b2s_sst;

/* Blocks (= partial sums) of the two SST transport passes; equals b2s_mesh_part_blocks. */
B2S_API int b2s_sst_part_blocks(const b2s_mesh* m);

/* Face viscosities and source of the momentum equations and the turbulent heat diffusivity
 * (turbulence.py:235-261, 399-417) from U (Up = [p, U], [1+dim][nc]), its gradient
 * (gUp [1+dim][dim][nc]) and mu_t: mu_f [nf], mu_b [nb] (walls: mu Re_y / u+^2 from Spalding's
 * law), yplus [nb] (optional, 0 off walls), tsrc [dim][nc] = div(mu_t (grad U)^T), and, both or
 * neither, kT_f [nf] / kT_b [nb] = k/cp + mu_t/Pr_t (walls k/cp). */
B2S_API int b2s_sst_momentum_terms_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_sst* t, const double* Up,
                                     const double* gUp, const double* mut, double* mu_f, double* mu_b,
                                     double* yplus, double* tsrc, double* kT_f, double* kT_b, b2s_stream_t s);

/* Boundary values of k and omega (KWb [2][nb]) and the mask of fixed faces (fixed [nb], 0/1):
 * fixed at inlets and at open faces with inflow (Fb < 0), zero-gradient elsewhere. */
B2S_API int b2s_sst_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_sst* t, const double* KW,
                            const double* Fb, double* KWb, double* fixed, b2s_stream_t s);

/* Per cell, from grad U (gU [dim][dim][nc]), k/omega, their gradients (gKW [2][dim][nc]) and mu_t:
 * coef [8][nc] = (mu + sigma_k mu_t, mu + sigma_w mu_t, Sc_k, Sp_k, Sc_w, Sp_w, |S|, near-wall
 * omega of wall cells). */
B2S_API int b2s_sst_sources_d(const b2s_mesh* m, const b2s_sst* t, const double* gU, const double* KW,
                              const double* gKW, const double* mut, double* coef, b2s_stream_t s);

/* Transport system of field q (0 k, 1 omega): off-diagonals into val [nnz], the unrelaxed
 * diagonal (+ Sp V) into diag [nc], the right-hand side (+ Sc V) into b [nc], each block's
 * maximum diagonal into part_max [b2s_sst_part_blocks]. */
B2S_API int b2s_sst_transport_assemble_d(const b2s_mesh* m, const b2s_sst* t, int q, const double* KW,
                                         const double* KWb, const double* fixed, const double* gKW, const double* F,
                                         const double* Fb, const double* coef, double* val, double* diag, double* b,
                                         double* part_max, b2s_stream_t s);

/* Completes the system of b2s_sst_transport_assemble_d: for omega the wall cells are pinned to
 * coef[7] (diag and b += 1e10 max(diag) x (1, value)); the residual sums |b - A phi| and
 * |diag phi| over the cells above the floor and not pinned go to part_res (2 quantities x
 * blocks); val's diagonal, inv [nc] and br [nc] receive the relaxed system. */
B2S_API int b2s_sst_transport_finish_d(const b2s_mesh* m, const b2s_sst* t, int q, const double* KW,
                                       const double* coef, const double* part_max, double* val, double* diag,
                                       double* b, double* inv, double* br, double* part_res, b2s_stream_t s);

/* New state from the solves (KWn [2][nc]): k, omega floored into KW [2][nc], and
 * mu_t = rho a1 k / max(a1 omega, |S| F2) into mut [nc]. */
B2S_API int b2s_sst_update_d(const b2s_mesh* m, const b2s_sst* t, const double* KWn, const double* coef,
                             double* KW, double* mut, b2s_stream_t s);

#ifdef __cplusplus
}
#endif

#endif
