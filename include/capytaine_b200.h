/* capytaine_b200 — C ABI of the B200 (sm_100a) Delhommeau BEM hot path.
 *
 * Every entry point takes plain pointers and sizes.  Pointers named *_dev are
 * CUDA device pointers (any allocator: torch, cudaMalloc, cupy); pointers named
 * *_host are host pointers.  `stream` is a cudaStream_t passed as void* (NULL =
 * legacy default stream).  Work is enqueued on the stream; functions return
 * before it completes unless stated otherwise.  Every function returns a
 * status code (BEM_OK = 0); bem_last_error() gives a message for the calling
 * thread.
 *
 * Array conventions follow capytaine: points and vectors are (n, 3) row-major
 * float64; faces are (N, 4) int32, 0-based, triangles stored with their last
 * vertex repeated (capytaine meshes/meshes.py:454-469); influence matrices are
 * column-major (Fortran order) complex arrays, entry (I, J) at I + J*ld.
 */
#ifndef CAPYTAINE_B200_H
#define CAPYTAINE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define BEM_OK 0
#define BEM_ERR_INVALID_ARGUMENT 1
#define BEM_ERR_CUDA 2
#define BEM_ERR_NAN 3             /* NaN in an influence matrix (engines.py:400-405)   */
#define BEM_ERR_SINGULAR 4        /* zero pivot in the LU factorisation                */
#define BEM_ERR_NOT_CONVERGED 5   /* iterative refinement / GMRES did not converge    */
#define BEM_ERR_OUT_OF_MEMORY 6
#define BEM_ERR_UNSUPPORTED 7     /* option outside the implemented path               */
#define BEM_ERR_TIMEOUT 8         /* a bounded device-side wait gave up                */
#define BEM_PENDING 9             /* bem_request_poll: the request is still running    */

/* ---- enums (values of libDelhommeau constants.f90:40-52) ------------------ */
#define BEM_GRID_LEGACY 0
#define BEM_GRID_SCALED_NEMOH3 1
#define BEM_GF_HIGH_FREQ 0
#define BEM_GF_LOW_FREQ 1
#define BEM_GF_LOW_FREQ_WITH_RANKINE_PART 2

#define BEM_DTYPE_C128 0          /* complex128 outputs                               */
#define BEM_DTYPE_C64 1           /* complex64 outputs                                */

#define BEM_PREC_FP64 0           /* every term in float64                            */
#define BEM_PREC_MIXED 1          /* float32 wave term, float64 Rankine terms             */

/* Message describing the last error raised on the calling thread. */
const char* bem_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int bem_version(void);
/* Number of kernels this library has launched since it was loaded (all devices,
 * all threads): instrumentation for benchmarks. */
long long bem_launch_count(void);
/* Optional device timing per kernel class (no counterpart in the reference:
 * benchmark instrumentation).  While enabled, launches of the classes below
 * are bracketed by CUDA events recorded on their launch stream.  enable(0/1)
 * discards what was recorded; read() waits for the recorded events and returns
 * the summed duration and the number of bracketed launches of one class.
 * Classes: 0 assemble, 1 float64 DMMA GEMM, 2 tcgen05 TF32 update, 3 Gauss-
 * Jordan diagonal inverse, 4 mixed panel, 5 mixed block substitution, 6 float64
 * diagonal LU, 7 float64 panel, 8 float64 triangular solve, 9 tall GEMM. */
int bem_kernel_timer_enable(int on);
int bem_kernel_timer_read(int kernel_class, double* total_ms_host, long long* launches_host);
const char* bem_kernel_class_name(int kernel_class);

/* ---- tabulation of the Delhommeau integrals ------------------------------- */
/* Grid of the tabulation.  Replace delhommeau_integrals::default_r_spacing and
 * default_z_spacing (libs/libDelhommeau/src/Delhommeau_integrals.f90:208-270),
 * called from capytaine green_functions/delhommeau.py:253-258.  Host output. */
int bem_default_r_spacing(int nr, double rmax, int grid_shape, double* r_range_host);
int bem_default_z_spacing(int nz, double zmin, int grid_shape, double* z_range_host);

/* Five tabulated integrals on the (r, z) grid by Simpson integration over theta.
 * Replaces delhommeau_integrals::construct_tabulation
 * (Delhommeau_integrals.f90:43-153,190-204), called from delhommeau.py:259-261.
 * table_dev: float64, C-order (nr, nz, 5). */
int bem_construct_tabulation(const double* r_range_dev, int nr, const double* z_range_dev, int nz,
                             int nb_integration_points, double* table_dev, void* stream);

/* Reciprocals of the denominators of the 3-point Lagrange weights of a grid
 * (range, n values, host): out[3 c + i] = 1 / prod_{k != i} (u_i - u_k) for
 * the stencil u = range[c - 1 .. c + 1] centred on node c (1 <= c <= n - 2;
 * the other rows are zero).  Given to the assembly (bem_assembly_args
 * r_inv_den_dev / z_inv_den_dev), the interpolation of the tabulated integrals
 * (Delhommeau_integrals.f90:383-392) multiplies instead of dividing; the
 * weights change by an ulp at most.  No counterpart in the reference. */
int bem_tabulation_inverse_denominators(const double* range_host, int n, double* out_host);

/* ---- assembly of the influence matrices ----------------------------------- */
typedef struct {
  /* collocation side (mesh1 or a raw list of points) */
  int32_t n;                       /* number of collocation points (rows)                      */
  const double* points_dev;        /* (n, 3)                                                   */
  const double* dot_normals_dev;   /* (n, 3) if adjoint_double_layer else (nb_faces, 3)        */
  /* source side (mesh2) */
  int32_t nb_faces;                /* columns                                                  */
  int32_t nb_vertices;
  const double* vertices_dev;      /* (nb_vertices, 3)                                         */
  const int32_t* faces_dev;        /* (nb_faces, 4), 0-based                                   */
  const double* centers_dev;       /* (nb_faces, 3)                                            */
  const double* normals_dev;       /* (nb_faces, 3)                                            */
  const double* areas_dev;         /* (nb_faces)                                               */
  const double* radii_dev;         /* (nb_faces)                                               */
  int32_t nb_quad_points;
  const double* quad_points_dev;   /* (nb_faces, nb_quad_points, 3)                            */
  const double* quad_weights_dev;  /* (nb_faces, nb_quad_points)                               */
  /* tabulation (nr or nz <= 1 selects direct integration, as the reference) */
  int32_t tabulation_nb_integration_points;
  int32_t tabulation_grid_shape;
  int32_t nr;
  int32_t nz;
  const double* r_range_dev;
  const double* z_range_dev;
  const double* table_dev;         /* (nr, nz, 5) C-order float64                              */
  const float* table32_dev;        /* optional float32 copy for BEM_PREC_MIXED (may be NULL)   */
  /* problem */
  double wavenumber;               /* 0 and +inf are allowed (no wave term)                    */
  double free_surface;             /* +inf: Rankine kernel only (no free surface)              */
  int32_t gf_singularities;        /* BEM_GF_*                                                 */
  int32_t adjoint_double_layer;    /* 1: K (derivative w.r.t. collocation point), 0: D          */
  int32_t early_dot_product;       /* 1: K (n, N); 0: three gradient planes                    */
  int32_t diagonal_term;           /* add 1/2 (1 on free-surface panels) on the diagonal       */
  int32_t precision;               /* BEM_PREC_*                                               */
  /* outputs */
  int32_t out_dtype;               /* BEM_DTYPE_*                                              */
  void* S_dev;                     /* (n, N) column-major, leading dimension lds               */
  void* K_dev;                     /* (n, N) column-major (ldk), or 3 planes ldk*N apart       */
  int64_t lds;
  int64_t ldk;
  int64_t k_plane_stride;          /* elements between gradient planes when !early_dot_product */
  int32_t* nan_flag_dev;           /* optional: set to 1 if a NaN was produced                  */
  /* optional: reciprocal Lagrange denominators of the table's r and z grids
   * (3 per node, bem_tabulation_inverse_denominators); NULL: divided each time */
  const double* r_inv_den_dev;     /* (nr, 3)                                                  */
  const double* z_inv_den_dev;     /* (nz, 3)                                                  */
} bem_assembly_args;

/* S and K (or D, or the full gradient) for one wavenumber, infinite depth.
 * Replaces matrices::build_matrices, add_diagonal_term and add_rankine_term_only
 * (libs/libDelhommeau/src/matrices.f90:28-432), called from capytaine
 * green_functions/delhommeau.py:377-390 and 498-515. */
int bem_assemble(const bem_assembly_args* args, void* stream);

/* Wavenumber-independent part of the assembly, kept for reuse across
 * frequencies (no counterpart in the reference, which recomputes it for every
 * frequency in matrices.f90:28-432): out(I, J) = (direct + reflected Rankine G,
 * dot normal . their gradient), unscaled, column-major complex128 with leading
 * dimension ld, the diagonal term excluded.  Same arguments as bem_assemble
 * (S/K unused); the reflected-term sign follows the variant in force at
 * args->wavenumber.  Needs a free surface, early_dot_product and
 * gf_singularities high_freq or low_freq. */
int bem_assemble_rankine_part(const bem_assembly_args* args, void* out_dev, int64_t ld, void* stream);

/* S and K of a mesh with itself at args->wavenumber (finite, > 0) from a Rankine
 * part made by bem_assemble_rankine_part with the same arguments: the wave term
 * (Green_wave.f90:50-271) is evaluated once per unordered pair of faces and
 * written to both entries (it is symmetric, its horizontal gradient changes
 * sign).  Same results as bem_assemble up to rounding.  Needs n == nb_faces, one
 * quadrature point per face, the same device array for points_dev, centers_dev
 * and quad_points_dev (collocation at the quadrature points), float64
 * precision and complex128 outputs. */
int bem_assemble_wave_symmetric(const bem_assembly_args* args, const void* rankine_dev, int64_t ld, void* stream);

/* bem_assemble_wave_symmetric for nk wavenumbers (host array) in one launch per
 * 64 of them (a small mesh alone does not fill the GPU): the outputs of
 * wavenumber i are args->S_dev + i * s_stride and args->K_dev + i * k_stride
 * (complex128 elements); args->wavenumber is not used.  Same results as nk
 * calls of bem_assemble_wave_symmetric.  No counterpart in the reference
 * (matrices.f90:28-432 is called once per wavenumber). */
int bem_assemble_wave_symmetric_batched(const bem_assembly_args* args, const void* rankine_dev, int64_t ld,
                                        const double* wavenumbers_host, int nk, int64_t s_stride, int64_t k_stride,
                                        void* stream);

/* bem_assemble_wave_symmetric_batched that also writes K rounded to float32
 * into the planes of a mixed-LU workspace (lu_work_dev of
 * bem_clu_workspace_bytes(npad, ...), matrices first .. first + nk - 1), the
 * way bem_clu_factor converts it; bem_clu_factor_planes then factors them
 * without reading K again.  K and S are written as by the batched call.  No
 * counterpart in the reference (matrices.f90:28-432 writes complex128 only). */
int bem_assemble_wave_symmetric_batched_lu(const bem_assembly_args* args, const void* rankine_dev, int64_t ld,
                                           const double* wavenumbers_host, int nk, int64_t s_stride,
                                           int64_t k_stride, void* lu_work_dev, int npad, int first, void* stream);

/* S and K of a mesh with itself at one wavenumber (finite, > 0) with no cached
 * Rankine part: bem_assemble_rankine_part into K_dev, then the wave term once
 * per unordered pair of faces added in place.  Same requirements as
 * bem_assemble_wave_symmetric; same results as bem_assemble up to rounding.
 * One frequency of a body that is not seen again (a request of the server). */
int bem_assemble_symmetric(const bem_assembly_args* args, void* stream);

/* S and K in water of depth `depth` (finite, > 0), Delhommeau's method:
 * bem_assemble's terms plus the Rankine images through the sea bottom, the
 * four infinite-depth wave terms of the point and the face and of their
 * images through the bottom (scaled by Delhommeau's factor), and four Rankine
 * images per exponential of the Prony decomposition prony_dev (device, 2 x nexp
 * float64: growth rates, then amplitudes; nexp <= 64).  method: 0 = legacy
 * (one-point free-surface image), 1 = newer.  args->precision must be
 * BEM_PREC_FP64 (every term in float64); complex128 or complex64 outputs; K
 * with the dot product taken or the three gradient planes, as bem_assemble.
 * The variant args->gf_singularities is used as given (the caller applies
 * delhommeau.py:467-487).  Replaces the finite-depth branch of
 * matrices::build_matrices (libs/libDelhommeau/src/matrices.f90:197-305,
 * Green_wave.f90:311-508), called from delhommeau.py:492-515. */
int bem_assemble_finite_depth(const bem_assembly_args* args, double depth, int method, const double* prony_dev,
                              int nexp, void* stream);

/* Any collocation points (args->n) against a mesh (args->nb_faces panels, one
 * quadrature point per face, the same device array for centers_dev and
 * quad_points_dev) at nk wavenumbers, from a Rankine part made by
 * bem_assemble_rankine_part with the same arguments: the wave term of every
 * entry plus the cached part, outputs as in bem_assemble_wave_symmetric_batched.
 * Same results as bem_assemble per wavenumber up to rounding.  The first block
 * column of a mesh with symmetries (its whole mesh against the reference
 * sub-mesh) across a frequency sweep.  No counterpart in the reference. */
int bem_assemble_wave_cached(const bem_assembly_args* args, const void* rankine_dev, int64_t ld,
                             const double* wavenumbers_host, int nk, int64_t s_stride, int64_t k_stride, void* stream);

/* ---- dense complex128 linear algebra (batched) ---------------------------- */
/* Matrices are column-major complex128 (interleaved re, im), `batch` of them
 * `stride` elements apart.  n must be a multiple of 64: pad the system with the
 * identity (bem_zpad_identity) and the right-hand sides with zeros. */

/* Zero rows and columns n..npad-1 and put ones on their diagonal. */
int bem_zpad_identity(void* A_dev, int64_t lda, int64_t stride, int batch, int n, int npad, void* stream);

/* C = alpha A B + beta C (alpha, beta real), float64 tensor-core MMAs. */
int bem_zgemm(int M, int N, int K, double alpha, const void* A_dev, int64_t lda, int64_t strideA,
              const void* B_dev, int64_t ldb, int64_t strideB, double beta, void* C_dev, int64_t ldc,
              int64_t strideC, int batch, void* stream);

/* Workspace of bem_zlu_factor / bem_zlu_solve in bytes (inverted diagonal
 * blocks and completion flags). */
int64_t bem_zlu_workspace_bytes(int n, int batch);

/* In-place LU factorisation P A = L U, partial pivoting within each 64-row
 * diagonal block.  Replaces LAPACK zgetrf behind scipy.linalg.lu_factor
 * (capytaine tools/block_circulant_matrices.py:361-378, bem/engines.py:326-338).
 * piv_dev: batch x n ints (row permutation inside each block); info_dev: batch
 * ints, 0 or the 1-based column of the first zero pivot (as LAPACK's info). */
int bem_zlu_factor(void* A_dev, int n, int64_t lda, int64_t stride, int batch, int* piv_dev, int* info_dev,
                   void* work_dev, void* stream);

/* Solve A X = B in place for nrhs <= 64 columns with the factors of
 * bem_zlu_factor.  Replaces LAPACK zgetrs behind scipy.linalg.lu_solve
 * (tools/block_circulant_matrices.py:382-385).  err_dev: one int set to 1 when
 * a bounded wait of the persistent kernel timed out (result invalid). */
int bem_zlu_solve(const void* A_dev, int n, int64_t lda, int64_t stride, int batch, const int* piv_dev,
                  const void* work_dev, void* B_dev, int64_t ldb, int64_t strideB, int nrhs, int* err_dev,
                  void* stream);

/* Float64 solve with a residual check: X solves K X = B with the factors of
 * bem_zlu_factor (LU_dev: the factored copy of K, npad x npad, ldlu, strideLU)
 * and the residual r = b - K x is evaluated in float64 against the
 * unfactored K (n x n, ldk, strideK) after each solve; while the worst
 * relative residual |r| / |b| of a column exceeds tol, x += LU^{-1} r.  The
 * factorisation pivots inside its 64-row diagonal blocks only, where LAPACK's
 * zgetrf searches the whole column: this check reports, and the iteration
 * repairs, any accuracy that the restricted pivoting loses (a well-pivoted
 * factorisation converges in one iteration).  B, X, R: complex128 npad x nrhs
 * (rows n..npad-1 of B zero), nrhs <= 16; ts_work_dev sized by
 * bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch); norms_dev 2*batch*nrhs + 2
 * doubles; iters_out / resid_out: iterations taken and the final worst
 * relative residual.  BEM_ERR_NOT_CONVERGED (X holds the last iterate) as
 * bem_refine_solve.  Replaces zgetrs behind scipy.linalg.lu_solve
 * (tools/block_circulant_matrices.py:382-385) together with the check that
 * zgetrf's full-column pivoting makes unnecessary there. */
int bem_zlu_refine_solve(const void* K_dev, int64_t ldk, int64_t strideK, int n, const void* LU_dev, int npad,
                         int64_t ldlu, int64_t strideLU, int batch, const int* piv_dev, void* lu_work_dev,
                         const void* B_dev, void* X_dev, void* R_dev, int64_t ldb, int64_t strideB, int nrhs,
                         double tol, int max_iter, void* ts_work_dev, double* norms_dev, int* err_dev,
                         int* iters_out, double* resid_out, void* stream);

/* ---- right-hand sides, potentials, forces --------------------------------- */
/* Columns 0..ndof-1: radiation BC -1j*omega*(dof . n) (dofn_dev: ndof x n);
 * columns ndof..ndof+nhead-1: diffraction BC -(u_Airy . n) in water of depth
 * water_depth (> 0; +inf: infinite depth): depth profiles cosh(k(z+h))/cosh(kh)
 * and sinh(k(z+h))/cosh(kh) when 0 <= kh < 20, else e^{kz}.  Zero where
 * hull_dev[i] == 0 (lid panels; hull_dev may be NULL).  One batch entry per
 * frequency (omega_dev, wavenumber_dev: batch doubles; the wavenumbers are the
 * roots of the dispersion relation in that depth).  Replaces
 * bem/problems_and_results.py:373-381, 440-449 and bem/airy_waves.py:56-95. */
int bem_build_rhs(int n, int batch, const double* omega_dev, const double* wavenumber_dev, double g,
                  double water_depth, int ndof, const double* dofn_dev, int nhead, const double* headings_dev,
                  const double* centers_dev, const double* normals_dev, const int32_t* hull_dev, void* B_dev,
                  int64_t ldb, int64_t strideB, void* stream);

/* Y = alpha A X + beta Y, A (M x K) complex128, X (K x nrhs), nrhs <= 16:
 * the potential S @ sigma (bem/solver.py:197-198) and residuals. */
int64_t bem_zgemm_ts_workspace_bytes(int M, int K, int nrhs, int batch);
int bem_zgemm_ts(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                 int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re, double beta_im,
                 void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* work_dev, void* stream);

/* F[b][c][d] = i omega_b rho sum_i phi[b][i][c] wdof[d][i] with
 * wdof[d][i] = -(dof_d . n_i) area_i on hull panels (0 on lid panels).
 * Replaces bodies/bodies.py:238-250 applied to bem/solver.py:199-207. */
int bem_integrate_pressure(int n, int batch, int nrhs, int ndof, const void* phi_dev, int64_t ldp, int64_t strideP,
                           const double* omega_dev, double rho, const double* wdof_dev, void* F_dev, void* stream);

/* Froude-Krylov force of each heading: F[b][h][d] = sum_i p0_i wdof[d][i],
 * p0 = rho g cih(z) exp(i k (x cos beta + y sin beta)), cih the depth profile
 * of bem_build_rhs (exp(k z) in infinite depth) (airy_waves.py:19-53,98-102). */
int bem_froude_krylov(int n, int batch, int ndof, int nhead, const double* wavenumber_dev, double rho, double g,
                      double water_depth, const double* headings_dev, const double* centers_dev,
                      const double* wdof_dev, void* F_dev, void* stream);

/* ---- tensor-core complex update (mixed precision) ------------------------- */
/* C -= A B for complex A (m x k) and B (k x n) on the tcgen05 tensor cores with
 * TF32 inputs and FP32 accumulation, C stored as two float32 planes (Cr, Ci),
 * column-major with leading dimension ldc, trailing block starting at
 * (c_row0, c_col0), m and n multiples of 128.  Operands are packed K-major with
 * K' = kp = 2k (multiple of 32):
 *   Aop[b][a_row0 + i][:] = [Re A(i, :), Im A(i, :)]
 *   Bop[b][b_row0 + 2*j0 + t][:]       = [Re B(:, j0+t); -Im B(:, j0+t)]
 *   Bop[b][b_row0 + 2*j0 + 128 + t][:] = [Im B(:, j0+t);  Re B(:, j0+t)]
 * for each group of 128 columns j0 and t < 128.  err_dev is set to 1 when a
 * bounded wait inside the kernel gave up.  This is the trailing update of the
 * mixed-precision LU that replaces zgetrf's (tools/block_circulant_matrices.py:378). */
int bem_cgemm_tf32_update(const float* Aop_dev, int64_t a_rows, int a_row0, const float* Bop_dev, int64_t b_rows,
                          int b_row0, int kp, float* Cr_dev, float* Ci_dev, int64_t ldc, int64_t c_stride,
                          int c_row0, int c_col0, int m, int n, int batch, int* err_dev, void* stream);

/* ---- mixed-precision solve ------------------------------------------------- */
/* Workspace of bem_clu_factor / bem_clu_solve (float32 planes of K, packed
 * tensor-core operands, inverted diagonal blocks, flags); 1024-byte aligned. */
int64_t bem_clu_workspace_bytes(int npad, int batch);

/* Float32 block LU of the complex128 matrices K (n x n, leading dimension ldk,
 * `batch` of them strideK apart): copy to float32 planes padded to npad
 * (multiple of 128) with the identity, then K = L U with L unit block lower
 * (L_ik = K_ik K_kk^{-1}) and U block upper, 128-wide blocks; each diagonal
 * block is inverted by Gauss-Jordan elimination with partial pivoting among
 * its rows, trailing updates run on the tcgen05 tensor cores (TF32 inputs,
 * FP32 accumulation).  piv_dev (batch x npad ints) is reserved: no row
 * permutation leaves the diagonal blocks.  info_dev: batch ints, 0 or the
 * 1-based column of the first zero pivot; err_dev: bounded-wait timeout flag.
 * Replaces the LU of tools/block_circulant_matrices.py:361-378 in the
 * mixed-precision engine. */
int bem_clu_factor(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch, int* piv_dev,
                   int* info_dev, void* work_dev, int* err_dev, void* stream);

/* bem_clu_factor for a batch of matrices of different sizes held in one
 * padded batch: matrix b is identity-padded beyond its active size
 * active_host[b] (a multiple of 128, <= npad; host array), and the
 * tensor-core updates skip every tile beyond it (those updates are exact
 * no-ops: the padding's off-diagonal blocks are zero), so each matrix costs
 * the flops of its own size.  Same factors as bem_clu_factor, bit for bit.
 * No counterpart in the reference (capytaine solves one problem at a time,
 * bem/solver.py:327-369). */
int bem_clu_factor_grouped(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch,
                           const int* active_host, int* piv_dev, int* info_dev, void* work_dev, int* err_dev,
                           void* stream);

/* bem_clu_factor of matrices already in the workspace's float32 planes
 * (written by bem_assemble_wave_symmetric_batched_lu): the identity padding
 * beyond n, then the same factorisation, bit for bit.  Replaces the same
 * zgetrf as bem_clu_factor (tools/block_circulant_matrices.py:374-385). */
int bem_clu_factor_planes(int n, int npad, int batch, int* piv_dev, int* info_dev, void* work_dev, int* err_dev,
                          void* stream);

/* B <- (LU)^{-1} B with the float32 block factors; B complex128 (npad x nrhs, ldb); piv_dev reserved. */
int bem_clu_solve(void* work_dev, int npad, int batch, const int* piv_dev, void* B_dev, int64_t ldb,
                  int64_t strideB, int nrhs, int* err_dev, void* stream);

/* No counterpart in the reference: a test of the bounded waits.  bem_clu_solve
 * with the iteration limit of the flag waits of its block substitutions given
 * (spin_limit > 0 polls of ~64 ns; bem_clu_solve uses 4e6) and, when
 * withheld_block >= 0, that block row's completion flag never published, so
 * that every wait on it runs out: each waiting block then sets *err_dev = 1
 * and finishes (its result is invalid, every access stays in bounds), and the
 * stream remains usable.  withheld_block = -1 gives bem_clu_solve's result. */
int bem_clu_solve_bounded(void* work_dev, int npad, int batch, const int* piv_dev, void* B_dev, int64_t ldb,
                          int64_t strideB, int nrhs, long long spin_limit, int withheld_block, int* err_dev,
                          void* stream);

/* Iterative refinement: X solves K X = B to a relative residual below tol in
 * every column (residual r = b - K x evaluated in float64 against the float64
 * K, correction from the float32 LU, solved in place in R).  B, X, R:
 * complex128 npad x nrhs (rows n..npad-1 of B zero), nrhs <= 16; work_dev the
 * factorisation of bem_clu_factor; ts_work_dev sized by
 * bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch); norms_dev: 2*batch*nrhs + 2
 * doubles.  The convergence test runs on the device: iterations are enqueued
 * in groups of four and those after convergence return at once, so the stream
 * is synchronised once per group.  Returns BEM_ERR_NOT_CONVERGED (X holds the
 * last iterate) when max_iter is reached or when a group of iterations does
 * not halve the residual (the float32 factors are too far from K for the
 * iteration to contract).  Replaces the lu_solve of
 * tools/block_circulant_matrices.py:382-385. */
int bem_refine_solve(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch, void* work_dev,
                     const int* piv_dev, const void* B_dev, void* X_dev, void* R_dev, int64_t ldb, int64_t strideB,
                     int nrhs, double tol, int max_iter, void* ts_work_dev, double* norms_dev, int* err_dev,
                     int* iters_out, double* resid_out, void* stream);

/* ---- GMRES ------------------------------------------------------------------ */
/* Workspace of bem_gmres_solve in bytes (the Krylov basis V and the basis Z of
 * preconditioned vectors, both restart + 1 vectors per system, Hessenberg
 * matrices, rotations, per-system state, tall-GEMM partial sums); -1 for bad
 * sizes. */
int64_t bem_gmres_workspace_bytes(int n, int npad, int nrhs, int batch, int restart);

/* Restarted GMRES, x0 = 0, for each of the nrhs columns of each of the `batch`
 * matrices A (n x n complex128, column-major, lda, strideA apart).  Column c of
 * B (ldb, strideB; rows < n read) converges when |b - A x| <= max(atol, rtol |b|);
 * inner iterations stop when the (preconditioned) Arnoldi residual meets the
 * adaptive inner tolerance, as scipy.sparse.linalg.gmres does.  restart <= 64
 * (capytaine/SciPy: 20), at most max_cycles restart cycles.
 * precond_work_dev: NULL for plain GMRES, or the factorisation of
 * bem_clu_factor (npad multiple of 128, err_dev required) used as the right
 * preconditioner M^-1 = (LU)^-1 with float32 factors and float64 products, in
 * the flexible form (z_k = M^-1 v_k kept, x += Z y at the end of a cycle, so
 * that the rounding of the float32 substitutions cannot make the final update
 * disagree with the Arnoldi products): GMRES-based iterative refinement of the
 * mixed-precision LU.  X (ldb,
 * strideB): rows < n written.  work_dev: bem_gmres_workspace_bytes, 256-byte
 * aligned.  iters_out: largest number of inner iterations over the systems;
 * resid_out: largest |b - A x| / |b| over the systems with |b| >= atol (the
 * others are solved by x = 0, as SciPy does).  Synchronises the stream once per group
 * of four inner iterations and once per cycle.  Returns BEM_ERR_NOT_CONVERGED
 * when a system breaks down or max_cycles is reached.  Replaces
 * scipy.sparse.linalg.gmres behind capytaine's solve_gmres
 * (bem/engines.py:74-89). */
int bem_gmres_solve(const void* A_dev, int64_t lda, int64_t strideA, int n, int npad, int batch, const void* B_dev,
                    void* X_dev, int64_t ldb, int64_t strideB, int nrhs, double atol, double rtol, int restart,
                    int max_cycles, void* precond_work_dev, void* work_dev, int* err_dev, int* iters_out,
                    double* resid_out, void* stream);

/* ---- symmetric meshes ------------------------------------------------------ */
/* out[f][o][c][r] = sum_{i < mi} W[o][i] in[f][src[i]][c][r] for o < mo, r < rows,
 * c < cols, f < nf, complex128; element (f, b, c, r) of `in` at
 * in + f*in_fstride + b*in_bstride + c*in_cstride + r (elements), likewise for
 * `out`.  W: mo x mi row-major complex128 on the device; source_dev: mi int32
 * block indices, or NULL for src[i] = i.  `out` must not overlap `in`.
 * cols <= 65535 and nf * ceil(mo / 8) <= 65535.
 * With the first column of blocks of a mesh with reflection or rotation
 * symmetry as `in` (rows of block j at j * n_sub) and the group's Fourier
 * weights as W, it writes the independent systems of the block-diagonalised
 * matrix; with vectors it takes right-hand sides to those systems and
 * solutions back.  Replaces BlockCirculantMatrix.block_diagonalize, the
 * np.fft.fft / ifft of the right-hand sides in LUDecomposedBlockCirculantMatrix
 * .solve and NestedBlockCirculantMatrix.to_BlockCirculantMatrix
 * (tools/block_circulant_matrices.py:138-162, 226-266, 276-301, 410-419). */
int bem_block_combine(const void* in_dev, int64_t in_fstride, int64_t in_bstride, int64_t in_cstride, void* out_dev,
                      int64_t out_fstride, int64_t out_bstride, int64_t out_cstride, const void* weights_dev,
                      const int32_t* source_dev, int mi, int mo, int rows, int cols, int nf, void* stream);

/* ---- whole frequency-solves, LU handles, requests ------------------------- */
/* Opaque handles owned by the library until bem_release. */
typedef struct bem_context bem_context;
typedef struct bem_lu bem_lu;
typedef struct bem_request bem_request;

/* Parameters of the Delhommeau Green function, as the keywords of
 * Delhommeau.__init__ (green_functions/delhommeau.py:30-41, 116-140): reference
 * defaults 676, 100.0, 372, -251.0, 1001, BEM_GRID_SCALED_NEMOH3,
 * BEM_GF_LOW_FREQ.  tabulation_nr or _nz <= 1: no table (direct integration). */
typedef struct {
  int32_t tabulation_nr;
  double tabulation_rmax;
  int32_t tabulation_nz;
  double tabulation_zmin;
  int32_t tabulation_nb_integration_points;
  int32_t tabulation_grid_shape;  /* BEM_GRID_*                                   */
  int32_t gf_singularities;       /* BEM_GF_HIGH_FREQ or BEM_GF_LOW_FREQ          */
} bem_green_function_params;

/* A mesh in host memory, with the per-face arrays capytaine computes
 * (meshes/geometry.py:35-85) and passes to matrices::build_matrices
 * (matrices.f90:28-90): the quadrature is the default one point per face (the
 * centre, weight = area, meshes/meshes.py:472-486).  hull_mask: 1 for hull
 * faces, 0 for lid faces (irregular-frequency removal, meshes.py:655-737);
 * NULL: every face is hull. */
typedef struct {
  int32_t nb_faces;
  int32_t nb_vertices;
  const double* vertices;   /* (nb_vertices, 3)            */
  const int32_t* faces;     /* (nb_faces, 4), 0-based      */
  const double* centers;    /* (nb_faces, 3)               */
  const double* normals;    /* (nb_faces, 3)               */
  const double* areas;      /* (nb_faces)                  */
  const double* radii;      /* (nb_faces)                  */
  const int32_t* hull_mask; /* (nb_faces) or NULL          */
} bem_mesh_desc;

typedef struct {
  int32_t iterations;          /* most refinement (or GMRES) iterations of a solve     */
  double residual;             /* worst final relative residual |b - K x| / |b|         */
  int32_t escalated_to_gmres;  /* solves whose refinement continued with GMRES         */
} bem_solve_stats;

/* A context on `device`: the tabulation of the Green function built on the
 * device (delhommeau.py:208-261, Delhommeau_integrals.f90:190-204) and kept
 * until bem_release.  Replaces Delhommeau.__init__.  Synchronous. */
int bem_context_create(int device, const bem_green_function_params* params, bem_context** out);
/* Copies of the context's grid (nr, nz) and table (nr, nz, 5 C-order) to host
 * memory (any pointer may be NULL), and replacement of the table by a host copy
 * (a table loaded from capytaine's npz cache, delhommeau.py:221-251). */
int bem_context_tabulation(const bem_context* ctx, double* r_range_host, double* z_range_host, double* table_host);
int bem_context_set_tabulation(bem_context* ctx, const double* table_host);

/* The frequency-solves of one body in infinite depth, host buffers in and out:
 * for each of the nomega angular frequencies (finite, > 0; k = omega^2 / g),
 * S and K assembled on the device (the wavenumber-independent Rankine part
 * once for the call), K factored (precision BEM_PREC_MIXED: float32 block LU
 * with tcgen05 trailing updates and float64-residual refinement to 1e-10,
 * continued with preconditioned GMRES when it stops contracting;
 * BEM_PREC_FP64: float64 block LU with the residual refined to 1e-13), the
 * radiation problems of the ndof dofs (dof_normals: ndof x nb_faces, the
 * normal component dof(x_i) . n_i of each dof's motion at the face centres,
 * problems_and_results.py:440-449) and the diffraction problems of the nhead
 * wave directions (radians, Airy waves, airy_waves.py:56-95), the potential
 * S sigma, the forces on the hull faces (bodies/bodies.py:238-250) and the
 * coefficients (problems_and_results.py:583-592):
 *   added_mass[w][i][j] = Re F_ij / omega^2, damping[w][i][j] = Im F_ij / omega
 *   (i the radiating dof, j the influenced one; ndof x ndof per frequency),
 *   excitation[w][h][j] = diffraction + Froude-Krylov force, complex as
 *   (re, im) pairs (nhead x ndof x 2 doubles per frequency; NULL if nhead = 0).
 * ndof + nhead <= 64.  The variant overrides of delhommeau.py:466-490 apply
 * (faces on the free surface force low_freq).  Synchronous; calls on one
 * context from several host threads may overlap (each call has its own stream
 * and buffers).  Replaces the solve_all loop of one body over its problems
 * (bem/solver.py:268-372) for the indirect method. */
int bem_solve_frequency(const bem_context* ctx, const bem_mesh_desc* mesh, int nomega, const double* omegas,
                        int ndof, const double* dof_normals, int nhead, const double* headings, double rho, double g,
                        int precision, double* added_mass, double* damping, double* excitation,
                        bem_solve_stats* stats);

/* bem_solve_frequency on a worker thread: returns at once with a request; the
 * mesh, its arrays and the input and output buffers must stay valid until
 * bem_request_poll has reported completion.  bem_request_poll(req, wait = 0)
 * returns BEM_PENDING while the request runs, else its status (wait != 0
 * blocks until it completes); release the request with bem_release.  No
 * counterpart in the reference (capytaine runs problems in joblib processes,
 * bem/solver.py:327-369). */
int bem_solve_submit(const bem_context* ctx, const bem_mesh_desc* mesh, int nomega, const double* omegas, int ndof,
                     const double* dof_normals, int nhead, const double* headings, double rho, double g,
                     int precision, double* added_mass, double* damping, double* excitation, bem_request** out);
int bem_request_poll(bem_request* req, int wait, bem_solve_stats* stats);

/* LU handle of a complex128 matrix K (n x n, column-major, leading dimension
 * ldk, device memory): the library copies K (kept for the residuals) and
 * factors it (precision as bem_solve_frequency).  Replaces lu_decompose /
 * LUDecomposedMatrix (tools/block_circulant_matrices.py:361-378) behind
 * DefaultMatrixEngine.linear_solver (bem/engines.py:300-346), which keeps the
 * factors in its cache in place of K.  Synchronous; BEM_ERR_SINGULAR for a
 * zero pivot. */
int bem_lu_factor(const bem_context* ctx, const void* K_dev, int64_t ldk, int n, int precision, bem_lu** out);
/* X (n x nrhs, ldx, device) solving K X = B (ldb, device) with the handle's
 * factors, refined against the kept K as bem_solve_frequency's solves.
 * Replaces lu_solve (tools/block_circulant_matrices.py:382-385).
 * Synchronous. */
int bem_lu_solve(bem_lu* lu, const void* B_dev, int64_t ldb, int nrhs, void* X_dev, int64_t ldx,
                 bem_solve_stats* stats);
/* Frees a context, an LU handle or a finished request (a running request is
 * waited for).  NULL is accepted. */
int bem_release(void* handle);

/* ---- allocation-free variant ---------------------------------------------- */
/* No counterpart in the reference.  Same operation and arguments as
 * bem_zgemm_ts without the workspace: for callers that can only pass buffers
 * they already own (a fixed device pool that allows no further allocation, or
 * a loop where a cudaMalloc is unacceptable).  The split-K partial sums live in
 * a static device array of bem_zgemm_ts_static_capacity() = 524288 complex128
 * entries (8 MiB, held on every GPU that loads the library until exit);
 * M * nrhs * batch must not exceed it and batch must not exceed 65535 (else
 * BEM_ERR_INVALID_ARGUMENT).  The first call on a device (and the first after
 * its context was reset and re-created) looks the array up: make it before
 * any stream capture.  Calls that overlap on the GPU share the array and race. */
int64_t bem_zgemm_ts_static_capacity(void);
int bem_zgemm_ts_static(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                        int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re,
                        double beta_im, void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CAPYTAINE_B200_H */
