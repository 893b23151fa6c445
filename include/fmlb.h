/*
 * fmlb.h — C ABI of libfmlb.so, the B200 (sm_100a) implementation of the
 * andersx/fml kernel-ridge-regression hot path.
 *
 * Conventions
 *   - Every pointer argument is DEVICE memory unless stated otherwise; the
 *     caller owns all buffers. Arrays are C-order (row-major).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream). Calls are asynchronous on that stream unless stated.
 *   - Return value: FMLB_OK (0) or a negative error code; the message of the
 *     last error on the calling thread is in fmlb_last_error_string().
 *   - Descriptors are rows: a descriptor matrix of n descriptors of length d
 *     is an (n, d) array with leading dimension ld >= d. The reference's
 *     Python wrappers take the transpose, (d, n), and hand f2py Fortran-order
 *     arrays whose columns are descriptors; the memory layout is the same.
 *
 * Each entry point names the reference routine it replaces (file:line in the
 * andersx/fml tree).
 */
#ifndef FMLB_H
#define FMLB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FMLB_OK 0
#define FMLB_EINVAL (-22)    /* invalid argument (shape, size, pointer) */
#define FMLB_ENOMEM (-12)    /* workspace too small */
#define FMLB_ECUDA (-5)      /* CUDA launch / runtime error */
#define FMLB_ENOTSUP (-95)   /* size outside what the kernels support */
#define FMLB_ETIMEDOUT (-110)/* a bounded device-side wait gave up */

/* Message describing the last error returned on this thread ("" if none). */
const char *fmlb_last_error_string(void);

/* ABI version of this library. */
int fmlb_version(void);

/* ------------------------------------------------------------------------
 * Sorted Coulomb matrices for a packed ragged batch of molecules.
 * Replaces fgenerate_coulomb_matrix, fml/representations/frepresentations.f90:23-110
 * (called per molecule by Molecule.generate_coulomb_matrix, fml/fml.py:64-66).
 *
 *   charges  (total_atoms,)    nuclear charges
 *   coords   (total_atoms, 3)  Cartesian coordinates
 *   offsets  (nmol + 1,) int   molecule m owns atoms [offsets[m], offsets[m+1])
 *   nmax     padded size; each output row holds nmax*(nmax+1)/2 values
 *   cm       (nmol, ldcm) float64 output, ldcm >= nmax*(nmax+1)/2 (may be NULL)
 *   cm32     (nmol, ldcm32) float32 copy of the same values (may be NULL);
 *            columns beyond nmax*(nmax+1)/2 are zeroed up to ldcm32
 *   order    (nmol, nmax) int: original atom index at each sorted position,
 *            -1 past the molecule's atom count (may be NULL)
 * Row-norm order: descending, ties -> higher original index first
 * (the reference's repeated minloc filled from the end, :86-91).
 *   status   device int (may be NULL): set to 1 when a molecule has more than
 *            nmax atoms (the reference writes out of bounds there); that
 *            molecule's row is written as zeros.
 * Errors: FMLB_EINVAL if nmax is outside 1..255 or a leading dimension is short.
 * ---------------------------------------------------------------------- */
int fmlb_coulomb_matrices(const double *charges, const double *coords, const int *offsets,
                          int nmol, int nmax, double *cm, int ldcm, float *cm32, int ldcm32,
                          int *order, int *status, void *stream);

/* Packed form of fmlb_vector_kernels_f64: X1 (total_atoms1, d) rows with
 * molecule offsets O1 (nm1 + 1), likewise X2 / O2; amax1 / amax2 bound the
 * atoms of one molecule. With kind 1 and X1 = X2 this is the molecule kernel
 * of fget_alpha (fml/kernels/fkernels.f90:380-440, wrapper get_alpha,
 * kernels.py:119-126). */
int fmlb_vector_kernels_packed_f64(int kind, const double *X1, const int *O1, int nm1, int amax1,
                                   const double *X2, const int *O2, int nm2, int amax2, int d,
                                   const double *sigmas_host, int nsig, double *K, int *status,
                                   void *stream);

/* Atomic KRR from precomputed atom-pair distances (fml/kernels/fkernels.f90:541-702,
 * wrappers get_alpha_from_distance / get_prediction_from_distance,
 * kernels.py:110-134):
 * fmlb_segment_exp_sum_f64: S[p, q] = sum over rows R[p]..R[p+1] and columns
 *   C[q]..C[q+1] of exp(c M[r, s]) (M row-major, rows x cols); with M the
 *   atom distance matrix and R = C the molecule offsets, S is the transposed
 *   molecule kernel of fget_alpha_from_distance (:586-597).
 * fmlb_exp_weighted_colsum_f64: v[s] = sum_r exp(c M[r, s]) w[r], the per-atom
 *   sums of fget_prediction_from_distance (:688-693); scratch of
 *   fmlb_exp_colsum_scratch_doubles(cols) device doubles. Deterministic. */
int fmlb_segment_exp_sum_f64(const double *M, long long ldm, int rows, int cols, const int *R,
                             int np, const int *C, int nq, double c, double *S, long long lds,
                             void *stream);
size_t fmlb_exp_colsum_scratch_doubles(int cols);
int fmlb_exp_weighted_colsum_f64(const double *M, long long ldm, int rows, int cols, double c,
                                 const double *w, double *v, double *scratch, void *stream);

/* ------------------------------------------------------------------------
 * Batched XYZ ingestion (host code, no GPU): many .xyz files parsed with the
 * rules of Molecule.read_xyz (fml/fml.py:109-132) into one packed ragged
 * buffer, on `nthreads` host threads (<= 0: all cores).
 *
 * fmlb_xyz_scan: per file the declared atom count (line 1; may be NULL) and
 *   the number of atom lines (lines 3.. up to the first with fewer than 4
 *   tokens), which sizes the molecule as in the reference.
 * fmlb_xyz_parse: with offsets (nfiles + 1) from the parsed counts, writes
 *   charges (A,), coords (A, 3) and, when not NULL, symbol_index (A,) (index
 *   of the element in the caller's table: table_symbols / table_charges,
 *   the reference's NUCLEAR_CHARGE). Pass page-locked buffers to follow with
 *   one asynchronous copy per array. charges and coords may be NULL when
 *   offsets[nfiles] == 0 (no atoms in the batch).
 * Numbers follow Python's int() and float() for ASCII text (signs, fractions,
 * exponents, inf / infinity / nan in any case, PEP 515 digit-group
 * underscores); tokens split on str.split()'s ASCII whitespace.
 * Errors: FMLB_EINVAL with the file and line in the error string (unreadable
 * file, bad atom count, unknown element, a coordinate that is not a number).
 * ---------------------------------------------------------------------- */
int fmlb_xyz_scan(const char *const *paths, int nfiles, int *natoms_declared, int *natoms_parsed,
                  int nthreads);
int fmlb_xyz_parse(const char *const *paths, int nfiles, const int *offsets,
                   const char *const *table_symbols, const double *table_charges, int ntable,
                   double *charges, double *coords, int *symbol_index, int nthreads);

/* Unsorted Coulomb matrices: one packed lower triangle per molecule in the
 * input atom order, the replacement for fgenerate_unsorted_coulomb_matrix
 * (fml/representations/frepresentations.f90:112-202) as called by
 * Molecule.generate_unsorted_coulomb_matrix (fml/fml.py:68-70). cm (nmol, ldcm),
 * zero padded; status as for fmlb_coulomb_matrices. */
int fmlb_unsorted_coulomb_matrices(const double *charges, const double *coords, const int *offsets,
                                   int nmol, int nmax, double *cm, int ldcm, int *status,
                                   void *stream);

/* ------------------------------------------------------------------------
 * Local / atomic Coulomb matrices: one packed lower-triangle row per atom.
 * Replaces fgenerate_local_coulomb_matrix (kind 0,
 * fml/representations/frepresentations.f90:204-294) and
 * fgenerate_atomic_coulomb_matrix (kind 1, :297-390), as called by
 * Molecule.generate_local_coulomb_matrix / generate_atomic_coulomb_matrix,
 * fml/fml.py:72-78.
 *
 *   cm   (total_atoms, ldcm) float64, row offsets[m] + k holds the matrix of
 *        central atom k of molecule m, nmax(nmax+1)/2 entries, zero padded.
 *        kind 0: k first, then the other atoms by descending row norm;
 *        kind 1: all atoms by ascending distance to k.
 *   status device int (may be NULL): 1 if a molecule has more than nmax atoms.
 * ---------------------------------------------------------------------- */
int fmlb_local_coulomb_matrices(const double *charges, const double *coords, const int *offsets,
                                int nmol, int nmax, int kind, double *cm, int ldcm, int *status,
                                void *stream);

/* ------------------------------------------------------------------------
 * Atomic vector kernels over per-atom descriptors.
 * Replaces fget_vector_kernels_gaussian (kind 0, fml/kernels/fkernels.f90:106-162)
 * and fget_vector_kernels_laplacian (kind 1, :23-104), as called by
 * get_atomic_kernels_gaussian / get_atomic_kernels_laplacian,
 * fml/kernels/kernels.py:351-411.
 *
 *   X1 (nm1, amax1, d), X2 (nm2, amax2, d) float64 device; N1/N2 atom counts.
 *   K  (nsig, nm1, nm2): sum over atom pairs of exp(c_k * dist), dist the
 *      squared L2 (kind 0, c_k = -0.5/sigma_k^2) or the L1 distance (kind 1,
 *      c_k = -1/sigma_k).
 *   sigmas_host host array of nsig (1..32) values; amax1, amax2 1..128.
 * ---------------------------------------------------------------------- */
int fmlb_vector_kernels_f64(int kind, const double *X1, const int *N1, int nm1, int amax1,
                            const double *X2, const int *N2, int nm2, int amax2, int d,
                            const double *sigmas_host, int nsig, double *K, int *status,
                            void *stream);

/* ------------------------------------------------------------------------
 * ARAD descriptors for a packed ragged batch of molecules.
 * Replaces ARAD.describe, fml/arad.py:70-145 (non-periodic path), as called
 * by Molecule.generate_arad_descriptor, fml/fml.py:80-86.
 *
 *   out  (nmol, size, 5, size) float64: channel 0 sorted neighbour distances
 *        (padding 1e100), 1/2 PTP row/column, 3/4 damped mean cos/sin.
 *   cut  neighbour cut-off (Angstrom).
 *   status device int (may be NULL): 1 if a molecule has more than `size`
 *        atoms (its rows are padding only), 2 if a charge has no
 *        periodic-table position (its channels 1/2 hold -1).
 * Errors: FMLB_EINVAL if size is outside 1..128.
 * ---------------------------------------------------------------------- */
int fmlb_arad_descriptors(const double *charges, const double *coords, const int *offsets,
                          int nmol, int size, double cut, double *out, int *status, void *stream);

/* ------------------------------------------------------------------------
 * Gaussian and Laplacian kernel matrices, plain FP64 (direct differences).
 * Replace fgaussian_kernel / flaplacian_kernel, fml/kernels/fkernels.f90:317-377
 * (wrappers gaussian_kernel / laplacian_kernel, fml/kernels/kernels.py:136-196).
 *
 *   A (na, lda), B (nb, ldb): descriptor rows of length d
 *   K: nsigma matrices (na, nb), matrix s at K + s*sigma_stride, row stride ldk
 *      gaussian:  K_s[j,i] = exp(-0.5/sigma_s^2 * sum_k (A[j,k]-B[i,k])^2)
 *      laplacian: K_s[j,i] = exp(-1/sigma_s   * sum_k |A[j,k]-B[i,k]|)
 *   symmetric != 0: A == B (same pointer, na == nb); only tiles on or below
 *      the diagonal are computed and mirrored (results are bit-identical to
 *      the full computation, which is exactly symmetric).
 * ---------------------------------------------------------------------- */
int fmlb_gaussian_kernel_f64(const double *A, int na, int lda, const double *B, int nb, int ldb,
                             int d, const double *sigmas_host, int nsigma, double *K,
                             long long ldk, long long sigma_stride, int symmetric, void *stream);
int fmlb_laplacian_kernel_f64(const double *A, int na, int lda, const double *B, int nb, int ldb,
                              int d, const double *sigmas_host, int nsigma, double *K,
                              long long ldk, long long sigma_stride, int symmetric, void *stream);

/* ------------------------------------------------------------------------
 * ARAD molecular kernels.
 * Replace fget_kernels_arad (fml/kernels/farad_kernels.f90:439-616) and
 * fget_symmetric_kernels_arad (:619-755), core atomic_distl2 (:29-90);
 * wrappers get_atomic_kernels_arad / get_atomic_symmetric_kernels_arad,
 * fml/kernels/kernels.py:229-349.
 *
 *   X1 (nm1, amax, 5, amax), X2 (nm2, amax, 5, amax) float64 ARAD descriptors
 *   Z1 (nm1, amax, 2), Z2 (nm2, amax, 2) float64 PTP (row, column) per atom
 *   N1 (nm1,), N2 (nm2,) int atom counts (<= amax)
 *   sigmas_host (nsigma,) HOST array; K (nsigma, nm1, nm2) float64 output
 *   symmetric != 0: set 2 is set 1 (X2/Z2/N2 ignored), only i <= j computed
 *      and mirrored, with the symmetric routine's sine table (:689-698).
 *   precision: 0 = FP64 (parity path), 1 = FP32 arithmetic, FP64 output.
 *   workspace: device scratch of fmlb_arad_workspace_bytes(...) bytes.
 * Errors: FMLB_ENOTSUP if amax > 64; FMLB_ENOMEM if ws_bytes is too small.
 * ---------------------------------------------------------------------- */
size_t fmlb_arad_workspace_bytes(int nm1, int nm2, int amax, int symmetric);

/* Atom-level ARAD kernel, fget_atomic_kernels_arad
 * (fml/kernels/farad_kernels.f90:757-899), FP64 in the reference's order:
 *   K[s, i, j] = exp(l2(i, j) * -1/sigma_s^2) for every atom i of set 1 and j
 *   of set 2, l2 = self_i + self_j - 2 atomic_distl2(i, j) stoch(z_i, z_j),
 *   |l2| < 5e-12 -> 0.
 *   Q1 (na1, 5, amax) per-atom ARAD descriptors, Z1 (na1, 2) PTP row/column,
 *   N1 (na1,) neighbour counts; the same for set 2 (same amax).
 *   K (nsigma, na1, na2) row-major; nsigma <= 16.
 *   workspace: fmlb_arad_atomic_workspace_bytes(na1, na2, amax) bytes. */
size_t fmlb_arad_atomic_workspace_bytes(int na1, int na2, int amax);
/* The atom-pair l2 distances themselves, fget_atomic_distance_arad
 * (fml/kernels/farad_kernels.f90:902-1030): D[i, j] = l2(i, j) as above, D
 * (na1, na2) row-major; same workspace as fmlb_arad_atomic_kernels. */
int fmlb_arad_atomic_distances(const double *Q1, const double *Z1, const int *N1, int na1,
                               const double *Q2, const double *Z2, const int *N2, int na2,
                               int amax, double width, double cut_distance, double r_width,
                               double c_width, double *D, void *workspace, size_t ws_bytes,
                               void *stream);
int fmlb_arad_atomic_kernels(const double *Q1, const double *Z1, const int *N1, int na1,
                             const double *Q2, const double *Z2, const int *N2, int na2, int amax,
                             const double *sigmas_host, int nsigma, double width,
                             double cut_distance, double r_width, double c_width, double *K,
                             void *workspace, size_t ws_bytes, void *stream);
int fmlb_arad_kernels(const double *X1, const double *Z1, const int *N1, int nm1,
                      const double *X2, const double *Z2, const int *N2, int nm2, int amax,
                      const double *sigmas_host, int nsigma, double width, double cut_distance,
                      double r_width, double c_width, int symmetric, int precision, double *K,
                      void *workspace, size_t ws_bytes, void *stream);

/* The regularised kernel matrix of fget_alpha_arad (fml/kernels/
 * farad_kernels.f90:231-389): K (nm, nm) = the symmetric FP64 ARAD kernel for
 * one sigma with that routine's fixed width 0.2, cut 6, r_width 1, c_width 0.5
 * and eps 1e-11, plus lambda on the diagonal. X, Z, N and the workspace as
 * for fmlb_arad_kernels (fmlb_arad_workspace_bytes(nm, nm, amax, 1)). The
 * rest of the routine is fmlb_potrf_f64, fmlb_potri_f64 and fmlb_gemv_f64. */
int fmlb_arad_alpha_kernel_f64(const double *X, const double *Z, const int *N, int nm, int amax,
                               double sigma, double lambda, double *K, void *workspace,
                               size_t ws_bytes, void *stream);

/* Atom-pair ARAD distances of two molecule sets, the replacement for
 * atomic_arad_l2_distance_all (fml/math/farad.f90:452-600) as called by
 * get_l2_distance_arad (fml/math/distance.py:120-189).
 *   D (nm1, nm2, amax, amax) float64: l2 of atom i1 of molecule i and atom j1
 *     of molecule j, zero past each molecule's atoms.
 * X, Z, N as for fmlb_arad_kernels; workspace of
 * fmlb_arad_workspace_bytes(nm1, nm2, amax, 0) bytes. */
int fmlb_arad_distances(const double *X1, const double *Z1, const int *N1, int nm1,
                        const double *X2, const double *Z2, const int *N2, int nm2, int amax,
                        double width, double cut_distance, double r_width, double c_width,
                        double *D, void *workspace, size_t ws_bytes, void *stream);

/* Generic distance matrices, the replacement for fml/math/fdistance.f90 as
 * called by manhattan_distance / l2_distance / p_distance
 * (fml/math/distance.py:58-117):
 *   kind 0 fmanhattan_distance, 1 fl2_distance, 2 fp_distance_integer
 *   (p_int), 3 fp_distance_double (p_real).
 * A (na, d), B (nb, d) row-major device rows; D (na, nb) with row stride ldd,
 * D[j, i] = dist(A_j, B_i). The p forms raise the signed difference as the
 * reference does. */
int fmlb_distance_matrix_f64(int kind, const double *A, int na, int lda, const double *B, int nb,
                             int ldb, int d, int p_int, double p_real, double *D, long long ldd,
                             void *stream);

/* ------------------------------------------------------------------------
 * Cholesky factorisation and solve, FP64.
 * Replace LAPACK dpotrf('U') / dpotrs('U') as called by fcho_solve,
 * fml/math/fcho_solve.f90:23-47 (wrapper cho_solve, fml/math/cho_solve.py:33-58).
 *
 * A is an (n, n) row-major matrix with row stride lda. The factorisation
 * reads the triangle i >= j of the row-major array and overwrites it with L,
 * A = L L^T. For the reference's C-order numpy argument this is the upper
 * triangle of the Fortran view, A = U^T U with U = L^T, i.e. dpotrf('U').
 *
 *   work     device scratch of fmlb_potrf_workspace_bytes(n) bytes; keeps the
 *            inverted diagonal blocks that fmlb_potrs_f64 reuses.
 *   info     device int: 0, or the 1-based column of the first non-positive
 *            pivot (LAPACK convention); work after a failed pivot is skipped.
 * fmlb_potrs_f64 solves A x = b in place in x (n,) given the factor and work.
 * ---------------------------------------------------------------------- */
size_t fmlb_potrf_workspace_bytes(int n);
int fmlb_potrf_f64(double *A, long long lda, int n, void *work, int *info, void *stream);
int fmlb_potrs_f64(const double *L, long long lda, int n, const void *work, double *x,
                   void *stream);

/* Inverse from the factor, the replacement for LAPACK dpotri('U') after
 * dpotrf('U') as fcho_invert calls them (fml/math/fcho_solve.f90:49-68,
 * wrapper cho_invert, fml/math/cho_solve.py:27-30).
 *
 *   A     the factor from fmlb_potrf_f64 (triangle i >= j); on return that
 *         triangle holds inv(A). The other triangle is not touched.
 *   work  the fmlb_potrf_f64 workspace (inverted diagonal blocks).
 *   V     device scratch (n, ldv), ldv >= n: receives L^-T.
 *   info  the fmlb_potrf_f64 info (device, may be NULL): when non-zero the
 *         inversion is skipped.
 * n <= 65535. */
int fmlb_potri_f64(double *A, long long lda, int n, const void *work, double *V, long long ldv,
                   const int *info, void *stream);

/* Trailing update of the blocked factorisation: C -= P P^T on the triangle
 * i >= j of the row-major (m, m) matrix C, P is (m, k) with stride ldp; the
 * other triangle of C is not touched. strip_cols = 0 updates the whole lower
 * triangle, strip_cols > 0 only its first strip_cols columns. `info` (device,
 * may be NULL): when it holds a non-zero value the update is skipped. The
 * step fmlb_potrf_f64 runs per panel (the LAPACK dsyrk call inside dpotrf,
 * fcho_solve.f90:35). */
int fmlb_syrk_lower_f64(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                        int strip_cols, const int *info, void *stream);

/* FP64-accurate Cholesky factorisation with the trailing updates on the int8
 * tensor cores, the replacement for LAPACK dpotrf('U') as fcho_solve calls it
 * (fml/math/fcho_solve.f90:35) when an iterative refinement follows.
 * Same storage, result layout, workspace prefix (the inverted diagonal blocks
 * that fmlb_potrs_f64 reads) and info as fmlb_potrf_f64; only the bulk and
 * strip trailing updates (C -= P P^T with k = the outer panel width) change:
 * P's rows are split into nslices (1..8) 8-bit digit planes (a signed leading
 * digit, lower digits stored around a zero point) with one power-of-two
 * scale per row, the s(s+1)/2 leading digit products run as tcgen05.mma
 * kind::i8 with exact int32 accumulation, and the epilogue combines them in
 * FP64 and adds the zero-point terms (the Ozaki scheme). Six planes give the
 * accuracy of seven truncated 7-bit planes; seven or eight are below the
 * FP64 rounding bound.
 *   work  fmlb_potrf_ozaki_workspace_bytes(n, nslices) bytes
 *   info  LAPACK-style (> 0: first non-positive pivot); FMLB_ETIMEDOUT (< 0)
 *         if a bounded device-side wait of the tensor-core kernel gave up. */
size_t fmlb_potrf_ozaki_workspace_bytes(int n, int nslices);
int fmlb_potrf_ozaki_f64(double *A, long long lda, int n, int nslices, void *work,
                         size_t ws_bytes, int *info, void *stream);

/* The int8 emulated trailing update on its own (the step above): C -= P P^T
 * on the triangle i >= j of the row-major (m, m) C, or its first strip_cols
 * columns; P is (m, k), k <= 8192. work: fmlb_syrk_ozaki_workspace_bytes
 * (m, k, nslices) bytes (digit planes and row exponents). info (device):
 * skipped when non-zero; FMLB_ETIMEDOUT stored on a device-side timeout.
 * (The LAPACK dsyrk call inside dpotrf, fcho_solve.f90:35.) */
size_t fmlb_syrk_ozaki_workspace_bytes(int m, int k, int nslices);
int fmlb_syrk_lower_ozaki(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                          int strip_cols, int nslices, void *work, size_t ws_bytes, int *info,
                          void *stream);

/* Test hooks of the tensor-core kernels (fmlb_gaussian_kernel_tc,
 * fmlb_syrk_lower_ozaki, fmlb_potrf_ozaki_f64) for later launches from the
 * calling host thread: wait_cycles > 0 sets the clock-cycle limit of every
 * device-side mbarrier wait (0 restores the default, about 2 s); skip_loads
 * != 0 makes the TMA producer issue no copies, so the waits run out with
 * nothing in flight and the kernel reports FMLB_ETIMEDOUT. No reference
 * counterpart (failure-path testing). */
int fmlb_tc_test_hooks(long long wait_cycles, int skip_loads);

/* Double-double iterative refinement after an in-place factorisation of
 * A = K + lambda I (fmlb_potrf_f64 or fmlb_potrf_ozaki_f64), reading K from
 * the strict upper triangle the factorisation leaves untouched and the
 * diagonal from `diag` (saved before factoring with fmlb_get_diagonal_f64).
 * The reference solves once (fml/math/fcho_solve.f90:35-42); this extends it
 * past the FP64 residual floor. x = x + x_lo is kept in double-double; per
 * step r = y - A (x + x_lo) in double-double, (x, x_lo) += solve(L, r).
 * resid (device, iters + 1, may be NULL): ||r||_2 before each step and after
 * the last. scratch: fmlb_krr_refine_dd_scratch_doubles(n). Deterministic. */
int fmlb_get_diagonal_f64(const double *A, long long lda, int n, double *diag, void *stream);
size_t fmlb_krr_refine_dd_scratch_doubles(int n);
int fmlb_krr_refine_dd(const double *A, long long lda, int n, const double *diag,
                       const void *work, const double *y, double *x, double *x_lo, int iters,
                       double *resid, double *scratch, void *stream);

/* FP64 residual and iterative refinement after fmlb_potrf_f64 (the reference
 * solves once, fml/math/fcho_solve.f90:35-42, and leaves the residual to the
 * user). For (K + lambda I) x = y with K full and symmetric (row-major, both
 * triangles; fmlb_symmetrize_lower_f64 mirrors the lower triangle into the
 * upper one) and L / work its factor:
 *   per step: r = y - (K + lambda I) x in FP64, x += solve(L, r);
 *   resid (device, iters + 1 doubles, may be NULL): ||r||_2 before every step
 *   and after the last one (iters = 0 computes the residual only).
 * scratch: fmlb_krr_refine_scratch_doubles(n) device doubles. Deterministic. */
size_t fmlb_krr_refine_scratch_doubles(int n);
int fmlb_symmetrize_lower_f64(double *A, long long lda, int n, void *stream);
int fmlb_krr_refine_f64(const double *K, long long ldk, int n, double lambda, const double *L,
                        long long ldl, const void *work, const double *y, double *x, int iters,
                        double *resid, double *scratch, void *stream);

/* ------------------------------------------------------------------------
 * KRR helpers, FP64.
 * fmlb_add_diagonal_f64: A[i, i] += lambda (the user-side K + lambda I that
 *   precedes cho_solve).
 * fmlb_kernel_predict_f64: y[s, q] = sum_t k_s(Xq[q], Xt[t]) * alpha[s, t] for
 *   every sigma s without storing the kernel matrix; kind 0 = Gaussian,
 *   1 = Laplacian (same kernels as fmlb_gaussian_kernel_f64 /
 *   fmlb_laplacian_kernel_f64). Replaces the user-side prediction
 *   gaussian_kernel(Xq, Xt, sigma) @ alpha (pattern of fget_prediction,
 *   fml/kernels/fkernels.f90:480-539). nsigma <= 8. Deterministic.
 * fmlb_gemv_f64: y[r] = sum_c M[r, c] x[c] (row-major M, leading dimension
 *   ldm); the user-side K_test @ alpha for a test kernel that was stored, e.g.
 *   the ARAD kernel from fmlb_arad_kernels. Deterministic.
 * ---------------------------------------------------------------------- */
int fmlb_gemv_f64(const double *M, long long ldm, int rows, int cols, const double *x, double *y,
                  void *stream);
int fmlb_add_diagonal_f64(double *A, long long lda, int n, double lambda, void *stream);
size_t fmlb_kernel_predict_workspace_bytes(int nq, int nt, int nsigma);
int fmlb_kernel_predict_f64(int kind, const double *Xq, int nq, int ldq, const double *Xt, int nt,
                            int ldt, int d, const double *sigmas_host, int nsigma,
                            const double *alpha, long long lda_alpha, double *y, long long ldy,
                            void *workspace, size_t ws_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Laplacian kernel matrix in FP32 (mixed precision), the FP32 form of
 * flaplacian_kernel (fml/kernels/fkernels.f90:351-377): same arguments as
 * fmlb_laplacian_kernel_f64 with an FP32 output. Descriptors are read in FP64
 * and converted to FP32; the L1 sums are FP32. Relative error against the FP64
 * kernel about 1e-6 * sum|a-b| / sigma.
 * ---------------------------------------------------------------------- */
int fmlb_laplacian_kernel_f32(const double *A, int na, int lda, const double *B, int nb, int ldb,
                              int d, const double *sigmas_host, int nsigma, float *K,
                              long long ldk, long long sigma_stride, int symmetric, void *stream);

/* ------------------------------------------------------------------------
 * Gaussian kernel matrix on the tcgen05 tensor cores (mixed precision).
 * Mixed-precision form of fgaussian_kernel (fml/kernels/fkernels.f90:317-349):
 * K_s[i, j] = exp(-(|x_i|^2 + |x_j|^2 - 2 x_i.x_j) / (2 sigma_s^2)) on
 * descriptors centred by mu, x_i.x_j from BF16 hi/lo splits with three BF16
 * products accumulated in FP32; FP32 output (nsigma, na, nb), stride ldk.
 * Diagonal entries of a symmetric build are exactly 1 and the result is
 * exactly symmetric. Error against the FP64 kernel: about 6e-5 absolute at
 * sigma = 100 on Coulomb matrices of 4..29 atoms (1e-5 relative in d^2 for
 * distinct molecules).
 *   mu        (d,) device, centring vector (fmlb_column_mean_f64 of the set)
 *   workspace fmlb_tc_operand_bytes(na, d) (+ fmlb_tc_operand_bytes(nb, d)
 *             when not symmetric) bytes
 *   status    device int: 0, or 1..3 when a bounded device-side wait gave up
 *             (the result is then incomplete)
 * nsigma <= 8.
 * ---------------------------------------------------------------------- */
size_t fmlb_tc_operand_bytes(int n, int d);
int fmlb_column_mean_f64(const double *X, int n, int ldx, int d, double *mu, void *stream);
int fmlb_gaussian_kernel_tc(const double *A, int na, int lda, const double *B, int nb, int ldb,
                            int d, const double *mu, const double *sigmas_host, int nsigma,
                            float *K, long long ldk, long long sigma_stride, int symmetric,
                            void *workspace, size_t ws_bytes, int *status, void *stream);

/* ------------------------------------------------------------------------
 * Batched KRR: many independent problems of uneven size in ONE persistent
 * launch (the user-side composition of gaussian_kernel, cho_solve and the
 * prediction, fml/kernels/kernels.py:167-196 and fml/math/cho_solve.py:33-58,
 * per problem). `grid` CTAs (<= 0: one per SM) pull problems from a device
 * queue in the order `order` (largest first is best); each CTA runs a whole
 * problem: kernel matrix (Gaussian of descriptor rows, or precomputed),
 * + lambda I, blocked FP64 Cholesky, solve, prediction of its test rows.
 *   problems  device array of nprob records of fmlb_batch_problem_bytes()
 *             bytes (layout in fml_b200/batched.py)
 *   counter   device int (work-queue head; reset by the call)
 *   X (rows, ldx) descriptors, Y targets, pred outputs, buf: per-problem
 *             matrices + workspaces (fmlb_batch_buffer_doubles(n) each)
 *   info      device int per problem: LAPACK-style Cholesky info (0 = ok)
 * ---------------------------------------------------------------------- */
size_t fmlb_batch_problem_bytes(void);
size_t fmlb_batch_buffer_doubles(int n);
int fmlb_krr_batched_f64(const void *problems, const int *order, int nprob, int *counter,
                         const double *X, int ldx, int d, const double *Y, double *pred,
                         double *buf, int *info, int grid, void *stream);

/* Allocation-free form of fmlb_kernel_predict_f64 (same arguments minus the
 * workspace, same results). It has no counterpart in the reference: it exists
 * for callers that cannot allocate device memory on the call path (a server
 * whose device memory is all reserved by its own arena up front, or a host
 * framework that hands the library only input and output buffers). Its
 * scratch is an 8 MiB array inside the library image, held by every GPU that
 * loads the library until the process exits, so
 *   ceil(nt / 1024) * nsigma * nq <= 1048576
 * and larger calls return FMLB_EINVAL. The first call on each device looks up
 * the array's device address (with that device current); make it before any
 * stream capture. All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int fmlb_kernel_predict_f64_noalloc(int kind, const double *Xq, int nq, int ldq, const double *Xt,
                                    int nt, int ldt, int d, const double *sigmas_host, int nsigma,
                                    const double *alpha, long long lda_alpha, double *y,
                                    long long ldy, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FMLB_H */
