// FP64 residual and iterative refinement for the KRR solve
// (K + lambda I) x = y, after the factorisation of fmlb_potrf_f64:
//
//   r = y - (K + lambda I) x        (FP64, K read once, warp per row)
//   ||r||_2                         (fixed-order two-pass reduction)
//   x += (K + lambda I)^-1 r        (fmlb_potrs_f64 with the same factor)
//
// The reference solves once with LAPACK (fml/math/fcho_solve.f90:35-42) and
// leaves the residual to the user; here it is computed on the device and can
// drive refinement steps. fmlb_symmetrize_lower_f64 builds the full matrix
// the residual needs from the triangle the factorisation reads.
#include <math.h>

#include <algorithm>

#include "common.cuh"
#include "dd.cuh"
#include "fmlb.h"

namespace fmlb {
namespace {

constexpr int RF_TPB = 256;
constexpr int RF_PARTS = 1024;  // partial sums of the norm (fixed)

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// r[i] = y[i] - sum_j K[i, j] x[j] - lambda x[i]; warp per row, lanes stride
// the row (coalesced), fixed shuffle tree
__global__ void __launch_bounds__(RF_TPB)
residual_kernel(const double *__restrict__ K, long long ldk, int n, double lambda,
                const double *__restrict__ y, const double *__restrict__ x,
                double *__restrict__ r) {
    const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *k = K + (size_t)row * ldk;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(k[j], x[j], s);
    s = warp_sum_d(s);
    if (lane == 0) r[row] = y[row] - s - lambda * x[row];
}

// part[b] = sum of r[i]^2 over the fixed slice b of the vector
__global__ void __launch_bounds__(RF_TPB)
sumsq_partial_kernel(const double *__restrict__ r, int n, double *__restrict__ part) {
    __shared__ double red[RF_TPB / 32];
    const int per = (n + RF_PARTS - 1) / RF_PARTS;
    const int b = blockIdx.x, i0 = b * per, i1 = min(n, i0 + per);
    double s = 0.0;
    for (int i = i0 + (int)threadIdx.x; i < i1; i += RF_TPB) s = fma(r[i], r[i], s);
    s = warp_sum_d(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < RF_TPB / 32; ++w) t += red[w];
        part[b] = t;
    }
}

__global__ void norm_final_kernel(const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double red[RF_TPB / 32];
    double s = 0.0;
    for (int b = threadIdx.x; b < RF_PARTS; b += RF_TPB) s += part[b];
    s = warp_sum_d(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < RF_TPB / 32; ++w) t += red[w];
        *out = sqrt(t);
    }
}

__global__ void axpy_kernel(double *__restrict__ x, const double *__restrict__ d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += d[i];
}

// A[j, i] = A[i, j] for j < i: the upper triangle from the lower one
__global__ void symmetrize_kernel(double *__restrict__ A, long long lda, int n) {
    const int i = blockIdx.y * 32 + threadIdx.y, j = blockIdx.x * 32 + threadIdx.x;
    if (i < n && j < i) A[(size_t)j * lda + i] = A[(size_t)i * lda + j];
}

// ---- double-double residual from the upper triangle ---------------------------
// After an in-place factorisation of A = K + lambda I (factor in the lower
// triangle) the strict upper triangle still holds K; the diagonal was saved.
// r = y - A x with x = x_hi + x_lo, in double-double:
//   row pass     s_row[i] = sum_{j > i} A[i, j] x_j      (warp per row)
//   column pass  s_col[c][j] = sum_{i in chunk c, i < j} A[i, j] x_i
//                (thread per column, rows in chunks of DD_CHUNK)
//   combine      r_i = y_i - s_row[i] - sum_c s_col[c][i] - diag_i x_i
// every sum in a fixed order (deterministic).
constexpr int DD_CHUNK = 1024;
constexpr int DD_COLS = 256;

__device__ __forceinline__ dd warp_sum_dd(dd v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        dd w;
        w.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
        w.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
        v = dd_add(v, w);
    }
    return v;
}

__global__ void __launch_bounds__(RF_TPB)
upper_rows_dd_kernel(const double *__restrict__ A, long long lda, int n,
                     const double *__restrict__ xh, const double *__restrict__ xl,
                     double *__restrict__ srow) {
    const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *a = A + (size_t)row * lda;
    dd s0{0.0, 0.0}, s1{0.0, 0.0};
    int j = row + 1 + lane;
    for (; j + 32 < n; j += 64) {
        s0 = dd_add(s0, dd_mul_d(dd{xh[j], xl[j]}, a[j]));
        s1 = dd_add(s1, dd_mul_d(dd{xh[j + 32], xl[j + 32]}, a[j + 32]));
    }
    if (j < n) s0 = dd_add(s0, dd_mul_d(dd{xh[j], xl[j]}, a[j]));
    dd s = warp_sum_dd(dd_add(s0, s1));
    if (lane == 0) {
        srow[2 * (size_t)row] = s.hi;
        srow[2 * (size_t)row + 1] = s.lo;
    }
}

__global__ void __launch_bounds__(DD_COLS)
upper_cols_dd_kernel(const double *__restrict__ A, long long lda, int n,
                     const double *__restrict__ xh, const double *__restrict__ xl,
                     double *__restrict__ scol) {
    const int j = blockIdx.x * DD_COLS + threadIdx.x;
    const int c = blockIdx.y;
    const int i0 = c * DD_CHUNK;
    if (i0 >= (int)(blockIdx.x * DD_COLS + DD_COLS) || j >= n || i0 >= j) return;
    const int i1 = min(i0 + DD_CHUNK, j);
    dd s0{0.0, 0.0}, s1{0.0, 0.0};
    int i = i0;
    for (; i + 1 < i1; i += 2) {
        s0 = dd_add(s0, dd_mul_d(dd{xh[i], xl[i]}, A[(size_t)i * lda + j]));
        s1 = dd_add(s1, dd_mul_d(dd{xh[i + 1], xl[i + 1]}, A[(size_t)(i + 1) * lda + j]));
    }
    if (i < i1) s0 = dd_add(s0, dd_mul_d(dd{xh[i], xl[i]}, A[(size_t)i * lda + j]));
    const dd s = dd_add(s0, s1);
    scol[2 * ((size_t)c * n + j)] = s.hi;
    scol[2 * ((size_t)c * n + j) + 1] = s.lo;
}

__global__ void combine_residual_dd_kernel(int n, const double *__restrict__ y,
                                           const double *__restrict__ diag,
                                           const double *__restrict__ xh,
                                           const double *__restrict__ xl,
                                           const double *__restrict__ srow,
                                           const double *__restrict__ scol,
                                           double *__restrict__ r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dd acc{srow[2 * (size_t)i], srow[2 * (size_t)i + 1]};
    const int nc = i > 0 ? (i - 1) / DD_CHUNK + 1 : 0;  // chunks holding rows < i
    for (int c = 0; c < nc; ++c)
        acc = dd_add(acc, dd{scol[2 * ((size_t)c * n + i)], scol[2 * ((size_t)c * n + i) + 1]});
    acc = dd_add(acc, dd_mul_d(dd{xh[i], xl[i]}, diag[i]));
    const dd res = dd_add_d(dd_neg(acc), y[i]);
    r[i] = res.hi + res.lo;
}

// x_hi + x_lo += d in double-double
__global__ void dd_axpy_kernel(double *__restrict__ xh, double *__restrict__ xl,
                               const double *__restrict__ d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const dd v = dd_add_d(dd{xh[i], xl[i]}, d[i]);
    xh[i] = v.hi;
    xl[i] = v.lo;
}

__global__ void get_diagonal_kernel(const double *__restrict__ A, long long lda, int n,
                                    double *__restrict__ diag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) diag[i] = A[(size_t)i * lda + i];
}

int residual_norm_dd(const double *A, long long lda, int n, const double *diag, const double *y,
                     const double *xh, const double *xl, double *r, double *part, double *srow,
                     double *scol, double *out, cudaStream_t st) {
    upper_rows_dd_kernel<<<ceil_div((long)n * 32, RF_TPB), RF_TPB, 0, st>>>(A, lda, n, xh, xl,
                                                                           srow);
    FMLB_TRY(launch_status("upper_rows_dd_kernel"));
    const dim3 grid(ceil_div(n, DD_COLS), ceil_div(n, DD_CHUNK));
    upper_cols_dd_kernel<<<grid, DD_COLS, 0, st>>>(A, lda, n, xh, xl, scol);
    FMLB_TRY(launch_status("upper_cols_dd_kernel"));
    combine_residual_dd_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, y, diag, xh, xl, srow, scol,
                                                                 r);
    FMLB_TRY(launch_status("combine_residual_dd_kernel"));
    if (out) {
        sumsq_partial_kernel<<<RF_PARTS, RF_TPB, 0, st>>>(r, n, part);
        FMLB_TRY(launch_status("sumsq_partial_kernel"));
        norm_final_kernel<<<1, RF_TPB, 0, st>>>(part, out);
        FMLB_TRY(launch_status("norm_final_kernel"));
    }
    return FMLB_OK;
}

int residual_norm(const double *K, long long ldk, int n, double lambda, const double *y,
                  const double *x, double *r, double *part, double *out, cudaStream_t st) {
    residual_kernel<<<ceil_div((long)n * 32, RF_TPB), RF_TPB, 0, st>>>(K, ldk, n, lambda, y, x,
                                                                      r);
    FMLB_TRY(launch_status("residual_kernel"));
    if (out) {
        sumsq_partial_kernel<<<RF_PARTS, RF_TPB, 0, st>>>(r, n, part);
        FMLB_TRY(launch_status("sumsq_partial_kernel"));
        norm_final_kernel<<<1, RF_TPB, 0, st>>>(part, out);
        FMLB_TRY(launch_status("norm_final_kernel"));
    }
    return FMLB_OK;
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_krr_refine_scratch_doubles(int n) {
    return (size_t)std::max(n, 0) + fmlb::RF_PARTS;
}

extern "C" int fmlb_symmetrize_lower_f64(double *A, long long lda, int n, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_symmetrize_lower_f64: bad sizes");
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A, "fmlb_symmetrize_lower_f64: null pointer");
    const dim3 grid(ceil_div(n, 32), ceil_div(n, 32)), block(32, 32);
    symmetrize_kernel<<<grid, block, 0, FMLB_STREAM(stream)>>>(A, lda, n);
    return launch_status("symmetrize_kernel");
}

extern "C" int fmlb_krr_refine_f64(const double *K, long long ldk, int n, double lambda,
                                   const double *L, long long ldl, const void *work,
                                   const double *y, double *x, int iters, double *resid,
                                   double *scratch, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && ldk >= n && ldl >= n && iters >= 0,
                 "fmlb_krr_refine_f64: bad sizes");
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(K && L && work && y && x && scratch, "fmlb_krr_refine_f64: null pointer");
    double *r = scratch, *part = scratch + n;
    for (int it = 0; it < iters; ++it) {
        FMLB_TRY(residual_norm(K, ldk, n, lambda, y, x, r, part, resid ? resid + it : nullptr,
                               st));
        FMLB_TRY(fmlb_potrs_f64(L, ldl, n, work, r, st));
        axpy_kernel<<<ceil_div(n, 256), 256, 0, st>>>(x, r, n);
        FMLB_TRY(launch_status("axpy_kernel"));
    }
    if (resid)
        FMLB_TRY(residual_norm(K, ldk, n, lambda, y, x, r, part, resid + iters, st));
    return FMLB_OK;
}

extern "C" int fmlb_get_diagonal_f64(const double *A, long long lda, int n, double *diag,
                                     void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_get_diagonal_f64: bad sizes");
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A && diag, "fmlb_get_diagonal_f64: null pointer");
    get_diagonal_kernel<<<ceil_div(n, 256), 256, 0, FMLB_STREAM(stream)>>>(A, lda, n, diag);
    return launch_status("get_diagonal_kernel");
}

extern "C" size_t fmlb_krr_refine_dd_scratch_doubles(int n) {
    if (n <= 0) return fmlb::RF_PARTS;
    const size_t nc = (size_t)(n + fmlb::DD_CHUNK - 1) / fmlb::DD_CHUNK;
    return (size_t)n + fmlb::RF_PARTS + 2 * (size_t)n + 2 * nc * n;
}

extern "C" int fmlb_krr_refine_dd(const double *A, long long lda, int n, const double *diag,
                                  const void *work, const double *y, double *x, double *x_lo,
                                  int iters, double *resid, double *scratch, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && lda >= n && iters >= 0, "fmlb_krr_refine_dd: bad sizes");
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A && diag && work && y && x && x_lo && scratch,
                 "fmlb_krr_refine_dd: null pointer");
    double *r = scratch, *part = r + n, *srow = part + RF_PARTS, *scol = srow + 2 * (size_t)n;
    for (int it = 0; it < iters; ++it) {
        FMLB_TRY(residual_norm_dd(A, lda, n, diag, y, x, x_lo, r, part, srow, scol,
                                  resid ? resid + it : nullptr, st));
        FMLB_TRY(fmlb_potrs_f64(A, lda, n, work, r, st));
        dd_axpy_kernel<<<ceil_div(n, 256), 256, 0, st>>>(x, x_lo, r, n);
        FMLB_TRY(launch_status("dd_axpy_kernel"));
    }
    if (resid)
        FMLB_TRY(residual_norm_dd(A, lda, n, diag, y, x, x_lo, r, part, srow, scol,
                                  resid + iters, st));
    return FMLB_OK;
}
