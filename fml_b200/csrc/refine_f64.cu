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
