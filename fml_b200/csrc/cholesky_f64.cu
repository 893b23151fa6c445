// Plain-FP64 blocked right-looking Cholesky factorisation and solve, the
// replacement for LAPACK dpotrf('U') / dpotrs('U') as fcho_solve calls them
// (fml/math/fcho_solve.f90:35-42).
//
// Storage: row-major (n, n), factor L in the triangle i >= j (A = L L^T); the
// other triangle is never read or written. For the reference's C-order
// argument this is its dpotrf('U') factor U = L^T.
//
// Per panel of NB columns:
//   1. potf2 + inversion of the diagonal block in shared memory (one CTA); a
//      non-positive pivot records the LAPACK info (1-based column) and every
//      later kernel returns early;
//   2. panel solve L21 = A21 L11^-T as a product with the stored inverse;
//   3. trailing update A22 -= L21 L21^T over the tiles on or below the diagonal.
// The inverted diagonal blocks are kept in the workspace for the solve.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int NB = 64;    // panel width
constexpr int TPB = 256;

__device__ __forceinline__ bool failed(const int *info) { return *(volatile const int *)info != 0; }

// ---- 1. diagonal block ----------------------------------------------------
__global__ void __launch_bounds__(TPB)
potf2_block_kernel(double *__restrict__ A, long long lda, int k0, int kn,
                   double *__restrict__ Linv, int *__restrict__ info) {
    __shared__ double L[NB][NB + 1];
    __shared__ double tmp[NB];
    __shared__ int bad;
    if (failed(info)) return;
    const int tid = threadIdx.x;
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        double v = 0.0;
        if (r < kn && c <= r) v = A[(size_t)(k0 + r) * lda + (k0 + c)];
        else if (r == c) v = 1.0;  // identity padding past kn keeps the block SPD
        L[r][c] = v;
    }
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < NB; ++j) {
        if (tid == 0) {
            const double d = L[j][j];
            if (!(d > 0.0)) bad = j + 1;
            else L[j][j] = sqrt(d);
        }
        __syncthreads();
        if (bad) break;
        const double djj = L[j][j];
        for (int i = j + 1 + tid; i < NB; i += TPB) L[i][j] /= djj;
        __syncthreads();
        // trailing update of the block: L[i][c] -= L[i][j] * L[c][j], j < c <= i
        const int m = NB - j - 1;
        for (int t = tid; t < m * m; t += TPB) {
            const int i = j + 1 + t / m, c = j + 1 + t % m;
            if (c <= i) L[i][c] = fma(-L[i][j], L[c][j], L[i][c]);
        }
        __syncthreads();
    }
    if (bad) {
        if (tid == 0) atomicCAS(info, 0, k0 + bad);
        return;
    }
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        if (r < kn && c <= r) A[(size_t)(k0 + r) * lda + (k0 + c)] = L[r][c];
    }
    __syncthreads();
    // in-place inverse of the lower-triangular block, last column first:
    // column j of inv(L) is -inv(L22) l / l_jj with inv(L22) already in place
    for (int j = NB - 1; j >= 0; --j) {
        if (tid == 0) L[j][j] = 1.0 / L[j][j];
        __syncthreads();
        const int i = j + 1 + tid;
        if (i < NB) {
            double s = 0.0;
            for (int k = j + 1; k <= i; ++k) s = fma(L[i][k], L[k][j], s);
            tmp[i] = s;
        }
        __syncthreads();
        if (i < NB) L[i][j] = -L[j][j] * tmp[i];
        __syncthreads();
    }
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        Linv[t] = (c <= r) ? L[r][c] : 0.0;
    }
}

// ---- 2. panel solve: rows [r0, n) of columns [k0, k0+kn): X <- X Linv^T ----
__global__ void __launch_bounds__(TPB)
panel_trsm_kernel(double *__restrict__ A, long long lda, int n, int k0, int kn,
                  const double *__restrict__ Linv, const int *__restrict__ info) {
    extern __shared__ double trsm_smem[];
    double(*Li)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(trsm_smem);
    double(*P)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(trsm_smem + NB * (NB + 1));
    if (failed(info)) return;
    const int r0 = k0 + kn + blockIdx.x * NB;
    const int tid = threadIdx.x;
    for (int t = tid; t < NB * NB; t += TPB) Li[t / NB][t % NB] = Linv[t];
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        P[r][c] = (r0 + r < n && c < kn) ? A[(size_t)(r0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    // out[r][c] = sum_{k <= c} P[r][k] * Linv[c][k]
    const int c = tid & 63, rq = tid >> 6;  // 4 row groups of 16 rows
    double out[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) out[i] = 0.0;
    for (int k = 0; k <= c; ++k) {
        const double l = Li[c][k];
#pragma unroll
        for (int i = 0; i < 16; ++i) out[i] = fma(P[rq * 16 + i][k], l, out[i]);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int r = r0 + rq * 16 + i;
        if (r < n && c < kn) A[(size_t)r * lda + k0 + c] = out[i];
    }
}

constexpr size_t kTrsmSmem = 2 * NB * (NB + 1) * sizeof(double);

// ---- 3. trailing update: C -= L21 L21^T on tiles at or below the diagonal ----
// 128x128 tile per CTA, 8x8 outputs per thread, k-chunks of 16.
constexpr int TM = 128, TK = 16;
__global__ void __launch_bounds__(TPB)
syrk_update_kernel(double *__restrict__ A, long long lda, int n, int k0, int kn,
                   const int *__restrict__ info) {
    __shared__ double As[TK][TM + 2];
    __shared__ double Bs[TK][TM + 2];
    if (failed(info)) return;
    const long long t = blockIdx.x;
    int by = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)by * (by + 1) / 2 > t) --by;
    while ((long long)(by + 1) * (by + 2) / 2 <= t) ++by;
    const int bx = (int)(t - (long long)by * (by + 1) / 2);
    const int base = k0 + kn;
    const int row0 = base + by * TM, col0 = base + bx * TM;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;

    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

    const int lk = threadIdx.x & 15, lr = threadIdx.x >> 4;
    for (int kk0 = 0; kk0 < kn; kk0 += TK) {
        const int k = k0 + kk0 + lk;
        const bool kin = kk0 + lk < kn;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int ra = row0 + lr + 16 * r, rb = col0 + lr + 16 * r;
            As[lk][lr + 16 * r] = (ra < n && kin) ? A[(size_t)ra * lda + k] : 0.0;
            Bs[lk][lr + 16 * r] = (rb < n && kin) ? A[(size_t)rb * lda + k] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            double a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = row0 + ty + 16 * i;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = col0 + tx + 16 * j;
            if (r < n && c <= r) {
                double *p = A + (size_t)r * lda + c;
                *p -= acc[i][j];
            }
        }
    }
}

// ---- solve ------------------------------------------------------------------
// forward step: y_k = Linv_k * x_k; x_j -= L[j, k-block] y_k for rows j after the block
constexpr int SOLVE_ROWS = 256;
__global__ void __launch_bounds__(TPB)
forward_step_kernel(const double *__restrict__ L, long long lda, int n, int k0, int kn,
                    const double *__restrict__ Linv, double *__restrict__ x,
                    double *__restrict__ y) {
    __shared__ double yk[NB];
    const int tid = threadIdx.x;
    if (tid < NB) {
        double s = 0.0;
        if (tid < kn)
            for (int c = 0; c <= tid; ++c) s = fma(Linv[tid * NB + c], x[k0 + c], s);
        yk[tid] = s;
    }
    __syncthreads();
    if (blockIdx.x == 0 && tid < kn) y[k0 + tid] = yk[tid];
    const int r = k0 + kn + blockIdx.x * SOLVE_ROWS + tid;
    if (r < n) {
        const double *row = L + (size_t)r * lda + k0;
        double s = 0.0;
        for (int c = 0; c < kn; ++c) s = fma(row[c], yk[c], s);
        x[r] -= s;
    }
}

// backward step: x_k = Linv_k^T y_k; y_j -= sum_r L[k0+r, j] x_k[r] for j < k0
__global__ void __launch_bounds__(TPB)
backward_step_kernel(const double *__restrict__ L, long long lda, int n, int k0, int kn,
                     const double *__restrict__ Linv, double *__restrict__ y,
                     double *__restrict__ x) {
    __shared__ double xk[NB];
    const int tid = threadIdx.x;
    if (tid < NB) {
        double s = 0.0;
        if (tid < kn)
            for (int r = tid; r < kn; ++r) s = fma(Linv[r * NB + tid], y[k0 + r], s);
        xk[tid] = s;
    }
    __syncthreads();
    if (blockIdx.x == 0 && tid < kn) x[k0 + tid] = xk[tid];
    const int j = blockIdx.x * SOLVE_ROWS + tid;
    if (j < k0) {
        double s = 0.0;
        for (int r = 0; r < kn; ++r) s = fma(L[(size_t)(k0 + r) * lda + j], xk[r], s);
        y[j] -= s;
    }
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_potrf_workspace_bytes(int n) {
    if (n <= 0) return 256;
    const size_t nblk = (size_t)(n + fmlb::NB - 1) / fmlb::NB;
    return nblk * fmlb::NB * fmlb::NB * sizeof(double) + ((size_t)n * sizeof(double) + 255) / 256 * 256;
}

extern "C" int fmlb_potrf_f64(double *A, long long lda, int n, void *work, int *info,
                              void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_potrf_f64: bad n=%d / lda=%lld", n, lda);
    FMLB_REQUIRE(info, "fmlb_potrf_f64: info pointer is null");
    FMLB_TRY(cuda_status(cudaMemsetAsync(info, 0, sizeof(int), st), "fmlb_potrf_f64: clear info"));
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A && work, "fmlb_potrf_f64: null pointer");
    double *Linv = static_cast<double *>(work);
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(panel_trsm_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kTrsmSmem),
                         "fmlb_potrf_f64: shared memory attribute"));
    for (int k0 = 0, kb = 0; k0 < n; k0 += NB, ++kb) {
        const int kn = std::min(NB, n - k0);
        double *Li = Linv + (size_t)kb * NB * NB;
        potf2_block_kernel<<<1, TPB, 0, st>>>(A, lda, k0, kn, Li, info);
        FMLB_TRY(launch_status("potf2_block_kernel"));
        const int rest = n - k0 - kn;
        if (rest <= 0) break;
        panel_trsm_kernel<<<ceil_div(rest, NB), TPB, kTrsmSmem, st>>>(A, lda, n, k0, kn, Li, info);
        FMLB_TRY(launch_status("panel_trsm_kernel"));
        const long long T = ceil_div(rest, TM);
        syrk_update_kernel<<<(unsigned)(T * (T + 1) / 2), TPB, 0, st>>>(A, lda, n, k0, kn, info);
        FMLB_TRY(launch_status("syrk_update_kernel"));
    }
    return FMLB_OK;
}

extern "C" int fmlb_potrs_f64(const double *L, long long lda, int n, const void *work, double *x,
                              void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_potrs_f64: bad n=%d / lda=%lld", n, lda);
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(L && work && x, "fmlb_potrs_f64: null pointer");
    const double *Linv = static_cast<const double *>(work);
    const size_t nblk = (size_t)(n + NB - 1) / NB;
    // y lives after the inverted blocks in the workspace (written by potrs only)
    double *y = const_cast<double *>(Linv + nblk * NB * NB);
    for (int k0 = 0, kb = 0; k0 < n; k0 += NB, ++kb) {
        const int kn = std::min(NB, n - k0);
        const int rest = n - k0 - kn;
        const int grid = std::max(1, ceil_div(rest, SOLVE_ROWS));
        forward_step_kernel<<<grid, TPB, 0, st>>>(L, lda, n, k0, kn, Linv + (size_t)kb * NB * NB,
                                                  x, y);
        FMLB_TRY(launch_status("forward_step_kernel"));
    }
    for (int kb = (int)nblk - 1; kb >= 0; --kb) {
        const int k0 = kb * NB, kn = std::min(NB, n - k0);
        const int grid = std::max(1, ceil_div(k0, SOLVE_ROWS));
        backward_step_kernel<<<grid, TPB, 0, st>>>(L, lda, n, k0, kn, Linv + (size_t)kb * NB * NB,
                                                   y, x);
        FMLB_TRY(launch_status("backward_step_kernel"));
    }
    return FMLB_OK;
}
