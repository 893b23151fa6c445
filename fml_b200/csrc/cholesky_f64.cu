// Plain-FP64 blocked right-looking Cholesky factorisation and solve, the
// replacement for LAPACK dpotrf('U') / dpotrs('U') as fcho_solve calls them
// (fml/math/fcho_solve.f90:35-42).
//
// Storage: row-major (n, n), factor L in the triangle i >= j (A = L L^T); the
// other triangle is never read or written. For the reference's C-order
// argument this is its dpotrf('U') factor U = L^T.
//
// Per panel of NB = 128 columns:
//   1. potf2 + in-place inversion of the diagonal block in shared memory (one
//      CTA); a non-positive pivot records the LAPACK info (1-based column) and
//      every later kernel of the factorisation returns at once;
//   2. panel solve L21 = A21 L11^-T as a product with the stored inverse;
//   3. trailing update A22 -= L21 L21^T on the FP64 tensor cores
//      (mma.sync m8n8k4 f64), 128x128 tiles on or below the diagonal, operands
//      streamed through a 3-stage cp.async pipeline.
// The inverted diagonal blocks stay in the workspace for the solve.
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int NB = 128;  // panel width
constexpr int TPB = 256;

__device__ __forceinline__ bool failed(const int *info) {
    return info && *(volatile const int *)info != 0;
}

// ---- 1. diagonal block ----------------------------------------------------
// The 128 x 128 block is factored in four 32-column steps. In step J one warp
// factors (and inverts) the 32 x 32 diagonal sub-block in registers with warp
// shuffles only; the whole CTA then solves the 32-column sub-panel below it
// and updates the rest of the block. The block inverse is assembled from the
// sub-block inverses: inv(L)_IJ = -inv(L_II) sum_{K=J}^{I-1} L_IK inv(L)_KJ,
// with the off-diagonal blocks kept (transposed) in the unused upper triangle.
constexpr int LDL = NB + 1;
constexpr int SB = 32, NSB = NB / SB, LDW = SB + 1;
constexpr size_t kPotf2Smem = ((size_t)NB * LDL + (size_t)NSB * SB * LDW + SB * LDW) *
                              sizeof(double);

// lane i holds row i of the sub-block in d[0..31]; on return d holds the
// factor row and x holds column `lane` of the inverse. Returns the 1-based
// failing column or 0.
__device__ __forceinline__ int warp_potrf_inv32(double (&d)[SB], double (&x)[SB]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < SB; ++j) {
        const double piv = __shfl_sync(full, d[j], j);
        if (!(piv > 0.0)) return j + 1;
        const double r = sqrt(piv), inv = 1.0 / r;
        d[j] = (lane == j) ? r : (lane > j ? d[j] * inv : d[j]);
#pragma unroll
        for (int c = j + 1; c < SB; ++c) {
            const double dcj = __shfl_sync(full, d[j], c);
            if (lane >= c) d[c] = fma(-d[j], dcj, d[c]);
        }
    }
    // column `lane` of the inverse by forward substitution
#pragma unroll
    for (int k = 0; k < SB; ++k) {
        double s = (k == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int q = 0; q < k; ++q) s = fma(-__shfl_sync(full, d[q], k), x[q], s);
        x[k] = s / __shfl_sync(full, d[k], k);
    }
    return 0;
}

__global__ void __launch_bounds__(TPB)
potf2_block_kernel(double *__restrict__ A, long long lda, int k0, int kn,
                   double *__restrict__ Linv, int *__restrict__ info) {
    extern __shared__ double potf2_smem[];
    double(*L)[LDL] = reinterpret_cast<double(*)[LDL]>(potf2_smem);
    double(*W)[SB][LDW] = reinterpret_cast<double(*)[SB][LDW]>(potf2_smem + NB * LDL);
    double(*T)[LDW] = reinterpret_cast<double(*)[LDW]>(potf2_smem + NB * LDL + NSB * SB * LDW);
    __shared__ int bad;
    if (failed(info)) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t >> 7, c = t & (NB - 1);
        double v = 0.0;
        if (r < kn && c <= r) v = A[(size_t)(k0 + r) * lda + (k0 + c)];
        else if (r == c) v = 1.0;  // identity padding past kn keeps the block SPD
        L[r][c] = v;
    }
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int J = 0; J < NSB; ++J) {
        const int b0 = J * SB;
        if (warp == 0) {
            double d[SB], x[SB];
#pragma unroll
            for (int c = 0; c < SB; ++c) d[c] = L[b0 + lane][b0 + c];
            const int f = warp_potrf_inv32(d, x);
            if (f) {
                if (lane == 0) bad = b0 + f;
            } else {
#pragma unroll
                for (int c = 0; c < SB; ++c) {
                    if (c <= lane) L[b0 + lane][b0 + c] = d[c];
                    W[J][c][lane] = x[c];  // inverse: row c, column lane
                }
            }
        }
        __syncthreads();
        if (bad) {
            if (tid == 0) atomicCAS(info, 0, k0 + bad);
            return;
        }
        const int r0 = b0 + SB;
        // sub-panel solve: L[r][b0..b0+31] <- L[r][b0..] inv(D)^T, one row per thread
        for (int r = r0 + tid; r < NB; r += TPB) {
            double a[SB];
#pragma unroll
            for (int k = 0; k < SB; ++k) a[k] = L[r][b0 + k];
#pragma unroll
            for (int c = 0; c < SB; ++c) {
                double sacc = 0.0;
#pragma unroll
                for (int k = 0; k <= c; ++k) sacc = fma(a[k], W[J][c][k], sacc);
                L[r][b0 + c] = sacc;
            }
        }
        __syncthreads();
        // update of the rest of the block: L[r][c] -= sum_k X[r][k] X[c][k], r0 <= c <= r
        for (int r = r0 + (tid >> 4); r < NB; r += TPB / 16) {
            for (int c = r0 + (tid & 15); c <= r; c += 16) {
                double sacc = 0.0;
#pragma unroll 8
                for (int k = 0; k < SB; ++k) sacc = fma(L[r][b0 + k], L[c][b0 + k], sacc);
                L[r][c] -= sacc;
            }
        }
        __syncthreads();
    }
    // factor back to global
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t >> 7, c = t & (NB - 1);
        if (r < kn && c <= r) A[(size_t)(k0 + r) * lda + (k0 + c)] = L[r][c];
    }
    // block inverse; inv(L)_IJ for I > J is stored transposed at L[b0J + c][b0I + r]
    for (int I = 1; I < NSB; ++I) {
        for (int J = 0; J < I; ++J) {
            // T = sum_{K=J}^{I-1} L_IK inv(L)_KJ
            for (int t = tid; t < SB * SB; t += TPB) {
                const int r = t >> 5, c = t & 31;
                double sacc = 0.0;
                for (int K = J; K < I; ++K) {
                    for (int q = 0; q < SB; ++q) {
                        const double lik = L[I * SB + r][K * SB + q];
                        const double inv = (K == J) ? W[J][q][c] : L[J * SB + c][K * SB + q];
                        sacc = fma(lik, inv, sacc);
                    }
                }
                T[r][c] = sacc;
            }
            __syncthreads();
            for (int t = tid; t < SB * SB; t += TPB) {
                const int r = t >> 5, c = t & 31;
                double sacc = 0.0;
                for (int q = 0; q <= r; ++q) sacc = fma(W[I][r][q], T[q][c], sacc);
                L[J * SB + c][I * SB + r] = -sacc;
            }
            __syncthreads();
        }
    }
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t >> 7, c = t & (NB - 1);
        const int I = r / SB, J = c / SB;
        double v = 0.0;
        if (I == J) v = (c <= r) ? W[I][r - I * SB][c - J * SB] : 0.0;
        else if (I > J) v = L[c][r];
        Linv[t] = v;
    }
}

// ---- 2. panel solve: rows [r0, n) of columns [k0, k0+kn): X <- X Linv^T ----
constexpr int TRSM_ROWS = 64;
constexpr size_t kTrsmSmem = (size_t)(NB + TRSM_ROWS) * LDL * sizeof(double);

__global__ void __launch_bounds__(TPB)
panel_trsm_kernel(double *__restrict__ A, long long lda, int n, int k0, int kn,
                  const double *__restrict__ Linv, const int *__restrict__ info) {
    extern __shared__ double trsm_smem[];
    double(*Li)[LDL] = reinterpret_cast<double(*)[LDL]>(trsm_smem);
    double(*P)[LDL] = reinterpret_cast<double(*)[LDL]>(trsm_smem + NB * LDL);
    if (failed(info)) return;
    const int r0 = k0 + kn + blockIdx.x * TRSM_ROWS;
    const int tid = threadIdx.x;
    for (int t = tid; t < NB * NB; t += TPB) Li[t / NB][t % NB] = Linv[t];
    for (int t = tid; t < TRSM_ROWS * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        P[r][c] = (r0 + r < n && c < kn) ? A[(size_t)(r0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    // out[r][c] = sum_{k <= c} P[r][k] * Linv[c][k]
    const int c = tid & (NB - 1), rq = tid / NB;  // 2 row groups of 32 rows
    double out[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) out[i] = 0.0;
    for (int k = 0; k <= c; ++k) {
        const double l = Li[c][k];
#pragma unroll
        for (int i = 0; i < 32; ++i) out[i] = fma(P[rq * 32 + i][k], l, out[i]);
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int r = r0 + rq * 32 + i;
        if (r < n && c < kn) A[(size_t)r * lda + k0 + c] = out[i];
    }
}

// ---- 3. trailing update on the FP64 tensor cores ---------------------------
// C (m x m, stride ldc) -= P P^T on the triangle c <= r, P is (m x k).
// CTA tile 128 rows x 64 columns, 4 warps as 2 x 2, warp tile 64x32 =
// 8 x 4 m8n8 fragments; two CTAs fit per SM so one CTA's prologue and
// read-modify-write epilogue overlap the other's tensor-core work.
constexpr int SY_TM = 128, SY_TN = 64, SY_TK = 16, SY_LD = 20, SY_STAGES = 3, SY_TPB = 128;
constexpr int SY_STAGE_DOUBLES = (SY_TM + SY_TN) * SY_LD;
constexpr size_t kSyrkSmem = (size_t)SY_STAGES * SY_STAGE_DOUBLES * sizeof(double);

__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Loads rows [row0, row0+ROWS) x k-columns [kc0, kc0+16) of P into a ROWS x
// SY_LD stage buffer; out-of-range rows / columns are zero-filled.
template <int ROWS, bool kAligned16>
__device__ __forceinline__ void syrk_load_tile(double *dst, const double *__restrict__ P,
                                               long long ldp, int m, int k, int row0, int kc0) {
    const int tid = threadIdx.x;
    if (kAligned16) {
#pragma unroll
        for (int i = 0; i < (ROWS * SY_TK / 2) / SY_TPB; ++i) {
            const int c = tid + i * SY_TPB;
            const int r = c >> 3, kc = (c & 7) * 2;
            const int gr = row0 + r, gk = kc0 + kc;
            int bytes = 0;
            if (gr < m) bytes = min(max(k - gk, 0), 2) * 8;
            const double *src = bytes ? P + (size_t)gr * ldp + gk : P;
            cp_async_16(dst + r * SY_LD + kc, src, bytes);
        }
    } else {
#pragma unroll
        for (int i = 0; i < (ROWS * SY_TK) / SY_TPB; ++i) {
            const int c = tid + i * SY_TPB;
            const int r = c >> 4, kc = c & 15;
            const int gr = row0 + r, gk = kc0 + kc;
            const bool ok = gr < m && gk < k;
            cp_async_8(dst + r * SY_LD + kc, ok ? P + (size_t)gr * ldp + gk : P, ok ? 8 : 0);
        }
    }
}

template <bool kAligned16>
__global__ void __launch_bounds__(SY_TPB, 2)
syrk_dmma_kernel(double *__restrict__ C, long long ldc, int m, const double *__restrict__ P,
                 long long ldp, int k, const int *__restrict__ info) {
    extern __shared__ __align__(16) double sy_smem[];
    if (failed(info)) return;
    // tile t -> (row block by of 128, column block bx of 64), bx <= 2 by + 1
    const long long t = blockIdx.x;
    int by = (int)((sqrt(4.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)by * by + by > t) --by;
    while ((long long)(by + 1) * (by + 1) + (by + 1) <= t) ++by;
    const int bx = (int)(t - (long long)by * by - by);
    const int row0 = by * SY_TM, col0 = bx * SY_TN;
    if (col0 >= m || row0 >= m) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wr = warp >> 1, wc = warp & 1;
    const int g = lane >> 2, tq = lane & 3;

    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (k + SY_TK - 1) / SY_TK;
#pragma unroll
    for (int s = 0; s < SY_STAGES - 1; ++s) {
        if (s < nk) {
            double *st = sy_smem + s * SY_STAGE_DOUBLES;
            syrk_load_tile<SY_TM, kAligned16>(st, P, ldp, m, k, row0, s * SY_TK);
            syrk_load_tile<SY_TN, kAligned16>(st + SY_TM * SY_LD, P, ldp, m, k, col0, s * SY_TK);
        }
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<SY_STAGES - 2>();
        __syncthreads();
        const int nxt = kt + SY_STAGES - 1;
        if (nxt < nk) {
            double *st = sy_smem + (nxt % SY_STAGES) * SY_STAGE_DOUBLES;
            syrk_load_tile<SY_TM, kAligned16>(st, P, ldp, m, k, row0, nxt * SY_TK);
            syrk_load_tile<SY_TN, kAligned16>(st + SY_TM * SY_LD, P, ldp, m, k, col0, nxt * SY_TK);
        }
        cp_async_commit();
        const double *As = sy_smem + (kt % SY_STAGES) * SY_STAGE_DOUBLES;
        const double *Bs = As + SY_TM * SY_LD;
#pragma unroll
        for (int kk = 0; kk < SY_TK / 4; ++kk) {
            double a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[(wr * 64 + i * 8 + g) * SY_LD + kk * 4 + tq];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(wc * 32 + j * 8 + g) * SY_LD + kk * 4 + tq];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], a[i], b[j]);
        }
    }
    cp_async_wait<0>();
    // fragment (i, j): rows wr*64 + i*8 + g, columns wc*32 + j*8 + 2*tq + {0, 1}
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = row0 + wr * 64 + i * 8 + g;
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + wc * 32 + j * 8 + 2 * tq;
            double *p = C + (size_t)r * ldc + c;
            if (c <= r) p[0] -= acc[i][j][0];
            if (c + 1 <= r) p[1] -= acc[i][j][1];
        }
    }
}

template <bool kAligned16>
int launch_syrk_impl(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                     const int *info, cudaStream_t st) {
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "syrk: cudaGetDevice"));
    if (attr_dev != dev) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(syrk_dmma_kernel<kAligned16>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kSyrkSmem), "syrk smem attribute"));
        attr_dev = dev;
    }
    const long long Tr = ceil_div(m, SY_TM);
    const long long ntiles = Tr * Tr + Tr;  // row block by holds 2 by + 2 column tiles
    syrk_dmma_kernel<kAligned16><<<(unsigned)ntiles, SY_TPB, kSyrkSmem, st>>>(C, ldc, m, P, ldp, k,
                                                                            info);
    return launch_status("syrk_dmma_kernel");
}

int launch_syrk(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                const int *info, cudaStream_t st) {
    if (m <= 0 || k <= 0) return FMLB_OK;
    if (((uintptr_t)P % 16 == 0) && (ldp % 2 == 0))
        return launch_syrk_impl<true>(C, ldc, m, P, ldp, k, info, st);
    return launch_syrk_impl<false>(C, ldc, m, P, ldp, k, info, st);
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

int set_smem_attrs() {
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "potrf: cudaGetDevice"));
    if (attr_dev == dev) return FMLB_OK;
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(potf2_block_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kPotf2Smem), "potf2 smem attribute"));
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(panel_trsm_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kTrsmSmem), "trsm smem attribute"));
    attr_dev = dev;
    return FMLB_OK;
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_potrf_workspace_bytes(int n) {
    if (n <= 0) return 256;
    const size_t nblk = (size_t)(n + fmlb::NB - 1) / fmlb::NB;
    return nblk * fmlb::NB * fmlb::NB * sizeof(double) +
           ((size_t)n * sizeof(double) + 255) / 256 * 256;
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
    FMLB_TRY(set_smem_attrs());
    double *Linv = static_cast<double *>(work);
    for (int k0 = 0, kb = 0; k0 < n; k0 += NB, ++kb) {
        const int kn = std::min(NB, n - k0);
        double *Li = Linv + (size_t)kb * NB * NB;
        potf2_block_kernel<<<1, TPB, kPotf2Smem, st>>>(A, lda, k0, kn, Li, info);
        FMLB_TRY(launch_status("potf2_block_kernel"));
        const int rest = n - k0 - kn;
        if (rest <= 0) break;
        panel_trsm_kernel<<<ceil_div(rest, TRSM_ROWS), TPB, kTrsmSmem, st>>>(A, lda, n, k0, kn, Li,
                                                                            info);
        FMLB_TRY(launch_status("panel_trsm_kernel"));
        const size_t base = (size_t)(k0 + kn);
        FMLB_TRY(launch_syrk(A + base * lda + base, lda, rest, A + base * lda + k0, lda, kn, info,
                             st));
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

extern "C" int fmlb_syrk_lower_f64(double *C, long long ldc, int m, const double *P,
                                   long long ldp, int k, const int *info, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(m >= 0 && k >= 0 && ldc >= m && ldp >= k, "fmlb_syrk_lower_f64: bad sizes");
    if (m == 0 || k == 0) return FMLB_OK;
    FMLB_REQUIRE(C && P, "fmlb_syrk_lower_f64: null pointer");
    return launch_syrk(C, ldc, m, P, ldp, k, info, FMLB_STREAM(stream));
}
