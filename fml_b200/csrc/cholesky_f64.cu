// Plain-FP64 blocked right-looking Cholesky factorisation and solve, the
// replacement for LAPACK dpotrf('U') / dpotrs('U') as fcho_solve calls them
// (fml/math/fcho_solve.f90:35-42).
//
// Storage: row-major (n, n), factor L in the triangle i >= j (A = L L^T); the
// other triangle is never read or written. For the reference's C-order
// argument this is its dpotrf('U') factor U = L^T.
//
// Two levels of blocking. Inner panels of NB = 128 columns:
//   1. potf2 + inversion of the diagonal block in shared memory (one CTA); a
//      non-positive pivot records the LAPACK info (1-based column) and every
//      later kernel of the factorisation returns at once;
//   2. panel solve L21 = A21 L11^-T as a product with the stored inverse;
// outer panels of 256, 512 or 1024 columns (wider at larger n):
//   3. trailing update A22 -= L21 L21^T with k = the outer width, on the FP64
//      tensor cores (mma.sync m8n8k4 f64), 128x64 tiles on or below the
//      diagonal, operands streamed through a 3-stage cp.async pipeline;
// with the next outer panel factored on a second stream under step 3.
// The inverted diagonal blocks stay in the workspace for the solve (section 4).
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "ozaki.cuh"

namespace fmlb {
namespace {

constexpr int NB = 128;  // panel width
constexpr int TPB = 256;

__device__ __forceinline__ bool failed(const int *info) {
    return info && *(volatile const int *)info != 0;
}

// Programmatic dependent launch (kernels launched with programmatic stream
// serialization; in a kernel launched without it both are no-ops).
// griddepcontrol.wait returns once the previous kernel of the stream has
// completed and its writes are visible, so every read of data that kernel
// may write comes after it. The panel chain (diagonal block, panel solve,
// update inside the outer panel) signals its dependent only at its end, so
// the next kernel's CTAs do not sit on SMs the concurrent bulk update needs;
// the solve's step kernels signal at their start and read their rows of the
// factor, which no step writes, before waiting.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- 1. diagonal block ----------------------------------------------------
// The 128 x 128 block is factored in four 32-column steps. In step J one warp
// factors (and inverts) the 32 x 32 diagonal sub-block in registers with warp
// shuffles only; the whole CTA then solves the 32-column sub-panel below it
// and updates the rest of the block. The block inverse is assembled from the
// sub-block inverses: inv(L)_IJ = -inv(L_II) sum_{K=J}^{I-1} L_IK inv(L)_KJ,
// with the off-diagonal blocks kept (transposed) in the unused upper triangle.
constexpr int LDL = NB + 1;
constexpr int SB = 32, NSB = NB / SB, LDW = SB + 1;
constexpr size_t kPotf2Smem =
    ((size_t)NB * LDL + (size_t)NSB * SB * LDW + (size_t)(NSB - 1) * SB * LDW) * sizeof(double);

// One warp factors the 32 x 32 diagonal sub-block at L[b0.., b0..] in place
// and writes its inverse into W (row-major). Lane r holds row r of the block
// in registers; the entries other lanes need come by shuffles. The column
// steps are unrolled by template recursion, so every register index is a
// constant. The arithmetic (order of the FMAs, reciprocal-multiply scaling,
// the division in the substitution) is that of right-looking elimination
// and forward substitution in shared memory, bit for bit.
template <int J>
struct WarpFactor32 {
    __device__ __forceinline__ static void run(double (&a)[SB], int lane, int &fail) {
        const double piv = __shfl_sync(0xffffffffu, a[J], J);
        if (!(piv > 0.0) && !fail) fail = J + 1;  // later columns are NaN and not stored
        const double r = sqrt(piv), inv = 1.0 / r;
        if (lane == J) a[J] = r;
        else if (lane > J) a[J] *= inv;
        const double lij = a[J];
#pragma unroll
        for (int c = J + 1; c < SB; ++c) {
            const double lcj = __shfl_sync(0xffffffffu, a[J], c);  // L[c][J]
            if (c <= lane) a[c] = fma(-lij, lcj, a[c]);
        }
        WarpFactor32<J + 1>::run(a, lane, fail);
    }
};
template <>
struct WarpFactor32<SB> {
    __device__ __forceinline__ static void run(double (&)[SB], int, int &) {}
};
// Column `lane` of the inverse by forward substitution, right-looking: once
// w[K] = W[K][lane] is final it is subtracted from every later row's sum, so
// the serial chain per step is one division and one FMA. Each row's sum takes
// its terms in ascending column order, as the left-looking loop does; v[K]
// holds that sum until step K turns it into w[K].
template <int K>
struct WarpInverse32 {
    __device__ __forceinline__ static void run(const double (&a)[SB], double (&v)[SB], int lane) {
        const double lkk = __shfl_sync(0xffffffffu, a[K], K);
        v[K] = (K < lane) ? 0.0 : v[K] / lkk;
#pragma unroll
        for (int r = K + 1; r < SB; ++r) {
            const double lrk = __shfl_sync(0xffffffffu, a[K], r);  // L[r][K]
            if (K >= lane) v[r] = fma(-lrk, v[K], v[r]);
        }
        WarpInverse32<K + 1>::run(a, v, lane);
    }
};
template <>
struct WarpInverse32<SB> {
    __device__ __forceinline__ static void run(const double (&)[SB], double (&)[SB], int) {}
};

// Returns the 1-based failing column or 0 (the same value in every lane).
__device__ __forceinline__ int warp_potrf_inv32(double (*L)[NB + 1], int b0, double (*W)[SB + 1]) {
    const int lane = threadIdx.x & 31;
    double a[SB];
#pragma unroll
    for (int c = 0; c < SB; ++c) a[c] = c <= lane ? L[b0 + lane][b0 + c] : 0.0;
    int fail = 0;
    WarpFactor32<0>::run(a, lane, fail);
    if (fail) return fail;
#pragma unroll
    for (int c = 0; c < SB; ++c)
        if (c <= lane) L[b0 + lane][b0 + c] = a[c];
    double w[SB];
#pragma unroll
    for (int k = 0; k < SB; ++k) w[k] = (k == lane) ? 1.0 : 0.0;
    WarpInverse32<0>::run(a, w, lane);
#pragma unroll
    for (int k = 0; k < SB; ++k) W[k][lane] = w[k];
    __syncwarp();
    return 0;
}

__global__ void __launch_bounds__(TPB, 1)
potf2_block_kernel(double *__restrict__ A, long long lda, int k0, int kn,
                   double *__restrict__ Linv, int *__restrict__ info) {
    extern __shared__ double potf2_smem[];
    double(*L)[LDL] = reinterpret_cast<double(*)[LDL]>(potf2_smem);
    double(*W)[SB][LDW] = reinterpret_cast<double(*)[SB][LDW]>(potf2_smem + NB * LDL);
    // T[J]: sum_{K=J}^{I-1} L_IK inv(L)_KJ for every J < I of one block row I
    double(*T)[SB][LDW] =
        reinterpret_cast<double(*)[SB][LDW]>(potf2_smem + NB * LDL + NSB * SB * LDW);
    __shared__ int bad;
    pdl_wait();
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
            const int f = warp_potrf_inv32(L, b0, W[J]);
            if (f && lane == 0) bad = b0 + f;
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
        // update of the rest of the block: L[r][c] -= sum_k X[r][k] X[c][k], r0 <= c <= r;
        // two columns per step, so two independent FMA chains share the row loads
        for (int r = r0 + (tid >> 4); r < NB; r += TPB / 16) {
            for (int c = r0 + (tid & 15); c <= r; c += 32) {
                const bool two = c + 16 <= r;
                const int c2 = two ? c + 16 : c;
                double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
                for (int k = 0; k < SB; ++k) {
                    const double x = L[r][b0 + k];
                    s0 = fma(x, L[c][b0 + k], s0);
                    s1 = fma(x, L[c2][b0 + k], s1);
                }
                L[r][c] -= s0;
                if (two) L[r][c2] -= s1;
            }
        }
        __syncthreads();
    }
    // factor back to global
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t >> 7, c = t & (NB - 1);
        if (r < kn && c <= r) A[(size_t)(k0 + r) * lda + (k0 + c)] = L[r][c];
    }
    // block inverse; inv(L)_IJ for I > J is stored transposed at L[b0J + c][b0I + r].
    // Block row I needs the rows before it only, so its J < I blocks are formed
    // together: T[J] for every J, then inv(L)_IJ = -inv(L_II) T[J].
    // Thread tid forms, for every J, the four rows r = tid / 32 + 8 i of column
    // c = tid % 32: the column operand is loaded once for four independent FMA
    // chains (each entry's sum in the same order as one chain per entry).
    static_assert(TPB == 8 * SB, "four rows per thread and column block");
    const int rq = tid >> 5, cq = tid & 31;
    for (int I = 1; I < NSB; ++I) {
        for (int J = 0; J < I; ++J) {
            double sacc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int K = J; K < I; ++K) {
                for (int q = 0; q < SB; ++q) {
                    const double inv = (K == J) ? W[J][q][cq] : L[J * SB + cq][K * SB + q];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        sacc[i] = fma(L[I * SB + rq + 8 * i][K * SB + q], inv, sacc[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) T[J][rq + 8 * i][cq] = sacc[i];
        }
        __syncthreads();
        for (int J = 0; J < I; ++J) {
            double sacc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int q = 0; q <= rq + 24; ++q) {
                const double tq = T[J][q][cq];
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (q <= rq + 8 * i) sacc[i] = fma(W[I][rq + 8 * i][q], tq, sacc[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) L[J * SB + cq][I * SB + rq + 8 * i] = -sacc[i];
        }
        __syncthreads();
    }
    for (int t = tid; t < NB * NB; t += TPB) {
        const int r = t >> 7, c = t & (NB - 1);
        const int I = r / SB, J = c / SB;
        double v = 0.0;
        if (I == J) v = (c <= r) ? W[I][r - I * SB][c - J * SB] : 0.0;
        else if (I > J) v = L[c][r];
        Linv[t] = v;
    }
    pdl_launch_dependents();
}

// ---- 2. panel solve: rows [r0, n) of columns [k0, k0+kn): X <- X Linv^T ----
constexpr int TRSM_ROWS = 64;
constexpr size_t kTrsmSmem = (size_t)(NB + TRSM_ROWS) * LDL * sizeof(double);

// Rows [r0, r0 + TRSM_ROWS) (clipped to rend) of columns [k0, k0 + kn):
// out[r][c] = sum_{k <= c} X[r][k] * Linv[c][k], in place.
__device__ __forceinline__ void trsm_rows(double *__restrict__ A, long long lda, int r0, int rend,
                                          int k0, int kn, const double *__restrict__ Linv,
                                          double *smem) {
    double(*Li)[LDL] = reinterpret_cast<double(*)[LDL]>(smem);
    double(*P)[LDL] = reinterpret_cast<double(*)[LDL]>(smem + NB * LDL);
    const int tid = threadIdx.x;
    for (int t = tid; t < NB * NB; t += TPB) Li[t / NB][t % NB] = Linv[t];
    for (int t = tid; t < TRSM_ROWS * NB; t += TPB) {
        const int r = t / NB, c = t % NB;
        P[r][c] = (r0 + r < rend && c < kn) ? A[(size_t)(r0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
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
        if (r < rend && c < kn) A[(size_t)r * lda + k0 + c] = out[i];
    }
}

__global__ void __launch_bounds__(TPB)
panel_trsm_kernel(double *__restrict__ A, long long lda, int n, int k0, int kn,
                  const double *__restrict__ Linv, const int *__restrict__ info) {
    extern __shared__ double trsm_smem[];
    pdl_wait();
    if (failed(info)) return;
    trsm_rows(A, lda, k0 + kn + blockIdx.x * TRSM_ROWS, n, k0, kn, Linv, trsm_smem);
    pdl_launch_dependents();
}

// Rows [0, rend) of columns [k0, k0 + kn): X <- X Linv^T (the inverse's
// column-block step, section 5).
__global__ void __launch_bounds__(TPB)
rows_trsm_kernel(double *__restrict__ A, long long lda, int rend, int k0, int kn,
                 const double *__restrict__ Linv, const int *__restrict__ info) {
    extern __shared__ double trsm_smem[];
    if (failed(info)) return;
    trsm_rows(A, lda, blockIdx.x * TRSM_ROWS, rend, k0, kn, Linv, trsm_smem);
}

// ---- 3. trailing update on the FP64 tensor cores ---------------------------
// C (m x m, stride ldc) -= P P^T on the triangle c <= r, P is (m x k).
// CTA tile 128 rows x 64 columns, 4 warps as 2 x 2, warp tile 64x32 =
// 8 x 4 m8n8 fragments; two CTAs fit per SM so one CTA's prologue and
// read-modify-write epilogue overlap the other's tensor-core work.
constexpr int SY_TM = 128, SY_TN = 64, SY_TK = 16, SY_LD = 20, SY_STAGES = 3, SY_TPB = 128;
constexpr int SY_STAGE_DOUBLES = (SY_TM + SY_TN) * SY_LD;
constexpr int SY_CLD = SY_TN + 8;  // row pitch of the epilogue's C tile in shared memory
static_assert(SY_TM * SY_CLD <= SY_STAGES * SY_STAGE_DOUBLES, "C tile must fit in the stages");
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
                 long long ldp, int k, int strip_tiles, const int *__restrict__ info) {
    extern __shared__ __align__(16) double sy_smem[];
    pdl_wait();
    if (failed(info)) return;
    const long long t = blockIdx.x;
    int by, bx;
    if (strip_tiles > 0) {  // only the first strip_tiles column tiles of every row block
        by = (int)(t / strip_tiles);
        bx = (int)(t % strip_tiles);
        if (bx > 2 * by + 1) return;
    } else {  // tile t -> (row block by of 128, column block bx of 64), bx <= 2 by + 1
        by = (int)((sqrt(4.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)by * by + by > t) --by;
        while ((long long)(by + 1) * (by + 1) + (by + 1) <= t) ++by;
        bx = (int)(t - (long long)by * by - by);
    }
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
    __syncthreads();  // every warp is done with the stage buffers
    // Epilogue through shared memory: one coalesced pass loads the C tile,
    // the fragments are subtracted there, one coalesced masked pass stores it
    // (keeps the 64 read-modify-writes per thread from serialising).
    double *Cs = sy_smem;  // SY_TM x SY_CLD doubles, fits in the stage area
    const int tid = threadIdx.x;
    for (int e = tid; e < SY_TM * (SY_TN / 2); e += SY_TPB) {
        const int r = e / (SY_TN / 2), c = (e % (SY_TN / 2)) * 2;
        const int gr = row0 + r, gc = col0 + c;
        double v0 = 0.0, v1 = 0.0;
        if (gr < m) {
            const double *src = C + (size_t)gr * ldc + gc;
            if (gc < m) v0 = src[0];
            if (gc + 1 < m) v1 = src[1];
        }
        Cs[r * SY_CLD + c] = v0;
        Cs[r * SY_CLD + c + 1] = v1;
    }
    __syncthreads();
    // fragment (i, j): rows wr*64 + i*8 + g, columns wc*32 + j*8 + 2*tq + {0, 1}
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int rl = wr * 64 + i * 8 + g;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cl = wc * 32 + j * 8 + 2 * tq;
            Cs[rl * SY_CLD + cl] -= acc[i][j][0];
            Cs[rl * SY_CLD + cl + 1] -= acc[i][j][1];
        }
    }
    __syncthreads();
    for (int e = tid; e < SY_TM * (SY_TN / 2); e += SY_TPB) {
        const int r = e / (SY_TN / 2), c = (e % (SY_TN / 2)) * 2;
        const int gr = row0 + r, gc = col0 + c;
        if (gr >= m) continue;
        double *dst = C + (size_t)gr * ldc + gc;
        if (gc < m && gc <= gr) dst[0] = Cs[r * SY_CLD + c];
        if (gc + 1 < m && gc + 1 <= gr) dst[1] = Cs[r * SY_CLD + c + 1];
    }
    pdl_launch_dependents();
}

// Launch with programmatic stream serialization when `pdl` is set (the kernel
// orders its dependent reads with griddepcontrol.wait).
template <typename... KArgs, typename... Args>
int launch_maybe_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                     cudaStream_t st, const char *name, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    FMLB_TRY(cuda_status(cudaLaunchKernelEx(&cfg, kernel, args...), name));
    return launch_status(name);
}

template <bool kAligned16>
int launch_syrk_impl(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                     int strip_cols, const int *info, cudaStream_t st, bool pdl) {
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
    const int strip_tiles = strip_cols > 0 ? ceil_div(std::min(strip_cols, m), SY_TN) : 0;
    // full: row block by holds 2 by + 2 column tiles; strip: strip_tiles per row block
    const long long ntiles = strip_tiles ? Tr * strip_tiles : Tr * Tr + Tr;
    return launch_maybe_pdl(pdl, syrk_dmma_kernel<kAligned16>, dim3((unsigned)ntiles),
                            dim3(SY_TPB), kSyrkSmem, st, "syrk_dmma_kernel", C, ldc, m, P, ldp, k,
                            strip_tiles, info);
}

// strip_cols = 0: lower triangle of the m x m block; > 0: only its first
// strip_cols columns (the lower part of that column strip).
int launch_syrk(double *C, long long ldc, int m, const double *P, long long ldp, int k,
                const int *info, cudaStream_t st, int strip_cols = 0, bool pdl = false) {
    if (m <= 0 || k <= 0) return FMLB_OK;
    if (((uintptr_t)P % 16 == 0) && (ldp % 2 == 0))
        return launch_syrk_impl<true>(C, ldc, m, P, ldp, k, strip_cols, info, st, pdl);
    return launch_syrk_impl<false>(C, ldc, m, P, ldp, k, strip_cols, info, st, pdl);
}

// ---- 4. triangular solves with the factor (potrs) ---------------------------
// Right-looking, one launch per 128-block column and direction. Every thread
// block reads its rows (forward) or columns (backward) of the factor once,
// coalesced; the block that owns the next diagonal block also applies that
// block's stored inverse, so the next launch starts from a finished
// sub-vector. All reductions run in a fixed order (deterministic).
constexpr int SOLVE_WARPS = TPB / 32;

constexpr int FWD_ROWS = 32;   // rows per thread block past the next diagonal block
constexpr int BWD_COLS = 32;   // columns per thread block before the previous one

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// out[t] = sum_{c <= t} Linv[t][c] in[c], t < kn (lower-triangular block
// inverse, row-major 128 x 128); warp per row, four rows in flight per warp.
__device__ __forceinline__ void tri_lower_apply(const double *__restrict__ Linv,
                                                const double *in, double *out, int kn) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t0 = warp; t0 < kn; t0 += 4 * SOLVE_WARPS) {
        double s[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int t = t0 + q * SOLVE_WARPS;
            s[q] = 0.0;
#pragma unroll
            for (int i = 0; i < NB / 32; ++i) {
                const int c = lane + 32 * i;
                if (t < kn && c <= t) s[q] = fma(Linv[t * NB + c], in[c], s[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double v = warp_sum(s[q]);
            const int t = t0 + q * SOLVE_WARPS;
            if (lane == 0 && t < kn) out[t] = v;
        }
    }
}

// out[t] = sum_{r >= t} Linv[r][t] in[r], t < kn (the transposed inverse);
// thread t with 2 row halves reduced through shared memory.
__device__ __forceinline__ void tri_upper_apply(const double *__restrict__ Linv,
                                                const double *in, double *out, int kn,
                                                double *red) {
    const int t = threadIdx.x & (NB - 1), h = threadIdx.x >> 7;  // TPB = 2 NB
    double s = 0.0;
    if (t < kn) {
        const int r1 = min(kn, (h + 1) * (NB / 2));
#pragma unroll 32
        for (int r = h * (NB / 2); r < r1; ++r)
            if (r >= t) s = fma(Linv[r * NB + t], in[r], s);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    if (h == 0 && t < kn) out[t] = red[t] + red[t + NB];
}

// y[0..kn) = Linv_0 x[0..kn)
__global__ void __launch_bounds__(TPB)
solve_first_forward_kernel(const double *__restrict__ Linv0, const double *__restrict__ x,
                           double *__restrict__ y, int kn) {
    tri_lower_apply(Linv0, x, y, kn);
}

// x[k0..k0+kn) = Linv_k^T y[k0..k0+kn)
__global__ void __launch_bounds__(TPB)
solve_first_backward_kernel(const double *__restrict__ Linvk, const double *__restrict__ y,
                            double *__restrict__ x, int kn) {
    __shared__ double red[TPB];
    pdl_launch_dependents();
    pdl_wait();
    tri_upper_apply(Linvk, y, x, kn, red);
}

// L2 prefetch of a 128 x 128 block (the next diagonal block's inverse), so
// that the owner block's final step reads it from L2
__device__ __forceinline__ void prefetch_block_l2(const double *p) {
    for (int t = threadIdx.x; t < NB * NB / 16; t += blockDim.x)  // one 128-byte line each
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p + (size_t)t * 16));
}

// Forward step for block column k (y_k final): x[r] -= L[r, k0:k0+kn] y_k for
// r >= k0 + kn. Thread block 0 owns the next diagonal block and then writes
// y_{k+1} = Linv_{k+1} x_{k+1}. Every lane reads its four entries of y_k
// directly, so a warp's row loads, y_k loads and x loads all go out together;
// each warp keeps eight rows in flight.
__global__ void __launch_bounds__(TPB)
forward_step_kernel(const double *__restrict__ L, long long lda, int n, int k0, int kn,
                    const double *__restrict__ LinvNext, double *__restrict__ x,
                    double *__restrict__ y) {
    __shared__ double xn[NB];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool owner = blockIdx.x == 0;
    pdl_launch_dependents();
    if (owner && LinvNext != nullptr) prefetch_block_l2(LinvNext);
    double ykr[NB / 32];
    bool waited = false;
    const int nb0 = k0 + kn;
    int rb, re;
    if (owner) {
        rb = nb0;
        re = min(n, nb0 + NB);
    } else {
        rb = nb0 + NB + (blockIdx.x - 1) * FWD_ROWS;
        re = min(n, rb + FWD_ROWS);
    }
    constexpr int G = 8;  // rows per warp in flight
    for (int r0 = rb + warp; r0 < re; r0 += G * SOLVE_WARPS) {
        double s[G], xr[G], lv[G][NB / 32];
#pragma unroll
        for (int q = 0; q < G; ++q) {  // the factor's rows: not written by any step
            const int r = r0 + q * SOLVE_WARPS;
            const bool ok = r < re;
            const double *row = L + (size_t)min(r, n - 1) * lda + k0;
#pragma unroll
            for (int i = 0; i < NB / 32; ++i) {
                const int c = lane + 32 * i;
                lv[q][i] = (ok && c < kn) ? row[c] : 0.0;
            }
        }
        if (!waited) {
            pdl_wait();
            waited = true;
#pragma unroll
            for (int i = 0; i < NB / 32; ++i) {
                const int c = lane + 32 * i;
                ykr[i] = c < kn ? y[k0 + c] : 0.0;
            }
        }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int r = r0 + q * SOLVE_WARPS;
            const bool ok = r < re;
            s[q] = 0.0;
            xr[q] = (ok && lane == 0) ? x[r] : 0.0;
#pragma unroll
            for (int i = 0; i < NB / 32; ++i) {
                const int c = lane + 32 * i;
                if (ok && c < kn) s[q] = fma(lv[q][i], ykr[i], s[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const double sq = warp_sum(s[q]);
            const int r = r0 + q * SOLVE_WARPS;
            if (lane == 0 && r < re) {
                const double v = xr[q] - sq;
                x[r] = v;
                if (owner) xn[r - nb0] = v;
            }
        }
    }
    if (!waited) pdl_wait();
    if (owner && LinvNext != nullptr) {
        __syncthreads();
        tri_lower_apply(LinvNext, xn, y + nb0, re - rb);
    }
}

// Backward step for block column k (x_k final): y[j] -= sum_r L[k0 + r, j]
// x_k[r] for j < k0. Thread block 0 owns the previous diagonal block's 128
// columns (2 row halves per column) and then writes x_{k-1} = Linv_{k-1}^T
// y_{k-1}; the others own 32 columns each (8 row groups per column). Partial
// sums are added in a fixed order.
__global__ void __launch_bounds__(TPB)
backward_step_kernel(const double *__restrict__ L, long long lda, int k0, int kn,
                     const double *__restrict__ LinvPrev, double *__restrict__ y,
                     double *__restrict__ x) {
    __shared__ double xk[NB];
    __shared__ double yp[NB];
    __shared__ double red[TPB];
    const int tid = threadIdx.x;
    const bool owner = blockIdx.x == 0;
    pdl_launch_dependents();
    if (owner) prefetch_block_l2(LinvPrev);
    pdl_wait();
    if (tid < NB) xk[tid] = tid < kn ? x[k0 + tid] : 0.0;
    __syncthreads();
    const int pb = k0 - NB;  // first column of the previous diagonal block (k0 >= NB here)
    const int W = owner ? NB : BWD_COLS;          // columns of this thread block
    const int G = TPB / W;                        // row groups per column
    const int rows_per = NB / G;
    const int cb = owner ? pb : (blockIdx.x - 1) * BWD_COLS;
    const int ce = owner ? k0 : min(pb, cb + BWD_COLS);
    const int col = tid % W, g = tid / W;
    const int j = cb + col;
    double s = 0.0;
    if (j < ce) {
        const int rbeg = g * rows_per;
#pragma unroll 32
        for (int rr = 0; rr < rows_per; ++rr) {
            const int r = rbeg + rr;
            if (r < kn) s = fma(L[(size_t)(k0 + r) * lda + j], xk[r], s);
        }
    }
    red[tid] = s;
    __syncthreads();
    if (g == 0 && j < ce) {
        double t = 0.0;
        for (int q = 0; q < G; ++q) t += red[q * W + col];
        const double v = y[j] - t;
        y[j] = v;
        if (owner) yp[col] = v;
    }
    if (owner) {
        __syncthreads();
        tri_upper_apply(LinvPrev, yp, x + pb, NB, red);
    }
}

// ---- 5. inverse from the factor (potri) ------------------------------------
// inv(A) = L^-T L^-1 = V V^T with V = L^-T (upper triangular). V solves
// V L^T = I column block by column block, right-looking:
//   V[:, i] = U[:, i] Linv_ii^T                      (rows_trsm_kernel)
//   U[:, j] -= V[:, i] L[j, i]^T for blocks j > i    (gemm_nt_dmma_kernel)
// with U = I initially (only rows above block i+1 are non-zero). Then the
// lower triangle of V V^T (gemm_nt_dmma_kernel, triangle mode, k from the
// tile's first row on since V is upper triangular). 2n^3/3 flops, as LAPACK
// dpotri; both products on the FP64 tensor cores with the trailing update's
// tiles (128 x 64, DMMA m8n8k4, 3-stage cp.async).
//
// kTri = false: C (M x N) -= A B^T, A (M x K), B (N x K), all row-major.
// kTri = true:  C (M x M, triangle c <= r) = A A^T with A upper triangular
//               (B = A, the k-loop of row block r0 starts at r0).
template <bool kAligned16, bool kTri>
__global__ void __launch_bounds__(SY_TPB, 2)
gemm_nt_dmma_kernel(double *__restrict__ C, long long ldc, int M, int N,
                    const double *__restrict__ A, long long lda, const double *__restrict__ B,
                    long long ldb, int K, int tiles_n, const int *__restrict__ info) {
    extern __shared__ __align__(16) double sy_smem[];
    if (failed(info)) return;
    const long long t = blockIdx.x;
    int by, bx;
    if (kTri) {  // tile t -> (by, bx <= 2 by + 1), as the trailing update
        by = (int)((sqrt(4.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)by * by + by > t) --by;
        while ((long long)(by + 1) * (by + 1) + (by + 1) <= t) ++by;
        bx = (int)(t - (long long)by * by - by);
    } else {
        by = (int)(t / tiles_n);
        bx = (int)(t % tiles_n);
    }
    const int row0 = by * SY_TM, col0 = bx * SY_TN;
    if (row0 >= M || col0 >= N) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wr = warp >> 1, wc = warp & 1;
    const int g = lane >> 2, tq = lane & 3;

    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int kt0 = kTri ? row0 / SY_TK : 0;  // row0 is a multiple of SY_TK
    const int nk = (K + SY_TK - 1) / SY_TK;
#pragma unroll
    for (int s = 0; s < SY_STAGES - 1; ++s) {
        if (kt0 + s < nk) {
            double *st = sy_smem + s * SY_STAGE_DOUBLES;
            syrk_load_tile<SY_TM, kAligned16>(st, A, lda, M, K, row0, (kt0 + s) * SY_TK);
            syrk_load_tile<SY_TN, kAligned16>(st + SY_TM * SY_LD, B, ldb, N, K, col0,
                                              (kt0 + s) * SY_TK);
        }
        cp_async_commit();
    }
    for (int kt = kt0; kt < nk; ++kt) {
        cp_async_wait<SY_STAGES - 2>();
        __syncthreads();
        const int nxt = kt + SY_STAGES - 1;
        if (nxt < nk) {
            double *st = sy_smem + ((nxt - kt0) % SY_STAGES) * SY_STAGE_DOUBLES;
            syrk_load_tile<SY_TM, kAligned16>(st, A, lda, M, K, row0, nxt * SY_TK);
            syrk_load_tile<SY_TN, kAligned16>(st + SY_TM * SY_LD, B, ldb, N, K, col0,
                                              nxt * SY_TK);
        }
        cp_async_commit();
        const double *As = sy_smem + ((kt - kt0) % SY_STAGES) * SY_STAGE_DOUBLES;
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
    __syncthreads();
    double *Cs = sy_smem;  // SY_TM x SY_CLD
    const int tid = threadIdx.x;
    for (int e = tid; e < SY_TM * (SY_TN / 2); e += SY_TPB) {
        const int r = e / (SY_TN / 2), c = (e % (SY_TN / 2)) * 2;
        const int gr = row0 + r, gc = col0 + c;
        double v0 = 0.0, v1 = 0.0;
        if (!kTri && gr < M) {
            const double *src = C + (size_t)gr * ldc + gc;
            if (gc < N) v0 = src[0];
            if (gc + 1 < N) v1 = src[1];
        }
        Cs[r * SY_CLD + c] = v0;
        Cs[r * SY_CLD + c + 1] = v1;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int rl = wr * 64 + i * 8 + g;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cl = wc * 32 + j * 8 + 2 * tq;
            if (kTri) {
                Cs[rl * SY_CLD + cl] += acc[i][j][0];
                Cs[rl * SY_CLD + cl + 1] += acc[i][j][1];
            } else {
                Cs[rl * SY_CLD + cl] -= acc[i][j][0];
                Cs[rl * SY_CLD + cl + 1] -= acc[i][j][1];
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < SY_TM * (SY_TN / 2); e += SY_TPB) {
        const int r = e / (SY_TN / 2), c = (e % (SY_TN / 2)) * 2;
        const int gr = row0 + r, gc = col0 + c;
        if (gr >= M) continue;
        double *dst = C + (size_t)gr * ldc + gc;
        if (gc < N && (!kTri || gc <= gr)) dst[0] = Cs[r * SY_CLD + c];
        if (gc + 1 < N && (!kTri || gc + 1 <= gr)) dst[1] = Cs[r * SY_CLD + c + 1];
    }
}

template <bool kTri>
int launch_gemm_nt(double *C, long long ldc, int M, int N, const double *A, long long lda,
                   const double *B, long long ldb, int K, const int *info, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0) return FMLB_OK;
    const bool al = (uintptr_t)A % 16 == 0 && lda % 2 == 0 && (uintptr_t)B % 16 == 0 &&
                    ldb % 2 == 0;
    const long long Tr = ceil_div(M, SY_TM);
    const int tiles_n = ceil_div(N, SY_TN);
    const long long ntiles = kTri ? Tr * Tr + Tr : Tr * tiles_n;
    if (al) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(gemm_nt_dmma_kernel<true, kTri>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kSyrkSmem), "gemm smem attribute"));
        gemm_nt_dmma_kernel<true, kTri><<<(unsigned)ntiles, SY_TPB, kSyrkSmem, st>>>(
            C, ldc, M, N, A, lda, B, ldb, K, tiles_n, info);
    } else {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(gemm_nt_dmma_kernel<false, kTri>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kSyrkSmem), "gemm smem attribute"));
        gemm_nt_dmma_kernel<false, kTri><<<(unsigned)ntiles, SY_TPB, kSyrkSmem, st>>>(
            C, ldc, M, N, A, lda, B, ldb, K, tiles_n, info);
    }
    return launch_status("gemm_nt_dmma_kernel");
}

// V = I on the leading (n, n) block of a row-major buffer with stride ldv
__global__ void identity_kernel(double *__restrict__ V, long long ldv, int n) {
    const int r = blockIdx.y, c = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n && c < n) V[(size_t)r * ldv + c] = (r == c) ? 1.0 : 0.0;
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
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(rows_trsm_kernel,
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

// Per host thread, device and caller stream: the high-priority stream that
// runs the panel chain (strip update, diagonal block, panel solve) of the
// lookahead, and two events to order it against the caller's stream.
// Factorisations issued on different caller streams get different panel
// streams, so they can overlap: one's narrow final steps run under another's
// bulk updates. Past kPerCaller caller streams a thread shares one entry per
// device; its panel stream then serialises those callers' panel chains, which
// is slower but still ordered correctly, since every wait names the event
// recorded by the same call. The streams and events live for the life of the
// host thread and do not survive cudaDeviceReset: a process that resets a
// device must not factor on it again from the same thread.
struct Lookahead {
    cudaStream_t panel = nullptr;
    cudaEvent_t main_done = nullptr, panel_done = nullptr;
};

static int lookahead_for(cudaStream_t caller, Lookahead **out) {
    using namespace fmlb;
    constexpr int kPerCaller = 16;
    struct Entry {
        int dev = -1;
        cudaStream_t caller = nullptr;
        Lookahead la;
    };
    static thread_local Entry by_caller[kPerCaller];
    static thread_local Lookahead shared_per_dev[64];
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_potrf_f64: cudaGetDevice"));
    FMLB_REQUIRE(dev >= 0 && dev < 64, "fmlb_potrf_f64: device %d out of range", dev);
    Lookahead *lp = nullptr;
    for (int i = 0; i < kPerCaller && !lp; ++i)
        if (by_caller[i].dev == dev && by_caller[i].caller == caller) lp = &by_caller[i].la;
    for (int i = 0; i < kPerCaller && !lp; ++i)
        if (by_caller[i].dev < 0) {
            by_caller[i].dev = dev;
            by_caller[i].caller = caller;
            lp = &by_caller[i].la;
        }
    if (!lp) lp = &shared_per_dev[dev];
    Lookahead &L = *lp;
    if (!L.panel) {
        int lo = 0, hi = 0;
        FMLB_TRY(cuda_status(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priorities"));
        FMLB_TRY(cuda_status(cudaStreamCreateWithPriority(&L.panel, cudaStreamNonBlocking, hi),
                             "fmlb_potrf_f64: panel stream"));
        FMLB_TRY(cuda_status(cudaEventCreateWithFlags(&L.main_done, cudaEventDisableTiming),
                             "fmlb_potrf_f64: event"));
        FMLB_TRY(cuda_status(cudaEventCreateWithFlags(&L.panel_done, cudaEventDisableTiming),
                             "fmlb_potrf_f64: event"));
    }
    *out = &L;
    return FMLB_OK;
}

static int panel_factor(double *A, long long lda, int n, int k0, double *Li, int *info,
                        cudaStream_t st, bool after_kernel) {
    using namespace fmlb;
    const int kn = std::min(NB, n - k0);
    // the chain of one outer panel: each kernel follows the previous one of
    // the stream with a programmatic dependency; the first block of an outer
    // panel is launched normally, as what precedes it may be a memset or an
    // event wait rather than a kernel of the chain
    FMLB_TRY(launch_maybe_pdl(after_kernel, potf2_block_kernel, dim3(1), dim3(TPB), kPotf2Smem, st,
                              "potf2_block_kernel", A, lda, k0, kn, Li, info));
    const int rest = n - k0 - kn;
    if (rest > 0)
        FMLB_TRY(launch_maybe_pdl(true, panel_trsm_kernel, dim3(ceil_div(rest, TRSM_ROWS)),
                                  dim3(TPB), kTrsmSmem, st, "panel_trsm_kernel", A, lda, n, k0, kn,
                                  (const double *)Li, (const int *)info));
    return FMLB_OK;
}

// Factor the outer panel of columns [K0, K0 + width) on stream st: per inner
// panel of NB columns, the diagonal block and the panel solve (all rows below),
// then the update of the rest of the outer panel's columns by that inner panel.
static int factor_outer_panel(double *A, long long lda, int n, int K0, int width, double *Linv,
                              int *info, cudaStream_t st) {
    using namespace fmlb;
    const int end = std::min(K0 + width, n);
    for (int k0 = K0; k0 < end; k0 += NB) {
        FMLB_TRY(panel_factor(A, lda, n, k0, Linv + (size_t)(k0 / NB) * NB * NB, info, st,
                              k0 > K0));
        const size_t b = (size_t)(k0 + NB);
        const int rem = end - (int)b;
        if (rem > 0)
            FMLB_TRY(launch_syrk(A + b * lda + b, lda, n - (int)b, A + b * lda + k0, lda, NB, info,
                                 st, rem, true));
    }
    return FMLB_OK;
}

// Outer panel width: wide panels give the trailing update a long k-loop
// (k = 512: ~28 TFLOP/s against ~17 at k = 128 on B200) and fewer steps.
// Measured at n = 32768 on B200: 455 ms (512), 436 ms (768), 429 ms (1024).
static int outer_width(int n) {
    return n >= 16384 ? 8 * fmlb::NB : n >= 8192 ? 4 * fmlb::NB : 2 * fmlb::NB;
}

// Two-level blocked factorisation with a lookahead of depth one. For outer
// panel K (factored), with outer block K+1 the next:
//   panel stream:  strip update of outer block K+1 by panel K (k = width),
//                  then the factorisation of outer panel K+1;
//   caller stream: update of the trailing matrix past block K+1 by panel K.
// The two regions are disjoint, so the panel chain runs under the bulk update.
// With `oz` set, the strip and bulk updates run on the int8 tensor cores
// (ozaki_f64.cu): panel K's rows below it are split into digit planes once,
// on the caller stream, before either update reads them; the next split waits
// for the panel stream, so the planes are never overwritten while read.
static int potrf_blocked(double *A, long long lda, int n, void *work, int *info,
                         cudaStream_t st, const fmlb::OzakiSlices *oz) {
    using namespace fmlb;
    FMLB_TRY(set_smem_attrs());
    Lookahead *la = nullptr;
    FMLB_TRY(lookahead_for(st, &la));
    double *Linv = static_cast<double *>(work);
    const int W = outer_width(n);
    const int nob = ceil_div(n, W);
    FMLB_TRY(factor_outer_panel(A, lda, n, 0, W, Linv, info, st));
    bool panel_used = false;
    for (int K = 0; K + 1 < nob; ++K) {
        const int K0 = K * W;
        const size_t base = (size_t)(K0 + W);  // first row / column of outer block K+1
        const int rest = n - (int)base;
        if (panel_used)  // outer panel K was factored on the panel stream
            FMLB_TRY(cuda_status(cudaStreamWaitEvent(st, la->panel_done, 0), "wait panel"));
        if (oz)  // digit planes of panel K, rows [base, n)
            FMLB_TRY(ozaki_split(A + base * lda + K0, lda, rest, W, *oz, info, st));
        FMLB_TRY(cuda_status(cudaEventRecord(la->main_done, st), "record main"));
        FMLB_TRY(cuda_status(cudaStreamWaitEvent(la->panel, la->main_done, 0), "wait main"));
        if (oz)
            FMLB_TRY(ozaki_syrk(A + base * lda + base, lda, rest, *oz, 0, W, info, la->panel));
        else
            FMLB_TRY(launch_syrk(A + base * lda + base, lda, rest, A + base * lda + K0, lda, W,
                                 info, la->panel, W));
        FMLB_TRY(factor_outer_panel(A, lda, n, (int)base, W, Linv, info, la->panel));
        FMLB_TRY(cuda_status(cudaEventRecord(la->panel_done, la->panel), "record panel"));
        panel_used = true;
        const int rest2 = rest - W;
        if (rest2 > 0) {
            const size_t b2 = base + W;
            if (oz)
                FMLB_TRY(ozaki_syrk(A + b2 * lda + b2, lda, rest2, *oz, W, 0, info, st));
            else
                FMLB_TRY(launch_syrk(A + b2 * lda + b2, lda, rest2, A + b2 * lda + K0, lda, W,
                                     info, st));
        }
    }
    if (panel_used)
        FMLB_TRY(cuda_status(cudaStreamWaitEvent(st, la->panel_done, 0), "join panel stream"));
    return FMLB_OK;
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
    return potrf_blocked(A, lda, n, work, info, st, nullptr);
}

extern "C" size_t fmlb_potrf_ozaki_workspace_bytes(int n, int nslices) {
    if (n <= 0 || nslices <= 0) return 256;
    const int W = outer_width(n);
    return (fmlb_potrf_workspace_bytes(n) + 255) / 256 * 256 +
           fmlb::ozaki_slice_bytes(n, W, nslices);
}

extern "C" int fmlb_potrf_ozaki_f64(double *A, long long lda, int n, int nslices, void *work,
                                    size_t ws_bytes, int *info, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_potrf_ozaki_f64: bad n=%d / lda=%lld", n, lda);
    FMLB_REQUIRE(nslices >= 1 && nslices <= OZAKI_MAX_SLICES,
                 "fmlb_potrf_ozaki_f64: nslices must be 1..%d", OZAKI_MAX_SLICES);
    FMLB_REQUIRE(info, "fmlb_potrf_ozaki_f64: info pointer is null");
    FMLB_TRY(cuda_status(cudaMemsetAsync(info, 0, sizeof(int), st),
                         "fmlb_potrf_ozaki_f64: clear info"));
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A && work, "fmlb_potrf_ozaki_f64: null pointer");
    const size_t need = fmlb_potrf_ozaki_workspace_bytes(n, nslices);
    if (ws_bytes < need) {
        set_error("fmlb_potrf_ozaki_f64: workspace %zu < %zu bytes", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    OzakiSlices oz;
    const size_t off = (fmlb_potrf_workspace_bytes(n) + 255) / 256 * 256;
    FMLB_TRY(ozaki_bind(static_cast<char *>(work) + off, n, outer_width(n), nslices, oz));
    return potrf_blocked(A, lda, n, work, info, st, &oz);
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
    solve_first_forward_kernel<<<1, TPB, 0, st>>>(Linv, x, y, std::min(NB, n));
    FMLB_TRY(launch_status("solve_first_forward_kernel"));
    for (int k0 = 0, kb = 0; k0 + NB < n; k0 += NB, ++kb) {
        const int rest = n - k0 - NB;  // rows past this block column
        const int grid = 1 + ceil_div(std::max(0, rest - NB), FWD_ROWS);
        FMLB_TRY(launch_maybe_pdl(true, forward_step_kernel, dim3(grid), dim3(TPB), 0, st,
                                  "forward_step_kernel", L, lda, n, k0, (int)NB,
                                  (const double *)(Linv + (size_t)(kb + 1) * NB * NB), x, y));
    }
    {
        const int kb = (int)nblk - 1, k0 = kb * NB;
        FMLB_TRY(launch_maybe_pdl(true, solve_first_backward_kernel, dim3(1), dim3(TPB), 0, st,
                                  "solve_first_backward_kernel",
                                  (const double *)(Linv + (size_t)kb * NB * NB),
                                  (const double *)(y + k0), x + k0, n - k0));
    }
    for (int kb = (int)nblk - 1; kb >= 1; --kb) {
        const int k0 = kb * NB, kn = std::min(NB, n - k0);
        const int grid = 1 + ceil_div(k0 - NB, BWD_COLS);
        FMLB_TRY(launch_maybe_pdl(true, backward_step_kernel, dim3(grid), dim3(TPB), 0, st,
                                  "backward_step_kernel", L, lda, k0, kn,
                                  (const double *)(Linv + (size_t)(kb - 1) * NB * NB), y, x));
    }
    return FMLB_OK;
}

extern "C" int fmlb_syrk_lower_f64(double *C, long long ldc, int m, const double *P,
                                   long long ldp, int k, int strip_cols, const int *info,
                                   void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(m >= 0 && k >= 0 && ldc >= m && ldp >= k && strip_cols >= 0,
                 "fmlb_syrk_lower_f64: bad sizes");
    if (m == 0 || k == 0) return FMLB_OK;
    FMLB_REQUIRE(C && P, "fmlb_syrk_lower_f64: null pointer");
    return launch_syrk(C, ldc, m, P, ldp, k, info, FMLB_STREAM(stream), strip_cols);
}

extern "C" int fmlb_potri_f64(double *A, long long lda, int n, const void *work, double *V,
                              long long ldv, const int *info, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(n >= 0 && lda >= n && ldv >= n, "fmlb_potri_f64: bad n=%d / lda / ldv", n);
    if (n == 0) return FMLB_OK;
    FMLB_REQUIRE(A && work && V, "fmlb_potri_f64: null pointer");
    FMLB_REQUIRE(n <= 65535, "fmlb_potri_f64: n=%d above 65535", n);
    FMLB_TRY(set_smem_attrs());
    const double *Linv = static_cast<const double *>(work);
    identity_kernel<<<dim3(ceil_div(n, 256), n), 256, 0, st>>>(V, ldv, n);
    FMLB_TRY(launch_status("identity_kernel"));
    for (int k0 = 0, kb = 0; k0 < n; k0 += NB, ++kb) {
        const int kn = std::min(NB, n - k0), R = k0 + kn;
        rows_trsm_kernel<<<ceil_div(R, TRSM_ROWS), TPB, kTrsmSmem, st>>>(
            V, ldv, R, k0, kn, Linv + (size_t)kb * NB * NB, info);
        FMLB_TRY(launch_status("rows_trsm_kernel"));
        if (R < n)
            FMLB_TRY(launch_gemm_nt<false>(V + R, ldv, R, n - R, V + k0, ldv,
                                           A + (size_t)R * lda + k0, lda, kn, info, st));
    }
    return launch_gemm_nt<true>(A, lda, n, n, V, ldv, V, ldv, n, info, st);
}
