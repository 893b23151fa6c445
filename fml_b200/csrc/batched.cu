// Batched KRR: many independent problems of uneven size (training size n,
// sigma, lambda per problem) trained and evaluated in ONE persistent launch.
//
// One CTA per SM pulls whole problems from a device work queue (problems are
// queued largest first); for each problem it runs the FP64 path of the
// reference's user-side KRR end to end, with CTA-level routines:
//   K = exp(-|x_i - x_j|^2 / (2 sigma^2)) (lower triangle, direct differences,
//   fgaussian_kernel fml/kernels/fkernels.f90:317-349), K + lambda I,
//   blocked Cholesky (64-column panels: shared-memory factor + inverse of the
//   diagonal block, panel solve, trailing update on the FP64 tensor cores),
//   the two triangular solves (fcho_solve.f90:35-42), and the prediction
//   sum_t k(x_q, x_t) alpha_t of the problem's test molecules.
// There are no dependencies between CTAs (each owns its problems), so the
// kernel cannot deadlock; a problem's LAPACK-style info goes to info[p].
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int BT = 64;     // tile / panel size
constexpr int BTPB = 256;  // threads (8 warps)

// kind 0: Gaussian kernel on descriptor rows (built here);
// kind 1: kernel matrix precomputed in buf (e.g. the ARAD kernel), lower
//         triangle used; the test kernel (nt x n) precomputed at ktest.
struct BatchProblem {
    long long x_train;   // row offset of the training descriptors in X
    long long x_test;    // row offset of the test descriptors
    long long y;         // offset of the training targets in Y
    long long pred;      // offset of the predictions
    long long kbuf;      // offset (doubles) of this problem's n x n matrix
    long long work;      // offset (doubles) of the inverted diagonal blocks + vectors
    long long ktest;     // kind 1: offset (doubles) of the nt x n test kernel
    int n, nt, kind, pad;
    double sigma, lambda;
};

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

struct BatchSmem {
    double a[BT][BT + 1];   // tile / diagonal block
    double b[BT][BT + 1];   // second operand / inverse
    double v[2 * BT];
    int bad;
    int prob;
};

// ---- K build: lower-triangle tiles, direct FP64 differences -------------------
__device__ void cta_gauss_build(BatchSmem &sm, const double *__restrict__ X, int ldx, int d, int n,
                                double scale, double lambda, double *__restrict__ K) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int nt = (n + BT - 1) / BT;
    for (int bi = 0; bi < nt; ++bi) {
        for (int bj = 0; bj <= bi; ++bj) {
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int k0 = 0; k0 < d; k0 += BT) {
                __syncthreads();
                for (int t = tid; t < BT * BT; t += BTPB) {
                    const int r = t / BT, kk = t % BT;
                    const int ra = bi * BT + r, rb = bj * BT + r, k = k0 + kk;
                    sm.a[kk][r] = (ra < n && k < d) ? X[(size_t)ra * ldx + k] : 0.0;
                    sm.b[kk][r] = (rb < n && k < d) ? X[(size_t)rb * ldx + k] : 0.0;
                }
                __syncthreads();
                const int kmax = min(BT, d - k0);
                for (int kk = 0; kk < kmax; ++kk) {
                    double av[4], bv[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) av[i] = sm.a[kk][ty + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; ++j) bv[j] = sm.b[kk][tx + 16 * j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const double t = av[i] - bv[j];
                            acc[i][j] = fma(t, t, acc[i][j]);
                        }
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = bi * BT + ty + 16 * i;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = bj * BT + tx + 16 * j;
                    if (r < n && c <= r) {
                        double v = exp(scale * acc[i][j]);
                        if (r == c) v += lambda;
                        K[(size_t)r * n + c] = v;
                    }
                }
            }
        }
    }
    __syncthreads();
}

// ---- Cholesky ----------------------------------------------------------------
// diagonal block at (k0, k0), kn <= 64 columns: factor in sm.a, inverse in sm.b
__device__ bool cta_potf2(BatchSmem &sm, double *__restrict__ K, int n, int k0, int kn,
                          double *__restrict__ Linv, int *info) {
    const int tid = threadIdx.x;
    __syncthreads();
    for (int t = tid; t < BT * BT; t += BTPB) {
        const int r = t / BT, c = t % BT;
        double v = 0.0;
        if (r < kn && c <= r) v = K[(size_t)(k0 + r) * n + k0 + c];
        else if (r == c) v = 1.0;
        sm.a[r][c] = v;
    }
    if (tid == 0) sm.bad = 0;
    __syncthreads();
    for (int j = 0; j < BT; ++j) {
        const double dj = sm.a[j][j];
        if (!(dj > 0.0)) {
            if (tid == 0) sm.bad = k0 + j + 1;
            break;
        }
        const double r = sqrt(dj), inv = 1.0 / r;
        __syncthreads();
        if (tid == 0) sm.a[j][j] = r;
        for (int i = j + 1 + tid; i < BT; i += BTPB) sm.a[i][j] *= inv;
        __syncthreads();
        const int m = BT - j - 1;
        for (int t = tid; t < m * m; t += BTPB) {
            const int i = j + 1 + t / m, c = j + 1 + t % m;
            if (c <= i) sm.a[i][c] = fma(-sm.a[i][j], sm.a[c][j], sm.a[i][c]);
        }
        __syncthreads();
    }
    __syncthreads();
    if (sm.bad) {
        if (tid == 0 && *info == 0) *info = sm.bad;
        return false;
    }
    // inverse: column c solves L x = e_c (threads 0..63, one column each)
    if (tid < BT) {
        const int c = tid;
        for (int i = 0; i < BT; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = c; k < i; ++k) s = fma(-sm.a[i][k], sm.b[k][c], s);
            sm.b[i][c] = (i < c) ? 0.0 : s / sm.a[i][i];
        }
    }
    __syncthreads();
    for (int t = tid; t < BT * BT; t += BTPB) {
        const int r = t / BT, c = t % BT;
        if (r < kn && c <= r) K[(size_t)(k0 + r) * n + k0 + c] = sm.a[r][c];
        Linv[t] = sm.b[r][c];
    }
    __syncthreads();
    return true;
}

// rows [k0+kn, n) of the panel: X <- X Linv^T (Linv in sm.b)
__device__ void cta_trsm(BatchSmem &sm, double *__restrict__ K, int n, int k0, int kn) {
    const int tid = threadIdx.x;
    for (int r0 = k0 + kn; r0 < n; r0 += BT) {
        __syncthreads();
        for (int t = tid; t < BT * BT; t += BTPB) {
            const int r = t / BT, c = t % BT;
            sm.a[r][c] = (r0 + r < n && c < kn) ? K[(size_t)(r0 + r) * n + k0 + c] : 0.0;
        }
        __syncthreads();
        const int c = tid & (BT - 1), rq = tid >> 6;  // 4 groups of 16 rows
        double out[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) out[i] = 0.0;
        for (int k = 0; k <= c; ++k) {
            const double l = sm.b[c][k];
#pragma unroll
            for (int i = 0; i < 16; ++i) out[i] = fma(sm.a[rq * 16 + i][k], l, out[i]);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = r0 + rq * 16 + i;
            if (r < n && c < kn) K[(size_t)r * n + k0 + c] = out[i];
        }
    }
    __syncthreads();
}

// trailing update C -= P P^T on the lower tiles past the panel, FP64 tensor
// cores: 8 warps as 4 x 2, warp tile 16 x 32 (2 x 4 m8n8 fragments)
__device__ void cta_syrk(BatchSmem &sm, double *__restrict__ K, int n, int k0, int kn) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wr = warp >> 1, wc = warp & 1, g = lane >> 2, tq = lane & 3;
    const int base = k0 + kn;
    const int m = n - base;
    const int nt = (m + BT - 1) / BT;
    for (int bi = 0; bi < nt; ++bi) {
        for (int bj = 0; bj <= bi; ++bj) {
            __syncthreads();
            for (int t = tid; t < BT * BT; t += BTPB) {
                const int r = t / BT, c = t % BT;
                const int ra = base + bi * BT + r, rb = base + bj * BT + r;
                sm.a[r][c] = (ra < n && c < kn) ? K[(size_t)ra * n + k0 + c] : 0.0;
                sm.b[r][c] = (rb < n && c < kn) ? K[(size_t)rb * n + k0 + c] : 0.0;
            }
            __syncthreads();
            double acc[2][4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
            for (int kk = 0; kk < BT; kk += 4) {
                double av[2], bv[4];
#pragma unroll
                for (int i = 0; i < 2; ++i) av[i] = sm.a[wr * 16 + i * 8 + g][kk + tq];
#pragma unroll
                for (int j = 0; j < 4; ++j) bv[j] = sm.b[wc * 32 + j * 8 + g][kk + tq];
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], av[i], bv[j]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = base + bi * BT + wr * 16 + i * 8 + g;
                if (r >= n) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = base + bj * BT + wc * 32 + j * 8 + 2 * tq;
                    double *p = K + (size_t)r * n + c;
                    if (c <= r) p[0] -= acc[i][j][0];
                    if (c + 1 <= r) p[1] -= acc[i][j][1];
                }
            }
        }
    }
    __syncthreads();
}

// x <- (L L^T)^-1 x with the stored inverted diagonal blocks
__device__ void cta_potrs(BatchSmem &sm, const double *__restrict__ L, int n,
                          const double *__restrict__ Linv, double *__restrict__ x) {
    const int tid = threadIdx.x;
    const int nb = (n + BT - 1) / BT;
    // forward: y_k = Linv_k (x_k - sum_{j<k} L_kj y_j), y kept in x
    for (int kb = 0; kb < nb; ++kb) {
        const int k0 = kb * BT, kn = min(BT, n - k0);
        __syncthreads();
        if (tid < kn) {
            double s = x[k0 + tid];
            for (int c = 0; c < k0; ++c) s = fma(-L[(size_t)(k0 + tid) * n + c], x[c], s);
            sm.v[tid] = s;
        }
        __syncthreads();
        if (tid < kn) {
            const double *li = Linv + (size_t)kb * BT * BT + tid * BT;
            double s = 0.0;
            for (int c = 0; c <= tid; ++c) s = fma(li[c], sm.v[c], s);
            x[k0 + tid] = s;
        }
    }
    // backward: x_k = Linv_k^T (y_k - sum_{j>k} L_jk^T x_j)
    for (int kb = nb - 1; kb >= 0; --kb) {
        const int k0 = kb * BT, kn = min(BT, n - k0);
        __syncthreads();
        if (tid < kn) {
            double s = x[k0 + tid];
            for (int r = k0 + kn; r < n; ++r) s = fma(-L[(size_t)r * n + k0 + tid], x[r], s);
            sm.v[tid] = s;
        }
        __syncthreads();
        if (tid < kn) {
            double s = 0.0;
            for (int r = tid; r < kn; ++r) s = fma(Linv[(size_t)kb * BT * BT + r * BT + tid], sm.v[r], s);
            x[k0 + tid] = s;
        }
    }
    __syncthreads();
}

// pred[q] = sum_t exp(scale |xq - xt|^2) alpha_t
__device__ void cta_predict(BatchSmem &sm, const double *__restrict__ X, int ldx, int d,
                            long long xq, int nq, long long xt, int n, double scale,
                            const double *__restrict__ alpha, double *__restrict__ pred) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int q0 = 0; q0 < nq; q0 += BT) {
        double out[4] = {0.0, 0.0, 0.0, 0.0};
        for (int t0 = 0; t0 < n; t0 += BT) {
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int k0 = 0; k0 < d; k0 += BT) {
                __syncthreads();
                for (int t = tid; t < BT * BT; t += BTPB) {
                    const int r = t / BT, kk = t % BT;
                    const int ra = q0 + r, rb = t0 + r, k = k0 + kk;
                    sm.a[kk][r] = (ra < nq && k < d) ? X[(size_t)(xq + ra) * ldx + k] : 0.0;
                    sm.b[kk][r] = (rb < n && k < d) ? X[(size_t)(xt + rb) * ldx + k] : 0.0;
                }
                __syncthreads();
                const int kmax = min(BT, d - k0);
                for (int kk = 0; kk < kmax; ++kk) {
                    double av[4], bv[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) av[i] = sm.a[kk][ty + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; ++j) bv[j] = sm.b[kk][tx + 16 * j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const double t = av[i] - bv[j];
                            acc[i][j] = fma(t, t, acc[i][j]);
                        }
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = t0 + tx + 16 * j;
                if (c < n) {
                    const double a = alpha[c];
#pragma unroll
                    for (int i = 0; i < 4; ++i) out[i] = fma(exp(scale * acc[i][j]), a, out[i]);
                }
            }
        }
        // reduce over the 16 threads of a row group (tx), fixed order
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            double v = out[i];
            for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int r = q0 + ty + 16 * i;
            if (tx == 0 && r < nq) pred[r] = v;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(BTPB, 1)
krr_batched_kernel(const BatchProblem *__restrict__ probs, const int *__restrict__ order,
                   int nprob, int *__restrict__ counter, const double *__restrict__ X, int ldx,
                   int d, const double *__restrict__ Y, double *__restrict__ pred,
                   double *__restrict__ buf, int *__restrict__ info) {
    extern __shared__ __align__(16) uint8_t bsm_raw[];
    BatchSmem &sm = *reinterpret_cast<BatchSmem *>(bsm_raw);
    const int tid = threadIdx.x;
    for (;;) {
        __syncthreads();
        if (tid == 0) sm.prob = atomicAdd(counter, 1);
        __syncthreads();
        const int qi = sm.prob;
        if (qi >= nprob) break;
        const int p = order[qi];
        const BatchProblem pr = probs[p];
        const int n = pr.n;
        double *K = buf + pr.kbuf;
        double *Linv = buf + pr.work;
        double *alpha = Linv + (size_t)((n + BT - 1) / BT) * BT * BT;
        const double scale = -0.5 / (pr.sigma * pr.sigma);
        if (pr.kind == 0) {
            cta_gauss_build(sm, X + (size_t)pr.x_train * ldx, ldx, d, n, scale, pr.lambda, K);
        } else {
            for (int t = tid; t < n; t += BTPB) K[(size_t)t * n + t] += pr.lambda;
            __syncthreads();
        }
        bool ok = true;
        for (int k0 = 0; k0 < n && ok; k0 += BT) {
            const int kn = min(BT, n - k0);
            ok = cta_potf2(sm, K, n, k0, kn, Linv + (size_t)(k0 / BT) * BT * BT, &info[p]);
            if (!ok) break;
            cta_trsm(sm, K, n, k0, kn);
            cta_syrk(sm, K, n, k0, kn);
        }
        for (int t = tid; t < n; t += BTPB) alpha[t] = Y[pr.y + t];
        __syncthreads();
        if (ok) cta_potrs(sm, K, n, Linv, alpha);
        if (pr.kind == 0) {
            cta_predict(sm, X, ldx, d, pr.x_test, pr.nt, pr.x_train, n, scale, alpha,
                        pred + pr.pred);
        } else {  // pred = K_test alpha, one warp per test row
            const double *Kt = buf + pr.ktest;
            const int warp = tid >> 5, lane = tid & 31;
            for (int q = warp; q < pr.nt; q += BTPB / 32) {
                double v = 0.0;
                for (int t = lane; t < n; t += 32) v = fma(Kt[(size_t)q * n + t], alpha[t], v);
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) pred[pr.pred + q] = v;
            }
            __syncthreads();
        }
    }
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_batch_problem_bytes(void) { return sizeof(fmlb::BatchProblem); }

extern "C" size_t fmlb_batch_buffer_doubles(int n) {
    if (n <= 0) return 0;
    const size_t nb = (size_t)(n + fmlb::BT - 1) / fmlb::BT;
    return (size_t)n * n + nb * fmlb::BT * fmlb::BT + (size_t)n;
}

extern "C" int fmlb_krr_batched_f64(const void *problems, const int *order, int nprob,
                                    int *counter, const double *X, int ldx, int d,
                                    const double *Y, double *pred, double *buf, int *info,
                                    int grid, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(nprob >= 0 && d >= 1 && ldx >= d, "fmlb_krr_batched_f64: bad sizes");
    if (nprob == 0) return FMLB_OK;
    FMLB_REQUIRE(problems && order && counter && X && Y && pred && buf && info,
                 "fmlb_krr_batched_f64: null pointer");
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_krr_batched_f64: cudaGetDevice"));
    if (attr_dev != dev) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(krr_batched_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)sizeof(BatchSmem)),
                             "fmlb_krr_batched_f64: smem attribute"));
        attr_dev = dev;
    }
    if (grid <= 0) grid = sm_count();
    FMLB_TRY(cuda_status(cudaMemsetAsync(counter, 0, sizeof(int), st), "clear counter"));
    krr_batched_kernel<<<grid, BTPB, sizeof(BatchSmem), st>>>(
        static_cast<const BatchProblem *>(problems), order, nprob, counter, X, ldx, d, Y, pred,
        buf, info);
    return launch_status("krr_batched_kernel");
}
