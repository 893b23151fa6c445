// Plain-FP64 Gaussian and Laplacian kernel matrices by direct differences,
// the FP64 parity path of fkernels.f90:317-377.
//
// K_s[j, i] = exp(scale_s * sum_k f(A[j,k] - B[i,k])), f = square (Gaussian,
// scale = -0.5/sigma^2) or abs (Laplacian, scale = -1/sigma). Every sigma is
// emitted from one pass over the descriptors.
//
// Tiling: a 64x64 output tile per 256-thread CTA, descriptors staged through
// shared memory in k-chunks of 16, 4x4 outputs per thread with a stride-16
// mapping so global stores are coalesced. Symmetric mode launches only the
// tiles on or below the diagonal and writes the mirror through a shared-memory
// transpose.
#include <math.h>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, TPB = 256, MAXSIG = 32;

struct SigmaScales {
    double s[MAXSIG];
};

template <bool kL1>
__global__ void __launch_bounds__(TPB)
distance_kernel_f64(const double *__restrict__ A, int na, int lda, const double *__restrict__ B,
                    int nb, int ldb, int d, SigmaScales sc, int nsig, double *__restrict__ K,
                    long long ldk, long long sstride, int symmetric) {
    // the staging tiles and the transpose tile share one buffer: the
    // transpose is only used after the last k-chunk
    __shared__ double smem_raw[BM * (BN + 1)];
    double(*As)[BM + 1] = reinterpret_cast<double(*)[BM + 1]>(smem_raw);
    double(*Bs)[BN + 1] = reinterpret_cast<double(*)[BN + 1]>(smem_raw + BK * (BM + 1));
    double(*T)[BN + 1] = reinterpret_cast<double(*)[BN + 1]>(smem_raw);

    int by, bx;
    if (symmetric) {
        const long long t = blockIdx.x;
        by = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)by * (by + 1) / 2 > t) --by;
        while ((long long)(by + 1) * (by + 2) / 2 <= t) ++by;
        bx = (int)(t - (long long)by * (by + 1) / 2);
    } else {
        bx = blockIdx.x;
        by = blockIdx.y;
    }
    const int row0 = by * BM, col0 = bx * BN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;

    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

    // loader mapping: 16 consecutive k of one row per half-warp
    const int lk = threadIdx.x & 15, lr = threadIdx.x >> 4;  // lr in 0..15
    for (int k0 = 0; k0 < d; k0 += BK) {
        const int k = k0 + lk;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int ra = row0 + lr + 16 * r;
            As[lk][lr + 16 * r] = (ra < na && k < d) ? A[(size_t)ra * lda + k] : 0.0;
            const int rb = col0 + lr + 16 * r;
            Bs[lk][lr + 16 * r] = (rb < nb && k < d) ? B[(size_t)rb * ldb + k] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double t = a[i] - b[j];
                    if (kL1)
                        acc[i][j] += fabs(t);
                    else
                        acc[i][j] = fma(t, t, acc[i][j]);
                }
        }
        __syncthreads();
    }

    const bool mirror = symmetric && by > bx;
    for (int s = 0; s < nsig; ++s) {
        double *Ks = K + s * sstride;
        const double scale = sc.s[s];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = row0 + ty + 16 * i;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = col0 + tx + 16 * j;
                const double v = exp(scale * acc[i][j]);
                if (r < na && c < nb) Ks[(size_t)r * ldk + c] = v;
                if (mirror) T[tx + 16 * j][ty + 16 * i] = v;
            }
        }
        if (mirror) {
            __syncthreads();
            // T[c_local][r_local] -> K[col0 + c_local][row0 + r_local], coalesced in r
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int cl = ty + 16 * i;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int rl = tx + 16 * j;
                    const int gr = col0 + cl, gc = row0 + rl;
                    if (gr < nb && gc < na) Ks[(size_t)gr * ldk + gc] = T[cl][rl];
                }
            }
            __syncthreads();
        }
    }
}

template <bool kL1>
int launch_distance(const double *A, int na, int lda, const double *B, int nb, int ldb, int d,
                    const double *sigmas, int nsigma, double *K, long long ldk, long long sstride,
                    int symmetric, cudaStream_t st, const char *name) {
    FMLB_REQUIRE(na >= 0 && nb >= 0 && d >= 1, "%s: bad sizes na=%d nb=%d d=%d", name, na, nb, d);
    FMLB_REQUIRE(lda >= d && ldb >= d, "%s: leading dimension < d", name);
    FMLB_REQUIRE(ldk >= nb, "%s: ldk < nb", name);
    FMLB_REQUIRE(nsigma >= 1 && sigmas, "%s: need at least one sigma", name);
    FMLB_REQUIRE(nsigma == 1 || sstride >= (long long)na * ldk || sstride <= -(long long)na * ldk,
                 "%s: sigma_stride overlaps matrices", name);
    if (symmetric) FMLB_REQUIRE(A == B && na == nb && lda == ldb, "%s: symmetric needs A == B", name);
    if (na == 0 || nb == 0) return FMLB_OK;
    for (int s0 = 0; s0 < nsigma; s0 += MAXSIG) {
        const int ns = nsigma - s0 < MAXSIG ? nsigma - s0 : MAXSIG;
        SigmaScales sc;
        for (int s = 0; s < ns; ++s) {
            const double sg = sigmas[s0 + s];
            sc.s[s] = kL1 ? -1.0 / sg : -0.5 / (sg * sg);  // fkernels.f90:334 / :367
        }
        double *Ks = K + s0 * sstride;
        if (symmetric) {
            const long long nt = ceil_div(na, BM);
            const long long nblk = nt * (nt + 1) / 2;
            FMLB_REQUIRE(nblk < (1LL << 31), "%s: too many tiles", name);
            distance_kernel_f64<kL1><<<(unsigned)nblk, TPB, 0, st>>>(A, na, lda, B, nb, ldb, d, sc,
                                                                       ns, Ks, ldk, sstride, 1);
        } else {
            dim3 grid(ceil_div(nb, BN), ceil_div(na, BM));
            FMLB_REQUIRE(grid.y <= 65535, "%s: na too large for one launch", name);
            distance_kernel_f64<kL1><<<grid, TPB, 0, st>>>(A, na, lda, B, nb, ldb, d, sc, ns, Ks,
                                                             ldk, sstride, 0);
        }
        FMLB_TRY(launch_status(name));
    }
    return FMLB_OK;
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_gaussian_kernel_f64(const double *A, int na, int lda, const double *B, int nb,
                                        int ldb, int d, const double *sigmas_host, int nsigma,
                                        double *K, long long ldk, long long sigma_stride,
                                        int symmetric, void *stream) {
    return fmlb::launch_distance<false>(A, na, lda, B, nb, ldb, d, sigmas_host, nsigma, K, ldk,
                                        sigma_stride, symmetric, FMLB_STREAM(stream),
                                        "fmlb_gaussian_kernel_f64");
}

extern "C" int fmlb_laplacian_kernel_f64(const double *A, int na, int lda, const double *B, int nb,
                                         int ldb, int d, const double *sigmas_host, int nsigma,
                                         double *K, long long ldk, long long sigma_stride,
                                         int symmetric, void *stream) {
    return fmlb::launch_distance<true>(A, na, lda, B, nb, ldb, d, sigmas_host, nsigma, K, ldk,
                                       sigma_stride, symmetric, FMLB_STREAM(stream),
                                       "fmlb_laplacian_kernel_f64");
}
