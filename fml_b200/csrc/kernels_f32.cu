// Laplacian kernel matrix in FP32, the mixed-precision form of
// flaplacian_kernel (fml/kernels/fkernels.f90:351-377):
//
//   K_s[j, i] = exp(-1/sigma_s * sum_k |A[j,k] - B[i,k]|)
//
// CUDA-core kernel (the L1 distance is not a contraction): 128 x 128 output
// tile per 256-thread CTA, FP64 descriptors converted to FP32 while staged
// through shared memory in k-chunks of 32 (the row operand negated), 8 x 8
// outputs per thread as 8 x 4 column pairs in packed FP32x2 arithmetic
// (b - a and the abs-add, two terms per instruction; operands fetched as
// float4), every sigma emitted from one pass. b + (-a) is a - b negated
// exactly, so the sums equal the scalar |a - b| accumulation bit for bit. The next k-chunk's global loads are issued into registers
// before the current chunk is computed, so their latency hides under the
// arithmetic. Symmetric builds compute the tiles on or below the diagonal and
// write the mirror through a shared-memory transpose.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int LB = 128, LK = 32, LTPB = 256, LMAXSIG = 8, LPAD = 4;
constexpr size_t kLapSmem = (size_t)LB * (LB + 1) * sizeof(float);  // transpose tile (>= stages)

struct LapScales {
    float s[LMAXSIG];  // -log2(e) / sigma
};

__global__ void __launch_bounds__(LTPB, 2)
laplacian_f32_kernel(const double *__restrict__ A, int na, int lda, const double *__restrict__ B,
                     int nb, int ldb, int d, const __grid_constant__ LapScales sc, int nsig,
                     float *__restrict__ K,
                     long long ldk, long long sstride, int symmetric) {
    extern __shared__ float lap_smem[];
    float(*As)[LB + LPAD] = reinterpret_cast<float(*)[LB + LPAD]>(lap_smem);
    float(*Bs)[LB + LPAD] = reinterpret_cast<float(*)[LB + LPAD]>(lap_smem + LK * (LB + LPAD));
    float(*T)[LB + 1] = reinterpret_cast<float(*)[LB + 1]>(lap_smem);

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
    const int row0 = by * LB, col0 = bx * LB;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;

    float2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.0f, 0.0f);

    // loader: 32 consecutive k of one row per warp, 8 rows per pass; the
    // chunk is held in registers (converted) until the previous one is done
    const int lk = threadIdx.x & 31, lr = threadIdx.x >> 5;
    float pa[LB / 8], pb[LB / 8];
    auto fetch = [&](int k0) {
        const int k = k0 + lk;
#pragma unroll
        for (int r = 0; r < LB / 8; ++r) {
            const int rr = lr + 8 * r;
            const int ra = row0 + rr, rb = col0 + rr;
            pa[r] = (ra < na && k < d) ? (float)A[(size_t)ra * lda + k] : 0.0f;
            pb[r] = (rb < nb && k < d) ? (float)B[(size_t)rb * ldb + k] : 0.0f;
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < d; k0 += LK) {
#pragma unroll
        for (int r = 0; r < LB / 8; ++r) {
            As[lk][lr + 8 * r] = -pa[r];
            Bs[lk][lr + 8 * r] = pb[r];
        }
        __syncthreads();
        if (k0 + LK < d) fetch(k0 + LK);  // in flight during the arithmetic below
#pragma unroll 2
        for (int kk = 0; kk < LK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[kk][ty * 8]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[kk][ty * 8 + 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 8]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 8 + 4]);
            const float na[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};  // -A
            const float2 b2[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w),
                                  make_float2(b1.x, b1.y), make_float2(b1.z, b1.w)};
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float2 na2 = make_float2(na[i], na[i]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 dd = __fadd2_rn(b2[j], na2);
                    acc[i][j] = __fadd2_rn(acc[i][j], make_float2(fabsf(dd.x), fabsf(dd.y)));
                }
            }
        }
        __syncthreads();
    }

    // epilogue through shared memory: the L1 sums go to T once, then every
    // sigma is written with coalesced stores (and the mirror, column-wise)
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T[ty * 8 + i][tx * 8 + 2 * j] = acc[i][j].x;
            T[ty * 8 + i][tx * 8 + 2 * j + 1] = acc[i][j].y;
        }
    __syncthreads();
    const bool mirror = symmetric && by > bx;
    for (int s = 0; s < nsig; ++s) {
        float *Ks = K + s * sstride;
        const float c = sc.s[s];
        for (int e = threadIdx.x; e < LB * LB; e += LTPB) {
            const int rl = e >> 7, cl = e & (LB - 1);
            const int r = row0 + rl, col = col0 + cl;
            if (r < na && col < nb) {
                float v;
                asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(v) : "f"(T[rl][cl] * c));
                Ks[(size_t)r * ldk + col] = v;
            }
        }
        if (mirror) {
            for (int e = threadIdx.x; e < LB * LB; e += LTPB) {
                const int cl = e >> 7, rl = e & (LB - 1);
                const int gr = col0 + cl, gc = row0 + rl;
                if (gr < nb && gc < na) {
                    float v;
                    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(v) : "f"(T[rl][cl] * c));
                    Ks[(size_t)gr * ldk + gc] = v;
                }
            }
        }
    }
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_laplacian_kernel_f32(const double *A, int na, int lda, const double *B, int nb,
                                         int ldb, int d, const double *sigmas_host, int nsigma,
                                         float *K, long long ldk, long long sigma_stride,
                                         int symmetric, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(na >= 0 && nb >= 0 && d >= 1 && lda >= d && ldb >= d,
                 "fmlb_laplacian_kernel_f32: bad sizes");
    FMLB_REQUIRE(ldk >= nb, "fmlb_laplacian_kernel_f32: ldk < nb");
    FMLB_REQUIRE(nsigma >= 1 && sigmas_host, "fmlb_laplacian_kernel_f32: need at least one sigma");
    if (symmetric)
        FMLB_REQUIRE(A == B && na == nb && lda == ldb,
                     "fmlb_laplacian_kernel_f32: symmetric needs A == B");
    if (na == 0 || nb == 0) return FMLB_OK;
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_laplacian_kernel_f32: cudaGetDevice"));
    if (attr_dev != dev) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(laplacian_f32_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kLapSmem),
                             "fmlb_laplacian_kernel_f32: smem attribute"));
        attr_dev = dev;
    }
    for (int s0 = 0; s0 < nsigma; s0 += LMAXSIG) {
        const int ns = std::min(LMAXSIG, nsigma - s0);
        LapScales sc;
        for (int s = 0; s < ns; ++s) sc.s[s] = (float)(-1.4426950408889634 / sigmas_host[s0 + s]);
        float *Ks = K + (long long)s0 * sigma_stride;
        if (symmetric) {
            const long long nt = ceil_div(na, LB);
            laplacian_f32_kernel<<<(unsigned)(nt * (nt + 1) / 2), LTPB, kLapSmem, st>>>(
                A, na, lda, B, nb, ldb, d, sc, ns, Ks, ldk, sigma_stride, 1);
        } else {
            dim3 grid(ceil_div(nb, LB), ceil_div(na, LB));
            laplacian_f32_kernel<<<grid, LTPB, kLapSmem, st>>>(A, na, lda, B, nb, ldb, d, sc, ns, Ks,
                                                                ldk, sigma_stride, 0);
        }
        FMLB_TRY(launch_status("laplacian_f32_kernel"));
    }
    return FMLB_OK;
}
