// Gaussian kernel matrix on the 5th-generation tensor cores (tcgen05), the
// mixed-precision form of fgaussian_kernel (fml/kernels/fkernels.f90:317-349):
//
//   K_s[i, j] = exp(-(|x_i|^2 + |x_j|^2 - 2 x_i . x_j) / (2 sigma_s^2))
//
// on mean-centred descriptors, with x . y from BF16 hi/lo splits
// (x = hi + lo): x.y ~ hi.hi + hi.lo + lo.hi, three BF16 MMAs accumulated in
// FP32 in tensor memory, and every sigma emitted by the epilogue.
//
// Structure (one persistent CTA per SM, 192 threads):
//   warp 0      TMA producer: per k-chunk of 64, four 128 x 64 BF16 tiles
//               (A hi, A lo, B hi, B lo), 128B-swizzled, into a 3-stage ring;
//   warp 1      allocates 256 TMEM columns (two 128 x 128 FP32 accumulators)
//               and one thread issues tcgen05.mma (M=128, N=128, K=16);
//   warps 2..5  epilogue: tcgen05.ld of their 32-lane quarter, d^2, exp for
//               every sigma, FP32 stores (and the mirrored tile for
//               symmetric builds), overlapping the next tile's MMAs.
// Every mbarrier wait is bounded; a wait that runs out records an error code
// in *status and the CTA winds down instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 64, TC_STAGES = 3, TC_THREADS = 192;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 2;          // 16 KB per operand tile
constexpr int TC_STAGE_BYTES = 4 * TC_TILE_BYTES;          // A hi, A lo, B hi, B lo
constexpr int TC_TMEM_COLS = 2 * TC_BN;
constexpr int TC_MAXSIG = 8;
constexpr size_t kTcSmem = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024 /* align */ + 256;
constexpr long long kWaitBudget = 4000000000LL;            // clock cycles (~2 s)

enum TcStatus { TC_OK = 0, TC_TIMEOUT_FULL = 1, TC_TIMEOUT_EMPTY = 2, TC_TIMEOUT_TMEM = 3 };

struct TcParams {
    float scale[TC_MAXSIG];  // -log2(e) / (2 sigma^2)
    int nsig;
    int na, nb;              // logical rows of A and B
    int ntile_a, ntile_b;    // 128-row tiles of A and B
    int nk;                  // k-chunks of 64
    int symmetric;
    long long ldk, sstride;  // output row stride and sigma stride (elements)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `bar` with the given parity; false after the budget.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kWaitBudget) return false;
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart, descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc_sw128(const void *p) {
    const uint64_t addr = smem_u32(p);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;        // start address
    d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;              // version
    d |= (uint64_t)2 << 61;              // 128-byte swizzle
    return d;
}

// Instruction descriptor, kind::f16: BF16 A and B, FP32 accumulator, both
// K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                            ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void tile_coords(int t, const TcParams &p, int &ta, int &tb) {
    if (p.symmetric) {  // lower triangle of tiles, row-major: ta >= tb
        int r = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
        while (r * (r + 1) / 2 > t) --r;
        while ((r + 1) * (r + 2) / 2 <= t) ++r;
        ta = r;
        tb = t - r * (r + 1) / 2;
    } else {
        ta = t / p.ntile_b;
        tb = t % p.ntile_b;
    }
}

__device__ __forceinline__ float fast_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__global__ void __launch_bounds__(TC_THREADS, 1)
gauss_tc_kernel(const __grid_constant__ CUtensorMap mapAhi, const __grid_constant__ CUtensorMap mapAlo,
                const __grid_constant__ CUtensorMap mapBhi, const __grid_constant__ CUtensorMap mapBlo,
                const float *__restrict__ normA, const float *__restrict__ normB, TcParams p,
                float *__restrict__ K, int *__restrict__ status) {
    extern __shared__ uint8_t tc_smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TC_STAGES * TC_STAGE_BYTES);
    uint64_t *full = bars, *empty = bars + TC_STAGES;
    uint64_t *tmem_full = bars + 2 * TC_STAGES, *tmem_empty = tmem_full + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tmem_empty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = p.symmetric ? p.ntile_a * (p.ntile_a + 1) / 2 : p.ntile_a * p.ntile_b;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tmem_full[a], 1);
            mbar_init(&tmem_empty[a], 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int ta, tb;
                tile_coords(t, p, ta, tb);
                for (int kc = 0; kc < p.nk; ++kc) {
                    if (!mbar_wait(&empty[stage], phase ^ 1)) {
                        atomicCAS(status, 0, TC_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + stage * TC_STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], TC_STAGE_BYTES);
                    tma_load_2d(st, &mapAhi, &full[stage], kc * TC_BK, ta * TC_BM);
                    tma_load_2d(st + TC_TILE_BYTES, &mapAlo, &full[stage], kc * TC_BK, ta * TC_BM);
                    tma_load_2d(st + 2 * TC_TILE_BYTES, &mapBhi, &full[stage], kc * TC_BK,
                                tb * TC_BN);
                    tma_load_2d(st + 3 * TC_TILE_BYTES, &mapBlo, &full[stage], kc * TC_BK,
                                tb * TC_BN);
                    if (++stage == TC_STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int lt = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++lt) {
                const int acc = lt & 1;
                const uint32_t acc_phase = (lt >> 1) & 1;
                if (!mbar_wait(&tmem_empty[acc], acc_phase ^ 1)) {
                    atomicCAS(status, 0, TC_TIMEOUT_TMEM);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t dacc = tmem_base + (uint32_t)(acc * TC_BN);
                for (int kc = 0; kc < p.nk; ++kc) {
                    if (!mbar_wait(&full[stage], phase)) {
                        atomicCAS(status, 0, TC_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    uint8_t *st = smem + stage * TC_STAGE_BYTES;
                    const uint64_t ahi = smem_desc_sw128(st);
                    const uint64_t alo = smem_desc_sw128(st + TC_TILE_BYTES);
                    const uint64_t bhi = smem_desc_sw128(st + 2 * TC_TILE_BYTES);
                    const uint64_t blo = smem_desc_sw128(st + 3 * TC_TILE_BYTES);
#pragma unroll
                    for (int k = 0; k < TC_BK / 16; ++k) {
                        // advance 16 BF16 = 32 bytes inside the 128-byte swizzle row
                        const uint64_t off = (uint64_t)((k * 32) >> 4);
                        const uint32_t first = (kc == 0 && k == 0) ? 0u : 1u;
                        mma_bf16(dacc, ahi + off, bhi + off, first);
                        mma_bf16(dacc, ahi + off, blo + off, 1u);
                        mma_bf16(dacc, alo + off, bhi + off, 1u);
                    }
                    mma_commit(&empty[stage]);  // frees the stage once these MMAs finish
                    if (++stage == TC_STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                mma_commit(&tmem_full[acc]);
            }
        }
    } else {
        // --------------------------------------------------------------- epilogue
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int row_local = q * 32 + lane;
        const bool vec_ok = ((p.ldk & 3) == 0) && ((p.sstride & 3) == 0) &&
                            ((reinterpret_cast<uintptr_t>(K) & 15) == 0);
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++lt) {
            int ta, tb;
            tile_coords(t, p, ta, tb);
            const int acc = lt & 1;
            const uint32_t acc_phase = (lt >> 1) & 1;
            if (!mbar_wait(&tmem_full[acc], acc_phase)) {
                atomicCAS(status, 0, TC_TIMEOUT_TMEM);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int grow = ta * TC_BM + row_local;
            const bool row_ok = grow < p.na;
            const float nr = row_ok ? normA[grow] : 0.0f;
            const bool diag_tile = p.symmetric && ta == tb;
            for (int c0 = 0; c0 < TC_BN; c0 += 32) {
                uint32_t v[32];
                tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * TC_BN + c0), v);
                const int gcol0 = tb * TC_BN + c0;
                float d2[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int gcol = gcol0 + j;
                    const float nc = gcol < p.nb ? normB[gcol] : 0.0f;
                    float x = fmaxf(nr + nc - 2.0f * __uint_as_float(v[j]), 0.0f);
                    if (diag_tile && gcol == grow) x = 0.0f;  // exact zero distance
                    d2[j] = x;
                }
                if (!row_ok) continue;
                for (int s = 0; s < p.nsig; ++s) {
                    const float sc = p.scale[s];
                    float *Ks = K + s * p.sstride;
#pragma unroll
                    for (int j4 = 0; j4 < 32; j4 += 4) {
                        float kv[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) kv[i] = fast_exp2(d2[j4 + i] * sc);
                        const int gcol = gcol0 + j4;
                        // direct tile: on diagonal tiles only the lower triangle (c <= r)
                        const bool full4 = gcol + 3 < p.nb && (!diag_tile || gcol + 3 <= grow);
                        if (full4 && vec_ok) {
                            *reinterpret_cast<float4 *>(Ks + (size_t)grow * p.ldk + gcol) =
                                make_float4(kv[0], kv[1], kv[2], kv[3]);
                        } else {
#pragma unroll
                            for (int i = 0; i < 4; ++i)
                                if (gcol + i < p.nb && (!diag_tile || gcol + i <= grow))
                                    Ks[(size_t)grow * p.ldk + gcol + i] = kv[i];
                        }
                        // mirrored tile: lanes hold consecutive rows -> coalesced stores
                        if (p.symmetric) {
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const int c = gcol + i;
                                if (c < p.nb && (!diag_tile || c < grow))
                                    Ks[(size_t)c * p.ldk + grow] = kv[i];
                            }
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tmem_empty[acc]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                     "r"(TC_TMEM_COLS));
}

// ---- operand preparation ----------------------------------------------------
// hi = bf16(x - mu), lo = bf16(x - mu - hi), norms = |x - mu|^2 (FP64 -> FP32);
// rows past n and columns past d are zero.
__global__ void split_center_kernel(const double *__restrict__ X, int n, int ldx, int d,
                                    const double *__restrict__ mu, int n_pad, int d_pad,
                                    __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                    float *__restrict__ norms) {
    const int row = blockIdx.x;
    if (row >= n_pad) return;
    double acc = 0.0;
    for (int k = threadIdx.x; k < d_pad; k += blockDim.x) {
        double v = 0.0;
        if (row < n && k < d) v = X[(size_t)row * ldx + k] - mu[k];
        const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        const __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
        hi[(size_t)row * d_pad + k] = h;
        lo[(size_t)row * d_pad + k] = l;
        acc += v * v;
    }
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) norms[row] = (float)v;
    }
}

// column means of X (n rows), one thread per column
__global__ void column_mean_kernel(const double *__restrict__ X, int n, int ldx, int d,
                                   double *__restrict__ mu) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += X[(size_t)i * ldx + k];
    mu[k] = n ? s / n : 0.0;
}

// ---- host: tensor maps --------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

int make_map(CUtensorMap *m, const void *base, int rows, int cols) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is unavailable");
        return FMLB_ECUDA;
    }
    FMLB_REQUIRE(((uintptr_t)base % 16) == 0, "tensor base not 16-byte aligned");
    FMLB_REQUIRE(cols % TC_BK == 0 && rows % TC_BM == 0, "padded operand shape");
    const cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t gstride[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {TC_BK, TC_BM};
    const cuuint32_t estride[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), gdim,
                    gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return FMLB_ECUDA;
    }
    return FMLB_OK;
}

struct SplitView {
    __nv_bfloat16 *hi, *lo;
    float *norms;
    int n_pad, d_pad;
};

}  // namespace
}  // namespace fmlb

// Workspace of one operand set: hi and lo BF16 (n_pad x d_pad) + FP32 norms.
extern "C" size_t fmlb_tc_operand_bytes(int n, int d) {
    if (n <= 0 || d <= 0) return 256;
    const size_t n_pad = (size_t)(n + 127) / 128 * 128, d_pad = (size_t)(d + 63) / 64 * 64;
    return 2 * n_pad * d_pad * 2 + n_pad * 4 + 512;
}

static int prepare_operand(const double *X, int n, int ldx, int d, const double *mu, void *ws,
                           fmlb::SplitView &v, cudaStream_t st) {
    using namespace fmlb;
    v.n_pad = (n + 127) / 128 * 128;
    v.d_pad = (d + 63) / 64 * 64;
    char *p = static_cast<char *>(ws);
    p = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(p) + 255) & ~(uintptr_t)255);
    v.hi = reinterpret_cast<__nv_bfloat16 *>(p);
    v.lo = v.hi + (size_t)v.n_pad * v.d_pad;
    v.norms = reinterpret_cast<float *>(v.lo + (size_t)v.n_pad * v.d_pad);
    split_center_kernel<<<v.n_pad, 128, 0, st>>>(X, n, ldx, d, mu, v.n_pad, v.d_pad, v.hi, v.lo,
                                                  v.norms);
    return launch_status("split_center_kernel");
}

extern "C" int fmlb_column_mean_f64(const double *X, int n, int ldx, int d, double *mu,
                                    void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(n >= 0 && d >= 1 && ldx >= d && mu, "fmlb_column_mean_f64: bad arguments");
    column_mean_kernel<<<ceil_div(d, 128), 128, 0, FMLB_STREAM(stream)>>>(X, n, ldx, d, mu);
    return launch_status("column_mean_kernel");
}

extern "C" int fmlb_gaussian_kernel_tc(const double *A, int na, int lda, const double *B, int nb,
                                       int ldb, int d, const double *mu, const double *sigmas_host,
                                       int nsigma, float *K, long long ldk,
                                       long long sigma_stride, int symmetric, void *workspace,
                                       size_t ws_bytes, int *status, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(na >= 0 && nb >= 0 && d >= 1 && lda >= d && ldb >= d,
                 "fmlb_gaussian_kernel_tc: bad sizes");
    FMLB_REQUIRE(nsigma >= 1 && nsigma <= TC_MAXSIG && sigmas_host,
                 "fmlb_gaussian_kernel_tc: nsigma must be 1..%d", TC_MAXSIG);
    FMLB_REQUIRE(ldk >= nb, "fmlb_gaussian_kernel_tc: ldk < nb");
    FMLB_REQUIRE(nsigma == 1 || sigma_stride >= (long long)(na - 1) * ldk + nb,
                 "fmlb_gaussian_kernel_tc: sigma_stride %lld overlaps the previous sigma's "
                 "(na - 1) * ldk + nb = %lld elements", sigma_stride,
                 (long long)(na - 1) * ldk + nb);
    FMLB_REQUIRE(mu && status && K, "fmlb_gaussian_kernel_tc: null pointer");
    if (symmetric)
        FMLB_REQUIRE(A == B && na == nb && lda == ldb, "fmlb_gaussian_kernel_tc: symmetric needs A == B");
    if (na == 0 || nb == 0) return FMLB_OK;
    const size_t need_a = fmlb_tc_operand_bytes(na, d);
    const size_t need = need_a + (symmetric ? 0 : fmlb_tc_operand_bytes(nb, d));
    if (!workspace || ws_bytes < need) {
        set_error("fmlb_gaussian_kernel_tc: workspace %zu < %zu bytes", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    SplitView va, vb;
    FMLB_TRY(prepare_operand(A, na, lda, d, mu, workspace, va, st));
    if (symmetric) {
        vb = va;
    } else {
        FMLB_TRY(prepare_operand(B, nb, ldb, d, mu, static_cast<char *>(workspace) + need_a, vb, st));
    }
    CUtensorMap mAhi, mAlo, mBhi, mBlo;
    FMLB_TRY(make_map(&mAhi, va.hi, va.n_pad, va.d_pad));
    FMLB_TRY(make_map(&mAlo, va.lo, va.n_pad, va.d_pad));
    FMLB_TRY(make_map(&mBhi, vb.hi, vb.n_pad, vb.d_pad));
    FMLB_TRY(make_map(&mBlo, vb.lo, vb.n_pad, vb.d_pad));
    TcParams p;
    for (int s = 0; s < nsigma; ++s)
        p.scale[s] = (float)(-1.4426950408889634 / (2.0 * sigmas_host[s] * sigmas_host[s]));
    p.nsig = nsigma;
    p.na = na;
    p.nb = nb;
    p.ntile_a = va.n_pad / TC_BM;
    p.ntile_b = vb.n_pad / TC_BN;
    p.nk = va.d_pad / TC_BK;
    p.symmetric = symmetric ? 1 : 0;
    p.ldk = ldk;
    p.sstride = sigma_stride;
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_gaussian_kernel_tc: cudaGetDevice"));
    if (attr_dev != dev) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(gauss_tc_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)kTcSmem),
                             "fmlb_gaussian_kernel_tc: smem attribute"));
        attr_dev = dev;
    }
    const long long ntiles = symmetric ? (long long)p.ntile_a * (p.ntile_a + 1) / 2
                                       : (long long)p.ntile_a * p.ntile_b;
    FMLB_REQUIRE(ntiles < (1LL << 31), "fmlb_gaussian_kernel_tc: too many tiles");
    const int grid = (int)std::min<long long>(ntiles, sm_count());
    gauss_tc_kernel<<<grid, TC_THREADS, kTcSmem, st>>>(mAhi, mAlo, mBhi, mBlo, va.norms, vb.norms,
                                                       p, K, status);
    return launch_status("gauss_tc_kernel");
}
