// Gaussian kernel matrix on the 5th-generation tensor cores (tcgen05), the
// mixed-precision form of fgaussian_kernel (fml/kernels/fkernels.f90:317-349):
//
//   K_s[i, j] = exp(-(|x_i|^2 + |x_j|^2 - 2 x_i . x_j) / (2 sigma_s^2))
//
// on mean-centred descriptors, with x . y from BF16 hi/lo splits
// (x = hi + lo): x.y ~ hi.hi + hi.lo + lo.hi, three BF16 MMAs accumulated in
// FP32 in tensor memory, and every sigma emitted by the epilogue.
//
// Structure (one persistent CTA per SM, 320 threads):
//   warp 0      TMA producer: per k-chunk of 64, four 128 x 64 BF16 tiles
//               (A hi, A lo, B hi, B lo), 128B-swizzled, into a 3-stage ring;
//   warp 1      allocates 256 TMEM columns (two 128 x 128 FP32 accumulators)
//               and one thread issues tcgen05.mma (M=128, N=128, K=16);
//   warps 2..9  epilogue, two warps per 32-lane TMEM quarter (64 columns
//               each): tcgen05.ld, d^2, release of the accumulator, then exp
//               for every sigma and streaming FP32 stores: the mirrored tile
//               (symmetric builds) from registers, the direct tile through a
//               shared-memory transpose so every store is one coalesced row;
//               the next tile's MMAs run meanwhile in the other accumulator.
// Every mbarrier wait is bounded; a wait that runs out records an error code
// in *status and the CTA winds down instead of hanging, after its own copies
// and MMAs in flight have finished.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "tc_common.cuh"

namespace fmlb {
namespace {

using namespace tc;

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 64, TC_STAGES = 2, TC_THREADS = 320;
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 2;          // 16 KB per operand tile
constexpr int TC_STAGE_BYTES = 4 * TC_TILE_BYTES;          // A hi, A lo, B hi, B lo
constexpr int TC_TMEM_COLS = 2 * TC_BN;
constexpr int TC_MAXSIG = 8;
constexpr int TC_PITCH = 33;                               // floats per transposed row
constexpr int TC_BOX_FLOATS = 32 * 32;                     // one 32 x 32 FP32 store box
constexpr int TC_RING = 3;                                 // store boxes per epilogue warp
constexpr int TC_WARP_STG = TC_RING * TC_BOX_FLOATS;
static_assert(32 * TC_PITCH <= TC_WARP_STG, "the transposed fallback tile fits the boxes");
constexpr int TC_STG_BYTES = TC_EPI_WARPS * TC_WARP_STG * 4;
constexpr size_t kTcSmem =
    (size_t)TC_STAGES * TC_STAGE_BYTES + TC_STG_BYTES + 1024 /* align */ + 256;
static_assert(kTcSmem <= 232448, "dynamic shared memory of one CTA");

enum TcStatus { TC_OK = 0, TC_TIMEOUT_FULL = 1, TC_TIMEOUT_EMPTY = 2, TC_TIMEOUT_TMEM = 3,
                TC_TIMEOUT_DRAIN = 4 };

struct TcParams {
    float scale[TC_MAXSIG];  // -log2(e) / (2 sigma^2)
    int nsig;
    int na, nb;              // logical rows of A and B
    int ntile_a, ntile_b;    // 128-row tiles of A and B
    int nk;                  // k-chunks of 64
    int symmetric;
    long long ldk, sstride;  // output row stride and sigma stride (elements)
    long long budget;        // clock cycles of every mbarrier wait
    int skip_loads;          // test hook: the producer issues no copies
    int tma_store;           // K is written by TMA bulk-tensor stores (aligned K)
};

// L2 policies: the BF16 operands (re-read by every tile of their row / column
// block) are kept, the K boxes (written once) are evicted first.
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        ".L2::cache_hint [%0], [%1, {%3, %4}], [%2], %5;\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "l"(pol)
        : "memory");
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

// 3-D tiled TMA store of a shared-memory box (bulk async-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int x, int y,
                                             int z, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group.L2::cache_hint"
        " [%0, {%2, %3, %4}], [%1], %5;\n" ::"l"(reinterpret_cast<uint64_t>(map)),
        "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n"); }
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// the box a ring slot held is free once at most TC_RING - 1 newer groups are
// still reading (every slot use is its own commit group)
__device__ __forceinline__ void bulk_wait_ring_slot() {
    static_assert(TC_RING == 3, "the wait count below is TC_RING - 1");
    asm volatile("cp.async.bulk.wait_group.read 2;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ float fast_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__global__ void __launch_bounds__(TC_THREADS, 1)
gauss_tc_kernel(const __grid_constant__ CUtensorMap mapAhi, const __grid_constant__ CUtensorMap mapAlo,
                const __grid_constant__ CUtensorMap mapBhi, const __grid_constant__ CUtensorMap mapBlo,
                const __grid_constant__ CUtensorMap mapK, const float *__restrict__ normA,
                const float *__restrict__ normB, const __grid_constant__ TcParams p,
                float *__restrict__ K,
                int *__restrict__ status) {
    extern __shared__ uint8_t tc_smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    float *stg_all = reinterpret_cast<float *>(smem + TC_STAGES * TC_STAGE_BYTES);
    uint64_t *bars =
        reinterpret_cast<uint64_t *>(smem + TC_STAGES * TC_STAGE_BYTES + TC_STG_BYTES);
    uint64_t *full = bars, *empty = bars + TC_STAGES;
    uint64_t *tmem_full = bars + 2 * TC_STAGES, *tmem_empty = tmem_full + 2;
    uint64_t *mma_done = tmem_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = p.symmetric ? p.ntile_a * (p.ntile_a + 1) / 2 : p.ntile_a * p.ntile_b;
    const long long budget = p.budget;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tmem_full[a], 1);
            mbar_init(&tmem_empty[a], TC_EPI_WARPS);
        }
        mbar_init(mma_done, 1);
        mbar_fence_init();
    }
    if (warp == 1) tmem_alloc(tmem_slot, TC_TMEM_COLS);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            const uint64_t keep = l2_evict_last();
            long long issued = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok && !p.skip_loads; t += gridDim.x) {
                int ta, tb;
                tile_coords(t, p, ta, tb);
                for (int kc = 0; kc < p.nk; ++kc, ++issued) {
                    const int stage = (int)(issued % TC_STAGES);
                    const uint32_t phase = (uint32_t)((issued / TC_STAGES) & 1);
                    if (!mbar_wait(&empty[stage], phase ^ 1, budget)) {
                        atomicCAS(status, 0, TC_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + stage * TC_STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], TC_STAGE_BYTES);
                    tma_load_2d(st, &mapAhi, &full[stage], kc * TC_BK, ta * TC_BM, keep);
                    tma_load_2d(st + TC_TILE_BYTES, &mapAlo, &full[stage], kc * TC_BK, ta * TC_BM,
                                keep);
                    tma_load_2d(st + 2 * TC_TILE_BYTES, &mapBhi, &full[stage], kc * TC_BK,
                                tb * TC_BN, keep);
                    tma_load_2d(st + 3 * TC_TILE_BYTES, &mapBlo, &full[stage], kc * TC_BK,
                                tb * TC_BN, keep);
                }
            }
            // every copy this thread issued has landed before the CTA winds down
            for (long long l = issued > TC_STAGES ? issued - TC_STAGES : 0; l < issued; ++l)
                if (!mbar_wait(&full[l % TC_STAGES], (uint32_t)((l / TC_STAGES) & 1), budget))
                    atomicCAS(status, 0, TC_TIMEOUT_DRAIN);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            long long consumed = 0;
            int lt = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++lt) {
                const int acc = lt & 1;
                const uint32_t acc_phase = (lt >> 1) & 1;
                if (!mbar_wait(&tmem_empty[acc], acc_phase ^ 1, budget)) {
                    atomicCAS(status, 0, TC_TIMEOUT_TMEM);
                    break;
                }
                fence_after_sync();
                const uint32_t dacc = tmem_base + (uint32_t)(acc * TC_BN);
                for (int kc = 0; kc < p.nk; ++kc, ++consumed) {
                    const int stage = (int)(consumed % TC_STAGES);
                    const uint32_t phase = (uint32_t)((consumed / TC_STAGES) & 1);
                    if (!mbar_wait(&full[stage], phase, budget)) {
                        atomicCAS(status, 0, TC_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                    fence_after_sync();
                    uint8_t *st = smem + stage * TC_STAGE_BYTES;
                    const uint64_t ahi = smem_desc_kmajor(st, 128);
                    const uint64_t alo = smem_desc_kmajor(st + TC_TILE_BYTES, 128);
                    const uint64_t bhi = smem_desc_kmajor(st + 2 * TC_TILE_BYTES, 128);
                    const uint64_t blo = smem_desc_kmajor(st + 3 * TC_TILE_BYTES, 128);
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
                }
                if (!ok) break;
                mma_commit(&tmem_full[acc]);
            }
            // every MMA issued has finished before TMEM is released
            mma_commit(mma_done);
            if (!mbar_wait(mma_done, 0, budget)) atomicCAS(status, 0, TC_TIMEOUT_DRAIN);
        }
    } else {
        // --------------------------------------------------------------- epilogue
        // Two warps per TMEM lane quarter, 64 columns each. Both 32-column
        // chunks are drained into registers first and TMEM is released, then
        // every sigma is written through a ring of TC_RING 32 x 32 boxes per
        // warp (direct and mirrored box of each chunk in consecutive slots,
        // one TMA store and commit group per slot use), so a box is refilled
        // while the stores of the two before it are still being read.
        // Diagonal tiles (and K without TMA alignment) take per-element
        // stores through a shared-memory transpose.
        const int q = warp & 3;
        const int half = (warp - 2) >> 2;
        float *stg = stg_all + (warp - 2) * TC_WARP_STG;  // 1024-byte aligned boxes
        int slot = 0;
        const uint64_t stream_out = l2_evict_first();
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++lt) {
            int ta, tb;
            tile_coords(t, p, ta, tb);
            const int acc = lt & 1;
            const uint32_t acc_phase = (lt >> 1) & 1;
            if (!mbar_wait(&tmem_full[acc], acc_phase, budget)) {
                atomicCAS(status, 0, TC_TIMEOUT_TMEM);
                break;
            }
            fence_after_sync();
            const int row0 = ta * TC_BM + q * 32;           // this warp's first row
            const int grow = row0 + lane;
            const int gcol0 = tb * TC_BN + half * 64;       // this warp's first column
            const bool row_ok = grow < p.na;
            const float nr = row_ok ? normA[grow] : 0.0f;
            const bool diag_tile = p.symmetric && ta == tb;
            float d2[64];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                uint32_t v[32];
                tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) +
                              (uint32_t)(acc * TC_BN + half * 64 + c * 32), v);
                // the norms are padded to whole tiles (zero past nb) and
                // 16-byte aligned at every 32-column chunk
                float ncol[32];
                const float4 *nb4 = reinterpret_cast<const float4 *>(normB + gcol0 + c * 32);
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4) {
                    const float4 t4 = __ldg(nb4 + j4);
                    ncol[4 * j4] = t4.x;
                    ncol[4 * j4 + 1] = t4.y;
                    ncol[4 * j4 + 2] = t4.z;
                    ncol[4 * j4 + 3] = t4.w;
                }
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int gcol = gcol0 + c * 32 + j;
                    float x = fmaxf(nr + ncol[j] - 2.0f * __uint_as_float(v[j]), 0.0f);
                    if (diag_tile && gcol == grow) x = 0.0f;  // exact zero distance
                    d2[c * 32 + j] = x;
                }
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tmem_empty[acc]);  // the next-but-one tile may start
            const bool tma = p.tma_store && !diag_tile;
            for (int s = 0; s < p.nsig; ++s) {
                const float sc = p.scale[s];
                float *Ks = K + s * p.sstride;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int cb = gcol0 + c * 32;
                    float kv[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) kv[j] = fast_exp2(d2[c * 32 + j] * sc);
                    if (tma) {
                        // direct box K[row0 + r][cb + j], row r = lane, 128-byte
                        // swizzle: 16-byte chunk j4 of row r at chunk j4 ^ (r & 7)
                        if (lane == 0) bulk_wait_ring_slot();
                        __syncwarp();
                        float *dbox = stg + slot * TC_BOX_FLOATS;
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4)
                            *reinterpret_cast<float4 *>(dbox + lane * 32 + ((j4 ^ (lane & 7)) << 2)) =
                                make_float4(kv[4 * j4], kv[4 * j4 + 1], kv[4 * j4 + 2],
                                            kv[4 * j4 + 3]);
                        fence_proxy_async();
                        __syncwarp();
                        if (lane == 0) {  // boxes wholly outside K are not issued
                            if (row0 < p.na && cb < p.nb)
                                tma_store_3d(&mapK, dbox, cb, row0, s, stream_out);
                            bulk_commit();
                        }
                        slot = slot == TC_RING - 1 ? 0 : slot + 1;
                        // mirrored box K[cb + j][row0 + lane]: row j, column lane
                        if (p.symmetric) {
                            if (lane == 0) bulk_wait_ring_slot();
                            __syncwarp();
                            float *mbox = stg + slot * TC_BOX_FLOATS;
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                mbox[j * 32 + (((lane >> 2) ^ (j & 7)) << 2) + (lane & 3)] = kv[j];
                            fence_proxy_async();
                            __syncwarp();
                            if (lane == 0) {
                                if (row0 < p.nb && cb < p.na)
                                    tma_store_3d(&mapK, mbox, row0, cb, s, stream_out);
                                bulk_commit();
                            }
                            slot = slot == TC_RING - 1 ? 0 : slot + 1;
                        }
                    } else {
                        // the whole ring is free once every earlier store has read it
                        if (lane == 0) bulk_wait_read();
                        __syncwarp();
                        // mirrored tile K[col][row]: lanes write 32 consecutive rows
                        if (p.symmetric && row_ok) {
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const int col = cb + j;
                                if (col < p.nb && (!diag_tile || col < grow))
                                    __stcs(Ks + (size_t)col * p.ldk + grow, kv[j]);
                            }
                        }
                        // direct tile K[row][col] through the transpose
#pragma unroll
                        for (int j = 0; j < 32; ++j) stg[lane * TC_PITCH + j] = kv[j];
                        __syncwarp();
                        const int col = cb + lane;
                        for (int rr = 0; rr < 32; ++rr) {
                            const int r = row0 + rr;
                            if (r < p.na && col < p.nb && (!diag_tile || col <= r))
                                __stcs(Ks + (size_t)r * p.ldk + col, stg[rr * TC_PITCH + lane]);
                        }
                        __syncwarp();
                    }
                }
            }
        }
        if (lane == 0) bulk_wait_all();  // every store of this warp is complete
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 1) tmem_dealloc(tmem_base, TC_TMEM_COLS);
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

// column means of X (n rows): a CTA per 32 columns, 32 row groups of one warp
// each (row r to group r mod 32, coalesced 32-column segments), the groups'
// partial sums combined by a fixed shared-memory tree
constexpr int CM_ROWG = 32;
__global__ void __launch_bounds__(32 * CM_ROWG)
column_mean_kernel(const double *__restrict__ X, int n, int ldx, int d, double *__restrict__ mu) {
    __shared__ double part[CM_ROWG][33];
    const int c = threadIdx.x, g = threadIdx.y;
    const int k = blockIdx.x * 32 + c;
    double s = 0.0;
    if (k < d) {
#pragma unroll 8
        for (int i = g; i < n; i += CM_ROWG) s += X[(size_t)i * ldx + k];
    }
    part[g][c] = s;
    __syncthreads();
    for (int h = CM_ROWG / 2; h > 0; h >>= 1) {
        if (g < h) part[g][c] += part[g + h][c];
        __syncthreads();
    }
    if (g == 0 && k < d) mu[k] = n ? part[0][c] / n : 0.0;
}

// ---- host: tensor maps --------------------------------------------------------
int make_map(CUtensorMap *m, const void *base, int rows, int cols) {
    EncodeTiledFn fn = encode_tiled_fn();
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
    column_mean_kernel<<<ceil_div(d, 32), dim3(32, CM_ROWG), 0, FMLB_STREAM(stream)>>>(X, n, ldx,
                                                                                  d, mu);
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
    const TestHooks hooks = test_hooks();
    p.budget = hooks.wait_budget;
    p.skip_loads = hooks.skip_loads;
    // K written by TMA stores when its rows and sigma planes start on 16 bytes
    CUtensorMap mK;
    memset(&mK, 0, sizeof mK);
    p.tma_store = ((uintptr_t)K % 16 == 0) && (ldk % 4 == 0) &&
                  (nsigma == 1 || sigma_stride % 4 == 0) && ldk * 4 < (1LL << 40) &&
                  (long long)sigma_stride * 4 < (1LL << 40);
    if (p.tma_store) {
        EncodeTiledFn fn = encode_tiled_fn();
        const cuuint64_t gdim[3] = {(cuuint64_t)nb, (cuuint64_t)na, (cuuint64_t)nsigma};
        const cuuint64_t gstride[2] = {(cuuint64_t)ldk * 4,
                                       (cuuint64_t)(nsigma > 1 ? sigma_stride : (long long)na * ldk) * 4};
        const cuuint32_t box[3] = {32, 32, 1};
        const cuuint32_t estride[3] = {1, 1, 1};
        if (!fn || fn(&mK, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, K, gdim, gstride, box, estride,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                      CU_TENSOR_MAP_L2_PROMOTION_NONE,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            p.tma_store = 0;  // the per-element store path needs no map
    }
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
    gauss_tc_kernel<<<grid, TC_THREADS, kTcSmem, st>>>(mAhi, mAlo, mBhi, mBlo, mK, va.norms, vb.norms,
                                                       p, K, status);
    return launch_status("gauss_tc_kernel");
}
