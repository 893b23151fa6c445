// FP64 trailing update C -= P P^T of the Cholesky factorisation on the int8
// tensor cores: the Ozaki splitting scheme (K. Ozaki, T. Ogita, S. Oishi,
// S. M. Rump, "Error-free transformations of matrix multiplication by using
// fast routines of matrix multiplication and its applications", Numer.
// Algorithms 59, 2012; int8 form: H. Ootomo, K. Ozaki, R. Yokota, "DGEMM on
// integer matrix multiplication unit", IJHPCA 2024), written for tcgen05.
//
// Splitting. Each row r of P (k columns) gets the exponent e_r with
// max_c |P[r, c]| < 2^e_r, so x = P[r, c] 2^-(e_r + 1) lies in (-1/2, 1/2),
// and s base-256 digits by repeated flooring, all exact in FP64:
//     d_1 = floor(256 x) in [-128, 127];  u_t = floor(256 rem_{t-1}) in [0, 255]
// (a remainder 1 - |tiny| that rounds to 1.0 after a leading -1 is carried
// back into the digit, so every remainder stays in [0, 1))
// stored as signed bytes with a zero point: v_t = u_t - 128 in [-128, 127], so
//     x = xt + c + rho,   xt = d_1 / 256 + sum_{t>1} v_t 256^-t,
//     c = 128 sum_{t=2..s} 256^-t,   0 <= rho < 256^-s.
// With c' = c + 256^-s / 2 the error x - (xt + c') is zero-mean, and so are
// the dropped digit products below (v_t is centred), which keeps the errors
// of the k-term sums from adding up coherently. Then, summing over k,
//     x_r . x_c ~ xt_r . xt_c + c' (S_r + S_c) + k c'^2,   S_r = sum_k xt_r,k,
// and the product of two rows keeps the digit pairs (t, u) with t + u <= s + 1,
// grouped by diagonal q = t + u - 1:
//     xt_r . xt_c ~ 256^-(s + 1) sum_{q=1..s} D_q 256^(s - q),
//     D_q = sum_{t + u = q + 1} dig_t[r, :] . dig_u[c, :]       (exact in int32)
// s (s + 1) / 2 signed int8 products in all, every D_q accumulated exactly in
// its own TMEM accumulator and combined once, in FP64, by the epilogue
// (Horner in 256), which adds the zero-point terms and scales by
// 2^(e_r + e_c + 2). |dig| <= 128 bounds |D_q| by (q + 1) 2^14 k < 2^31 for
// k <= 8192. Six planes carry the accuracy of seven truncated 7-bit ones
// (21 products instead of 28); the error of one entry stays below
// k (s + 3) 2^(e_r + e_c + 2 - 8 s).
//
// Kernel (one CTA per SM at a time, four tiles per CTA, 320 threads), output
// tile 128 x 64:
//   warp 0      TMA producer: per 32-byte k step, the s digit planes of the
//               128 A rows and 64 B rows (one 3-D box each, 32-byte swizzle)
//               into a ring as deep as shared memory allows (5 stages at
//               s = 6, at most 8);
//   warp 1      allocates 512 TMEM columns (s <= 8 accumulators of 64 int32
//               columns) and issues tcgen05.mma kind::i8 (M 128, N 64, K 32);
//   warps 2..9  epilogue, two warps per TMEM lane quarter (32 columns each):
//               drain the s accumulators into FP64 (Horner), release TMEM to
//               the next tile's MMAs, scale by the row and column exponents,
//               and subtract from C through a shared-memory transpose
//               (coalesced read-modify-write of the lower triangle).
// Every mbarrier wait is bounded; a wait that runs out stores FMLB_ETIMEDOUT
// in *info, and every kernel that reads info returns at once.
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "ozaki.cuh"
#include "tc_common.cuh"

namespace fmlb {
namespace {

constexpr int OZ_BM = 128, OZ_BN = 128;
#ifndef OZ_PASS_DIAGONALS
#define OZ_PASS_DIAGONALS 4
#endif
// Diagonals (int32 accumulators of 128 columns) per pass, and the TMEM buffers
// the 512 columns hold: with two, a pass's MMAs run while the epilogue drains
// the previous pass.
constexpr int OZ_PASS_Q = OZ_PASS_DIAGONALS;
constexpr int OZ_TMEM_BUFS = 4 / OZ_PASS_Q;  // 512 columns: 2 buffers of 2, 1 of 3 or 4
constexpr int OZ_MAX_PASSES = (8 + OZ_PASS_Q - 1) / OZ_PASS_Q;
static_assert(OZ_PASS_Q >= 2 && OZ_PASS_Q <= 4, "passes of 2 to 4 diagonals");
constexpr int OZ_KB = 32;          // int8 k values (bytes) per stage: one MMA K step
constexpr int OZ_MAX_STAGES = 8;  // the ring depth is set per launch from shared memory
constexpr int OZ_THREADS = 320;    // 10 warps
constexpr int OZ_EPI_WARPS = 8;
constexpr int OZ_TMEM_COLS = 512;
constexpr int OZ_CPITCH = OZ_BN + 1;  // doubles per row of the staged C tile (odd: rows of
                                      // one column fall in 16 distinct banks per half-warp)
constexpr int OZ_A_PLANE = OZ_BM * OZ_KB;   // 4096 bytes per A digit plane per stage
constexpr int OZ_B_PLANE = OZ_BN * OZ_KB;   // 4096
constexpr int OZ_CTILE_BYTES = OZ_BM * OZ_CPITCH * (int)sizeof(double);  // 132096
constexpr int OZ_COLF_BYTES = OZ_BN * (int)sizeof(double);
constexpr int OZ_ALIGN = 256;  // shared-memory base: the 32-byte swizzle atom
constexpr int OZ_NONFINITE = 0x7fffffff;    // exponent marking a row with Inf / NaN

constexpr long long kOzDefaultBudget = 4000000000LL;  // clock cycles (~2 s)
constexpr int OZ_SMEM_LIMIT = 232448 - 64;  // opt-in shared memory per CTA, less static
constexpr int OZ_BAR_BYTES = (2 * OZ_MAX_STAGES + 2 * OZ_TMEM_BUFS + 2) * 8 + 8;

struct OzParams {
    int m;             // rows (= columns) of C
    int p_row0;        // slice row of C's row 0 (and column 0)
    int ns;            // digit planes
    int nkb;           // 32-byte k steps
    int strip_cols;    // > 0: only the first strip_cols columns
    int strip_tiles;   // column tiles per row block in strip mode
    long long ntiles;
    long long ldc;
    int exp_bias;      // -8 (ns + 1)
    int npass;         // passes: diagonals [0, Q), [Q, 2Q), ... [.., ns)
    double zp_c;       // c' (zero point of the digit planes)
    double zp_kc2;     // kp c'^2
    int skip_loads;    // test hook: the producer issues no copies
    int stages;        // depth of the operand ring
};

// Tensor maps of the digit planes, one per pass (boxes of that pass's planes).
struct OzMaps {
    CUtensorMap m[OZ_MAX_PASSES];
};

// Instruction descriptor, kind::i8: signed A and B, int32 accumulator, both
// K-major, M = 128, N = 128.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(OZ_BN >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
__device__ __forceinline__ uint32_t idesc_i8(int, int) { return kIdescI8; }

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Tile t -> (row0, col0) of the lower triangle of 128 x 128 tiles (row block
// `by` holds column tiles 0 .. by), or of the first strip_tiles column tiles
// of every row block. Tiles run in bands of OZ_BAND row blocks and, inside a
// band, in groups of OZ_BAND column tiles (a 1024 x 1024 block of C), so the
// ~148 tiles in flight at a time share their digit planes through L2. Band
// b holds b + 1 groups below and on the diagonal. The enumeration covers a
// superset of C; false for tiles outside C.
constexpr int OZ_BAND = 8;
constexpr int OZ_GROUP = OZ_BAND * OZ_BAND;  // tiles of a band x group block
__device__ __forceinline__ bool oz_tile(long long t, const OzParams &p, int &row0, int &col0) {
    int by, bx;
    if (p.strip_tiles > 0) {
        const int band = (int)(t / (OZ_BAND * p.strip_tiles));
        const int w = (int)(t % (OZ_BAND * p.strip_tiles));
        by = band * OZ_BAND + w / p.strip_tiles;
        bx = w % p.strip_tiles;
    } else {
        // bands before band b: OZ_GROUP b (b + 1) / 2 tiles
        int b = (int)((sqrt(8.0 * (double)t / OZ_GROUP + 1.0) - 1.0) * 0.5);
        while ((long long)OZ_GROUP * b * (b + 1) / 2 > t) --b;
        while ((long long)OZ_GROUP * (b + 1) * (b + 2) / 2 <= t) ++b;
        const int u = (int)(t - (long long)OZ_GROUP * b * (b + 1) / 2);
        const int g = u / OZ_GROUP, w = u % OZ_GROUP;
        by = b * OZ_BAND + w / OZ_BAND;
        bx = g * OZ_BAND + w % OZ_BAND;
    }
    if (bx > by) return false;
    row0 = by * OZ_BM;
    col0 = bx * OZ_BN;
    return row0 < p.m && col0 < p.m;
}

__device__ __forceinline__ void oz_fail(int *info) { atomicCAS(info, 0, FMLB_ETIMEDOUT); }

// 2^(e + 1) for a row or column exponent in [-500, 500] (the scaled product
// core * 2^(e_r+1) * 2^(e_c+1) then equals ldexp(core, e_r + e_c + 2)), else 0.
__device__ __forceinline__ double oz_pow2_factor(int e) {
    return (e >= -500 && e <= 500) ? __longlong_as_double((long long)(e + 1 + 1023) << 52) : 0.0;
}

// First tile t' >= t of this CTA's sequence (stride gridDim.x) inside C, or ntiles.
__device__ __forceinline__ long long oz_next_tile(long long t, const OzParams &p, int &row0,
                                                  int &col0) {
    for (; t < p.ntiles; t += gridDim.x)
        if (oz_tile(t, p, row0, col0)) return t;
    return p.ntiles;
}

// 8-byte asynchronous global -> shared copies (completion per thread).
__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(tc::smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Pass q0..q1 of the diagonals needs the digit planes 0..q1-1.
__device__ __forceinline__ void oz_pass(const OzParams &p, int ps, int &q0, int &q1) {
    q0 = ps * OZ_PASS_Q;
    q1 = min(p.ns, q0 + OZ_PASS_Q);
}

__global__ void __launch_bounds__(OZ_THREADS, 1)
ozaki_syrk_kernel(const __grid_constant__ OzMaps maps,
                  const int *__restrict__ exps, const double *__restrict__ rsum, OzParams p,
                  double *__restrict__ C, int *__restrict__ info, long long budget) {
    extern __shared__ uint8_t oz_smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(oz_smem_raw) + OZ_ALIGN - 1) & ~(uintptr_t)(OZ_ALIGN - 1));
    const int stage_bytes = p.ns * (OZ_A_PLANE + OZ_B_PLANE);  // B planes after ns A planes
    const int nst = p.stages;
    // C tile, 128 x 129: column 128 holds the tile's column digit sums S_c
    double *cs = reinterpret_cast<double *>(smem + nst * stage_bytes);
    // 2^(e_c + 1) per column of the tile, 0 where the exact scaling needs ldexp
    double *colf = reinterpret_cast<double *>(smem + nst * stage_bytes + OZ_CTILE_BYTES);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + nst * stage_bytes + OZ_CTILE_BYTES +
                                                  OZ_COLF_BYTES);
    uint64_t *full = bars, *empty = bars + OZ_MAX_STAGES;
    uint64_t *tmem_full = bars + 2 * OZ_MAX_STAGES, *tmem_empty = tmem_full + OZ_TMEM_BUFS,
             *mma_done = tmem_empty + OZ_TMEM_BUFS, *epi_bar = mma_done + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(epi_bar + 1);
    __shared__ int abort_cta;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        abort_cta = *(volatile const int *)info != 0;
        for (int s = 0; s < nst; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < OZ_TMEM_BUFS; ++b) {
            tc::mbar_init(&tmem_full[b], 1);
            tc::mbar_init(&tmem_empty[b], OZ_EPI_WARPS);
        }
        tc::mbar_init(mma_done, 1);
        tc::mbar_init(epi_bar, OZ_EPI_WARPS * 32);
        tc::mbar_fence_init();
    }
    __syncthreads();
    if (abort_cta) return;  // a failed factorisation: the whole CTA leaves together
    if (warp == 1) tc::tmem_alloc(tmem_slot, OZ_TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            long long issued = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
                int row0, col0;
                if (!oz_tile(t, p, row0, col0)) continue;
                for (int ps = 0; ps < p.npass && ok; ++ps) {
                    int q0, q1;
                    oz_pass(p, ps, q0, q1);
                    const CUtensorMap *map = &maps.m[ps];  // boxes of q1 planes
                    for (int kb = 0; kb < p.nkb && !p.skip_loads; ++kb, ++issued) {
                        const int st = (int)(issued % nst);
                        const uint32_t ph = (uint32_t)((issued / nst) & 1);
                        if (!tc::mbar_wait(&empty[st], ph ^ 1, budget)) {
                            oz_fail(info);
                            ok = false;
                            break;
                        }
                        uint8_t *sa = smem + st * stage_bytes;
                        uint8_t *sb = sa + p.ns * OZ_A_PLANE;
                        tc::mbar_arrive_expect_tx(&full[st], (uint32_t)(q1 * (OZ_A_PLANE + OZ_B_PLANE)));
                        tc::tma_load_3d(sa, map, &full[st], kb * OZ_KB, p.p_row0 + row0, 0);
                        tc::tma_load_3d(sb, map, &full[st], kb * OZ_KB, p.p_row0 + col0, 0);
                    }
                }
            }
            // every copy this thread issued has landed before the CTA winds down
            for (long long l = std::max(0LL, issued - (long long)nst); l < issued; ++l)
                if (!tc::mbar_wait(&full[l % nst], (uint32_t)((l / nst) & 1), budget))
                    oz_fail(info);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            long long consumed = 0;
            int lp = 0;  // passes issued
            bool ok = true;
            for (long long t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
                int row0, col0;
                if (!oz_tile(t, p, row0, col0)) continue;
                for (int ps = 0; ps < p.npass; ++ps, ++lp) {
                    int q0, q1;
                    oz_pass(p, ps, q0, q1);
                    const int buf = lp % OZ_TMEM_BUFS;
                    if (!tc::mbar_wait(&tmem_empty[buf], (uint32_t)(((lp / OZ_TMEM_BUFS) & 1) ^ 1),
                                       budget)) {
                        oz_fail(info);
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    for (int kb = 0; kb < p.nkb; ++kb, ++consumed) {
                        const int st = (int)(consumed % nst);
                        const uint32_t ph = (uint32_t)((consumed / nst) & 1);
                        if (!tc::mbar_wait(&full[st], ph, budget)) {
                            oz_fail(info);
                            ok = false;
                            break;
                        }
                        tc::fence_after_sync();
                        const uint8_t *sa = smem + st * stage_bytes;
                        const uint8_t *sb = sa + p.ns * OZ_A_PLANE;
                        const uint64_t da = tc::smem_desc_kmajor(sa, OZ_KB);
                        const uint64_t db = tc::smem_desc_kmajor(sb, OZ_KB);
                        for (int q = q0; q < q1; ++q) {
                            const uint32_t dacc =
                                tmem_base + (uint32_t)((buf * OZ_PASS_Q + q - q0) * OZ_BN);
                            for (int a = 0; a <= q; ++a) {
                                const int b = q - a;
                                // plane offsets in 16-byte units of the descriptor address
                                mma_i8(dacc, da + (uint64_t)((a * OZ_A_PLANE) >> 4),
                                       db + (uint64_t)((b * OZ_B_PLANE) >> 4), idesc_i8(a, b),
                                       (kb > 0 || a > 0) ? 1u : 0u);
                            }
                        }
                        tc::mma_commit(&empty[st]);  // frees the stage once these MMAs finish
                    }
                    if (!ok) break;
                    tc::mma_commit(&tmem_full[buf]);
                }
            }
            // every MMA issued has finished before TMEM is released
            tc::mma_commit(mma_done);
            if (!tc::mbar_wait(mma_done, 0, budget)) oz_fail(info);
        }
    } else {
        // --------------------------------------------------------------- epilogue
        // C's tile is staged in shared memory (cs, rows of 129 doubles) by
        // cp.async while the tile's first pass runs on the tensor cores, and
        // written back once after its last pass, both with one coalesced row
        // segment of 32 columns per warp instruction (element i * 256 + e of
        // the tile for thread e). Two warps per TMEM lane quarter, 64 columns
        // (two chunks of 32) each: per pass and chunk, drain the pass's
        // accumulators into FP64 (Horner in 256), scale, and subtract from
        // this lane's row of cs. TMEM is released after the second chunk's
        // drain, so the next pass's MMAs overlap that chunk's arithmetic.
        const int qw = warp & 3;
        const int half = (warp - 2) >> 2;
        const int e = threadIdx.x - 64;           // 0 .. 255
        const int rl = qw * 32 + lane;            // this lane's row of the tile
        double *csr = cs + rl * OZ_CPITCH;
        int lp = 0;
        uint32_t nsync = 0;
        bool ok = true;
        // every epilogue thread arrives; bounded wait, so a warp that gave up
        // cannot hold the others
        auto epi_sync = [&]() -> bool {
            tc::mbar_arrive(epi_bar);
            const bool r = tc::mbar_wait(epi_bar, nsync & 1, budget);
            ++nsync;
            return r;
        };
        auto tile_elem = [&](int i, int r0, int c0, int &r, int &c, size_t &g) -> bool {
            const int idx = i * (OZ_EPI_WARPS * 32) + e;
            r = idx >> 7;
            c = idx & (OZ_BN - 1);
            const int gr = r0 + r, gc = c0 + c;
            g = (size_t)gr * p.ldc + gc;
            return gr < p.m && gc <= gr && (p.strip_cols == 0 || gc < p.strip_cols);
        };
        auto prefetch = [&](int r0, int c0) {
            for (int i = 0; i < OZ_BM * OZ_BN / (OZ_EPI_WARPS * 32); ++i) {
                int r, c;
                size_t g;
                if (tile_elem(i, r0, c0, r, c, g)) cp_async8(cs + r * OZ_CPITCH + c, C + g);
            }
            cp_async_commit();
        };
        int row0 = 0, col0 = 0;
        long long t = oz_next_tile(blockIdx.x, p, row0, col0);
        if (t < p.ntiles) prefetch(row0, col0);
        while (t < p.ntiles && ok) {
            const int grow = row0 + rl;
            const int er = grow < p.m ? exps[p.p_row0 + grow] : 0;
            const double sr = grow < p.m ? rsum[p.p_row0 + grow] : 0.0;
            const double rowf = oz_pow2_factor(er);
            if (e < OZ_BN) {  // the tile's column data; read after the tile-start barrier
                const int gc = col0 + e;
                const int ec = gc < p.m ? exps[p.p_row0 + gc] : 0;
                colf[e] = oz_pow2_factor(ec);
                cs[e * OZ_CPITCH + OZ_BN] = gc < p.m ? rsum[p.p_row0 + gc] : 0.0;
            }
            for (int ps = 0; ps < p.npass && ok; ++ps, ++lp) {
                int q0, q1;
                oz_pass(p, ps, q0, q1);
                const bool last = ps == p.npass - 1;
                // Horner over diagonals q0 .. q1-1 carries 256^(q1-1-q): scale by 256^-(q1+1)
                const double pbias = __longlong_as_double((long long)(1023 - 8 * (q1 + 1)) << 52);
                const int buf = lp % OZ_TMEM_BUFS;
                if (!tc::mbar_wait(&tmem_full[buf], (uint32_t)((lp / OZ_TMEM_BUFS) & 1), budget)) {
                    oz_fail(info);
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                if (ps == 0) {  // the tile's C has landed in cs (every thread's copies)
                    cp_async_wait_all();
                    if (!epi_sync()) {
                        oz_fail(info);
                        ok = false;
                        break;
                    }
                }
                for (int cc = 0; cc < 2; ++cc) {
                    const int cb = half * 64 + cc * 32;  // chunk's first column in the tile
                    double acc[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[j] = 0.0;
                    for (int q = q0; q < q1; ++q) {
                        uint32_t v[32];
                        tc::tmem_ld32(tmem_base + ((uint32_t)(qw * 32) << 16) +
                                          (uint32_t)((buf * OZ_PASS_Q + q - q0) * OZ_BN + cb), v);
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            acc[j] = fma(acc[j], 256.0, (double)(int)v[j]);
                    }
                    if (cc == 1) {
                        tc::fence_before_sync();
                        __syncwarp();
                        if (lane == 0) tc::mbar_arrive(&tmem_empty[buf]);  // the buffer is free
                    }
                    // last pass: (acc 256^-(s+1) + c' (S_r + S_c) + k c'^2) 2^(e_r + e_c + 2),
                    // earlier passes: acc 256^-(q1+1) 2^(e_r + e_c + 2); fixed order, no
                    // contraction. Both power-of-two scalings are exact multiplications
                    // (core * 2^(e_r+1) is normal), so the result is ldexp's, rounded once.
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const double f = colf[cb + j];
                        double core = __dmul_rn(acc[j], pbias);
                        if (last)
                            core = __dadd_rn(
                                __dadd_rn(core, __dmul_rn(p.zp_c,
                                                          __dadd_rn(sr, cs[(cb + j) * OZ_CPITCH + OZ_BN]))),
                                p.zp_kc2);
                        double v;
                        if (rowf != 0.0 && f != 0.0) {
                            v = __dmul_rn(__dmul_rn(core, rowf), f);
                        } else {  // a non-finite row or column, or an exponent outside +-500
                            const int gc = col0 + cb + j;
                            const int ec = gc < p.m ? exps[p.p_row0 + gc] : 0;
                            v = (er == OZ_NONFINITE || ec == OZ_NONFINITE)
                                    ? __longlong_as_double(0x7ff8000000000000LL)
                                    : ldexp(core, er + ec + 2);
                        }
                        csr[cb + j] = __dsub_rn(csr[cb + j], v);
                    }
                }
            }
            if (!ok) break;
            if (!epi_sync()) {  // every pass's subtraction is in cs
                oz_fail(info);
                break;
            }
            for (int i = 0; i < OZ_BM * OZ_BN / (OZ_EPI_WARPS * 32); ++i) {
                int r, c;
                size_t g;
                if (tile_elem(i, row0, col0, r, c, g)) C[g] = cs[r * OZ_CPITCH + c];
            }
            // the next tile's C into the elements this thread has just written back
            t = oz_next_tile(t + gridDim.x, p, row0, col0);
            if (t < p.ntiles) prefetch(row0, col0);
        }
        cp_async_wait_all();  // no copy lands after the CTA has left
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) tc::tmem_dealloc(tmem_base, OZ_TMEM_COLS);
}

// ---- splitting --------------------------------------------------------------
// One CTA (128 threads) per row of P (rows [0, m), k columns, stride ldp):
// exps[r], ns digit planes (row-major, kp >= k columns zero-padded, plane
// stride pstride bytes) and the row sum rsum[r] = S_r of the zero-point
// digits (per-plane integer sums, combined in FP64 in plane order). Each
// thread owns 8 consecutive columns per sweep.
constexpr int SL_TPB = 128;

__global__ void __launch_bounds__(SL_TPB)
ozaki_slice_kernel(const double *__restrict__ P, long long ldp, int m, int k, int kp, int ns,
                   int8_t *__restrict__ planes, long long pstride, long long ldpl,
                   int *__restrict__ exps, double *__restrict__ rsum,
                   const int *__restrict__ info) {
    __shared__ double red[SL_TPB / 32];
    __shared__ int tsum[OZAKI_MAX_SLICES][SL_TPB / 32];
    __shared__ int bad_row, abort_cta;
    const int r = blockIdx.x, tid = threadIdx.x;
    if (tid == 0) {
        abort_cta = info && *(volatile const int *)info != 0;
        bad_row = 0;
    }
    __syncthreads();
    if (abort_cta || r >= m) return;
    const double *row = P + (size_t)r * ldp;
    double mx = 0.0;
    for (int c = tid; c < k; c += SL_TPB) {
        const double v = row[c];
        if (!isfinite(v)) bad_row = 1;
        mx = fmax(mx, fabs(v));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) red[tid >> 5] = mx;
    __syncthreads();
    mx = fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1): |P[r, :]| < 2^e
    if (tid == 0) exps[r] = bad_row ? OZ_NONFINITE : e;
    int psum[OZAKI_MAX_SLICES];
#pragma unroll
    for (int t = 0; t < OZAKI_MAX_SLICES; ++t) psum[t] = 0;
    for (int c0 = tid * 8; c0 < kp; c0 += SL_TPB * 8) {
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int c = c0 + i;
            const double v = c < k ? row[c] : 0.0;
            x[i] = (bad_row || !isfinite(v)) ? 0.0 : ldexp(v, -(e + 1));  // in (-1/2, 1/2)
        }
#pragma unroll
        for (int t = 0; t < OZAKI_MAX_SLICES; ++t) {
            if (t >= ns) break;
            uint64_t word = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                x[i] *= 256.0;
                double d = floor(x[i]);             // [-128, 127] first, then [0, 255]
                x[i] -= d;
                // a tiny negative leading value gives d = -1 and a remainder
                // 1 - |x| that rounds to 1.0: carry it back into the digit
                if (x[i] >= 1.0) {
                    x[i] -= 1.0;
                    d += 1.0;
                }
                const int v = (int)d - (t ? 128 : 0);  // zero point of the lower planes
                psum[t] += v;
                word |= (uint64_t)((uint32_t)v & 0xffu) << (8 * i);
            }
            *reinterpret_cast<uint64_t *>(planes + t * pstride + (size_t)r * ldpl + c0) = word;
        }
    }
#pragma unroll
    for (int t = 0; t < OZAKI_MAX_SLICES; ++t) {
        int v = psum[t];
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) tsum[t][tid >> 5] = v;
    }
    __syncthreads();
    if (tid == 0) {
        double sr = 0.0;
        for (int t = 0; t < ns; ++t) {
            const int tt = tsum[t][0] + tsum[t][1] + tsum[t][2] + tsum[t][3];
            sr = __dadd_rn(sr, ldexp((double)tt, -8 * (t + 1)));
        }
        rsum[r] = sr;
    }
}

int make_plane_map(CUtensorMap *map, const int8_t *base, int rows, long long ldpl, int kp,
                   long long pstride, int ns, int box_rows) {
    tc::EncodeTiledFn fn = tc::encode_tiled_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is unavailable");
        return FMLB_ECUDA;
    }
    FMLB_REQUIRE(((uintptr_t)base % 16) == 0 && ldpl % 16 == 0 && pstride % 16 == 0,
                 "ozaki: digit planes not 16-byte aligned");
    const cuuint64_t gdim[3] = {(cuuint64_t)kp, (cuuint64_t)rows, (cuuint64_t)ns};
    const cuuint64_t gstride[2] = {(cuuint64_t)ldpl, (cuuint64_t)pstride};
    const cuuint32_t box[3] = {(cuuint32_t)OZ_KB, (cuuint32_t)box_rows, (cuuint32_t)ns};
    const cuuint32_t estride[3] = {1, 1, 1};
    CUresult res = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t *>(base), gdim,
                      gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (res != CUDA_SUCCESS) {
        set_error("ozaki: cuTensorMapEncodeTiled failed (%d)", (int)res);
        return FMLB_ECUDA;
    }
    return FMLB_OK;
}

// Deepest operand ring (<= OZ_MAX_STAGES) whose shared memory fits a CTA.
// (two stages at 6 planes, one at 7 or 8 beside the 129 KB C tile).
int oz_stages(int ns) {
    const int sb = ns * (OZ_A_PLANE + OZ_B_PLANE);
    const int room = OZ_SMEM_LIMIT - OZ_CTILE_BYTES - OZ_COLF_BYTES - OZ_BAR_BYTES - OZ_ALIGN;
    return std::max(1, std::min(OZ_MAX_STAGES, room / sb));
}

size_t oz_smem_bytes(int ns) {
    return (size_t)oz_stages(ns) * ns * (OZ_A_PLANE + OZ_B_PLANE) + OZ_CTILE_BYTES +
           OZ_COLF_BYTES + OZ_BAR_BYTES + OZ_ALIGN;
}

thread_local tc::TestHooks t_hooks = {0, 0};

}  // namespace

tc::TestHooks tc::test_hooks() {
    tc::TestHooks h = t_hooks;
    if (h.wait_budget <= 0) h.wait_budget = kOzDefaultBudget;
    return h;
}

int ozaki_split(const double *P, long long ldp, int m, int k, const OzakiSlices &s, const int *info,
                cudaStream_t st) {
    if (m <= 0) return FMLB_OK;
    FMLB_REQUIRE(m <= s.rows && k <= s.kp, "ozaki: panel %d x %d exceeds the slice buffer %d x %d",
                 m, k, s.rows, s.kp);
    ozaki_slice_kernel<<<m, SL_TPB, 0, st>>>(P, ldp, m, k, s.kp, s.ns, s.planes, s.pstride,
                                             s.ldpl, s.exps, s.rsum, info);
    return launch_status("ozaki_slice_kernel");
}

int ozaki_syrk(double *C, long long ldc, int m, const OzakiSlices &s, int p_row0, int strip_cols,
               int *info, cudaStream_t st) {
    if (m <= 0) return FMLB_OK;
    FMLB_REQUIRE(s.ns >= 1 && s.ns <= OZAKI_MAX_SLICES, "ozaki: 1..%d slices", OZAKI_MAX_SLICES);
    FMLB_REQUIRE(s.kp % OZ_KB == 0 && s.kp <= 8192, "ozaki: k must be a multiple of 32, <= 8192");
    FMLB_REQUIRE(p_row0 >= 0 && p_row0 + m <= s.rows, "ozaki: rows outside the slice buffer");
    // boxes of 128 rows and the planes each pass reads (planes 0 .. q1-1 for
    // its last diagonal q1-1)
    OzMaps maps;
    memset(&maps, 0, sizeof maps);
    const int npass = (s.ns + OZ_PASS_Q - 1) / OZ_PASS_Q;
    for (int ps = 0; ps < npass; ++ps)
        FMLB_TRY(make_plane_map(&maps.m[ps], s.planes, s.rows, s.ldpl, s.kp, s.pstride,
                                std::min(s.ns, (ps + 1) * OZ_PASS_Q), OZ_BM));
    OzParams p;
    p.m = m;
    p.p_row0 = p_row0;
    p.ns = s.ns;
    p.nkb = s.kp / OZ_KB;
    p.strip_cols = strip_cols > 0 ? std::min(strip_cols, m) : 0;
    const long long Tr = ceil_div(m, OZ_BM);
    p.strip_tiles = p.strip_cols > 0 ? ceil_div(p.strip_cols, OZ_BN) : 0;
    const long long nband = ceil_div(Tr, OZ_BAND);
    p.ntiles = p.strip_tiles ? nband * OZ_BAND * p.strip_tiles
                             : (long long)OZ_GROUP * nband * (nband + 1) / 2;
    p.npass = npass;
    p.ldc = ldc;
    p.exp_bias = -8 * (s.ns + 1);
    double zc = ldexp(1.0, -8 * s.ns - 1);  // half an ulp of the last digit
    for (int t = 2; t <= s.ns; ++t) zc += ldexp(128.0, -8 * t);
    p.zp_c = zc;
    p.zp_kc2 = (double)s.kp * zc * zc;
    const tc::TestHooks hooks = tc::test_hooks();
    p.skip_loads = hooks.skip_loads;
    p.stages = oz_stages(s.ns);
    const size_t smem = oz_smem_bytes(s.ns);
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "ozaki: cudaGetDevice"));
    if (attr_dev != dev) {
        FMLB_TRY(cuda_status(cudaFuncSetAttribute(ozaki_syrk_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  OZ_SMEM_LIMIT),
                             "ozaki: smem attribute"));
        attr_dev = dev;
    }
    // four tiles per CTA: CTAs retire while the update runs, so the
    // factorisation's high-priority panel chain gets SMs (a persistent grid
    // held every SM until the update ended and serialised the lookahead)
    const int grid = (int)std::min<long long>(
        p.ntiles, std::max<long long>(sm_count(), (p.ntiles + 3) / 4));
    ozaki_syrk_kernel<<<grid, OZ_THREADS, smem, st>>>(maps, s.exps, s.rsum, p, C, info,
                                                       hooks.wait_budget);
    return launch_status("ozaki_syrk_kernel");
}

size_t ozaki_slice_bytes(int rows, int kp, int ns) {
    return (size_t)ns * rows * kp + (size_t)rows * (sizeof(int) + sizeof(double)) + 512;
}

int ozaki_bind(void *ws, int rows, int kp, int ns, OzakiSlices &s) {
    FMLB_REQUIRE(kp % OZ_KB == 0, "ozaki: padded k must be a multiple of 32");
    char *p = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(ws) + 255) & ~(uintptr_t)255);
    s.planes = reinterpret_cast<int8_t *>(p);
    s.rows = rows;
    s.kp = kp;
    s.ns = ns;
    s.ldpl = kp;
    s.pstride = (long long)rows * kp;
    s.rsum = reinterpret_cast<double *>(p + (size_t)ns * rows * kp);  // 8-byte aligned: kp % 32 == 0
    s.exps = reinterpret_cast<int *>(s.rsum + rows);
    return FMLB_OK;
}

}  // namespace fmlb

extern "C" size_t fmlb_syrk_ozaki_workspace_bytes(int m, int k, int nslices) {
    if (m <= 0 || k <= 0 || nslices <= 0) return 256;
    const int kp = (k + 31) / 32 * 32;
    return fmlb::ozaki_slice_bytes(m, kp, nslices);
}

extern "C" int fmlb_syrk_lower_ozaki(double *C, long long ldc, int m, const double *P,
                                     long long ldp, int k, int strip_cols, int nslices,
                                     void *work, size_t ws_bytes, int *info, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(m >= 0 && k >= 0 && ldc >= m && ldp >= k && strip_cols >= 0,
                 "fmlb_syrk_lower_ozaki: bad sizes");
    FMLB_REQUIRE(nslices >= 1 && nslices <= OZAKI_MAX_SLICES,
                 "fmlb_syrk_lower_ozaki: nslices must be 1..%d", OZAKI_MAX_SLICES);
    FMLB_REQUIRE(k <= 8192, "fmlb_syrk_lower_ozaki: k=%d above 8192", k);
    if (m == 0 || k == 0) return FMLB_OK;
    FMLB_REQUIRE(C && P && info, "fmlb_syrk_lower_ozaki: null pointer");
    const size_t need = fmlb_syrk_ozaki_workspace_bytes(m, k, nslices);
    if (!work || ws_bytes < need) {
        set_error("fmlb_syrk_lower_ozaki: workspace %zu < %zu bytes", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    OzakiSlices s;
    FMLB_TRY(ozaki_bind(work, m, (k + 31) / 32 * 32, nslices, s));
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_TRY(ozaki_split(P, ldp, m, k, s, info, st));
    return ozaki_syrk(C, ldc, m, s, 0, strip_cols, info, st);
}

extern "C" int fmlb_tc_test_hooks(long long wait_cycles, int skip_loads) {
    using namespace fmlb;
    FMLB_REQUIRE(wait_cycles >= 0, "fmlb_tc_test_hooks: negative wait budget");
    t_hooks.wait_budget = wait_cycles;
    t_hooks.skip_loads = skip_loads ? 1 : 0;
    return FMLB_OK;
}
