// Atomic KRR from precomputed atom-pair distances, the kernels of
// fget_alpha_from_distance / fget_prediction_from_distance
// (fml/kernels/fkernels.f90:541-702):
//
//   fmlb_segment_exp_sum_f64:  S[p, q] = sum_{r in R_p} sum_{s in C_q} exp(c M[r, s])
//     (the molecule kernel of fget_alpha_from_distance, :586-597, is S with
//     R = C = the molecules' atom ranges and M = D);
//   fmlb_exp_weighted_colsum_f64:  v[s] = sum_r exp(c M[r, s]) w[r]
//     (the per-atom sums csa of fget_prediction_from_distance, :688-693).
//
// Both are HBM-bound reads of M; reductions run in a fixed order.
#include <math.h>

#include <algorithm>

#include "common.cuh"
#include "fmlb.h"

namespace fmlb {
namespace {

constexpr int SE_TPB = 256;
constexpr int CS_TPB = 256;
constexpr int CS_SPLIT = 64;  // row slices of the column sums (fixed)

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One CTA per output (p, q): threads stride the block's entries row by row.
__global__ void __launch_bounds__(SE_TPB)
segment_exp_sum_kernel(const double *__restrict__ M, long long ldm, int rows, int cols,
                       const int *__restrict__ R, int np, const int *__restrict__ C, int nq,
                       double c, double *__restrict__ S, long long lds) {
    __shared__ double red[SE_TPB / 32];
    const long long t = blockIdx.x;
    const int p = (int)(t / nq), q = (int)(t % nq);
    // ranges clipped to the matrix (the host checks the offsets as well)
    const int r0 = min(max(R[p], 0), rows), r1 = min(max(R[p + 1], r0), rows);
    const int c0 = min(max(C[q], 0), cols), c1 = min(max(C[q + 1], c0), cols);
    const int w = c1 - c0;
    double acc = 0.0;
    const long long cnt = (long long)(r1 - r0) * w;
    for (long long e = threadIdx.x; e < cnt; e += SE_TPB) {
        const int r = r0 + (int)(e / w), s = c0 + (int)(e % w);
        acc += exp(c * M[(size_t)r * ldm + s]);
    }
    acc = warp_sum_d(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int k = 0; k < SE_TPB / 32; ++k) v += red[k];
        S[(size_t)p * lds + q] = v;
    }
}

// part[b, s] = sum over the rows of slice b of exp(c M[r, s]) w[r]; thread per column.
__global__ void __launch_bounds__(CS_TPB)
exp_colsum_partial_kernel(const double *__restrict__ M, long long ldm, int rows, int cols,
                          double c, const double *__restrict__ w, double *__restrict__ part) {
    const int s = blockIdx.x * CS_TPB + threadIdx.x;
    const int b = blockIdx.y;
    const int per = (rows + CS_SPLIT - 1) / CS_SPLIT;
    const int r0 = b * per, r1 = min(rows, r0 + per);
    if (s >= cols) return;
    double acc = 0.0;
    for (int r = r0; r < r1; ++r) acc += exp(c * M[(size_t)r * ldm + s]) * w[r];
    part[(size_t)b * cols + s] = acc;
}

__global__ void exp_colsum_final_kernel(const double *__restrict__ part, int cols,
                                        double *__restrict__ v) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= cols) return;
    double acc = 0.0;
    for (int b = 0; b < CS_SPLIT; ++b) acc += part[(size_t)b * cols + s];
    v[s] = acc;
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_segment_exp_sum_f64(const double *M, long long ldm, int rows, int cols,
                                        const int *R, int np, const int *C, int nq, double c,
                                        double *S, long long lds, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(rows >= 0 && cols >= 0 && ldm >= cols && np >= 0 && nq >= 0 && lds >= nq,
                 "fmlb_segment_exp_sum_f64: bad sizes");
    if ((long long)np * nq == 0) return FMLB_OK;
    FMLB_REQUIRE(M && R && C && S, "fmlb_segment_exp_sum_f64: null pointer");
    FMLB_REQUIRE((long long)np * nq < 0x7fffffffLL, "fmlb_segment_exp_sum_f64: too many blocks");
    segment_exp_sum_kernel<<<(unsigned)((long long)np * nq), SE_TPB, 0, FMLB_STREAM(stream)>>>(
        M, ldm, rows, cols, R, np, C, nq, c, S, lds);
    return launch_status("segment_exp_sum_kernel");
}

extern "C" size_t fmlb_exp_colsum_scratch_doubles(int cols) {
    return (size_t)fmlb::CS_SPLIT * (size_t)std::max(cols, 0);
}

extern "C" int fmlb_exp_weighted_colsum_f64(const double *M, long long ldm, int rows, int cols,
                                            double c, const double *w, double *v,
                                            double *scratch, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(rows >= 0 && cols >= 0 && ldm >= cols, "fmlb_exp_weighted_colsum_f64: bad sizes");
    if (cols == 0) return FMLB_OK;
    FMLB_REQUIRE(v && scratch && (rows == 0 || (M && w)),
                 "fmlb_exp_weighted_colsum_f64: null pointer");
    cudaStream_t st = FMLB_STREAM(stream);
    const dim3 grid(ceil_div(cols, CS_TPB), CS_SPLIT);
    exp_colsum_partial_kernel<<<grid, CS_TPB, 0, st>>>(M, ldm, rows, cols, c, w, scratch);
    FMLB_TRY(launch_status("exp_colsum_partial_kernel"));
    exp_colsum_final_kernel<<<ceil_div(cols, 256), 256, 0, st>>>(scratch, cols, v);
    return launch_status("exp_colsum_final_kernel");
}
