// Generic FP64 distance matrices between descriptor sets, the replacement for
// fml/math/fdistance.f90:
//   kind 0  fmanhattan_distance  (:23-46)   D = sum |a - b|
//   kind 1  fl2_distance         (:49-80)   D = sqrt(sum (a - b)^2)
//   kind 2  fp_distance_integer  (:120-155) D = (sum (a - b)^p)^(1/p), integer p
//   kind 3  fp_distance_double   (:83-118)  D = (sum (a - b)^p)^(1/p), real p
// The p forms raise the signed difference, as the reference does (no abs):
// odd p keeps signs, a real p gives NaN for negative differences.
//
// A (na, d) and B (nb, d) are row-major rows (the reference's columns);
// D (na, nb) row-major, D[j, i] = dist(A_j, B_i). 64 x 64 output tile per
// 256-thread CTA, descriptors staged through shared memory in chunks of 16
// features, 4 x 4 outputs per thread; each output accumulates in feature order.
#include <math.h>

#include "common.cuh"
#include "fmlb.h"

namespace fmlb {
namespace {

constexpr int DM = 64, DN = 64, DK = 16, DTPB = 256;

// x^p by binary exponentiation (p >= 0), 1/x^|p| for p < 0
__device__ __forceinline__ double ipow(double x, int p) {
    unsigned int e = p < 0 ? 0u - (unsigned int)p : (unsigned int)p;
    double r = (e & 1u) ? x : 1.0;
    while (e >>= 1) {
        x = x * x;
        if (e & 1u) r = r * x;
    }
    return p < 0 ? 1.0 / r : r;
}

template <int KIND>
__global__ void __launch_bounds__(DTPB)
distance_matrix_kernel(const double *__restrict__ A, int na, int lda,
                       const double *__restrict__ B, int nb, int ldb, int d, int ip, double dp,
                       double *__restrict__ D, long long ldd) {
    __shared__ double As[DK][DM + 1];
    __shared__ double Bs[DK][DN + 1];
    const int row0 = blockIdx.y * DM, col0 = blockIdx.x * DN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    const int lk = threadIdx.x & 15, lr = threadIdx.x >> 4;
    for (int k0 = 0; k0 < d; k0 += DK) {
        const int k = k0 + lk;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int ra = row0 + lr + 16 * r;
            As[lk][lr + 16 * r] = (ra < na && k < d) ? A[(size_t)ra * lda + k] : 0.0;
            const int rb = col0 + lr + 16 * r;
            Bs[lk][lr + 16 * r] = (rb < nb && k < d) ? B[(size_t)rb * ldb + k] : 0.0;
        }
        __syncthreads();
        const int kn = min(DK, d - k0);  // padded features would add pow(0, p) terms
        for (int kk = 0; kk < kn; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double t = __dsub_rn(a[i], b[j]);
                    double term;
                    if (KIND == 0) term = fabs(t);
                    else if (KIND == 1) term = __dmul_rn(t, t);
                    else if (KIND == 2) term = ipow(t, ip);
                    else term = pow(t, dp);
                    acc[i][j] = __dadd_rn(acc[i][j], term);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty + 16 * i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx + 16 * j;
            double v = acc[i][j];
            if (KIND == 1) v = sqrt(v);
            else if (KIND >= 2) v = pow(v, KIND == 2 ? 1.0 / (double)ip : 1.0 / dp);
            if (r < na && c < nb) D[(size_t)r * ldd + c] = v;
        }
    }
}

template <int KIND>
int launch_dm(const double *A, int na, int lda, const double *B, int nb, int ldb, int d, int ip,
              double dp, double *D, long long ldd, cudaStream_t st) {
    const dim3 grid(ceil_div(nb, DN), ceil_div(na, DM));
    distance_matrix_kernel<KIND><<<grid, DTPB, 0, st>>>(A, na, lda, B, nb, ldb, d, ip, dp, D, ldd);
    return launch_status("distance_matrix_kernel");
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_distance_matrix_f64(int kind, const double *A, int na, int lda,
                                        const double *B, int nb, int ldb, int d, int p_int,
                                        double p_real, double *D, long long ldd, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(kind >= 0 && kind <= 3, "fmlb_distance_matrix_f64: kind must be 0..3");
    FMLB_REQUIRE(na >= 0 && nb >= 0 && d >= 0 && lda >= d && ldb >= d && ldd >= nb,
                 "fmlb_distance_matrix_f64: bad sizes");
    FMLB_REQUIRE(ceil_div(na, DM) <= 65535, "fmlb_distance_matrix_f64: na too large");
    if (na == 0 || nb == 0) return FMLB_OK;
    FMLB_REQUIRE(A && B && D, "fmlb_distance_matrix_f64: null pointer");
    cudaStream_t st = FMLB_STREAM(stream);
    switch (kind) {
        case 0: return launch_dm<0>(A, na, lda, B, nb, ldb, d, 0, 0.0, D, ldd, st);
        case 1: return launch_dm<1>(A, na, lda, B, nb, ldb, d, 0, 0.0, D, ldd, st);
        case 2: return launch_dm<2>(A, na, lda, B, nb, ldb, d, p_int, 0.0, D, ldd, st);
        default: return launch_dm<3>(A, na, lda, B, nb, ldb, d, 0, p_real, D, ldd, st);
    }
}
