// Atomic vector kernels over per-atom descriptors (local / atomic Coulomb
// matrices):
//
//   K[k, i, j] = sum_{ia < n1[i], ja < n2[j]} exp(c_k * d(x1[i, ia], x2[j, ja]))
//
//   Gaussian  (fkernels.f90:106-162): d = sum_f (a_f - b_f)^2, c_k = -0.5 / sigma_k^2
//   Laplacian (fkernels.f90:23-104):  d = sum_f |a_f - b_f|,   c_k = -1 / sigma_k
//
// Layout: X (nm, amax, d) row-major FP64 (molecule, atom, feature); K
// (nsig, nm1, nm2) row-major, the reference's kernels(k, i, j) order.
//
// One CTA per molecule pair. Feature chunks of both molecules' atoms are staged
// in shared memory; each thread owns up to PP atom pairs (p = ja * n1 + ia, the
// reference's column-major atomic_distance order) and accumulates d in feature
// order, as the reference's sum does. exp(c_k d) is summed per thread into a
// per-sigma slot and the slots are combined by a fixed tree, so the result does
// not depend on scheduling.
#include <math.h>

#include "common.cuh"
#include "fmlb.h"

namespace fmlb {
namespace {

constexpr int VK_TPB = 64;     // threads per CTA
constexpr int VK_FCH = 32;     // features per shared-memory chunk
constexpr int VK_FS = 33;      // padded row stride of a chunk
constexpr int VK_MAX_ATOMS = 128;
constexpr int VK_MAX_SIGMAS = 32;

struct Coefs {
    double c[VK_MAX_SIGMAS];
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// PP atom pairs per thread per pass: the distance sums of the PP pairs are
// independent chains, interleaved feature by feature.
// Packed mode (O1 / O2 not null): molecule m's atoms are rows O[m] .. O[m+1]
// of a (total_atoms, d) matrix; N and amax then bound the counts only.
template <int KIND, int PP>
__global__ void __launch_bounds__(VK_TPB)
vector_kernels_kernel(const double *__restrict__ X1, const int *__restrict__ N1, int nm1,
                      int amax1, const double *__restrict__ X2, const int *__restrict__ N2,
                      int nm2, int amax2, int d, const Coefs coef, int nsig,
                      double *__restrict__ K, int *__restrict__ status,
                      const int *__restrict__ O1, const int *__restrict__ O2) {
    extern __shared__ double sm[];
    double *A = sm;                                   // [amax1][VK_FS]
    double *B = A + (size_t)amax1 * VK_FS;            // [amax2][VK_FS]
    double *acc = B + (size_t)amax2 * VK_FS;          // [nsig][VK_TPB]
    double *red = acc + (size_t)nsig * VK_TPB;        // [nsig][VK_TPB / 32]
    const long long pair = blockIdx.x;
    const int i = (int)(pair / nm2), j = (int)(pair % nm2);
    const int t = threadIdx.x;
    int ni = O1 ? O1[i + 1] - O1[i] : N1[i], nj = O2 ? O2[j + 1] - O2[j] : N2[j];
    if (ni < 0 || ni > amax1 || nj < 0 || nj > amax2) {  // rejected on the host as well
        if (t == 0 && status) atomicCAS(status, 0, 1);
        ni = min(max(ni, 0), amax1);
        nj = min(max(nj, 0), amax2);
    }
    for (int k = 0; k < nsig; ++k) acc[k * VK_TPB + t] = 0.0;
    const double *x1 = X1 + (O1 ? (size_t)O1[i] : (size_t)i * amax1) * d;
    const double *x2 = X2 + (O2 ? (size_t)O2[j] : (size_t)j * amax2) * d;
    const int np = ni * nj;
    for (int p0 = 0; p0 < np; p0 += VK_TPB * PP) {
        double dist[PP];
        int oa[PP], ob[PP];
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            const int p = min(p0 + t + q * VK_TPB, np - 1);
            const int ja = p / ni;
            oa[q] = (p - ja * ni) * VK_FS;
            ob[q] = ja * VK_FS;
            dist[q] = 0.0;
        }
        for (int f0 = 0; f0 < d; f0 += VK_FCH) {
            const int fc = min(VK_FCH, d - f0);
            __syncthreads();
            for (int e = t; e < ni * VK_FCH; e += VK_TPB) {
                const int a = e / VK_FCH, f = e - a * VK_FCH;
                if (f < fc) A[a * VK_FS + f] = x1[(size_t)a * d + f0 + f];
            }
            for (int e = t; e < nj * VK_FCH; e += VK_TPB) {
                const int b = e / VK_FCH, f = e - b * VK_FCH;
                if (f < fc) B[b * VK_FS + f] = x2[(size_t)b * d + f0 + f];
            }
            __syncthreads();
#pragma unroll 4
            for (int f = 0; f < fc; ++f) {
#pragma unroll
                for (int q = 0; q < PP; ++q) {
                    const double e = __dsub_rn(A[oa[q] + f], B[ob[q] + f]);
                    dist[q] = __dadd_rn(dist[q], KIND == 0 ? __dmul_rn(e, e) : fabs(e));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            if (p0 + t + q * VK_TPB < np)
                for (int k = 0; k < nsig; ++k)
                    acc[k * VK_TPB + t] += exp(dist[q] * coef.c[k]);
        }
    }
    // fixed-order combination: shuffle tree per warp, then the warps in order
    const int lane = t & 31, warp = t >> 5;
    for (int k = 0; k < nsig; ++k) {
        const double s = warp_sum_d(acc[k * VK_TPB + t]);
        if (lane == 0) red[k * (VK_TPB / 32) + warp] = s;
    }
    __syncthreads();
    for (int k = t; k < nsig; k += VK_TPB) {
        double s = 0.0;
        for (int w = 0; w < VK_TPB / 32; ++w) s += red[k * (VK_TPB / 32) + w];
        K[((size_t)k * nm1 + i) * nm2 + j] = s;
    }
}

size_t vk_smem_bytes(int amax1, int amax2, int nsig) {
    return sizeof(double) * ((size_t)(amax1 + amax2) * VK_FS + (size_t)nsig * VK_TPB +
                             (size_t)nsig * (VK_TPB / 32));
}

template <int KIND, int PP>
int launch_vk(const double *X1, const int *N1, int nm1, int amax1, const double *X2,
              const int *N2, int nm2, int amax2, int d, const Coefs &coef, int nsig, double *K,
              int *status, const int *O1, const int *O2, cudaStream_t st) {
    const size_t smem = vk_smem_bytes(amax1, amax2, nsig);
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(vector_kernels_kernel<KIND, PP>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem),
                         "cudaFuncSetAttribute"));
    vector_kernels_kernel<KIND, PP><<<(unsigned)((long long)nm1 * nm2), VK_TPB, smem, st>>>(
        X1, N1, nm1, amax1, X2, N2, nm2, amax2, d, coef, nsig, K, status, O1, O2);
    return launch_status(KIND == 0 ? "vector_kernels_kernel<gaussian>"
                                   : "vector_kernels_kernel<laplacian>");
}

// pairs per thread: the smallest of 2, 4, 6, 9, 12, 16 that covers the
// largest molecule pair in one pass (16 and several passes above that)
template <int KIND>
int launch_vk_pp(int pairs, const double *X1, const int *N1, int nm1, int amax1,
                 const double *X2, const int *N2, int nm2, int amax2, int d, const Coefs &coef,
                 int nsig, double *K, int *status, const int *O1, const int *O2,
                 cudaStream_t st) {
#define FMLB_VK(PP)                                                                            \
    if (pairs <= PP * VK_TPB || PP == 16)                                                     \
        return launch_vk<KIND, PP>(X1, N1, nm1, amax1, X2, N2, nm2, amax2, d, coef, nsig, K,  \
                                   status, O1, O2, st);
    FMLB_VK(2) FMLB_VK(4) FMLB_VK(6) FMLB_VK(9) FMLB_VK(12) FMLB_VK(16)
#undef FMLB_VK
    return FMLB_OK;
}

}  // namespace
}  // namespace fmlb

static int vector_kernels_impl(int kind, const double *X1, const int *N1, int nm1, int amax1,
                               const double *X2, const int *N2, int nm2, int amax2, int d,
                               const double *sigmas_host, int nsig, double *K, int *status,
                               const int *O1, const int *O2, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(kind == 0 || kind == 1, "fmlb_vector_kernels_f64: kind must be 0 or 1");
    FMLB_REQUIRE(nm1 >= 0 && nm2 >= 0 && d >= 0, "fmlb_vector_kernels_f64: bad sizes");
    FMLB_REQUIRE(amax1 >= 1 && amax1 <= VK_MAX_ATOMS && amax2 >= 1 && amax2 <= VK_MAX_ATOMS,
                 "fmlb_vector_kernels_f64: atoms per molecule must be 1..%d", VK_MAX_ATOMS);
    FMLB_REQUIRE(nsig >= 1 && nsig <= VK_MAX_SIGMAS,
                 "fmlb_vector_kernels_f64: nsig=%d outside 1..%d", nsig, VK_MAX_SIGMAS);
    FMLB_REQUIRE(sigmas_host, "fmlb_vector_kernels_f64: null sigmas");
    if ((long long)nm1 * nm2 == 0) return FMLB_OK;
    FMLB_REQUIRE(X1 && (N1 || O1) && X2 && (N2 || O2) && K,
                 "fmlb_vector_kernels_f64: null pointer");
    Coefs coef;
    for (int k = 0; k < nsig; ++k) {
        FMLB_REQUIRE(sigmas_host[k] > 0.0, "fmlb_vector_kernels_f64: sigma %d not positive", k);
        coef.c[k] = kind == 0 ? -0.5 / (sigmas_host[k] * sigmas_host[k]) : -1.0 / sigmas_host[k];
    }
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE((long long)nm1 * nm2 < 0x7fffffffLL,
                 "fmlb_vector_kernels_f64: too many molecule pairs");
    const int pairs = amax1 * amax2;
    if (kind == 0)
        return launch_vk_pp<0>(pairs, X1, N1, nm1, amax1, X2, N2, nm2, amax2, d, coef, nsig, K,
                               status, O1, O2, st);
    return launch_vk_pp<1>(pairs, X1, N1, nm1, amax1, X2, N2, nm2, amax2, d, coef, nsig, K,
                           status, O1, O2, st);
}

extern "C" int fmlb_vector_kernels_f64(int kind, const double *X1, const int *N1, int nm1,
                                       int amax1, const double *X2, const int *N2, int nm2,
                                       int amax2, int d, const double *sigmas_host, int nsig,
                                       double *K, int *status, void *stream) {
    return vector_kernels_impl(kind, X1, N1, nm1, amax1, X2, N2, nm2, amax2, d, sigmas_host,
                               nsig, K, status, nullptr, nullptr, stream);
}

// Packed form: X (total_atoms, d) rows with molecule offsets O (nm + 1);
// amax bounds the atoms of one molecule (checked on the device through
// status). The molecule kernel of fget_alpha (fkernels.f90:380-440) is the
// Laplacian form with X1 = X2.
extern "C" int fmlb_vector_kernels_packed_f64(int kind, const double *X1, const int *O1, int nm1,
                                              int amax1, const double *X2, const int *O2, int nm2,
                                              int amax2, int d, const double *sigmas_host,
                                              int nsig, double *K, int *status, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(nm1 == 0 || O1, "fmlb_vector_kernels_packed_f64: null offsets");
    FMLB_REQUIRE(nm2 == 0 || O2, "fmlb_vector_kernels_packed_f64: null offsets");
    return vector_kernels_impl(kind, X1, nullptr, nm1, amax1, X2, nullptr, nm2, amax2, d,
                               sigmas_host, nsig, K, status, O1, O2, stream);
}
