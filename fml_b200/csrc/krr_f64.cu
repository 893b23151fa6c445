// KRR helpers on the FP64 path:
//   * fmlb_add_diagonal_f64: A[i, i] += lambda (the user-side K + lambda*I);
//   * fmlb_kernel_predict_f64: y_s[q] = sum_t k_s(Xq[q], Xt[t]) alpha_s[t] for
//     every sigma, with the kernel matrix never written to memory (the user-side
//     prediction K_test @ alpha, fused; reference pattern fget_prediction,
//     fml/kernels/fkernels.f90:480-539);
//   * fmlb_gemv_f64: y = M x for a stored kernel matrix (the user-side
//     K_test @ alpha when the test kernel was built separately, e.g. ARAD).
// The prediction is split over the training set into fixed chunks whose
// partial sums are reduced in a second pass in a fixed order (deterministic).
#include <math.h>

#include <algorithm>

#include <limits.h>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, TPB = 256, MAXSIG = 8;
constexpr int CHUNK = 1024;  // training points per split

struct Scales {
    double s[MAXSIG];
};

__global__ void add_diagonal_kernel(double *A, long long lda, int n, double lam) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) A[(size_t)i * lda + i] += lam;
}

template <bool kL1>
__global__ void __launch_bounds__(TPB)
predict_partial_kernel(const double *__restrict__ Q, int nq, int ldq, const double *__restrict__ T,
                       int nt, int ldt, int d, Scales sc, int nsig,
                       const double *__restrict__ alpha, long long lda_alpha,
                       double *__restrict__ partial) {
    __shared__ double As[BK][BM + 1];
    __shared__ double Bs[BK][BN + 1];
    __shared__ double red[MAXSIG][BM];
    const int row0 = blockIdx.x * BM;
    const int split = blockIdx.y;
    const int t_begin = split * CHUNK, t_end = min(nt, t_begin + CHUNK);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int lk = threadIdx.x & 15, lr = threadIdx.x >> 4;

    double out[MAXSIG][4];
#pragma unroll
    for (int s = 0; s < MAXSIG; ++s)
#pragma unroll
        for (int i = 0; i < 4; ++i) out[s][i] = 0.0;

    for (int col0 = t_begin; col0 < t_end; col0 += BN) {
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        for (int k0 = 0; k0 < d; k0 += BK) {
            const int k = k0 + lk;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int ra = row0 + lr + 16 * r;
                As[lk][lr + 16 * r] = (ra < nq && k < d) ? Q[(size_t)ra * ldq + k] : 0.0;
                const int rb = col0 + lr + 16 * r;
                Bs[lk][lr + 16 * r] = (rb < t_end && k < d) ? T[(size_t)rb * ldt + k] : 0.0;
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
                        if (kL1) acc[i][j] += fabs(t);
                        else acc[i][j] = fma(t, t, acc[i][j]);
                    }
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx + 16 * j;
            if (c < t_end) {
#pragma unroll
                for (int s = 0; s < MAXSIG; ++s) {
                    if (s < nsig) {
                        const double a = alpha[s * lda_alpha + c];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            out[s][i] = fma(exp(sc.s[s] * acc[i][j]), a, out[s][i]);
                    }
                }
            }
        }
    }
    // reduce over the 16 threads (tx) sharing each row, in a fixed order
#pragma unroll
    for (int s = 0; s < MAXSIG; ++s) {
        if (s < nsig) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                double v = out[s][i];
                for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (tx == 0) red[s][ty + 16 * i] = v;
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nsig * BM; t += TPB) {
        const int s = t / BM, r = t % BM;
        if (row0 + r < nq) partial[((size_t)split * nsig + s) * nq + row0 + r] = red[s][r];
    }
}

__global__ void reduce_splits_kernel(const double *__restrict__ partial, int nsplit, int nsig,
                                     int nq, double *__restrict__ y, long long ldy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsig * nq) return;
    const int s = t / nq, q = t % nq;
    double v = 0.0;
    for (int p = 0; p < nsplit; ++p) v += partial[((size_t)p * nsig + s) * nq + q];
    y[s * ldy + q] = v;
}

// one warp per row, lanes stride the columns, fixed shuffle tree (deterministic)
__global__ void gemv_rows_kernel(const double *__restrict__ M, long long ldm, int rows, int cols,
                                 const double *__restrict__ x, double *__restrict__ y) {
    const int warp = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const double *m = M + (size_t)warp * ldm;
    double v = 0.0;
    for (int t = lane; t < cols; t += 32) v = fma(m[t], x[t], v);
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) y[warp] = v;
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_gemv_f64(const double *M, long long ldm, int rows, int cols, const double *x,
                             double *y, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(rows >= 0 && cols >= 0 && ldm >= cols, "fmlb_gemv_f64: bad sizes");
    if (rows == 0) return FMLB_OK;
    FMLB_REQUIRE(M && x && y, "fmlb_gemv_f64: null pointer");
    gemv_rows_kernel<<<ceil_div(rows, 8), 256, 0, FMLB_STREAM(stream)>>>(M, ldm, rows, cols, x, y);
    return launch_status("gemv_rows_kernel");
}

extern "C" int fmlb_add_diagonal_f64(double *A, long long lda, int n, double lam, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(n >= 0 && lda >= n, "fmlb_add_diagonal_f64: bad sizes");
    if (n == 0) return FMLB_OK;
    add_diagonal_kernel<<<ceil_div(n, 256), 256, 0, FMLB_STREAM(stream)>>>(A, lda, n, lam);
    return launch_status("add_diagonal_kernel");
}

extern "C" size_t fmlb_kernel_predict_workspace_bytes(int nq, int nt, int nsigma) {
    if (nq <= 0 || nt <= 0 || nsigma <= 0) return 256;
    const size_t nsplit = (size_t)(nt + fmlb::CHUNK - 1) / fmlb::CHUNK;
    return nsplit * nsigma * nq * sizeof(double);
}

extern "C" int fmlb_kernel_predict_f64(int kind, const double *Xq, int nq, int ldq,
                                       const double *Xt, int nt, int ldt, int d,
                                       const double *sigmas_host, int nsigma, const double *alpha,
                                       long long lda_alpha, double *y, long long ldy,
                                       void *workspace, size_t ws_bytes, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(kind == 0 || kind == 1, "fmlb_kernel_predict_f64: kind must be 0 (gaussian) "
                                         "or 1 (laplacian)");
    FMLB_REQUIRE(nq >= 0 && nt >= 0 && d >= 1 && ldq >= d && ldt >= d,
                 "fmlb_kernel_predict_f64: bad sizes");
    FMLB_REQUIRE(nsigma >= 1 && nsigma <= MAXSIG && sigmas_host,
                 "fmlb_kernel_predict_f64: nsigma must be 1..%d", MAXSIG);
    FMLB_REQUIRE(lda_alpha >= nt && ldy >= nq, "fmlb_kernel_predict_f64: bad alpha / y stride");
    FMLB_REQUIRE((long long)nsigma * nq < INT_MAX,
                 "fmlb_kernel_predict_f64: nsigma * nq = %lld must stay below 2^31",
                 (long long)nsigma * nq);
    if (nq == 0) return FMLB_OK;
    if (nt == 0) {
        for (int s = 0; s < nsigma; ++s)
            FMLB_TRY(cuda_status(cudaMemsetAsync(y + s * ldy, 0, sizeof(double) * nq, st),
                                 "fmlb_kernel_predict_f64: memset"));
        return FMLB_OK;
    }
    const size_t need = fmlb_kernel_predict_workspace_bytes(nq, nt, nsigma);
    if (ws_bytes < need || !workspace) {
        set_error("fmlb_kernel_predict_f64: workspace %zu < %zu bytes", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    Scales sc;
    for (int s = 0; s < nsigma; ++s) {
        const double sg = sigmas_host[s];
        sc.s[s] = kind == 1 ? -1.0 / sg : -0.5 / (sg * sg);
    }
    const int nsplit = ceil_div(nt, CHUNK);
    double *partial = static_cast<double *>(workspace);
    dim3 grid(ceil_div(nq, BM), nsplit);
    FMLB_REQUIRE(grid.y <= 65535, "fmlb_kernel_predict_f64: training set too large");
    if (kind == 0)
        predict_partial_kernel<false><<<grid, TPB, 0, st>>>(Xq, nq, ldq, Xt, nt, ldt, d, sc,
                                                            nsigma, alpha, lda_alpha, partial);
    else
        predict_partial_kernel<true><<<grid, TPB, 0, st>>>(Xq, nq, ldq, Xt, nt, ldt, d, sc, nsigma,
                                                           alpha, lda_alpha, partial);
    FMLB_TRY(launch_status("predict_partial_kernel"));
    reduce_splits_kernel<<<ceil_div((long)nsigma * nq, 256), 256, 0, st>>>(partial, nsplit, nsigma,
                                                                          nq, y, ldy);
    return launch_status("reduce_splits_kernel");
}

// ---------------------------------------------------------------------------
// Allocation-free prediction.
//
// Some callers cannot allocate device memory on the call path: an inference
// server whose memory is reserved up front by its own arena, a host library
// that receives only its input and output buffers from a framework that owns
// all device allocations, or code that must not reach cudaMalloc's implicit
// synchronisation. For them this variant keeps its split partial sums in the
// file-scope array below instead of a caller-provided workspace. The array is
// part of the module image: every GPU that loads the library holds it
// (8 MiB) until the process exits.
//
// The array's name in host code is only a host-side stand-in, so its device
// address is looked up once per device with cudaGetSymbolAddress, with that
// device current, on the first call made on that device. Make that first call
// before any stream capture. All calls share the array; a call fully
// overwrites the part it reads, so nothing needs clearing between calls, but
// calls that overlap on the GPU (different streams, or host threads) race on
// it and must be serialised by the caller. The looked-up address is cached per
// device for the life of the process: it does not survive cudaDeviceReset
// (after which the module may load at another address), so a process that
// resets a device must not call this entry point on it again.
// ---------------------------------------------------------------------------
#include <mutex>

namespace fmlb {
namespace {

constexpr size_t kNoAllocScratchDoubles = (size_t)1 << 20;  // 8 MiB
__device__ __align__(256) double g_predict_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

int noalloc_scratch(double **out) {
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_kernel_predict_f64_noalloc: cudaGetDevice"));
    FMLB_REQUIRE(dev >= 0 && dev < kMaxDevices,
                 "fmlb_kernel_predict_f64_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        FMLB_TRY(cuda_status(cudaGetSymbolAddress(&p, g_predict_scratch),
                             "fmlb_kernel_predict_f64_noalloc: cudaGetSymbolAddress"));
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return FMLB_OK;
}

}  // namespace
}  // namespace fmlb

extern "C" int fmlb_kernel_predict_f64_noalloc(int kind, const double *Xq, int nq, int ldq,
                                               const double *Xt, int nt, int ldt, int d,
                                               const double *sigmas_host, int nsigma,
                                               const double *alpha, long long lda_alpha,
                                               double *y, long long ldy, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(kind == 0 || kind == 1, "fmlb_kernel_predict_f64_noalloc: kind must be 0 "
                                         "(gaussian) or 1 (laplacian)");
    FMLB_REQUIRE(nq >= 0 && nt >= 0 && d >= 1 && ldq >= d && ldt >= d,
                 "fmlb_kernel_predict_f64_noalloc: bad sizes");
    FMLB_REQUIRE(nsigma >= 1 && nsigma <= MAXSIG && sigmas_host,
                 "fmlb_kernel_predict_f64_noalloc: nsigma must be 1..%d", MAXSIG);
    FMLB_REQUIRE(lda_alpha >= nt && ldy >= nq,
                 "fmlb_kernel_predict_f64_noalloc: bad alpha / y stride");
    if (nq == 0) return FMLB_OK;
    if (nt == 0) {
        for (int s = 0; s < nsigma; ++s)
            FMLB_TRY(cuda_status(cudaMemsetAsync(y + s * ldy, 0, sizeof(double) * nq, st),
                                 "fmlb_kernel_predict_f64_noalloc: memset"));
        return FMLB_OK;
    }
    const int nsplit = ceil_div(nt, CHUNK);
    const size_t need = (size_t)nsplit * nsigma * nq;
    FMLB_REQUIRE(need <= kNoAllocScratchDoubles,
                 "fmlb_kernel_predict_f64_noalloc: ceil(nt/%d) * nsigma * nq = %zu exceeds the "
                 "fixed scratch of %zu doubles (8 MiB); split the queries or use "
                 "fmlb_kernel_predict_f64 with a workspace",
                 CHUNK, need, kNoAllocScratchDoubles);
    double *partial = nullptr;
    FMLB_TRY(noalloc_scratch(&partial));
    Scales sc;
    for (int s = 0; s < nsigma; ++s) {
        const double sg = sigmas_host[s];
        sc.s[s] = kind == 1 ? -1.0 / sg : -0.5 / (sg * sg);
    }
    dim3 grid(ceil_div(nq, BM), nsplit);
    FMLB_REQUIRE(grid.y <= 65535, "fmlb_kernel_predict_f64_noalloc: training set too large");
    if (kind == 0)
        predict_partial_kernel<false><<<grid, TPB, 0, st>>>(Xq, nq, ldq, Xt, nt, ldt, d, sc,
                                                            nsigma, alpha, lda_alpha, partial);
    else
        predict_partial_kernel<true><<<grid, TPB, 0, st>>>(Xq, nq, ldq, Xt, nt, ldt, d, sc, nsigma,
                                                           alpha, lda_alpha, partial);
    FMLB_TRY(launch_status("predict_partial_kernel"));
    reduce_splits_kernel<<<ceil_div((long)nsigma * nq, 256), 256, 0, st>>>(partial, nsplit, nsigma,
                                                                          nq, y, ldy);
    return launch_status("reduce_splits_kernel");
}
