// ARAD molecular kernels: fget_kernels_arad / fget_symmetric_kernels_arad,
// fml/kernels/farad_kernels.f90:439-755, core atomic_distl2 :29-90.
//
//   K[s, I, J] = sum_{i1 < n_I, j1 < n_J} exp(-l2(i1, j1) / sigma_s^2)
//   l2 = self(I, i1) + self(J, j1) - 2 * S(i1, j1) * stoch(i1, j1), |l2| < eps -> 0
//   S  = sum over neighbour pairs (m1, m2) within the cut of
//        exp(-(r1 - r2)^2 / (4 w^2)) xi1 xi2 stoch(m1, m2) (1 + c1 c2 + s1 s2),
//        only where (r1 - r2)^2 < (8 w)^2.
//
// Stage 1 (arad_prep_kernel) turns each descriptor into its neighbour-list
// prefix length (the reference's early exit at r > cut), the sine factors xi
// and the self terms. Stage 2 evaluates molecule pairs.
//
// The FP64 path keeps the reference's operation order (explicit _rn
// intrinsics, no contracted FMA). The FP32 path is the fast path; its
// neighbour data is re-packed as float4 {r, xi, xi*c, xi*s} + float2 {row, col}.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int MAXSIG = 16;

struct SigmaTable {
    double inv_sigma2[MAXSIG];  // -1 / sigma^2 (farad_kernels.f90:511)
};

struct AradParams {
    double width, cut, rw2, cw2, inv_width, maxg2, inv_cut;
};

// Per-set workspace views.
struct SetWs {
    int *nnb;        // (nm, amax)      neighbour prefix length
    double *xi;      // (nm, amax, amax) sine factors (FP64 path)
    double *self;    // (nm, amax)      self terms (FP64 path)
    float4 *pk;      // (nm, amax, amax) {r, xi, xi*c, xi*s} (FP32 path)
    float2 *pz;      // (nm, amax, amax) {row, col}         (FP32 path)
    float *self32;   // (nm, amax)
};

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t set_ws_bytes(int nm, int amax) {
    const size_t a2 = (size_t)nm * amax * amax, a1 = (size_t)nm * amax;
    return align256(a1 * sizeof(int)) + align256(a2 * sizeof(double)) +
           align256(a1 * sizeof(double)) + align256(a2 * sizeof(float4)) +
           align256(a2 * sizeof(float2)) + align256(a1 * sizeof(float));
}

SetWs carve(char *&p, int nm, int amax) {
    const size_t a2 = (size_t)nm * amax * amax, a1 = (size_t)nm * amax;
    SetWs w;
    w.nnb = reinterpret_cast<int *>(p); p += align256(a1 * sizeof(int));
    w.xi = reinterpret_cast<double *>(p); p += align256(a2 * sizeof(double));
    w.self = reinterpret_cast<double *>(p); p += align256(a1 * sizeof(double));
    w.pk = reinterpret_cast<float4 *>(p); p += align256(a2 * sizeof(float4));
    w.pz = reinterpret_cast<float2 *>(p); p += align256(a2 * sizeof(float2));
    w.self32 = reinterpret_cast<float *>(p); p += align256(a1 * sizeof(float));
    return w;
}

// atomic_distl2 in FP64, reference order (farad_kernels.f90:58-88).
// x = descriptor of one atom (5, amax); xi = its sine factors.
__device__ double distl2_f64(const double *x1, const double *xi1, int n1, const double *x2,
                             const double *xi2, int n2, int amax, const AradParams &P) {
    double aad = 0.0;
    for (int m1 = 0; m1 < n1; ++m1) {
        const double r1 = x1[m1];
        const double p1 = x1[amax + m1], g1 = x1[2 * amax + m1];
        const double c1 = x1[3 * amax + m1], s1 = x1[4 * amax + m1];
        const double e1 = xi1[m1];
        for (int m2 = 0; m2 < n2; ++m2) {
            const double r2 = x2[m2];
            const double dr = __dsub_rn(r2, r1);
            const double t = __dmul_rn(dr, dr);
            if (t < P.maxg2) {
                double d = __dmul_rn(__dmul_rn(exp(__dmul_rn(t, P.inv_width)), e1), xi2[m2]);
                const double dp = __dsub_rn(p1, x2[amax + m2]);
                const double dg = __dsub_rn(g1, x2[2 * amax + m2]);
                const double st = __ddiv_rn(
                    __dmul_rn(__ddiv_rn(P.rw2, __dadd_rn(P.rw2, __dmul_rn(dp, dp))), P.cw2),
                    __dadd_rn(P.cw2, __dmul_rn(dg, dg)));
                d = __dmul_rn(d, st);
                const double ang = __dadd_rn(__dadd_rn(1.0, __dmul_rn(c1, x2[3 * amax + m2])),
                                             __dmul_rn(s1, x2[4 * amax + m2]));
                aad = __dadd_rn(aad, __dmul_rn(d, ang));
            }
        }
    }
    return aad;
}

// FP32 form over the packed neighbour records.
__device__ __forceinline__ float distl2_f32(const float4 *a, const float2 *za, int n1,
                                            const float4 *b, const float2 *zb, int n2,
                                            float inv_w_log2, float maxg2, float rw2, float cw2) {
    float aad = 0.0f;
    for (int m1 = 0; m1 < n1; ++m1) {
        const float4 u = a[m1];
        const float2 zu = za[m1];
        for (int m2 = 0; m2 < n2; ++m2) {
            const float4 v = b[m2];
            const float dr = v.x - u.x;
            const float t = dr * dr;
            if (t < maxg2) {
                const float2 zv = zb[m2];
                const float dp = zu.x - zv.x, dg = zu.y - zv.y;
                const float st = __fdividef(rw2, rw2 + dp * dp) * __fdividef(cw2, cw2 + dg * dg);
                const float g = fmaf(u.z, v.z, fmaf(u.w, v.w, u.y * v.y));
                aad = fmaf(exp2f(t * inv_w_log2) * st, g, aad);
            }
        }
    }
    return aad;
}

// Stage 1: one thread per (molecule, atom).
__global__ void arad_prep_kernel(const double *__restrict__ X, const int *__restrict__ N, int nm,
                                 int amax, AradParams P, int conditional_sine, SetWs w) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nm * amax) return;
    const int m = (int)(gid / amax), a = (int)(gid % amax);
    const int n = min(max(N[m], 0), amax);  // counts beyond amax are clamped
    const size_t base = (size_t)m * amax + a;
    if (a >= n) {
        w.nnb[base] = 0;
        w.self[base] = 0.0;
        w.self32[base] = 0.0f;
        return;
    }
    const double *x = X + base * 5 * amax;
    // neighbour prefix: the loop of atomic_distl2 exits at the first r > cut
    int cnt = 0;
    while (cnt < n && !(x[cnt] > P.cut)) ++cnt;
    w.nnb[base] = cnt;
    double *xi = w.xi + base * amax;
    float4 *pk = w.pk + base * amax;
    float2 *pz = w.pz + base * amax;
    for (int k = 0; k < n; ++k) {
        const double r = x[k];
        double s = 0.0;  // farad_kernels.f90:516 zero-initialised table
        if (!conditional_sine || r < P.cut) s = __dsub_rn(1.0, sin(__dmul_rn(r, P.inv_cut)));
        xi[k] = s;
        if (k < cnt) {
            const double c = x[3 * amax + k], sn = x[4 * amax + k];
            pk[k] = make_float4((float)r, (float)s, (float)(s * c), (float)(s * sn));
            pz[k] = make_float2((float)x[amax + k], (float)x[2 * amax + k]);
        }
    }
    w.self[base] = distl2_f64(x, xi, cnt, x, xi, cnt, amax, P);
    const float inv_w_log2 = (float)(P.inv_width * 1.4426950408889634);
    w.self32[base] = distl2_f32(pk, pz, cnt, pk, pz, cnt, inv_w_log2, (float)P.maxg2,
                                (float)P.rw2, (float)P.cw2);
}

__device__ __forceinline__ void pair_index(long long t, int symmetric, int nm2, int &I, int &J) {
    if (symmetric) {
        int j = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)j * (j + 1) / 2 > t) --j;
        while ((long long)(j + 1) * (j + 2) / 2 <= t) ++j;
        J = j;
        I = (int)(t - (long long)j * (j + 1) / 2);
    } else {
        I = (int)(t / nm2);
        J = (int)(t % nm2);
    }
}

// Stage 2: one warp per molecule pair; lanes stride over atom pairs.
template <bool kF64>
__global__ void __launch_bounds__(128)
arad_pair_kernel(const double *__restrict__ X1, const double *__restrict__ Z1,
                 const int *__restrict__ N1, SetWs w1, int nm1, const double *__restrict__ X2,
                 const double *__restrict__ Z2, const int *__restrict__ N2, SetWs w2, int nm2,
                 int amax, AradParams P, SigmaTable sig, int nsig, int symmetric,
                 double *__restrict__ K) {
    const int lane = threadIdx.x & 31;
    const long long npairs = symmetric ? (long long)nm1 * (nm1 + 1) / 2 : (long long)nm1 * nm2;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const double eps = (double)5.0e-12f;  // single-precision literal in the source (:505)
    const float inv_w_log2 = (float)(P.inv_width * 1.4426950408889634);
    const float maxg2 = (float)P.maxg2, rw2f = (float)P.rw2, cw2f = (float)P.cw2;

    for (long long t = warp0; t < npairs; t += nwarps) {
        int I, J;
        pair_index(t, symmetric, nm2, I, J);
        const int nI = min(max(N1[I], 0), amax), nJ = min(max(N2[J], 0), amax);
        double acc[MAXSIG];
#pragma unroll
        for (int s = 0; s < MAXSIG; ++s) acc[s] = 0.0;
        const int P2 = nI * nJ;
        for (int p = lane; p < P2; p += 32) {
            const int i1 = p / nJ, j1 = p - i1 * nJ;
            const size_t b1 = (size_t)I * amax + i1, b2 = (size_t)J * amax + j1;
            const double dz1 = __dsub_rn(Z1[b1 * 2 + 0], Z2[b2 * 2 + 0]);
            const double dz2 = __dsub_rn(Z1[b1 * 2 + 1], Z2[b2 * 2 + 1]);
            const double stoch = __ddiv_rn(
                __dmul_rn(__ddiv_rn(P.rw2, __dadd_rn(P.rw2, __dmul_rn(dz1, dz1))), P.cw2),
                __dadd_rn(P.cw2, __dmul_rn(dz2, dz2)));
            double l2;
            if (kF64) {
                const double S = distl2_f64(X1 + b1 * 5 * amax, w1.xi + b1 * amax, w1.nnb[b1],
                                            X2 + b2 * 5 * amax, w2.xi + b2 * amax, w2.nnb[b2],
                                            amax, P);
                l2 = __dsub_rn(__dadd_rn(w1.self[b1], w2.self[b2]),
                               __dmul_rn(__dmul_rn(2.0, S), stoch));
            } else {
                const float S = distl2_f32(w1.pk + b1 * amax, w1.pz + b1 * amax, w1.nnb[b1],
                                           w2.pk + b2 * amax, w2.pz + b2 * amax, w2.nnb[b2],
                                           inv_w_log2, maxg2, rw2f, cw2f);
                l2 = (double)(w1.self32[b1] + w2.self32[b2] - 2.0f * S * (float)stoch);
            }
            if (fabs(l2) < eps) l2 = 0.0;  // :594
#pragma unroll
            for (int s = 0; s < MAXSIG; ++s)
                if (s < nsig) acc[s] += exp(l2 * sig.inv_sigma2[s]);
        }
#pragma unroll
        for (int s = 0; s < MAXSIG; ++s) {
            if (s < nsig) {
                double v = acc[s];
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) {
                    K[((size_t)s * nm1 + I) * nm2 + J] = v;
                    if (symmetric) K[((size_t)s * nm1 + J) * nm2 + I] = v;  // :744
                }
            }
        }
    }
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_arad_workspace_bytes(int nm1, int nm2, int amax, int symmetric) {
    if (nm1 < 0 || nm2 < 0 || amax < 1) return 0;
    return fmlb::set_ws_bytes(nm1, amax) + (symmetric ? 0 : fmlb::set_ws_bytes(nm2, amax));
}

extern "C" int fmlb_arad_kernels(const double *X1, const double *Z1, const int *N1, int nm1,
                                 const double *X2, const double *Z2, const int *N2, int nm2,
                                 int amax, const double *sigmas_host, int nsigma, double width,
                                 double cut_distance, double r_width, double c_width,
                                 int symmetric, int precision, double *K, void *workspace,
                                 size_t ws_bytes, void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(nm1 >= 0 && amax >= 1, "fmlb_arad_kernels: bad sizes");
    FMLB_REQUIRE(nsigma >= 1 && sigmas_host, "fmlb_arad_kernels: need at least one sigma");
    FMLB_REQUIRE(precision == 0 || precision == 1, "fmlb_arad_kernels: precision must be 0 or 1");
    if (symmetric) {
        X2 = X1; Z2 = Z1; N2 = N1; nm2 = nm1;
    }
    FMLB_REQUIRE(nm2 >= 0, "fmlb_arad_kernels: bad nm2");
    const size_t need = fmlb_arad_workspace_bytes(nm1, nm2, amax, symmetric);
    if (ws_bytes < need || (need && !workspace)) {
        set_error("fmlb_arad_kernels: workspace %zu bytes < required %zu", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    if (nm1 == 0 || nm2 == 0) return FMLB_OK;
    FMLB_REQUIRE(X1 && Z1 && N1 && X2 && Z2 && N2 && K, "fmlb_arad_kernels: null pointer");

    AradParams P;
    P.width = width;
    P.cut = cut_distance;
    P.rw2 = r_width * r_width;
    P.cw2 = c_width * c_width;
    P.inv_width = -1.0 / (4.0 * width * width);      // :58
    P.maxg2 = (8.0 * width) * (8.0 * width);          // :60
    P.inv_cut = (4.0 * atan(1.0)) / (2.0 * cut_distance);  // :502, :510

    char *p = static_cast<char *>(workspace);
    SetWs w1 = carve(p, nm1, amax);
    SetWs w2 = symmetric ? w1 : carve(p, nm2, amax);
    const int tpb = 128;
    {
        const long long n = (long long)nm1 * amax;
        arad_prep_kernel<<<ceil_div(n, tpb), tpb, 0, st>>>(X1, N1, nm1, amax, P, symmetric ? 0 : 1,
                                                           w1);
        FMLB_TRY(launch_status("arad_prep_kernel"));
    }
    if (!symmetric) {
        const long long n = (long long)nm2 * amax;
        arad_prep_kernel<<<ceil_div(n, tpb), tpb, 0, st>>>(X2, N2, nm2, amax, P, 1, w2);
        FMLB_TRY(launch_status("arad_prep_kernel"));
    }
    const long long npairs = symmetric ? (long long)nm1 * (nm1 + 1) / 2 : (long long)nm1 * nm2;
    const int blocks = (int)std::min<long long>(ceil_div(npairs, tpb / 32), (long long)sm_count() * 64);
    for (int s0 = 0; s0 < nsigma; s0 += MAXSIG) {
        const int ns = nsigma - s0 < MAXSIG ? nsigma - s0 : MAXSIG;
        SigmaTable sig;
        for (int s = 0; s < ns; ++s)
            sig.inv_sigma2[s] = -1.0 / (sigmas_host[s0 + s] * sigmas_host[s0 + s]);
        double *Ks = K + (size_t)s0 * nm1 * nm2;
        if (precision == 0)
            arad_pair_kernel<true><<<blocks, tpb, 0, st>>>(X1, Z1, N1, w1, nm1, X2, Z2, N2, w2, nm2,
                                                           amax, P, sig, ns, symmetric, Ks);
        else
            arad_pair_kernel<false><<<blocks, tpb, 0, st>>>(X1, Z1, N1, w1, nm1, X2, Z2, N2, w2,
                                                            nm2, amax, P, sig, ns, symmetric, Ks);
        FMLB_TRY(launch_status("arad_pair_kernel"));
    }
    return FMLB_OK;
}
