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
    double eps;  // |l2| below eps counts as 0
};

// Per-set workspace views.
struct SetWs {
    int *nnb;             // (nm, amax)       neighbour prefix length
    double *xi;           // (nm, amax, amax) sine factors (FP64 path)
    double *self;         // (nm, amax)       self terms (FP64 path)
    float4 *pk;           // (nm, amax, amax) {r, xi, xi*c, xi*s} (FP32 paths)
    float2 *pz;           // (nm, amax, amax) {row, col}         (generic FP32 path)
    float *self32;        // (nm, amax)       self terms (generic FP32 path)
    signed char *cls;     // (nm, amax, amax) element class of each neighbour (fast path)
    signed char *acls;    // (nm, amax)       element class of each atom (fast path)
    float *selff;         // (nm, amax)       self terms (fast path)
    float4 *spk;          // (nm, amax, amax) records of each molecule sorted by r (paired path)
    int *smeta;           // (nm, amax, amax) atom | class << 16 | 1 << 24 of each sorted record
    int *nrec;            // (nm)             records per molecule
};

// Element classes (distinct periodic-table positions) of the fast FP32 path:
// the stoichiometric factor between two classes comes from a small table.
constexpr int FC_MAXC = 16;
constexpr int FC_NPOS = 8 * 34;  // (row 0..7) * 34 + (col 0..33)
struct ClassInfo {
    int flag;                 // 0: fast path usable; otherwise why not
    int ncls;
    int present[FC_NPOS];
    signed char map[FC_NPOS]; // position -> class, -1 if absent
    float stoch[FC_MAXC * FC_MAXC];
};

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t set_ws_bytes(int nm, int amax) {
    const size_t a2 = (size_t)nm * amax * amax, a1 = (size_t)nm * amax;
    return align256(a1 * sizeof(int)) + align256(a2 * sizeof(double)) +
           align256(a1 * sizeof(double)) + align256(a2 * sizeof(float4)) +
           align256(a2 * sizeof(float2)) + align256(a1 * sizeof(float)) + align256(a2) +
           align256(a1) + align256(a1 * sizeof(float)) + align256(a2 * sizeof(float4)) +
           align256(a2 * sizeof(int)) + align256((size_t)nm * sizeof(int));
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
    w.cls = reinterpret_cast<signed char *>(p); p += align256(a2);
    w.acls = reinterpret_cast<signed char *>(p); p += align256(a1);
    w.selff = reinterpret_cast<float *>(p); p += align256(a1 * sizeof(float));
    w.spk = reinterpret_cast<float4 *>(p); p += align256(a2 * sizeof(float4));
    w.smeta = reinterpret_cast<int *>(p); p += align256(a2 * sizeof(int));
    w.nrec = reinterpret_cast<int *>(p); p += align256((size_t)nm * sizeof(int));
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

// FP32 form over the packed neighbour records. The records hold the distance
// pre-scaled by rs = sqrt(-inv_width * log2 e), so exp(dr^2 inv_width) =
// exp2(-(dr')^2) and the window (dr)^2 < (8 w)^2 is (dr')^2 < maxg2s.
__device__ __forceinline__ float distl2_f32(const float4 *a, const float2 *za, int n1,
                                            const float4 *b, const float2 *zb, int n2,
                                            float maxg2s, float rw2, float cw2) {
    float aad = 0.0f;
    for (int m1 = 0; m1 < n1; ++m1) {
        const float4 u = a[m1];
        const float2 zu = za[m1];
        for (int m2 = 0; m2 < n2; ++m2) {
            const float4 v = b[m2];
            const float dr = v.x - u.x;
            const float t = dr * dr;
            if (t < maxg2s) {
                const float2 zv = zb[m2];
                const float dp = zu.x - zv.x, dg = zu.y - zv.y;
                const float st = __fdividef(rw2, rw2 + dp * dp) * __fdividef(cw2, cw2 + dg * dg);
                const float g = fmaf(u.z, v.z, fmaf(u.w, v.w, u.y * v.y));
                aad = fmaf(exp2f(-t) * st, g, aad);
            }
        }
    }
    return aad;
}

__host__ __device__ inline double fp32_scale(const AradParams &P) {
    return sqrt(-P.inv_width * 1.4426950408889634);
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
            pk[k] = make_float4((float)(r * fp32_scale(P)), (float)s, (float)(s * c),
                                (float)(s * sn));
            pz[k] = make_float2((float)x[amax + k], (float)x[2 * amax + k]);
        }
    }
    w.self[base] = distl2_f64(x, xi, cnt, x, xi, cnt, amax, P);
    const float maxg2s = (float)(P.maxg2 * fp32_scale(P) * fp32_scale(P));
    w.self32[base] = distl2_f32(pk, pz, cnt, pk, pz, cnt, maxg2s, (float)P.rw2, (float)P.cw2);
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
// kDist: store every atom pair's l2 in D (nm1, nm2, amax, amax) instead of
// the kernel sums (atomic_arad_l2_distance_all, farad.f90:452-600).
template <bool kF64, bool kDist = false>
__global__ void __launch_bounds__(128)
arad_pair_kernel(const double *__restrict__ X1, const double *__restrict__ Z1,
                 const int *__restrict__ N1, SetWs w1, int nm1, const double *__restrict__ X2,
                 const double *__restrict__ Z2, const int *__restrict__ N2, SetWs w2, int nm2,
                 int amax, AradParams P, SigmaTable sig, int nsig, int symmetric,
                 double *__restrict__ K, const ClassInfo *fast_ci,
                 double *__restrict__ D = nullptr) {
    // when the fast FP32 kernel handled this call, the generic one does nothing
    if (fast_ci && fast_ci->flag == 0) return;
    const int lane = threadIdx.x & 31;
    const long long npairs = symmetric ? (long long)nm1 * (nm1 + 1) / 2 : (long long)nm1 * nm2;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const double eps = P.eps;
    const float maxg2s = (float)(P.maxg2 * fp32_scale(P) * fp32_scale(P));
    const float rw2f = (float)P.rw2, cw2f = (float)P.cw2;

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
                                           maxg2s, rw2f, cw2f);
                l2 = (double)(w1.self32[b1] + w2.self32[b2] - 2.0f * S * (float)stoch);
            }
            if (fabs(l2) < eps) l2 = 0.0;  // :594
            if (kDist) {  // farad.f90:589
                D[(((size_t)I * nm2 + J) * amax + i1) * amax + j1] = l2;
                continue;
            }
#pragma unroll
            for (int s = 0; s < MAXSIG; ++s)
                if (s < nsig) acc[s] += exp(l2 * sig.inv_sigma2[s]);
        }
        if (kDist) continue;
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

// ---------------------------------------------------------------------------
// Fast FP32 path.
//
// Molecule I's neighbour records (one record = one neighbour m1 of one atom
// i1) are packed, whole atoms at a time, into passes of 32 lanes; molecule J
// is staged in shared memory. A work item (pass p, atom j1 of J) lets every
// lane sum its record against all of j1's neighbours (broadcast reads), then a
// segmented warp scan forms S(i1, j1) for every atom i1 of the pass at the
// last lane of its segment, which applies the kernel exponentials for every
// sigma. Self terms come from the same code (J = I), so l2 cancels exactly for
// identical environments.
// ---------------------------------------------------------------------------
constexpr int FC_BM = 8, FC_WARPS = 8, FC_MAXREC = 1024, FC_MAXA = 32, FC_MAXSIG = 8;
constexpr int FC_SST = FC_MAXC + 1;

__device__ __forceinline__ int ptp_pos(double row, double col) {
    const double r = rint(row), c = rint(col);
    if (r != row || c != col || r < 0.0 || r > 7.0 || c < 0.0 || c > 33.0) return -1;
    return (int)r * 34 + (int)c;
}

// marks the periodic-table positions of the atoms and their neighbours
__global__ void arad_class_scan_kernel(const double *__restrict__ X, const double *__restrict__ Z,
                                       const int *__restrict__ N, int nm, int amax, double cut,
                                       ClassInfo *ci) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nm * amax) return;
    const int m = (int)(gid / amax), a = (int)(gid % amax);
    const int n = min(max(N[m], 0), amax);
    if (a >= n) return;
    const size_t base = (size_t)m * amax + a;
    int pos = ptp_pos(Z[base * 2 + 0], Z[base * 2 + 1]);
    if (pos < 0) { atomicOr(&ci->flag, 1); return; }
    atomicOr(&ci->present[pos], 1);
    const double *x = X + base * 5 * amax;
    for (int k = 0; k < n && !(x[k] > cut); ++k) {
        pos = ptp_pos(x[amax + k], x[2 * amax + k]);
        if (pos < 0) { atomicOr(&ci->flag, 1); return; }
        atomicOr(&ci->present[pos], 1);
    }
}

// one thread: class ids and the stoichiometric table (farad_kernels.f90:80-81)
__global__ void arad_class_build_kernel(ClassInfo *ci, double rw2, double cw2) {
    int rows[FC_MAXC], cols[FC_MAXC];
    int nc = 0;
    for (int pos = 0; pos < FC_NPOS; ++pos) {
        ci->map[pos] = -1;
        if (ci->present[pos]) {
            if (nc == FC_MAXC) { ci->flag |= 2; break; }
            rows[nc] = pos / 34;
            cols[nc] = pos % 34;
            ci->map[pos] = (signed char)nc;
            ++nc;
        }
    }
    ci->ncls = nc;
    for (int a = 0; a < FC_MAXC; ++a)
        for (int b = 0; b < FC_MAXC; ++b) {
            double v = 0.0;
            if (a < nc && b < nc) {
                const double dr = (double)(rows[a] - rows[b]), dc = (double)(cols[a] - cols[b]);
                v = rw2 / (rw2 + dr * dr) * cw2 / (cw2 + dc * dc);
            }
            ci->stoch[a * FC_MAXC + b] = (float)v;
        }
}

// element classes of every neighbour record and atom (after the class build)
__global__ void arad_class_assign_kernel(const double *__restrict__ X, const double *__restrict__ Z,
                                         const int *__restrict__ N, int nm, int amax,
                                         const ClassInfo *ci, SetWs w) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nm * amax) return;
    const int m = (int)(gid / amax), a = (int)(gid % amax);
    const int n = min(max(N[m], 0), amax);
    const size_t base = (size_t)m * amax + a;
    if (a >= n) { w.acls[base] = 0; return; }
    int pos = ptp_pos(Z[base * 2 + 0], Z[base * 2 + 1]);
    w.acls[base] = pos >= 0 ? max((int)ci->map[pos], 0) : 0;
    const double *x = X + base * 5 * amax;
    const int cnt = w.nnb[base];
    for (int k = 0; k < cnt; ++k) {
        pos = ptp_pos(x[amax + k], x[2 * amax + k]);
        w.cls[base * amax + k] = pos >= 0 ? (signed char)max((int)ci->map[pos], 0) : 0;
    }
}

// Paired path (at most FC_PC element classes): the records of J are stored two
// at a time, (r0, r1, xi0, xi1) and (xc0, xc1, xs0, xs1), so every lane
// evaluates two neighbour pairs per step with packed FP32x2 arithmetic
// (FADD2 / FMUL2 / FFMA2) and fetches both stoichiometric factors with one
// load from a per-class pair table. An atom with an odd neighbour count gets
// a padding record (r = 1e18, xi = 0) whose window test and exponential are 0.
constexpr int FC_PC = 8;
constexpr int FC_PTS = FC_PC * FC_PC + 1;  // pair-table row stride (float2): conflict-free rows
constexpr int FC_SS = FC_MAXA + 1;         // S row stride: lanes adding to different atoms i1
                                           // of one column j1 hit different banks

struct FastSmem {
    float4 recI[FC_MAXREC];      // molecule I, dense by atom, 32 records per pass
    int metaI[FC_MAXREC];        // atom | seg_start << 8 | cls << 16 | active << 24 | tail << 25
    float selfI[FC_MAXA];
    int aclsI[FC_MAXA];
    union {
        struct {
            float4 rec[FC_MAXREC];       // molecule J, dense by atom
            signed char cls[FC_MAXREC];  // element class of each record of J
        } s;
        struct {
            float4 a[FC_MAXREC / 2];     // (r0, r1, xi0, xi1) per record pair
            float4 b[FC_MAXREC / 2];     // (xc0, xc1, xs0, xs1)
            int k[FC_MAXREC / 2];        // cls0 * FC_PC + cls1: column of the pair table
        } p;
    } J;
    int offJ[FC_MAXA + 1];       // record offsets (scalar path) or pair offsets (paired path)
    float selfJ[FC_MAXA];
    int aclsJ[FC_MAXA];
    float stoch[FC_MAXC * FC_SST];  // row stride 17: lanes of different classes hit distinct banks
    float2 pt[FC_PC * FC_PTS];   // pt[c1][ca * FC_PC + cb] = (stoch(c1, ca), stoch(c1, cb))
    union {
        float f[FC_MAXA * FC_SS];      // scalar path: S(i1, j1), row stride FC_SS
        long long q[FC_MAXA * FC_SS];  // paired path: S(i1, j1) in fixed point (2^-32 units)
    } S;
    float passLo[FC_MAXREC / 32], passHi[FC_MAXREC / 32];  // r band of each I pass (paired)
    float red[FC_WARPS][FC_MAXSIG];
    int npassI, nI, nJ;
};

// Molecule I, dense: pass p holds records [32 p, 32 p + 32). Whole CTA; the
// caller synchronises before the records are read.
__device__ void fast_load_I(FastSmem &sm, const SetWs &w, int I, int amax, int nI,
                            bool use_self) {
    __shared__ int offI[FC_MAXA + 1];
    if (threadIdx.x < 32) {  // exclusive prefix of the neighbour counts (nI <= 32)
        const int a = threadIdx.x;
        const int cnt = a < nI ? w.nnb[(size_t)I * amax + a] : 0;
        int incl = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (a >= d) incl += o;
        }
        offI[a] = incl - cnt;
        if (a == 31) {
            offI[32] = incl;
            sm.npassI = (incl + 31) / 32;
            sm.nI = nI;
        }
    }
    __syncthreads();
    const int nrec = offI[32];
    const int nslot = sm.npassI * 32;
    for (int slot = nrec + threadIdx.x; slot < nslot; slot += blockDim.x) {
        sm.metaI[slot] = ((slot & 31) << 8);  // inactive lane, own segment, no tail
        sm.recI[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int t = threadIdx.x; t < nI * amax; t += blockDim.x) {
        const int a = t / amax, k = t % amax;
        const int beg = offI[a], cnt = offI[a + 1] - beg;
        if (k < cnt) {
            const int slot = beg + k;
            // segment = this atom's records inside this pass
            const int seg = max(beg, slot & ~31) & 31;
            const bool tail = (k == cnt - 1) || ((slot & 31) == 31);
            const size_t src = ((size_t)I * amax + a) * amax + k;
            sm.metaI[slot] = a | (seg << 8) | ((int)w.cls[src] << 16) | (1 << 24) |
                             ((tail ? 1 : 0) << 25);
            sm.recI[slot] = w.pk[src];
        }
    }
    for (int a = threadIdx.x; a < nI; a += blockDim.x) {
        sm.selfI[a] = use_self ? w.selff[(size_t)I * amax + a] : 0.0f;
        sm.aclsI[a] = w.acls[(size_t)I * amax + a];
    }
}

// Molecule J, dense by atom. Whole CTA; the caller synchronises before the
// records are read.
__device__ void fast_load_J(FastSmem &sm, const SetWs &w, int J, int amax, int nJ,
                            bool use_self) {
    if (threadIdx.x < 32) {  // exclusive prefix of the neighbour counts (nJ <= 32)
        const int a = threadIdx.x;
        const int cnt = a < nJ ? w.nnb[(size_t)J * amax + a] : 0;
        int incl = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (a >= d) incl += o;
        }
        sm.offJ[a] = incl - cnt;
        if (a == 31) {
            sm.offJ[32] = incl;
            sm.nJ = nJ;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nJ * amax; t += blockDim.x) {
        const int a = t / amax, k = t % amax;
        if (k < sm.offJ[a + 1] - sm.offJ[a]) {
            const int d = sm.offJ[a] + k;
            const size_t src = ((size_t)J * amax + a) * amax + k;
            sm.J.s.rec[d] = w.pk[src];
            sm.J.s.cls[d] = w.cls[src];
        }
    }
    for (int a = threadIdx.x; a < nJ; a += blockDim.x) {
        sm.selfJ[a] = use_self ? w.selff[(size_t)J * amax + a] : 0.0f;
        sm.aclsJ[a] = w.acls[(size_t)J * amax + a];
    }
}

// Molecule J in record pairs (paired path). Whole CTA; the caller synchronises
// before the records are read.
__device__ void fast_load_J_pairs(FastSmem &sm, const SetWs &w, int J, int amax, int nJ,
                                  bool use_self) {
    if (threadIdx.x < 32) {  // exclusive prefix of the padded pair counts (nJ <= 32)
        const int a = threadIdx.x;
        const int np = a < nJ ? (w.nnb[(size_t)J * amax + a] + 1) >> 1 : 0;
        int incl = np;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (a >= d) incl += o;
        }
        sm.offJ[a] = incl - np;
        if (a == 31) {
            sm.offJ[32] = incl;
            sm.nJ = nJ;
        }
    }
    __syncthreads();
    const int hp = (amax + 1) >> 1;
    for (int t = threadIdx.x; t < nJ * hp; t += blockDim.x) {
        const int a = t / hp, q = t - a * hp;
        const int beg = sm.offJ[a];
        if (q < sm.offJ[a + 1] - beg) {
            const size_t base = (size_t)J * amax + a;
            const int cnt = w.nnb[base];
            const size_t src = base * amax + 2 * q;
            const float4 r0 = w.pk[src];
            const int c0 = w.cls[src];
            float4 r1 = make_float4(1.0e18f, 0.0f, 0.0f, 0.0f);
            int c1 = 0;
            if (2 * q + 1 < cnt) {
                r1 = w.pk[src + 1];
                c1 = w.cls[src + 1];
            }
            sm.J.p.a[beg + q] = make_float4(r0.x, r1.x, r0.y, r1.y);
            sm.J.p.b[beg + q] = make_float4(r0.z, r1.z, r0.w, r1.w);
            sm.J.p.k[beg + q] = c0 * FC_PC + c1;
        }
    }
    for (int a = threadIdx.x; a < nJ; a += blockDim.x) {
        sm.selfJ[a] = use_self ? w.selff[(size_t)J * amax + a] : 0.0f;
        sm.aclsJ[a] = w.acls[(size_t)J * amax + a];
    }
}

__device__ __forceinline__ float set_lt(float a, float b) {  // 1.0f if a < b, else 0.0f
    float r;
    asm("set.lt.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// Paired work item over molecule I in radius bands: lane = one record of
// pass p and one of pass p + 1 (records of I sorted by r, 32 per pass),
// against the record pairs of atom j1 of J, two records per step with packed
// FP32x2 arithmetic; each J record pair is loaded once for four
// neighbour-pair evaluations. Every term is computed with the same operations
// as in fast_item. Records of j1 outside the (8w)^2 window of every lane of
// the two passes (j1's records are sorted by r) are skipped, and terms outside
// a record's own window are masked: both are exactly zero. The lane's sums are
// added to S(i1, j1) in 2^-32 fixed point, so the result does not depend on
// the order of the additions.
__device__ __forceinline__ void fast_item_band2(FastSmem &sm, int p, int j1, float maxg2s,
                                                float wd) {
    const int lane = threadIdx.x & 31;
    const bool two = p + 1 < sm.npassI;
    const float4 u0 = sm.recI[p * 32 + lane];
    const int meta0 = sm.metaI[p * 32 + lane];
    const float4 u1 = two ? sm.recI[(p + 1) * 32 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int meta1 = two ? sm.metaI[(p + 1) * 32 + lane] : 0;
    const float2 *ptrow0 = sm.pt + ((meta0 >> 16) & 0xff) * FC_PTS;
    const float2 *ptrow1 = sm.pt + ((meta1 >> 16) & 0xff) * FC_PTS;
    const float2 nux0 = make_float2(-u0.x, -u0.x), uy0 = make_float2(u0.y, u0.y),
                 uz0 = make_float2(u0.z, u0.z), uw0 = make_float2(u0.w, u0.w);
    const float2 nux1 = make_float2(-u1.x, -u1.x), uy1 = make_float2(u1.y, u1.y),
                 uz1 = make_float2(u1.z, u1.z), uw1 = make_float2(u1.w, u1.w);
    const int beg = sm.offJ[j1], end = sm.offJ[j1 + 1];
    const float lo = sm.passLo[p] - wd, hi = sm.passHi[two ? p + 1 : p] + wd;
    bool below = false, before = false;
    if (beg + lane < end) {
        const float4 A = sm.J.p.a[beg + lane];
        below = !(A.y > lo);
        before = A.x < hi;
    }
    const int mb = beg + __popc(__ballot_sync(0xffffffffu, below));
    const int me = beg + __popc(__ballot_sync(0xffffffffu, before));
    float2 acc0 = make_float2(0.0f, 0.0f), acc1 = make_float2(0.0f, 0.0f);
#pragma unroll 2
    for (int m = mb; m < me; ++m) {
        const float4 A = sm.J.p.a[m];
        const float4 B = sm.J.p.b[m];
        const int k = sm.J.p.k[m];
        const float2 st0 = ptrow0[k], st1 = ptrow1[k];
        const float2 rj = make_float2(A.x, A.y), xj = make_float2(A.z, A.w);
        const float2 cj = make_float2(B.x, B.y), sj = make_float2(B.z, B.w);
        {
            const float2 dr = __fadd2_rn(rj, nux0);
            const float2 t = __fmul2_rn(dr, dr);
            float e0, e1;
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e0) : "f"(-t.x));
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e1) : "f"(-t.y));
            const float2 g = __ffma2_rn(sj, uw0, __ffma2_rn(cj, uz0, __fmul2_rn(xj, uy0)));
            const float2 win = make_float2(set_lt(t.x, maxg2s), set_lt(t.y, maxg2s));
            const float2 eg = __fmul2_rn(__fmul2_rn(make_float2(e0, e1), st0), win);
            acc0 = __ffma2_rn(eg, g, acc0);
        }
        {
            const float2 dr = __fadd2_rn(rj, nux1);
            const float2 t = __fmul2_rn(dr, dr);
            float e0, e1;
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e0) : "f"(-t.x));
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e1) : "f"(-t.y));
            const float2 g = __ffma2_rn(sj, uw1, __ffma2_rn(cj, uz1, __fmul2_rn(xj, uy1)));
            const float2 win = make_float2(set_lt(t.x, maxg2s), set_lt(t.y, maxg2s));
            const float2 eg = __fmul2_rn(__fmul2_rn(make_float2(e0, e1), st1), win);
            acc1 = __ffma2_rn(eg, g, acc1);
        }
    }
    if ((meta0 >> 24) & 1) {
        const long long f = __float2ll_rn((acc0.x + acc0.y) * 4294967296.0f);
        if (f)
            atomicAdd(reinterpret_cast<unsigned long long *>(&sm.S.q[(meta0 & 0xff) * FC_SS + j1]),
                      (unsigned long long)f);
    }
    if ((meta1 >> 24) & 1) {
        const long long f = __float2ll_rn((acc1.x + acc1.y) * 4294967296.0f);
        if (f)
            atomicAdd(reinterpret_cast<unsigned long long *>(&sm.S.q[(meta1 & 0xff) * FC_SS + j1]),
                      (unsigned long long)f);
    }
}

// Work item (pass p, atom j1): the segment sums of the pass against j1 are
// added into S[i1][j1] by each segment's last lane (an atom split across two
// passes contributes two partial sums; two terms commute, so the result does
// not depend on their order).
__device__ __forceinline__ void fast_item(FastSmem &sm, int p, int j1, float maxg2s) {
    const int lane = threadIdx.x & 31;
    const float4 u = sm.recI[p * 32 + lane];
    const int meta = sm.metaI[p * 32 + lane];
    const float *strow = sm.stoch + ((meta >> 16) & 0xff) * FC_SST;
    const int beg = sm.offJ[j1], end = sm.offJ[j1 + 1];
    float acc = 0.0f;
#pragma unroll 4
    for (int m2 = beg; m2 < end; ++m2) {
        const float4 q = sm.J.s.rec[m2];
        const float dr = q.x - u.x;
        const float t = dr * dr;
        float e;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(-t));
        const float g = fmaf(u.w, q.w, fmaf(u.z, q.z, u.y * q.y));
        const float eg = e * strow[sm.J.s.cls[m2]];
        if (t < maxg2s) acc = fmaf(eg, g, acc);
    }
    const int seg = (meta >> 8) & 0xff;
    float v = acc;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const float o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane - d >= seg) v += o;
    }
    if ((meta >> 25) & 1) atomicAdd(&sm.S.f[(meta & 0xff) * FC_SS + j1], v);
}

// All work items of one molecule pair, S cleared first. Whole CTA.
__device__ __forceinline__ void fast_pair_sums(FastSmem &sm, int nJ, float maxg2s, bool paired) {
    if (paired) {
        for (int t = threadIdx.x; t < FC_MAXA * FC_SS; t += blockDim.x) sm.S.q[t] = 0;
    } else {
        for (int t = threadIdx.x; t < FC_MAXA * FC_SS; t += blockDim.x) sm.S.f[t] = 0.0f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    const int items = sm.npassI * nJ;
    if (paired) {
        // skip margin slightly wider than the window: only records whose every
        // term is masked are skipped
        const float wd = sqrtf(maxg2s) * 1.0001f;
        const int items2 = ((sm.npassI + 1) >> 1) * nJ;
        for (int it = warp; it < items2; it += FC_WARPS)
            fast_item_band2(sm, 2 * (it / nJ), it % nJ, maxg2s, wd);
    } else {
        for (int it = warp; it < items; it += FC_WARPS) fast_item(sm, it / nJ, it % nJ, maxg2s);
    }
    __syncthreads();
}

__device__ __forceinline__ float s_value(const FastSmem &sm, int idx, bool paired) {
    return paired ? (float)((double)sm.S.q[idx] * 2.3283064365386963e-10) : sm.S.f[idx];
}

// Molecule I for the paired path: its records sorted by r (prepared once per
// set by arad_sort_records_kernel), 32 per pass, with the r band of each
// pass. Whole CTA; the caller synchronises before the records are read.
__device__ void fast_load_I_band(FastSmem &sm, const SetWs &w, int I, int amax, int nI,
                                 bool use_self) {
    const int nrec = w.nrec[I];
    const int npass = (nrec + 31) / 32;
    const size_t base = (size_t)I * amax * amax;
    for (int slot = threadIdx.x; slot < npass * 32; slot += blockDim.x) {
        if (slot < nrec) {
            sm.recI[slot] = w.spk[base + slot];
            sm.metaI[slot] = w.smeta[base + slot];
        } else {
            sm.recI[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
            sm.metaI[slot] = 0;  // inactive
        }
    }
    for (int p = threadIdx.x; p < npass; p += blockDim.x) {
        sm.passLo[p] = w.spk[base + 32 * p].x;
        sm.passHi[p] = w.spk[base + min(32 * p + 31, nrec - 1)].x;
    }
    for (int a = threadIdx.x; a < nI; a += blockDim.x) {
        sm.selfI[a] = use_self ? w.selff[(size_t)I * amax + a] : 0.0f;
        sm.aclsI[a] = w.acls[(size_t)I * amax + a];
    }
    if (threadIdx.x == 0) {
        sm.npassI = npass;
        sm.nI = nI;
    }
}

// Class tables of the CTA: the stoichiometric table (row stride FC_SST) and,
// for the paired path, the pair table.
__device__ __forceinline__ void fast_load_tables(FastSmem &sm, const ClassInfo *ci, bool paired) {
    for (int t = threadIdx.x; t < FC_MAXC * FC_MAXC; t += blockDim.x)
        sm.stoch[(t / FC_MAXC) * FC_SST + t % FC_MAXC] = ci->stoch[t];
    if (paired)
        for (int t = threadIdx.x; t < FC_PC * FC_PC * FC_PC; t += blockDim.x) {
            const int c1 = t / (FC_PC * FC_PC), k = t % (FC_PC * FC_PC);
            const int ca = k / FC_PC, cb = k % FC_PC;
            sm.pt[c1 * FC_PTS + k] =
                make_float2(ci->stoch[c1 * FC_MAXC + ca], ci->stoch[c1 * FC_MAXC + cb]);
        }
}

__device__ __forceinline__ void pair_block(long long t, int symmetric, int nbj, int &bi, int &bj) {
    if (symmetric) {  // blocks bi <= bj
        int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while ((long long)r * (r + 1) / 2 > t) --r;
        while ((long long)(r + 1) * (r + 2) / 2 <= t) ++r;
        bj = r;
        bi = (int)(t - (long long)r * (r + 1) / 2);
    } else {
        bi = (int)(t / nbj);
        bj = (int)(t % nbj);
    }
}

// Records of one molecule sorted by r (ties by atom, then neighbour index):
// the I-side layout of the paired path. One CTA per molecule, bitonic sort
// of 64-bit keys (r bits << 32 | atom * 32 + k) in shared memory.
__global__ void __launch_bounds__(FC_WARPS * 32)
arad_sort_records_kernel(SetWs w, const int *__restrict__ N, int nm, int amax,
                         const ClassInfo *ci) {
    __shared__ unsigned long long key[FC_MAXREC];
    __shared__ int off[FC_MAXA + 1];
    if (ci->flag || ci->ncls > FC_PC) return;
    const int I = blockIdx.x;
    if (I >= nm) return;
    const int nI = min(max(N[I], 0), amax);
    if (threadIdx.x < 32) {
        const int a = threadIdx.x;
        const int cnt = a < nI ? w.nnb[(size_t)I * amax + a] : 0;
        int incl = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (a >= d) incl += o;
        }
        off[a] = incl - cnt;
        if (a == 31) off[32] = incl;
    }
    __syncthreads();
    const int nrec = off[32];
    int len = 1;
    while (len < nrec) len <<= 1;
    for (int t = threadIdx.x; t < len; t += blockDim.x) key[t] = ~0ull;
    __syncthreads();
    for (int t = threadIdx.x; t < nI * amax; t += blockDim.x) {
        const int a = t / amax, k = t % amax;
        if (k < off[a + 1] - off[a]) {
            const float r = w.pk[((size_t)I * amax + a) * amax + k].x;
            key[off[a] + k] = ((unsigned long long)__float_as_uint(r) << 32) |
                              (unsigned)(a * FC_MAXA + k);
        }
    }
    __syncthreads();
    for (int size = 2; size <= len; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < len; t += blockDim.x) {
                const int partner = t ^ stride;
                if (partner > t) {
                    const bool up = (t & size) == 0;
                    const unsigned long long x = key[t], y = key[partner];
                    if ((x > y) == up) {
                        key[t] = y;
                        key[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    const size_t base = (size_t)I * amax * amax;
    for (int t = threadIdx.x; t < nrec; t += blockDim.x) {
        const int idx = (int)(key[t] & 0xffffffffu), a = idx / FC_MAXA, k = idx % FC_MAXA;
        const size_t src = ((size_t)I * amax + a) * amax + k;
        w.spk[base + t] = w.pk[src];
        w.smeta[base + t] = a | ((int)w.cls[src] << 16) | (1 << 24);
    }
    if (threadIdx.x == 0) w.nrec[I] = nrec;
}

// Self terms S(a, a) through the same passes, scan and partial sums as the
// pair kernel, so that l2 = s + s - 2 S cancels exactly for an atom with itself.
__global__ void __launch_bounds__(FC_WARPS * 32)
arad_fast_self_kernel(SetWs w, const int *__restrict__ N, int nm, int amax, AradParams P,
                      const ClassInfo *ci) {
    extern __shared__ __align__(16) unsigned char fc_smem_raw[];
    FastSmem &sm = *reinterpret_cast<FastSmem *>(fc_smem_raw);
    if (ci->flag) return;
    const int I = blockIdx.x;
    if (I >= nm) return;
    const bool paired = ci->ncls <= FC_PC;
    fast_load_tables(sm, ci, paired);
    const int nI = min(max(N[I], 0), amax);
    if (paired) {
        fast_load_I_band(sm, w, I, amax, nI, false);
        fast_load_J_pairs(sm, w, I, amax, nI, false);
    } else {
        fast_load_I(sm, w, I, amax, nI, false);
        fast_load_J(sm, w, I, amax, nI, false);
    }
    __syncthreads();
    const float maxg2s = (float)(P.maxg2 * fp32_scale(P) * fp32_scale(P));
    fast_pair_sums(sm, nI, maxg2s, paired);
    for (int a = threadIdx.x; a < nI; a += blockDim.x)
        w.selff[(size_t)I * amax + a] = s_value(sm, a * FC_SS + a, paired);
}

__global__ void __launch_bounds__(FC_WARPS * 32)
arad_fast_pair_kernel(SetWs w1, const int *__restrict__ N1, int nm1, SetWs w2,
                      const int *__restrict__ N2, int nm2, int amax, AradParams P,
                      const ClassInfo *ci, SigmaTable sig, int nsig, int symmetric,
                      double *__restrict__ K) {
    extern __shared__ __align__(16) unsigned char fc_smem_raw[];
    FastSmem &sm = *reinterpret_cast<FastSmem *>(fc_smem_raw);
    if (ci->flag) return;
    const int nbj = (nm2 + FC_BM - 1) / FC_BM;
    int bi, bj;
    pair_block(blockIdx.x, symmetric, nbj, bi, bj);
    const bool paired = ci->ncls <= FC_PC;
    fast_load_tables(sm, ci, paired);
    const float maxg2s = (float)(P.maxg2 * fp32_scale(P) * fp32_scale(P));
    const float eps = 5.0e-12f;
    float sc[FC_MAXSIG];
#pragma unroll
    for (int s = 0; s < FC_MAXSIG; ++s)
        sc[s] = s < nsig ? (float)(sig.inv_sigma2[s] * 1.4426950408889634) : 0.0f;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int il = 0; il < FC_BM; ++il) {
        const int I = bi * FC_BM + il;
        if (I >= nm1) break;
        __syncthreads();
        const int nI = min(max(N1[I], 0), amax);
        if (paired)
            fast_load_I_band(sm, w1, I, amax, nI, true);
        else
            fast_load_I(sm, w1, I, amax, nI, true);
        for (int jl = 0; jl < FC_BM; ++jl) {
            const int J = bj * FC_BM + jl;
            if (J >= nm2) break;
            if (symmetric && J < I) continue;
            __syncthreads();
            const int nJ = min(max(N2[J], 0), amax);
            if (paired)
                fast_load_J_pairs(sm, w2, J, amax, nJ, true);
            else
                fast_load_J(sm, w2, J, amax, nJ, true);
            __syncthreads();
            fast_pair_sums(sm, nJ, maxg2s, paired);
            // phase 2: l2 and the kernel exponentials of every atom pair
            float kacc[FC_MAXSIG];
#pragma unroll
            for (int s = 0; s < FC_MAXSIG; ++s) kacc[s] = 0.0f;
            for (int t = threadIdx.x; t < nI * nJ; t += blockDim.x) {
                const int a = t / nJ, j1 = t - a * nJ;
                const float stz = sm.stoch[sm.aclsI[a] * FC_SST + sm.aclsJ[j1]];
                float l2 = sm.selfI[a] + sm.selfJ[j1] -
                           2.0f * s_value(sm, a * FC_SS + j1, paired) * stz;
                if (fabsf(l2) < eps) l2 = 0.0f;  // farad_kernels.f90:594
#pragma unroll
                for (int s = 0; s < FC_MAXSIG; ++s) {
                    if (s < nsig) {
                        float e;
                        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(l2 * sc[s]));
                        kacc[s] += e;
                    }
                }
            }
#pragma unroll
            for (int s = 0; s < FC_MAXSIG; ++s) {
                float v = kacc[s];
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) sm.red[warp][s] = v;
            }
            __syncthreads();
            if (threadIdx.x < nsig) {
                const int s = threadIdx.x;
                double v = 0.0;
                for (int q = 0; q < FC_WARPS; ++q) v += (double)sm.red[q][s];
                K[((size_t)s * nm1 + I) * nm2 + J] = v;
                if (symmetric) K[((size_t)s * nm1 + J) * nm2 + I] = v;
            }
        }
    }
}

// The fast kernels' shared memory is dynamic (above the 48 KB static limit);
// the attribute is set once per device.
int fast_smem_attrs() {
    static int attr_dev = -1;
    int dev = 0;
    FMLB_TRY(cuda_status(cudaGetDevice(&dev), "fmlb_arad_kernels: cudaGetDevice"));
    if (attr_dev == dev) return FMLB_OK;
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(arad_fast_self_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)sizeof(FastSmem)),
                         "fmlb_arad_kernels: self kernel smem attribute"));
    FMLB_TRY(cuda_status(cudaFuncSetAttribute(arad_fast_pair_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)sizeof(FastSmem)),
                         "fmlb_arad_kernels: pair kernel smem attribute"));
    attr_dev = dev;
    return FMLB_OK;
}

// ---- atom-level ARAD kernel (fget_atomic_kernels_arad, farad_kernels.f90:757-899)
// Every atom is its own environment: descriptor (5, amax), neighbour count n.
// Per atom: the prefix length of the neighbour list (the exit at r > cut of
// atomic_distl2, :68 / :72), the sine factors 1 - sin(r inv_cut) for every
// listed neighbour (:836-850, unconditional) and the self term (:855-868).
__global__ void arad_atom_prep_kernel(const double *__restrict__ Q, const int *__restrict__ N,
                                      int na, int amax, AradParams P, int *__restrict__ nnb,
                                      double *__restrict__ sines, double *__restrict__ self) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= na) return;
    const double *q = Q + (size_t)i * 5 * amax;
    const int n = min(max(N[i], 0), amax);
    double *si = sines + (size_t)i * amax;
    int pre = 0;
    while (pre < n && !(q[pre] > P.cut)) ++pre;
    for (int m = 0; m < amax; ++m) si[m] = m < n ? 1.0 - sin(__dmul_rn(q[m], P.inv_cut)) : 0.0;
    nnb[i] = pre;
    self[i] = distl2_f64(q, si, pre, q, si, pre, amax, P);
}

// K[s, i, j] = exp(l2(i, j) inv_sigma2[s]), l2 = self_i + self_j - 2 d(i, j) stoch
// (:873-891); thread per atom pair, j fastest (coalesced rows of K). With
// kDistance the l2 itself is stored, K[i, j] = l2(i, j) (the distances of
// fget_atomic_distance_arad, :902-1030).
template <bool kDistance>
__global__ void __launch_bounds__(128)
arad_atom_pair_kernel(const double *__restrict__ Q1, const double *__restrict__ Z1,
                      const int *__restrict__ nnb1, const double *__restrict__ S1,
                      const double *__restrict__ self1, int na1,
                      const double *__restrict__ Q2, const double *__restrict__ Z2,
                      const int *__restrict__ nnb2, const double *__restrict__ S2,
                      const double *__restrict__ self2, int na2, int amax, AradParams P,
                      SigmaTable sig, int nsig, double *__restrict__ K) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const double eps = (double)5.0e-12f;  // :823, a single-precision literal in the source
    for (int i = blockIdx.y; i < na1; i += gridDim.y) {
        if (j >= na2) continue;
        double l2 = distl2_f64(Q1 + (size_t)i * 5 * amax, S1 + (size_t)i * amax, nnb1[i],
                               Q2 + (size_t)j * 5 * amax, S2 + (size_t)j * amax, nnb2[j], amax,
                               P);
        const double dz1 = __dsub_rn(Z1[2 * i], Z2[2 * j]);
        const double dz2 = __dsub_rn(Z1[2 * i + 1], Z2[2 * j + 1]);
        const double st = __ddiv_rn(
            __dmul_rn(__ddiv_rn(P.rw2, __dadd_rn(P.rw2, __dmul_rn(dz1, dz1))), P.cw2),
            __dadd_rn(P.cw2, __dmul_rn(dz2, dz2)));
        l2 = __dsub_rn(__dadd_rn(self1[i], self2[j]), __dmul_rn(__dmul_rn(2.0, l2), st));
        if (fabs(l2) < eps) l2 = 0.0;
        if (kDistance) {
            K[(size_t)i * na2 + j] = l2;
        } else {
            for (int s = 0; s < nsig; ++s)
                K[((size_t)s * na1 + i) * na2 + j] = exp(__dmul_rn(l2, sig.inv_sigma2[s]));
        }
    }
}

size_t atom_ws_bytes(int na, int amax) {
    return align256((size_t)na * sizeof(int)) + align256((size_t)na * amax * sizeof(double)) +
           align256((size_t)na * sizeof(double));
}

}  // namespace
}  // namespace fmlb

extern "C" size_t fmlb_arad_atomic_workspace_bytes(int na1, int na2, int amax) {
    if (na1 < 0 || na2 < 0 || amax < 1) return 0;
    return fmlb::atom_ws_bytes(na1, amax) + fmlb::atom_ws_bytes(na2, amax);
}

static int arad_atomic_impl(const double *Q1, const double *Z1, const int *N1, int na1,
                            const double *Q2, const double *Z2, const int *N2, int na2, int amax,
                            const double *sigmas_host, int nsigma, double width,
                            double cut_distance, double r_width, double c_width, double *K,
                            void *workspace, size_t ws_bytes, bool distance, cudaStream_t st) {
    using namespace fmlb;
    const char *what = distance ? "fmlb_arad_atomic_distances" : "fmlb_arad_atomic_kernels";
    FMLB_REQUIRE(na1 >= 0 && na2 >= 0 && amax >= 1, "%s: bad sizes", what);
    if (!distance)
        FMLB_REQUIRE(nsigma >= 1 && nsigma <= MAXSIG && sigmas_host,
                     "%s: nsigma must be 1..%d", what, MAXSIG);
    const size_t need = fmlb_arad_atomic_workspace_bytes(na1, na2, amax);
    if (ws_bytes < need || (need && !workspace)) {
        set_error("%s: workspace %zu bytes < required %zu", what, ws_bytes, need);
        return FMLB_ENOMEM;
    }
    if (na1 == 0 || na2 == 0) return FMLB_OK;
    FMLB_REQUIRE(Q1 && Z1 && N1 && Q2 && Z2 && N2 && K, "%s: null pointer", what);
    AradParams P;
    P.width = width;
    P.cut = cut_distance;
    P.rw2 = r_width * r_width;
    P.cw2 = c_width * c_width;
    P.inv_width = -1.0 / (4.0 * width * width);      // :58
    P.maxg2 = (8.0 * width) * (8.0 * width);          // :60
    P.inv_cut = (4.0 * atan(1.0)) / (2.0 * cut_distance);  // :828
    P.eps = (double)5.0e-12f;                                // :823
    SigmaTable sig;
    for (int s = 0; s < (distance ? 0 : nsigma); ++s)
        sig.inv_sigma2[s] = -1.0 / (sigmas_host[s] * sigmas_host[s]);
    char *p = static_cast<char *>(workspace);
    int *nnb1 = reinterpret_cast<int *>(p); p += align256((size_t)na1 * sizeof(int));
    double *S1 = reinterpret_cast<double *>(p); p += align256((size_t)na1 * amax * sizeof(double));
    double *self1 = reinterpret_cast<double *>(p); p += align256((size_t)na1 * sizeof(double));
    int *nnb2 = reinterpret_cast<int *>(p); p += align256((size_t)na2 * sizeof(int));
    double *S2 = reinterpret_cast<double *>(p); p += align256((size_t)na2 * amax * sizeof(double));
    double *self2 = reinterpret_cast<double *>(p);
    arad_atom_prep_kernel<<<ceil_div(na1, 128), 128, 0, st>>>(Q1, N1, na1, amax, P, nnb1, S1,
                                                               self1);
    FMLB_TRY(launch_status("arad_atom_prep_kernel"));
    arad_atom_prep_kernel<<<ceil_div(na2, 128), 128, 0, st>>>(Q2, N2, na2, amax, P, nnb2, S2,
                                                               self2);
    FMLB_TRY(launch_status("arad_atom_prep_kernel"));
    const dim3 grid(ceil_div(na2, 128), std::min(na1, 65535));
    if (distance)
        arad_atom_pair_kernel<true><<<grid, 128, 0, st>>>(Q1, Z1, nnb1, S1, self1, na1, Q2, Z2,
                                                          nnb2, S2, self2, na2, amax, P, sig, 0,
                                                          K);
    else
        arad_atom_pair_kernel<false><<<grid, 128, 0, st>>>(Q1, Z1, nnb1, S1, self1, na1, Q2, Z2,
                                                           nnb2, S2, self2, na2, amax, P, sig,
                                                           nsigma, K);
    return launch_status("arad_atom_pair_kernel");
}

extern "C" int fmlb_arad_atomic_kernels(const double *Q1, const double *Z1, const int *N1, int na1,
                                        const double *Q2, const double *Z2, const int *N2, int na2,
                                        int amax, const double *sigmas_host, int nsigma,
                                        double width, double cut_distance, double r_width,
                                        double c_width, double *K, void *workspace,
                                        size_t ws_bytes, void *stream) {
    return arad_atomic_impl(Q1, Z1, N1, na1, Q2, Z2, N2, na2, amax, sigmas_host, nsigma, width,
                            cut_distance, r_width, c_width, K, workspace, ws_bytes, false,
                            FMLB_STREAM(stream));
}

extern "C" int fmlb_arad_atomic_distances(const double *Q1, const double *Z1, const int *N1,
                                          int na1, const double *Q2, const double *Z2,
                                          const int *N2, int na2, int amax, double width,
                                          double cut_distance, double r_width, double c_width,
                                          double *D, void *workspace, size_t ws_bytes,
                                          void *stream) {
    return arad_atomic_impl(Q1, Z1, N1, na1, Q2, Z2, N2, na2, amax, nullptr, 0, width,
                            cut_distance, r_width, c_width, D, workspace, ws_bytes, true,
                            FMLB_STREAM(stream));
}

extern "C" size_t fmlb_arad_workspace_bytes(int nm1, int nm2, int amax, int symmetric) {
    if (nm1 < 0 || nm2 < 0 || amax < 1) return 0;
    return fmlb::set_ws_bytes(nm1, amax) + (symmetric ? 0 : fmlb::set_ws_bytes(nm2, amax)) +
           fmlb::align256(sizeof(fmlb::ClassInfo));
}

static int arad_kernels_impl(const double *X1, const double *Z1, const int *N1, int nm1,
                             const double *X2, const double *Z2, const int *N2, int nm2,
                             int amax, const double *sigmas_host, int nsigma, double width,
                             double cut_distance, double r_width, double c_width, int symmetric,
                             int precision, double eps, double *K, void *workspace,
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
    P.eps = eps;

    char *p = static_cast<char *>(workspace);
    SetWs w1 = carve(p, nm1, amax);
    SetWs w2 = symmetric ? w1 : carve(p, nm2, amax);
    ClassInfo *ci = reinterpret_cast<ClassInfo *>(p);
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
    // fast FP32 path: amax <= 32 and at most 16 element classes (decided on the device)
    const bool try_fast = precision == 1 && amax <= FC_MAXA;
    if (try_fast) {
        FMLB_TRY(cuda_status(cudaMemsetAsync(ci, 0, sizeof(ClassInfo), st), "clear class info"));
        arad_class_scan_kernel<<<ceil_div((long long)nm1 * amax, tpb), tpb, 0, st>>>(
            X1, Z1, N1, nm1, amax, P.cut, ci);
        if (!symmetric)
            arad_class_scan_kernel<<<ceil_div((long long)nm2 * amax, tpb), tpb, 0, st>>>(
                X2, Z2, N2, nm2, amax, P.cut, ci);
        arad_class_build_kernel<<<1, 1, 0, st>>>(ci, P.rw2, P.cw2);
        arad_class_assign_kernel<<<ceil_div((long long)nm1 * amax, tpb), tpb, 0, st>>>(
            X1, Z1, N1, nm1, amax, ci, w1);
        if (!symmetric)
            arad_class_assign_kernel<<<ceil_div((long long)nm2 * amax, tpb), tpb, 0, st>>>(
                X2, Z2, N2, nm2, amax, ci, w2);
        FMLB_TRY(fast_smem_attrs());
        arad_sort_records_kernel<<<nm1, FC_WARPS * 32, 0, st>>>(w1, N1, nm1, amax, ci);
        if (!symmetric)
            arad_sort_records_kernel<<<nm2, FC_WARPS * 32, 0, st>>>(w2, N2, nm2, amax, ci);
        arad_fast_self_kernel<<<nm1, FC_WARPS * 32, sizeof(FastSmem), st>>>(w1, N1, nm1, amax, P,
                                                                            ci);
        if (!symmetric)
            arad_fast_self_kernel<<<nm2, FC_WARPS * 32, sizeof(FastSmem), st>>>(w2, N2, nm2, amax,
                                                                                P, ci);
        FMLB_TRY(launch_status("arad fast-path preparation"));
    }
    const long long npairs = symmetric ? (long long)nm1 * (nm1 + 1) / 2 : (long long)nm1 * nm2;
    const int blocks = (int)std::min<long long>(ceil_div(npairs, tpb / 32), (long long)sm_count() * 64);
    const int chunk = try_fast ? FC_MAXSIG : MAXSIG;
    for (int s0 = 0; s0 < nsigma; s0 += chunk) {
        const int ns = nsigma - s0 < chunk ? nsigma - s0 : chunk;
        SigmaTable sig;
        for (int s = 0; s < ns; ++s)
            sig.inv_sigma2[s] = -1.0 / (sigmas_host[s0 + s] * sigmas_host[s0 + s]);
        double *Ks = K + (size_t)s0 * nm1 * nm2;
        if (precision == 0) {
            arad_pair_kernel<true><<<blocks, tpb, 0, st>>>(X1, Z1, N1, w1, nm1, X2, Z2, N2, w2, nm2,
                                                           amax, P, sig, ns, symmetric, Ks, nullptr);
        } else {
            if (try_fast) {
                const long long nbi = ceil_div(nm1, FC_BM), nbj = ceil_div(nm2, FC_BM);
                const long long nblk = symmetric ? nbi * (nbi + 1) / 2 : nbi * nbj;
                FMLB_REQUIRE(nblk < (1LL << 31), "fmlb_arad_kernels: too many molecule blocks");
                arad_fast_pair_kernel<<<(unsigned)nblk, FC_WARPS * 32, sizeof(FastSmem), st>>>(
                    w1, N1, nm1, w2, N2, nm2, amax, P, ci, sig, ns, symmetric, Ks);
                FMLB_TRY(launch_status("arad_fast_pair_kernel"));
            }
            arad_pair_kernel<false><<<blocks, tpb, 0, st>>>(X1, Z1, N1, w1, nm1, X2, Z2, N2, w2,
                                                            nm2, amax, P, sig, ns, symmetric, Ks,
                                                            try_fast ? ci : nullptr);
        }
        FMLB_TRY(launch_status("arad_pair_kernel"));
    }
    return FMLB_OK;
}

extern "C" int fmlb_arad_kernels(const double *X1, const double *Z1, const int *N1, int nm1,
                                 const double *X2, const double *Z2, const int *N2, int nm2,
                                 int amax, const double *sigmas_host, int nsigma, double width,
                                 double cut_distance, double r_width, double c_width,
                                 int symmetric, int precision, double *K, void *workspace,
                                 size_t ws_bytes, void *stream) {
    // eps: the single-precision literal 5.0e-12 of farad_kernels.f90:505 / :679
    return arad_kernels_impl(X1, Z1, N1, nm1, X2, Z2, N2, nm2, amax, sigmas_host, nsigma, width,
                             cut_distance, r_width, c_width, symmetric, precision,
                             (double)5.0e-12f, K, workspace, ws_bytes, stream);
}

// The kernel matrix of fget_alpha_arad (farad_kernels.f90:231-393): the
// symmetric FP64 ARAD kernel for one sigma with the routine's fixed
// parameters (width 0.2, cut 6, r_width 1, c_width 0.5, :237-240) and its eps
// (the single-precision literal 1.0e-11, :309), plus lambda on the diagonal
// (:385-389).
extern "C" int fmlb_arad_alpha_kernel_f64(const double *X, const double *Z, const int *N,
                                          int nm, int amax, double sigma, double lambda,
                                          double *K, void *workspace, size_t ws_bytes,
                                          void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(sigma > 0.0, "fmlb_arad_alpha_kernel_f64: sigma must be positive");
    FMLB_TRY(arad_kernels_impl(X, Z, N, nm, X, Z, N, nm, amax, &sigma, 1, 0.2, 6.0, 1.0, 0.5, 1,
                               0, (double)1.0e-11f, K, workspace, ws_bytes, stream));
    return fmlb_add_diagonal_f64(K, nm, nm, lambda, stream);
}

// atomic_arad_l2_distance_all (farad.f90:452-600), called by
// get_l2_distance_arad (fml/math/distance.py:120-189): D (nm1, nm2, amax, amax)
// with l2 of every atom pair, zero past each molecule's atoms. Sine factors
// for every listed neighbour in both sets (:519-539), eps the single-precision
// literal 5.0e-12 (:509).
extern "C" int fmlb_arad_distances(const double *X1, const double *Z1, const int *N1, int nm1,
                                   const double *X2, const double *Z2, const int *N2, int nm2,
                                   int amax, double width, double cut_distance, double r_width,
                                   double c_width, double *D, void *workspace, size_t ws_bytes,
                                   void *stream) {
    using namespace fmlb;
    cudaStream_t st = FMLB_STREAM(stream);
    FMLB_REQUIRE(nm1 >= 0 && nm2 >= 0 && amax >= 1, "fmlb_arad_distances: bad sizes");
    const size_t need = fmlb_arad_workspace_bytes(nm1, nm2, amax, 0);
    if (ws_bytes < need || (need && !workspace)) {
        set_error("fmlb_arad_distances: workspace %zu bytes < required %zu", ws_bytes, need);
        return FMLB_ENOMEM;
    }
    if (nm1 == 0 || nm2 == 0) return FMLB_OK;
    FMLB_REQUIRE(X1 && Z1 && N1 && X2 && Z2 && N2 && D, "fmlb_arad_distances: null pointer");
    AradParams P;
    P.width = width;
    P.cut = cut_distance;
    P.rw2 = r_width * r_width;
    P.cw2 = c_width * c_width;
    P.inv_width = -1.0 / (4.0 * width * width);
    P.maxg2 = (8.0 * width) * (8.0 * width);
    P.inv_cut = (4.0 * atan(1.0)) / (2.0 * cut_distance);  // farad.f90:515
    P.eps = (double)5.0e-12f;
    char *p = static_cast<char *>(workspace);
    SetWs w1 = carve(p, nm1, amax);
    SetWs w2 = carve(p, nm2, amax);
    const int tpb = 128;
    arad_prep_kernel<<<ceil_div((long long)nm1 * amax, tpb), tpb, 0, st>>>(X1, N1, nm1, amax, P,
                                                                           0, w1);
    FMLB_TRY(launch_status("arad_prep_kernel"));
    arad_prep_kernel<<<ceil_div((long long)nm2 * amax, tpb), tpb, 0, st>>>(X2, N2, nm2, amax, P,
                                                                           0, w2);
    FMLB_TRY(launch_status("arad_prep_kernel"));
    FMLB_TRY(cuda_status(cudaMemsetAsync(D, 0, sizeof(double) * nm1 * nm2 * amax * amax, st),
                         "fmlb_arad_distances: clear D"));
    const long long npairs = (long long)nm1 * nm2;
    const int blocks =
        (int)std::min<long long>(ceil_div(npairs, tpb / 32), (long long)sm_count() * 64);
    SigmaTable sig{};
    arad_pair_kernel<true, true><<<blocks, tpb, 0, st>>>(X1, Z1, N1, w1, nm1, X2, Z2, N2, w2, nm2,
                                                         amax, P, sig, 0, 0, nullptr, nullptr,
                                                         D);
    return launch_status("arad_pair_kernel<distance>");
}
