// Descriptor generation: sorted Coulomb matrices and ARAD descriptors for a
// packed ragged batch of molecules, one launch per batch.
//
// Both kernels keep the reference's FP64 arithmetic order (explicit _rn
// intrinsics, so no FMA is contracted) so the row-norm sort permutation of the
// Coulomb matrix is bit-exact with the reference.
#include <math.h>
#include <string.h>

#include "common.cuh"

namespace fmlb {
namespace {

constexpr int kWarpsPerBlock = 4;

// 0.5 * Z**2.4 for integral Z, evaluated on the host with the C library's
// pow(), i.e. the same libm call the reference's `**` compiles to
// (frepresentations.f90:66). Passed by value as a kernel parameter.
struct DiagTable {
    double v[128];
};

// Periodic-table position (row, column) per Z; -1 where undefined.
struct PtpTable {
    signed char row[128];
    signed char col[128];
};

__device__ __forceinline__ double cm_diag(double z, const DiagTable &t) {
    double r = rint(z);
    if (r == z && r >= 0.0 && r < 128.0) return t.v[(int)r];
    return __dmul_rn(0.5, pow(z, 2.4));
}

// Z_a Z_b / |R_b - R_a| for a < b, in the order of frepresentations.f90:75-76.
__device__ __forceinline__ double cm_pair(const double *X, const double *Y, const double *Zc,
                                          const double *Q, int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    double dx = __dsub_rn(X[b], X[a]);
    double dy = __dsub_rn(Y[b], Y[a]);
    double dz = __dsub_rn(Zc[b], Zc[a]);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return __ddiv_rn(__dmul_rn(Q[a], Q[b]), __dsqrt_rn(s));
}

// |R_b - R_a| for a < b (the distance matrix of frepresentations.f90:336-342)
__device__ __forceinline__ double cm_dist(const double *X, const double *Y, const double *Zc,
                                          int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    double dx = __dsub_rn(X[b], X[a]);
    double dy = __dsub_rn(Y[b], Y[a]);
    double dz = __dsub_rn(Zc[b], Zc[a]);
    return __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// One warp per molecule.
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
cm_sorted_kernel(const double *__restrict__ charges, const double *__restrict__ coords,
                 const int *__restrict__ offsets, int nmol, int nmax, double *__restrict__ cm,
                 int ldcm, float *__restrict__ cm32, int ldcm32, int *__restrict__ order,
                 DiagTable diag, int *__restrict__ status) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mol = blockIdx.x * kWarpsPerBlock + warp;
    if (mol >= nmol) return;
    const int per_warp = 5 * nmax + (nmax + 1) / 2 + 1;
    double *X = smem + warp * per_warp;
    double *Y = X + nmax, *Zc = Y + nmax, *Q = Zc + nmax, *N = Q + nmax;
    int *S = reinterpret_cast<int *>(N + nmax);

    const int a0 = offsets[mol];
    int n = offsets[mol + 1] - a0;
    const int L = nmax * (nmax + 1) / 2;
    if (n < 0 || n > nmax) {
        if (lane == 0 && status) atomicCAS(status, 0, 1);
        n = 0;  // emit a zero row, stay in bounds
    }
    for (int t = lane; t < n; t += 32) {
        X[t] = coords[3 * (size_t)(a0 + t) + 0];
        Y[t] = coords[3 * (size_t)(a0 + t) + 1];
        Zc[t] = coords[3 * (size_t)(a0 + t) + 2];
        Q[t] = charges[a0 + t];
    }
    __syncwarp();
    // row norms: diagonal first, then the other atoms in index order
    // (single-thread order of the loops at frepresentations.f90:65-84)
    for (int i = lane; i < n; i += 32) {
        double s = cm_diag(Q[i], diag);
        for (int j = 0; j < n; ++j)
            if (j != i) s = __dadd_rn(s, cm_pair(X, Y, Zc, Q, i, j));
        N[i] = s;
    }
    __syncwarp();
    // rank: descending norm, ties -> higher index first (minloc fill, :86-91)
    // (NaN norms are ranked as -inf so the ranks always form a permutation)
    for (int i = lane; i < n; i += 32) {
        const double ni = isnan(N[i]) ? -INFINITY : N[i];
        int r = 0;
        for (int j = 0; j < n; ++j) {
            const double nj = isnan(N[j]) ? -INFINITY : N[j];
            r += (nj > ni) || (nj == ni && j > i);
        }
        S[r] = i;
    }
    __syncwarp();
    // packed lower triangle of the sorted matrix (:93-104)
    double *crow = cm ? cm + (size_t)mol * ldcm : nullptr;
    float *frow = cm32 ? cm32 + (size_t)mol * ldcm32 : nullptr;
    for (int idx = lane; idx < L; idx += 32) {
        int m = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
        while (m * (m + 1) / 2 > idx) --m;
        while ((m + 1) * (m + 2) / 2 <= idx) ++m;
        const int q = idx - m * (m + 1) / 2;
        double v = 0.0;
        if (m < n) v = (q == m) ? cm_diag(Q[S[m]], diag) : cm_pair(X, Y, Zc, Q, S[m], S[q]);
        if (crow) crow[idx] = v;
        if (frow) frow[idx] = (float)v;
    }
    if (frow)
        for (int idx = L + lane; idx < ldcm32; idx += 32) frow[idx] = 0.0f;
    if (order)
        for (int p = lane; p < nmax; p += 32) order[(size_t)mol * nmax + p] = p < n ? S[p] : -1;
}

// ---------------------------------------------------------------------------
// Unsorted Coulomb matrix, fgenerate_unsorted_coulomb_matrix
// (frepresentations.f90:112-202): the packed lower triangle in the input atom
// order. One warp per molecule.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
cm_unsorted_kernel(const double *__restrict__ charges, const double *__restrict__ coords,
                   const int *__restrict__ offsets, int nmol, int nmax, double *__restrict__ cm,
                   int ldcm, DiagTable diag, int *__restrict__ status) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mol = blockIdx.x * kWarpsPerBlock + warp;
    if (mol >= nmol) return;
    double *X = smem + (size_t)warp * 4 * nmax;
    double *Y = X + nmax, *Zc = Y + nmax, *Q = Zc + nmax;
    const int a0 = offsets[mol];
    int n = offsets[mol + 1] - a0;
    const int L = nmax * (nmax + 1) / 2;
    if (n < 0 || n > nmax) {  // rejected on the host; emit a zero row, stay in bounds
        if (lane == 0 && status) atomicCAS(status, 0, 1);
        n = 0;
    }
    for (int t = lane; t < n; t += 32) {
        X[t] = coords[3 * (size_t)(a0 + t) + 0];
        Y[t] = coords[3 * (size_t)(a0 + t) + 1];
        Zc[t] = coords[3 * (size_t)(a0 + t) + 2];
        Q[t] = charges[a0 + t];
    }
    __syncwarp();
    double *row = cm + (size_t)mol * ldcm;
    for (int idx = lane; idx < L; idx += 32) {  // :184-192
        int m = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
        while (m * (m + 1) / 2 > idx) --m;
        while ((m + 1) * (m + 2) / 2 <= idx) ++m;
        const int q = idx - m * (m + 1) / 2;
        double v = 0.0;
        if (m < n) v = (q == m) ? cm_diag(Q[m], diag) : cm_pair(X, Y, Zc, Q, m, q);
        row[idx] = v;
    }
    for (int idx = L + lane; idx < ldcm; idx += 32) row[idx] = 0.0;
}

// ---------------------------------------------------------------------------
// Local and atomic Coulomb matrices, one row per atom: the packed lower
// triangle of the molecule's Coulomb matrix with the atoms reordered around
// the central atom k.
//   kind 0, fgenerate_local_coulomb_matrix (frepresentations.f90:204-294):
//     k first, then the others in the row-norm order of the sorted matrix
//     (descending norm, ties -> higher index first, :262-277);
//   kind 1, fgenerate_atomic_coulomb_matrix (:297-390): every atom by its
//     distance to k, ascending, ties -> lower index first (minloc, :366-371).
// One warp per molecule; FP64 in the reference's operation order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
cm_local_kernel(const double *__restrict__ charges, const double *__restrict__ coords,
                const int *__restrict__ offsets, int nmol, int nmax, int kind,
                double *__restrict__ cm, int ldcm, DiagTable diag, int *__restrict__ status) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mol = blockIdx.x * kWarpsPerBlock + warp;
    if (mol >= nmol) return;
    const int per_warp = 5 * nmax + nmax;  // X Y Z Q N (doubles) + S, O (ints)
    double *X = smem + warp * per_warp;
    double *Y = X + nmax, *Zc = Y + nmax, *Q = Zc + nmax, *N = Q + nmax;
    int *S = reinterpret_cast<int *>(N + nmax), *O = S + nmax;
    const int a0 = offsets[mol];
    const int n = offsets[mol + 1] - a0;
    const int L = nmax * (nmax + 1) / 2;
    if (n < 0 || n > nmax) {  // rejected on the host; stay in bounds regardless
        if (lane == 0 && status) atomicCAS(status, 0, 1);
        return;
    }
    for (int t = lane; t < n; t += 32) {
        X[t] = coords[3 * (size_t)(a0 + t) + 0];
        Y[t] = coords[3 * (size_t)(a0 + t) + 1];
        Zc[t] = coords[3 * (size_t)(a0 + t) + 2];
        Q[t] = charges[a0 + t];
    }
    __syncwarp();
    if (kind == 0) {
        // row norms (:238-259: diagonal, then every other atom in index order)
        for (int i = lane; i < n; i += 32) {
            double s = cm_diag(Q[i], diag);
            for (int j = 0; j < n; ++j)
                if (j != i) s = __dadd_rn(s, cm_pair(X, Y, Zc, Q, i, j));
            N[i] = s;
        }
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const double ni = isnan(N[i]) ? -INFINITY : N[i];
            int r = 0;
            for (int j = 0; j < n; ++j) {
                const double nj = isnan(N[j]) ? -INFINITY : N[j];
                r += (nj > ni) || (nj == ni && j > i);
            }
            S[r] = i;
        }
        __syncwarp();
    }
    for (int k = 0; k < n; ++k) {
        if (kind == 0) {  // k, then the sorted atoms without k (:268-277)
            for (int t = lane; t < n; t += 32) {
                if (t == 0) {
                    O[0] = k;
                } else {
                    int pos = 0;  // position of k in the sorted order
                    while (S[pos] != k) ++pos;
                    O[t] = S[t - 1 + (t - 1 >= pos ? 1 : 0)];
                }
            }
        } else {  // ascending distance to k, ties -> lower index (:366-371)
            for (int i = lane; i < n; i += 32) {
                const double di = i == k ? 0.0 : cm_dist(X, Y, Zc, i, k);
                int r = 0;
                for (int j = 0; j < n; ++j) {
                    const double dj = j == k ? 0.0 : cm_dist(X, Y, Zc, j, k);
                    r += (dj < di) || (dj == di && j < i);
                }
                O[r] = i;
            }
        }
        __syncwarp();
        double *row = cm + (size_t)(a0 + k) * ldcm;
        for (int idx = lane; idx < L; idx += 32) {
            int m = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
            while (m * (m + 1) / 2 > idx) --m;
            while ((m + 1) * (m + 2) / 2 <= idx) ++m;
            const int q = idx - m * (m + 1) / 2;
            double v = 0.0;
            if (m < n) v = (q == m) ? cm_diag(Q[O[m]], diag) : cm_pair(X, Y, Zc, Q, O[m], O[q]);
            row[idx] = v;
        }
        for (int idx = L + lane; idx < ldcm; idx += 32) row[idx] = 0.0;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// ARAD descriptor, fml/arad.py:70-145. One CTA per molecule, one warp per
// central atom.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pairwise_sum_small(const double *v, const int *sel, int n) {
    // numpy's pairwise summation for n <= 128 (8 partial sums, then a tree),
    // which np.sum applies to the contiguous array at fml/arad.py:137.
    if (n < 8) {
        double r = -0.0;
        for (int i = 0; i < n; ++i) r = __dadd_rn(r, v[sel[i]]);
        return r;
    }
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = v[sel[j]];
    int i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], v[sel[i + j]]);
    double res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                           __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
    for (; i < n; ++i) res = __dadd_rn(res, v[sel[i]]);
    return res;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
arad_describe_kernel(const double *__restrict__ charges, const double *__restrict__ coords,
                     const int *__restrict__ offsets, int nmol, int size, double cut,
                     double *__restrict__ out, PtpTable ptp, int *__restrict__ status) {
    extern __shared__ double smem[];
    const int mol = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *X = smem, *Y = X + size, *Zc = Y + size, *PR = Zc + size, *PC = PR + size;
    const int per_warp = 5 * size + (size + 1) / 2 + 1;
    double *W = PC + size + warp * per_warp;
    double *CX = W, *CY = CX + size, *CZ = CY + size, *D = CZ + size, *DMP = D + size;
    int *SEL = reinterpret_cast<int *>(DMP + size);

    const int a0 = offsets[mol];
    int n = offsets[mol + 1] - a0;
    if (n < 0 || n > size) {
        if (threadIdx.x == 0 && status) atomicCAS(status, 0, 1);
        n = 0;
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        X[t] = coords[3 * (size_t)(a0 + t) + 0];
        Y[t] = coords[3 * (size_t)(a0 + t) + 1];
        Zc[t] = coords[3 * (size_t)(a0 + t) + 2];
        const double z = charges[a0 + t];
        const double zr = rint(z);
        int r = -1, c = -1;
        if (zr == z && zr >= 0.0 && zr < 128.0) {
            r = ptp.row[(int)zr];
            c = ptp.col[(int)zr];
        }
        if (r < 0 && status) atomicCAS(status, 0, 2);
        PR[t] = (double)r;
        PC[t] = (double)c;
    }
    __syncthreads();

    const double eps = 100.0 * 2.220446049250313e-16;  // fml/arad.py:42
    const double pi = 3.141592653589793;                // numpy.pi
    const double two_cut = __dmul_rn(2.0, cut);
    double *mol_out = out + (size_t)mol * size * 5 * size;

    for (int i = warp; i < size; i += kWarpsPerBlock) {
        double *row = mol_out + (size_t)i * 5 * size;
        if (i >= n) {  // rows past the molecule: M[:, 0, :] = 1e100 (:93)
            for (int p = lane; p < size; p += 32) {
                row[p] = 1e100;
                row[size + p] = row[2 * size + p] = row[3 * size + p] = row[4 * size + p] = 0.0;
            }
            continue;
        }
        // displacements, distances and damping (:97-108)
        for (int k = lane; k < n; k += 32) {
            const double cx = __dsub_rn(X[k], X[i]);
            const double cy = __dsub_rn(Y[k], Y[i]);
            const double cz = __dsub_rn(Zc[k], Zc[i]);
            CX[k] = cx;
            CY[k] = cy;
            CZ[k] = cz;
            const double d = __dsqrt_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz)));
            D[k] = d;
            DMP[k] = __dsub_rn(1.0, sin(__ddiv_rn(__dmul_rn(pi, d), two_cut)));
        }
        __syncwarp();
        // stable argsort by distance (:110); NaN sorts last like numpy
        for (int k = lane; k < n; k += 32) {
            const double dk = isnan(D[k]) ? INFINITY : D[k];
            int r = 0;
            for (int q = 0; q < n; ++q) {
                const double dq = isnan(D[q]) ? INFINITY : D[q];
                r += (dq < dk) || (dq == dk && q < k);
            }
            SEL[r] = k;
        }
        __syncwarp();
        // neighbours kept: sorted prefix with D < cut (:121)
        int m = 0;
        for (int k = lane; k < n; k += 32) m += (D[k] < cut);
        for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
        const double norm = pairwise_sum_small(DMP, SEL, m);  // :137
        for (int p = lane; p < size; p += 32) {
            if (p >= m) {
                row[p] = 1e100;
                row[size + p] = row[2 * size + p] = row[3 * size + p] = row[4 * size + p] = 0.0;
                continue;
            }
            const int j = SEL[p];
            const double dj = D[j];
            double cs = 0.0, ss = 0.0;
            for (int q = 0; q < m; ++q) {
                const int k = SEL[q];
                const double sp = __dadd_rn(
                    __dadd_rn(__dmul_rn(CX[j], CX[k]), __dmul_rn(CY[j], CY[k])),
                    __dmul_rn(CZ[j], CZ[k]));
                const double nn = __dmul_rn(dj, D[k]);
                double c = 1.0, s = 0.0;  // masked angle 0 (:29-33)
                if (fabs(__dsub_rn(sp, nn)) > eps && fabs(nn) > eps) {
                    // cos(arccos(x)) = x and sin(arccos(x)) = sqrt((1-x)(1+x));
                    // |x| > 1 gives NaN as arccos does
                    const double x = __ddiv_rn(sp, nn);
                    if (fabs(x) <= 1.0) {
                        c = x;
                        s = __dsqrt_rn(__dmul_rn(__dsub_rn(1.0, x), __dadd_rn(1.0, x)));
                    } else {
                        c = s = __longlong_as_double(0x7ff8000000000000LL);
                    }
                }
                const double w = DMP[k];
                if (q == 0) {
                    cs = __dmul_rn(c, w);
                    ss = __dmul_rn(s, w);
                } else {
                    cs = __dadd_rn(cs, __dmul_rn(c, w));
                    ss = __dadd_rn(ss, __dmul_rn(s, w));
                }
            }
            row[p] = dj;                          // :138
            row[size + p] = PR[j];                // :139
            row[2 * size + p] = PC[j];            // :140
            row[3 * size + p] = __ddiv_rn(cs, norm);  // :141
            row[4 * size + p] = __ddiv_rn(ss, norm);  // :142
        }
        __syncwarp();
    }
}

DiagTable make_diag_table() {
    DiagTable t;
    for (int z = 0; z < 128; ++z) t.v[z] = 0.5 * pow((double)z, 2.4);
    return t;
}

}  // namespace
}  // namespace fmlb

// PTP table (period row, group column), the reference's fml/arad.py:43-68.
// Z = 101 -> (7, 32) (last of its two dict entries) and Z = 102 -> (7, 14),
// as the reference table has them.
static void fill_ptp(fmlb::PtpTable &t) {
    memset(t.row, -1, sizeof t.row);
    memset(t.col, -1, sizeof t.col);
    auto set = [&](int z, int r, int c) { t.row[z] = (signed char)r; t.col[z] = (signed char)c; };
    set(1, 1, 1);
    set(2, 1, 8);
    const int light[2] = {3, 11};
    for (int p = 0; p < 2; ++p) {
        set(light[p], 2 + p, 1);
        set(light[p] + 1, 2 + p, 2);
        for (int k = 0; k < 6; ++k) set(light[p] + 2 + k, 2 + p, 3 + k);
    }
    const int mid[2][3] = {{19, 21, 31}, {37, 39, 49}};
    for (int p = 0; p < 2; ++p) {
        set(mid[p][0], 4 + p, 1);
        set(mid[p][0] + 1, 4 + p, 2);
        for (int k = 0; k < 10; ++k) set(mid[p][1] + k, 4 + p, 9 + k);
        for (int k = 0; k < 6; ++k) set(mid[p][2] + k, 4 + p, 3 + k);
    }
    const int heavy[2][4] = {{55, 57, 72, 81}, {87, 89, 104, 113}};
    for (int p = 0; p < 2; ++p) {
        set(heavy[p][0], 6 + p, 1);
        set(heavy[p][0] + 1, 6 + p, 2);
        for (int k = 0; k < 15; ++k) set(heavy[p][1] + k, 6 + p, 19 + k);
        for (int k = 0; k < 9; ++k) set(heavy[p][2] + k, 6 + p, 10 + k);
        for (int k = 0; k < 6; ++k) set(heavy[p][3] + k, 6 + p, 3 + k);
    }
    set(101, 7, 32);
    set(102, 7, 14);
}

extern "C" int fmlb_coulomb_matrices(const double *charges, const double *coords,
                                     const int *offsets, int nmol, int nmax, double *cm, int ldcm,
                                     float *cm32, int ldcm32, int *order, int *status,
                                     void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(nmol >= 0, "fmlb_coulomb_matrices: nmol < 0");
    FMLB_REQUIRE(nmax >= 1 && nmax <= 255, "fmlb_coulomb_matrices: nmax=%d outside 1..255", nmax);
    const int L = nmax * (nmax + 1) / 2;
    FMLB_REQUIRE(!cm || ldcm >= L, "fmlb_coulomb_matrices: ldcm=%d < %d", ldcm, L);
    FMLB_REQUIRE(!cm32 || ldcm32 >= L, "fmlb_coulomb_matrices: ldcm32=%d < %d", ldcm32, L);
    FMLB_REQUIRE(nmol == 0 || (charges && coords && offsets), "fmlb_coulomb_matrices: null input");
    if (nmol == 0) return FMLB_OK;
    static const DiagTable diag = make_diag_table();
    const int per_warp = 5 * nmax + (nmax + 1) / 2 + 1;
    const size_t smem = sizeof(double) * per_warp * kWarpsPerBlock;
    cm_sorted_kernel<<<ceil_div(nmol, kWarpsPerBlock), kWarpsPerBlock * 32, smem,
                       FMLB_STREAM(stream)>>>(charges, coords, offsets, nmol, nmax, cm, ldcm,
                                              cm32, ldcm32, order, diag, status);
    return launch_status("cm_sorted_kernel");
}

extern "C" int fmlb_unsorted_coulomb_matrices(const double *charges, const double *coords,
                                              const int *offsets, int nmol, int nmax, double *cm,
                                              int ldcm, int *status, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(nmol >= 0, "fmlb_unsorted_coulomb_matrices: nmol < 0");
    FMLB_REQUIRE(nmax >= 1 && nmax <= 255,
                 "fmlb_unsorted_coulomb_matrices: nmax=%d outside 1..255", nmax);
    const int L = nmax * (nmax + 1) / 2;
    FMLB_REQUIRE(ldcm >= L, "fmlb_unsorted_coulomb_matrices: ldcm=%d < %d", ldcm, L);
    FMLB_REQUIRE(nmol == 0 || (charges && coords && offsets && cm),
                 "fmlb_unsorted_coulomb_matrices: null pointer");
    if (nmol == 0) return FMLB_OK;
    static const DiagTable diag = make_diag_table();
    const size_t smem = sizeof(double) * 4 * nmax * kWarpsPerBlock;
    cm_unsorted_kernel<<<ceil_div(nmol, kWarpsPerBlock), kWarpsPerBlock * 32, smem,
                         FMLB_STREAM(stream)>>>(charges, coords, offsets, nmol, nmax, cm, ldcm,
                                                diag, status);
    return launch_status("cm_unsorted_kernel");
}

extern "C" int fmlb_local_coulomb_matrices(const double *charges, const double *coords,
                                           const int *offsets, int nmol, int nmax, int kind,
                                           double *cm, int ldcm, int *status, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(nmol >= 0, "fmlb_local_coulomb_matrices: nmol < 0");
    FMLB_REQUIRE(nmax >= 1 && nmax <= 255, "fmlb_local_coulomb_matrices: nmax=%d outside 1..255",
                 nmax);
    FMLB_REQUIRE(kind == 0 || kind == 1, "fmlb_local_coulomb_matrices: kind must be 0 or 1");
    const int L = nmax * (nmax + 1) / 2;
    FMLB_REQUIRE(ldcm >= L, "fmlb_local_coulomb_matrices: ldcm=%d < %d", ldcm, L);
    FMLB_REQUIRE(nmol == 0 || (charges && coords && offsets && cm),
                 "fmlb_local_coulomb_matrices: null pointer");
    if (nmol == 0) return FMLB_OK;
    static const DiagTable diag = make_diag_table();
    const size_t smem = sizeof(double) * (5 * nmax + nmax) * kWarpsPerBlock;
    cm_local_kernel<<<ceil_div(nmol, kWarpsPerBlock), kWarpsPerBlock * 32, smem,
                      FMLB_STREAM(stream)>>>(charges, coords, offsets, nmol, nmax, kind, cm, ldcm,
                                             diag, status);
    return launch_status("cm_local_kernel");
}

extern "C" int fmlb_arad_descriptors(const double *charges, const double *coords,
                                     const int *offsets, int nmol, int size, double cut,
                                     double *out, int *status, void *stream) {
    using namespace fmlb;
    FMLB_REQUIRE(nmol >= 0, "fmlb_arad_descriptors: nmol < 0");
    FMLB_REQUIRE(size >= 1 && size <= 128, "fmlb_arad_descriptors: size=%d outside 1..128", size);
    FMLB_REQUIRE(nmol == 0 || (charges && coords && offsets && out),
                 "fmlb_arad_descriptors: null pointer");
    if (nmol == 0) return FMLB_OK;
    static const PtpTable ptp = [] { PtpTable t; fill_ptp(t); return t; }();
    const int per_warp = 5 * size + (size + 1) / 2 + 1;
    const size_t smem = sizeof(double) * (5 * size + per_warp * kWarpsPerBlock);
    arad_describe_kernel<<<nmol, kWarpsPerBlock * 32, smem, FMLB_STREAM(stream)>>>(
        charges, coords, offsets, nmol, size, cut, out, ptp, status);
    return launch_status("arad_describe_kernel");
}
