// Internal interface of the int8 (Ozaki) emulation of the FP64 trailing
// update, used by the Cholesky factorisation (cholesky_f64.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fmlb {

constexpr int OZAKI_MAX_SLICES = 8;

// Digit planes of a panel: ns planes of rows x kp int8 (row stride ldpl,
// plane stride pstride bytes), one exponent and one zero-point digit sum per
// row.
struct OzakiSlices {
    int8_t *planes = nullptr;
    int *exps = nullptr;
    double *rsum = nullptr;
    int rows = 0, kp = 0, ns = 0;
    long long ldpl = 0, pstride = 0;
};

// Bytes of a slice buffer for `rows` rows of kp (multiple of 32) columns.
size_t ozaki_slice_bytes(int rows, int kp, int ns);
// Lays out a slice buffer in `ws` (at least ozaki_slice_bytes bytes).
int ozaki_bind(void *ws, int rows, int kp, int ns, OzakiSlices &s);
// Splits rows [0, m) x columns [0, k) of P into s (returns at once when *info != 0).
int ozaki_split(const double *P, long long ldp, int m, int k, const OzakiSlices &s,
                const int *info, cudaStream_t st);
// C (m x m, lower triangle; first strip_cols columns if > 0) -= P P^T with
// P = slice rows [p_row0, p_row0 + m).
int ozaki_syrk(double *C, long long ldc, int m, const OzakiSlices &s, int p_row0, int strip_cols,
               int *info, cudaStream_t st);

}  // namespace fmlb
