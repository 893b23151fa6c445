/*
 * CPU ORACLE — test infrastructure, not product code.
 *
 * Plain-C FP64 restatement of the reference's Fortran routines on the KRR hot
 * path. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm may load this library; the product (fml_b200) never does.
 *
 * Every routine cites the reference file:line it restates (paths are relative
 * to the andersx/fml tree). Arithmetic is written in the same order as the
 * Fortran source and is compiled with -ffp-contract=off so that no FMA is
 * introduced. Parallelism follows the reference: one OpenMP loop over the
 * outermost molecule / column index.
 *
 * Layout convention (C order, matching the numpy arrays the reference's
 * Python wrappers hand to f2py):
 *   descriptors  X   (n, d)              row = one descriptor
 *   kernel       K   (na, nb)            K[j*nb + i] = k(A_j, B_i)
 *   ARAD         Q   (nm, amax, 5, amax) Q[((m*amax + a)*5 + ch)*amax + k]
 *   PTP          Z   (nm, amax, 2)
 *   ARAD kernel  K   (nsigma, nm1, nm2)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Sorted Coulomb matrix: frepresentations.f90:23-110                         */
/* ------------------------------------------------------------------------ */
/*
 * charges[n], coords[n*3] (row-major), output cm[nmax*(nmax+1)/2].
 * order_out (optional, n ints): order_out[p] = original 0-based atom index
 * placed at sorted position p.
 * Returns 0, or -1 when n > nmax (the Fortran writes out of bounds there).
 */
int orc_cm_sorted(int n, const double *charges, const double *coords, int nmax,
                  double *cm, int *order_out)
{
    if (n > nmax || n < 0) return -1;
    const int len = nmax * (nmax + 1) / 2;
    for (int t = 0; t < len; ++t) cm[t] = 0.0;
    if (n == 0) return 0;

    double *pair = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *row_norms = (double *)malloc(sizeof(double) * n);
    int *sorted_atoms = (int *)malloc(sizeof(int) * n);

    /* :62-70 diagonal 0.5 * Z**2.4 seeds the row norms */
    for (int i = 0; i < n; ++i) {
        double pn = 0.5 * pow(charges[i], 2.4);
        row_norms[i] = 0.0 + pn;
        pair[i * n + i] = pn;
    }
    /* :72-84 off-diagonal Z_i Z_j / |R_j - R_i|, accumulated in loop order */
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            double dx = coords[j * 3 + 0] - coords[i * 3 + 0];
            double dy = coords[j * 3 + 1] - coords[i * 3 + 1];
            double dz = coords[j * 3 + 2] - coords[i * 3 + 2];
            double s = dx * dx;
            s = s + dy * dy;
            s = s + dz * dz;
            double pn = charges[i] * charges[j] / sqrt(s);
            row_norms[j] = row_norms[j] + pn;
            row_norms[i] = row_norms[i] + pn;
            pair[i * n + j] = pn;
            pair[j * n + i] = pn;
        }
    }
    /* :86-91 repeated minloc (first index of the minimum), filled from the end */
    for (int it = 0; it < n; ++it) {
        int jmin = 0;
        for (int j = 1; j < n; ++j)
            if (row_norms[j] < row_norms[jmin]) jmin = j;
        sorted_atoms[n - it - 1] = jmin;
        row_norms[jmin] = DBL_MAX;
    }
    /* :93-104 packed lower triangle of the sorted matrix, row by row */
    for (int m = 0; m < n; ++m) {
        int i = sorted_atoms[m];
        int idx = m * (m + 1) / 2;
        for (int q = 0; q <= m; ++q) cm[idx + q] = pair[i * n + sorted_atoms[q]];
    }
    if (order_out)
        for (int m = 0; m < n; ++m) order_out[m] = sorted_atoms[m];
    free(pair);
    free(row_norms);
    free(sorted_atoms);
    return 0;
}

/* Batch form: offsets[nmol+1] into the packed atom arrays; cm (nmol, len). */
int orc_cm_sorted_batch(int nmol, const int *offsets, const double *charges,
                        const double *coords, int nmax, double *cm, int *order_out)
{
    const int len = nmax * (nmax + 1) / 2;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
    for (int m = 0; m < nmol; ++m) {
        int a0 = offsets[m], n = offsets[m + 1] - offsets[m];
        int rc = orc_cm_sorted(n, charges + a0, coords + 3 * (size_t)a0, nmax,
                               cm + (size_t)m * len,
                               order_out ? order_out + (size_t)m * nmax : NULL);
        if (rc) bad |= 1;
    }
    return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Unsorted Coulomb matrix: frepresentations.f90:112-202 (identity order)     */
/* ------------------------------------------------------------------------ */
int orc_cm_unsorted_batch(int nmol, const int *offsets, const double *charges,
                          const double *coords, int nmax, double *cm)
{
    const int len = nmax * (nmax + 1) / 2;
    int bad = 0;
    for (int mol = 0; mol < nmol; ++mol) {
        const int a0 = offsets[mol], n = offsets[mol + 1] - offsets[mol];
        double *row = cm + (size_t)mol * len;
        for (int t = 0; t < len; ++t) row[t] = 0.0;
        if (n < 0 || n > nmax) { bad = 1; continue; }
        const double *z = charges + a0, *r = coords + 3 * (size_t)a0;
        for (int m = 0; m < n; ++m) {           /* :184-192 */
            const int idx = m * (m + 1) / 2;
            for (int q = 0; q <= m; ++q) {
                double v;
                if (q == m) {
                    v = 0.5 * pow(z[m], 2.4);    /* :161-165 */
                } else {                          /* :167-178, i = q < j = m */
                    double dx = r[3 * m + 0] - r[3 * q + 0];
                    double dy = r[3 * m + 1] - r[3 * q + 1];
                    double dz = r[3 * m + 2] - r[3 * q + 2];
                    double s2 = dx * dx;
                    s2 = s2 + dy * dy;
                    s2 = s2 + dz * dz;
                    v = z[q] * z[m] / sqrt(s2);
                }
                row[idx + q] = v;
            }
        }
    }
    return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Local / atomic Coulomb matrices: frepresentations.f90:204-294 / :297-390   */
/* ------------------------------------------------------------------------ */
/* One molecule: cm (n, len) rows, kind 0 local, 1 atomic. Returns -1 if n > nmax. */
int orc_cm_local(int n, const double *charges, const double *coords, int nmax, int kind,
                 double *cm)
{
    if (n > nmax || n < 0) return -1;
    const int len = nmax * (nmax + 1) / 2;
    for (size_t t = 0; t < (size_t)n * len; ++t) cm[t] = 0.0;
    if (n == 0) return 0;
    double *pair = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *dist = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *row_norms = (double *)malloc(sizeof(double) * n);
    int *sorted_atoms = (int *)malloc(sizeof(int) * n);
    int *order = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) { /* :238-244, :344-346 */
        double pn = 0.5 * pow(charges[i], 2.4);
        row_norms[i] = 0.0 + pn;
        pair[i * n + i] = pn;
        dist[i * n + i] = 0.0;
    }
    for (int i = 0; i < n; ++i) /* :246-259, :336-354 */
        for (int j = i + 1; j < n; ++j) {
            double dx = coords[j * 3 + 0] - coords[i * 3 + 0];
            double dy = coords[j * 3 + 1] - coords[i * 3 + 1];
            double dz = coords[j * 3 + 2] - coords[i * 3 + 2];
            double s = dx * dx;
            s = s + dy * dy;
            s = s + dz * dz;
            double d = sqrt(s);
            double pn = charges[i] * charges[j] / d;
            row_norms[j] = row_norms[j] + pn;
            row_norms[i] = row_norms[i] + pn;
            pair[i * n + j] = pn;
            pair[j * n + i] = pn;
            dist[i * n + j] = d;
            dist[j * n + i] = d;
        }
    for (int it = 0; it < n; ++it) { /* :262-266 */
        int jmin = 0;
        for (int j = 1; j < n; ++j)
            if (row_norms[j] < row_norms[jmin]) jmin = j;
        sorted_atoms[n - it - 1] = jmin;
        row_norms[jmin] = DBL_MAX;
    }
    for (int k = 0; k < n; ++k) {
        if (kind == 0) { /* :268-277: k, then the sorted atoms without k */
            order[0] = k;
            int m = 0;
            for (int i = 0; i < n - 1; ++i) {
                if (sorted_atoms[i] == k) m = 1;
                order[i + 1] = sorted_atoms[i + m];
            }
        } else { /* :366-371: repeated minloc over the distances to k */
            double *col = (double *)malloc(sizeof(double) * n);
            for (int i = 0; i < n; ++i) col[i] = dist[i * n + k];
            for (int it = 0; it < n; ++it) {
                int jmin = 0;
                for (int j = 1; j < n; ++j)
                    if (col[j] < col[jmin]) jmin = j;
                order[it] = jmin;
                col[jmin] = DBL_MAX;
            }
            free(col);
        }
        for (int m = 0; m < n; ++m) { /* :281-291 / :375-386 */
            int idx = m * (m + 1) / 2;
            for (int q = 0; q <= m; ++q)
                cm[(size_t)k * len + idx + q] = pair[order[m] * n + order[q]];
        }
    }
    free(pair); free(dist); free(row_norms); free(sorted_atoms); free(order);
    return 0;
}

/* Batch: rows of every atom, cm (total_atoms, len). */
int orc_cm_local_batch(int nmol, const int *offsets, const double *charges,
                       const double *coords, int nmax, int kind, double *cm)
{
    const int len = nmax * (nmax + 1) / 2;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
    for (int m = 0; m < nmol; ++m) {
        int a0 = offsets[m], n = offsets[m + 1] - offsets[m];
        if (orc_cm_local(n, charges + a0, coords + 3 * (size_t)a0, nmax, kind,
                         cm + (size_t)a0 * len))
            bad |= 1;
    }
    return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Atomic vector kernels: fkernels.f90:23-104 (Laplacian, Gaussian)           */
/* ------------------------------------------------------------------------ */
/* X (nm, amax, d) row-major; K (nsig, nm1, nm2); kind 0 Gaussian, 1 Laplacian */
void orc_vector_kernels(int kind, const double *X1, const int *N1, int nm1, int amax1,
                        const double *X2, const int *N2, int nm2, int amax2, int d,
                        const double *sigmas, int nsig, double *K)
{
#pragma omp parallel for schedule(dynamic)
    for (int j = 0; j < nm2; ++j) {
        double *ad = (double *)malloc(sizeof(double) * (size_t)amax1 * amax2);
        for (int i = 0; i < nm1; ++i) {
            int ni = N1[i], nj = N2[j];
            for (int ja = 0; ja < nj; ++ja)
                for (int ia = 0; ia < ni; ++ia) {
                    const double *a = X1 + ((size_t)i * amax1 + ia) * d;
                    const double *b = X2 + ((size_t)j * amax2 + ja) * d;
                    double s = 0.0;
                    for (int f = 0; f < d; ++f) {
                        double t = a[f] - b[f];
                        s = s + (kind == 0 ? t * t : fabs(t));
                    }
                    ad[(size_t)ja * ni + ia] = s; /* column-major (ia fastest) */
                }
            for (int k = 0; k < nsig; ++k) {
                double c = kind == 0 ? -0.5 / (sigmas[k] * sigmas[k]) : -1.0 / sigmas[k];
                double acc = 0.0;
                for (int t = 0; t < ni * nj; ++t) acc = acc + exp(ad[t] * c);
                K[((size_t)k * nm1 + i) * nm2 + j] = acc;
            }
        }
        free(ad);
    }
}

/* ------------------------------------------------------------------------ */
/* Atomic Laplacian KRR: fkernels.f90:380-702. Atom descriptors are rows      */
/* Q (na, nv); molecule m owns atoms off[m] .. off[m+1].                      */
/* ------------------------------------------------------------------------ */
/* fget_alpha's matrix before lambda, :409-432: ltcl(i, j) for i <= j as the
 * reference builds it (ltc over all na atoms, then summed per molecule).
 * K (nm, nm) receives both triangles (the lower mirrored). */
void orc_atomic_laplacian_kernel(const double *Q, int na, int nv, const int *off, int nm,
                                 double sigma, double *K)
{
    const double inv_sigma = -1.0 / sigma;
#pragma omp parallel
    {
        double *ltc = (double *)malloc(sizeof(double) * (na > 0 ? na : 1));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nm; ++j) {
            for (int i = 0; i < na; ++i) {
                double acc = 0.0;
                for (int k = off[j]; k < off[j + 1]; ++k) {
                    double s = 0.0;
                    for (int f = 0; f < nv; ++f)
                        s = s + fabs(Q[(size_t)k * nv + f] - Q[(size_t)i * nv + f]);
                    acc = acc + exp(inv_sigma * s);
                }
                ltc[i] = acc;
            }
            for (int i = 0; i <= j; ++i) {
                double t = 0.0;
                for (int a = off[i]; a < off[i + 1]; ++a) t = t + ltc[a];
                K[(size_t)i * nm + j] = t;
                K[(size_t)j * nm + i] = t;
            }
        }
        free(ltc);
    }
}

/* fget_prediction, :508-535: csa over all test atoms, then per-molecule sums. */
void orc_atomic_laplacian_predict(const double *Q, int na, const double *Q2, int na2, int nv,
                                  const int *off2, int nm2, const double *alpha, double sigma,
                                  double *Y)
{
    const double inv_sigma = -1.0 / sigma;
    double *csa = (double *)calloc(na2 > 0 ? na2 : 1, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < na2; ++i) {
        double acc = 0.0;
        for (int j = 0; j < na; ++j) {
            double s = 0.0;
            for (int f = 0; f < nv; ++f) s = s + fabs(Q[(size_t)j * nv + f] - Q2[(size_t)i * nv + f]);
            acc = acc + exp(inv_sigma * s) * alpha[j];
        }
        csa[i] = acc;
    }
    for (int j = 0; j < nm2; ++j) {
        double t = 0.0;
        for (int a = off2[j]; a < off2[j + 1]; ++a) t = t + csa[a];
        Y[j] = t;
    }
    free(csa);
}

/* fget_alpha_from_distance's matrix before lambda, :577-597; D (na, na)
 * row-major is the numpy array, d(k, i) = D[k][i]. */
void orc_distance_mol_kernel(const double *D, int na, const int *off, int nm, double dgamma,
                             double *K)
{
    const double inv_gamma = -1.0 / dgamma;
    double *ltc = (double *)malloc(sizeof(double) * (size_t)(nm > 0 ? nm : 1) * (na > 0 ? na : 1));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nm; ++j) {
            double acc = 0.0;
            for (int k = off[j]; k < off[j + 1]; ++k) acc = acc + exp(inv_gamma * D[(size_t)k * na + i]);
            ltc[(size_t)j * na + i] = acc;
        }
    for (int j = 0; j < nm; ++j)
        for (int i = 0; i < nm; ++i) {
            double t = 0.0;
            for (int a = off[i]; a < off[i + 1]; ++a) t = t + ltc[(size_t)j * na + a];
            K[(size_t)i * nm + j] = t;
        }
    free(ltc);
}

/* fget_prediction_from_distance, :681-698 (csa starts at zero here). */
void orc_distance_predict(const double *D2, int na, int na2, const int *off2, int nm2,
                          const double *alpha, double dgamma, double *Y)
{
    const double inv_gamma = -1.0 / dgamma;
    double *csa = (double *)calloc(na2 > 0 ? na2 : 1, sizeof(double));
    for (int i = 0; i < na2; ++i)
        for (int j = 0; j < na; ++j)
            csa[i] = csa[i] + exp(inv_gamma * D2[(size_t)j * na2 + i]) * alpha[j];
    for (int j = 0; j < nm2; ++j) {
        double t = 0.0;
        for (int a = off2[j]; a < off2[j + 1]; ++a) t = t + csa[a];
        Y[j] = t;
    }
    free(csa);
}

/* ------------------------------------------------------------------------ */
/* Distance matrices: fdistance.f90:23-155. A (na, nv), B (nb, nv) rows;      */
/* D (na, nb). kind 0 manhattan, 1 l2, 2 integer p, 3 real p.                 */
/* ------------------------------------------------------------------------ */
void orc_distance_matrix(int kind, const double *A, int na, const double *B, int nb, int nv,
                         int p_int, double p_real, double *D)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < na; ++j) {
            double s = 0.0;
            for (int k = 0; k < nv; ++k) {
                double t = A[(size_t)j * nv + k] - B[(size_t)i * nv + k];
                double term;
                if (kind == 0) term = fabs(t);
                else if (kind == 1) term = t * t;
                else if (kind == 2) term = pow(t, (double)p_int);
                else term = pow(t, p_real);
                s = s + term;
            }
            if (kind == 1) s = sqrt(s);
            else if (kind == 2) s = pow(s, 1.0 / (double)p_int);
            else if (kind == 3) s = pow(s, 1.0 / p_real);
            D[(size_t)j * nb + i] = s;
        }
}

/* ------------------------------------------------------------------------ */
/* Gaussian kernel: fkernels.f90:317-349                                      */
/* ------------------------------------------------------------------------ */
void orc_gaussian_kernel(const double *A, int na, const double *B, int nb, int d,
                         double sigma, double *K)
{
    const double inv_sigma = -0.5 / (sigma * sigma); /* :334 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nb; ++i) {                 /* :338-339 OMP over columns of B */
        const double *b = B + (size_t)i * d;
        for (int j = 0; j < na; ++j) {
            const double *a = A + (size_t)j * d;
            double s = 0.0;
            for (int k = 0; k < d; ++k) {          /* :341-342 sum(temp*temp) */
                double t = a[k] - b[k];
                s = s + t * t;
            }
            K[(size_t)j * nb + i] = exp(inv_sigma * s);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Laplacian kernel: fkernels.f90:351-377                                     */
/* ------------------------------------------------------------------------ */
void orc_laplacian_kernel(const double *A, int na, const double *B, int nb, int d,
                          double sigma, double *K)
{
    const double inv_sigma = -1.0 / sigma; /* :367 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nb; ++i) {
        const double *b = B + (size_t)i * d;
        for (int j = 0; j < na; ++j) {
            const double *a = A + (size_t)j * d;
            double s = 0.0;
            for (int k = 0; k < d; ++k) s = s + fabs(a[k] - b[k]); /* :372 */
            K[(size_t)j * nb + i] = exp(inv_sigma * s);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Several sigmas from one pass (fkernels.f90:317-377, the loops above): the  */
/* pair sum s of each (j, i) is formed once, in the same order as the single- */
/* sigma routines, and exp(inv_sigma * s) is taken per sigma, so every K_k is  */
/* bit-identical to orc_gaussian_kernel / orc_laplacian_kernel at sigma_k.     */
/* kind 0: Gaussian (sum of squares, inv_sigma = -0.5/sigma^2, :334, :341);    */
/* kind 1: Laplacian (sum of |a - b|, inv_sigma = -1/sigma, :367, :372).       */
/* K is (nsig, na, nb) row-major.                                              */
/* ------------------------------------------------------------------------ */
void orc_kernels_multi(int kind, const double *A, int na, const double *B, int nb, int d,
                       const double *sigmas, int nsig, double *K)
{
    double inv[16];
    for (int q = 0; q < nsig && q < 16; ++q)
        inv[q] = kind == 0 ? -0.5 / (sigmas[q] * sigmas[q]) : -1.0 / sigmas[q];
    const size_t plane = (size_t)na * nb;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nb; ++i) {
        const double *b = B + (size_t)i * d;
        for (int j = 0; j < na; ++j) {
            const double *a = A + (size_t)j * d;
            double s = 0.0;
            if (kind == 0) {
                for (int k = 0; k < d; ++k) {
                    double t = a[k] - b[k];
                    s = s + t * t;
                }
            } else {
                for (int k = 0; k < d; ++k) s = s + fabs(a[k] - b[k]);
            }
            for (int q = 0; q < nsig && q < 16; ++q)
                K[q * plane + (size_t)j * nb + i] = exp(inv[q] * s);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* ARAD atom-pair distance: farad_kernels.f90:29-90 (atomic_distl2)           */
/* ------------------------------------------------------------------------ */
/* x1, x2: one atom's descriptor (5, amax) row-major; s1, s2: sine factors.   */
static double orc_atomic_distl2(const double *x1, const double *x2, int n1, int n2,
                                const double *s1, const double *s2, int amax,
                                double width, double cut, double r_width, double c_width)
{
    const double inv_width = -1.0 / (4.0 * width * width); /* :58 */
    const double maxgausdist2 = (8.0 * width) * (8.0 * width); /* :60 */
    const double rw2 = r_width * r_width, cw2 = c_width * c_width;
    const double *r1 = x1, *p1 = x1 + amax, *g1 = x1 + 2 * amax, *c1 = x1 + 3 * amax,
                 *z1 = x1 + 4 * amax;
    const double *r2 = x2, *p2 = x2 + amax, *g2 = x2 + 2 * amax, *c2 = x2 + 3 * amax,
                 *z2 = x2 + 4 * amax;
    double aadist = 0.0;
    for (int m1 = 0; m1 < n1; ++m1) {
        if (r1[m1] > cut) break;                        /* :68 */
        for (int m2 = 0; m2 < n2; ++m2) {
            if (r2[m2] > cut) break;                    /* :72 */
            double dr = r2[m2] - r1[m1];
            double r2v = dr * dr;                       /* :74 */
            if (r2v < maxgausdist2) {                   /* :76 */
                double d = exp(r2v * inv_width) * s1[m1] * s2[m2]; /* :78 */
                double dp = p1[m1] - p2[m2], dg = g1[m1] - g2[m2];
                d = d * (rw2 / (rw2 + dp * dp) * cw2 / (cw2 + dg * dg)); /* :80-81 */
                aadist = aadist + d * (1.0 + c1[m1] * c2[m2] + z1[m1] * z2[m2]); /* :83 */
            }
        }
    }
    return aadist;
}

/* sin factor tables, farad_kernels.f90:521-545 (non-symmetric: only r < cut)
 * and :689-698 (symmetric: unconditional). sin[(m*amax + a)*amax + k]. */
static double *orc_arad_sines(const double *Q, const int *N, int nm, int amax, double cut,
                              int conditional)
{
    const double pi = 4.0 * atan(1.0);
    const double inv_cut = pi / (2.0 * cut); /* :510 */
    double *s = (double *)calloc((size_t)nm * amax * amax, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int m = 0; m < nm; ++m) {
        int ni = N[m];
        for (int k = 0; k < ni; ++k)
            for (int a = 0; a < ni; ++a) {
                double r = Q[(((size_t)m * amax + a) * 5 + 0) * amax + k];
                if (!conditional || r < cut)
                    s[((size_t)m * amax + a) * amax + k] = 1.0 - sin(r * inv_cut);
            }
    }
    return s;
}

/* self terms selfl2, farad_kernels.f90:550-568 */
static double *orc_arad_self(const double *Q, const int *N, const double *S, int nm, int amax,
                             double width, double cut, double rw, double cw)
{
    double *self = (double *)calloc((size_t)nm * amax, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int m = 0; m < nm; ++m) {
        int ni = N[m];
        for (int a = 0; a < ni; ++a) {
            const double *x = Q + ((size_t)m * amax + a) * 5 * amax;
            const double *s = S + ((size_t)m * amax + a) * amax;
            self[(size_t)m * amax + a] =
                orc_atomic_distl2(x, x, ni, ni, s, s, amax, width, cut, rw, cw);
        }
    }
    return self;
}

static double orc_arad_pair(const double *Q1, const double *Z1, const int *N1, const double *S1,
                            const double *self1, int i, const double *Q2, const double *Z2,
                            const int *N2, const double *S2, const double *self2, int j,
                            int amax, double width, double cut, double rw, double cw,
                            const double *inv_sigma2, int nsig, double eps, double *ad,
                            double *out)
{
    /* eps: the single-precision literal 5.0e-12 of :505 / :679, or 1.0e-11 (:309)
     * for fget_alpha_arad */
    const double rw2 = rw * rw, cw2 = cw * cw;
    int ni = N1[i], nj = N2[j];
    for (int j1 = 0; j1 < nj; ++j1) {
        for (int i1 = 0; i1 < ni; ++i1) {
            const double *x1 = Q1 + ((size_t)i * amax + i1) * 5 * amax;
            const double *x2 = Q2 + ((size_t)j * amax + j1) * 5 * amax;
            double l2 = orc_atomic_distl2(x1, x2, ni, nj, S1 + ((size_t)i * amax + i1) * amax,
                                          S2 + ((size_t)j * amax + j1) * amax, amax, width, cut,
                                          rw, cw);
            double dz1 = Z1[((size_t)i * amax + i1) * 2 + 0] - Z2[((size_t)j * amax + j1) * 2 + 0];
            double dz2 = Z1[((size_t)i * amax + i1) * 2 + 1] - Z2[((size_t)j * amax + j1) * 2 + 1];
            /* :590-592 */
            l2 = self1[(size_t)i * amax + i1] + self2[(size_t)j * amax + j1] -
                 2.0 * l2 * (rw2 / (rw2 + dz1 * dz1) * cw2 / (cw2 + dz2 * dz2));
            if (fabs(l2) < eps) l2 = 0.0; /* :594 */
            ad[(size_t)j1 * ni + i1] = l2; /* column-major like atomic_distance(:ni,:nj) */
        }
    }
    /* :602-604 sum(exp(atomic_distance(:ni,:nj) * inv_sigma2(k))), column-major order */
    for (int k = 0; k < nsig; ++k) {
        double s = 0.0;
        for (int t = 0; t < ni * nj; ++t) s = s + exp(ad[t] * inv_sigma2[k]);
        out[k] = s;
    }
    return 0.0;
}

/* fget_atomic_kernels_arad: farad_kernels.f90:757-899. Q (na, 5, amax) per-atom
 * descriptors, Z (na, 2), N (na,) neighbour counts; K (nsig, na1, na2). */
static void orc_arad_atomic(const double *Q1, const double *Q2, const double *Z1,
                            const double *Z2, const int *N1, const int *N2,
                            const double *sigmas, int na1, int na2, int nsig, int amax,
                            double width, double cut, double rw, double cw, double *K,
                            int distance)
{
    const double pi = 4.0 * atan(1.0);
    const double inv_cut = pi / (2.0 * cut); /* :828 */
    const double eps = 5.0e-12f;            /* :823 */
    const double rw2 = rw * rw, cw2 = cw * cw;
    double *s1 = (double *)calloc((size_t)na1 * amax, sizeof(double));
    double *s2 = (double *)calloc((size_t)na2 * amax, sizeof(double));
    double *self1 = (double *)calloc((size_t)na1, sizeof(double));
    double *self2 = (double *)calloc((size_t)na2, sizeof(double));
    for (int i = 0; i < na1; ++i) /* :836-842 */
        for (int m = 0; m < N1[i]; ++m)
            s1[(size_t)i * amax + m] = 1.0 - sin(Q1[((size_t)i * 5) * amax + m] * inv_cut);
    for (int i = 0; i < na2; ++i) /* :844-850 */
        for (int m = 0; m < N2[i]; ++m)
            s2[(size_t)i * amax + m] = 1.0 - sin(Q2[((size_t)i * 5) * amax + m] * inv_cut);
    for (int i = 0; i < na1; ++i) { /* :855-860 */
        const double *x = Q1 + (size_t)i * 5 * amax, *s = s1 + (size_t)i * amax;
        self1[i] = orc_atomic_distl2(x, x, N1[i], N1[i], s, s, amax, width, cut, rw, cw);
    }
    for (int i = 0; i < na2; ++i) { /* :862-868 */
        const double *x = Q2 + (size_t)i * 5 * amax, *s = s2 + (size_t)i * amax;
        self2[i] = orc_atomic_distl2(x, x, N2[i], N2[i], s, s, amax, width, cut, rw, cw);
    }
#pragma omp parallel for schedule(dynamic)
    for (int j = 0; j < na2; ++j) /* :873-891 */
        for (int i = 0; i < na1; ++i) {
            double l2 = orc_atomic_distl2(Q1 + (size_t)i * 5 * amax, Q2 + (size_t)j * 5 * amax,
                                          N1[i], N2[j], s1 + (size_t)i * amax,
                                          s2 + (size_t)j * amax, amax, width, cut, rw, cw);
            const double dz1 = Z1[2 * i] - Z2[2 * j], dz2 = Z1[2 * i + 1] - Z2[2 * j + 1];
            l2 = self1[i] + self2[j] -
                 2.0 * l2 * (rw2 / (rw2 + dz1 * dz1) * cw2 / (cw2 + dz2 * dz2));
            if (fabs(l2) < eps) l2 = 0.0;
            if (distance) { /* fget_atomic_distance_arad stores l2 (:1019) */
                K[(size_t)i * na2 + j] = l2;
                continue;
            }
            for (int k = 0; k < nsig; ++k)
                K[((size_t)k * na1 + i) * na2 + j] = exp(l2 * (-1.0 / (sigmas[k] * sigmas[k])));
        }
    free(s1); free(s2); free(self1); free(self2);
}

void orc_arad_atomic_kernels(const double *Q1, const double *Q2, const double *Z1,
                             const double *Z2, const int *N1, const int *N2,
                             const double *sigmas, int na1, int na2, int nsig, int amax,
                             double width, double cut, double rw, double cw, double *K)
{
    orc_arad_atomic(Q1, Q2, Z1, Z2, N1, N2, sigmas, na1, na2, nsig, amax, width, cut, rw, cw,
                    K, 0);
}

/* fget_atomic_distance_arad: farad_kernels.f90:902-1030; D[i, j] = l2(i, j). */
void orc_arad_atomic_distances(const double *Q1, const double *Q2, const double *Z1,
                               const double *Z2, const int *N1, const int *N2, int na1, int na2,
                               int amax, double width, double cut, double rw, double cw,
                               double *D)
{
    orc_arad_atomic(Q1, Q2, Z1, Z2, N1, N2, NULL, na1, na2, 0, amax, width, cut, rw, cw, D, 1);
}

/* fget_kernels_arad: farad_kernels.f90:439-616. K (nsig, nm1, nm2). */
void orc_arad_kernels(const double *Q1, const double *Q2, const double *Z1, const double *Z2,
                      const int *N1, const int *N2, const double *sigmas, int nm1, int nm2,
                      int nsig, int amax, double width, double cut, double rw, double cw,
                      double *K)
{
    double *inv_sigma2 = (double *)malloc(sizeof(double) * (nsig > 0 ? nsig : 1));
    for (int k = 0; k < nsig; ++k) inv_sigma2[k] = -1.0 / (sigmas[k] * sigmas[k]); /* :511 */
    double *S1 = orc_arad_sines(Q1, N1, nm1, amax, cut, 1);
    double *S2 = orc_arad_sines(Q2, N2, nm2, amax, cut, 1);
    double *self1 = orc_arad_self(Q1, N1, S1, nm1, amax, width, cut, rw, cw);
    double *self2 = orc_arad_self(Q2, N2, S2, nm2, amax, width, cut, rw, cw);
#pragma omp parallel
    {
        double *ad = (double *)malloc(sizeof(double) * (size_t)amax * amax);
        double *out = (double *)malloc(sizeof(double) * (nsig > 0 ? nsig : 1));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nm2; ++j) { /* :576-577 OMP over molecules of set 2 */
            for (int i = 0; i < nm1; ++i) {
                orc_arad_pair(Q1, Z1, N1, S1, self1, i, Q2, Z2, N2, S2, self2, j, amax, width,
                              cut, rw, cw, inv_sigma2, nsig, (double)5.0e-12f, ad, out);
                for (int k = 0; k < nsig; ++k)
                    K[((size_t)k * nm1 + i) * nm2 + j] = out[k];
            }
        }
        free(ad);
        free(out);
    }
    free(inv_sigma2);
    free(S1);
    free(S2);
    free(self1);
    free(self2);
}

static void orc_arad_symmetric(const double *Q1, const double *Z1, const int *N1,
                               const double *sigmas, int nm1, int nsig, int amax, double width,
                               double cut, double rw, double cw, double eps, double *K);

/* atomic_arad_l2_distance_all: farad.f90:452-600 (its atomic_distl2,
 * :62-123, is the same function as farad_kernels.f90:29-90). Sines for every
 * listed neighbour of both sets (:519-539), eps 5.0e-12 single-precision
 * (:509). D (nm1, nm2, amax, amax), zero past each molecule's atoms. */
void orc_arad_l2_distance_all(const double *Q1, const double *Q2, const double *Z1,
                              const double *Z2, const int *N1, const int *N2, int nm1, int nm2,
                              int amax, double width, double cut, double rw, double cw, double *D)
{
    const double eps = 5.0e-12f;
    const double rw2 = rw * rw, cw2 = cw * cw;
    double *S1 = orc_arad_sines(Q1, N1, nm1, amax, cut, 0);
    double *S2 = orc_arad_sines(Q2, N2, nm2, amax, cut, 0);
    double *self1 = orc_arad_self(Q1, N1, S1, nm1, amax, width, cut, rw, cw);
    double *self2 = orc_arad_self(Q2, N2, S2, nm2, amax, width, cut, rw, cw);
    for (size_t t = 0; t < (size_t)nm1 * nm2 * amax * amax; ++t) D[t] = 0.0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < nm2; ++j) {
        for (int i = 0; i < nm1; ++i) {
            for (int i1 = 0; i1 < N1[i]; ++i1) {
                for (int j1 = 0; j1 < N2[j]; ++j1) {
                    const size_t a = (size_t)i * amax + i1, b = (size_t)j * amax + j1;
                    double l2 = orc_atomic_distl2(Q1 + a * 5 * amax, Q2 + b * 5 * amax, N1[i],
                                                  N2[j], S1 + a * amax, S2 + b * amax, amax,
                                                  width, cut, rw, cw);
                    double dz1 = Z1[a * 2 + 0] - Z2[b * 2 + 0];
                    double dz2 = Z1[a * 2 + 1] - Z2[b * 2 + 1];
                    l2 = self1[a] + self2[b] -
                         2.0 * l2 * (rw2 / (rw2 + dz1 * dz1) * cw2 / (cw2 + dz2 * dz2));
                    if (fabs(l2) < eps) l2 = 0.0;
                    D[(((size_t)i * nm2 + j) * amax + i1) * amax + j1] = l2; /* :587 */
                }
            }
        }
    }
    free(S1);
    free(S2);
    free(self1);
    free(self2);
}

/* fget_symmetric_kernels_arad: farad_kernels.f90:619-755. K (nsig, nm, nm). */
void orc_arad_symmetric_kernels(const double *Q1, const double *Z1, const int *N1,
                                const double *sigmas, int nm1, int nsig, int amax, double width,
                                double cut, double rw, double cw, double *K)
{
    orc_arad_symmetric(Q1, Z1, N1, sigmas, nm1, nsig, amax, width, cut, rw, cw,
                       (double)5.0e-12f, K);
}

/* The matrix fget_alpha_arad factors (farad_kernels.f90:231-389): the
 * symmetric kernel for one sigma with width 0.2, cut 6, r_width 1,
 * c_width 0.5 (:237-240), eps the single-precision literal 1.0e-11 (:309),
 * then lambda added to the diagonal (:385-389). K (nm, nm). */
void orc_arad_alpha_kernel(const double *Q1, const double *Z1, const int *N1, int nm1, int amax,
                           double sigma, double lambda, double *K)
{
    orc_arad_symmetric(Q1, Z1, N1, &sigma, nm1, 1, amax, 0.2, 6.0, 1.0, 0.5,
                       (double)1.0e-11f, K);
    for (int i = 0; i < nm1; ++i) K[(size_t)i * nm1 + i] = K[(size_t)i * nm1 + i] + lambda;
}

static void orc_arad_symmetric(const double *Q1, const double *Z1, const int *N1,
                               const double *sigmas, int nm1, int nsig, int amax, double width,
                               double cut, double rw, double cw, double eps, double *K)
{
    double *inv_sigma2 = (double *)malloc(sizeof(double) * (nsig > 0 ? nsig : 1));
    for (int k = 0; k < nsig; ++k) inv_sigma2[k] = -1.0 / (sigmas[k] * sigmas[k]); /* :685 */
    double *S1 = orc_arad_sines(Q1, N1, nm1, amax, cut, 0);
    double *self1 = orc_arad_self(Q1, N1, S1, nm1, amax, width, cut, rw, cw);
#pragma omp parallel
    {
        double *ad = (double *)malloc(sizeof(double) * (size_t)amax * amax);
        double *out = (double *)malloc(sizeof(double) * (nsig > 0 ? nsig : 1));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nm1; ++j) {      /* :717-718 */
            for (int i = 0; i <= j; ++i) {   /* :720 only i <= j */
                orc_arad_pair(Q1, Z1, N1, S1, self1, i, Q1, Z1, N1, S1, self1, j, amax, width,
                              cut, rw, cw, inv_sigma2, nsig, eps, ad, out);
                for (int k = 0; k < nsig; ++k) {
                    K[((size_t)k * nm1 + i) * nm1 + j] = out[k];
                    K[((size_t)k * nm1 + j) * nm1 + i] = out[k]; /* :744 mirror */
                }
            }
        }
        free(ad);
        free(out);
    }
    free(inv_sigma2);
    free(S1);
    free(self1);
}

/* ------------------------------------------------------------------------ */
/* Cholesky: restatement of LAPACK dpotrf('U') / dpotrs('U') as called by     */
/* fcho_solve.f90:35-42 (unblocked "dpotf2" column order, Golub & Van Loan    */
/* Algorithm 4.2.1). A is the numpy (n, n) array in C order; its upper        */
/* triangle A[i][j], i <= j, is the Fortran A(i,j) upper triangle.            */
/* On exit the upper triangle holds U with A = U^T U. Returns LAPACK info:    */
/* 0, or the 1-based column of the first non-positive pivot.                  */
/* ------------------------------------------------------------------------ */
int orc_potrf_upper(int n, double *A)
{
    for (int j = 0; j < n; ++j) {
        double ajj = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) ajj -= A[(size_t)k * n + j] * A[(size_t)k * n + j];
        if (!(ajj > 0.0)) {
            A[(size_t)j * n + j] = ajj;
            return j + 1;
        }
        ajj = sqrt(ajj);
        A[(size_t)j * n + j] = ajj;
#pragma omp parallel for schedule(static)
        for (int c = j + 1; c < n; ++c) {
            double s = A[(size_t)j * n + c];
            for (int k = 0; k < j; ++k) s -= A[(size_t)k * n + j] * A[(size_t)k * n + c];
            A[(size_t)j * n + c] = s / ajj;
        }
    }
    return 0;
}

/* dpotrs('U', nrhs=1): solve U^T z = b, then U x = z, in place in x. */
void orc_potrs_upper(int n, const double *U, double *x)
{
    for (int i = 0; i < n; ++i) {
        double s = x[i];
        for (int k = 0; k < i; ++k) s -= U[(size_t)k * n + i] * x[k];
        x[i] = s / U[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int k = i + 1; k < n; ++k) s -= U[(size_t)i * n + k] * x[k];
        x[i] = s / U[(size_t)i * n + i];
    }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
