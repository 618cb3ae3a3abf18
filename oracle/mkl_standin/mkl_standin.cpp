// mkl_standin.cpp -- implementations behind oracle/mkl_standin/include/mkl.h.
//
// Test infrastructure: lets the reference's own FGMRES / BCGSTAB sources run
// here (oracle/_ref) so the NumPy oracle can be checked against them.  Each
// routine follows the published definition of the MKL/BLAS/LAPACK routine it
// stands for; none of them is tuned.
//
//  * pardiso (mtype 13, complex unsymmetric, 1-based CSR): phase 11 records
//    the pattern, 22 factors, 33 solves one right-hand side, -1 releases.
//    The factorization is Gaussian elimination with partial pivoting kept in
//    band storage: rows are only swapped within the lower bandwidth, so the
//    fill stays inside kl + ku columns to the right of the diagonal.  The
//    band widths are measured from the CSR pattern.
//  * DFTI: complex double, 1D, strided, out of place; the transform
//    y_k = s * sum_j x_j exp(-+2 pi i j k / n) is evaluated directly, with the
//    angle reduced as (j*k mod n) before the cos/sin.
//  * zgels (trans = "N", m >= n): Householder QR and a triangular solve.
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mkl.h"
#include "mkl_dfti.h"

typedef std::complex<double> zc;

static void standin_missing(const char *name) {
    fprintf(stderr, "mkl stand-in: %s is not provided (not on the FGMRES path)\n", name);
    abort();
}

#define MISSING(ret, name) \
    extern "C" ret name(...) { standin_missing(#name); return (ret)0; }
#define MISSING_V(name) \
    extern "C" void name(...) { standin_missing(#name); }

MISSING_V(zgemm) MISSING_V(ztrsm) MISSING_V(zgetrf) MISSING_V(zlaswp) MISSING_V(mkl_zomatadd)
MISSING_V(zsyrk) MISSING_V(zsymm) MISSING_V(zpotrf) MISSING_V(mkl_zimatcopy) MISSING_V(zgetri)
MISSING_V(mkl_zomatcopy) MISSING_V(zgesvd) MISSING_V(zaxpby) MISSING_V(zgetrs) MISSING_V(zgecon)
MISSING_V(dgemm) MISSING_V(dgemv) MISSING_V(dsymv) MISSING_V(dsymm) MISSING_V(daxpby) MISSING_V(dgesvd)
MISSING_V(mkl_dimatcopy) MISSING_V(mkl_domatcopy) MISSING_V(mkl_domatadd) MISSING_V(mkl_dcsrgemv)
MISSING_V(mkl_zdnscsr) MISSING_V(dsyrk) MISSING_V(dpotrf) MISSING_V(dtrsm) MISSING_V(dgetrf)
MISSING_V(dgetri) MISSING_V(dlaswp) MISSING_V(dscal) MISSING_V(daxpy) MISSING_V(dcopy)
MISSING(double, ddot) MISSING(double, dnrm2) MISSING_V(dgeqrf) MISSING_V(zgeqrf) MISSING_V(dgels)
MISSING_V(zlaset) MISSING_V(dlaset) MISSING_V(zungqr) MISSING_V(dorgqr) MISSING_V(zgesv) MISSING_V(dgesv)
MISSING_V(zhemm) MISSING_V(ztrmm) MISSING_V(dtrmm)

extern "C" void mkl_set_num_threads(int) {}

// ---------------------------------------------------------------- BLAS 1/2
void zdotc(zc *pres, const int *n, const zc *x, const int *incx, const zc *y, const int *incy) {
    zc s = 0.0;
    for (int i = 0; i < *n; i++) s += std::conj(x[(long)i * *incx]) * y[(long)i * *incy];
    *pres = s;
}

void zaxpy(const int *n, const zc *alpha, const zc *x, const int *incx, zc *y, const int *incy) {
    for (int i = 0; i < *n; i++) y[(long)i * *incy] += *alpha * x[(long)i * *incx];
}

double dznrm2(const int *n, const zc *x, const int *incx) {
    // scaled sum of squares, as the reference BLAS does, to avoid overflow
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < *n; i++) {
        const double parts[2] = {x[(long)i * *incx].real(), x[(long)i * *incx].imag()};
        for (double v : parts) {
            if (v != 0.0) {
                double a = std::fabs(v);
                if (scale < a) {
                    ssq = 1.0 + ssq * (scale / a) * (scale / a);
                    scale = a;
                } else {
                    ssq += (a / scale) * (a / scale);
                }
            }
        }
    }
    return scale * std::sqrt(ssq);
}

void zcopy(const int *n, const zc *x, const int *incx, zc *y, const int *incy) {
    for (int i = 0; i < *n; i++) y[(long)i * *incy] = x[(long)i * *incx];
}

void zdscal(const int *n, const double *a, zc *x, const int *incx) {
    for (int i = 0; i < *n; i++) x[(long)i * *incx] *= *a;
}

void zscal(const int *n, const zc *a, zc *x, const int *incx) {
    for (int i = 0; i < *n; i++) x[(long)i * *incx] *= *a;
}

void zgemv(const char *trans, const int *m, const int *n, const zc *alpha, const zc *a, const int *lda,
           const zc *x, const int *incx, const zc *beta, zc *y, const int *incy) {
    const char t = trans[0];
    const bool no = (t == 'n' || t == 'N');
    const int ylen = no ? *m : *n;
    std::vector<zc> acc(ylen, 0.0);
    for (int j = 0; j < *n; j++)
        for (int i = 0; i < *m; i++) {
            zc aij = a[i + (long)*lda * j];
            if (no) acc[i] += aij * x[(long)j * *incx];
            else if (t == 'c' || t == 'C') acc[j] += std::conj(aij) * x[(long)i * *incx];
            else acc[j] += aij * x[(long)i * *incx];
        }
    for (int i = 0; i < ylen; i++) {
        zc yi = (*beta == zc(0.0)) ? zc(0.0) : *beta * y[(long)i * *incy];
        y[(long)i * *incy] = yi + *alpha * acc[i];
    }
}

void mkl_zcsrgemv(const char *transa, const int *m, const zc *a, const int *ia, const int *ja, const zc *x,
                  zc *y) {
    if (!(transa[0] == 'n' || transa[0] == 'N')) standin_missing("mkl_zcsrgemv(trans)");
    for (int i = 0; i < *m; i++) {
        zc s = 0.0;
        for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) s += a[p] * x[ja[p] - 1];
        y[i] = s;
    }
}

template <typename T>
static double lange_impl(const char *norm, int m, int n, const T *a, int lda) {
    const char c = norm[0];
    double r = 0.0;
    if (c == 'F' || c == 'f' || c == 'E' || c == 'e') {
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) r += std::norm(a[i + (long)lda * j]);
        return std::sqrt(r);
    }
    if (c == 'M' || c == 'm') {
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) r = std::max(r, (double)std::abs(a[i + (long)lda * j]));
        return r;
    }
    if (c == '1' || c == 'O' || c == 'o') {
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int i = 0; i < m; i++) s += std::abs(a[i + (long)lda * j]);
            r = std::max(r, s);
        }
        return r;
    }
    if (c == 'I' || c == 'i') {
        for (int i = 0; i < m; i++) {
            double s = 0.0;
            for (int j = 0; j < n; j++) s += std::abs(a[i + (long)lda * j]);
            r = std::max(r, s);
        }
        return r;
    }
    standin_missing("lange(norm)");
    return 0.0;
}

double zlange(const char *norm, const int *m, const int *n, const zc *a, const int *lda, double *) {
    return lange_impl(norm, *m, *n, a, *lda);
}
double dlange(const char *norm, const int *m, const int *n, const double *a, const int *lda, double *) {
    return lange_impl(norm, *m, *n, a, *lda);
}
float clange(const char *norm, const int *m, const int *n, const std::complex<float> *a, const int *lda, float *) {
    return (float)lange_impl(norm, *m, *n, a, *lda);
}

void zlacpy(const char *uplo, const int *m, const int *n, const zc *a, const int *lda, zc *b, const int *ldb) {
    const char u = uplo[0];
    for (int j = 0; j < *n; j++)
        for (int i = 0; i < *m; i++) {
            if ((u == 'U' || u == 'u') && i > j) continue;
            if ((u == 'L' || u == 'l') && i < j) continue;
            b[i + (long)*ldb * j] = a[i + (long)*lda * j];
        }
}
void dlacpy(const char *uplo, const int *m, const int *n, const double *a, const int *lda, double *b,
            const int *ldb) {
    const char u = uplo[0];
    for (int j = 0; j < *n; j++)
        for (int i = 0; i < *m; i++) {
            if ((u == 'U' || u == 'u') && i > j) continue;
            if ((u == 'L' || u == 'l') && i < j) continue;
            b[i + (long)*ldb * j] = a[i + (long)*lda * j];
        }
}

// ------------------------------------------------------------------ zgels
// Least squares min ||b - A x|| for a full-rank m x n A (m >= n), one or more
// right-hand sides, by Householder QR: A = Q R, x = R^{-1} (Q^H b)[0:n].
void zgels(const char *trans, const int *m, const int *n, const int *nrhs, zc *a, const int *lda, zc *b,
           const int *ldb, zc *work, const int *lwork, int *info) {
    *info = 0;
    if (*lwork == -1) {
        work[0] = zc((double)std::max(1, *n * 64), 0.0);
        return;
    }
    if (!(trans[0] == 'n' || trans[0] == 'N') || *m < *n) standin_missing("zgels(trans/m<n)");
    const int M = *m, N = *n, LDA = *lda, LDB = *ldb;
    for (int k = 0; k < N; k++) {
        // Householder vector v for column k (rows k..M-1): H = I - tau v v^H,
        // H^H x = (alpha, 0, ...) with |alpha| = ||x||.
        double xnorm = 0.0;
        for (int i = k; i < M; i++) xnorm += std::norm(a[i + (long)LDA * k]);
        xnorm = std::sqrt(xnorm);
        if (xnorm == 0.0) continue;
        zc x0 = a[k + (long)LDA * k];
        double ax0 = std::abs(x0);
        zc phase = (ax0 == 0.0) ? zc(1.0) : x0 / ax0;
        zc alpha = -phase * xnorm;
        std::vector<zc> v(M - k);
        v[0] = x0 - alpha;
        for (int i = k + 1; i < M; i++) v[i - k] = a[i + (long)LDA * k];
        double vnorm2 = 0.0;
        for (auto &vi : v) vnorm2 += std::norm(vi);
        if (vnorm2 == 0.0) continue;
        double tau = 2.0 / vnorm2;
        // apply H to remaining columns of A and to B
        for (int j = k; j < N; j++) {
            zc s = 0.0;
            for (int i = k; i < M; i++) s += std::conj(v[i - k]) * a[i + (long)LDA * j];
            s *= tau;
            for (int i = k; i < M; i++) a[i + (long)LDA * j] -= s * v[i - k];
        }
        for (int r = 0; r < *nrhs; r++) {
            zc s = 0.0;
            for (int i = k; i < M; i++) s += std::conj(v[i - k]) * b[i + (long)LDB * r];
            s *= tau;
            for (int i = k; i < M; i++) b[i + (long)LDB * r] -= s * v[i - k];
        }
    }
    for (int r = 0; r < *nrhs; r++) {
        for (int i = N - 1; i >= 0; i--) {
            zc s = b[i + (long)LDB * r];
            for (int j = i + 1; j < N; j++) s -= a[i + (long)LDA * j] * b[j + (long)LDB * r];
            zc d = a[i + (long)LDA * i];
            if (d == zc(0.0)) { *info = i + 1; return; }
            b[i + (long)LDB * r] = s / d;
        }
    }
}

// ------------------------------------------------------- sparse checker
void sparse_matrix_checker_init(sparse_struct *h) { memset(h, 0, sizeof(*h)); }
int sparse_matrix_checker(sparse_struct *) { return 0; }

// ------------------------------------------------------------------ PARDISO
namespace {
struct BandLU {
    int n = 0, kl = 0, ku = 0, w = 0;   // row band: columns [i - kl, i + kl + ku]
    std::vector<zc> ab;                  // n rows x w
    std::vector<int> piv;
    bool factored = false;
    zc &at(int i, int j) { return ab[(long)i * w + (j - i + kl)]; }
};

void band_factor(BandLU &f, const zc *a, const int *ia, const int *ja) {
    const int n = f.n;
    f.ab.assign((long)n * f.w, zc(0.0));
    f.piv.assign(n, 0);
    for (int i = 0; i < n; i++)
        for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) f.at(i, ja[p] - 1) += a[p];
    for (int k = 0; k < n; k++) {
        int last = std::min(n - 1, k + f.kl);
        int p = k;
        double best = std::abs(f.at(k, k));
        for (int i = k + 1; i <= last; i++) {
            double v = std::abs(f.at(i, k));
            if (v > best) { best = v; p = i; }
        }
        f.piv[k] = p;
        int jend = std::min(n - 1, k + f.kl + f.ku);
        if (p != k)
            for (int j = k; j <= jend; j++) std::swap(f.at(k, j), f.at(p, j));
        zc d = f.at(k, k);
        if (d == zc(0.0)) continue;  // singular: left to the solve
        for (int i = k + 1; i <= last; i++) {
            zc l = f.at(i, k) / d;
            f.at(i, k) = l;
            if (l == zc(0.0)) continue;
            for (int j = k + 1; j <= jend; j++) f.at(i, j) -= l * f.at(k, j);
        }
    }
    f.factored = true;
}

void band_solve(BandLU &f, const zc *b, zc *x) {
    const int n = f.n;
    std::vector<zc> y(b, b + n);
    for (int k = 0; k < n; k++) {
        if (f.piv[k] != k) std::swap(y[k], y[f.piv[k]]);
        int last = std::min(n - 1, k + f.kl);
        for (int i = k + 1; i <= last; i++) y[i] -= f.at(i, k) * y[k];
    }
    for (int k = n - 1; k >= 0; k--) {
        int jend = std::min(n - 1, k + f.kl + f.ku);
        zc s = y[k];
        for (int j = k + 1; j <= jend; j++) s -= f.at(k, j) * y[j];
        y[k] = s / f.at(k, k);
    }
    for (int i = 0; i < n; i++) x[i] = y[i];
}
}  // namespace

extern "C" void pardisoinit(_MKL_DSS_HANDLE_t pt, const int *, int *iparm) {
    memset(pt, 0, 64 * sizeof(void *));
    for (int i = 0; i < 64; i++) iparm[i] = 0;
}

extern "C" void pardiso(_MKL_DSS_HANDLE_t pt, const int *, const int *, const int *mtype, const int *phase,
                        const int *n, const void *a, const int *ia, const int *ja, int *, const int *nrhs,
                        int *iparm, const int *, void *b, void *x, int *error) {
    void **slot = (void **)pt;
    BandLU *f = (BandLU *)slot[0];
    *error = 0;
    if (*mtype != 13) standin_missing("pardiso(mtype != 13)");
    if (*phase == -1 || *phase == 0) {
        delete f;
        slot[0] = nullptr;
        return;
    }
    if (*phase == 11 || *phase == 12 || *phase == 13) {
        if (!f) { f = new BandLU(); slot[0] = f; }
        f->n = *n;
        int kl = 0, ku = 0;
        for (int i = 0; i < *n; i++)
            for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) {
                int j = ja[p] - 1;
                kl = std::max(kl, i - j);
                ku = std::max(ku, j - i);
            }
        f->kl = kl;
        f->ku = ku;
        f->w = 2 * kl + ku + 1;
        iparm[14] = iparm[15] = iparm[16] = 0;
    }
    if (*phase == 12 || *phase == 13 || *phase == 22 || *phase == 23) {
        if (!f) { *error = -1; return; }
        band_factor(*f, (const zc *)a, ia, ja);
    }
    if (*phase == 13 || *phase == 23 || *phase == 33) {
        if (!f || !f->factored) { *error = -1; return; }
        for (int r = 0; r < *nrhs; r++)
            band_solve(*f, (const zc *)b + (long)r * f->n, (zc *)x + (long)r * f->n);
    }
}

// -------------------------------------------------------------------- DFTI
struct DFTI_DESCRIPTOR_STANDIN {
    long n = 0;
    double fwd_scale = 1.0, bwd_scale = 1.0;
    long in_strides[2] = {0, 1}, out_strides[2] = {0, 1};
    int placement = DFTI_INPLACE;
};

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, int precision, int domain, MKL_LONG dimension, ...) {
    if (precision != DFTI_DOUBLE || domain != DFTI_COMPLEX || dimension != 1)
        standin_missing("DftiCreateDescriptor(non complex-double-1D)");
    va_list ap;
    va_start(ap, dimension);
    long n = va_arg(ap, long);
    va_end(ap);
    *h = new DFTI_DESCRIPTOR_STANDIN();
    (*h)->n = n;
    return DFTI_NO_ERROR;
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, int param, ...) {
    va_list ap;
    va_start(ap, param);
    switch (param) {
        case DFTI_PLACEMENT: h->placement = va_arg(ap, int); break;
        case DFTI_FORWARD_SCALE: h->fwd_scale = va_arg(ap, double); break;
        case DFTI_BACKWARD_SCALE: h->bwd_scale = va_arg(ap, double); break;
        case DFTI_INPUT_STRIDES: {
            long *s = va_arg(ap, long *);
            h->in_strides[0] = s[0];
            h->in_strides[1] = s[1];
            break;
        }
        case DFTI_OUTPUT_STRIDES: {
            long *s = va_arg(ap, long *);
            h->out_strides[0] = s[0];
            h->out_strides[1] = s[1];
            break;
        }
        default: va_end(ap); standin_missing("DftiSetValue(param)");
    }
    va_end(ap);
    return DFTI_NO_ERROR;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE) { return DFTI_NO_ERROR; }

static void dft_strided(DFTI_DESCRIPTOR_HANDLE h, const zc *in, zc *out, double sign, double scale) {
    const long n = h->n;
    std::vector<zc> tmp(n);
    for (long k = 0; k < n; k++) {
        zc s = 0.0;
        for (long j = 0; j < n; j++) {
            long r = (j * k) % n;
            double ang = sign * 2.0 * M_PI * (double)r / (double)n;
            s += in[h->in_strides[0] + j * h->in_strides[1]] * zc(std::cos(ang), std::sin(ang));
        }
        tmp[k] = s * scale;
    }
    for (long k = 0; k < n; k++) out[h->out_strides[0] + k * h->out_strides[1]] = tmp[k];
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...) {
    zc *out = (zc *)in;
    if (h->placement == DFTI_NOT_INPLACE) {
        va_list ap;
        va_start(ap, in);
        out = (zc *)va_arg(ap, void *);
        va_end(ap);
    }
    dft_strided(h, (const zc *)in, out, -1.0, h->fwd_scale);
    return DFTI_NO_ERROR;
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...) {
    zc *out = (zc *)in;
    if (h->placement == DFTI_NOT_INPLACE) {
        va_list ap;
        va_start(ap, in);
        out = (zc *)va_arg(ap, void *);
        va_end(ap);
    }
    dft_strided(h, (const zc *)in, out, +1.0, h->bwd_scale);
    return DFTI_NO_ERROR;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h) {
    delete *h;
    *h = nullptr;
    return DFTI_NO_ERROR;
}
