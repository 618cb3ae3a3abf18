// setup.cpp -- host (FP64) set-up of a solve: PML coefficient tables, the
// z-averaged medium of the preconditioner, dL (mode R), the kz table, the FFT
// plan, device uploads and the block LU factor.  Replaces the set-up block of
// FGMRES (Source/FGMRES.cpp:72-298).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "helm3d_internal.h"

namespace h3d {

static const double kPi = 3.141592653589793238462643;

// d(x) = 1000 x^2 (Source/functions.cpp:893-906)
static double d_pml(double x) { return 1000.0 * x * x; }

// alpha(size_m, double) (Source/functions.cpp:1839-1878): -i w / (d(x) - i w)
// inside the PML, 1 outside; the left test i < pml includes i = pml - 1/2.
static zc alpha(int n, int pml, double i, double omega) {
    if (pml == 0) return zc(1.0, 0.0);
    const double h = 1.0 / pml;
    if (i < pml || i >= (n - pml)) {
        double x;
        if (i < pml) x = 1.0 - i * h;
        else x = 1.0 + (i - n + 1) * h;
        return zc(0.0, -omega) / zc(d_pml(x), -omega);
    }
    return zc(1.0, 0.0);
}

// cm[i] = alpha(i) alpha(i-1/2)/h^2, cp[i] = alpha(i) alpha(i+1/2)/h^2
// (beta2D_pml cases -1/+1, -2/+2: Source/functions.cpp:2385-2399)
static void pml_table(int n, int pml, double h, double omega, std::vector<zc> &cm, std::vector<zc> &cp) {
    cm.resize(n);
    cp.resize(n);
    const double h2 = h * h;
    for (int i = 0; i < n; i++) {
        const zc a = alpha(n, pml, (double)i, omega);
        cm[i] = a * alpha(n, pml, i - 0.5, omega) / h2;
        cp[i] = a * alpha(n, pml, i + 0.5, omega) / h2;
    }
}

// ------------------------------------------------------------------------
// Eigen-decomposition D = W diag(lam) W^{-1} of the z operator with its PML
// (tridiagonal: sub cm[i+1], diagonal -(cm+cp)[i], super cp[i]).  D is
// upper Hessenberg; its complex Schur form D = Z T Z^H is computed by the
// single-shift QR algorithm with Wilkinson shifts, deflation and bulge
// chasing by complex Givens rotations (Golub & Van Loan, Matrix
// Computations, sec. 7.5); eigenvectors of T by back substitution, W = Z Y;
// W^{-1} by Gaussian elimination with partial pivoting.
static bool schur_hessenberg(int n, std::vector<zc> &H, std::vector<zc> &Z) {
    auto h = [&](int i, int j) -> zc & { return H[(size_t)i * n + j]; };
    auto z = [&](int i, int j) -> zc & { return Z[(size_t)i * n + j]; };
    Z.assign((size_t)n * n, zc(0, 0));
    for (int i = 0; i < n; i++) z(i, i) = 1.0;
    double anorm = 0;
    for (auto &v : H) anorm = std::max(anorm, std::abs(v));
    const double eps = 2.220446049250313e-16;
    int hi = n - 1, iter = 0, total = 0;
    while (hi > 0) {
        int lo = hi;
        while (lo > 0) {
            double sc = std::abs(h(lo - 1, lo - 1)) + std::abs(h(lo, lo));
            if (sc == 0.0) sc = anorm;
            if (std::abs(h(lo, lo - 1)) <= eps * sc) {
                h(lo, lo - 1) = 0.0;
                break;
            }
            lo--;
        }
        if (lo == hi) {
            hi--;
            iter = 0;
            continue;
        }
        if (++total > 100 * n) return false;
        iter++;
        const zc a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
        const zc half = (a - d) * 0.5;
        const zc disc = std::sqrt(half * half + b * c);
        const zc m1 = (a + d) * 0.5 + disc, m2 = (a + d) * 0.5 - disc;
        zc mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
        if (iter % 11 == 10) mu = d + 0.75 * std::abs(h(hi, hi - 1));  // exceptional shift
        zc x = h(lo, lo) - mu, y = h(lo + 1, lo);
        for (int k = lo; k < hi; k++) {
            const double ax = std::abs(x), nrm = std::hypot(ax, std::abs(y));
            double cs;
            zc sn;
            if (nrm == 0.0) {
                cs = 1.0;
                sn = 0.0;
            } else if (ax == 0.0) {
                cs = 0.0;
                sn = 1.0;
            } else {
                cs = ax / nrm;
                sn = (x / ax) * std::conj(y) / nrm;
            }
            for (int j = std::max(lo, k - 1); j < n; j++) {
                const zc t1 = h(k, j), t2 = h(k + 1, j);
                h(k, j) = cs * t1 + sn * t2;
                h(k + 1, j) = -std::conj(sn) * t1 + cs * t2;
            }
            for (int i = 0; i <= std::min(k + 2, hi); i++) {
                const zc t1 = h(i, k), t2 = h(i, k + 1);
                h(i, k) = cs * t1 + std::conj(sn) * t2;
                h(i, k + 1) = -sn * t1 + cs * t2;
            }
            for (int i = 0; i < n; i++) {
                const zc t1 = z(i, k), t2 = z(i, k + 1);
                z(i, k) = cs * t1 + std::conj(sn) * t2;
                z(i, k + 1) = -sn * t1 + cs * t2;
            }
            if (k < hi - 1) {
                x = h(k + 1, k);
                y = h(k + 2, k);
            }
        }
    }
    return true;
}

static bool invert(int n, std::vector<zc> A, std::vector<zc> &Ainv) {
    Ainv.assign((size_t)n * n, zc(0, 0));
    for (int i = 0; i < n; i++) Ainv[(size_t)i * n + i] = 1.0;
    for (int k = 0; k < n; k++) {
        int p = k;
        for (int i = k + 1; i < n; i++)
            if (std::abs(A[(size_t)i * n + k]) > std::abs(A[(size_t)p * n + k])) p = i;
        if (std::abs(A[(size_t)p * n + k]) == 0.0) return false;
        if (p != k)
            for (int j = 0; j < n; j++) {
                std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
                std::swap(Ainv[(size_t)k * n + j], Ainv[(size_t)p * n + j]);
            }
        const zc inv = 1.0 / A[(size_t)k * n + k];
        for (int j = 0; j < n; j++) {
            A[(size_t)k * n + j] *= inv;
            Ainv[(size_t)k * n + j] *= inv;
        }
        for (int i = 0; i < n; i++) {
            if (i == k) continue;
            const zc f = A[(size_t)i * n + k];
            if (f == zc(0, 0)) continue;
            for (int j = 0; j < n; j++) {
                A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
                Ainv[(size_t)i * n + j] -= f * Ainv[(size_t)k * n + j];
            }
        }
    }
    return true;
}

static bool zpml_eigen(const std::vector<zc> &cm, const std::vector<zc> &cp, std::vector<zc> &lam,
                       std::vector<zc> &W, std::vector<zc> &Wi, double *resid) {
    const int n = (int)cm.size();
    std::vector<zc> D((size_t)n * n, zc(0, 0));
    for (int i = 0; i < n; i++) {
        D[(size_t)i * n + i] = -(cm[i] + cp[i]);
        if (i + 1 < n) {
            D[(size_t)i * n + i + 1] = cp[i];
            D[(size_t)(i + 1) * n + i] = cm[i + 1];
        }
    }
    std::vector<zc> T = D, Z;
    if (!schur_hessenberg(n, T, Z)) return false;
    lam.resize(n);
    for (int k = 0; k < n; k++) lam[k] = T[(size_t)k * n + k];
    double tnorm = 0;
    for (auto &v : T) tnorm = std::max(tnorm, std::abs(v));
    const double small = 1e-14 * std::max(tnorm, 1e-300);
    W.assign((size_t)n * n, zc(0, 0));
    std::vector<zc> y(n);
    for (int k = 0; k < n; k++) {
        std::fill(y.begin(), y.end(), zc(0, 0));
        y[k] = 1.0;
        for (int j = k - 1; j >= 0; j--) {
            zc sum = 0.0;
            for (int l = j + 1; l <= k; l++) sum += T[(size_t)j * n + l] * y[l];
            zc den = T[(size_t)j * n + j] - lam[k];
            if (std::abs(den) < small) den = small;
            y[j] = -sum / den;
        }
        double nrm = 0;
        for (int i = 0; i < n; i++) {
            zc v = 0.0;
            for (int l = 0; l <= k; l++) v += Z[(size_t)i * n + l] * y[l];
            W[(size_t)i * n + k] = v;
            nrm += std::norm(v);
        }
        nrm = std::sqrt(nrm);
        for (int i = 0; i < n; i++) W[(size_t)i * n + k] /= nrm;
    }
    if (!invert(n, W, Wi)) return false;
    // residual max_k ||D w_k - lam_k w_k|| / ||D||
    double r = 0, dn = 0;
    for (auto &v : D) dn = std::max(dn, std::abs(v));
    for (int k = 0; k < n; k++)
        for (int i = 0; i < n; i++) {
            zc v = -lam[k] * W[(size_t)i * n + k];
            for (int j = std::max(0, i - 1); j <= std::min(n - 1, i + 1); j++) v += D[(size_t)i * n + j] * W[(size_t)j * n + k];
            r = std::max(r, std::abs(v) / dn);
        }
    *resid = r;
    return r < 1e-8;
}

void build_fft_plan(int n, FftPlan &plan, std::vector<zc> &tables) {
    plan = FftPlan();
    plan.n = n;
    int rem = n;
    std::vector<int> rad;
    while (rem % 8 == 0) { rad.push_back(8); rem /= 8; }
    while (rem % 4 == 0) { rad.push_back(4); rem /= 4; }
    while (rem % 2 == 0) { rad.push_back(2); rem /= 2; }
    for (int p : {3, 5, 7}) while (rem % p == 0) { rad.push_back(p); rem /= p; }
    for (int p = 11; rem > 1; p += 2)
        while (rem % p == 0) { rad.push_back(p); rem /= p; }
    if (rad.empty()) rad.push_back(1);
    plan.npass = (int)rad.size();
    tables.clear();
    int span = 1;
    for (int s = 0; s < plan.npass; s++) {
        const int r = rad[s];
        plan.radix[s] = r;
        plan.span[s] = span;
        plan.twoff[s] = (int)tables.size();
        for (int k = 0; k < span; k++)
            for (int q = 0; q < r; q++) {
                const long e = (long)q * k;
                const long mod = (long)span * r;
                const double ang = -2.0 * kPi * (double)(e % mod) / (double)mod;
                tables.push_back(zc(std::cos(ang), std::sin(ang)));
            }
        plan.dftoff[s] = (int)tables.size();
        for (int t = 0; t < r; t++) {
            const double ang = -2.0 * kPi * (double)t / (double)r;
            tables.push_back(zc(std::cos(ang), std::sin(ang)));
        }
        span *= r;
    }
    plan.twlen = (int)tables.size();
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int set_error(helm3d_ctx *c, int code, const std::string &msg) {
    if (c) c->last_error = msg;
    return code;
}

int cuda_check(helm3d_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return HELM3D_OK;
    // a failed call leaves its error as the thread's last error; clear it
    // (possible for the non-sticky ones, e.g. a failed allocation), so that
    // the next launch check of this or another context does not report it
    cudaGetLastError();
    const int code = (e == cudaErrorMemoryAllocation) ? HELM3D_ERR_OOM : HELM3D_ERR_CUDA;
    return set_error(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

static int dalloc(helm3d_ctx *c, void **p, size_t bytes, const char *what) {
    if (*p) return HELM3D_OK;
    const int rc = cuda_check(c, cudaMalloc(p, bytes), what);
    if (rc == HELM3D_OK) c->bytes += bytes;
    return rc;
}

// upload a complex table in the preconditioner precision
static int upload_c(helm3d_ctx *c, void **dst, const std::vector<zc> &v, const char *what) {
    const size_t esz = c->c64 ? 8 : 16;
    int rc = dalloc(c, dst, v.size() * esz + 16, what);
    if (rc) return rc;
    if (c->c64) {
        std::vector<float> tmp(2 * v.size());
        for (size_t i = 0; i < v.size(); i++) {
            tmp[2 * i] = (float)v[i].real();
            tmp[2 * i + 1] = (float)v[i].imag();
        }
        return cuda_check(c, cudaMemcpy(*dst, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice), what);
    }
    return cuda_check(c, cudaMemcpy(*dst, v.data(), v.size() * 16, cudaMemcpyHostToDevice), what);
}

static int upload_c64(helm3d_ctx *c, double2 **dst, const std::vector<zc> &v, const char *what) {
    int rc = dalloc(c, (void **)dst, v.size() * 16 + 16, what);
    if (rc) return rc;
    return cuda_check(c, cudaMemcpy(*dst, v.data(), v.size() * 16, cudaMemcpyHostToDevice), what);
}

// Everything that depends on the grid and options only: PML tables, the kz
// table or the z eigenbasis, the FFT plan, uploads and allocations.
int ctx_setup_grid(helm3d_ctx *c) {
    const helm3d_grid &g = c->grid;
    const helm3d_opts &o = c->opts;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double w = g.omega;
    pml_table(nx, g.pml_x, g.hx, w, c->cmx, c->cpx);
    pml_table(ny, g.pml_y, g.hy, w, c->cmy, c->cpy);
    pml_table(nz, g.pml_z, g.hz, w, c->cmz, c->cpz);

    // kz table
    const double lz = g.lz > 0 ? g.lz : nz * g.hz;
    c->kz2.assign(nz, 0.0);
    for (int k = 0; k < nz; k++) {
        double v;
        if (o.kz_symbol == HELM3D_KZ_DISCRETE) {
            const double sn = std::sin(kPi * k / nz);
            v = 4.0 / (g.hz * g.hz) * sn * sn;
        } else if (o.kz_symbol == HELM3D_KZ_CONTINUOUS) {
            const int kk = std::min(k, nz - k);
            v = (2.0 * kPi * kk / lz) * (2.0 * kPi * kk / lz);
        } else {
            // Source/FGMRES.cpp:182-190: k < nz/2 - 1 -> k, else nz - k
            const int kk = (k < nz / 2 - 1) ? k : nz - k;
            v = 4.0 * kPi * kPi * (double)kk * (double)kk / (lz * lz);
        }
        c->kz2[k] = v;
    }
    int rc;
    if ((rc = upload_c(c, &c->d_cmx, c->cmx, "cmx")) || (rc = upload_c(c, &c->d_cpx, c->cpx, "cpx")) ||
        (rc = upload_c(c, &c->d_cmy, c->cmy, "cmy")) || (rc = upload_c(c, &c->d_cpy, c->cpy, "cpy")))
        return rc;
    if ((rc = upload_c64(c, &c->d_cmx64, c->cmx, "cmx64")) || (rc = upload_c64(c, &c->d_cpx64, c->cpx, "cpx64")) ||
        (rc = upload_c64(c, &c->d_cmy64, c->cmy, "cmy64")) || (rc = upload_c64(c, &c->d_cpy64, c->cpy, "cpy64")) ||
        (rc = upload_c64(c, &c->d_cmz64, c->cmz, "cmz64")) || (rc = upload_c64(c, &c->d_cpz64, c->cpz, "cpz64")))
        return rc;
    // alpha_x(i) alpha_y(j) and conj(1 / (alpha_x(i) alpha_y(j))): the
    // symmetrizing scale of the 2D systems used by the adjoint sweep
    if (o.mode == HELM3D_MODE_N) {
        std::vector<zc> dxy((size_t)2 * ny * nx);
        for (int j = 0; j < ny; j++) {
            const zc ay = alpha(ny, g.pml_y, (double)j, w);
            for (int i = 0; i < nx; i++) {
                const zc d = alpha(nx, g.pml_x, (double)i, w) * ay;
                dxy[(size_t)j * nx + i] = d;
                dxy[((size_t)ny + j) * nx + i] = std::conj(1.0 / d);
            }
        }
        if ((rc = upload_c(c, &c->d_dxy, dxy, "alpha_x alpha_y"))) return rc;
    }
    // per-mode complex shift added to the 2D diagonal: -kz^2 (FFT) or the
    // eigenvalue lambda_k of the z operator (PML eigenbasis)
    c->zeig = (o.mode == HELM3D_MODE_N && o.z_transform == HELM3D_ZT_PML_EIGEN);
    c->zshift.assign(nz, zc(0, 0));
    if (c->zeig) {
        double resid = 0;
        if (!zpml_eigen(c->cmz, c->cpz, c->zshift, c->zW, c->zWi, &resid))
            return set_error(c, HELM3D_ERR_ARG, "eigen-decomposition of the z operator failed (residual " +
                                                    std::to_string(resid) + ")");
        // conjugate transposes for the adjoint preconditioner Wi^H D^{-H} W^H
        std::vector<zc> wh((size_t)nz * nz), wih((size_t)nz * nz);
        for (int a = 0; a < nz; a++)
            for (int b = 0; b < nz; b++) {
                wh[(size_t)a * nz + b] = std::conj(c->zW[(size_t)b * nz + a]);
                wih[(size_t)a * nz + b] = std::conj(c->zWi[(size_t)b * nz + a]);
            }
        if ((rc = upload_c64(c, &c->d_zW64, c->zW, "z eigenvectors c128")) ||
            (rc = upload_c64(c, &c->d_zWi64, c->zWi, "z eigenvectors inverse c128")) ||
            (rc = upload_c64(c, &c->d_zWH64, wh, "z eigenvectors^H")) ||
            (rc = upload_c64(c, &c->d_zWiH64, wih, "z eigenvectors inverse^H")))
            return rc;
        // complex64 planes: the transforms run on the tensor cores (3xTF32);
        // HELM3D_ZT_TENSOR=0 in the environment keeps the FP64 kernels
        const char *env = std::getenv("HELM3D_ZT_TENSOR");
        c->ztc = c->c64 && ztc_supported(nz) && !(env && env[0] == '0');
        if (c->ztc) {
            const std::vector<zc> *mats[4] = {&c->zWi, &c->zW, &wh, &wih};
            for (int q = 0; q < 4; q++) {
                std::vector<float> b;
                ztc_prepare(*mats[q], nz, b);
                if ((rc = dalloc(c, (void **)&c->d_ztc[q], b.size() * 4, "tensor-core z-transform")) ||
                    (rc = cuda_check(c, cudaMemcpy(c->d_ztc[q], b.data(), b.size() * 4, cudaMemcpyHostToDevice),
                                     "tensor-core z-transform")))
                    return rc;
            }
        }
    } else {
        for (int k = 0; k < nz; k++) c->zshift[k] = -c->kz2[k];
    }
    if ((rc = upload_c(c, &c->d_kz2, c->zshift, "mode shifts"))) return rc;
    // FFT tables
    std::vector<zc> tw;
    build_fft_plan(nz, c->plan, tw);
    if ((rc = upload_c(c, &c->d_tw, tw, "fft tables"))) return rc;
    // medium tables, planes, status, factor storage
    const size_t esz = c->c64 ? 8 : 16;
    if ((rc = dalloc(c, &c->d_base2d, esz * c->plane + 16, "base2d"))) return rc;
    if (o.mode == HELM3D_MODE_N && (rc = dalloc(c, (void **)&c->d_s2, sizeof(double) * c->N, "s2"))) return rc;
    if (o.mode == HELM3D_MODE_R && (rc = dalloc(c, (void **)&c->d_dl, sizeof(double2) * c->N, "dL"))) return rc;
    if ((rc = dalloc(c, &c->d_planes, esz * c->N + 256, "planes"))) return rc;
    c->planes_R = 1;
    if ((rc = dalloc(c, (void **)&c->d_status, 64, "status"))) return rc;
    c->ldg = (nx + 3) & ~3;
    c->Gt_bytes = esz * (size_t)nz * ny * nx * c->ldg;
    if ((rc = dalloc(c, &c->d_Gt, c->Gt_bytes, "block LU factor"))) return rc;
    if ((rc = dalloc(c, (void **)&c->d_gscale, sizeof(float) * (size_t)nz * ny, "block scales"))) return rc;
    if (c->c64 && nx <= 256 && (rc = dalloc(c, &c->d_gpack, gpack_bytes(nx, ny, nz), "packed factor"))) return rc;
    return HELM3D_OK;
}

// The medium-dependent tables.  Mode N: s2 is copied to the device and the
// z-mean of s2 (base2d = omega^2 s0^2 (1 + i beta_prec)) is formed by a kernel,
// which also flags non-finite values (status bit 4).  Mode R: the reference's
// c0 (q1 running mean) and dL are formed on the host in FP64.
int ctx_setup_medium(helm3d_ctx *c, const double *s2, bool s2_on_device) {
    const helm3d_grid &g = c->grid;
    const helm3d_opts &o = c->opts;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double w2 = g.omega * g.omega;
    int rc = cuda_check(c, cudaMemsetAsync(c->d_status, 0, 64, c->stream), "status reset");
    if (rc) return rc;
    if (o.mode == HELM3D_MODE_N) {
        rc = cuda_check(c, cudaMemcpyAsync(c->d_s2, s2, sizeof(double) * c->N,
                                           s2_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream),
                        "s2");
        if (rc) return rc;
        int zlo = g.pml_z, zhi = nz - g.pml_z;
        if (zhi <= zlo) {
            zlo = 0;
            zhi = nz;
        }
        return timed(c, HELM3D_K_KRYLOV, 1, [&] {
            return launch_base2d(c->c64, c->d_s2, nz, c->plane, zlo, zhi, w2, o.beta_prec, c->d_base2d, c->d_status,
                                 c->stream);
        });
    }
    // mode R (host)
    std::vector<double> s2h;
    if (s2_on_device) {
        s2h.resize(c->N);
        rc = cuda_check(c, cudaMemcpy(s2h.data(), s2, sizeof(double) * c->N, cudaMemcpyDeviceToHost), "s2");
        if (rc) return rc;
        s2 = s2h.data();
    }
    for (long q = 0; q < c->N; q++)
        if (!std::isfinite(s2[q])) return set_error(c, HELM3D_ERR_NONFINITE, "medium has NaN/Inf");
    c->base2d.assign((size_t)nx * ny, zc(0, 0));
    // SetSoundSpeed2D (Source/functions.cpp:1686-1738) over the physical x,y
    // range and the non-sponge z range, j outer / i inner; with q1 the
    // accumulator carries over between columns.  Then the edge extension
    // into the x,y PML (Source/functions.cpp:2636-2673).
    const int spg = g.spg_z, nzp = nz - 2 * spg;
    std::vector<double> s0((size_t)nx * ny, 0.0);
    double acc = 0.0;
    for (int j = g.pml_y; j < ny - g.pml_y; j++)
        for (int i = g.pml_x; i < nx - g.pml_x; i++) {
            double col = 0.0;
            for (int k = spg; k < nz - spg; k++) col += s2[((long)k * ny + j) * nx + i];
            acc = o.quirk_q1 ? (acc + col) / nzp : col / nzp;
            const double c0 = std::sqrt(1.0 / acc);
            s0[(size_t)j * nx + i] = 1.0 / (c0 * c0);
        }
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < g.pml_x; i++) s0[(size_t)j * nx + i] = s0[(size_t)j * nx + g.pml_x];
        for (int i = nx - g.pml_x; i < nx; i++) s0[(size_t)j * nx + i] = s0[(size_t)j * nx + nx - g.pml_x - 1];
    }
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < g.pml_y; j++) s0[(size_t)j * nx + i] = s0[(size_t)g.pml_y * nx + i];
        for (int j = ny - g.pml_y; j < ny; j++) s0[(size_t)j * nx + i] = s0[(size_t)(ny - g.pml_y - 1) * nx + i];
    }
    for (size_t q = 0; q < s0.size(); q++)
        c->base2d[q] = w2 * (o.s2_l0 > 0 ? o.s2_l0 : s0[q]) * zc(1.0, o.beta_prec);   // q3
    // dL (Source/functions.cpp:1740-1824)
    std::vector<zc> dl((size_t)c->N, zc(0, 0));
    const long pl = c->plane;
    for (int k = spg; k <= nz - spg && k < nz; k++)
        for (long q = 0; q < pl; q++)
            dl[(size_t)k * pl + q] = w2 * (zc(1.0, o.beta_prec) * s0[q] - s2[(size_t)k * pl + q]);
    const double sigma = 0.3, lzz = g.lz > 0 ? g.lz : nz * g.hz;
    const double z0 = spg * g.hz, zN = (nz - spg) * g.hz, L0 = z0, Ln = lzz - zN;
    for (int k = 0; k < spg; k++) {
        const double zp = k * g.hz;
        const double e = std::exp(-(zp - z0) * (zp - z0) / (L0 * L0) / (sigma * sigma));
        for (long q = 0; q < pl; q++) dl[(size_t)k * pl + q] = dl[(size_t)spg * pl + q] * e;
    }
    for (int k = nz - spg + 1; k < nz; k++) {
        const double zp = k * g.hz;
        const double e = std::exp(-(zp - zN) * (zp - zN) / (Ln * Ln) / (sigma * sigma));
        for (long q = 0; q < pl; q++) dl[(size_t)k * pl + q] = dl[(size_t)(nz - spg) * pl + q] * e;
    }
    if ((rc = upload_c64(c, &c->d_dl, dl, "dL"))) return rc;
    return upload_c(c, &c->d_base2d, c->base2d, "base2d");
}

// The modes skipped by opts.kz_skip_ratio (the reference's SAVE_MEM rule,
// Source/FGMRES.cpp:197-206: kww >= ratio * k2): kww = -Re of the mode's
// shift (kz^2, or -Re lambda_k), k2 = omega^2 s2_l0 when s2_l0 > 0 (mode R
// HOMO: the reference's kk = omega / c_z), else the largest omega^2 s0^2 of
// the 2D medium (Re base2d).  Their slots, list and inverse diagonals (zero in
// mode R) go to the device; the factor and sweep kernels leave those modes.
static int setup_kz_skip(helm3d_ctx *c) {
    const helm3d_opts &o = c->opts;
    const helm3d_grid &g = c->grid;
    const int nz = g.nz;
    c->nskip = 0;
    c->kzslot_h.assign(nz, -1);
    if (!(o.kz_skip_ratio > 0)) return HELM3D_OK;
    int rc;
    double k2 = 0.0;
    if (o.s2_l0 > 0) {
        k2 = g.omega * g.omega * o.s2_l0;
    } else {
        const size_t esz = c->c64 ? 8 : 16;
        std::vector<unsigned char> b(esz * (size_t)c->plane);
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "base2d")) ||
            (rc = cuda_check(c, cudaMemcpy(b.data(), c->d_base2d, b.size(), cudaMemcpyDeviceToHost), "base2d")))
            return rc;
        for (long l = 0; l < c->plane; l++) {
            double re;
            if (c->c64) {
                float f;
                std::memcpy(&f, b.data() + 8 * l, 4);
                re = f;
            } else {
                std::memcpy(&re, b.data() + 16 * l, 8);
            }
            k2 = std::max(k2, re);
        }
    }
    std::vector<int> list;
    for (int k = 0; k < nz; k++)
        if (-c->zshift[k].real() >= o.kz_skip_ratio * k2) {
            c->kzslot_h[k] = (int)list.size();
            list.push_back(k);
        }
    c->nskip = (int)list.size();
    if (c->nskip == 0) return HELM3D_OK;
    const size_t esz = c->c64 ? 8 : 16;
    const size_t inv_bytes = esz * (size_t)c->plane * c->nskip;
    if (inv_bytes > c->kzinv_bytes) {
        if (c->d_kzinv) {
            cudaFree(c->d_kzinv);
            c->bytes -= c->kzinv_bytes;
            c->d_kzinv = nullptr;
        }
        if ((rc = dalloc(c, &c->d_kzinv, inv_bytes, "skipped modes' diagonals"))) return rc;
        c->kzinv_bytes = inv_bytes;
    }
    if ((rc = dalloc(c, (void **)&c->d_kzslot, sizeof(int) * nz, "skipped modes")) ||
        (rc = dalloc(c, (void **)&c->d_kzlist, sizeof(int) * nz, "skipped modes")) ||
        (rc = cuda_check(c, cudaMemcpy(c->d_kzslot, c->kzslot_h.data(), sizeof(int) * nz, cudaMemcpyHostToDevice),
                         "skipped modes")) ||
        (rc = cuda_check(c, cudaMemcpy(c->d_kzlist, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice),
                         "skipped modes")))
        return rc;
    rc = launch_kzinv(c->c64, c->d_kzlist, c->nskip, g.nx, g.ny, c->d_cmx, c->d_cpx, c->d_cmy, c->d_cpy,
                      c->d_base2d, c->d_kz2, o.mode == HELM3D_MODE_R, c->d_kzinv, c->stream);
    if (rc) return set_error(c, rc, "skipped modes' diagonals launch failed");
    if (o.verbose) std::printf("helm3d: %d of %d kz modes skipped (ratio %g, k2 %g)\n", c->nskip, nz,
                               o.kz_skip_ratio, k2);
    return HELM3D_OK;
}

int ctx_factor(helm3d_ctx *c) {
    if (!factor_supported(c->c64, c->grid.nx))
        return set_error(c, HELM3D_ERR_ARG, "nx beyond the supported block size of the factor");
    int rc;
    FactorArgs a;
    a.n = c->grid.nx;
    a.ny = c->grid.ny;
    a.nz = c->grid.nz;
    a.ldg = c->ldg;
    a.Gt = c->d_Gt;
    a.cmx = c->d_cmx;
    a.cpx = c->d_cpx;
    a.cmy = c->d_cmy;
    a.cpy = c->d_cpy;
    a.base2d = c->d_base2d;
    a.kz2 = c->d_kz2;
    a.status = c->d_status;
    if ((rc = setup_kz_skip(c))) return rc;
    a.kzslot = c->nskip > 0 ? c->d_kzslot : nullptr;
    const int nv = factor_variants(c->c64, a.n);
    if (nv > 1) {
        // the launch shapes of this block size, timed once per process; the
        // device status (set-up flags included) is kept across the tuning runs
        char shape[96];
        std::snprintf(shape, sizeof(shape), "%d|%d|%d|%d", c->c64 ? 64 : 128, a.n, a.ny, a.nz);
        int st0 = 0;
        rc = cuda_check(c, cudaMemcpyAsync(&st0, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                        "status");
        if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "status");
        if (rc) return rc;
        c->tv_factor = tune_pick(c, "FACTOR", shape, nv, [&](int v) { return launch_factor(c->c64, a, c->stream, v); });
        rc = cuda_check(c, cudaMemcpyAsync(c->d_status, &st0, sizeof(int), cudaMemcpyHostToDevice, c->stream),
                        "status");
        if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "status");
        if (rc) return rc;
    } else {
        c->tv_factor = 0;
    }
    rc = timed(c, HELM3D_K_FACTOR, 1, [&] { return launch_factor(c->c64, a, c->stream, c->tv_factor); });
    if (rc) return set_error(c, rc, std::string("factor launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    // complex64: the blocks' power-of-two scales for the FP16 sweep
    if (c->c64) {
        rc = timed(c, HELM3D_K_FACTOR, 1,
                   [&] { return launch_gscale(c->d_Gt, a.n, a.ny, a.nz, a.ldg, c->d_gscale, c->stream); });
        if (rc) return set_error(c, rc, "block scales launch failed");
        if (c->d_gpack) {
            rc = timed(c, HELM3D_K_FACTOR, 1, [&] {
                return launch_gpack(c->d_Gt, a.n, a.ny, a.nz, a.ldg, c->d_gscale, c->d_gpack, c->stream);
            });
            if (rc) return set_error(c, rc, "factor packing launch failed");
        }
    }
    int st = 0;
    rc = cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status");
    if (rc) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "factor");
    if (rc) return rc;
    if (st & 16) return set_error(c, HELM3D_ERR_NONFINITE, "medium has NaN/Inf");
    if (st & 1) return set_error(c, HELM3D_ERR_SINGULAR, "zero pivot in the block LU factor");
    if (st & 2) return set_error(c, HELM3D_ERR_CUDA, "factor: a bounded wait expired");
    if (st & 8) return set_error(c, HELM3D_ERR_CUDA, "factor: an index check failed");
    return HELM3D_OK;
}

}  // namespace h3d
