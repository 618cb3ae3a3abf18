// solver.cpp -- the outer Krylov drivers on the device.
//
// FGMRES follows the reference's restarted loop (Source/FGMRES.cpp:464-684)
// with three stated changes: the Arnoldi coefficients are V_i^H w (correct
// Gram-Schmidt, applied twice: CGS2) instead of the conjugate the reference
// computes (:511); the least-squares problem is updated by Givens rotations
// instead of a fresh zgels every step (:552-570); and the true residual and
// the preconditioner are applied once per iteration plus once per cycle
// instead of three times per iteration (:503,579,601).
//   mode N: flexible, right preconditioned: z_j = M^{-1} v_j, w = A z_j,
//           x = x0 + Z y.
//   mode R: GMRES on K = I - dL L0^{-1} (the preconditioner is inside the
//           operator), x = x0 + V y, u = L0^{-1} x.
// BiCGStab follows BCGSTAB (Source/BcGSTAB.cpp:397-560): right
// preconditioned, iterate kept in u-space, shadow residual 2 r0.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "helm3d_internal.h"

namespace h3d {

#define RC(x)                          \
    do {                               \
        int _rc = (x);                 \
        if (_rc) return _rc;           \
    } while (0)

static Reduce reducer(helm3d_ctx *c) {
    Reduce r;
    r.partials = c->d_partials;
    r.nblocks = c->red_blocks;
    r.cap = c->red_cap;
    return r;
}

int ensure_krylov(helm3d_ctx *c, int m) {
    if (c->m_alloc >= m && c->d_V) return HELM3D_OK;
    auto fre = [&](void *p) { if (p) cudaFree(p); };
    fre(c->d_V);
    fre(c->d_Z);
    fre(c->d_vs);
    fre(c->d_h);
    fre(c->d_partials);
    c->d_V = c->d_Z = nullptr;
    c->d_vs = nullptr;
    c->d_h = nullptr;
    c->d_partials = nullptr;
    const size_t vb = sizeof(double2) * (size_t)c->N;
    RC(cuda_check(c, cudaMalloc((void **)&c->d_V, vb * (m + 1)), "Krylov basis V"));
    if (c->opts.mode == HELM3D_MODE_N) RC(cuda_check(c, cudaMalloc((void **)&c->d_Z, vb * m), "Krylov basis Z"));
    RC(cuda_check(c, cudaMalloc((void **)&c->d_vs, sizeof(double) * (m + 2)), "scales"));
    RC(cuda_check(c, cudaMalloc((void **)&c->d_h, sizeof(double2) * 4 * (m + 2)), "h"));
    c->red_cap = std::max(m + 2, 8);
    c->red_blocks = 2 * device_info().sm_count;
    RC(cuda_check(c, cudaMalloc((void **)&c->d_partials, sizeof(double2) * c->red_cap * c->red_blocks), "partials"));
    c->m_alloc = m;
    c->bytes += vb * (m + 1) + (c->d_Z ? vb * m : 0);
    return HELM3D_OK;
}

static int ensure_vec(helm3d_ctx *c, double2 **p, const char *what) {
    if (*p) return HELM3D_OK;
    RC(cuda_check(c, cudaMalloc((void **)p, sizeof(double2) * (size_t)c->N), what));
    c->bytes += sizeof(double2) * (size_t)c->N;
    return HELM3D_OK;
}

// ---------------------------------------------------------------- operators
static SweepArgs sweep_args(helm3d_ctx *c) {
    SweepArgs s;
    s.n = c->grid.nx;
    s.ny = c->grid.ny;
    s.nz = c->grid.nz;
    s.ldg = c->ldg;
    s.Gt = c->d_Gt;
    s.cmy = c->d_cmy;
    s.cpy = c->d_cpy;
    s.planes = c->d_planes;
    s.nrhs = 1;
    s.rhs_stride = 0;
    s.status = c->d_status;
    return s;
}

// planes = FFT_z(xscale * x); per-kz block sweep in place
static int prec_to_planes(helm3d_ctx *c, const double2 *x, double xscale) {
    RC(timed(c, HELM3D_K_FFT_FWD, 1, [&] {
        if (c->zeig)
            return launch_ztrans_forward(c->c64, x, xscale, c->d_planes, c->grid.nz, c->plane, c->d_zWi64, c->stream);
        return launch_fft_forward(c->c64, x, xscale, c->d_planes, c->grid.nz, c->plane, c->plan, c->d_tw, c->stream);
    }));
    const SweepArgs s = sweep_args(c);
    return timed(c, HELM3D_K_SWEEP, 1, [&] { return launch_sweep(c->c64, s, c->stream); });
}

int apply_prec(helm3d_ctx *c, const double2 *x, double xscale, double2 *y) {
    RC(prec_to_planes(c, x, xscale));
    return timed(c, HELM3D_K_FFT_INV, 1, [&] {
        if (c->zeig) return launch_ztrans_inverse(c->c64, c->d_planes, y, c->grid.nz, c->plane, c->d_zW64, c->stream);
        return launch_fft_inverse(c->c64, c->d_planes, y, c->grid.nz, c->plane, c->plan, c->d_tw, 0, nullptr, 0.0,
                                  nullptr, c->stream);
    });
}

static StencilArgs stencil_args(helm3d_ctx *c, const double2 *x, double xscale, double2 *y, const double2 *f) {
    StencilArgs a;
    a.nx = c->grid.nx;
    a.ny = c->grid.ny;
    a.nz = c->grid.nz;
    a.cmx = c->d_cmx64;
    a.cpx = c->d_cpx64;
    a.cmy = c->d_cmy64;
    a.cpy = c->d_cpy64;
    a.cmz = c->d_cmz64;
    a.cpz = c->d_cpz64;
    a.s2 = c->d_s2;
    a.w2 = c->grid.omega * c->grid.omega;
    a.beta_phys = c->opts.beta_phys;
    a.x = x;
    a.xscale = xscale;
    a.y = y;
    a.f = f;
    return a;
}

int apply_op(helm3d_ctx *c, const double2 *x, double xscale, double2 *y) {
    if (c->opts.mode == HELM3D_MODE_N) {
        const StencilArgs a = stencil_args(c, x, xscale, y, nullptr);
        return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, false, c->stream); });
    }
    // mode R: y = xscale*x - dL * L0^{-1}(xscale*x), dL fused into the inverse FFT
    RC(prec_to_planes(c, x, xscale));
    return timed(c, HELM3D_K_FFT_INV, 1, [&] {
        return launch_fft_inverse(c->c64, c->d_planes, y, c->grid.nz, c->plane, c->plan, c->d_tw, 1, x, xscale,
                                  c->d_dl, c->stream);
    });
}

int apply_op_adjoint(helm3d_ctx *c, const double2 *x, double xscale, double2 *y) {
    if (c->opts.mode != HELM3D_MODE_N) return set_error(c, HELM3D_ERR_ARG, "adjoint operator is mode N only");
    const StencilArgs a = stencil_args(c, x, xscale, y, nullptr);
    return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, true, c->stream); });
}

static int axpby(helm3d_ctx *c, double2 a, const double2 *x, double2 b, double2 *y) {
    return timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_axpby(a, x, b, y, c->N, c->stream); });
}

// r = f - A x
static int residual(helm3d_ctx *c, const double2 *f, const double2 *x, double2 *r, bool adjoint) {
    if (c->opts.mode == HELM3D_MODE_N) {
        const StencilArgs a = stencil_args(c, x, 1.0, r, f);
        return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, adjoint, c->stream); });
    }
    RC(apply_op(c, x, 1.0, r));
    return axpby(c, make_double2(1, 0), f, make_double2(-1, 0), r);
}

// small pinned host mirror of device scalars
struct Pinned {
    double2 *h = nullptr;
    explicit Pinned(size_t n) { cudaMallocHost((void **)&h, sizeof(double2) * n); }
    ~Pinned() { if (h) cudaFreeHost(h); }
};

static int norm2(helm3d_ctx *c, const double2 *x, const int *box, double2 *d_out, double *host_out) {
    int full[6] = {0, c->grid.nx, 0, c->grid.ny, 0, c->grid.nz};
    const Reduce red = reducer(c);
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_norm2_box(x, c->grid.nx, c->grid.ny, c->grid.nz, box ? box : full, red, d_out, c->stream);
    }));
    double2 v;
    RC(cuda_check(c, cudaMemcpyAsync(&v, d_out, sizeof(double2), cudaMemcpyDeviceToHost, c->stream), "norm"));
    RC(cuda_check(c, cudaStreamSynchronize(c->stream), "norm sync"));
    *host_out = v.x;
    return HELM3D_OK;
}

static void phys_box(helm3d_ctx *c, int box[6]) {
    const helm3d_grid &g = c->grid;
    const int zl = std::max(g.spg_z, g.pml_z);
    box[0] = g.pml_x;
    box[1] = g.nx - g.pml_x;
    box[2] = g.pml_y;
    box[3] = g.ny - g.pml_y;
    box[4] = zl;
    box[5] = g.nz - zl;
}

static int check_status(helm3d_ctx *c) {
    int st = 0;
    RC(cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status"));
    RC(cuda_check(c, cudaStreamSynchronize(c->stream), "status sync"));
    if (st & 6) return set_error(c, HELM3D_ERR_CUDA, "a bounded wait expired in a kernel");
    return HELM3D_OK;
}

// --------------------------------------------------------------- FGMRES
int fgmres(helm3d_ctx *c, const double2 *f, double2 *u, bool adjoint, helm3d_stats *st) {
    const helm3d_opts &o = c->opts;
    const bool flexible = (o.mode == HELM3D_MODE_N);
    if (adjoint && !flexible) return set_error(c, HELM3D_ERR_ARG, "adjoint solve is mode N only");
    const int m = std::max(1, o.restart);
    RC(ensure_krylov(c, m));
    RC(ensure_vec(c, &c->d_r, "residual"));
    const long N = c->N;
    const size_t vb = sizeof(double2) * (size_t)N;
    double2 *V = c->d_V, *Z = c->d_Z;
    double2 *d_h1 = c->d_h, *d_h2 = c->d_h + (m + 2), *d_nrm = c->d_h + 2 * (m + 2), *d_y = c->d_h + 3 * (m + 2);
    Pinned hb(3 * (m + 2));
    if (!hb.h) return set_error(c, HELM3D_ERR_OOM, "pinned host buffer");

    cudaEventRecord(c->ev0, c->stream);
    double nf2;
    RC(norm2(c, f, nullptr, d_nrm, &nf2));
    const double nf = std::sqrt(nf2);
    if (!std::isfinite(nf)) return set_error(c, HELM3D_ERR_NONFINITE, "right-hand side has NaN/Inf");
    RC(cuda_check(c, cudaMemsetAsync(u, 0, vb, c->stream), "x0"));
    if (st) st->history_len = 0;
    if (nf == 0.0) {
        if (st) {
            st->iterations = 0;
            st->relres = 0;
            st->relres_phys = 0;
        }
        return HELM3D_OK;
    }
    const double tol = o.tol;
    int it = 0, restarts = 0;
    bool x_zero = true;
    std::vector<zc> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1);
    std::vector<double> vs_h(m + 2);
    int status = HELM3D_OK;
    double relres = 1.0;
    while (true) {
        // r0 = f - A x0 into V_0
        if (x_zero) {
            RC(cuda_check(c, cudaMemcpyAsync(V, f, vb, cudaMemcpyDeviceToDevice, c->stream), "r0"));
        } else {
            RC(residual(c, f, u, V, adjoint));
        }
        double beta2;
        RC(norm2(c, V, nullptr, d_nrm, &beta2));
        const double beta = std::sqrt(beta2);
        relres = beta / nf;
        if (!std::isfinite(beta)) return set_error(c, HELM3D_ERR_NONFINITE, "residual is NaN/Inf");
        if (relres <= tol || it >= o.max_iter) break;
        vs_h[0] = 1.0 / beta;
        RC(cuda_check(c, cudaMemcpyAsync(c->d_vs, vs_h.data(), sizeof(double), cudaMemcpyHostToDevice, c->stream),
                      "vs0"));
        std::fill(H.begin(), H.end(), zc(0, 0));
        std::fill(gv.begin(), gv.end(), zc(0, 0));
        gv[0] = beta;
        int k = 0;
        for (int j = 0; j < m; j++) {
            double2 *w = V + (size_t)(j + 1) * N;
            if (flexible) {
                double2 *z = Z + (size_t)j * N;
                if (adjoint) {
                    // M^H is not yet available: M^{-1} serves as the
                    // (flexible) preconditioner of the adjoint system
                    RC(apply_prec(c, V + (size_t)j * N, vs_h[j], z));
                    RC(apply_op_adjoint(c, z, 1.0, w));
                } else {
                    RC(apply_prec(c, V + (size_t)j * N, vs_h[j], z));
                    RC(apply_op(c, z, 1.0, w));
                }
            } else {
                RC(apply_op(c, V + (size_t)j * N, vs_h[j], w));
            }
            // Classical Gram-Schmidt, repeated only when needed ("twice is
            // enough"): h1 = V^H w with ||w||^2 from the same pass, w -= V h1
            // with ||w||^2 after; a second pass runs when the norm dropped
            // below 1/sqrt(2) of its value.
            const Reduce red = reducer(c);
            RC(timed(c, HELM3D_K_KRYLOV, 2,
                     [&] { return launch_dots(V, N, c->d_vs, j + 1, w, N, red, d_h1, c->stream, true); }));
            RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
                return launch_update(V, N, c->d_vs, j + 1, d_h1, w, N, 1, red, d_nrm, c->stream);
            }));
            RC(cuda_check(c, cudaMemcpyAsync(hb.h, d_h1, sizeof(double2) * 3 * (m + 2), cudaMemcpyDeviceToHost,
                                             c->stream),
                          "h"));
            RC(cuda_check(c, cudaStreamSynchronize(c->stream), "h sync"));
            for (int i = 0; i <= j; i++) H[(size_t)i * m + j] = zc(hb.h[i].x, hb.h[i].y);
            if (hb.h[2 * (m + 2)].x < 0.5 * hb.h[j + 1].x) {
                RC(timed(c, HELM3D_K_KRYLOV, 2,
                         [&] { return launch_dots(V, N, c->d_vs, j + 1, w, N, red, d_h2, c->stream); }));
                RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
                    return launch_update(V, N, c->d_vs, j + 1, d_h2, w, N, 1, red, d_nrm, c->stream);
                }));
                RC(cuda_check(c, cudaMemcpyAsync(hb.h + (m + 2), d_h2, sizeof(double2) * 2 * (m + 2),
                                                 cudaMemcpyDeviceToHost, c->stream),
                              "h2"));
                RC(cuda_check(c, cudaStreamSynchronize(c->stream), "h2 sync"));
                for (int i = 0; i <= j; i++) H[(size_t)i * m + j] += zc(hb.h[(m + 2) + i].x, hb.h[(m + 2) + i].y);
                c->reorth++;
            }
            const double hn = std::sqrt(std::max(0.0, hb.h[2 * (m + 2)].x));
            if (!std::isfinite(hn)) return set_error(c, HELM3D_ERR_NONFINITE, "Arnoldi norm is NaN/Inf");
            H[(size_t)(j + 1) * m + j] = hn;
            // Givens
            for (int i = 0; i < j; i++) {
                const zc a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
                H[(size_t)(i + 1) * m + j] = -std::conj(sn[i]) * a + cs[i] * b;
            }
            {
                const zc a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
                const double den = std::hypot(std::abs(a), std::abs(b));
                if (den == 0.0) {
                    cs[j] = 1.0;
                    sn[j] = 0.0;
                } else if (std::abs(a) == 0.0) {
                    cs[j] = 0.0;
                    sn[j] = 1.0;
                } else {
                    cs[j] = std::abs(a) / den;
                    sn[j] = (a / std::abs(a)) * std::conj(b) / den;
                }
                H[(size_t)j * m + j] = cs[j] * a + sn[j] * b;
                H[(size_t)(j + 1) * m + j] = 0.0;
                gv[j + 1] = -std::conj(sn[j]) * gv[j];
                gv[j] = cs[j] * gv[j];
            }
            it++;
            k = j + 1;
            const double est = std::abs(gv[j + 1]) / nf;
            if (st && st->history && st->history_len < st->history_cap) st->history[st->history_len++] = est;
            if (o.verbose) fprintf(stderr, "helm3d: it %d  est relres %.3e\n", it, est);
            if (hn == 0.0 || est <= tol || it >= o.max_iter) break;
            vs_h[j + 1] = 1.0 / hn;
            RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_set_scale(d_nrm, c->d_vs, j + 1, c->stream); }));
        }
        // y = H^{-1} g (upper triangular k x k), x += basis * y
        std::vector<zc> y(k);
        for (int i = k - 1; i >= 0; i--) {
            zc s = gv[i];
            for (int q = i + 1; q < k; q++) s -= H[(size_t)i * m + q] * y[q];
            y[i] = s / H[(size_t)i * m + i];
        }
        RC(cuda_check(c, cudaMemcpyAsync(d_y, y.data(), sizeof(double2) * k, cudaMemcpyHostToDevice, c->stream),
                      "y"));
        RC(timed(c, HELM3D_K_KRYLOV, 1, [&] {
            return flexible ? launch_combine(Z, N, nullptr, k, d_y, u, N, c->stream)
                            : launch_combine(V, N, c->d_vs, k, d_y, u, N, c->stream);
        }));
        RC(cuda_check(c, cudaStreamSynchronize(c->stream), "combine"));
        x_zero = false;
        restarts++;
        if (it >= o.max_iter) {
            RC(residual(c, f, u, c->d_r, adjoint));
            double r2;
            RC(norm2(c, c->d_r, nullptr, d_nrm, &r2));
            relres = std::sqrt(r2) / nf;
            if (relres > tol) status = HELM3D_ERR_NOT_CONVERGED;
            break;
        }
    }
    // true residual (full and physical domain)
    RC(residual(c, f, u, c->d_r, adjoint));
    double r2, rp2, fp2;
    RC(norm2(c, c->d_r, nullptr, d_nrm, &r2));
    int box[6];
    phys_box(c, box);
    RC(norm2(c, c->d_r, box, d_nrm, &rp2));
    RC(norm2(c, f, box, d_nrm, &fp2));
    relres = std::sqrt(r2) / nf;
    if (!flexible) {
        // u = L0^{-1} w
        RC(ensure_vec(c, &c->d_t, "tmp"));
        RC(cuda_check(c, cudaMemcpyAsync(c->d_t, u, vb, cudaMemcpyDeviceToDevice, c->stream), "w copy"));
        RC(apply_prec(c, c->d_t, 1.0, u));
    }
    cudaEventRecord(c->ev1, c->stream);
    RC(check_status(c));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (st) {
        st->iterations += it;
        st->restarts += restarts;
        st->relres = relres;
        st->relres_phys = std::sqrt(rp2) / nf;   // relative to ||f|| as the reference (:591-592)
        st->ms_solve += ms;
        (void)fp2;
    }
    if (status == HELM3D_OK && relres > tol && o.max_iter > 0 && it >= o.max_iter) status = HELM3D_ERR_NOT_CONVERGED;
    return status;
}

// -------------------------------------------------------------- BiCGStab
// dot <a, b> = sum conj(a) b on the device, returned to the host
static int zdot(helm3d_ctx *c, const double2 *a, const double2 *b, zc *out) {
    const Reduce red = reducer(c);
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] { return launch_dots(a, c->N, nullptr, 1, b, c->N, red, c->d_h, c->stream); }));
    double2 v;
    RC(cuda_check(c, cudaMemcpyAsync(&v, c->d_h, sizeof(double2), cudaMemcpyDeviceToHost, c->stream), "dot"));
    RC(cuda_check(c, cudaStreamSynchronize(c->stream), "dot sync"));
    *out = zc(v.x, v.y);
    return HELM3D_OK;
}

int bicgstab(helm3d_ctx *c, const double2 *f, double2 *u, helm3d_stats *st) {
    const helm3d_opts &o = c->opts;
    RC(ensure_krylov(c, std::max(1, o.restart)));
    const long N = c->N;
    const size_t vb = sizeof(double2) * (size_t)N;
    if (!c->d_bic) {
        RC(cuda_check(c, cudaMalloc((void **)&c->d_bic, vb * 8), "BiCGStab vectors"));
        c->bytes += vb * 8;
    }
    double2 *r = c->d_bic, *p = r + N, *rst = p + N, *Ay = rst + N, *yv = Ay + N, *s = yv + N, *Az = s + N,
            *zv = Az + N;
    cudaEventRecord(c->ev0, c->stream);
    double nf2;
    RC(norm2(c, f, nullptr, c->d_h + 1, &nf2));
    const double nf = std::sqrt(nf2);
    if (!std::isfinite(nf)) return set_error(c, HELM3D_ERR_NONFINITE, "right-hand side has NaN/Inf");
    RC(cuda_check(c, cudaMemsetAsync(u, 0, vb, c->stream), "x0"));
    if (nf == 0.0) return HELM3D_OK;
    // x0 = 0: r0 = f, p0 = r0, r* = 2 r0 (Source/BcGSTAB.cpp:433-437)
    RC(cuda_check(c, cudaMemcpyAsync(r, f, vb, cudaMemcpyDeviceToDevice, c->stream), "r0"));
    RC(cuda_check(c, cudaMemcpyAsync(p, f, vb, cudaMemcpyDeviceToDevice, c->stream), "p0"));
    RC(cuda_check(c, cudaMemsetAsync(rst, 0, vb, c->stream), "rst"));
    RC(axpby(c, make_double2(2, 0), f, make_double2(0, 0), rst));
    int it = 0, status = HELM3D_OK;
    double relres = 1.0;
    const bool modeN = o.mode == HELM3D_MODE_N;
    // right preconditioned operator B = A M^{-1} (mode N) or K (mode R);
    // the u-space update uses M^{-1} p (mode N) or L0^{-1} p (mode R)
    auto opB = [&](const double2 *x, double2 *yout, double2 *pre) -> int {
        RC(apply_prec(c, x, 1.0, pre));
        if (modeN) return apply_op(c, pre, 1.0, yout);
        return timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_sub_dl(x, c->d_dl, pre, yout, N, c->stream); });
    };
    for (it = 0; it < o.max_iter;) {
        RC(opB(p, Ay, yv));
        zc rr, ra;
        RC(zdot(c, rst, r, &rr));
        RC(zdot(c, rst, Ay, &ra));
        if (ra == zc(0, 0)) { status = HELM3D_ERR_BREAKDOWN; break; }
        const zc alpha = rr / ra;
        // s = r - alpha Ay
        RC(cuda_check(c, cudaMemcpyAsync(s, r, vb, cudaMemcpyDeviceToDevice, c->stream), "s"));
        RC(axpby(c, make_double2(-alpha.real(), -alpha.imag()), Ay, make_double2(1, 0), s));
        RC(opB(s, Az, zv));
        zc as, aa;
        RC(zdot(c, Az, s, &as));
        RC(zdot(c, Az, Az, &aa));
        if (aa == zc(0, 0)) { status = HELM3D_ERR_BREAKDOWN; break; }
        const zc om = as / aa;
        // x += alpha y + omega z
        RC(axpby(c, make_double2(alpha.real(), alpha.imag()), yv, make_double2(1, 0), u));
        RC(axpby(c, make_double2(om.real(), om.imag()), zv, make_double2(1, 0), u));
        // r_new = s - omega Az (into r)
        zc rr_old = rr;
        RC(cuda_check(c, cudaMemcpyAsync(r, s, vb, cudaMemcpyDeviceToDevice, c->stream), "r"));
        RC(axpby(c, make_double2(-om.real(), -om.imag()), Az, make_double2(1, 0), r));
        zc rrn;
        RC(zdot(c, rst, r, &rrn));
        if (rr_old == zc(0, 0) || om == zc(0, 0)) { status = HELM3D_ERR_BREAKDOWN; break; }
        const zc beta = (alpha / om) * rrn / rr_old;
        // p = r + beta (p - omega Ay)
        RC(axpby(c, make_double2(-om.real(), -om.imag()), Ay, make_double2(1, 0), p));
        RC(axpby(c, make_double2(1, 0), r, make_double2(beta.real(), beta.imag()), p));

        it++;
        double r2;
        RC(norm2(c, r, nullptr, c->d_h + 1, &r2));
        relres = std::sqrt(r2) / nf;
        if (st && st->history && st->history_len < st->history_cap) st->history[st->history_len++] = relres;
        if (!std::isfinite(relres)) return set_error(c, HELM3D_ERR_NONFINITE, "BiCGStab residual is NaN/Inf");
        if (relres <= o.tol) break;
    }
    // true residual of the u-space system
    RC(ensure_vec(c, &c->d_r, "residual"));
    if (modeN) {
        RC(residual(c, f, u, c->d_r, false));
    } else {
        // A_R u = L0 u - dL u is not formed directly: K(L0 u) = A_R u.  The
        // BiCGStab recursion residual r is reported for mode R.
        RC(cuda_check(c, cudaMemcpyAsync(c->d_r, r, vb, cudaMemcpyDeviceToDevice, c->stream), "r"));
    }
    double r2, rp2;
    RC(norm2(c, c->d_r, nullptr, c->d_h + 1, &r2));
    int box[6];
    phys_box(c, box);
    RC(norm2(c, c->d_r, box, c->d_h + 1, &rp2));
    cudaEventRecord(c->ev1, c->stream);
    RC(check_status(c));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    relres = std::sqrt(r2) / nf;
    if (st) {
        st->iterations += it;
        st->relres = relres;
        st->relres_phys = std::sqrt(rp2) / nf;
        st->ms_solve += ms;
    }
    if (status == HELM3D_OK && relres > o.tol) status = HELM3D_ERR_NOT_CONVERGED;
    return status;
}

}  // namespace h3d
