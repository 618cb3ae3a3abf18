// solver.cpp -- the outer Krylov drivers on the device.
//
// FGMRES follows the reference's restarted loop (Source/FGMRES.cpp:464-684)
// with three stated changes: the Arnoldi coefficients are V_i^H w (correct
// Gram-Schmidt, with a second pass when the first lost more than half of
// ||w||^2) instead of the conjugate the reference computes (:511); the
// least-squares problem is updated by Givens rotations instead of a fresh
// zgels every step (:552-570); and the true residual and the preconditioner
// are applied once per iteration plus once per cycle instead of three times
// per iteration (:503,579,601).
//   mode N: flexible, right preconditioned: z_j = M^{-1} v_j, w = A z_j,
//           x = x0 + Z y.
//   mode R: GMRES on K = I - dL L0^{-1} (the preconditioner is inside the
//           operator), x = x0 + V y, u = L0^{-1} x.
// Several right-hand sides (the reference's loop over sources,
// Source/main.cpp) are iterated in lockstep: one operator / preconditioner
// launch per Arnoldi step serves the whole batch, each right-hand side keeps
// its own basis, Hessenberg matrix and Givens rotations, and a right-hand
// side that has converged stops contributing columns (and leaves the batch
// at the next restart).
// BiCGStab follows BCGSTAB (Source/BcGSTAB.cpp:397-560): right
// preconditioned, iterate kept in u-space, shadow residual 2 r0.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "helm3d_internal.h"

namespace h3d {

#define RC(x)                          \
    do {                               \
        int _rc = (x);                 \
        if (_rc) return _rc;           \
    } while (0)

static const ScaleBatch kNoScale{nullptr, 0};
static VecBatch one(const double2 *p) { return VecBatch{const_cast<double2 *>(p), 0}; }

static Reduce reducer(helm3d_ctx *c) {
    Reduce r;
    r.partials = c->d_partials;
    r.nblocks = c->red_blocks;
    r.cap = c->red_cap;
    r.rmax = c->r_alloc;
    r.update = c->tv_update;
    return r;
}

// small per-right-hand-side device scalars, each region m+2 long:
// h1 | h2 | norms | y | alpha | delta  (DCGS2 dots span h1 and h2)
static int scalars_per_rhs(int m) { return 6 * (m + 2); }

// bytes of the device Arnoldi state for R right-hand sides and restart m
static size_t arn_bytes(int m, int R) {
    return sizeof(double2) * (size_t)R * ((size_t)(m + 1) * m + 2 * m + (m + 1)) +
           sizeof(double) * (size_t)R * (m + 3) + sizeof(int) * ((size_t)4 * R + kArnFlags) + 256;
}

// the state arrays of a batch of B (restart m) carved from c->d_arn:
// doubles first (est, nf, tol, beta), then ints (frozen, k, it, max_iter, flags)
static ArnState arn_state(helm3d_ctx *c, int m, int B) {
    ArnState a;
    const int R = c->r_alloc;
    char *q = (char *)c->d_arn;
    a.H = (double2 *)q;
    q += sizeof(double2) * (size_t)R * (m + 1) * m;
    a.cs = (double2 *)q;
    q += sizeof(double2) * (size_t)R * m;
    a.sn = (double2 *)q;
    q += sizeof(double2) * (size_t)R * m;
    a.g = (double2 *)q;
    q += sizeof(double2) * (size_t)R * (m + 1);
    a.est = (double *)q;
    q += sizeof(double) * (size_t)R * m;
    a.nf = (double *)q;
    a.tol = a.nf + R;
    a.beta = a.tol + R;
    q += sizeof(double) * (size_t)3 * R;
    a.frozen = (int *)q;
    a.k = a.frozen + R;
    a.it = a.k + R;
    a.max_iter = a.it + R;
    a.flags = a.max_iter + R;
    a.m = m;
    a.B = B;
    a.h = c->d_h;
    a.M2 = m + 2;
    a.SH = scalars_per_rhs(m);
    a.vs = c->d_vs;
    return a;
}

static void drop_graphs(helm3d_ctx *c) {
    for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
}

static void free_krylov(helm3d_ctx *c) {
    drop_graphs(c);
    void *bufs[] = {c->d_V, c->d_Z, c->d_vs, c->d_h, c->d_partials, c->d_Fw, c->d_Uw, c->d_arn};
    for (void *p : bufs)
        if (p) cudaFree(p);
    c->d_V = c->d_Z = c->d_h = c->d_partials = c->d_Fw = c->d_Uw = nullptr;
    c->d_arn = nullptr;
    c->d_vs = nullptr;
    c->bytes -= c->kry_bytes;
    c->kry_bytes = 0;
    c->m_alloc = c->r_alloc = 0;
}

int ensure_krylov(helm3d_ctx *c, int m, int R) {
    if (c->d_V && c->m_alloc >= m && c->r_alloc >= R) return HELM3D_OK;
    m = std::max(m, c->m_alloc);
    R = std::max(R, c->r_alloc);
    free_krylov(c);
    const size_t vb = sizeof(double2) * (size_t)c->N;
    size_t total = 0;
    auto get = [&](void **p, size_t bytes, const char *what) {
        total += bytes;
        return cuda_check(c, cudaMalloc(p, bytes), what);
    };
    c->red_cap = std::max(2 * m + 4, 8);
    c->red_blocks = reduce_blocks(0);
    // partials for the largest reduction grid the autotuner may pick
    int red_max = 0;
    for (int v = 0; v < kReduceVariants; v++) red_max = std::max(red_max, reduce_blocks(v));
    int rc;
    if ((rc = get((void **)&c->d_V, vb * (m + 1) * R, "Krylov basis V")) ||
        (c->opts.mode == HELM3D_MODE_N &&
         (rc = get((void **)&c->d_Z, (c->z64 ? sizeof(float2) : sizeof(double2)) * (size_t)c->N * m * R,
                   "Krylov basis Z"))) ||
        (rc = get((void **)&c->d_vs, sizeof(double) * (m + 2) * R, "basis scales")) ||
        (rc = get((void **)&c->d_h, sizeof(double2) * scalars_per_rhs(m) * R, "Krylov scalars")) ||
        (rc = get((void **)&c->d_partials, sizeof(double2) * c->red_cap * red_max * R, "partials")) ||
        (rc = get((void **)&c->d_Fw, vb * R, "packed right-hand sides")) ||
        (rc = get((void **)&c->d_Uw, vb * R, "packed iterates")) ||
        (rc = get(&c->d_arn, arn_bytes(m, R), "Arnoldi state"))) {
        c->kry_bytes = 0;
        free_krylov(c);
        return rc;
    }
    c->m_alloc = m;
    c->r_alloc = R;
    c->kry_bytes = total;
    c->bytes += total;
    return HELM3D_OK;
}

static int ensure_vec(helm3d_ctx *c, double2 **p, const char *what) {
    if (*p) return HELM3D_OK;
    RC(cuda_check(c, cudaMalloc((void **)p, sizeof(double2) * (size_t)c->N), what));
    c->bytes += sizeof(double2) * (size_t)c->N;
    return HELM3D_OK;
}

// spectral planes for R right-hand sides
static int ensure_planes(helm3d_ctx *c, int R) {
    if (c->planes_R >= R && c->d_planes) return HELM3D_OK;
    const size_t esz = c->c64 ? 8 : 16;
    drop_graphs(c);   // captured launches hold the old planes
    if (c->d_planes) {
        RC(cuda_check(c, cudaStreamSynchronize(c->stream), "planes sync"));
        cudaFree(c->d_planes);
        c->bytes -= esz * c->N * c->planes_R + 256;
        c->d_planes = nullptr;
        c->planes_R = 0;
    }
    RC(cuda_check(c, cudaMalloc(&c->d_planes, esz * c->N * R + 256), "planes"));
    c->bytes += esz * c->N * R + 256;
    c->planes_R = R;
    return HELM3D_OK;
}

// ---------------------------------------------------------------- operators
static PlaneLayout layout(helm3d_ctx *c, int R) {
    return PlaneLayout{c->grid.nx, c->grid.ny, c->grid.nz, R, c->plane};
}

static SweepArgs sweep_args(helm3d_ctx *c, int R, bool adjoint) {
    SweepArgs s;
    s.n = c->grid.nx;
    s.ny = c->grid.ny;
    s.nz = c->grid.nz;
    s.ldg = c->ldg;
    s.Gt = c->d_Gt;
    s.cmy = c->d_cmy;
    s.cpy = c->d_cpy;
    s.planes = c->d_planes;
    s.R = R;
    s.dxy = adjoint ? c->d_dxy : nullptr;
    s.status = c->d_status;
    s.gscale = c->d_gscale;
    s.gpack = c->d_gpack;
    if (c->nskip > 0) {
        s.kzslot = c->d_kzslot;
        s.kzlist = c->d_kzlist;
        s.nskip = c->nskip;
        s.kzinv = c->d_kzinv;
    }
    sweep_variant(c->tv_sweep[adjoint ? 1 : 0], s);
    return s;
}

static int check_batch(helm3d_ctx *c, int R) {
    if (R < 1 || R > kMaxBatch) return set_error(c, HELM3D_ERR_ARG, "batch of right-hand sides out of range");
    return HELM3D_OK;
}

// planes = Z-transform(xscale sc_r x_r); per-kz block sweep in place.
// M^{-1} = T^{-1} diag_k(S_k^{-1}) T with T the z-FFT or Wi (eigenbasis);
// M^{-H} = T^H diag_k(S_k^{-H}) T^{-H}: the same FFT pair (F^H = nz F^{-1}),
// or W^H forward and Wi^H inverse.
static int prec_to_planes(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, int R,
                          bool adjoint) {
    RC(check_batch(c, R));
    RC(ensure_planes(c, R));
    const PlaneLayout L = layout(c, R);
    RC(timed(c, HELM3D_K_FFT_FWD, 1, [&] {
        if (c->ztc)
            return launch_ztc_forward(x, xscale, sc, c->d_planes, L, c->d_ztc[adjoint ? 2 : 0], c->d_status,
                                      c->stream);
        if (c->zeig)
            return launch_ztrans_forward(c->c64, x, xscale, sc, c->d_planes, L, adjoint ? c->d_zWH64 : c->d_zWi64,
                                         c->stream);
        return launch_fft_forward(c->c64, x, xscale, sc, c->d_planes, L, c->plan, c->d_tw, c->stream);
    }));
    const SweepArgs s = sweep_args(c, R, adjoint);
    return timed(c, HELM3D_K_SWEEP, 1, [&] { return launch_sweep(c->c64, s, c->stream); });
}

static int prec_common(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y,
                       int R, bool adjoint) {
    RC(prec_to_planes(c, x, xscale, sc, R, adjoint));
    const PlaneLayout L = layout(c, R);
    return timed(c, HELM3D_K_FFT_INV, 1, [&] {
        if (c->ztc) return launch_ztc_inverse(c->d_planes, L, y, c->d_ztc[adjoint ? 3 : 1], c->d_status, c->stream);
        if (c->zeig)
            return launch_ztrans_inverse(c->c64, c->d_planes, L, y, adjoint ? c->d_zWiH64 : c->d_zW64, c->stream);
        return launch_fft_inverse(c->c64, c->d_planes, L, y, c->plan, c->d_tw, 0, VecBatch{nullptr, 0}, 0.0,
                                  kNoScale, nullptr, c->stream);
    });
}

int apply_prec(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y, int R) {
    return prec_common(c, x, xscale, sc, y, R, false);
}

int apply_prec_adjoint(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y,
                       int R) {
    if (c->opts.mode != HELM3D_MODE_N || !c->d_dxy)
        return set_error(c, HELM3D_ERR_ARG, "adjoint preconditioner is mode N only");
    return prec_common(c, x, xscale, sc, y, R, true);
}

static StencilArgs stencil_args(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc,
                                const VecBatch &y, const VecBatch &f, int R) {
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
    a.sc = sc;
    a.y = y;
    a.f = f;
    a.R = R;
    a.zchunk = stencil_zchunk(c->tv_stencil);
    a.src_fast = stencil_src_fast(c->tv_stencil);
    a.smem = stencil_smem(c->tv_stencil);
    return a;
}

int apply_op(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y, int R) {
    RC(check_batch(c, R));
    if (c->opts.mode == HELM3D_MODE_N) {
        const StencilArgs a = stencil_args(c, x, xscale, sc, y, VecBatch{nullptr, 0}, R);
        return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, false, c->stream); });
    }
    // mode R: y = s x - dL * L0^{-1}(s x), dL fused into the inverse FFT
    RC(prec_to_planes(c, x, xscale, sc, R, false));
    const PlaneLayout L = layout(c, R);
    return timed(c, HELM3D_K_FFT_INV, 1, [&] {
        return launch_fft_inverse(c->c64, c->d_planes, L, y, c->plan, c->d_tw, 1, x, xscale, sc, c->d_dl,
                                  c->stream);
    });
}

int apply_op_adjoint(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y,
                     int R) {
    RC(check_batch(c, R));
    if (c->opts.mode != HELM3D_MODE_N) return set_error(c, HELM3D_ERR_ARG, "adjoint operator is mode N only");
    const StencilArgs a = stencil_args(c, x, xscale, sc, y, VecBatch{nullptr, 0}, R);
    return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, true, c->stream); });
}

static int axpby(helm3d_ctx *c, double2 a, const VecBatch &x, double2 b, const VecBatch &y, int R) {
    return timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_axpby(a, x, b, y, c->N, R, c->stream); });
}

// r_r = f_r - A x_r
static int residual(helm3d_ctx *c, const VecBatch &f, const VecBatch &x, const VecBatch &r, int R, bool adjoint) {
    if (c->opts.mode == HELM3D_MODE_N) {
        const StencilArgs a = stencil_args(c, x, 1.0, kNoScale, r, f, R);
        return timed(c, HELM3D_K_STENCIL, 1, [&] { return launch_stencil(a, adjoint, c->stream); });
    }
    RC(apply_op(c, x, 1.0, kNoScale, r, R));
    return axpby(c, make_double2(1, 0), f, make_double2(-1, 0), r, R);
}

static int fetch(helm3d_ctx *c, const double2 *d, size_t n, double2 *h, const char *what) {
    RC(cuda_check(c, cudaMemcpyAsync(h, d, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream), what));
    return cuda_check(c, cudaStreamSynchronize(c->stream), what);
}

static void full_box(helm3d_ctx *c, int box[6]) {
    box[0] = 0;
    box[1] = c->grid.nx;
    box[2] = 0;
    box[3] = c->grid.ny;
    box[4] = 0;
    box[5] = c->grid.nz;
}

// the physical domain: the grid without its PML (and mode R's sponge) layers
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

// ||x_r||^2 into out[r * sOut].x (full grid) and, with phys, out[r * sOut + 1].x
// (physical domain); no host synchronization
static int norms(helm3d_ctx *c, const VecBatch &x, int R, bool phys, double2 *out, long sOut) {
    const Reduce red = reducer(c);
    int box[6];
    full_box(c, box);
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_norm2_box(x, R, c->grid.nx, c->grid.ny, c->grid.nz, box, red, out, sOut, c->stream);
    }));
    if (!phys) return HELM3D_OK;
    phys_box(c, box);
    return timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_norm2_box(x, R, c->grid.nx, c->grid.ny, c->grid.nz, box, red, out + 1, sOut, c->stream);
    });
}

int check_status(helm3d_ctx *c) {
    int st = 0;
    RC(cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status"));
    RC(cuda_check(c, cudaStreamSynchronize(c->stream), "status sync"));
    if (st & 6) return set_error(c, HELM3D_ERR_CUDA, "a bounded wait expired in a kernel");
    if (st & 8) return set_error(c, HELM3D_ERR_CUDA, "an index check failed in a kernel");
    return HELM3D_OK;
}

// complex Givens rotation zeroing b in (a, b)
static void givens(zc a, zc b, zc &cs, zc &sn) {
    const double den = std::hypot(std::abs(a), std::abs(b));
    if (den == 0.0) {
        cs = 1.0;
        sn = 0.0;
    } else if (std::abs(a) == 0.0) {
        cs = 0.0;
        sn = 1.0;
    } else {
        cs = std::abs(a) / den;
        sn = (a / std::abs(a)) * std::conj(b) / den;
    }
}

// Mode N (flexible) uses DCGS2, the low-synchronization Gram-Schmidt with
// delayed reorthogonalization, unless HELM3D_GS=cgs2 selects classical
// Gram-Schmidt with the conditional second pass.
static bool lowsync(const helm3d_ctx *c) { return c->opts.mode == HELM3D_MODE_N && c->gs_lowsync; }

// The Z basis from vector offset off (in elements), leading dimension ld:
// complex64 when the context keeps it so (z64), else complex128.
static VecBatch zbasis(const helm3d_ctx *c, long off, long ld) {
    if (c->z64) return VecBatch{reinterpret_cast<double2 *>(reinterpret_cast<float2 *>(c->d_Z) + off), ld, true};
    return VecBatch{c->d_Z + off, ld};
}

// ------------------------------------------------ restart cycle as a graph
// One Arnoldi step j of a batch of B, kernels only: the operator and
// preconditioner applications, classical Gram-Schmidt with its norms, the
// predicated second pass and the device Givens update, which arms (or not)
// the conditional node of step j + 1.
static int arnoldi_step(helm3d_ctx *c, int m, int B, int j, bool adjoint, const ArnState &a, bool has_next,
                        cudaGraphConditionalHandle next) {
    const long N = c->N;
    const long ldV = (long)(m + 1) * N, ldZ = (long)m * N;
    const int M2 = m + 2, SH = scalars_per_rhs(m);
    double2 *V = c->d_V, *Hd = c->d_h;
    double2 *d_h1 = Hd, *d_h2 = Hd + M2, *d_nrm = Hd + 2 * M2;
    const Reduce red = reducer(c);
    const VecBatch Vall{V, ldV}, Vj{V + (size_t)j * N, ldV}, w{V + (size_t)(j + 1) * N, ldV};
    const ScaleBatch vsb{c->d_vs, M2}, vsj{c->d_vs + j, M2};
    if (c->opts.mode == HELM3D_MODE_N) {
        const VecBatch zj = zbasis(c, (long)j * N, ldZ);
        if (adjoint) {
            RC(apply_prec_adjoint(c, Vj, 1.0, vsj, zj, B));
            RC(apply_op_adjoint(c, zj, 1.0, kNoScale, w, B));
        } else {
            RC(apply_prec(c, Vj, 1.0, vsj, zj, B));
            RC(apply_op(c, zj, 1.0, kNoScale, w, B));
        }
    } else {
        RC(apply_op(c, Vj, 1.0, vsj, w, B));
    }
    if (lowsync(c)) {
        // DCGS2: one reduction (w against V_0..V_j, the lagged second
        // projection of V_j), the bookkeeping, one update pass
        RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
            return launch_dots2(Vall, N, vsb, j, w, N, B, red, d_h1, SH, c->stream, nullptr, a.frozen);
        }));
        RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_lagged(a, j, c->stream); }));
        RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
            return launch_update2(Vall, N, j, Hd + 4 * M2, SH, M2, w, N, B, red, d_nrm, SH, c->stream, nullptr,
                                  a.frozen);
        }));
        return timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_post(a, j, has_next, next, c->stream); });
    }
    RC(timed(c, HELM3D_K_KRYLOV, 2,
             [&] { return launch_dots(Vall, N, vsb, j + 1, w, N, B, red, d_h1, SH, c->stream, true); }));
    RC(timed(c, HELM3D_K_KRYLOV, 2,
             [&] { return launch_update(Vall, N, vsb, j + 1, d_h1, SH, w, N, B, 1, red, d_nrm, SH, c->stream); }));
    RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_reorth_check(a, j, c->stream); }));
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_dots(Vall, N, vsb, j + 1, w, N, B, red, d_h2, SH, c->stream, false, a.flags);
    }));
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_update(Vall, N, vsb, j + 1, d_h2, SH, w, N, B, 1, red, d_nrm, SH, c->stream, a.flags);
    }));
    return timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_givens(a, j, has_next, next, c->stream); });
}

// end of a cycle: y = R^{-1} g on the device, x += Z y (mode R: V y)
static int cycle_tail(helm3d_ctx *c, int m, int B, const ArnState &a) {
    const long N = c->N;
    const long ldV = (long)(m + 1) * N, ldZ = (long)m * N;
    const int M2 = m + 2, SH = scalars_per_rhs(m);
    double2 *d_y = c->d_h + 3 * M2;
    if (lowsync(c)) {
        // the open column of the last step (skipped when every right-hand
        // side stopped inside the cycle)
        RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
            return launch_dots_tail(VecBatch{c->d_V, ldV}, N, ScaleBatch{c->d_vs, M2}, m, a.flags + 4, N, B,
                                    reducer(c), c->d_h, SH, c->stream, a.flags + 5, a.frozen);
        }));
        RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_lagged_final(a, c->stream); }));
    }
    RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_backsub(a, c->stream); }));
    return timed(c, HELM3D_K_KRYLOV, 1, [&] {
        return c->opts.mode == HELM3D_MODE_N
                   ? launch_combine(zbasis(c, 0, ldZ), N, kNoScale, m, d_y, SH, VecBatch{c->d_Uw, N}, N, B,
                                    c->stream, a.flags + 2)
                   : launch_combine(VecBatch{c->d_V, ldV}, N, ScaleBatch{c->d_vs, M2}, m, d_y, SH,
                                    VecBatch{c->d_Uw, N}, N, B, c->stream, a.flags + 2);
    });
}

// Adds the restart cycle of context c (a batch of B) to graph G as one more
// chain of root nodes: m conditional (IF) nodes in sequence, the body of
// node j holding step j, then the tail.  Step 0 always runs; the bookkeeping
// kernel of step j sets the condition of step j + 1.  The chain's kernels
// are recorded on c's launch count per step (per_step) and at the tail.
// Every allocation happens before the captures.
static bool add_cycle(cudaGraph_t G, helm3d_ctx *c, int m, int B, bool adjoint, long long &per_step,
                      long long &tail) {
    if (ensure_planes(c, B)) return false;
    const ArnState a = arn_state(c, m, B);
    cudaStream_t cap = nullptr;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaStream_t saved = c->stream;
    const bool prof = c->prof;
    const long long launches0 = c->launches;
    c->stream = cap;
    c->prof = false;
    bool ok = true;
    std::vector<cudaGraphConditionalHandle> hs(m);
    for (int j = 0; ok && j < m; j++)
        ok = cudaGraphConditionalHandleCreate(&hs[j], G, j == 0 ? 1u : 0u, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNode_t prev = nullptr;
    for (int j = 0; ok && j < m; j++) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hs[j];
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        ok = cudaGraphAddNode(&node, G, prev ? &prev : nullptr, prev ? 1 : 0, &cp) == cudaSuccess;
        if (!ok) break;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
             cudaSuccess;
        if (!ok) break;
        const long long l0 = c->launches;
        const int rc = arnoldi_step(c, m, B, j, adjoint, a, j + 1 < m, j + 1 < m ? hs[j + 1] : 0);
        cudaGraph_t out = nullptr;
        ok = cudaStreamEndCapture(cap, &out) == cudaSuccess && rc == HELM3D_OK;
        per_step = c->launches - l0;
        prev = node;
    }
    if (ok) {
        ok = cudaStreamBeginCaptureToGraph(cap, G, &prev, nullptr, 1, cudaStreamCaptureModeRelaxed) == cudaSuccess;
        if (ok) {
            const long long l0 = c->launches;
            const int rc = cycle_tail(c, m, B, a);
            cudaGraph_t out = nullptr;
            ok = cudaStreamEndCapture(cap, &out) == cudaSuccess && rc == HELM3D_OK;
            tail = c->launches - l0;
        }
    }
    cudaStreamDestroy(cap);
    c->stream = saved;
    c->prof = prof;
    c->launches = launches0;
    if (!ok) cudaGetLastError();
    return ok;
}

// The cycle graph of one context for a batch of B, built once per
// (B, adjoint) and kept until the workspace moves.  Returns the index in
// c->graphs, or -1 when graphs are unavailable (the caller then launches the
// steps itself).
static int cycle_graph(helm3d_ctx *c, int m, int B, bool adjoint) {
    for (size_t q = 0; q < c->graphs.size(); q++)
        if (c->graphs[q].B == B && c->graphs[q].adjoint == adjoint) return (int)q;
    cudaGraph_t G = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long per_step = 0, tail = 0;
    bool ok = cudaGraphCreate(&G, 0) == cudaSuccess && add_cycle(G, c, m, B, adjoint, per_step, tail);
    if (ok) ok = cudaGraphInstantiate(&exec, G, 0) == cudaSuccess;
    if (G) cudaGraphDestroy(G);
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return -1;
    }
    c->graphs.push_back({B, adjoint, exec, per_step, tail});
    return (int)c->graphs.size() - 1;
}

// ------------------------------------------------------------- autotuning
int tune_solve(helm3d_ctx *c, int R, bool adjoint) {
    const bool any_forced = std::getenv("HELM3D_FORCE_SWEEP") || std::getenv("HELM3D_FORCE_STENCIL") ||
                            std::getenv("HELM3D_FORCE_REDUCE") || std::getenv("HELM3D_FORCE_UPDATE");
    if (!tune_enabled() && !any_forced) {
        c->tv_sweep[0] = c->tv_sweep[1] = 0;
        c->tv_stencil = 0;
        c->tv_update = 0;
        c->red_blocks = reduce_blocks(0);
        return HELM3D_OK;
    }
    const helm3d_grid &g = c->grid;
    const int m = c->m_alloc;
    const long N = c->N, ldV = (long)(m + 1) * N;
    char shape[128];
    // the sweep, in place on zeroed planes of R right-hand sides
    RC(cuda_check(c, cudaMemsetAsync(c->d_planes, 0, (c->c64 ? 8 : 16) * (size_t)N * R, c->stream), "tune planes"));
    const int adj = adjoint ? 1 : 0;
    std::snprintf(shape, sizeof(shape), "%d|%d|%d|%d|%d|%d", c->c64 ? 64 : 128, g.nx, g.ny, g.nz, R, adj);
    const SweepArgs s0 = sweep_args(c, R, adjoint);
    c->tv_sweep[adj] = tune_pick(c, "SWEEP", shape, kSweepVariants, [&](int v) {
        SweepArgs t = s0;
        sweep_variant(v, t);
        return launch_sweep(c->c64, t, c->stream);
    });
    if (c->opts.mode == HELM3D_MODE_N) {
        // the stencil from Z_0 (its FGMRES input: complex64 when the
        // context keeps Z so) into V_1 of every right-hand side
        std::snprintf(shape, sizeof(shape), "%d|%d|%d|%d|%d", g.nx, g.ny, g.nz, R, c->z64 ? 64 : 128);
        StencilArgs a0 = stencil_args(c, zbasis(c, 0, (long)m * N), 1.0, kNoScale, VecBatch{c->d_V + N, ldV},
                                      VecBatch{nullptr, 0}, R);
        c->tv_stencil = tune_pick(c, "STENCIL", shape, kStencilVariants, [&](int v) {
            StencilArgs t = a0;
            t.zchunk = stencil_zchunk(v);
            t.src_fast = stencil_src_fast(v);
            t.smem = stencil_smem(v);
            return launch_stencil(t, adjoint, c->stream);
        });
    }
    // the Gram-Schmidt reduction at mid-cycle depth (read-only on V)
    const int j = std::min(m - 1, std::max(0, m / 2));
    std::snprintf(shape, sizeof(shape), "%ld|%d|%d", N, R, j);
    const int rv = tune_pick(c, "REDUCE", shape, kReduceVariants, [&](int v) {
        Reduce red = reducer(c);
        red.nblocks = reduce_blocks(v);
        return launch_dots2(VecBatch{c->d_V, ldV}, N, ScaleBatch{c->d_vs, m + 2}, j,
                            VecBatch{c->d_V + (size_t)(j + 1) * N, ldV}, N, R, red, c->d_h, scalars_per_rhs(m),
                            c->stream, nullptr, nullptr);
    });
    c->red_blocks = reduce_blocks(rv);
    // the DCGS2 update pass at the same depth, in place on V_j and V_{j+1}
    // (the solve overwrites both): its basis loads one by one or 8 batched
    if (c->opts.mode == HELM3D_MODE_N && lowsync(c)) {
        std::snprintf(shape, sizeof(shape), "%ld|%d|%d", N, R, j);
        const int M2 = m + 2;
        c->tv_update = tune_pick(c, "UPDATE", shape, kUpdateVariants, [&](int v) {
            Reduce red = reducer(c);
            red.update = v;
            return launch_update2(VecBatch{c->d_V, ldV}, N, j, c->d_h + 4 * M2, scalars_per_rhs(m), M2,
                                  VecBatch{c->d_V + (size_t)(j + 1) * N, ldV}, N, R, red, c->d_h + 2 * M2,
                                  scalars_per_rhs(m), c->stream, nullptr, nullptr);
        });
    }
    return HELM3D_OK;
}

// --------------------------------------------------------------- FGMRES
namespace {
// host state of one right-hand side of the batch
struct Rhs {
    int orig = 0;             // position in the caller's f/u
    double nf = 0;            // ||f||
    int it = 0, restarts = 0;
    double relres = 1, relres_phys = 1;
    int status = HELM3D_OK;
    bool done = false;
    bool frozen = false;      // converged inside the current cycle: no more columns
    int k = 0;                // columns of the current cycle
    double beta = 0;
    std::vector<zc> H, cs, sn, gv;
};
}  // namespace

// One FGMRES solve of a lockstep batch of R right-hand sides on one context,
// as a sequence of restart cycles: begin(); then, while the batch is not
// done, cycle_begin() (true residual, retirement, the cycle's batch B), the
// cycle itself (a graph launch, the steps launched one by one with device
// bookkeeping, or the host-driven cycle) and cycle_end(); then finish().  A
// group of contexts runs the cycles of all its contexts as one graph launch.
struct FgmresRun {
    helm3d_ctx *c;
    const double2 *f;
    double2 *u;
    int R;
    bool adjoint;
    helm3d_stats *st;
    int m = 1, M2 = 3, SH = 0;
    long N = 0, ldV = 0, ldZ = 0;
    size_t vb = 0;
    bool flexible = false;
    double2 *hbuf = nullptr;     // pinned mirror of the Krylov scalars (the context's h_scal)
    std::vector<Rhs> S;
    std::vector<int> act;        // packed position p -> right-hand side
    bool x_zero = true;
    int B = 0;                   // batch of the current cycle
    std::vector<double> vs0;
    std::vector<double2> ybuf;
    std::vector<int> iv;         // device cycle state of the current cycle (host side)
    std::vector<double> dv, est;
    std::vector<double2> g0;

    FgmresRun(helm3d_ctx *c_, const double2 *f_, double2 *u_, int R_, bool adj, helm3d_stats *st_)
        : c(c_), f(f_), u(u_), R(R_), adjoint(adj), st(st_) {}
    bool done() const { return act.empty(); }
    bool device_cycle() const { return lowsync(c) || graphs_usable(); }
    bool graphs_usable() const { return c->use_graphs && !c->prof && !c->opts.verbose; }

    int fetch_scalars(int n, const char *what) { return fetch(c, c->d_h, (size_t)SH * n, hbuf, what); }

    // Drop the finished right-hand sides from the packed batch: their iterate
    // goes to u, the rest move down (iterate, right-hand side, and V_0 when
    // it holds the current residual).
    int retire(bool move_v0) {
        double2 *V = c->d_V, *Fw = c->d_Fw, *Uw = c->d_Uw;
        size_t q = 0;
        for (size_t p = 0; p < act.size(); p++) {
            Rhs &r = S[act[p]];
            if (r.done) {
                RC(cuda_check(c, cudaMemcpyAsync(u + (size_t)r.orig * N, Uw + p * N, vb, cudaMemcpyDeviceToDevice,
                                                 c->stream),
                              "retire"));
                continue;
            }
            if (q != p) {
                RC(cuda_check(c, cudaMemcpyAsync(Fw + q * N, Fw + p * N, vb, cudaMemcpyDeviceToDevice, c->stream),
                              "pack f"));
                RC(cuda_check(c, cudaMemcpyAsync(Uw + q * N, Uw + p * N, vb, cudaMemcpyDeviceToDevice, c->stream),
                              "pack u"));
                if (move_v0)
                    RC(cuda_check(c, cudaMemcpyAsync(V + q * ldV, V + p * ldV, vb, cudaMemcpyDeviceToDevice,
                                                     c->stream),
                                  "pack v0"));
            }
            act[q++] = act[p];
        }
        act.resize(q);
        return HELM3D_OK;
    }

    int begin() {
        const helm3d_opts &o = c->opts;
        flexible = (o.mode == HELM3D_MODE_N);
        if (adjoint && !flexible) return set_error(c, HELM3D_ERR_ARG, "adjoint solve is mode N only");
        RC(check_batch(c, R));
        m = std::max(1, o.restart);
        RC(ensure_krylov(c, m, R));
        RC(ensure_planes(c, R));
        RC(tune_solve(c, R, adjoint));
        N = c->N;
        vb = sizeof(double2) * (size_t)N;
        ldV = (long)(m + 1) * N;
        ldZ = (long)m * N;
        M2 = m + 2;
        SH = scalars_per_rhs(m);
        // the pinned mirror lives in the context: pinning and unpinning host
        // memory are driver calls (cudaFreeHost also waits for the device),
        // kept out of every solve after the first of a size
        const size_t need = (size_t)SH * R;
        if (c->h_scal_cap < need) {
            if (c->h_scal) cudaFreeHost(c->h_scal);
            c->h_scal = nullptr;
            c->h_scal_cap = 0;
            if (cudaMallocHost((void **)&c->h_scal, sizeof(double2) * need) != cudaSuccess) {
                cudaGetLastError();
                c->h_scal = nullptr;
                return set_error(c, HELM3D_ERR_OOM, "pinned host buffer");
            }
            c->h_scal_cap = need;
        }
        hbuf = c->h_scal;
        cudaEventRecord(c->ev0, c->stream);
        RC(cuda_check(c, cudaMemcpyAsync(c->d_Fw, f, vb * R, cudaMemcpyDeviceToDevice, c->stream), "f copy"));
        RC(cuda_check(c, cudaMemsetAsync(c->d_Uw, 0, vb * R, c->stream), "x0"));
        RC(cuda_check(c, cudaMemsetAsync(u, 0, vb * R, c->stream), "u0"));
        RC(norms(c, VecBatch{c->d_Fw, N}, R, false, c->d_h + 2 * M2, SH));
        RC(fetch_scalars(R, "norms of f"));
        S.assign(R, Rhs());
        act.clear();
        for (int r = 0; r < R; r++) {
            Rhs &q = S[r];
            q.orig = r;
            q.nf = std::sqrt(hbuf[(size_t)r * SH + 2 * M2].x);
            if (!std::isfinite(q.nf)) return set_error(c, HELM3D_ERR_NONFINITE, "right-hand side has NaN/Inf");
            q.H.assign((size_t)(m + 1) * m, zc(0, 0));
            q.cs.assign(m, zc(0, 0));
            q.sn.assign(m, zc(0, 0));
            q.gv.assign(m + 1, zc(0, 0));
            act.push_back(r);
        }
        if (st) st->history_len = 0;
        for (int r : act)
            if (S[r].nf == 0.0) {
                S[r].done = true;
                S[r].relres = S[r].relres_phys = 0;
            }
        RC(retire(false));
        x_zero = true;
        vs0.assign(R, 0.0);
        ybuf.assign((size_t)M2 * R, make_double2(0, 0));
        return HELM3D_OK;
    }

    // r0 = f - A x0 into V_0 of every active right-hand side, its norms, the
    // stop test and retirement; B = 0 when the batch is done
    int cycle_begin() {
        const helm3d_opts &o = c->opts;
        B = 0;
        if (act.empty()) return HELM3D_OK;
        double2 *V = c->d_V;
        const int A = (int)act.size();
        const VecBatch V0{V, ldV};
        if (x_zero) {
            RC(cuda_check(c, cudaMemcpy2DAsync(V, sizeof(double2) * ldV, c->d_Fw, vb, vb, A,
                                               cudaMemcpyDeviceToDevice, c->stream),
                          "r0"));
        } else {
            RC(residual(c, VecBatch{c->d_Fw, N}, VecBatch{c->d_Uw, N}, V0, A, adjoint));
        }
        RC(norms(c, V0, A, true, c->d_h + 2 * M2, SH));
        RC(fetch_scalars(A, "residual norms"));
        bool any_done = false;
        for (int p = 0; p < A; p++) {
            Rhs &r = S[act[p]];
            const double b2 = hbuf[(size_t)p * SH + 2 * M2].x, p2 = hbuf[(size_t)p * SH + 2 * M2 + 1].x;
            r.beta = std::sqrt(b2);
            if (!std::isfinite(r.beta)) return set_error(c, HELM3D_ERR_NONFINITE, "residual is NaN/Inf");
            r.relres = r.beta / r.nf;
            r.relres_phys = std::sqrt(p2) / r.nf;   // relative to ||f|| as the reference (:591-592)
            if (r.relres <= o.tol || r.it >= o.max_iter) {
                r.done = true;
                r.status = (r.relres <= o.tol || o.max_iter == 0) ? HELM3D_OK : HELM3D_ERR_NOT_CONVERGED;
                any_done = true;
            }
        }
        if (any_done) RC(retire(true));
        if (act.empty()) return HELM3D_OK;
        B = (int)act.size();
        for (int p = 0; p < B; p++) {
            Rhs &r = S[act[p]];
            vs0[p] = 1.0 / r.beta;
            std::fill(r.H.begin(), r.H.end(), zc(0, 0));
            std::fill(r.gv.begin(), r.gv.end(), zc(0, 0));
            r.gv[0] = r.beta;
            r.frozen = false;
            r.k = 0;
        }
        return cuda_check(c, cudaMemcpy2DAsync(c->d_vs, sizeof(double) * M2, vs0.data(), sizeof(double),
                                               sizeof(double), B, cudaMemcpyHostToDevice, c->stream),
                          "vs0");
    }

    // the device cycle state of the batch in (before the graph or the steps)
    int upload_state() {
        const helm3d_opts &o = c->opts;
        const ArnState a = arn_state(c, m, B);
        const int Ra = c->r_alloc;
        dv.assign((size_t)2 * Ra, 0.0);
        iv.assign((size_t)4 * Ra + kArnFlags, 0);
        g0.assign((size_t)B, make_double2(0, 0));
        for (int p = 0; p < B; p++) {
            const Rhs &r = S[act[p]];
            dv[p] = r.nf;
            dv[Ra + p] = o.tol;
            iv[2 * Ra + p] = r.it;
            iv[3 * Ra + p] = o.max_iter;
            g0[p] = make_double2(r.beta, 0.0);
        }
        RC(cuda_check(c, cudaMemcpyAsync(a.nf, dv.data(), sizeof(double) * dv.size(), cudaMemcpyHostToDevice,
                                         c->stream),
                      "cycle state"));
        RC(cuda_check(c, cudaMemcpyAsync(a.frozen, iv.data(), sizeof(int) * iv.size(), cudaMemcpyHostToDevice,
                                         c->stream),
                      "cycle state"));
        return cuda_check(c, cudaMemcpy2DAsync(a.g, sizeof(double2) * (m + 1), g0.data(), sizeof(double2),
                                               sizeof(double2), B, cudaMemcpyHostToDevice, c->stream),
                          "cycle state");
    }

    // a device cycle without a graph: the steps one by one, the host checking
    // after each whether some right-hand side is still active
    int run_steps() {
        const ArnState a = arn_state(c, m, B);
        for (int j = 0; j < m; j++) {
            RC(arnoldi_step(c, m, B, j, adjoint, a, false, 0));
            int active = 0;
            RC(cuda_check(c, cudaMemcpyAsync(&active, a.flags + 5, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                          "active"));
            RC(cuda_check(c, cudaStreamSynchronize(c->stream), "step"));
            if (c->opts.verbose) fprintf(stderr, "helm3d: step %d, %s\n", j + 1, active ? "active" : "done");
            if (!active) break;
        }
        return cycle_tail(c, m, B, a);
    }

    // the device cycle state out; per_step / tail: kernels of a graph launch
    // (counted here), or -1 when the steps were launched (already counted)
    int cycle_end_device(long long per_step, long long tail) {
        const ArnState a = arn_state(c, m, B);
        const int Ra = c->r_alloc;
        est.assign((size_t)Ra * m, 0.0);
        RC(cuda_check(c, cudaMemcpyAsync(iv.data(), a.frozen, sizeof(int) * iv.size(), cudaMemcpyDeviceToHost,
                                         c->stream),
                      "cycle result"));
        RC(cuda_check(c, cudaMemcpyAsync(est.data(), a.est, sizeof(double) * est.size(), cudaMemcpyDeviceToHost,
                                         c->stream),
                      "cycle result"));
        RC(cuda_check(c, cudaStreamSynchronize(c->stream), "cycle"));
        const int *flags = iv.data() + 4 * Ra;
        if (flags[3]) return set_error(c, HELM3D_ERR_NONFINITE, "Arnoldi norm is NaN/Inf");
        const int kmax = flags[2];
        c->reorth += flags[1];
        if (per_step >= 0) c->launches += (flags[4] + 1) * per_step + tail;   // steps run = last step index + 1
        for (int p = 0; p < B; p++) {
            Rhs &r = S[act[p]];
            r.it = iv[2 * Ra + p];
            r.k = iv[Ra + p];
        }
        for (int j = 0; j < kmax; j++) {
            double e = 0;
            for (int p = 0; p < B; p++)
                if (S[act[p]].k > j) e = std::max(e, est[(size_t)p * m + j]);
            if (st && st->history && st->history_len < st->history_cap) st->history[st->history_len++] = e;
        }
        return cycle_done();
    }

    int cycle_done() {
        x_zero = false;
        for (int p = 0; p < B; p++) S[act[p]].restarts++;
        return HELM3D_OK;
    }

    // the host-driven cycle (classical Gram-Schmidt, host Givens): mode R
    // without graphs, or HELM3D_GS=cgs2 without graphs
    int run_host_cycle();

    int finish() {
        if (!flexible) {
            // u = L0^{-1} w for every right-hand side (in place: the forward
            // transform reads all of u before the inverse writes it)
            RC(apply_prec(c, VecBatch{u, N}, 1.0, kNoScale, VecBatch{u, N}, R));
        }
        cudaEventRecord(c->ev1, c->stream);
        RC(check_status(c));
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        int status = HELM3D_OK;
        for (const Rhs &r : S) {
            if (r.status) status = r.status;
            if (st) {
                st->iterations += r.it;
                st->restarts += r.restarts;
                st->relres = std::max(st->relres, r.relres);
                st->relres_phys = std::max(st->relres_phys, r.relres_phys);
            }
        }
        if (st) st->ms_solve += ms;
        return status;
    }
};

int FgmresRun::run_host_cycle() {
    const helm3d_opts &o = c->opts;
    const double tol = o.tol;
    double2 *V = c->d_V, *Uw = c->d_Uw, *Hd = c->d_h;
    double2 *d_h1 = Hd, *d_h2 = Hd + M2, *d_nrm = Hd + 2 * M2, *d_y = Hd + 3 * M2;
    const Reduce red = reducer(c);
    const VecBatch Vall{V, ldV};
    const ScaleBatch vsb{c->d_vs, M2};
    for (int j = 0; j < m; j++) {
        const VecBatch Vj{V + (size_t)j * N, ldV}, w{V + (size_t)(j + 1) * N, ldV};
        const ScaleBatch vsj{c->d_vs + j, M2};
        if (flexible) {
            const VecBatch zj = zbasis(c, (long)j * N, ldZ);
            if (adjoint) {
                // A^H M^{-H} = (M^{-1} A)^H: the adjoint of the forward
                // preconditioned operator, with the same singular values
                RC(apply_prec_adjoint(c, Vj, 1.0, vsj, zj, B));
                RC(apply_op_adjoint(c, zj, 1.0, kNoScale, w, B));
            } else {
                RC(apply_prec(c, Vj, 1.0, vsj, zj, B));
                RC(apply_op(c, zj, 1.0, kNoScale, w, B));
            }
        } else {
            RC(apply_op(c, Vj, 1.0, vsj, w, B));
        }
        // Classical Gram-Schmidt, repeated only when needed ("twice is
        // enough"): h1 = V^H w with ||w||^2 from the same pass, w -= V h1
        // with ||w||^2 after; a second pass runs when the norm of some
        // right-hand side dropped below 1/sqrt(2) of its value.
        RC(timed(c, HELM3D_K_KRYLOV, 2,
                 [&] { return launch_dots(Vall, N, vsb, j + 1, w, N, B, red, d_h1, SH, c->stream, true); }));
        RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
            return launch_update(Vall, N, vsb, j + 1, d_h1, SH, w, N, B, 1, red, d_nrm, SH, c->stream);
        }));
        RC(fetch_scalars(B, "Arnoldi coefficients"));
        bool again = false;
        for (int p = 0; p < B; p++) {
            const Rhs &r = S[act[p]];
            const double2 *h = hbuf + (size_t)p * SH;
            if (!r.frozen && h[2 * M2].x < H3D_REORTH_ETA2 * h[j + 1].x) again = true;
        }
        for (int p = 0; p < B; p++) {
            Rhs &r = S[act[p]];
            const double2 *h = hbuf + (size_t)p * SH;
            for (int i = 0; i <= j; i++) r.H[(size_t)i * m + j] = zc(h[i].x, h[i].y);
        }
        if (again) {
            RC(timed(c, HELM3D_K_KRYLOV, 2,
                     [&] { return launch_dots(Vall, N, vsb, j + 1, w, N, B, red, d_h2, SH, c->stream); }));
            RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
                return launch_update(Vall, N, vsb, j + 1, d_h2, SH, w, N, B, 1, red, d_nrm, SH, c->stream);
            }));
            RC(fetch_scalars(B, "Arnoldi second pass"));
            for (int p = 0; p < B; p++) {
                Rhs &r = S[act[p]];
                const double2 *h = hbuf + (size_t)p * SH + M2;
                for (int i = 0; i <= j; i++) r.H[(size_t)i * m + j] += zc(h[i].x, h[i].y);
            }
            c->reorth++;
        }
        double est_max = 0;
        bool all_frozen = true;
        for (int p = 0; p < B; p++) {
            Rhs &r = S[act[p]];
            if (r.frozen) continue;
            const double hn = std::sqrt(std::max(0.0, hbuf[(size_t)p * SH + 2 * M2].x));
            if (!std::isfinite(hn)) return set_error(c, HELM3D_ERR_NONFINITE, "Arnoldi norm is NaN/Inf");
            std::vector<zc> &H = r.H;
            H[(size_t)(j + 1) * m + j] = hn;
            for (int i = 0; i < j; i++) {
                const zc a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = r.cs[i] * a + r.sn[i] * b;
                H[(size_t)(i + 1) * m + j] = -std::conj(r.sn[i]) * a + r.cs[i] * b;
            }
            const zc a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
            givens(a, b, r.cs[j], r.sn[j]);
            H[(size_t)j * m + j] = r.cs[j] * a + r.sn[j] * b;
            H[(size_t)(j + 1) * m + j] = 0.0;
            r.gv[j + 1] = -std::conj(r.sn[j]) * r.gv[j];
            r.gv[j] = r.cs[j] * r.gv[j];
            r.it++;
            r.k = j + 1;
            const double est = std::abs(r.gv[j + 1]) / r.nf;
            est_max = std::max(est_max, est);
            if (hn == 0.0 || est <= tol || r.it >= o.max_iter) r.frozen = true;
            else all_frozen = false;
        }
        if (st && st->history && st->history_len < st->history_cap) st->history[st->history_len++] = est_max;
        if (o.verbose) fprintf(stderr, "helm3d: step %d  max est relres %.3e over %d rhs\n", j + 1, est_max, B);
        if (all_frozen) break;
        RC(timed(c, HELM3D_K_KRYLOV, 1, [&] { return launch_set_scale(d_nrm, SH, c->d_vs, M2, j + 1, B, c->stream); }));
    }
    // y = H^{-1} g (upper triangular k x k) per right-hand side, zero
    // padded to the longest; x += basis * y
    int kmax = 0;
    for (int p = 0; p < B; p++) kmax = std::max(kmax, S[act[p]].k);
    for (int p = 0; p < B; p++) {
        const Rhs &r = S[act[p]];
        double2 *y = ybuf.data() + (size_t)p * M2;
        std::vector<zc> yz(r.k);
        for (int i = r.k - 1; i >= 0; i--) {
            zc s = r.gv[i];
            for (int q = i + 1; q < r.k; q++) s -= r.H[(size_t)i * m + q] * yz[q];
            yz[i] = s / r.H[(size_t)i * m + i];
        }
        for (int i = 0; i < kmax; i++) y[i] = i < r.k ? make_double2(yz[i].real(), yz[i].imag()) : make_double2(0, 0);
    }
    if (kmax > 0) {
        RC(cuda_check(c, cudaMemcpy2DAsync(d_y, sizeof(double2) * SH, ybuf.data(), sizeof(double2) * M2,
                                           sizeof(double2) * kmax, B, cudaMemcpyHostToDevice, c->stream),
                      "y"));
        RC(timed(c, HELM3D_K_KRYLOV, 1, [&] {
            return flexible ? launch_combine(zbasis(c, 0, ldZ), N, kNoScale, kmax, d_y, SH, VecBatch{Uw, N}, N, B,
                                             c->stream)
                            : launch_combine(Vall, N, vsb, kmax, d_y, SH, VecBatch{Uw, N}, N, B, c->stream);
        }));
    }
    return cycle_done();
}

int fgmres(helm3d_ctx *c, const double2 *f, double2 *u, int R, bool adjoint, helm3d_stats *st) {
    FgmresRun run(c, f, u, R, adjoint, st);
    RC(run.begin());
    while (!run.done()) {
        RC(run.cycle_begin());
        if (run.B == 0) break;
        const int gi = run.graphs_usable() ? cycle_graph(c, run.m, run.B, adjoint) : -1;
        if (gi >= 0) {
            RC(run.upload_state());
            RC(cuda_check(c, cudaGraphLaunch(c->graphs[gi].exec, c->stream), "cycle graph"));
            RC(run.cycle_end_device(c->graphs[gi].kernels_per_step, c->graphs[gi].tail_kernels));
        } else if (lowsync(c)) {
            RC(run.upload_state());
            RC(run.run_steps());
            RC(run.cycle_end_device(-1, 0));
        } else {
            RC(run.run_host_cycle());
        }
    }
    return run.finish();
}

// ------------------------------------------------- groups of contexts
// A group graph: the cycles of several contexts (each with its batch size)
// as independent chains of one graph, so that the kernels of grids of
// different sizes run side by side on the GPU.
namespace {
struct GroupGraph {
    std::vector<int> key;                  // batch per context (0: not in the cycle)
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> per_step, tail;
};
struct StreamGuard {
    std::vector<helm3d_ctx *> cs;
    std::vector<cudaStream_t> saved;
    ~StreamGuard() {
        for (size_t i = 0; i < cs.size(); i++) cs[i]->stream = saved[i];
    }
};
}  // namespace

int fgmres_group(helm3d_ctx *const *cs, int n, const double2 *const *f, double2 *const *u, const int *R,
                 helm3d_stats *const *st) {
    // one stream for the call: the group graph and every context's set-up
    // and read-back work are ordered on it
    StreamGuard guard;
    cudaStream_t gs = cs[0]->stream;
    for (int i = 0; i < n; i++) {
        guard.cs.push_back(cs[i]);
        guard.saved.push_back(cs[i]->stream);
        cs[i]->stream = gs;
    }
    std::vector<std::unique_ptr<FgmresRun>> runs;
    for (int i = 0; i < n; i++) {
        runs.emplace_back(new FgmresRun(cs[i], f[i], u[i], R[i], false, st[i]));
        RC(runs.back()->begin());
    }
    std::vector<GroupGraph> graphs;
    struct Cleanup {
        std::vector<GroupGraph> *g;
        ~Cleanup() {
            for (auto &x : *g)
                if (x.exec) cudaGraphExecDestroy(x.exec);
        }
    } cleanup{&graphs};
    bool use_group = true;
    for (int i = 0; i < n; i++) use_group = use_group && runs[i]->graphs_usable();
    for (;;) {
        std::vector<int> key(n, 0);
        bool any = false;
        for (int i = 0; i < n; i++) {
            if (runs[i]->done()) continue;
            RC(runs[i]->cycle_begin());
            key[i] = runs[i]->B;
            any = any || key[i] > 0;
        }
        if (!any) break;
        int gi = -1;
        if (use_group) {
            for (size_t q = 0; q < graphs.size(); q++)
                if (graphs[q].key == key) gi = (int)q;
            if (gi < 0) {
                GroupGraph g;
                g.key = key;
                g.per_step.assign(n, 0);
                g.tail.assign(n, 0);
                cudaGraph_t G = nullptr;
                bool ok = cudaGraphCreate(&G, 0) == cudaSuccess;
                for (int i = 0; ok && i < n; i++)
                    if (key[i] > 0) ok = add_cycle(G, cs[i], runs[i]->m, key[i], false, g.per_step[i], g.tail[i]);
                if (ok) ok = cudaGraphInstantiate(&g.exec, G, 0) == cudaSuccess;
                if (G) cudaGraphDestroy(G);
                if (ok) {
                    graphs.push_back(g);
                    gi = (int)graphs.size() - 1;
                } else {
                    cudaGetLastError();
                    use_group = false;   // the contexts' own cycles from here on
                }
            }
        }
        if (gi >= 0) {
            for (int i = 0; i < n; i++)
                if (key[i] > 0) RC(runs[i]->upload_state());
            RC(cuda_check(cs[0], cudaGraphLaunch(graphs[gi].exec, gs), "group cycle graph"));
            for (int i = 0; i < n; i++)
                if (key[i] > 0) RC(runs[i]->cycle_end_device(graphs[gi].per_step[i], graphs[gi].tail[i]));
            continue;
        }
        for (int i = 0; i < n; i++) {
            if (key[i] == 0) continue;
            FgmresRun &run = *runs[i];
            helm3d_ctx *c = cs[i];
            const int g1 = run.graphs_usable() ? cycle_graph(c, run.m, run.B, false) : -1;
            if (g1 >= 0) {
                RC(run.upload_state());
                RC(cuda_check(c, cudaGraphLaunch(c->graphs[g1].exec, c->stream), "cycle graph"));
                RC(run.cycle_end_device(c->graphs[g1].kernels_per_step, c->graphs[g1].tail_kernels));
            } else if (lowsync(c)) {
                RC(run.upload_state());
                RC(run.run_steps());
                RC(run.cycle_end_device(-1, 0));
            } else {
                RC(run.run_host_cycle());
            }
        }
    }
    int worst = HELM3D_OK;
    for (int i = 0; i < n; i++) {
        const int rc = runs[i]->finish();
        if (rc && rc != HELM3D_ERR_NOT_CONVERGED) return rc;
        if (rc) worst = rc;
    }
    return worst;
}

// -------------------------------------------------------------- BiCGStab
// dot <a, b> = sum conj(a) b on the device, returned to the host
static int zdot(helm3d_ctx *c, const double2 *a, const double2 *b, zc *out) {
    const Reduce red = reducer(c);
    RC(timed(c, HELM3D_K_KRYLOV, 2, [&] {
        return launch_dots(one(a), c->N, kNoScale, 1, one(b), c->N, 1, red, c->d_h, 0, c->stream);
    }));
    double2 v;
    RC(fetch(c, c->d_h, 1, &v, "dot"));
    *out = zc(v.x, v.y);
    return HELM3D_OK;
}

static int norm2_one(helm3d_ctx *c, const double2 *x, bool phys, double *full, double *ph) {
    RC(norms(c, one(x), 1, phys, c->d_h + 1, 0));
    double2 v[2];
    RC(fetch(c, c->d_h + 1, phys ? 2 : 1, v, "norm"));
    *full = v[0].x;
    if (ph) *ph = v[1].x;
    return HELM3D_OK;
}

static int axpby1(helm3d_ctx *c, double2 a, const double2 *x, double2 b, double2 *y) {
    return axpby(c, a, one(x), b, one(y), 1);
}

int bicgstab(helm3d_ctx *c, const double2 *f, double2 *u, helm3d_stats *st) {
    const helm3d_opts &o = c->opts;
    RC(ensure_krylov(c, 1, 1));
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
    RC(norm2_one(c, f, false, &nf2, nullptr));
    const double nf = std::sqrt(nf2);
    if (!std::isfinite(nf)) return set_error(c, HELM3D_ERR_NONFINITE, "right-hand side has NaN/Inf");
    RC(cuda_check(c, cudaMemsetAsync(u, 0, vb, c->stream), "x0"));
    if (nf == 0.0) return HELM3D_OK;
    // x0 = 0: r0 = f, p0 = r0, r* = 2 r0 (Source/BcGSTAB.cpp:433-437)
    RC(cuda_check(c, cudaMemcpyAsync(r, f, vb, cudaMemcpyDeviceToDevice, c->stream), "r0"));
    RC(cuda_check(c, cudaMemcpyAsync(p, f, vb, cudaMemcpyDeviceToDevice, c->stream), "p0"));
    RC(cuda_check(c, cudaMemsetAsync(rst, 0, vb, c->stream), "rst"));
    RC(axpby1(c, make_double2(2, 0), f, make_double2(0, 0), rst));
    int it = 0, status = HELM3D_OK;
    double relres = 1.0;
    const bool modeN = o.mode == HELM3D_MODE_N;
    // right preconditioned operator B = A M^{-1} (mode N) or K (mode R);
    // the u-space update uses M^{-1} p (mode N) or L0^{-1} p (mode R)
    auto opB = [&](const double2 *x, double2 *yout, double2 *pre) -> int {
        RC(apply_prec(c, one(x), 1.0, kNoScale, one(pre), 1));
        if (modeN) return apply_op(c, one(pre), 1.0, kNoScale, one(yout), 1);
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
        RC(axpby1(c, make_double2(-alpha.real(), -alpha.imag()), Ay, make_double2(1, 0), s));
        RC(opB(s, Az, zv));
        zc as, aa;
        RC(zdot(c, Az, s, &as));
        RC(zdot(c, Az, Az, &aa));
        if (aa == zc(0, 0)) { status = HELM3D_ERR_BREAKDOWN; break; }
        const zc om = as / aa;
        // x += alpha y + omega z
        RC(axpby1(c, make_double2(alpha.real(), alpha.imag()), yv, make_double2(1, 0), u));
        RC(axpby1(c, make_double2(om.real(), om.imag()), zv, make_double2(1, 0), u));
        // r_new = s - omega Az (into r)
        zc rr_old = rr;
        RC(cuda_check(c, cudaMemcpyAsync(r, s, vb, cudaMemcpyDeviceToDevice, c->stream), "r"));
        RC(axpby1(c, make_double2(-om.real(), -om.imag()), Az, make_double2(1, 0), r));
        zc rrn;
        RC(zdot(c, rst, r, &rrn));
        if (rr_old == zc(0, 0) || om == zc(0, 0)) { status = HELM3D_ERR_BREAKDOWN; break; }
        const zc beta = (alpha / om) * rrn / rr_old;
        // p = r + beta (p - omega Ay)
        RC(axpby1(c, make_double2(-om.real(), -om.imag()), Ay, make_double2(1, 0), p));
        RC(axpby1(c, make_double2(1, 0), r, make_double2(beta.real(), beta.imag()), p));

        it++;
        // the recursion's residual, over the whole grid or (stop_phys, as the
        // reference's test, Source/BcGSTAB.cpp:503-505) the physical domain
        double r2, rp2 = 0.0;
        RC(norm2_one(c, r, o.stop_phys != 0, &r2, &rp2));
        relres = std::sqrt(o.stop_phys ? rp2 : r2) / nf;
        if (st && st->history && st->history_len < st->history_cap) st->history[st->history_len++] = relres;
        if (!std::isfinite(relres)) return set_error(c, HELM3D_ERR_NONFINITE, "BiCGStab residual is NaN/Inf");
        if (relres <= o.tol) break;
    }
    // true residual of the u-space system
    RC(ensure_vec(c, &c->d_r, "residual"));
    if (modeN) {
        RC(residual(c, one(f), one(u), one(c->d_r), 1, false));
    } else {
        // A_R u = L0 u - dL u is not formed directly: K(L0 u) = A_R u.  The
        // BiCGStab recursion residual r is reported for mode R.
        RC(cuda_check(c, cudaMemcpyAsync(c->d_r, r, vb, cudaMemcpyDeviceToDevice, c->stream), "r"));
    }
    double r2, rp2;
    RC(norm2_one(c, c->d_r, true, &r2, &rp2));
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
    if (status == HELM3D_OK && (o.stop_phys ? std::sqrt(rp2) / nf : relres) > o.tol)
        status = HELM3D_ERR_NOT_CONVERGED;
    return status;
}

}  // namespace h3d
