// capi.cpp -- the extern "C" entry points of include/helm3d.h.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <memory>
#include <new>
#include <vector>

#include "helm3d_internal.h"

using namespace h3d;

namespace {

// message of the last failed helm3d_create on this thread (no context exists then)
thread_local std::string g_create_error;

// A vector argument of `count` complex values: device pointers are used in
// place, host data is staged through *slot (capacity *cap values).
struct VecArg {
    helm3d_ctx *c;
    double2 *dev = nullptr;
    bool staged = false;
    int rc = HELM3D_OK;
    VecArg(helm3d_ctx *ctx, const void *p, size_t count, bool copy_in, double2 **slot, size_t *cap) : c(ctx) {
        if (!p) { rc = set_error(c, HELM3D_ERR_ARG, "null vector argument"); return; }
        if (is_device_ptr(p)) { dev = (double2 *)p; return; }
        staged = true;
        if (*slot && *cap < count) {
            rc = cuda_check(c, cudaStreamSynchronize(c->stream), "staging sync");
            if (rc) return;
            cudaFree(*slot);
            c->bytes -= sizeof(double2) * *cap;
            *slot = nullptr;
            *cap = 0;
        }
        if (!*slot) {
            rc = cuda_check(c, cudaMalloc((void **)slot, sizeof(double2) * count), "staging buffer");
            if (rc) return;
            c->bytes += sizeof(double2) * count;
            *cap = count;
        }
        dev = *slot;
        if (copy_in)
            rc = cuda_check(c, cudaMemcpyAsync(dev, p, sizeof(double2) * count, cudaMemcpyHostToDevice, c->stream),
                            "copy in");
    }
    int copy_out(void *p, size_t count) {
        if (!staged) return HELM3D_OK;
        int r = cuda_check(c, cudaMemcpyAsync(p, dev, sizeof(double2) * count, cudaMemcpyDeviceToHost, c->stream),
                           "copy out");
        if (r) return r;
        return cuda_check(c, cudaStreamSynchronize(c->stream), "copy out sync");
    }
};

// Right-hand sides per lockstep batch: at most kMaxBatch, and as many as the
// Krylov bases (V, Z), packed iterates, planes, staging and `extra` further
// vectors of each fit in 85% of the free device memory (plus what the
// context's Krylov workspace already holds).
int batch_size(helm3d_ctx *c, int nrhs, bool staged, int extra = 0) {
    const int m = std::max(1, c->opts.restart);
    const size_t vb = sizeof(double2) * (size_t)c->N;
    const size_t per =
        vb * ((size_t)(m + 1) + (c->opts.mode == HELM3D_MODE_N ? m : 0) + 2 + (staged ? 2 : 0) + extra) +
        (c->c64 ? 8 : 16) * (size_t)c->N;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const size_t avail = (size_t)(0.85 * (double)(fr + c->kry_bytes));
    int R = (int)std::min<size_t>(avail / std::max<size_t>(per, 1), (size_t)kMaxBatch);
    return std::max(1, std::min(R, nrhs));
}

int validate(const helm3d_grid *g, const helm3d_opts *o) {
    if (!g || !o) return HELM3D_ERR_ARG;
    if (g->nx < 2 || g->ny < 2 || g->nz < 1) return HELM3D_ERR_ARG;
    if (!(g->hx > 0) || !(g->hy > 0) || !(g->hz > 0) || !(g->omega > 0)) return HELM3D_ERR_ARG;
    if (g->pml_x < 0 || g->pml_y < 0 || g->pml_z < 0 || g->spg_z < 0) return HELM3D_ERR_ARG;
    if (2 * g->pml_x >= g->nx || 2 * g->pml_y >= g->ny) return HELM3D_ERR_ARG;
    if (o->mode == HELM3D_MODE_R && 2 * g->spg_z >= g->nz) return HELM3D_ERR_ARG;
    if (o->mode != HELM3D_MODE_R && o->mode != HELM3D_MODE_N) return HELM3D_ERR_ARG;
    if (o->precision != HELM3D_PREC_C64 && o->precision != HELM3D_PREC_C128) return HELM3D_ERR_ARG;
    if (o->kz_symbol < 0 || o->kz_symbol > 2) return HELM3D_ERR_ARG;
    if (o->z_transform != HELM3D_ZT_FFT && o->z_transform != HELM3D_ZT_PML_EIGEN) return HELM3D_ERR_ARG;
    if (o->restart < 1 || o->restart > 1000 || o->max_iter < 0 || !(o->tol >= 0)) return HELM3D_ERR_ARG;
    if (g->nz > 4096) return HELM3D_ERR_ARG;
    return HELM3D_OK;
}

}  // namespace

// Start of a call that runs the operator or the preconditioner: refused
// after a failed set-up or factor of this context (that error again), else
// the device status word is cleared, so that a bounded wait that expired or
// an index check that failed in an earlier call is not reported again (the
// factor's own bits were reported when it ran).
int h3d::begin_call(helm3d_ctx *c) {
    if (c->factor_rc)
        return set_error(c, c->factor_rc,
                         std::string("the context's last set-up or factor failed: ") + helm3d_status_string(c->factor_rc));
    return cuda_check(c, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream), "status reset");
}

extern "C" {

int helm3d_default_opts(helm3d_opts *o) {
    if (!o) return HELM3D_ERR_ARG;
    memset(o, 0, sizeof(*o));
    o->mode = HELM3D_MODE_N;
    o->precision = HELM3D_PREC_C64;
    o->kz_symbol = HELM3D_KZ_DISCRETE;
    o->beta_prec = 0.25;
    o->beta_phys = 0.0;
    o->s2_l0 = 0.0;
    o->quirk_q1 = 1;
    o->restart = 20;
    o->max_iter = 2000;
    o->tol = 1e-8;
    o->stop_phys = 0;
    o->device = 0;
    o->verbose = 0;
    return HELM3D_OK;
}

const char *helm3d_status_string(int s) {
    switch (s) {
        case HELM3D_OK: return "ok";
        case HELM3D_ERR_ARG: return "bad argument";
        case HELM3D_ERR_OOM: return "out of device memory";
        case HELM3D_ERR_CUDA: return "CUDA error";
        case HELM3D_ERR_SINGULAR: return "singular block in the factor";
        case HELM3D_ERR_NOT_CONVERGED: return "not converged";
        case HELM3D_ERR_BREAKDOWN: return "Krylov breakdown";
        case HELM3D_ERR_NONFINITE: return "non-finite value";
        case HELM3D_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char *helm3d_last_error(const helm3d_ctx *c) { return c ? c->last_error.c_str() : g_create_error.c_str(); }

size_t helm3d_device_bytes(const helm3d_ctx *c) { return c ? c->bytes : 0; }

int helm3d_set_stream(helm3d_ctx *c, void *stream) {
    if (!c) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return HELM3D_OK;
}

int helm3d_profile(helm3d_ctx *c, int enable) {
    if (!c) return HELM3D_ERR_ARG;
    c->prof = enable != 0;
    return HELM3D_OK;
}

int helm3d_profile_read(helm3d_ctx *c, double *ms, long long *launches, int nkinds) {
    if (!c || nkinds < 0) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    int rc = cuda_check(c, cudaStreamSynchronize(c->stream), "profile sync");
    if (rc) return rc;
    for (auto &e : c->prof_ev) {
        float t = 0;
        if (cudaEventElapsedTime(&t, e.a, e.b) == cudaSuccess) c->prof_ms[e.kind] += t;
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    c->prof_ev.clear();
    for (int k = 0; k < nkinds && k < HELM3D_K_COUNT; k++) {
        if (ms) ms[k] = c->prof_ms[k];
        if (launches) launches[k] = c->prof_n[k];
    }
    for (int k = 0; k < HELM3D_K_COUNT; k++) {
        c->prof_ms[k] = 0;
        c->prof_n[k] = 0;
    }
    return HELM3D_OK;
}

long long helm3d_kernel_launches(const helm3d_ctx *c) { return c ? c->launches : 0; }

int helm3d_create(const helm3d_grid *grid, const double *s2, const helm3d_opts *opts, helm3d_ctx **out) {
    if (!out) return HELM3D_ERR_ARG;
    *out = nullptr;
    int rc = validate(grid, opts);
    if (rc) return rc;
    if (!s2) return HELM3D_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return HELM3D_ERR_NO_DEVICE;
    }
    if (opts->device < 0 || opts->device >= ndev) return HELM3D_ERR_ARG;
    helm3d_ctx *c = new (std::nothrow) helm3d_ctx();
    if (!c) return HELM3D_ERR_OOM;
    c->grid = *grid;
    c->opts = *opts;
    c->device = opts->device;
    c->c64 = opts->precision == HELM3D_PREC_C64;
    // Z_j = M^{-1} V_j is the complex64 preconditioner's output: kept in
    // complex64 (HELM3D_Z64=0 in the environment keeps it in complex128)
    {
        const char *zenv = std::getenv("HELM3D_Z64");
        c->z64 = c->c64 && opts->mode == HELM3D_MODE_N && !(zenv && zenv[0] == '0');
    }
    c->plane = (long)grid->nx * grid->ny;
    c->N = c->plane * grid->nz;
    if (cudaSetDevice(c->device) != cudaSuccess) {
        delete c;
        return HELM3D_ERR_CUDA;
    }
    auto fail = [&](int code) {
        g_create_error = c->last_error;
        helm3d_destroy(c);
        return code;
    };
    if ((rc = cuda_check(c, cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking), "stream")) ||
        (rc = cuda_check(c, cudaEventCreate(&c->ev0), "event")) ||
        (rc = cuda_check(c, cudaEventCreate(&c->ev1), "event")))
        return fail(rc);
    c->stream = c->own_stream;
    // HELM3D_GRAPH=0 keeps the host-driven restart cycle (no CUDA graphs)
    const char *genv = std::getenv("HELM3D_GRAPH");
    c->use_graphs = !(genv && genv[0] == '0');
    // HELM3D_GS=cgs2 selects classical Gram-Schmidt with the conditional
    // second pass for mode N instead of DCGS2
    const char *gsenv = std::getenv("HELM3D_GS");
    c->gs_lowsync = !(gsenv && std::strcmp(gsenv, "cgs2") == 0);
    auto t0 = std::chrono::steady_clock::now();
    if ((rc = ctx_setup_grid(c)) || (rc = ctx_setup_medium(c, s2, is_device_ptr(s2))) || (rc = ctx_factor(c)))
        return fail(rc);
    c->ms_factor = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    g_create_error.clear();
    *out = c;
    return HELM3D_OK;
}

int helm3d_set_medium(helm3d_ctx *c, const double *s2) {
    if (!c || !s2) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    int rc = ctx_setup_medium(c, s2, is_device_ptr(s2));
    if (!rc) rc = ctx_factor(c);
    c->factor_rc = rc;
    return rc;
}


static int solve_common(helm3d_ctx *c, const double *f, double *u, int nrhs, helm3d_stats *st, int which) {
    if (!c || !f || !u || nrhs < 1) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    if (int rc = begin_call(c)) return rc;
    if (st) {
        st->iterations = 0;
        st->restarts = 0;
        st->ms_solve = 0;
        st->relres = 0;
        st->relres_phys = 0;
        st->history_len = 0;
    }
    const bool staged = !is_device_ptr(f) || !is_device_ptr(u);
    const int B = which == 1 ? 1 : batch_size(c, nrhs, staged);
    int worst = HELM3D_OK;
    for (int r0 = 0; r0 < nrhs; r0 += B) {
        const int R = std::min(B, nrhs - r0);
        const size_t count = (size_t)R * c->N;
        const double *fr = f + 2 * (size_t)r0 * c->N;
        double *ur = u + 2 * (size_t)r0 * c->N;
        VecArg fa(c, fr, count, true, &c->d_f, &c->f_cap);
        if (fa.rc) return fa.rc;
        VecArg ua(c, ur, count, false, &c->d_u, &c->u_cap);
        if (ua.rc) return ua.rc;
        int rc;
        if (which == 0) rc = fgmres(c, fa.dev, ua.dev, R, false, st);
        else if (which == 1) rc = bicgstab(c, fa.dev, ua.dev, st);
        else rc = fgmres(c, fa.dev, ua.dev, R, true, st);
        if (rc && rc != HELM3D_ERR_NOT_CONVERGED) return rc;
        if (rc) worst = rc;
        int rc2 = ua.copy_out(ur, count);
        if (rc2) return rc2;
    }
    if (st) st->status = worst;
    return worst;
}

int helm3d_solve(helm3d_ctx *c, const double *f, double *u, int nrhs, helm3d_stats *st) {
    return solve_common(c, f, u, nrhs, st, 0);
}

int helm3d_solve_medium(helm3d_ctx *c, const double *s2, const double *f, double *u, int nrhs,
                        helm3d_stats *st) {
    if (!c || !s2 || !f || !u || nrhs < 1) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    const size_t count = (size_t)nrhs * c->N;
    // host right-hand sides that fit one lockstep batch go to the staging
    // buffer on a copy stream while the medium is factored: the staging
    // buffer and the stream are made first, the copy is issued after the
    // medium's own upload (so that it does not queue behind the sources)
    bool pre = !is_device_ptr(f) && batch_size(c, nrhs, true) >= nrhs;
    if (pre) {
        int rc = HELM3D_OK;
        if (!c->copy_stream) {
            rc = cuda_check(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy stream");
            if (!rc) rc = cuda_check(c, cudaEventCreateWithFlags(&c->ev_copy0, cudaEventDisableTiming), "copy event");
            if (!rc) rc = cuda_check(c, cudaEventCreateWithFlags(&c->ev_copy, cudaEventDisableTiming), "copy event");
            if (rc) return rc;
        }
        if (c->d_f && c->f_cap < count) {
            rc = cuda_check(c, cudaStreamSynchronize(c->stream), "staging sync");
            if (rc) return rc;
            cudaFree(c->d_f);
            c->bytes -= sizeof(double2) * c->f_cap;
            c->d_f = nullptr;
            c->f_cap = 0;
        }
        if (!c->d_f) {
            rc = cuda_check(c, cudaMalloc((void **)&c->d_f, sizeof(double2) * count), "staging buffer");
            if (rc) return rc;
            c->bytes += sizeof(double2) * count;
            c->f_cap = count;
        }
    }
    int rc = ctx_setup_medium(c, s2, is_device_ptr(s2));
    if (!rc && pre) {
        // after the medium's upload and the context's earlier work on the
        // staging buffer (both on the context's stream)
        rc = cuda_check(c, cudaEventRecord(c->ev_copy0, c->stream), "copy order");
        if (!rc) rc = cuda_check(c, cudaStreamWaitEvent(c->copy_stream, c->ev_copy0, 0), "copy order");
        if (!rc)
            rc = cuda_check(c, cudaMemcpyAsync(c->d_f, f, sizeof(double2) * count, cudaMemcpyHostToDevice, c->copy_stream),
                            "copy in");
        if (!rc) rc = cuda_check(c, cudaEventRecord(c->ev_copy, c->copy_stream), "copy order");
        if (rc) {
            cudaStreamSynchronize(c->copy_stream);
            c->factor_rc = rc;
            return rc;
        }
    } else {
        pre = false;
    }
    if (!rc) rc = ctx_factor(c);
    c->factor_rc = rc;
    if (pre) {
        // the solve reads the copy on the context's stream; a failed factor
        // still waits for it, so that no copy outlives the call
        const int rc2 = cuda_check(c, cudaStreamWaitEvent(c->stream, c->ev_copy, 0), "copy order");
        if (rc) {
            cudaEventSynchronize(c->ev_copy);
            return rc;
        }
        if (rc2) {
            cudaEventSynchronize(c->ev_copy);
            return rc2;
        }
    }
    if (rc) return rc;
    rc = solve_common(c, pre ? (const double *)c->d_f : f, u, nrhs, st, 0);
    if (pre) cudaEventSynchronize(c->ev_copy);   // f is not read after the call returns
    return rc;
}

int helm3d_solve_group(helm3d_ctx *const *ctxs, int n, const double *const *f, double *const *u, const int *nrhs,
                       helm3d_stats *stats) {
    if (!ctxs || n < 1 || !f || !u || !nrhs) return HELM3D_ERR_ARG;
    for (int i = 0; i < n; i++) {
        helm3d_ctx *c = ctxs[i];
        if (!c) return HELM3D_ERR_ARG;
        if (!f[i] || !u[i] || nrhs[i] < 1) return set_error(c, HELM3D_ERR_ARG, "solve_group: bad vector arguments");
        if (c->device != ctxs[0]->device) return set_error(c, HELM3D_ERR_ARG, "solve_group: contexts on two devices");
        for (int q = 0; q < i; q++)
            if (ctxs[q] == c) return set_error(c, HELM3D_ERR_ARG, "solve_group: a context appears twice");
    }
    cudaSetDevice(ctxs[0]->device);
    // every context's work (staging included) on the first context's stream
    // for the call
    struct Guard {
        std::vector<helm3d_ctx *> cs;
        std::vector<cudaStream_t> saved;
        ~Guard() {
            for (size_t i = 0; i < cs.size(); i++) cs[i]->stream = saved[i];
        }
    } guard;
    for (int i = 0; i < n; i++) {
        guard.cs.push_back(ctxs[i]);
        guard.saved.push_back(ctxs[i]->stream);
        ctxs[i]->stream = ctxs[0]->stream;
        if (int rc = begin_call(ctxs[i])) return rc;
        if (stats) {
            helm3d_stats &s = stats[i];
            s.iterations = 0;
            s.restarts = 0;
            s.ms_solve = 0;
            s.relres = 0;
            s.relres_phys = 0;
            s.history_len = 0;
            s.status = HELM3D_OK;
        }
    }
    // batch per context, each sized after the earlier contexts' workspace
    std::vector<int> Bc(n);
    int rounds = 0;
    for (int i = 0; i < n; i++) {
        helm3d_ctx *c = ctxs[i];
        const bool staged = !is_device_ptr(f[i]) || !is_device_ptr(u[i]);
        Bc[i] = batch_size(c, nrhs[i], staged);
        int rc = ensure_krylov(c, std::max(1, c->opts.restart), Bc[i]);
        if (rc) return rc;
        rounds = std::max(rounds, (nrhs[i] + Bc[i] - 1) / Bc[i]);
    }
    int worst = HELM3D_OK;
    for (int t = 0; t < rounds; t++) {
        std::vector<helm3d_ctx *> cs;
        std::vector<const double2 *> fd;
        std::vector<double2 *> ud;
        std::vector<int> Rs;
        std::vector<helm3d_stats *> sts;
        std::vector<std::unique_ptr<VecArg>> fa, ua;
        std::vector<double *> uh;
        std::vector<size_t> counts;
        for (int i = 0; i < n; i++) {
            const int r0 = t * Bc[i];
            if (r0 >= nrhs[i]) continue;
            helm3d_ctx *c = ctxs[i];
            const int R = std::min(Bc[i], nrhs[i] - r0);
            const size_t count = (size_t)R * c->N;
            const double *fr = f[i] + 2 * (size_t)r0 * c->N;
            double *ur = u[i] + 2 * (size_t)r0 * c->N;
            fa.emplace_back(new VecArg(c, fr, count, true, &c->d_f, &c->f_cap));
            if (fa.back()->rc) return fa.back()->rc;
            ua.emplace_back(new VecArg(c, ur, count, false, &c->d_u, &c->u_cap));
            if (ua.back()->rc) return ua.back()->rc;
            cs.push_back(c);
            fd.push_back(fa.back()->dev);
            ud.push_back(ua.back()->dev);
            Rs.push_back(R);
            sts.push_back(stats ? &stats[i] : nullptr);
            uh.push_back(ur);
            counts.push_back(count);
        }
        int rc = fgmres_group(cs.data(), (int)cs.size(), fd.data(), ud.data(), Rs.data(), sts.data());
        if (rc && rc != HELM3D_ERR_NOT_CONVERGED) return rc;
        if (rc) worst = rc;
        for (size_t q = 0; q < cs.size(); q++) {
            if (sts[q] && rc) sts[q]->status = rc;
            const int rc2 = ua[q]->copy_out(uh[q], counts[q]);
            if (rc2) return rc2;
        }
    }
    return worst;
}

int helm3d_solve_bicgstab(helm3d_ctx *c, const double *f, double *u, helm3d_stats *st) {
    return solve_common(c, f, u, 1, st, 1);
}

int helm3d_solve_adjoint(helm3d_ctx *c, const double *g, double *lam, helm3d_stats *st) {
    if (c && c->opts.mode != HELM3D_MODE_N) return set_error(c, HELM3D_ERR_ARG, "adjoint solve is mode N only");
    return solve_common(c, g, lam, 1, st, 2);
}

// device memory released when the scope ends
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int alloc(helm3d_ctx *c, size_t bytes, const char *what) { return cuda_check(c, cudaMalloc(&p, bytes), what); }
};

static int apply_common(helm3d_ctx *c, const double *x, double *y, int which) {
    if (!c || !x || !y) return HELM3D_ERR_ARG;
    cudaSetDevice(c->device);
    if (int rc = begin_call(c)) return rc;
    VecArg xa(c, x, c->N, true, &c->d_f, &c->f_cap);
    if (xa.rc) return xa.rc;
    VecArg ya(c, y, c->N, false, &c->d_u, &c->u_cap);
    if (ya.rc) return ya.rc;
    const VecBatch xb{xa.dev, 0}, yb{ya.dev, 0};
    const ScaleBatch one{nullptr, 0};
    int rc;
    if (which == 0) rc = apply_op(c, xb, 1.0, one, yb, 1);
    else if (which == 1) rc = apply_op_adjoint(c, xb, 1.0, one, yb, 1);
    else if (which == 2) rc = apply_prec(c, xb, 1.0, one, yb, 1);
    else rc = apply_prec_adjoint(c, xb, 1.0, one, yb, 1);
    if (rc) return rc;
    rc = ya.copy_out(y, c->N);
    if (rc) return rc;
    return check_status(c);
}

int helm3d_apply_op(helm3d_ctx *c, const double *x, double *y) { return apply_common(c, x, y, 0); }
int helm3d_apply_op_adjoint(helm3d_ctx *c, const double *x, double *y) { return apply_common(c, x, y, 1); }
int helm3d_apply_prec(helm3d_ctx *c, const double *x, double *y) { return apply_common(c, x, y, 2); }
int helm3d_apply_prec_adjoint(helm3d_ctx *c, const double *x, double *y) { return apply_common(c, x, y, 3); }

int helm3d_apply_prec_batch(helm3d_ctx *c, const double *x, double *y, int nrhs, int adjoint) {
    if (!c || !x || !y) return HELM3D_ERR_ARG;
    if (nrhs < 1 || nrhs > kMaxBatch) return set_error(c, HELM3D_ERR_ARG, "apply_prec_batch: nrhs must be 1..16");
    if (adjoint && c->opts.mode != HELM3D_MODE_N)
        return set_error(c, HELM3D_ERR_ARG, "adjoint preconditioner is mode N only");
    cudaSetDevice(c->device);
    if (int rc = begin_call(c)) return rc;
    const size_t cnt = (size_t)c->N * nrhs;
    VecArg xa(c, x, cnt, true, &c->d_f, &c->f_cap);
    if (xa.rc) return xa.rc;
    VecArg ya(c, y, cnt, false, &c->d_u, &c->u_cap);
    if (ya.rc) return ya.rc;
    // the sweep shape: forced (HELM3D_FORCE_SWEEP), else the one the last
    // solve of this context was tuned to
    const int forced = tune_forced("SWEEP");
    if (forced >= 0) c->tv_sweep[adjoint ? 1 : 0] = forced < kSweepVariants ? forced : 0;
    const VecBatch xb{xa.dev, c->N}, yb{ya.dev, c->N};
    const ScaleBatch one{nullptr, 0};
    int rc = adjoint ? apply_prec_adjoint(c, xb, 1.0, one, yb, nrhs) : apply_prec(c, xb, 1.0, one, yb, nrhs);
    if (rc) return rc;
    rc = ya.copy_out(y, cnt);
    if (rc) return rc;
    return check_status(c);
}

int helm3d_misfit_grad(helm3d_ctx *c, const double *f, int nsrc, const long long *recv, int nrecv, const double *data,
                       double *grad, double *misfit, helm3d_stats *st) {
    if (!c) return HELM3D_ERR_ARG;
    if (!f || !grad || nsrc < 1 || nrecv < 0 || (nrecv > 0 && (!recv || !data)))
        return set_error(c, HELM3D_ERR_ARG, "misfit_grad: bad arguments");
    if (c->opts.mode != HELM3D_MODE_N) return set_error(c, HELM3D_ERR_ARG, "misfit gradient is mode N only");
    cudaSetDevice(c->device);
    if (int rc = begin_call(c)) return rc;
    if (st) {
        st->iterations = 0;
        st->restarts = 0;
        st->ms_solve = 0;
        st->relres = 0;
        st->relres_phys = 0;
        st->history_len = 0;
    }
    const long N = c->N;
    int rc;
    // receivers: checked on the host, used from the device
    std::vector<long long> hrecv((size_t)nrecv);
    DevBuf d_recv, d_data, d_grad, d_u, d_lam, d_adj, d_res;
    if (nrecv > 0) {
        if ((rc = cuda_check(c, cudaMemcpy(hrecv.data(), recv, sizeof(long long) * nrecv, cudaMemcpyDefault),
                             "receivers")))
            return rc;
        for (long long q : hrecv)
            if (q < 0 || q >= N) return set_error(c, HELM3D_ERR_ARG, "misfit_grad: receiver index out of range");
        if ((rc = d_recv.alloc(c, sizeof(long long) * nrecv, "receivers")) ||
            (rc = cuda_check(c, cudaMemcpy(d_recv.p, hrecv.data(), sizeof(long long) * nrecv, cudaMemcpyHostToDevice),
                             "receivers")))
            return rc;
    }
    const double2 *dd = (const double2 *)data;
    if (nrecv > 0 && !is_device_ptr(data)) {
        const size_t b = sizeof(double2) * (size_t)nsrc * nrecv;
        if ((rc = d_data.alloc(c, b, "data")) ||
            (rc = cuda_check(c, cudaMemcpy(d_data.p, data, b, cudaMemcpyHostToDevice), "data")))
            return rc;
        dd = (const double2 *)d_data.p;
    }
    const bool gdev = is_device_ptr(grad);
    double *g = grad;
    if (!gdev) {
        if ((rc = d_grad.alloc(c, sizeof(double) * N, "gradient"))) return rc;
        g = (double *)d_grad.p;
    }
    if ((rc = cuda_check(c, cudaMemsetAsync(g, 0, sizeof(double) * N, c->stream), "gradient zero"))) return rc;
    const bool fstaged = !is_device_ptr(f);
    const int B = batch_size(c, nsrc, fstaged, 3);
    const size_t vb = sizeof(double2) * (size_t)N;
    if ((rc = d_u.alloc(c, vb * B, "wavefields")) || (rc = d_lam.alloc(c, vb * B, "adjoint wavefields")) ||
        (rc = d_adj.alloc(c, vb * B, "adjoint sources")) ||
        (nrecv > 0 && (rc = d_res.alloc(c, sizeof(double2) * (size_t)B * nrecv, "receiver residuals"))))
        return rc;
    double2 *U = (double2 *)d_u.p, *Lam = (double2 *)d_lam.p, *Adj = (double2 *)d_adj.p, *Res = (double2 *)d_res.p;
    std::vector<double2> hres((size_t)B * std::max(nrecv, 0));
    const double w2 = c->grid.omega * c->grid.omega;
    double J = 0.0;
    int worst = HELM3D_OK;
    for (int r0 = 0; r0 < nsrc; r0 += B) {
        const int R = std::min(B, nsrc - r0);
        VecArg fa(c, f + 2 * (size_t)r0 * N, (size_t)R * N, true, &c->d_f, &c->f_cap);
        if (fa.rc) return fa.rc;
        // forward wavefields
        rc = fgmres(c, fa.dev, U, R, false, st);
        if (rc && rc != HELM3D_ERR_NOT_CONVERGED) return rc;
        if (rc) worst = rc;
        // receiver residuals P u - d, misfit, adjoint sources P^T (d - P u)
        if ((rc = cuda_check(c, cudaMemsetAsync(Adj, 0, vb * R, c->stream), "adjoint source zero"))) return rc;
        if (nrecv > 0) {
            rc = timed(c, HELM3D_K_KRYLOV, 2, [&] {
                int r1 = launch_receiver_residual(VecBatch{U, N}, R, (const long long *)d_recv.p, nrecv,
                                                  dd + (size_t)r0 * nrecv, nrecv, Res, c->stream);
                if (r1) return r1;
                return launch_adjoint_source(Res, R, (const long long *)d_recv.p, nrecv, -1.0, VecBatch{Adj, N},
                                             c->stream);
            });
            if (rc) return set_error(c, rc, "misfit_grad: receiver kernels");
            if ((rc = cuda_check(c, cudaMemcpyAsync(hres.data(), Res, sizeof(double2) * (size_t)R * nrecv,
                                                    cudaMemcpyDeviceToHost, c->stream),
                                 "residuals")) ||
                (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "residuals")))
                return rc;
            for (size_t q = 0; q < (size_t)R * nrecv; q++) J += 0.5 * (hres[q].x * hres[q].x + hres[q].y * hres[q].y);
        }
        // adjoint wavefields A^H lam = P^T (d - P u)
        rc = fgmres(c, Adj, Lam, R, true, st);
        if (rc && rc != HELM3D_ERR_NOT_CONVERGED) return rc;
        if (rc) worst = rc;
        rc = timed(c, HELM3D_K_KRYLOV, 1, [&] {
            return launch_grad_accum(VecBatch{Lam, N}, VecBatch{U, N}, R, w2, c->opts.beta_phys, g, N, c->stream);
        });
        if (rc) return set_error(c, rc, "misfit_grad: gradient kernel");
    }
    if (!gdev && (rc = cuda_check(c, cudaMemcpyAsync(grad, g, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream),
                                  "gradient out")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "misfit_grad"))) return rc;
    if (misfit) *misfit = J;
    if (st) st->status = worst;
    return worst;
}

int helm3d_destroy(helm3d_ctx *c) {
    if (!c) return HELM3D_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *bufs[] = {c->d_Gt, c->d_gscale, c->d_gpack, c->d_kzslot, c->d_kzlist, c->d_kzinv, c->d_tw, c->d_cmx, c->d_cpx, c->d_cmy, c->d_cpy, c->d_base2d, c->d_kz2, c->d_zW, c->d_zWi, c->d_zW64, c->d_zWi64, c->d_zWH64, c->d_zWiH64, c->d_dxy,
                    c->d_cmx64, c->d_cpx64, c->d_cmy64, c->d_cpy64, c->d_cmz64, c->d_cpz64, c->d_s2, c->d_dl,
                    c->d_planes, c->d_status, c->d_V, c->d_Z, c->d_vs, c->d_h, c->d_partials, c->d_f, c->d_u,
                    c->d_r, c->d_t, c->d_t2, c->d_bic, c->d_Fw, c->d_Uw};
    for (void *p : bufs)
        if (p) cudaFree(p);
    for (float *p : c->d_ztc)
        if (p) cudaFree(p);
    for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
    if (c->d_arn) cudaFree(c->d_arn);
    for (auto &e : c->prof_ev) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    if (c->h_scal) cudaFreeHost(c->h_scal);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->ev_copy0) cudaEventDestroy(c->ev_copy0);
    if (c->ev_copy) cudaEventDestroy(c->ev_copy);
    delete c;
    return HELM3D_OK;
}

}  // extern "C"
