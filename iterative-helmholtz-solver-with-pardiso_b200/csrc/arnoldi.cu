// arnoldi.cu -- the per-step bookkeeping of the lockstep batched FGMRES on
// the device: the Gram-Schmidt second-pass test, the Givens update of the
// Hessenberg column and the right-hand side g, the convergence estimate, and
// the back substitution y = R^{-1} g at the end of a cycle.  One thread per
// right-hand side (a batch holds at most 16); the arithmetic is the host
// loop's (FGMRES restart cycle, Source/FGMRES.cpp:464-684, with Givens
// rotations in place of the per-step zgels) in the same order, in FP64.
//
// These kernels let a whole restart cycle run as one CUDA graph: the Givens
// kernel of step j decides, on the device, whether step j + 1 runs (graph
// conditional node) -- it runs while some right-hand side of the batch has
// not converged, reached the iteration limit or broken down.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

constexpr int kArnThreads = 32;   // >= kMaxBatch

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cmag(double2 a) { return hypot(a.x, a.y); }

__global__ void __launch_bounds__(kArnThreads) reorth_check_kernel(ArnState a, int j) {
    const int p = threadIdx.x;
    int need = 0;
    if (p < a.B && !a.frozen[p]) {
        const double2 *h = a.h + (long)p * a.SH;
        need = h[2 * a.M2].x < H3D_REORTH_ETA2 * h[j + 1].x;
    }
    need = __syncthreads_or(need);
    if (p == 0) {
        a.flags[0] = need;
        if (need) a.flags[1] += 1;
    }
}

// Column j of H holds V^H w above the diagonal and H[j+1][j] below it
// (unrotated): apply the earlier rotations, make rotation j, update g, the
// iteration count and the estimate; returns whether right-hand side p stops
// (converged, iteration limit, breakdown or non-finite).
__device__ bool finalize_column(const ArnState &a, int p, int j) {
    const int m = a.m;
    double2 *H = a.H + (long)p * (m + 1) * m;
    double2 *cs = a.cs + (long)p * m, *sn = a.sn + (long)p * m, *g = a.g + (long)p * (m + 1);
    const double hn = cmag(H[(long)(j + 1) * m + j]);
    for (int i = 0; i < j; i++) {
        const double2 x = H[(long)i * m + j], y = H[(long)(i + 1) * m + j];
        H[(long)i * m + j] = cadd(cmul(cs[i], x), cmul(sn[i], y));
        H[(long)(i + 1) * m + j] = csub(cmul(cs[i], y), cmul(cconj(sn[i]), x));
    }
    const double2 x = H[(long)j * m + j], y = H[(long)(j + 1) * m + j];
    const double ax = cmag(x), den = hypot(ax, cmag(y));
    double2 c, s;
    if (den == 0.0) {
        c = make_double2(1, 0);
        s = make_double2(0, 0);
    } else if (ax == 0.0) {
        c = make_double2(0, 0);
        s = make_double2(1, 0);
    } else {
        c = make_double2(ax / den, 0.0);
        // (x / |x|) conj(y) / den
        s = cmul(make_double2(x.x / ax, x.y / ax), cconj(y));
        s = make_double2(s.x / den, s.y / den);
    }
    cs[j] = c;
    sn[j] = s;
    H[(long)j * m + j] = cadd(cmul(c, x), cmul(s, y));
    H[(long)(j + 1) * m + j] = make_double2(0, 0);
    const double2 gj = g[j];
    g[j + 1] = make_double2(-(s.x * gj.x + s.y * gj.y), -(s.x * gj.y - s.y * gj.x));   // -conj(s) g[j]
    g[j] = cmul(c, gj);
    const int it = a.it[p] + 1;
    a.it[p] = it;
    a.k[p] = j + 1;
    const double est = cmag(g[j + 1]) / a.nf[p];
    a.est[(long)p * m + j] = est;
    const bool bad = !isfinite(hn) || !isfinite(est);
    if (bad) atomicOr(&a.flags[3], 1);
    const bool frozen = bad || hn == 0.0 || est <= a.tol[p] || it >= a.max_iter[p];
    a.frozen[p] = frozen ? 1 : 0;
    return frozen;
}

__global__ void __launch_bounds__(kArnThreads) givens_kernel(ArnState a, int j, int has_next,
                                                             cudaGraphConditionalHandle next) {
    const int p = threadIdx.x;
    const int m = a.m;
    int active = 0;
    // a right-hand side that has stopped gets zero scales: its further basis
    // vectors are exact zeros (the zero-padded combine then adds nothing)
    if (p < a.B && a.frozen[p]) a.vs[(long)p * a.M2 + j + 1] = 0.0;
    if (p < a.B && !a.frozen[p]) {
        const double2 *h1 = a.h + (long)p * a.SH, *h2 = h1 + a.M2;
        const bool second = a.flags[0] != 0;
        double2 *H = a.H + (long)p * (m + 1) * m;
        const double hn = sqrt(fmax(0.0, h1[2 * a.M2].x));
        // column j: V^H w (both passes), then ||w|| below the diagonal
        for (int i = 0; i <= j; i++) H[(long)i * m + j] = second ? cadd(h1[i], h2[i]) : h1[i];
        H[(long)(j + 1) * m + j] = make_double2(hn, 0.0);
        const bool frozen = finalize_column(a, p, j);
        a.vs[(long)p * a.M2 + j + 1] = (!frozen && hn > 0.0) ? 1.0 / hn : 0.0;
        active = !frozen;
    }
    active = __syncthreads_or(active);
    if (p == 0) {
        a.flags[4] = j;
        a.flags[5] = active;
        if (has_next) cudaGraphSetConditional(next, active ? 1u : 0u);
    }
}

// ------------------------------------------------ DCGS2 (mode N, flexible)
// Step j computed w = A z_j with z_j = M^{-1} (vs_j V_j), where V_j is still
// the tentative vector of step j - 1 (projected once).  From the one
// reduction of dots2 this kernel
//   * reorthogonalizes V_j: s_i = a_i vs_j, nrm^2 = g vs_j^2 - sum |s_i|^2;
//   * finalizes column j - 1, whose subdiagonal was left open: with
//     beta = ||w_{j-1}'|| of the last update, H[i][j-1] += beta s_i and
//     H[j][j-1] = beta nrm, then its Givens rotation (convergence is known
//     one step late);
//   * writes column j (unrotated) against the final basis: c_i = b_i (i < j),
//     c_j = (b_j - sum conj(s_i) b_i) / nrm;
//   * writes the update coefficients in stored-vector terms (alpha for V_j,
//     delta for w) and the new scale of V_j.
// Frozen right-hand sides are skipped by the passes that follow.
__global__ void __launch_bounds__(kArnThreads) lagged_kernel(ArnState a, int j) {
    const int p = threadIdx.x;
    if (p >= a.B || a.frozen[p]) return;
    const int m = a.m, M2 = a.M2;
    double2 *hp = a.h + (long)p * a.SH;
    const double2 *b = hp, *av = hp + j + 1;
    double2 *alpha = hp + 4 * M2, *delta = hp + 5 * M2;
    double *vs = a.vs + (long)p * M2;
    double2 *H = a.H + (long)p * (m + 1) * m;
    const double sj = vs[j];
    double nrm = 1.0;
    if (j > 0) {
        double ss = 0.0;
        for (int i = 0; i < j; i++) {
            const double2 si = cscale(av[i], sj);
            ss += si.x * si.x + si.y * si.y;
        }
        const double n2 = hp[2 * j + 1].x * sj * sj - ss;
        nrm = n2 > 0.0 ? sqrt(n2) : 0.0;
        const double beta = a.beta[p];
        for (int i = 0; i < j; i++) {
            const double2 si = cscale(av[i], sj);
            H[(long)i * m + j - 1] = cadd(H[(long)i * m + j - 1], cscale(si, beta));
        }
        H[(long)j * m + j - 1] = make_double2(beta * nrm, 0.0);
        if (finalize_column(a, p, j - 1)) return;
    }
    // nrm > 0 here: nrm = 0 makes H[j][j-1] = 0, a breakdown that stops p
    double2 cj = b[j];
    for (int i = 0; i < j; i++) cj = csub(cj, cmul(cconj(cscale(av[i], sj)), b[i]));
    cj = cscale(cj, 1.0 / nrm);
    for (int i = 0; i < j; i++) H[(long)i * m + j] = b[i];
    H[(long)j * m + j] = cj;
    const double2 cn = cscale(cj, 1.0 / nrm);
    for (int i = 0; i < j; i++) {
        const double2 si = cscale(av[i], sj);
        alpha[i] = cscale(si, vs[i] / sj);
        delta[i] = cscale(csub(b[i], cmul(cn, si)), vs[i]);
    }
    delta[j] = cscale(cj, sj / nrm);
    if (j > 0) vs[j] = sj / nrm;
}

// After the update pass of step j: beta = ||w'||, the scale of the new
// tentative vector V_{j+1}, the breakdown and non-finite checks, and whether
// step j + 1 runs (some right-hand side still active).
__global__ void __launch_bounds__(kArnThreads) post_kernel(ArnState a, int j, int has_next,
                                                           cudaGraphConditionalHandle next) {
    const int p = threadIdx.x;
    int active = 0;
    if (p < a.B) {
        double *vs = a.vs + (long)p * a.M2;
        if (a.frozen[p]) {
            vs[j + 1] = 0.0;
        } else {
            const double beta = sqrt(fmax(0.0, a.h[(long)p * a.SH + 2 * a.M2].x));
            if (!isfinite(beta)) {
                atomicOr(&a.flags[3], 1);
                a.frozen[p] = 1;
                vs[j + 1] = 0.0;
            } else {
                a.beta[p] = beta;
                vs[j + 1] = beta > 0.0 ? 1.0 / beta : 0.0;
                active = 1;
            }
        }
    }
    active = __syncthreads_or(active);
    if (p == 0) {
        a.flags[4] = j;
        a.flags[5] = active;
        if (has_next) cudaGraphSetConditional(next, active ? 1u : 0u);
    }
}

// End of a cycle: the open column jl = flags[4] of every still active
// right-hand side, from the reorthogonalization dots of V_{jl+1} (a_i at
// slots 0 .. jl, g at jl + 1).
__global__ void __launch_bounds__(kArnThreads) lagged_final_kernel(ArnState a) {
    const int p = threadIdx.x;
    if (p >= a.B || a.frozen[p] || !a.flags[5]) return;
    const int m = a.m, jl = a.flags[4], t = jl + 1;
    const double2 *hp = a.h + (long)p * a.SH;
    const double st = a.vs[(long)p * a.M2 + t];
    double2 *H = a.H + (long)p * (m + 1) * m;
    double ss = 0.0;
    for (int i = 0; i <= jl; i++) {
        const double2 si = cscale(hp[i], st);
        ss += si.x * si.x + si.y * si.y;
    }
    const double n2 = hp[t].x * st * st - ss;
    const double nrm = n2 > 0.0 ? sqrt(n2) : 0.0;
    const double beta = a.beta[p];
    for (int i = 0; i <= jl; i++)
        H[(long)i * m + jl] = cadd(H[(long)i * m + jl], cscale(cscale(hp[i], st), beta));
    H[(long)t * m + jl] = make_double2(beta * nrm, 0.0);
    finalize_column(a, p, jl);
    a.frozen[p] = 1;
}

__global__ void __launch_bounds__(kArnThreads) backsub_kernel(ArnState a) {
    const int p = threadIdx.x;
    const int m = a.m;
    int k = 0;
    if (p < a.B) {
        k = a.k[p];
        const double2 *H = a.H + (long)p * (m + 1) * m, *g = a.g + (long)p * (m + 1);
        double2 *y = a.h + (long)p * a.SH + 3 * a.M2;
        for (int i = k - 1; i >= 0; i--) {
            double2 s = g[i];
            for (int q = i + 1; q < k; q++) s = csub(s, cmul(H[(long)i * m + q], y[q]));
            y[i] = cmul(s, cinv(H[(long)i * m + i]));
        }
        for (int i = k; i < m; i++) y[i] = make_double2(0, 0);
    }
    // longest column count of the batch (kArnThreads lanes, one warp)
    for (int off = 16; off > 0; off >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, off));
    if (p == 0) a.flags[2] = k;
}

static inline int ok() { return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA; }

int launch_reorth_check(const ArnState &a, int j, cudaStream_t s) {
    reorth_check_kernel<<<1, kArnThreads, 0, s>>>(a, j);
    return ok();
}

int launch_givens(const ArnState &a, int j, bool has_next, cudaGraphConditionalHandle next, cudaStream_t s) {
    givens_kernel<<<1, kArnThreads, 0, s>>>(a, j, has_next ? 1 : 0, next);
    return ok();
}

int launch_lagged(const ArnState &a, int j, cudaStream_t s) {
    lagged_kernel<<<1, kArnThreads, 0, s>>>(a, j);
    return ok();
}

int launch_post(const ArnState &a, int j, bool has_next, cudaGraphConditionalHandle next, cudaStream_t s) {
    post_kernel<<<1, kArnThreads, 0, s>>>(a, j, has_next ? 1 : 0, next);
    return ok();
}

int launch_lagged_final(const ArnState &a, cudaStream_t s) {
    lagged_final_kernel<<<1, kArnThreads, 0, s>>>(a);
    return ok();
}

int launch_backsub(const ArnState &a, cudaStream_t s) {
    backsub_kernel<<<1, kArnThreads, 0, s>>>(a);
    return ok();
}

}  // namespace h3d
