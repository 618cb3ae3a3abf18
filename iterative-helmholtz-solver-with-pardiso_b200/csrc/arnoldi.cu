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
        double2 *cs = a.cs + (long)p * m, *sn = a.sn + (long)p * m, *g = a.g + (long)p * (m + 1);
        const double hn = sqrt(fmax(0.0, h1[2 * a.M2].x));
        // column j: V^H w (both passes), then ||w|| below the diagonal
        for (int i = 0; i <= j; i++) H[(long)i * m + j] = second ? cadd(h1[i], h2[i]) : h1[i];
        H[(long)(j + 1) * m + j] = make_double2(hn, 0.0);
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
        a.vs[(long)p * a.M2 + j + 1] = (!frozen && hn > 0.0) ? 1.0 / hn : 0.0;
        active = !frozen;
    }
    active = __syncthreads_or(active);
    if (p == 0 && has_next) cudaGraphSetConditional(next, active ? 1u : 0u);
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

int launch_backsub(const ArnState &a, cudaStream_t s) {
    backsub_kernel<<<1, kArnThreads, 0, s>>>(a);
    return ok();
}

}  // namespace h3d
