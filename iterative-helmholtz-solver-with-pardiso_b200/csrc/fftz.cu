// fftz.cu -- batched complex FFT along z (stride nx*ny), replacing the
// reference's nx*ny separate strided DFTI calls (Source/functions.cpp:
// 5858-5881, 6041-6046): forward unscaled, backward scaled 1/nz.
//
// One CTA owns TW consecutive z-columns (w = i + nx*j) and all nz rows.
// Loads and stores move whole rows of TW columns (coalesced, 512 B per warp
// for complex128).  The transform runs in shared memory as a mixed-radix
// Stockham sequence of passes (ping-pong buffers, natural order out): pass s
// with radix r and span p maps task i (k = i mod p) to
//     u_q = x[i + q*(n/r)] * w_{p r}^{q k},   U = DFT_r(u),
//     y[(i - k) r + k + q p] = U_q.
// Radices 2..8 are unrolled; any other prime factor uses a generic loop.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

struct FftK {
    int n, npass;
    int radix[kMaxPasses];
    int span[kMaxPasses];
    int twoff[kMaxPasses];
    int dftoff[kMaxPasses];
};

template <typename R, bool INV>
__device__ __forceinline__ cplx<R> tw_load(const cplx<R> *tw, int idx) {
    cplx<R> t = tw[idx];
    if (INV) t.y = -t.y;
    return t;
}

template <typename R, int RR, bool INV, int TW>
__device__ __forceinline__ void radix_task(const cplx<R> *__restrict__ src, cplx<R> *__restrict__ dst,
                                           const cplx<R> *__restrict__ tw, int twoff, int dftoff, int i,
                                           int m, int p, int col) {
    const int k = i % p;
    const int j = (i - k) * RR + k;
    cplx<R> u[RR];
#pragma unroll
    for (int q = 0; q < RR; q++) u[q] = src[(i + q * m) * TW + col];
    if (p > 1) {
#pragma unroll
        for (int q = 1; q < RR; q++) u[q] = cmul(u[q], tw_load<R, INV>(tw, twoff + k * RR + q));
    }
    cplx<R> U[RR];
    if (RR == 2) {
        U[0] = cadd(u[0], u[1]);
        U[1] = csub(u[0], u[1]);
    } else if (RR == 4) {
        cplx<R> a = cadd(u[0], u[2]), b = csub(u[0], u[2]);
        cplx<R> c = cadd(u[1], u[3]), d = csub(u[1], u[3]);
        // -i*d (forward) or +i*d (inverse)
        cplx<R> e = INV ? mkc<R>(-d.y, d.x) : mkc<R>(d.y, -d.x);
        U[0] = cadd(a, c);
        U[2] = csub(a, c);
        U[1] = cadd(b, e);
        U[3] = csub(b, e);
    } else {
#pragma unroll
        for (int q = 0; q < RR; q++) {
            cplx<R> acc = u[0];
#pragma unroll
            for (int t = 1; t < RR; t++) acc = cfma(u[t], tw_load<R, INV>(tw, dftoff + (q * t) % RR), acc);
            U[q] = acc;
        }
    }
#pragma unroll
    for (int q = 0; q < RR; q++) dst[(j + q * p) * TW + col] = U[q];
}

template <typename R, bool INV, int TW>
__device__ void radix_task_generic(const cplx<R> *__restrict__ src, cplx<R> *__restrict__ dst,
                                   const cplx<R> *__restrict__ tw, int twoff, int dftoff, int r, int i, int m,
                                   int p, int col) {
    const int k = i % p;
    const int j = (i - k) * r + k;
    for (int q = 0; q < r; q++) {
        cplx<R> acc = mkc<R>(0, 0);
        for (int t = 0; t < r; t++) {
            cplx<R> ut = src[(i + t * m) * TW + col];
            if (p > 1 && t > 0) ut = cmul(ut, tw_load<R, INV>(tw, twoff + k * r + t));
            acc = cfma(ut, tw_load<R, INV>(tw, dftoff + (q * t) % r), acc);
        }
        dst[(j + q * p) * TW + col] = acc;
    }
}

template <typename R, bool INV, int TW>
__device__ cplx<R> *fft_passes(cplx<R> *A, cplx<R> *B, const FftK &fp, const cplx<R> *tw, int col, int grp,
                               int ngrp) {
    cplx<R> *src = A, *dst = B;
    for (int s = 0; s < fp.npass; s++) {
        const int r = fp.radix[s], p = fp.span[s], m = fp.n / r;
        const int to = fp.twoff[s], dof = fp.dftoff[s];
        for (int i = grp; i < m; i += ngrp) {
            switch (r) {
                case 2: radix_task<R, 2, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                case 3: radix_task<R, 3, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                case 4: radix_task<R, 4, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                case 5: radix_task<R, 5, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                case 7: radix_task<R, 7, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                case 8: radix_task<R, 8, INV, TW>(src, dst, tw, to, dof, i, m, p, col); break;
                default: radix_task_generic<R, INV, TW>(src, dst, tw, to, dof, r, i, m, p, col); break;
            }
        }
        __syncthreads();
        cplx<R> *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

constexpr int kFftThreads = 256;

// plane index of (row k, column w = i + nx*j) for right-hand side r
__device__ __forceinline__ long plane_index(const PlaneLayout &L, int r, int k, long w) {
    const long j = w / L.nx, i = w - j * L.nx;
    return (long)k * L.plane * L.R + (j * L.R + r) * L.nx + i;
}

template <typename R, int TW>
__global__ void __launch_bounds__(kFftThreads) fftz_forward_kernel(FftK fp, VecBatch x, double scale, ScaleBatch sc,
                                                                   cplx<R> *__restrict__ out, PlaneLayout L,
                                                                   const cplx<R> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smem_raw);
    cplx<R> *B = A + (size_t)fp.n * TW;
    const int col = threadIdx.x % TW, grp = threadIdx.x / TW, ngrp = kFftThreads / TW;
    const int r = blockIdx.y;
    const long plane = L.plane;
    const double2 *xr = x.p + r * x.stride;
    const double s = scale * (sc.p ? sc.p[r * sc.stride] : 1.0);
    const long w = (long)blockIdx.x * TW + col;
    const bool valid = w < plane;
    for (int row = grp; row < fp.n; row += ngrp) {
        double2 v = valid ? xr[(long)row * plane + w] : make_double2(0.0, 0.0);
        A[row * TW + col] = cvt<cplx<R>, double2>(make_double2(v.x * s, v.y * s));
    }
    __syncthreads();
    cplx<R> *res = fft_passes<R, false, TW>(A, B, fp, tw, col, grp, ngrp);
    if (valid)
        for (int row = grp; row < fp.n; row += ngrp) out[plane_index(L, r, row, w)] = res[row * TW + col];
}

template <typename R, int TW>
__global__ void __launch_bounds__(kFftThreads) fftz_inverse_kernel(FftK fp, const cplx<R> *__restrict__ in,
                                                                   PlaneLayout L, VecBatch y,
                                                                   const cplx<R> *__restrict__ tw, int mode,
                                                                   VecBatch wv, double scale, ScaleBatch sc,
                                                                   const double2 *__restrict__ dl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smem_raw);
    cplx<R> *B = A + (size_t)fp.n * TW;
    const int col = threadIdx.x % TW, grp = threadIdx.x / TW, ngrp = kFftThreads / TW;
    const int r = blockIdx.y;
    const long plane = L.plane;
    const long w = (long)blockIdx.x * TW + col;
    const bool valid = w < plane;
    for (int row = grp; row < fp.n; row += ngrp)
        A[row * TW + col] = valid ? in[plane_index(L, r, row, w)] : mkc<R>(0, 0);
    __syncthreads();
    cplx<R> *res = fft_passes<R, true, TW>(A, B, fp, tw, col, grp, ngrp);
    if (!valid) return;
    const double inv_n = 1.0 / (double)fp.n;
    double2 *yr = y.p + r * y.stride;
    const double2 *wr = mode == 1 ? wv.p + r * wv.stride : nullptr;
    const double s = scale * (sc.p ? sc.p[r * sc.stride] : 1.0);
    for (int row = grp; row < fp.n; row += ngrp) {
        const long idx = (long)row * plane + w;
        double2 t = cvt<double2, cplx<R>>(res[row * TW + col]);
        t.x *= inv_n;
        t.y *= inv_n;
        if (mode == 1) {
            const double2 a = wr[idx], d = dl[idx];
            t = make_double2(s * a.x - (d.x * t.x - d.y * t.y), s * a.y - (d.x * t.y + d.y * t.x));
        }
        if (y.c64) reinterpret_cast<float2 *>(y.p)[r * y.stride + idx] = cvt<float2, double2>(t);
        else yr[idx] = t;
    }
}

static FftK to_k(const FftPlan &p) {
    FftK k;
    k.n = p.n;
    k.npass = p.npass;
    for (int s = 0; s < kMaxPasses; s++) {
        k.radix[s] = p.radix[s];
        k.span[s] = p.span[s];
        k.twoff[s] = p.twoff[s];
        k.dftoff[s] = p.dftoff[s];
    }
    return k;
}

template <typename R> static int pick_tw(int n) {
    // two buffers of n x TW elements must fit the opt-in shared memory
    const size_t cap = device_info().smem_optin;
    if ((size_t)2 * n * 32 * sizeof(cplx<R>) <= cap) return 32;
    if ((size_t)2 * n * 16 * sizeof(cplx<R>) <= cap) return 16;
    return 0;
}

template <typename R, int TW>
static int fwd_impl(const VecBatch &x, double scale, const ScaleBatch &sc, void *planes, const PlaneLayout &L,
                    const FftPlan &plan, const void *tw, cudaStream_t s) {
    size_t smem = (size_t)2 * plan.n * TW * sizeof(cplx<R>);
    auto kern = fftz_forward_kernel<R, TW>;
    if (!smem_limit_max(kern, smem))
        return HELM3D_ERR_CUDA;
    dim3 grid((unsigned)((L.plane + TW - 1) / TW), (unsigned)L.R);
    kern<<<grid, kFftThreads, smem, s>>>(to_k(plan), x, scale, sc, (cplx<R> *)planes, L, (const cplx<R> *)tw);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

template <typename R, int TW>
static int inv_impl(const void *planes, const PlaneLayout &L, const VecBatch &y, const FftPlan &plan, const void *tw,
                    int mode, const VecBatch &w, double scale, const ScaleBatch &sc, const double2 *dl,
                    cudaStream_t s) {
    size_t smem = (size_t)2 * plan.n * TW * sizeof(cplx<R>);
    auto kern = fftz_inverse_kernel<R, TW>;
    if (!smem_limit_max(kern, smem))
        return HELM3D_ERR_CUDA;
    dim3 grid((unsigned)((L.plane + TW - 1) / TW), (unsigned)L.R);
    kern<<<grid, kFftThreads, smem, s>>>(to_k(plan), (const cplx<R> *)planes, L, y, (const cplx<R> *)tw, mode, w,
                                         scale, sc, dl);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_fft_forward(bool c64, const VecBatch &x, double scale, const ScaleBatch &sc, void *planes,
                       const PlaneLayout &L, const FftPlan &plan, const void *tw, cudaStream_t s) {
    if (c64) {
        int tw_ = pick_tw<float>(plan.n);
        if (tw_ == 32) return fwd_impl<float, 32>(x, scale, sc, planes, L, plan, tw, s);
        if (tw_ == 16) return fwd_impl<float, 16>(x, scale, sc, planes, L, plan, tw, s);
    } else {
        int tw_ = pick_tw<double>(plan.n);
        if (tw_ == 32) return fwd_impl<double, 32>(x, scale, sc, planes, L, plan, tw, s);
        if (tw_ == 16) return fwd_impl<double, 16>(x, scale, sc, planes, L, plan, tw, s);
    }
    return HELM3D_ERR_ARG;
}

int launch_fft_inverse(bool c64, const void *planes, const PlaneLayout &L, const VecBatch &y, const FftPlan &plan,
                       const void *tw, int mode, const VecBatch &w, double scale, const ScaleBatch &sc,
                       const double2 *dl, cudaStream_t s) {
    if (c64) {
        int tw_ = pick_tw<float>(plan.n);
        if (tw_ == 32) return inv_impl<float, 32>(planes, L, y, plan, tw, mode, w, scale, sc, dl, s);
        if (tw_ == 16) return inv_impl<float, 16>(planes, L, y, plan, tw, mode, w, scale, sc, dl, s);
    } else {
        int tw_ = pick_tw<double>(plan.n);
        if (tw_ == 32) return inv_impl<double, 32>(planes, L, y, plan, tw, mode, w, scale, sc, dl, s);
        if (tw_ == 16) return inv_impl<double, 16>(planes, L, y, plan, tw, mode, w, scale, sc, dl, s);
    }
    return HELM3D_ERR_ARG;
}

}  // namespace h3d
