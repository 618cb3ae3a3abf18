// krylov.cu -- complex128 vector kernels of the outer Krylov loop: the
// Gram-Schmidt dot products and updates (the reference's zdotc/zaxpy loop,
// Source/FGMRES.cpp:508-517), norms (dznrm2, :519; the physical-domain norm
// after reducePML3D, :590-592), the solution update x = x0 + Z y (zgemv,
// :575) and small helpers.  Every kernel takes a batch of R right-hand sides
// (blockIdx.y = r, per-r pointer strides).  Reductions are two-level and
// deterministic: fixed-size per-block partials, then one pass over the blocks.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

constexpr int kRedThreads = 256;
constexpr int kDotChunk = 8;

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    }
    return v;
}

// block sum of CH complex values per thread; result valid in thread 0
template <int CH> __device__ __forceinline__ void block_sum(double2 (&acc)[CH], double2 *sh /* [8][CH] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < CH; q++) acc[q] = warp_sum(acc[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < CH; q++) sh[warp * CH + q] = acc[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kRedThreads / 32; w++)
#pragma unroll
            for (int q = 0; q < CH; q++) {
                acc[q].x += sh[w * CH + q].x;
                acc[q].y += sh[w * CH + q].y;
            }
    }
    __syncthreads();
}

// partials[r][b][i] = sum over this block's l of conj(V_i[l]) w[l] * vs[i]
// (i < nv); with wnorm, partials[r][b][nv].x = sum |w[l]|^2 as well
__global__ void __launch_bounds__(kRedThreads) dots_kernel(const double2 *__restrict__ V, long ldv, long sV,
                                                           const double *__restrict__ vs, long sVs, int nv,
                                                           const double2 *__restrict__ w, long sW, long N, int wnorm,
                                                           double2 *__restrict__ partials, int cap, const int *pred) {
    __shared__ double2 sh[(kRedThreads / 32) * (kDotChunk + 1)];
    if (pred && *pred == 0) return;
    const int r = blockIdx.y;
    V += r * sV;
    w += r * sW;
    if (vs) vs += r * sVs;
    partials += (long)r * gridDim.x * cap;
    const long stride = (long)gridDim.x * blockDim.x;
    for (int c0 = 0; c0 < nv || (c0 == 0 && wnorm); c0 += kDotChunk) {
        double2 acc[kDotChunk + 1];
#pragma unroll
        for (int q = 0; q <= kDotChunk; q++) acc[q] = make_double2(0, 0);
        const bool with_norm = wnorm && c0 == 0;
        for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
            const double2 wl = w[l];
#pragma unroll
            for (int q = 0; q < kDotChunk; q++)
                if (c0 + q < nv) acc[q] = cfma(make_double2(V[(c0 + q) * ldv + l].x, -V[(c0 + q) * ldv + l].y), wl, acc[q]);
            if (with_norm) acc[kDotChunk].x += wl.x * wl.x + wl.y * wl.y;
        }
        block_sum<kDotChunk + 1>(acc, sh);
        if (threadIdx.x == 0) {
            for (int q = 0; q < kDotChunk && c0 + q < nv; q++)
                partials[(long)blockIdx.x * cap + c0 + q] = cscale(acc[q], vs ? vs[c0 + q] : 1.0);
            if (with_norm) partials[(long)blockIdx.x * cap + nv] = acc[kDotChunk];
        }
    }
}

// Low-synchronization Gram-Schmidt (DCGS2, delayed reorthogonalization): one
// pass over V_0 .. V_j and the new vector w gives, per right-hand side,
//   slots 0 .. j       b_i = vs_i <V_i, w>      (i <= j)
//   slots j+1 .. 2j    a_i = vs_i <V_i, V_j>    (i < j: the lagged second
//                                                projection of V_j)
//   slot 2j+1          g   = <V_j, V_j>
// A right-hand side with skip[r] set writes zero partials and reads nothing.
__global__ void __launch_bounds__(kRedThreads) dots2_kernel(const double2 *__restrict__ V, long ldv, long sV,
                                                            const double *__restrict__ vs, long sVs, int j,
                                                            const double2 *__restrict__ w, long sW, long N,
                                                            double2 *__restrict__ partials, int cap,
                                                            const int *pred, const int *skip) {
    __shared__ double2 sh[(kRedThreads / 32) * (2 * kDotChunk + 2)];
    if (pred && *pred == 0) return;
    const int r = blockIdx.y;
    partials += (long)r * gridDim.x * cap + (long)blockIdx.x * cap;
    if (skip && skip[r]) {
        for (int q = threadIdx.x; q < 2 * j + 2; q += blockDim.x) partials[q] = make_double2(0, 0);
        return;
    }
    V += r * sV;
    w += r * sW;
    vs += r * sVs;
    const double2 *__restrict__ vj = V + (long)j * ldv;
    const long stride = (long)gridDim.x * blockDim.x;
    for (int c0 = 0; c0 < j || c0 == 0; c0 += kDotChunk) {
        // acc[q]: <V_{c0+q}, w>; acc[kDotChunk+q]: <V_{c0+q}, V_j>; then <V_j, w>, |V_j|^2
        double2 acc[2 * kDotChunk + 2];
#pragma unroll
        for (int q = 0; q < 2 * kDotChunk + 2; q++) acc[q] = make_double2(0, 0);
        const bool first = c0 == 0;
        for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
            const double2 wl = w[l], xl = vj[l];
#pragma unroll
            for (int q = 0; q < kDotChunk; q++)
                if (c0 + q < j) {
                    const double2 v = V[(c0 + q) * ldv + l];
                    const double2 vc = make_double2(v.x, -v.y);
                    acc[q] = cfma(vc, wl, acc[q]);
                    acc[kDotChunk + q] = cfma(vc, xl, acc[kDotChunk + q]);
                }
            if (first) {
                acc[2 * kDotChunk] = cfma(make_double2(xl.x, -xl.y), wl, acc[2 * kDotChunk]);
                acc[2 * kDotChunk + 1].x += xl.x * xl.x + xl.y * xl.y;
            }
        }
        block_sum<2 * kDotChunk + 2>(acc, sh);
        if (threadIdx.x == 0) {
            for (int q = 0; q < kDotChunk && c0 + q < j; q++) {
                partials[c0 + q] = cscale(acc[q], vs[c0 + q]);
                partials[j + 1 + c0 + q] = cscale(acc[kDotChunk + q], vs[c0 + q]);
            }
            if (first) {
                partials[j] = cscale(acc[2 * kDotChunk], vs[j]);
                partials[2 * j + 1] = acc[2 * kDotChunk + 1];
            }
        }
    }
}

// The delayed reorthogonalization of the last tentative vector V_t of a
// cycle, t = *jl + 1 (read on the device: the number of steps a graph ran
// is decided on the device): slots 0 .. t-1 a_i = vs_i <V_i, V_t>, slot t
// g = <V_t, V_t>.
__global__ void __launch_bounds__(kRedThreads) dots_tail_kernel(const double2 *__restrict__ V, long ldv, long sV,
                                                                const double *__restrict__ vs, long sVs,
                                                                const int *jl, long N,
                                                                double2 *__restrict__ partials, int cap,
                                                                const int *pred, const int *skip) {
    __shared__ double2 sh[(kRedThreads / 32) * (kDotChunk + 1)];
    if (pred && *pred == 0) return;
    const int t = *jl + 1;
    const int r = blockIdx.y;
    partials += (long)r * gridDim.x * cap + (long)blockIdx.x * cap;
    if (skip && skip[r]) {
        for (int q = threadIdx.x; q <= t; q += blockDim.x) partials[q] = make_double2(0, 0);
        return;
    }
    V += r * sV;
    vs += r * sVs;
    const double2 *__restrict__ vt = V + (long)t * ldv;
    const long stride = (long)gridDim.x * blockDim.x;
    for (int c0 = 0; c0 < t; c0 += kDotChunk) {
        double2 acc[kDotChunk + 1];
#pragma unroll
        for (int q = 0; q <= kDotChunk; q++) acc[q] = make_double2(0, 0);
        const bool first = c0 == 0;
        for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
            const double2 xl = vt[l];
#pragma unroll
            for (int q = 0; q < kDotChunk; q++)
                if (c0 + q < t) {
                    const double2 v = V[(c0 + q) * ldv + l];
                    acc[q] = cfma(make_double2(v.x, -v.y), xl, acc[q]);
                }
            if (first) acc[kDotChunk].x += xl.x * xl.x + xl.y * xl.y;
        }
        block_sum<kDotChunk + 1>(acc, sh);
        if (threadIdx.x == 0) {
            for (int q = 0; q < kDotChunk && c0 + q < t; q++) partials[c0 + q] = cscale(acc[q], vs[c0 + q]);
            if (first) partials[t] = acc[kDotChunk];
        }
    }
}

// out[r][i] = sum_b partials[r][b][i]: one block of kFinalThreads per (i, r),
// threads stride over the block partials, then a fixed shuffle tree
// (deterministic: the order depends only on nblocks).  With nv_dev the
// count is min(nv, *nv_dev + nv_add).
constexpr int kFinalThreads = 128;
__global__ void __launch_bounds__(kFinalThreads) reduce_partials_kernel(const double2 *__restrict__ partials,
                                                                        int nblocks, int cap, int nv,
                                                                        double2 *__restrict__ out, long sOut,
                                                                        const int *pred,
                                                                        const int *nv_dev = nullptr,
                                                                        int nv_add = 0) {
    __shared__ double2 sh[kFinalThreads / 32];
    if (pred && *pred == 0) return;
    const int i = blockIdx.x, r = blockIdx.y;
    if (nv_dev) nv = min(nv, *nv_dev + nv_add);
    if (i >= nv) return;
    partials += (long)r * nblocks * cap;
    double2 s = make_double2(0, 0);
    for (int b = threadIdx.x; b < nblocks; b += kFinalThreads) {
        const double2 p = partials[(long)b * cap + i];
        s.x += p.x;
        s.y += p.y;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = sh[0];
        for (int w = 1; w < kFinalThreads / 32; w++) t = cadd(t, sh[w]);
        out[r * sOut + i] = t;
    }
}

// w -= sum_i coef[i] vs[i] V_i ; post 1: ||w_new||^2 partial into partials[r][b][0]
__global__ void __launch_bounds__(kRedThreads) update_kernel(const double2 *__restrict__ V, long ldv, long sV,
                                                             const double *__restrict__ vs, long sVs, int nv,
                                                             const double2 *__restrict__ coef, long sCoef,
                                                             double2 *__restrict__ w, long sW, long N, int post,
                                                             double2 *__restrict__ partials, int cap,
                                                             const int *pred) {
    extern __shared__ double2 sc[];  // nv coefficients (coef * vs)
    __shared__ double2 sh[(kRedThreads / 32)];
    if (pred && *pred == 0) return;
    const int r = blockIdx.y;
    V += r * sV;
    w += r * sW;
    coef += r * sCoef;
    if (vs) vs += r * sVs;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) sc[i] = cscale(coef[i], vs ? vs[i] : 1.0);
    __syncthreads();
    double2 nrm[1] = {make_double2(0, 0)};
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
        double2 acc = w[l];
        for (int i = 0; i < nv; i++) acc = cfms(sc[i], V[i * ldv + l], acc);
        w[l] = acc;
        nrm[0].x += acc.x * acc.x + acc.y * acc.y;
    }
    if (post == 1) {
        block_sum<1>(nrm, sh);
        if (threadIdx.x == 0) partials[(long)r * gridDim.x * cap + (long)blockIdx.x * cap] = nrm[0];
    }
}

// The DCGS2 update pass: with alpha = coef[0 .. j-1], delta = coef[M2 .. M2+j]
//   V_j <- V_j - sum_{i<j} alpha_i V_i                 (j > 0)
//   w   <- w - sum_{i<j} delta_i V_i - delta_j V_j(old)
// and ||w||^2 partials; skip[r] set: zero partials, nothing read or written.
// U > 1: the basis loads of U consecutive i issued together ahead of their
// FMAs (more bytes in flight per thread; the FMA order, and so the result,
// is the same as U = 1).
template <int U>
__global__ void __launch_bounds__(kRedThreads) update2_kernel(double2 *__restrict__ V, long ldv, long sV, int j,
                                                              const double2 *__restrict__ coef, long sCoef, int M2,
                                                              double2 *__restrict__ w, long sW, long N,
                                                              double2 *__restrict__ partials, int cap,
                                                              const int *pred, const int *skip) {
    extern __shared__ double2 sc[];  // alpha[j], delta[j + 1]
    __shared__ double2 sh[(kRedThreads / 32)];
    if (pred && *pred == 0) return;
    const int r = blockIdx.y;
    if (skip && skip[r]) {
        if (threadIdx.x == 0) partials[(long)r * gridDim.x * cap + (long)blockIdx.x * cap] = make_double2(0, 0);
        return;
    }
    V += r * sV;
    w += r * sW;
    coef += r * sCoef;
    double2 *alpha = sc, *delta = sc + j;
    for (int i = threadIdx.x; i < j; i += blockDim.x) alpha[i] = coef[i];
    for (int i = threadIdx.x; i <= j; i += blockDim.x) delta[i] = coef[M2 + i];
    __syncthreads();
    double2 *__restrict__ vj = V + (long)j * ldv;
    double2 nrm[1] = {make_double2(0, 0)};
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
        double2 x = vj[l];
        double2 acc = cfms(delta[j], x, w[l]);
        int i = 0;
        if (U > 1) {
            for (; i + U <= j; i += U) {
                double2 v[U];
#pragma unroll
                for (int q = 0; q < U; q++) v[q] = V[(long)(i + q) * ldv + l];
#pragma unroll
                for (int q = 0; q < U; q++) {
                    x = cfms(alpha[i + q], v[q], x);
                    acc = cfms(delta[i + q], v[q], acc);
                }
            }
        }
        for (; i < j; i++) {
            const double2 v = V[i * ldv + l];
            x = cfms(alpha[i], v, x);
            acc = cfms(delta[i], v, acc);
        }
        if (j > 0) vj[l] = x;
        w[l] = acc;
        nrm[0].x += acc.x * acc.x + acc.y * acc.y;
    }
    block_sum<1>(nrm, sh);
    if (threadIdx.x == 0) partials[(long)r * gridDim.x * cap + (long)blockIdx.x * cap] = nrm[0];
}

// x += sum_i y[i] zs[i] Z_i  (i < *nzv_dev when given, else nzv); Z complex128 or complex64
template <typename TZ>
__global__ void __launch_bounds__(kRedThreads) combine_kernel(const TZ *__restrict__ Z, long ldz, long sZ,
                                                              const double *__restrict__ zs, long sZs, int nzv,
                                                              const double2 *__restrict__ y, long sY,
                                                              double2 *__restrict__ x, long sX, long N,
                                                              const int *nzv_dev) {
    extern __shared__ double2 sc[];
    if (nzv_dev) nzv = min(nzv, *nzv_dev);
    const int r = blockIdx.y;
    Z += r * sZ;
    y += r * sY;
    x += r * sX;
    if (zs) zs += r * sZs;
    for (int i = threadIdx.x; i < nzv; i += blockDim.x) sc[i] = cscale(y[i], zs ? zs[i] : 1.0);
    __syncthreads();
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
        double2 acc = x[l];
        for (int i = 0; i < nzv; i++) acc = cfma(sc[i], cvt<double2, TZ>(Z[i * ldz + l]), acc);
        x[l] = acc;
    }
}

__global__ void __launch_bounds__(kRedThreads) norm2_box_kernel(const double2 *__restrict__ x, long sX, int nx, int ny,
                                                                int x0, int x1, int y0, int y1, int z0, int z1,
                                                                double2 *__restrict__ partials, int cap) {
    __shared__ double2 sh[(kRedThreads / 32)];
    const int r = blockIdx.y;
    x += r * sX;
    const long bx = x1 - x0, by = y1 - y0, bz = z1 - z0;
    const long total = bx * by * bz;
    double2 acc[1] = {make_double2(0, 0)};
    const long stride = (long)gridDim.x * blockDim.x;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
        const long i = q % bx, t = q / bx;
        const long j = t % by, k = t / by;
        const double2 v = x[((k + z0) * ny + (j + y0)) * (long)nx + (i + x0)];
        acc[0].x += v.x * v.x + v.y * v.y;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partials[(long)r * gridDim.x * cap + (long)blockIdx.x * cap] = acc[0];
}

__global__ void axpby_kernel(double2 a, const double2 *__restrict__ x, long sX, double2 b, double2 *__restrict__ y,
                             long sY, long N) {
    const int r = blockIdx.y;
    x += r * sX;
    y += r * sY;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
        const double2 yv = y[l], xv = x[l];
        y[l] = cadd(cmul(a, xv), cmul(b, yv));
    }
}

__global__ void sub_dl_kernel(const double2 *__restrict__ x, const double2 *__restrict__ dl,
                              const double2 *__restrict__ t, double2 *__restrict__ y, long N) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) y[l] = csub(x[l], cmul(dl[l], t[l]));
}

// vs[r][j] = 1 / sqrt(nrm[r].x)
__global__ void set_scale_kernel(const double2 *nrm, long sNrm, double *vs, long sVs, int j, int R) {
    const int r = threadIdx.x;
    if (r < R) {
        const double s = sqrt(nrm[r * sNrm].x);
        vs[r * sVs + j] = s > 0 ? 1.0 / s : 0.0;
    }
}

template <typename R>
__global__ void base2d_kernel(const double *__restrict__ s2, int nz, long plane, int zlo, int zhi, double w2,
                              double beta, cplx<R> *__restrict__ out, int *status) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= plane) return;
    double s = 0.0;
    bool bad = false;
    for (int k = 0; k < nz; k++) {
        const double v = s2[(long)k * plane + q];
        bad |= !isfinite(v);
        if (k >= zlo && k < zhi) s += v;
    }
    s *= w2 / (double)(zhi - zlo);
    out[q] = cvt<cplx<R>, double2>(make_double2(s, s * beta));
    if (bad) atomicOr(status, 16);
}

static inline bool ok() { return cudaGetLastError() == cudaSuccess; }

static int grid_for(long N, int R = 1) {
    const long b = (N + kRedThreads - 1) / kRedThreads;
    const long cap = (4L * device_info().sm_count + R - 1) / R;
    return (int)(b < cap ? (b < 1 ? 1 : b) : (cap < 1 ? 1 : cap));
}

int launch_dots(const VecBatch &V, long ldv, const ScaleBatch &vs, int nv, const VecBatch &w, long N, int R,
                const Reduce &red, double2 *out, long sOut, cudaStream_t s, bool wnorm, const int *pred) {
    const int nout = nv + (wnorm ? 1 : 0);
    if (nout > red.cap || R > red.rmax) return HELM3D_ERR_ARG;
    const int nb = red.nblocks;
    dots_kernel<<<dim3(nb, R), kRedThreads, 0, s>>>(V.p, ldv, V.stride, vs.p, vs.stride, nv, w.p, w.stride, N,
                                                    wnorm ? 1 : 0, red.partials, red.cap, pred);
    reduce_partials_kernel<<<dim3(nout, R), kFinalThreads, 0, s>>>(red.partials, nb, red.cap, nout, out, sOut,
                                                                    pred);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_update(const VecBatch &V, long ldv, const ScaleBatch &vs, int nv, const double2 *coef, long sCoef,
                  const VecBatch &w, long N, int R, int post, const Reduce &red, double2 *out, long sOut,
                  cudaStream_t s, const int *pred) {
    if (R > red.rmax) return HELM3D_ERR_ARG;
    const int nb = post ? red.nblocks : grid_for(N, R);
    update_kernel<<<dim3(nb, R), kRedThreads, sizeof(double2) * (nv > 0 ? nv : 1), s>>>(
        V.p, ldv, V.stride, vs.p, vs.stride, nv, coef, sCoef, w.p, w.stride, N, post, red.partials, red.cap, pred);
    if (post == 1)
        reduce_partials_kernel<<<dim3(1, R), kFinalThreads, 0, s>>>(red.partials, nb, red.cap, 1, out, sOut, pred);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_dots2(const VecBatch &V, long ldv, const ScaleBatch &vs, int j, const VecBatch &w, long N, int R,
                 const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred, const int *skip) {
    const int nout = 2 * j + 2;
    if (nout > red.cap || R > red.rmax) return HELM3D_ERR_ARG;
    const int nb = red.nblocks;
    dots2_kernel<<<dim3(nb, R), kRedThreads, 0, s>>>(V.p, ldv, V.stride, vs.p, vs.stride, j, w.p, w.stride, N,
                                                     red.partials, red.cap, pred, skip);
    reduce_partials_kernel<<<dim3(nout, R), kFinalThreads, 0, s>>>(red.partials, nb, red.cap, nout, out, sOut,
                                                                    pred);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_dots_tail(const VecBatch &V, long ldv, const ScaleBatch &vs, int tmax, const int *jl, long N, int R,
                     const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred, const int *skip) {
    if (tmax + 1 > red.cap || R > red.rmax) return HELM3D_ERR_ARG;
    const int nb = red.nblocks;
    dots_tail_kernel<<<dim3(nb, R), kRedThreads, 0, s>>>(V.p, ldv, V.stride, vs.p, vs.stride, jl, N, red.partials,
                                                         red.cap, pred, skip);
    reduce_partials_kernel<<<dim3(tmax + 1, R), kFinalThreads, 0, s>>>(red.partials, nb, red.cap, tmax + 1, out,
                                                                        sOut, pred, jl, 2);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_update2(const VecBatch &V, long ldv, int j, const double2 *coef, long sCoef, int M2, const VecBatch &w,
                   long N, int R, const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred,
                   const int *skip) {
    if (R > red.rmax) return HELM3D_ERR_ARG;
    const int nb = red.nblocks;
    const size_t smem = sizeof(double2) * (2 * j + 1);
    if (red.update == 1)
        update2_kernel<8><<<dim3(nb, R), kRedThreads, smem, s>>>(V.p, ldv, V.stride, j, coef, sCoef, M2, w.p,
                                                                 w.stride, N, red.partials, red.cap, pred, skip);
    else
        update2_kernel<1><<<dim3(nb, R), kRedThreads, smem, s>>>(V.p, ldv, V.stride, j, coef, sCoef, M2, w.p,
                                                                 w.stride, N, red.partials, red.cap, pred, skip);
    reduce_partials_kernel<<<dim3(1, R), kFinalThreads, 0, s>>>(red.partials, nb, red.cap, 1, out, sOut, pred);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_combine(const VecBatch &Z, long ldz, const ScaleBatch &zs, int nzv, const double2 *y, long sY,
                   const VecBatch &x, long N, int R, cudaStream_t s, const int *nzv_dev) {
    const dim3 grid(grid_for(N, R), R);
    const size_t sm = sizeof(double2) * (nzv > 0 ? nzv : 1);
    if (Z.c64)
        combine_kernel<float2><<<grid, kRedThreads, sm, s>>>(reinterpret_cast<const float2 *>(Z.p), ldz, Z.stride,
                                                             zs.p, zs.stride, nzv, y, sY, x.p, x.stride, N, nzv_dev);
    else
        combine_kernel<double2><<<grid, kRedThreads, sm, s>>>(Z.p, ldz, Z.stride, zs.p, zs.stride, nzv, y, sY, x.p,
                                                              x.stride, N, nzv_dev);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_norm2_box(const VecBatch &x, int R, int nx, int ny, int nz, const int box[6], const Reduce &red,
                     double2 *out, long sOut, cudaStream_t s) {
    (void)nz;
    if (R > red.rmax) return HELM3D_ERR_ARG;
    norm2_box_kernel<<<dim3(red.nblocks, R), kRedThreads, 0, s>>>(x.p, x.stride, nx, ny, box[0], box[1], box[2],
                                                                  box[3], box[4], box[5], red.partials, red.cap);
    reduce_partials_kernel<<<dim3(1, R), kFinalThreads, 0, s>>>(red.partials, red.nblocks, red.cap, 1, out, sOut,
                                                                 nullptr);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_axpby(double2 a, const VecBatch &x, double2 b, const VecBatch &y, long N, int R, cudaStream_t s) {
    axpby_kernel<<<dim3(grid_for(N, R), R), kRedThreads, 0, s>>>(a, x.p, x.stride, b, y.p, y.stride, N);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_sub_dl(const double2 *x, const double2 *dl, const double2 *t, double2 *y, long N, cudaStream_t s) {
    sub_dl_kernel<<<grid_for(N), kRedThreads, 0, s>>>(x, dl, t, y, N);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_set_scale(const double2 *nrm, long sNrm, double *vs, long sVs, int j, int R, cudaStream_t s) {
    set_scale_kernel<<<1, 32 * ((R + 31) / 32), 0, s>>>(nrm, sNrm, vs, sVs, j, R);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_base2d(bool c64, const double *s2, int nz, long plane, int zlo, int zhi, double w2, double beta,
                  void *base2d, int *status, cudaStream_t s) {
    const unsigned grid = (unsigned)((plane + 255) / 256);
    if (c64) base2d_kernel<float><<<grid, 256, 0, s>>>(s2, nz, plane, zlo, zhi, w2, beta, (float2 *)base2d, status);
    else base2d_kernel<double><<<grid, 256, 0, s>>>(s2, nz, plane, zlo, zhi, w2, beta, (double2 *)base2d, status);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

Dev &device_info() {
    static Dev d;
    static bool init = false;
    if (!init) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
            d.sm_count = p.multiProcessorCount;
            d.smem_optin = p.sharedMemPerBlockOptin;
        }
        init = true;
    }
    return d;
}

}  // namespace h3d
