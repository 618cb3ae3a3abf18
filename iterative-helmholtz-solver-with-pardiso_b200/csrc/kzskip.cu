// kzskip.cu -- the kz modes skipped by opts.kz_skip_ratio, the reference's
// SAVE_MEM switch (Source/FGMRES.cpp:197-206: a kz system with
// kww >= ratio * k2 is neither factored nor solved; its part of the
// solution is zero, Source/functions.cpp:6020-6024).  The factor and sweep
// kernels return at once for such a mode; here its planes are set: to zero
// (mode R, as the reference), or divided by the diagonal of the mode's 2D
// operator (mode N, where zero stalls FGMRES on the 7-point operator).
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

// kzinv[slot][j][i] = 1 / (-(cmx + cpx)[i] - (cmy + cpy)[j] + base2d[j][i] + shift[kz]), or 0
template <typename R>
__global__ void __launch_bounds__(256) kzinv_kernel(const int *__restrict__ kzlist, int nx, int ny,
                                                    const cplx<R> *__restrict__ cmx, const cplx<R> *__restrict__ cpx,
                                                    const cplx<R> *__restrict__ cmy, const cplx<R> *__restrict__ cpy,
                                                    const cplx<R> *__restrict__ base2d,
                                                    const cplx<R> *__restrict__ shift, int zero,
                                                    cplx<R> *__restrict__ kzinv) {
    const int slot = blockIdx.y;
    const long plane = (long)nx * ny;
    const int kz = kzlist[slot];
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < plane; l += (long)gridDim.x * blockDim.x) {
        const int j = (int)(l / nx), i = (int)(l - (long)j * nx);
        cplx<R> out = mkc<R>(0, 0);
        if (!zero) {
            const double dr = -((double)cmx[i].x + cpx[i].x + cmy[j].x + cpy[j].x) + base2d[l].x + shift[kz].x;
            const double di = -((double)cmx[i].y + cpx[i].y + cmy[j].y + cpy[j].y) + base2d[l].y + shift[kz].y;
            const double m2 = dr * dr + di * di;
            out = mkc<R>((R)(dr / m2), (R)(-di / m2));
        }
        kzinv[(long)slot * plane + l] = out;
    }
}

int launch_kzinv(bool c64, const int *kzlist, int nskip, int nx, int ny, const void *cmx, const void *cpx,
                 const void *cmy, const void *cpy, const void *base2d, const void *shift, bool zero, void *kzinv,
                 cudaStream_t s) {
    if (nskip <= 0) return HELM3D_OK;
    const dim3 grid((unsigned)(((long)nx * ny + 255) / 256), (unsigned)nskip);
    if (c64)
        kzinv_kernel<float><<<grid, 256, 0, s>>>(kzlist, nx, ny, (const float2 *)cmx, (const float2 *)cpx,
                                                 (const float2 *)cmy, (const float2 *)cpy, (const float2 *)base2d,
                                                 (const float2 *)shift, zero ? 1 : 0, (float2 *)kzinv);
    else
        kzinv_kernel<double><<<grid, 256, 0, s>>>(kzlist, nx, ny, (const double2 *)cmx, (const double2 *)cpx,
                                                  (const double2 *)cmy, (const double2 *)cpy, (const double2 *)base2d,
                                                  (const double2 *)shift, zero ? 1 : 0, (double2 *)kzinv);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

// planes of mode kzlist[slot] (plane kz holds line j, right-hand side r, row
// i at ((kz ny + j) R + r) nx + i) times kzinv[slot][j][i] (conjugated for
// the adjoint: the inverse of the conjugate transpose of a diagonal)
template <typename R, bool ADJ>
__global__ void __launch_bounds__(256) kzskip_apply_kernel(const int *__restrict__ kzlist, int nx, int ny, int nr,
                                                           const cplx<R> *__restrict__ kzinv,
                                                           cplx<R> *__restrict__ planes) {
    const int slot = blockIdx.z, j = blockIdx.y;
    const int kz = kzlist[slot];
    const cplx<R> *d = kzinv + ((long)slot * ny + j) * nx;
    cplx<R> *p = planes + ((long)kz * ny + j) * nr * nx;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nr * nx; q += gridDim.x * blockDim.x) {
        const int i = q % nx;
        cplx<R> v = d[i];
        if (ADJ) v.y = -v.y;
        p[q] = cmul(v, p[q]);
    }
}

template <typename R> static void kzskip_go(const SweepArgs &a, cudaStream_t s) {
    const dim3 grid((unsigned)((a.R * a.n + 255) / 256), (unsigned)a.ny, (unsigned)a.nskip);
    if (a.dxy)
        kzskip_apply_kernel<R, true><<<grid, 256, 0, s>>>(a.kzlist, a.n, a.ny, a.R, (const cplx<R> *)a.kzinv,
                                                         (cplx<R> *)a.planes);
    else
        kzskip_apply_kernel<R, false><<<grid, 256, 0, s>>>(a.kzlist, a.n, a.ny, a.R, (const cplx<R> *)a.kzinv,
                                                          (cplx<R> *)a.planes);
}

int launch_kzskip_apply(bool c64, const SweepArgs &a, cudaStream_t s) {
    if (a.nskip <= 0) return HELM3D_OK;
    if (!a.kzlist || !a.kzinv) return HELM3D_ERR_ARG;
    if (c64) kzskip_go<float>(a, s);
    else kzskip_go<double>(a, s);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
