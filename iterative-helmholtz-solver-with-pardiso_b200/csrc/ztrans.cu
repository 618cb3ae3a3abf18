// ztrans.cu -- dense transform along z with the eigenvectors of the z
// operator with its PML (the HELM3D_ZT_PML_EIGEN preconditioner):
//   forward  planes[k][w] = sum_j Wi[k][j] (scale x[j][w])   (complex128 in, P out)
//   inverse  y[k][w]      = sum_j W[k][j] planes[j][w]        (P in, complex128 out)
// for every z-column w = i + nx*j of the grid, in FP64 whatever the plane
// precision (W is far from unitary: cond(W) ~ 1e4 for 12-point PMLs at
// nz = 128).  One CTA owns 32 consecutive
// columns: the nz x 32 input tile is staged in shared memory with coalesced
// row loads; warp q accumulates output rows k = 4q + 32t .. 4q + 32t + 3
// (four at a time, lane = column) over j, the matrix entries being warp-wide
// broadcast loads through L1.  The matrix (nz^2 elements) stays in L1/L2.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

constexpr int kZtCols = 32, kZtWarps = 8, kZtRows = 4;

template <typename R, bool FWD>
__global__ void __launch_bounds__(kZtCols *kZtWarps) ztrans_kernel(int nz, long plane, const void *__restrict__ in,
                                                                   double scale, void *__restrict__ out,
                                                                   const double2 *__restrict__ M) {
    typedef cplx<R> Cx;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *tile = reinterpret_cast<double2 *>(smem_raw);  // [nz][kZtCols]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long w = (long)blockIdx.x * kZtCols + lane;
    const bool valid = w < plane;
    for (int j = warp; j < nz; j += kZtWarps) {
        double2 v = make_double2(0, 0);
        if (valid) {
            if (FWD) {
                const double2 x = reinterpret_cast<const double2 *>(in)[(long)j * plane + w];
                v = make_double2(scale * x.x, scale * x.y);
            } else {
                v = cvt<double2, Cx>(reinterpret_cast<const Cx *>(in)[(long)j * plane + w]);
            }
        }
        tile[j * kZtCols + lane] = v;
    }
    __syncthreads();
    for (int k0 = warp * kZtRows; k0 < nz; k0 += kZtWarps * kZtRows) {
        double2 acc[kZtRows];
#pragma unroll
        for (int r = 0; r < kZtRows; r++) acc[r] = make_double2(0, 0);
        for (int j = 0; j < nz; j++) {
            const double2 t = tile[j * kZtCols + lane];
#pragma unroll
            for (int r = 0; r < kZtRows; r++)
                if (k0 + r < nz) acc[r] = cfma(__ldg(&M[(long)(k0 + r) * nz + j]), t, acc[r]);
        }
        if (!valid) continue;
#pragma unroll
        for (int r = 0; r < kZtRows; r++) {
            const int k = k0 + r;
            if (k >= nz) break;
            if (FWD) reinterpret_cast<Cx *>(out)[(long)k * plane + w] = cvt<Cx, double2>(acc[r]);
            else reinterpret_cast<double2 *>(out)[(long)k * plane + w] = acc[r];
        }
    }
}

template <typename R, bool FWD>
static int zt_impl(int nz, long plane, const void *in, double scale, void *out, const void *M, cudaStream_t s) {
    const size_t smem = (size_t)nz * kZtCols * sizeof(double2);
    auto kern = ztrans_kernel<R, FWD>;
    if (smem > device_info().smem_optin) return HELM3D_ERR_ARG;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return HELM3D_ERR_CUDA;
    const unsigned grid = (unsigned)((plane + kZtCols - 1) / kZtCols);
    kern<<<grid, kZtCols * kZtWarps, smem, s>>>(nz, plane, in, scale, out, (const double2 *)M);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_ztrans_forward(bool c64, const double2 *x, double scale, void *planes, int nz, long plane, const double2 *Wi,
                          cudaStream_t s) {
    return c64 ? zt_impl<float, true>(nz, plane, x, scale, planes, Wi, s)
               : zt_impl<double, true>(nz, plane, x, scale, planes, Wi, s);
}

int launch_ztrans_inverse(bool c64, const void *planes, double2 *y, int nz, long plane, const double2 *W,
                          cudaStream_t s) {
    return c64 ? zt_impl<float, false>(nz, plane, planes, 1.0, y, W, s)
               : zt_impl<double, false>(nz, plane, planes, 1.0, y, W, s);
}

}  // namespace h3d
