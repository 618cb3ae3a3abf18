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

// plane index of (row k, column w = i + nx*j) for right-hand side r
__device__ __forceinline__ long zt_plane_index(const PlaneLayout &L, int r, int k, long w) {
    const long j = w / L.nx, i = w - j * L.nx;
    return (long)k * L.plane * L.R + (j * L.R + r) * L.nx + i;
}

template <typename R, bool FWD>
__global__ void __launch_bounds__(kZtCols *kZtWarps) ztrans_kernel(PlaneLayout L, VecBatch vec, double scale,
                                                                   ScaleBatch sc, cplx<R> *__restrict__ planes,
                                                                   const double2 *__restrict__ M) {
    typedef cplx<R> Cx;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *tile = reinterpret_cast<double2 *>(smem_raw);  // [nz][kZtCols]
    const int nz = L.nz;
    const long plane = L.plane;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r = blockIdx.y;
    double2 *v_r = vec.p + r * vec.stride;
    const double s = scale * (sc.p ? sc.p[r * sc.stride] : 1.0);
    const long w = (long)blockIdx.x * kZtCols + lane;
    const bool valid = w < plane;
    for (int j = warp; j < nz; j += kZtWarps) {
        double2 v = make_double2(0, 0);
        if (valid) {
            if (FWD) {
                const double2 x = v_r[(long)j * plane + w];
                v = make_double2(s * x.x, s * x.y);
            } else {
                v = cvt<double2, Cx>(planes[zt_plane_index(L, r, j, w)]);
            }
        }
        tile[j * kZtCols + lane] = v;
    }
    __syncthreads();
    for (int k0 = warp * kZtRows; k0 < nz; k0 += kZtWarps * kZtRows) {
        double2 acc[kZtRows];
#pragma unroll
        for (int q = 0; q < kZtRows; q++) acc[q] = make_double2(0, 0);
        for (int j = 0; j < nz; j++) {
            const double2 t = tile[j * kZtCols + lane];
#pragma unroll
            for (int q = 0; q < kZtRows; q++)
                if (k0 + q < nz) acc[q] = cfma(__ldg(&M[(long)(k0 + q) * nz + j]), t, acc[q]);
        }
        if (!valid) continue;
#pragma unroll
        for (int q = 0; q < kZtRows; q++) {
            const int k = k0 + q;
            if (k >= nz) break;
            if (FWD) planes[zt_plane_index(L, r, k, w)] = cvt<Cx, double2>(acc[q]);
            else if (vec.c64) reinterpret_cast<float2 *>(vec.p)[r * vec.stride + (long)k * plane + w] = cvt<float2, double2>(acc[q]);
            else v_r[(long)k * plane + w] = acc[q];
        }
    }
}

template <typename R, bool FWD>
static int zt_impl(const PlaneLayout &L, const VecBatch &vec, double scale, const ScaleBatch &sc, void *planes,
                   const double2 *M, cudaStream_t s) {
    const size_t smem = (size_t)L.nz * kZtCols * sizeof(double2);
    auto kern = ztrans_kernel<R, FWD>;
    if (smem > device_info().smem_optin) return HELM3D_ERR_ARG;
    if (!smem_limit_max(kern, smem))
        return HELM3D_ERR_CUDA;
    const dim3 grid((unsigned)((L.plane + kZtCols - 1) / kZtCols), (unsigned)L.R);
    kern<<<grid, kZtCols * kZtWarps, smem, s>>>(L, vec, scale, sc, (cplx<R> *)planes, M);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_ztrans_forward(bool c64, const VecBatch &x, double scale, const ScaleBatch &sc, void *planes,
                          const PlaneLayout &L, const double2 *Wi, cudaStream_t s) {
    return c64 ? zt_impl<float, true>(L, x, scale, sc, planes, Wi, s)
               : zt_impl<double, true>(L, x, scale, sc, planes, Wi, s);
}

int launch_ztrans_inverse(bool c64, const void *planes, const PlaneLayout &L, const VecBatch &y, const double2 *W,
                          cudaStream_t s) {
    const ScaleBatch none = {nullptr, 0};
    return c64 ? zt_impl<float, false>(L, y, 1.0, none, (void *)planes, W, s)
               : zt_impl<double, false>(L, y, 1.0, none, (void *)planes, W, s);
}

}  // namespace h3d
