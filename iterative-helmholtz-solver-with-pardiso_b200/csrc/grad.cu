// grad.cu -- kernels of the L2 data-misfit gradient with respect to the
// squared slowness s2 (no counterpart in the reference, which has no adjoint).
//
// For A(s2) u_s = f_s, J = 1/2 sum_s ||P u_s - d_s||^2 with P the sampling at
// the receiver indices, and lam_s = A^{-H} P^T (d_s - P u_s):
//   dJ/ds2_l = sum_s Re(conj(lam_s[l]) dA/ds2_l u_s[l]),
//   dA/ds2_l = omega^2 (1 + i beta) at cell l (the diagonal mass term).
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

__global__ void receiver_residual_kernel(const double2 *__restrict__ u, long sU, const long long *__restrict__ recv,
                                         int nrecv, const double2 *__restrict__ d, long sD,
                                         double2 *__restrict__ res) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (q < nrecv) res[(long)r * nrecv + q] = csub(u[r * sU + recv[q]], d[r * sD + q]);
}

__global__ void adjoint_source_kernel(const double2 *__restrict__ res, const long long *__restrict__ recv, int nrecv,
                                      double sign, double2 *__restrict__ y, long sY) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (q < nrecv) {
        const double2 v = res[(long)r * nrecv + q];
        double *dst = reinterpret_cast<double *>(y + r * sY + recv[q]);
        atomicAdd(dst, sign * v.x);
        atomicAdd(dst + 1, sign * v.y);
    }
}

// one pass over the cells, all sources of the batch per cell: g is read and
// written once per batch
__global__ void __launch_bounds__(256) grad_accum_kernel(const double2 *__restrict__ lam, long sL,
                                                         const double2 *__restrict__ u, long sU, int R, double w2,
                                                         double beta, double *__restrict__ g, long N) {
    const double2 dA = make_double2(w2, w2 * beta);
    const long stride = (long)gridDim.x * blockDim.x;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += stride) {
        double acc = 0.0;
        for (int r = 0; r < R; r++) {
            const double2 du = cmul(dA, u[r * sU + l]);
            const double2 lv = lam[r * sL + l];
            acc += lv.x * du.x + lv.y * du.y;   // Re(conj(lam) du)
        }
        g[l] += acc;
    }
}

static inline bool ok() { return cudaGetLastError() == cudaSuccess; }

int launch_receiver_residual(const VecBatch &u, int R, const long long *recv, int nrecv, const double2 *d, long sD,
                             double2 *res, cudaStream_t s) {
    if (nrecv <= 0) return HELM3D_OK;
    receiver_residual_kernel<<<dim3((nrecv + 255) / 256, R), 256, 0, s>>>(u.p, u.stride, recv, nrecv, d, sD, res);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_adjoint_source(const double2 *res, int R, const long long *recv, int nrecv, double sign,
                          const VecBatch &y, cudaStream_t s) {
    if (nrecv <= 0) return HELM3D_OK;
    adjoint_source_kernel<<<dim3((nrecv + 255) / 256, R), 256, 0, s>>>(res, recv, nrecv, sign, y.p, y.stride);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_grad_accum(const VecBatch &lam, const VecBatch &u, int R, double w2, double beta, double *g, long N,
                      cudaStream_t s) {
    const long b = (N + 255) / 256;
    const long cap = 8L * device_info().sm_count;
    grad_accum_kernel<<<(unsigned)(b < cap ? b : cap), 256, 0, s>>>(lam.p, lam.stride, u.p, u.stride, R, w2, beta, g,
                                                                    N);
    return ok() ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
