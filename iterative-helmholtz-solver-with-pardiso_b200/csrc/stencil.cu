// stencil.cu -- the complex 7-point PML-stretched operator (mode N) and its
// conjugate transpose, complex128:
//   (A u)_ijk = sum_a [cp_a (u_{+a} - u) + cm_a (u_{-a} - u)]
//               + omega^2 s2_ijk (1 + i beta) u_ijk,        u = 0 off the grid
// with cp_a(i) = alpha(i) alpha(i+1/2)/h^2 and cm_a(i) = alpha(i) alpha(i-1/2)/h^2
// (the reference's 5-point form, beta2D_pml, Source/functions.cpp:2347-2402,
// carried to z).  A thread owns one (i, j) column and marches along z with
// the z neighbours in registers; x/y neighbours come through L1.  The grid's
// z dimension enumerates (source, z chunk) pairs, source-major or
// source-minor (autotuned).
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

constexpr int kStX = 32, kStY = 8;

template <bool ADJ>
__global__ void __launch_bounds__(kStX *kStY) stencil_kernel(StencilArgs a) {
    const int i = blockIdx.x * kStX + threadIdx.x;
    const int j = blockIdx.y * kStY + threadIdx.y;
    if (i >= a.nx || j >= a.ny) return;
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    // source-minor order: the R sources of a z chunk are adjacent in launch
    // order and run together, so their reads of s2 and the coefficient
    // tables meet in L2 instead of coming from DRAM once per source
    const int r = a.src_fast ? (int)(blockIdx.z % a.R) : (int)(blockIdx.z / nzc);
    const int zc = a.src_fast ? (int)(blockIdx.z / a.R) : (int)(blockIdx.z - r * nzc);
    const int k0 = zc * a.zchunk;
    const int k1 = min(a.nz, k0 + a.zchunk);
    const long plane = (long)a.nx * a.ny;
    const long col = (long)j * a.nx + i;
    const double2 *x = a.x.p + r * a.x.stride;
    double2 *yout = a.y.p + r * a.y.stride;
    const double2 *fin = a.f.p ? a.f.p + r * a.f.stride : nullptr;
    const double xs = a.xscale * (a.sc.p ? a.sc.p[r * a.sc.stride] : 1.0);

    // per-axis couplings at this (i, j); for ADJ the ones that multiply the
    // neighbours are conj(cp[i-1]) (from i-1) and conj(cm[i+1]) (from i+1)
    double2 c_xm, c_xp, c_ym, c_yp, diag_xy;
    {
        const double2 cmx = a.cmx[i], cpx = a.cpx[i], cmy = a.cmy[j], cpy = a.cpy[j];
        diag_xy = make_double2(-(cmx.x + cpx.x + cmy.x + cpy.x), -(cmx.y + cpx.y + cmy.y + cpy.y));
        if (!ADJ) {
            c_xm = cmx;
            c_xp = cpx;
            c_ym = cmy;
            c_yp = cpy;
        } else {
            diag_xy.y = -diag_xy.y;
            c_xm = i > 0 ? a.cpx[i - 1] : make_double2(0, 0);
            c_xp = i + 1 < a.nx ? a.cmx[i + 1] : make_double2(0, 0);
            c_ym = j > 0 ? a.cpy[j - 1] : make_double2(0, 0);
            c_yp = j + 1 < a.ny ? a.cmy[j + 1] : make_double2(0, 0);
            c_xm.y = -c_xm.y;
            c_xp.y = -c_xp.y;
            c_ym.y = -c_ym.y;
            c_yp.y = -c_yp.y;
        }
    }
    const bool hxm = i > 0, hxp = i + 1 < a.nx, hym = j > 0, hyp = j + 1 < a.ny;
    double2 um = k0 > 0 ? x[(long)(k0 - 1) * plane + col] : make_double2(0, 0);
    double2 uc = x[(long)k0 * plane + col];
    for (int k = k0; k < k1; k++) {
        const long idx = (long)k * plane + col;
        const double2 up = k + 1 < a.nz ? x[idx + plane] : make_double2(0, 0);
        double2 czm, czp;
        const double2 cmz = a.cmz[k], cpz = a.cpz[k];
        double2 diag = make_double2(diag_xy.x - (cmz.x + cpz.x), diag_xy.y + (ADJ ? 1.0 : -1.0) * (cmz.y + cpz.y));
        if (!ADJ) {
            czm = cmz;
            czp = cpz;
        } else {
            czm = k > 0 ? a.cpz[k - 1] : make_double2(0, 0);
            czp = k + 1 < a.nz ? a.cmz[k + 1] : make_double2(0, 0);
            czm.y = -czm.y;
            czp.y = -czp.y;
        }
        const double s = a.w2 * a.s2[idx];
        // omega^2 s2 (1 + i beta), conjugated for the adjoint
        diag.x += s;
        diag.y += (ADJ ? -1.0 : 1.0) * s * a.beta_phys;
        double2 acc = cmul(diag, uc);
        if (hxm) acc = cfma(c_xm, x[idx - 1], acc);
        if (hxp) acc = cfma(c_xp, x[idx + 1], acc);
        if (hym) acc = cfma(c_ym, x[idx - a.nx], acc);
        if (hyp) acc = cfma(c_yp, x[idx + a.nx], acc);
        acc = cfma(czm, um, acc);
        acc = cfma(czp, up, acc);
        acc.x *= xs;
        acc.y *= xs;
        if (fin) {
            const double2 fv = fin[idx];
            acc = make_double2(fv.x - acc.x, fv.y - acc.y);
        }
        yout[idx] = acc;
        um = uc;
        uc = up;
    }
}

int launch_stencil(const StencilArgs &a, bool adjoint, cudaStream_t s) {
    dim3 block(kStX, kStY);
    if (a.zchunk < 1) return HELM3D_ERR_ARG;
    dim3 grid((a.nx + kStX - 1) / kStX, (a.ny + kStY - 1) / kStY, ((a.nz + a.zchunk - 1) / a.zchunk) * a.R);
    if (adjoint) stencil_kernel<true><<<grid, block, 0, s>>>(a);
    else stencil_kernel<false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
