// stencil.cu -- the complex 7-point PML-stretched operator (mode N) and its
// conjugate transpose, complex128:
//   (A u)_ijk = sum_a [cp_a (u_{+a} - u) + cm_a (u_{-a} - u)]
//               + omega^2 s2_ijk (1 + i beta) u_ijk,        u = 0 off the grid
// with cp_a(i) = alpha(i) alpha(i+1/2)/h^2 and cm_a(i) = alpha(i) alpha(i-1/2)/h^2
// (the reference's 5-point form, beta2D_pml, Source/functions.cpp:2347-2402,
// carried to z).  A thread owns one (i, j) column and marches along z with
// the z neighbours in registers; x/y neighbours come through L1
// (stencil_kernel) or from the plane's tile staged in shared memory
// (stencil_smem_kernel).  The grid's z dimension enumerates (source, z chunk)
// pairs, source-major or source-minor (autotuned).  The input x is complex128,
// or complex64 (TX = float2: FGMRES's Z basis of a complex64 preconditioner),
// widened to complex128 as it is read; the arithmetic and y are complex128.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "helm3d_internal.h"

namespace h3d {

__device__ __forceinline__ uint32_t smem_u32_st(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

constexpr int kStX = 32, kStY = 8;

template <bool ADJ, typename TX>
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
    const TX *x = reinterpret_cast<const TX *>(a.x.p) + r * a.x.stride;
    double2 *yout = a.y.p + r * a.y.stride;
    const double2 *fin = a.f.p ? a.f.p + r * a.f.stride : nullptr;
    const double xs = a.xscale * (a.sc.p ? a.sc.p[r * a.sc.stride] : 1.0);
    auto X = [&](long l) { return cvt<double2, TX>(x[l]); };

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
    double2 um = k0 > 0 ? X((long)(k0 - 1) * plane + col) : make_double2(0, 0);
    double2 uc = X((long)k0 * plane + col);
    for (int k = k0; k < k1; k++) {
        const long idx = (long)k * plane + col;
        const double2 up = k + 1 < a.nz ? X(idx + plane) : make_double2(0, 0);
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
        if (hxm) acc = cfma(c_xm, X(idx - 1), acc);
        if (hxp) acc = cfma(c_xp, X(idx + 1), acc);
        if (hym) acc = cfma(c_ym, X(idx - a.nx), acc);
        if (hyp) acc = cfma(c_yp, X(idx + a.nx), acc);
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

// ---------------------------------------------------------------------------
// The same operator with each z-plane's (x, y) tile staged in shared memory.
// A CTA owns a 32 x 8 tile of (i, j) columns and marches along z; plane k's
// tile with its one-point halo (34 x 10 complex) is copied into shared
// memory by 16- or 8-byte asynchronous copies (cp.async, zero-filled off the grid,
// which is the operator's u = 0 there), three planes ahead of the one being
// computed, in a ring of four plane buffers.  The x/y neighbours come from
// the tile, the z neighbours from the tiles of planes k - 1 (kept in a
// register) and k + 1.  One CTA barrier per plane.
constexpr int kSsX = 32, kSsY = 8, kSsHX = kSsX + 2, kSsHY = kSsY + 2, kSsBuf = 4;

// one element of x (B = 16 bytes complex128, 8 bytes complex64)
template <int B> __device__ __forceinline__ void cp_async_el(void *dst_smem, const void *src, bool valid);
template <> __device__ __forceinline__ void cp_async_el<16>(void *dst_smem, const void *src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32_st(dst_smem)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
template <> __device__ __forceinline__ void cp_async_el<8>(void *dst_smem, const void *src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32_st(dst_smem)), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <bool ADJ, typename TX>
__global__ void __launch_bounds__(kSsX *kSsY) stencil_smem_kernel(StencilArgs a) {
    __shared__ __align__(16) TX tile[kSsBuf][kSsHY][kSsHX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kSsX + tx;
    const int i = blockIdx.x * kSsX + tx;
    const int j = blockIdx.y * kSsY + ty;
    const int gi0 = blockIdx.x * kSsX - 1, gj0 = blockIdx.y * kSsY - 1;   // the tile's halo origin
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    const int r = a.src_fast ? (int)(blockIdx.z % a.R) : (int)(blockIdx.z / nzc);
    const int zc = a.src_fast ? (int)(blockIdx.z / a.R) : (int)(blockIdx.z - r * nzc);
    const int k0 = zc * a.zchunk;
    const int k1 = min(a.nz, k0 + a.zchunk);
    const long plane = (long)a.nx * a.ny;
    const TX *x = reinterpret_cast<const TX *>(a.x.p) + r * a.x.stride;
    double2 *yout = a.y.p + r * a.y.stride;
    const double2 *fin = a.f.p ? a.f.p + r * a.f.stride : nullptr;
    const double xs = a.xscale * (a.sc.p ? a.sc.p[r * a.sc.stride] : 1.0);
    const bool own = i < a.nx && j < a.ny;
    auto T = [&](int b, int hy, int hx) { return cvt<double2, TX>(tile[b][hy][hx]); };
    const long col = own ? (long)j * a.nx + i : 0;

    // plane k (any k: off the grid reads zeros) into ring buffer b
    auto load = [&](int k, int b) {
        for (int e = tid; e < kSsHX * kSsHY; e += kSsX * kSsY) {
            const int hy = e / kSsHX, hx = e - hy * kSsHX;
            const int gi = gi0 + hx, gj = gj0 + hy;
            const bool in = k >= 0 && k < a.nz && gi >= 0 && gi < a.nx && gj >= 0 && gj < a.ny;
            cp_async_el<sizeof(TX)>(&tile[b][hy][hx], in ? x + (long)k * plane + (long)gj * a.nx + gi : x, in);
        }
        cp_async_commit();
    };

    double2 c_xm = make_double2(0, 0), c_xp = c_xm, c_ym = c_xm, c_yp = c_xm, diag_xy = c_xm;
    if (own) {
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
    load(k0, 0);
    load(k0 + 1, 1);
    load(k0 + 2, 2);
    double2 um = (own && k0 > 0) ? cvt<double2, TX>(x[(long)(k0 - 1) * plane + col]) : make_double2(0, 0);
    for (int k = k0; k < k1; k++) {
        const int q = k - k0, b = q & (kSsBuf - 1), bp = (q + 1) & (kSsBuf - 1);
        cp_async_wait<1>();   // planes k and k + 1 have landed (k + 2 may be in flight)
        __syncthreads();      // ... for every thread's copies; and buffer (k - 1) is free
        if (k + 3 <= k1) load(k + 3, (q + 3) & (kSsBuf - 1));
        else cp_async_commit();   // an empty group keeps the count of groups per plane
        if (!own) continue;
        const long idx = (long)k * plane + col;
        const double2 uc = T(b, ty + 1, tx + 1);
        const double2 up = T(bp, ty + 1, tx + 1);
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
        acc = cfma(c_xm, T(b, ty + 1, tx), acc);
        acc = cfma(c_xp, T(b, ty + 1, tx + 2), acc);
        acc = cfma(c_ym, T(b, ty, tx + 1), acc);
        acc = cfma(c_yp, T(b, ty + 2, tx + 1), acc);
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
    }
    cp_async_wait<0>();   // no copy into this CTA's shared memory outlives it
}

template <typename TX> static void stencil_go(const StencilArgs &a, bool adjoint, cudaStream_t s) {
    if (a.smem) {
        dim3 block(kSsX, kSsY);
        dim3 grid((a.nx + kSsX - 1) / kSsX, (a.ny + kSsY - 1) / kSsY, ((a.nz + a.zchunk - 1) / a.zchunk) * a.R);
        if (adjoint) stencil_smem_kernel<true, TX><<<grid, block, 0, s>>>(a);
        else stencil_smem_kernel<false, TX><<<grid, block, 0, s>>>(a);
        return;
    }
    dim3 block(kStX, kStY);
    dim3 grid((a.nx + kStX - 1) / kStX, (a.ny + kStY - 1) / kStY, ((a.nz + a.zchunk - 1) / a.zchunk) * a.R);
    if (adjoint) stencil_kernel<true, TX><<<grid, block, 0, s>>>(a);
    else stencil_kernel<false, TX><<<grid, block, 0, s>>>(a);
}

int launch_stencil(const StencilArgs &a, bool adjoint, cudaStream_t s) {
    if (a.zchunk < 1 || a.y.c64 || a.f.c64) return HELM3D_ERR_ARG;
    if (a.x.c64) stencil_go<float2>(a, adjoint, s);
    else stencil_go<double2>(a, adjoint, s);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
