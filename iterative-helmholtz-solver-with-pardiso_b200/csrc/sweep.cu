// sweep.cu -- forward/backward block sweep over y-lines for every kz (the
// per-kz 2D solve; replaces PARDISO phase 33, Source/functions.cpp:5959,
// and DirSolveFastDiagStruct, Source/HODLR/BinaryTreesHODLR.cpp:2971-3018).
//
// With G_j = S_j^{-1} from the factor:
//   forward   y_0 = G_0 f_0,   y_j = G_j (f_j - cmy[j] y_{j-1})
//   backward  x_{ny-1} = y_{ny-1},   x_j = y_j - cpy[j] G_j x_{j+1}
// in place on the plane of each kz.  One CTA per (kz, right-hand side).
//
// G_j^T (row m = column m of G, contiguous) streams from HBM through a ring
// of shared-memory stages filled by 1D bulk copies (cp.async.bulk with
// mbarrier completion) that a dedicated producer warp issues as far ahead as
// the ring allows, independently of the y_{j-1} -> y_j dependence chain.
// Each of the 8 consumer warps owns RW = 32/G rows of y: lane (il, g) owns
// row i = w*RW + il and accumulates G^T[m][i] v[m] over the rows m = g, g+G,
// ... of every stage; the G partial sums of a row meet by warp shuffles, so a
// y-line ends with one named barrier among the consumer warps and no
// shared-memory reduction.  v[m] is formed on the fly from the previous
// line's result and the current line's right-hand side, both double-buffered
// in shared memory; the next line's right-hand side is prefetched into
// registers while the current line streams.
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"

namespace h3d {

template <typename R> struct SweepK {
    int n, ny, ldg;
    const cplx<R> *Gt;
    const cplx<R> *cmy, *cpy;
    cplx<R> *planes;
    long rhs_stride;
    int rows_per_stage;  // rows of G^T per ring stage
    int nstage;          // ring depth
    uint32_t stage_bytes;
    int *status;
};

constexpr uint32_t kSweepWaitLimit = 1u << 20;
constexpr int kSweepConsumerWarps = 8;
constexpr int kSweepMaxN = 256;

__device__ __forceinline__ void consumer_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kSweepConsumerWarps * 32) : "memory");
}

// G^T source of stage `seq`: forward lines 0..ny-1, then backward lines
// ny-2..0, each line split in chunks of rows_per_stage rows
template <typename R>
__device__ __forceinline__ const cplx<R> *stage_src(const SweepK<R> &a, int kz, long seq, int cpl, int *rows) {
    const long line_seq = seq / cpl;
    const int chunk = (int)(seq % cpl);
    const int line = line_seq < a.ny ? (int)line_seq : (int)(2 * a.ny - 2 - line_seq);
    const int r0 = chunk * a.rows_per_stage;
    *rows = min(a.rows_per_stage, a.n - r0);
    return a.Gt + (((long)kz * a.ny + line) * a.n + r0) * (long)a.ldg;
}

template <typename R, int G>
__global__ void __launch_bounds__((kSweepConsumerWarps + 1) * 32, 1) sweep_kernel(SweepK<R> a) {
    typedef cplx<R> Cx;
    constexpr int RW = 32 / G;  // rows of y per warp
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, ldg = a.ldg;
    const int kz = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cx *ring = reinterpret_cast<Cx *>(smem_raw);
    Cx *ybuf = reinterpret_cast<Cx *>(smem_raw + (size_t)a.nstage * a.stage_bytes);  // [2][kSweepMaxN]
    Cx *fbuf = ybuf + 2 * kSweepMaxN;                                                 // [2][kSweepMaxN]
    uint64_t *full = reinterpret_cast<uint64_t *>(fbuf + 2 * kSweepMaxN);
    uint64_t *empty = full + a.nstage;
    Cx *P = a.planes + (long)blockIdx.y * a.rhs_stride + (long)kz * ny * n;
    const int cpl = (n + a.rows_per_stage - 1) / a.rows_per_stage;
    const long nseq = (long)(2 * ny - 1) * cpl;

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kSweepConsumerWarps);
        }
        fence_mbar_init_cluster();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) fbuf[i] = P[i];  // f_0
    __syncthreads();

    if (warp == kSweepConsumerWarps) {
        // producer warp: one lane streams every stage of the chain
        if (lane == 0) {
            bool dead = false;
            for (long seq = 0; seq < nseq; seq++) {
                const int s = (int)(seq % a.nstage);
                const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
                if (!dead && !mbar_wait_bounded_cta(smem_u32(&empty[s]), ph ^ 1u, kSweepWaitLimit)) {
                    dead = true;
                    atomicOr(a.status, 4);
                }
                int rows;
                const Cx *src = stage_src(a, kz, seq, cpl, &rows);
                const uint32_t bytes = (uint32_t)rows * ldg * (uint32_t)sizeof(Cx);
                mbar_expect_tx(&full[s], bytes);
                bulk_g2s(ring + (size_t)s * (a.stage_bytes / sizeof(Cx)), src, bytes, &full[s]);
            }
        }
        return;
    }

    const int il = lane % RW, g = lane / RW;
    const int i = warp * RW + il;
    const bool own = i < n;
    bool dead = false;
    long seq = 0;
    for (int step = 0; step < 2 * ny - 1; step++) {
        const bool fwd = step < ny;
        const int line = fwd ? step : 2 * ny - 2 - step;
        const Cx *yprev = ybuf + ((step + 1) & 1) * kSweepMaxN;  // y_{line-1} (fwd) / x_{line+1} (bwd)
        Cx *ycur = ybuf + (step & 1) * kSweepMaxN;
        const Cx *fcur = fbuf + (step & 1) * kSweepMaxN;
        const Cx c = fwd ? (line > 0 ? a.cmy[line] : mkc<R>(0, 0)) : mkc<R>(0, 0);
        // prefetch: next line's right-hand side (forward) or this line's y (backward)
        Cx pre = mkc<R>(0, 0);
        if (own && g == 0) {
            if (fwd && line + 1 < ny) pre = P[(long)(line + 1) * n + i];
            else if (!fwd) pre = P[(long)line * n + i];
        }
        Cx acc = mkc<R>(0, 0);
        for (int ch = 0; ch < cpl; ch++, seq++) {
            const int s = (int)(seq % a.nstage);
            const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
            if (!dead && !mbar_wait_bounded_cta(smem_u32(&full[s]), ph, kSweepWaitLimit)) {
                dead = true;
                atomicOr(a.status, 4);
            }
            const Cx *st = ring + (size_t)s * (a.stage_bytes / sizeof(Cx));
            const int r0 = ch * a.rows_per_stage;
            const int rows = min(a.rows_per_stage, n - r0);
            if (own) {
#pragma unroll 4
                for (int ml = g; ml < rows; ml += G) {
                    const int m = r0 + ml;
                    Cx v;
                    if (fwd) v = (line > 0) ? cfms(c, yprev[m], fcur[m]) : fcur[m];
                    else v = yprev[m];
                    acc = cfma(st[(long)ml * ldg + i], v, acc);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&empty[s]);
        }
#pragma unroll
        for (int off = RW; off < 32; off <<= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        }
        if (own && g == 0) {
            Cx out;
            if (fwd) {
                out = acc;
                if (line + 1 < ny) fbuf[((step + 1) & 1) * kSweepMaxN + i] = pre;
            } else {
                out = cfms(a.cpy[line], acc, pre);
            }
            ycur[i] = out;
            P[(long)line * n + i] = out;
        }
        consumer_barrier();
    }
}

template <typename R, int G> static int sweep_impl(const SweepArgs &sa, cudaStream_t st) {
    typedef cplx<R> Cx;
    SweepK<R> k;
    k.n = sa.n;
    k.ny = sa.ny;
    k.ldg = sa.ldg;
    k.Gt = (const Cx *)sa.Gt;
    k.cmy = (const Cx *)sa.cmy;
    k.cpy = (const Cx *)sa.cpy;
    k.planes = (Cx *)sa.planes;
    k.rhs_stride = sa.rhs_stride;
    k.status = sa.status;
    // ~16 KB stages, as many as fit in ~200 KB
    const size_t row_bytes = (size_t)sa.ldg * sizeof(Cx);
    int rows = (int)((16 * 1024) / row_bytes);
    if (rows < 1) rows = 1;
    if (rows > sa.n) rows = sa.n;
    k.rows_per_stage = rows;
    k.stage_bytes = (uint32_t)(((size_t)rows * row_bytes + 127) & ~(size_t)127);
    int nst = (int)((200 * 1024) / k.stage_bytes);
    if (nst > 32) nst = 32;
    if (nst < 2) nst = 2;
    k.nstage = nst;
    const size_t smem = (size_t)nst * k.stage_bytes + sizeof(Cx) * 4 * kSweepMaxN + 2 * nst * sizeof(uint64_t);
    auto kern = sweep_kernel<R, G>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return HELM3D_ERR_CUDA;
    kern<<<dim3((unsigned)sa.nz, (unsigned)sa.nrhs), (kSweepConsumerWarps + 1) * 32, smem, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_sweep(bool c64, const SweepArgs &sa, cudaStream_t s) {
    if (sa.n < 1 || sa.n > kSweepMaxN) return HELM3D_ERR_ARG;
    const int g = sa.n <= 64 ? 4 : (sa.n <= 128 ? 2 : 1);
    if (c64) {
        if (g == 4) return sweep_impl<float, 4>(sa, s);
        if (g == 2) return sweep_impl<float, 2>(sa, s);
        return sweep_impl<float, 1>(sa, s);
    }
    if (g == 4) return sweep_impl<double, 4>(sa, s);
    if (g == 2) return sweep_impl<double, 2>(sa, s);
    return sweep_impl<double, 1>(sa, s);
}

}  // namespace h3d
