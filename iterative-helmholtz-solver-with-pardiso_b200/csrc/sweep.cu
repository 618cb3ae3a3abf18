// sweep.cu -- forward/backward block sweep over y-lines for every kz (the
// per-kz 2D solve; replaces PARDISO phase 33, Source/functions.cpp:5959,
// and DirSolveFastDiagStruct, Source/HODLR/BinaryTreesHODLR.cpp:2971-3018).
//
// With G_j = S_j^{-1} from the factor:
//   forward   y_0 = G_0 f_0,   y_j = G_j (f_j - cmy[j] y_{j-1})
//   backward  x_{ny-1} = y_{ny-1},   x_j = y_j - cpy[j] G_j x_{j+1}
// in place on the plane of each kz.  One CTA per (kz, right-hand side).
//
// The block product y = G v reads G^T row by row (G^T[m][:] = column m of
// G, contiguous): warp w accumulates v[m] * G^T[m][:] for m = w, w + NW, ...
// with lane l owning rows l, l + 32, ...; the NW partial vectors are summed
// through shared memory.  G^T streams from HBM through a ring of shared
// memory stages filled by 1D bulk copies (cp.async.bulk) issued by one
// thread; the copies run ahead of the dependence chain y_{j-1} -> y_j, so
// the stream is limited by bandwidth rather than by the per-line latency.
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

// stage s of the global sequence: fwd lines 0..ny-1 then bwd lines ny-2..0,
// each line split in chunks of rows_per_stage rows of G^T
template <typename R>
__device__ __forceinline__ const cplx<R> *stage_src(const SweepK<R> &a, int kz, long seq, int chunks_per_line,
                                                    int *rows) {
    const long line_seq = seq / chunks_per_line;
    const int chunk = (int)(seq % chunks_per_line);
    const int line = line_seq < a.ny ? (int)line_seq : (int)(2 * a.ny - 2 - line_seq);
    const int r0 = chunk * a.rows_per_stage;
    *rows = min(a.rows_per_stage, a.n - r0);
    return a.Gt + (((long)kz * a.ny + line) * a.n + r0) * (long)a.ldg;
}

template <typename R, int NW, int RB>
__global__ void __launch_bounds__(NW * 32, 1) sweep_kernel(SweepK<R> a) {
    typedef cplx<R> Cx;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, ldg = a.ldg;
    const int kz = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cx *ring = reinterpret_cast<Cx *>(smem_raw);                                    // nstage * stage
    Cx *vec = reinterpret_cast<Cx *>(smem_raw + (size_t)a.nstage * a.stage_bytes);  // [32*RB] current v
    Cx *prev = vec + 32 * RB;                                                        // [32*RB] y_{j-1} / x_{j+1}
    Cx *red = prev + 32 * RB;                                                        // [NW][32*RB]
    uint64_t *full = reinterpret_cast<uint64_t *>(red + NW * 32 * RB);
    uint64_t *empty = full + a.nstage;
    Cx *P = a.planes + (long)blockIdx.y * a.rhs_stride + (long)kz * ny * n;

    const int cpl = (n + a.rows_per_stage - 1) / a.rows_per_stage;  // chunks per line
    const long nseq = (long)(2 * ny - 1) * cpl;
    bool dead = false;

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW);
        }
        fence_mbar_init_cluster();
    }
    __syncthreads();

    // producer: thread 0 keeps up to nstage copies in flight
    long issued = 0;
    auto produce = [&](long upto) {
        while (issued < upto && issued < nseq) {
            const int s = (int)(issued % a.nstage);
            const uint32_t ph = (uint32_t)((issued / a.nstage) & 1);
            if (!dead && !mbar_wait_bounded_cta(smem_u32(&empty[s]), ph ^ 1u, kSweepWaitLimit)) {
                dead = true;
                atomicOr(a.status, 4);
            }
            int rows;
            const Cx *src = stage_src(a, kz, issued, cpl, &rows);
            const uint32_t bytes = (uint32_t)rows * ldg * sizeof(Cx);
            mbar_expect_tx(&full[s], bytes);
            bulk_g2s(ring + (size_t)s * (a.stage_bytes / sizeof(Cx)), src, bytes, &full[s]);
            issued++;
        }
    };
    if (threadIdx.x == 0) produce(a.nstage);

    long seq = 0;
    for (int step = 0; step < 2 * ny - 1; step++) {
        const bool fwd = step < ny;
        const int line = fwd ? step : 2 * ny - 2 - step;
        // v for this line
        for (int i = threadIdx.x; i < n; i += NW * 32) {
            Cx v;
            if (fwd) {
                v = P[(long)line * n + i];
                if (line > 0) v = cfms(a.cmy[line], prev[i], v);
            } else {
                v = prev[i];  // x_{line+1}
            }
            vec[i] = v;
        }
        __syncthreads();
        Cx acc[RB];
#pragma unroll
        for (int ra = 0; ra < RB; ra++) acc[ra] = mkc<R>(0, 0);
        for (int c = 0; c < cpl; c++, seq++) {
            const int s = (int)(seq % a.nstage);
            const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
            if (!dead && !mbar_wait_bounded_cta(smem_u32(&full[s]), ph, kSweepWaitLimit)) {
                dead = true;
                atomicOr(a.status, 4);
            }
            const Cx *st = ring + (size_t)s * (a.stage_bytes / sizeof(Cx));
            const int r0 = c * a.rows_per_stage;
            const int rows = min(a.rows_per_stage, n - r0);
            for (int m = warp; m < rows; m += NW) {
                const Cx vm = vec[r0 + m];
                const Cx *g = st + (long)m * ldg;
#pragma unroll
                for (int ra = 0; ra < RB; ra++) {
                    const int i = lane + 32 * ra;
                    if (i < n) acc[ra] = cfma(g[i], vm, acc[ra]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&empty[s]);
            if (threadIdx.x == 0) produce(seq + 1 + a.nstage);
        }
#pragma unroll
        for (int ra = 0; ra < RB; ra++) red[warp * 32 * RB + lane + 32 * ra] = acc[ra];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += NW * 32) {
            Cx y = red[i];
            for (int w = 1; w < NW; w++) y = cadd(y, red[w * 32 * RB + i]);
            if (fwd) {
                prev[i] = y;
                P[(long)line * n + i] = y;
            } else {
                const Cx x = cfms(a.cpy[line], y, P[(long)line * n + i]);
                prev[i] = x;
                P[(long)line * n + i] = x;
            }
        }
        __syncthreads();
    }
}

template <typename R, int NW, int RB> static int sweep_impl(const SweepArgs &sa, cudaStream_t st) {
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
    // ring: ~24 KB stages, as many as fit in ~160 KB
    const size_t row_bytes = (size_t)sa.ldg * sizeof(Cx);
    int rows = (int)((24 * 1024) / row_bytes);
    if (rows < 1) rows = 1;
    if (rows > sa.n) rows = sa.n;
    k.rows_per_stage = rows;
    k.stage_bytes = (uint32_t)(((size_t)rows * row_bytes + 127) & ~(size_t)127);
    int nst = (int)((160 * 1024) / k.stage_bytes);
    if (nst > 8) nst = 8;
    if (nst < 2) nst = 2;
    k.nstage = nst;
    const size_t smem = (size_t)nst * k.stage_bytes + sizeof(Cx) * (2 + NW) * 32 * RB + 2 * nst * sizeof(uint64_t) + 16;
    auto kern = sweep_kernel<R, NW, RB>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return HELM3D_ERR_CUDA;
    kern<<<dim3((unsigned)sa.nz, (unsigned)sa.nrhs), NW * 32, smem, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_sweep(bool c64, const SweepArgs &sa, cudaStream_t s) {
    const int rb = (sa.n + 31) / 32;
    if (c64) {
        switch (rb) {
            case 1: return sweep_impl<float, 8, 1>(sa, s);
            case 2: return sweep_impl<float, 8, 2>(sa, s);
            case 3: return sweep_impl<float, 8, 3>(sa, s);
            case 4: return sweep_impl<float, 8, 4>(sa, s);
            case 5: case 6: return sweep_impl<float, 8, 6>(sa, s);
            case 7: case 8: return sweep_impl<float, 8, 8>(sa, s);
        }
    } else {
        switch (rb) {
            case 1: return sweep_impl<double, 8, 1>(sa, s);
            case 2: return sweep_impl<double, 8, 2>(sa, s);
            case 3: return sweep_impl<double, 8, 3>(sa, s);
            case 4: return sweep_impl<double, 8, 4>(sa, s);
            case 5: case 6: return sweep_impl<double, 8, 6>(sa, s);
            case 7: case 8: return sweep_impl<double, 8, 8>(sa, s);
        }
    }
    return HELM3D_ERR_ARG;
}

}  // namespace h3d
