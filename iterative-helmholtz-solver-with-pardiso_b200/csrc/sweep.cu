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
// row i = w*RW + il and accumulates G^T[m][i] v[m][r] over the rows m = g,
// g+G, ... of every stage for all RR right-hand sides r (one G element feeds
// RR complex FMAs); the G partial sums of a row meet by warp shuffles.  The
// row owner also forms the next line's v[i][r] (f_{j+1} - cmy y_j forward,
// x_j backward) into a double-buffered shared array, so a y-line ends with
// one named barrier among the consumer warps and no shared-memory reduction.
// The next line's right-hand side is prefetched into registers while the
// current line streams.  Planes of R right-hand sides are laid out
// [kz][line][r][i].
#include <cuda_runtime.h>

#include <cstdlib>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"

namespace h3d {

template <typename R> struct SweepK {
    int n, ny, ldg, nrhs;
    const cplx<R> *Gt;
    const cplx<R> *cmy, *cpy;
    cplx<R> *planes;
    const cplx<R> *dxy;  // adjoint: [2][ny][n] = alpha_x alpha_y, conj(1 / (alpha_x alpha_y))
    int rows_per_stage;  // rows of G^T per ring stage
    int nstage;          // ring depth
    uint32_t stage_bytes;
    int *status;
    uint32_t wait_limit;  // polls of a producer/consumer wait before it gives up (status bit 2)
    int expire_test;      // HELM3D_TEST_EXPIRE_WAIT: the consumers first wait on a barrier that
                          // nothing arrives on, so that the wait expires (tests of the status path)
    const int *kzslot;    // >= 0: a skipped mode (launch_kzskip_apply handles it), or null
};

// Polls of a bounded wait.  Waits between the producer and the consumers use
// SweepK::wait_limit (this value unless HELM3D_WAIT_LIMIT sets it, to make
// a wait expire in a test); the final drain of the producer's own copies
// always uses this value, so that no copy is in flight when the CTA exits.
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

// G groups of lanes split the rows m of each stage; RR right-hand sides.
// ADJ: the conjugate-transposed solve S^{-H} v = conj(Dxy)^{-1} conj(S^{-1}
// (Dxy conj(v))), Dxy = diag(alpha_x(i) alpha_y(j)): Dxy^{-1} S is complex
// symmetric (every coupling is alpha(node) alpha(half node) / h^2), so the
// same factor serves; the input is scaled and conjugated where it is loaded
// and the output where it is stored.
// The producer lane waits (bounded) for its last copies to land before it
// returns, so that no bulk copy into this CTA's shared memory is still in
// flight when the CTA can exit: the final use of each of the last
// min(nstage, issued) ring slots.
__device__ __forceinline__ void sweep_drain(uint64_t *full, int nstage, long issued) {
    for (long k = 1; k <= nstage && k <= issued; k++) {
        const long seq = issued - k;
        mbar_wait_bounded_cta(smem_u32(&full[seq % nstage]), (uint32_t)((seq / nstage) & 1), kSweepWaitLimit);
    }
}

template <typename R, bool ADJ>
__device__ __forceinline__ cplx<R> adj_in(const SweepK<R> &a, int line, int i, cplx<R> f) {
    if (!ADJ) return f;
    return cmul(a.dxy[(long)line * a.n + i], mkc<R>(f.x, -f.y));
}
template <typename R, bool ADJ>
__device__ __forceinline__ cplx<R> adj_out(const SweepK<R> &a, int line, int i, cplx<R> x) {
    if (!ADJ) return x;
    return cmul(mkc<R>(x.x, -x.y), a.dxy[(long)(a.ny + line) * a.n + i]);
}

template <typename R, int G, int RR, bool ADJ>
__global__ void __launch_bounds__((kSweepConsumerWarps + 1) * 32, 1) sweep_kernel(SweepK<R> a) {
    typedef cplx<R> Cx;
    constexpr int RW = 32 / G;  // rows of y per warp
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, ldg = a.ldg, Rn = a.nrhs;
    const int kz = blockIdx.x;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cx *ring = reinterpret_cast<Cx *>(smem_raw);
    Cx *vbuf = reinterpret_cast<Cx *>(smem_raw + (size_t)a.nstage * a.stage_bytes);  // [2][n][RR]
    uint64_t *full = reinterpret_cast<uint64_t *>(vbuf + 2 * (size_t)n * RR);
    uint64_t *empty = full + a.nstage;
    uint64_t *never = empty + a.nstage;         // no thread arrives on it
    Cx *P = a.planes + (long)kz * ny * Rn * n;  // line j, rhs r, row i at ((j*Rn + r)*n + i)
    const int cpl = (n + a.rows_per_stage - 1) / a.rows_per_stage;
    const long nseq = (long)(2 * ny - 1) * cpl;

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kSweepConsumerWarps);
        }
        mbar_init(never, 1);
        fence_mbar_init_cluster();
    }
    for (int q = threadIdx.x; q < n * RR; q += blockDim.x) {  // v of line 0: f_0
        const int m = q / RR, r = q - (q / RR) * RR;
        vbuf[q] = r < Rn ? adj_in<R, ADJ>(a, 0, m, P[(long)r * n + m]) : mkc<R>(0, 0);
    }
    __syncthreads();

    if (warp == kSweepConsumerWarps) {
        // producer warp: one lane streams every stage of the chain
        if (lane == 0) {
            long seq = 0;
            for (; seq < nseq; seq++) {
                const int s = (int)(seq % a.nstage);
                const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
                if (!mbar_wait_bounded_cta(smem_u32(&empty[s]), ph ^ 1u, a.wait_limit)) {
                    // stop issuing: the consumers' bounded waits on full[] expire in turn
                    atomicOr(a.status, 4);
                    break;
                }
                int rows;
                const Cx *src = stage_src(a, kz, seq, cpl, &rows);
                const uint32_t bytes = (uint32_t)rows * ldg * (uint32_t)sizeof(Cx);
                mbar_expect_tx(&full[s], bytes);
                bulk_g2s(ring + (size_t)s * (a.stage_bytes / sizeof(Cx)), src, bytes, &full[s]);
            }
            sweep_drain(full, a.nstage, seq);
        }
        return;
    }

    const int il = lane % RW, g = lane / RW;
    const int i = warp * RW + il;
    const bool own = i < n;
    bool dead = false;
    if (a.expire_test && !mbar_wait_bounded_cta(smem_u32(never), 0u, a.wait_limit)) {
        dead = true;
        atomicOr(a.status, 4);
    }
    long seq = 0;
    for (int step = 0; step < 2 * ny - 1; step++) {
        const bool fwd = step < ny;
        const int line = fwd ? step : 2 * ny - 2 - step;
        const Cx *v = vbuf + (size_t)(step & 1) * n * RR;
        Cx *vnext = vbuf + (size_t)((step + 1) & 1) * n * RR;
        // prefetch: next line's right-hand side (forward) or this line's y (backward)
        Cx pre[RR];
#pragma unroll
        for (int r = 0; r < RR; r++) {
            pre[r] = mkc<R>(0, 0);
            if (own && g == 0 && r < Rn) {
                if (fwd && line + 1 < ny) pre[r] = adj_in<R, ADJ>(a, line + 1, i, P[((long)(line + 1) * Rn + r) * n + i]);
                else if (!fwd) pre[r] = P[((long)line * Rn + r) * n + i];
            }
        }
        Cx acc[RR];
#pragma unroll
        for (int r = 0; r < RR; r++) acc[r] = mkc<R>(0, 0);
        for (int ch = 0; ch < cpl; ch++, seq++) {
            const int s = (int)(seq % a.nstage);
            const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
            if (!dead && !mbar_wait_bounded_cta(smem_u32(&full[s]), ph, a.wait_limit)) {
                dead = true;
                atomicOr(a.status, 4);
            }
            const Cx *st = ring + (size_t)s * (a.stage_bytes / sizeof(Cx));
            const int r0 = ch * a.rows_per_stage;
            const int rows = min(a.rows_per_stage, n - r0);
            if (own) {
#pragma unroll 2
                for (int ml = g; ml < rows; ml += G) {
                    const Cx gv = st[(long)ml * ldg + i];
                    const Cx *vm = v + (size_t)(r0 + ml) * RR;
#pragma unroll
                    for (int r = 0; r < RR; r++) acc[r] = cfma(gv, vm[r], acc[r]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&empty[s]);
        }
#pragma unroll
        for (int r = 0; r < RR; r++)
#pragma unroll
            for (int off = RW; off < 32; off <<= 1) {
                acc[r].x += __shfl_xor_sync(0xffffffffu, acc[r].x, off);
                acc[r].y += __shfl_xor_sync(0xffffffffu, acc[r].y, off);
            }
        if (own && g == 0) {
            const Cx cn = (fwd && line + 1 < ny) ? a.cmy[line + 1] : mkc<R>(0, 0);
            const Cx cp = fwd ? mkc<R>(0, 0) : a.cpy[line];
#pragma unroll
            for (int r = 0; r < RR; r++) {
                if (r >= Rn) break;
                Cx out, vn;
                bool last;  // out is the final x of this line
                if (fwd) {
                    out = acc[r];                                          // y_line
                    last = line + 1 == ny;
                    vn = last ? out : cfms(cn, out, pre[r]);               // f_{line+1} - cmy y_line, or x_{ny-1}
                } else {
                    out = cfms(cp, acc[r], pre[r]);                        // x_line = y_line - cpy G x_{line+1}
                    last = true;
                    vn = out;
                }
                P[((long)line * Rn + r) * n + i] = last ? adj_out<R, ADJ>(a, line, i, out) : out;
                vnext[(size_t)i * RR + r] = vn;
            }
        }
        consumer_barrier();
    }
}

// ------------------------------------------------------------------------
// Register-tiled variant for complex64 batches of RR >= 4 right-hand sides.
// Each line is Y (n x RR) = G_j V.  The CW consumer warps form GM groups of
// CW / GM warps; group g takes the rows m = g, g + GM, ... of every stage,
// so the 32 lanes of a warp always read one G row and one v row (contiguous,
// no bank conflicts).  Thread t of a group owns a tile of TM = 4 rows x
// TR = 4 right-hand sides: per m it loads 4 G and 4 v entries (four 16-byte
// shared loads) for 16 complex FMAs.  At the end of a line groups 1..GM-1
// leave their partial tiles in shared memory and group 0 adds them and
// finishes the tile (next line's v into shared memory, x or y into the
// planes).  Producer warp, ring and mbarriers as in sweep_kernel.
constexpr int kTileM = 4, kTileR = 4;

template <int CW> __device__ __forceinline__ void consumer_barrier_n() {
    asm volatile("bar.sync 1, %0;" ::"n"(CW * 32) : "memory");
}

template <int RR, int GM, bool ADJ, int CW>
__global__ void __launch_bounds__((CW + 1) * 32, 1) sweep_tiled_kernel(SweepK<float> a) {
    typedef float2 Cx;
    constexpr int RB = RR / kTileR;             // right-hand-side blocks
    constexpr int NQ = kTileM * kTileR;          // outputs per tile
    constexpr int TPG = CW * 32 / GM;            // threads (tiles) per group
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, ldg = a.ldg, Rn = a.nrhs;
    const int kz = blockIdx.x;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cx *ring = reinterpret_cast<Cx *>(smem_raw);
    Cx *vbuf = reinterpret_cast<Cx *>(smem_raw + (size_t)a.nstage * a.stage_bytes);  // [2][n][RR]
    Cx *red = vbuf + 2 * (size_t)n * RR;                                               // [GM-1][NQ][TPG]
    uint64_t *full = reinterpret_cast<uint64_t *>(red + (size_t)(GM - 1) * NQ * TPG);
    uint64_t *empty = full + a.nstage;
    Cx *P = a.planes + (long)kz * ny * Rn * n;
    const int cpl = (n + a.rows_per_stage - 1) / a.rows_per_stage;
    const long nseq = (long)(2 * ny - 1) * cpl;
    const int NB = (n + kTileM - 1) / kTileM;   // row blocks

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CW);
        }
        fence_mbar_init_cluster();
    }
    for (int q = threadIdx.x; q < 2 * n * RR; q += blockDim.x) {
        const int m = (q / RR) % n, r = q % RR;
        vbuf[q] = (q < n * RR && r < Rn) ? adj_in<float, ADJ>(a, 0, m, P[(long)r * n + m]) : make_float2(0, 0);
    }
    __syncthreads();

    if (warp == CW) {
        if (lane == 0) {
            long seq = 0;
            for (; seq < nseq; seq++) {
                const int s = (int)(seq % a.nstage);
                const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
                if (!mbar_wait_bounded_cta(smem_u32(&empty[s]), ph ^ 1u, a.wait_limit)) {
                    // stop issuing: the consumers' bounded waits on full[] expire in turn
                    atomicOr(a.status, 4);
                    break;
                }
                int rows;
                const Cx *src = stage_src(a, kz, seq, cpl, &rows);
                const uint32_t bytes = (uint32_t)rows * ldg * (uint32_t)sizeof(Cx);
                mbar_expect_tx(&full[s], bytes);
                bulk_g2s(ring + (size_t)s * (a.stage_bytes / sizeof(Cx)), src, bytes, &full[s]);
            }
            sweep_drain(full, a.nstage, seq);
        }
        return;
    }

    const int t = threadIdx.x;
    const int g = t / TPG, tile = t % TPG;
    const int rb = tile % RB, ib = tile / RB;
    const bool busy = ib < NB;                  // threads past the last tile only synchronize
    const int i0 = ib * kTileM, r0 = rb * kTileR;
    bool dead = false;
    long seq = 0;
    for (int step = 0; step < 2 * ny - 1; step++) {
        const bool fwd = step < ny;
        const int line = fwd ? step : 2 * ny - 2 - step;
        const Cx *v = vbuf + (size_t)(step & 1) * n * RR;
        Cx *vnext = vbuf + (size_t)((step + 1) & 1) * n * RR;
        // group 0 prefetches the values it needs to finish the tile
        Cx pre[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            pre[q] = make_float2(0, 0);
            const int i = i0 + q / kTileR, r = r0 + q % kTileR;
            if (g == 0 && busy && i < n && r < Rn) {
                if (fwd && line + 1 < ny)
                    pre[q] = adj_in<float, ADJ>(a, line + 1, i, P[((long)(line + 1) * Rn + r) * n + i]);
                else if (!fwd)
                    pre[q] = P[((long)line * Rn + r) * n + i];
            }
        }
        float2 acc[kTileM][kTileR];
#pragma unroll
        for (int x = 0; x < kTileM; x++)
#pragma unroll
            for (int y = 0; y < kTileR; y++) acc[x][y] = make_float2(0, 0);
        for (int ch = 0; ch < cpl; ch++, seq++) {
            const int s = (int)(seq % a.nstage);
            const uint32_t ph = (uint32_t)((seq / a.nstage) & 1);
            if (!dead && !mbar_wait_bounded_cta(smem_u32(&full[s]), ph, a.wait_limit)) {
                dead = true;
                atomicOr(a.status, 4);
            }
            const Cx *st = ring + (size_t)s * (a.stage_bytes / sizeof(Cx));
            const int m0 = ch * a.rows_per_stage;
            const int rows = min(a.rows_per_stage, n - m0);
            if (busy) {
#pragma unroll 2
                for (int ml = g; ml < rows; ml += GM) {
                    const float4 ga = *reinterpret_cast<const float4 *>(st + (long)ml * ldg + i0);
                    const float4 gb = *reinterpret_cast<const float4 *>(st + (long)ml * ldg + i0 + 2);
                    const float4 va = *reinterpret_cast<const float4 *>(v + (size_t)(m0 + ml) * RR + r0);
                    const float4 vb = *reinterpret_cast<const float4 *>(v + (size_t)(m0 + ml) * RR + r0 + 2);
                    const float2 gg[4] = {make_float2(ga.x, ga.y), make_float2(ga.z, ga.w), make_float2(gb.x, gb.y),
                                          make_float2(gb.z, gb.w)};
                    const float2 vv[4] = {make_float2(va.x, va.y), make_float2(va.z, va.w), make_float2(vb.x, vb.y),
                                          make_float2(vb.z, vb.w)};
#pragma unroll
                    for (int x = 0; x < kTileM; x++)
#pragma unroll
                        for (int y = 0; y < kTileR; y++) acc[x][y] = cfma(gg[x], vv[y], acc[x][y]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&empty[s]);
        }
        // partial tiles of groups 1..GM-1 to shared memory ([q][tile]: a warp's stores are contiguous)
        if (GM > 1) {
            if (g > 0) {
#pragma unroll
                for (int q = 0; q < NQ; q++) red[((size_t)(g - 1) * NQ + q) * TPG + tile] = acc[q / kTileR][q % kTileR];
            }
            consumer_barrier_n<CW>();
        }
        if (g == 0 && busy) {
            const Cx cn = (fwd && line + 1 < ny) ? a.cmy[line + 1] : make_float2(0, 0);
            const Cx cp = fwd ? make_float2(0, 0) : a.cpy[line];
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int x = q / kTileR, y = q % kTileR;
                float2 sum = acc[x][y];
#pragma unroll
                for (int h = 1; h < GM; h++) {
                    const float2 o = red[((size_t)(h - 1) * NQ + q) * TPG + tile];
                    sum.x += o.x;
                    sum.y += o.y;
                }
                const int i = i0 + x, r = r0 + y;
                if (i >= n || r >= Rn) continue;
                Cx out, vn;
                bool last;
                if (fwd) {
                    out = sum;
                    last = line + 1 == ny;
                    vn = last ? out : cfms(cn, out, pre[q]);
                } else {
                    out = cfms(cp, sum, pre[q]);
                    last = true;
                    vn = out;
                }
                P[((long)line * Rn + r) * n + i] = last ? adj_out<float, ADJ>(a, line, i, out) : out;
                vnext[(size_t)i * RR + r] = vn;
            }
        }
        consumer_barrier_n<CW>();
    }
}

// RR right-hand sides per CTA, one CTA per kz
constexpr int kTiledWarps = 8;

template <int RR, bool ADJ> static int sweep_tiled_rr(const SweepArgs &sa, cudaStream_t st) {
    typedef float2 Cx;
    SweepK<float> k;
    k.n = sa.n;
    k.ny = sa.ny;
    k.ldg = sa.ldg;
    k.nrhs = sa.R;
    k.Gt = (const Cx *)sa.Gt;
    k.cmy = (const Cx *)sa.cmy;
    k.cpy = (const Cx *)sa.cpy;
    k.planes = (Cx *)sa.planes;
    k.dxy = (const Cx *)sa.dxy;
    k.status = sa.status;
    k.kzslot = sa.kzslot;
    k.expire_test = 0;
    k.wait_limit = wait_limit_polls(kSweepWaitLimit);
    // groups: the largest power of two GM with tiles <= threads per group
    constexpr int CT = kTiledWarps * 32;
    const int tiles = ((sa.n + kTileM - 1) / kTileM) * (RR / kTileR);
    int gm = 1;
    while (gm < kTiledWarps && tiles <= CT / (gm * 2)) gm *= 2;
    if (tiles > CT) return HELM3D_ERR_ARG;
    const size_t vbytes = sizeof(Cx) * 2 * (size_t)sa.n * RR;
    const size_t rbytes = sizeof(Cx) * (size_t)(gm - 1) * kTileM * kTileR * (CT / gm);
    const size_t budget = device_info().smem_optin - vbytes - rbytes - 1024;
    const size_t row_bytes = (size_t)sa.ldg * sizeof(Cx);
    int rows = (int)(((size_t)sa.stage_kb * 1024) / row_bytes);
    if (rows < 1) rows = 1;
    if (rows > sa.n) rows = sa.n;
    k.rows_per_stage = rows;
    k.stage_bytes = (uint32_t)(((size_t)rows * row_bytes + 127) & ~(size_t)127);
    const size_t ring_max = (size_t)sa.ring_kb * 1024;
    size_t ring_cap = budget < ring_max ? budget : ring_max;
    int nst = (int)(ring_cap / k.stage_bytes);
    if (nst > 32) nst = 32;
    if (nst < 2) return HELM3D_ERR_ARG;
    k.nstage = nst;
    const size_t smem = (size_t)nst * k.stage_bytes + vbytes + rbytes + 2 * nst * sizeof(uint64_t);
    auto pick = [&](auto kern) -> int {
        if (!smem_limit_max(kern, smem))
            return HELM3D_ERR_CUDA;
        kern<<<dim3((unsigned)sa.nz), (kTiledWarps + 1) * 32, smem, st>>>(k);
        return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
    };
    switch (gm) {
        case 1: return pick(sweep_tiled_kernel<RR, 1, ADJ, kTiledWarps>);
        case 2: return pick(sweep_tiled_kernel<RR, 2, ADJ, kTiledWarps>);
        case 4: return pick(sweep_tiled_kernel<RR, 4, ADJ, kTiledWarps>);
        default: return pick(sweep_tiled_kernel<RR, 8, ADJ, kTiledWarps>);
    }
}

template <bool ADJ> static int sweep_tiled(const SweepArgs &sa, cudaStream_t s) {
    if (sa.R <= 4) return sweep_tiled_rr<4, ADJ>(sa, s);
    if (sa.R <= 8) return sweep_tiled_rr<8, ADJ>(sa, s);
    return sweep_tiled_rr<16, ADJ>(sa, s);
}

template <typename R, int G, int RR, bool ADJ> static int sweep_impl(const SweepArgs &sa, cudaStream_t st) {
    typedef cplx<R> Cx;
    SweepK<R> k;
    k.n = sa.n;
    k.ny = sa.ny;
    k.ldg = sa.ldg;
    k.nrhs = sa.R;
    k.Gt = (const Cx *)sa.Gt;
    k.cmy = (const Cx *)sa.cmy;
    k.cpy = (const Cx *)sa.cpy;
    k.planes = (Cx *)sa.planes;
    k.dxy = (const Cx *)sa.dxy;
    k.status = sa.status;
    k.kzslot = sa.kzslot;
    k.wait_limit = wait_limit_polls(kSweepWaitLimit);
    {
        const char *e = std::getenv("HELM3D_TEST_EXPIRE_WAIT");
        k.expire_test = (e && *e && *e != '0') ? 1 : 0;
    }
    const size_t vbytes = sizeof(Cx) * 2 * (size_t)sa.n * RR;
    const size_t budget = device_info().smem_optin - vbytes - 1024;
    // stages of about stage_kb, as many as fit the rest of shared memory
    // (at most ring_kb)
    const size_t row_bytes = (size_t)sa.ldg * sizeof(Cx);
    int rows = (int)(((size_t)sa.stage_kb * 1024) / row_bytes);
    if (rows < 1) rows = 1;
    if (rows > sa.n) rows = sa.n;
    k.rows_per_stage = rows;
    k.stage_bytes = (uint32_t)(((size_t)rows * row_bytes + 127) & ~(size_t)127);
    const size_t ring_max = (size_t)sa.ring_kb * 1024;
    size_t ring_cap = budget < ring_max ? budget : ring_max;
    int nst = (int)(ring_cap / k.stage_bytes);
    if (nst > 32) nst = 32;
    if (nst < 2) return HELM3D_ERR_ARG;
    k.nstage = nst;
    const size_t smem = (size_t)nst * k.stage_bytes + vbytes + (2 * nst + 1) * sizeof(uint64_t);
    auto kern = sweep_kernel<R, G, RR, ADJ>;
    if (!smem_limit_max(kern, smem))
        return HELM3D_ERR_CUDA;
    kern<<<dim3((unsigned)sa.nz), (kSweepConsumerWarps + 1) * 32, smem, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

template <typename R, int G, bool ADJ> static int sweep_rr(const SweepArgs &sa, cudaStream_t s) {
    if (sa.R <= 1) return sweep_impl<R, G, 1, ADJ>(sa, s);
    if (sa.R <= 2) return sweep_impl<R, G, 2, ADJ>(sa, s);
    if (sa.R <= 4) return sweep_impl<R, G, 4, ADJ>(sa, s);
    if (sa.R <= 8) return sweep_impl<R, G, 8, ADJ>(sa, s);
    return sweep_impl<R, G, 16, ADJ>(sa, s);
}

template <typename R, int G> static int sweep_g(const SweepArgs &sa, cudaStream_t s) {
    return sa.dxy ? sweep_rr<R, G, true>(sa, s) : sweep_rr<R, G, false>(sa, s);
}

void sweep_variant(int v, SweepArgs &a) {
    static const int kStage[kSweepVariants] = {16, 8, 32, 16, 8, 32, 16, 16, 16, 16};
    static const int kRingKb[kSweepVariants] = {200, 200, 200, 100, 100, 100, 200, 200, 200, 200};
    static const int kTcMc[kSweepVariants] = {0, 0, 0, 0, 0, 0, 32, 16, 32, 0};
    static const int kTcF16[kSweepVariants] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 0};
    static const int kTcPack[kSweepVariants] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1};
    if (v < 0 || v >= kSweepVariants) v = 0;
    a.stage_kb = kStage[v];
    a.ring_kb = kRingKb[v];
    a.tc_mc = kTcMc[v];
    a.tc_f16 = kTcF16[v];
    a.tc_pack = kTcPack[v];
}

static int launch_sweep_kernels(bool c64, const SweepArgs &sa, cudaStream_t s);

int launch_sweep(bool c64, const SweepArgs &sa, cudaStream_t s) {
    const int rc = launch_sweep_kernels(c64, sa, s);
    if (rc || sa.nskip <= 0) return rc;
    return launch_kzskip_apply(c64, sa, s);   // the skipped modes, which the sweep kernels left
}

static int launch_sweep_kernels(bool c64, const SweepArgs &sa, cudaStream_t s) {
    if (sa.n < 1 || sa.n > kSweepMaxN || sa.R < 1 || sa.R > kMaxBatch) return HELM3D_ERR_ARG;
    // the tensor-core kernel where it applies (complex64, n <= 256, shared memory fits)
    if (c64 && sa.tc_mc && sweep_tc_supported(sa)) return launch_sweep_tc(sa, sa.tc_mc, s);
    if (c64 && sa.tc_pack && sweep_tcp_supported(sa)) return launch_sweep_tcp(sa, s);
    // complex64 batches of 3 or more: the register-tiled kernel (its 16-byte
    // tile loads need ldg, the padded row length, to be a multiple of 4)
    if (c64 && sa.R >= 3 && sa.ldg % 4 == 0) return sa.dxy ? sweep_tiled<true>(sa, s) : sweep_tiled<false>(sa, s);
    const int g = sa.n <= 64 ? 4 : (sa.n <= 128 ? 2 : 1);
    if (c64) {
        if (g == 4) return sweep_g<float, 4>(sa, s);
        if (g == 2) return sweep_g<float, 2>(sa, s);
        return sweep_g<float, 1>(sa, s);
    }
    if (g == 4) return sweep_g<double, 4>(sa, s);
    if (g == 2) return sweep_g<double, 2>(sa, s);
    return sweep_g<double, 1>(sa, s);
}

}  // namespace h3d
