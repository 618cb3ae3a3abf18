// sweep_tc.cu -- the block sweep of sweep.cu for complex64 batches of
// right-hand sides on the 5th-generation tensor cores (tcgen05, kind::tf32,
// FP32-class products by 3xTF32: a_hi b_hi + a_hi b_lo + a_lo b_hi, as two
// MMAs per K step: a_hi [b_hi; b_lo] with N = 4 RR, and a_lo b_hi).
// Same recurrence (the per-kz 2D solve replacing PARDISO phase 33,
// Source/functions.cpp:5959, and DirSolveFastDiagStruct,
// Source/HODLR/BinaryTreesHODLR.cpp:2971-3018):
//   forward   y_0 = G_0 f_0,   y_j = G_j (f_j - cmy[j] y_{j-1})
//   backward  x_{ny-1} = y_{ny-1},   x_j = y_j - cpy[j] G_j x_{j+1}
// One CTA per kz, all RR (8 or 16, padded) right-hand sides at once: each
// line is the real GEMM
//   D[i][2r + c] = sum_K A[i][K] B[2r + c][K],   K = 2m + c'  (m < n, c' = re/im)
// with A = G_j (row i, complex interleaved along K: the natural layout of
// G) and B the real form of the line's input v (B[2r][2m] = Re v[m][r],
// B[2r][2m+1] = -Im v, B[2r+1][2m] = Im v, B[2r+1][2m+1] = Re v), so that
// D[i][2r] + i D[i][2r+1] = (G_j v)[i][r].  M = 128 (rows i, n <= 128),
// N = 2 RR, K = 2 n padded to the chunk.
//
// Roles (15 warps):
//   * warp 12, one lane: streams G_j^T (rows m, i contiguous, as the factor
//     stores it) chunk by chunk (MC rows m) into a ring of shared-memory
//     stages with 1D bulk copies, as far ahead as the ring allows;
//   * warps 0-3 (converters): thread i of warp i / 32 reads G^T[m][i] for
//     every m of the chunk, splits it into tf32 hi + lo and stores both into
//     TMEM (lane i, column K), one of three chunk buffers, running ahead of
//     the MMAs as far as the buffers allow;
//   * warps 4-11 (epilogue): at the end of a line read D from TMEM (warp
//     4 + e: lanes 32 (e % 4) + [0, 32), the columns of half the right-hand
//     sides), finish the line (y or x into the planes), write the next
//     line's v to shared memory and from it the next B (hi and lo, canonical
//     no-swizzle K-major layout, 16-byte units in address order so that the
//     stores of a warp are contiguous);
//   * warps 13 and 14, one lane each: issue the MMAs of a line (A from TMEM,
//     B from shared memory) chunk by chunk as the buffers fill, and commit
//     them to the buffer-free barriers and, after the last chunk, to the
//     accumulator-ready barrier.  The issuing thread waits about 70 cycles
//     per tcgen05.mma whatever its N (measured on the B200), while two
//     issuers' MMAs run side by side, so the line's MMAs are split between
//     two issuers: with two row blocks issuer u takes row block u, with one
//     issuer 0 takes the a_hi [b_hi; b_lo] products and issuer 1 the
//     a_lo b_hi products, into an accumulator of their own.
// The dependence chain per line is MMAs -> epilogue -> B; the conversion of
// the next chunks and the bulk copies run beside it.  Ring positions advance
// by counters (no integer division in the loops).  Every wait is bounded; on
// expiry bit 2 of *status is set and the kernel runs on without waiting
// (results then invalid), waits (bounded) for its own MMAs and bulk copies,
// frees its TMEM and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kTcConvWarps = 4;          // warps 0-3: G^T chunks -> TMEM
constexpr int kTcEpiWarps = 8;           // warps 4-11: finish each line, build the next B
constexpr int kTcProducerWarp = kTcConvWarps + kTcEpiWarps;
constexpr int kTcMmaWarp = kTcProducerWarp + 1;   // first of the MMA issuers
constexpr int kTcMmaWarps = 2;
constexpr int kTcThreads = (kTcMmaWarp + kTcMmaWarps) * 32;
constexpr int kTcMaxN = 256;             // two row blocks of MMA M = 128
constexpr int kTcBuf = 3;                // TMEM A chunk buffers
constexpr uint32_t kTcCols = 512;        // TMEM columns: D of row block rb at 4 RR rb, buffers from 128
constexpr uint32_t kTcWaitLimit = 1u << 22;

struct SweepTcK {
    int n, ny, ldg, nrhs;
    const float *gscale; // FP16 products: power-of-two scale of each block G_j ([nz][ny])
    int npad;            // n rounded up to the chunk (K = 2 npad)
    int cpl;             // chunks per line
    int nstage;          // bulk-copy ring depth
    uint32_t stage_bytes;
    const float2 *Gt;
    const float2 *cmy, *cpy;
    float2 *planes;
    const float2 *dxy;   // adjoint scaling table (see sweep.cu), or null
    int *status;
    const int *kzslot;   // >= 0: a skipped mode (launch_kzskip_apply handles it), or null
};

__device__ __forceinline__ void tc_epilogue_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
}

template <bool ADJ> __device__ __forceinline__ float2 tc_adj_in(const SweepTcK &a, int line, int i, float2 f) {
    if (!ADJ) return f;
    return cmul(a.dxy[(long)line * a.n + i], make_float2(f.x, -f.y));
}
template <bool ADJ> __device__ __forceinline__ float2 tc_adj_out(const SweepTcK &a, int line, int i, float2 x) {
    if (!ADJ) return x;
    return cmul(make_float2(x.x, -x.y), a.dxy[(long)(a.ny + line) * a.n + i]);
}

// MB row blocks of 128 rows i (n <= 128 MB).  TMEM: the accumulator of row
// block rb at columns [2 NR rb, 2 NR (rb + 1)) (with one row block, the
// a_lo b_hi products in their own at [2 NR, 3 NR)); chunk buffer b at 128 + b BW,
// row block rb's hi at + 2 KC rb, its lo KC further (3 buffers fit for
// MB = 1 with MC <= 32 and for MB = 2 with MC = 16, or MC = 32 with F16).
//
// F16: the products in kind::f16 (K = 16 per MMA, half the MMAs of tf32)
// with FP16 hi/lo splits (11 + 11 significant bits, as tf32's), G_j scaled
// by its power-of-two block scale and each right-hand side's v by a power of
// two chosen per line from its largest entry (so that the largest scaled
// entries lie in [2^13, 2^14) and the lo parts stay normal), the
// accumulator unscaled exactly in the epilogue.  A packs one complex m per
// TMEM column (re | im as two halves).
template <int RR, int MC, int MB, bool ADJ, bool F16>
__global__ void __launch_bounds__(kTcThreads, 1) sweep_tc_kernel(SweepTcK a) {
    constexpr int NR = 2 * RR;        // B rows = D columns
    constexpr int KC = F16 ? MC : 2 * MC;   // TMEM columns of hi, and of lo, per chunk (K = 2 MC)
    constexpr int RH = RR / 2;        // right-hand sides per epilogue warp
    constexpr int BW = MB * 2 * KC;   // TMEM columns of one chunk buffer
    static_assert((MB == 2 ? 4 * NR : 3 * NR) <= 128 && 128 + kTcBuf * BW <= (int)kTcCols, "TMEM layout");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, ldg = a.ldg, Rn = a.nrhs, npad = a.npad, cpl = a.cpl;
    const int Kp = 2 * npad;
    const int kz = blockIdx.x;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nsteps = 2 * ny - 1;
    const long nseq = (long)nsteps * cpl;

    unsigned char *ring = smem_raw;
    float *Bhi = reinterpret_cast<float *>(smem_raw + (size_t)a.nstage * a.stage_bytes);
    // B_lo follows B_hi as further 8-row groups (FP16: half the bytes)
    float *Blo = Bhi + (size_t)NR * Kp / (F16 ? 2 : 1);
    const int vld = npad + 2;         // padded row of vst (bank spread across right-hand sides)
    float2 *vst = reinterpret_cast<float2 *>(Bhi + 2 * (size_t)NR * Kp / (F16 ? 2 : 1));   // [RR][vld]
    float *vmax = reinterpret_cast<float *>(vst + (size_t)RR * vld);       // F16: [4][RR]
    uint64_t *raw_full = reinterpret_cast<uint64_t *>(vmax + 4 * RR);
    uint64_t *raw_empty = raw_full + a.nstage;
    uint64_t *a_full = raw_empty + a.nstage;
    uint64_t *a_empty = a_full + kTcBuf;
    uint64_t *b_full = a_empty + kTcBuf;
    uint64_t *d_full = b_full + 1;
    uint64_t *fin = d_full + 1;       // [kTcMmaWarps]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(fin + kTcMmaWarps);
    float2 *P = a.planes + (long)kz * ny * Rn * n;   // line j, rhs r, row i at ((j*Rn + r)*n + i)

    if (warp == 0) tmem_alloc(tslot, kTcCols);
    if (tid == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&raw_full[s], 1);
            mbar_init(&raw_empty[s], kTcConvWarps);
        }
        for (int b = 0; b < kTcBuf; b++) {
            mbar_init(&a_full[b], kTcConvWarps);
            mbar_init(&a_empty[b], kTcMmaWarps);
        }
        mbar_init(b_full, kTcEpiWarps);
        mbar_init(d_full, kTcMmaWarps);
        for (int u = 0; u < kTcMmaWarps; u++) mbar_init(&fin[u], 1);
        fence_mbar_init_cluster();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    bool dead = false;
    auto fail = [&]() {
        if (!dead) atomicOr(a.status, 4);
        dead = true;
    };
    auto wait = [&](uint64_t *bar, uint32_t parity) {
        if (!dead && !mbar_wait_bounded_cta(smem_u32(bar), parity, kTcWaitLimit)) fail();
    };

    if (warp == kTcProducerWarp) {
        // ---------------------------------------------------- producer
        if (lane == 0) {
            // G^T rows of chunk c of step t: forward lines 0..ny-1, then
            // backward lines ny-2..0, MC rows m per chunk
            RingPos rp;
            int t = 0, c = 0;
            long issued = 0;
            for (long seq = 0; seq < nseq; seq++) {
                if (seq >= a.nstage) wait(&raw_empty[rp.slot], rp.phase ^ 1u);
                if (dead) break;   // stop issuing once a wait has expired
                const int line = t < ny ? t : 2 * ny - 2 - t;
                const int m0 = c * MC;
                const int rows = min(MC, n - m0);
                const float2 *src = a.Gt + (((long)kz * ny + line) * n + m0) * (long)ldg;
                const uint32_t bytes = (uint32_t)rows * ldg * 8u;
                mbar_expect_tx(&raw_full[rp.slot], bytes);
                bulk_g2s(ring + (size_t)rp.slot * a.stage_bytes, src, bytes, &raw_full[rp.slot]);
                rp.next(a.nstage);
                issued++;
                if (++c == cpl) {
                    c = 0;
                    t++;
                }
            }
            // the copies still in flight land before the CTA exits: the
            // last use of every slot (rp is one past the final use)
            for (int k = 0; k < a.nstage && k < issued; k++) {
                int sl = rp.slot - 1 - k;
                uint32_t ph = rp.phase;
                if (sl < 0) {
                    sl += a.nstage;
                    ph ^= 1u;
                }
                mbar_wait_bounded_cta(smem_u32(&raw_full[sl]), ph, kTcWaitLimit);
            }
        }
    } else if (warp >= kTcMmaWarp) {
        // -------------------------------------------------- MMA issuers
        if (lane == 0) {
            const int u = warp - kTcMmaWarp;
            // Blo follows Bhi as further 8-row groups of the same layout, so
            // one descriptor with N = 2 NR rows covers [B_hi; B_lo]
            const uint32_t idesc2 = F16 ? umma_idesc_f16(2 * NR) : umma_idesc_tf32(2 * NR);
            const uint32_t idesc1 = F16 ? umma_idesc_f16(NR) : umma_idesc_tf32(NR);
            constexpr int KE = F16 ? 8 : 4;   // K elements per 16-byte core-matrix row
            constexpr int KS = F16 ? 16 : 8;  // K per MMA
            const uint32_t sbo = (uint32_t)(Kp / KE) * 128u;
            // descriptor of B at K = 0; K steps advance its start address
            // field (16-byte units: one core matrix of 128 bytes is 8), which
            // stays below 2^14 for any shared-memory address
            const uint64_t db0 = umma_desc(smem_u32(Bhi), 128, sbo);
            // what issuer u issues: D_rb[0, 2NR) (+)= a_hi [b_hi; b_lo] and
            // D_rb[0, NR) += a_lo b_hi for row block rb = u (two row blocks),
            // or with one row block the a_hi products into D_a = [0, 2NR)
            // (issuer 0) and the a_lo products into D_b = [2NR, 3NR) (issuer 1)
            const bool hi_part = MB == 2 || u == 0, lo_part = MB == 2 || u == 1;
            const int rb = MB == 2 ? u : 0;
            const uint32_t d_hi = tmem + (uint32_t)(rb * 2 * NR);
            const uint32_t d_lo = MB == 2 ? d_hi : tmem + (uint32_t)(2 * NR);
            RingPos bp;
            for (int t = 0; t < nsteps; t++) {
                wait(b_full, (uint32_t)(t & 1));
                tc_fence_after();
                for (int c = 0; c < cpl; c++) {
                    const int b = bp.slot;
                    wait(&a_full[b], bp.phase);
                    tc_fence_after();
                    // 8 TMEM columns of A per MMA: 8 tf32, or 16 fp16 in pairs
                    const uint32_t ahi0 = tmem + 128u + (uint32_t)(b * BW + rb * 2 * KC);
                    const uint64_t dbc = db0 + (uint64_t)((c * 2 * MC / KE) * 8);
#pragma unroll
                    for (int ks = 0; ks < 2 * MC / KS; ks++) {
                        const uint64_t db = dbc + (uint64_t)(ks * (KS / KE) * 8);
                        const uint32_t ahi = ahi0 + (uint32_t)(ks * 8);
                        const uint32_t first = (c > 0 || ks > 0) ? 1u : 0u;
                        if constexpr (F16) {
                            if (hi_part) umma_f16_ts(d_hi, ahi, db, idesc2, first);
                            if (lo_part) umma_f16_ts(d_lo, ahi + (uint32_t)KC, db, idesc1, MB == 2 ? 1u : first);
                        } else {
                            if (hi_part) umma_tf32_ts(d_hi, ahi, db, idesc2, first);
                            if (lo_part) umma_tf32_ts(d_lo, ahi + (uint32_t)KC, db, idesc1, MB == 2 ? 1u : first);
                        }
                    }
                    umma_commit(&a_empty[b]);
                    bp.next(kTcBuf);
                }
                umma_commit(d_full);
            }
            // every MMA of this issuer complete before the TMEM is freed
            umma_commit(&fin[u]);
            mbar_wait_bounded_cta(smem_u32(&fin[u]), 0u, kTcWaitLimit);
        }
    } else if (warp < kTcConvWarps) {
        // --------------------------------------------------- converters
        // warp q: TMEM lanes 32 q + [0, 32) = rows i of G_j, every m of the chunk
        const int q = warp;
        const int i = 32 * q + lane;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
        RingPos rp, bp;
        int c = 0, t = 0;
        float gs = F16 ? a.gscale[(long)kz * ny] : 1.f;   // scale of the current line's block
        for (long seq = 0; seq < nseq; seq++) {
            const int s = rp.slot, b = bp.slot;
            wait(&raw_full[s], rp.phase);
            if (seq >= kTcBuf) wait(&a_empty[b], bp.phase ^ 1u);
            tc_fence_after();
            const int rows = min(MC, n - c * MC);
            const float2 *raw = reinterpret_cast<const float2 *>(ring + (size_t)s * a.stage_bytes);
            if constexpr (F16) {
                // one complex m per TMEM column: (re | im) hi, and lo, in FP16
#pragma unroll
                for (int rb = 0; rb < MB; rb++) {
                    const int row = i + 128 * rb;
                    const uint32_t col = 128u + (uint32_t)(b * BW + rb * 2 * KC);
#pragma unroll
                    for (int h = 0; h < MC / 16; h++) {
                        float hv[16], lv[16];
#pragma unroll
                        for (int k = 0; k < 16; k++) {
                            const int ml = 16 * h + k;
                            float2 g = make_float2(0.f, 0.f);
                            if (row < n && ml < rows) g = raw[(size_t)ml * ldg + row];
                            const uint2 pk = f16_split2(g.x * gs, g.y * gs);
                            hv[k] = __uint_as_float(pk.x);
                            lv[k] = __uint_as_float(pk.y);
                        }
                        tmem_st16(trow + col + (uint32_t)(16 * h), hv);
                        tmem_st16(trow + col + (uint32_t)(KC + 16 * h), lv);
                        tmem_wait_st();
                    }
                }
            } else {
            // row block rb, 16 rows m at a time: 32 hi and 32 lo columns (K = 2 m + re/im)
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
                const int row = i + 128 * rb;
                const uint32_t col = 128u + (uint32_t)(b * BW + rb * 2 * KC);
#pragma unroll
                for (int h = 0; h < MC / 16; h++) {
                    float hv[32], lv[32];
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int ml = 16 * h + k;
                        float2 g = make_float2(0.f, 0.f);
                        if (row < n && ml < rows) g = raw[(size_t)ml * ldg + row];
                        tf32_split_fast(g.x, hv[2 * k], lv[2 * k]);
                        tf32_split_fast(g.y, hv[2 * k + 1], lv[2 * k + 1]);
                    }
                    tmem_st32(trow + col + (uint32_t)(32 * h), hv);
                    tmem_st32(trow + col + (uint32_t)(KC + 32 * h), lv);
                    tmem_wait_st();
                }
            }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_local(&raw_empty[s]);
                mbar_arrive_local(&a_full[b]);
            }
            rp.next(a.nstage);
            bp.next(kTcBuf);
            if (++c == cpl) {
                c = 0;
                if (F16 && ++t < nsteps) gs = a.gscale[(long)kz * ny + (t < ny ? t : 2 * ny - 2 - t)];
            }
        }
    } else {
        // ----------------------------------------------------- epilogue
        // warp 4 + e: TMEM lanes 32 (e % 4) + [0, 32), right-hand sides
        // (e / 4) RH + [0, RH)
        const int ew = warp - kTcConvWarps;
        const int q = ew & 3, wg = ew >> 2;
        const int i = 32 * q + lane;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);

        // B (hi, lo) of the next line from vst.  16-byte units in address
        // order: row & 7, then the K quad kq, then the 8-row group rg; the
        // NR / 8 groups are split among the warps (WPR warps each), a warp
        // writing 4 consecutive K quads of its group per pass (512
        // contiguous bytes)
        constexpr int WPR = kTcEpiWarps / (NR / 8);
        // FP16: the power-of-two scale of right-hand side r's next v, from
        // the per-quarter maxima in vmax (the same value in every thread)
        auto v_scale = [&](int r) -> float {
            float mx = 0.f;
#pragma unroll
            for (int qq = 0; qq < 4; qq++) mx = fmaxf(mx, vmax[qq * RR + r]);
            return pow2_scale_13(mx);
        };
        auto build_b = [&]() {
            const int rg = ew / WPR, rlo = lane & 7;
            const int row = rg * 8 + rlo, r = row >> 1;
            const float2 *vrow = vst + (size_t)r * vld;
            if constexpr (F16) {
                // 16-byte units of 8 K = 4 complex m, in address order (row & 7, K octet, 8-row group)
                const int ko_n = Kp / 8;
                const float sv = v_scale(r);
                for (int ko = (ew % WPR) * 4 + (lane >> 3); ko < ko_n; ko += 4 * WPR) {
                    const int u = (rg * ko_n + ko) * 8 + rlo;
                    const float4 va = *reinterpret_cast<const float4 *>(vrow + 4 * ko);
                    const float4 vb = *reinterpret_cast<const float4 *>(vrow + 4 * ko + 2);
                    float e[8];
                    if ((row & 1) == 0) {   // (Re v, -Im v)
                        e[0] = va.x; e[1] = -va.y; e[2] = va.z; e[3] = -va.w;
                        e[4] = vb.x; e[5] = -vb.y; e[6] = vb.z; e[7] = -vb.w;
                    } else {                // (Im v, Re v)
                        e[0] = va.y; e[1] = va.x; e[2] = va.w; e[3] = va.z;
                        e[4] = vb.y; e[5] = vb.x; e[6] = vb.w; e[7] = vb.z;
                    }
                    uint4 h, l;
                    uint2 p0 = f16_split2(e[0] * sv, e[1] * sv), p1 = f16_split2(e[2] * sv, e[3] * sv);
                    uint2 p2 = f16_split2(e[4] * sv, e[5] * sv), p3 = f16_split2(e[6] * sv, e[7] * sv);
                    h = make_uint4(p0.x, p1.x, p2.x, p3.x);
                    l = make_uint4(p0.y, p1.y, p2.y, p3.y);
                    reinterpret_cast<uint4 *>(Bhi)[u] = h;
                    reinterpret_cast<uint4 *>(Blo)[u] = l;
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive_local(b_full);
                return;
            }
            const int kq_n = Kp / 4;
            for (int kq = (ew % WPR) * 4 + (lane >> 3); kq < kq_n; kq += 4 * WPR) {
                const int u = (rg * kq_n + kq) * 8 + rlo;
                const float4 vv = *reinterpret_cast<const float4 *>(vrow + 2 * kq);
                float4 e;
                if ((row & 1) == 0) e = make_float4(vv.x, -vv.y, vv.z, -vv.w);   // (Re v, -Im v)
                else e = make_float4(vv.y, vv.x, vv.w, vv.z);                   // (Im v, Re v)
                float4 h, l;
                tf32_split_fast(e.x, h.x, l.x);
                tf32_split_fast(e.y, h.y, l.y);
                tf32_split_fast(e.z, h.z, l.z);
                tf32_split_fast(e.w, h.w, l.w);
                reinterpret_cast<float4 *>(Bhi)[u] = h;
                reinterpret_cast<float4 *>(Blo)[u] = l;
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive_local(b_full);
        };

        // FP16: this warp's per-right-hand-side maxima of the next v into
        // vmax[q][r] (one writer per entry; every reader of the previous
        // values is past the B-ready barrier by then)
        auto put_vmax = [&](float (&am)[RH]) {
            if constexpr (F16) {
#pragma unroll
                for (int k = 0; k < RH; k++) {
                    // non-negative floats order like their bit patterns
                    const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(am[k]));
                    if (lane == 0) vmax[q * RR + wg * RH + k] = __uint_as_float(m);
                }
            }
        };
        float sv_cur[RH];   // scales of the v this thread's line is multiplied with
#pragma unroll
        for (int k = 0; k < RH; k++) sv_cur[k] = 1.f;

        // line 0's input: f_0 of this thread's rows and right-hand sides
        {
            float am[RH];
#pragma unroll
            for (int k = 0; k < RH; k++) am[k] = 0.f;
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
                const int m = i + 128 * rb;
                if (m >= npad) continue;
#pragma unroll
                for (int k = 0; k < RH; k++) {
                    const int r = wg * RH + k;
                    const float2 f = (r < Rn && m < n) ? tc_adj_in<ADJ>(a, 0, m, P[(long)r * n + m])
                                                       : make_float2(0.f, 0.f);
                    vst[(size_t)r * vld + m] = f;
                    am[k] = fmaxf(am[k], fmaxf(fabsf(f.x), fabsf(f.y)));
                }
            }
            put_vmax(am);
        }
        tc_epilogue_barrier();
        if constexpr (F16) {
#pragma unroll
            for (int k = 0; k < RH; k++) sv_cur[k] = v_scale(wg * RH + k);
        }
        build_b();

        // What finishing step t needs besides G v, loaded one step ahead (the
        // planes do not fit in L2): f_{line+1} forward (and its adjoint
        // scale), y_line backward.  Written by this same thread earlier, or
        // untouched input.  Row i + 128 rb of row block rb.
        auto load_pre = [&](int t, float2 (&v)[MB][RH], float2 (&dx)[MB]) {
            const bool fwd = t < ny;
            const int line = fwd ? t : 2 * ny - 2 - t;
            const bool nxt = fwd && line + 1 < ny;
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
                const int row = i + 128 * rb;
#pragma unroll
                for (int k = 0; k < RH; k++) {
                    const int r = wg * RH + k;
                    v[rb][k] = make_float2(0.f, 0.f);
                    if (row < n && r < Rn) {
                        if (nxt) v[rb][k] = P[((long)(line + 1) * Rn + r) * n + row];
                        else if (!fwd) v[rb][k] = P[((long)line * Rn + r) * n + row];
                    }
                }
                dx[rb] = (ADJ && nxt && row < n) ? a.dxy[(long)(line + 1) * n + row] : make_float2(0.f, 0.f);
            }
        };
        float2 pv[MB][RH], pvn[MB][RH], dx[MB], dxn[MB];
        load_pre(0, pv, dx);

        for (int t = 0; t < nsteps; t++) {
            if (t + 1 < nsteps) load_pre(t + 1, pvn, dxn);
            const bool fwd = t < ny;
            const int line = fwd ? t : 2 * ny - 2 - t;
            const bool last_fwd = fwd && line + 1 == ny;
            const float2 cn = (fwd && !last_fwd) ? a.cmy[line + 1] : make_float2(0.f, 0.f);
            const float2 cp = fwd ? make_float2(0.f, 0.f) : a.cpy[line];
            const float igs = F16 ? pow2_inv(a.gscale[(long)kz * ny + line]) : 1.f;
            float us[RH];   // exact unscaling: 1 / (block scale * right-hand-side scale)
#pragma unroll
            for (int k = 0; k < RH; k++) us[k] = F16 ? igs * pow2_inv(sv_cur[k]) : 1.f;
            float am[RH];
#pragma unroll
            for (int k = 0; k < RH; k++) am[k] = 0.f;
            wait(d_full, (uint32_t)(t & 1));
            tc_fence_after();
            // this line's y / x, stored to the planes after the next B is
            // handed over (the stores are off the line-to-line chain)
            float2 outs[MB][RH];
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
                const int row = i + 128 * rb;
                // D = a_hi b_hi (+ a_lo b_hi with two row blocks) (columns c) +
                // a_hi b_lo (columns NR + c); with one row block a_lo b_hi at 2 NR + c
                const uint32_t dcol = (uint32_t)(rb * 2 * NR + wg * RR);
                float d[2 * RR], d3[RR];
                if constexpr (RR == 16) {
                    tmem_ld16_nowait(trow + dcol, d);
                    tmem_ld16_nowait(trow + dcol + (uint32_t)NR, d + RR);
                    if constexpr (MB == 1) tmem_ld16_nowait(trow + dcol + (uint32_t)(2 * NR), d3);
                } else {
                    tmem_ld8_nowait(trow + dcol, d);
                    tmem_ld8_nowait(trow + dcol + (uint32_t)NR, d + RR);
                    if constexpr (MB == 1) tmem_ld8_nowait(trow + dcol + (uint32_t)(2 * NR), d3);
                }
                tmem_wait_ld(d);
                if constexpr (MB == 1) {
                    tmem_wait_ld(d3);
                } else {
#pragma unroll
                    for (int k = 0; k < RR; k++) d3[k] = 0.f;
                }
#pragma unroll
                for (int k = 0; k < RH; k++) {
                    const int r = wg * RH + k;
                    const float2 pk = pv[rb][k];
                    const float2 pre = (ADJ && fwd && !last_fwd) ? cmul(dx[rb], make_float2(pk.x, -pk.y)) : pk;
                    const float2 acc = make_float2((d[2 * k] + d[RR + 2 * k] + d3[2 * k]) * us[k],
                                                   (d[2 * k + 1] + d[RR + 2 * k + 1] + d3[2 * k + 1]) * us[k]);
                    float2 out, vn;
                    bool fin_x;   // out is this line's final x
                    if (fwd) {
                        out = acc;                                        // y_line
                        fin_x = last_fwd;
                        vn = fin_x ? out : cfms(cn, out, pre);            // f_{line+1} - cmy y_line, or x_{ny-1}
                    } else {
                        out = cfms(cp, acc, pre);                         // x_line = y_line - cpy G x_{line+1}
                        fin_x = true;
                        vn = out;
                    }
                    const bool valid = row < n && r < Rn;
                    outs[rb][k] = fin_x ? tc_adj_out<ADJ>(a, line, row, out) : out;
                    if (row < npad) vst[(size_t)r * vld + row] = valid ? vn : make_float2(0.f, 0.f);
                    if (valid) am[k] = fmaxf(am[k], fmaxf(fabsf(vn.x), fabsf(vn.y)));
                }
            }
            tc_fence_before();
            if (t + 1 < nsteps) {
                put_vmax(am);
                tc_epilogue_barrier();
                if constexpr (F16) {
#pragma unroll
                    for (int k = 0; k < RH; k++) sv_cur[k] = v_scale(wg * RH + k);
                }
                build_b();
            }
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
                const int row = i + 128 * rb;
#pragma unroll
                for (int k = 0; k < RH; k++) {
                    const int r = wg * RH + k;
                    if (row < n && r < Rn) P[((long)line * Rn + r) * n + row] = outs[rb][k];
                }
            }
#pragma unroll
            for (int rb = 0; rb < MB; rb++) {
#pragma unroll
                for (int k = 0; k < RH; k++) pv[rb][k] = pvn[rb][k];
                dx[rb] = dxn[rb];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, kTcCols);
}

// ------------------------------------------------------------------- host
// Power-of-two scale of every block G_j (kz, line) for the FP16 products:
// its largest |re| or |im| scaled into [2^13, 2^14).
__global__ void __launch_bounds__(256) gscale_kernel(const float2 *Gt, int n, int ldg, float *gscale) {
    __shared__ float wmax[8];
    const float2 *g = Gt + (long)blockIdx.x * n * ldg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float mx = 0.f;
    for (int m = warp; m < n; m += 8)
        for (int i = lane; i < n; i += 32) {
            const float2 v = g[(long)m * ldg + i];
            mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (lane == 0) wmax[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) mx = fmaxf(mx, wmax[w]);
        gscale[blockIdx.x] = pow2_scale_13(mx);
    }
}

int launch_gscale(const void *Gt, int n, int ny, int nz, int ldg, float *gscale, cudaStream_t s) {
    gscale_kernel<<<dim3((unsigned)(ny * nz)), 256, 0, s>>>((const float2 *)Gt, n, ldg, gscale);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

// The launch shape of a batch: RR right-hand sides (8 or 16), chunk rows MC,
// row blocks MB, FP16 or TF32 products, ring depth and shared memory; false
// when it does not fit.
struct TcShape {
    int RR, MC, MB, npad, nstage;
    bool f16;
    uint32_t stage_bytes;
    size_t smem;
};

static bool tc_shape(const SweepArgs &sa, int mc, TcShape &sh) {
    if (sa.n < 1 || sa.n > kTcMaxN || sa.R < 1 || sa.R > 16) return false;
    sh.f16 = sa.tc_f16 != 0;
    if (sh.f16 && !sa.gscale) return false;
    sh.RR = sa.R <= 8 ? 8 : 16;
    sh.MB = sa.n > 128 ? 2 : 1;
    // FP16 products: 32-row chunks; TF32: as asked, 16-row chunks with two row blocks (TMEM)
    sh.MC = sh.f16 ? 32 : ((sh.MB == 2 || mc == 16) ? 16 : 32);
    sh.npad = ((sa.n + sh.MC - 1) / sh.MC) * sh.MC;
    sh.stage_bytes = (uint32_t)((((size_t)sh.MC * sa.ldg * 8) + 127) & ~(size_t)127);
    // B hi and lo: tf32 words, or FP16 halves (half the bytes)
    const size_t bbytes = 2 * sizeof(float) * (size_t)(2 * sh.RR) * (2 * sh.npad) / (sh.f16 ? 2 : 1);
    const size_t vbytes = sizeof(float2) * (size_t)sh.RR * (sh.npad + 2) + sizeof(float) * 4 * sh.RR;
    const size_t fixed = bbytes + vbytes + sizeof(uint64_t) * (2 * kTcBuf + 2 + kTcMmaWarps) + 16;
    const size_t optin = device_info().smem_optin;
    const size_t per_stage = sh.stage_bytes + 2 * sizeof(uint64_t);
    if (fixed + 2 * per_stage > optin) return false;
    int nst = (int)((optin - fixed) / per_stage);
    const int ring_cap = (int)(((size_t)sa.ring_kb * 1024) / sh.stage_bytes);
    if (nst > ring_cap) nst = ring_cap;
    if (nst > 8) nst = 8;
    if (nst < 2) return false;
    sh.nstage = nst;
    sh.smem = (size_t)nst * per_stage + fixed;
    return true;
}

bool sweep_tc_supported(const SweepArgs &sa) {
    TcShape sh;
    return tc_shape(sa, sa.tc_mc, sh);
}

template <int RR, int MC, int MB, bool ADJ, bool F16>
static int sweep_tc_impl(const SweepArgs &sa, const TcShape &sh, cudaStream_t st) {
    SweepTcK k;
    k.n = sa.n;
    k.ny = sa.ny;
    k.ldg = sa.ldg;
    k.nrhs = sa.R;
    k.gscale = sa.gscale;
    k.npad = sh.npad;
    k.cpl = sh.npad / MC;
    k.Gt = (const float2 *)sa.Gt;
    k.cmy = (const float2 *)sa.cmy;
    k.cpy = (const float2 *)sa.cpy;
    k.planes = (float2 *)sa.planes;
    k.dxy = (const float2 *)sa.dxy;
    k.status = sa.status;
    k.kzslot = sa.kzslot;
    k.stage_bytes = sh.stage_bytes;
    k.nstage = sh.nstage;
    auto kern = sweep_tc_kernel<RR, MC, MB, ADJ, F16>;
    if (!smem_limit_max(kern, sh.smem))
        return HELM3D_ERR_CUDA;
    kern<<<dim3((unsigned)sa.nz), kTcThreads, sh.smem, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

template <bool ADJ> static int sweep_tc_adj(const SweepArgs &sa, const TcShape &sh, cudaStream_t s) {
    if (sh.f16) {
        if (sh.MB == 2) {
            if (sh.RR == 8) return sweep_tc_impl<8, 32, 2, ADJ, true>(sa, sh, s);
            return sweep_tc_impl<16, 32, 2, ADJ, true>(sa, sh, s);
        }
        if (sh.RR == 8) return sweep_tc_impl<8, 32, 1, ADJ, true>(sa, sh, s);
        return sweep_tc_impl<16, 32, 1, ADJ, true>(sa, sh, s);
    }
    if (sh.MB == 2) {
        if (sh.RR == 8) return sweep_tc_impl<8, 16, 2, ADJ, false>(sa, sh, s);
        return sweep_tc_impl<16, 16, 2, ADJ, false>(sa, sh, s);
    }
    if (sh.MC == 16) {
        if (sh.RR == 8) return sweep_tc_impl<8, 16, 1, ADJ, false>(sa, sh, s);
        return sweep_tc_impl<16, 16, 1, ADJ, false>(sa, sh, s);
    }
    if (sh.RR == 8) return sweep_tc_impl<8, 32, 1, ADJ, false>(sa, sh, s);
    return sweep_tc_impl<16, 32, 1, ADJ, false>(sa, sh, s);
}

int launch_sweep_tc(const SweepArgs &sa, int mc, cudaStream_t s) {
    TcShape sh;
    if (!tc_shape(sa, mc, sh)) return HELM3D_ERR_ARG;
    return sa.dxy ? sweep_tc_adj<true>(sa, sh, s) : sweep_tc_adj<false>(sa, sh, s);
}

}  // namespace h3d
