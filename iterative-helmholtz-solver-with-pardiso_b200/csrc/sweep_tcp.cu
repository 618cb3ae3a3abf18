// sweep_tcp.cu -- the tensor-core block sweep of complex64 batches with the
// factor packed once, after the block LU factor, into FP16 hi/lo tiles in
// the tensor core's shared-memory operand layout, so that the sweep streams
// them by bulk copies straight into the MMAs' A operand: no per-sweep
// conversion of G and no TMEM copy of it.  Same recurrence as sweep.cu and
// sweep_tc.cu (the per-kz 2D solve replacing PARDISO phase 33,
// Source/functions.cpp:5959, and DirSolveFastDiagStruct,
// Source/HODLR/BinaryTreesHODLR.cpp:2971-3018):
//   forward   y_0 = G_0 f_0,   y_j = G_j (f_j - cmy[j] y_{j-1})
//   backward  x_{ny-1} = y_{ny-1},   x_j = y_j - cpy[j] G_j x_{j+1}
// and the same real GEMM per line as sweep_tc.cu,
//   D[i][2r + c] = sum_K A[i][K] B[2r + c][K],   K = 2m + (re, im),
// A = s_j G_j (s_j the block's power-of-two scale) as FP16 hi + lo, B the
// real form of the line's input v scaled per right-hand side by a power of
// two, as FP16 hi + lo; D = a_hi b_hi + a_hi b_lo + a_lo b_hi in FP32
// (kind::f16, K = 16 per MMA), unscaled exactly in the epilogue.
//
// Packed factor (launch_gpack): block (kz, j), chunk c (complex m in
// [16 c, 16 c + 16)) is two tiles, hi then lo, of n8 = n rounded to 8 rows i,
// each row 32 FP16 values along K (m re, m im, ...): 8-row groups of 512
// bytes, each 4 core matrices (8 rows x 16 bytes, K-adjacent 128 bytes
// apart).  Rows i >= n and m >= n are zero.  Same bytes as the complex64
// block (8 per entry).  A row block of 128 rows read through a tile of fewer
// rows takes its last rows from whatever shared memory follows; those rows
// of D are never read.
//
// Roles (11 warps): warps 0-7 epilogue (as sweep_tc.cu: D from TMEM, finish
// the line, the next B), warp 8 one lane: bulk copies of the packed chunks
// into a ring of stages, warps 9-10 one lane each: the MMAs (A and B from
// shared memory), split between the two issuers as in sweep_tc.cu, each
// chunk's MMAs committed to the stage's empty barrier.  Every wait is
// bounded; on expiry bit 2 of *status is set, the producer stops issuing and
// drains its copies, the issuers wait (bounded) for their MMAs, TMEM is freed
// and the kernel returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kTpEpiWarps = 8;            // warps 0-7
constexpr int kTpProducerWarp = 8;
constexpr int kTpMmaWarp = 9;             // warps 9, 10
constexpr int kTpMmaWarps = 2;
constexpr int kTpThreads = (kTpMmaWarp + kTpMmaWarps) * 32;
constexpr int kTpMC = 16;                 // complex m per chunk
constexpr uint32_t kTpRowBytes = 64;      // one tile row: 32 FP16 along K
constexpr uint32_t kTpSbo = 8 * kTpRowBytes;   // 8-row group
constexpr uint32_t kTpCols = 128;         // TMEM: the accumulators only
constexpr uint32_t kTpWaitLimit = 1u << 22;

struct SweepTpK {
    int n, ny, nrhs, npad, cpl, nstage;
    uint32_t tile_bytes;    // one tile: n8 rows x 64 bytes
    const unsigned char *Gp;
    const float *gscale;
    const float2 *cmy, *cpy;
    float2 *planes;
    const float2 *dxy;      // adjoint scaling table (see sweep.cu), or null
    int *status;
    const int *kzslot;      // >= 0: a skipped mode (launch_kzskip_apply handles it), or null
};

__device__ __forceinline__ void tp_epilogue_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kTpEpiWarps * 32) : "memory");
}

template <bool ADJ> __device__ __forceinline__ float2 tp_adj_in(const SweepTpK &a, int line, int i, float2 f) {
    if (!ADJ) return f;
    return cmul(a.dxy[(long)line * a.n + i], make_float2(f.x, -f.y));
}
template <bool ADJ> __device__ __forceinline__ float2 tp_adj_out(const SweepTpK &a, int line, int i, float2 x) {
    if (!ADJ) return x;
    return cmul(make_float2(x.x, -x.y), a.dxy[(long)(a.ny + line) * a.n + i]);
}

// RR right-hand sides (8 or 16, padded), MB row blocks of 128 rows.  TMEM:
// the accumulator of row block rb at columns [2 NR rb, 2 NR (rb + 1)); with
// one row block the a_lo b_hi products in their own at [2 NR, 3 NR).
template <int RR, int MB, bool ADJ>
__global__ void __launch_bounds__(kTpThreads, 1) sweep_tcp_kernel(SweepTpK a) {
    constexpr int NR = 2 * RR;        // B rows = D columns
    constexpr int RH = RR / 2;        // right-hand sides per epilogue warp
    static_assert((MB == 2 ? 4 * NR : 3 * NR) <= (int)kTpCols, "TMEM layout");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int n = a.n, ny = a.ny, Rn = a.nrhs, npad = a.npad, cpl = a.cpl;
    const int Kp = 2 * npad;
    const int kz = blockIdx.x;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nsteps = 2 * ny - 1;
    const long nseq = (long)nsteps * cpl;
    const uint32_t stage_bytes = 2 * a.tile_bytes;

    unsigned char *ring = smem_raw;
    float *Bhi = reinterpret_cast<float *>(smem_raw + (size_t)a.nstage * stage_bytes);
    float *Blo = Bhi + (size_t)NR * Kp / 2;   // B_lo follows B_hi as further 8-row groups
    const int vld = npad + 2;                 // padded row of vst
    float2 *vst = reinterpret_cast<float2 *>(Bhi + (size_t)NR * Kp);   // [RR][vld]
    float *vmax = reinterpret_cast<float *>(vst + (size_t)RR * vld);   // [4][RR]
    uint64_t *full = reinterpret_cast<uint64_t *>(vmax + 4 * RR);      // [nstage]
    uint64_t *empty = full + a.nstage;                                 // [nstage]
    uint64_t *b_full = empty + a.nstage;
    uint64_t *d_full = b_full + 1;
    uint64_t *fin = d_full + 1;                                        // [kTpMmaWarps]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(fin + kTpMmaWarps);
    float2 *P = a.planes + (long)kz * ny * Rn * n;   // line j, rhs r, row i at ((j*Rn + r)*n + i)

    if (warp == 0) tmem_alloc(tslot, kTpCols);
    if (tid == 0) {
        for (int s = 0; s < a.nstage; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTpMmaWarps);
        }
        mbar_init(b_full, kTpEpiWarps);
        mbar_init(d_full, kTpMmaWarps);
        for (int u = 0; u < kTpMmaWarps; u++) mbar_init(&fin[u], 1);
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
        if (!dead && !mbar_wait_bounded_cta(smem_u32(bar), parity, kTpWaitLimit)) fail();
    };

    if (warp == kTpProducerWarp) {
        // ---------------------------------------------------- producer
        if (lane == 0) {
            // chunk c of step t: forward lines 0..ny-1, then backward lines
            // ny-2..0; its hi and lo tiles into the first and second half of
            // the stage
            const size_t block_bytes = (size_t)cpl * 2 * a.tile_bytes;
            RingPos rp;
            int t = 0, c = 0;
            long issued = 0;
            for (long seq = 0; seq < nseq; seq++) {
                if (seq >= a.nstage) wait(&empty[rp.slot], rp.phase ^ 1u);
                if (dead) break;   // stop issuing once a wait has expired
                const int line = t < ny ? t : 2 * ny - 2 - t;
                const unsigned char *src =
                    a.Gp + ((size_t)kz * ny + line) * block_bytes + (size_t)c * 2 * a.tile_bytes;
                unsigned char *dst = ring + (size_t)rp.slot * stage_bytes;
                mbar_expect_tx(&full[rp.slot], 2 * a.tile_bytes);
                bulk_g2s(dst, src, a.tile_bytes, &full[rp.slot]);
                bulk_g2s(dst + a.tile_bytes, src + a.tile_bytes, a.tile_bytes, &full[rp.slot]);
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
                mbar_wait_bounded_cta(smem_u32(&full[sl]), ph, kTpWaitLimit);
            }
        }
    } else if (warp >= kTpMmaWarp) {
        // -------------------------------------------------- MMA issuers
        if (lane == 0) {
            const int u = warp - kTpMmaWarp;
            // B: Blo follows Bhi as further 8-row groups, so one descriptor
            // with N = 2 NR rows covers [B_hi; B_lo].  K steps advance the
            // descriptors' start address field (16-byte units), which stays
            // below 2^14 for any shared-memory address.
            const uint32_t idesc2 = umma_idesc_f16(2 * NR), idesc1 = umma_idesc_f16(NR);
            const uint64_t db0 = umma_desc(smem_u32(Bhi), 128, (uint32_t)(Kp / 8) * 128u);
            // issuer u: row block u (two row blocks), or with one row block
            // the a_hi products into D_a (u = 0) and the a_lo products into D_b (u = 1)
            const bool hi_part = MB == 2 || u == 0, lo_part = MB == 2 || u == 1;
            const int rb = MB == 2 ? u : 0;
            const uint32_t d_hi = tmem + (uint32_t)(rb * 2 * NR);
            const uint32_t d_lo = MB == 2 ? d_hi : tmem + (uint32_t)(2 * NR);
            // A: the stage's hi tile from row block rb's first 8-row group
            const uint64_t da0 = umma_desc(smem_u32(ring) + (uint32_t)rb * 16u * kTpSbo, 128, kTpSbo);
            RingPos sp;
            for (int t = 0; t < nsteps; t++) {
                wait(b_full, (uint32_t)(t & 1));
                tc_fence_after();
                for (int c = 0; c < cpl; c++) {
                    wait(&full[sp.slot], sp.phase);
                    tc_fence_after();
                    const uint64_t dah = da0 + (uint64_t)(((uint32_t)sp.slot * stage_bytes) >> 4);
                    const uint64_t dal = dah + (uint64_t)(a.tile_bytes >> 4);
                    const uint64_t dbc = db0 + (uint64_t)(c * 2 * kTpMC / 8 * 8);
#pragma unroll
                    for (int ks = 0; ks < 2 * kTpMC / 16; ks++) {
                        // K = 16: two core matrices of A (256 bytes along the row
                        // group), two of B
                        const uint64_t db = dbc + (uint64_t)(ks * 16);
                        const uint64_t ka = (uint64_t)(ks * 16);
                        const uint32_t first = (c > 0 || ks > 0) ? 1u : 0u;
                        if (hi_part) umma_f16_ss(d_hi, dah + ka, db, idesc2, first);
                        if (lo_part) umma_f16_ss(d_lo, dal + ka, db, idesc1, MB == 2 ? 1u : first);
                    }
                    umma_commit(&empty[sp.slot]);
                    sp.next(a.nstage);
                }
                umma_commit(d_full);
            }
            // every MMA of this issuer complete before the TMEM is freed
            umma_commit(&fin[u]);
            mbar_wait_bounded_cta(smem_u32(&fin[u]), 0u, kTpWaitLimit);
        }
    } else {
        // ----------------------------------------------------- epilogue
        // warp e: TMEM lanes 32 (e % 4) + [0, 32), right-hand sides
        // (e / 4) RH + [0, RH)
        const int ew = warp;
        const int q = ew & 3, wg = ew >> 2;
        const int i = 32 * q + lane;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);

        // B (hi, lo) of the next line from vst: 16-byte units of 8 K = 4
        // complex m, in address order (row & 7, K octet, 8-row group); the
        // NR / 8 groups split among the warps (WPR warps each)
        constexpr int WPR = kTpEpiWarps / (NR / 8);
        // the power-of-two scale of right-hand side r's next v, from the
        // per-quarter maxima in vmax (the same value in every thread)
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
                const uint2 p0 = f16_split2(e[0] * sv, e[1] * sv), p1 = f16_split2(e[2] * sv, e[3] * sv);
                const uint2 p2 = f16_split2(e[4] * sv, e[5] * sv), p3 = f16_split2(e[6] * sv, e[7] * sv);
                reinterpret_cast<uint4 *>(Bhi)[u] = make_uint4(p0.x, p1.x, p2.x, p3.x);
                reinterpret_cast<uint4 *>(Blo)[u] = make_uint4(p0.y, p1.y, p2.y, p3.y);
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive_local(b_full);
        };
        // this warp's per-right-hand-side maxima of the next v into vmax[q][r]
        // (one writer per entry; every reader of the previous values is past
        // the B-ready barrier by then)
        auto put_vmax = [&](float (&am)[RH]) {
#pragma unroll
            for (int k = 0; k < RH; k++) {
                // non-negative floats order like their bit patterns
                const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(am[k]));
                if (lane == 0) vmax[q * RR + wg * RH + k] = __uint_as_float(m);
            }
        };
        float sv_cur[RH];   // scales of the v this thread's line is multiplied with

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
                    const float2 f = (r < Rn && m < n) ? tp_adj_in<ADJ>(a, 0, m, P[(long)r * n + m])
                                                       : make_float2(0.f, 0.f);
                    vst[(size_t)r * vld + m] = f;
                    am[k] = fmaxf(am[k], fmaxf(fabsf(f.x), fabsf(f.y)));
                }
            }
            put_vmax(am);
        }
        tp_epilogue_barrier();
#pragma unroll
        for (int k = 0; k < RH; k++) sv_cur[k] = v_scale(wg * RH + k);
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
            const float igs = pow2_inv(a.gscale[(long)kz * ny + line]);
            float us[RH];   // exact unscaling: 1 / (block scale * right-hand-side scale)
#pragma unroll
            for (int k = 0; k < RH; k++) us[k] = igs * pow2_inv(sv_cur[k]);
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
                    outs[rb][k] = fin_x ? tp_adj_out<ADJ>(a, line, row, out) : out;
                    if (row < npad) vst[(size_t)r * vld + row] = valid ? vn : make_float2(0.f, 0.f);
                    if (valid) am[k] = fmaxf(am[k], fmaxf(fabsf(vn.x), fabsf(vn.y)));
                }
            }
            tc_fence_before();
            if (t + 1 < nsteps) {
                put_vmax(am);
                tp_epilogue_barrier();
#pragma unroll
                for (int k = 0; k < RH; k++) sv_cur[k] = v_scale(wg * RH + k);
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
    if (warp == 0) tmem_dealloc(tmem, kTpCols);
}

// ------------------------------------------------------------- the packing
// One CTA per block (kz, j): 16-byte units (row i, chunk c, K core kc) =
// complex m = 16 c + 4 kc + [0, 4) of row i, as (re, im) FP16 pairs of the
// hi parts and of the lo parts of s_j G[i][m] (s_j = gscale).  Consecutive
// threads take consecutive rows: coalesced reads of G^T[m][i], 128-byte runs
// of writes.
__global__ void __launch_bounds__(256) gpack_kernel(const float2 *Gt, int n, int ldg, int n8, int cpl,
                                                    const float *gscale, unsigned char *Gp) {
    const long blk = blockIdx.x;
    const float2 *g = Gt + blk * n * (long)ldg;
    const uint32_t tile = (uint32_t)n8 * kTpRowBytes;
    unsigned char *out = Gp + (size_t)blk * cpl * 2 * tile;
    const float gs = gscale[blk];
    const int units = n8 * cpl * 4;
    for (int uix = threadIdx.x; uix < units; uix += blockDim.x) {
        const int i = uix % n8, rest = uix / n8;
        const int c = rest >> 2, kc = rest & 3;
        uint32_t hv[4], lv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int m = kTpMC * c + 4 * kc + k;
            float2 v = make_float2(0.f, 0.f);
            if (i < n && m < n) v = g[(long)m * ldg + i];
            const uint2 p = f16_split2(v.x * gs, v.y * gs);
            hv[k] = p.x;
            lv[k] = p.y;
        }
        const uint32_t off = (uint32_t)(i >> 3) * kTpSbo + (uint32_t)kc * 128u + (uint32_t)(i & 7) * 16u;
        unsigned char *ct = out + (size_t)c * 2 * tile;
        *reinterpret_cast<uint4 *>(ct + off) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<uint4 *>(ct + tile + off) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    }
}

size_t gpack_bytes(int n, int ny, int nz) {
    const size_t n8 = (size_t)((n + 7) & ~7), cpl = (size_t)((n + kTpMC - 1) / kTpMC);
    return (size_t)nz * ny * cpl * 2 * n8 * kTpRowBytes;
}

int launch_gpack(const void *Gt, int n, int ny, int nz, int ldg, const float *gscale, void *Gp, cudaStream_t s) {
    if (n < 1 || n > 256) return HELM3D_ERR_ARG;
    const int n8 = (n + 7) & ~7, cpl = (n + kTpMC - 1) / kTpMC;
    gpack_kernel<<<dim3((unsigned)(ny * nz)), 256, 0, s>>>((const float2 *)Gt, n, ldg, n8, cpl, gscale,
                                                          (unsigned char *)Gp);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

// ------------------------------------------------------------------ launch
// The launch shape of a batch: RR right-hand sides (8 or 16), MB row blocks,
// ring depth and shared memory; false when it does not fit.
struct TpShape {
    int RR, MB, npad, cpl, nstage;
    uint32_t tile_bytes;
    size_t smem;
};

static bool tp_shape(const SweepArgs &sa, TpShape &sh) {
    if (!sa.gpack || !sa.gscale || sa.n < 1 || sa.n > 256 || sa.R < 1 || sa.R > 16) return false;
    sh.RR = sa.R <= 8 ? 8 : 16;
    sh.MB = sa.n > 128 ? 2 : 1;
    sh.npad = ((sa.n + kTpMC - 1) / kTpMC) * kTpMC;
    sh.cpl = sh.npad / kTpMC;
    const int n8 = (sa.n + 7) & ~7;
    sh.tile_bytes = (uint32_t)n8 * kTpRowBytes;
    const size_t stage = 2 * (size_t)sh.tile_bytes;
    const size_t NR = 2 * (size_t)sh.RR, Kp = 2 * (size_t)sh.npad;
    const size_t bbytes = 2 * NR * Kp * 2;   // B hi and lo, FP16
    const size_t vbytes = sizeof(float2) * (size_t)sh.RR * (sh.npad + 2) + sizeof(float) * 4 * sh.RR;
    const size_t fixed = bbytes + vbytes + sizeof(uint64_t) * (2 + kTpMmaWarps) + 16;
    // a row block read through the last stage's lo tile runs past the ring
    // by (128 MB - n8) rows: that much must be allocated after it
    const size_t tail = std::max(fixed, (size_t)(128 * sh.MB - n8) * kTpRowBytes);
    const size_t optin = device_info().smem_optin;
    const size_t per_stage = stage + 2 * sizeof(uint64_t);
    if (tail + 2 * per_stage > optin) return false;
    int nst = (int)((optin - tail) / per_stage);
    const int ring_cap = (int)(((size_t)sa.ring_kb * 1024) / stage);
    if (nst > ring_cap) nst = ring_cap;
    if (nst > 8) nst = 8;
    if (nst < 2) return false;
    sh.nstage = nst;
    sh.smem = (size_t)nst * stage + tail + 2 * sizeof(uint64_t) * nst;
    return true;
}

bool sweep_tcp_supported(const SweepArgs &sa) {
    TpShape sh;
    return tp_shape(sa, sh);
}

template <int RR, int MB, bool ADJ> static int sweep_tcp_impl(const SweepArgs &sa, const TpShape &sh, cudaStream_t st) {
    SweepTpK k;
    k.n = sa.n;
    k.ny = sa.ny;
    k.nrhs = sa.R;
    k.npad = sh.npad;
    k.cpl = sh.cpl;
    k.nstage = sh.nstage;
    k.tile_bytes = sh.tile_bytes;
    k.Gp = (const unsigned char *)sa.gpack;
    k.gscale = sa.gscale;
    k.cmy = (const float2 *)sa.cmy;
    k.cpy = (const float2 *)sa.cpy;
    k.planes = (float2 *)sa.planes;
    k.dxy = (const float2 *)sa.dxy;
    k.status = sa.status;
    k.kzslot = sa.kzslot;
    auto kern = sweep_tcp_kernel<RR, MB, ADJ>;
    if (!smem_limit_max(kern, sh.smem)) return HELM3D_ERR_CUDA;
    kern<<<dim3((unsigned)sa.nz), kTpThreads, sh.smem, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

template <bool ADJ> static int sweep_tcp_adj(const SweepArgs &sa, const TpShape &sh, cudaStream_t s) {
    if (sh.MB == 2) return sh.RR == 8 ? sweep_tcp_impl<8, 2, ADJ>(sa, sh, s) : sweep_tcp_impl<16, 2, ADJ>(sa, sh, s);
    return sh.RR == 8 ? sweep_tcp_impl<8, 1, ADJ>(sa, sh, s) : sweep_tcp_impl<16, 1, ADJ>(sa, sh, s);
}

int launch_sweep_tcp(const SweepArgs &sa, cudaStream_t s) {
    TpShape sh;
    if (!tp_shape(sa, sh)) return HELM3D_ERR_ARG;
    return sa.dxy ? sweep_tcp_adj<true>(sa, sh, s) : sweep_tcp_adj<false>(sa, sh, s);
}

}  // namespace h3d
