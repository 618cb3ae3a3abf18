// factor_tc2.cu -- the block-tridiagonal factor of blocklu.cu for complex64
// blocks of 128 < n <= 224 on a pair of CTAs per kz (a thread-block cluster
// of 2), the block resident in the two CTAs' tensor memory and the trailing
// updates of the panel-blocked Gauss-Jordan elimination on the tensor cores
// (tcgen05, kind::tf32, 3xTF32).  Same recurrence as blocklu.cu and
// factor_tc.cu (replacing PARDISO phases 11/22, Source/FGMRES.cpp:274-284, and
// DirFactFastDiagStructOnline, Source/HODLR/BinaryTreesHODLR.cpp:2870-2969):
// S_0 = D_0, S_j = D_j - cmy[j] cpy[j-1] G_{j-1}, G_j = S_j^{-1}, by
// Gauss-Jordan with partial pivoting, G_j^T written row-major for the sweep.
//
// Rows.  CTA 0 of the pair holds physical rows [0, n0), CTA 1 rows [n0, n)
// (n0 = ceil(n/2) <= 112), one row per TMEM lane (lane = row - first row);
// every CTA holds all 2 ncol real columns (ncol = n rounded up to the panel
// width 16): TMEM columns [0, 2 ncol) hold M (2j, 2j+1 = Re, Im of column j),
// [2 ncol, 2 ncol + 32) and [2 ncol + 32, 2 ncol + 64) the panel's X = panel
// - E_R as tf32 hi / lo.  Each CTA runs its own tcgen05 GEMMs (M = 128 rows,
// its own lanes) with its own copy of B (the real form of the panel's pivot
// rows) in shared memory.
//
// Pivot steps across the pair.  At step k each warp of both CTAs reduces its
// candidates to one 32-bit key (redux.sync.max): the top 24 bits of
// |re| + |im| of column k and 255 - row, so that the largest magnitude wins
// and ties go to the lowest row (magnitudes equal to 2^-15 relative count as
// ties).  The warp's winning lane writes the key and its row's 16 panel
// entries into the step's slot in the shared memory of both CTAs, and one
// lane arrives on both CTAs' step barrier (8 arrivals per phase: 4 warps
// per CTA); every row thread then picks the largest of the 8 keys.  The
// slots alternate by phase parity: a slot is rewritten two phases later,
// after every warp of both CTAs has arrived once more, so after every reader
// is done with it.  The same barrier carries one more phase per panel, after
// which the panel's pivot rows (written by their owners into both CTAs'
// shared memory) are complete in both CTAs.
//
// Frames.  The block is never unscrambled.  Physical row g of M holds
// logical row rho[g], physical column q logical column kap[q].  In-place
// Gauss-Jordan without row exchanges on A[g][q] = S[rho[g]][kap[q]] leaves
// M[g][q] = S^{-1}[kap[sigma[g]]][rho[perm[q]]] with perm[k] the pivot row
// of step k and sigma its inverse, so the next frame is rho' = kap o sigma,
// kap' = rho o perm.  The next Schur complement is formed in place in that
// frame, M <- D[rho'][kap'] - c M (D tridiagonal: three entries per row, at
// the physical columns kapinv of logical columns i-1, i, i+1), and G_j^T is
// written to global memory as G^T[kap'[q]][rho'[g]] = M[g][q] (the 8-byte
// stores of a warp scatter within one row of G^T and merge in L2).
//
// Look-ahead.  After panel p's pivot rows are in place, the MMA warp first
// updates the next panel's 16 columns (commit: next_ready), then every other
// column outside panels p and p+1 (commit: rest_done).  The row threads run
// panel p+1's pivot steps as soon as next_ready arrives; rest_done is waited
// for only before panel p+1's X and pivot rows are written, so the trailing
// GEMM runs under the next panel's pivot chain.
//
// Every wait is bounded: on expiry bit 1 of *status is set and the kernel
// runs on without waiting (results invalid), waits (bounded) for its MMAs,
// meets its peer at a final cluster barrier (so that no store into a
// CTA's shared memory can land after it exits), frees its TMEM and returns.
// A zero pivot, or a column without a finite candidate, sets bit 0.
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kF2RowWarps = 4;
constexpr int kF2Warps = kF2RowWarps * 2;        // row warps of the pair
constexpr int kF2Threads = (kF2RowWarps + 1) * 32;
constexpr int kF2B = 16;                         // panel width
constexpr int kF2MaxN = 224;                     // 2 ncol + 64 X columns <= 512
constexpr int kF2Tab = 256;
constexpr uint32_t kF2Cols = 512;
constexpr uint32_t kF2WaitLimit = 1u << 22;

struct F2K {
    int n, ny, ldg;
    float2 *Gt;
    const float2 *cmx, *cpx, *cmy, *cpy, *base2d, *kz2;
    int *status;
};

// one warp's candidate of a pivot step: its key and its row's panel entries
struct __align__(16) F2Slot {
    uint32_t key, pad[3];
    float4 v[kF2B / 2];
};

struct F2Smem {
    float *Bhi, *Blo;   // [2 kF2MaxN rows][2 kF2B] canonical K-major each
    float2 *Y;          // [kF2B][kF2MaxN]: the panel's pivot rows
    F2Slot *slot;       // [2][kF2Warps]
    int *rho, *kap;     // [2][kF2Tab] each: the frame, double-buffered by line
    int *kapinv, *perm, *sigma;   // [kF2Tab]
    uint64_t *stepbar, *b_ready, *next_ready, *rest_done, *fin;
    uint32_t *tslot;
};

constexpr size_t kF2BBytes = sizeof(float) * 2 * kF2MaxN * 2 * kF2B;
constexpr size_t kF2SmemBytes = 2 * kF2BBytes + sizeof(float2) * kF2B * kF2MaxN + sizeof(F2Slot) * 2 * kF2Warps +
                                sizeof(int) * 7 * kF2Tab + 5 * sizeof(uint64_t) + 16 + 1024;

__device__ __forceinline__ F2Smem f2_carve(unsigned char *raw) {
    F2Smem s;
    uintptr_t b = (reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023);
    s.Bhi = reinterpret_cast<float *>(b);
    s.Blo = s.Bhi + 2 * kF2MaxN * 2 * kF2B;
    s.Y = reinterpret_cast<float2 *>(s.Blo + 2 * kF2MaxN * 2 * kF2B);
    s.slot = reinterpret_cast<F2Slot *>(s.Y + kF2B * kF2MaxN);
    s.rho = reinterpret_cast<int *>(s.slot + 2 * kF2Warps);
    s.kap = s.rho + 2 * kF2Tab;
    s.kapinv = s.kap + 2 * kF2Tab;
    s.perm = s.kapinv + kF2Tab;
    s.sigma = s.perm + kF2Tab;
    uintptr_t m = reinterpret_cast<uintptr_t>(s.sigma + kF2Tab);
    m = (m + 15) & ~uintptr_t(15);
    s.stepbar = reinterpret_cast<uint64_t *>(m);
    s.b_ready = s.stepbar + 1;
    s.next_ready = s.stepbar + 2;
    s.rest_done = s.stepbar + 3;
    s.fin = s.stepbar + 4;
    s.tslot = reinterpret_cast<uint32_t *>(s.stepbar + 5);
    return s;
}

__device__ __forceinline__ void f2_row_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kF2RowWarps * 32) : "memory");
}

__device__ __forceinline__ void st_cluster_v4f32(uint32_t addr, float4 v) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

// The tridiagonal D_line in logical row i: diagonal, and the couplings to
// logical columns i - 1 (sub) and i + 1 (sup).
struct F2Drow {
    float2 diag, sub, sup;
};
__device__ __forceinline__ F2Drow f2_drow(const F2K &a, int line, int i, float2 kzv) {
    F2Drow d;
    const float2 cyd = make_float2(-(a.cmy[line].x + a.cpy[line].x), -(a.cmy[line].y + a.cpy[line].y));
    d.diag = cadd(cadd(cyd, a.base2d[(long)line * a.n + i]), kzv);
    d.diag.x -= a.cmx[i].x + a.cpx[i].x;
    d.diag.y -= a.cmx[i].y + a.cpx[i].y;
    d.sub = a.cmx[i];
    d.sup = a.cpx[i];
    return d;
}

__global__ void __launch_bounds__(kF2Threads, 1) factor_tc2_kernel(F2K a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    F2Smem sm = f2_carve(smem_raw);
    const int n = a.n, ny = a.ny;
    const uint32_t rank = cluster_ctarank(), peer = rank ^ 1u;
    const int kz = blockIdx.x >> 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n0 = (n + 1) >> 1;
    const int nr = rank == 0 ? n0 : n - n0;       // rows of this CTA
    const int gbase = rank == 0 ? 0 : n0;
    const int ncol = (n + kF2B - 1) / kF2B * kF2B;
    const int npan = ncol / kF2B;
    const uint32_t kXhi = 2u * ncol, kXlo = 2u * ncol + 32u;

    if (warp == 0) tmem_alloc(sm.tslot, kF2Cols);
    for (int q = tid; q < kF2Tab; q += kF2Threads) {
        sm.rho[q] = q;
        sm.kap[q] = q;
        sm.kapinv[q] = q;
        sm.perm[q] = 0;
        sm.sigma[q] = 0;   // every entry stays a valid index, even for a failed step
    }
    if (tid == 0) {
        mbar_init(sm.stepbar, kF2Warps);
        mbar_init(sm.b_ready, kF2RowWarps);
        mbar_init(sm.next_ready, 1);
        mbar_init(sm.rest_done, 1);
        mbar_init(sm.fin, 1);
        fence_mbar_init_cluster();
    }
    tc_fence_before();
    cluster_sync_all();   // both CTAs' barriers exist before any remote arrive
    tc_fence_after();
    const uint32_t tmem = *sm.tslot;
    bool dead = false;
    auto wait_cta = [&](uint64_t *bar, uint32_t parity) {
        if (!dead && !mbar_wait_bounded_cta(smem_u32(bar), parity, kF2WaitLimit)) {
            dead = true;
            atomicOr(a.status, 2);
        }
    };

    if (warp == kF2RowWarps) {
        // ---------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t sbo = (uint32_t)(2 * kF2B / 4) * 128u;
            const uint32_t bhi = smem_u32(sm.Bhi), blo = smem_u32(sm.Blo);
            // D[:, c0 + [0, len)) += X B[c0 + [0, len), :]^T, 3xTF32, in chunks of N <= 256
            auto issue = [&](int c0, int len) {
                for (int off = 0; off < len; off += 256) {
                    const int nn = len - off < 256 ? len - off : 256;
                    const int col = c0 + off;
                    const uint32_t idesc = umma_idesc_tf32(nn);
                    const uint32_t boff = (uint32_t)(col / 8) * sbo;
#pragma unroll
                    for (int ks = 0; ks < 2 * kF2B / 8; ks++) {
                        const uint32_t koff = (uint32_t)ks * 256u;
                        const uint64_t dh = umma_desc(bhi + boff + koff, 128, sbo);
                        const uint64_t dl = umma_desc(blo + boff + koff, 128, sbo);
                        const uint32_t xh = tmem + kXhi + (uint32_t)(ks * 8), xl = tmem + kXlo + (uint32_t)(ks * 8);
                        const uint32_t d = tmem + (uint32_t)col;
                        umma_tf32_ts(d, xh, dh, idesc, 1u);
                        umma_tf32_ts(d, xh, dl, idesc, 1u);
                        umma_tf32_ts(d, xl, dh, idesc, 1u);
                    }
                }
            };
            uint32_t ph = 0;
            for (int line = 0; line < ny; line++) {
                for (int p = 0; p < npan; p++) {
                    wait_cta(sm.b_ready, ph);
                    ph ^= 1u;
                    tc_fence_after();
                    if (p + 1 < npan) {
                        issue(2 * kF2B * (p + 1), 2 * kF2B);
                        umma_commit(sm.next_ready);
                        issue(0, 2 * kF2B * p);
                        issue(2 * kF2B * (p + 2), 2 * ncol - 2 * kF2B * (p + 2));
                    } else {
                        issue(0, 2 * kF2B * p);
                    }
                    umma_commit(sm.rest_done);
                }
            }
            umma_commit(sm.fin);
            mbar_wait_bounded_cta(smem_u32(sm.fin), 0u, kF2WaitLimit);
        }
    } else {
        // ----------------------------------------------------- row threads
        const int t = tid;                       // TMEM lane t
        const int g = gbase + t;                 // physical row
        const bool valid = t < nr;
        const int wg = (int)rank * kF2RowWarps + warp;
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
        const uint32_t bar_loc = mapa_u32(smem_u32(sm.stepbar), rank);
        const uint32_t bar_peer = mapa_u32(smem_u32(sm.stepbar), peer);
        const uint32_t slot_peer = mapa_u32(smem_u32(sm.slot), peer);
        const uint32_t y_peer = mapa_u32(smem_u32(sm.Y), peer);
        const float2 kzv = a.kz2[kz];
        uint32_t xph = 0, ph_next = 0, ph_rest = 0;
        int cur = 0;
        auto xwait = [&]() {
            if (!dead && !mbar_wait_bounded_cluster(smem_u32(sm.stepbar), xph, kF2WaitLimit)) {
                dead = true;
                atomicOr(a.status, 2);
            }
            xph ^= 1u;
        };

        // ---- S_0 = D_0 (identity frame)
        {
            F2Drow d = f2_drow(a, 0, valid ? g : 0, kzv);
#pragma unroll 1
            for (int c = 0; c < ncol / 16; c++) {
                float f[32];
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    const int q = 16 * c + e;
                    float2 s = make_float2(0.f, 0.f);
                    if (valid && q < n) {
                        if (q == g) s = d.diag;
                        else if (q == g - 1) s = d.sub;
                        else if (q == g + 1) s = d.sup;
                    }
                    f[2 * e] = s.x;
                    f[2 * e + 1] = s.y;
                }
                tmem_st32(trow + (uint32_t)(32 * c), f);
            }
            tmem_wait_st();
        }

        for (int line = 0; line < ny; line++) {
            bool used = false;
            int my_step = -1;
            for (int p = 0; p < npan; p++) {
                const int k0 = p * kF2B, bl = min(kF2B, n - k0);
                if (p > 0) {
                    wait_cta(sm.next_ready, ph_next);
                    ph_next ^= 1u;
                }
                // ---- the panel's columns into registers
                float2 P[kF2B];
                {
                    float f[32];
                    tc_fence_after();
                    tmem_ld32_nowait(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_ld(f);
#pragma unroll
                    for (int e = 0; e < kF2B; e++) P[e] = make_float2(f[2 * e], f[2 * e + 1]);
                }
                // ---- the panel's pivot steps across the pair
#pragma unroll
                for (int kk = 0; kk < kF2B; kk++) {
                    if (kk >= bl) break;
                    const int k = k0 + kk, sl = (int)(xph & 1u);
                    const float2 v = P[kk];
                    uint32_t key = 0;
                    if (valid && !used) {
                        const float av = fabsf(v.x) + fabsf(v.y);
                        if (av == av) key = (__float_as_uint(av) & 0xFFFFFF00u) | (uint32_t)(255 - g);
                    }
                    const uint32_t kw = __reduce_max_sync(0xffffffffu, key);
                    const bool win = kw != 0u ? key == kw : lane == 0;
                    if (win) {
                        F2Slot *s = sm.slot + sl * kF2Warps + wg;
                        const uint32_t rs = slot_peer + (uint32_t)((sl * kF2Warps + wg) * sizeof(F2Slot));
                        s->key = kw;
                        st_cluster_u32(rs, kw);
                        if (kw != 0u) {
#pragma unroll
                            for (int e = 0; e < kF2B / 2; e++) {
                                const float4 q4 = make_float4(P[2 * e].x, P[2 * e].y, P[2 * e + 1].x, P[2 * e + 1].y);
                                s->v[e] = q4;
                                st_cluster_v4f32(rs + 16u + 16u * (uint32_t)e, q4);
                            }
                        }
                    }
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive_cluster(bar_loc);
                        mbar_arrive_cluster(bar_peer);
                    }
                    xwait();
                    uint32_t kmax = 0;
                    int wsel = 0;
#pragma unroll
                    for (int w2 = 0; w2 < kF2Warps; w2++) {
                        const uint32_t kk2 = sm.slot[sl * kF2Warps + w2].key;
                        if (kk2 > kmax) {
                            kmax = kk2;
                            wsel = w2;
                        }
                    }
                    const int r = kmax != 0u ? 255 - (int)(kmax & 0xFFu) : -1;
                    float2 prow[kF2B];
                    float2 pinv = make_float2(0.f, 0.f);
                    if (r < 0) {
                        // no finite candidate in the column: flagged, the block is invalid
#pragma unroll
                        for (int e = 0; e < kF2B; e++) prow[e] = make_float2(0.f, 0.f);
                        if (t == 0 && rank == 0) atomicOr(a.status, 1);
                    } else {
                        const F2Slot *s = sm.slot + sl * kF2Warps + wsel;
#pragma unroll
                        for (int e = 0; e < kF2B / 2; e++) {
                            const float4 q4 = s->v[e];
                            prow[2 * e] = make_float2(q4.x, q4.y);
                            prow[2 * e + 1] = make_float2(q4.z, q4.w);
                        }
                        const float2 pv = prow[kk];
                        if (pv.x == 0.f && pv.y == 0.f) {
                            if (t == 0 && rank == 0) atomicOr(a.status, 1);
                        } else {
                            // 1 / pv with two divisions, scaled against overflow of |pv|^2
                            const float sc = 1.f / fmaxf(fabsf(pv.x), fabsf(pv.y));
                            const float ax = pv.x * sc, ay = pv.y * sc;
                            const float rd = sc / (ax * ax + ay * ay);
                            pinv = make_float2(ax * rd, -ay * rd);
                        }
                    }
                    if (t == 0) sm.perm[k] = r >= 0 ? r : 0;
                    if (valid && g == r) {
#pragma unroll
                        for (int e = 0; e < kF2B; e++) P[e] = e == kk ? pinv : cmul(prow[e], pinv);
                        used = true;
                        my_step = k;
                    } else {
                        // row -= (c / pv) * pivot row; column k becomes -c / pv
                        const float2 sfac = cmul(v, pinv);
#pragma unroll
                        for (int e = 0; e < kF2B; e++)
                            P[e] = e == kk ? make_float2(-sfac.x, -sfac.y) : cfms(sfac, prow[e], P[e]);
                    }
                }

                // ---- the previous panel's trailing GEMM is done: X, the
                // panel's own columns and its pivot rows can be written
                if (p > 0) {
                    wait_cta(sm.rest_done, ph_rest);
                    ph_rest ^= 1u;
                }
                tc_fence_after();
                {
                    float xh[32], xl[32], f[32];
#pragma unroll
                    for (int e = 0; e < kF2B; e++) {
                        float2 x = make_float2(0.f, 0.f);
                        if (e < bl) {
                            x = P[e];
                            if (my_step == k0 + e) x.x -= 1.f;
                        }
                        tf32_split_fast(x.x, xh[2 * e], xl[2 * e]);
                        tf32_split_fast(x.y, xh[2 * e + 1], xl[2 * e + 1]);
                        f[2 * e] = P[e].x;
                        f[2 * e + 1] = P[e].y;
                    }
                    tmem_st32(trow + kXhi, xh);
                    tmem_st32(trow + kXlo, xl);
                    tmem_st32(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_st();
                }
                // ---- the panel's pivot rows (their values before its update,
                // outside the panel) into Y of both CTAs
                const bool piv = my_step >= k0 && my_step < k0 + bl;
                if (__any_sync(0xffffffffu, piv)) {
                    const int yr = piv ? my_step - k0 : 0;
                    float2 *yrow = sm.Y + (size_t)yr * kF2MaxN;
                    const uint32_t yrp = y_peer + (uint32_t)(yr * kF2MaxN * sizeof(float2));
#pragma unroll 1
                    for (int c = 0; c < ncol / 16; c++) {
                        float f[32];
                        tmem_ld32_nowait(trow + (uint32_t)(32 * c), f);
                        tmem_wait_ld(f);
                        if (piv) {
#pragma unroll
                            for (int e = 0; e < 8; e++) {
                                const float4 q4 = make_float4(f[4 * e], f[4 * e + 1], f[4 * e + 2], f[4 * e + 3]);
                                reinterpret_cast<float4 *>(yrow + 16 * c)[e] = q4;
                                st_cluster_v4f32(yrp + (uint32_t)((16 * c + 2 * e) * sizeof(float2)), q4);
                            }
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive_cluster(bar_loc);
                    mbar_arrive_cluster(bar_peer);
                }
                xwait();
                // ---- B = real form of Y (rows 2j + c, K = 2kk + c'), hi and lo,
                // 16-byte units in address order (row & 7, K quad, 8-row group)
#pragma unroll 4
                for (int u = t; u < 2 * ncol * (2 * kF2B / 4); u += kF2RowWarps * 32) {
                    const int rlo = u & 7, kq = (u >> 3) & 7, rg = u >> 6;
                    const int row = rg * 8 + rlo, j = row >> 1;
                    const int kk0 = 2 * kq;
                    const float2 y0 = kk0 < bl ? sm.Y[(size_t)kk0 * kF2MaxN + j] : make_float2(0.f, 0.f);
                    const float2 y1 = kk0 + 1 < bl ? sm.Y[(size_t)(kk0 + 1) * kF2MaxN + j] : make_float2(0.f, 0.f);
                    float4 e;
                    if ((row & 1) == 0) e = make_float4(y0.x, -y0.y, y1.x, -y1.y);   // (Re y, -Im y)
                    else e = make_float4(y0.y, y0.x, y1.y, y1.x);                   // (Im y, Re y)
                    float4 h, l;
                    tf32_split_fast(e.x, h.x, l.x);
                    tf32_split_fast(e.y, h.y, l.y);
                    tf32_split_fast(e.z, h.z, l.z);
                    tf32_split_fast(e.w, h.w, l.w);
                    reinterpret_cast<float4 *>(sm.Bhi)[u] = h;
                    reinterpret_cast<float4 *>(sm.Blo)[u] = l;
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive_local(sm.b_ready);
            }

            // ---- the line's last GEMM done: the next frame
            wait_cta(sm.rest_done, ph_rest);
            ph_rest ^= 1u;
            tc_fence_after();
            f2_row_barrier();
            const int nxt = cur ^ 1;
            int *rho = sm.rho + cur * kF2Tab, *kap = sm.kap + cur * kF2Tab;
            int *rho2 = sm.rho + nxt * kF2Tab, *kap2 = sm.kap + nxt * kF2Tab;
            for (int k = t; k < n; k += kF2RowWarps * 32) sm.sigma[sm.perm[k]] = k;
            f2_row_barrier();
            for (int q = t; q < n; q += kF2RowWarps * 32) {
                rho2[q] = kap[sm.sigma[q]];
                kap2[q] = rho[sm.perm[q]];
            }
            f2_row_barrier();
            for (int q = t; q < n; q += kF2RowWarps * 32) sm.kapinv[kap2[q]] = q;
            f2_row_barrier();
            cur = nxt;

            // ---- G_line^T to global in the new frame, and S_{line+1} in place
            {
                const int i = valid ? rho2[g] : 0;
                const bool more = line + 1 < ny;
                float2 cc = make_float2(0.f, 0.f);
                F2Drow d = {};
                int qd = -1, qs = -1, qp = -1;
                if (more) {
                    cc = cmul(a.cmy[line + 1], a.cpy[line]);
                    d = f2_drow(a, line + 1, i, kzv);
                    qd = sm.kapinv[i];
                    qs = i > 0 ? sm.kapinv[i - 1] : -1;
                    qp = i + 1 < n ? sm.kapinv[i + 1] : -1;
                }
                float2 *gout = a.Gt + ((long)kz * ny + line) * (long)n * a.ldg;
#pragma unroll 1
                for (int c = 0; c < ncol / 16; c++) {
                    float f[32];
                    tmem_ld32_nowait(trow + (uint32_t)(32 * c), f);
                    tmem_wait_ld(f);
#pragma unroll
                    for (int e = 0; e < 16; e++) {
                        const int q = 16 * c + e;
                        const float2 m = make_float2(f[2 * e], f[2 * e + 1]);
                        float2 s = make_float2(0.f, 0.f);
                        if (valid && q < n) {
                            gout[(long)kap2[q] * a.ldg + i] = m;
                            s = make_float2(-(cc.x * m.x - cc.y * m.y), -(cc.x * m.y + cc.y * m.x));
                            if (q == qd) s = cadd(s, d.diag);
                            else if (q == qs) s = cadd(s, d.sub);
                            else if (q == qp) s = cadd(s, d.sup);
                        }
                        f[2 * e] = s.x;
                        f[2 * e + 1] = s.y;
                    }
                    if (more) tmem_st32(trow + (uint32_t)(32 * c), f);
                }
                tmem_wait_st();
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();   // the peer is done with this CTA's shared memory
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, kF2Cols);
}

bool factor_tc2_supported(bool c64, int n) { return c64 && n > 128 && n <= kF2MaxN; }

int launch_factor_tc2(const FactorArgs &fa, cudaStream_t st) {
    if (fa.n <= 128 || fa.n > kF2MaxN) return HELM3D_ERR_ARG;
    if (kF2SmemBytes > device_info().smem_optin) return HELM3D_ERR_ARG;
    F2K k;
    k.n = fa.n;
    k.ny = fa.ny;
    k.ldg = fa.ldg;
    k.Gt = (float2 *)fa.Gt;
    k.cmx = (const float2 *)fa.cmx;
    k.cpx = (const float2 *)fa.cpx;
    k.cmy = (const float2 *)fa.cmy;
    k.cpy = (const float2 *)fa.cpy;
    k.base2d = (const float2 *)fa.base2d;
    k.kz2 = (const float2 *)fa.kz2;
    k.status = fa.status;
    if (!smem_limit_max(factor_tc2_kernel, kF2SmemBytes)) return HELM3D_ERR_CUDA;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * fa.nz), 1, 1);
    cfg.blockDim = dim3(kF2Threads, 1, 1);
    cfg.dynamicSmemBytes = kF2SmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, factor_tc2_kernel, k) != cudaSuccess) return HELM3D_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
