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
// Panels.  A panel's 16 pivot steps touch only the panel's columns, n x 16
// complex values, so both CTAs run all of them, on the whole panel, with the
// same arithmetic and therefore the same pivots: at the start of a panel
// each CTA sends its rows' panel entries into both CTAs' shared memory
// (cluster stores, then one arrive per warp on the peer's barrier, release
// at cluster scope), and thread t of each CTA takes physical rows t and
// t + 128 into registers.  A step is then local to the CTA: the pivot
// candidate of each warp is one 32-bit key (redux.sync.max): the top 24
// bits of |re| + |im| and 255 - row, so that the largest magnitude wins and
// ties go to the lowest row (magnitudes equal to 2^-15 relative count as
// ties); the warps' keys and winning rows go through shared memory slots
// alternating by step parity, one CTA barrier per step.  After the steps
// each CTA keeps X and the panel of its own rows, and the panel's pivot
// rows (their other columns live in their owner's TMEM) are exchanged the
// same way as the panel entries.  Two exchanges between the CTAs per panel.
//
// Frames.  The block is never unscrambled.  Physical row g of M holds
// logical row rho[g], physical column q logical column kap[q].  In-place
// Gauss-Jordan without row exchanges on A[g][q] = S[rho[g]][kap[q]] leaves
// M[g][q] = S^{-1}[kap[sigma[g]]][rho[perm[q]]] with perm[k] the pivot row
// of step k and sigma its inverse (the step of row g), so the next frame is
// rho' = kap o sigma, kap' = rho o perm.  The next Schur complement is
// formed in place in that frame, M <- D[rho'][kap'] - c M (D tridiagonal:
// three entries per row, at the physical columns kapinv of logical columns
// i-1, i, i+1), and G_j^T is written to global memory as
// G^T[kap'[q]][rho'[g]] = M[g][q] (the 8-byte stores of a warp scatter
// within one row of G^T and merge in L2).
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
constexpr int kF2RowThreads = kF2RowWarps * 32;
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
    const int *kzslot;   // >= 0: a skipped mode (nothing to do, in both CTAs), or null
};

struct F2Smem {
    float *Bhi, *Blo;   // [2 kF2MaxN rows][2 kF2B] canonical K-major each
    float2 *Y;          // [kF2B][kF2Yld]: the panel's pivot rows
    float2 *PF;         // [kF2MaxN][kF2PFld]: the panel's entries of every row
    float2 *wrow;       // [2][kF2RowWarps][kF2B]: each warp's candidate row, by step parity
    uint32_t *wkey;     // [2][kF2RowWarps]
    int *rho, *kap;     // [2][kF2Tab] each: the frame, double-buffered by line
    int *kapinv, *perm, *stepof;   // [kF2Tab]; stepof[g]: the step that pivoted row g
    uint64_t *pan_bar, *y_bar, *b_ready, *next_ready, *rest_done, *fin;
    uint32_t *tslot;
};

constexpr size_t kF2BBytes = sizeof(float) * 2 * kF2MaxN * 2 * kF2B;
// row stride of PF: 18 complex (144 bytes) instead of 16, so that a warp's
// row-per-thread accesses (16-byte and 8-byte) fall on distinct banks
constexpr int kF2PFld = kF2B + 2;
// row stride of Y: 226 complex, so that the B build's reads of four pivot
// rows at the same column fall on distinct banks (16-byte aligned rows)
constexpr int kF2Yld = kF2MaxN + 2;
constexpr size_t kF2SmemBytes = 2 * kF2BBytes + sizeof(float2) * (kF2B * kF2Yld + kF2PFld * kF2MaxN) +
                                sizeof(float2) * 2 * kF2RowWarps * kF2B + sizeof(uint32_t) * 2 * kF2RowWarps +
                                sizeof(int) * 7 * kF2Tab + 6 * sizeof(uint64_t) + 16 + 1024 + 16;

__device__ __forceinline__ F2Smem f2_carve(unsigned char *raw) {
    F2Smem s;
    uintptr_t b = (reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023);
    s.Bhi = reinterpret_cast<float *>(b);
    s.Blo = s.Bhi + 2 * kF2MaxN * 2 * kF2B;
    s.Y = reinterpret_cast<float2 *>(s.Blo + 2 * kF2MaxN * 2 * kF2B);
    s.PF = s.Y + kF2B * kF2Yld;
    s.wrow = s.PF + kF2MaxN * kF2PFld;
    s.wkey = reinterpret_cast<uint32_t *>(s.wrow + 2 * kF2RowWarps * kF2B);
    s.rho = reinterpret_cast<int *>(s.wkey + 2 * kF2RowWarps);
    s.kap = s.rho + 2 * kF2Tab;
    s.kapinv = s.kap + 2 * kF2Tab;
    s.perm = s.kapinv + kF2Tab;
    s.stepof = s.perm + kF2Tab;
    uintptr_t m = reinterpret_cast<uintptr_t>(s.stepof + kF2Tab);
    m = (m + 15) & ~uintptr_t(15);
    s.pan_bar = reinterpret_cast<uint64_t *>(m);
    s.y_bar = s.pan_bar + 1;
    s.b_ready = s.pan_bar + 2;
    s.next_ready = s.pan_bar + 3;
    s.rest_done = s.pan_bar + 4;
    s.fin = s.pan_bar + 5;
    s.tslot = reinterpret_cast<uint32_t *>(s.pan_bar + 6);
    return s;
}

__device__ __forceinline__ void f2_row_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kF2RowThreads) : "memory");
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

// pivot key of an entry of row g (0 when the row is not a candidate)
__device__ __forceinline__ uint32_t f2_key(float2 v, bool cand, int g) {
    if (!cand) return 0u;
    const float av = fabsf(v.x) + fabsf(v.y);
    if (!(av == av)) return 0u;
    return (__float_as_uint(av) & 0xFFFFFF00u) | (uint32_t)(255 - g);
}

__global__ void __launch_bounds__(kF2Threads, 1) factor_tc2_kernel(F2K a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    F2Smem sm = f2_carve(smem_raw);
    const int n = a.n, ny = a.ny;
    const uint32_t rank = cluster_ctarank(), peer = rank ^ 1u;
    const int kz = blockIdx.x >> 1;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
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
        sm.stepof[q] = -1;   // not pivoted in this line yet
    }
    if (tid == 0) {
        mbar_init(sm.pan_bar, kF2RowWarps);   // the peer's 4 row warps
        mbar_init(sm.y_bar, kF2RowWarps);
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
    auto wait_cluster = [&](uint64_t *bar, uint32_t parity) {
        if (!dead && !mbar_wait_bounded_cluster(smem_u32(bar), parity, kF2WaitLimit)) {
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
        const int g = gbase + t;                 // this CTA's physical row in lane t
        const bool valid = t < nr;
        const int g1 = t + kF2RowThreads;        // the second row of the panel steps (g0 = t)
        const bool has1 = g1 < n;
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
        const uint32_t panbar_peer = mapa_u32(smem_u32(sm.pan_bar), peer);
        const uint32_t ybar_peer = mapa_u32(smem_u32(sm.y_bar), peer);
        const uint32_t pf_peer = mapa_u32(smem_u32(sm.PF), peer);
        const uint32_t y_peer = mapa_u32(smem_u32(sm.Y), peer);
        const float2 kzv = a.kz2[kz];
        uint32_t ph_pan = 0, ph_y = 0, ph_next = 0, ph_rest = 0;
        int cur = 0;

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
            bool used0 = false, used1 = false;
            for (int p = 0; p < npan; p++) {
                const int k0 = p * kF2B, bl = min(kF2B, n - k0);
                if (p > 0) {
                    wait_cta(sm.next_ready, ph_next);
                    ph_next ^= 1u;
                }
                // ---- this CTA's rows of the panel into both CTAs' PF
                {
                    float f[32];
                    tc_fence_after();
                    tmem_ld32_nowait(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_ld(f);
                    if (valid) {
                        float4 *dst = reinterpret_cast<float4 *>(sm.PF + (size_t)g * kF2PFld);
                        const uint32_t rdst = pf_peer + (uint32_t)(g * kF2PFld * sizeof(float2));
#pragma unroll
                        for (int e = 0; e < kF2B / 2; e++) {
                            const float4 q4 = make_float4(f[4 * e], f[4 * e + 1], f[4 * e + 2], f[4 * e + 3]);
                            dst[e] = q4;
                            st_cluster_v4f32(rdst + 16u * (uint32_t)e, q4);
                        }
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(panbar_peer);
                }
                f2_row_barrier();
                wait_cluster(sm.pan_bar, ph_pan);
                ph_pan ^= 1u;
                float2 P0[kF2B], P1[kF2B];
                {
                    const float4 *s0 = reinterpret_cast<const float4 *>(sm.PF + (size_t)t * kF2PFld);
                    const float4 *s1 = reinterpret_cast<const float4 *>(sm.PF + (size_t)(has1 ? g1 : t) * kF2PFld);
#pragma unroll
                    for (int e = 0; e < kF2B / 2; e++) {
                        const float4 x0 = s0[e], x1 = s1[e];
                        P0[2 * e] = make_float2(x0.x, x0.y);
                        P0[2 * e + 1] = make_float2(x0.z, x0.w);
                        P1[2 * e] = make_float2(x1.x, x1.y);
                        P1[2 * e + 1] = make_float2(x1.z, x1.w);
                    }
                }
                // ---- the panel's pivot steps, in each CTA on the whole panel.
                // The rows rotate by one column per step, so that the column
                // of step kk is always P[0] (no register indexed by kk): after
                // step kk, P[e] holds panel column (kk + 1 + e) mod 16.
                // A pivot row is left unscaled in its step (its multiplier is
                // 0, its new column 1) and scaled by its 1 / pv after the
                // panel: every later step is linear in the row, so this gives
                // the same rows as scaling it in its step. Each step issues
                // the next step's warp reduction right after the update of
                // the next pivot column, before the other columns.
                float2 sc0 = make_float2(1.f, 0.f), sc1 = sc0;
                bool piv0 = false, piv1 = false;
                uint32_t key0 = f2_key(P0[0], !used0, t);
                uint32_t key1 = f2_key(P1[0], has1 && !used1, g1);
                uint32_t key = key0 > key1 ? key0 : key1;
                uint32_t kw = __reduce_max_sync(0xffffffffu, key);
#pragma unroll 1
                for (int kk = 0; kk < bl; kk++) {
                    const int k = k0 + kk, buf = k & 1;
                    if (lane == 0) sm.wkey[buf * kF2RowWarps + warp] = kw;
                    if (kw != 0u && key == kw) {
                        // the winning row in register order: w[0] the pivot, w[1 + e] = prow[e]
                        float4 *w = reinterpret_cast<float4 *>(sm.wrow + (size_t)(buf * kF2RowWarps + warp) * kF2B);
                        if (key0 == kw) {
#pragma unroll
                            for (int e = 0; e < kF2B / 2; e++)
                                w[e] = make_float4(P0[2 * e].x, P0[2 * e].y, P0[2 * e + 1].x, P0[2 * e + 1].y);
                        } else {
#pragma unroll
                            for (int e = 0; e < kF2B / 2; e++)
                                w[e] = make_float4(P1[2 * e].x, P1[2 * e].y, P1[2 * e + 1].x, P1[2 * e + 1].y);
                        }
                    }
                    f2_row_barrier();
                    const uint4 kv = *reinterpret_cast<const uint4 *>(sm.wkey + buf * kF2RowWarps);
                    uint32_t kmax = kv.x;
                    int wsel = 0;
                    if (kv.y > kmax) {
                        kmax = kv.y;
                        wsel = 1;
                    }
                    if (kv.z > kmax) {
                        kmax = kv.z;
                        wsel = 2;
                    }
                    if (kv.w > kmax) {
                        kmax = kv.w;
                        wsel = 3;
                    }
                    const int r = kmax != 0u ? 255 - (int)(kmax & 0xFFu) : -1;
                    // the pivot row, rotated like the rows: prow[e] = column (kk + 1 + e) mod 16
                    const float4 *w = reinterpret_cast<const float4 *>(sm.wrow + (size_t)(buf * kF2RowWarps + wsel) * kF2B);
                    float2 prow[kF2B], pv = make_float2(0.f, 0.f);
#pragma unroll
                    for (int e = 0; e < kF2B / 2; e++) {
                        const float4 q4 = w[e];
                        if (e == 0) pv = make_float2(q4.x, q4.y);
                        else prow[2 * e - 1] = make_float2(q4.x, q4.y);
                        prow[2 * e] = make_float2(q4.z, q4.w);
                    }
                    float2 pinv = make_float2(0.f, 0.f);
                    if (r < 0 || (pv.x == 0.f && pv.y == 0.f)) {
                        // no finite candidate, or an exactly zero pivot: flagged, the block is invalid
                        if (t == 0 && rank == 0) atomicOr(a.status, 1);
                    } else {
                        pinv = pivot_inv(pv);
                    }
                    if (t == 0) sm.perm[k] = r >= 0 ? r : 0;
                    // row -= (c / pv) * pivot row, column k becomes -c / pv
                    const bool ip0 = t == r, ip1 = g1 == r;
                    float2 s0 = cmul(P0[0], pinv), s1 = cmul(P1[0], pinv);
                    if (ip0) {
                        s0 = make_float2(0.f, 0.f);
                        sc0 = pinv;
                        used0 = piv0 = true;
                        sm.stepof[t] = k;
                    }
                    if (ip1) {
                        s1 = make_float2(0.f, 0.f);
                        sc1 = pinv;
                        used1 = piv1 = true;
                        sm.stepof[g1] = k;
                    }
                    P0[0] = cfms(s0, prow[0], P0[1]);
                    P1[0] = cfms(s1, prow[0], P1[1]);
                    key0 = f2_key(P0[0], !used0, t);
                    key1 = f2_key(P1[0], has1 && !used1, g1);
                    key = key0 > key1 ? key0 : key1;
                    kw = __reduce_max_sync(0xffffffffu, key);
#pragma unroll
                    for (int e = 1; e < kF2B - 1; e++) {
                        P0[e] = cfms(s0, prow[e], P0[e + 1]);
                        P1[e] = cfms(s1, prow[e], P1[e + 1]);
                    }
                    P0[kF2B - 1] = ip0 ? make_float2(1.f, 0.f) : make_float2(-s0.x, -s0.y);
                    P1[kF2B - 1] = ip1 ? make_float2(1.f, 0.f) : make_float2(-s1.x, -s1.y);
                }
                // the panel's pivot rows scaled by their 1 / pv
                if (piv0) {
#pragma unroll
                    for (int e = 0; e < kF2B; e++) P0[e] = cmul(P0[e], sc0);
                }
                if (piv1) {
#pragma unroll
                    for (int e = 0; e < kF2B; e++) P1[e] = cmul(P1[e], sc1);
                }
                // ---- the panel after its steps back into PF, in column order
                // (P[e] holds column (bl + e) mod 16)
                {
                    float2 *d0 = sm.PF + (size_t)t * kF2PFld;
                    float2 *d1 = sm.PF + (size_t)(has1 ? g1 : t) * kF2PFld;
#pragma unroll
                    for (int e = 0; e < kF2B; e++) d0[(bl + e) & (kF2B - 1)] = P0[e];
                    if (has1) {
#pragma unroll
                        for (int e = 0; e < kF2B; e++) d1[(bl + e) & (kF2B - 1)] = P1[e];
                    }
                }
                f2_row_barrier();

                // ---- the previous panel's trailing GEMM is done: X and the
                // panel's own columns of this CTA's rows into TMEM
                if (p > 0) {
                    wait_cta(sm.rest_done, ph_rest);
                    ph_rest ^= 1u;
                }
                tc_fence_after();
                const int my_step = valid ? sm.stepof[g] : -1;
                const bool piv = valid && my_step >= k0 && my_step < k0 + bl;
                {
                    float xh[32], xl[32], f[32];
                    const float4 *src = reinterpret_cast<const float4 *>(sm.PF + (size_t)(valid ? g : 0) * kF2PFld);
#pragma unroll
                    for (int e = 0; e < kF2B / 2; e++) {
                        const float4 q4 = src[e];
                        f[4 * e] = q4.x;
                        f[4 * e + 1] = q4.y;
                        f[4 * e + 2] = q4.z;
                        f[4 * e + 3] = q4.w;
                    }
                    if (!valid) {
#pragma unroll
                        for (int e = 0; e < 32; e++) f[e] = 0.f;
                    }
#pragma unroll
                    for (int e = 0; e < kF2B; e++) {
                        float2 x = make_float2(0.f, 0.f);
                        if (e < bl) {
                            x = make_float2(f[2 * e], f[2 * e + 1]);
                            if (piv && my_step == k0 + e) x.x -= 1.f;
                        }
                        tf32_split_fast(x.x, xh[2 * e], xl[2 * e]);
                        tf32_split_fast(x.y, xh[2 * e + 1], xl[2 * e + 1]);
                    }
                    tmem_st32(trow + kXhi, xh);
                    tmem_st32(trow + kXlo, xl);
                    tmem_st32(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_st();
                }
                // every read of this panel's PF is done before this CTA's
                // pivot rows go out (the peer writes the next panel's PF only
                // after it has them)
                f2_row_barrier();
                // ---- the panel's pivot rows of this CTA (their values before
                // the panel's update, outside the panel) into Y of both CTAs
                if (__any_sync(0xffffffffu, piv)) {
                    const int yr = piv ? my_step - k0 : 0;
                    float2 *yrow = sm.Y + (size_t)yr * kF2Yld;
                    const uint32_t yrp = y_peer + (uint32_t)(yr * kF2Yld * sizeof(float2));
                    // two 32-column loads in flight per wait
                    const int nc = ncol / 16;
#pragma unroll 1
                    for (int c = 0; c < nc; c += 2) {
                        float f[2][32];
                        tmem_ld32_nowait(trow + (uint32_t)(32 * c), f[0]);
                        if (c + 1 < nc) tmem_ld32_nowait(trow + (uint32_t)(32 * (c + 1)), f[1]);
                        tmem_wait_ld(f[0]);
                        tmem_wait_ld(f[1]);
                        if (piv) {
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                if (c + h >= nc) break;
#pragma unroll
                                for (int e = 0; e < 8; e++) {
                                    const float4 q4 = make_float4(f[h][4 * e], f[h][4 * e + 1], f[h][4 * e + 2],
                                                                  f[h][4 * e + 3]);
                                    reinterpret_cast<float4 *>(yrow + 16 * (c + h))[e] = q4;
                                    st_cluster_v4f32(yrp + (uint32_t)((16 * (c + h) + 2 * e) * sizeof(float2)), q4);
                                }
                            }
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(ybar_peer);
                f2_row_barrier();
                wait_cluster(sm.y_bar, ph_y);
                ph_y ^= 1u;
                // ---- B = real form of Y (rows 2j + c, K = 2kk + c'), hi and lo:
                // each pair (column j of Y, K quad kq) gives the 16-byte units of
                // rows 2j, (Re y, -Im y), and 2j + 1, (Im y, Re y), adjacent in
                // address order (row & 7, K quad, 8-row group); the TF32 split
                // is odd in its argument, so one split serves both rows
#pragma unroll 2
                for (int v = t; v < ncol * (2 * kF2B / 4); v += kF2RowThreads) {
                    const int jlo = v & 3, kq = (v >> 2) & 7, j = (v >> 5) * 4 + jlo;
                    const int kk0 = 2 * kq;
                    const float2 y0 = kk0 < bl ? sm.Y[(size_t)kk0 * kF2Yld + j] : make_float2(0.f, 0.f);
                    const float2 y1 = kk0 + 1 < bl ? sm.Y[(size_t)(kk0 + 1) * kF2Yld + j] : make_float2(0.f, 0.f);
                    float4 h, l;   // split of (Re y0, Im y0, Re y1, Im y1)
                    tf32_split_fast(y0.x, h.x, l.x);
                    tf32_split_fast(y0.y, h.y, l.y);
                    tf32_split_fast(y1.x, h.z, l.z);
                    tf32_split_fast(y1.y, h.w, l.w);
                    const int u0 = (v >> 5) * 64 + kq * 8 + 2 * jlo;
                    float4 *bh = reinterpret_cast<float4 *>(sm.Bhi) + u0;
                    float4 *bl4 = reinterpret_cast<float4 *>(sm.Blo) + u0;
                    bh[0] = make_float4(h.x, -h.y, h.z, -h.w);
                    bh[1] = make_float4(h.y, h.x, h.w, h.z);
                    bl4[0] = make_float4(l.x, -l.y, l.z, -l.w);
                    bl4[1] = make_float4(l.y, l.x, l.w, l.z);
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
            const int *rho = sm.rho + cur * kF2Tab, *kap = sm.kap + cur * kF2Tab;
            int *rho2 = sm.rho + nxt * kF2Tab, *kap2 = sm.kap + nxt * kF2Tab;
            for (int q = t; q < n; q += kF2RowThreads) {
                int st = sm.stepof[q];
                st = (st >= 0 && st < n) ? st : 0;   // a failed step leaves rows unpivoted (status set)
                rho2[q] = kap[st];
                kap2[q] = rho[sm.perm[q]];
            }
            f2_row_barrier();
            for (int q = t; q < n; q += kF2RowThreads) {
                sm.kapinv[kap2[q]] = q;
                sm.stepof[q] = -1;   // for the next line
            }
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
    k.kzslot = fa.kzslot;
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
