// factor_tc.cu -- the block-tridiagonal factor of blocklu.cu for complex64
// blocks of n <= 128 with the block resident in tensor memory and the
// Gauss-Jordan elimination blocked by panels of 16 columns, the trailing
// updates on the 5th-generation tensor cores (tcgen05, kind::tf32, 3xTF32).
// Same recurrence (replacing PARDISO phases 11/22, Source/FGMRES.cpp:274-284,
// and DirFactFastDiagStructOnline, Source/HODLR/BinaryTreesHODLR.cpp:
// 2870-2969): S_0 = D_0, S_j = D_j - cmy[j] cpy[j-1] G_{j-1}, G_j = S_j^{-1},
// by Gauss-Jordan with partial pivoting (the pivot of column k is the row,
// among those not yet pivoted, with the largest |re| + |im|; ties to the
// lowest row), G_j^T written row-major for the sweep.
//
// Blocking.  Step k of in-place Gauss-Jordan changes every column j != k by
// M[:, j] -= c_k p_k[j] with c_k the current column k (its pivot entry minus
// one) and p_k the normalized pivot row, so the 16 steps of a panel act on
// the columns outside it as M_J <- M_J + X M_J[R, :], R the panel's pivot
// rows and X = (the panel's columns after its 16 steps) - E_R (E_R: ones
// at (r_k, k)).  The panel's steps run on CUDA cores with the panel in
// registers (thread i = row i); X M[R, :] is one tcgen05 GEMM per panel
// (M = 128 rows, N = 2 n_pad real columns, K = 32) accumulated into the
// block in TMEM; the panel's own columns, which that product does not
// describe, are then rewritten from registers.
//
// Layout per CTA (one CTA per kz, all ny lines in sequence):
//   TMEM (512 columns x 128 lanes): the block M (lane i = row i, column
//     2j / 2j + 1 = Re / Im M[i][j]) at [0, 256); X hi at [256, 288), X lo at
//     [288, 320) (lane i, column 2kk + re/im);
//   shared memory: G_{j-1} (row-major, padded rows) for the next Schur
//     complement and the write-out; B = real form of M[R, :] (hi and lo,
//     canonical no-swizzle K-major, 2 n_pad rows x 32); the gathered pivot
//     rows; the per-warp pivot keys and rows (double-buffered by step
//     parity, so one barrier per step); the pivot order.
// Warps 0-3: row threads; warp 4, one lane: MMA issuer.  Every wait is
// bounded: on expiry bit 1 of *status is set and the kernel runs on without
// waiting (results invalid), waits (bounded) for its MMAs, frees its TMEM
// and returns.  A zero pivot sets bit 0.
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kFtRowWarps = 4;
constexpr int kFtThreads = (kFtRowWarps + 1) * 32;
constexpr int kFtNP = 128;              // rows = TMEM lanes, padded columns
constexpr int kFtB = 16;                // panel width
constexpr uint32_t kFtCols = 512;
constexpr uint32_t kFtXhi = 256, kFtXlo = 288;
constexpr int kFtGld = kFtNP + 1;       // padded row of G in shared memory (float2)
constexpr int kFtYld = kFtNP + 2;       // padded row of the gathered pivot rows (float2)
constexpr uint32_t kFtWaitLimit = 1u << 22;

struct FactorTcK {
    int n, ny, ldg;
    float2 *Gt;
    const float2 *cmx, *cpx, *cmy, *cpy, *base2d, *kz2;
    int *status;
    const int *kzslot;   // >= 0: a skipped mode (nothing to do), or null
};

struct FtSmem {
    float2 *G;          // [kFtNP][kFtGld]
    float *Bhi, *Blo;   // [2 kFtNP rows][2 kFtB] canonical each
    float2 *Y;          // [kFtB][kFtYld]
    float2 *wrow;       // [2][4][kFtB]
    uint32_t *ckey;     // [2][4]: each warp's pivot key, by step parity
    int *perm;          // [kFtNP]
    uint64_t *b_ready, *mma_done, *fin;
    uint32_t *tslot;
};

constexpr size_t kFtSmemBytes = sizeof(float2) * kFtNP * kFtGld + 2 * sizeof(float) * 2 * kFtNP * 2 * kFtB +
                                sizeof(float2) * kFtB * kFtYld + sizeof(float2) * 2 * 4 * kFtB +
                                sizeof(float) * 8 + sizeof(int) * 8 + sizeof(int) * kFtNP + 3 * sizeof(uint64_t) +
                                16 + 128;

__device__ __forceinline__ FtSmem ft_carve(unsigned char *raw) {
    FtSmem s;
    s.Bhi = reinterpret_cast<float *>(raw);                       // 1024-aligned base
    s.Blo = s.Bhi + 2 * kFtNP * 2 * kFtB;
    s.G = reinterpret_cast<float2 *>(s.Blo + 2 * kFtNP * 2 * kFtB);
    s.Y = s.G + kFtNP * kFtGld;
    s.wrow = s.Y + kFtB * kFtYld;
    s.ckey = reinterpret_cast<uint32_t *>(s.wrow + 2 * 4 * kFtB);
    s.perm = reinterpret_cast<int *>(s.ckey + 8);
    uintptr_t b = reinterpret_cast<uintptr_t>(s.perm + kFtNP);
    b = (b + 15) & ~uintptr_t(15);
    s.b_ready = reinterpret_cast<uint64_t *>(b);
    s.mma_done = s.b_ready + 1;
    s.fin = s.b_ready + 2;
    s.tslot = reinterpret_cast<uint32_t *>(s.b_ready + 3);
    return s;
}

__device__ __forceinline__ void ft_row_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kFtRowWarps * 32) : "memory");
}

__global__ void __launch_bounds__(kFtThreads, 1) factor_tc_kernel(FactorTcK a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FtSmem sm = ft_carve(smem_raw);
    const int n = a.n, ny = a.ny;
    const int kz = blockIdx.x;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npan = (n + kFtB - 1) / kFtB;
    const int ncol = ((n + 7) / 8) * 8;          // complex columns the GEMM covers (N = 2 ncol, a multiple of 16)

    if (warp == 0) tmem_alloc(sm.tslot, kFtCols);
    if (tid == 0) {
        mbar_init(sm.b_ready, kFtRowWarps);
        mbar_init(sm.mma_done, 1);
        mbar_init(sm.fin, 1);
        fence_mbar_init_cluster();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *sm.tslot;
    bool dead = false;
    auto wait = [&](uint64_t *bar, uint32_t parity) {
        if (!dead && !mbar_wait_bounded_cta(smem_u32(bar), parity, kFtWaitLimit)) {
            dead = true;
            atomicOr(a.status, 2);
        }
    };

    if (warp == kFtRowWarps) {
        // ---------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_tf32(2 * ncol);
            const uint32_t sbo = (uint32_t)(2 * kFtB / 4) * 128u;
            const uint32_t bhi = smem_u32(sm.Bhi), blo = smem_u32(sm.Blo);
            uint32_t ph = 0;
            for (int line = 0; line < ny; line++) {
                for (int p = 0; p < npan; p++) {
                    wait(sm.b_ready, ph);
                    tc_fence_after();
#pragma unroll
                    for (int ks = 0; ks < 2 * kFtB / 8; ks++) {
                        const uint32_t koff = (uint32_t)ks * 256u;   // 8 K = two core matrices of 128 B
                        const uint64_t dh = umma_desc(bhi + koff, 128, sbo), dl = umma_desc(blo + koff, 128, sbo);
                        const uint32_t xh = tmem + kFtXhi + (uint32_t)(ks * 8), xl = tmem + kFtXlo + (uint32_t)(ks * 8);
                        umma_tf32_ts(tmem, xh, dh, idesc, 1u);
                        umma_tf32_ts(tmem, xh, dl, idesc, 1u);
                        umma_tf32_ts(tmem, xl, dh, idesc, 1u);
                    }
                    umma_commit(sm.mma_done);
                    ph ^= 1u;
                }
            }
            umma_commit(sm.fin);
            mbar_wait_bounded_cta(smem_u32(sm.fin), 0u, kFtWaitLimit);
        }
    } else {
        // ----------------------------------------------------- row threads
        const int t = tid;                        // row t, TMEM lane t
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
        uint32_t ph = 0;
        const float2 kzv = a.kz2[kz];
        for (int line = 0; line < ny; line++) {
            // ---- S_line = D_line - cmy[line] cpy[line-1] G_{line-1} into TMEM
            {
                const float2 cyd = make_float2(-(a.cmy[line].x + a.cpy[line].x), -(a.cmy[line].y + a.cpy[line].y));
                const float2 cc = line > 0 ? cmul(a.cmy[line], a.cpy[line - 1]) : make_float2(0.f, 0.f);
                float2 diag = make_float2(0.f, 0.f), sub = diag, sup = diag;
                if (t < n) {
                    diag = cadd(cadd(cyd, a.base2d[(long)line * n + t]), kzv);
                    diag.x -= a.cmx[t].x + a.cpx[t].x;
                    diag.y -= a.cmx[t].y + a.cpx[t].y;
                    sub = a.cmx[t];
                    sup = a.cpx[t];
                }
                const float2 *grow = sm.G + (size_t)t * kFtGld;
#pragma unroll 1
                for (int q = 0; q < kFtNP / 16; q++) {
                    float v[32];
#pragma unroll
                    for (int e = 0; e < 16; e++) {
                        const int j = 16 * q + e;
                        float2 s = make_float2(0.f, 0.f);
                        if (t >= n || j >= n) {
                            if (t == j) s = make_float2(1.f, 0.f);
                        } else {
                            if (line > 0) {
                                const float2 g = grow[j];
                                s = make_float2(-(cc.x * g.x - cc.y * g.y), -(cc.x * g.y + cc.y * g.x));
                            }
                            if (j == t) s = cadd(s, diag);
                            else if (j == t + 1) s = cadd(s, sup);
                            else if (j == t - 1) s = cadd(s, sub);
                        }
                        v[2 * e] = s.x;
                        v[2 * e + 1] = s.y;
                    }
                    tmem_st32(trow + (uint32_t)(32 * q), v);
                }
                tmem_wait_st();
            }

            bool used = false;
            int my_step = -1;
            for (int p = 0; p < npan; p++) {
                const int k0 = p * kFtB, bl = min(kFtB, n - k0);
                // ---- the panel's columns into registers
                float2 P[kFtB];
                {
                    float f[32];
                    tc_fence_after();
                    tmem_ld32_nowait(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_ld(f);
#pragma unroll
                    for (int e = 0; e < kFtB; e++) P[e] = make_float2(f[2 * e], f[2 * e + 1]);
                }
                // ---- the panel's steps (CUDA cores), in a rolled loop: the row
                // rotates by one column per step, so that the column of step kk
                // is always P[0]; after step kk, P[e] holds panel column
                // (kk + 1 + e) mod 16.  The pivot of a column is the candidate
                // row with the largest key: the top 24 bits of |re| + |im| and
                // 255 - row (ties, to 2^-15 relative, go to the lowest row),
                // reduced per warp by redux.sync and across the 4 warps through
                // shared memory slots alternating by step parity.  The pivot
                // row keeps its values in its step (multiplier 0, new column 1)
                // and is scaled by its 1 / pv after the panel: every later step
                // is linear in the row.  The next step's warp reduction is
                // issued right after the update of the next pivot column.
                float2 psc = make_float2(1.f, 0.f);
                bool pivp = false;
                uint32_t key = 0;
                {
                    const float av = fabsf(P[0].x) + fabsf(P[0].y);
                    if (!used && t < n && av == av) key = (__float_as_uint(av) & 0xFFFFFF00u) | (uint32_t)(255 - t);
                }
                uint32_t kw = __reduce_max_sync(0xffffffffu, key);
#pragma unroll 1
                for (int kk = 0; kk < bl; kk++) {
                    const int k = k0 + kk, buf = k & 1;
                    if (lane == 0) sm.ckey[buf * 4 + warp] = kw;
                    if (kw != 0u && key == kw) {
                        // the winning row in register order: w[0] the pivot, w[1 + e] = prow[e]
                        float4 *w = reinterpret_cast<float4 *>(sm.wrow + (buf * 4 + warp) * kFtB);
#pragma unroll
                        for (int e = 0; e < kFtB / 2; e++) w[e] = make_float4(P[2 * e].x, P[2 * e].y, P[2 * e + 1].x, P[2 * e + 1].y);
                    }
                    ft_row_barrier();
                    const uint4 kv = *reinterpret_cast<const uint4 *>(sm.ckey + buf * 4);
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
                    const float4 *w = reinterpret_cast<const float4 *>(sm.wrow + (buf * 4 + wsel) * kFtB);
                    float2 prow[kFtB], pv = make_float2(0.f, 0.f);
#pragma unroll
                    for (int e = 0; e < kFtB / 2; e++) {
                        const float4 q4 = w[e];
                        if (e == 0) pv = make_float2(q4.x, q4.y);
                        else prow[2 * e - 1] = make_float2(q4.x, q4.y);
                        prow[2 * e] = make_float2(q4.z, q4.w);
                    }
                    float2 pinv = make_float2(0.f, 0.f);
                    if (r < 0 || (pv.x == 0.f && pv.y == 0.f)) {
                        // no finite candidate, or an exactly zero pivot: flagged, the block is invalid
                        if (t == 0) atomicOr(a.status, 1);
                    } else {
                        pinv = pivot_inv(pv);
                    }
                    // row -= (c / pv) * pivot row, column k becomes -c / pv
                    const bool ip = t == r;
                    float2 sfac = cmul(P[0], pinv);
                    if (ip) {
                        sfac = make_float2(0.f, 0.f);
                        psc = pinv;
                        used = pivp = true;
                        my_step = k;
                        sm.perm[k] = t;
                    }
                    P[0] = cfms(sfac, prow[0], P[1]);
                    key = 0;
                    {
                        const float av = fabsf(P[0].x) + fabsf(P[0].y);
                        if (!used && t < n && av == av) key = (__float_as_uint(av) & 0xFFFFFF00u) | (uint32_t)(255 - t);
                    }
                    kw = __reduce_max_sync(0xffffffffu, key);
#pragma unroll
                    for (int e = 1; e < kFtB - 1; e++) P[e] = cfms(sfac, prow[e], P[e + 1]);
                    P[kFtB - 1] = ip ? make_float2(1.f, 0.f) : make_float2(-sfac.x, -sfac.y);
                }
                // the panel's pivot row scaled by its 1 / pv
                if (pivp) {
#pragma unroll
                    for (int e = 0; e < kFtB; e++) P[e] = cmul(P[e], psc);
                }
                // back to column order (P[e] holds column (bl + e) mod 16;
                // only a partial last panel is not back in order), through
                // this thread's row of G, which holds nothing during the panels
                if (bl < kFtB) {
                    float2 *tmp = sm.G + (size_t)t * kFtGld;
#pragma unroll
                    for (int e = 0; e < kFtB; e++) tmp[(bl + e) & (kFtB - 1)] = P[e];
#pragma unroll
                    for (int e = 0; e < kFtB; e++) P[e] = tmp[e];
                }

                // ---- X = panel - E_R into TMEM (tf32 hi / lo)
                {
                    float xh[32], xl[32];
#pragma unroll
                    for (int e = 0; e < kFtB; e++) {
                        float2 x = make_float2(0.f, 0.f);
                        if (e < bl) {
                            x = P[e];
                            if (my_step == k0 + e) x.x -= 1.f;
                        }
                        tf32_split_fast(x.x, xh[2 * e], xl[2 * e]);
                        tf32_split_fast(x.y, xh[2 * e + 1], xl[2 * e + 1]);
                    }
                    tmem_st32(trow + kFtXhi, xh);
                    tmem_st32(trow + kFtXlo, xl);
                }
                // ---- the pivot rows of this panel (values before its update) into Y
                const bool piv = my_step >= k0 && my_step < k0 + bl;
                if (__any_sync(0xffffffffu, piv)) {
                    float2 *yrow = sm.Y + (size_t)(piv ? my_step - k0 : 0) * kFtYld;
#pragma unroll 1
                    for (int q = 0; q < kFtNP / 16; q++) {
                        float f[32];
                        tmem_ld32_nowait(trow + (uint32_t)(32 * q), f);
                        tmem_wait_ld(f);
                        if (piv) {
#pragma unroll
                            for (int e = 0; e < 16; e++) yrow[16 * q + e] = make_float2(f[2 * e], f[2 * e + 1]);
                        }
                    }
                }
                tmem_wait_st();
                tc_fence_before();
                ft_row_barrier();
                // ---- B = real form of Y (rows 2j + c, K = 2kk + c'), hi and lo,
                // 16-byte units in address order (row & 7, K quad, 8-row group)
#pragma unroll 4
                for (int u = t; u < 2 * ncol * (2 * kFtB / 4); u += kFtRowWarps * 32) {
                    const int rlo = u & 7, kq = (u >> 3) & 7, rg = u >> 6;
                    const int row = rg * 8 + rlo, j = row >> 1;
                    const int kk0 = 2 * kq;
                    const float2 y0 = kk0 < bl ? sm.Y[(size_t)kk0 * kFtYld + j] : make_float2(0.f, 0.f);
                    const float2 y1 = kk0 + 1 < bl ? sm.Y[(size_t)(kk0 + 1) * kFtYld + j] : make_float2(0.f, 0.f);
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
                // ---- M += X B^T done: rewrite the panel's own columns
                wait(sm.mma_done, ph);
                ph ^= 1u;
                tc_fence_after();
                {
                    float f[32];
#pragma unroll
                    for (int e = 0; e < kFtB; e++) {
                        f[2 * e] = P[e].x;
                        f[2 * e + 1] = P[e].y;
                    }
                    tmem_st32(trow + (uint32_t)(2 * k0), f);
                    tmem_wait_st();
                }
            }

            // ---- G = M with rows and columns unscrambled: G[step of row t][perm[j]] = M[t][j]
            ft_row_barrier();
            {
                const int rt = (t < n) ? my_step : t;
                float2 *gdst = sm.G + (size_t)(rt >= 0 ? rt : 0) * kFtGld;
#pragma unroll 1
                for (int q = 0; q < kFtNP / 16; q++) {
                    float f[32];
                    tmem_ld32_nowait(trow + (uint32_t)(32 * q), f);
                    tmem_wait_ld(f);
                    if (t < n && rt >= 0) {
#pragma unroll
                        for (int e = 0; e < 16; e++) {
                            const int j = 16 * q + e;
                            if (j < n) gdst[sm.perm[j]] = make_float2(f[2 * e], f[2 * e + 1]);
                        }
                    }
                }
            }
            tc_fence_before();
            ft_row_barrier();
            // ---- G_line^T to global: row m of G^T = column m of G
            if (t < n) {
                float2 *gout = a.Gt + ((long)kz * ny + line) * (long)n * a.ldg;
                const float2 *grow = sm.G + (size_t)t * kFtGld;
                for (int m = 0; m < n; m++) gout[(long)m * a.ldg + t] = grow[m];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, kFtCols);
}

bool factor_tc_supported(bool c64, int n) { return c64 && n >= 1 && n <= kFtNP; }

int launch_factor_tc(const FactorArgs &fa, cudaStream_t st) {
    if (fa.n < 1 || fa.n > kFtNP) return HELM3D_ERR_ARG;
    if (kFtSmemBytes > device_info().smem_optin) return HELM3D_ERR_ARG;
    FactorTcK k;
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
    if (!smem_limit_max(factor_tc_kernel, kFtSmemBytes))
        return HELM3D_ERR_CUDA;
    factor_tc_kernel<<<dim3((unsigned)fa.nz), kFtThreads, kFtSmemBytes, st>>>(k);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

}  // namespace h3d
