// ztc.cu -- the PML-eigenbasis z-transforms of the complex64 preconditioner
// on the 5th-generation tensor cores (tcgen05, kind::tf32), with FP32-class
// accuracy by three TF32 products (3xTF32: a_hi b_hi + a_hi b_lo + a_lo b_hi).
//
//   forward  planes[k][w] = sum_j M[k][j] (s x[j][w])    (complex128 in, complex64 out)
//   inverse  y[k][w]      = sum_j M[k][j] planes[j][w]   (complex64 in, complex128 out)
//
// As a real GEMM per tile of 128 z-columns w (one right-hand side):
//   D[p][n] = sum_K A[p][K] B[n][K],   p < 128, K = 2j + (re, im), n = 2k + (re, im)
// with A[p][2j] = Re x[j][w_p], A[p][2j+1] = Im x[j][w_p] and B the real form
// of M: B[2k][2j] = Re M, B[2k][2j+1] = -Im M, B[2k+1][2j] = Im M,
// B[2k+1][2j+1] = Re M.  M = 128 rows (tile positions), N = 2 nz (padded to 16,
// split in two MMAs above 256), K = 2 nz padded to the chunk.
//
// Per CTA (persistent over tiles, 256 threads, one CTA per SM):
//   * B streams chunk by chunk (KC real K per chunk, hi and lo halves already
//     in the tensor-core layout in global memory, prepared once per grid) by a
//     1D bulk copy into a two-stage shared-memory ring;
//   * all threads convert the A chunk (FP64 or FP32 input -> tf32 hi/lo) into
//     the other half of the stage, one 16-byte store per (position, pair of j);
//   * thread 0 issues the 3 x (KC / 8) MMAs of the chunk into the TMEM
//     accumulator (128 lanes x N fp32 columns) and commits them to the stage's
//     mbarrier, which gates the refill of that stage two chunks later;
//   * after the last chunk every warp reads its 32 TMEM lanes (tcgen05.ld
//     32x32b) and writes the outputs of its positions.
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 rows x
// 16 bytes per core matrix, K-adjacent core matrices LBO = 128 bytes apart,
// 8-row groups SBO = KC/4 * 128 bytes apart.  Every wait is bounded; on
// expiry the kernel sets bit 2 of *status, stops issuing work, waits (bounded)
// for its own MMAs, frees its TMEM and returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kZcThreads = 256;
constexpr int kZcM = 128;                  // tile positions (MMA M)
constexpr uint32_t kZcWaitLimit = 1u << 22;

// -------------------------------------------------------------- the kernel
struct ZtcArgs {
    int nz, nzq;            // nz and nz padded to 8 (output rows)
    int N, K, KC;           // GEMM N = 2 nzq, K = 2 nz padded to KC, chunk
    int nchunks;
    long plane;             // nx*ny
    PlaneLayout L;
    VecBatch vec;           // forward: input x; inverse: output y
    double scale;
    ScaleBatch sc;
    void *planes;           // complex64 planes
    const float *B;         // [nchunks][2 (hi, lo)][N rows x KC] in canonical layout
    int ntiles, tiles_per_rhs;
    uint32_t tmem_cols;
    int *status;
};

__device__ __forceinline__ long zc_plane_index(const PlaneLayout &L, int r, int k, long w) {
    const long j = w / L.nx, i = w - j * L.nx;
    return (long)k * L.plane * L.R + (j * L.R + r) * L.nx + i;
}

// Where one thread's A values of a tile come from: position w of right-hand
// side r; element j at base + j * step (double2 for the forward transform,
// float2 planes for the inverse), times s.
struct ZtcSrc {
    const void *base;
    long step;
    double s;
    bool valid;
};

template <bool FWD>
__device__ __forceinline__ ZtcSrc ztc_src(const ZtcArgs &a, int tile, int p) {
    ZtcSrc q;
    const int r = tile / a.tiles_per_rhs;
    const long w = (long)(tile - r * a.tiles_per_rhs) * kZcM + p;
    q.valid = w < a.plane;
    if (FWD) {
        q.base = a.vec.p + r * a.vec.stride + (q.valid ? w : 0);
        q.step = a.plane;
        q.s = a.scale * (a.sc.p ? a.sc.p[r * a.sc.stride] : 1.0);
    } else {
        q.base = reinterpret_cast<const float2 *>(a.planes) + (q.valid ? zc_plane_index(a.L, r, 0, w) : 0);
        q.step = a.L.plane * a.L.R;
        q.s = 1.0;
    }
    return q;
}

// the 2 JP complex values (j = j0 + 2 jp + {0, 1}, jp = half, half + 2, ...)
// one thread converts for one chunk, as 4 JP doubles
template <bool FWD, int JP>
__device__ __forceinline__ void ztc_load(const ZtcArgs &a, const ZtcSrc &q, int j0, int half, double (&v)[4 * JP]) {
#pragma unroll
    for (int t = 0; t < JP; t++) {
        const int jp = half + 2 * t;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int jj = j0 + 2 * jp + e;
            double re = 0.0, im = 0.0;
            if (q.valid && jj < a.nz) {
                if (FWD) {
                    const double2 x = __ldg(reinterpret_cast<const double2 *>(q.base) + (long)jj * q.step);
                    re = q.s * x.x;
                    im = q.s * x.y;
                } else {
                    const float2 x = __ldg(reinterpret_cast<const float2 *>(q.base) + (long)jj * q.step);
                    re = x.x;
                    im = x.y;
                }
            }
            v[4 * t + 2 * e] = re;
            v[4 * t + 2 * e + 1] = im;
        }
    }
}

template <bool FWD, int KC>
__global__ void __launch_bounds__(kZcThreads, 1) ztc_kernel(ZtcArgs a) {
    constexpr int JP = KC / 8;   // 16-byte A stores per thread per chunk
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int N = a.N;
    const uint32_t bbytes = 2u * (uint32_t)N * KC * 4u;         // hi + lo
    const uint32_t abytes = (uint32_t)kZcM * KC * 4u;           // one of hi / lo
    const uint32_t stage_bytes = bbytes + 2u * abytes;
    unsigned char *stage0 = smem_raw;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + 2 * stage_bytes);   // b_bar[2], mma_bar[2]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 4);
    volatile int *s_dead = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t *b_bar = bars, *mma_bar = bars + 2;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(a.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int q = 0; q < 4; q++) mbar_init(&bars[q], 1);
        fence_mbar_init_cluster();
        *s_dead = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // `dead` is read from shared memory right after a barrier, so every
    // thread takes the same branches; a thread whose bounded wait expires
    // sets it (and bit 2 of *status) for the next barrier to publish.
    auto fail = [&]() {
        *s_dead = 1;
        atomicOr(a.status, 4);
    };
    const int p = tid & (kZcM - 1), half = tid >> 7;
    const int nch = a.nchunks;
    const int my_tiles = blockIdx.x < a.ntiles ? (a.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long total = (long)my_tiles * nch;
    int dead = 0;
    long last_commit = -1;   // chunk of thread 0's last commit
    // the (tile, chunk) sequence of this CTA; the inputs of chunk g + 1 are
    // loaded into the other register buffer while chunk g is converted and
    // multiplied (two buffers, no copy, so the loads stay in flight)
    double bufA[4 * JP], bufB[4 * JP];
    ZtcSrc src_nxt = ztc_src<FWD>(a, blockIdx.x, p);
    if (total > 0) ztc_load<FWD, JP>(a, src_nxt, 0, half, bufA);
    // one chunk; returns false to leave the loop (dead)
    auto chunk = [&](long g, double (&cur)[4 * JP], double (&nxt)[4 * JP]) -> bool {
        const int tile = blockIdx.x + (int)(g / nch) * gridDim.x;
        const int c = (int)(g % nch);
        if (g + 1 < total) {
            const int c1 = (int)((g + 1) % nch);
            if (c1 == 0) src_nxt = ztc_src<FWD>(a, tile + gridDim.x, p);
            ztc_load<FWD, JP>(a, src_nxt, c1 * (KC / 2), half, nxt);
        }
        const int st = (int)(g & 1);
        unsigned char *sbase = stage0 + st * stage_bytes;
        float *Bs = reinterpret_cast<float *>(sbase);
        unsigned char *Ahi = sbase + bbytes, *Alo = Ahi + abytes;
        // the MMAs that read this stage two chunks ago must be complete
        if (g >= 2 && !dead &&
            !mbar_wait_bounded_cta(smem_u32(&mma_bar[st]), (uint32_t)(((g - 2) >> 1) & 1), kZcWaitLimit))
            fail();
        if (tid == 0 && !dead && !*s_dead) {
            mbar_expect_tx(&b_bar[st], bbytes);
            bulk_g2s(Bs, a.B + (size_t)c * (bbytes / 4), bbytes, &b_bar[st]);
        }
#pragma unroll
        for (int t = 0; t < JP; t++) {
            const int jp = half + 2 * t;
            float4 hi, lo;
            tf32_split(cur[4 * t + 0], hi.x, lo.x);
            tf32_split(cur[4 * t + 1], hi.y, lo.y);
            tf32_split(cur[4 * t + 2], hi.z, lo.z);
            tf32_split(cur[4 * t + 3], hi.w, lo.w);
            const uint32_t off = canon_off(p, 4 * jp, KC);
            *reinterpret_cast<float4 *>(Ahi + off) = hi;
            *reinterpret_cast<float4 *>(Alo + off) = lo;
        }
        fence_proxy_async_smem();
        __syncthreads();
        dead = *s_dead;
        if (tid == 0 && !dead) {
            if (!mbar_wait_bounded_cta(smem_u32(&b_bar[st]), (uint32_t)((g >> 1) & 1), kZcWaitLimit)) {
                fail();
            } else {
                tc_fence_after();
                const uint32_t sbo = (uint32_t)(KC / 4) * 128u;
                const uint32_t bs = smem_u32(Bs), ah = smem_u32(Ahi), al = smem_u32(Alo);
                const uint32_t blo = bs + bbytes / 2;
                for (int part = 0; part * 256 < N; part++) {
                    const int n_part = N - part * 256 < 256 ? N - part * 256 : 256;
                    const uint32_t idesc = umma_idesc_tf32(n_part, kZcM);
                    const uint32_t brow = (uint32_t)(part * 256 / 8) * sbo;   // row offset of this part
                    const uint32_t td = tmem + (uint32_t)(part * 256);
#pragma unroll
                    for (int ks = 0; ks < KC / 8; ks++) {
                        const uint32_t koff = (uint32_t)ks * 256u;           // 2 core matrices of 128 B
                        const uint32_t acc0 = (c > 0 || ks > 0) ? 1u : 0u;
                        umma_tf32(td, umma_desc(al + koff, 128, sbo), umma_desc(bs + brow + koff, 128, sbo), idesc,
                                  acc0);
                        umma_tf32(td, umma_desc(ah + koff, 128, sbo), umma_desc(blo + brow + koff, 128, sbo), idesc,
                                  1u);
                        umma_tf32(td, umma_desc(ah + koff, 128, sbo), umma_desc(bs + brow + koff, 128, sbo), idesc,
                                  1u);
                    }
                }
                umma_commit(&mma_bar[st]);
                last_commit = g;
            }
        }
        if (c != nch - 1) return true;

        // epilogue of the tile: wait for its last MMAs, read 32 lanes per warp
        if (!dead && !mbar_wait_bounded_cta(smem_u32(&mma_bar[st]), (uint32_t)((g >> 1) & 1), kZcWaitLimit))
            fail();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        dead = *s_dead;
        if (dead) return false;
        const int r = tile / a.tiles_per_rhs;
        const int q = warp & 3, colhalf = warp >> 2;
        const long we = (long)(tile - r * a.tiles_per_rhs) * kZcM + 32 * q + lane;   // TMEM lane = position
        const bool ve = we < a.plane;
        long oidx0 = 0, ostep = 0;
        if (ve) {
            if (FWD) {
                oidx0 = zc_plane_index(a.L, r, 0, we);
                ostep = a.L.plane * a.L.R;
            } else {
                oidx0 = we;
                ostep = a.plane;
            }
        }
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
        for (int cc = 2 * colhalf; cc < N / 16; cc += 4) {
            // two 16-column loads in flight, one wait
            float v[32];
            tmem_ld16_nowait(trow + (uint32_t)(cc * 16), v);
            const bool two = cc + 1 < N / 16;
            if (two) tmem_ld16_nowait(trow + (uint32_t)((cc + 1) * 16), v + 16);
            tmem_wait_ld(v);
            if (!ve) continue;
#pragma unroll
            for (int t = 0; t < 16; t++) {
                const int k = cc * 8 + t;
                if (k >= a.nz || (t >= 8 && !two)) break;
                if (FWD) {
                    reinterpret_cast<float2 *>(a.planes)[oidx0 + (long)k * ostep] = make_float2(v[2 * t], v[2 * t + 1]);
                } else {
                    double2 *yo = a.vec.p + r * a.vec.stride;
                    yo[oidx0 + (long)k * ostep] = make_double2((double)v[2 * t], (double)v[2 * t + 1]);
                }
            }
        }
        // the next tile's first MMA overwrites the accumulator
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        return true;
    };
    for (long g = 0; g < total; g += 2) {
        if (!chunk(g, bufA, bufB)) break;
        if (g + 1 < total && !chunk(g + 1, bufB, bufA)) break;
    }
    // free the accumulator once every MMA this CTA issued has completed
    if (tid == 0 && last_commit >= 0)
        mbar_wait_bounded_cta(smem_u32(&mma_bar[last_commit & 1]), (uint32_t)((last_commit >> 1) & 1),
                              kZcWaitLimit);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols)
                     : "memory");
}

// ------------------------------------------------------------------- host
// The GEMM shape of an nz-point transform, or false when it does not fit
// (N above 512 TMEM columns).
static bool ztc_shape(int nz, int &N, int &K, int &KC) {
    const int nzq = (nz + 7) & ~7;
    N = 2 * nzq;
    if (N > 512) return false;
    KC = N <= 256 ? 32 : 16;
    K = ((2 * nz + KC - 1) / KC) * KC;
    return true;
}

bool ztc_supported(int nz) {
    int N, K, KC;
    return ztc_shape(nz, N, K, KC);
}

size_t ztc_prepared_floats(int nz) {
    int N, K, KC;
    if (!ztc_shape(nz, N, K, KC)) return 0;
    return (size_t)2 * N * K;
}

// B in the canonical chunked layout, hi then lo per chunk, for the nz x nz
// row-major complex matrix M.
void ztc_prepare(const std::vector<zc> &M, int nz, std::vector<float> &out) {
    int N, K, KC;
    if (!ztc_shape(nz, N, K, KC)) {
        out.clear();
        return;
    }
    out.assign((size_t)2 * N * K, 0.0f);
    for (int n = 0; n < N; n++) {
        const int k = n >> 1, cn = n & 1;
        for (int kk = 0; kk < K; kk++) {
            const int j = kk >> 1, cj = kk & 1;
            double v = 0.0;
            if (k < nz && j < nz) {
                const zc m = M[(size_t)k * nz + j];
                // [Re -Im; Im Re]
                v = cn == 0 ? (cj == 0 ? m.real() : -m.imag()) : (cj == 0 ? m.imag() : m.real());
            }
            float hi, lo;
            tf32_split(v, hi, lo);
            const int c = kk / KC, kc = kk - c * KC;
            const size_t base = (size_t)c * 2 * N * KC;
            const size_t off = canon_off(n, kc, KC) / 4;
            out[base + off] = hi;
            out[base + (size_t)N * KC + off] = lo;
        }
    }
}

template <bool FWD>
static int ztc_launch(const PlaneLayout &L, const VecBatch &vec, double scale, const ScaleBatch &sc, void *planes,
                      const float *B, int *status, cudaStream_t s) {
    ZtcArgs a;
    if (!ztc_shape(L.nz, a.N, a.K, a.KC)) return HELM3D_ERR_ARG;
    a.nz = L.nz;
    a.nzq = a.N / 2;
    a.nchunks = a.K / a.KC;
    a.plane = L.plane;
    a.L = L;
    a.vec = vec;
    a.scale = scale;
    a.sc = sc;
    a.planes = planes;
    a.B = B;
    a.tiles_per_rhs = (int)((L.plane + kZcM - 1) / kZcM);
    a.ntiles = a.tiles_per_rhs * L.R;
    a.tmem_cols = a.N <= 256 ? 256u : 512u;
    a.status = status;
    const size_t stage = (size_t)2 * a.N * a.KC * 4 + (size_t)2 * kZcM * a.KC * 4;
    const size_t smem = 2 * stage + 4 * sizeof(uint64_t) + 16;   // stages, barriers, TMEM slot, flag
    if (smem > device_info().smem_optin) return HELM3D_ERR_ARG;
    auto kern = a.KC == 32 ? ztc_kernel<FWD, 32> : ztc_kernel<FWD, 16>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return HELM3D_ERR_CUDA;
    const int grid = a.ntiles < device_info().sm_count ? a.ntiles : device_info().sm_count;
    kern<<<grid, kZcThreads, smem, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

int launch_ztc_forward(const VecBatch &x, double scale, const ScaleBatch &sc, void *planes, const PlaneLayout &L,
                       const float *B, int *status, cudaStream_t s) {
    return ztc_launch<true>(L, x, scale, sc, planes, B, status, s);
}

int launch_ztc_inverse(const void *planes, const PlaneLayout &L, const VecBatch &y, const float *B, int *status,
                       cudaStream_t s) {
    return ztc_launch<false>(L, y, 1.0, ScaleBatch{nullptr, 0}, (void *)planes, B, status, s);
}

}  // namespace h3d
