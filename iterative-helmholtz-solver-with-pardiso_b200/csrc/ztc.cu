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
// One persistent CTA per SM walks its tiles chunk by chunk (KC real K per
// chunk) through a ring of S shared-memory stages, each holding the A chunk
// (hi, lo) and the B chunk (hi, lo), with warp-specialized roles:
//   * warps 0-7 (converters): thread (p, half) loads its position's inputs
//     kZcDepth chunks ahead into registers (the loads stay in flight), splits
//     them into tf32 hi/lo and stores them into the stage (one 16-byte store
//     per pair of j), then arrives on the stage's a_full barrier;
//   * warp 16 (producer): one bulk copy per chunk of B (hi and lo, already in
//     the tensor-core layout in global memory, prepared once per grid; the
//     same for every tile, so it comes from L2);
//   * warp 17 (MMA): 3 x (KC / 8) MMAs per chunk into the tile's TMEM
//     accumulator, committed to the stage's empty barrier (which gates its
//     refill); after the tile's last chunk a commit to the accumulator's
//     full barrier;
//   * warps 8-15 (epilogue): warps w and w + 4 read TMEM lanes 32 (w % 4) +
//     [0, 32) (tcgen05.ld 32x32b), each half the columns, 64 columns per
//     wait; the accumulator is freed as soon as its last load has landed,
//     and the outputs of those positions are stored after that
// Two accumulators (2 N <= 512 TMEM columns, nz <= 128) let the epilogue of
// one tile run under the MMAs of the next; above that one accumulator.
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 rows x
// 16 bytes per core matrix, K-adjacent core matrices LBO = 128 bytes apart,
// 8-row groups SBO = KC/4 * 128 bytes apart.  Every wait is bounded; on
// expiry the kernel sets bit 2 of *status, every role stops issuing work,
// the producer waits (bounded) for its copies in flight and the MMA warp for
// its MMAs, TMEM is freed and the kernel returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace h3d {

constexpr int kZcM = 128;                    // tile positions (MMA M)
constexpr int kZcConvWarps = 8;              // warps 0-7
constexpr int kZcEpiWarps = 8;               // warps 8-15
constexpr int kZcProducerWarp = 16;
constexpr int kZcMmaWarp = 17;
constexpr int kZcThreads = 18 * 32;
constexpr int kZcDepth = 4;                  // input chunks in flight per converter thread
constexpr int kZcMaxStages = 8;
constexpr uint32_t kZcStageBudget = 200u * 1024u;
constexpr uint32_t kZcWaitLimit = 1u << 22;

// -------------------------------------------------------------- the kernel
struct ZtcArgs {
    int nz, nzq;            // nz and nz padded to 8 (output rows)
    int N, K, KC;           // GEMM N = 2 nzq, K = 2 nz padded to KC, chunk
    int nchunks;
    int nstage;             // shared-memory stages
    int nacc;               // TMEM accumulators (1 or 2)
    long plane;             // nx*ny
    PlaneLayout L;
    VecBatch vec;           // forward: input x; inverse: output y
    double scale;
    ScaleBatch sc;
    void *planes;           // complex64 planes
    const float *B;         // [nchunks][2 (hi, lo)][N rows x KC] in canonical layout
    int ntiles, tiles_per_rhs;
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

template <bool FWD> struct ZtcIn;
template <> struct ZtcIn<true> { typedef double2 T; };
template <> struct ZtcIn<false> { typedef float2 T; };

// the 2 JP complex inputs (j = j0 + 2 jp + {0, 1}, jp = half, half + 2, ...)
// of one thread for one chunk; zeros outside the grid
template <bool FWD, int JP>
__device__ __forceinline__ void ztc_load(const ZtcArgs &a, const ZtcSrc &q, int j0, int half,
                                         typename ZtcIn<FWD>::T (&v)[2 * JP]) {
    typedef typename ZtcIn<FWD>::T In;
#pragma unroll
    for (int t = 0; t < JP; t++) {
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int jj = j0 + 2 * (half + 2 * t) + e;
            In x;
            x.x = 0;
            x.y = 0;
            if (q.valid && jj < a.nz) x = __ldg(reinterpret_cast<const In *>(q.base) + (long)jj * q.step);
            v[2 * t + e] = x;
        }
    }
}

// The (tile, chunk) cursor of one CTA's sequence, with the thread's source.
template <bool FWD> struct ZtcCursor {
    int tile, c;
    ZtcSrc src;
    __device__ __forceinline__ void start(const ZtcArgs &a, int p) {
        tile = blockIdx.x;
        c = 0;
        src = ztc_src<FWD>(a, tile, p);
    }
    __device__ __forceinline__ void next(const ZtcArgs &a, int p) {
        if (++c == a.nchunks) {
            c = 0;
            tile += gridDim.x;
            if (tile < a.ntiles) src = ztc_src<FWD>(a, tile, p);
        }
    }
};

template <bool FWD, int KC>
__global__ void __launch_bounds__(kZcThreads, 1) ztc_kernel(ZtcArgs a) {
    constexpr int JP = KC / 8;   // 16-byte A stores (pairs of j) per converter thread per chunk
    typedef typename ZtcIn<FWD>::T In;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int N = a.N, S = a.nstage, nch = a.nchunks;
    const uint32_t abytes = (uint32_t)kZcM * KC * 4u;         // one of hi / lo
    const uint32_t bbytes = 2u * (uint32_t)N * KC * 4u;       // hi + lo
    const uint32_t stage_bytes = 2u * abytes + bbytes;
    uint64_t *a_full = reinterpret_cast<uint64_t *>(smem_raw + (size_t)S * stage_bytes);
    uint64_t *b_full = a_full + kZcMaxStages;
    uint64_t *empty = b_full + kZcMaxStages;
    uint64_t *acc_full = empty + kZcMaxStages;
    uint64_t *acc_empty = acc_full + 2;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(acc_empty + 2);
    volatile int *s_dead = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) tmem_alloc(tslot, 512);
    if (tid == 0) {
        for (int q = 0; q < S; q++) {
            mbar_init(&a_full[q], kZcConvWarps);
            mbar_init(&b_full[q], 1);
            mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < 2; q++) {
            mbar_init(&acc_full[q], 1);
            mbar_init(&acc_empty[q], kZcEpiWarps);
        }
        fence_mbar_init_cluster();
        *s_dead = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int my_tiles = blockIdx.x < a.ntiles ? (a.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long total = (long)my_tiles * nch;
    bool dead = false;
    auto fail = [&]() {
        if (!dead) atomicOr(a.status, 4);
        dead = true;
        *s_dead = 1;
    };
    auto wait = [&](uint64_t *bar, uint32_t parity) {
        if (!dead && !mbar_wait_bounded_cta(smem_u32(bar), parity, kZcWaitLimit)) fail();
    };
    auto stage = [&](int s) { return smem_raw + (size_t)s * stage_bytes; };

    if (warp < kZcConvWarps) {
        // ------------------------------------------------------ converters
        const int p = tid & (kZcM - 1), half = tid >> 7;
        In buf[kZcDepth][2 * JP];
        float bs[kZcDepth];   // the chunk's input scale, in FP32
        ZtcCursor<FWD> lc;   // loads: kZcDepth chunks ahead of the conversions
        lc.start(a, p);
#pragma unroll
        for (int d = 0; d < kZcDepth; d++) {
            if (d < total) {
                ztc_load<FWD, JP>(a, lc.src, lc.c * (KC / 2), half, buf[d]);
                bs[d] = (float)lc.src.s;
                lc.next(a, p);
            }
        }
        RingPos sp;
        for (long g0 = 0; g0 < total && !dead; g0 += kZcDepth) {
#pragma unroll
            for (int d = 0; d < kZcDepth; d++) {
                const long g = g0 + d;
                if (g < total && !dead) {
                    wait(&empty[sp.slot], sp.phase ^ 1u);   // the MMAs that read the stage last are done
                    // warp-uniform from here (the stores end in a __syncwarp)
                    if (__any_sync(0xffffffffu, dead || *s_dead)) dead = true;
                    if (!dead) {
                        unsigned char *Ahi = stage(sp.slot), *Alo = Ahi + abytes;
#pragma unroll
                        for (int t = 0; t < JP; t++) {
                            const In x0 = buf[d][2 * t], x1 = buf[d][2 * t + 1];
                            // in FP32: the input rounded once to FP32 (the
                            // planes' own precision), then hi + lo with lo
                            // left in FP32 (the tensor core reads its tf32
                            // part): 22 significant bits, as the FP64 split
                            const float s = bs[d];
                            float4 hi, lo;
                            tf32_split_fast((float)x0.x * s, hi.x, lo.x);
                            tf32_split_fast((float)x0.y * s, hi.y, lo.y);
                            tf32_split_fast((float)x1.x * s, hi.z, lo.z);
                            tf32_split_fast((float)x1.y * s, hi.w, lo.w);
                            const uint32_t off = canon_off(p, 4 * (half + 2 * t), KC);
                            *reinterpret_cast<float4 *>(Ahi + off) = hi;
                            *reinterpret_cast<float4 *>(Alo + off) = lo;
                        }
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) mbar_arrive_local(&a_full[sp.slot]);
                    }
                    sp.next(S);
                    if (g + kZcDepth < total) {
                        ztc_load<FWD, JP>(a, lc.src, lc.c * (KC / 2), half, buf[d]);
                        bs[d] = (float)lc.src.s;
                        lc.next(a, p);
                    }
                }
            }
        }
    } else if (warp == kZcProducerWarp) {
        // -------------------------------------------------------- producer
        if (lane == 0) {
            RingPos sp;
            int c = 0;
            long issued = 0;
            for (long g = 0; g < total && !dead; g++) {
                wait(&empty[sp.slot], sp.phase ^ 1u);
                if (*s_dead) dead = true;
                if (dead) break;
                unsigned char *Bs = stage(sp.slot) + 2u * abytes;
                mbar_expect_tx(&b_full[sp.slot], bbytes);
                bulk_g2s(Bs, a.B + (size_t)c * (bbytes / 4), bbytes, &b_full[sp.slot]);
                issued++;
                sp.next(S);
                if (++c == nch) c = 0;
            }
            // the copies still in flight land before the CTA exits: the last
            // use of every slot (sp is one past the final use)
            for (int k = 0; k < S && k < issued; k++) {
                int sl = sp.slot - 1 - k;
                uint32_t ph = sp.phase;
                if (sl < 0) {
                    sl += S;
                    ph ^= 1u;
                }
                mbar_wait_bounded_cta(smem_u32(&b_full[sl]), ph, kZcWaitLimit);
            }
        }
    } else if (warp == kZcMmaWarp) {
        // ------------------------------------------------------------- MMA
        if (lane == 0) {
            RingPos sp, ap;
            const uint32_t sbo = (uint32_t)(KC / 4) * 128u;
            bool any = false;
            RingPos last;   // accumulator of the last tile committed
            for (int i = 0; i < my_tiles && !dead; i++) {
                wait(&acc_empty[ap.slot], ap.phase ^ 1u);   // its previous tile's outputs are read
                tc_fence_after();
                const uint32_t tacc = tmem + (uint32_t)(ap.slot * N);
                for (int c = 0; c < nch && !dead; c++) {
                    wait(&a_full[sp.slot], sp.phase);
                    wait(&b_full[sp.slot], sp.phase);
                    if (*s_dead) dead = true;
                    if (dead) break;
                    tc_fence_after();
                    const uint32_t ah = smem_u32(stage(sp.slot)), al = ah + abytes;
                    const uint32_t bh = ah + 2u * abytes, bl = bh + bbytes / 2;
                    for (int part = 0; part * 256 < N; part++) {
                        const int n_part = N - part * 256 < 256 ? N - part * 256 : 256;
                        const uint32_t idesc = umma_idesc_tf32(n_part, kZcM);
                        const uint32_t brow = (uint32_t)(part * 256 / 8) * sbo;   // row offset of this part
                        const uint32_t td = tacc + (uint32_t)(part * 256);
#pragma unroll
                        for (int ks = 0; ks < KC / 8; ks++) {
                            const uint32_t koff = (uint32_t)ks * 256u;   // 2 core matrices of 128 B
                            const uint32_t acc0 = (c > 0 || ks > 0) ? 1u : 0u;
                            umma_tf32(td, umma_desc(al + koff, 128, sbo), umma_desc(bh + brow + koff, 128, sbo),
                                      idesc, acc0);
                            umma_tf32(td, umma_desc(ah + koff, 128, sbo), umma_desc(bl + brow + koff, 128, sbo),
                                      idesc, 1u);
                            umma_tf32(td, umma_desc(ah + koff, 128, sbo), umma_desc(bh + brow + koff, 128, sbo),
                                      idesc, 1u);
                        }
                    }
                    umma_commit(&empty[sp.slot]);
                    sp.next(S);
                }
                if (dead) break;
                umma_commit(&acc_full[ap.slot]);
                any = true;
                last = ap;
                ap.next(a.nacc);
            }
            // every MMA issued has completed before TMEM is freed
            if (any) mbar_wait_bounded_cta(smem_u32(&acc_full[last.slot]), last.phase, kZcWaitLimit);
        }
    } else {
        // -------------------------------------------------------- epilogue
        const int q = warp & 3;   // TMEM lanes 32 q + [0, 32) (a warp reads its own quarter)
        const int eh = (warp - kZcConvWarps) >> 2;   // which half of the 16-column groups
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
        const int G = N / 16, gsplit = (G + 1) / 2;
        const int g_lo = eh == 0 ? 0 : gsplit, g_hi = eh == 0 ? gsplit : G;
        RingPos ap;
        for (int i = 0; i < my_tiles && !dead; i++) {
            const int tile = blockIdx.x + i * gridDim.x;
            wait(&acc_full[ap.slot], ap.phase);
            // warp-uniform from here (tcgen05.ld is warp-collective)
            if (__any_sync(0xffffffffu, dead || *s_dead)) dead = true;
            if (dead) break;
            tc_fence_after();
            const int r = tile / a.tiles_per_rhs;
            const long we = (long)(tile - r * a.tiles_per_rhs) * kZcM + 32 * q + lane;   // TMEM lane = position
            const bool ve = we < a.plane;
            long oidx0 = 0, ostep = 0;
            if (ve) {
                if (FWD) {
                    oidx0 = zc_plane_index(a.L, r, 0, we);
                    ostep = a.L.plane * a.L.R;
                } else {
                    oidx0 = r * a.vec.stride + we;
                    ostep = a.plane;
                }
            }
            const uint32_t tacc = trow + (uint32_t)(ap.slot * N);
            if (g_lo >= g_hi) {
                // no columns for this warp (N = 16): only the release
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_local(&acc_empty[ap.slot]);
            }
            for (int g0 = g_lo; g0 < g_hi; g0 += 4) {
                // up to four 16-column loads in flight, one wait
                const int ng = g_hi - g0 < 4 ? g_hi - g0 : 4;
                float v[2][32];
                tmem_ld16_nowait(tacc + (uint32_t)(g0 * 16), v[0]);
                if (ng > 1) tmem_ld16_nowait(tacc + (uint32_t)((g0 + 1) * 16), v[0] + 16);
                if (ng > 2) tmem_ld16_nowait(tacc + (uint32_t)((g0 + 2) * 16), v[1]);
                if (ng > 3) tmem_ld16_nowait(tacc + (uint32_t)((g0 + 3) * 16), v[1] + 16);
                tmem_wait_ld(v[0]);
                tmem_wait_ld(v[1]);
                if (g0 + 4 >= g_hi) {
                    // the accumulator's last columns of this warp are in registers
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_local(&acc_empty[ap.slot]);
                }
                if (!ve) continue;
#pragma unroll
                for (int t = 0; t < 32; t++) {
                    const int k = g0 * 8 + t;
                    if (k >= a.nz || t >= 8 * ng) break;
                    const float re = v[t >> 4][(2 * t) & 31], im = v[t >> 4][(2 * t + 1) & 31];
                    if (FWD) {
                        reinterpret_cast<float2 *>(a.planes)[oidx0 + (long)k * ostep] = make_float2(re, im);
                    } else if (a.vec.c64) {
                        reinterpret_cast<float2 *>(a.vec.p)[oidx0 + (long)k * ostep] = make_float2(re, im);
                    } else {
                        a.vec.p[oidx0 + (long)k * ostep] = make_double2((double)re, (double)im);
                    }
                }
            }
            ap.next(a.nacc);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// ------------------------------------------------------------------- host
// The GEMM shape of an nz-point transform, or false when it does not fit
// (N above 512 TMEM columns).
static bool ztc_shape(int nz, int &N, int &K, int &KC) {
    const int nzq = (nz + 7) & ~7;
    N = 2 * nzq;
    if (N > 512) return false;
    KC = N <= 256 ? 16 : 8;
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
    a.nacc = 2 * a.N <= 512 ? 2 : 1;
    a.status = status;
    const size_t stage = (size_t)2 * a.N * a.KC * 4 + (size_t)2 * kZcM * a.KC * 4;
    a.nstage = (int)(kZcStageBudget / stage);
    if (a.nstage > kZcMaxStages) a.nstage = kZcMaxStages;
    if (a.nstage < 2) return HELM3D_ERR_ARG;
    // stages, barriers (3 per stage slot, 2 per accumulator), TMEM slot, flag
    const size_t smem = (size_t)a.nstage * stage + (3 * kZcMaxStages + 4) * sizeof(uint64_t) + 16;
    if (smem > device_info().smem_optin) return HELM3D_ERR_ARG;
    auto kern = a.KC == 16 ? ztc_kernel<FWD, 16> : ztc_kernel<FWD, 8>;
    if (!smem_limit_max(kern, smem))
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
