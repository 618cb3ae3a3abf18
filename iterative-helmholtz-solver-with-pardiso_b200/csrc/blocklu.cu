// blocklu.cu -- batched block-tridiagonal factorization of the per-kz 2D
// systems (replaces PARDISO phase 11/22, Source/FGMRES.cpp:274-284, and the
// HODLR recurrence DirFactFastDiagStructOnline,
// Source/HODLR/BinaryTreesHODLR.cpp:2870-2969, without compression).
//
// For fixed kz the 5-point PML matrix is block tridiagonal over y-lines:
//   cmy[j] u_{j-1} + D_j u_j + cpy[j] u_{j+1} = f_j,
// D_j tridiagonal (x couplings cmx/cpx, diagonal -(cmx+cpx) - (cmy+cpy)
// + omega^2 s0^2 (1 + i beta) - kz^2).  The y couplings are scalars per line
// (alpha_y depends on j only), so the Schur recurrence is
//   S_0 = D_0,   S_j = D_j - cmy[j] cpy[j-1] G_{j-1},   G_j = S_j^{-1}.
// Each G_j is formed by Gauss-Jordan elimination with partial pivoting
// (rows chosen among the not yet pivoted ones by max |re| + |im|) and
// stored transposed (G_j^T row-major) for the sweep.
//
// Execution: one thread-block cluster of C CTAs per kz, all ny lines in
// sequence.  The NP x NP block (n padded with an identity) lives in
// registers: lane l of every warp owns rows l, l+32, ...; CTA q, warp w owns
// columns q*NPC + w*CB + [0, CB).  At pivot step k the warp owning column k
// picks the pivot row by a warp argmax and writes the column, the pivot row
// index and value into a 4-slot ring in the shared memory of every CTA of
// the cluster, then arrives on each CTA's `full` mbarrier.  Every warp waits
// on its CTA's `full` barrier, fetches the pivot-row entries of its columns
// by warp shuffles (the row lives in the same lane of every warp), updates
// its registers and releases the slot on the `empty` barrier of every CTA
// (the producer of the step that reuses the slot may sit in any of them).
// No CTA-wide barrier runs inside the elimination.  All waits are bounded; on expiry bit 1 of *status is set and
// the kernel runs on without waiting (results are then invalid).
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "helm3d_internal.h"
#include "ptx.cuh"

namespace h3d {

constexpr int kRing = 4;
constexpr uint32_t kWaitLimit = 1u << 20;

// Optional self-checks (compile with -DHELM3D_CHECKS): an index out of range
// sets bit 3 of *status and the access is skipped.
#ifdef HELM3D_CHECKS
#define H3D_OK_IDX(cond) ((cond) ? true : (atomicOr(a.status, 8), false))
#else
#define H3D_OK_IDX(cond) true
#endif

template <typename R> struct FactorK {
    int n, ny, nz, ldg;
    cplx<R> *Gt;
    const cplx<R> *cmx, *cpx, *cmy, *cpy, *base2d;
    const cplx<R> *kz2;  // complex shift of mode kz
    int *status;
    const int *kzslot;   // >= 0: a skipped mode (nothing to do), or null
};

template <typename R> __device__ __forceinline__ R cabs1(cplx<R> a) { return fabs(a.x) + fabs(a.y); }

// bounded wait on a local mbarrier; cluster-scope acquire only when other
// CTAs of the cluster arrive on it
template <int C> __device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    if constexpr (C == 1) return mbar_wait_bounded_cta(addr, parity, kWaitLimit);
    else return mbar_wait_bounded_cluster(addr, parity, kWaitLimit);
}

// Predicated selects in inline PTX.  Written as plain `if (a == q) x = S[q]`
// chains, the compiler folds the unrolled selects back into one dynamically
// indexed load, which moves the whole register tile to local memory.
__device__ __forceinline__ float2 csel(bool p, float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %4, 0;\n\tselp.f32 %0, %2, %5, q;\n\tselp.f32 %1, %3, %6, q;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "r"((unsigned)p), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ double2 csel(bool p, double2 a, double2 b) {
    double2 r;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %4, 0;\n\tselp.f64 %0, %2, %5, q;\n\tselp.f64 %1, %3, %6, q;\n\t}"
        : "=d"(r.x), "=d"(r.y)
        : "d"(a.x), "d"(a.y), "r"((unsigned)p), "d"(b.x), "d"(b.y));
    return r;
}

template <int CB, typename Cx> __device__ __forceinline__ Cx sel_col(const Cx (&row)[CB], int b) {
    Cx x = row[0];
#pragma unroll
    for (int q = 1; q < CB; q++) x = csel(b == q, row[q], x);
    return x;
}

template <int RB, int CB, typename Cx> __device__ __forceinline__ Cx sel_row(const Cx (&S)[RB][CB], int a, int b) {
    Cx x = S[0][b];
#pragma unroll
    for (int q = 1; q < RB; q++) x = csel(a == q, S[q][b], x);
    return x;
}

template <typename R> struct Smem {
    cplx<R> *sGT, *ringcol, *ringpv, *pinvs;
    int *ringr, *perm, *rinv;
    uint64_t *full, *empty;
};

template <typename R, int NP, int NPC>
__device__ __forceinline__ Smem<R> carve(unsigned char *raw) {
    Smem<R> s;
    s.sGT = reinterpret_cast<cplx<R> *>(raw);
    s.ringcol = s.sGT + NPC * NP;
    s.ringpv = s.ringcol + kRing * NP;
    s.pinvs = s.ringpv + kRing;
    s.ringr = reinterpret_cast<int *>(s.pinvs + NP);
    s.perm = s.ringr + kRing;
    s.rinv = s.perm + NP;
    uintptr_t b = reinterpret_cast<uintptr_t>(s.rinv + NP);
    b = (b + 15) & ~uintptr_t(15);
    s.full = reinterpret_cast<uint64_t *>(b);
    s.empty = s.full + kRing;
    return s;
}

template <typename R, int NP, int NPC> constexpr size_t factor_smem_bytes() {
    return sizeof(cplx<R>) * ((size_t)NPC * NP + (size_t)kRing * NP + kRing + NP) + sizeof(int) * (kRing + 2 * NP) +
           16 + sizeof(uint64_t) * 2 * kRing;
}

// MB: CTAs per SM the register budget is planned for (2 lets two kz chains
// share an SM and hide each other's pivot-step latency)
template <typename R, int NP, int NW, int CB, int C, int MB>
__global__ void __launch_bounds__(NW * 32, MB) factor_kernel(FactorK<R> a) {
    constexpr int RB = NP / 32;
    constexpr int NPC = NP / C;
    static_assert(NW * CB == NPC, "columns per CTA must equal warps x columns per warp");
    static_assert(NP % 32 == 0, "padded size must be a multiple of 32");
    typedef cplx<R> Cx;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<R> sm = carve<R, NP, NPC>(smem_raw);

    const uint32_t rank = (C > 1) ? cluster_ctarank() : 0u;
    const int kz = blockIdx.x / C;
    if (a.kzslot && a.kzslot[kz] >= 0) return;   // a skipped mode (kz_skip_ratio): not factored / swept
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n, ny = a.ny;
    const int col0 = (int)rank * NPC + warp * CB;
    bool dead = false;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; s++) {
            mbar_init(&sm.full[s], 32);
            mbar_init(&sm.empty[s], NW * C);
        }
        fence_mbar_init_cluster();
    }
    if (C > 1) cluster_sync_all();
    else __syncthreads();

    const Cx kzv = a.kz2[kz];
    Cx S[RB][CB];
    long t = 0;  // global pivot step counter (line * n + k)

    for (int line = 0; line < ny; line++) {
        // ---- S_line = D_line - cmy[line] cpy[line-1] G_{line-1}
        {
            const Cx cyd = mkc<R>(-(a.cmy[line].x + a.cpy[line].x), -(a.cmy[line].y + a.cpy[line].y));
            const Cx cc = line > 0 ? cmul(a.cmy[line], a.cpy[line - 1]) : mkc<R>(0, 0);
#pragma unroll
            for (int ra = 0; ra < RB; ra++) {
                const int i = lane + 32 * ra;
#pragma unroll
                for (int b = 0; b < CB; b++) {
                    const int j = col0 + b;
                    Cx v = mkc<R>(0, 0);
                    if (i >= n || j >= n) {
                        if (i == j) v = mkc<R>(1, 0);
                    } else {
                        if (line > 0) {
                            Cx gij = sm.sGT[(warp * CB + b) * NP + i];
                            v = mkc<R>(-(cc.x * gij.x - cc.y * gij.y), -(cc.x * gij.y + cc.y * gij.x));
                        }
                        if (i == j) {
                            Cx d = cadd(cadd(cyd, a.base2d[(long)line * n + i]), kzv);
                            d.x -= a.cmx[i].x + a.cpx[i].x;
                            d.y -= a.cmx[i].y + a.cpx[i].y;
                            v = cadd(v, d);
                        } else if (j == i + 1) {
                            v = cadd(v, a.cpx[i]);
                        } else if (j == i - 1) {
                            v = cadd(v, a.cmx[i]);
                        }
                    }
                    S[ra][b] = v;
                }
            }
        }

        // ---- Gauss-Jordan with partial pivoting, pivot search one step ahead:
        // the warp owning column k+1 updates that column first, searches and
        // publishes pivot k+1, then updates its other columns.
        uint32_t used = 0;
        const long t0 = t;
        auto publish = [&](int k) {
            // owner warp of column k: pick the pivot among unused rows and
            // write column k, the row index and the value into ring slot s
            const long tk = t0 + k;
            const int s = (int)(tk % kRing);
            const uint32_t ph = (uint32_t)((tk / kRing) & 1);
            const int ob = (k % NPC) % CB;
            if (!dead && !mbar_wait<C>(smem_u32(&sm.empty[s]), ph ^ 1u)) {
                dead = true;
                atomicOr(a.status, 2);
            }
            R best = (R)-1;
            int bi = NP;
#pragma unroll
            for (int ra = 0; ra < RB; ra++) {
                const int i = lane + 32 * ra;
                const R v = cabs1<R>(sel_col<CB>(S[ra], ob));
                if (i < n && !((used >> ra) & 1u) && v > best) {
                    best = v;
                    bi = i;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const R ov = __shfl_xor_sync(0xffffffffu, best, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            const int r = bi < n ? bi : k;  // no candidate only if the block is broken
            Cx pvs = mkc<R>(0, 0);
#pragma unroll
            for (int ra = 0; ra < RB; ra++) pvs = csel((r >> 5) == ra, sel_col<CB>(S[ra], ob), pvs);
            const Cx pv = shfl_c(pvs, r & 31);
            if constexpr (C == 1) {
#pragma unroll
                for (int ra = 0; ra < RB; ra++) sm.ringcol[s * NP + lane + 32 * ra] = sel_col<CB>(S[ra], ob);
                if (lane == 0) {
                    sm.ringpv[s] = pv;
                    sm.ringr[s] = r;
                    sm.perm[k] = r;
                }
                mbar_arrive_local(&sm.full[s]);
            } else {
                const uint32_t a_col = smem_u32(&sm.ringcol[s * NP]);
                const uint32_t a_pv = smem_u32(&sm.ringpv[s]);
                const uint32_t a_r = smem_u32(&sm.ringr[s]);
                const uint32_t a_perm = smem_u32(&sm.perm[k]);
                const uint32_t a_full = smem_u32(&sm.full[s]);
#pragma unroll
                for (int q = 0; q < C; q++) {
#pragma unroll
                    for (int ra = 0; ra < RB; ra++)
                        st_cluster_c(mapa_u32(a_col + (lane + 32 * ra) * (uint32_t)sizeof(Cx), q),
                                     sel_col<CB>(S[ra], ob));
                    if (lane == 0) {
                        st_cluster_c(mapa_u32(a_pv, q), pv);
                        st_cluster_u32(mapa_u32(a_r, q), (uint32_t)r);
                        st_cluster_u32(mapa_u32(a_perm, q), (uint32_t)r);
                    }
                }
#pragma unroll
                for (int q = 0; q < C; q++) mbar_arrive_cluster(mapa_u32(a_full, q));
            }
        };
        auto owns = [&](int k) { return (int)rank == k / NPC && warp == (k % NPC) / CB; };
        if (owns(0)) publish(0);
        for (int k = 0; k < n; k++, t++) {
            const int s = (int)(t % kRing);
            const uint32_t ph = (uint32_t)((t / kRing) & 1);
            if (!dead && !mbar_wait<C>(smem_u32(&sm.full[s]), ph)) {
                dead = true;
                atomicOr(a.status, 2);
            }
            int r = sm.ringr[s];
            if (!H3D_OK_IDX(r >= 0 && r < n)) r = 0;
            const Cx pv = sm.ringpv[s];
            Cx colk[RB];
#pragma unroll
            for (int ra = 0; ra < RB; ra++) colk[ra] = sm.ringcol[s * NP + lane + 32 * ra];
            Cx pinv;
            if (pv.x == (R)0 && pv.y == (R)0) {
                pinv = mkc<R>(0, 0);
                if (lane == 0) atomicOr(a.status, 1);
            } else {
                pinv = cinv(pv);
            }
            if (threadIdx.x == 0) sm.pinvs[k] = pinv;
            const int rl = r & 31, ar = r >> 5;
            Cx prow[CB];
#pragma unroll
            for (int b = 0; b < CB; b++) prow[b] = cmul(shfl_c(sel_row<RB, CB>(S, ar, b), rl), pinv);
            // The pivot row is left unscaled (it holds pv times the
            // normalized row, and 1 in column k) and divided by pv when G is
            // written out, so that every other element takes one complex FMA
            // with the column entry zeroed in the pivot row.
#pragma unroll
            for (int ra = 0; ra < RB; ra++) colk[ra] = csel((lane + 32 * ra) == r, mkc<R>(0, 0), colk[ra]);
            // element update of column slot b for step k
            auto update_col = [&](int b) {
                if ((col0 + b) == k) {
#pragma unroll
                    for (int ra = 0; ra < RB; ra++) {
                        const Cx e = mkc<R>(-(colk[ra].x * pinv.x - colk[ra].y * pinv.y),
                                            -(colk[ra].x * pinv.y + colk[ra].y * pinv.x));
                        S[ra][b] = csel((lane + 32 * ra) == r, mkc<R>(1, 0), e);
                    }
                } else {
#pragma unroll
                    for (int ra = 0; ra < RB; ra++) S[ra][b] = cfms(colk[ra], prow[b], S[ra][b]);
                }
            };
            if (lane == rl) used |= 1u << ar;
            const bool ahead = (k + 1 < n) && owns(k + 1);
            const int obn = ((k + 1) % NPC) % CB;
            if (ahead) {
#pragma unroll
                for (int b = 0; b < CB; b++)
                    if (b == obn) update_col(b);
                publish(k + 1);
            }
#pragma unroll
            for (int b = 0; b < CB; b++)
                if (!ahead || b != obn) update_col(b);
            __syncwarp();
            // Release slot s on the `empty` barrier of every CTA: whichever CTA
            // produces the next step that uses slot s, its barrier has then
            // completed exactly one phase per use of the slot, so the producer
            // can wait on the parity of the global step count.
            if (lane == 0 && (t + kRing) / n < ny) {
                if constexpr (C == 1) {
                    mbar_arrive_local(&sm.empty[s]);
                } else {
                    const uint32_t a_empty = smem_u32(&sm.empty[s]);
#pragma unroll
                    for (int q = 0; q < C; q++) mbar_arrive_cluster(mapa_u32(a_empty, (uint32_t)q));
                }
            }
        }

        // ---- G = A_final with rows/columns unscrambled: G[rinv[i]][perm[j]] = A[i][j]
        if (C > 1) cluster_sync_all();
        else __syncthreads();
        for (int q = threadIdx.x; q < NP; q += NW * 32) {
            const int p = q < n ? sm.perm[q] : q;
            if (H3D_OK_IDX(p >= 0 && p < NP)) sm.rinv[p] = q;
        }
        __syncthreads();
#pragma unroll
        for (int ra = 0; ra < RB; ra++) {
            const int i = lane + 32 * ra;
            const int ri = sm.rinv[i];
            // row i was the pivot of step ri: divide by its pivot
            const Cx sc = (ri >= 0 && ri < n) ? sm.pinvs[ri] : mkc<R>(1, 0);
#pragma unroll
            for (int b = 0; b < CB; b++) {
                const int j = col0 + b;
                const int pj = j < n ? sm.perm[j] : j;
                if (!H3D_OK_IDX(pj >= 0 && pj < NP && ri >= 0 && ri < NP)) continue;
                const Cx g = cmul(S[ra][b], sc);
                if constexpr (C == 1) {
                    sm.sGT[pj * NP + ri] = g;
                } else {
                    const int q = pj / NPC;
                    st_cluster_c(mapa_u32(smem_u32(&sm.sGT[(pj % NPC) * NP + ri]), (uint32_t)q), g);
                }
            }
        }
        if (C > 1) cluster_sync_all();
        else __syncthreads();
        cplx<R> *gout = a.Gt + ((long)kz * ny + line) * (long)n * a.ldg;
        for (int idx = threadIdx.x; idx < NPC * n; idx += NW * 32) {
            const int jl = idx / n, i = idx - jl * n;
            const int jg = (int)rank * NPC + jl;
            if (jg < n) gout[(long)jg * a.ldg + i] = sm.sGT[jl * NP + i];
        }
    }
}

// ------------------------------------------------------------------ launch
template <typename R, int NP, int NW, int CB, int C, int MB>
static int launch_cfg(const FactorArgs &fa, cudaStream_t st) {
    FactorK<R> k;
    k.n = fa.n;
    k.ny = fa.ny;
    k.nz = fa.nz;
    k.ldg = fa.ldg;
    k.Gt = (cplx<R> *)fa.Gt;
    k.cmx = (const cplx<R> *)fa.cmx;
    k.cpx = (const cplx<R> *)fa.cpx;
    k.cmy = (const cplx<R> *)fa.cmy;
    k.cpy = (const cplx<R> *)fa.cpy;
    k.base2d = (const cplx<R> *)fa.base2d;
    k.kz2 = (const cplx<R> *)fa.kz2;
    k.kzslot = fa.kzslot;
    k.status = fa.status;
    constexpr size_t smem = factor_smem_bytes<R, NP, NP / C>();
    auto kern = factor_kernel<R, NP, NW, CB, C, MB>;
    if (!smem_limit_max(kern, smem))
        return HELM3D_ERR_CUDA;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(fa.nz * C), 1, 1);
    cfg.blockDim = dim3(NW * 32, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kern, k) != cudaSuccess) return HELM3D_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? HELM3D_OK : HELM3D_ERR_CUDA;
}

// The launch shapes of the factor (padded block NP, warps NW, columns per
// warp CB, cluster size C, CTAs per SM planned MB), smallest NP first; for a
// block size n the autotuner times every shape of the smallest NP >= n (the
// first is the default).
typedef int (*FactorLaunch)(const FactorArgs &, cudaStream_t);
struct FactorShape {
    int np;
    FactorLaunch fn;
};
static const FactorShape kShapes64[] = {
    {32, launch_cfg<float, 32, 4, 8, 1, 1>},
    {64, launch_cfg<float, 64, 8, 8, 1, 1>},
    {96, launch_cfg<float, 96, 12, 8, 1, 1>},
    {128, launch_cfg<float, 128, 16, 8, 1, 1>},
    {128, launch_cfg<float, 128, 8, 8, 2, 1>},
    {192, launch_cfg<float, 192, 12, 8, 2, 1>},
    {224, launch_cfg<float, 224, 7, 8, 4, 1>},
    {224, launch_cfg<float, 224, 7, 4, 8, 2>},
    {256, launch_cfg<float, 256, 8, 8, 4, 1>},
    {256, launch_cfg<float, 256, 8, 4, 8, 2>},
};
static const FactorShape kShapes128[] = {
    {32, launch_cfg<double, 32, 8, 4, 1, 1>},
    {64, launch_cfg<double, 64, 16, 4, 1, 1>},
    {96, launch_cfg<double, 96, 12, 4, 2, 1>},
    {128, launch_cfg<double, 128, 8, 4, 4, 1>},
    {192, launch_cfg<double, 192, 12, 4, 4, 1>},
    {224, launch_cfg<double, 224, 7, 4, 8, 1>},
    {256, launch_cfg<double, 256, 8, 4, 8, 1>},
};

template <size_t K> static void shapes_for(const FactorShape (&t)[K], int n, int &first, int &count) {
    first = -1;
    count = 0;
    for (size_t q = 0; q < K; q++) {
        if (t[q].np < n) continue;
        if (first < 0) first = (int)q;
        if (t[q].np != t[first].np) break;
        count++;
    }
}

// After the register shapes, complex64 blocks have one more variant: the
// tensor-core factor, one CTA per kz for n <= 128 (factor_tc.cu), a CTA pair
// per kz for 128 < n <= 224 (factor_tc2.cu).
int factor_variants(bool c64, int n) {
    int first, count;
    if (c64) shapes_for(kShapes64, n, first, count);
    else shapes_for(kShapes128, n, first, count);
    return count + ((factor_tc_supported(c64, n) || factor_tc2_supported(c64, n)) ? 1 : 0);
}

bool factor_supported(bool c64, int n) { return n >= 1 && factor_variants(c64, n) > 0; }

int launch_factor(bool c64, const FactorArgs &fa, cudaStream_t s, int variant) {
    int first, count;
    if (c64) shapes_for(kShapes64, fa.n, first, count);
    else shapes_for(kShapes128, fa.n, first, count);
    if (count == 0) return HELM3D_ERR_ARG;
    if (variant == count && factor_tc_supported(c64, fa.n)) return launch_factor_tc(fa, s);
    if (variant == count && factor_tc2_supported(c64, fa.n)) return launch_factor_tc2(fa, s);
    if (variant < 0 || variant >= count) variant = 0;
    return (c64 ? kShapes64 : kShapes128)[first + variant].fn(fa, s);
}

}  // namespace h3d
