// helm3d_internal.h -- context and kernel launchers shared by the host code
// (setup.cpp, solver.cpp, capi.cpp) and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include <complex>
#include <functional>
#include <string>
#include <vector>

#include "../../include/helm3d.h"

namespace h3d {

typedef std::complex<double> zc;

// ----------------------------------------------------------------- FFT plan
// Stockham mixed-radix plan for length nz: pass s has radix r_s and span
// p_s = r_0 ... r_{s-1}; its twiddles tw[off_s + k*r_s + q] =
// exp(-2 pi i q k / (p_s r_s)) for k < p_s, q < r_s.
constexpr int kMaxPasses = 12;
struct FftPlan {
    int n = 0;
    int npass = 0;
    int radix[kMaxPasses];
    int span[kMaxPasses];
    int twoff[kMaxPasses];
    int dftoff[kMaxPasses];   // offset of the radix-r DFT table exp(-2 pi i t / r)
    int twlen = 0;
};

// device-side view of the tables one FFT launch needs
template <typename R> struct FftTables {
    const void *tw;   // cplx<R>*, pass twiddles then per-pass DFT roots
};

// --------------------------------------------------------- launch helpers
struct Dev {
    int sm_count = 148;
    size_t smem_optin = 227 * 1024;
};

// A batch of R complex128 vectors: vector r at p + r * stride.  With c64
// the vectors are complex64 (p points to float2 data, stride counted in
// float2): only where a kernel says it takes them (FGMRES's Z basis).
struct VecBatch {
    double2 *p;
    long stride;
    bool c64 = false;
};
// Per-vector real scales: scale of vector r at p[r * stride] (p may be null: 1).
struct ScaleBatch {
    const double *p;
    long stride;
};

// Spectral planes of R right-hand sides: plane k, y-line j holds the R
// vectors of length nx contiguously: index ((k*ny + j)*R + r)*nx + i.
struct PlaneLayout {
    int nx, ny, nz, R;
    long plane;               // nx*ny
};

// FFT along z (stride nx*ny) of every z-column, for R right-hand sides.
//   forward: planes = FFT(scale * sc_r * x_r)        (complex128 in, P out)
//   inverse: y_r = IFFT(planes_r) / nz, then epilogue mode 0: y_r = t;
//            mode 1: y_r = scale * sc_r * w_r - dl * t (mode R's K x).
int launch_fft_forward(bool c64, const VecBatch &x, double scale, const ScaleBatch &sc, void *planes,
                       const PlaneLayout &L, const FftPlan &plan, const void *tw, cudaStream_t s);
int launch_fft_inverse(bool c64, const void *planes, const PlaneLayout &L, const VecBatch &y, const FftPlan &plan,
                       const void *tw, int mode, const VecBatch &w, double scale, const ScaleBatch &sc,
                       const double2 *dl, cudaStream_t s);

// Dense z-transforms with the eigenvectors of the z operator (FP64 matrices
// W, Wi row-major nz x nz): planes = Wi (scale sc_r x_r); y_r = W planes_r.
int launch_ztrans_forward(bool c64, const VecBatch &x, double scale, const ScaleBatch &sc, void *planes,
                          const PlaneLayout &L, const double2 *Wi, cudaStream_t s);
int launch_ztrans_inverse(bool c64, const void *planes, const PlaneLayout &L, const VecBatch &y, const double2 *W,
                          cudaStream_t s);

// The same eigenbasis transforms for complex64 planes on the tensor cores
// (tcgen05 kind::tf32, three TF32 products per real product): B is the matrix
// prepared by ztc_prepare (real form, hi/lo split, tensor-core layout).
bool ztc_supported(int nz);
void ztc_prepare(const std::vector<std::complex<double>> &M, int nz, std::vector<float> &out);
int launch_ztc_forward(const VecBatch &x, double scale, const ScaleBatch &sc, void *planes, const PlaneLayout &L,
                       const float *B, int *status, cudaStream_t s);
int launch_ztc_inverse(const void *planes, const PlaneLayout &L, const VecBatch &y, const float *B, int *status,
                       cudaStream_t s);

// Block-tridiagonal factor of all nz systems: G^T of every (kz, y-line).
struct FactorArgs {
    int n, ny, nz, ldg;
    void *Gt;                 // cplx<P> [nz][ny][n][ldg]  (G^T per block)
    const void *cmx, *cpx;    // cplx<P>[n]
    const void *cmy, *cpy;    // cplx<P>[ny]
    const void *base2d;       // cplx<P>[ny][n]: omega^2 s0^2 (1 + i beta)
    const void *kz2;          // cplx<P>[nz]: complex shift of mode k (-kz^2 or lambda_k)
    int *status;              // device flag: bit 0 = zero pivot
    const int *kzslot = nullptr;   // [nz]: >= 0 for a skipped mode (not factored), or null
};
// variant: one of the factor_variants(c64, n) launch shapes (0: the default)
int launch_factor(bool c64, const FactorArgs &a, cudaStream_t s, int variant = 0);
int factor_variants(bool c64, int n);
// the tensor-core factor (complex64, n <= 128): the last factor variant
bool factor_tc_supported(bool c64, int n);
int launch_factor_tc(const FactorArgs &a, cudaStream_t s);
// the tensor-core factor on a CTA pair per kz (complex64, 128 < n <= 224):
// the last factor variant of those block sizes
bool factor_tc2_supported(bool c64, int n);
int launch_factor_tc2(const FactorArgs &a, cudaStream_t s);
bool factor_supported(bool c64, int n);

// Forward/backward block sweep over y-lines for every kz and all R
// right-hand sides of the planes, in place.
struct SweepArgs {
    int n, ny, nz, ldg;
    const void *Gt;
    const void *cmy, *cpy;
    void *planes;             // PlaneLayout with R right-hand sides
    int R;
    const void *dxy;          // null: S^{-1}; else S^{-H} with the [2][ny][n] alpha_x alpha_y table
    int *status;              // device flag: bit 2 = a bounded wait expired
    int stage_kb = 16;        // bulk-copy stage of G^T rows (KB, about)
    int ring_kb = 200;        // shared-memory ring of stages (KB, at most)
    int tc_mc = 0;            // complex64, n <= 256: the tensor-core sweep with G^T chunks of tc_mc rows (16, 32)
    int tc_f16 = 0;           // ... with FP16 hi/lo products (K = 16 per MMA), scaled by gscale
    const float *gscale = nullptr;   // [nz][ny] power-of-two scales of the blocks (launch_gscale)
    int tc_pack = 0;          // the tensor-core sweep on the packed factor (sweep_tcp.cu)
    const void *gpack = nullptr;     // the packed factor (launch_gpack), or null
    // skipped modes (kz_skip_ratio): kzslot[kz] >= 0 marks one (the sweep
    // kernels leave it), kzlist[slot] = kz, kzinv[slot] its inverse diagonal
    const int *kzslot = nullptr, *kzlist = nullptr;
    int nskip = 0;
    const void *kzinv = nullptr;
};
int launch_sweep(bool c64, const SweepArgs &a, cudaStream_t s);
// Skipped modes (opts.kz_skip_ratio, the reference's SAVE_MEM): kzinv[slot][j][i]
// = 1 / (the diagonal of mode kzlist[slot]'s 2D operator: -(cmx+cpx)[i]
// -(cmy+cpy)[j] + base2d[j][i] + shift[kz]), or 0 with zero (mode R: the
// reference sets those modes' solution to zero); launch_kzskip_apply scales
// those modes' planes by it (by its conjugate for the adjoint).
int launch_kzinv(bool c64, const int *kzlist, int nskip, int nx, int ny, const void *cmx, const void *cpx,
                 const void *cmy, const void *cpy, const void *base2d, const void *shift, bool zero, void *kzinv,
                 cudaStream_t s);
int launch_kzskip_apply(bool c64, const SweepArgs &a, cudaStream_t s);
// the sweep's launch variants the autotuner times: stage and ring sizes of
// the CUDA-core kernels (0-5), the tensor-core kernel's chunk (6, 7), the
// tensor-core kernel with FP16 products (8), the tensor-core kernel on the
// packed factor (9)
constexpr int kSweepVariants = 10;
// power-of-two scale of every complex64 block G_j for the FP16 products
int launch_gscale(const void *Gt, int n, int ny, int nz, int ldg, float *gscale, cudaStream_t s);
void sweep_variant(int v, SweepArgs &a);
bool sweep_tc_supported(const SweepArgs &a);   // shape and shared memory fit
int launch_sweep_tc(const SweepArgs &a, int mc, cudaStream_t s);
// the complex64 factor (n <= 256) packed once into FP16 hi/lo tiles of
// s_j G_j (s_j = gscale) in the tensor core's operand layout, gpack_bytes
// bytes (about those of the complex64 factor), for launch_sweep_tcp
size_t gpack_bytes(int n, int ny, int nz);
int launch_gpack(const void *Gt, int n, int ny, int nz, int ldg, const float *gscale, void *Gp, cudaStream_t s);
bool sweep_tcp_supported(const SweepArgs &a);
int launch_sweep_tcp(const SweepArgs &a, cudaStream_t s);
constexpr int kMaxBatch = 16;  // right-hand sides per preconditioner launch

// Classical Gram-Schmidt takes a second pass when the first left less than
// this fraction of ||w||^2 (0.5: Kahan's "twice is enough", eta = 1/sqrt 2)
#ifndef H3D_REORTH_ETA2
#define H3D_REORTH_ETA2 0.5
#endif

// 7-point PML operator y_r = A (xscale sc_r x_r) (adjoint: A^H), complex128.
struct StencilArgs {
    int nx, ny, nz;
    const double2 *cmx, *cpx, *cmy, *cpy, *cmz, *cpz;
    const double *s2;
    double w2;                // omega^2
    double beta_phys;
    VecBatch x;
    double xscale;
    ScaleBatch sc;
    VecBatch y;
    VecBatch f;               // if f.p: y = f - A x
    int R;
    int zchunk = 16;          // z points per thread (autotuned: 8, 16, 32, 64)
    int src_fast = 0;         // grid z order: 0 = z chunks within a source, 1 = sources within a z chunk
    int smem = 0;             // 1: x/y neighbours from the plane's tile staged in shared memory
};
int launch_stencil(const StencilArgs &a, bool adjoint, cudaStream_t s);

// ------------------------------------------------------ Krylov kernels
// All vectors complex128 of length N; a basis V_r of nv vectors (leading
// dimension ldv) per right-hand side r, with real scales vs (basis vector i
// of r is vs[r][i] V_r[i]).
struct Reduce {
    double2 *partials;        // [rmax][nblocks][cap] scratch
    int nblocks;
    int cap;
    int rmax;
    int update = 0;           // DCGS2 update pass variant (0: loads one by one, 1: 8 basis loads batched)
};
// out[r][i] = <vs_r[i] V_r[i], w_r>   (i < nv); with wnorm also out[r][nv].x = ||w_r||^2
// (pred: when given and *pred == 0 on the device, the kernels do nothing)
int launch_dots(const VecBatch &V, long ldv, const ScaleBatch &vs, int nv, const VecBatch &w, long N, int R,
                const Reduce &red, double2 *out, long sOut, cudaStream_t s, bool wnorm = false,
                const int *pred = nullptr);
// w_r -= sum_i coef[r][i] vs_r[i] V_r[i]; post 1: out[r].x = ||w_r||^2
int launch_update(const VecBatch &V, long ldv, const ScaleBatch &vs, int nv, const double2 *coef, long sCoef,
                  const VecBatch &w, long N, int R, int post, const Reduce &red, double2 *out, long sOut,
                  cudaStream_t s, const int *pred = nullptr);
// x_r += sum_i y[r][i] zs_r[i] Z_r[i]  (i < min(nzv, *nzv_dev) when nzv_dev is given)
int launch_combine(const VecBatch &Z, long ldz, const ScaleBatch &zs, int nzv, const double2 *y, long sY,
                   const VecBatch &x, long N, int R, cudaStream_t s, const int *nzv_dev = nullptr);

// ------------------------------------------- device-side Arnoldi bookkeeping
// Per right-hand side p of a lockstep batch of B (the host FGMRES state, on
// the device so that a whole restart cycle runs without the host):
struct ArnState {
    double2 *H;        // [B][m+1][m] Hessenberg columns, Givens-rotated (upper triangle = R)
    double2 *cs, *sn;  // [B][m] rotations
    double2 *g;        // [B][m+1] rotated right-hand side (g[0] = beta on entry)
    double *est;       // [B][m] |g[j+1]| / ||f|| after step j
    double *nf, *tol;  // [B]
    double *beta;      // [B] ||w'|| of the last update (DCGS2: the open column's scale)
    int *frozen, *k, *it, *max_iter;   // [B]
    int *flags;        // [kArnFlags]: [0] second Gram-Schmidt pass wanted, [1] second passes taken,
                       // [2] longest k, [3] error, [4] last step run, [5] some p still active
    int m, B;
    double2 *h;        // Krylov scalars: [B][SH], h1 at 0, h2 at M2, norms at 2 M2, y at 3 M2
    int SH, M2;
    double *vs;        // basis scales [B][M2]
};
constexpr int kArnFlags = 8;
// flags[0] = any unfrozen p with ||w||^2 after the first pass < 1/2 of before
int launch_reorth_check(const ArnState &a, int j, cudaStream_t s);
// column j of H (h1 + h2 when flags[0]), rotations, g, est, frozen, k, it,
// vs[j + 1]; sets `next` (if has_next) to "some p is still unfrozen"
int launch_givens(const ArnState &a, int j, bool has_next, cudaGraphConditionalHandle next, cudaStream_t s);
// DCGS2 (low-synchronization Gram-Schmidt with delayed reorthogonalization,
// flexible FGMRES): per step j one reduction (dots2) and one update pass
// (update2) over the basis.  Krylov scalars per right-hand side: dots at h
// (2 j + 2 slots), ||w'||^2 at 2 M2, update coefficients alpha at 4 M2 and
// delta at 5 M2.
int launch_dots2(const VecBatch &V, long ldv, const ScaleBatch &vs, int j, const VecBatch &w, long N, int R,
                 const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred, const int *skip);
int launch_update2(const VecBatch &V, long ldv, int j, const double2 *coef, long sCoef, int M2, const VecBatch &w,
                   long N, int R, const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred,
                   const int *skip);
// reorthogonalization dots of the cycle's last tentative vector V_{jl+1},
// jl = *jl on the device (tmax: the largest jl + 1)
int launch_dots_tail(const VecBatch &V, long ldv, const ScaleBatch &vs, int tmax, const int *jl, long N, int R,
                     const Reduce &red, double2 *out, long sOut, cudaStream_t s, const int *pred, const int *skip);
// finalize column j - 1, write column j and the update coefficients
int launch_lagged(const ArnState &a, int j, cudaStream_t s);
// beta, vs[j + 1], flags[4..5] and the condition of step j + 1
int launch_post(const ArnState &a, int j, bool has_next, cudaGraphConditionalHandle next, cudaStream_t s);
// finalize the open column of the cycle's last step
int launch_lagged_final(const ArnState &a, cudaStream_t s);
// y = R^{-1} g (k x k per p, zero padded to m) into h at 3 M2; flags[2] = max k
int launch_backsub(const ArnState &a, cudaStream_t s);
// out[r].x = ||x_r||^2 over the box [x0,x1) x [y0,y1) x [z0,z1)
int launch_norm2_box(const VecBatch &x, int R, int nx, int ny, int nz, const int box[6], const Reduce &red,
                     double2 *out, long sOut, cudaStream_t s);
// y_r = a x_r + b y_r
int launch_axpby(double2 a, const VecBatch &x, double2 b, const VecBatch &y, long N, int R, cudaStream_t s);
// y = x - dl * t  (mode R's K x from t = L0^{-1} x)
int launch_sub_dl(const double2 *x, const double2 *dl, const double2 *t, double2 *y, long N, cudaStream_t s);
// vs[r][j] = 1 / sqrt(nrm[r].x)
int launch_set_scale(const double2 *nrm, long sNrm, double *vs, long sVs, int j, int R, cudaStream_t s);
// base2d[q] = w2 (1 + i beta) mean_{zlo <= k < zhi} s2[k][q]  (P precision);
// sets bit 4 of *status when s2 holds NaN/Inf
int launch_base2d(bool c64, const double *s2, int nz, long plane, int zlo, int zhi, double w2, double beta,
                  void *base2d, int *status, cudaStream_t s);
// ---------------------------------------------------- misfit gradient
// res[r][q] = u_r[recv[q]] - d[r][q]   (q < nrecv; res stride nrecv, d stride sD)
int launch_receiver_residual(const VecBatch &u, int R, const long long *recv, int nrecv, const double2 *d, long sD,
                             double2 *res, cudaStream_t s);
// y_r[recv[q]] += sign * res[r][q]  (atomic: receivers may repeat)
int launch_adjoint_source(const double2 *res, int R, const long long *recv, int nrecv, double sign,
                          const VecBatch &y, cudaStream_t s);
// g += sum_r Re(conj(lam_r) w2 (1 + i beta) u_r)
int launch_grad_accum(const VecBatch &lam, const VecBatch &u, int R, double w2, double beta, double *g, long N,
                      cudaStream_t s);

Dev &device_info();

// Raise a kernel's dynamic shared-memory limit to the device maximum (less
// its static shared memory) and check that `need` fits.  The limit belongs to
// the function and is read by every launch, kernel nodes of instantiated
// CUDA graphs included, so it is only ever raised: lowering it to one
// launch's size would break a graph captured earlier with a larger size.
// Each launch still passes its own size (which sets its occupancy).
template <typename K> inline bool smem_limit_max(K kern, size_t need) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return false;
    const size_t cap = device_info().smem_optin - fa.sharedSizeBytes;
    if (need > cap) return false;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= cap) return true;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap) == cudaSuccess;
}

// ------------------------------------------------------------- autotuner
// The fastest of nvariants launch shapes of a kernel family for a problem
// shape: launch(v) runs variant v once on the context's stream; the choice is
// cached per (family, shape) for the process (and in HELM3D_TUNE_CACHE).
// Not for use inside a stream capture.
bool tune_enabled();
// The polls a kernel's bounded waits between its warps make before giving
// up: `dflt`, or HELM3D_WAIT_LIMIT (read at every launch) when set, so that
// a test can make such a wait expire and check the status it reports.
uint32_t wait_limit_polls(uint32_t dflt);
// HELM3D_FORCE_<family> as an integer, or -1 when unset
int tune_forced(const char *family);
// z chunk 16, 8, 32, 64; source-major (0-3) or source-minor (4-7) grid;
// 8-11: the shared-memory staged kernel, source-minor, z chunk 16, 32, 64, 8
constexpr int kStencilVariants = 12;
constexpr int kReduceVariants = 3;    // reduction blocks 2, 1, 4 per SM
constexpr int kUpdateVariants = 2;    // DCGS2 update pass: basis loads one by one, 8 batched
int stencil_zchunk(int v);
int stencil_src_fast(int v);
int stencil_smem(int v);
int reduce_blocks(int v);

}  // namespace h3d

// ---------------------------------------------------------------- context
struct helm3d_ctx {
    helm3d_grid grid;
    helm3d_opts opts;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool c64 = true;
    long N = 0;                // nx*ny*nz
    long plane = 0;            // nx*ny
    int ldg = 0;
    std::string last_error;
    long long launches = 0;
    double ms_factor = 0;      // wall time of set-up + factor in helm3d_create
    long long reorth = 0;      // Gram-Schmidt second passes taken
    cudaStream_t own_stream = nullptr;
    // helm3d_solve_medium: host right-hand sides copied in under the factor
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copy0 = nullptr, ev_copy = nullptr;

    // optional per-kernel-family profiler (helm3d_profile)
    struct ProfEv {
        int kind;
        cudaEvent_t a, b;
    };
    bool prof = false;
    std::vector<ProfEv> prof_ev;
    double prof_ms[HELM3D_K_COUNT] = {0};
    long long prof_n[HELM3D_K_COUNT] = {0};

    // host copies of the set-up tables (FP64)
    std::vector<h3d::zc> cmx, cpx, cmy, cpy, cmz, cpz;
    std::vector<double> kz2;
    std::vector<h3d::zc> base2d;   // [ny][nx]
    bool zeig = false;             // PML eigenbasis z-transform instead of the FFT
    std::vector<h3d::zc> zshift;   // per-mode diagonal shift: -kz^2 or lambda_k
    std::vector<h3d::zc> zW, zWi;  // z eigenvectors (row-major nz x nz) and inverse
    h3d::FftPlan plan;

    // device buffers
    void *d_Gt = nullptr;          // factor
    float *d_gscale = nullptr;     // [nz][ny] scales of the complex64 blocks (FP16 sweep)
    void *d_gpack = nullptr;       // complex64, n <= 256: the factor packed as FP16 hi/lo tiles (launch_gpack)
    size_t Gt_bytes = 0;
    void *d_tw = nullptr;          // FFT tables (precision P)
    void *d_cmx = nullptr, *d_cpx = nullptr, *d_cmy = nullptr, *d_cpy = nullptr;   // P precision
    void *d_base2d = nullptr, *d_kz2 = nullptr;                                    // P precision (kz2: complex mode shifts)
    void *d_zW = nullptr, *d_zWi = nullptr;                                        // P precision
    double2 *d_zW64 = nullptr, *d_zWi64 = nullptr;
    double2 *d_zWH64 = nullptr, *d_zWiH64 = nullptr;   // W^H, Wi^H (adjoint z-transforms)
    // tensor-core forms of Wi, W, W^H, Wi^H (complex64 eigenbasis path)
    bool ztc = false;
    bool z64 = false;              // mode N, complex64 preconditioner: FGMRES's Z_j = M^{-1} V_j kept in complex64
    // skipped modes (opts.kz_skip_ratio): per kz the slot or -1, the slots' kz,
    // the slots' inverse diagonals (cplx<P> [nskip][ny][nx])
    std::vector<int> kzslot_h;
    int nskip = 0;
    int *d_kzslot = nullptr, *d_kzlist = nullptr;
    void *d_kzinv = nullptr;
    size_t kzinv_bytes = 0;
    float *d_ztc[4] = {nullptr, nullptr, nullptr, nullptr};
    void *d_dxy = nullptr;         // [2][ny][nx] alpha_x alpha_y and conj(1 / (alpha_x alpha_y)), P precision
    double2 *d_cmx64 = nullptr, *d_cpx64 = nullptr, *d_cmy64 = nullptr, *d_cpy64 = nullptr;
    double2 *d_cmz64 = nullptr, *d_cpz64 = nullptr;
    double *d_s2 = nullptr;        // squared slowness (mode N operator)
    double2 *d_dl = nullptr;       // dL (mode R)
    void *d_planes = nullptr;      // spectral planes, P precision (planes_R right-hand sides)
    int planes_R = 0;
    int *d_status = nullptr;
    int factor_rc = HELM3D_OK;   // status of the last set-up and factor (set_medium)
    // Krylov workspace for r_alloc right-hand sides of restart length m_alloc
    int m_alloc = 0, r_alloc = 0;
    size_t kry_bytes = 0;
    double2 *d_V = nullptr, *d_Z = nullptr;
    double2 *d_Fw = nullptr, *d_Uw = nullptr;   // packed right-hand sides / iterates of the active batch
    void *d_arn = nullptr;                      // device-side Arnoldi state (ArnState arrays)
    // restart cycles captured as CUDA graphs, one per (batch size, adjoint)
    struct CycleGraph {
        int B;
        bool adjoint;
        cudaGraphExec_t exec;
        long long kernels_per_step, tail_kernels;
    };
    std::vector<CycleGraph> graphs;
    bool use_graphs = true;
    bool gs_lowsync = true;                     // mode N: DCGS2 (HELM3D_GS=cgs2: classical CGS2)
    // autotuned launch variants: the factor's, and the sweep's (forward,
    // adjoint) and stencil's of the current solve's batch (reduction blocks:
    // red_blocks)
    int tv_factor = 0;
    int tv_sweep[2] = {0, 0};
    int tv_stencil = 0;
    int tv_update = 0;
    size_t f_cap = 0, u_cap = 0;                // staging capacities (vectors) of d_f, d_u
    double *d_vs = nullptr;
    double2 *d_h = nullptr;        // small device scalars
    double2 *d_partials = nullptr;
    int red_blocks = 0, red_cap = 0;
    double2 *d_f = nullptr, *d_u = nullptr, *d_r = nullptr, *d_t = nullptr, *d_t2 = nullptr;
    double2 *d_bic = nullptr;      // BiCGStab vectors
    size_t bytes = 0;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double2 *h_scal = nullptr;     // pinned host mirror of the Krylov scalars, kept across solves
    size_t h_scal_cap = 0;         // its capacity (double2)
};

namespace h3d {
// Run one launch (or a short fixed sequence of `kernels` launches) of a kernel
// family: counts the launches and, when profiling, brackets them with events
// on the context's stream.
template <class F> int timed(helm3d_ctx *c, int kind, int kernels, F &&f) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (c->prof) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, c->stream);
    }
    const int rc = f();
    if (c->prof) {
        cudaEventRecord(b, c->stream);
        c->prof_ev.push_back({kind, a, b});
        c->prof_n[kind] += kernels;
    }
    c->launches += kernels;
    return rc;
}

int tune_pick(helm3d_ctx *c, const char *family, const std::string &shape, int nvariants,
              const std::function<int(int)> &launch);
// tune the solve-time kernels (sweep, stencil, reductions) of a batch of R
// (and the adjoint forms) on the context's own buffers, before any capture
int tune_solve(helm3d_ctx *c, int R, bool adjoint);
int ctx_setup_grid(helm3d_ctx *c);                                   // grid/option tables, allocations
int ctx_setup_medium(helm3d_ctx *c, const double *s2, bool s2_on_device);  // medium tables
int ctx_factor(helm3d_ctx *c);
// operators on R right-hand sides y_r = Op(xscale sc_r x_r) (R <= kMaxBatch)
int apply_prec(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y, int R);
int apply_op(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y, int R);
int apply_op_adjoint(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y,
                     int R);
// y_r = M^{-H} (xscale sc_r x_r)
int apply_prec_adjoint(helm3d_ctx *c, const VecBatch &x, double xscale, const ScaleBatch &sc, const VecBatch &y,
                       int R);
// FGMRES on R right-hand sides f + r N -> u + r N (device), iterated in lockstep
int fgmres(helm3d_ctx *c, const double2 *f, double2 *u, int R, bool adjoint, helm3d_stats *st);
// FGMRES on n contexts at once (R[i] <= kMaxBatch right-hand sides of device
// vectors f[i] -> u[i] each): every restart cycle of every context in one
// graph launch on the first context's stream
int fgmres_group(helm3d_ctx *const *cs, int n, const double2 *const *f, double2 *const *u, const int *R,
                 helm3d_stats *const *st);
int bicgstab(helm3d_ctx *c, const double2 *f, double2 *u, helm3d_stats *st);
int ensure_krylov(helm3d_ctx *c, int m, int R);
int set_error(helm3d_ctx *c, int code, const std::string &msg);
bool is_device_ptr(const void *p);   // device or managed memory
int cuda_check(helm3d_ctx *c, cudaError_t e, const char *what);
// Reads the context's device status word after the stream's work: a bounded
// wait that expired (bits 1, 2) or a failed index check (bit 3) in a kernel
// -> HELM3D_ERR_CUDA.  Synchronizes the stream; allocates nothing.
int check_status(helm3d_ctx *c);
// Start of a call that runs kernels on the context (see capi.cpp).
int begin_call(helm3d_ctx *c);
void build_fft_plan(int n, FftPlan &plan, std::vector<zc> &tables);
}  // namespace h3d
