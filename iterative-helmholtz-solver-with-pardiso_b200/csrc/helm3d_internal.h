// helm3d_internal.h -- context and kernel launchers shared by the host code
// (setup.cpp, solver.cpp, capi.cpp) and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>

#include <complex>
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

// FFT along z for a batch of columns [0, ncols) of nz-long columns with
// stride `plane` (= nx*ny).
//   forward: in = complex128 vector (times `scale`), out = planes of type P
//   inverse: in = planes of type P, out = complex128 vector scaled 1/nz,
//            then epilogue: mode 0 y = t; mode 1 y = scale*w - dl*t (mode R's
//            K x with x = scale*w).
int launch_fft_forward(bool c64, const double2 *x, double scale, void *planes, int nz, long plane,
                       const FftPlan &plan, const void *tw, cudaStream_t s);
int launch_fft_inverse(bool c64, const void *planes, double2 *y, int nz, long plane, const FftPlan &plan,
                       const void *tw, int mode, const double2 *w, double scale, const double2 *dl,
                       cudaStream_t s);

// Dense z-transforms with the eigenvectors of the z operator (FP64 matrices
// W, Wi row-major nz x nz): planes = Wi (scale x); y = W planes.
int launch_ztrans_forward(bool c64, const double2 *x, double scale, void *planes, int nz, long plane,
                          const double2 *Wi, cudaStream_t s);
int launch_ztrans_inverse(bool c64, const void *planes, double2 *y, int nz, long plane, const double2 *W,
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
};
int launch_factor(bool c64, const FactorArgs &a, cudaStream_t s);
bool factor_supported(bool c64, int n);

// Forward/backward block sweep over y-lines for every kz, in place on the
// planes (cplx<P> [nz][ny][n]).
struct SweepArgs {
    int n, ny, nz, ldg;
    const void *Gt;
    const void *cmy, *cpy;
    void *planes;
    int nrhs;
    long rhs_stride;          // elements between right-hand sides' planes
    int *status;              // device flag: bit 2 = a bounded wait expired
};
int launch_sweep(bool c64, const SweepArgs &a, cudaStream_t s);

// 7-point PML operator y = A x (adjoint: y = A^H x), complex128.
struct StencilArgs {
    int nx, ny, nz;
    const double2 *cmx, *cpx, *cmy, *cpy, *cmz, *cpz;
    const double *s2;
    double w2;                // omega^2
    double beta_phys;
    const double2 *x;
    double xscale;
    double2 *y;
    const double2 *f;         // if non-null: y = f - A x
};
int launch_stencil(const StencilArgs &a, bool adjoint, cudaStream_t s);

// ------------------------------------------------------ Krylov kernels
// All vectors complex128 of length N; V is a basis of nv vectors with
// leading dimension ldv and per-vector real scale vs[i] (the basis vector is
// vs[i] * V_i).
struct Reduce {
    double2 *partials;        // [nblocks][cap] scratch
    int nblocks;
    int cap;
};
// out[i] = sum_l conj(vs[i] V_i[l]) w[l]   (i < nv); with wnorm also
// out[nv].x = ||w||^2 from the same pass
int launch_dots(const double2 *V, long ldv, const double *vs, int nv, const double2 *w, long N,
                const Reduce &red, double2 *out, cudaStream_t s, bool wnorm = false);
// w -= sum_i coef[i] vs[i] V_i; then if redot: out[i] = <vs_i V_i, w_new>;
// if norm: out[0].x = ||w_new||^2.  (out may be null)
int launch_update(const double2 *V, long ldv, const double *vs, int nv, const double2 *coef, double2 *w,
                  long N, int post, const Reduce &red, double2 *out, cudaStream_t s);
// x += sum_i y[i] zs[i] Z_i
int launch_combine(const double2 *Z, long ldz, const double *zs, int nz_, const double2 *y, double2 *x, long N,
                   cudaStream_t s);
// out = ||x||^2 over the box [x0,x1) x [y0,y1) x [z0,z1) (whole grid by default)
int launch_norm2_box(const double2 *x, int nx, int ny, int nz, const int box[6], const Reduce &red,
                     double2 *out, cudaStream_t s);
// y = a*x + b*y
int launch_axpby(double2 a, const double2 *x, double2 b, double2 *y, long N, cudaStream_t s);
// y = x - dl * t  (mode R's K x from t = L0^{-1} x)
int launch_sub_dl(const double2 *x, const double2 *dl, const double2 *t, double2 *y, long N, cudaStream_t s);
// vs[j] = 1/sqrt(nrm[0]); h[j] = sqrt(nrm) etc. -- small device helpers
int launch_set_scale(const double2 *nrm, double *vs, int j, cudaStream_t s);
int launch_add_vec(const double2 *a, const double2 *b, double2 *out, int n, cudaStream_t s);
int launch_zero(void *p, size_t bytes, cudaStream_t s);
// base2d[q] = w2 (1 + i beta) mean_{zlo <= k < zhi} s2[k][q]  (P precision);
// sets bit 4 of *status when s2 holds NaN/Inf
int launch_base2d(bool c64, const double *s2, int nz, long plane, int zlo, int zhi, double w2, double beta,
                  void *base2d, int *status, cudaStream_t s);
// gradient accumulation g += Re(conj(lam) * w2 * u)  (d A / d s2 = w2 (1 + i beta))
int launch_grad_accum(const double2 *lam, const double2 *u, double w2, double beta, double *g, long N,
                      cudaStream_t s);
int launch_gather_residual(const double2 *u, const long long *recv, int nrecv, const double2 *d, double2 *res,
                           cudaStream_t s);
int launch_scatter_add(const double2 *vals, const long long *recv, int nrecv, double2 *y, double sign,
                       cudaStream_t s);

Dev &device_info();

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
    size_t Gt_bytes = 0;
    void *d_tw = nullptr;          // FFT tables (precision P)
    void *d_cmx = nullptr, *d_cpx = nullptr, *d_cmy = nullptr, *d_cpy = nullptr;   // P precision
    void *d_base2d = nullptr, *d_kz2 = nullptr;                                    // P precision (kz2: complex mode shifts)
    void *d_zW = nullptr, *d_zWi = nullptr;                                        // P precision
    double2 *d_zW64 = nullptr, *d_zWi64 = nullptr;
    double2 *d_cmx64 = nullptr, *d_cpx64 = nullptr, *d_cmy64 = nullptr, *d_cpy64 = nullptr;
    double2 *d_cmz64 = nullptr, *d_cpz64 = nullptr;
    double *d_s2 = nullptr;        // squared slowness (mode N operator)
    double2 *d_dl = nullptr;       // dL (mode R)
    void *d_planes = nullptr;      // spectral planes, P precision (one RHS)
    int *d_status = nullptr;
    // Krylov workspace
    int m_alloc = 0;
    double2 *d_V = nullptr, *d_Z = nullptr;
    double *d_vs = nullptr;
    double2 *d_h = nullptr;        // small device scalars
    double2 *d_partials = nullptr;
    int red_blocks = 0, red_cap = 0;
    double2 *d_f = nullptr, *d_u = nullptr, *d_r = nullptr, *d_t = nullptr, *d_t2 = nullptr;
    double2 *d_bic = nullptr;      // BiCGStab vectors
    size_t bytes = 0;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
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

int ctx_setup_grid(helm3d_ctx *c);                                   // grid/option tables, allocations
int ctx_setup_medium(helm3d_ctx *c, const double *s2, bool s2_on_device);  // medium tables
int ctx_factor(helm3d_ctx *c);
int apply_prec(helm3d_ctx *c, const double2 *x, double xscale, double2 *y);
int apply_op(helm3d_ctx *c, const double2 *x, double xscale, double2 *y);
int apply_op_adjoint(helm3d_ctx *c, const double2 *x, double xscale, double2 *y);
int apply_prec_adjoint(helm3d_ctx *c, const double2 *x, double xscale, double2 *y);
int fgmres(helm3d_ctx *c, const double2 *f, double2 *u, bool adjoint, helm3d_stats *st);
int bicgstab(helm3d_ctx *c, const double2 *f, double2 *u, helm3d_stats *st);
int ensure_krylov(helm3d_ctx *c, int m);
int set_error(helm3d_ctx *c, int code, const std::string &msg);
bool is_device_ptr(const void *p);   // device or managed memory
int cuda_check(helm3d_ctx *c, cudaError_t e, const char *what);
void build_fft_plan(int n, FftPlan &plan, std::vector<zc> &tables);
}  // namespace h3d
