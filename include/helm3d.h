/*
 * helm3d.h -- C ABI of the B200 3D Helmholtz solver.
 *
 * The solve is the reference's: a Krylov outer iteration preconditioned by
 * an FFT along z that splits the 3D problem into one shifted 2D system per
 * kz (dklyuchinskiy/Iterative-Helmholtz-solver-with-PARDISO).  The 2D
 * systems are factorised here by a batched block-tridiagonal block LU over
 * y-lines instead of PARDISO.  Every call returns a helm3d_status (0 = OK).
 *
 * Vectors are complex128, interleaved (re, im), laid out l = i + nx*j +
 * nx*ny*k (x fastest) as the reference's take_coord3D
 * (Source/functions.cpp:225-230).  A vector argument may be a device
 * pointer or a host pointer (pageable or pinned); host data is copied in and
 * out by the call.  A context owns the factor and all workspace; it is not
 * shared between threads.  Work is ordered on the context's stream.
 *
 * Two operators (helm3d_opts.mode):
 *   HELM3D_MODE_R  the reference's K w = (I - dL L0^{-1}) w = f, u = L0^{-1} w
 *                  (Source/FGMRES.cpp:464-684, Source/functions.cpp:5554-5575)
 *   HELM3D_MODE_N  the 7-point PML-stretched operator A u = f, with the FFT-z
 *                  operator as a flexible right preconditioner M.
 */
#ifndef HELM3D_H
#define HELM3D_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HELM3D_ABI_VERSION 1

typedef enum helm3d_status {
    HELM3D_OK = 0,
    HELM3D_ERR_ARG = 1,            /* bad argument or unsupported size */
    HELM3D_ERR_OOM = 2,            /* device allocation failed */
    HELM3D_ERR_CUDA = 3,           /* a CUDA call failed */
    HELM3D_ERR_SINGULAR = 4,       /* zero pivot in the block LU factor */
    HELM3D_ERR_NOT_CONVERGED = 5,  /* max_iter reached above tol */
    HELM3D_ERR_BREAKDOWN = 6,      /* Krylov breakdown (BiCGStab rho/omega = 0) */
    HELM3D_ERR_NONFINITE = 7,      /* NaN/Inf in the input or a residual */
    HELM3D_ERR_NO_DEVICE = 8       /* no usable CUDA device */
} helm3d_status;

typedef enum helm3d_mode { HELM3D_MODE_R = 0, HELM3D_MODE_N = 1 } helm3d_mode;

/* arithmetic and storage type of the preconditioner (FFT planes, factor,
 * sweep); the outer Krylov loop is always complex128 */
typedef enum helm3d_precision { HELM3D_PREC_C128 = 0, HELM3D_PREC_C64 = 1 } helm3d_precision;

/* kz^2 of plane k: (4/hz^2) sin^2(pi k/nz) | (2 pi min(k,nz-k)/Lz)^2 |
 * the reference's table (Source/FGMRES.cpp:182-190) */
typedef enum helm3d_kz_symbol {
    HELM3D_KZ_DISCRETE = 0,
    HELM3D_KZ_CONTINUOUS = 1,
    HELM3D_KZ_REFERENCE = 2
} helm3d_kz_symbol;

/* How the preconditioner separates z (mode N):
 *   HELM3D_ZT_FFT        the reference's FFT along z with the periodic kz^2
 *                        symbol (Source/functions.cpp:5858-5881);
 *   HELM3D_ZT_PML_EIGEN  the eigenvectors of the 1D z operator with its PML
 *                        (D_z = W diag(lambda) W^{-1}), applied as dense
 *                        z-transforms; the per-mode shift is lambda_k.  The
 *                        split into one shifted 2D system per z-mode and the
 *                        block LU are unchanged; M equals A when the medium
 *                        is z-invariant and beta_prec = 0. */
typedef enum helm3d_z_transform { HELM3D_ZT_FFT = 0, HELM3D_ZT_PML_EIGEN = 1 } helm3d_z_transform;

/* Grid: mirrors size_m (Source/definitions.h:55-68) for three axes. */
typedef struct helm3d_grid {
    int nx, ny, nz;          /* points per axis, PML/sponge included */
    double hx, hy, hz;       /* steps */
    int pml_x, pml_y, pml_z; /* PML points on each face (alpha != 1 there) */
    int spg_z;               /* sponge points at each z end (mode R) */
    double lz;               /* z period of the kz table; 0 -> nz*hz */
    double omega;            /* angular frequency */
} helm3d_grid;

typedef struct helm3d_opts {
    int mode;            /* helm3d_mode */
    int precision;       /* helm3d_precision */
    int kz_symbol;       /* helm3d_kz_symbol */
    double beta_prec;    /* complex shift of the preconditioner; mode R: beta_eq.  The FFT-z
                          * preconditioner needs damping (0.25); with HELM3D_ZT_PML_EIGEN a small
                          * shift (0.01) converges in far fewer iterations (measured at 128^3-200^3:
                          * 7-8 instead of 22-33) */
    double beta_phys;    /* mode N: physical damping in A */
    double s2_l0;        /* mode R: > 0 -> L0 uses this constant s^2 (HOMO, q3) */
    int quirk_q1;        /* mode R: c0 by the reference's running-sum mean (q1) */
    int restart;         /* FGMRES cycle length m */
    int max_iter;        /* total iteration cap */
    double tol;          /* relative residual target ||f - A u|| / ||f|| */
    int stop_phys;       /* 1: test the physical-domain residual instead */
    int device;          /* CUDA device ordinal */
    int verbose;
    int z_transform;     /* helm3d_z_transform (mode N; mode R always uses the FFT) */
    double kz_skip_ratio; /* > 0: the reference's SAVE_MEM (Source/FGMRES.cpp:197-206):
                           * mode k with kww >= ratio * k2 is not factored (kww its kz^2,
                           * -Re of its shift; k2 = omega^2 s2_l0 when s2_l0 > 0, else
                           * omega^2 times the largest s0^2 of the 2D medium); mode R sets
                           * its solution to zero as the reference does, mode N solves it
                           * by the diagonal of its 2D operator.  0 (default): off */
} helm3d_opts;

typedef struct helm3d_stats {
    int status;
    int iterations;       /* Krylov iterations over all right-hand sides */
    int restarts;
    double relres;        /* true ||f - A u|| / ||f|| over the whole grid */
    double relres_phys;   /* the same restricted to the physical domain */
    double ms_factor;     /* set-up + factor time of helm3d_create */
    double ms_solve;      /* device time of the last solve */
    double *history;      /* optional caller buffer: residual estimate per iteration */
    int history_cap;
    int history_len;
} helm3d_stats;

typedef struct helm3d_ctx helm3d_ctx;

/* Fill opts with defaults (mode N, C64 preconditioner, discrete kz symbol,
 * beta_prec 0.25, restart 20, tol 1e-8). */
int helm3d_default_opts(helm3d_opts *opts);

/* Set up a solve on one device: PML tables, media (s2 = 1/c^2, real,
 * nx*ny*nz, host or device), the kz table and the block LU factor of every
 * kz system.  Replaces FGMRES's set-up block (Source/FGMRES.cpp:72-298). */
int helm3d_create(const helm3d_grid *grid, const double *s2, const helm3d_opts *opts, helm3d_ctx **ctx);

/* New medium on the same grid: recompute dL / shifts and refactor. */
int helm3d_set_medium(helm3d_ctx *ctx, const double *s2);

/* Solve for nrhs right-hand sides f[r*N .. ] -> u[r*N ..] with FGMRES from
 * a zero initial guess.  The right-hand sides go through the iteration in
 * lockstep batches of up to 16 (as many as device memory holds), one
 * preconditioner and operator launch per step for the whole batch;
 * stats->iterations is summed over the right-hand sides and relres is the
 * largest.  Replaces FGMRES (Source/FGMRES.cpp:6-725, prototype
 * Source/templates.h:59), which the reference calls once per source. */
int helm3d_solve(helm3d_ctx *ctx, const double *f, double *u, int nrhs, helm3d_stats *stats);

/* helm3d_set_medium(ctx, s2) then helm3d_solve(ctx, f, u, nrhs, stats) in
 * one call, as the reference's FGMRES builds the medium, factors and solves
 * in one call (Source/FGMRES.cpp:72-298 then :300-725).  With host f (pinned
 * for the overlap) and nrhs in one lockstep batch, the right-hand sides are
 * copied to the device while the medium is set up and factored.  Returns the
 * factor's error (and leaves the context refusing solves, as
 * helm3d_set_medium does) or the solve's status. */
int helm3d_solve_medium(helm3d_ctx *ctx, const double *s2, const double *f, double *u, int nrhs,
                        helm3d_stats *stats);

/* Solve n contexts at once: grids of different sizes, each with its own
 * medium, options and factor, on one device.  Context i solves nrhs[i]
 * right-hand sides f[i] -> u[i] (host or device pointers, laid out as for
 * helm3d_solve).  The contexts iterate FGMRES in lockstep restart cycles,
 * and each cycle of all of them is one CUDA graph whose independent branches
 * (one per context) run side by side on the GPU, so that small grids that
 * cannot fill it alone share it.  The work is ordered on the first context's
 * stream; stats (n entries, or NULL) are per context.  A context may appear
 * only once.  No counterpart in the reference, which solves one grid per
 * run (Source/main.cpp:470). */
int helm3d_solve_group(helm3d_ctx *const *ctxs, int n, const double *const *f, double *const *u, const int *nrhs,
                       helm3d_stats *stats);

/* The same system by BiCGStab with the reference's shadow residual 2 r0.
 * Replaces BCGSTAB (Source/BcGSTAB.cpp:6-666, Source/templates.h:60). */
int helm3d_solve_bicgstab(helm3d_ctx *ctx, const double *f, double *u, helm3d_stats *stats);

/* Adjoint solve A^H lambda = g (mode N) by FGMRES right-preconditioned with
 * M^{-H}.  No counterpart in the reference. */
int helm3d_solve_adjoint(helm3d_ctx *ctx, const double *g, double *lambda, helm3d_stats *stats);

/* y = A x (mode N) or y = K x = x - dL L0^{-1} x (mode R,
 * ApplyCoeffMatrixA_CSR, Source/functions.cpp:5554-5575). */
int helm3d_apply_op(helm3d_ctx *ctx, const double *x, double *y);

/* y = A^H x (mode N). */
int helm3d_apply_op_adjoint(helm3d_ctx *ctx, const double *x, double *y);

/* y = M^{-1} x: forward FFT along z, one 2D solve per kz, inverse FFT
 * (Solve3DSparseUsingFT_CSR, Source/functions.cpp:5837-6061). */
int helm3d_apply_prec(helm3d_ctx *ctx, const double *x, double *y);

/* y = M^{-H} x (mode N): the conjugate transpose of the preconditioner, used
 * by the adjoint solve.  No counterpart in the reference, which has no
 * adjoint. */
int helm3d_apply_prec_adjoint(helm3d_ctx *ctx, const double *x, double *y);

/* y_r = M^{-1} x_r (adjoint != 0: M^{-H} x_r, mode N) for nrhs <= 16
 * vectors stored one after another (nrhs * nx*ny*nz complex each, host or
 * device pointers), as one batched preconditioner apply: each factor block
 * read from memory serves every vector.  Batched form of
 * Solve3DSparseUsingFT_CSR (Source/functions.cpp:5837-6061), which the
 * reference applies to one vector at a time. */
int helm3d_apply_prec_batch(helm3d_ctx *ctx, const double *x, double *y, int nrhs, int adjoint);

/* The same y = M^{-1} x for callers that cannot allocate device memory at
 * the point of use (inside an allocator or pool callback, with free memory
 * held by a caching allocator, or on a path that must avoid cudaMalloc's
 * device synchronization).  It allocates nothing: x and y must be device
 * pointers on the context's device, and the spectral planes use an 8 MiB
 * static device array of the library (nx*ny*nz*8 bytes for C64, *16 for
 * C128 must fit, else HELM3D_ERR_ARG).  The first call on a device looks the
 * array up and should come before any stream capture; the address is kept
 * for the process, so after cudaDeviceReset the call must not be used on
 * that device until the process restarts.  Calls that overlap on the GPU
 * race on the array.  No counterpart in the reference, which has no device
 * code. */
int helm3d_apply_prec_noalloc(helm3d_ctx *ctx, const double *x, double *y);

/* Gradient of J = 0.5 sum_s ||P u_s - d_s||^2 with respect to s2 (mode N),
 * where A u_s = f_s and P samples u at the nrecv grid indices recv (the same
 * for every source; repeats allowed): forward solves, adjoint solves
 * A^H lam_s = P^T (d_s - P u_s), then grad = sum_s Re(conj(lam_s) omega^2
 * (1 + i beta_phys) u_s), all batched over sources.  f: nsrc vectors, data:
 * nsrc*nrecv complex, grad: N doubles (overwritten), each host or device;
 * misfit: host (may be NULL).  No counterpart in the reference. */
int helm3d_misfit_grad(helm3d_ctx *ctx, const double *f, int nsrc, const long long *recv, int nrecv,
                       const double *data, double *grad, double *misfit, helm3d_stats *stats);

/* Order the context's work on a caller stream (cudaStream_t; NULL restores
 * the context's own stream). */
int helm3d_set_stream(helm3d_ctx *ctx, void *stream);

/* Kernel families timed by the optional profiler. */
typedef enum helm3d_kernel_kind {
    HELM3D_K_FACTOR = 0,   /* block LU factor */
    HELM3D_K_FFT_FWD = 1,  /* forward z-FFT */
    HELM3D_K_SWEEP = 2,    /* block sweep */
    HELM3D_K_FFT_INV = 3,  /* inverse z-FFT (+ mode R epilogue) */
    HELM3D_K_STENCIL = 4,  /* 7-point operator */
    HELM3D_K_KRYLOV = 5,   /* dots, updates, norms, combine */
    HELM3D_K_COUNT = 6
} helm3d_kernel_kind;

/* enable = 1: record CUDA events around every launch on the launching
 * stream; helm3d_profile_read returns the summed device time (ms) and launch
 * count per kind, and clears them. */
int helm3d_profile(helm3d_ctx *ctx, int enable);
int helm3d_profile_read(helm3d_ctx *ctx, double *ms, long long *launches, int nkinds);

/* Bytes of device memory held by the context. */
size_t helm3d_device_bytes(const helm3d_ctx *ctx);

/* Kernels launched by this context since creation (all entry points). */
long long helm3d_kernel_launches(const helm3d_ctx *ctx);

const char *helm3d_status_string(int status);
const char *helm3d_last_error(const helm3d_ctx *ctx);

int helm3d_destroy(helm3d_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* HELM3D_H */
