// compat.cpp -- FGMRES / BCGSTAB with the reference's prototypes
// (include/helm3d_compat.h), built on the C ABI in mode R.
//
// The set-up mirrors FGMRES's own (Source/FGMRES.cpp:72-93): the medium is
// built from the grid as SetSoundSpeed3D + HeteroSoundSpeed3DExtensionToPML
// do (Source/functions.cpp:1362-1456, 2675-2716), then c0, dL and the per-kz
// shifts are derived by helm3d_create in mode R (q1 running mean, reference
// kz table, HOMO's kk for L0).
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/helm3d.h"
#include "../../include/helm3d_compat.h"

namespace {

const double kPi = 3.141592653589793238462643;
const double kNu = 4.0;       // nu (Source/definitions.h:251)
const double kCz = 1280.0;    // c_z (Source/definitions.h:252)
int g_linear = 0;
int g_device = 0;

// SetSoundSpeed3D + the x,y edge extension, as squared slowness 1/c^2
std::vector<double> reference_s2(const size_m &x, const size_m &y, const size_m &z) {
    const int nx = x.n, ny = y.n, nz = z.n;
    const int px = x.pml_pts, py = y.pml_pts;
    std::vector<double> c((size_t)nx * ny * nz, 0.0);
    const double c3 = 600.0, c2 = (1500.0 - c3) / y.l, c1 = (1800.0 - c3 - c2 * y.l) / x.l;
    for (int k = 0; k < nz; k++)
        for (int j = py; j < ny - py; j++)
            for (int i = px; i < nx - px; i++) {
                double v = kCz;
                if (g_linear) v = c1 * ((double)i + 1 - px) * x.h + c2 * ((double)j + 1 - py) * y.h + c3;
                c[((size_t)k * ny + j) * nx + i] = v;
            }
    for (int k = 0; k < nz; k++) {
        double *p = &c[(size_t)k * ny * nx];
        for (int j = 0; j < ny; j++) {
            for (int i = 0; i < px; i++) p[(size_t)j * nx + i] = p[(size_t)j * nx + px];
            for (int i = nx - px; i < nx; i++) p[(size_t)j * nx + i] = p[(size_t)j * nx + nx - px - 1];
        }
        for (int i = 0; i < nx; i++) {
            for (int j = 0; j < py; j++) p[(size_t)j * nx + i] = p[(size_t)py * nx + i];
            for (int j = ny - py; j < ny; j++) p[(size_t)j * nx + i] = p[(size_t)(ny - py - 1) * nx + i];
        }
    }
    std::vector<double> s2(c.size());
    for (size_t q = 0; q < c.size(); q++) s2[q] = 1.0 / (c[q] * c[q]);
    return s2;
}

helm3d_ctx *make_ctx(const size_m &x, const size_m &y, const size_m &z, int restart, int max_iter, double tol,
                     double beta_eq, int stop_phys = 0) {
    helm3d_grid g;
    g.nx = x.n;
    g.ny = y.n;
    g.nz = z.n;
    g.hx = x.h;
    g.hy = y.h;
    g.hz = z.h;
    g.pml_x = x.pml_pts;
    g.pml_y = y.pml_pts;
    g.pml_z = 0;
    g.spg_z = z.spg_pts;
    g.lz = z.l;
    g.omega = 2.0 * kPi * kNu;
    helm3d_opts o;
    helm3d_default_opts(&o);
    o.mode = HELM3D_MODE_R;
    o.precision = HELM3D_PREC_C128;
    o.kz_symbol = HELM3D_KZ_REFERENCE;
    o.beta_prec = beta_eq;
    o.s2_l0 = g_linear ? 0.0 : 1.0 / (kCz * kCz);
    o.quirk_q1 = 1;
    o.restart = restart;
    o.max_iter = max_iter;
    o.tol = tol;
    o.stop_phys = stop_phys;
    o.device = g_device;
    const std::vector<double> s2 = reference_s2(x, y, z);
    helm3d_ctx *ctx = nullptr;
    const int rc = helm3d_create(&g, s2.data(), &o, &ctx);
    if (rc != HELM3D_OK) {
        fprintf(stderr, "!!! helm3d set-up failed: %s (%s) !!!\n", helm3d_status_string(rc), helm3d_last_error(nullptr));
        return nullptr;
    }
    return ctx;
}

// NullifySource2D(x, y, u + plane z.n/2, size2D/2, 1) (Source/functions.cpp:
// 6628-6644): zeroes the points l = 0, 1 to the left, right, below and above
// index size2D/2 of the middle z plane, with the reference's flat indexing
// (for even x.n the "left" point is the last one of the row below)
void nullify_source_cross(const size_m &x, const size_m &y, const size_m &z, dtype *u) {
    const long size2D = (long)x.n * y.n;
    dtype *plane = u + (long)(z.n / 2) * size2D;
    const long src = size2D / 2, jsrc = src / x.n, isrc = src - (long)x.n * jsrc;
    for (long l = 0; l <= 1; l++) {
        plane[isrc - l + x.n * jsrc] = 0.0;
        plane[isrc + l + x.n * jsrc] = 0.0;
        plane[isrc + x.n * (jsrc - l)] = 0.0;
        plane[isrc + x.n * (jsrc + l)] = 0.0;
    }
}

}  // namespace

extern "C" void helm3d_compat_set_linear_media(int on) { g_linear = on ? 1 : 0; }
extern "C" void helm3d_compat_set_device(int device) { g_device = device; }

void FGMRES(size_m x, size_m y, size_m z, int m, int rest, const point source, dtype *x_sol, dtype *x_orig,
            const dtype *f, double thresh, double &diff_sol, double beta_eq) {
    (void)source;
    (void)x_orig;
    (void)thresh;
    helm3d_ctx *ctx = make_ctx(x, y, z, m > 0 ? m : 1, (m > 0 ? m : 1) * (rest > 0 ? rest : 1), 1e-4, beta_eq);
    if (!ctx) return;
    helm3d_stats st = {};
    const int rc = helm3d_solve(ctx, reinterpret_cast<const double *>(f), reinterpret_cast<double *>(x_sol), 1, &st);
    if (rc != HELM3D_OK && rc != HELM3D_ERR_NOT_CONVERGED)
        fprintf(stderr, "!!! helm3d FGMRES failed: %s (%s) !!!\n", helm3d_status_string(rc), helm3d_last_error(ctx));
    printf("helm3d FGMRES: %d iterations, relative residual %e (physical domain %e)\n", st.iterations, st.relres,
           st.relres_phys);
    diff_sol = st.relres_phys;
    helm3d_destroy(ctx);
}

void BCGSTAB(size_m x, size_m y, size_m z, int m, const point source, dtype *x_sol, dtype *x_orig, const dtype *f,
             double thresh, double &diff_sol, double beta_eq) {
    (void)source;
    (void)x_orig;
    (void)thresh;
    const size_t n = (size_t)x.n * y.n * z.n;
    double nf = 0.0;
    for (size_t q = 0; q < n; q++) nf += std::norm(f[q]);
    nf = std::sqrt(nf);
    // RES_EXIT = 1e-8 on the absolute residual of the physical domain
    // (Source/BcGSTAB.cpp:503-505, 564), at most m iterations
    const double tol = nf > 0 ? 1e-8 / nf : 0.0;
    helm3d_ctx *ctx = make_ctx(x, y, z, 1, m > 0 ? m : 1, tol, beta_eq, 1);
    if (!ctx) return;
    helm3d_stats st = {};
    const int rc = helm3d_solve_bicgstab(ctx, reinterpret_cast<const double *>(f), reinterpret_cast<double *>(x_sol),
                                         &st);
    if (rc != HELM3D_OK && rc != HELM3D_ERR_NOT_CONVERGED)
        fprintf(stderr, "!!! helm3d BCGSTAB failed: %s (%s) !!!\n", helm3d_status_string(rc), helm3d_last_error(ctx));
    printf("helm3d BCGSTAB: %d iterations, relative residual %e (physical domain %e)\n", st.iterations, st.relres,
           st.relres_phys);
    diff_sol = st.relres_phys;
    helm3d_destroy(ctx);
    // the HOMO build zeroes the source cross of its solution and of x_orig
    // (Source/BcGSTAB.cpp:532-533)
    if (!g_linear) {
        nullify_source_cross(x, y, z, x_sol);
        if (x_orig) nullify_source_cross(x, y, z, x_orig);
    }
}
