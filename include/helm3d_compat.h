/*
 * helm3d_compat.h -- the reference's solver entry points, served by helm3d.
 *
 * Declares FGMRES and BCGSTAB with exactly the reference's prototypes
 * (Source/templates.h:59-60) and its grid/point types (size_m, point:
 * Source/definitions.h:55-75; dtype = std::complex<double>,
 * Source/definitions.h:10).  The types are declared in the global namespace
 * with the reference's names and layouts, so the C++ symbols of
 * libhelm3d.so are the ones the reference's main (Source/main.cpp:470-471)
 * links against: build the reference without Source/FGMRES.cpp and
 * Source/BcGSTAB.cpp and link libhelm3d.so instead.  A translation unit that
 * already has the reference's definitions.h defines HELM3D_COMPAT_NO_TYPES
 * before including this header.
 *
 * Semantics follow the reference's defaults (definitions.h): HOMO media with
 * c_z = 1280 m/s unless helm3d_compat_set_linear_media(1) selects the linear
 * model c = c1 x + c2 y + c3 (Source/functions.cpp:1362-1456); nu = 4 Hz; the
 * L0 shift kk^2 (1 + i beta_eq) with kk = omega / c_z under HOMO; the exit at a
 * relative residual of REL_RES_EXIT = 1e-4 (here measured over the whole grid,
 * which bounds the reference's physical-domain residual from above).
 * Errors are printed to stderr and leave x_sol as it was, as the reference
 * prints PARDISO errors and carries on.
 */
#ifndef HELM3D_COMPAT_H
#define HELM3D_COMPAT_H

#include <complex>

#ifndef HELM3D_COMPAT_NO_TYPES
typedef std::complex<double> dtype;

struct size_m {
    double l;
    int n;
    double h;
    int pml_pts;
    int spg_pts;
    int n_nopml;
    double ta;
    double tc;
    double td;
    double c0, c1, c2, c3;
};

struct point {
    double x;
    double y;
    double z;
};
#endif

/* FGMRES (Source/FGMRES.cpp:6-725; Source/templates.h:59): restarted GMRES
 * with m iterations per cycle and `rest` cycles on (I - dL L0^{-1}) w = f,
 * then x_sol = L0^{-1} w.  x_orig (the HOMO analytic solution) is not used;
 * diff_sol receives the final relative residual over the physical domain. */
void FGMRES(size_m x, size_m y, size_m z, int m, int rest, const point source, dtype *x_sol, dtype *x_orig,
            const dtype *f, double thresh, double &diff_sol, double beta_eq);

/* BCGSTAB (Source/BcGSTAB.cpp:6-666; Source/templates.h:60): BiCGStab on the
 * same operator, shadow residual 2 r0, the iterate kept in u-space, up to m
 * iterations, exit when the absolute residual over the physical domain drops
 * below RES_EXIT = 1e-8 (Source/BcGSTAB.cpp:503-505, 564).  L0 is the 5-point
 * operator: the reference assembles BCGSTAB's 2D systems with its 9-point
 * routine, whose coefficients (a = c = 1, d = 0) make the four diagonal-
 * neighbour entries exactly zero (Source/functions.cpp:2497-2512, 3557-3559).
 * With the HOMO medium (the default) the source cross of x_sol and of x_orig
 * (when not NULL) is zeroed as the reference does (Source/BcGSTAB.cpp:532-533).
 * diff_sol receives the final relative residual over the physical domain. */
void BCGSTAB(size_m x, size_m y, size_m z, int m, const point source, dtype *x_sol, dtype *x_orig, const dtype *f,
             double thresh, double &diff_sol, double beta_eq);

extern "C" {
/* 1: the linear velocity model of SetSoundSpeed3D; 0 (default): HOMO. */
void helm3d_compat_set_linear_media(int on);
/* CUDA device used by FGMRES/BCGSTAB (default 0). */
void helm3d_compat_set_device(int device);
}

#endif /* HELM3D_COMPAT_H */
