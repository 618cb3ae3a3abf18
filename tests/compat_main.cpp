// compat_main.cpp -- calls FGMRES or BCGSTAB through include/helm3d_compat.h
// the way the reference's main does (Source/main.cpp:95-193, 470-471): grid
// from n_nopml / pml / spg without SOURCE_SHIFT, niter, restart, beta_eq.  The
// right-hand side is read from f.bin, the solution written to x_sol.bin.
//   compat_main fgmres  <n_nopml> <pml> <spg> <beta> <niter> <restart> <dir>
//   compat_main bcgstab <n_nopml> <pml> <spg> <beta> <niter> <dir>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "helm3d_compat.h"

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    const std::string solver = argv[1];
    const bool bcg = solver == "bcgstab";
    if (argc != (bcg ? 8 : 9)) return 2;
    const int n_nopml = atoi(argv[2]), pml = atoi(argv[3]), spg = atoi(argv[4]);
    const double beta = atof(argv[5]);
    const int niter = atoi(argv[6]), restart = bcg ? 1 : atoi(argv[7]);
    const std::string dir = argv[bcg ? 7 : 8];
    const double L = 3200.0;  // LENGTH (Source/definitions.h:222)
    size_m x, y, z;
    memset(&x, 0, sizeof(x));
    memset(&y, 0, sizeof(y));
    memset(&z, 0, sizeof(z));
    x.pml_pts = y.pml_pts = pml;
    z.pml_pts = 0;
    z.spg_pts = spg;
    x.n = y.n = n_nopml + 2 * pml;
    z.n = n_nopml + 2 * spg;
    x.n_nopml = y.n_nopml = n_nopml;
    z.n_nopml = n_nopml;
    x.l = y.l = L + (double)(2 * pml * L) / n_nopml;
    z.l = L + (double)(2 * spg * L) / n_nopml;
    x.h = x.l / x.n;
    y.h = y.l / y.n;
    z.h = z.l / z.n;
    point source = {x.l / 2, y.l / 2, z.l / 2};
    const size_t size = (size_t)x.n * y.n * z.n;
    std::vector<dtype> f(size), x_sol(size), x_orig(size);
    FILE *fh = fopen((dir + "/f.bin").c_str(), "rb");
    if (!fh || fread(f.data(), sizeof(dtype), size, fh) != size) return 3;
    fclose(fh);
    double diff_sol = 0;
    if (bcg) BCGSTAB(x, y, z, niter, source, x_sol.data(), x_orig.data(), f.data(), 1e-4, diff_sol, beta);
    else FGMRES(x, y, z, niter, restart, source, x_sol.data(), x_orig.data(), f.data(), 1e-4, diff_sol, beta);
    fh = fopen((dir + "/x_sol.bin").c_str(), "wb");
    fwrite(x_sol.data(), sizeof(dtype), size, fh);
    fclose(fh);
    printf("diff_sol %e\n", diff_sol);
    return 0;
}
