// compat_fgmres_main.cpp -- calls FGMRES through include/helm3d_compat.h the
// way the reference's main does (Source/main.cpp:95-193, 470): grid from
// n_nopml / pml / spg without SOURCE_SHIFT, niter, restart, beta_eq.  The
// right-hand side is read from f.bin, the solution written to x_sol.bin.
//   compat_fgmres_main <n_nopml> <pml> <spg> <beta> <niter> <restart> <dir>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "helm3d_compat.h"

int main(int argc, char **argv) {
    if (argc != 8) return 2;
    const int n_nopml = atoi(argv[1]), pml = atoi(argv[2]), spg = atoi(argv[3]);
    const double beta = atof(argv[4]);
    const int niter = atoi(argv[5]), restart = atoi(argv[6]);
    const std::string dir = argv[7];
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
    FGMRES(x, y, z, niter, restart, source, x_sol.data(), x_orig.data(), f.data(), 1e-4, diff_sol, beta);
    fh = fopen((dir + "/x_sol.bin").c_str(), "wb");
    fwrite(x_sol.data(), sizeof(dtype), size, fh);
    fclose(fh);
    printf("diff_sol %e\n", diff_sol);
    return 0;
}
