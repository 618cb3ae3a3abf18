// ref_driver.cpp -- runs the reference's own FGMRES path on a small grid and
// dumps what it computed, so the NumPy oracle can be checked against the
// reference itself (test infrastructure; built by oracle/Makefile into
// oracle/_ref/ref_driver with the MKL stand-in).
//
//   ref_driver setup  <n_nopml> <pml> <spg> <beta> <outdir>
//       calls SetSoundSpeed3D, HeteroSoundSpeed3DExtensionToPML,
//       SetSoundSpeed2D, HeteroSoundSpeed2DExtensionToPML, GenerateDeltaL and
//       GenSparseMatrixOnline2DwithPMLFast(-1, ...) exactly as FGMRES does
//       (Source/FGMRES.cpp:79-151) and writes sound2D, deltaL and the CSR
//       values of the base 2D matrix.
//   ref_driver fgmres <n_nopml> <pml> <spg> <beta> <niter> <restart> <outdir>
//       builds the grid as main does (Source/main.cpp:95-193, no
//       SOURCE_SHIFT), the RHS with GenRHSandSolutionViaSound3D
//       (Source/main.cpp:418) and calls FGMRES (Source/main.cpp:470); writes
//       f and x_sol.  FGMRES itself writes its convergence_*.dat file into
//       the working directory.
//   ref_driver bcgstab <n_nopml> <pml> <spg> <beta> <niter> <fscale> <outdir>
//       the same grid and RHS scaled by fscale (BCGSTAB stops on an absolute
//       residual, RES_EXIT = 1e-8, so the scale sets how many iterations it
//       runs), then BCGSTAB (Source/BcGSTAB.cpp:6-666, the call main has
//       commented out at Source/main.cpp:471); writes f and x_sol, and
//       BCGSTAB writes its convergence_*_BCGSTAB.dat file.
//   ref_driver setup9 <n_nopml> <pml> <spg> <outdir>
//       the base 2D matrix of BCGSTAB, GenSparseMatrixOnline2DwithPMLand9Pts
//       (-1, ...) (Source/BcGSTAB.cpp:143, Source/functions.cpp:3532-3679):
//       CSR values / ia / ja and the diagonal positions freqs.
//
// The reference is compiled with its own definitions.h, i.e. HOMO mode,
// nu = 4 Hz, c_z = 1280 m/s, LENGTH = 3200 m, REL_RES_EXIT = 1e-4.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "templates.h"

static void write_bin(const std::string &path, const void *p, size_t bytes) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) { perror(path.c_str()); exit(2); }
    fwrite(p, 1, bytes, f);
    fclose(f);
}

static void make_grid(int n_nopml, int pml, int spg, size_m &x, size_m &y, size_m &z) {
    memset(&x, 0, sizeof(x));
    memset(&y, 0, sizeof(y));
    memset(&z, 0, sizeof(z));
    x.pml_pts = y.pml_pts = pml;
    z.pml_pts = 0;
    z.spg_pts = spg;
    x.n = n_nopml + 2 * pml;
    y.n = n_nopml + 2 * pml;
    z.n = n_nopml + 2 * spg;
    x.n_nopml = x.n - 2 * x.pml_pts;
    y.n_nopml = y.n - 2 * y.pml_pts;
    z.n_nopml = z.n - 2 * z.spg_pts;
    x.l = LENGTH_X + (double)(2 * x.pml_pts * LENGTH_X) / (x.n_nopml);
    y.l = LENGTH_Y + (double)(2 * y.pml_pts * LENGTH_Y) / (y.n_nopml);
    z.l = LENGTH_Z + (double)(2 * z.spg_pts * LENGTH_Z) / (z.n_nopml);
    x.h = x.l / (x.n);
    y.h = y.l / (y.n);
    z.h = z.l / (z.n);
}

static point make_source(const size_m &x, const size_m &y, const size_m &z) {
    double xc = x.l, yc = y.l, zc = z.l;
    if (x.n % 2 != 0) xc += x.h;
    if (y.n % 2 != 0) yc += y.h;
    if (z.n % 2 != 0) zc += z.h;
    point source = {xc / 2.0, yc / 2.0, zc / 2.0};
    return source;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: ref_driver setup|fgmres ...\n");
        return 1;
    }
    const std::string mode = argv[1];
    if (mode == "setup" && argc == 7) {
        int n_nopml = atoi(argv[2]), pml = atoi(argv[3]), spg = atoi(argv[4]);
        double beta = atof(argv[5]);
        std::string out = argv[6];
        size_m x, y, z;
        make_grid(n_nopml, pml, spg, x, y, z);
        point source = make_source(x, y, z);
        int size = x.n * y.n * z.n, size2D = x.n * y.n;
        dtype *sound3D = alloc_arr<dtype>(size);
        dtype *sound2D = alloc_arr<dtype>(size2D);
        dtype *deltaL = alloc_arr<dtype>(size);
        SetSoundSpeed3D(x, y, z, sound3D, source);
        HeteroSoundSpeed3DExtensionToPML(x, y, z, sound3D);
        SetSoundSpeed2D(x, y, z, sound3D, sound2D, source);
        HeteroSoundSpeed2DExtensionToPML(x, y, sound2D);
        GenerateDeltaL(x, y, z, sound3D, sound2D, deltaL, beta);
        size_t nnz = ((size_t)x.n + (x.n - 1) * 2) * y.n + 2 * (size2D - x.n);
        zcsr *A = (zcsr *)malloc(sizeof(zcsr));
        A->values = alloc_arr<dtype>(nnz);
        A->ia = alloc_arr<int>((size_t)size2D + 1);
        A->ja = alloc_arr<int>(nnz);
        A->ia[size2D] = (int)nnz + 1;
        A->non_zeros = (int)nnz;
        int *freqs = alloc_arr<int>(size);
        GenSparseMatrixOnline2DwithPMLFast(-1, x, y, A, 0, freqs);
        write_bin(out + "/sound2D.bin", sound2D, sizeof(dtype) * size2D);
        write_bin(out + "/deltaL.bin", deltaL, sizeof(dtype) * size);
        write_bin(out + "/csr_values.bin", A->values, sizeof(dtype) * nnz);
        write_bin(out + "/csr_ia.bin", A->ia, sizeof(int) * (size2D + 1));
        write_bin(out + "/csr_ja.bin", A->ja, sizeof(int) * nnz);
        printf("setup done: nx=%d nz=%d hx=%.17g hz=%.17g nnz=%zu\n", x.n, z.n, x.h, z.h, nnz);
        return 0;
    }
    if (mode == "fgmres" && argc == 9) {
        int n_nopml = atoi(argv[2]), pml = atoi(argv[3]), spg = atoi(argv[4]);
        double beta = atof(argv[5]);
        int niter = atoi(argv[6]), restart = atoi(argv[7]);
        std::string out = argv[8];
        size_m x, y, z;
        make_grid(n_nopml, pml, spg, x, y, z);
        point source = make_source(x, y, z);
        int size = x.n * y.n * z.n;
        dtype *x_orig = alloc_arr<dtype>(size);
        dtype *x_sol = alloc_arr<dtype>(size);
        dtype *f = alloc_arr<dtype>(size);
        GenRHSandSolutionViaSound3D(x, y, z, x_orig, f, source);
        double thresh = 1e-4, diff_sol = 0;
        FGMRES(x, y, z, niter, restart, source, x_sol, x_orig, f, thresh, diff_sol, beta);
        write_bin(out + "/f.bin", f, sizeof(dtype) * size);
        write_bin(out + "/x_sol.bin", x_sol, sizeof(dtype) * size);
        write_bin(out + "/x_orig.bin", x_orig, sizeof(dtype) * size);
        printf("fgmres done: nx=%d nz=%d\n", x.n, z.n);
        return 0;
    }
    if (mode == "bcgstab" && argc == 9) {
        int n_nopml = atoi(argv[2]), pml = atoi(argv[3]), spg = atoi(argv[4]);
        double beta = atof(argv[5]);
        int niter = atoi(argv[6]);
        double fscale = atof(argv[7]);
        std::string out = argv[8];
        size_m x, y, z;
        make_grid(n_nopml, pml, spg, x, y, z);
        point source = make_source(x, y, z);
        int size = x.n * y.n * z.n;
        dtype *x_orig = alloc_arr<dtype>(size);
        dtype *x_sol = alloc_arr<dtype>(size);
        dtype *f = alloc_arr<dtype>(size);
        GenRHSandSolutionViaSound3D(x, y, z, x_orig, f, source);
        for (int q = 0; q < size; q++) {
            f[q] *= fscale;
            x_orig[q] *= fscale;
        }
        double thresh = 1e-4, diff_sol = 0;
        BCGSTAB(x, y, z, niter, source, x_sol, x_orig, f, thresh, diff_sol, beta);
        write_bin(out + "/f.bin", f, sizeof(dtype) * size);
        write_bin(out + "/x_sol.bin", x_sol, sizeof(dtype) * size);
        printf("bcgstab done: nx=%d nz=%d\n", x.n, z.n);
        return 0;
    }
    if (mode == "setup9" && argc == 6) {
        int n_nopml = atoi(argv[2]), pml = atoi(argv[3]), spg = atoi(argv[4]);
        std::string out = argv[5];
        size_m x, y, z;
        make_grid(n_nopml, pml, spg, x, y, z);
        int size2D = x.n * y.n;
        // the count BCGSTAB allocates (Source/BcGSTAB.cpp:98)
        int nnz = (x.n + (x.n - 1) * 2) * y.n + 2 * (size2D - x.n) + 4 * (x.n - 1) * (y.n - 1);
        zcsr *A = (zcsr *)malloc(sizeof(zcsr));
        A->values = alloc_arr<dtype>(nnz);
        A->ia = alloc_arr<int>((size_t)size2D + 1);
        A->ja = alloc_arr<int>(nnz);
        A->ia[size2D] = nnz + 1;
        A->non_zeros = nnz;
        int *freqs = alloc_arr<int>(size2D);
        GenSparseMatrixOnline2DwithPMLand9Pts(-1, x, y, A, 0, freqs);
        write_bin(out + "/csr9_values.bin", A->values, sizeof(dtype) * nnz);
        write_bin(out + "/csr9_ia.bin", A->ia, sizeof(int) * (size2D + 1));
        write_bin(out + "/csr9_ja.bin", A->ja, sizeof(int) * nnz);
        write_bin(out + "/csr9_freqs.bin", freqs, sizeof(int) * size2D);
        printf("setup9 done: nx=%d nnz=%d\n", x.n, nnz);
        return 0;
    }
    fprintf(stderr, "bad arguments\n");
    return 1;
}
