// noalloc.cu -- helm3d_apply_prec_noalloc: the preconditioner apply
// (forward z-FFT, per-kz block sweep, inverse z-FFT) with its scratch, the
// spectral planes, in a fixed device array of this library instead of memory
// the call allocates.
//
// Some callers cannot call cudaMalloc where they apply the preconditioner:
// code that runs inside a device-memory allocator or pool callback (it must
// not re-enter the allocator), processes whose free device memory is already
// reserved by a framework's caching allocator, and latency-bound loops that
// must stay off the driver's allocation path (cudaMalloc can synchronize the
// device).  This entry point allocates nothing: the caller passes device
// input and output vectors, the factor and tables were allocated when the
// context was created, and the planes live in kScratchBytes (8 MiB) of static
// device memory that every GPU which loads the library holds until the
// process exits.  Grids whose planes need more (nx*ny*nz*8 bytes for the
// complex64 preconditioner, *16 for complex128) are rejected.
//
// The array name is only a host-side stand-in for the device symbol: the
// device address is looked up once per device with cudaGetSymbolAddress (on
// the first call on that device, with the device current), cached, and
// passed to the kernels.  That first call should therefore come before any
// stream capture.  All calls share the array and it keeps the last call's
// contents; every call overwrites all planes it reads, so nothing needs
// clearing.  Calls whose work overlaps on the GPU (different streams or
// contexts at the same time) race on the array.  The address is cached per
// device ordinal for the life of the process: after cudaDeviceReset (or
// anything else that re-creates the device's primary context) the cached
// address is stale, and this entry point must not be used on that device
// until the process restarts.
#include <cuda_runtime.h>

#include <mutex>

#include "helm3d_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_plane_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" int helm3d_apply_prec_noalloc(helm3d_ctx *c, const double *x, double *y) {
    using namespace h3d;
    if (!c || !x || !y) return HELM3D_ERR_ARG;
    if (c->device < 0 || c->device >= kMaxDevices) return set_error(c, HELM3D_ERR_ARG, "device ordinal too large");
    int rc = cuda_check(c, cudaSetDevice(c->device), "set device");
    if (rc) return rc;
    const size_t need = (size_t)c->N * (c->c64 ? 8 : 16);
    if (need > kScratchBytes)
        return set_error(c, HELM3D_ERR_ARG,
                         "apply_prec_noalloc: nx*ny*nz*" + std::to_string(c->c64 ? 8 : 16) + " = " +
                             std::to_string(need) + " bytes of planes exceed the 8 MiB static scratch");
    for (const void *p : {(const void *)x, (const void *)y}) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, HELM3D_ERR_ARG, "apply_prec_noalloc takes device pointers only");
        }
        if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
            return set_error(c, HELM3D_ERR_ARG, "apply_prec_noalloc takes device pointers only");
        if (at.type == cudaMemoryTypeDevice && at.device != c->device)
            return set_error(c, HELM3D_ERR_ARG, "apply_prec_noalloc: x and y must be on the context's device");
    }
    if ((rc = begin_call(c))) return rc;
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[c->device]) {
            void *p = nullptr;
            rc = cuda_check(c, cudaGetSymbolAddress(&p, g_plane_scratch), "cudaGetSymbolAddress(scratch)");
            if (rc) return rc;
            g_scratch_addr[c->device] = p;
        }
        scratch = g_scratch_addr[c->device];
    }
    const VecBatch xb{(double2 *)x, 0}, yb{(double2 *)y, 0};
    const ScaleBatch one{nullptr, 0};
    const PlaneLayout L{c->grid.nx, c->grid.ny, c->grid.nz, 1, c->plane};
    rc = c->ztc    ? launch_ztc_forward(xb, 1.0, one, scratch, L, c->d_ztc[0], c->d_status, c->stream)
         : c->zeig ? launch_ztrans_forward(c->c64, xb, 1.0, one, scratch, L, c->d_zWi64, c->stream)
                   : launch_fft_forward(c->c64, xb, 1.0, one, scratch, L, c->plan, c->d_tw, c->stream);
    if (rc) return set_error(c, rc, "apply_prec_noalloc: forward FFT launch");
    SweepArgs s;
    s.n = c->grid.nx;
    s.ny = c->grid.ny;
    s.nz = c->grid.nz;
    s.ldg = c->ldg;
    s.Gt = c->d_Gt;
    s.cmy = c->d_cmy;
    s.cpy = c->d_cpy;
    s.planes = scratch;
    s.R = 1;
    s.dxy = nullptr;
    s.status = c->d_status;
    if (c->nskip > 0) {
        s.kzslot = c->d_kzslot;
        s.kzlist = c->d_kzlist;
        s.nskip = c->nskip;
        s.kzinv = c->d_kzinv;
    }
    rc = launch_sweep(c->c64, s, c->stream);
    if (rc) return set_error(c, rc, "apply_prec_noalloc: sweep launch");
    rc = c->ztc    ? launch_ztc_inverse(scratch, L, yb, c->d_ztc[1], c->d_status, c->stream)
         : c->zeig ? launch_ztrans_inverse(c->c64, scratch, L, yb, c->d_zW64, c->stream)
                   : launch_fft_inverse(c->c64, scratch, L, yb, c->plan, c->d_tw, 0, VecBatch{nullptr, 0}, 0.0, one,
                                      nullptr, c->stream);
    if (rc) return set_error(c, rc, "apply_prec_noalloc: inverse FFT launch");
    c->launches += 3;
    // a bounded wait that expired in the sweep or a tensor-core z-transform
    // leaves y invalid and sets a status bit: reported, not returned as OK
    return check_status(c);
}
