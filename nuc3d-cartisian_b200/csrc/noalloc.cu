// Allocation-free CRWENO5 reconstruction (nuc3d_reconstruct_crweno5_noalloc).
//
// nuc3d_reconstruct with scheme CRWENO5 needs scratch for the Thomas sweep
// (2 * nx * ny * nz doubles) and obtains it with cudaMallocAsync.  Some
// callers cannot let a library allocate device memory: a host code that
// reserves all device memory for its own pool at start-up, or a solver
// plug-in invoked where the host application forbids allocation.  For them
// this entry point runs the same line-solve kernel on a fixed scratch array
// that lives in the library's own device image.
//
// Limits and behaviour:
//  * the scratch is kNoAllocScratchDoubles doubles (4 MiB); every GPU that
//    loads the library holds it until the process exits.  Calls needing
//    more than 2 * nx * ny * nz > kNoAllocScratchDoubles are rejected with
//    NUC3D_ERR_INVALID.
//  * the array's host-side name is not a device address.  Every call looks
//    up the array's address on the current device with
//    cudaGetSymbolAddress (a host-side lookup that allocates nothing) and
//    checks the result, so a cudaDeviceReset or a re-created primary context
//    in the same process never leaves a stale address behind.  The first
//    call on a device also loads the library's device code there; make that
//    first call before any stream capture.
//  * the same argument rules as nuc3d_reconstruct(NUC3D_CRWENO5, ...),
//    nx <= 4096 included.
//  * all calls share one array per device and it keeps the last call's
//    contents.  Nothing in it has to start at zero: the kernel writes every
//    entry it reads before reading it.  Calls whose executions overlap on
//    the GPU (different streams, or different host threads) race on the
//    array; serialise them.
//  * no cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include "nuc3d_b200.h"
#include "op_kernels.h"

namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(1) << 19;  // 4 MiB of FP64
__device__ __align__(256) double g_crweno_scratch[kNoAllocScratchDoubles];

}  // namespace

extern "C" NUC3D_API int nuc3d_reconstruct_crweno5_noalloc(int upwind, int nx, int ny, int nz,
                                                           const double *d_in,
                                                           const double *d_halo_l,
                                                           const double *d_halo_r,
                                                           double *d_out, void *stream) {
    using nuc3d::set_last_error;
    if (upwind != 1 && upwind != -1)
        return set_last_error(NUC3D_ERR_INVALID, "weno error: no such direction");
    if (nx < 8 || ny < 1 || nz < 1)
        return set_last_error(NUC3D_ERR_INVALID, "need nx >= 8, ny, nz >= 1");
    if (nx > 4096) return set_last_error(NUC3D_ERR_INVALID, "crweno5 / hccs need nx <= 4096");
    if (!d_in || !d_halo_l || !d_halo_r || !d_out)
        return set_last_error(NUC3D_ERR_INVALID, "null buffer");
    const long long lines = (long long)ny * nz;
    const long long need = 2LL * nx * lines;
    if (need > (long long)kNoAllocScratchDoubles)
        return set_last_error(NUC3D_ERR_INVALID,
                              "crweno5 no-alloc: 2*nx*ny*nz exceeds the 524288-double "
                              "(4 MiB) static scratch; use nuc3d_reconstruct");
    // the device address of the array in the current context (never cached:
    // a reset device reloads the module and the array may move)
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_crweno_scratch);
    if (e != cudaSuccess || !p)
        return set_last_error(NUC3D_ERR_CUDA, e != cudaSuccess
                                                  ? cudaGetErrorString(e)
                                                  : "crweno5 no-alloc: no scratch address");
    double *const scratch = static_cast<double *>(p);
    e = nuc3d::op_crweno_into(upwind, nx, lines, d_in, d_halo_l, d_halo_r, d_out, scratch,
                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return set_last_error(NUC3D_ERR_CUDA, cudaGetErrorString(e));
    return NUC3D_OK;
}
