// hlld_rk_step_ct_static: the 2D RK + CT step with its scratch memory in a
// fixed device array that is part of the library, for callers that cannot
// allocate device memory themselves.
//
// Who cannot allocate: hosts whose device memory belongs to a pool or
// allocator they do not control (a framework's caching allocator, a
// fixed-budget embedded runtime), plugin hosts that hand a solver only its
// input and output arrays, and time-step loops that cannot afford the
// device-wide synchronisation a cudaMalloc or cudaFree may cause.  For them
// the scratch (face fluxes, corner EMF, the RK stage-0 copy, counters and,
// in the mixed form, the C2P roots of the first stage) lives in
// g_step_scratch below.
//
// Limits and rules:
//   - the array holds kStaticScratchBytes (64 MiB); hlld_step2d_scratch_bytes
//     says what a grid needs; with ng = 2 that is square grids up to
//     599 x 599 cells in FP64, 708 x 708 in the mixed form and 849 x 849 in
//     FP32; larger grids get HLLD_ERR_SCRATCH;
//   - every GPU that loads the library keeps the 64 MiB until the process
//     exits;
//   - all calls share the one array per device, so calls whose work overlaps
//     on the GPU (two streams, two host threads) race: serialise them on one
//     stream.  The step itself overwrites or zeroes everything it reads from
//     the array before reading it, so leftover contents of an earlier call are
//     harmless;
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it.
#include <cstdio>
#include <mutex>

#include "variants.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 128;

// The scratch.  In host code this name is a host-side stand-in, not a device
// address: only the pointer from cudaGetSymbolAddress may be passed to a kernel.
static __device__ __align__(256) unsigned char g_step_scratch[kStaticScratchBytes];

std::mutex g_mu;
void *g_dev_ptr[kMaxDevices] = {};

int scratch_for_current_device(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return hlld::report_error(HLLD_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return hlld::report_error(HLLD_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_step_scratch);
        if (e != cudaSuccess || !p)
            return hlld::report_error(HLLD_ERR_CUDA, "cudaGetSymbolAddress(g_step_scratch): %s",
                                      cudaGetErrorString(e));
        g_dev_ptr[dev] = p;
    }
    *out = g_dev_ptr[dev];
    return HLLD_OK;
}

}  // namespace

extern "C" {

int hlld_rk_step_ct_static(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt_host,
                           const double *dt_dev, int scheme, hlld_step_diag_t *diag,
                           void *stream) {
    size_t need = 0;
    int rc = hlld_step2d_scratch_bytes(g, &need);
    if (rc != HLLD_OK) return rc;
    if (need > kStaticScratchBytes)
        return hlld::report_error(HLLD_ERR_SCRATCH,
                                  "grid needs %zu bytes of scratch, the static array holds %zu: "
                                  "use hlld_rk_step_ct with caller-allocated scratch",
                                  need, kStaticScratchBytes);
    void *scratch = nullptr;
    if ((rc = scratch_for_current_device(&scratch)) != HLLD_OK) return rc;
    return hlld_rk_step_ct(g, s, scratch, kStaticScratchBytes, dt_host, dt_dev, scheme, diag,
                           stream);
}

}  // extern "C"
