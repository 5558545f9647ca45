// Allocation-free variant of the block-LU factorization entry point.
//
// Some callers cannot let a library call cudaMalloc/cudaFree: hosts whose own
// GPU memory manager owns the device heap (MATLAB's gpuArray manager, caching
// allocators of deep-learning frameworks) and may already have reserved most
// of it, and latency-critical callers for which the implicit device
// synchronization of cudaMalloc/cudaFree is not acceptable.  For them,
// wust_decomp_block_lu_noalloc runs the same factorization kernel as
// wust_decomp_block_lu, but its scratch (working page, row/column panels,
// grid-barrier word and status words) lives in one file-scope __device__
// array that is part of the loaded module: every GPU that loads the library
// holds kNoallocScratchBytes for it until the process exits.
//
// Limits and sharing rules:
//   * Ny <= WUST_NOALLOC_MAX_NY (1024); larger grids are rejected with
//     WUST_ERR_INVALID_INPUT before any device work.
//   * All calls on a device share the one array, which keeps whatever the
//     last call left in it.  The launcher clears the barrier and status words
//     at the start of every call; the working page and panels are fully
//     rewritten before they are read.  Two calls whose work overlaps on the
//     GPU (different streams, or host threads without ordering) race on the
//     array and corrupt each other's results; callers must serialize them.
//   * Every call looks up the array's device address (cudaGetSymbolAddress)
//     with the caller's device current, so a device reset between calls (a
//     host such as MATLAB can reset the GPU, which reloads the module,
//     possibly at another address) never leaves a stale pointer behind.  The
//     lookup allocates nothing, but the first one on a device may load the
//     module: make the first call on each device outside any stream capture.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int kNoallocMaxNy = WUST_NOALLOC_MAX_NY;
// Scratch of factor_launch for Ny = kNoallocMaxNy, rounded up to 256 bytes.
constexpr size_t kNoallocScratchBytes = (factor_scratch_bytes_for(kNoallocMaxNy) + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_factor_scratch[kNoallocScratchBytes];

// Device address of g_factor_scratch in the current device's context.  In
// host code the symbol names a host-side shadow, so kernels must be given
// this address, never &g_factor_scratch.
static void *noalloc_scratch_address() {
    void *ptr = nullptr;
    WUST_CUDA(cudaGetSymbolAddress(&ptr, g_factor_scratch));
    if (!ptr) fail(WUST_ERR_CUDA, "cudaGetSymbolAddress returned a null scratch address");
    return ptr;
}

static bool noalloc_device_pointer(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace wust

using namespace wust;

extern "C" int wust_decomp_block_lu_noalloc(const wust_c64 *Ld, const wust_c64 *Ll, const wust_c64 *Lu,
                                            const wust_c64 *Dd, const wust_c64 *Dl, const wust_c64 *Du,
                                            const wust_c64 *Ud, const wust_c64 *Ul, const wust_c64 *Uu, int Ny, int Nx,
                                            wust_c64 *invT, void *stream) {
    try {
        if (Ny < 3 || Nx < 2 || (long long)Ny * Nx > 2147483647LL)
            fail(WUST_ERR_INVALID_INPUT, "Block-LU grid must have an interior and fit int indexing.");
        if (Ny > kNoallocMaxNy)
            fail(WUST_ERR_INVALID_INPUT,
                 "decompBlockLU without allocation supports Ny <= %d (got %d); use wust_decomp_block_lu", kNoallocMaxNy,
                 Ny);
        if (factor_scratch_bytes(Ny) > kNoallocScratchBytes)
            fail(WUST_ERR_RUNTIME, "static scratch too small for Ny = %d", Ny);
        const wust_c64 *in[9] = {Dd, Dl, Du, Ld, Ll, Lu, Ud, Ul, Uu};
        for (const wust_c64 *p : in)
            if (!p || !noalloc_device_pointer(p)) fail(WUST_ERR_INVALID_INPUT, "decompBlockLU requires 9 gpuArray inputs.");
        if (!invT || !noalloc_device_pointer(invT))
            fail(WUST_ERR_INVALID_OUTPUT, "decompBlockLU requires a device invT output.");
        void *scratch = noalloc_scratch_address();
        Coefs<float2> co;
        co.Dd = (const float2 *)Dd; co.Dl = (const float2 *)Dl; co.Du = (const float2 *)Du;
        co.Ld = (const float2 *)Ld; co.Ll = (const float2 *)Ll; co.Lu = (const float2 *)Lu;
        co.Ud = (const float2 *)Ud; co.Ul = (const float2 *)Ul; co.Uu = (const float2 *)Uu;
        co.ny = Ny; co.nx = Nx;
        int hstat[3] = {0, 0, 0};
        factor_launch(co, (float2 *)invT, scratch, kNoallocScratchBytes, (cudaStream_t)stream, 10.0, hstat);
        if (hstat[2]) fail(WUST_ERR_DEVICE_TIMEOUT, "factorization grid barrier %d timed out", hstat[2]);
        if (hstat[0]) fail(WUST_ERR_SINGULAR_SCHUR_BLOCK, "getrf block %d is singular at pivot %d", hstat[0], hstat[1] + 1);
        return WUST_OK;
    } catch (const WustError &e) {
        set_last_error(e.message);
        return e.status;
    } catch (...) {
        set_last_error("unknown error");
        return WUST_ERR_RUNTIME;
    }
}
