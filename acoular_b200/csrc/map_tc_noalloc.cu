// Allocation-free variant of the tensor-core map (acb_map_tc_noalloc).
//
// acb_map_tc needs a scratch buffer for the split-BF16 copy of the real-embedded CSM and takes it
// from the caller.  Some callers cannot provide one: a real-time acquisition loop that must not
// call cudaMalloc (it can synchronise the whole device and stall the sample stream), or a host
// program that reaches this library through a plain C interface without any device allocator of
// its own.  For them the scratch lives in a fixed array in device memory that this library
// declares itself: every GPU that loads the library holds it (ACB_NOALLOC_SCRATCH_BYTES) until
// the process exits.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"

namespace {

constexpr size_t kScratchBytes = ACB_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The scratch array.  In host code this name is only a host-side handle for the symbol, not a
// device address; the device address is obtained once per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_map_tc_scratch[kScratchBytes];

std::mutex g_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up on first use and kept for
// the life of the process; a cudaDeviceReset of that device invalidates it).
int scratch_for_current_device(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        acb::set_cuda_error(e);
        return ACB_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return ACB_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_map_tc_scratch);
        if (e != cudaSuccess || !p) {
            acb::set_cuda_error(e);
            return ACB_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return ACB_OK;
}

}  // namespace

extern "C" {

int acb_map_tc_noalloc(const acb_map_params *p, int precision, const void *csm, const double *wavenumber,
                       const double *mpos, const double *gpos, double *out_map, double *out_steer_norm,
                       int *error_word, void *stream)
{
    // the argument checks of acb_map_tc, with its status codes: given no workspace it validates
    // everything and returns ACB_ERR_WORKSPACE, before any CUDA call, only when the arguments are good
    const int chk = acb_map_tc(p, precision, csm, wavenumber, mpos, gpos, out_map, out_steer_norm, nullptr, 0,
                               error_word, stream);
    if (chk != ACB_ERR_WORKSPACE) return chk;
    // the whole R' copy for this call must fit the fixed array; larger requests are rejected
    // before anything is enqueued (split the bins over several calls instead)
    const size_t need = acb_map_tc_workspace_bytes(p->num_mics, p->num_bins, precision);
    if (need == 0 || need > kScratchBytes) return ACB_ERR_SHAPE;
    void *scratch = nullptr;
    const int st = scratch_for_current_device(&scratch);
    if (st) return st;
    // every element of the scratch region this call uses is written by the call before it is
    // read, so nothing has to be cleared between calls
    return acb_map_tc(p, precision, csm, wavenumber, mpos, gpos, out_map, out_steer_norm, scratch, kScratchBytes,
                      error_word, stream);
}

}  // extern "C"
