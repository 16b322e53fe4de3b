// kc_noalloc.cu -- kc_sort_records_noalloc: the record sort for callers that
// cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc at the point where
// they need sorted records: code that runs with a fixed device-memory budget
// accounted up front (another framework's caching allocator owns the rest of
// the GPU), latency-critical request paths where an allocation can stall on
// the driver or synchronize the device, or callers that already hold the
// records in device memory and only have a stream to offer.  This entry point
// sorts the caller's device arrays in place and takes its working memory from
// a fixed array compiled into the library instead of allocating it.
//
// The scratch array is a file-scope __device__ array of 13 MiB.  In host code
// its name is only a host-side stand-in, not a device address, so the address
// is looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on that device.  With CUDA's lazy module
// loading (the default) a module's code and __device__ arrays are placed in
// device memory when the module is first used, so that first call also loads
// the module of this file (the array) and the sort kernels it launches; from
// then on the array and the kernels stay loaded on that device until the
// process exits, and no later call loads or allocates anything.  A call with
// n = 0 does only this set-up and can serve as a warm-up.
#include <cuda_runtime.h>

#include <array>
#include <mutex>
#include <string>

#include "kc.h"
#include "kc_host.h"
#include "kc_kernels.cuh"

namespace {

// 13 MiB: the LSD sort of KC_SORT_NOALLOC_MAX records needs a second copy of
// keys and counts (12 MiB) plus per-tile digit counts, offsets and the tile
// descriptors (under 1 MiB).
constexpr size_t SCRATCH_BYTES = 13ull << 20;

__device__ __align__(256) unsigned char g_sort_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
std::array<void *, MAX_DEVICES> g_scratch_ptr{};

// Device address of the scratch array on the current device (looked up, and
// the sort kernels loaded, on the first call for that device).
int scratch_for_current_device(void **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return kc::set_error(KC_ERR_NO_DEVICE, "no current CUDA device");
    }
    if (dev >= MAX_DEVICES) return kc::set_error(KC_ERR_INVALID, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return kc::set_error(KC_ERR_CUDA, std::string("cudaGetSymbolAddress of the sort scratch failed: ") +
                                                  cudaGetErrorString(e));
        }
        e = kc::preload_sort_in_scratch();
        if (e != cudaSuccess) {
            cudaGetLastError();
            return kc::set_error(KC_ERR_CUDA, std::string("loading the sort kernels failed: ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return KC_OK;
}

}  // namespace

extern "C" int kc_sort_records_noalloc(uint64_t *d_keys, uint32_t *d_counts, uint64_t n, uint32_t bits,
                                       void *stream)
{
    if ((!d_keys || !d_counts) && n) return kc::set_error(KC_ERR_INVALID, "bad argument");
    if (bits > 64) return kc::set_error(KC_ERR_INVALID, "bits must be <= 64");
    if (n > KC_SORT_NOALLOC_MAX)
        return kc::set_error(KC_ERR_INVALID, "kc_sort_records_noalloc sorts at most " +
                                                 std::to_string((unsigned long long)KC_SORT_NOALLOC_MAX) +
                                                 " records; got " + std::to_string((unsigned long long)n));
    const size_t need = kc::sort_tmp_bytes_in_scratch(n);
    if (need > SCRATCH_BYTES) return kc::set_error(KC_ERR_INVALID, "scratch array too small for this sort");
    void *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != KC_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call waits for its sort, which a stream being captured into a
    // graph cannot do: refuse before enqueuing anything
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();
        return kc::set_error(KC_ERR_CUDA, "kc_sort_records_noalloc: cannot query the stream's capture status");
    }
    if (cap != cudaStreamCaptureStatusNone)
        return kc::set_error(KC_ERR_INVALID, "kc_sort_records_noalloc waits for its sort and cannot be called on a "
                                             "stream that is being captured");
    if (n <= 1) return KC_OK;
    // nothing in the scratch has to start at zero: every pass writes all the
    // digit counts, offsets and records it later reads
    cudaError_t e =
        kc::launch_radix_sort_in_scratch(reinterpret_cast<unsigned long long *>(d_keys), d_counts, n, bits, scratch, st);
    // the call returns once the records are sorted
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return kc::set_error(KC_ERR_CUDA, std::string("kc_sort_records_noalloc: ") + cudaGetErrorString(e));
    }
    return KC_OK;
}
