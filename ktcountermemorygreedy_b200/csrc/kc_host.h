// kc_host.h -- host-side helpers shared by the C ABI translation units:
// error type, CUDA check macro, stream-ordered allocation scope, and the
// tile-aligned device layout of FASTQ inputs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "kc.h"
#include "kc_kernels.cuh"

namespace kc {

struct KcError {
    int code;
    std::string msg;
};

int set_error(int code, const std::string &msg);

#define CK(x)                                                                                            \
    do {                                                                                                 \
        cudaError_t e_ = (x);                                                                            \
        if (e_ != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            throw ::kc::KcError{e_ == cudaErrorMemoryAllocation ? KC_ERR_NOMEM : KC_ERR_CUDA,            \
                                std::string(#x) + ": " + cudaGetErrorString(e_)};                        \
        }                                                                                                \
    } while (0)

// Stream-ordered device allocations released together.
struct DevScope {
    cudaStream_t st = nullptr;
    std::vector<void *> ptrs;
    explicit DevScope(cudaStream_t s) : st(s) {}
    DevScope(const DevScope &) = delete;
    DevScope &operator=(const DevScope &) = delete;
    void *get(size_t bytes);
    template <class T>
    T *n(size_t count)
    {
        return static_cast<T *>(get(count * sizeof(T)));
    }
    void release(void *p);
    ~DevScope();
};

uint64_t bit_ceil64(uint64_t x);

}  // namespace kc

struct kc_input {
    uint8_t *base = nullptr;       // allocation (FRONT_PAD zero bytes, then tiles)
    uint8_t *buf = nullptr;        // first byte of tile 0
    uint64_t n_tiles = 0;
    std::vector<kc::Seg> segs;     // k and sample are filled in per job
    uint32_t *d_tile_seg = nullptr;
    std::vector<uint64_t> sizes;   // per file (including empty files)
    uint64_t total_bytes = 0;
    bool stream_owned = false;     // allocated with cudaMallocAsync on a job stream
};

namespace kc {

// Lays the files out tile-aligned in one device buffer.  When `scope` is
// given the allocations belong to it (per-job upload), otherwise they are
// long-lived (kc_input_upload).  `file_sample` (optional) assigns each file
// to a sample.
void build_input(kc_input &in, const kc_buffer *files, uint32_t n_files, cudaStream_t st, DevScope *scope,
                 std::vector<uint32_t> &tile_seg_host, const uint32_t *file_sample = nullptr);

}  // namespace kc
