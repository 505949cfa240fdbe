// Exclusive scan-gather that allocates nothing.
//
// Some callers cannot call cudaMalloc: host programs whose device memory is
// owned by another allocator (a framework's caching pool that has already
// reserved the device and expects to be the only allocator), and per-frame
// loops that may not take cudaMalloc / cudaFree's implicit device-wide
// synchronisation. sf_exclusive_scan_gather needs an sf_scan scratch, which
// sf_scan_create allocates; this variant instead runs the same single-pass
// look-back scan kernel over a scratch held in a file-scope __device__ array
// of fixed size, so it calls no cudaMalloc, cudaFree or other allocating
// routine.
//
// The array is shared by every call on a device and keeps the last call's
// contents: each call clears the partition ticket, the look-back status
// words and the error word before its kernel starts. Calls that overlap on
// the GPU (on different streams, or from different host threads) race on the
// array; callers must order them, e.g. by issuing them on one stream.
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "sf_handles.h"

namespace {

// Maximum element count: 2^24 (SF_SCAN_NOALLOC_MAX_ELEMS). The array holds a
// 64-byte line for the 64-bit total and the error word, a 64-byte ticket line,
// and one look-back status word per 4096-element partition (4096 words,
// 32 KiB): 32,896 bytes.
constexpr uint32_t kNoAllocMaxElems = SF_SCAN_NOALLOC_MAX_ELEMS;
static_assert(kNoAllocMaxElems == (1u << 24), "header and scratch size disagree");
constexpr size_t kNoAllocTotalsBytes = 64;
constexpr size_t kNoAllocScanBytes = 64 + (size_t)(kNoAllocMaxElems / 4096) * 8;
constexpr size_t kNoAllocBytes = kNoAllocTotalsBytes + kNoAllocScanBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device, found once per device by
// the first call on it. A cudaDeviceReset unloads the module that holds the
// array, so the cached address is not valid across one: callers that reset a
// device must not use this entry point afterwards in the same process.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

int na_fail(int code, const std::string& msg) { return sfk::set_error(code, msg); }

// Set-up, once per device, with that device current.
int noalloc_scratch(int device, unsigned char** out) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return na_fail(SF_ERR_CUDA, std::string("cudaGetSymbolAddress(static scan scratch): ") +
                                            cudaGetErrorString(e));
        g_noalloc_ptr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
    return SF_OK;
}

}  // namespace

extern "C" {

int sf_exclusive_scan_gather_noalloc(const uint32_t* gids, const uint32_t* counts, uint32_t* offsets,
                                     uint32_t n, sf_stream stream) {
    try {
        if (n > kNoAllocMaxElems)
            return na_fail(SF_ERR_SHAPE, "sf_exclusive_scan_gather_noalloc: " + std::to_string(n) +
                                             " elements exceed the static scratch maximum of " +
                                             std::to_string(kNoAllocMaxElems));
        if (n == 0) return SF_OK;
        if (!counts || !offsets) return na_fail(SF_ERR_ARG, "null buffer");
        if (sfk::scan_temp_bytes(n) > kNoAllocScanBytes)
            return na_fail(SF_ERR_SHAPE, "static scan scratch too small for the scan's partitions");
        int device = -1;
        cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess)
            return na_fail(SF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        if (device < 0 || device >= kMaxDevices) return na_fail(SF_ERR_ARG, "device ordinal out of range");
        unsigned char* base = nullptr;
        const int rc = noalloc_scratch(device, &base);
        if (rc != SF_OK) return rc;
        const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        auto* total = reinterpret_cast<unsigned long long*>(base);
        auto* err = reinterpret_cast<uint32_t*>(base + 8);
        // The total and error words start at zero; sfk::exclusive_scan clears
        // the ticket and the look-back words it uses.
        e = cudaMemsetAsync(base, 0, kNoAllocTotalsBytes, st);
        if (e == cudaSuccess)
            e = sfk::exclusive_scan(gids, counts, offsets, n, nullptr, n, base + kNoAllocTotalsBytes, total,
                                    err, st, sfk::lookback_test_knobs());
        // The error word comes back into a host stack variable (no pinned
        // buffer is allocated); a look-back wait that ran out is reported.
        uint32_t word = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&word, err, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return na_fail(SF_ERR_CUDA, std::string("static-scratch scan: ") + cudaGetErrorString(e));
        if (word & SF_DEV_ERR_TIMEOUT)
            return na_fail(SF_ERR_TIMEOUT, "static-scratch scan: device look-back wait timed out");
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return na_fail(SF_ERR_NOMEM, "host allocation failed");
    }
}

}  // extern "C"
