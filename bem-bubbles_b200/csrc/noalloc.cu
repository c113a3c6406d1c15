// Allocation-free entry point of the split-precision tensor-core GEMM.
//
// Some callers cannot allocate GPU memory themselves: code running under a host framework that owns
// the device heap (a memory-pool allocator, an embedding application that forbids the driver's
// allocator), real-time loops that must not allocate after start-up, and plug-ins that only get
// device pointers handed in.  bem_gemm_bf16x3 allocates its operand copies and the bf16 operand
// planes on every call, so those callers cannot use it.  bem_gemm_bf16x3_noalloc takes the caller's
// device pointers for A, B and C and keeps its only scratch -- the four bf16 operand planes and the
// error word -- in the file-scope device array below.  Every GPU that loads this library holds that
// array (BEM_NOALLOC_GEMM_MAX_N^2 * 8 bytes + 256 bytes, 8 MB) until the process exits.
#include <mutex>

#include "ctx.h"

namespace bemb {

constexpr size_t NOALLOC_PLANE_ELEMS = (size_t)BEM_NOALLOC_GEMM_MAX_N * BEM_NOALLOC_GEMM_MAX_N;
constexpr size_t NOALLOC_PLANES_BYTES = 4 * NOALLOC_PLANE_ELEMS * 2;  // four bf16 planes
constexpr size_t NOALLOC_BYTES = NOALLOC_PLANES_BYTES + 256;          // + the error word

// The scratch.  In host code this name is only a host-side stand-in for the device array; the device
// address comes from cudaGetSymbolAddress, once per device (noalloc_scratch below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static void* g_noalloc_ptr[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mutex;

// Device address of the scratch on the current device (looked up on the first call per device).
static int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return BEM_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BEM_ERR_CUDA;
        g_noalloc_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
    return BEM_OK;
}

}  // namespace bemb

namespace {
// Makes `device` current for the call and gives the caller's thread its own current device back on
// every return path (plug-in callers, e.g. under a framework driving several GPUs, keep theirs).
struct DeviceScope {
    int prev = -1;
    bool ok = false;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int gemm_noalloc(int device, int n, const float* A, const float* B, float* C, cudaStream_t s) {
    using namespace bemb;
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(device, &scratch);
    if (rc) return rc;
    int* err = reinterpret_cast<int*>(scratch + NOALLOC_PLANES_BYTES);
    // the error word must start at zero; the planes are overwritten in full (pads included)
    if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return BEM_ERR_CUDA;
    Ctx c;
    rc = tc_gemm(c, n, A, B, C, scratch, err, s);  // reports a refused launch itself
    if (rc) return rc;
    int herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return BEM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return BEM_ERR_CUDA;
    return herr ? BEM_ERR_CUDA : BEM_OK;
}
}  // namespace

// The stream must belong to `device` (or be the legacy default stream 0, then that device's).
extern "C" int bem_gemm_bf16x3_noalloc(int device, int n, const float* A, const float* B, float* C, void* stream) {
    using namespace bemb;
    if (n <= 0 || !A || !B || !C) return BEM_ERR_ARG;
    if (n > BEM_NOALLOC_GEMM_MAX_N) return BEM_ERR_ARG;  // the scratch holds planes up to this size
    DeviceScope scope(device);
    if (!scope.ok) return BEM_ERR_CUDA;
    return gemm_noalloc(device, n, A, B, C, static_cast<cudaStream_t>(stream));
}
