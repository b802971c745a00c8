// mqb_apply_static: circuit application for callers that cannot allocate device memory.
//
// mqb_apply needs a caller-provided workspace for the per-sample gate matrices that the matrix
// generation kernel writes and the tile kernels read.  Some callers cannot call cudaMalloc (or
// any allocating routine) when they apply a circuit: runtimes that reserve all device memory in a
// fixed pool at start-up, thin language bindings that only own the state buffers they pass in,
// and real-time loops that must not call into the allocator.  This entry point uses a fixed
// scratch array that lives in the library's own device memory instead.
//
// The scratch is a file-scope __device__ array of kStaticScratchBytes (4 MiB).  Every GPU that
// loads this library holds it until the process exits.  Its device address is looked up once per
// device with cudaGetSymbolAddress the first time the entry point runs with that device current,
// so that first call should come before any stream capture; a device reset invalidates the cached
// address (the entry point must not be used after cudaDeviceReset).  All calls share the one array:
// calls whose work overlaps on the GPU (different streams, or different host threads without
// ordering) race on it.  Nothing in it needs to start at zero: every call overwrites the
// matrices it reads before reading them.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/mqb200.h"
#include "mqb_internal.h"

namespace mqb {
void set_last_error(const char *msg);   // capi.cpp: the message mqb_last_error() returns on this thread
}

namespace {

constexpr size_t kStaticScratchBytes = size_t(4) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mutex;
void *g_static_ptr[kMaxDevices] = {nullptr};

int fail_static(int code, const char *fmt, ...) {
    char buf[320];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    mqb::set_last_error(buf);
    return code;
}

}  // namespace

extern "C" {

MQB_API int mqb_apply_static(mqb_program *prog, void *states, int64_t batch, const double *params,
                             int64_t param_stride, const double *custom, void *stream) {
    if (!prog || !states || batch < 1) return fail_static(MQB_ERR_INVALID, "mqb_apply_static: invalid argument");
    if (reinterpret_cast<uintptr_t>(states) & 15u)
        return fail_static(MQB_ERR_INVALID, "mqb_apply_static: states must be 16-byte aligned");
    size_t need = 0;
    int st = mqb_apply_workspace_size(prog, batch, &need);
    if (st != MQB_OK) return st;
    if (need > kStaticScratchBytes)
        return fail_static(MQB_ERR_WORKSPACE,
                           "mqb_apply_static: %zu bytes of gate matrices for batch %lld exceed the fixed scratch of "
                           "%zu bytes; use a smaller batch or mqb_apply with a workspace",
                           need, static_cast<long long>(batch), kStaticScratchBytes);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_static(MQB_ERR_CUDA, "mqb_apply_static: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail_static(MQB_ERR_INVALID, "mqb_apply_static: device %d not supported", dev);
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mutex);
        if (!g_static_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess || !p)
                return fail_static(MQB_ERR_CUDA, "mqb_apply_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_static_ptr[dev] = p;
        }
        scratch = g_static_ptr[dev];
    }
    mqb::JitBlock no_generated_kernels;   // loading a generated kernel would allocate device memory
    return mqb_apply(prog, states, batch, params, param_stride, custom, scratch, kStaticScratchBytes, stream);
}

}  // extern "C"
