// S4 matching for callers that cannot allocate device memory.
//
// Who needs this: code that holds descriptor and match buffers handed to it
// by another component but may not call cudaMalloc itself. Examples are a
// plug-in running inside a host process that owns all device allocations, and
// a latency-bound loop where cudaMalloc's implicit device-wide
// synchronisation is not acceptable. Such a caller cannot provide the S4
// workspace, so this entry point uses a scratch array that lives in the
// library's own device memory instead.
//
// The scratch is a file-scope __device__ array of kScratchBytes (4 MiB). Every
// GPU that loads the library holds it until the process exits. All calls on a
// device share the one array, and it keeps whatever the last call wrote. The
// S4 kernels fully write every region they later read, so nothing needs
// clearing between calls. Calls that overlap on the GPU (other streams, or
// other host threads on the same device) race on the array: serialise them.
//
// The array's device address belongs to the CUDA context that loaded the
// module. The first call on a device, with that device current, looks it up
// with cudaGetSymbolAddress and keeps it together with the context's unique
// id; a later call in another context (after cudaDeviceReset, for example)
// looks it up again, and a lookup that failed is retried on the next call.
// Make the first call on a device, and the first call after a device reset,
// before any stream capture. Argument errors are reported exactly as
// stitch_s4_match reports them; then requests whose S4 workspace would exceed
// kScratchBytes fail with INSUFFICIENT_WORKSPACE, before anything is
// enqueued. No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "s4_internal.hpp"
#include "stitch_b200.h"

namespace {

constexpr std::size_t kScratchBytes = std::size_t{4} << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_s4_scratch[kScratchBytes];

using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

struct DriverCalls {
    CtxGetCurrent get_current = nullptr;
    CtxGetId get_id = nullptr;
};

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry points
// (the library links no libcuda); both null when the driver lacks them.
const DriverCalls& driver_calls() {
    static const DriverCalls calls = [] {
        DriverCalls c;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && p)
            c.get_current = reinterpret_cast<CtxGetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && p)
            c.get_id = reinterpret_cast<CtxGetId>(p);
        if (!c.get_current || !c.get_id) c = DriverCalls{};
        return c;
    }();
    return calls;
}

// Unique id of the current context (ids are never reused within a process);
// 0 when there is none or it cannot be read.
unsigned long long current_context_id() {
    const DriverCalls& d = driver_calls();
    if (!d.get_current) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (d.get_current(&ctx) != CUDA_SUCCESS || !ctx || d.get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

struct Cached {
    unsigned long long context = 0;  // 0: nothing cached
    void* address = nullptr;
};
std::mutex g_lock;
Cached g_cache[kMaxDevices];

// Device address of g_s4_scratch in the current device's current context
// (null on failure). Only a successful lookup is kept; without context ids
// the address is looked up on every call.
void* scratch_on_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> hold(g_lock);
    Cached& c = g_cache[dev];
    if (ctx != 0 && c.context == ctx) return c.address;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_s4_scratch) != cudaSuccess || !p) {
        cudaGetLastError();  // the failure is reported by the return code, not left for the next call
        return nullptr;
    }
    // the lookup makes the device's primary context current if it was not
    const unsigned long long now = ctx != 0 ? ctx : current_context_id();
    c = Cached{now, now != 0 ? p : nullptr};
    return p;
}

}  // namespace

extern "C" int stitch_s4_match_static(const stitch_keypoints* a, const stitch_descriptors* da,
                                      const stitch_keypoints* b, const stitch_descriptors* db,
                                      const stitch_s4_config* config, const stitch_matches* output,
                                      void* stream) {
    using namespace stitch;
    if (!a || !da || !b || !db || !config || !output) return static_cast<int>(Status::INVALID_ARGUMENT);
    const auto& ka = *reinterpret_cast<const Keypoints*>(a);
    const auto& kb = *reinterpret_cast<const Keypoints*>(b);
    const auto& dA = *reinterpret_cast<const Descriptors*>(da);
    const auto& dB = *reinterpret_cast<const Descriptors*>(db);
    const auto& cfg = *reinterpret_cast<const s4::Config*>(config);
    const auto& out = *reinterpret_cast<const Matches*>(output);
    std::size_t need = 0;
    const Status q = b200::s4k::check_match_args(ka, dA, kb, dB, cfg, out, &need);
    if (q != Status::OK) return static_cast<int>(q);
    if (need > kScratchBytes) return static_cast<int>(Status::INSUFFICIENT_WORKSPACE);
    void* scratch = scratch_on_current_device();
    if (!scratch) return static_cast<int>(Status::CUDA_ERROR);
    return static_cast<int>(s4::s4_match(ka, dA, kb, dB, cfg, out, scratch, kScratchBytes,
                                         static_cast<cudaStream_t>(stream)));
}
