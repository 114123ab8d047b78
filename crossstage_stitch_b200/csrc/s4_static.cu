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
// The first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (once per device). Make
// that first call before any stream capture. Requests whose S4 workspace
// would exceed kScratchBytes fail with INSUFFICIENT_WORKSPACE before anything
// is enqueued. No cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>

#include "stage_api.hpp"
#include "stitch_b200.h"

#include <cuda_runtime.h>

namespace {

constexpr std::size_t kScratchBytes = std::size_t{4} << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_s4_scratch[kScratchBytes];

std::once_flag g_once[kMaxDevices];
void* g_addr[kMaxDevices];

// Device address of g_s4_scratch on the current device (null on failure).
void* scratch_on_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::call_once(g_once[dev], [dev] {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_s4_scratch) == cudaSuccess) g_addr[dev] = p;
    });
    return g_addr[dev];
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
    const auto& cfg = *reinterpret_cast<const s4::Config*>(config);
    std::size_t need = 0;
    const Status q = s4::s4_workspace_bytes(ka.capacity, kb.capacity, cfg, &need);
    if (q != Status::OK) return static_cast<int>(q);
    if (need > kScratchBytes) return static_cast<int>(Status::INSUFFICIENT_WORKSPACE);
    void* scratch = scratch_on_current_device();
    if (!scratch) return static_cast<int>(Status::CUDA_ERROR);
    return static_cast<int>(s4::s4_match(ka, *reinterpret_cast<const Descriptors*>(da), kb,
                                         *reinterpret_cast<const Descriptors*>(db), cfg,
                                         *reinterpret_cast<const Matches*>(output), scratch, kScratchBytes,
                                         static_cast<cudaStream_t>(stream)));
}
