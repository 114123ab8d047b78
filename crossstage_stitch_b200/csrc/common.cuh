// Shared host/device helpers for the stage kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstddef>
#include <cstdint>

#include "stage_api.hpp"

namespace stitch::b200 {

constexpr std::size_t kWorkspaceAlign = 256;
constexpr int kSmCount = 148;  // B200: grid sizing target, not a correctness input

// Kernel launches issued by this library (all threads, all devices); read
// through stitch_launch_count() to attribute device work to these kernels.
void note_launches(int n);

inline Status launch_status() {
    return cudaGetLastError() == cudaSuccess ? Status::OK : Status::CUDA_ERROR;
}

template <class T> inline T* at_offset(void* base, std::size_t offset) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + offset);
}

inline bool aligned(const void* p, std::size_t a) {
    return (reinterpret_cast<std::uintptr_t>(p) % a) == 0;
}

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

// Bump allocator over a workspace: every region starts on a 256-byte
// boundary; false on size_t overflow.
struct Layout {
    std::size_t cursor = 0;
    bool ok = true;
    std::size_t take(std::size_t count, std::size_t elem) {
        constexpr std::size_t kMax = ~std::size_t{0};
        if (!ok) return 0;
        if (cursor > kMax - (kWorkspaceAlign - 1)) { ok = false; return 0; }
        const std::size_t start = (cursor + kWorkspaceAlign - 1) / kWorkspaceAlign * kWorkspaceAlign;
        if (elem && count > (kMax - start) / elem) { ok = false; return 0; }
        cursor = start + count * elem;
        return start;
    }
};

}  // namespace stitch::b200
