// S4 kernels: exact brute-force top-2 neighbours and the ratio-test
// compaction, sm_100a.
//
// Reference semantics (file:line in the reference tree):
//   top-2 order: lower distance, then lower train index; the second
//   neighbour is a distinct index; missing = (+inf, -1) .... src/s4/s4.cu:115-135
//   binary distance = sum of byte popcounts (as double); float distance =
//   sum over dimensions, in order, of rounded squared differences  src/s4/s4.cu:164-181
//   accept: second exists and d1 == 0 ? d2 > 0 : d1 < ratio * d2,
//   optional mutual check ...................................... src/s4/s4.cu:212-239
//   compaction in query order, sqrt for L2, +inf above FLT_MAX .. src/s4/s4.cu:241-262
//
// Hot path (BINARY_U8, 32-byte rows): each thread owns one query row (eight
// 32-bit words in registers); train rows stream through shared memory and
// every thread scores them against its query with XOR + POPC. A neighbour is
// kept as the 32-bit key (distance << 23) | train_index, so "smaller key" is
// exactly the reference order and the top-2 update is three min/max ops.
// Train rows can be split over several blocks; a merge pass then takes the
// two smallest keys per query.
#pragma once

#include <cfloat>
#include <math_constants.h>

#include "common.cuh"

namespace stitch::b200::s4k {

using Top2 = ::stitch::s4::Top2;

constexpr int kQueryThreads = 128;
// Queries held per thread by the batched chain (1 measured fastest: 4 per
// thread cost more in occupancy than it saved in shared-memory reads).
constexpr int kQueriesPerThread = 1;
constexpr int kQueryTile = kQueryThreads * kQueriesPerThread;  // queries per batched popc block
constexpr int kTrainStage = 256;   // train rows per shared-memory stage
constexpr int kIndexBits = 23;     // train index bits of a key
constexpr std::uint32_t kEmptyKey = 0xffffffffu;
constexpr int kMaxPopcTrain = 1 << kIndexBits;

struct Side {
    const std::uint8_t* rows;
    int stride;
    int capacity;
    const int* count;
};

struct KnnJob {
    Side query, train;
    int q_tiles;         // ceil(query.capacity / (kQueryThreads * queries per thread))
    int splits;          // train partitions
    int rows_per_split;  // multiple of kTrainStage
    uint2* partial;      // [splits][query.capacity] (k1, k2); unused when splits == 1
    Top2* top2;          // [query.capacity]
};

template <class Job> struct OneJob {
    Job job;
    __device__ bool find(int block, Job* j, int* local) const {
        *j = job;
        *local = block;
        return true;
    }
};

// Device table of jobs with a block prefix (prefix[n] = total blocks).
template <class Job> struct JobTable {
    const Job* jobs;
    const int* prefix;
    int n;
    __device__ bool find(int block, Job* j, int* local) const {
        if (block >= prefix[n]) return false;
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= block) lo = mid; else hi = mid - 1;
        }
        *j = jobs[lo];
        *local = block - prefix[lo];
        return true;
    }
};

__device__ __forceinline__ bool counts_valid(const KnnJob& j, int* nq, int* nt) {
    *nq = *j.query.count;
    *nt = *j.train.count;
    return *nq >= 0 && *nq <= j.query.capacity && *nt >= 0 && *nt <= j.train.capacity;
}

__device__ __forceinline__ Top2 top2_from_keys(std::uint32_t k1, std::uint32_t k2) {
    Top2 t;
    t.first_index = k1 == kEmptyKey ? -1 : static_cast<int>(k1 & ((1u << kIndexBits) - 1));
    t.first_distance = k1 == kEmptyKey ? CUDART_INF : static_cast<double>(k1 >> kIndexBits);
    t.second_index = k2 == kEmptyKey ? -1 : static_cast<int>(k2 & ((1u << kIndexBits) - 1));
    t.second_distance = k2 == kEmptyKey ? CUDART_INF : static_cast<double>(k2 >> kIndexBits);
    return t;
}

__device__ __forceinline__ void keep2(std::uint32_t& k1, std::uint32_t& k2, std::uint32_t k) {
    k2 = min(k2, max(k1, k));
    k1 = min(k1, k);
}

// Block = kQ * 128 queries x one train partition. Thread t holds queries
// t, t + 128, ... of the tile in registers, so each staged train row read
// from shared memory serves kQ queries.
template <class Src, int kQ>
__global__ __launch_bounds__(kQueryThreads) void knn_popc_kernel(const __grid_constant__ Src src) {
    __shared__ uint4 stage[kTrainStage * 2];
    KnnJob j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    const int qt = local % j.q_tiles, split = local / j.q_tiles;
    int nq, nt;
    const bool ok = counts_valid(j, &nq, &nt);
    const int t0 = split * j.rows_per_split;
    const int t1 = ok ? min(nt, t0 + j.rows_per_split) : t0;
    uint4 qa[kQ], qb[kQ];
    std::uint32_t k1[kQ], k2[kQ];
#pragma unroll
    for (int u = 0; u < kQ; ++u) {
        const int q = (qt * kQ + u) * kQueryThreads + threadIdx.x;
        qa[u] = qb[u] = make_uint4(0, 0, 0, 0);
        if (ok && q < nq) {
            const uint4* row = reinterpret_cast<const uint4*>(j.query.rows + static_cast<std::size_t>(q) * j.query.stride);
            qa[u] = row[0];
            qb[u] = row[1];
        }
        k1[u] = k2[u] = kEmptyKey;
    }
    for (int base = t0; base < t1; base += kTrainStage) {
        const int rows = min(kTrainStage, t1 - base);
        for (int i = threadIdx.x; i < rows * 2; i += kQueryThreads) {
            const uint4* row = reinterpret_cast<const uint4*>(
                j.train.rows + static_cast<std::size_t>(base + (i >> 1)) * j.train.stride);
            stage[i] = row[i & 1];
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < rows; ++r) {
            const uint4 a = stage[2 * r], b = stage[2 * r + 1];
            const std::uint32_t idx = static_cast<std::uint32_t>(base + r);
#pragma unroll
            for (int u = 0; u < kQ; ++u) {
                const int d = __popc(qa[u].x ^ a.x) + __popc(qa[u].y ^ a.y) + __popc(qa[u].z ^ a.z) +
                              __popc(qa[u].w ^ a.w) + __popc(qb[u].x ^ b.x) + __popc(qb[u].y ^ b.y) +
                              __popc(qb[u].z ^ b.z) + __popc(qb[u].w ^ b.w);
                keep2(k1[u], k2[u], (static_cast<std::uint32_t>(d) << kIndexBits) | idx);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kQ; ++u) {
        const int q = (qt * kQ + u) * kQueryThreads + threadIdx.x;
        if (q >= j.query.capacity) continue;
        const bool active = ok && q < nq;
        const std::uint32_t a1 = active ? k1[u] : kEmptyKey, a2 = active ? k2[u] : kEmptyKey;
        if (j.splits == 1) {
            j.top2[q] = top2_from_keys(a1, a2);
        } else {
            j.partial[static_cast<std::size_t>(split) * j.query.capacity + q] = make_uint2(a1, a2);
        }
    }
}

// Thread per query: the two smallest keys over all train partitions.
template <class Src>
__global__ __launch_bounds__(256) void knn_merge_kernel(const __grid_constant__ Src src) {
    KnnJob j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    const int q = local * 256 + threadIdx.x;
    if (q >= j.query.capacity) return;
    std::uint32_t k1 = kEmptyKey, k2 = kEmptyKey;
    for (int s = 0; s < j.splits; ++s) {
        const uint2 p = j.partial[static_cast<std::size_t>(s) * j.query.capacity + q];
        keep2(k1, k2, p.x);
        keep2(k1, k2, p.y);
    }
    j.top2[q] = top2_from_keys(k1, k2);
}

// ---------------------------------------------------------------- generic

// (d, i) precedes (e, k): lower distance, then lower index; missing last.
__device__ __forceinline__ bool precedes(double d, int i, double e, int k) {
    return i >= 0 && (k < 0 || d < e || (d == e && i < k));
}

__device__ __forceinline__ void push(Top2& t, double d, int i) {
    if (i < 0 || i == t.first_index || i == t.second_index) return;
    if (precedes(d, i, t.first_distance, t.first_index)) {
        t.second_distance = t.first_distance;
        t.second_index = t.first_index;
        t.first_distance = d;
        t.first_index = i;
    } else if (precedes(d, i, t.second_distance, t.second_index)) {
        t.second_distance = d;
        t.second_index = i;
    }
}

// Any descriptor width, BINARY_U8 or FLOAT32: one warp per query, lanes take
// train rows round-robin, then the lane top-2s are merged across the warp.
template <bool kFloat>
__global__ __launch_bounds__(256) void knn_generic_kernel(Side query, Side train, int dim, Top2* out) {
    const int lane = threadIdx.x & 31;
    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    const int nq = *query.count, nt = *train.count;
    const bool ok = nq >= 0 && nq <= query.capacity && nt >= 0 && nt <= train.capacity;
    for (long long q = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
         q < query.capacity; q += warps) {
        Top2 t{CUDART_INF, CUDART_INF, -1, -1};
        if (ok && q < nq) {
            const std::uint8_t* qrow = query.rows + static_cast<std::size_t>(q) * query.stride;
            for (int r = lane; r < nt; r += 32) {
                const std::uint8_t* trow = train.rows + static_cast<std::size_t>(r) * train.stride;
                double d = 0.0;
                if constexpr (kFloat) {
                    const float* a = reinterpret_cast<const float*>(qrow);
                    const float* b = reinterpret_cast<const float*>(trow);
                    for (int k = 0; k < dim; ++k) {
                        const double delta = static_cast<double>(a[k]) - static_cast<double>(b[k]);
                        d = __dadd_rn(d, __dmul_rn(delta, delta));
                    }
                } else {
                    long long bits = 0;
                    for (int k = 0; k < dim; ++k) bits += __popc(static_cast<unsigned>(qrow[k] ^ trow[k]));
                    d = static_cast<double>(bits);
                }
                push(t, d, r);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double d1 = __shfl_xor_sync(0xffffffffu, t.first_distance, o);
            const double d2 = __shfl_xor_sync(0xffffffffu, t.second_distance, o);
            const int i1 = __shfl_xor_sync(0xffffffffu, t.first_index, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, t.second_index, o);
            push(t, d1, i1);
            push(t, d2, i2);
        }
        if (lane == 0) out[q] = t;
    }
}

// ------------------------------------------------------------ compaction

struct AcceptJob {
    const Top2* forward;
    const Top2* reverse;  // null without the mutual check
    int capacity;         // query rows
    double ratio;         // squared for L2
    int l2;
    ::stitch::Matches out;
};

// One block per query set: ratio test (+ mutual check) and a stable
// compaction in query order; writes the match count.
template <class Src>
__global__ __launch_bounds__(1024) void accept_kernel(const __grid_constant__ Src src) {
    __shared__ int warp_sum[32];
    AcceptJob j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int running = 0;
    for (int base = 0; base < j.capacity; base += 1024) {
        const int q = base + threadIdx.x;
        bool accept = false;
        Top2 p{};
        if (q < j.capacity) {
            p = j.forward[q];
            accept = p.second_index >= 0 &&
                     (p.first_distance == 0 ? p.second_distance > 0
                                            : p.first_distance < j.ratio * p.second_distance);
            if (accept && j.reverse) accept = j.reverse[p.first_index].first_index == q;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, accept);
        if (lane == 0) warp_sum[warp] = __popc(ballot);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < 32; ++w) {
            before += w < warp ? warp_sum[w] : 0;
            total += warp_sum[w];
        }
        if (accept) {
            const int at = running + before + __popc(ballot & ((1u << lane) - 1u));
            j.out.idx_a[at] = q;
            j.out.idx_b[at] = p.first_index;
            const double d = j.l2 ? sqrt(p.first_distance) : p.first_distance;
            j.out.distance[at] = d > FLT_MAX ? CUDART_INF_F : static_cast<float>(d);
        }
        running += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *j.out.d_count = running;
}

}  // namespace stitch::b200::s4k
