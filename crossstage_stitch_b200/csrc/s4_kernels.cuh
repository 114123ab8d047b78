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
    // optional block -> (job << 16 | block within the job) map: one load
    // instead of a binary search over the prefix
    const std::uint32_t* map = nullptr;
    int map_blocks = 0;
    __device__ bool find(int block, Job* j, int* local) const {
        if (map) {
            if (block >= map_blocks) return false;
            const std::uint32_t e = __ldg(map + block);
            *j = jobs[e >> 16];
            *local = static_cast<int>(e & 0xffffu);
            return true;
        }
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

// ------------------------------------------------- tensor-core matcher
//
// Exact Hamming distance on the 5th-generation tensor cores: every
// descriptor bit b becomes the int8 value +1 (b = 1) or -1 (b = 0), so for
// two 256-bit descriptors dot = 256 - 2 * Hamming, and tcgen05.mma
// kind::i8 (int32 accumulation, exact) gives dot for a 128-query x
// 256-train tile in TMEM. The block walks the same train partition as the
// popc kernel; each query's thread reads its row of dot products back with
// tcgen05.ld and keeps the two smallest (distance << 23 | train index)
// keys, so results equal knn_popc_kernel's bit for bit.
//
// Shared memory holds the expanded queries (128 rows x 256 bytes) and one
// train stage (kRowsB rows x 256 bytes: 256, 128 or 64) in the K-major
// 128-byte-swizzle layout tcgen05 reads: per 128-byte K block, 8-row groups
// of 1024 bytes, 16-byte chunk c of row r stored at chunk c ^ (r % 8). A
// narrower stage halves the shared memory and TMEM of a block, so more
// blocks share an SM and one block's staging and epilogue overlap another's
// MMA (2, 3 or 4 blocks per SM).
constexpr int kTcRowsA = kQueryThreads;       // 128 queries (MMA M)
constexpr int kTcBytesA = kTcRowsA * 256;
template <int kRowsB> struct TcShape {
    static_assert(kRowsB == 64 || kRowsB == 128 || kRowsB == 256, "MMA N and TMEM columns");
    static constexpr int rows_b = kRowsB;                                  // MMA N, TMEM columns
    static constexpr int bytes_b = kRowsB * 256;
    static constexpr int smem = kTcBytesA + bytes_b + 1024 + 64;            // + alignment slack + barrier/slot
    static constexpr int blocks_per_sm = (228 * 1024) / (smem + 1024);     // shared memory bound
    // kind::i8 instruction descriptor: s32 accumulator, signed A and B, both
    // K-major, N = kRowsB, M = 128
    static constexpr std::uint32_t idesc =
        (2u << 4) | (1u << 7) | (1u << 10) | ((kRowsB >> 3) << 17) | ((kTcRowsA >> 4) << 24);
    static_assert(blocks_per_sm * kRowsB <= 512, "TMEM columns of the resident blocks");
};
constexpr long long kTcWaitLimit = 1ll << 26;  // mbarrier polls before giving up

// Error word of the tensor-core matcher (one per translation unit): set when
// an MMA completion wait runs out (the block then stops, frees its TMEM and
// leaves its outputs unwritten).
static __device__ int g_tc_error;

__device__ __forceinline__ std::uint32_t smem_u32(const void* p) {
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

// Bits 0..3 of n as the int8 values +1 / -1 in bytes 0..3.
__device__ __forceinline__ std::uint32_t pm_one4(std::uint32_t n) {
    const std::uint32_t spread = (n * 0x00204081u) & 0x01010101u;
    return 0x01010101u | ((spread ^ 0x01010101u) * 0xFEu);
}

// Writes descriptor row `row` (32 bytes at src; zeros when src is null) of
// a tile of `rows` rows into the swizzled layout at `tile`.
__device__ __forceinline__ void stage_pm_row(std::uint8_t* tile, int rows, int row, const std::uint8_t* src) {
    uint4 w[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    if (src) {
        w[0] = reinterpret_cast<const uint4*>(src)[0];
        w[1] = reinterpret_cast<const uint4*>(src)[1];
    }
    const std::uint32_t words[8] = {w[0].x, w[0].y, w[0].z, w[0].w, w[1].x, w[1].y, w[1].z, w[1].w};
    std::uint8_t* base = tile + (row >> 3) * 1024 + (row & 7) * 128;
#pragma unroll
    for (int h = 0; h < 16; ++h) {  // 16 descriptor bits -> one 16-byte chunk
        const std::uint32_t bits = (words[h >> 1] >> (16 * (h & 1))) & 0xffffu;
        const int kb = h >> 3, c = h & 7;
        uint4 v;
        v.x = src ? pm_one4(bits & 0xf) : 0u;
        v.y = src ? pm_one4((bits >> 4) & 0xf) : 0u;
        v.z = src ? pm_one4((bits >> 8) & 0xf) : 0u;
        v.w = src ? pm_one4((bits >> 12) & 0xf) : 0u;
        *reinterpret_cast<uint4*>(base + kb * rows * 128 + ((c ^ (row & 7)) << 4)) = v;
    }
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ std::uint64_t sw128_desc(std::uint32_t addr) {
    return static_cast<std::uint64_t>((addr >> 4) & 0x3fffu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
           (2ull << 61);
}

// Packed top-2 of one stage's columns: in each 32-bit word the low 16-bit
// lane holds a key of an even column and the high lane one of the next odd
// column, key16 = (distance << 7) | (column - first) / 2 with distance =
// (256 - dot) / 2 <= 256 (so key16 <= 32895; 0xffff is empty). Within a
// lane, smaller key16 is exactly (smaller distance, then smaller column), so
// one min/max.u16x2 updates two candidates. The even and odd lanes are
// folded into the 32-bit (distance << 23 | train index) chains when the
// stage ends (fold_stage), which keeps the top-2 exact.
__device__ __forceinline__ void keep2x2(std::uint32_t& a1, std::uint32_t& a2, std::uint32_t x) {
    a2 = __vminu2(a2, __vmaxu2(a1, x));
    a1 = __vminu2(a1, x);
}

// 32 dot products v of columns first + c .. first + c + 31 (c even) into
// the packed chains; columns at or past `limit` (train rows past the end)
// are left out.
__device__ __forceinline__ void stage_keys32(const std::uint32_t (&v)[32], int c, int first, int limit,
                                             std::uint32_t (&p1)[4], std::uint32_t (&p2)[4]) {
    const std::uint32_t m0 = static_cast<std::uint32_t>(c >> 1);
    constexpr std::uint32_t kBias = (256u << 6) + (256u << 22);  // (256 - v) << 6 per lane, as one add
    if (first + c + 32 <= limit) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const std::uint32_t m = m0 + static_cast<std::uint32_t>(i);
            const std::uint32_t x = (kBias + (m | (m << 16))) - (v[2 * i] << 6) - (v[2 * i + 1] << 22);
            keep2x2(p1[i & 3], p2[i & 3], x);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const std::uint32_t m = m0 + static_cast<std::uint32_t>(i);
            std::uint32_t x = (kBias + (m | (m << 16))) - (v[2 * i] << 6) - (v[2 * i + 1] << 22);
            if (first + c + 2 * i >= limit) x |= 0x0000ffffu;
            if (first + c + 2 * i + 1 >= limit) x |= 0xffff0000u;
            keep2x2(p1[i & 3], p2[i & 3], x);
        }
    }
}

// The packed chains of a stage whose first column is train row `first`
// into the 32-bit key chains; the packed chains are emptied.
__device__ __forceinline__ void fold_stage(std::uint32_t (&p1)[4], std::uint32_t (&p2)[4], std::uint32_t first,
                                           std::uint32_t (&k1)[4], std::uint32_t (&k2)[4]) {
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const std::uint32_t w = r ? p2[ch] : p1[ch];
#pragma unroll
            for (int lane = 0; lane < 2; ++lane) {
                const std::uint32_t key = (w >> (16 * lane)) & 0xffffu;
                if (key != 0xffffu)
                    keep2(k1[ch], k2[ch], ((key >> 7) << 23) + first + 2 * (key & 127u) + static_cast<std::uint32_t>(lane));
            }
        }
        p1[ch] = p2[ch] = 0xffffffffu;
    }
}

template <class Src, int kRowsB>
__global__ __launch_bounds__(kQueryThreads, 1) void knn_tc_kernel(const __grid_constant__ Src src) {
    using Shape = TcShape<kRowsB>;
    constexpr int kTcRowsB = Shape::rows_b;
    constexpr int kTcBytesB = Shape::bytes_b;
    extern __shared__ std::uint8_t dyn[];
    KnnJob j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    std::uint8_t* tileA = reinterpret_cast<std::uint8_t*>((reinterpret_cast<std::uintptr_t>(dyn) + 1023) & ~std::uintptr_t(1023));
    std::uint8_t* tileB = tileA + kTcBytesA;
    auto* bar = reinterpret_cast<std::uint64_t*>(tileB + kTcBytesB);
    auto* tmem_slot = reinterpret_cast<std::uint32_t*>(bar + 1);
    auto* stop = reinterpret_cast<int*>(tmem_slot + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int qt = local % j.q_tiles, split = local / j.q_tiles;
    int nq, nt;
    const bool ok = counts_valid(j, &nq, &nt);
    const int t0 = split * j.rows_per_split;
    const int t1 = ok ? min(nt, t0 + j.rows_per_split) : t0;
    const int q = qt * kTcRowsA + tid;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTcRowsB));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *stop = 0;
    }
    stage_pm_row(tileA, kTcRowsA, tid,
                 ok && q < nq ? j.query.rows + static_cast<std::size_t>(q) * j.query.stride : nullptr);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const std::uint32_t tmem = *tmem_slot;
    // four independent (smallest, second) key pairs, merged at the end: keys
    // are distinct (they carry the train index), so the merge is exact
    std::uint32_t k1[4] = {kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey};
    std::uint32_t k2[4] = {kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey};
    std::uint32_t phase = 0;
    std::uint32_t p1[4] = {~0u, ~0u, ~0u, ~0u}, p2[4] = {~0u, ~0u, ~0u, ~0u};  // packed chains of a stage
    for (int base = t0; base < t1; base += kTcRowsB) {
        for (int r = tid; r < kTcRowsB; r += kQueryThreads)
            stage_pm_row(tileB, kTcRowsB, r,
                         base + r < t1 ? j.train.rows + static_cast<std::size_t>(base + r) * j.train.stride : nullptr);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const std::uint32_t a0 = smem_u32(tileA), b0 = smem_u32(tileB);
#pragma unroll
            for (int s = 0; s < 8; ++s) {  // K = 256 in slices of 32 bytes
                const std::uint32_t koff = (s & 3) * 32;  // within the 128-byte swizzle atom
                const std::uint64_t da = sw128_desc(a0 + (s >> 2) * kTcRowsA * 128 + koff);
                const std::uint64_t db = sw128_desc(b0 + (s >> 2) * kTcRowsB * 128 + koff);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(Shape::idesc), "r"(s));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(bar))
                         : "memory");
        }
        // bounded wait for the MMA chain of this stage
        std::uint32_t done = 0;
        for (long long it = 0; it < kTcWaitLimit && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(phase)
                : "memory");
        }
        if (!done) *stop = 1;
        __syncthreads();
        if (*stop) break;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // this thread's query row: 256 dot products in 8 loads of 32 columns
#pragma unroll 1
        for (int c = 0; c < kTcRowsB; c += 32) {
            std::uint32_t v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + (static_cast<std::uint32_t>(warp * 32) << 16) + static_cast<std::uint32_t>(c)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            stage_keys32(v, c, base, t1, p1, p2);
        }
        fold_stage(p1, p2, static_cast<std::uint32_t>(base), k1, k2);
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();  // TMEM and the train stage are free for the next stage
    }
    const bool failed = *stop != 0;
    if (failed && tid == 0) atomicExch(&g_tc_error, 1);
#pragma unroll
    for (int u = 1; u < 4; ++u) {
        keep2(k1[0], k2[0], k1[u]);
        keep2(k1[0], k2[0], k2[u]);
    }
    if (!failed && q < j.query.capacity) {
        const bool active = ok && q < nq;
        const std::uint32_t a1 = active ? k1[0] : kEmptyKey, a2 = active ? k2[0] : kEmptyKey;
        if (j.splits == 1) {
            j.top2[q] = top2_from_keys(a1, a2);
        } else {
            j.partial[static_cast<std::size_t>(split) * j.query.capacity + q] = make_uint2(a1, a2);
        }
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcRowsB));
}

// ------------------------------------------------ pipelined tensor cores
//
// The same exact top-2 search as knn_tc_kernel, with the three kinds of work
// of a stage overlapped instead of run one after the other. Warp roles:
//   warps 0-7   epilogue: warp w reads TMEM lane quarter w % 4 (its 32
//               queries) and column half w / 4 of an accumulator, keeping
//               four top-2 key chains per thread;
//   warps 8-11  producers: expand the queries once, then each train stage
//               (256 rows) into one of two shared-memory stage buffers;
//   warp 12     one thread issues the 8 MMAs of a stage into one of two TMEM
//               accumulators (2 x 256 columns) and commits them.
// Stage s uses buffer and accumulator s % 2. mbarriers order the roles:
// full[b] (producers -> MMA), done[b] (MMA completion -> epilogue, and to
// the producers: the buffer is free again), free[b] (epilogue -> MMA: the
// accumulator was read). Every wait is bounded: when one runs out the block
// sets the error word and a stop flag that ends every role, waits (bounded)
// for its last MMA, frees its TMEM and leaves its outputs unwritten. The two
// column halves of a query meet in shared memory at the end.
constexpr int kPipeEpiWarps = 8, kPipeProdWarps = 4;
constexpr int kPipeThreads = (kPipeEpiWarps + kPipeProdWarps + 1) * 32;
constexpr int kPipeStage = 256;                                   // train rows per stage (MMA N)
constexpr int kPipeBytesB = kPipeStage * 256;
constexpr int kPipeSmem = kTcBytesA + 2 * kPipeBytesB + 1024 + 2048;  // + alignment + barriers and exchange
constexpr std::uint32_t kPipeIdesc = TcShape<kPipeStage>::idesc;

__device__ __forceinline__ void bar_init(std::uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void bar_arrive(std::uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
// Waits for the completion of the phase of `parity`; false when the wait ran
// out (then the stop flag is set) or another role stopped the block.
__device__ __forceinline__ bool bar_wait(std::uint64_t* bar, std::uint32_t parity, volatile int* stop) {
    for (long long it = 0; it < kTcWaitLimit; ++it) {
        std::uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && *stop) return false;
    }
    *stop = 1;
    return false;
}

template <class Src>
__global__ __launch_bounds__(kPipeThreads, 1) void knn_tc_pipe_kernel(const __grid_constant__ Src src) {
    extern __shared__ std::uint8_t dyn[];
    KnnJob j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    std::uint8_t* tileA = reinterpret_cast<std::uint8_t*>((reinterpret_cast<std::uintptr_t>(dyn) + 1023) & ~std::uintptr_t(1023));
    std::uint8_t* tileB[2] = {tileA + kTcBytesA, tileA + kTcBytesA + kPipeBytesB};
    auto* full = reinterpret_cast<std::uint64_t*>(tileA + kTcBytesA + 2 * kPipeBytesB);
    std::uint64_t* done = full + 2;
    std::uint64_t* freeb = full + 4;
    auto* tmem_slot = reinterpret_cast<std::uint32_t*>(full + 6);
    auto* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);
    auto* last_issued = reinterpret_cast<int*>(tmem_slot + 2);
    auto* xchg = reinterpret_cast<uint2*>(full + 8);  // [128] keys of column half 1
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int qt = local % j.q_tiles, split = local / j.q_tiles;
    int nq, nt;
    const bool ok = counts_valid(j, &nq, &nt);
    const int t0 = split * j.rows_per_split;
    const int t1 = ok ? min(nt, t0 + j.rows_per_split) : t0;
    const int stages = t1 > t0 ? (t1 - t0 + kPipeStage - 1) / kPipeStage : 0;
    if (warp == kPipeEpiWarps + kPipeProdWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * kPipeStage));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            bar_init(&full[b], kPipeProdWarps * 32);
            bar_init(&done[b], 1);
            bar_init(&freeb[b], kPipeEpiWarps * 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *stop = 0;
        *last_issued = -1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const std::uint32_t tmem = *tmem_slot;
    std::uint32_t k1[4] = {kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey};
    std::uint32_t k2[4] = {kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey};
    const int qrow = 32 * (warp & 3) + lane;  // epilogue: the query of this thread
    if (warp < kPipeEpiWarps) {
        const int half = warp >> 2;
        std::uint32_t p1[4] = {~0u, ~0u, ~0u, ~0u}, p2[4] = {~0u, ~0u, ~0u, ~0u};  // packed chains of a stage
        for (int s = 0; s < stages; ++s) {
            const int b = s & 1;
            // the TMEM loads below are warp-collective: the warp goes on only together
            if (!__all_sync(0xffffffffu, bar_wait(&done[b], (s >> 1) & 1, stop))) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int base = t0 + s * kPipeStage + half * (kPipeStage / 2);
#pragma unroll 1
            for (int c = 0; c < kPipeStage / 2; c += 32) {
                std::uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(tmem + (static_cast<std::uint32_t>((warp & 3) * 32) << 16) +
                          static_cast<std::uint32_t>(b * kPipeStage + half * (kPipeStage / 2) + c)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                stage_keys32(v, c, base, t1, p1, p2);
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            bar_arrive(&freeb[b]);
            fold_stage(p1, p2, static_cast<std::uint32_t>(base), k1, k2);
        }
    } else if (warp < kPipeEpiWarps + kPipeProdWarps) {
        const int p = tid - kPipeEpiWarps * 32;  // 0 .. 127
        const int q = qt * kTcRowsA + p;
        stage_pm_row(tileA, kTcRowsA, p, ok && q < nq ? j.query.rows + static_cast<std::size_t>(q) * j.query.stride
                                                      : nullptr);
        for (int s = 0; s < stages; ++s) {
            const int b = s & 1;
            if (s >= 2 && !bar_wait(&done[b], ((s - 2) >> 1) & 1, stop)) break;
            const int base = t0 + s * kPipeStage;
            for (int r = p; r < kPipeStage; r += kPipeProdWarps * 32)
                stage_pm_row(tileB[b], kPipeStage, r,
                             base + r < t1 ? j.train.rows + static_cast<std::size_t>(base + r) * j.train.stride : nullptr);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bar_arrive(&full[b]);
        }
    } else if (lane == 0) {
        const std::uint32_t a0 = smem_u32(tileA);
        for (int s = 0; s < stages; ++s) {
            const int b = s & 1;
            if (!bar_wait(&full[b], (s >> 1) & 1, stop)) break;
            if (s >= 2 && !bar_wait(&freeb[b], ((s - 2) >> 1) & 1, stop)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const std::uint32_t b0 = smem_u32(tileB[b]);
            const std::uint32_t d = tmem + static_cast<std::uint32_t>(b * kPipeStage);
#pragma unroll
            for (int k = 0; k < 8; ++k) {  // K = 256 in slices of 32 bytes
                const std::uint32_t koff = (k & 3) * 32;  // within the 128-byte swizzle atom
                const std::uint64_t da = sw128_desc(a0 + (k >> 2) * kTcRowsA * 128 + koff);
                const std::uint64_t db = sw128_desc(b0 + (k >> 2) * kPipeStage * 128 + koff);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                    "l"(da), "l"(db), "r"(kPipeIdesc), "r"(k));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&done[b]))
                         : "memory");
            *last_issued = s;
        }
    }
    __syncthreads();
    const bool failed = *stop != 0;
    if (warp < kPipeEpiWarps) {
#pragma unroll
        for (int u = 1; u < 4; ++u) {
            keep2(k1[0], k2[0], k1[u]);
            keep2(k1[0], k2[0], k2[u]);
        }
        if (warp >= 4) xchg[qrow] = make_uint2(k1[0], k2[0]);
    }
    __syncthreads();
    if (failed && tid == 0) atomicExch(&g_tc_error, 1);
    if (!failed && warp < 4) {
        const uint2 o = xchg[qrow];
        keep2(k1[0], k2[0], o.x);
        keep2(k1[0], k2[0], o.y);
        const int q = qt * kTcRowsA + qrow;
        if (q < j.query.capacity) {
            const bool active = ok && q < nq;
            const std::uint32_t a1 = active ? k1[0] : kEmptyKey, a2 = active ? k2[0] : kEmptyKey;
            if (j.splits == 1) {
                j.top2[q] = top2_from_keys(a1, a2);
            } else {
                j.partial[static_cast<std::size_t>(split) * j.query.capacity + q] = make_uint2(a1, a2);
            }
        }
    }
    if (warp == kPipeEpiWarps + kPipeProdWarps) {
        // after a stop, MMAs may still be running: wait (bounded) for the last one
        const int last = *last_issued;
        if (failed && last >= 0) {
            volatile int never = 0;
            bar_wait(&done[last & 1], (last >> 1) & 1, &never);
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kPipeStage));
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

// Whether query q's forward neighbours pass the ratio test (and the mutual
// check when there is a reverse direction); *p gets its Top2.
__device__ __forceinline__ bool accepted(const AcceptJob& j, int q, Top2* p) {
    *p = j.forward[q];
    bool accept = p->second_index >= 0 &&
                  (p->first_distance == 0 ? p->second_distance > 0 : p->first_distance < j.ratio * p->second_distance);
    if (accept && j.reverse) accept = j.reverse[p->first_index].first_index == q;
    return accept;
}

__device__ __forceinline__ void write_match(const AcceptJob& j, int at, int q, const Top2& p) {
    j.out.idx_a[at] = q;
    j.out.idx_b[at] = p.first_index;
    const double d = j.l2 ? sqrt(p.first_distance) : p.first_distance;
    j.out.distance[at] = d > FLT_MAX ? CUDART_INF_F : static_cast<float>(d);
}

// The accept step of one large query set over many blocks: block b counts
// the accepted queries among b * 1024 .. b * 1024 + 1023 ...
template <class Src>
__global__ __launch_bounds__(1024) void accept_count_kernel(const __grid_constant__ Src src, int* counts) {
    AcceptJob j;
    int local;
    if (!src.find(0, &j, &local)) return;
    const int q = blockIdx.x * 1024 + threadIdx.x;
    Top2 p;
    const int n = __syncthreads_count(q < j.capacity && accepted(j, q, &p));
    if (threadIdx.x == 0) counts[blockIdx.x] = n;
}

// ... and then writes them after the accepted queries of all earlier
// blocks, in query order; the last block writes the match count.
template <class Src>
__global__ __launch_bounds__(1024) void accept_scatter_kernel(const __grid_constant__ Src src, const int* counts) {
    __shared__ int warp_sum[32];
    __shared__ int offset;
    AcceptJob j;
    int local;
    if (!src.find(0, &j, &local)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        int s = 0;
        for (int b = lane; b < static_cast<int>(blockIdx.x); b += 32) s += counts[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) offset = s;
    }
    const int q = blockIdx.x * 1024 + threadIdx.x;
    Top2 p{};
    const bool accept = q < j.capacity && accepted(j, q, &p);
    const unsigned ballot = __ballot_sync(0xffffffffu, accept);
    if (lane == 0) warp_sum[warp] = __popc(ballot);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
        before += w < warp ? warp_sum[w] : 0;
        total += warp_sum[w];
    }
    if (accept) write_match(j, offset + before + __popc(ballot & ((1u << lane) - 1u)), q, p);
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *j.out.d_count = offset + total;
}

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
