// Host side of S4: argument checks, workspace layout and launches.
//
// Checks and their order follow src/s4/s4.cu:79-109 (valid_input/valid_pair)
// and :269-334 (s4_knn_top2, s4_match, s4_forward_neighbors); the workspace
// query follows src/s4/s4_config.cpp:8-32 in its validation. The forward
// Top2 array sits at offset 0 of the workspace, where s4_forward_neighbors
// exposes it to later consumers.
#include <algorithm>
#include <cmath>
#include <limits>

#include "s4_internal.hpp"

namespace stitch::b200::s4k {

bool valid_side(const Keypoints& k, const Descriptors& d) {
    if (k.capacity < 0 || !k.d_count || !aligned(k.d_count, alignof(int)) || d.dim <= 0 ||
        d.row_stride_bytes <= 0)
        return false;
    std::size_t elem;
    if (d.type == DescriptorType::BINARY_U8) elem = 1;
    else if (d.type == DescriptorType::FLOAT32) elem = sizeof(float);
    else return false;
    if (static_cast<std::size_t>(d.dim) > std::numeric_limits<std::size_t>::max() / elem) return false;
    const std::size_t row = static_cast<std::size_t>(d.dim) * elem;
    if (row > static_cast<std::size_t>(d.row_stride_bytes) ||
        static_cast<std::size_t>(d.row_stride_bytes) % elem != 0 || (k.capacity && !d.data) ||
        !aligned(d.data, elem))
        return false;
    if (k.capacity) {
        const std::size_t last = static_cast<std::size_t>(k.capacity - 1);
        const std::size_t limit = std::numeric_limits<std::size_t>::max();
        if (last > (limit - row) / static_cast<std::size_t>(d.row_stride_bytes)) return false;
        const std::size_t bytes = last * static_cast<std::size_t>(d.row_stride_bytes) + row;
        if (reinterpret_cast<std::uintptr_t>(d.data) > std::numeric_limits<std::uintptr_t>::max() - bytes)
            return false;
    }
    return true;
}

bool valid_pair(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db) {
    return valid_side(a, da) && valid_side(b, db) && da.type == db.type && da.dim == db.dim;
}

bool popc_eligible(const Descriptors& q, const Descriptors& t, int capacity_train) {
    return q.type == DescriptorType::BINARY_U8 && q.dim == 32 && aligned(q.data, 16) &&
           aligned(t.data, 16) && q.row_stride_bytes % 16 == 0 && t.row_stride_bytes % 16 == 0 &&
           capacity_train < kMaxPopcTrain;
}

// Train partitions so that one pair of images fills about two waves of
// blocks; depends only on the capacities, so the workspace size does too.
void plan_split(int capacity_q, int capacity_t, int* q_tiles, int* splits, int* rows_per_split) {
    const int qt = std::max(1, ceil_div(std::max(capacity_q, 1), kQueryThreads));
    const int stages = std::max(1, ceil_div(std::max(capacity_t, 1), kTrainStage));
    int s = std::max(1, ceil_div(2 * kSmCount, qt));
    s = std::min(s, stages);
    const int per = ceil_div(stages, s) * kTrainStage;
    *q_tiles = qt;
    *rows_per_split = per;
    *splits = ceil_div(std::max(capacity_t, 1), per);
}

bool match_layout(int capacity_a, int capacity_b, bool cross, MatchLayout* out) {
    if (capacity_a < 0 || capacity_b < 0) return false;
    MatchLayout l{};
    const std::size_t a = static_cast<std::size_t>(capacity_a), b = static_cast<std::size_t>(capacity_b);
    l.forward = 0;
    std::size_t cursor = a * sizeof(Top2);
    l.reverse = cursor;
    if (cross) cursor += b * sizeof(Top2);
    plan_split(capacity_a, capacity_b, &l.fq_tiles, &l.fsplits, &l.frows);
    plan_split(capacity_b, capacity_a, &l.rq_tiles, &l.rsplits, &l.rrows);
    l.fpartial = cursor;
    if (l.fsplits > 1) cursor += static_cast<std::size_t>(l.fsplits) * a * sizeof(uint2);
    l.rpartial = cursor;
    if (cross && l.rsplits > 1) cursor += static_cast<std::size_t>(l.rsplits) * b * sizeof(uint2);
    l.accept_counts = cursor;
    cursor += static_cast<std::size_t>((capacity_a + 1023) / 1024) * sizeof(int);
    l.total = cursor;
    *out = l;
    return true;
}

KnnJob make_knn_job(const Keypoints& qk, const Descriptors& qd, const Keypoints& tk, const Descriptors& td,
                    int q_tiles, int splits, int rows, uint2* partial, Top2* top2) {
    KnnJob j{};
    j.query = Side{static_cast<const std::uint8_t*>(qd.data), qd.row_stride_bytes, qk.capacity, qk.d_count};
    j.train = Side{static_cast<const std::uint8_t*>(td.data), td.row_stride_bytes, tk.capacity, tk.d_count};
    j.q_tiles = q_tiles;
    j.splits = splits;
    j.rows_per_split = rows;
    j.partial = partial;
    j.top2 = top2;
    return j;
}

namespace {
// The tensor-core matcher measured 2.7x faster than __popc on the batched
// 64-pair workload (0.139 vs 0.375 ms per step), so it is the default. The
// choice belongs to the calling host thread.
thread_local int t_matcher = kMatcherTensor;
}  // namespace

int matcher() { return t_matcher; }

Status check_match_args(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db,
                        const s4::Config& config, const Matches& output, std::size_t* required) {
    *required = 0;
    if (s4::s4_workspace_bytes(a.capacity, b.capacity, config, required) != Status::OK ||
        !valid_pair(a, da, b, db) || output.capacity < a.capacity || !output.d_count ||
        !aligned(output.d_count, alignof(int)) ||
        (a.capacity && (!output.idx_a || !output.idx_b || !output.distance ||
                        !aligned(output.idx_a, alignof(int32_t)) || !aligned(output.idx_b, alignof(int32_t)) ||
                        !aligned(output.distance, alignof(float)))))
        return Status::INVALID_ARGUMENT;
    return Status::OK;
}
bool valid_matcher(int kind) { return kind >= kMatcherPopc && kind <= kMatcherTensorPipe; }

namespace {

// One direction of the exact top-2 search into `out` (capacity of the query
// side entries); partial may be null only when the plan has one split.
Status launch_direction(const Keypoints& qk, const Descriptors& qd, const Keypoints& tk,
                        const Descriptors& td, Top2* out, uint2* partial, int q_tiles, int splits,
                        int rows, cudaStream_t stream) {
    if (qk.capacity == 0) return Status::OK;
    if (popc_eligible(qd, td, tk.capacity)) {
        using Src = OneJob<KnnJob>;
        const Src src{make_knn_job(qk, qd, tk, td, q_tiles, splits, rows, partial, out)};
        if (is_tensor(matcher())) {
            // Two tensor-core blocks fit on an SM (shared memory), so a grid
            // above 2 x 148 blocks leaves a second, mostly idle wave: use the
            // largest train partition count whose grid fits one wave (never
            // more partitions than the workspace plan holds).
            const int stages = ceil_div(std::max(tk.capacity, 1), kTrainStage);
            const int want =
                std::min(splits, std::max(1, tc_blocks_per_sm(matcher()) * kSmCount / std::max(q_tiles, 1)));
            const int tc_rows = ceil_div(stages, want) * kTrainStage;
            const int tc_splits = ceil_div(std::max(tk.capacity, 1), tc_rows);
            const Src tc{make_knn_job(qk, qd, tk, td, q_tiles, tc_splits, tc_rows, partial, out)};
            if (!launch_tc(matcher(), q_tiles * tc_splits, tc, stream)) return Status::CUDA_ERROR;
            if (tc_splits > 1) knn_merge_kernel<Src><<<ceil_div(qk.capacity, 256), 256, 0, stream>>>(tc);
            note_launches(tc_splits > 1 ? 2 : 1);
        } else {
            knn_popc_kernel<Src, 1><<<q_tiles * splits, kQueryThreads, 0, stream>>>(src);
            if (splits > 1) knn_merge_kernel<Src><<<ceil_div(qk.capacity, 256), 256, 0, stream>>>(src);
            note_launches(splits > 1 ? 2 : 1);
        }
    } else {
        const Side q{static_cast<const std::uint8_t*>(qd.data), qd.row_stride_bytes, qk.capacity, qk.d_count};
        const Side t{static_cast<const std::uint8_t*>(td.data), td.row_stride_bytes, tk.capacity, tk.d_count};
        const int blocks = std::min(ceil_div(qk.capacity, 8), 65535);
        if (qd.type == DescriptorType::FLOAT32)
            knn_generic_kernel<true><<<blocks, 256, 0, stream>>>(q, t, qd.dim, out);
        else
            knn_generic_kernel<false><<<blocks, 256, 0, stream>>>(q, t, qd.dim, out);
        note_launches(1);
    }
    return launch_status();
}

}  // namespace

}  // namespace stitch::b200::s4k

namespace stitch::s4 {

using namespace ::stitch::b200;
using namespace ::stitch::b200::s4k;

Status s4_workspace_bytes(int capacity_a, int capacity_b, const Config& config, std::size_t* bytes) {
    if (!bytes) return Status::INVALID_ARGUMENT;
    *bytes = 0;
    if (capacity_a < 0 || capacity_b < 0 || !std::isfinite(config.ratio_threshold) ||
        config.ratio_threshold <= 0 || config.ratio_threshold >= 1)
        return Status::INVALID_ARGUMENT;
    if (capacity_a == 0) return Status::OK;
    MatchLayout l;
    if (!match_layout(capacity_a, capacity_b, config.cross_check, &l)) return Status::INVALID_ARGUMENT;
    *bytes = l.total;
    return Status::OK;
}

Status s4_knn_top2(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db,
                   Top2* output, cudaStream_t stream) {
    if (!valid_pair(a, da, b, db) || (a.capacity && (!output || !aligned(output, alignof(Top2)))))
        return Status::INVALID_ARGUMENT;
    if (!a.capacity) return Status::OK;
    // No workspace here: a single train partition writes Top2 directly.
    const int q_tiles = ceil_div(a.capacity, kQueryThreads);
    const int rows = std::max(kTrainStage, ceil_div(std::max(b.capacity, 1), kTrainStage) * kTrainStage);
    return launch_direction(a, da, b, db, output, nullptr, q_tiles, 1, rows, stream);
}

Status s4_match(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db,
                const Config& config, Matches output, void* workspace, std::size_t workspace_bytes,
                cudaStream_t stream) {
    std::size_t required = 0;
    if (check_match_args(a, da, b, db, config, output, &required) != Status::OK) return Status::INVALID_ARGUMENT;
    if (workspace_bytes < required || (required && !workspace)) return Status::INSUFFICIENT_WORKSPACE;
    if (required && (!aligned(workspace, alignof(Top2)) ||
                     reinterpret_cast<std::uintptr_t>(workspace) >
                         std::numeric_limits<std::uintptr_t>::max() - required))
        return Status::INVALID_ARGUMENT;
    if (!a.capacity)
        return cudaMemsetAsync(output.d_count, 0, sizeof(int), stream) == cudaSuccess ? Status::OK
                                                                                       : Status::CUDA_ERROR;
    MatchLayout l;
    match_layout(a.capacity, b.capacity, config.cross_check, &l);
    auto* forward = at_offset<Top2>(workspace, l.forward);
    auto* reverse = config.cross_check ? at_offset<Top2>(workspace, l.reverse) : nullptr;
    Status s = launch_direction(a, da, b, db, forward, at_offset<uint2>(workspace, l.fpartial), l.fq_tiles,
                                l.fsplits, l.frows, stream);
    if (s != Status::OK) return s;
    if (config.cross_check && b.capacity) {
        s = launch_direction(b, db, a, da, reverse, at_offset<uint2>(workspace, l.rpartial), l.rq_tiles,
                             l.rsplits, l.rrows, stream);
        if (s != Status::OK) return s;
    }
    AcceptJob aj{};
    aj.forward = forward;
    aj.reverse = reverse;
    aj.capacity = a.capacity;
    aj.l2 = da.type == DescriptorType::FLOAT32;
    aj.ratio = aj.l2 ? config.ratio_threshold * config.ratio_threshold : config.ratio_threshold;
    aj.out = output;
    if (a.capacity <= 1024) {
        accept_kernel<OneJob<AcceptJob>><<<1, 1024, 0, stream>>>(OneJob<AcceptJob>{aj});
        note_launches(1);
    } else {  // many blocks: counts per 1024 queries, then offsets and the compaction
        const int blocks = ceil_div(a.capacity, 1024);
        int* counts = at_offset<int>(workspace, l.accept_counts);
        accept_count_kernel<OneJob<AcceptJob>><<<blocks, 1024, 0, stream>>>(OneJob<AcceptJob>{aj}, counts);
        accept_scatter_kernel<OneJob<AcceptJob>><<<blocks, 1024, 0, stream>>>(OneJob<AcceptJob>{aj}, counts);
        note_launches(2);
    }
    return launch_status();
}

Status s4_forward_neighbors(int capacity_a, int capacity_b, const Config& config, const void* workspace,
                            std::size_t workspace_bytes, const Top2** output) {
    std::size_t required = 0;
    if (!output || s4_workspace_bytes(capacity_a, capacity_b, config, &required) != Status::OK ||
        !capacity_a || !workspace || workspace_bytes < required || !aligned(workspace, alignof(Top2)))
        return Status::INVALID_ARGUMENT;
    *output = static_cast<const Top2*>(workspace);
    return Status::OK;
}

}  // namespace stitch::s4

extern "C" {

int stitch_s4_set_matcher(int kind) {
    using namespace stitch::b200::s4k;
    if (!valid_matcher(kind)) return static_cast<int>(stitch::Status::INVALID_ARGUMENT);
    t_matcher = kind;
    return 0;
}

int stitch_s4_matcher(void) { return stitch::b200::s4k::matcher(); }

int stitch_s4_tc_errors(void) {
    using namespace stitch::b200::s4k;
    int mine = 0;
    if (cudaMemcpyFromSymbol(&mine, g_tc_error, sizeof(int)) != cudaSuccess) return -1;
    const int zero = 0;
    if (mine && cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    const int batch = take_batch_tc_error();
    return batch < 0 ? -1 : (mine | batch);
}

}  // extern "C"
