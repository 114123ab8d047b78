// Host side of S2 (detect) and S3 (describe): argument checks, workspace
// layouts and launches of the kernels in s2s3_kernels.cuh.
//
// Argument checks and their order follow src/s2_s3/s2.cu:333-356 and
// src/s2_s3/s3.cu:168-184; workspace queries follow
// src/s2_s3/s2_s3_config.cpp:121-202 (sizes differ: this layout is the one
// these kernels need).
#include <algorithm>
#include <cmath>
#include <mutex>

#include "s2s3_internal.hpp"

namespace stitch::b200::s2s3 {

bool valid_image_shape(int w, int h) { return w > 0 && h > 0 && w <= INT_MAX / h; }

bool valid_gray(const ImageView& im) {
    return im.data && im.format == PixelFormat::GRAY8 && valid_image_shape(im.width, im.height) &&
           im.pitch_bytes >= im.width;
}

bool valid_detect_config(const s2::Config& c) {
    return c.fast_threshold >= 1 && c.fast_threshold <= 254 && c.max_keypoints >= 0 &&
           c.max_keypoints <= INT_MAX / s2::kCandidateFactor && std::isfinite(c.harris_k) &&
           c.harris_k >= 0.0f;
}

bool detect_layout(int w, int h, int k, DetectLayout* out) {
    if (!out || !valid_image_shape(w, h) || k < 0 || k > INT_MAX / s2::kCandidateFactor) return false;
    DetectLayout l{};
    const std::size_t pixels = static_cast<std::size_t>(w) * static_cast<std::size_t>(h);
    // strict 3x3 maxima inside the edge margin: at most one per 2x2 cell
    const std::size_t cells = (w > 2 * kEdge && h > 2 * kEdge)
                                  ? static_cast<std::size_t>((w - 2 * kEdge + 1) / 2) *
                                        static_cast<std::size_t>((h - 2 * kEdge + 1) / 2)
                                  : 0;
    if (cells > static_cast<std::size_t>(INT_MAX)) return false;
    l.max_maxima = static_cast<int>(cells);
    l.candidates = s2::kCandidateFactor * k;
    l.tiles_x = ceil_div(w, kFastTileW);
    l.tiles = l.tiles_x * ceil_div(h, kFastTileH);
    l.select_blocks = static_cast<int>(std::max<std::size_t>(1, (pixels + kSelectPx - 1) / kSelectPx));
    Layout lay;
    l.hist = lay.take(DetectLayout::hist_bytes, 1);
    l.params = lay.take(1, sizeof(SelectParams));
    l.keys = lay.take(static_cast<std::size_t>(l.candidates), sizeof(std::uint64_t));
    l.maxima = lay.take(std::max<std::size_t>(cells, 1), sizeof(std::uint64_t));
    if (!lay.ok) return false;
    l.total = lay.cursor;
    *out = l;
    return true;
}

bool describe_layout(int w, int h, DescribeLayout* out, int pitch_align) {
    if (!out || !valid_image_shape(w, h)) return false;
    Layout lay;
    DescribeLayout l{};
    l.blur_pitch = (w + pitch_align - 1) / pitch_align * pitch_align;
    l.blurred = lay.take(static_cast<std::size_t>(l.blur_pitch) * static_cast<std::size_t>(h), 1);
    if (!lay.ok) return false;
    l.total = lay.cursor;
    l.tiles_x = ceil_div(w, kBlurTileW);
    l.tiles = l.tiles_x * ceil_div(h, kBlurTileH);
    *out = l;
    return true;
}

DetectJob make_detect_job(const ImageView& im, const s2::Config& c, const Keypoints& out,
                          void* ws, const DetectLayout& l) {
    DetectJob j{};
    j.image = im.data;
    j.width = im.width;
    j.height = im.height;
    j.pitch = im.pitch_bytes;
    j.threshold = c.fast_threshold;
    j.max_keypoints = c.max_keypoints;
    j.harris_k = c.harris_k;
    j.maxima = at_offset<std::uint64_t>(ws, l.maxima);
    j.max_maxima = l.max_maxima;
    j.hist = at_offset<std::uint32_t>(ws, l.hist);
    j.params = at_offset<SelectParams>(ws, l.params);
    j.keys = at_offset<std::uint64_t>(ws, l.keys);
    j.x = out.x;
    j.y = out.y;
    j.response = out.response;
    j.count = out.d_count;
    j.tiles_x = l.tiles_x;
    j.tiles_x_magic = l.tiles_x > 1 ? static_cast<std::uint32_t>((0x100000000ull + static_cast<std::uint64_t>(l.tiles_x) - 1) /
                                                                 static_cast<std::uint64_t>(l.tiles_x))
                                    : 0u;
    j.tiles = l.tiles;
    j.select_blocks = l.select_blocks;
    j.candidates = l.candidates;
    return j;
}

int sort_smem_bytes(int candidates) {
    int n = candidates < kSortCap ? candidates : kSortCap;
    int p = kSortChunk;  // the kernel sorts at least one 64-key chunk
    while (p < n) p <<= 1;
    return p * static_cast<int>(sizeof(std::uint64_t));
}

namespace {

// Opt the shared-memory sort kernels in to more than 48 KB of dynamic shared
// memory, once per device.
template <class Src> bool enable_sort_smem() {
    static std::once_flag flags[64];
    static bool ok[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    std::call_once(flags[dev], [&] {
        ok[dev] = cudaFuncSetAttribute(sort_topk_kernel<Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSortCap * static_cast<int>(sizeof(std::uint64_t))) == cudaSuccess;
    });
    return ok[dev];
}

bool record(cudaEvent_t ev, cudaStream_t s) { return !ev || cudaEventRecord(ev, s) == cudaSuccess; }

Status detect(const ImageView& image, const s2::Config& config, const Keypoints& output, void* ws,
              std::size_t ws_bytes, cudaStream_t stream, const s2_s3::detail::S2Marks* marks) {
    if (!valid_gray(image) || !valid_detect_config(config) || !output.d_count ||
        !aligned(output.d_count, alignof(int)) || output.capacity < config.max_keypoints ||
        (config.max_keypoints > 0 && (!output.x || !output.y)))
        return Status::INVALID_ARGUMENT;
    const cudaEvent_t e_fast = marks ? marks->after_fast : nullptr;
    const cudaEvent_t e_select = marks ? marks->after_select : nullptr;
    const cudaEvent_t e_harris = marks ? marks->after_harris : nullptr;
    if (config.max_keypoints == 0 || image.width <= 2 * s2::kEdge || image.height <= 2 * s2::kEdge) {
        if (cudaMemsetAsync(output.d_count, 0, sizeof(int), stream) != cudaSuccess ||
            !record(e_fast, stream) || !record(e_select, stream) || !record(e_harris, stream))
            return Status::CUDA_ERROR;
        return launch_status();
    }
    DetectLayout l;
    if (!detect_layout(image.width, image.height, config.max_keypoints, &l)) return Status::INVALID_ARGUMENT;
    if (!ws || !aligned(ws, kWorkspaceAlign)) return Status::INVALID_ARGUMENT;
    if (ws_bytes < l.total) return Status::INSUFFICIENT_WORKSPACE;
    using Src = OneJob<DetectJob>;
    if (!enable_sort_smem<Src>()) return Status::CUDA_ERROR;
    const Src src{make_detect_job(image, config, output, ws, l)};
    if (cudaMemsetAsync(src.job.hist, 0, DetectLayout::hist_bytes, stream) != cudaSuccess)
        return Status::CUDA_ERROR;
    const int fast_grid = std::min(l.tiles, kSmCount * kFastCtasPerSm);
    fast_kernel<Src><<<fast_grid, kFastThreads, 0, stream>>>(src, src.job.counters() + kTileQueue, l.tiles);
    if (!record(e_fast, stream)) return Status::CUDA_ERROR;
    select_kernel<Src><<<l.select_blocks, 256, 0, stream>>>(src);
    ties_kernel<Src><<<1, kTieThreads, 0, stream>>>(src);
    if (!record(e_select, stream)) return Status::CUDA_ERROR;
    const int harris_blocks = ceil_div(l.candidates, kHarrisThreads);
    harris_kernel<Src><<<harris_blocks, kHarrisThreads, 0, stream>>>(src);
    if (!record(e_harris, stream)) return Status::CUDA_ERROR;
    sort_topk_kernel<Src><<<1, kSortThreads, sort_smem_bytes(l.candidates), stream>>>(src);
    if (l.candidates > kSortCap)
        rank_topk_kernel<Src><<<harris_blocks, kHarrisThreads, 0, stream>>>(src);
    note_launches(l.candidates > kSortCap ? 7 : 6);
    return launch_status();
}

Status describe(const ImageView& image, const Keypoints& kp, const Descriptors& out, void* ws,
                std::size_t ws_bytes, cudaStream_t stream, const s2_s3::detail::S3Marks* marks) {
    if (!valid_gray(image) || kp.capacity < 0 || !kp.d_count || !aligned(kp.d_count, alignof(int)) ||
        (kp.capacity > 0 && (!kp.x || !kp.y || !out.data)) || out.type != DescriptorType::BINARY_U8 ||
        out.dim != s3::kDescriptorBytes || out.row_stride_bytes < s3::kDescriptorBytes)
        return Status::INVALID_ARGUMENT;
    DescribeLayout l;
    if (!describe_layout(image.width, image.height, &l) || !ws || !aligned(ws, kWorkspaceAlign))
        return Status::INVALID_ARGUMENT;
    if (ws_bytes < l.total) return Status::INSUFFICIENT_WORKSPACE;
    const cudaEvent_t e_blur = marks ? marks->after_blur : nullptr;
    if (kp.capacity == 0) return record(e_blur, stream) ? Status::OK : Status::CUDA_ERROR;
    using Src = OneJob<DescribeJob>;
    const Src src{make_describe_job(image, kp, out, ws, l)};
    blur_kernel<Src><<<l.tiles, 256, 0, stream>>>(src);
    if (!record(e_blur, stream)) return Status::CUDA_ERROR;
    describe_kernel<Src><<<ceil_div(kp.capacity, kDescKeys), kDescWarps * 32, 0, stream>>>(src);
    note_launches(2);
    return launch_status();
}

}  // namespace

DescribeJob make_describe_job(const ImageView& im, const Keypoints& kp, const Descriptors& out, void* ws,
                              const DescribeLayout& l) {
    DescribeJob j{};
    j.image = im.data;
    j.width = im.width;
    j.height = im.height;
    j.pitch = im.pitch_bytes;
    j.blurred = at_offset<std::uint8_t>(ws, l.blurred);
    j.blur_pitch = l.blur_pitch;
    j.x = kp.x;
    j.y = kp.y;
    j.count = kp.d_count;
    j.capacity = kp.capacity;
    j.out = static_cast<std::uint8_t*>(out.data);
    j.row_stride = out.row_stride_bytes;
    j.tiles_x = l.tiles_x;
    j.tiles = l.tiles;
    return j;
}

}  // namespace stitch::b200::s2s3

namespace stitch {

namespace s2 {
Status s2_workspace_bytes(int width, int height, const Config& config, std::size_t* bytes) {
    using namespace b200::s2s3;
    if (!bytes) return Status::INVALID_ARGUMENT;
    *bytes = 0;
    if (!valid_detect_config(config) || !valid_image_shape(width, height)) return Status::INVALID_ARGUMENT;
    if (config.max_keypoints == 0) return Status::OK;
    DetectLayout l;
    if (!detect_layout(width, height, config.max_keypoints, &l)) return Status::INVALID_ARGUMENT;
    *bytes = l.total;
    return Status::OK;
}

Status s2_detect(const ImageView& image, const Config& config, Keypoints output, void* workspace,
                 std::size_t workspace_bytes, cudaStream_t stream) {
    return b200::s2s3::detect(image, config, output, workspace, workspace_bytes, stream, nullptr);
}
}  // namespace s2

namespace s3 {
Status s3_workspace_bytes(int width, int height, std::size_t* bytes) {
    using namespace b200::s2s3;
    if (!bytes) return Status::INVALID_ARGUMENT;
    *bytes = 0;
    DescribeLayout l;
    if (!describe_layout(width, height, &l)) return Status::INVALID_ARGUMENT;
    *bytes = l.total;
    return Status::OK;
}

Status s3_describe(const ImageView& image, const Keypoints& keypoints, Descriptors output,
                   void* workspace, std::size_t workspace_bytes, cudaStream_t stream) {
    return b200::s2s3::describe(image, keypoints, output, workspace, workspace_bytes, stream, nullptr);
}
}  // namespace s3

namespace s2_s3::detail {
Status s2_detect_marked(const ImageView& image, const s2::Config& config, Keypoints output,
                        void* workspace, std::size_t workspace_bytes, cudaStream_t stream,
                        const S2Marks& marks) {
    return b200::s2s3::detect(image, config, output, workspace, workspace_bytes, stream, &marks);
}
Status s3_describe_marked(const ImageView& image, const Keypoints& keypoints, Descriptors output,
                          void* workspace, std::size_t workspace_bytes, cudaStream_t stream,
                          const S3Marks& marks) {
    return b200::s2s3::describe(image, keypoints, output, workspace, workspace_bytes, stream, &marks);
}
}  // namespace s2_s3::detail

}  // namespace stitch
