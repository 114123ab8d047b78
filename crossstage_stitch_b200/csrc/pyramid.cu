// Scale-pyramid S2/S3 of one image: layers 1..L-1 resized in a chain, then
// S2 and S3 of every layer in the same launches (the layers' jobs travel as
// kernel parameters; the FAST kernel also writes each layer's blur), each
// layer's keypoints and descriptors written by the describe kernel straight
// into the image's concatenated outputs in level-0 coordinates.
//
// The reference has no pyramid (docs/decisions/s2-s3-orb.md:84): its S2/S3
// are single-level (src/s2_s3/s2.cu, src/s2_s3/s3.cu). The layer semantics
// here are OpenCV ORB's (modules/features2d/src/orb.cpp: getScale, layer
// sizes, nfeaturesPerLevel, resize with INTER_LINEAR_EXACT, pt *= scale),
// and each layer runs the reference's single-level S2/S3 unchanged.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "s2s3_internal.hpp"

namespace stitch::b200::s2s3 {

bool valid_pyramid(int levels, float sf) {
    if (levels < 1 || levels > kMaxLevels) return false;
    return levels == 1 || (std::isfinite(sf) && sf > 1.0f && sf <= 16.0f);
}

LevelPlan level_plan(int w, int h, int k, int levels, float sf) {
    LevelPlan p;
    // budgets: cvRound of a float geometric series, the rest on the last layer
    if (levels == 1) {
        p.budget[0] = k;
    } else {
        const float factor = static_cast<float>(1.0 / static_cast<double>(sf));
        float d = static_cast<float>(k) * (1.0f - factor) /
                  (1.0f - static_cast<float>(std::pow(static_cast<double>(factor), static_cast<double>(levels))));
        int used = 0;
        for (int l = 0; l < levels - 1; ++l) {
            int n = static_cast<int>(std::lrintf(d));
            if (n > k - used) n = k - used;
            p.budget[l] = n;
            used += n;
            d = d * factor;
        }
        p.budget[levels - 1] = k - used > 0 ? k - used : 0;
    }
    for (int l = 0; l < levels; ++l) {
        const float s = static_cast<float>(std::pow(static_cast<double>(sf), static_cast<double>(l)));
        const float inv = 1.0f / s;
        const int lw = l ? static_cast<int>(std::lrintf(static_cast<float>(w) * inv)) : w;
        const int lh = l ? static_cast<int>(std::lrintf(static_cast<float>(h) * inv)) : h;
        if (lw <= 2 * kEdge || lh <= 2 * kEdge) break;
        p.width[l] = lw;
        p.height[l] = lh;
        p.scale[l] = s;
        p.levels = l + 1;
    }
    return p;
}

// Rows of the layer images start on 16-byte boundaries.
int layer_pitch(int width) { return (width + 15) / 16 * 16; }

bool pyramid_layout(int w, int h, int k, int levels, float sf, PyramidLayout* out, int resize_tile_h) {
    if (!out || !valid_image_shape(w, h) || k < 0 || k > INT_MAX / s2::kCandidateFactor ||
        !valid_pyramid(levels, sf))
        return false;
    PyramidLayout l{};
    if (resize_tile_h < 16 || resize_tile_h > kResizeTileH || resize_tile_h % 16) return false;
    l.resize_tile_h = resize_tile_h;
    l.plan = level_plan(w, h, k, levels, sf);
    const int n = l.plan.levels;
    // blur tiles of every layer (the describe layout's tile grid)
    l.blur_first[0] = 0;
    for (int i = 0; i < n; ++i)
        l.blur_first[i + 1] = l.blur_first[i] + ceil_div(l.plan.width[i], kBlurTileW) * ceil_div(l.plan.height[i], kBlurTileH);
    const std::size_t blur_total = static_cast<std::size_t>(std::max(l.blur_first[n], 1));
    Layout lay;
    l.counts = lay.take(static_cast<std::size_t>(n > 0 ? n : 1), sizeof(int));
    l.hists = lay.take(static_cast<std::size_t>(n > 0 ? n : 1) * kHistWords, sizeof(std::uint32_t));
    l.queue = lay.take(2, sizeof(std::uint32_t));  // FAST tile queue, blur-list count
    l.marks = lay.take(blur_total, sizeof(std::uint32_t));
    l.zeroed_bytes = lay.cursor;
    l.blur_list = lay.take(blur_total, sizeof(uint2));
    for (int i = 0; i < n; ++i) {
        const int lw = l.plan.width[i], lh = l.plan.height[i];
        const std::size_t kk = static_cast<std::size_t>(l.plan.budget[i] > 0 ? l.plan.budget[i] : 1);
        l.image[i] = i ? lay.take(static_cast<std::size_t>(layer_pitch(lw)) * static_cast<std::size_t>(lh), 1) : 0;
        l.kx[i] = lay.take(kk, sizeof(float));
        l.ky[i] = lay.take(kk, sizeof(float));
        l.kr[i] = lay.take(kk, sizeof(float));
        if (!detect_layout(lw, lh, l.plan.budget[i], &l.det[i]) || !describe_layout(lw, lh, &l.des[i], 16))
            return false;
        l.detect[i] = lay.take(l.det[i].total, 1);
        l.describe[i] = lay.take(l.des[i].total, 1);
        l.resize_tiles[i] = i ? ceil_div(lw, kResizeTileW) * ceil_div(lh, resize_tile_h) : 0;
    }
    if (!lay.ok) return false;
    l.total = lay.cursor;
    *out = l;
    return true;
}

void make_pyramid_jobs(const ImageView& im, const s2::Config& c, const Keypoints& out, const Descriptors& desc,
                       void* ws, const PyramidLayout& l, const PyramidShared& sh, PyramidJobs* jobs) {
    int* counts = sh.counts;
    const LevelPlan& p = l.plan;
    for (int i = 0; i < p.levels; ++i) {
        ImageView layer = im;
        if (i) {
            layer.data = at_offset<std::uint8_t>(ws, l.image[i]);
            layer.width = p.width[i];
            layer.height = p.height[i];
            layer.pitch_bytes = layer_pitch(p.width[i]);
            ResizeJob r{};
            r.src = i == 1 ? im.data : at_offset<std::uint8_t>(ws, l.image[i - 1]);
            r.src_width = p.width[i - 1];
            r.src_height = p.height[i - 1];
            r.src_pitch = i == 1 ? im.pitch_bytes : layer_pitch(p.width[i - 1]);
            r.dst = const_cast<std::uint8_t*>(layer.data);
            r.width = p.width[i];
            r.height = p.height[i];
            r.pitch = layer.pitch_bytes;
            r.tiles_x = ceil_div(p.width[i], kResizeTileW);
            r.tiles = l.resize_tiles[i];
            r.scale_x = linear_exact_scale(r.src_width, r.width);
            r.scale_y = linear_exact_scale(r.src_height, r.height);
            jobs->resize[i] = r;
        }
        s2::Config lc = c;
        lc.max_keypoints = p.budget[i];
        const Keypoints staged{at_offset<float>(ws, l.kx[i]), at_offset<float>(ws, l.ky[i]),
                               at_offset<float>(ws, l.kr[i]), p.budget[i], counts + i};
        DetectJob d = make_detect_job(layer, lc, staged, at_offset<void>(ws, l.detect[i]), l.det[i]);
        d.hist = sh.hists + static_cast<std::size_t>(i) * kHistWords;
        d.blur_marks = sh.blur_marks + l.blur_first[i];
        d.blur_list = sh.blur_list;
        d.blur_count = sh.blur_count;
        d.job = sh.job0 + i;
        jobs->detect[i] = d;
        DescribeJob s = make_describe_job(layer, staged, desc, at_offset<void>(ws, l.describe[i]), l.des[i]);
        s.response = staged.response;
        s.out_x = out.x;
        s.out_y = out.y;
        s.out_response = out.response;
        s.out_count = out.d_count;
        s.level_counts = counts;
        s.level = i;
        s.scale = p.scale[i];
        jobs->describe[i] = s;
    }
}

void pyramid_detect_blocks(const PyramidLayout& l, int i, int (&blocks)[kDetectKinds]) {
    const bool active = i < l.plan.levels && l.plan.budget[i] > 0;
    const DetectLayout& d = l.det[i];
    blocks[kFastKind] = active ? d.tiles : 0;
    blocks[kSelectKind] = active ? d.select_blocks : 0;
    blocks[kHarrisKind] = active ? ceil_div(d.candidates, kHarrisThreads) : 0;
    blocks[kSortKind] = active ? 1 : 0;
}

void pyramid_describe_blocks(const PyramidLayout& l, int i, int (&blocks)[kDescribeKinds]) {
    const bool active = i < l.plan.levels && l.plan.budget[i] > 0;
    blocks[kBlurKind] = 0;  // on demand: blur_tiles_kernel takes the flagged tiles from a list
    blocks[kDescKind] = active ? ceil_div(l.plan.budget[i], kDescKeys) : 0;
}

namespace {

using DetSrc = InlineTable<DetectJob, kMaxLevels, kDetectKinds>;
using DesSrc = InlineTable<DescribeJob, kMaxLevels, kDescribeKinds>;
static_assert(sizeof(DetSrc) <= 4096 && sizeof(DesSrc) <= 4096, "layer tables must fit the kernel parameters");

bool enable_pyramid_sort_smem() {
    static std::once_flag flags[64];
    static bool ok[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    std::call_once(flags[dev], [&] {
        ok[dev] = cudaFuncSetAttribute(sort_topk_kernel<DetSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSortCap * static_cast<int>(sizeof(std::uint64_t))) == cudaSuccess;
    });
    return ok[dev];
}

}  // namespace

Status pyramid_workspace_bytes(int w, int h, const s2::Config& c, int levels, float sf, std::size_t* bytes) {
    if (!bytes) return Status::INVALID_ARGUMENT;
    *bytes = 0;
    if (!valid_detect_config(c) || !valid_image_shape(w, h) || !valid_pyramid(levels, sf))
        return Status::INVALID_ARGUMENT;
    PyramidLayout l;
    if (!pyramid_layout(w, h, c.max_keypoints, levels, sf, &l, kSingleResizeTileH)) return Status::INVALID_ARGUMENT;
    *bytes = l.total;
    return Status::OK;
}

Status pyramid_detect_describe(const ImageView& image, const s2::Config& c, int levels, float sf,
                               const Keypoints& out, const Descriptors& desc, void* ws, std::size_t ws_bytes,
                               cudaStream_t stream) {
    if (!valid_gray(image) || !valid_detect_config(c) || !valid_pyramid(levels, sf) || !out.d_count ||
        !aligned(out.d_count, alignof(int)) || out.capacity < c.max_keypoints ||
        (c.max_keypoints > 0 && (!out.x || !out.y || !desc.data)) || desc.type != DescriptorType::BINARY_U8 ||
        desc.dim != s3::kDescriptorBytes || desc.row_stride_bytes < s3::kDescriptorBytes)
        return Status::INVALID_ARGUMENT;
    PyramidLayout l;
    if (!pyramid_layout(image.width, image.height, c.max_keypoints, levels, sf, &l, kSingleResizeTileH))
        return Status::INVALID_ARGUMENT;
    if (!ws || !aligned(ws, kWorkspaceAlign)) return Status::INVALID_ARGUMENT;
    if (ws_bytes < l.total) return Status::INSUFFICIENT_WORKSPACE;
    if (cudaMemsetAsync(out.d_count, 0, sizeof(int), stream) != cudaSuccess ||
        cudaMemsetAsync(ws, 0, l.zeroed_bytes, stream) != cudaSuccess)
        return Status::CUDA_ERROR;
    const int n = l.plan.levels;
    if (n == 0 || c.max_keypoints == 0) return launch_status();
    if (!enable_pyramid_sort_smem()) return Status::CUDA_ERROR;
    PyramidJobs jobs;
    std::uint32_t* queue = at_offset<std::uint32_t>(ws, l.queue);
    const PyramidShared sh{at_offset<int>(ws, l.counts), at_offset<std::uint32_t>(ws, l.hists),
                           at_offset<std::uint32_t>(ws, l.marks), at_offset<uint2>(ws, l.blur_list), queue + 1, 0};
    make_pyramid_jobs(image, c, out, desc, ws, l, sh, &jobs);
    int launches = 0;
    for (int i = 1; i < n; ++i) {
        resize_kernel<OneJob<ResizeJob>, kSingleResizeTileH>
            <<<l.resize_tiles[i], 256, 0, stream>>>(OneJob<ResizeJob>{jobs.resize[i]}, 0);
        ++launches;
    }
    DetSrc det{};
    DesSrc des{};
    det.n = des.n = n;
    int max_cand = 0;
    for (int i = 0; i < n; ++i) {
        det.jobs[i] = jobs.detect[i];
        des.jobs[i] = jobs.describe[i];
        int db[kDetectKinds], sb[kDescribeKinds];
        pyramid_detect_blocks(l, i, db);
        pyramid_describe_blocks(l, i, sb);
        for (int k = 0; k < kDetectKinds; ++k) det.first[k][i + 1] = det.first[k][i] + db[k];
        for (int k = 0; k < kDescribeKinds; ++k) des.first[k][i + 1] = des.first[k][i] + sb[k];
        if (db[kSortKind]) max_cand = max_cand > l.det[i].candidates ? max_cand : l.det[i].candidates;
    }
    auto blocks = [&](int kind) { return det.first[kind][n]; };
    if (blocks(kFastKind)) {
        fast_kernel<DetSrc><<<std::min(blocks(kFastKind), kSmCount * kFastCtasPerSm), kFastThreads, 0, stream>>>(
            det, queue, blocks(kFastKind));
        select_kernel<DetSrc><<<blocks(kSelectKind), 256, 0, stream>>>(det);
        ties_kernel<DetSrc><<<blocks(kSortKind), kTieThreads, 0, stream>>>(det);
        harris_kernel<DetSrc><<<blocks(kHarrisKind), kHarrisThreads, 0, stream>>>(det);
        sort_topk_kernel<DetSrc><<<blocks(kSortKind), kSortThreads, sort_smem_bytes(max_cand), stream>>>(det);
        launches += 5;
        if (max_cand > kSortCap) {
            rank_topk_kernel<DetSrc><<<blocks(kHarrisKind), kHarrisThreads, 0, stream>>>(det);
            ++launches;
        }
        blur_tiles_kernel<DesSrc><<<std::max(1, std::min(l.blur_first[n], kSmCount * kBlurCtasPerSm)), 256, 0, stream>>>(
            des, at_offset<uint2>(ws, l.blur_list), queue + 1);
        ++launches;
    }
    if (des.first[kDescKind][n]) {
        describe_kernel<DesSrc><<<des.first[kDescKind][n], kDescWarps * 32, 0, stream>>>(des);
        ++launches;
    }
    note_launches(launches);
    return launch_status();
}

}  // namespace stitch::b200::s2s3
