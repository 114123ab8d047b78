// Layouts and job builders shared by the per-image S2/S3 calls and the
// batched chain.
#pragma once

#include "s2s3_kernels.cuh"

namespace stitch::b200::s2s3 {

// S2 workspace of one image (or pyramid layer). `hist` holds the 256
// histogram bins and then the kDetectCounters counters, zeroed together
// (hist_bytes) before each run.
struct DetectLayout {
    std::size_t maxima, hist, params, keys, total;
    int max_maxima, candidates, tiles_x, tiles, select_blocks;
    static constexpr std::size_t hist_bytes = kHistWords * sizeof(std::uint32_t);
};

struct DescribeLayout {
    std::size_t blurred, total;  // blurred image first, at offset 0
    int blur_pitch;
    int tiles_x, tiles;
};

bool valid_image_shape(int w, int h);
bool valid_gray(const ImageView& im);
bool valid_detect_config(const s2::Config& c);
bool detect_layout(int w, int h, int k, DetectLayout* out);
// pitch_align 1: the blurred image is dense (the per-image S3 call); 16:
// rows start on 16-byte boundaries (the fused batched and pyramid paths).
bool describe_layout(int w, int h, DescribeLayout* out, int pitch_align = 1);
DetectJob make_detect_job(const ImageView& im, const s2::Config& c, const Keypoints& out, void* ws,
                          const DetectLayout& l);
DescribeJob make_describe_job(const ImageView& im, const Keypoints& kp, const Descriptors& out, void* ws,
                              const DescribeLayout& l);
// Dynamic shared memory of sort_topk_kernel for `candidates` keys.
int sort_smem_bytes(int candidates);

// ------------------------------------------------------- scale pyramid

// Layers of one image (OpenCV ORB level semantics): layer l has scale
// s_l = float(double(sf)^l) and size cvRound(W * (1.f / s_l)) x
// cvRound(H * (1.f / s_l)); layer l >= 1 is resized from layer l - 1. Only
// layers whose sides both exceed 2 * kEdge are built (smaller ones hold no
// keypoint). Budgets split K geometrically (cv::ORB's nfeaturesPerLevel),
// each share clamped so that the total is exactly K.
struct LevelPlan {
    int levels = 0;  // layers built
    int width[kMaxLevels] = {}, height[kMaxLevels] = {}, budget[kMaxLevels] = {};
    float scale[kMaxLevels] = {};
};

bool valid_pyramid(int levels, float scale_factor);
LevelPlan level_plan(int w, int h, int k, int levels, float scale_factor);

// Workspace of one image's pyramid. The head (layer counts int[levels],
// FAST histograms and counters u32[levels][kHistWords], the FAST tile queue
// and the blur-list count, the blur-tile flags u32[blur_total]) must be zero
// before each run (zeroed_bytes); the blur list uint2[blur_total] follows.
struct PyramidLayout {
    LevelPlan plan;
    std::size_t counts, hists, queue, marks, zeroed_bytes, blur_list;
    int blur_first[kMaxLevels + 1];  // first flag of each layer's blur tiles; blur_first[levels] = blur_total
    std::size_t image[kMaxLevels];  // dense layer images, l >= 1
    std::size_t kx[kMaxLevels], ky[kMaxLevels], kr[kMaxLevels];  // layer keypoints
    std::size_t detect[kMaxLevels], describe[kMaxLevels];
    DetectLayout det[kMaxLevels];
    DescribeLayout des[kMaxLevels];
    int resize_tiles[kMaxLevels];
    int resize_tile_h;  // output rows per resize block
    std::size_t total;
};

// resize_tile_h: 64 rows per resize block when many images share a launch;
// a single image's pyramid (kSingleResizeTileH) takes 16 to fill the GPU.
constexpr int kSingleResizeTileH = 16;
bool pyramid_layout(int w, int h, int k, int levels, float scale_factor, PyramidLayout* out,
                    int resize_tile_h = kResizeTileH);

struct PyramidJobs {
    ResizeJob resize[kMaxLevels];  // entries 1 .. levels-1
    DetectJob detect[kMaxLevels];
    DescribeJob describe[kMaxLevels];
};

// Buffers an image's layer jobs point into that are zeroed per run or shared
// by a whole launch: the layout's own head for the per-image call, the
// batch workspace's head in the batched chain.
struct PyramidShared {
    int* counts;               // [levels] layer keypoint counts
    std::uint32_t* hists;      // [levels][kHistWords]
    std::uint32_t* blur_marks; // [blur_first[levels]] this image's blur-tile flags
    uint2* blur_list;          // the launch's blur list
    std::uint32_t* blur_count; // and its length
    int job0;                  // describe-table index of layer 0
};

// Jobs of every layer over the workspace `ws` laid out by `l`.
void make_pyramid_jobs(const ImageView& im, const s2::Config& c, const Keypoints& out, const Descriptors& desc,
                       void* ws, const PyramidLayout& l, const PyramidShared& sh, PyramidJobs* jobs);

// Block count of each detect/describe kind for layer i (0 when inactive).
void pyramid_detect_blocks(const PyramidLayout& l, int layer, int (&blocks)[kDetectKinds]);
void pyramid_describe_blocks(const PyramidLayout& l, int layer, int (&blocks)[kDescribeKinds]);

Status pyramid_workspace_bytes(int w, int h, const s2::Config& c, int levels, float scale_factor,
                               std::size_t* bytes);
Status pyramid_detect_describe(const ImageView& image, const s2::Config& c, int levels, float scale_factor,
                               const Keypoints& out, const Descriptors& desc, void* ws, std::size_t ws_bytes,
                               cudaStream_t stream);

}  // namespace stitch::b200::s2s3
