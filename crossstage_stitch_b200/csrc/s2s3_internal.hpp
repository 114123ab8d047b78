// Layouts and job builders shared by the per-image S2/S3 calls and the
// batched chain.
#pragma once

#include "s2s3_kernels.cuh"

namespace stitch::b200::s2s3 {

struct DetectLayout {
    std::size_t maxima, hist, params, chunk_counts, keys, total;
    int chunks, candidates, tiles_x, tiles;
};

struct DescribeLayout {
    std::size_t blurred, total;  // blurred image first, at offset 0
    int tiles_x, tiles;
};

bool valid_image_shape(int w, int h);
bool valid_gray(const ImageView& im);
bool valid_detect_config(const s2::Config& c);
bool detect_layout(int w, int h, int k, DetectLayout* out);
bool describe_layout(int w, int h, DescribeLayout* out);
DetectJob make_detect_job(const ImageView& im, const s2::Config& c, const Keypoints& out, void* ws,
                          const DetectLayout& l);
DescribeJob make_describe_job(const ImageView& im, const Keypoints& kp, const Descriptors& out, void* ws,
                              const DescribeLayout& l);
// Dynamic shared memory of sort_topk_kernel for `candidates` keys.
int sort_smem_bytes(int candidates);

}  // namespace stitch::b200::s2s3
