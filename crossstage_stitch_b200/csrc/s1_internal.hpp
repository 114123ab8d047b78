// S1 pieces shared with the served form (server.cu).
#pragma once

#include "common.cuh"
#include "stitch_b200.h"

namespace stitch::b200::s1k {

struct Params {
    const std::uint8_t* src;
    int src_pitch, orig_w, orig_h;
    std::uint8_t* dst;
    int dst_pitch, work_w, work_h;
    float inv_sx, inv_sy, scale_area;
    int mode;  // 0 direct, 1 2x2 average, 2 4x4 average, 3 float box filter
};

constexpr int kBatchTileW = 64, kBatchTileH = 16;

// One image of a batched S1 launch: 64x16 output tiles.
struct BatchJob {
    Params p;
    int tiles_x, tiles;
};

// Checks one RGB8 -> GRAY8 image (the per-call rules of s1_preprocess) and
// fills its job; `si` gives the working size.
Status batch_job(const ImageView& in, const ImageView& out, const ScaleInfo& si, BatchJob* j);
// One launch over n jobs; device_prefix[i] is the first block of job i,
// device_prefix[n] == blocks.
Status batch_enqueue(const BatchJob* device_jobs, const int* device_prefix, int n, int blocks, cudaStream_t stream);

}  // namespace stitch::b200::s1k
