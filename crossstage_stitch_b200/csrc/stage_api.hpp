// C++ stage interface of the registration chain S2 -> S3 -> S4 -> S5.
//
// Names, argument lists and struct layouts are those of the reference's stage
// API, so a caller built against the reference headers (its harness, mock
// drivers and CUDA tests) links against this library without changes:
//   plain-data structs ........ src/common/types.hpp:13-70
//   Status codes .............. src/common/status.hpp:6-13
//   S2 ........................ src/s2_s3/s2.hpp:14-39
//   S3 ........................ src/s2_s3/s3.hpp:15-26
//   S2/S3 event-mark hooks .... src/s2_s3/s2_s3_marks.hpp:16-34
//   S4 ........................ src/s4/s4.hpp:8-60
//   S5 ........................ src/s5/s5.hpp:11-39
//   geometry helpers .......... src/common/geometry.hpp:119-163
// Contract shared by every stage: the caller allocates all buffers, stages
// never allocate or synchronise, arguments are checked before anything is
// enqueued, and the return value reports argument and launch errors only.
#pragma once

#include <cstddef>
#include <cstdint>

struct CUstream_st;
typedef struct CUstream_st* cudaStream_t;
struct CUevent_st;
typedef struct CUevent_st* cudaEvent_t;

namespace stitch {

enum class Status : int {
    OK = 0,
    INVALID_ARGUMENT,
    INSUFFICIENT_WORKSPACE,
    CUDA_ERROR,
    NOT_ENOUGH_POINTS,
    DEGENERATE,
};

enum class PixelFormat : int { RGB8 = 0, GRAY8 = 1 };

// Device image, rows pitch_bytes apart.
struct ImageView {
    uint8_t* data;
    int width;
    int height;
    int pitch_bytes;
    PixelFormat format;
};

// Working-resolution bookkeeping of one image; D maps original pixel
// coordinates to working coordinates (half-pixel convention).
struct ScaleInfo {
    int orig_w, orig_h;
    int work_w, work_h;
    double sx, sy;
    double D[9];
};

// Device SoA keypoints; valid rows are [0, *d_count).
struct Keypoints {
    float* x;
    float* y;
    float* response;
    int capacity;
    int* d_count;
};

enum class DescriptorType : int { BINARY_U8 = 0, FLOAT32 = 1 };

struct Descriptors {
    DescriptorType type;
    int dim;
    int row_stride_bytes;
    void* data;
};

struct Matches {
    int32_t* idx_a;
    int32_t* idx_b;
    float* distance;
    int capacity;
    int* d_count;
};

// B -> A homography in original (H) and working (H_s) coordinates.
struct HomographyResult {
    double H[9];
    double H_s[9];
    int num_matches;
    int num_inliers;
    double inlier_ratio;
    double inlier_coverage;
    double reproj_residual;
    Status status;
};

namespace s1 {
// src/s1/s1.hpp:14-20 and :40-46: S1 needs no device workspace; the gradient
// probe needs 32 bytes.
inline Status s1_workspace_bytes(int orig_w, int orig_h, double scale, std::size_t* bytes) {
    if (bytes == nullptr || orig_w <= 0 || orig_h <= 0 || !(scale > 0.0) || scale > 1.0)
        return Status::INVALID_ARGUMENT;
    *bytes = 0;
    return Status::OK;
}
inline Status s1_gradient_workspace_bytes(std::size_t* bytes) {
    if (bytes == nullptr) return Status::INVALID_ARGUMENT;
    *bytes = 32;
    return Status::OK;
}
Status s1_preprocess_single(const ImageView& in, double scale, ImageView* out, ScaleInfo* scale_info,
                            cudaStream_t stream);
Status s1_preprocess(const ImageView& img_a, const ImageView& img_b, double scale, ImageView* out_a,
                     ImageView* out_b, ScaleInfo* scale_a, ScaleInfo* scale_b, cudaStream_t stream);
Status s1_compute_gradient(const ImageView& gray_a, const ImageView& gray_b, void* d_workspace,
                           double* pinned_gradient_a, double* pinned_gradient_b, cudaStream_t stream);
Status s1_compute_gradient_single(const ImageView& gray, void* d_workspace, double* pinned_gradient,
                                  cudaStream_t stream);
}  // namespace s1

namespace s2 {
constexpr int kEdge = 31;
constexpr int kCandidateFactor = 2;
struct Config {
    int fast_threshold;  // 1..254
    int max_keypoints;   // K >= 0
    float harris_k;      // finite, >= 0
};
Status s2_workspace_bytes(int width, int height, const Config& config, std::size_t* bytes);
Status s2_detect(const ImageView& image, const Config& config, Keypoints output,
                 void* workspace, std::size_t workspace_bytes, cudaStream_t stream);
}  // namespace s2

namespace s3 {
constexpr int kDescriptorBytes = 32;
Status s3_workspace_bytes(int width, int height, std::size_t* bytes);
Status s3_describe(const ImageView& image, const Keypoints& keypoints, Descriptors output,
                   void* workspace, std::size_t workspace_bytes, cudaStream_t stream);
}  // namespace s3

namespace s2_s3::detail {
struct S2Marks {
    cudaEvent_t after_fast;
    cudaEvent_t after_select;
    cudaEvent_t after_harris;
};
struct S3Marks {
    cudaEvent_t after_blur;
};
Status s2_detect_marked(const ImageView& image, const s2::Config& config, Keypoints output,
                        void* workspace, std::size_t workspace_bytes, cudaStream_t stream,
                        const S2Marks& marks);
Status s3_describe_marked(const ImageView& image, const Keypoints& keypoints,
                          Descriptors output, void* workspace, std::size_t workspace_bytes,
                          cudaStream_t stream, const S3Marks& marks);
}  // namespace s2_s3::detail

namespace s4 {
struct Config {
    double ratio_threshold;  // finite, in (0, 1)
    bool cross_check;
};
// Missing neighbours: index -1, distance +inf.
struct Top2 {
    double first_distance;
    double second_distance;
    int first_index;
    int second_index;
};
Status s4_workspace_bytes(int capacity_a, int capacity_b, const Config& config, std::size_t* bytes);
Status s4_knn_top2(const Keypoints& a, const Descriptors& da, const Keypoints& b,
                   const Descriptors& db, Top2* output, cudaStream_t stream);
Status s4_match(const Keypoints& a, const Descriptors& da, const Keypoints& b,
                const Descriptors& db, const Config& config, Matches output, void* workspace,
                std::size_t workspace_bytes, cudaStream_t stream);
Status s4_forward_neighbors(int capacity_a, int capacity_b, const Config& config,
                            const void* workspace, std::size_t workspace_bytes,
                            const Top2** output);
}  // namespace s4

namespace s5 {
struct Config {
    int hypotheses;           // total R, including previous_hypotheses
    int previous_hypotheses;  // 0 restarts; otherwise extends the saved search
    int batch_size;           // 1..65535
    int refinement_steps;     // >= 0
    double threshold;         // reprojection distance, working pixels
    std::uint64_t seed;
    std::uint64_t generation;
};
Status s5_workspace_bytes(const Config& config, std::size_t* bytes);
Status estimate(const Keypoints& a, const Keypoints& b, const Matches& matches,
                const ScaleInfo& scale_a, const ScaleInfo& scale_b, const Config& config,
                std::uint8_t* inlier_mask, HomographyResult* output, void* workspace,
                std::size_t workspace_bytes, cudaStream_t stream);
}  // namespace s5

namespace s6 {
// src/s6/s6.hpp:13-19 and src/s6/geometry.hpp:9-33.
enum class BlendMode : int { Feather = 0, Multiband3 = 1, Multiband5 = 2 };
struct alignas(8) RenderStatistics {
    std::uint64_t union_pixels;
    std::uint64_t overlap_pixels;
};
struct GeometryPolicy {
    double denominator_tolerance = 1e-12;
    double inverse_tolerance = 1e-12;
    double snap_tolerance = 1e-10;
    std::size_t max_canvas_pixels = 16777216;
};
struct Geometry {
    int width = 0;
    int height = 0;
    int origin_x = 0;  // original A coordinates of canvas pixel (0, 0)
    int origin_y = 0;
    int width_a = 0;
    int height_a = 0;
    int width_b = 0;
    int height_b = 0;
    double denominator_tolerance = 1e-12;
    double snap_tolerance = 1e-10;
    double inverse[9] = {};  // A-original -> B-original, normalised by its largest entry
};
Status prepare_geometry(int width_a, int height_a, int width_b, int height_b, const double* h,
                        const GeometryPolicy& policy, Geometry* out);
int effective_reductions(const Geometry& geometry, BlendMode mode);
Status s6_workspace_bytes(const Geometry& geometry, BlendMode mode, std::size_t* bytes);
Status render(const ImageView& a, const ImageView& b, const Geometry& geometry, BlendMode mode,
              const ImageView& output, const ImageView& mask, void* workspace, std::size_t workspace_bytes,
              cudaStream_t stream, RenderStatistics* statistics = nullptr);
}  // namespace s6

}  // namespace stitch
