/* C ABI of the B200 registration chain S2 -> S3 -> S4 -> S5.
 *
 * Plain pointers and sizes only; every struct below has the layout of the
 * reference's C++ stage struct it mirrors, so callers may pass either. Return
 * values are the reference's Status codes (src/common/status.hpp:6-13):
 *   0 OK, 1 INVALID_ARGUMENT, 2 INSUFFICIENT_WORKSPACE, 3 CUDA_ERROR,
 *   4 NOT_ENOUGH_POINTS, 5 DEGENERATE.
 * Contract shared by every stage call (src/common/types.hpp:2,
 * src/s4/s4.hpp:40-51): the caller allocates every device buffer and
 * workspace; calls never allocate or synchronise; arguments are checked before
 * anything is enqueued and a failed check writes nothing; work is ordered on
 * the caller's stream (a cudaStream_t passed as void*, NULL = legacy default
 * stream); device failures surface when the caller synchronises.
 *
 * The same library also exports the reference's C++ entry points
 * (stitch::s2::s2_detect, ..., stitch::s5::estimate) with identical
 * signatures, so code compiled against the reference headers links unchanged.
 */
#ifndef STITCH_B200_H
#define STITCH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- types */

/* src/common/types.hpp:16-22. format: 0 RGB8, 1 GRAY8 (stages take GRAY8). */
typedef struct stitch_image_view {
    uint8_t* data;
    int width, height, pitch_bytes;
    int format;
} stitch_image_view;

/* src/common/types.hpp:25-30. D maps original to working coordinates. */
typedef struct stitch_scale_info {
    int orig_w, orig_h, work_w, work_h;
    double sx, sy;
    double D[9];
} stitch_scale_info;

/* src/common/types.hpp:33-39. Device SoA; *d_count lives on the device. */
typedef struct stitch_keypoints {
    float* x;
    float* y;
    float* response; /* may be NULL */
    int capacity;
    int* d_count;
} stitch_keypoints;

/* src/common/types.hpp:44-49. type: 0 BINARY_U8 (dim bytes), 1 FLOAT32. */
typedef struct stitch_descriptors {
    int type, dim, row_stride_bytes;
    void* data;
} stitch_descriptors;

/* src/common/types.hpp:52-58. */
typedef struct stitch_matches {
    int32_t* idx_a;
    int32_t* idx_b;
    float* distance;
    int capacity;
    int* d_count;
} stitch_matches;

/* src/common/types.hpp:61-70. H maps B -> A in original coordinates. */
typedef struct stitch_homography_result {
    double H[9];
    double H_s[9];
    int num_matches, num_inliers;
    double inlier_ratio, inlier_coverage, reproj_residual;
    int status;
} stitch_homography_result;

/* src/s2_s3/s2.hpp:19-23. */
typedef struct stitch_s2_config {
    int fast_threshold; /* 1..254 */
    int max_keypoints;  /* K >= 0 */
    float harris_k;     /* finite, >= 0 */
} stitch_s2_config;

/* src/s4/s4.hpp:8-11 (bool cross_check is one byte, then padding). */
typedef struct stitch_s4_config {
    double ratio_threshold; /* finite, in (0, 1) */
    uint8_t cross_check;
    uint8_t reserved[7];
} stitch_s4_config;

/* src/s4/s4.hpp:16-21. Missing neighbour: index -1, distance +inf. */
typedef struct stitch_s4_top2 {
    double first_distance, second_distance;
    int first_index, second_index;
} stitch_s4_top2;

/* src/s5/s5.hpp:11-19. */
typedef struct stitch_s5_config {
    int hypotheses;          /* total R, including previous_hypotheses */
    int previous_hypotheses; /* 0 restarts; else extends the saved search */
    int batch_size;          /* 1..65535 */
    int refinement_steps;    /* >= 0 */
    double threshold;        /* reprojection distance in working pixels */
    uint64_t seed;
    uint64_t generation;
} stitch_s5_config;

/* --------------------------------------------------------------- library */

/* ABI version of this header (no reference counterpart). */
int stitch_abi_version(void);
/* Kernels this library has launched so far, over all calls (no reference
 * counterpart; lets a caller attribute device work to these kernels). */
long long stitch_launch_count(void);
/* Name of a status code; src/common/status.hpp:15-25. */
const char* stitch_status_name(int status);

/* src/common/geometry.hpp:119-131 (make_scale_info). */
int stitch_make_scale_info(int width, int height, double scale, stitch_scale_info* out);
/* src/common/geometry.hpp:157-163 (to_original): H = D_A^-1 H_s D_B. */
int stitch_to_original(const double* h_s, const double* d_a, const double* d_b, double* h_out);

/* ------------------------------------------------------------------- S1 */

/* src/s1/s1.hpp:33-38 (stitch::s1::s1_preprocess): RGB8 images A and B to
 * GRAY8 at scale S in (0, 1] (15-bit integer gray, area resize), one launch.
 * Writes scale_a/scale_b (make_scale_info); out_a/out_b must already have
 * the working sizes. No device workspace (src/s1/s1.hpp:14-20). */
int stitch_s1_preprocess(const stitch_image_view* img_a, const stitch_image_view* img_b, double scale,
                         stitch_image_view* out_a, stitch_image_view* out_b, stitch_scale_info* scale_a,
                         stitch_scale_info* scale_b, void* stream);
/* src/s1/s1.hpp:25-27 (stitch::s1::s1_preprocess_single). */
int stitch_s1_preprocess_single(const stitch_image_view* img, double scale, stitch_image_view* out,
                                stitch_scale_info* scale_info, void* stream);
/* src/s1/s1.hpp:53-56 (stitch::s1::s1_compute_gradient): mean absolute
 * gradient of two GRAY8 images into pinned host doubles; workspace 32 device
 * bytes (src/s1/s1.hpp:40-46). */
int stitch_s1_compute_gradient(const stitch_image_view* gray_a, const stitch_image_view* gray_b, void* workspace,
                               double* pinned_gradient_a, double* pinned_gradient_b, void* stream);

/* ------------------------------------------------------------------- S2 */

/* src/s2_s3/s2.hpp:26-27 (stitch::s2::s2_workspace_bytes). */
int stitch_s2_workspace_bytes(int width, int height, const stitch_s2_config* config, size_t* bytes);
/* src/s2_s3/s2.hpp:38-39 (stitch::s2::s2_detect). Writes min(found, K)
 * keypoints sorted by Harris response, ties by raster index, and *d_count. */
int stitch_s2_detect(const stitch_image_view* image, const stitch_s2_config* config,
                     const stitch_keypoints* output, void* workspace, size_t workspace_bytes,
                     void* stream);
/* src/s2_s3/s2_s3_marks.hpp:27-29 (s2_detect_marked): cudaEvent_t marks
 * recorded after FAST, after the 2K selection and after Harris. */
int stitch_s2_detect_marked(const stitch_image_view* image, const stitch_s2_config* config,
                            const stitch_keypoints* output, void* workspace, size_t workspace_bytes,
                            void* stream, void* after_fast, void* after_select, void* after_harris);

/* ------------------------------------------------------------------- S3 */

/* src/s2_s3/s3.hpp:19 (stitch::s3::s3_workspace_bytes). The blurred image
 * sits at offset 0 of the workspace after a call. */
int stitch_s3_workspace_bytes(int width, int height, size_t* bytes);
/* src/s2_s3/s3.hpp:28-30 (stitch::s3::s3_describe). */
int stitch_s3_describe(const stitch_image_view* image, const stitch_keypoints* keypoints,
                       const stitch_descriptors* output, void* workspace, size_t workspace_bytes,
                       void* stream);
/* src/s2_s3/s2_s3_marks.hpp:32-34 (s3_describe_marked). */
int stitch_s3_describe_marked(const stitch_image_view* image, const stitch_keypoints* keypoints,
                              const stitch_descriptors* output, void* workspace, size_t workspace_bytes,
                              void* stream, void* after_blur);

/* -------------------------------------------------------- scale pyramid */

/* The pyramid-levels knob. No reference counterpart: the reference's S2/S3
 * are single-level (docs/decisions/s2-s3-orb.md:84). levels 1 (or 0) is the
 * reference's single-level path; levels 2..16 follow cv::ORB's layers with
 * scale_factor in (1, 16] taken as a float like cv::ORB::create's. */
typedef struct stitch_pyramid_config {
    int levels;
    float scale_factor;
} stitch_pyramid_config;

/* No reference counterpart. Workspace of stitch_pyramid_detect_describe. */
int stitch_pyramid_workspace_bytes(int width, int height, const stitch_s2_config* config,
                                   const stitch_pyramid_config* pyramid, size_t* bytes);
/* No reference counterpart. S2 + S3 over the scale pyramid of one image:
 * layer l (scale s_l = float(sf^l), size cvRound(W / s_l) x cvRound(H / s_l),
 * built from layer l-1 by INTER_LINEAR_EXACT resizing) gets its share of the
 * K keypoints (cv::ORB's geometric split, the total exactly K) and runs the
 * single-level S2 and S3 (src/s2_s3/s2.cu, src/s2_s3/s3.cu); keypoints come
 * out level by level in level-0 coordinates (x, y multiplied by s_l in
 * float), with their descriptors in the same rows. Layers with a side of at
 * most 62 pixels hold no keypoints. With levels 1 the results equal
 * stitch_s2_detect followed by stitch_s3_describe. */
int stitch_pyramid_detect_describe(const stitch_image_view* image, const stitch_s2_config* config,
                                   const stitch_pyramid_config* pyramid, const stitch_keypoints* keypoints,
                                   const stitch_descriptors* descriptors, void* workspace,
                                   size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------- S4 */

/* No reference counterpart. Chooses the exact binary matcher of the calling
 * host thread's later S4 launches (stitch_s4_* calls) and of the batch plans
 * and servers it creates afterwards: 0 the __popc tile kernel, 1 (the
 * default) the tcgen05 kind::i8 tensor-core kernel (descriptor bits as +-1
 * int8, Hamming = (256 - dot) / 2) with 256 train rows per MMA stage, 2 and
 * 3 the same kernel with 128 and 64 train rows per stage (smaller blocks,
 * more of them per SM), 4 the pipelined tensor-core kernel (train-stage
 * expansion, MMAs and the top-2 epilogue of consecutive stages overlapped by
 * warp roles, two shared-memory stages and two TMEM accumulators). The choice is per thread, so threads never race on
 * it; stitch_batch_set_matcher changes one plan's. Results are identical. stitch_s4_tc_errors reads and clears the tensor-core
 * kernel's error word (1: an MMA completion wait ran out; -1: read failed). */
int stitch_s4_set_matcher(int kind);
int stitch_s4_matcher(void);
int stitch_s4_tc_errors(void);

/* src/s4/s4.hpp:25-26 (stitch::s4::s4_workspace_bytes). */
int stitch_s4_workspace_bytes(int capacity_a, int capacity_b, const stitch_s4_config* config,
                              size_t* bytes);
/* src/s4/s4.hpp:36-38 (stitch::s4::s4_knn_top2). */
int stitch_s4_knn_top2(const stitch_keypoints* a, const stitch_descriptors* da, const stitch_keypoints* b,
                       const stitch_descriptors* db, stitch_s4_top2* output, void* stream);
/* src/s4/s4.hpp:52-55 (stitch::s4::s4_match). */
int stitch_s4_match(const stitch_keypoints* a, const stitch_descriptors* da, const stitch_keypoints* b,
                    const stitch_descriptors* db, const stitch_s4_config* config, const stitch_matches* output,
                    void* workspace, size_t workspace_bytes, void* stream);
/* No counterpart in the reference. stitch_s4_match without a workspace, for
 * callers that cannot allocate device memory (a plug-in whose host owns all
 * device allocations, or a loop that cannot afford cudaMalloc's implicit
 * device synchronisation). The workspace is a 4 MiB array in the library's
 * own device memory, held by every GPU that loads the library until exit;
 * requests needing more fail with INSUFFICIENT_WORKSPACE (up to 87374 query
 * and train rows each fit with the mutual check, 174734 without, at the
 * current workspace layout). The first call on a device
 * looks the array up (make it before any stream capture); all calls on a
 * device share the array, so calls that overlap on the GPU race. */
int stitch_s4_match_static(const stitch_keypoints* a, const stitch_descriptors* da, const stitch_keypoints* b,
                           const stitch_descriptors* db, const stitch_s4_config* config,
                           const stitch_matches* output, void* stream);
/* src/s4/s4.hpp:59-60 (stitch::s4::s4_forward_neighbors). */
int stitch_s4_forward_neighbors(int capacity_a, int capacity_b, const stitch_s4_config* config,
                                const void* workspace, size_t workspace_bytes, const stitch_s4_top2** output);

/* ------------------------------------------------------------------- S5 */

/* src/s5/s5.hpp:23 (stitch::s5::s5_workspace_bytes). */
int stitch_s5_workspace_bytes(const stitch_s5_config* config, size_t* bytes);
/* src/s5/s5.hpp:36-39 (stitch::s5::estimate). output: pinned host memory,
 * valid after the caller synchronises the stream. */
int stitch_s5_estimate(const stitch_keypoints* a, const stitch_keypoints* b, const stitch_matches* matches,
                       const stitch_scale_info* scale_a, const stitch_scale_info* scale_b,
                       const stitch_s5_config* config, uint8_t* inlier_mask, stitch_homography_result* output,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------- S6 */

/* src/s6/geometry.hpp:10-16 (stitch::s6::GeometryPolicy). */
typedef struct stitch_s6_policy {
    double denominator_tolerance, inverse_tolerance, snap_tolerance;
    size_t max_canvas_pixels;
} stitch_s6_policy;
/* src/s6/geometry.hpp:18-34 (stitch::s6::Geometry): the canvas (A's pixel
 * grid from origin) and the A -> B inverse, largest entry magnitude 1. */
typedef struct stitch_s6_geometry {
    int width, height, origin_x, origin_y;
    int width_a, height_a, width_b, height_b;
    double denominator_tolerance, snap_tolerance;
    double inverse[9];
} stitch_s6_geometry;
/* Blend modes of src/s6/s6.hpp:13: 0 feather, 1 multiband3, 2 multiband5.
 * Only the feather blend renders; the multiband modes return
 * INVALID_ARGUMENT from stitch_s6_workspace_bytes and stitch_s6_render. */
#define STITCH_S6_FEATHER 0

/* The reference's default GeometryPolicy (1e-12, 1e-12, 1e-10, 16777216). */
void stitch_s6_default_policy(stitch_s6_policy* policy);
/* src/s6/geometry.hpp:43-44 (stitch::s6::prepare_geometry): H maps B to A
 * (row-major doubles); policy NULL = the default. OK, INVALID_ARGUMENT,
 * DEGENERATE (horizon, singular, ill-conditioned) or INSUFFICIENT_WORKSPACE
 * (canvas over the policy's pixel budget); *out is zeroed on failure. */
int stitch_s6_prepare_geometry(int width_a, int height_a, int width_b, int height_b, const double* h,
                               const stitch_s6_policy* policy, stitch_s6_geometry* out);
/* src/s6/s6.hpp:26-27 (stitch::s6::s6_workspace_bytes): 0 for feather. */
int stitch_s6_workspace_bytes(const stitch_s6_geometry* geometry, int mode, size_t* bytes);
/* src/s6/s6.hpp:44-47 (stitch::s6::render): one launch; output RGB8 and
 * mask GRAY8 (0/1) of the canvas size, device memory; statistics NULL or
 * two device uint64 {union_pixels, overlap_pixels}, 8-byte aligned, reset
 * and filled by the call. */
int stitch_s6_render(const stitch_image_view* a, const stitch_image_view* b, const stitch_s6_geometry* geometry,
                     int mode, const stitch_image_view* output, const stitch_image_view* mask, void* workspace,
                     size_t workspace_bytes, void* stream, uint64_t* statistics);

/* --------------------------------------------------------- batched form */

/* One pair of the batched form. It bundles the per-pair arguments the
 * reference harness passes to s2_detect (x2), s3_describe (x2), s4_match and
 * estimate (harness/pipeline_runner.cu:366-413); every pair carries its own
 * knobs and image sizes. scale_a/scale_b map original to working
 * coordinates as in src/common/geometry.hpp:119-131; orig_w == 0 means the
 * identity at the image's size. s5.previous_hypotheses must be 0.
 * pyramid.levels 0 or 1 is the single-level path; more levels run S2/S3 as
 * stitch_pyramid_detect_describe does. */
typedef struct stitch_pair_desc {
    stitch_image_view image_a, image_b; /* device GRAY8 */
    stitch_scale_info scale_a, scale_b;
    stitch_s2_config s2;
    stitch_s4_config s4;
    stitch_s5_config s5;
    stitch_pyramid_config pyramid;
} stitch_pair_desc;

/* Opaque plan of a batch (host object; owns a pinned staging buffer for the
 * device job tables and, after stitch_batch_capture, a CUDA graph and the
 * device copy of the job tables that the graph reads). */
typedef struct stitch_batch stitch_batch;

/* No reference counterpart (batched form). Validates every pair with the
 * stage rules and lays out one device workspace holding all intermediates
 * and outputs. On INVALID_ARGUMENT, *bad_pair (if non-NULL) is the first
 * offending pair. */
int stitch_batch_create(int n_pairs, const stitch_pair_desc* pairs, stitch_batch** plan,
                        size_t* workspace_bytes, int* bad_pair);
/* No reference counterpart (batched form). Launch shapes of a plan, chosen
 * per plan by an autotuner (results never depend on them); 0 in a field
 * keeps its default. fast_ctas_per_sm: resident FAST blocks per SM in the
 * persistent FAST grid, 1..7 (default 7); blur_ctas_per_sm: the same for the
 * on-demand blur, 1..6 (default 6); matcher: 1 + an S4 matcher kind (0..4,
 * as for stitch_s4_set_matcher), or 0 for the creating thread's choice;
 * search_hpw: MSAC hypotheses per warp round, 4, 8, 16 or 32 (default: the
 * largest that still fills about two waves); resize_tile_h: pyramid rows per
 * resize block, 16, 32 or 64 (default 64). */
typedef struct stitch_batch_tuning {
    int fast_ctas_per_sm;
    int blur_ctas_per_sm;
    int matcher;
    int search_hpw;
    int resize_tile_h;
} stitch_batch_tuning;

/* No reference counterpart (batched form). stitch_batch_create with a
 * tuning (NULL: the defaults); INVALID_ARGUMENT for a field out of range. */
int stitch_batch_create_tuned(int n_pairs, const stitch_pair_desc* pairs, const stitch_batch_tuning* tuning,
                              stitch_batch** plan, size_t* workspace_bytes, int* bad_pair);
/* No reference counterpart (batched form). Enqueues the whole chain for all
 * pairs on `stream`: results are identical, bit for bit, to calling the
 * stages pair by pair. results_pinned (n entries, may be NULL) receives the
 * homography results once the stream completes. */
int stitch_batch_enqueue(stitch_batch* plan, void* workspace, size_t workspace_bytes,
                         stitch_homography_result* results_pinned, void* stream);
/* No reference counterpart (batched form). Captures stitch_batch_enqueue with
 * these arguments into a CUDA graph held by the plan (the stream must not be
 * capturing already); stitch_batch_launch replays it. The call runs the chain
 * once uncaptured and keeps a device copy of the plan's job tables, which the
 * replays read: a replay starts with a kernel, not a host-to-device copy (so
 * it never waits for an image upload on another stream), and depends on
 * nothing left in `workspace`. The call synchronises `stream`. */
int stitch_batch_capture(stitch_batch* plan, void* workspace, size_t workspace_bytes,
                         stitch_homography_result* results_pinned, void* stream);
int stitch_batch_launch(stitch_batch* plan, void* stream);
/* No reference counterpart (batched form). Device views of pair `pair`'s
 * outputs inside `workspace` (any pointer argument may be NULL). */
int stitch_batch_pair_outputs(const stitch_batch* plan, void* workspace, int pair, stitch_keypoints* kp_a,
                              stitch_keypoints* kp_b, stitch_descriptors* desc_a, stitch_descriptors* desc_b,
                              stitch_matches* matches, uint8_t** inlier_mask, stitch_homography_result** result);
void stitch_batch_destroy(stitch_batch* plan);
/* No reference counterpart (batched form). The S4 matcher of this plan's
 * later enqueues and captures (0 __popc, 1 tensor cores; see
 * stitch_s4_set_matcher, whose choice a plan takes when it is created). */
int stitch_batch_set_matcher(stitch_batch* plan, int kind);
/* Per-kernel timing hook of the batched form (like the reference's S2/S3
 * event marks, src/s2_s3/s2_s3_marks.hpp:16-34): `events` holds
 * STITCH_BATCH_MARKS cudaEvent_t recorded, in order, after the table upload,
 * the pyramid resize chain, fast_nms, select+scatter, harris, sort, blur,
 * describe, knn (tensor-core or popc matcher), knn_merge, accept, prepare,
 * search and finish kernels
 * (a skipped kernel still records its mark). Applies to later enqueues and
 * captures; NULL turns the marks off. */
#define STITCH_BATCH_MARKS 14
int stitch_batch_set_marks(stitch_batch* plan, void* const* events, int count);

/* ---------------------------------------------------------- served form */

/* No reference counterpart (served form). The server owns no device memory:
 * `arena` (256-byte aligned, arena_bytes long, on `device`) is the caller's,
 * and its size is the HBM admission budget. Requests are admitted in
 * arrival order into batches of at most max_batch pairs (0: 64) that fit in
 * the arena; up to `streams` batches (0: 2) run at once. */
typedef struct stitch_server_config {
    void* arena;
    size_t arena_bytes;
    int device;
    int max_batch;
    int streams;
} stitch_server_config;

/* One pair to register. The images are host rows (pinned memory lets the
 * copies overlap; pageable memory works, synchronously) and must stay valid
 * until the request's result is polled. With rgb = 0 they are GRAY8 and
 * scale_a/scale_b are as in stitch_pair_desc. With rgb = 1 they are RGB8:
 * the server runs S1 (src/s1/s1.hpp:33-38) at `scale` (0 means 1) on the
 * device first, registers the working-size GRAY8 images, and returns H in
 * the original coordinates (scale_a/scale_b are then ignored). With
 * retry_hypotheses > s5.hypotheses, a result whose status is not OK or
 * whose inlier count is below retry_min_inliers is retried once by
 * extending the saved S5 search to retry_hypotheses on the resident
 * keypoints and matches (the controller's R escalation,
 * src/controller/reuse.cpp:5-22: no resampling, same result as a fresh run
 * with retry_hypotheses). `tag` is returned with the result.
 * S6 (rgb = 1 only): with host_panorama not NULL, after registration (and
 * any retry) the server renders the feather panorama of the two original
 * RGB images from the returned H (stitch_s6_prepare_geometry with the
 * default policy, then stitch_s6_render) into host_panorama as packed rows
 * of 3 * canvas width bytes and, when host_mask is not NULL, the 0/1 union
 * mask into host_mask (packed rows of canvas width bytes).
 * panorama_capacity is the largest canvas, in pixels, the buffers hold;
 * that much device memory is part of the request's arena footprint. Pinned
 * buffers keep the dispatcher from blocking on the copies. */
typedef struct stitch_request {
    const uint8_t* host_a;
    const uint8_t* host_b;
    int width_a, height_a, pitch_a;
    int width_b, height_b, pitch_b;
    stitch_scale_info scale_a, scale_b;
    stitch_s2_config s2;
    stitch_s4_config s4;
    stitch_s5_config s5;
    stitch_pyramid_config pyramid;
    int rgb;
    double scale;
    int retry_hypotheses;
    int retry_min_inliers;
    uint64_t tag;
    uint8_t* host_panorama;
    uint8_t* host_mask;
    size_t panorama_capacity;
} stitch_request;

/* Completed request. Times are milliseconds on a steady clock since the
 * server was created: submit (stitch_server_submit), launch (its batch
 * enqueued) and done (the dispatcher saw its batch complete, results on the
 * host). status is 0 unless the request could not run; attempts is 2 when
 * the S5 extension retry ran. render_status is -1 when no panorama was
 * asked for; otherwise the registration's status when it was not OK, else
 * the status of the geometry (DEGENERATE, or INSUFFICIENT_WORKSPACE for a
 * canvas above panorama_capacity or the default 16777216-pixel budget) or
 * of the render; with 0 the canvas size, its origin in A's pixels and the
 * union/overlap pixel counts describe the panorama written. */
typedef struct stitch_server_result {
    uint64_t tag;
    double submit_ms, launch_ms, done_ms;
    int batch_pairs;
    int status;
    int attempts;
    stitch_homography_result result;
    int render_status;
    int canvas_width, canvas_height, origin_x, origin_y;
    uint64_t union_pixels, overlap_pixels;
} stitch_server_result;

typedef struct stitch_server stitch_server;

/* No reference counterpart (served form). Starts the dispatcher thread. */
int stitch_server_create(const stitch_server_config* config, stitch_server** server);
/* No reference counterpart. The device-memory footprint a request takes in
 * an arena (the request alone in a batch); host computation only, the same
 * checks as stitch_server_submit. For placing requests across GPUs. */
int stitch_server_request_bytes(const stitch_request* request, size_t* bytes);
/* No reference counterpart. Queues one request (thread-safe, returns at
 * once). INVALID_ARGUMENT for knobs or sizes the stages reject;
 * INSUFFICIENT_WORKSPACE when the request alone needs more than the arena. */
int stitch_server_submit(stitch_server* server, const stitch_request* request);
/* No reference counterpart. Moves up to `max` completed results to `out`. */
int stitch_server_poll(stitch_server* server, stitch_server_result* out, int max, int* count);
/* No reference counterpart. Requests submitted and not yet polled-ready. */
int stitch_server_outstanding(stitch_server* server);
/* No reference counterpart. Finishes the queued requests, then stops. */
void stitch_server_destroy(stitch_server* server);

#ifdef __cplusplus
}
#endif

#endif /* STITCH_B200_H */
