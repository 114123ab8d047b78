// extern "C" wrappers over the C++ stage API. The C structs of
// include/stitch_b200.h have the layouts of the C++ structs (checked below),
// so arguments are reinterpreted, never copied field by field. No exception
// crosses this boundary: the stage functions do not throw.
#include <atomic>
#include <cmath>
#include <cstddef>

#include "stitch_b200.h"
#include "stage_api.hpp"

namespace {

using namespace stitch;

#define SAME_LAYOUT(C, CPP)                                                        \
    static_assert(sizeof(C) == sizeof(CPP) && alignof(C) == alignof(CPP), #C)

SAME_LAYOUT(stitch_image_view, ImageView);
SAME_LAYOUT(stitch_scale_info, ScaleInfo);
SAME_LAYOUT(stitch_keypoints, Keypoints);
SAME_LAYOUT(stitch_descriptors, Descriptors);
SAME_LAYOUT(stitch_matches, Matches);
SAME_LAYOUT(stitch_homography_result, HomographyResult);
SAME_LAYOUT(stitch_s2_config, s2::Config);
SAME_LAYOUT(stitch_s4_config, s4::Config);
SAME_LAYOUT(stitch_s4_top2, s4::Top2);
SAME_LAYOUT(stitch_s5_config, s5::Config);
static_assert(offsetof(stitch_homography_result, status) == offsetof(HomographyResult, status), "result");
static_assert(offsetof(stitch_s5_config, seed) == offsetof(s5::Config, seed), "s5 config");
static_assert(offsetof(stitch_scale_info, D) == offsetof(ScaleInfo, D), "scale info");
static_assert(offsetof(stitch_s4_config, cross_check) == offsetof(s4::Config, cross_check), "s4 config");
SAME_LAYOUT(stitch_s6_policy, s6::GeometryPolicy);
SAME_LAYOUT(stitch_s6_geometry, s6::Geometry);
static_assert(offsetof(stitch_s6_policy, max_canvas_pixels) == offsetof(s6::GeometryPolicy, max_canvas_pixels),
              "s6 policy");
static_assert(offsetof(stitch_s6_geometry, inverse) == offsetof(s6::Geometry, inverse), "s6 geometry");
static_assert(offsetof(stitch_s6_geometry, snap_tolerance) == offsetof(s6::Geometry, snap_tolerance), "s6 geometry");

template <class T, class C> const T& as(const C* p) { return *reinterpret_cast<const T*>(p); }

int code(Status s) { return static_cast<int>(s); }
constexpr int kInvalid = static_cast<int>(Status::INVALID_ARGUMENT);

cudaStream_t stream_of(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

namespace stitch::b200 {
namespace s2s3 {  // pyramid.cu
Status pyramid_workspace_bytes(int w, int h, const s2::Config& c, int levels, float scale_factor,
                               std::size_t* bytes);
Status pyramid_detect_describe(const ImageView& image, const s2::Config& c, int levels, float scale_factor,
                               const Keypoints& out, const Descriptors& desc, void* ws, std::size_t ws_bytes,
                               cudaStream_t stream);
}  // namespace s2s3
static std::atomic<long long> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace stitch::b200

extern "C" {

int stitch_abi_version(void) { return 3; }

long long stitch_launch_count(void) { return stitch::b200::g_launches.load(std::memory_order_relaxed); }

const char* stitch_status_name(int status) {
    switch (status) {
        case 0: return "OK";
        case 1: return "INVALID_ARGUMENT";
        case 2: return "INSUFFICIENT_WORKSPACE";
        case 3: return "CUDA_ERROR";
        case 4: return "NOT_ENOUGH_POINTS";
        case 5: return "DEGENERATE";
        default: return "UNKNOWN";
    }
}

int stitch_make_scale_info(int w, int h, double s, stitch_scale_info* out) {
    if (!out || w <= 0 || h <= 0 || !(s > 0.0) || s > 1.0) return kInvalid;
    const long ww = std::lround(static_cast<double>(w) * s), wh = std::lround(static_cast<double>(h) * s);
    out->orig_w = w;
    out->orig_h = h;
    out->work_w = static_cast<int>(ww < 1 ? 1 : ww);
    out->work_h = static_cast<int>(wh < 1 ? 1 : wh);
    out->sx = static_cast<double>(out->work_w) / w;
    out->sy = static_cast<double>(out->work_h) / h;
    const double d[9] = {out->sx, 0, 0.5 * (out->sx - 1.0), 0, out->sy, 0.5 * (out->sy - 1.0), 0, 0, 1};
    for (int i = 0; i < 9; ++i) out->D[i] = d[i];
    return 0;
}

int stitch_to_original(const double* h_s, const double* d_a, const double* d_b, double* h_out) {
    if (!h_s || !d_a || !d_b || !h_out) return kInvalid;
    const double* m = d_a;
    const double c00 = m[4] * m[8] - m[5] * m[7];
    const double c01 = m[5] * m[6] - m[3] * m[8];
    const double c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (std::fabs(det) < 1e-300) return static_cast<int>(Status::DEGENERATE);
    const double inv = 1.0 / det;
    const double ia[9] = {c00 * inv, (m[2] * m[7] - m[1] * m[8]) * inv, (m[1] * m[5] - m[2] * m[4]) * inv,
                          c01 * inv, (m[0] * m[8] - m[2] * m[6]) * inv, (m[2] * m[3] - m[0] * m[5]) * inv,
                          c02 * inv, (m[1] * m[6] - m[0] * m[7]) * inv, (m[0] * m[4] - m[1] * m[3]) * inv};
    double t[9], r[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[3 * i + j] = ia[3 * i] * h_s[j] + ia[3 * i + 1] * h_s[j + 3] + ia[3 * i + 2] * h_s[j + 6];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[3 * i + j] = t[3 * i] * d_b[j] + t[3 * i + 1] * d_b[j + 3] + t[3 * i + 2] * d_b[j + 6];
    for (int i = 0; i < 9; ++i) h_out[i] = r[i];
    return 0;
}

int stitch_s2_workspace_bytes(int w, int h, const stitch_s2_config* c, size_t* bytes) {
    if (!c) return kInvalid;
    return code(s2::s2_workspace_bytes(w, h, as<s2::Config>(c), bytes));
}

int stitch_s2_detect(const stitch_image_view* im, const stitch_s2_config* c, const stitch_keypoints* out,
                     void* ws, size_t ws_bytes, void* stream) {
    if (!im || !c || !out) return kInvalid;
    return code(s2::s2_detect(as<ImageView>(im), as<s2::Config>(c), as<Keypoints>(out), ws, ws_bytes,
                              stream_of(stream)));
}

int stitch_s2_detect_marked(const stitch_image_view* im, const stitch_s2_config* c, const stitch_keypoints* out,
                            void* ws, size_t ws_bytes, void* stream, void* e_fast, void* e_select,
                            void* e_harris) {
    if (!im || !c || !out) return kInvalid;
    const s2_s3::detail::S2Marks marks{static_cast<cudaEvent_t>(e_fast), static_cast<cudaEvent_t>(e_select),
                                       static_cast<cudaEvent_t>(e_harris)};
    return code(s2_s3::detail::s2_detect_marked(as<ImageView>(im), as<s2::Config>(c), as<Keypoints>(out), ws,
                                                ws_bytes, stream_of(stream), marks));
}

int stitch_s3_workspace_bytes(int w, int h, size_t* bytes) { return code(s3::s3_workspace_bytes(w, h, bytes)); }

int stitch_s3_describe(const stitch_image_view* im, const stitch_keypoints* kp, const stitch_descriptors* out,
                       void* ws, size_t ws_bytes, void* stream) {
    if (!im || !kp || !out) return kInvalid;
    return code(s3::s3_describe(as<ImageView>(im), as<Keypoints>(kp), as<Descriptors>(out), ws, ws_bytes,
                                stream_of(stream)));
}

int stitch_s3_describe_marked(const stitch_image_view* im, const stitch_keypoints* kp,
                              const stitch_descriptors* out, void* ws, size_t ws_bytes, void* stream,
                              void* e_blur) {
    if (!im || !kp || !out) return kInvalid;
    const s2_s3::detail::S3Marks marks{static_cast<cudaEvent_t>(e_blur)};
    return code(s2_s3::detail::s3_describe_marked(as<ImageView>(im), as<Keypoints>(kp), as<Descriptors>(out), ws,
                                                  ws_bytes, stream_of(stream), marks));
}

int stitch_pyramid_workspace_bytes(int w, int h, const stitch_s2_config* c, const stitch_pyramid_config* p,
                                   size_t* bytes) {
    if (!c || !p) return kInvalid;
    return code(b200::s2s3::pyramid_workspace_bytes(w, h, as<s2::Config>(c), p->levels ? p->levels : 1,
                                                    p->scale_factor, bytes));
}

int stitch_pyramid_detect_describe(const stitch_image_view* im, const stitch_s2_config* c,
                                   const stitch_pyramid_config* p, const stitch_keypoints* kp,
                                   const stitch_descriptors* desc, void* ws, size_t ws_bytes, void* stream) {
    if (!im || !c || !p || !kp || !desc) return kInvalid;
    return code(b200::s2s3::pyramid_detect_describe(as<ImageView>(im), as<s2::Config>(c), p->levels ? p->levels : 1,
                                                    p->scale_factor, as<Keypoints>(kp), as<Descriptors>(desc), ws,
                                                    ws_bytes, stream_of(stream)));
}

int stitch_s4_workspace_bytes(int ca, int cb, const stitch_s4_config* c, size_t* bytes) {
    if (!c) return kInvalid;
    return code(s4::s4_workspace_bytes(ca, cb, as<s4::Config>(c), bytes));
}

int stitch_s4_knn_top2(const stitch_keypoints* a, const stitch_descriptors* da, const stitch_keypoints* b,
                       const stitch_descriptors* db, stitch_s4_top2* out, void* stream) {
    if (!a || !da || !b || !db) return kInvalid;
    return code(s4::s4_knn_top2(as<Keypoints>(a), as<Descriptors>(da), as<Keypoints>(b), as<Descriptors>(db),
                                reinterpret_cast<s4::Top2*>(out), stream_of(stream)));
}

int stitch_s4_match(const stitch_keypoints* a, const stitch_descriptors* da, const stitch_keypoints* b,
                    const stitch_descriptors* db, const stitch_s4_config* c, const stitch_matches* out, void* ws,
                    size_t ws_bytes, void* stream) {
    if (!a || !da || !b || !db || !c || !out) return kInvalid;
    return code(s4::s4_match(as<Keypoints>(a), as<Descriptors>(da), as<Keypoints>(b), as<Descriptors>(db),
                             as<s4::Config>(c), as<Matches>(out), ws, ws_bytes, stream_of(stream)));
}

int stitch_s4_forward_neighbors(int ca, int cb, const stitch_s4_config* c, const void* ws, size_t ws_bytes,
                                const stitch_s4_top2** out) {
    if (!c) return kInvalid;
    return code(s4::s4_forward_neighbors(ca, cb, as<s4::Config>(c), ws, ws_bytes,
                                         reinterpret_cast<const s4::Top2**>(out)));
}

int stitch_s5_workspace_bytes(const stitch_s5_config* c, size_t* bytes) {
    if (!c) return kInvalid;
    return code(s5::s5_workspace_bytes(as<s5::Config>(c), bytes));
}

int stitch_s5_estimate(const stitch_keypoints* a, const stitch_keypoints* b, const stitch_matches* m,
                       const stitch_scale_info* sa, const stitch_scale_info* sb, const stitch_s5_config* c,
                       uint8_t* mask, stitch_homography_result* out, void* ws, size_t ws_bytes, void* stream) {
    if (!a || !b || !m || !sa || !sb || !c) return kInvalid;
    return code(s5::estimate(as<Keypoints>(a), as<Keypoints>(b), as<Matches>(m), as<ScaleInfo>(sa),
                             as<ScaleInfo>(sb), as<s5::Config>(c), mask, reinterpret_cast<HomographyResult*>(out),
                             ws, ws_bytes, stream_of(stream)));
}

}  // extern "C"
