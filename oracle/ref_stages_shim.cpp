// Test infrastructure only. extern "C" entry points over the reference's own
// S1..S6 stage functions, linked with the reference sources built for sm_100a
// by `make -C oracle ref`. Arguments use the same plain-data layouts as
// include/stitch_b200.h, so tests pass identical structs to both libraries.
#include "common/types.hpp"
#include "s1/s1.hpp"
#include "s2_s3/s2.hpp"
#include "s2_s3/s3.hpp"
#include "s4/s4.hpp"
#include "s5/s5.hpp"
#include "s6/s6.hpp"

using namespace stitch;

namespace {
int code(Status s) { return static_cast<int>(s); }
cudaStream_t st(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {
int ref_s1_preprocess(const ImageView* a, const ImageView* b, double scale, ImageView* oa, ImageView* ob,
                      ScaleInfo* sa, ScaleInfo* sb, void* s) {
    return code(s1::s1_preprocess(*a, *b, scale, oa, ob, sa, sb, st(s)));
}
int ref_s1_compute_gradient(const ImageView* a, const ImageView* b, void* ws, double* ga, double* gb, void* s) {
    return code(s1::s1_compute_gradient(*a, *b, ws, ga, gb, st(s)));
}
int ref_s2_workspace_bytes(int w, int h, const s2::Config* c, std::size_t* b) {
    return code(s2::s2_workspace_bytes(w, h, *c, b));
}
int ref_s2_detect(const ImageView* im, const s2::Config* c, const Keypoints* out, void* ws, std::size_t n,
                  void* s) {
    return code(s2::s2_detect(*im, *c, *out, ws, n, st(s)));
}
int ref_s3_workspace_bytes(int w, int h, std::size_t* b) { return code(s3::s3_workspace_bytes(w, h, b)); }
int ref_s3_describe(const ImageView* im, const Keypoints* kp, const Descriptors* out, void* ws, std::size_t n,
                    void* s) {
    return code(s3::s3_describe(*im, *kp, *out, ws, n, st(s)));
}
int ref_s4_workspace_bytes(int ca, int cb, const s4::Config* c, std::size_t* b) {
    return code(s4::s4_workspace_bytes(ca, cb, *c, b));
}
int ref_s4_match(const Keypoints* a, const Descriptors* da, const Keypoints* b, const Descriptors* db,
                 const s4::Config* c, const Matches* out, void* ws, std::size_t n, void* s) {
    return code(s4::s4_match(*a, *da, *b, *db, *c, *out, ws, n, st(s)));
}
int ref_s4_knn_top2(const Keypoints* a, const Descriptors* da, const Keypoints* b, const Descriptors* db,
                    s4::Top2* out, void* s) {
    return code(s4::s4_knn_top2(*a, *da, *b, *db, out, st(s)));
}
int ref_s5_workspace_bytes(const s5::Config* c, std::size_t* b) { return code(s5::s5_workspace_bytes(*c, b)); }
int ref_s5_estimate(const Keypoints* a, const Keypoints* b, const Matches* m, const ScaleInfo* sa,
                    const ScaleInfo* sb, const s5::Config* c, std::uint8_t* mask, HomographyResult* out, void* ws,
                    std::size_t n, void* s) {
    return code(s5::estimate(*a, *b, *m, *sa, *sb, *c, mask, out, ws, n, st(s)));
}
int ref_s6_prepare_geometry(int wa, int ha, int wb, int hb, const double* h, const s6::GeometryPolicy* p,
                            s6::Geometry* out) {
    return code(s6::prepare_geometry(wa, ha, wb, hb, h, *p, out));
}
int ref_s6_render(const ImageView* a, const ImageView* b, const s6::Geometry* g, int mode, const ImageView* out,
                  const ImageView* mask, void* ws, std::size_t n, void* s, std::uint64_t* statistics) {
    return code(s6::render(*a, *b, *g, static_cast<s6::BlendMode>(mode), *out, *mask, ws, n, st(s),
                           reinterpret_cast<s6::RenderStatistics*>(statistics)));
}
}
