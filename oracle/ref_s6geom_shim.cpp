// Test infrastructure only. extern "C" access to the reference's own S6 host
// geometry (src/s6/geometry.cpp), compiled from the reference tree by
// `make -C oracle ref`; tests use it to pin the oracle's and the library's
// prepare_geometry bit for bit. Structs have the layouts of
// include/stitch_b200.h (stitch_s6_policy, stitch_s6_geometry).
#include "s6/geometry.hpp"

extern "C" int ref_s6_prepare_geometry(int wa, int ha, int wb, int hb, const double* h,
                                       const stitch::s6::GeometryPolicy* policy, stitch::s6::Geometry* out) {
    return static_cast<int>(stitch::s6::prepare_geometry(wa, ha, wb, hb, h, *policy, out));
}
