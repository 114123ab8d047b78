// Test infrastructure only. extern "C" access to the reference's own host
// solver (src/s5/s5_math.hpp) and geometry (src/common/geometry.hpp), compiled
// from the reference tree by `make -C oracle ref`; tests use it to pin the C
// oracle's S5 math bit for bit.
#include <cstdint>

#include "common/geometry.hpp"
#include "s5/s5_math.hpp"

using namespace stitch::s5::detail;

namespace {
struct Pts {
    const Point* p;
    Point operator()(int i) const { return p[i]; }
};
struct Keep {
    const unsigned char* k;
    bool operator()(int i) const { return k == nullptr || k[i] != 0; }
};
}  // namespace

extern "C" {
int ref_fit(int n, const double* pts4, const unsigned char* keep, double* out) {
    return fit(n, Pts{reinterpret_cast<const Point*>(pts4)}, Keep{keep}, out) ? 1 : 0;
}
void ref_sample_four(int n, std::uint64_t seed, int h, int* out) { sample_four(n, seed, h, out); }
double ref_residual2(const double* h, double ax, double ay, double bx, double by) {
    return residual_squared(h, Point{ax, ay, bx, by});
}
int ref_nondegenerate(const double* pts4) { return nondegenerate_four(reinterpret_cast<const Point*>(pts4)) ? 1 : 0; }
int ref_valid_domain(const double* h, int w, int hgt) { return valid_domain(h, w, hgt) ? 1 : 0; }
int ref_normalize(double* h) { return normalize(h) ? 1 : 0; }
int ref_mat3_inverse(const double* m, double* out) { return stitch::mat3_inverse(m, out) ? 1 : 0; }
}
