// S6: the B -> A canvas geometry (host) and the fused feather render
// (device) of two RGB8 images.
//
// Reference semantics (file:line in the reference tree):
//   geometry  src/s6/geometry.cpp:10-198 (80-bit long double: H normalised by
//             its largest entry; the four B corners must stay on one side of
//             the horizon; inclusive canvas floor(min) .. ceil(max) after
//             snapping near-integers; the canvas budget; the conditioning
//             test on size-normalised coordinates with scaled partial
//             pivoting; the inverse normalised by its largest entry)
//   feather   src/s6/s6.cu:147-215 (per canvas pixel: A at the pixel, B through
//             the inverse with the denominator guard; bilinear samples of the
//             pixel-centre grid after snapping near-integers; each image
//             weighted by its distance-to-edge score; quantised
//             floor(clamp(255 c) + 0.5)); the union mask in {0, 1}
//   checks    src/s6/s6.cu:300-345 (argument order, overlap rules, the
//             optional statistics counters)
// Only the feather blend is built; the multiband modes are rejected.
// The device arithmetic is double and float with every product and sum
// rounded on its own (no contraction), which the CPU oracle restates.
#include <algorithm>
#include <cmath>
#include <limits>
#include <utility>

#include "common.cuh"
#include "stitch_b200.h"

namespace stitch::b200::s6k {

using Real = long double;

namespace {

bool valid_policy(const s6::GeometryPolicy& p) {
    return std::isfinite(p.denominator_tolerance) && p.denominator_tolerance > 0 && p.denominator_tolerance < 1 &&
           std::isfinite(p.inverse_tolerance) && p.inverse_tolerance > 0 && p.inverse_tolerance < 1 &&
           std::isfinite(p.snap_tolerance) && p.snap_tolerance >= 0 && p.snap_tolerance < 0.5 &&
           p.max_canvas_pixels > 0;
}

void mul3(const Real* a, const Real* b, Real* out) {
    Real t[9] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) t[3 * r + c] += a[3 * r + k] * b[3 * k + c];
    std::copy(t, t + 9, out);
}

bool scale_by_largest(Real* m) {
    Real big = 0;
    for (int i = 0; i < 9; ++i) {
        if (!std::isfinite(m[i])) return false;
        big = std::max(big, std::fabs(m[i]));
    }
    if (big == 0) return false;
    for (int i = 0; i < 9; ++i) m[i] /= big;
    return true;
}

Real row_norm(const Real* m) {
    Real n = 0;
    for (int r = 0; r < 3; ++r) n = std::max(n, std::fabs(m[3 * r]) + std::fabs(m[3 * r + 1]) + std::fabs(m[3 * r + 2]));
    return n;
}

// Gauss-Jordan on [M | I] with row pivots chosen by |a| / row scale; fails
// when a pivot score is not above the tolerance or the condition number
// ||M||_inf ||M^-1||_inf reaches 1 / tolerance.
bool invert3(const Real* m, Real tol, Real* inv) {
    Real a[3][6] = {}, rs[3] = {};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            a[r][c] = m[3 * r + c];
            rs[r] = std::max(rs[r], std::fabs(a[r][c]));
        }
        if (rs[r] == 0) return false;
        a[r][r + 3] = 1;
    }
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        Real best = 0;
        for (int r = col; r < 3; ++r) {
            const Real sc = std::fabs(a[r][col]) / rs[r];
            if (sc > best) {
                best = sc;
                piv = r;
            }
        }
        if (!std::isfinite(best) || best <= tol) return false;
        if (piv != col) {
            for (int c = 0; c < 6; ++c) std::swap(a[piv][c], a[col][c]);
            std::swap(rs[piv], rs[col]);
        }
        const Real d = a[col][col];
        for (int c = 0; c < 6; ++c) a[col][c] /= d;
        for (int r = 0; r < 3; ++r) {
            if (r == col) continue;
            const Real f = a[r][col];
            for (int c = 0; c < 6; ++c) a[r][c] -= f * a[col][c];
        }
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            if (!std::isfinite(a[r][c + 3])) return false;
            inv[3 * r + c] = a[r][c + 3];
        }
    const Real cond = row_norm(m) * row_norm(inv);
    return std::isfinite(cond) && cond * tol < 1;
}

Real snap(Real x, const s6::GeometryPolicy& p) {
    const Real near = std::round(x);
    const Real floor_tol = 16 * std::numeric_limits<double>::epsilon() * std::max(Real(1), std::fabs(x));
    return std::fabs(x - near) <= std::max(Real(p.snap_tolerance), floor_tol) ? near : x;
}

bool valid_geometry(const s6::Geometry& g) {
    if (g.width <= 0 || g.height <= 0 ||
        static_cast<std::size_t>(g.width) > std::numeric_limits<std::size_t>::max() / static_cast<std::size_t>(g.height) ||
        g.width_a <= 0 || g.height_a <= 0 || g.width_b <= 0 || g.height_b <= 0 || g.origin_x > 0 || g.origin_y > 0)
        return false;
    if (static_cast<long long>(g.origin_x) + g.width - 1 < g.width_a - 1LL ||
        static_cast<long long>(g.origin_y) + g.height - 1 < g.height_a - 1LL)
        return false;
    double big = 0;
    for (double v : g.inverse) {
        if (!std::isfinite(v)) return false;
        big = std::max(big, std::fabs(v));
    }
    return big > 0 && std::isfinite(g.denominator_tolerance) && g.denominator_tolerance > 0 &&
           g.denominator_tolerance < 1 && std::isfinite(g.snap_tolerance) && g.snap_tolerance >= 0 &&
           g.snap_tolerance < 0.5;
}

bool valid_mode(s6::BlendMode m) {
    return m == s6::BlendMode::Feather || m == s6::BlendMode::Multiband3 || m == s6::BlendMode::Multiband5;
}

struct Span {
    std::uintptr_t first, last;  // half-open
};

bool image_span(const ImageView& v, PixelFormat f, Span* s) {
    const std::size_t ch = f == PixelFormat::RGB8 ? 3 : 1;
    if (!v.data || v.width <= 0 || v.height <= 0 || v.pitch_bytes <= 0 || v.format != f) return false;
    const std::size_t row = static_cast<std::size_t>(v.width) * ch;
    if (row > static_cast<std::size_t>(v.pitch_bytes)) return false;
    const auto max = std::numeric_limits<std::uintptr_t>::max();
    const auto rows = static_cast<std::size_t>(v.height - 1), pitch = static_cast<std::size_t>(v.pitch_bytes);
    if (rows > (max - row) / pitch) return false;
    const std::size_t span = rows * pitch + row;
    s->first = reinterpret_cast<std::uintptr_t>(v.data);
    if (s->first > max - span) return false;
    s->last = s->first + span;
    return true;
}

bool overlap(const Span& a, const Span& b) { return a.first < b.last && b.first < a.last; }

}  // namespace

// ------------------------------------------------------------------ device

// Snaps a sample coordinate within max(tolerance, 16 eps max(1, |x|)) of an
// integer onto it; inside the pixel-centre grid [0, n - 1]?
__device__ __forceinline__ bool centre_coord(double& x, int n, double tol) {
    if (!isfinite(x)) return false;
    const double near = nearbyint(x);
    const double roundoff = __dmul_rn(16 * 2.2204460492503131e-16, fmax(1.0, fabs(x)));
    if (fabs(__dsub_rn(x, near)) <= fmax(tol, roundoff)) x = near;
    return x >= 0 && x <= n - 1.0;
}

// Distance-to-edge score min((x + .5) / w, (w - .5 - x) / w, (y + .5) / h,
// (h - .5 - y) / h) with two divisions: correctly rounded division by a
// positive number preserves order, so the smaller of two quotients over the
// same w is the quotient of the smaller numerator (both numerators >= 0.5).
__device__ __forceinline__ double edge_score(double x, double y, double w, double h) {
    return fmin(__ddiv_rn(fmin(__dadd_rn(x, 0.5), __dsub_rn(__dsub_rn(w, 0.5), x)), w),
                __ddiv_rn(fmin(__dadd_rn(y, 0.5), __dsub_rn(__dsub_rn(h, 0.5), y)), h));
}

// General bilinear sample of the pixel-centre grid at (x, y).
__device__ __forceinline__ bool sample(const ImageView& im, double x, double y, float* rgb, double& score,
                                       double tol) {
    if (!centre_coord(x, im.width, tol) || !centre_coord(y, im.height, tol)) return false;
    const int x0 = static_cast<int>(floor(x)), y0 = static_cast<int>(floor(y));
    const int x1 = x0 < im.width - 1 ? x0 + 1 : x0;
    const int y1 = y0 < im.height - 1 ? y0 + 1 : y0;
    const double ax = __dsub_rn(x, x0), ay = __dsub_rn(y, y0);
    const double bx = __dsub_rn(1.0, ax), by = __dsub_rn(1.0, ay);
    const std::uint8_t* r0 = im.data + static_cast<std::size_t>(y0) * im.pitch_bytes;
    const std::uint8_t* r1 = im.data + static_cast<std::size_t>(y1) * im.pitch_bytes;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double v0 = __dadd_rn(__dmul_rn(bx, r0[3 * x0 + c]), __dmul_rn(ax, r0[3 * x1 + c]));
        const double v1 = __dadd_rn(__dmul_rn(bx, r1[3 * x0 + c]), __dmul_rn(ax, r1[3 * x1 + c]));
        rgb[c] = static_cast<float>(__ddiv_rn(__dadd_rn(__dmul_rn(by, v0), __dmul_rn(ay, v1)), 255.0));
    }
    score = edge_score(x, y, im.width, im.height);
    return true;
}

// The same sample at integer (x, y), which is where A is sampled: no snap
// moves it, both bilinear weights are exactly 0, so each channel is the byte
// p itself and the colour is (float)(p / 255.0), read from `unit`.
__device__ __forceinline__ bool sample_at_pixel(const ImageView& im, int x, int y, const float* unit, float* rgb,
                                                double& score) {
    if (x < 0 || x >= im.width || y < 0 || y >= im.height) return false;
    const std::uint8_t* px = im.data + static_cast<std::size_t>(y) * im.pitch_bytes + 3 * x;
#pragma unroll
    for (int c = 0; c < 3; ++c) rgb[c] = unit[px[c]];
    score = edge_score(x, y, im.width, im.height);
    return true;
}

__device__ __forceinline__ std::uint8_t quantize(float c) {
    return static_cast<std::uint8_t>(floorf(__fadd_rn(fminf(255.0f, fmaxf(0.0f, __fmul_rn(255.0f, c))), 0.5f)));
}

struct FeatherArgs {
    ImageView a, b, out, mask;
    s6::Geometry g;
    unsigned long long* stats;  // {union, overlap} or null
};

constexpr int kS6BlockX = 32, kS6BlockY = 8;

__global__ __launch_bounds__(kS6BlockX * kS6BlockY) void feather_kernel(const __grid_constant__ FeatherArgs p) {
    __shared__ unsigned long long sums[2];
    __shared__ float unit[256];
    static_assert(kS6BlockX * kS6BlockY == 256, "one byte value per thread");
    const s6::Geometry& g = p.g;
    const int x = blockIdx.x * kS6BlockX + threadIdx.x, y = blockIdx.y * kS6BlockY + threadIdx.y;
    const int t = threadIdx.y * kS6BlockX + threadIdx.x;
    unit[t] = static_cast<float>(__ddiv_rn(static_cast<double>(t), 255.0));
    if (t < 2) sums[t] = 0;
    __syncthreads();
    bool ma = false, mb = false;
    if (x < g.width && y < g.height) {
        const int ia = x + g.origin_x, ja = y + g.origin_y;  // no overflow: origin <= 0 < x
        const double xa = ia, ya = ja;
        float ra[3] = {}, rb[3] = {};
        double sa = 0, sb = 0;
        ma = sample_at_pixel(p.a, ia, ja, unit, ra, sa);
        const double* m = g.inverse;
        const double den = __dadd_rn(__dadd_rn(__dmul_rn(m[6], xa), __dmul_rn(m[7], ya)), m[8]);
        const double den_scale = __dadd_rn(__dadd_rn(fabs(__dmul_rn(m[6], xa)), fabs(__dmul_rn(m[7], ya))), fabs(m[8]));
        if (isfinite(den) && den_scale > 0 && fabs(den) > __dmul_rn(g.denominator_tolerance, den_scale)) {
            const double xb = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], xa), __dmul_rn(m[1], ya)), m[2]), den);
            const double yb = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], xa), __dmul_rn(m[4], ya)), m[5]), den);
            mb = sample(p.b, xb, yb, rb, sb, g.snap_tolerance);
        }
        p.mask.data[static_cast<std::size_t>(y) * p.mask.pitch_bytes + x] = ma || mb ? 1 : 0;
        std::uint8_t* o = p.out.data + static_cast<std::size_t>(y) * p.out.pitch_bytes + 3 * x;
        const double sw = __dadd_rn(sa, sb);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float col = ma && mb ? static_cast<float>(__ddiv_rn(
                                             __dadd_rn(__dmul_rn(sa, ra[c]), __dmul_rn(sb, rb[c])), sw))
                                       : (ma ? ra[c] : rb[c]);
            o[c] = quantize(col);
        }
    }
    if (p.stats) {
        const unsigned u = __ballot_sync(0xffffffffu, ma || mb), v = __ballot_sync(0xffffffffu, ma && mb);
        if ((t & 31) == 0) {
            if (u) atomicAdd(&sums[0], static_cast<unsigned long long>(__popc(u)));
            if (v) atomicAdd(&sums[1], static_cast<unsigned long long>(__popc(v)));
        }
        __syncthreads();
        if (t == 0) {
            if (sums[0]) atomicAdd(&p.stats[0], sums[0]);
            if (sums[1]) atomicAdd(&p.stats[1], sums[1]);
        }
    }
}

}  // namespace stitch::b200::s6k

namespace stitch::s6 {

using namespace b200::s6k;

Status prepare_geometry(int width_a, int height_a, int width_b, int height_b, const double* h,
                        const GeometryPolicy& policy, Geometry* out) {
    if (!out) return Status::INVALID_ARGUMENT;
    Real mtx[9] = {};  // copied first: h may alias out->inverse
    if (h) std::copy(h, h + 9, mtx);
    *out = Geometry{};
    if (!h || width_a <= 0 || height_a <= 0 || width_b <= 0 || height_b <= 0 || !valid_policy(policy))
        return Status::INVALID_ARGUMENT;
    if (!scale_by_largest(mtx)) return Status::DEGENERATE;
    const Real bx = Real(width_b) - 1, by = Real(height_b) - 1;
    const Real dscale = std::fabs(mtx[6]) * bx + std::fabs(mtx[7]) * by + std::fabs(mtx[8]);
    if (!(dscale > 0) || !std::isfinite(dscale)) return Status::DEGENERATE;
    const Real dfloor = policy.denominator_tolerance * dscale;
    Real x0 = 0, y0 = 0, x1 = Real(width_a) - 1, y1 = Real(height_a) - 1;
    int side = 0;
    for (int corner = 0; corner < 4; ++corner) {
        const Real cx = (corner & 1) ? bx : 0, cy = (corner & 2) ? by : 0;
        const Real w = mtx[6] * cx + mtx[7] * cy + mtx[8];
        if (!std::isfinite(w) || std::fabs(w) <= dfloor) return Status::DEGENERATE;
        const int sg = w > 0 ? 1 : -1;
        if (side && sg != side) return Status::DEGENERATE;
        side = sg;
        const Real px = (mtx[0] * cx + mtx[1] * cy + mtx[2]) / w;
        const Real py = (mtx[3] * cx + mtx[4] * cy + mtx[5]) / w;
        if (!std::isfinite(px) || !std::isfinite(py)) return Status::DEGENERATE;
        x0 = std::min(x0, px);
        y0 = std::min(y0, py);
        x1 = std::max(x1, px);
        y1 = std::max(y1, py);
    }
    x0 = std::floor(snap(x0, policy));
    y0 = std::floor(snap(y0, policy));
    x1 = std::ceil(snap(x1, policy));
    y1 = std::ceil(snap(y1, policy));
    const Real cw = x1 - x0 + 1, ch = y1 - y0 + 1;
    constexpr int imax = std::numeric_limits<int>::max(), imin = std::numeric_limits<int>::min();
    if (x0 < imin || y0 < imin || x0 > imax || y0 > imax || !std::isfinite(cw) || !std::isfinite(ch) || cw < 1 ||
        ch < 1 || cw > imax || ch > imax)
        return Status::INSUFFICIENT_WORKSPACE;
    const auto uw = static_cast<std::size_t>(cw), uh = static_cast<std::size_t>(ch);
    if (uw > std::numeric_limits<std::size_t>::max() / uh || uw > policy.max_canvas_pixels / uh)
        return Status::INSUFFICIENT_WORKSPACE;
    // condition test in size-normalised coordinates (centred, scaled by the
    // larger extent), so that a pixel translation is not called singular
    const Real na_s = std::max({Real(1), Real(width_a) - 1, Real(height_a) - 1});
    const Real nb_s = std::max({Real(1), bx, by});
    const Real cax = (Real(width_a) - 1) / 2, cay = (Real(height_a) - 1) / 2;
    const Real na[9] = {1 / na_s, 0, -cax / na_s, 0, 1 / na_s, -cay / na_s, 0, 0, 1};
    const Real nb_inv[9] = {nb_s, 0, bx / 2, 0, nb_s, by / 2, 0, 0, 1};
    Real t[9], hn[9], hn_inv[9], inv[9];
    mul3(na, mtx, t);
    mul3(t, nb_inv, hn);
    if (!scale_by_largest(hn) || !invert3(hn, policy.inverse_tolerance, hn_inv)) return Status::DEGENERATE;
    mul3(nb_inv, hn_inv, t);
    mul3(t, na, inv);
    if (!scale_by_largest(inv)) return Status::DEGENERATE;
    Geometry g{};
    g.width = static_cast<int>(cw);
    g.height = static_cast<int>(ch);
    g.origin_x = static_cast<int>(x0);
    g.origin_y = static_cast<int>(y0);
    g.width_a = width_a;
    g.height_a = height_a;
    g.width_b = width_b;
    g.height_b = height_b;
    g.denominator_tolerance = policy.denominator_tolerance;
    g.snap_tolerance = policy.snap_tolerance;
    for (int i = 0; i < 9; ++i) {
        g.inverse[i] = static_cast<double>(inv[i]);
        if (!std::isfinite(g.inverse[i])) return Status::DEGENERATE;
    }
    *out = g;
    return Status::OK;
}

int effective_reductions(const Geometry& g, BlendMode mode) {
    if (!valid_mode(mode) || !valid_geometry(g)) return -1;
    if (mode == BlendMode::Feather) return 0;
    int n = 0, w = g.width, h = g.height;
    const int want = mode == BlendMode::Multiband3 ? 3 : 5;
    while ((w > 1 || h > 1) && n < want) {
        w = w / 2 + w % 2;
        h = h / 2 + h % 2;
        ++n;
    }
    return n;
}

Status s6_workspace_bytes(const Geometry& g, BlendMode mode, std::size_t* bytes) {
    if (!bytes) return Status::INVALID_ARGUMENT;
    *bytes = 0;
    if (!valid_geometry(g) || mode != BlendMode::Feather) return Status::INVALID_ARGUMENT;
    return Status::OK;  // the feather blend is fused and needs no workspace
}

Status render(const ImageView& a, const ImageView& b, const Geometry& g, BlendMode mode, const ImageView& output,
              const ImageView& mask, void* workspace, std::size_t available, cudaStream_t stream,
              RenderStatistics* statistics) {
    if (!valid_geometry(g) || mode != BlendMode::Feather) return Status::INVALID_ARGUMENT;
    if (a.width != g.width_a || a.height != g.height_a || b.width != g.width_b || b.height != g.height_b ||
        output.width != g.width || output.height != g.height || mask.width != g.width || mask.height != g.height)
        return Status::INVALID_ARGUMENT;
    Span spans[4];
    if (!image_span(a, PixelFormat::RGB8, &spans[0]) || !image_span(b, PixelFormat::RGB8, &spans[1]) ||
        !image_span(output, PixelFormat::RGB8, &spans[2]) || !image_span(mask, PixelFormat::GRAY8, &spans[3]))
        return Status::INVALID_ARGUMENT;
    for (int i = 0; i < 4; ++i)
        for (int k = i + 1; k < 4; ++k)
            if (!(i == 0 && k == 1) && overlap(spans[i], spans[k])) return Status::INVALID_ARGUMENT;
    if (statistics) {
        const auto at = reinterpret_cast<std::uintptr_t>(statistics);
        const auto max = std::numeric_limits<std::uintptr_t>::max();
        if (at % alignof(RenderStatistics) || at > max - sizeof(RenderStatistics)) return Status::INVALID_ARGUMENT;
        const Span counters{at, at + sizeof(RenderStatistics)};
        for (const auto& sp : spans)
            if (overlap(sp, counters)) return Status::INVALID_ARGUMENT;
        if (workspace && available) {
            const auto w = reinterpret_cast<std::uintptr_t>(workspace);
            if (w > max - available || overlap(counters, Span{w, w + available})) return Status::INVALID_ARGUMENT;
        }
    }
    if (statistics && cudaMemsetAsync(statistics, 0, sizeof(RenderStatistics), stream) != cudaSuccess)
        return Status::CUDA_ERROR;
    FeatherArgs args{a, b, output, mask, g, reinterpret_cast<unsigned long long*>(statistics)};
    const dim3 block(kS6BlockX, kS6BlockY);
    const dim3 grid(b200::ceil_div(g.width, kS6BlockX), b200::ceil_div(g.height, kS6BlockY));
    if (grid.y > 65535) return Status::INVALID_ARGUMENT;
    feather_kernel<<<grid, block, 0, stream>>>(args);
    b200::note_launches(1);
    return b200::launch_status();
}

}  // namespace stitch::s6

extern "C" {

void stitch_s6_default_policy(stitch_s6_policy* p) {
    if (!p) return;
    const stitch::s6::GeometryPolicy d{};
    *reinterpret_cast<stitch::s6::GeometryPolicy*>(p) = d;
}

int stitch_s6_prepare_geometry(int wa, int ha, int wb, int hb, const double* h, const stitch_s6_policy* policy,
                               stitch_s6_geometry* out) {
    using namespace stitch::s6;
    const GeometryPolicy p = policy ? *reinterpret_cast<const GeometryPolicy*>(policy) : GeometryPolicy{};
    return static_cast<int>(prepare_geometry(wa, ha, wb, hb, h, p, reinterpret_cast<Geometry*>(out)));
}

int stitch_s6_workspace_bytes(const stitch_s6_geometry* g, int mode, size_t* bytes) {
    using namespace stitch::s6;
    if (!g) return static_cast<int>(stitch::Status::INVALID_ARGUMENT);
    return static_cast<int>(
        s6_workspace_bytes(*reinterpret_cast<const Geometry*>(g), static_cast<BlendMode>(mode), bytes));
}

int stitch_s6_render(const stitch_image_view* a, const stitch_image_view* b, const stitch_s6_geometry* g, int mode,
                     const stitch_image_view* output, const stitch_image_view* mask, void* workspace,
                     size_t workspace_bytes, void* stream, uint64_t* statistics) {
    using namespace stitch;
    if (!a || !b || !g || !output || !mask) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(s6::render(
        *reinterpret_cast<const ImageView*>(a), *reinterpret_cast<const ImageView*>(b),
        *reinterpret_cast<const s6::Geometry*>(g), static_cast<s6::BlendMode>(mode),
        *reinterpret_cast<const ImageView*>(output), *reinterpret_cast<const ImageView*>(mask), workspace,
        workspace_bytes, static_cast<cudaStream_t>(stream), reinterpret_cast<s6::RenderStatistics*>(statistics)));
}

}  // extern "C"
