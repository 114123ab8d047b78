// The MSAC residual divides both projected coordinates by z through one
// correctly rounded reciprocal (Markstein's theorem). This checks, on the
// device, that each quotient equals the plain division bit for bit and that
// the residual equals the plain two-division form bit for bit, over seeded
// random operands: wide exponent ranges for the quotient, random homographies
// and pixel coordinates (plus far-out ones) for the residual.
#include <cstdio>
#include <cstdint>

#include "s5_kernels.cuh"

using stitch::b200::s5k::div_by_recip;
using stitch::b200::s5k::Pt;
using stitch::b200::s5k::residual2;

__device__ std::uint64_t mix(std::uint64_t v) {
    v += 0x9e3779b97f4a7c15ULL;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
    return v ^ (v >> 31);
}

// A double with a random 52-bit mantissa, random sign and exponent in [lo, hi].
__device__ double rnd(std::uint64_t& s, int lo, int hi) {
    s = mix(s);
    const int e = lo + static_cast<int>(s % static_cast<std::uint64_t>(hi - lo + 1));
    s = mix(s);
    const double m = 1.0 + static_cast<double>(s >> 12) * 0x1p-52;
    return ((s & 1) ? -1.0 : 1.0) * ldexp(m, e);
}

__device__ double residual_plain(const double* h, const Pt& p) {
    const double z = h[6] * p.bx + h[7] * p.by + h[8];
    if (!stitch::b200::s5k::fin(z) || fabs(z) < 1e-15) return DBL_MAX;
    const double dx = (h[0] * p.bx + h[1] * p.by + h[2]) / z - p.ax;
    const double dy = (h[3] * p.bx + h[4] * p.by + h[5]) / z - p.ay;
    const double r = dx * dx + dy * dy;
    return stitch::b200::s5k::fin(r) ? r : DBL_MAX;
}

__global__ void check(unsigned long long n, unsigned long long* bad) {
    unsigned long long local = 0;
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        std::uint64_t s = i * 0x2545f4914f6cdd1dULL + 12345;
        // quotients: |b| in [2^-49, 2^996] (1/b normal), a over a wide range
        const double a = rnd(s, -300, 300), b = rnd(s, -49, 996);
        const double q = a / b;
        if (fabs(q) >= 0x1p-1022 && fabs(q) <= DBL_MAX &&
            __double_as_longlong(div_by_recip(a, b, __drcp_rn(b))) != __double_as_longlong(q))
            ++local;
        // guarded division (any operands, zeros and extremes included): raw bits,
        // so the sign of a zero counts
        {
            s = mix(s);
            const int kind = static_cast<int>(s & 7);
            const double ga = kind == 0 ? 0.0 : kind == 1 ? -0.0 : rnd(s, kind == 2 ? -1074 : -1022, kind == 3 ? 1023 : 200);
            const double gb = rnd(s, kind == 4 ? -1074 : -1022, kind == 5 ? 1023 : 200);
            if (__double_as_longlong(stitch::b200::s5k::div_guarded(ga, gb, stitch::b200::s5k::recip_or_nan(gb))) !=
                __double_as_longlong(ga / gb))
                ++local;
        }
        // residuals: a homography near the identity or random, pixel or far-out points
        double h[9];
        s = mix(s);
        const bool wild = (s & 7) == 0;
        for (int k = 0; k < 9; ++k) h[k] = wild ? rnd(s, -30, 30) : 0.0;
        if (!wild) {
            h[0] = 1.0 + rnd(s, -12, -4); h[1] = rnd(s, -12, -4); h[2] = rnd(s, -2, 9);
            h[3] = rnd(s, -12, -4); h[4] = 1.0 + rnd(s, -12, -4); h[5] = rnd(s, -2, 9);
            h[6] = rnd(s, -30, -12); h[7] = rnd(s, -30, -12); h[8] = 1.0;
        }
        s = mix(s);
        const int span = (s & 15) == 0 ? 40 : 12;
        const Pt p{fabs(rnd(s, -2, span)), fabs(rnd(s, -2, span)), fabs(rnd(s, -2, span)), fabs(rnd(s, -2, span))};
        if (__double_as_longlong(residual2(h, p)) != __double_as_longlong(residual_plain(h, p))) ++local;
    }
    if (local) atomicAdd(bad, local);
}

int main() {
    unsigned long long* bad = nullptr;
    if (cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess) return 1;
    cudaMemset(bad, 0, sizeof(unsigned long long));
    const unsigned long long n = 1ull << 27;
    check<<<148 * 16, 256>>>(n, bad);
    unsigned long long h = 0;
    if (cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    printf("inputs %llu mismatch %llu\n", n, h);
    cudaFree(bad);
    return 0;
}
