// S5 kernels: batched MSAC homography (B -> A) with counter-based sampling,
// sm_100a. This translation unit must be compiled with -fmad=false: every
// double product and sum below is rounded on its own, exactly as in the
// reference's solver evaluated without contraction, so results are
// reproducible bit for bit against the CPU oracle.
//
// Reference semantics (file:line in the reference tree):
//   solver math ............ src/s5/s5_math.hpp:98-263
//   prepare / reuse checks .. src/s5/s5.cu:35-83
//   hypothesis generation ... src/s5/s5.cu:85-99
//   MSAC score: 128 lanes, lane l sums terms l, l+128, ... in order, then a
//   halving tree ............ src/s5/s5.cu:101-122
//   winner: valid, then lower loss, then lower hypothesis index
//                             src/s5/s5.cu:124-132
//   finish: serial re-score, refinement accepted on a strictly lower loss,
//   inlier mask r^2 <= tau^2, telemetry, H = D_A^-1 H_s D_B
//                             src/s5/s5.cu:139-212
//
// Layout of the work: a warp owns HPW consecutive hypotheses; lanes
// 0..HPW-1 each draw one sample and test it for degeneracy, then the whole
// warp fits each usable sample (the 8x9 system in shared memory, entries split
// over the lanes) and scores it. Lane l of the warp plays the reference's
// virtual lanes l, l+32, l+64 and l+96, so both the per-lane sums and the
// reduction tree are the reference's, operation for operation.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace stitch::b200::s5k {

struct Pt {
    double ax, ay, bx, by;
};

struct Model {
    double h[9];
    double loss;
    int hypothesis;
    int valid;
};

// Persistent per-pair search state at offset 0 of the S5 workspace.
struct State {
    Model best;  // raw winner over hypotheses [0, evaluated)
    HomographyResult result;
    const float* ax;
    const float* ay;
    const float* bx;
    const float* by;
    const std::int32_t* idx_a;
    const std::int32_t* idx_b;
    const int* count_a;
    const int* count_b;
    const int* count_m;
    int na, nb, nm;
    int cap_a, cap_b, cap_m;
    int evaluated;
    int batch_size;
    double threshold;
    std::uint64_t seed, generation;
    ScaleInfo scale_a, scale_b;
    int status;
    // bits of the smallest loss of a fully scored model of this search (or
    // of the previous winner), +inf when none: a pruning bound shared by
    // every warp of the pair (nonnegative doubles order like their bits)
    unsigned long long bound;
};

constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;  // +inf

constexpr int kSearchThreads = 256;
constexpr int kSearchWarps = kSearchThreads / 32;
constexpr int kMaxSearchBlocks = 2 * kSmCount;
constexpr int kStagePoints = 4096;  // matched points staged in shared memory per search block
constexpr int kFinishThreads = 256;
constexpr int kFinishChunk = 256;

// Inputs of one pair, as the caller passed them.
struct PairIO {
    Keypoints a, b;
    Matches m;
    ScaleInfo sa, sb;
    ::stitch::s5::Config c;
    State* state;
    Model* block_best;  // [kMaxSearchBlocks]
    int search_blocks;  // blocks the search launch used for this pair
    int hpw;            // hypotheses per warp
    std::uint8_t* mask;
    double inverse_a[9];  // D_A^-1 (host)
    double d_b[9];        // D_B
    HomographyResult* result_out;  // optional second copy of the result (batched form)
};

template <class Job> struct OneJob {
    Job job;
    __device__ bool find(int block, Job* j, int* local) const {
        *j = job;
        *local = block;
        return true;
    }
};

template <class Job> struct JobTable {
    const Job* jobs;
    const int* prefix;
    int n;
    // optional block -> (job << 16 | block within the job) map: one load
    // instead of a binary search over the prefix
    const std::uint32_t* map = nullptr;
    int map_blocks = 0;
    __device__ bool find(int block, Job* j, int* local) const {
        if (map) {
            if (block >= map_blocks) return false;
            const std::uint32_t e = __ldg(map + block);
            *j = jobs[e >> 16];
            *local = static_cast<int>(e & 0xffffu);
            return true;
        }
        if (block >= prefix[n]) return false;
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= block) lo = mid; else hi = mid - 1;
        }
        *j = jobs[lo];
        *local = block - prefix[lo];
        return true;
    }
};

// ------------------------------------------------------------ solver math

__device__ __forceinline__ bool fin(double x) { return x == x && x <= DBL_MAX && x >= -DBL_MAX; }

__device__ __forceinline__ void mat3_mul(const double* a, const double* b, double* out) {
    double t[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            t[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[j + 3] + a[3 * i + 2] * b[j + 6];
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = t[i];
}

// Divide by the largest magnitude; entries finite and |det| > 1e-15.
__device__ __forceinline__ bool h_normalize(double* h) {
    double scale = 0.0;
    for (int i = 0; i < 9; ++i) {
        if (!fin(h[i])) return false;
        if (fabs(h[i]) > scale) scale = fabs(h[i]);
    }
    if (!(scale > 0.0)) return false;
    for (int i = 0; i < 9; ++i) h[i] /= scale;
    const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                       h[2] * (h[3] * h[7] - h[4] * h[6]);
    return fin(det) && fabs(det) > 1e-15;
}

// Squared forward reprojection error of B -> A; DBL_MAX when the projective
// denominator is not finite or too close to zero.
__device__ __forceinline__ double residual2(const double* h, const Pt& p) {
    const double z = h[6] * p.bx + h[7] * p.by + h[8];
    if (!fin(z) || fabs(z) < 1e-15) return DBL_MAX;
    const double dx = (h[0] * p.bx + h[1] * p.by + h[2]) / z - p.ax;
    const double dy = (h[3] * p.bx + h[4] * p.by + h[5]) / z - p.ay;
    const double r = dx * dx + dy * dy;
    return fin(r) ? r : DBL_MAX;
}

// SplitMix64 finaliser on a counter (public-domain algorithm, S. Vigna).
__device__ __forceinline__ std::uint64_t splitmix64(std::uint64_t v) {
    v += 0x9e3779b97f4a7c15ULL;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
    return v ^ (v >> 31);
}

// Four distinct indices in [0, n): draw k = counter seed ^ (4h + k) mod
// (n - k), stepped past the earlier draws in ascending order.
__device__ __forceinline__ void sample_four(int n, std::uint64_t seed, int h, int* s) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int v = static_cast<int>(splitmix64(seed ^ (static_cast<std::uint64_t>(h) * 4 + k)) %
                                 static_cast<std::uint64_t>(n - k));
        // earlier draws in ascending order
        int lo[3] = {s[0], s[1], s[2]};
        if (k >= 2 && lo[0] > lo[1]) { const int t = lo[0]; lo[0] = lo[1]; lo[1] = t; }
        if (k >= 3) {
            if (lo[1] > lo[2]) { const int t = lo[1]; lo[1] = lo[2]; lo[2] = t; }
            if (lo[0] > lo[1]) { const int t = lo[0]; lo[0] = lo[1]; lo[1] = t; }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < k && v >= lo[i]) ++v;
        s[k] = v;
    }
}

__device__ __forceinline__ double coord(const Pt& p, int image, int axis) {
    return image ? (axis ? p.by : p.bx) : (axis ? p.ay : p.ax);
}

// No three of the four points (in either image) nearly collinear.
__device__ __forceinline__ bool nondegenerate(const Pt* p) {
#pragma unroll
    for (int image = 0; image < 2; ++image) {
        double scale = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < i; ++j) {
                const double dx = coord(p[i], image, 0) - coord(p[j], image, 0);
                const double dy = coord(p[i], image, 1) - coord(p[j], image, 1);
                const double d = dx * dx + dy * dy;
                if (d > scale) scale = d;
            }
        if (!(scale > 0.0) || !fin(scale)) return false;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = i + 1; j < 4; ++j)
#pragma unroll
                for (int k = j + 1; k < 4; ++k) {
                    const double x1 = coord(p[j], image, 0) - coord(p[i], image, 0);
                    const double y1 = coord(p[j], image, 1) - coord(p[i], image, 1);
                    const double x2 = coord(p[k], image, 0) - coord(p[i], image, 0);
                    const double y2 = coord(p[k], image, 1) - coord(p[i], image, 1);
                    if (fabs(x1 * y2 - y1 * x2) <= 1e-8 * scale) return false;
                }
    }
    return true;
}

// Entry `col` of the two design rows of one normalised correspondence
// (x, y) -> (u, v): row 0 = {x, y, 1, 0, 0, 0, -u x, -u y, u},
// row 1 = {0, 0, 0, x, y, 1, -v x, -v y, v}.
__device__ __forceinline__ double design(int row, int col, double x, double y, double u, double v) {
    if (row == 0) {
        switch (col) {
            case 0: return x; case 1: return y; case 2: return 1.0;
            case 3: case 4: case 5: return 0.0;
            case 6: return -u * x; case 7: return -u * y; default: return u;
        }
    }
    switch (col) {
        case 0: case 1: case 2: return 0.0;
        case 3: return x; case 4: return y; case 5: return 1.0;
        case 6: return -v * x; case 7: return -v * y; default: return v;
    }
}

// Gauss-Jordan with partial pivoting on the 8x9 normal equations, h33 = 1,
// then denormalisation and scaling; m is destroyed.
__device__ __forceinline__ bool solve_normalised(double (*m)[9], double cax, double cay, double cbx,
                                                 double cby, double sa, double sb, double* out) {
    double max_entry = 0.0;
    for (int i = 0; i < 8; ++i)
        if (fabs(m[i][i]) > max_entry) max_entry = fabs(m[i][i]);
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        for (int r = c + 1; r < 8; ++r)
            if (fabs(m[r][c]) > fabs(m[piv][c])) piv = r;
        if (!fin(m[piv][c]) || fabs(m[piv][c]) <= 1e-12 * max_entry) return false;
        for (int jx = c; jx < 9; ++jx) {
            const double t = m[c][jx]; m[c][jx] = m[piv][jx]; m[piv][jx] = t;
        }
        const double div = m[c][c];
        for (int jx = c; jx < 9; ++jx) m[c][jx] /= div;
        for (int r = 0; r < 8; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
            for (int jx = c; jx < 9; ++jx) m[r][jx] -= f * m[c][jx];
        }
    }
    double h[9];
    for (int i = 0; i < 8; ++i) h[i] = m[i][8];
    h[8] = 1.0;
    const double den_a[9] = {1.0 / sa, 0, cax, 0, 1.0 / sa, cay, 0, 0, 1};
    const double nrm_b[9] = {sb, 0, -sb * cbx, 0, sb, -sb * cby, 0, 0, 1};
    double tmp[9];
    mat3_mul(den_a, h, tmp);
    mat3_mul(tmp, nrm_b, out);
    return h_normalize(out);
}

// Gauss-Jordan of solve_normalised, run by all 32 lanes of a warp on M in
// shared memory (warp-private). Every entry goes through the serial
// solver's exact sequence of operations, so the model is bit-identical;
// lanes only split the independent per-entry work. Returns the same
// validity on every lane, and every lane holds the model in out.
__device__ inline bool warp_solve(double (*M)[9], double cax, double cay, double cbx, double cby, double sa,
                                  double sb, double* out) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    double max_entry = 0.0;
    for (int i = 0; i < 8; ++i)
        if (fabs(M[i][i]) > max_entry) max_entry = fabs(M[i][i]);
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        for (int r = c + 1; r < 8; ++r)
            if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
        const double pv = M[piv][c];
        if (!fin(pv) || fabs(pv) <= 1e-12 * max_entry) return false;
        __syncwarp();
        if (lane >= c && lane < 9) {
            const double t = M[c][lane];
            M[c][lane] = M[piv][lane];
            M[piv][lane] = t;
        }
        __syncwarp();
        const double div = M[c][c];
        __syncwarp();
        if (lane >= c && lane < 9) M[c][lane] /= div;
        __syncwarp();
        // entries (r, jx), r != c, jx >= c: M[r][jx] -= f_r * M[c][jx] with
        // f_r = M[r][c] read before any entry of row r changes
        double f[3], pr[3];
        int rr[3], jj[3];
        bool own[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int e = lane + 32 * s;
            rr[s] = e / 9;
            jj[s] = e % 9;
            own[s] = e < 72 && rr[s] != c && jj[s] >= c;
            f[s] = own[s] ? M[rr[s]][c] : 0.0;
            pr[s] = own[s] ? M[c][jj[s]] : 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 3; ++s)
            if (own[s]) M[rr[s]][jj[s]] -= f[s] * pr[s];
        __syncwarp();
    }
    double h[9];
    for (int i = 0; i < 8; ++i) h[i] = M[i][8];
    h[8] = 1.0;
    __syncwarp();
    const double den_a[9] = {1.0 / sa, 0, cax, 0, 1.0 / sa, cay, 0, 0, 1};
    const double nrm_b[9] = {sb, 0, -sb * cbx, 0, sb, -sb * cby, 0, 0, 1};
    double tmp[9];
    mat3_mul(den_a, h, tmp);
    mat3_mul(tmp, nrm_b, out);
    return h_normalize(out);
}

// Minimal 4-point model computed by a whole warp (all lanes pass the same
// points): normalisation on every lane, the 72 normal-matrix entries split
// over the lanes (each summed over the 4 points in order), then
// warp_solve. Bit-identical to fit4.
__device__ inline bool warp_fit4(const Pt* p, double (*M)[9], double* out) {
    const int lane = threadIdx.x & 31;
    double cax = 0, cay = 0, cbx = 0, cby = 0;
    for (int i = 0; i < 4; ++i) { cax += p[i].ax; cay += p[i].ay; cbx += p[i].bx; cby += p[i].by; }
    cax /= 4; cay /= 4; cbx /= 4; cby /= 4;
    double va = 0.0, vb = 0.0;
    for (int i = 0; i < 4; ++i) {
        va += (p[i].ax - cax) * (p[i].ax - cax) + (p[i].ay - cay) * (p[i].ay - cay);
        vb += (p[i].bx - cbx) * (p[i].bx - cbx) + (p[i].by - cby) * (p[i].by - cby);
    }
    if (!(va > 0.0) || !(vb > 0.0) || !fin(va) || !fin(vb)) return false;
    const double sa = sqrt(2.0 * 4 / va);
    const double sb = sqrt(2.0 * 4 / vb);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const int e = lane + 32 * s;
        if (e >= 72) continue;
        const int r = e / 9, c = e % 9;
        double acc = 0.0;
        for (int i = 0; i < 4; ++i) {
            const double x = (p[i].bx - cbx) * sb, y = (p[i].by - cby) * sb;
            const double u = (p[i].ax - cax) * sa, v = (p[i].ay - cay) * sa;
            acc += design(0, r, x, y, u, v) * design(0, c, x, y, u, v) +
                   design(1, r, x, y, u, v) * design(1, c, x, y, u, v);
        }
        M[r][c] = acc;
    }
    return warp_solve(M, cax, cay, cbx, cby, sa, sb, out);
}

// Minimal 4-point model on one thread with the 8x9 system in registers:
// every loop is unrolled and the pivot row swap is a predicated select per
// entry, so no entry is indexed at run time. Same operations, in the same
// order per entry, as fit4; bit-identical results.
__device__ __forceinline__ bool fit4_regs(const Pt* p, double* out) {
    double cax = 0, cay = 0, cbx = 0, cby = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) { cax += p[i].ax; cay += p[i].ay; cbx += p[i].bx; cby += p[i].by; }
    cax /= 4; cay /= 4; cbx /= 4; cby /= 4;
    double va = 0.0, vb = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        va += (p[i].ax - cax) * (p[i].ax - cax) + (p[i].ay - cay) * (p[i].ay - cay);
        vb += (p[i].bx - cbx) * (p[i].bx - cbx) + (p[i].by - cby) * (p[i].by - cby);
    }
    if (!(va > 0.0) || !(vb > 0.0) || !fin(va) || !fin(vb)) return false;
    const double sa = sqrt(2.0 * 4 / va);
    const double sb = sqrt(2.0 * 4 / vb);
    double m[8][9];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 9; ++c) m[r][c] = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double x = (p[i].bx - cbx) * sb, y = (p[i].by - cby) * sb;
        const double u = (p[i].ax - cax) * sa, v = (p[i].ay - cay) * sa;
        const double r0[9] = {x, y, 1, 0, 0, 0, -u * x, -u * y, u};
        const double r1[9] = {0, 0, 0, x, y, 1, -v * x, -v * y, v};
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int c = 0; c < 9; ++c) m[r][c] += r0[r] * r0[c] + r1[r] * r1[c];
    }
    double max_entry = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (fabs(m[i][i]) > max_entry) max_entry = fabs(m[i][i]);
    // A failed pivot makes the model invalid; the loop still runs to the
    // end (an early exit would stop full unrolling) and the values computed
    // after a failure are discarded.
    bool solvable = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        double best = fabs(m[c][c]);
        double pv = m[c][c];
#pragma unroll
        for (int r = c + 1; r < 8; ++r)
            if (fabs(m[r][c]) > best) { best = fabs(m[r][c]); piv = r; pv = m[r][c]; }
        solvable = solvable && fin(pv) && !(fabs(pv) <= 1e-12 * max_entry);
        // (loops run over all columns with a compile-time skip of jx < c, a
        // form that keeps every entry in a register after unrolling)
#pragma unroll
        for (int r = c + 1; r < 8; ++r) {
            const bool sw = r == piv;
#pragma unroll
            for (int jx = 0; jx < 9; ++jx) {
                if (jx < c) continue;
                const double a = m[c][jx], b = m[r][jx];
                m[c][jx] = sw ? b : a;
                m[r][jx] = sw ? a : b;
            }
        }
        const double div = m[c][c];
#pragma unroll
        for (int jx = 0; jx < 9; ++jx)
            if (jx >= c) m[c][jx] /= div;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
#pragma unroll
            for (int jx = 0; jx < 9; ++jx)
                if (jx >= c) m[r][jx] -= f * m[c][jx];
        }
    }
    if (!solvable) return false;
    double h[9];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = m[i][8];
    h[8] = 1.0;
    const double den_a[9] = {1.0 / sa, 0, cax, 0, 1.0 / sa, cay, 0, 0, 1};
    const double nrm_b[9] = {sb, 0, -sb * cbx, 0, sb, -sb * cby, 0, 0, 1};
    double tmp[9];
    mat3_mul(den_a, h, tmp);
    mat3_mul(tmp, nrm_b, out);
    return h_normalize(out);
}

// Minimal 4-point model (one thread).
__device__ inline bool fit4(const Pt* p, double* out) {
    double cax = 0, cay = 0, cbx = 0, cby = 0;
    for (int i = 0; i < 4; ++i) { cax += p[i].ax; cay += p[i].ay; cbx += p[i].bx; cby += p[i].by; }
    cax /= 4; cay /= 4; cbx /= 4; cby /= 4;
    double va = 0.0, vb = 0.0;
    for (int i = 0; i < 4; ++i) {
        va += (p[i].ax - cax) * (p[i].ax - cax) + (p[i].ay - cay) * (p[i].ay - cay);
        vb += (p[i].bx - cbx) * (p[i].bx - cbx) + (p[i].by - cby) * (p[i].by - cby);
    }
    if (!(va > 0.0) || !(vb > 0.0) || !fin(va) || !fin(vb)) return false;
    const double sa = sqrt(2.0 * 4 / va);
    const double sb = sqrt(2.0 * 4 / vb);
    double m[8][9];
    for (int r = 0; r < 8; ++r)
        for (int c = 0; c < 9; ++c) m[r][c] = 0.0;
    for (int i = 0; i < 4; ++i) {
        const double x = (p[i].bx - cbx) * sb, y = (p[i].by - cby) * sb;
        const double u = (p[i].ax - cax) * sa, v = (p[i].ay - cay) * sa;
        const double r0[9] = {x, y, 1, 0, 0, 0, -u * x, -u * y, u};
        const double r1[9] = {0, 0, 0, x, y, 1, -v * x, -v * y, v};
        for (int r = 0; r < 8; ++r)
            for (int c = 0; c < 9; ++c) m[r][c] += r0[r] * r0[c] + r1[r] * r1[c];
    }
    return solve_normalised(m, cax, cay, cbx, cby, sa, sb, out);
}

__device__ __forceinline__ bool valid_domain(const double* h, int width, int height) {
    const double z[4] = {h[8], h[6] * (width - 1) + h[8], h[7] * (height - 1) + h[8],
                         h[6] * (width - 1) + h[7] * (height - 1) + h[8]};
    for (int i = 0; i < 4; ++i)
        if (!fin(z[i]) || fabs(z[i]) < 1e-15 || (z[i] > 0.0) != (z[0] > 0.0)) return false;
    return true;
}

__device__ __forceinline__ bool better(const Model& a, const Model& b) {
    return a.valid && (!b.valid || a.loss < b.loss || (a.loss == b.loss && a.hypothesis < b.hypothesis));
}

__device__ __forceinline__ Pt gather(const PairIO& j, int i) {
    const int ia = j.m.idx_a[i], ib = j.m.idx_b[i];
    return Pt{static_cast<double>(j.a.x[ia]), static_cast<double>(j.a.y[ia]), static_cast<double>(j.b.x[ib]),
              static_cast<double>(j.b.y[ib])};
}

// Match i of the pair: from the staged float4 copy when it is staged.
__device__ __forceinline__ Pt point_at(const PairIO& j, const float4* pts, int i) {
    if (i < kStagePoints) {
        const float4 q = pts[i];
        return Pt{q.x, q.y, q.z, q.w};
    }
    return gather(j, i);
}

__device__ __forceinline__ bool same_scale(const ScaleInfo& a, const ScaleInfo& b) {
    if (a.orig_w != b.orig_w || a.orig_h != b.orig_h || a.work_w != b.work_w || a.work_h != b.work_h ||
        a.sx != b.sx || a.sy != b.sy)
        return false;
    for (int i = 0; i < 9; ++i)
        if (a.D[i] != b.D[i]) return false;
    return true;
}

// --------------------------------------------------------------- prepare

// Restart or validate an extension, then check counts, indices and
// coordinates of every match. One block per pair.
template <class Src>
__global__ __launch_bounds__(256) void prepare_kernel(const __grid_constant__ Src src) {
    __shared__ int go, bad;
    PairIO j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    State* s = j.state;
    if (threadIdx.x == 0) {
        const int na = *j.a.d_count, nb = *j.b.d_count, nm = *j.m.d_count;
        const auto& c = j.c;
        if (c.previous_hypotheses == 0) {
            s->best = Model{};
            s->ax = j.a.x; s->ay = j.a.y; s->bx = j.b.x; s->by = j.b.y;
            s->idx_a = j.m.idx_a; s->idx_b = j.m.idx_b;
            s->count_a = j.a.d_count; s->count_b = j.b.d_count; s->count_m = j.m.d_count;
            s->na = na; s->nb = nb; s->nm = nm;
            s->cap_a = j.a.capacity; s->cap_b = j.b.capacity; s->cap_m = j.m.capacity;
            s->evaluated = 0; s->batch_size = c.batch_size; s->threshold = c.threshold;
            s->seed = c.seed; s->generation = c.generation;
            s->scale_a = j.sa; s->scale_b = j.sb;
            s->status = static_cast<int>(Status::OK);
        } else if (s->evaluated != c.previous_hypotheses || s->generation != c.generation ||
                   s->seed != c.seed || s->threshold != c.threshold || s->batch_size != c.batch_size ||
                   s->ax != j.a.x || s->ay != j.a.y || s->bx != j.b.x || s->by != j.b.y ||
                   s->idx_a != j.m.idx_a || s->idx_b != j.m.idx_b || s->count_a != j.a.d_count ||
                   s->count_b != j.b.d_count || s->count_m != j.m.d_count || s->cap_a != j.a.capacity ||
                   s->cap_b != j.b.capacity || s->cap_m != j.m.capacity || s->na != na || s->nb != nb ||
                   s->nm != nm || !same_scale(s->scale_a, j.sa) || !same_scale(s->scale_b, j.sb)) {
            s->status = static_cast<int>(Status::INVALID_ARGUMENT);
        }
        s->bound = s->best.valid && fin(s->best.loss) ? static_cast<unsigned long long>(__double_as_longlong(s->best.loss))
                                                      : kInfBits;
        int g = s->status == static_cast<int>(Status::OK);
        if (g && (na < 0 || na > j.a.capacity || nb < 0 || nb > j.b.capacity || nm < 0 || nm > j.m.capacity)) {
            s->status = static_cast<int>(Status::INVALID_ARGUMENT);
            g = 0;
        }
        go = g;
        bad = 0;
    }
    __syncthreads();
    if (!go) return;
    const int na = s->na, nb = s->nb, nm = s->nm;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) {
        const int ia = j.m.idx_a[i], ib = j.m.idx_b[i];
        if (ia < 0 || ia >= na || ib < 0 || ib >= nb) { bad = 1; continue; }
        const Pt q = gather(j, i);
        if (!fin(q.ax) || !fin(q.ay) || !fin(q.bx) || !fin(q.by)) bad = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (bad) s->status = static_cast<int>(Status::INVALID_ARGUMENT);
        else if (nm < 4) s->status = static_cast<int>(Status::NOT_ENOUGH_POINTS);
    }
}

// ---------------------------------------------------------------- search

struct SearchJob {
    PairIO io;
    int first, count;  // hypotheses [first, first + count)
    Model* prefit;     // models of these hypotheses from fit_kernel, or null (fit in the search)
};

constexpr int kFitThreads = 128;

// One thread per hypothesis h in [first, first + count): the counter-based
// sample, the degeneracy test, the 4-point fit and the domain test, the same
// functions the search runs in place, into prefit[h - first] (valid = 0 for
// a rejected sample). A thread owns the whole 8x9 system, so this kernel
// runs with all the registers it needs, apart from the scoring.
template <class Src>
__global__ __launch_bounds__(kFitThreads) void fit_kernel(const __grid_constant__ Src src) {
    SearchJob sj;
    int block;
    if (!src.find(blockIdx.x, &sj, &block)) return;
    const PairIO& j = sj.io;
    const State* s = j.state;
    const int h = sj.first + block * kFitThreads + threadIdx.x;
    if (h >= sj.first + sj.count) return;
    Model m{};
    m.hypothesis = h;
    m.valid = 0;
    if (s->status == static_cast<int>(Status::OK)) {
        const int nm = s->nm;
        int idx[4] = {0, 0, 0, 0};
        sample_four(nm, j.c.seed, h, idx);
        Pt f[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = gather(j, idx[k]);
        m.valid = nondegenerate(f) && fit4_regs(f, m.h) && valid_domain(m.h, s->scale_b.work_w, s->scale_b.work_h);
    }
    sj.prefit[h - sj.first] = m;
}

// Block b of a pair walks warp rounds b*8 + w, b*8 + w + 8*blocks, ...; a
// round is HPW consecutive hypotheses. The block's best model goes to
// block_best[b].
// Three blocks per SM: the register-resident 4-point fit then spills to
// L1-backed local memory, but it is a small share of the work, and the
// scoring loop gains the occupancy (1 block: 0.62 ms, 3 blocks: 0.43 ms for
// 64 pairs x 2000 hypotheses x ~530 matches).
constexpr int kPruneEvery = 128;  // points between the pruning checks of a model (multiple of 128)

// kPrefit: the models come from fit_kernel (sj.prefit) and the kernel only
// scores (batched form: 0.387 -> 0.367 ms per step with the fit kernel
// included; 4 and 5 blocks per SM spill in the scoring loop and are slower).
template <class Src, bool kPrefit>
__global__ __launch_bounds__(kSearchThreads, 3) void search_kernel(const __grid_constant__ Src src) {
    extern __shared__ float4 pts[];
    __shared__ Model warp_best[kSearchWarps];
    SearchJob sj;
    int block;
    if (!src.find(blockIdx.x, &sj, &block)) return;
    const PairIO& j = sj.io;
    const State* s = j.state;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the warp's best model so far lives in shared memory, written by lane 0
    // (registers stay with the scoring loop)
    Model& best = warp_best[warp];
    if (lane == 0) best.valid = 0;
    __syncwarp();
    const bool ok = s->status == static_cast<int>(Status::OK);
    const int nm = ok ? s->nm : 0;
    const int staged = min(nm, kStagePoints);
    for (int i = threadIdx.x; i < staged; i += kSearchThreads) {
        const int ia = j.m.idx_a[i], ib = j.m.idx_b[i];
        pts[i] = make_float4(j.a.x[ia], j.a.y[ia], j.b.x[ib], j.b.y[ib]);
    }
    __syncthreads();
    if (ok) {
        const double thr2 = j.c.threshold * j.c.threshold;
        const int bw = s->scale_b.work_w, bh = s->scale_b.work_h;
        const std::uint64_t seed = j.c.seed;
        const int hpw = j.hpw;
        const int rounds = (sj.count + hpw - 1) / hpw;
        const int stride = j.search_blocks * kSearchWarps;
        for (int round = block * kSearchWarps + warp; round < rounds; round += stride) {
            const int h0 = sj.first + round * hpw;
            const int hend = min(sj.first + sj.count, h0 + hpw);
            // lanes 0..hpw-1 build one model each (system in registers)
            double hm[9];
            int valid = 0;
            if (kPrefit) {
                valid = lane < hend - h0 ? sj.prefit[h0 + lane - sj.first].valid : 0;
            } else if (lane < hend - h0) {
                int idx[4] = {0, 0, 0, 0};
                sample_four(nm, seed, h0 + lane, idx);
                Pt f[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (idx[k] < kStagePoints) {
                        const float4 q = pts[idx[k]];
                        f[k] = Pt{q.x, q.y, q.z, q.w};
                    } else {
                        f[k] = gather(j, idx[k]);
                    }
                }
                valid = nondegenerate(f) && fit4_regs(f, hm) && valid_domain(hm, bw, bh);
            }
            // then the whole warp scores the valid models one by one
            for (int k = 0; k < hend - h0; ++k) {
                if (!__shfl_sync(0xffffffffu, valid, k)) continue;
                double h[9];
                if (kPrefit) {
                    const Model& mk = sj.prefit[h0 + k - sj.first];  // the same address on every lane
#pragma unroll
                    for (int e = 0; e < 9; ++e) h[e] = mk.h[e];
                } else {
#pragma unroll
                    for (int e = 0; e < 9; ++e) h[e] = __shfl_sync(0xffffffffu, hm[e], k);
                }
                // Exact pruning against the smallest loss of a fully scored
                // model so far (this warp's best, or the pair's bound that
                // every warp publishes to): every term is >= 0 and a
                // correctly rounded sum of nonnegative values is nondecreasing
                // in each operand, so the tree sum of the partial accumulators
                // never exceeds the final loss. Once it is above that loss the
                // model cannot win (ties need equal losses).
                const double shared_bound =
                    __longlong_as_double(static_cast<long long>(*reinterpret_cast<volatile unsigned long long*>(&j.state->bound)));
                const double bound = best.valid && best.loss < shared_bound ? best.loss : shared_bound;
                const bool prune = bound <= DBL_MAX;
                // Lane l accumulates the points l, l+32, l+64, l+96 (virtual
                // lanes, slots 0..3) and every 128 after them in order: four
                // points per step, four independent FP64 chains. A point past
                // nm adds +0.0, which leaves a sum of nonnegative terms
                // (started at +0.0) bit for bit unchanged.
                double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
                bool lost = false;
                for (int base = 0; base < nm; base += 128) {  // warp-uniform trip count
                    const int i0 = base + lane, i1 = i0 + 32, i2 = i0 + 64, i3 = i0 + 96;
                    if (base + 128 <= nm) {  // every slot of the step holds a point
                        const Pt p0 = point_at(j, pts, i0), p1 = point_at(j, pts, i1);
                        const Pt p2 = point_at(j, pts, i2), p3 = point_at(j, pts, i3);
                        const double r0 = residual2(h, p0), r1 = residual2(h, p1);
                        const double r2 = residual2(h, p2), r3 = residual2(h, p3);
                        acc0 += r0 < thr2 ? r0 : thr2;
                        acc1 += r1 < thr2 ? r1 : thr2;
                        acc2 += r2 < thr2 ? r2 : thr2;
                        acc3 += r3 < thr2 ? r3 : thr2;
                    } else {
                        // the last, partial step: a virtual lane past nm adds
                        // +0.0, a no-op on a sum of nonnegative terms, so the
                        // chains with no point left (warp-uniform) are skipped
                        const double r0 = residual2(h, point_at(j, pts, min(i0, nm - 1)));
                        acc0 += i0 < nm ? (r0 < thr2 ? r0 : thr2) : 0.0;
                        if (base + 32 < nm) {
                            const double r1 = residual2(h, point_at(j, pts, min(i1, nm - 1)));
                            acc1 += i1 < nm ? (r1 < thr2 ? r1 : thr2) : 0.0;
                        }
                        if (base + 64 < nm) {
                            const double r2 = residual2(h, point_at(j, pts, min(i2, nm - 1)));
                            acc2 += i2 < nm ? (r2 < thr2 ? r2 : thr2) : 0.0;
                        }
                        if (base + 96 < nm) {
                            const double r3 = residual2(h, point_at(j, pts, min(i3, nm - 1)));
                            acc3 += i3 < nm ? (r3 < thr2 ? r3 : thr2) : 0.0;
                        }
                    }
                    if (prune && (base & (kPruneEvery - 1)) == kPruneEvery - 128 && base + 128 < nm) {
                        double part = (acc0 + acc2) + (acc1 + acc3);
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
                        if (__shfl_sync(0xffffffffu, part > bound ? 1 : 0, 0)) {
                            lost = true;
                            break;
                        }
                    }
                }
                if (lost) continue;
                // virtual lanes l, l+32, l+64, l+96: strides 64 and 32 of the tree
                double v = (acc0 + acc2) + (acc1 + acc3);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) {
                    Model cand;
#pragma unroll
                    for (int e = 0; e < 9; ++e) cand.h[e] = h[e];
                    cand.loss = v;
                    cand.hypothesis = h0 + k;
                    cand.valid = fin(v);
                    if (better(cand, best)) best = cand;
                    if (cand.valid) atomicMin(&j.state->bound, static_cast<unsigned long long>(__double_as_longlong(v)));
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Model b = warp_best[0];
        for (int w = 1; w < kSearchWarps; ++w)
            if (better(warp_best[w], b)) b = warp_best[w];
        j.block_best[block] = b;
    }
}

// ---------------------------------------------------------------- finish

// Sum over i < nm of f(i) in index order (one dependent chain, as the
// reference's single-thread loop), with the terms computed by the block.
template <class F>
__device__ double ordered_sum(int nm, double* buf /*kFinishChunk shared*/, F term) {
    __shared__ double total;
    if (threadIdx.x == 0) total = 0.0;
    for (int base = 0; base < nm; base += kFinishChunk) {
        const int n = min(kFinishChunk, nm - base);
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = term(base + i);
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = total;
#pragma unroll 8
            for (int i = 0; i < n; ++i) t += buf[i];
            total = t;
        }
    }
    __syncthreads();
    const double r = total;
    __syncthreads();
    return r;
}

// Least-squares refit over the points with keep[i] != 0: the centroid,
// scale and normal-matrix sums each run in index order as in the reference;
// the 72 matrix entries are accumulated by 72 threads side by side.
__device__ inline bool block_fit(const PairIO& j, int nm, const std::uint8_t* keep, double* out, double (*dv)[10],
                          std::uint8_t* ckeep /*kFinishChunk shared*/) {
    __shared__ double sums[6];
    __shared__ int kept;
    __shared__ double m[8][9];
    __shared__ int ok;
    const int t = threadIdx.x;
    if (t < 6) sums[t] = 0.0;
    if (t == 6) kept = 0;
    if (t < 72) m[t / 9][t % 9] = 0.0;
    // Each sum below starts at +0.0 and runs in index order on one thread
    // over terms the block computed beforehand; a dropped point contributes
    // +0.0, which leaves such a sum bit-identical to skipping the point
    // (round-to-nearest never turns a sum that starts at +0.0 into -0.0).
    // pass 1: centroids
    int mine = 0;
    for (int base = 0; base < nm; base += kFinishChunk) {
        const int n = min(kFinishChunk, nm - base);
        __syncthreads();
        for (int i = t; i < n; i += blockDim.x) {
            const Pt p = gather(j, base + i);
            const bool k = keep[base + i] != 0;
            mine += k ? 1 : 0;
            dv[i][0] = k ? p.ax : 0.0;
            dv[i][1] = k ? p.ay : 0.0;
            dv[i][2] = k ? p.bx : 0.0;
            dv[i][3] = k ? p.by : 0.0;
        }
        __syncthreads();
        if (t < 4) {
            double a = sums[t];
#pragma unroll 8
            for (int i = 0; i < n; ++i) a += dv[i][t];
            sums[t] = a;
        }
    }
    if (mine) atomicAdd(&kept, mine);
    __syncthreads();
    const int count = kept;
    if (count < 4) return false;
    const double cax = sums[0] / count, cay = sums[1] / count, cbx = sums[2] / count, cby = sums[3] / count;
    // pass 2: spreads
    for (int base = 0; base < nm; base += kFinishChunk) {
        const int n = min(kFinishChunk, nm - base);
        __syncthreads();
        for (int i = t; i < n; i += blockDim.x) {
            const Pt p = gather(j, base + i);
            const bool k = keep[base + i] != 0;
            dv[i][0] = k ? (p.ax - cax) * (p.ax - cax) + (p.ay - cay) * (p.ay - cay) : 0.0;
            dv[i][1] = k ? (p.bx - cbx) * (p.bx - cbx) + (p.by - cby) * (p.by - cby) : 0.0;
        }
        __syncthreads();
        if (t == 0 || t == 32) {
            const int col = t ? 1 : 0;
            double a = sums[4 + col];
#pragma unroll 8
            for (int i = 0; i < n; ++i) a += dv[i][col];
            sums[4 + col] = a;
        }
    }
    __syncthreads();
    const double va = sums[4], vb = sums[5];
    if (!(va > 0.0) || !(vb > 0.0) || !fin(va) || !fin(vb)) return false;
    const double sa = sqrt(2.0 * count / va);
    const double sb = sqrt(2.0 * count / vb);
    // pass 3: normal matrix, entry (r, c) on thread 9r + c. Each point's ten
    // design values are computed once (by the point's thread) into dv; a
    // matrix thread reads its four factors by index:
    // dv = {x, y, 1, 0, u, v, -u x, -u y, -v x, -v y},
    // row 0 = dv[{0,1,2,3,3,3,6,7,4}], row 1 = dv[{3,3,3,0,1,2,8,9,5}].
    constexpr unsigned char kRow0[9] = {0, 1, 2, 3, 3, 3, 6, 7, 4};
    constexpr unsigned char kRow1[9] = {3, 3, 3, 0, 1, 2, 8, 9, 5};
    const int r = t / 9, c = t % 9;
    const int i0r = t < 72 ? kRow0[r] : 0, i0c = t < 72 ? kRow0[c] : 0;
    const int i1r = t < 72 ? kRow1[r] : 0, i1c = t < 72 ? kRow1[c] : 0;
    for (int base = 0; base < nm; base += kFinishChunk) {
        const int n = min(kFinishChunk, nm - base);
        __syncthreads();
        for (int i = t; i < n; i += blockDim.x) {
            const Pt p = gather(j, base + i);
            ckeep[i] = keep[base + i];
            const double x = (p.bx - cbx) * sb, y = (p.by - cby) * sb;
            const double u = (p.ax - cax) * sa, v = (p.ay - cay) * sa;
            double* d = dv[i];
            d[0] = x; d[1] = y; d[2] = 1.0; d[3] = 0.0; d[4] = u; d[5] = v;
            d[6] = -u * x; d[7] = -u * y; d[8] = -v * x; d[9] = -v * y;
        }
        __syncthreads();
        if (t < 72) {
            double acc = m[r][c];
#pragma unroll 4
            for (int i = 0; i < n; ++i) {
                const double* d = dv[i];
                const double term = d[i0r] * d[i0c] + d[i1r] * d[i1c];
                acc += ckeep[i] ? term : 0.0;
            }
            m[r][c] = acc;
        }
    }
    __syncthreads();
    if (t < 32) {
        const bool solved = warp_solve(m, cax, cay, cbx, cby, sa, sb, out);
        if (t == 0) ok = solved;
    }
    __syncthreads();
    return ok;
}

// One block per pair: fold the search blocks' winners into the saved raw
// winner, refine, and build the mask and the result.
template <class Src>
__global__ __launch_bounds__(kFinishThreads, 1) void finish_kernel(const __grid_constant__ Src src) {
    __shared__ int red_src[kFinishThreads];
    __shared__ double buf[kFinishChunk];
    __shared__ std::uint8_t ckeep[kFinishChunk];
    __shared__ double dv[kFinishChunk][10];
    __shared__ Model model, cand;
    __shared__ HomographyResult res;
    __shared__ int cand_ok, inl;
    __shared__ double mins[4][kFinishThreads / 32];
    PairIO j;
    int local;
    if (!src.find(blockIdx.x, &j, &local)) return;
    State* s = j.state;
    const int t = threadIdx.x;
    const double nanv = __longlong_as_double(0x7ff8000000000000ll);
    // 1. raw winner: index of the best block result (-1: none)
    int src_i = -1;
    for (int i = t; i < j.search_blocks; i += kFinishThreads)
        if (src_i < 0 ? j.block_best[i].valid != 0 : better(j.block_best[i], j.block_best[src_i])) src_i = i;
    red_src[t] = src_i;
    __syncthreads();
    for (int o = kFinishThreads / 2; o > 0; o >>= 1) {
        if (t < o) {
            const int other = red_src[t + o], mine = red_src[t];
            if (other >= 0 && (mine < 0 || better(j.block_best[other], j.block_best[mine]))) red_src[t] = other;
        }
        __syncthreads();
    }
    const int status0 = s->status;
    if (t == 0) {
        if (status0 == static_cast<int>(Status::OK) && red_src[0] >= 0 &&
            better(j.block_best[red_src[0]], s->best))
            s->best = j.block_best[red_src[0]];
        HomographyResult r{};
        for (int i = 0; i < 9; ++i) r.H[i] = r.H_s[i] = nanv;
        r.reproj_residual = nanv;
        r.num_matches = (s->nm >= 0 && s->nm <= j.m.capacity) ? s->nm : 0;
        r.status = static_cast<Status>(status0);
        if (status0 == static_cast<int>(Status::OK) && !s->best.valid) r.status = Status::DEGENERATE;
        res = r;
        model = s->best;
    }
    for (int i = t; i < j.m.capacity; i += kFinishThreads) j.mask[i] = 0;
    __syncthreads();
    if (res.status == Status::OK) {
        const int nm = s->nm;
        const double thr2 = j.c.threshold * j.c.threshold;
        const int bw = s->scale_b.work_w, bh = s->scale_b.work_h;
        {
            double h[9];
            for (int e = 0; e < 9; ++e) h[e] = model.h[e];
            const double loss = ordered_sum(nm, buf, [&](int i) {
                const double r = residual2(h, gather(j, i));
                return r < thr2 ? r : thr2;
            });
            if (t == 0) model.loss = loss;
        }
        __syncthreads();
        for (int step = 0; step < j.c.refinement_steps; ++step) {
            double h[9];
            for (int e = 0; e < 9; ++e) h[e] = model.h[e];
            // inliers of the current model, kept in the mask buffer
            for (int i = t; i < nm; i += kFinishThreads) j.mask[i] = residual2(h, gather(j, i)) <= thr2;
            __syncthreads();
            double ch[9];
            const bool fitted = block_fit(j, nm, j.mask, ch, dv, ckeep);
            if (t == 0) {
                cand_ok = fitted && valid_domain(ch, bw, bh);
                for (int e = 0; e < 9; ++e) cand.h[e] = ch[e];
            }
            __syncthreads();
            if (!cand_ok) break;
            double hc[9];
            for (int e = 0; e < 9; ++e) hc[e] = cand.h[e];
            const double closs = ordered_sum(nm, buf, [&](int i) {
                const double r = residual2(hc, gather(j, i));
                return r < thr2 ? r : thr2;
            });
            const bool take = fin(closs) && closs < model.loss;
            __syncthreads();
            if (!take) break;
            if (t == 0) {
                for (int e = 0; e < 9; ++e) model.h[e] = cand.h[e];
                model.loss = closs;
            }
            __syncthreads();
        }
        // mask, inlier count, residual sum (index order), inlier extent
        double h[9];
        for (int e = 0; e < 9; ++e) h[e] = model.h[e];
        if (t == 0) inl = 0;
        __syncthreads();
        double mnx = DBL_MAX, mny = DBL_MAX, mxx = -DBL_MAX, mxy = -DBL_MAX;
        int cnt = 0;
        for (int i = t; i < j.m.capacity; i += kFinishThreads) {
            std::uint8_t in = 0;
            if (i < nm) {
                const Pt q = gather(j, i);
                if (residual2(h, q) <= thr2) {
                    in = 1;
                    ++cnt;
                    mnx = fmin(mnx, q.ax); mxx = fmax(mxx, q.ax);
                    mny = fmin(mny, q.ay); mxy = fmax(mxy, q.ay);
                }
            }
            j.mask[i] = in;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        if ((t & 31) == 0) {
            atomicAdd(&inl, cnt);
            mins[0][t >> 5] = mnx; mins[1][t >> 5] = mny; mins[2][t >> 5] = mxx; mins[3][t >> 5] = mxy;
        }
        const double sum = ordered_sum(nm, buf, [&](int i) {
            const double r = residual2(h, gather(j, i));
            return r <= thr2 ? r : 0.0;
        });
        if (t == 0) {
            double a = DBL_MAX, bb = DBL_MAX, c = -DBL_MAX, d = -DBL_MAX;
            for (int w = 0; w < kFinishThreads / 32; ++w) {
                a = fmin(a, mins[0][w]); bb = fmin(bb, mins[1][w]);
                c = fmax(c, mins[2][w]); d = fmax(d, mins[3][w]);
            }
            HomographyResult r = res;
            r.num_inliers = inl;
            if (r.num_inliers < 4) {
                r.status = Status::DEGENERATE;
                r.num_inliers = 0;
                cand_ok = 0;  // clear the mask below
            } else {
                r.inlier_ratio = static_cast<double>(r.num_inliers) / nm;
                r.reproj_residual = sqrt(sum / r.num_inliers);
                const double w = fmax(1.0, static_cast<double>(s->scale_a.work_w - 1));
                const double hh = fmax(1.0, static_cast<double>(s->scale_a.work_h - 1));
                r.inlier_coverage = fmin(1.0, (c - a) / w) * fmin(1.0, (d - bb) / hh);
                for (int e = 0; e < 9; ++e) r.H_s[e] = h[e];
                double tmp[9];
                mat3_mul(j.inverse_a, h, tmp);
                mat3_mul(tmp, j.d_b, r.H);
                cand_ok = 1;
                if (!h_normalize(r.H) || !valid_domain(r.H, s->scale_b.orig_w, s->scale_b.orig_h)) {
                    r.status = Status::DEGENERATE;
                    r.num_inliers = 0;
                    r.inlier_ratio = r.inlier_coverage = 0.0;
                    r.reproj_residual = nanv;
                    for (int e = 0; e < 9; ++e) r.H[e] = r.H_s[e] = nanv;
                    cand_ok = 0;
                }
            }
            res = r;
        }
        __syncthreads();
        if (!cand_ok)
            for (int i = t; i < j.m.capacity; i += kFinishThreads) j.mask[i] = 0;
    }
    if (t == 0) {
        s->evaluated = j.c.hypotheses;
        s->result = res;
        if (j.result_out) *j.result_out = res;
    }
}

}  // namespace stitch::b200::s5k
