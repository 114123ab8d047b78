// S2 (FAST-9 + NMS + 2K pre-selection + Harris + top-K) and S3 (7x7 blur +
// IC angle + rBRIEF-256) kernels for sm_100a.
//
// Every kernel reads its image and buffers from a "job". A job source is
// either one job passed by value (the per-image stage call) or a device table
// of jobs plus a block-prefix array (the batched chain, where one launch
// covers every image of every pair). Results are identical either way.
//
// Reference semantics (file:line in the reference tree):
//   FAST score        src/s2_s3/s2.cu:37-67   (cornerScore<16>, circle order)
//   NMS + histogram   src/s2_s3/s2.cu:81-106
//   2K threshold      src/s2_s3/s2.cu:108-139 (SelectParams)
//   raster compaction src/s2_s3/s2.cu:141-235 (all above, then first ties)
//   Harris            src/s2_s3/s2.cu:247-285 (no-FMA float formula, key)
//   top-K order       src/s2_s3/s2.cu:287-310 (descending key)
//   blur              src/s2_s3/s3.cu:41-73
//   describe          src/s2_s3/s3.cu:75-157
#pragma once

#include "common.cuh"

namespace stitch::b200::s2s3 {

// ---------------------------------------------------------------- jobs

struct SelectParams {
    std::uint32_t threshold;  // FAST score at the 2K boundary
    std::uint32_t above;      // maxima with score > threshold
    std::uint32_t ties;       // maxima at the threshold that are kept
    std::uint32_t selected;   // above + ties
};

// Per-job counters of the detect kernels, after the 256 histogram bins.
enum DetectCounter { kListed = 0, kAboveWritten = 1, kTiesWritten = 2, kTileQueue = 3, kDetectCounters = 4 };
constexpr int kHistWords = 256 + kDetectCounters;  // one job's histogram and counters

struct alignas(16) DetectJob {  // 16-byte multiple: copied into shared memory in 16-byte chunks
    const std::uint8_t* image;
    int width, height, pitch;
    int threshold, max_keypoints;
    float harris_k;
    // workspace
    std::uint64_t* maxima;         // NMS maxima listed by the FAST kernel: (score << 32) | raster index
    int max_maxima;                // capacity of `maxima`
    std::uint32_t* hist;           // [256] scores of the listed maxima, then DetectCounter words;
                                   // all zeroed before the FAST launch
    SelectParams* params;
    std::uint64_t* keys;           // [candidates]
    // output
    float* x;
    float* y;
    float* response;  // may be null
    int* count;
    // On-demand S3 blur (pyramid and batched paths; null elsewhere): the
    // blur tiles that final keypoints sample are flagged in blur_marks
    // (one word per tile, zeroed every run) and listed once each in
    // blur_list as (describe job, tile) behind the launch-wide *blur_count.
    std::uint32_t* blur_marks;
    uint2* blur_list;
    std::uint32_t* blur_count;
    int job;  // this job's index in the describe table of the launch
    // launch bookkeeping
    int tiles_x, tiles, select_blocks, candidates;
    std::uint32_t tiles_x_magic;  // ceil(2^32 / tiles_x), 0 for one tile column (see fast_origin)
    __host__ __device__ std::uint32_t* counters() const { return hist + 256; }
};

struct DescribeJob {
    const std::uint8_t* image;
    int width, height, pitch;
    std::uint8_t* blurred;  // rows of blur_pitch bytes
    int blur_pitch;
    const float* x;
    const float* y;
    const int* count;
    int capacity;
    std::uint8_t* out;  // rows of row_stride bytes
    int row_stride;
    int tiles_x, tiles;  // blur tiles
    // Pyramid layer (level_counts != null): the layer's keypoints are in
    // layer coordinates in x/y/response; the describe kernel writes them,
    // multiplied by `scale`, and their descriptors to the image's
    // concatenated outputs after the keypoints of lower layers
    // (level_counts[0..level-1]) and adds the layer's count to *out_count.
    const float* response;
    float* out_x;
    float* out_y;
    float* out_response;  // may be null
    int* out_count;
    const int* level_counts;
    int level;
    float scale;
};

// One pyramid layer: `dst` (dense) resized from `src` by fixed-point
// bilinear interpolation (cv::resize INTER_LINEAR_EXACT on 8-bit images).
struct ResizeJob {
    const std::uint8_t* src;
    int src_width, src_height, src_pitch;
    std::uint8_t* dst;
    int width, height, pitch;
    int tiles_x, tiles;
    double scale_x, scale_y;  // linear_exact_scale of each axis, computed by the host
};

// Per-image job passed by value.
template <class Job> struct OneJob {
    Job job;
    __device__ bool find(int block, int /*kind*/, Job* j, int* local) const {
        *j = job;
        *local = block;
        return true;
    }
    __device__ Job at(int /*index*/) const { return job; }
};

// Device table: prefix[kind * (n + 1) + i] is the first block of job i for
// launch kind `kind`; blocks past the end are idle. With map[kind] set, entry
// b of it is (job << 16 | block within the job) for block b of that kind, so
// a block finds its job in one load instead of a binary search over the
// prefix (each step of which waits on the previous one).
constexpr int kMapKinds = 16;
template <class Job> struct JobTable {
    const Job* jobs;
    const int* prefix;
    int n;
    const std::uint32_t* map[kMapKinds] = {};
    int map_blocks[kMapKinds] = {};
    __device__ bool find(int block, int kind, Job* j, int* local) const {
        if (const std::uint32_t* m = map[kind]) {
            if (block >= map_blocks[kind]) return false;
            const std::uint32_t e = __ldg(m + block);
            *j = jobs[e >> 16];
            *local = static_cast<int>(e & 0xffffu);
            return true;
        }
        const int* p = prefix + kind * (n + 1);
        if (block >= p[n]) return false;
        int lo = 0, hi = n - 1;
        while (lo < hi) {  // largest i with p[i] <= block
            const int mid = (lo + hi + 1) >> 1;
            if (p[mid] <= block) lo = mid; else hi = mid - 1;
        }
        *j = jobs[lo];
        *local = block - p[lo];
        return true;
    }
    __device__ Job at(int index) const { return jobs[index]; }
};

// A few jobs passed by value (the layers of one image's pyramid):
// first[kind][i] is the first block of job i; linear search.
template <class Job, int kJobs, int kKinds> struct InlineTable {
    Job jobs[kJobs];
    int first[kKinds][kJobs + 1];
    int n;
    __device__ bool find(int block, int kind, Job* j, int* local) const {
        if (block >= first[kind][n]) return false;
        int i = 0;
        while (i + 1 < n && first[kind][i + 1] <= block) ++i;
        *j = jobs[i];
        *local = block - first[kind][i];
        return true;
    }
    __device__ Job at(int index) const { return jobs[index]; }
};

// Launch kinds of the detect table: kFastKind entries are the FAST tiles of
// each job (looked up by tile index from the persistent FAST kernel's
// queue), kSelectKind blocks walk a job's maxima list, kSortKind is one
// block per job (tie selection, then the top-K sort).
enum DetectKind { kFastKind = 0, kSelectKind = 1, kHarrisKind = 2, kSortKind = 3, kDetectKinds = 4 };
enum DescribeKind { kBlurKind = 0, kDescKind = 1, kDescribeKinds = 2 };

constexpr int kFastTileW = 64, kFastTileH = 64;

// Origin (x0, y0) of FAST tile `local` of a job: local / tiles_x by a
// multiply-high with ceil(2^32 / tiles_x), which is the quotient or one
// above it (the error term local * (magic - 2^32 / tiles_x) / 2^32 is below
// 1), then corrected.
__device__ __forceinline__ int2 fast_origin(const DetectJob& j, int local) {
    int ty = j.tiles_x_magic ? static_cast<int>(__umulhi(static_cast<std::uint32_t>(local), j.tiles_x_magic)) : local;
    if (ty * j.tiles_x > local) --ty;
    return make_int2((local - ty * j.tiles_x) * kFastTileW, ty * kFastTileH);
}
constexpr int kFastInW = kFastTileW + 8, kFastInH = kFastTileH + 8;  // halo 4 = FAST 3 + NMS 1
constexpr int kFastScW = kFastTileW + 2, kFastScH = kFastTileH + 2;
constexpr int kSelectPx = 65536;   // image pixels per select block (a job's maxima list is walked
                                   // by ceil(W * H / kSelectPx) blocks)
constexpr int kFastThreads = 256;
constexpr int kFastCtasPerSm = 7;  // resident FAST blocks per SM (shared memory); the persistent grid is 148 x this
constexpr int kTieThreads = 1024;
// Largest offset of a rotated rBRIEF sample from its keypoint: the pattern's
// coordinates lie within a radius of 18.39 px (|x|, |y| <= 13), so a rotated
// coordinate rounds to at most 18.
constexpr int kSampleRadius = 18;
constexpr int kHarrisThreads = 256;
constexpr int kSortCap = 16384;    // candidates sorted in shared memory by one block
constexpr int kSortThreads = 1024;
constexpr int kSortChunk = 64;      // keys a warp sorts in registers (2 per lane)
constexpr int kBlurTileW = 64, kBlurTileH = 64;
constexpr int kDescWarps = 8;
constexpr int kDescRounds = 4;                        // keypoints per warp of a describe block
constexpr int kDescKeys = kDescWarps * kDescRounds;  // keypoints per describe block
constexpr int kEdge = 31;
constexpr int kResizeTileW = 128, kResizeTileH = 64;  // tallest tile; a job's tile_h may be smaller
constexpr int kMaxLevels = 16;
static_assert(kMaxLevels <= kMapKinds && kDetectKinds <= kMapKinds, "block map kinds");

// ------------------------------------------------------------- FAST + NMS

// float32 taps of a 7-tap, sigma-2 Gaussian (exp in float64, normalised,
// rounded to float32); equal to cv::getGaussianKernel(7, 2, CV_32F).
__device__ __forceinline__ float blur_tap(int i) {
    switch (i) {
        case 0: case 6: return 0x1.1f5f62p-4f;
        case 1: case 5: return 0x1.0c70fcp-3f;
        case 2: case 4: return 0x1.869472p-3f;
        default: return 0x1.ba95c0p-3f;
    }
}

// Border reflection without repeating the edge pixel (BORDER_REFLECT_101).
__device__ __forceinline__ int reflect101(int i, int n) {
    if (n == 1) return 0;
    while (i < 0 || i >= n) i = i < 0 ? -i : 2 * n - 2 - i;
    return i;
}

// FAST-9 score of the pixel at p (row stride `stride`), 0 when it is not a
// corner. With d_k = centre - ring_k over the 16-pixel circle, a 9-pixel arc
// scores min(d) when darker and min(-d) when brighter; the raw score is the
// largest over the 16 arcs of both kinds, the pixel is a corner iff the raw
// score exceeds the threshold, and it then scores raw - 1. Both kinds run
// at once as unsigned 16-bit lanes q_k = (d_k + 256) | (256 - d_k) << 16
// (all in [1, 511]), which is c + r_k * 0xffff for c = (v + 256) |
// (256 - v) << 16: one multiply-add per ring pixel, no borrow between the
// lanes. 9-wide arc minima come from 3-wide ones through the 3-input 16x2
// minimum (min3(m3[k], m3[k+3], m3[k+6])), and the 16 arcs are folded with
// the 3-input maximum. (CUDA 12.9 ptxas at -O1 and above miscompiles the
// signed max(min(arc), -max(arc)) form of this score on sm_100; this
// unsigned form is exact at every optimisation level.)
__device__ __forceinline__ int fast_score(const std::uint8_t* p, int stride, int thr) {
    const unsigned v = p[0];
    const unsigned c = (v + 256u) | ((256u - v) << 16);
    const unsigned r[16] = {p[3 * stride],      p[3 * stride + 1],  p[2 * stride + 2],  p[stride + 3],
                            p[3],               p[-stride + 3],     p[-2 * stride + 2], p[-3 * stride + 1],
                            p[-3 * stride],     p[-3 * stride - 1], p[-2 * stride - 2], p[-stride - 3],
                            p[-3],              p[stride - 3],      p[2 * stride - 2],  p[3 * stride - 1]};
    unsigned q[16], m3[16], m9[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) q[k] = c + r[k] * 0xffffu;
#pragma unroll
    for (int k = 0; k < 16; ++k) m3[k] = __vimin3_u16x2(q[k], q[(k + 1) & 15], q[(k + 2) & 15]);
#pragma unroll
    for (int k = 0; k < 16; ++k) m9[k] = __vimin3_u16x2(m3[k], m3[(k + 3) & 15], m3[(k + 6) & 15]);
    const unsigned b0 = __vimax3_u16x2(m9[0], m9[1], m9[2]), b1 = __vimax3_u16x2(m9[3], m9[4], m9[5]);
    const unsigned b2 = __vimax3_u16x2(m9[6], m9[7], m9[8]), b3 = __vimax3_u16x2(m9[9], m9[10], m9[11]);
    const unsigned b4 = __vimax3_u16x2(m9[12], m9[13], m9[14]);
    const unsigned best = __vmaxu2(__vimax3_u16x2(b0, b1, b2), __vimax3_u16x2(b3, b4, m9[15]));
    const unsigned lo = best & 0xffffu, hi = best >> 16;
    const int score = static_cast<int>(lo > hi ? lo : hi) - 256;
    return score > thr ? score - 1 : 0;
}

// Compass test of two pixels in 16-bit lanes (values 0..255), a necessary
// condition for a FAST-9 corner: every 9-pixel arc of the circle holds one of
// the compass pixels s0, s8 (3 below, 3 above) and one of s4, s12 (3 right,
// 3 left), so an arc brighter than v + t needs
// min(max(s0, s8), max(s4, s12)) >= v + t + 1 and one darker than v - t needs
// max(min(s0, s8), min(s4, s12)) <= v - t - 1. x >= y per lane is the top bit
// of (x | 0x8000) - y, with no borrow between lanes for x, y < 0x8000.
// thr1 = (t + 1) in both lanes. Returns 0x8000 per passing lane.
__device__ __forceinline__ std::uint32_t compass_pass2(std::uint32_t v, std::uint32_t s0, std::uint32_t s4,
                                                       std::uint32_t s8, std::uint32_t s12, std::uint32_t thr1) {
    const std::uint32_t hi = __vminu2(__vmaxu2(s0, s8), __vmaxu2(s4, s12));
    const std::uint32_t lo = __vmaxu2(__vminu2(s0, s8), __vminu2(s4, s12));
    constexpr std::uint32_t kTop = 0x80008000u;
    const std::uint32_t bright = ((hi | kTop) - (v + thr1)) & kTop;  // min(...) >= v + t + 1
    const std::uint32_t dark = ((v | kTop) - (lo + thr1)) & kTop;    // v >= max(...) + t + 1
    return bright | dark;
}

// Shared-memory tile of the FAST kernel: rows of kInStride bytes holding
// image columns x0-16 .. x0+79; the halo-4 column c (image x0-4+c) is at byte
// c + kInOff. Scores: rows of kScStride bytes, position (r, c) = image
// (y0-1+r, x0-1+c).
constexpr int kInStride = 96, kInOff = 12;
constexpr int kScStride = 68;
constexpr int kScGroups = kScStride / 4;  // groups of 4 positions per score row

// Bytes k of wa and wb as a float pair (rows r, r + 1 of one column), each
// exact: the float 2^23 + b (byte b placed in the low mantissa) minus 2^23.
__device__ __forceinline__ float2 byte_pair(std::uint32_t wa, std::uint32_t wb, int k) {
    const float2 biased = make_float2(__uint_as_float(__byte_perm(wa, 0x4B000000u, 0x7440u + k)),
                                      __uint_as_float(__byte_perm(wb, 0x4B000000u, 0x7440u + k)));
    return __fadd2_rn(biased, make_float2(-8388608.0f, -8388608.0f));
}

// A blur tap in both lanes of a packed pair. The sm_100 packed FP32 add and
// multiply round each lane exactly as __fadd_rn / __fmul_rn do, so two rows
// (or two columns) of the blur run in one instruction stream.
__device__ __forceinline__ float2 tap_pair(int t) { return make_float2(blur_tap(t), blur_tap(t)); }

// Rounds a blur sum half-to-even after clamping to [0, 255] (clamping the
// float first gives the same byte for every finite sum).
__device__ __forceinline__ std::uint32_t blur_byte(float acc) {
    return static_cast<std::uint32_t>(__float2int_rn(fminf(fmaxf(acc, 0.0f), 255.0f)));
}

// Asynchronous 16-byte copy, global to shared memory (both 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(gmem) : "memory");
}

// The FAST kernel's block map and job array where its source has them
// (tables staged by a plan); elsewhere the job is looked up in place.
template <class S> __device__ __forceinline__ const std::uint32_t* fast_map(const S&) { return nullptr; }
template <class S> __device__ __forceinline__ const DetectJob* fast_jobs(const S&) { return nullptr; }
template <> __device__ __forceinline__ const std::uint32_t* fast_map(const JobTable<DetectJob>& s) {
    return s.map[kFastKind];
}
template <class S> __device__ __forceinline__ int fast_map_tiles(const S&) { return 0; }
template <> __device__ __forceinline__ int fast_map_tiles(const JobTable<DetectJob>& s) { return s.map_blocks[kFastKind]; }
template <> __device__ __forceinline__ const DetectJob* fast_jobs(const JobTable<DetectJob>& s) { return s.jobs; }

// Stages rows y0-4 .. y0+67 and columns x0-16 .. x0+79 of the job's image in
// `in` (byte c of row r = image (y0-4+r, x0-16+c)). The FAST test never reads
// a position outside the image, so rows are clamped into it and the bytes of
// columns outside it are left as they are. With a 16-byte aligned image (base
// and pitch) every 16-byte chunk within a row's pitch (within the width on
// the last row) is one asynchronous copy, and a chunk that straddles the end
// of the last row is copied byte by byte; other images are loaded byte by
// byte with clamped columns. Asynchronous copies complete at the caller's
// cp_async_wait_all.
__device__ __forceinline__ void stage_fast_tile(const DetectJob& j, int local, std::uint8_t (*in)[kInStride]) {
    const int tid = threadIdx.x;
    const int W = j.width, H = j.height;
    const int2 org = fast_origin(j, local);
    const int y0 = org.y, x0 = org.x;
    const bool vec = ((reinterpret_cast<std::uintptr_t>(j.image) | static_cast<std::uintptr_t>(j.pitch)) & 15) == 0;
    if (vec) {
        constexpr int kChunks = kInStride / 16;  // 6 per row
        for (int i = tid; i < kFastInH * kChunks; i += kFastThreads) {
            const int r = i / kChunks, q = i - r * kChunks;
            const int gy = min(max(y0 - 4 + r, 0), H - 1);
            const int cx = x0 - 16 + 16 * q;
            const int limit = gy == H - 1 ? W : j.pitch;  // bytes of the row that may be read
            const std::uint8_t* row = j.image + static_cast<std::size_t>(gy) * j.pitch;
            if (cx >= 0 && cx + 16 <= limit) {
                cp_async16(&in[r][16 * q], row + cx);
            } else if (cx >= 0 && cx < W) {
                for (int b = 0; b < 16 && cx + b < W; ++b) in[r][16 * q + b] = row[cx + b];
            }
        }
    } else {
        for (int i = tid; i < kFastInH * kInStride; i += kFastThreads) {
            const int r = i / kInStride, c = i - r * kInStride;
            const int gy = min(max(y0 - 4 + r, 0), H - 1), gx = min(max(x0 - 16 + c, 0), W - 1);
            in[r][c] = j.image[static_cast<std::size_t>(gy) * j.pitch + gx];
        }
    }
}

// FAST-9 + strict 3x3 NMS, persistent: each block takes 64x64 tiles of
// every job of the launch from a device queue (`*queue`, zero at launch; tile
// t of `total` is looked up through the source's kFastKind entries), while
// the next tile's bytes are copied into the other half of a double buffer.
// The jobs of the current and the next tile sit in shared memory. Per tile:
//   1. the compass test on the tile plus a 1-pixel ring, 4 positions per
//      thread in 16-bit lanes; groups with a survivor are listed;
//   2. the groups are expanded into one list of survivor positions, scored
//      on full warps (every other position scores 0);
//   3. each survivor of the tile inside the 31-pixel edge margin that is a
//      strict 3x3 maximum goes into the job's maxima list as
//      (score << 32) | raster index (one atomic per warp), its score into the
//      tile's histogram, which is added to the job's at the end of the tile.
// No maxima map and no blur are written.
template <class Src>
__global__ __launch_bounds__(kFastThreads, kFastCtasPerSm) void fast_kernel(const __grid_constant__ Src src,
                                                                          std::uint32_t* queue, int total) {
    static_assert(sizeof(DetectJob) % 16 == 0, "jobs are copied in 16-byte chunks");
    __shared__ __align__(16) std::uint8_t in[2][kFastInH][kInStride];
    __shared__ __align__(16) std::uint8_t sc[kFastScH][kScStride];
    __shared__ std::uint16_t cand[kFastScH * kScGroups];
    __shared__ std::uint16_t pos[kFastScH * kFastScW];  // survivor positions r * kScStride + c
    __shared__ std::uint32_t hist[256];
    __shared__ DetectJob jobs[2];  // jobs of the tiles in in[0] and in[1] (kept here, not in registers)
    __shared__ int locals[2];
    __shared__ int n_cand, n_pos, next;
    __shared__ int ahead_tile;          // with a block map: the tile after `next`, taken from the queue
    __shared__ std::uint32_t ahead_entry;  // and its block-map entry (job << 16 | tile within the job)
    const int tid = threadIdx.x, lane = tid & 31;
    // With a block map, total is capped by the map; the job of the tile after
    // the current one is copied into shared memory asynchronously while the
    // current tile is tested, and the queue index and map entry of the tile
    // after that are fetched a tile ahead, so no thread waits on the lookup.
    const std::uint32_t* map = fast_map(src);
    if (map) total = min(total, fast_map_tiles(src));
    hist[tid] = 0;
    if (tid == 0) {
        n_cand = 0;
        n_pos = 0;
        next = static_cast<int>(atomicAdd(queue, 1u));
        if (next < total && !src.find(next, kFastKind, &jobs[0], &locals[0])) next = total;
        if (map) {
            const int t = static_cast<int>(atomicAdd(queue, 1u));
            ahead_tile = t;
            if (t < total) cp_async4(&ahead_entry, map + t);
        }
    }
    __syncthreads();
    int tile = next, buf = 0;
    if (tile < total) stage_fast_tile(jobs[0], locals[0], in[0]);
    cp_async_wait_all();
    __syncthreads();
    while (tile < total) {
        const DetectJob& j = jobs[buf];
        const int local = locals[buf];
        const int W = j.width, H = j.height;
        const int2 org = fast_origin(j, local);
        const int y0 = org.y, x0 = org.x;
        std::uint8_t (*cur)[kInStride] = in[buf];
        int ahead = total;  // thread 0 with a block map: the queue index of the tile after next
        if (tid == 0) {
            if (map) {
                const int t = ahead_tile;
                next = t;
                if (t < total) {
                    const std::uint32_t e = ahead_entry;
                    locals[buf ^ 1] = static_cast<int>(e & 0xffffu);
                    const auto* g = reinterpret_cast<const char*>(fast_jobs(src) + (e >> 16));
                    auto* d = reinterpret_cast<char*>(&jobs[buf ^ 1]);
#pragma unroll
                    for (int k = 0; k < static_cast<int>(sizeof(DetectJob) / 16); ++k) cp_async16(d + 16 * k, g + 16 * k);
                    ahead = static_cast<int>(atomicAdd(queue, 1u));
                }
            } else {
                int t = static_cast<int>(atomicAdd(queue, 1u));
                if (t < total && !src.find(t, kFastKind, &jobs[buf ^ 1], &locals[buf ^ 1])) t = total;
                next = t;
            }
        }
        // 1. compass test: thread (q, rb) takes positions 4q .. 4q+3 of rows rb,
        // rb + 15, rb + 30, ...; groups with a survivor are listed as
        // (group << 4 | survivor bits)
        const std::uint32_t thr1 = static_cast<std::uint32_t>(j.threshold + 1) * 0x00010001u;
        {
            constexpr int kRowSets = 256 / kScGroups;  // 15
            const int q = tid % kScGroups, rb = tid / kScGroups, c = 4 * q;
            unsigned colmask = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gx = x0 - 1 + c + k;
                if (c + k < kFastScW && gx >= 3 && gx < W - 3) colmask |= 1u << k;
            }
            for (int it = 0; it < (kFastScH + kRowSets - 1) / kRowSets; ++it) {  // same trip count everywhere
                const int r = rb + it * kRowSets;
                unsigned bits = 0;
                if (rb < kRowSets && r < kFastScH) {
                    *reinterpret_cast<std::uint32_t*>(&sc[r][c]) = 0u;
                    const int gy = y0 - 1 + r;
                    if (colmask && gy >= 3 && gy < H - 3) {
                        const int w = q + 3;  // word holding halo columns c .. c+3 (bytes c+12 .. c+15)
                        const auto* mid = reinterpret_cast<const std::uint32_t*>(&cur[r + 3][0]);
                        const auto* bot = reinterpret_cast<const std::uint32_t*>(&cur[r + 6][0]);
                        const auto* top = reinterpret_cast<const std::uint32_t*>(&cur[r][0]);
                        const std::uint32_t a0 = mid[w], a1 = mid[w + 1], a2 = mid[w + 2];
                        const std::uint32_t v = __funnelshift_r(a0, a1, 24);   // centres, halo columns c+3 .. c+6
                        const std::uint32_t s12 = a0;                          // 3 left
                        const std::uint32_t s4 = __funnelshift_r(a1, a2, 16);  // 3 right
                        const std::uint32_t s0 = __funnelshift_r(bot[w], bot[w + 1], 24);  // 3 down
                        const std::uint32_t s8 = __funnelshift_r(top[w], top[w + 1], 24);  // 3 up
                        const std::uint32_t plo =
                            compass_pass2(__byte_perm(v, 0, 0x4140), __byte_perm(s0, 0, 0x4140),
                                          __byte_perm(s4, 0, 0x4140), __byte_perm(s8, 0, 0x4140),
                                          __byte_perm(s12, 0, 0x4140), thr1);
                        const std::uint32_t phi =
                            compass_pass2(__byte_perm(v, 0, 0x4342), __byte_perm(s0, 0, 0x4342),
                                          __byte_perm(s4, 0, 0x4342), __byte_perm(s8, 0, 0x4342),
                                          __byte_perm(s12, 0, 0x4342), thr1);
                        bits = (((plo >> 15) & 1u) | ((plo >> 30) & 2u) | ((phi >> 13) & 4u) | ((phi >> 28) & 8u)) &
                               colmask;
                    }
                }
                const unsigned m = __ballot_sync(0xffffffffu, bits != 0);
                int base = 0;
                if (lane == 0 && m) base = atomicAdd(&n_cand, __popc(m));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (bits)
                    cand[base + __popc(m & ((1u << lane) - 1u))] =
                        static_cast<std::uint16_t>(((r * kScGroups + q) << 4) | bits);
            }
        }
        if (tid == 0 && map) cp_async_wait_all();  // the next tile's job
        __syncthreads();
        // the next tile's bytes travel while this one is scored
        const int nt = next;
        if (tid == 0 && map) {
            ahead_tile = ahead;
            if (ahead < total) cp_async4(&ahead_entry, map + ahead);
        }
        if (nt < total) stage_fast_tile(jobs[buf ^ 1], locals[buf ^ 1], in[buf ^ 1]);
        const int nc = n_cand;
        // 2. the survivor groups expanded into one position list (each warp
        // reserves its share with one shared atomic), then scored on full warps
        for (int base = 0; base < nc; base += kFastThreads) {  // block-uniform trip count
            const int i = base + tid;
            unsigned bits = 0;
            int pos0 = 0;
            if (i < nc) {
                const int e = cand[i];
                const int grp = e >> 4, r = grp / kScGroups, c0 = 4 * (grp - r * kScGroups);
                bits = e & 0xfu;
                pos0 = r * kScStride + c0;
            }
            const int cnt = __popc(bits);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            int first = 0;
            if (lane == 31 && incl) first = atomicAdd(&n_pos, incl);
            first = __shfl_sync(0xffffffffu, first, 31);
            int o = first + incl - cnt;
            for (unsigned b = bits; b; b &= b - 1) pos[o++] = static_cast<std::uint16_t>(pos0 + __ffs(b) - 1);
        }
        __syncthreads();
        const int np = n_pos;
        for (int k = tid; k < np; k += kFastThreads) {
            const int e = pos[k];
            const int r = e / kScStride, c = e - r * kScStride;
            sc[r][c] = static_cast<std::uint8_t>(fast_score(&cur[r + 3][c + 3 + kInOff], kInStride, j.threshold));
        }
        __syncthreads();
        // 3. strict 3x3 maxima inside the 31-pixel edge margin: only listed
        // survivors can score above 0, so only they are tested (the ring
        // rows and columns hold neighbours only). Each warp appends its maxima
        // to the job's list with one atomic, and their scores to the tile's
        // histogram.
        for (int k0 = 0; k0 < np; k0 += kFastThreads) {  // block-uniform trip count
            const int k = k0 + tid;
            unsigned v = 0;
            std::uint32_t px = 0;
            if (k < np) {
                const int e = pos[k];
                const int r = e / kScStride, c = e - r * kScStride;
                const int gy = y0 - 1 + r, gx = x0 - 1 + c;
                if (r >= 1 && r <= kFastTileH && c >= 1 && c <= kFastTileW && gy >= kEdge && gy < H - kEdge &&
                    gx >= kEdge && gx < W - kEdge) {
                    const unsigned s0 = sc[r][c];
                    if (s0 && s0 > sc[r - 1][c - 1] && s0 > sc[r - 1][c] && s0 > sc[r - 1][c + 1] &&
                        s0 > sc[r][c - 1] && s0 > sc[r][c + 1] && s0 > sc[r + 1][c - 1] && s0 > sc[r + 1][c] &&
                        s0 > sc[r + 1][c + 1]) {
                        v = s0;
                        px = static_cast<std::uint32_t>(gy) * static_cast<std::uint32_t>(W) + static_cast<std::uint32_t>(gx);
                    }
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, v != 0);
            if (m) {
                const int leader = __ffs(m) - 1;
                std::uint32_t first = 0;
                if (lane == leader) first = atomicAdd(&j.counters()[kListed], static_cast<std::uint32_t>(__popc(m)));
                first = __shfl_sync(0xffffffffu, first, leader);
                if (v) {
                    const std::uint32_t slot = first + static_cast<std::uint32_t>(__popc(m & ((1u << lane) - 1u)));
                    if (slot < static_cast<std::uint32_t>(j.max_maxima))
                        j.maxima[slot] = (static_cast<std::uint64_t>(v) << 32) | px;
                    atomicAdd(&hist[v], 1u);
                }
            }
        }
        __syncthreads();
        // the tile's histogram into the job's
        if (hist[tid]) {
            atomicAdd(&j.hist[tid], hist[tid]);
            hist[tid] = 0;
        }
        if (tid == 0) {
            n_cand = 0;
            n_pos = 0;
        }
        cp_async_wait_all();
        __syncthreads();
        tile = nt;
        buf ^= 1;
    }
}

// --------------------------------------------------------- 2K selection

// All 256 threads: suffix[s] = number of maxima with score >= s (s >= 1),
// then the unique threshold s with suffix[s] >= cap > suffix[s + 1]; with at
// most cap maxima, everything is kept (threshold 1).
__device__ __forceinline__ SelectParams select_params(const std::uint32_t* hist, std::uint32_t cap,
                                                     std::uint32_t* suffix /*[257] shared*/,
                                                     SelectParams* out /*shared*/) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    __shared__ std::uint32_t warp_total[8];
    const std::uint32_t own = t ? hist[t] : 0u;
    std::uint32_t v = own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const std::uint32_t n = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o < 32) v += n;
    }
    if (lane == 0) warp_total[warp] = v;
    __syncthreads();
    for (int w = warp + 1; w < 8; ++w) v += warp_total[w];
    suffix[t] = v;
    if (t == 0) suffix[256] = 0;
    __syncthreads();
    const std::uint32_t total = suffix[1];
    if (total <= cap) {
        if (t == 1) *out = SelectParams{1u, total - own, own, total};
    } else if (t >= 1 && suffix[t] >= cap && suffix[t + 1] < cap) {
        *out = SelectParams{static_cast<std::uint32_t>(t), suffix[t + 1], cap - suffix[t + 1], cap};
    }
    __syncthreads();
    return *out;
}

// Pre-selection over a job's maxima list: every block of the job derives the
// same threshold from the histogram; block 0 publishes the parameters and
// the keypoint count min(selected, K). The maxima above the threshold go to
// keys[0, above), and when every maximum at the threshold is kept (selected
// below the cap, or the cap falls exactly on a score boundary) those go to
// keys[above, selected); otherwise the tie kernel picks them. The order
// inside each range is not the raster order: the keys are sorted later by
// (response, raster index), which no order of equal sets changes.
template <class Src>
__global__ __launch_bounds__(256) void select_kernel(const __grid_constant__ Src src) {
    __shared__ std::uint32_t suffix[257];
    __shared__ SelectParams sp;
    DetectJob j;
    int local;
    if (!src.find(blockIdx.x, kSelectKind, &j, &local)) return;
    const SelectParams p = select_params(j.hist, static_cast<std::uint32_t>(j.candidates), suffix, &sp);
    if (local == 0 && threadIdx.x == 0) {
        *j.params = p;
        *j.count = static_cast<int>(min(p.selected, static_cast<std::uint32_t>(j.max_keypoints)));
    }
    const bool all_ties = p.ties == j.hist[p.threshold];
    std::uint32_t* ctr = j.counters();
    const std::uint32_t n = min(ctr[kListed], static_cast<std::uint32_t>(j.max_maxima));
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const std::uint32_t stride = static_cast<std::uint32_t>(j.select_blocks) * 256u;
    for (std::uint32_t i0 = static_cast<std::uint32_t>(local) * 256u; i0 < n; i0 += stride) {  // block-uniform
        const std::uint32_t i = i0 + threadIdx.x;
        bool above = false, tie = false;
        std::uint32_t px = 0;
        if (i < n) {
            const std::uint64_t e = j.maxima[i];
            const auto score = static_cast<std::uint32_t>(e >> 32);
            px = static_cast<std::uint32_t>(e);
            above = score > p.threshold;
            tie = all_ties && score == p.threshold;
        }
        const unsigned ma = __ballot_sync(0xffffffffu, above), mt = __ballot_sync(0xffffffffu, tie);
        std::uint32_t ba = 0, bt = 0;
        if (lane == 0) {
            if (ma) ba = atomicAdd(&ctr[kAboveWritten], static_cast<std::uint32_t>(__popc(ma)));
            if (mt) bt = atomicAdd(&ctr[kTiesWritten], static_cast<std::uint32_t>(__popc(mt)));
        }
        ba = __shfl_sync(0xffffffffu, ba, 0) + __popc(ma & below);
        bt = __shfl_sync(0xffffffffu, bt, 0) + __popc(mt & below);
        if (above && ba < p.above) j.keys[ba] = px;  // always true when list and histogram agree
        if (tie && bt < p.ties) j.keys[p.above + bt] = px;
    }
}

// The first `ties` maxima at the threshold score in raster order, when the
// select kernel could not take every tie: a most-significant-digit radix
// select over their raster indices (unique) finds the ties-th smallest, P,
// and every tie at or below P goes to keys[above, selected). One block per
// job; the reference's equivalent is the raster-order scatter of the first
// ties (src/s2_s3/s2.cu:182-235).
template <class Src>
__global__ __launch_bounds__(kTieThreads) void ties_kernel(const __grid_constant__ Src src) {
    __shared__ std::uint32_t bins[256];
    __shared__ std::uint32_t pick[2];  // digit, maxima before it
    DetectJob j;
    int local;
    if (!src.find(blockIdx.x, kSortKind, &j, &local)) return;
    const SelectParams p = *j.params;
    if (p.selected == 0 || p.ties == j.hist[p.threshold]) return;  // nothing to pick, or all written
    std::uint32_t* ctr = j.counters();
    const std::uint32_t n = min(ctr[kListed], static_cast<std::uint32_t>(j.max_maxima));
    const std::uint32_t T = p.threshold;
    std::uint32_t prefix = 0, need = p.ties;
    for (int shift = 24; shift >= 0; shift -= 8) {
        const std::uint32_t high = shift == 24 ? 0u : (0xffffffffu << (shift + 8));
        for (int b = threadIdx.x; b < 256; b += kTieThreads) bins[b] = 0;
        __syncthreads();
        for (std::uint32_t i = threadIdx.x; i < n; i += kTieThreads) {
            const std::uint64_t e = j.maxima[i];
            const auto px = static_cast<std::uint32_t>(e);
            if (static_cast<std::uint32_t>(e >> 32) == T && (px & high) == prefix)
                atomicAdd(&bins[(px >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            std::uint32_t run = 0, d = 0;
            while (d < 255 && run + bins[d] < need) run += bins[d++];
            pick[0] = d;
            pick[1] = run;
        }
        __syncthreads();
        prefix |= pick[0] << shift;
        need -= pick[1];
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    for (std::uint32_t i0 = 0; i0 < n; i0 += kTieThreads) {  // block-uniform
        const std::uint32_t i = i0 + threadIdx.x;
        bool keep = false;
        std::uint32_t px = 0;
        if (i < n) {
            const std::uint64_t e = j.maxima[i];
            px = static_cast<std::uint32_t>(e);
            keep = static_cast<std::uint32_t>(e >> 32) == T && px <= prefix;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        std::uint32_t b = 0;
        if (lane == 0 && m) b = atomicAdd(&ctr[kTiesWritten], static_cast<std::uint32_t>(__popc(m)));
        b = __shfl_sync(0xffffffffu, b, 0) + __popc(m & below);
        if (keep && b < p.ties) j.keys[p.above + b] = px;
    }
}

// ------------------------------------------------------------- Harris

// Monotone float -> unsigned order (never 0 for a finite input).
__device__ __forceinline__ std::uint32_t order_bits(float v) {
    const std::uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_order_bits(std::uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// (1 / (4 * 7 * 255))^4 evaluated in float32, as ORB's HarrisResponses does.
constexpr float kHarrisScale4 = 0x1.bb9da2p-52f;

// Harris response over the 7x7 window of 3x3 Sobel gradients centred on
// (x, y): integer sums, then det - k * trace^2 in float32 with every product
// and sum rounded separately.
__device__ __forceinline__ float harris_response(const std::uint8_t* img, int pitch, int x, int y, float k) {
    int p[9][9];
    const std::uint8_t* base = img + static_cast<std::size_t>(y - 4) * pitch + (x - 4);
#pragma unroll
    for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int c = 0; c < 9; ++c) p[r][c] = base[static_cast<std::size_t>(r) * pitch + c];
    int a = 0, b = 0, cc = 0;
#pragma unroll
    for (int i = 1; i < 8; ++i)
#pragma unroll
        for (int jx = 1; jx < 8; ++jx) {
            const int ix = (p[i][jx + 1] - p[i][jx - 1]) * 2 + (p[i - 1][jx + 1] - p[i - 1][jx - 1]) +
                           (p[i + 1][jx + 1] - p[i + 1][jx - 1]);
            const int iy = (p[i + 1][jx] - p[i - 1][jx]) * 2 + (p[i + 1][jx - 1] - p[i - 1][jx - 1]) +
                           (p[i + 1][jx + 1] - p[i - 1][jx + 1]);
            a += ix * ix;
            b += iy * iy;
            cc += ix * iy;
        }
    const float fa = static_cast<float>(a), fb = static_cast<float>(b), fc = static_cast<float>(cc);
    const float trace = __fadd_rn(fa, fb);
    const float det = __fsub_rn(__fmul_rn(fa, fb), __fmul_rn(fc, fc));
    const float penalty = __fmul_rn(__fmul_rn(k, trace), trace);
    return __fmul_rn(__fsub_rn(det, penalty), kHarrisScale4);
}

// Replaces each pre-selected pixel index by its sort key
// (order_bits(response) << 32) | (0xffffffff - index): larger key = better,
// equal responses prefer the smaller raster index.
template <class Src>
__global__ __launch_bounds__(kHarrisThreads) void harris_kernel(const __grid_constant__ Src src) {
    DetectJob j;
    int local;
    if (!src.find(blockIdx.x, kHarrisKind, &j, &local)) return;
    const int slot = local * kHarrisThreads + threadIdx.x;
    if (slot >= j.candidates) return;
    const std::uint32_t selected = j.params->selected;
    if (static_cast<std::uint32_t>(slot) >= selected) return;
    const auto px = static_cast<std::uint32_t>(j.keys[slot]);
    const int x = static_cast<int>(px % static_cast<std::uint32_t>(j.width));
    const int y = static_cast<int>(px / static_cast<std::uint32_t>(j.width));
    const float r = harris_response(j.image, j.pitch, x, y, j.harris_k);
    j.keys[slot] = (static_cast<std::uint64_t>(order_bits(r)) << 32) | (0xffffffffu - px);
}

// ------------------------------------------------------------- top-K

// Flags the blur tiles within kSampleRadius of the keypoint at (x, y) (the
// describe kernel samples nothing else of the blurred layer around it) and
// lists each newly flagged tile once for blur_tiles_kernel.
__device__ __forceinline__ void mark_blur_tiles(const DetectJob& j, int x, int y) {
    const int tx0 = max(x - kSampleRadius, 0) / kBlurTileW, tx1 = min(x + kSampleRadius, j.width - 1) / kBlurTileW;
    const int ty0 = max(y - kSampleRadius, 0) / kBlurTileH, ty1 = min(y + kSampleRadius, j.height - 1) / kBlurTileH;
    const int tiles_x = (j.width + kBlurTileW - 1) / kBlurTileW;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int t = ty * tiles_x + tx;
            if (atomicExch(&j.blur_marks[t], 1u) == 0u)
                j.blur_list[atomicAdd(j.blur_count, 1u)] = make_uint2(static_cast<unsigned>(j.job), static_cast<unsigned>(t));
        }
}

__device__ __forceinline__ void write_keypoint(const DetectJob& j, int rank, std::uint64_t key) {
    const std::uint32_t px = 0xffffffffu - static_cast<std::uint32_t>(key);
    const std::uint32_t x = px % static_cast<std::uint32_t>(j.width), y = px / static_cast<std::uint32_t>(j.width);
    j.x[rank] = static_cast<float>(x);
    j.y[rank] = static_cast<float>(y);
    if (j.response) j.response[rank] = from_order_bits(static_cast<std::uint32_t>(key >> 32));
    if (j.blur_marks) mark_blur_tiles(j, static_cast<int>(x), static_cast<int>(y));
}

// One block per image: bitonic sort (descending) of up to kSortCap keys in
// shared memory, then the first min(K, selected) become the keypoints.
template <class Src>
__global__ __launch_bounds__(kSortThreads) void sort_topk_kernel(const __grid_constant__ Src src) {
    extern __shared__ std::uint64_t sk[];
    DetectJob j;
    int local;
    if (!src.find(blockIdx.x, kSortKind, &j, &local)) return;
    const int n = static_cast<int>(j.params->selected);
    if (n > kSortCap || n == 0) return;
    int N = kSortChunk;  // at least one 64-key chunk (zero keys pad and sort last)
    while (N < n) N <<= 1;
    for (int i = threadIdx.x; i < N; i += kSortThreads) sk[i] = i < n ? j.keys[i] : 0ull;
    __syncthreads();
    // Bitonic network, keys unique: a compare-exchange of i < q = i + s puts
    // the larger key first where (i & k) == 0 (those runs end up descending).
    // Exchanges closer than 64 keys run in registers, a warp holding keys
    // c*64 + lane and c*64 + lane + 32 of chunk c; wider ones in shared memory.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto chunk_pass = [&](int k_lo, int k_hi, int s_top) {
        for (int c = warp; c < N / kSortChunk; c += kSortThreads / 32) {
            const int e0 = c * kSortChunk + lane;
            std::uint64_t v0 = sk[e0], v1 = sk[e0 + 32];
            for (int k = k_lo; k <= k_hi; k <<= 1) {
                for (int s = min(k >> 1, s_top); s > 0; s >>= 1) {
                    if (s == 32) {  // v0 (key e0) is the lower of the pair
                        const bool desc = (e0 & k) == 0;
                        const std::uint64_t hi = v0 > v1 ? v0 : v1, lo = v0 > v1 ? v1 : v0;
                        v0 = desc ? hi : lo;
                        v1 = desc ? lo : hi;
                    } else {
                        const bool lower = (lane & s) == 0;
                        const std::uint64_t p0 = __shfl_xor_sync(0xffffffffu, v0, s);
                        const std::uint64_t p1 = __shfl_xor_sync(0xffffffffu, v1, s);
                        const bool keep_hi0 = lower == ((e0 & k) == 0);
                        const bool keep_hi1 = lower == (((e0 + 32) & k) == 0);
                        v0 = keep_hi0 ? (v0 > p0 ? v0 : p0) : (v0 > p0 ? p0 : v0);
                        v1 = keep_hi1 ? (v1 > p1 ? v1 : p1) : (v1 > p1 ? p1 : v1);
                    }
                }
            }
            sk[e0] = v0;
            sk[e0 + 32] = v1;
        }
        __syncthreads();
    };
    chunk_pass(2, kSortChunk, kSortChunk / 2);  // runs up to 64 keys: registers only
    for (int k = 2 * kSortChunk; k <= N; k <<= 1) {
        for (int s = k >> 1; s >= kSortChunk; s >>= 1) {
            for (int t = threadIdx.x; t < (N >> 1); t += kSortThreads) {
                const int i = (t / s) * (s << 1) + (t % s);
                const int q = i + s;
                const std::uint64_t a = sk[i], b = sk[q];
                const bool descending = (i & k) == 0;
                if (descending ? (a < b) : (a > b)) { sk[i] = b; sk[q] = a; }
            }
            __syncthreads();
        }
        chunk_pass(k, k, kSortChunk / 2);
    }
    const int limit = min(n, j.max_keypoints);
    for (int i = threadIdx.x; i < limit; i += kSortThreads) write_keypoint(j, i, sk[i]);
}

// Fallback for images with more than kSortCap pre-selected points: the rank
// of a key is the number of larger keys (keys are unique). Launched over the
// same blocks as the Harris kernel.
template <class Src>
__global__ __launch_bounds__(kHarrisThreads) void rank_topk_kernel(const __grid_constant__ Src src) {
    __shared__ std::uint64_t tile[kHarrisThreads];
    DetectJob j;
    int local;
    if (!src.find(blockIdx.x, kHarrisKind, &j, &local)) return;
    const int n = static_cast<int>(j.params->selected);
    if (n <= kSortCap) return;
    const int slot = local * kHarrisThreads + static_cast<int>(threadIdx.x);
    if (local * kHarrisThreads >= n) return;  // block-uniform
    const std::uint64_t key = slot < n ? j.keys[slot] : 0ull;
    int rank = 0;
    for (int b0 = 0; b0 < n; b0 += kHarrisThreads) {
        const int q = b0 + static_cast<int>(threadIdx.x);
        tile[threadIdx.x] = q < n ? j.keys[q] : 0ull;
        __syncthreads();
        const int m = min(kHarrisThreads, n - b0);
        for (int i = 0; i < m; ++i) rank += tile[i] > key;
        __syncthreads();
    }
    if (slot < n && rank < j.max_keypoints) write_keypoint(j, rank, key);
}

// ------------------------------------------------------ pyramid layers

// Source index and 8-bit weight of the right neighbour for destination
// index v of a src -> dst linear resize: f = (v + 0.5) * scale - 0.5 in
// double with scale = 1 / (dst / src), weight rint((f - floor f) * 256).
// Indices left of the source (every index when src == 1) read pixel 0 with
// weight 0, indices past the last interval read pixel src - 1 with weight 0.
__host__ __device__ inline double linear_exact_scale(int src, int dst) {
    return 1.0 / (static_cast<double>(dst) / static_cast<double>(src));
}

__device__ __forceinline__ int2 linear_exact_tap(int v, int src, double scale) {
    const double f = scale * (static_cast<double>(v) + 0.5) - 0.5;
    const double fl = floor(f);
    if (src == 1 || fl < 0.0) return make_int2(0, 0);
    if (fl >= static_cast<double>(src - 1)) return make_int2(src - 1, 0);
    return make_int2(static_cast<int>(fl), static_cast<int>(rint((f - fl) * 256.0)));
}

// One block = one tile of 128 x kTileH (16..64) layer pixels:
//   1. per-column and per-row taps in shared memory (double, as above);
//   2. the tile's exact source window (rows of the first and last row taps,
//      columns from the first column tap rounded down to 16 bytes) is
//      staged in shared memory with 16-byte asynchronous copies;
//   3. warp w makes the band of kTileH / 8 consecutive rows starting at row
//      w * kTileH / 8, lane l columns 4l .. 4l + 3:
//        h(r, c) = src[r][c0] * (256 - wx) + src[r][c0 + 1] * wx   (< 2^16)
//        out = (h(ra, c) * (256 - wy) + h(rb, c) * wy + 2^15) >> 16,
//      the integer form of the 8-bit fixed-point horizontal pass followed by
//      the vertical pass with one final rounding. The band's source rows are
//      walked once, top to bottom: a row's h comes from two byte permutes of
//      aligned shared-memory words and one 16x8-bit dot product per column,
//      and every output row whose lower source row it is goes out with the
//      previous source row's h. A whole warp shares one band, so its lanes
//      take the same branches.
// Blocks whose source is not 16-byte aligned or whose window exceeds the
// staging buffer (layer ratios above about 1.45), and lanes whose bytes do
// not fit two 8-byte pools, read the source bytes from global memory per
// output row instead, with the same result.
constexpr int kRawStride = 256;  // bytes of a staged source row: 16 chunks of 16
template <int kTileH> __host__ __device__ constexpr int resize_raw_rows() { return kTileH * 3 / 2 + 6; }

__device__ __forceinline__ std::uint32_t resize_out(std::uint32_t ha, std::uint32_t hb, std::uint32_t wy) {
    return (ha * (256u - wy) + hb * wy + 32768u) >> 16;
}

template <class Src, int kTileH>
__global__ __launch_bounds__(256, 5) void resize_kernel(const __grid_constant__ Src src, int kind) {
    static_assert(kTileH >= 16 && kTileH <= kResizeTileH && kTileH % 16 == 0, "resize tile height");
    constexpr int kBand = kTileH / 8, kRows = resize_raw_rows<kTileH>();
    __shared__ int2 xtap[kResizeTileW];
    __shared__ int2 ytap[kTileH];
    __shared__ __align__(16) std::uint8_t raw[kRows][kRawStride];
    ResizeJob j;
    int local;
    if (!src.find(blockIdx.x, kind, &j, &local)) return;
    const int y0 = (local / j.tiles_x) * kTileH;
    const int x0 = (local % j.tiles_x) * kResizeTileW;
    const int t = threadIdx.x;
    // 1. taps (columns and rows past the layer edge repeat the last one)
    if (t < kResizeTileW) xtap[t] = linear_exact_tap(min(x0 + t, j.width - 1), j.src_width, j.scale_x);
    else if (t < kResizeTileW + kTileH)
        ytap[t - kResizeTileW] = linear_exact_tap(min(y0 + t - kResizeTileW, j.height - 1), j.src_height, j.scale_y);
    __syncthreads();
    // 2. source window: rows ry0 .. ry1, 16-byte chunks from column rx0
    const int ry0 = ytap[0].x, ry1 = min(ytap[kTileH - 1].x + 1, j.src_height - 1);
    const int rx0 = xtap[0].x & ~15, rx1 = min(xtap[kResizeTileW - 1].x + 1, j.src_width - 1);
    const int nrow = ry1 - ry0 + 1, nchunk = (rx1 - rx0) / 16 + 1;
    const bool staged = ((reinterpret_cast<std::uintptr_t>(j.src) | static_cast<std::uintptr_t>(j.src_pitch)) & 15) == 0 &&
                        nrow <= kRows && nchunk <= kRawStride / 16;  // block-uniform
    if (staged) {
        const int q = t & 15, col = rx0 + 16 * q;
        if (q < nchunk) {
            for (int r = t >> 4; r < nrow; r += 16) {
                const int gy = ry0 + r;
                const std::uint8_t* p = j.src + static_cast<std::size_t>(gy) * j.src_pitch + col;
                // bytes of the row that may be read: the pitch, the width on the last row
                if (col + 16 <= (gy < j.src_height - 1 ? j.src_pitch : j.src_width)) {
                    cp_async16(&raw[r][16 * q], p);
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) raw[r][16 * q + k] = col + k < j.src_width ? p[k] : 0;
                }
            }
        }
        cp_async_wait_all();
    }
    __syncthreads();
    // 3. bands
    const int r0 = (t >> 5) * kBand;
    const int r_end = r0 + min(kBand, j.height - y0 - r0);  // band rows inside the layer
    const int c = 4 * (t & 31), x = x0 + c;
    if (r_end <= r0 || x >= j.width) return;
    int2 tx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) tx[k] = xtap[c + k];
    std::uint32_t wx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) wx[k] = (256u - tx[k].y) | (static_cast<std::uint32_t>(tx[k].y) << 16);
    const int nx = min(4, j.width - x);
    std::uint8_t* dst = j.dst + static_cast<std::size_t>(y0 + r0) * j.pitch + x;
    const bool word_store = nx == 4 && ((reinterpret_cast<std::uintptr_t>(j.dst) | static_cast<std::uintptr_t>(j.pitch)) & 3) == 0;
    auto emit = [&](const std::uint32_t (&ha)[4], const std::uint32_t (&hb)[4], std::uint32_t wy) {
        std::uint32_t v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = resize_out(ha[k], hb[k], wy);
        if (word_store) {
            *reinterpret_cast<std::uint32_t*>(dst) = __byte_perm(__byte_perm(v[0], v[1], 0x0040), __byte_perm(v[2], v[3], 0x0040), 0x5410);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < nx) dst[k] = static_cast<std::uint8_t>(v[k]);
        }
        dst += j.pitch;
    };
    // the lane's bytes: pool A = 8 bytes at column `base` (columns 0, 1),
    // pool B = 8 bytes at base + 4 * kb (columns 2, 3)
    const int base = tx[0].x & ~3;
    const int o0 = tx[0].x - base, o1 = tx[1].x - base;
    const int kb = (tx[2].x - base) >> 2;
    const int o2 = tx[2].x - base - 4 * kb, o3 = tx[3].x - base - 4 * kb;
    const bool fits = staged && o1 + 1 <= 7 && o3 + 1 <= 7 && base - rx0 + 4 * kb + 8 <= kRawStride;
    if (!fits) {
        int xb[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) xb[k] = min(tx[k].x + 1, j.src_width - 1);
        for (int rr = r0; rr < r_end; ++rr) {
            const int2 ty = ytap[rr];
            const std::uint8_t* A = j.src + static_cast<std::size_t>(ty.x) * j.src_pitch;
            const std::uint8_t* B = j.src + static_cast<std::size_t>(min(ty.x + 1, j.src_height - 1)) * j.src_pitch;
            std::uint32_t ha[4], hb[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const std::uint32_t wa = __ldg(A + tx[k].x) | (static_cast<std::uint32_t>(__ldg(A + xb[k])) << 8);
                const std::uint32_t wb = __ldg(B + tx[k].x) | (static_cast<std::uint32_t>(__ldg(B + xb[k])) << 8);
                ha[k] = __dp2a_lo(wx[k], wa, 0u);
                hb[k] = __dp2a_lo(wx[k], wb, 0u);
            }
            emit(ha, hb, static_cast<std::uint32_t>(ty.y));
        }
        return;
    }
    const std::uint32_t sel_a = static_cast<std::uint32_t>(o0 | ((o0 + 1) << 4) | (o1 << 8) | ((o1 + 1) << 12));
    const std::uint32_t sel_b = static_cast<std::uint32_t>(o2 | ((o2 + 1) << 4) | (o3 << 8) | ((o3 + 1) << 12));
    const std::uint8_t* lane_bytes = &raw[0][0] + (base - rx0);
    const int s_last = min(ytap[r_end - 1].x + 1, j.src_height - 1);
    int rr = r0;
    int2 ty = ytap[rr];
    int s = ty.x;
    std::uint32_t pa[4] = {0u, 0u, 0u, 0u};  // h of source row s - 1
    while (rr < r_end && s <= s_last) {  // s <= rb of row rr throughout (monotone taps)
        s = max(s, ty.x);  // skips source rows no output row reads (layer ratios above 2)
        const auto* w = reinterpret_cast<const std::uint32_t*>(lane_bytes + (s - ry0) * kRawStride);
        const std::uint32_t pool_a = __byte_perm(w[0], w[1], sel_a), pool_b = __byte_perm(w[kb], w[kb + 1], sel_b);
        const std::uint32_t h[4] = {__dp2a_lo(wx[0], pool_a, 0u), __dp2a_hi(wx[1], pool_a, 0u),
                                    __dp2a_lo(wx[2], pool_b, 0u), __dp2a_hi(wx[3], pool_b, 0u)};
        // every row whose lower source row is s (ra = s - 1, or ra = s at the bottom edge)
        while (rr < r_end && min(ty.x + 1, j.src_height - 1) == s) {
            if (ty.x == s) emit(h, h, static_cast<std::uint32_t>(ty.y));
            else emit(pa, h, static_cast<std::uint32_t>(ty.y));
            if (++rr < r_end) ty = ytap[rr];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) pa[k] = h[k];
        ++s;
    }
}

// ------------------------------------------------------------- S3 blur

// One block = one 64x64 tile: rows pass into a float tile with a 3-row halo,
// then the columns pass; per output the taps are summed first to last with
// each product and sum rounded separately, then rounded half-to-even and
// clamped to [0, 255].
template <class Src>
__global__ __launch_bounds__(256) void blur_kernel(const __grid_constant__ Src src) {
    __shared__ std::uint8_t in[kBlurTileH + 6][kBlurTileW + 6];
    __shared__ float rows[kBlurTileH + 6][kBlurTileW];
    DescribeJob j;
    int local;
    if (!src.find(blockIdx.x, kBlurKind, &j, &local)) return;
    const int W = j.width, H = j.height;
    const int y0 = (local / j.tiles_x) * kBlurTileH;
    const int x0 = (local % j.tiles_x) * kBlurTileW;
    for (int i = threadIdx.x; i < (kBlurTileH + 6) * (kBlurTileW + 6); i += 256) {
        const int r = i / (kBlurTileW + 6), c = i - r * (kBlurTileW + 6);
        const int gy = reflect101(y0 - 3 + r, H), gx = reflect101(x0 - 3 + c, W);
        in[r][c] = j.image[static_cast<std::size_t>(gy) * j.pitch + gx];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < (kBlurTileH + 6) * kBlurTileW; i += 256) {
        const int r = i / kBlurTileW, c = i - r * kBlurTileW;
        float acc = 0.0f;
#pragma unroll
        for (int t = 0; t < 7; ++t) acc = __fadd_rn(acc, __fmul_rn(blur_tap(t), static_cast<float>(in[r][c + t])));
        rows[r][c] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kBlurTileH * kBlurTileW; i += 256) {
        const int r = i / kBlurTileW, c = i - r * kBlurTileW;
        const int gy = y0 + r, gx = x0 + c;
        if (gx >= W || gy >= H) continue;
        float acc = 0.0f;
#pragma unroll
        for (int t = 0; t < 7; ++t) acc = __fadd_rn(acc, __fmul_rn(blur_tap(t), rows[r + t][c]));
        // Clamping the float to [0, 255] before rounding half-to-even gives
        // the same byte as rounding then clamping the integer, for every
        // finite acc, and keeps signed integer min/max out of this kernel.
        j.blurred[static_cast<std::size_t>(gy) * j.blur_pitch + gx] =
            static_cast<std::uint8_t>(__float2int_rn(fminf(fmaxf(acc, 0.0f), 255.0f)));
    }
}

// The S3 blur of the 64x64 tiles listed by the keypoint writers (on-demand
// blur of the pyramid and batched paths): the same bytes as blur_kernel
// (per output the taps summed first to last, each product and sum rounded on
// its own, then rounded half-to-even and clamped), with both passes on the
// sm_100 packed FP32x2 add and multiply (two rows, or two columns, per
// instruction, each lane rounded as the scalar op). Persistent: block b takes
// list entries b, b + gridDim.x, ... (the list is complete when the kernel
// starts). A tile is staged with its reflect-101 halo: 16-byte loads for
// interior tiles of 16-byte aligned images, reflected byte loads otherwise.
constexpr int kBlurInH = kBlurTileH + 8;  // staged rows of a blur tile: rows y0-4 .. y0+kBlurTileH+3 (halo 3, rounded to 4)

// Origin of blur tile `tile` of job j.
__device__ __forceinline__ void blur_tile_origin(const DescribeJob& j, unsigned tile, int* x0, int* y0) {
    const int tiles_x = (j.width + kBlurTileW - 1) / kBlurTileW;
    *y0 = (static_cast<int>(tile) / tiles_x) * kBlurTileH;
    *x0 = (static_cast<int>(tile) % tiles_x) * kBlurTileW;
}

__device__ __forceinline__ bool aligned16(const DescribeJob& j) {
    return ((reinterpret_cast<std::uintptr_t>(j.image) | static_cast<std::uintptr_t>(j.pitch)) & 15) == 0;
}

// Asynchronous staging of a blur tile of a 16-byte aligned image: row r of
// `in` is image row reflect101(y0 - 4 + r) (the reflected halo rows are whole
// image rows), byte c is column x0 - 16 + c. Chunks inside a row's pitch
// (inside the width on the last image row) are 16-byte copies, a chunk
// straddling the end of the last row is copied byte by byte; the reflected
// halo columns are filled by blur_fix_columns once the copies are complete.
__device__ __forceinline__ void blur_stage_async(const DescribeJob& j, int x0, int y0, std::uint8_t (*in)[kInStride]) {
    const int tid = threadIdx.x;
    constexpr int kChunks = kInStride / 16;
    for (int i = tid; i < kBlurInH * kChunks; i += 256) {
        const int r = i / kChunks, q = i - r * kChunks;
        const int gy = reflect101(y0 - 4 + r, j.height);
        const int cx = x0 - 16 + 16 * q;
        const int limit = gy == j.height - 1 ? j.width : j.pitch;
        const std::uint8_t* row = j.image + static_cast<std::size_t>(gy) * j.pitch;
        if (cx >= 0 && cx + 16 <= limit) {
            cp_async16(&in[r][16 * q], row + cx);
        } else if (cx >= 0 && cx < j.width) {
            for (int b = 0; b < 16 && cx + b < j.width; ++b) in[r][16 * q + b] = row[cx + b];
        }
    }
}

// Whether the 7x7 blur of the tile at x0 reads columns outside the image.
__device__ __forceinline__ bool blur_needs_columns(int x0, int W) { return x0 < 3 || x0 + kBlurTileW + 3 > W; }

// Reflect-101 halo columns of a staged tile: column -k is column k, column
// W - 1 + k is column W - 1 - k (k = 1..3), copied inside `in`.
__device__ __forceinline__ void blur_fix_columns(int x0, int W, std::uint8_t (*in)[kInStride]) {
    for (int i = threadIdx.x; i < kBlurInH * 6; i += 256) {  // sources are interior columns, never written here
        const int r = i / 6, k = i % 6;
        const int off = x0 - 16;  // column of byte 0
        int dst, srcc;
        if (k < 3) {  // left edge
            dst = -(k + 1);
            srcc = k + 1;
        } else {      // right edge
            dst = W - 1 + (k - 2);
            srcc = W - 1 - (k - 2);
        }
        const int db = dst - off, sb = srcc - off;
        if (db >= 0 && db < kInStride && sb >= 0 && sb < kInStride && dst >= x0 - 3 && dst <= x0 + kBlurTileW + 2)
            in[r][db] = in[r][sb];
    }
}

constexpr int kBlurCtasPerSm = 6;  // resident blur blocks per SM; the persistent grid is 148 x this
template <class Src>
__global__ __launch_bounds__(256, kBlurCtasPerSm) void blur_tiles_kernel(const __grid_constant__ Src src, const uint2* list,
                                                            const std::uint32_t* count) {
    __shared__ __align__(16) std::uint8_t in2[2][kBlurInH][kInStride];  // rows y0-4 .., columns x0-16 ..
    __shared__ __align__(16) float rows[kBlurTileH + 6][kBlurTileW];
    __shared__ std::size_t row_at[kBlurInH];
    __shared__ int col_at[kInStride];
    const int tid = threadIdx.x;
    const int n = static_cast<int>(*count);
    // tiles of aligned images are copied asynchronously, the next one while this one is blurred
    auto prefetch = [&](int i, std::uint8_t (*dst)[kInStride]) {
        const uint2 e = list[i];
        const DescribeJob jn = src.at(static_cast<int>(e.x));
        if (!aligned16(jn)) return;
        int x0, y0;
        blur_tile_origin(jn, e.y, &x0, &y0);
        blur_stage_async(jn, x0, y0, dst);
    };
    int buf = 0;
    if (static_cast<int>(blockIdx.x) < n) prefetch(blockIdx.x, in2[0]);
    for (int i = blockIdx.x; i < n; i += gridDim.x, buf ^= 1) {
        std::uint8_t (*in)[kInStride] = in2[buf];
        const uint2 e = list[i];
        const DescribeJob j = src.at(static_cast<int>(e.x));
        const int W = j.width, H = j.height;
        int x0, y0;
        blur_tile_origin(j, e.y, &x0, &y0);
        if (!aligned16(j)) {  // unaligned image: reflected byte loads
            if (tid < kBlurInH) row_at[tid] = static_cast<std::size_t>(reflect101(y0 - 4 + tid, H)) * j.pitch;
            else if (tid < kBlurInH + kInStride) col_at[tid - kBlurInH] = reflect101(x0 - 16 + (tid - kBlurInH), W);
            __syncthreads();
            for (int k = tid; k < kBlurInH * (kInStride / 4); k += 256) {
                const int r = k / (kInStride / 4), b = 4 * (k - r * (kInStride / 4));
                const std::uint8_t* row = j.image + row_at[r];
                *reinterpret_cast<std::uint32_t*>(&in[r][b]) =
                    static_cast<std::uint32_t>(row[col_at[b]]) | (static_cast<std::uint32_t>(row[col_at[b + 1]]) << 8) |
                    (static_cast<std::uint32_t>(row[col_at[b + 2]]) << 16) |
                    (static_cast<std::uint32_t>(row[col_at[b + 3]]) << 24);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (aligned16(j) && blur_needs_columns(x0, W)) {
            blur_fix_columns(x0, W, in);
            __syncthreads();
        }
        if (i + static_cast<int>(gridDim.x) < n) prefetch(i + gridDim.x, in2[buf ^ 1]);
        // rows pass: image rows y0-3 .. y0+34, two rows x 4 outputs per item
        static_assert((kBlurTileH + 6) % 2 == 0, "rows pass takes row pairs");
        for (int g = tid; g < (kBlurTileH + 6) / 2 * (kBlurTileW / 4); g += 256) {
            const int rp = g / (kBlurTileW / 4), q = g - rp * (kBlurTileW / 4), rr = 2 * rp;
            const auto* ra = reinterpret_cast<const std::uint32_t*>(&in[rr + 1][0]);
            const auto* rb = reinterpret_cast<const std::uint32_t*>(&in[rr + 2][0]);
            const std::uint32_t a0 = ra[q + 3], a1 = ra[q + 4], a2 = ra[q + 5];  // bytes 4q+12 .. 4q+23
            const std::uint32_t b0 = rb[q + 3], b1 = rb[q + 4], b2 = rb[q + 5];
            // output 4q+k reads halo columns 4q+k+1 .. 4q+k+7, tap t on column
            // 4q+k+1+t; lane x holds row rr, lane y row rr + 1. The columns
            // stream in once and every output adds its taps in order (0 + a
            // nonnegative product is the product).
            float2 out[4];
#pragma unroll
            for (int m = 1; m <= 10; ++m) {
                const std::uint32_t wa = m < 4 ? a0 : m < 8 ? a1 : a2, wb = m < 4 ? b0 : m < 8 ? b1 : b2;
                const float2 xm = byte_pair(wa, wb, m & 3);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int t = m - 1 - k;
                    if (t == 0) out[k] = __fmul2_rn(tap_pair(0), xm);
                    else if (t > 0 && t < 7) out[k] = __fadd2_rn(out[k], __fmul2_rn(tap_pair(t), xm));
                }
            }
            *reinterpret_cast<float4*>(&rows[rr][4 * q]) = make_float4(out[0].x, out[1].x, out[2].x, out[3].x);
            *reinterpret_cast<float4*>(&rows[rr + 1][4 * q]) = make_float4(out[0].y, out[1].y, out[2].y, out[3].y);
        }
        __syncthreads();
        // columns pass: rows 2p, 2p+1 and columns 4q .. 4q+3 per thread and step
        for (int pr = tid / (kBlurTileW / 4), q = tid % (kBlurTileW / 4); pr < kBlurTileH / 2;
             pr += 256 / (kBlurTileW / 4)) {
            float2 lo[2], hi[2];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const float4 v = *reinterpret_cast<const float4*>(&rows[2 * pr + r][4 * q]);
                const float2 vl = make_float2(v.x, v.y), vh = make_float2(v.z, v.w);
#pragma unroll
                for (int o = 0; o < 2; ++o) {
                    const int t = r - o;
                    if (t == 0) {
                        lo[o] = __fmul2_rn(tap_pair(0), vl);
                        hi[o] = __fmul2_rn(tap_pair(0), vh);
                    } else if (t > 0 && t < 7) {
                        lo[o] = __fadd2_rn(lo[o], __fmul2_rn(tap_pair(t), vl));
                        hi[o] = __fadd2_rn(hi[o], __fmul2_rn(tap_pair(t), vh));
                    }
                }
            }
#pragma unroll
            for (int o = 0; o < 2; ++o) {
                const int gy = y0 + 2 * pr + o, gx = x0 + 4 * q;
                if (gy >= H || gx >= W) continue;
                const std::uint32_t packed = blur_byte(lo[o].x) | (blur_byte(lo[o].y) << 8) |
                                             (blur_byte(hi[o].x) << 16) | (blur_byte(hi[o].y) << 24);
                std::uint8_t* dst = j.blurred + static_cast<std::size_t>(gy) * j.blur_pitch + gx;
                if (gx + 3 < W && (reinterpret_cast<std::uintptr_t>(dst) & 3) == 0) {
                    *reinterpret_cast<std::uint32_t*>(dst) = packed;
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (gx + k < W) dst[k] = static_cast<std::uint8_t>(packed >> (8 * k));
                }
            }
        }
        __syncthreads();  // before the next tile's staging
    }
}

// ---------------------------------------------------------- S3 describe

// Global (not __constant__): each thread reads a different pair, which the
// constant cache would serialise.
__device__ const int4 kOrbPattern[256] = {
#include "orb_pattern_31.inc"
};

// Half-widths of the rows of the radius-15 orientation disc, v = 0..15:
// 15 15 15 15 14 14 14 13 13 12 11 10 9 8 6 3 (one byte per row).
__device__ __forceinline__ int disc_half_width(int v) {
    constexpr unsigned long long lo = 0x0d0e0e0e0f0f0f0full;  // rows 0..7, row 0 in the low byte
    constexpr unsigned long long hi = 0x030608090a0b0c0dull;  // rows 8..15, row 8 in the low byte
    return v < 8 ? static_cast<int>((lo >> (8 * v)) & 0xff)
                 : static_cast<int>((hi >> (8 * (v - 8))) & 0xff);
}

// Weights of the orientation disc for 4-byte loads: the disc's 31 rows are
// read as 9 aligned words each (279 (row, word) slots, slot = 9 row + word),
// the first word starting a = (x - 15) & 3 bytes left of column x - 15. Byte
// k of word w is column u = 4w + k - a - 15 of row v = row - 15; inside the
// disc its weights are u (for m10) and v (for m01) as signed bytes, outside 0.
constexpr int kDiscSlots = 288;  // 9 rounds of 32 lanes over the 279 slots
__device__ __forceinline__ uint2 disc_weights(int a, int slot) {
    const int row = slot / 9, word = slot - 9 * row;
    const int v = row - 15, av = v < 0 ? -v : v;
    std::uint32_t wu = 0, wv = 0;
    if (row < 31) {
        const int hw = disc_half_width(av);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int u = 4 * word + k - a - 15;
            if ((u < 0 ? -u : u) <= hw) {
                wu |= (static_cast<std::uint32_t>(u) & 0xffu) << (8 * k);
                wv |= (static_cast<std::uint32_t>(v) & 0xffu) << (8 * k);
            }
        }
    }
    return make_uint2(wu, wv);
}

// acc + sum of the four unsigned bytes of `bytes` times the four signed bytes of `w`
__device__ __forceinline__ int dot4_us(std::uint32_t bytes, std::uint32_t w, int acc) {
    int d;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(bytes), "r"(w), "r"(acc));
    return d;
}

// cv::fastAtan2 in degrees [0, 360): odd polynomial of the smaller/larger
// magnitude ratio, every step rounded in float32.
__device__ __forceinline__ float fast_atan2_deg(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const bool wide = ax >= ay;
    const float eps = 0x1p-52f;
    const float t = wide ? __fdiv_rn(ay, __fadd_rn(ax, eps)) : __fdiv_rn(ax, __fadd_rn(ay, eps));
    const float t2 = __fmul_rn(t, t);
    float p = __fadd_rn(__fmul_rn(-0x1.4515b2p+1f, t2), 0x1.1d3f7ep+3f);
    p = __fadd_rn(__fmul_rn(p, t2), -0x1.2aaddcp+4f);
    p = __fadd_rn(__fmul_rn(p, t2), 0x1.ca44dep+5f);
    p = __fmul_rn(p, t);
    float a = wide ? p : __fsub_rn(90.0f, p);
    if (x < 0) a = __fsub_rn(180.0f, a);
    if (y < 0) a = __fsub_rn(360.0f, a);
    return a;
}

__device__ __forceinline__ int rotated_sample(const std::uint8_t* centre, int stride, float fx, float fy,
                                              float a, float b) {
    const int ix = __float2int_rn(__fsub_rn(__fmul_rn(fx, a), __fmul_rn(fy, b)));
    const int iy = __float2int_rn(__fadd_rn(__fmul_rn(fx, b), __fmul_rn(fy, a)));
    return centre[iy * stride + ix];
}

// One warp per keypoint, kDescRounds keypoints per warp (the block stages
// the pattern once for its kDescKeys keypoints): intensity-centroid moments
// over the radius-15 disc of the unblurred image (lane l sums column l - 15),
// the angle on lane 0 (float fastAtan2, cos/sin evaluated in double then
// rounded to float), then lane l packs pattern pairs 8l..8l+7 of the blurred
// image into descriptor byte l.
// 8 blocks per SM (32 registers): the kernel waits on scattered patch loads,
// so resident warps matter more than the few registers it spills.
template <class Src>
__global__ __launch_bounds__(kDescWarps * 32, 8) void describe_kernel(const __grid_constant__ Src src) {
    __shared__ float4 pat[8][32];  // pat[k][l] = pair 8l + k as floats (x0, y0, x1, y1)
    __shared__ uint2 disc_w[4][kDiscSlots];  // disc_weights(a, slot)
    DescribeJob j;
    int local;
    if (!src.find(blockIdx.x, kDescKind, &j, &local)) return;
    // The grid covers the capacity; blocks past the keypoint count leave now.
    const int count = min(*j.count, j.capacity);
    int base = 0;  // first output row of this layer
    if (j.level_counts) {
        if (local == 0 && threadIdx.x == 0) atomicAdd(j.out_count, count);
        for (int m = 0; m < j.level; ++m) base += j.level_counts[m];
    }
    if (local * kDescKeys >= count) return;
    {
        const int p = threadIdx.x;  // 256 threads, one pattern pair each
        const int4 q = kOrbPattern[p];
        pat[p & 7][p >> 3] = make_float4(static_cast<float>(q.x), static_cast<float>(q.y), static_cast<float>(q.z),
                                         static_cast<float>(q.w));
    }
    // word loads of the disc need 4-byte aligned rows (block-uniform)
    const bool words = ((reinterpret_cast<std::uintptr_t>(j.image) | static_cast<std::uintptr_t>(j.pitch)) & 3) == 0;
    if (words)
        for (int e = threadIdx.x; e < 4 * kDiscSlots; e += kDescWarps * 32)
            disc_w[e / kDiscSlots][e % kDiscSlots] = disc_weights(e / kDiscSlots, e % kDiscSlots);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int u = lane - 15, au = u < 0 ? -u : u;
    const int pitch = j.pitch, blur_pitch = j.blur_pitch;
    for (int r = 0; r < kDescRounds; ++r) {
        const int index = local * kDescKeys + r * kDescWarps + (threadIdx.x >> 5);
        if (index >= count) break;
        std::uint8_t* row = j.out + static_cast<std::size_t>(base + index) * j.row_stride;
        const float fx = j.x[index], fy = j.y[index];
        const int x = __float2int_rn(fx);
        const int y = __float2int_rn(fy);
        if (j.level_counts && lane == 0) {
            j.out_x[base + index] = __fmul_rn(fx, j.scale);
            j.out_y[base + index] = __fmul_rn(fy, j.scale);
            if (j.out_response) j.out_response[base + index] = j.response[index];
        }
        if (x < kEdge || x >= j.width - kEdge || y < kEdge || y >= j.height - kEdge) {
            row[lane] = 0;
            continue;
        }
        // Moments as exact integer sums over the disc. With aligned rows each
        // lane takes slots lane, lane + 32, ... of the disc's words (four
        // pixels per load, weighted by two byte dot products); otherwise lane
        // l owns column u = l - 15 and walks the 31 rows.
        int m10 = 0, m01 = 0;
        if (words) {
            const int xs = x - 15, a = xs & 3;
            const std::uint8_t* top = j.image + static_cast<std::size_t>(y - 15) * pitch + (xs - a);
#pragma unroll
            for (int k = 0; k < kDiscSlots / 32; ++k) {
                const int slot = 32 * k + lane;
                if (slot < 279) {
                    const int row = (slot * 57) >> 9, word = slot - 9 * row;  // slot / 9 for slot < 288
                    const std::uint32_t d =
                        __ldg(reinterpret_cast<const unsigned int*>(top + static_cast<std::size_t>(row) * pitch + 4 * word));
                    const uint2 w = disc_w[a][slot];
                    m10 = dot4_us(d, w.x, m10);
                    m01 = dot4_us(d, w.y, m01);
                }
            }
        } else {
            const std::uint8_t* centre = j.image + static_cast<std::size_t>(y) * pitch + x;
#pragma unroll
            for (int v = -15; v <= 15; ++v) {
                const int av = v < 0 ? -v : v;
                if (lane < 31 && au <= disc_half_width(av)) {
                    const int val = centre[v * pitch + u];
                    m10 += u * val;
                    m01 += v * val;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m10 += __shfl_xor_sync(0xffffffffu, m10, o);
            m01 += __shfl_xor_sync(0xffffffffu, m01, o);
        }
        float a = 0.0f, b = 0.0f;
        if (lane == 0) {
            const float angle = __fmul_rn(fast_atan2_deg(static_cast<float>(m01), static_cast<float>(m10)),
                                          0x1.1df46ap-6f);
            // one sincos for both: it equals cos() and sin() bit for bit on every
            // float in [0, 6.2832] (all the angles this can produce; checked
            // exhaustively by tests/test_gpu_sincos.py)
            double sd, cd;
            sincos(static_cast<double>(angle), &sd, &cd);
            a = static_cast<float>(cd);
            b = static_cast<float>(sd);
        }
        a = __shfl_sync(0xffffffffu, a, 0);
        b = __shfl_sync(0xffffffffu, b, 0);
        const std::uint8_t* smooth = j.blurred + static_cast<std::size_t>(y) * blur_pitch + x;
        int value = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float4 q = pat[k][lane];
            const int t0 = rotated_sample(smooth, blur_pitch, q.x, q.y, a, b);
            const int t1 = rotated_sample(smooth, blur_pitch, q.z, q.w, a, b);
            value |= (t0 < t1) << k;
        }
        row[lane] = static_cast<std::uint8_t>(value);
    }
}

}  // namespace stitch::b200::s2s3
