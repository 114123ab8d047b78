// S1: RGB8 -> GRAY8 with an area resize to scale S in (0, 1], and the
// mean-absolute-gradient probe of the GRAY8 result.
//
// Reference semantics (file:line in the reference tree):
//   gray      src/s1/s1.cu:33-36   (9798 R + 19235 G + 3735 B + 2^14) >> 15
//   modes     src/s1/s1.cu:38-107  S = 1 direct; exact 2x2 and 4x4 averages;
//                                  otherwise a float box filter whose weighted
//                                  sum is accumulated with a fused multiply-add
//                                  (nvcc contracts total += g * (wx * wy))
//   params    src/s1/s1.cu:116-141 inv_s = float(W) / float(W_s), area scale
//                                  1 / (inv_sx * inv_sy), all in float
//   gradient  src/s1/s1.cu:147-205 (sum |dI/dx| + sum |dI/dy|) / (255 edges)
//   host      src/s1/s1.cu:209-320 argument order, one launch for a pair
//
// Both images of a pair run in one launch (blockIdx.z selects the image);
// each thread produces 4 horizontally adjacent outputs.
#include <cmath>

#include "s1_internal.hpp"
#include "s2s3_kernels.cuh"

namespace stitch::b200::s1k {

struct Pair {
    Params img[2];
};

__device__ __forceinline__ int gray15(const std::uint8_t* rgb) {
    return (9798 * rgb[0] + 19235 * rgb[1] + 3735 * rgb[2] + 16384) >> 15;
}

__device__ __forceinline__ int s1_pixel(const Params& p, int xd, int yd) {
    if (p.mode == 0) return gray15(p.src + static_cast<std::size_t>(yd) * p.src_pitch + 3 * xd);
    if (p.mode == 1) {
        const std::uint8_t* r0 = p.src + static_cast<std::size_t>(2 * yd) * p.src_pitch + 6 * xd;
        const std::uint8_t* r1 = r0 + p.src_pitch;
        return (gray15(r0) + gray15(r0 + 3) + gray15(r1) + gray15(r1 + 3) + 2) >> 2;
    }
    if (p.mode == 2) {
        int sum = 0;
#pragma unroll
        for (int dy = 0; dy < 4; ++dy) {
            const std::uint8_t* r = p.src + static_cast<std::size_t>(4 * yd + dy) * p.src_pitch + 12 * xd;
#pragma unroll
            for (int dx = 0; dx < 4; ++dx) sum += gray15(r + 3 * dx);
        }
        return __float2int_rn(__fmul_rn(static_cast<float>(sum), 0.0625f));
    }
    const float fsy1 = __fmul_rn(static_cast<float>(yd), p.inv_sy);
    const float fsy2 = __fmul_rn(static_cast<float>(yd + 1), p.inv_sy);
    const float fsx1 = __fmul_rn(static_cast<float>(xd), p.inv_sx);
    const float fsx2 = __fmul_rn(static_cast<float>(xd + 1), p.inv_sx);
    const int y_start = static_cast<int>(floorf(fsy1)), y_end = static_cast<int>(ceilf(fsy2));
    const int x_start = static_cast<int>(floorf(fsx1)), x_end = static_cast<int>(ceilf(fsx2));
    float total = 0.0f;
    for (int ys = y_start; ys < y_end && ys < p.orig_h; ++ys) {
        const float wy = fmaxf(0.0f, __fsub_rn(fminf(static_cast<float>(ys + 1), fsy2),
                                               fmaxf(static_cast<float>(ys), fsy1)));
        if (wy <= 0.0f) continue;
        const std::uint8_t* row = p.src + static_cast<std::size_t>(ys) * p.src_pitch;
        for (int xs = x_start; xs < x_end && xs < p.orig_w; ++xs) {
            const float wx = fmaxf(0.0f, __fsub_rn(fminf(static_cast<float>(xs + 1), fsx2),
                                                   fmaxf(static_cast<float>(xs), fsx1)));
            if (wx <= 0.0f) continue;
            total = __fmaf_rn(static_cast<float>(gray15(row + 3 * xs)), __fmul_rn(wx, wy), total);
        }
    }
    return __float2int_rn(__fmul_rn(total, p.scale_area));
}

constexpr int kS1BlockX = 16, kS1BlockY = 16;  // 16 x 4-output columns x 16 rows per block

__global__ __launch_bounds__(kS1BlockX * kS1BlockY) void s1_kernel(const __grid_constant__ Pair pair) {
    const Params& p = pair.img[blockIdx.z];
    const int x = 4 * (blockIdx.x * kS1BlockX + threadIdx.x);
    const int y = blockIdx.y * kS1BlockY + threadIdx.y;
    if (y >= p.work_h || x >= p.work_w) return;
    std::uint8_t* dst = p.dst + static_cast<std::size_t>(y) * p.dst_pitch + x;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (x + k < p.work_w) dst[k] = static_cast<std::uint8_t>(s1_pixel(p, x + k, y));
}

// Batched form: one launch over the images of many requests; each block
// finds its (image, 64x16 output tile) through a device job table.
template <class Src>
__global__ __launch_bounds__(256) void s1_batch_kernel(const __grid_constant__ Src src) {
    BatchJob j;
    int local;
    if (!src.find(blockIdx.x, 0, &j, &local)) return;
    const Params& p = j.p;
    const int x = (local % j.tiles_x) * kBatchTileW + 4 * (threadIdx.x & 15);
    const int y = (local / j.tiles_x) * kBatchTileH + (threadIdx.x >> 4);
    if (y >= p.work_h || x >= p.work_w) return;
    std::uint8_t* dst = p.dst + static_cast<std::size_t>(y) * p.dst_pitch + x;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (x + k < p.work_w) dst[k] = static_cast<std::uint8_t>(s1_pixel(p, x + k, y));
}

Status batch_job(const ImageView& in, const ImageView& out, const ScaleInfo& si, BatchJob* j);

Status batch_enqueue(const BatchJob* device_jobs, const int* device_prefix, int n, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return Status::OK;
    using Src = s2s3::JobTable<BatchJob>;
    s1_batch_kernel<Src><<<blocks, 256, 0, stream>>>(Src{device_jobs, device_prefix, n});
    note_launches(1);
    return launch_status();
}

// Sum of |I(x+1, y) - I(x, y)| and |I(x, y+1) - I(x, y)| per image into
// acc[blockIdx.z] (unsigned 64-bit, order-free).
struct GradPair {
    const std::uint8_t* src[2];
    int pitch[2], width[2], height[2];
    unsigned long long* acc;
    double* out;
};

__global__ __launch_bounds__(256) void gradient_kernel(const __grid_constant__ GradPair g) {
    __shared__ unsigned long long block_sum;
    const int z = blockIdx.z;
    const int w = g.width[z], h = g.height[z];
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    if (threadIdx.x == 0 && threadIdx.y == 0) block_sum = 0;
    __syncthreads();
    unsigned d = 0;
    if (x < w && y < h) {
        const std::uint8_t* row = g.src[z] + static_cast<std::size_t>(y) * g.pitch[z];
        const int c = row[x];
        if (x + 1 < w) d += static_cast<unsigned>(abs(static_cast<int>(row[x + 1]) - c));
        if (y + 1 < h) d += static_cast<unsigned>(abs(static_cast<int>(row[x + g.pitch[z]]) - c));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if (threadIdx.x == 0 && d) atomicAdd(&block_sum, static_cast<unsigned long long>(d));
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0 && block_sum) atomicAdd(&g.acc[z], block_sum);
}

__global__ void gradient_normalize_kernel(const __grid_constant__ GradPair g, int images) {
    const int z = threadIdx.x;
    if (z >= images) return;
    const unsigned long long edges = static_cast<unsigned long long>(g.height[z]) * (g.width[z] - 1) +
                                     static_cast<unsigned long long>(g.width[z]) * (g.height[z] - 1);
    g.out[z] = edges == 0 ? 0.0 : static_cast<double>(g.acc[z]) / (255.0 * static_cast<double>(edges));
}

namespace {

int mode_of(int ow, int oh, int ww, int wh) {
    if (ow == ww && oh == wh) return 0;
    if (ow == 2 * ww && oh == 2 * wh) return 1;
    if (ow == 4 * ww && oh == 4 * wh) return 2;
    return 3;
}

Status fill(const ImageView& in, const ImageView& out, const ScaleInfo& si, Params* p) {
    if (!in.data || !out.data || in.format != PixelFormat::RGB8 || out.format != PixelFormat::GRAY8 ||
        in.width <= 0 || in.height <= 0 || out.width != si.work_w || out.height != si.work_h ||
        in.pitch_bytes < in.width * 3 || out.pitch_bytes < out.width)
        return Status::INVALID_ARGUMENT;
    p->src = in.data;
    p->src_pitch = in.pitch_bytes;
    p->orig_w = in.width;
    p->orig_h = in.height;
    p->dst = out.data;
    p->dst_pitch = out.pitch_bytes;
    p->work_w = out.width;
    p->work_h = out.height;
    p->inv_sx = static_cast<float>(in.width) / static_cast<float>(out.width);
    p->inv_sy = static_cast<float>(in.height) / static_cast<float>(out.height);
    p->scale_area = 1.0f / (p->inv_sx * p->inv_sy);
    p->mode = mode_of(in.width, in.height, out.width, out.height);
    return Status::OK;
}

Status scale_info(int w, int h, double s, ScaleInfo* out) {
    return static_cast<Status>(stitch_make_scale_info(w, h, s, reinterpret_cast<stitch_scale_info*>(out)));
}

Status launch(const Pair& pair, int images, cudaStream_t stream) {
    int mw = pair.img[0].work_w, mh = pair.img[0].work_h;
    if (images == 2) {
        mw = mw > pair.img[1].work_w ? mw : pair.img[1].work_w;
        mh = mh > pair.img[1].work_h ? mh : pair.img[1].work_h;
    }
    const dim3 block(kS1BlockX, kS1BlockY);
    const dim3 grid(ceil_div(ceil_div(mw, 4), kS1BlockX), ceil_div(mh, kS1BlockY), images);
    s1_kernel<<<grid, block, 0, stream>>>(pair);
    note_launches(1);
    return launch_status();
}

bool valid_gray(const ImageView& g) {
    return g.data && g.format == PixelFormat::GRAY8 && g.width >= 2 && g.height >= 2 && g.pitch_bytes >= g.width;
}

Status gradient(const ImageView* imgs, int n, void* ws, double* const* pinned, cudaStream_t stream) {
    GradPair g{};
    int mw = 0, mh = 0;
    for (int z = 0; z < n; ++z) {
        g.src[z] = imgs[z].data;
        g.pitch[z] = imgs[z].pitch_bytes;
        g.width[z] = imgs[z].width;
        g.height[z] = imgs[z].height;
        mw = mw > imgs[z].width ? mw : imgs[z].width;
        mh = mh > imgs[z].height ? mh : imgs[z].height;
    }
    g.acc = static_cast<unsigned long long*>(ws);
    g.out = reinterpret_cast<double*>(static_cast<unsigned char*>(ws) + 16);
    if (cudaMemsetAsync(ws, 0, 16, stream) != cudaSuccess) return Status::CUDA_ERROR;
    gradient_kernel<<<dim3(ceil_div(mw, 32), ceil_div(mh, 8), n), dim3(32, 8), 0, stream>>>(g);
    gradient_normalize_kernel<<<1, 32, 0, stream>>>(g, n);
    note_launches(2);
    for (int z = 0; z < n; ++z)
        if (cudaMemcpyAsync(pinned[z], g.out + z, sizeof(double), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
            return Status::CUDA_ERROR;
    return launch_status();
}

}  // namespace

Status batch_job(const ImageView& in, const ImageView& out, const ScaleInfo& si, BatchJob* j) {
    const Status s = fill(in, out, si, &j->p);
    if (s != Status::OK) return s;
    j->tiles_x = ceil_div(out.width, kBatchTileW);
    j->tiles = j->tiles_x * ceil_div(out.height, kBatchTileH);
    return Status::OK;
}

}  // namespace stitch::b200::s1k

namespace stitch::s1 {

using namespace b200::s1k;

Status s1_preprocess_single(const ImageView& in, double scale, ImageView* out, ScaleInfo* scale_info_out,
                            cudaStream_t stream) {
    if (!out || !scale_info_out || !(scale > 0.0) || scale > 1.0) return Status::INVALID_ARGUMENT;
    Status s = scale_info(in.width, in.height, scale, scale_info_out);
    if (s != Status::OK) return s;
    Pair pair{};
    s = fill(in, *out, *scale_info_out, &pair.img[0]);
    if (s != Status::OK) return s;
    return launch(pair, 1, stream);
}

Status s1_preprocess(const ImageView& img_a, const ImageView& img_b, double scale, ImageView* out_a,
                     ImageView* out_b, ScaleInfo* scale_a, ScaleInfo* scale_b, cudaStream_t stream) {
    if (!out_a || !out_b || !scale_a || !scale_b || !(scale > 0.0) || scale > 1.0) return Status::INVALID_ARGUMENT;
    Status s = scale_info(img_a.width, img_a.height, scale, scale_a);
    if (s != Status::OK) return s;
    s = scale_info(img_b.width, img_b.height, scale, scale_b);
    if (s != Status::OK) return s;
    Pair pair{};
    s = fill(img_a, *out_a, *scale_a, &pair.img[0]);
    if (s != Status::OK) return s;
    s = fill(img_b, *out_b, *scale_b, &pair.img[1]);
    if (s != Status::OK) return s;
    return launch(pair, 2, stream);
}

Status s1_compute_gradient(const ImageView& gray_a, const ImageView& gray_b, void* d_workspace,
                           double* pinned_gradient_a, double* pinned_gradient_b, cudaStream_t stream) {
    if (!valid_gray(gray_a) || !valid_gray(gray_b) || !d_workspace || !pinned_gradient_a || !pinned_gradient_b)
        return Status::INVALID_ARGUMENT;
    const ImageView imgs[2] = {gray_a, gray_b};
    double* const pinned[2] = {pinned_gradient_a, pinned_gradient_b};
    return gradient(imgs, 2, d_workspace, pinned, stream);
}

Status s1_compute_gradient_single(const ImageView& gray, void* d_workspace, double* pinned_gradient,
                                  cudaStream_t stream) {
    if (!valid_gray(gray) || !d_workspace || !pinned_gradient) return Status::INVALID_ARGUMENT;
    double* const pinned[1] = {pinned_gradient};
    return gradient(&gray, 1, d_workspace, pinned, stream);
}

}  // namespace stitch::s1

extern "C" {

int stitch_s1_preprocess(const stitch_image_view* img_a, const stitch_image_view* img_b, double scale,
                         stitch_image_view* out_a, stitch_image_view* out_b, stitch_scale_info* scale_a,
                         stitch_scale_info* scale_b, void* stream) {
    using namespace stitch;
    if (!img_a || !img_b) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(s1::s1_preprocess(
        *reinterpret_cast<const ImageView*>(img_a), *reinterpret_cast<const ImageView*>(img_b), scale,
        reinterpret_cast<ImageView*>(out_a), reinterpret_cast<ImageView*>(out_b), reinterpret_cast<ScaleInfo*>(scale_a),
        reinterpret_cast<ScaleInfo*>(scale_b), static_cast<cudaStream_t>(stream)));
}

int stitch_s1_preprocess_single(const stitch_image_view* img, double scale, stitch_image_view* out,
                                stitch_scale_info* scale_info, void* stream) {
    using namespace stitch;
    if (!img) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(s1::s1_preprocess_single(*reinterpret_cast<const ImageView*>(img), scale,
                                                      reinterpret_cast<ImageView*>(out),
                                                      reinterpret_cast<ScaleInfo*>(scale_info),
                                                      static_cast<cudaStream_t>(stream)));
}

int stitch_s1_compute_gradient(const stitch_image_view* gray_a, const stitch_image_view* gray_b, void* workspace,
                               double* pinned_a, double* pinned_b, void* stream) {
    using namespace stitch;
    if (!gray_a || !gray_b) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(s1::s1_compute_gradient(*reinterpret_cast<const ImageView*>(gray_a),
                                                    *reinterpret_cast<const ImageView*>(gray_b), workspace, pinned_a,
                                                    pinned_b, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
