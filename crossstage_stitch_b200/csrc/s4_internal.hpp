// S4 layout and job builders shared by the per-pair call and the batched chain.
#pragma once

#include <mutex>

#include "s4_kernels.cuh"

namespace stitch::b200::s4k {

struct MatchLayout {
    std::size_t forward, reverse, fpartial, rpartial, accept_counts, total;  // accept_counts: int per 1024 queries
    int fq_tiles, fsplits, frows;  // forward direction plan
    int rq_tiles, rsplits, rrows;  // reverse direction plan
};

bool valid_side(const Keypoints& k, const Descriptors& d);
bool valid_pair(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db);
bool popc_eligible(const Descriptors& q, const Descriptors& t, int capacity_train);

// Binary matcher of an S4 launch: kMatcherPopc (the __popc tile kernel) or
// kMatcherTensor (tcgen05 kind::i8). Results are identical; the choice only
// changes speed. The stage calls use the calling host thread's choice
// (stitch_s4_set_matcher), so threads never race on it; a batch plan and a
// server take the creating thread's choice when they are made, and a plan can
// be given its own (stitch_batch_set_matcher).
constexpr int kMatcherPopc = 0, kMatcherTensor = 1, kMatcherTensor128 = 2, kMatcherTensor64 = 3,
              kMatcherTensorPipe = 4;
// Train rows per tensor-core stage of a tensor-core matcher kind.
constexpr int tc_rows(int kind) { return kind == kMatcherTensor64 ? 64 : kind == kMatcherTensor128 ? 128 : 256; }
constexpr bool is_tensor(int kind) { return kind != kMatcherPopc; }
int matcher();
bool valid_matcher(int kind);
// Host-only argument checks of s4_match, in its order: INVALID_ARGUMENT or
// OK, with *required the workspace bytes the call needs.
Status check_match_args(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db,
                        const s4::Config& config, const Matches& output, std::size_t* required);
// Opts the tensor-core kernel for a job source in to its shared memory
// (once per device); false if the device refuses.
template <class Src, int kRowsB> bool enable_tc_smem() {
    static std::once_flag flags[64];
    static bool ok[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    std::call_once(flags[dev], [&] {
        ok[dev] = cudaFuncSetAttribute(knn_tc_kernel<Src, kRowsB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TcShape<kRowsB>::smem) == cudaSuccess;
    });
    return ok[dev];
}
// Launches the tensor-core matcher of `kind` over `blocks` blocks.
template <class Src> bool enable_pipe_smem() {
    static std::once_flag flags[64];
    static bool ok[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    std::call_once(flags[dev], [&] {
        ok[dev] = cudaFuncSetAttribute(knn_tc_pipe_kernel<Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kPipeSmem) == cudaSuccess;
    });
    return ok[dev];
}
template <class Src> bool launch_tc(int kind, int blocks, const Src& src, cudaStream_t s) {
    if (kind == kMatcherTensorPipe) {
        if (!enable_pipe_smem<Src>()) return false;
        knn_tc_pipe_kernel<Src><<<blocks, kPipeThreads, kPipeSmem, s>>>(src);
        return true;
    }
    switch (tc_rows(kind)) {
        case 64:
            if (!enable_tc_smem<Src, 64>()) return false;
            knn_tc_kernel<Src, 64><<<blocks, kQueryThreads, TcShape<64>::smem, s>>>(src);
            return true;
        case 128:
            if (!enable_tc_smem<Src, 128>()) return false;
            knn_tc_kernel<Src, 128><<<blocks, kQueryThreads, TcShape<128>::smem, s>>>(src);
            return true;
        default:
            if (!enable_tc_smem<Src, 256>()) return false;
            knn_tc_kernel<Src, 256><<<blocks, kQueryThreads, TcShape<256>::smem, s>>>(src);
            return true;
    }
}
constexpr int tc_blocks_per_sm(int kind) {
    return kind == kMatcherTensorPipe ? 1
         : tc_rows(kind) == 64 ? TcShape<64>::blocks_per_sm
                               : tc_rows(kind) == 128 ? TcShape<128>::blocks_per_sm : TcShape<256>::blocks_per_sm;
}
// Reads and clears the tensor-core error word of the batched chain's
// translation unit (batch.cu).
int take_batch_tc_error();
void plan_split(int capacity_q, int capacity_t, int* q_tiles, int* splits, int* rows_per_split);
bool match_layout(int capacity_a, int capacity_b, bool cross, MatchLayout* out);
KnnJob make_knn_job(const Keypoints& qk, const Descriptors& qd, const Keypoints& tk, const Descriptors& td,
                    int q_tiles, int splits, int rows, uint2* partial, Top2* top2);

}  // namespace stitch::b200::s4k
