// Host side of S5: argument checks, workspace size and launches.
//
// Checks and their order follow src/s5/s5.cu:214-246 and
// src/s5/s5_config.cpp:8-19. The workspace holds the persistent search state
// (offset 0) and one best model per search block; its size depends on
// neither R nor the match count, so one allocation serves every extension.
// Compile with -fmad=false (see s5_kernels.cuh).
#include <algorithm>
#include <cmath>
#include <limits>

#include "s5_internal.hpp"

namespace stitch::b200::s5k {

std::size_t state_bytes() { return (sizeof(State) + kWorkspaceAlign - 1) / kWorkspaceAlign * kWorkspaceAlign; }

std::size_t estimate_workspace_bytes() { return state_bytes() + kMaxSearchBlocks * sizeof(Model); }

bool host_mat3_inverse(const double* m, double* out) {
    const double c00 = m[4] * m[8] - m[5] * m[7];
    const double c01 = m[5] * m[6] - m[3] * m[8];
    const double c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (std::fabs(det) < 1e-300) return false;
    const double inv = 1.0 / det;
    const double r[9] = {c00 * inv, (m[2] * m[7] - m[1] * m[8]) * inv, (m[1] * m[5] - m[2] * m[4]) * inv,
                         c01 * inv, (m[0] * m[8] - m[2] * m[6]) * inv, (m[2] * m[3] - m[0] * m[5]) * inv,
                         c02 * inv, (m[1] * m[6] - m[0] * m[7]) * inv, (m[0] * m[4] - m[1] * m[3]) * inv};
    std::copy(r, r + 9, out);
    return true;
}

bool valid_config(const ::stitch::s5::Config& c) {
    return c.hypotheses > 0 && c.previous_hypotheses >= 0 && c.previous_hypotheses <= c.hypotheses &&
           c.batch_size > 0 && c.batch_size <= 65535 && c.refinement_steps >= 0 && std::isfinite(c.threshold) &&
           c.threshold > 0.0 && std::isfinite(c.threshold * c.threshold);
}

bool valid_keypoints(const Keypoints& p) {
    return p.capacity >= 0 && p.d_count && (p.capacity == 0 || (p.x && p.y));
}

bool valid_scale(const ScaleInfo& s) {
    if (s.orig_w <= 0 || s.orig_h <= 0 || s.work_w <= 0 || s.work_h <= 0 || !(s.sx > 0.0) || !(s.sy > 0.0) ||
        !std::isfinite(s.sx) || !std::isfinite(s.sy))
        return false;
    for (double x : s.D)
        if (!std::isfinite(x)) return false;
    return true;
}

Status check_and_build(const Keypoints& a, const Keypoints& b, const Matches& m, const ScaleInfo& sa,
                       const ScaleInfo& sb, const ::stitch::s5::Config& c, std::uint8_t* mask,
                       const void* output, void* ws, std::size_t bytes, PairIO* io) {
    if (!valid_config(c)) return Status::INVALID_ARGUMENT;
    if (!valid_keypoints(a) || !valid_keypoints(b) || m.capacity < 0 || !m.d_count ||
        (m.capacity > 0 && (!m.idx_a || !m.idx_b || !mask)) || !output || !valid_scale(sa) || !valid_scale(sb))
        return Status::INVALID_ARGUMENT;
    if (bytes < estimate_workspace_bytes()) return Status::INSUFFICIENT_WORKSPACE;
    if (!ws || !aligned(ws, kWorkspaceAlign)) return Status::INVALID_ARGUMENT;
    PairIO j{};
    double inverse_b[9];
    if (!host_mat3_inverse(sa.D, j.inverse_a) || !host_mat3_inverse(sb.D, inverse_b))
        return Status::INVALID_ARGUMENT;
    for (int i = 0; i < 9; ++i) {
        if (!std::isfinite(j.inverse_a[i]) || !std::isfinite(inverse_b[i])) return Status::INVALID_ARGUMENT;
        j.d_b[i] = sb.D[i];
    }
    j.a = a;
    j.b = b;
    j.m = m;
    j.sa = sa;
    j.sb = sb;
    j.c = c;
    j.state = static_cast<State*>(ws);
    j.block_best = at_offset<Model>(ws, state_bytes());
    j.mask = mask;
    *io = j;
    return Status::OK;
}

int plan_search(int count, int hpw) {
    if (count <= 0) return 0;
    const int rounds = ceil_div(count, hpw);
    return std::min(kMaxSearchBlocks, ceil_div(rounds, kSearchWarps));
}

int search_smem_bytes(int match_capacity) {
    return std::min(std::max(match_capacity, 1), kStagePoints) * static_cast<int>(sizeof(float4));
}

bool enable_search_smem_once(const void* fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kStagePoints * static_cast<int>(sizeof(float4))) == cudaSuccess;
}

}  // namespace stitch::b200::s5k

namespace stitch::s5 {

using namespace ::stitch::b200;
using namespace ::stitch::b200::s5k;

Status s5_workspace_bytes(const Config& c, std::size_t* bytes) {
    if (!bytes || !valid_config(c)) return Status::INVALID_ARGUMENT;
    *bytes = estimate_workspace_bytes();
    return Status::OK;
}

Status estimate(const Keypoints& a, const Keypoints& b, const Matches& matches, const ScaleInfo& scale_a,
                const ScaleInfo& scale_b, const Config& config, std::uint8_t* inlier_mask,
                HomographyResult* output, void* workspace, std::size_t workspace_bytes, cudaStream_t stream) {
    PairIO io;
    const Status chk = check_and_build(a, b, matches, scale_a, scale_b, config, inlier_mask, output, workspace,
                                       workspace_bytes, &io);
    if (chk != Status::OK) return chk;
    constexpr int kHpw = 8;
    const int count = config.hypotheses - config.previous_hypotheses;
    io.hpw = kHpw;
    io.search_blocks = plan_search(count, kHpw);
    prepare_kernel<OneJob<PairIO>><<<1, 256, 0, stream>>>(OneJob<PairIO>{io});
    note_launches(1);
    if (cudaGetLastError() != cudaSuccess) return Status::CUDA_ERROR;
    if (io.search_blocks > 0) {
        using Src = OneJob<SearchJob>;
        static const bool smem_ok =
            enable_search_smem_once(reinterpret_cast<const void*>(search_kernel<Src, false>));
        (void)smem_ok;
        SearchJob sj{io, config.previous_hypotheses, count, nullptr};
        search_kernel<Src, false>
            <<<io.search_blocks, kSearchThreads, search_smem_bytes(matches.capacity), stream>>>(Src{sj});
        note_launches(1);
        if (cudaGetLastError() != cudaSuccess) return Status::CUDA_ERROR;
    }
    finish_kernel<OneJob<PairIO>><<<1, kFinishThreads, 0, stream>>>(OneJob<PairIO>{io});
    note_launches(1);
    if (cudaGetLastError() != cudaSuccess) return Status::CUDA_ERROR;
    if (cudaMemcpyAsync(output, &io.state->result, sizeof(*output), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return Status::CUDA_ERROR;
    return Status::OK;
}

}  // namespace stitch::s5
