// S5 helpers shared by the per-pair call and the batched chain.
#pragma once

#include "s5_kernels.cuh"

namespace stitch::b200::s5k {

std::size_t state_bytes();
std::size_t estimate_workspace_bytes();
bool host_mat3_inverse(const double* m, double* out);
bool valid_config(const ::stitch::s5::Config& c);
// Argument checks of one pair in the reference's order; fills *io.
Status check_and_build(const Keypoints& a, const Keypoints& b, const Matches& m, const ScaleInfo& sa,
                       const ScaleInfo& sb, const ::stitch::s5::Config& c, std::uint8_t* mask,
                       const void* output, void* ws, std::size_t bytes, PairIO* io);
// Search blocks for `count` hypotheses at `hpw` hypotheses per warp round.
int plan_search(int count, int hpw);
int search_smem_bytes(int match_capacity);
bool enable_search_smem_once(const void* fn);

}  // namespace stitch::b200::s5k
