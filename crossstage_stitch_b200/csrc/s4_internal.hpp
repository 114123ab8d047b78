// S4 layout and job builders shared by the per-pair call and the batched chain.
#pragma once

#include "s4_kernels.cuh"

namespace stitch::b200::s4k {

struct MatchLayout {
    std::size_t forward, reverse, fpartial, rpartial, total;
    int fq_tiles, fsplits, frows;  // forward direction plan
    int rq_tiles, rsplits, rrows;  // reverse direction plan
};

bool valid_side(const Keypoints& k, const Descriptors& d);
bool valid_pair(const Keypoints& a, const Descriptors& da, const Keypoints& b, const Descriptors& db);
bool popc_eligible(const Descriptors& q, const Descriptors& t, int capacity_train);
void plan_split(int capacity_q, int capacity_t, int* q_tiles, int* splits, int* rows_per_split);
bool match_layout(int capacity_a, int capacity_b, bool cross, MatchLayout* out);
KnnJob make_knn_job(const Keypoints& qk, const Descriptors& qd, const Keypoints& tk, const Descriptors& td,
                    int q_tiles, int splits, int rows, uint2* partial, Top2* top2);

}  // namespace stitch::b200::s4k
