// Batched registration: one launch per stage kernel covers every pair.
#pragma once

#include <cstddef>
#include <vector>

#include "s2s3_internal.hpp"
#include "s4_internal.hpp"
#include "s5_internal.hpp"
#include "stitch_b200.h"

namespace stitch::b200::batch {

// Device outputs of one pair inside the batch workspace (offsets).
struct PairOffsets {
    std::size_t kx[2], ky[2], kr[2], kcount[2], desc[2];
    std::size_t s2ws[2], s3ws[2];
    std::size_t ia, ib, dist, mcount, mask, s4ws, s5ws;
    s2s3::DetectLayout det[2];
    s2s3::DescribeLayout des[2];
    s4k::MatchLayout match;
};

class Plan {
public:
    int n = 0;
    std::vector<stitch_pair_desc> pairs;
    std::vector<PairOffsets> off;
    std::size_t results = 0;      // HomographyResult[n]
    std::size_t tables = 0;       // job tables + prefixes (device copy of `staging`)
    std::size_t table_bytes = 0;
    std::size_t total = 0;
    // launch shapes
    int det_blocks[s2s3::kDetectKinds] = {};
    int des_blocks[s2s3::kDescribeKinds] = {};
    int knn_blocks = 0, merge_blocks = 0, n_knn = 0;
    int search_blocks = 0;
    int sort_smem = 0, search_smem = 0;
    bool rank_fallback = false;
    int hpw = 8;
    // host staging of the tables (pinned), filled for one workspace address
    unsigned char* staging = nullptr;
    const void* staged_for = nullptr;
    // captured graph
    void* graph = nullptr;       // cudaGraph_t
    void* graph_exec = nullptr;  // cudaGraphExec_t
    std::size_t offsets[16] = {};  // table offsets inside the table block
    cudaEvent_t marks[STITCH_BATCH_MARKS] = {};
    bool marked = false;

    ~Plan();
    // Histograms follow the counts region (int[3n]) at the workspace start.
    std::size_t hists_offset() const {
        Layout lay;
        lay.take(3 * static_cast<std::size_t>(n), sizeof(int));
        return lay.take(2 * static_cast<std::size_t>(n) * 256, sizeof(std::uint32_t));
    }
    Status build(int n_pairs, const stitch_pair_desc* p, int* bad_pair);
    Status stage_tables(void* ws);
    Status enqueue(void* ws, std::size_t bytes, stitch_homography_result* host_results, cudaStream_t s);
};

}  // namespace stitch::b200::batch
