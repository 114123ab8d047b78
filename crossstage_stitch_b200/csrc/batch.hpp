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
    std::size_t models;  // S5 models of the pair's hypotheses (fit_kernel -> search_kernel)
    s2s3::DetectLayout det[2];
    s2s3::DescribeLayout des[2];
    s4k::MatchLayout match;
    // scale pyramid (levels > 1): layer workspace, first layer count and
    // first detect job of each image
    bool pyramid[2];
    s2s3::PyramidLayout pyr[2];
    std::size_t pyrws[2];
    int layer0[2], job0[2];
    std::size_t mark0[2];  // first blur-tile flag of each image (all its layers)
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
    int n_det = 0;     // detect/describe jobs: one per image, one per layer of a pyramid image
    int n_layers = 0;  // layer counts kept after the 3n image and match counts
    int n_resize = 0;  // resize jobs (layers 1.. of every pyramid image)
    int max_levels = 1;
    // zeroed head of the workspace: counts, then FAST histograms and counters
    // u32[n_det][kHistWords], the FAST tile queue and blur-list count (2
    // words), the blur-tile flags u32[blur_total]; `zeroed` bytes in all.
    // The blur list uint2[blur_total] follows the head.
    std::size_t hists = 0, queue = 0, blur_flags = 0, zeroed = 0, blur_list = 0;
    std::size_t blur_total = 0;
    int det_blocks[s2s3::kDetectKinds] = {};
    int des_blocks[s2s3::kDescribeKinds] = {};
    int rs_blocks[s2s3::kMaxLevels] = {};  // resize launch of layer kind + 1
    int knn_blocks = 0, merge_blocks = 0, n_knn = 0;
    int search_blocks = 0, fit_blocks = 0;
    int sort_smem = 0, search_smem = 0;
    bool rank_fallback = false;
    int hpw = 8;
    // binary matcher of this plan's S4 launches (s4k::kMatcherPopc or
    // kMatcherTensor): the building thread's choice, or stitch_batch_set_matcher's
    int matcher = s4k::kMatcherTensor;
    stitch_batch_tuning tuning{};  // launch shapes (0: default)
    // host staging of the tables (pinned), filled for one workspace address;
    // either allocated by build() or lent by the caller (use_staging)
    unsigned char* staging = nullptr;
    bool owns_staging = false;
    const void* staged_for = nullptr;
    // captured graph, and the device copy of the tables its replays read
    void* graph = nullptr;       // cudaGraph_t
    void* graph_exec = nullptr;  // cudaGraphExec_t
    unsigned char* graph_tables = nullptr;
    std::size_t offsets[20] = {};  // table offsets inside the table block
    // block -> job maps of the detect, describe and resize kinds (one table,
    // kinds one after the other; see s2s3::JobTable), when every job index
    // and block within a job fits 16 bits and the plan owns its staging
    bool block_map = false;
    int det_total[s2s3::kDetectKinds] = {}, des_total[s2s3::kDescribeKinds] = {}, rs_total[s2s3::kMaxLevels] = {};
    std::size_t det_first[s2s3::kDetectKinds] = {}, des_first[s2s3::kDescribeKinds] = {},
                rs_first[s2s3::kMaxLevels] = {};  // entry index of each kind's map
    // and of the S4/S5 launches: knn, knn merge, accept, pair (prepare and
    // finish), search, fit
    enum { kMapKnn, kMapMerge, kMapAccept, kMapPair, kMapSearch, kMapFit, kMapS45 };
    int s45_total[kMapS45] = {};
    std::size_t s45_first[kMapS45] = {};
    cudaEvent_t marks[STITCH_BATCH_MARKS] = {};
    bool marked = false;

    ~Plan();
    int resize_kinds() const { return max_levels > 1 ? max_levels - 1 : 1; }
    // Validates the pairs and lays out the workspace (host work only), then,
    // with alloc_staging, allocates the pinned staging of the job tables.
    // Every count, total, offset and block-map total it derives is reset and
    // recomputed, so calling it again on the same plan gives the layout of a
    // fresh plan (tests/test_plan_rebuild.py builds one plan twice and
    // compares).
    Status build(int n_pairs, const stitch_pair_desc* p, int* bad_pair, bool alloc_staging = true);
    // Lends a pinned buffer of at least table_bytes as the staging.
    void use_staging(unsigned char* buf) {
        staging = buf;
        owns_staging = false;
        staged_for = nullptr;
    }
    Status stage_tables(void* ws);
    // S4 train split of one matching direction of pair i.
    struct KnnShape {
        int splits, rows, blocks, merge_blocks;
    };
    int knn_want_splits() const;
    KnnShape knn_shape(int i, int dir, int want_splits) const;
    // Blocks of the detect and describe kinds of job (pair i, side s, layer l).
    void job_blocks(int i, int s, int l, int (&db)[s2s3::kDetectKinds], int (&sb)[s2s3::kDescribeKinds]) const;
    // With device_tables (graph capture), the kernels read the job tables
    // there, already uploaded for `ws`, instead of uploading them into `ws`.
    Status enqueue(void* ws, std::size_t bytes, stitch_homography_result* host_results, cudaStream_t s,
                   const unsigned char* device_tables = nullptr);
};

}  // namespace stitch::b200::batch
