// Batched registration of N uneven pairs: every stage kernel is launched once
// for the whole batch; each block finds its (pair, image, tile) through a
// device job table and a block-prefix array. The per-pair stage semantics
// are unchanged, so results equal the per-pair calls bit for bit.
//
// With a scale pyramid (levels > 1) an image contributes one detect and one
// describe job per layer and one resize job per layer above the first; the
// resize chain runs first, one launch per layer depth over all images.
//
// Workspace layout (one caller allocation, 256-byte aligned regions):
//   counts   int[3n + L]  keypoint counts (2 per pair), match counts and the
//                         L pyramid layer counts, zeroed every run
//   hists    u32[J][256]  FAST histograms of the J detect jobs, zeroed every run
//   results  HomographyResult[n]
//   tables   job tables + prefixes, copied from pinned host staging by every
//            enqueue (a captured graph reads its own device copy instead)
//   per pair: keypoints x/y/response, descriptors, S2 and S3 workspaces per
//             image (or its pyramid workspace), matches, inlier mask, S4 and
//             S5 workspaces
#include <algorithm>
#include <iterator>
#include <cstring>
#include <mutex>

#include "batch.hpp"

namespace stitch::b200::batch {

namespace {

using s2s3::DescribeJob;
using s2s3::DetectJob;
using s2s3::ResizeJob;
using s4k::AcceptJob;
using s4k::KnnJob;
using s5k::PairIO;
using s5k::SearchJob;

template <class T> T* at(void* base, std::size_t off) { return at_offset<T>(base, off); }

const ImageView& view(const stitch_image_view& v) { return *reinterpret_cast<const ImageView*>(&v); }

// Clears the counts and histograms at the start of the workspace. A kernel,
// not a memset: a graph replay then holds no copy-engine work before its
// first stage kernel, so it never queues behind an image upload running on
// another stream.
__global__ void zero_words_kernel(std::uint32_t* __restrict__ p, std::size_t words) {
    for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < words;
         i += static_cast<std::size_t>(gridDim.x) * blockDim.x)
        p[i] = 0;
}

bool small_image(const stitch_image_view& v) { return v.width <= 2 * s2::kEdge || v.height <= 2 * s2::kEdge; }

// Device job tables, in this order inside the table block.
enum Table {
    kDetJobs, kDetPrefix, kDesJobs, kDesPrefix, kKnnJobs, kKnnPrefix, kMergePrefix, kAccJobs, kAccPrefix,
    kPairJobs, kPairPrefix, kSearchJobs, kSearchPrefix, kFitPrefix, kRsJobs, kRsPrefix, kBlockMap, kTables
};

void set_attributes_once() {
    static std::once_flag flag;
    std::call_once(flag, [] {
        static_assert(kTables <= 20, "table offsets");
        cudaFuncSetAttribute(s2s3::sort_topk_kernel<s2s3::JobTable<DetectJob>>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             s2s3::kSortCap * static_cast<int>(sizeof(std::uint64_t)));
        s5k::enable_search_smem_once(
            reinterpret_cast<const void*>(s5k::search_kernel<s5k::JobTable<SearchJob>, true>));
    });
}

}  // namespace

Plan::~Plan() {
    if (graph_exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph_exec));
    if (graph_tables) cudaFree(graph_tables);
    if (graph) cudaGraphDestroy(static_cast<cudaGraph_t>(graph));
    if (staging && owns_staging) cudaFreeHost(staging);
}

Status Plan::build(int n_pairs, const stitch_pair_desc* p, int* bad_pair, bool alloc_staging) {
    if (n_pairs <= 0 || !p) return Status::INVALID_ARGUMENT;
    matcher = s4k::matcher();
    n = n_pairs;
    pairs.assign(p, p + n);
    off.assign(n, PairOffsets{});
    // 1. validate and fill identity scales
    for (int i = 0; i < n; ++i) {
        auto& q = pairs[i];
        const auto& c2 = *reinterpret_cast<const s2::Config*>(&q.s2);
        const auto& c4 = *reinterpret_cast<const s4::Config*>(&q.s4);
        const auto& c5 = *reinterpret_cast<const s5::Config*>(&q.s5);
        if (q.pyramid.levels == 0) q.pyramid.levels = 1;
        bool ok = s2s3::valid_gray(view(q.image_a)) && s2s3::valid_gray(view(q.image_b)) &&
                  s2s3::valid_detect_config(c2) && std::isfinite(c4.ratio_threshold) && c4.ratio_threshold > 0 &&
                  c4.ratio_threshold < 1 && s5k::valid_config(c5) && c5.previous_hypotheses == 0 &&
                  s2s3::valid_pyramid(q.pyramid.levels, q.pyramid.scale_factor);
        for (int s = 0; s < 2 && ok; ++s) {
            stitch_scale_info& si = s ? q.scale_b : q.scale_a;
            const stitch_image_view& im = s ? q.image_b : q.image_a;
            if (si.orig_w == 0) {
                stitch_make_scale_info(im.width, im.height, 1.0, &si);
            }
        }
        if (!ok) {
            if (bad_pair) *bad_pair = i;
            return Status::INVALID_ARGUMENT;
        }
    }
    // 2. jobs per image: one single-level job, or one per pyramid layer
    n_det = n_layers = n_resize = 0;
    max_levels = 1;
    for (int i = 0; i < n; ++i) {
        auto& o = off[i];
        const auto& q = pairs[i];
        for (int s = 0; s < 2; ++s) {
            const stitch_image_view& im = s ? q.image_b : q.image_a;
            o.pyramid[s] = q.pyramid.levels > 1;
            o.job0[s] = n_det;
            o.layer0[s] = n_layers;
            if (!o.pyramid[s]) {
                ++n_det;
                continue;
            }
            if (!s2s3::pyramid_layout(im.width, im.height, q.s2.max_keypoints, q.pyramid.levels,
                                      q.pyramid.scale_factor, &o.pyr[s],
                                      tuning.resize_tile_h ? tuning.resize_tile_h : s2s3::kResizeTileH)) {
                if (bad_pair) *bad_pair = i;
                return Status::INVALID_ARGUMENT;
            }
            const int L = o.pyr[s].plan.levels;
            n_det += L;
            n_layers += L;
            n_resize += L > 1 ? L - 1 : 0;
            max_levels = std::max(max_levels, L);
        }
    }
    // 3. layout: blur-tile flags per image first (they sit in the zeroed head)
    blur_total = 0;
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < 2; ++s) {
            auto& o = off[i];
            const stitch_image_view& im = s ? pairs[i].image_b : pairs[i].image_a;
            o.mark0[s] = blur_total;
            if (o.pyramid[s]) {
                blur_total += static_cast<std::size_t>(o.pyr[s].blur_first[o.pyr[s].plan.levels]);
            } else {
                blur_total += static_cast<std::size_t>(ceil_div(im.width, s2s3::kBlurTileW)) *
                              static_cast<std::size_t>(ceil_div(im.height, s2s3::kBlurTileH));
            }
        }
    Layout lay;
    const std::size_t counts = lay.take(3 * static_cast<std::size_t>(n) + n_layers, sizeof(int));
    hists = lay.take(static_cast<std::size_t>(std::max(n_det, 1)) * s2s3::kHistWords, sizeof(std::uint32_t));
    queue = lay.take(2, sizeof(std::uint32_t));
    blur_flags = lay.take(std::max<std::size_t>(blur_total, 1), sizeof(std::uint32_t));
    zeroed = lay.cursor;
    blur_list = lay.take(std::max<std::size_t>(blur_total, 1), sizeof(uint2));
    results = lay.take(n, sizeof(HomographyResult));
    for (int i = 0; i < n; ++i) {
        auto& o = off[i];
        const auto& q = pairs[i];
        const int k = q.s2.max_keypoints;
        const std::size_t kk = static_cast<std::size_t>(std::max(k, 1));
        for (int s = 0; s < 2; ++s) {
            const stitch_image_view& im = s ? q.image_b : q.image_a;
            o.kx[s] = lay.take(kk, sizeof(float));
            o.ky[s] = lay.take(kk, sizeof(float));
            o.kr[s] = lay.take(kk, sizeof(float));
            o.kcount[s] = counts + (2 * static_cast<std::size_t>(i) + s) * sizeof(int);
            o.desc[s] = lay.take(kk, 32);
            if (o.pyramid[s]) {
                o.pyrws[s] = lay.take(o.pyr[s].total, 1);
                continue;
            }
            if (!s2s3::detect_layout(im.width, im.height, k, &o.det[s]) ||
                !s2s3::describe_layout(im.width, im.height, &o.des[s], 16)) {
                if (bad_pair) *bad_pair = i;
                return Status::INVALID_ARGUMENT;
            }
            o.s2ws[s] = lay.take(o.det[s].total, 1);
            o.s3ws[s] = lay.take(o.des[s].total, 1);
        }
        o.ia = lay.take(kk, sizeof(std::int32_t));
        o.ib = lay.take(kk, sizeof(std::int32_t));
        o.dist = lay.take(kk, sizeof(float));
        o.mcount = counts + (2 * static_cast<std::size_t>(n) + i) * sizeof(int);
        o.mask = lay.take(kk, 1);
        s4k::match_layout(k, k, q.s4.cross_check != 0, &o.match);
        o.s4ws = lay.take(o.match.total, 1);
        o.s5ws = lay.take(s5k::estimate_workspace_bytes(), 1);
        o.models = lay.take(static_cast<std::size_t>(std::max(q.s5.hypotheses, 1)), sizeof(s5k::Model));
    }
    // 4. launch shapes (block counts are final once stage_tables has run)
    int max_cand = 0, max_cap_m = 1;
    for (int i = 0; i < n; ++i) {
        const auto& q = pairs[i];
        for (int s = 0; s < 2; ++s) {
            const stitch_image_view& im = s ? q.image_b : q.image_a;
            if (off[i].pyramid[s]) {
                for (int l = 0; l < off[i].pyr[s].plan.levels; ++l) {
                    int b[s2s3::kDetectKinds];
                    s2s3::pyramid_detect_blocks(off[i].pyr[s], l, b);
                    if (b[s2s3::kSortKind]) max_cand = std::max(max_cand, off[i].pyr[s].det[l].candidates);
                }
            } else if (q.s2.max_keypoints > 0 && !small_image(im)) {
                max_cand = std::max(max_cand, off[i].det[s].candidates);
            }
        }
        max_cap_m = std::max(max_cap_m, q.s2.max_keypoints);
    }
    sort_smem = s2s3::sort_smem_bytes(max_cand);
    rank_fallback = max_cand > s2s3::kSortCap;
    search_smem = s5k::search_smem_bytes(max_cap_m);
    // S4: one train partition per block unless the batch is too small to fill the GPU
    n_knn = 0;
    for (int i = 0; i < n; ++i) n_knn += pairs[i].s4.cross_check ? 2 : 1;
    const int want_splits = knn_want_splits();
    knn_blocks = merge_blocks = 0;
    // S5: hypotheses per warp round, as large as still fills about two waves
    long long rounds_at = 0;
    hpw = 32;
    for (int h : {32, 16, 8, 4}) {
        if (tuning.search_hpw && h != tuning.search_hpw) continue;
        hpw = h;
        rounds_at = 0;
        for (int i = 0; i < n; ++i) rounds_at += s5k::plan_search(pairs[i].s5.hypotheses, h);
        if (tuning.search_hpw || rounds_at >= 2 * kSmCount) break;
    }
    search_blocks = static_cast<int>(rounds_at);
    // block totals of every detect, describe and resize kind, for the block
    // -> job maps (the same per-job counts stage_tables lays out)
    std::fill(std::begin(det_total), std::end(det_total), 0);
    std::fill(std::begin(des_total), std::end(des_total), 0);
    std::fill(std::begin(rs_total), std::end(rs_total), 0);
    std::fill(std::begin(s45_total), std::end(s45_total), 0);
    bool map_fits = alloc_staging && n_det < (1 << 16) && n_resize < (1 << 16);
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < 2; ++s) {
            const int L = off[i].pyramid[s] ? off[i].pyr[s].plan.levels : 1;
            for (int l = 0; l < L; ++l) {
                int db[s2s3::kDetectKinds], sb[s2s3::kDescribeKinds];
                job_blocks(i, s, l, db, sb);
                for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) {
                    det_total[kind] += db[kind];
                    map_fits = map_fits && db[kind] < (1 << 16);
                }
                for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) {
                    des_total[kind] += sb[kind];
                    map_fits = map_fits && sb[kind] < (1 << 16);
                }
                if (l > 0) {
                    rs_total[l - 1] += off[i].pyr[s].resize_tiles[l];
                    map_fits = map_fits && off[i].pyr[s].resize_tiles[l] < (1 << 16);
                }
            }
        }
    std::size_t map_entries = 0;
    for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) {
        det_first[kind] = map_entries;
        map_entries += static_cast<std::size_t>(det_total[kind]);
    }
    for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) {
        des_first[kind] = map_entries;
        map_entries += static_cast<std::size_t>(des_total[kind]);
    }
    for (int kind = 0; kind < resize_kinds(); ++kind) {
        rs_first[kind] = map_entries;
        map_entries += static_cast<std::size_t>(rs_total[kind]);
    }
    map_fits = map_fits && n_knn < (1 << 16) && n < (1 << 16);
    for (int i = 0; i < n; ++i) {
        for (int dir = 0; dir < (pairs[i].s4.cross_check ? 2 : 1); ++dir) {
            const KnnShape ks = knn_shape(i, dir, want_splits);
            s45_total[kMapKnn] += ks.blocks;
            s45_total[kMapMerge] += ks.merge_blocks;
            map_fits = map_fits && ks.blocks < (1 << 16) && ks.merge_blocks < (1 << 16);
        }
        const int sb = s5k::plan_search(pairs[i].s5.hypotheses, hpw);
        const int fb = sb > 0 ? ceil_div(pairs[i].s5.hypotheses, s5k::kFitThreads) : 0;
        s45_total[kMapSearch] += sb;
        s45_total[kMapFit] += fb;
        map_fits = map_fits && sb < (1 << 16) && fb < (1 << 16);
    }
    s45_total[kMapAccept] = s45_total[kMapPair] = n;
    for (int m = 0; m < kMapS45; ++m) {
        s45_first[m] = map_entries;
        map_entries += static_cast<std::size_t>(s45_total[m]);
    }
    block_map = map_fits;
    // 5. table block layout
    std::size_t cur = 0;
    auto put = [&](int t, std::size_t bytes) {
        cur = (cur + 15) / 16 * 16;
        offsets[t] = cur;
        cur += bytes;
    };
    const std::size_t nd = static_cast<std::size_t>(n_det), nr = static_cast<std::size_t>(n_resize);
    put(kDetJobs, nd * sizeof(DetectJob));
    put(kDetPrefix, s2s3::kDetectKinds * (nd + 1) * sizeof(int));
    put(kDesJobs, nd * sizeof(DescribeJob));
    put(kDesPrefix, s2s3::kDescribeKinds * (nd + 1) * sizeof(int));
    put(kKnnJobs, n_knn * sizeof(KnnJob));
    put(kKnnPrefix, (n_knn + 1) * sizeof(int));
    put(kMergePrefix, (n_knn + 1) * sizeof(int));
    put(kAccJobs, n * sizeof(AcceptJob));
    put(kAccPrefix, (n + 1) * sizeof(int));
    put(kPairJobs, n * sizeof(PairIO));
    put(kPairPrefix, (n + 1) * sizeof(int));
    put(kSearchJobs, n * sizeof(SearchJob));
    put(kSearchPrefix, (n + 1) * sizeof(int));
    put(kFitPrefix, (n + 1) * sizeof(int));
    put(kRsJobs, nr * sizeof(ResizeJob));
    put(kRsPrefix, static_cast<std::size_t>(resize_kinds()) * (nr + 1) * sizeof(int));
    put(kBlockMap, block_map ? map_entries * sizeof(std::uint32_t) : 0);
    table_bytes = cur;
    tables = lay.take(table_bytes, 1);
    if (!lay.ok) return Status::INVALID_ARGUMENT;
    total = lay.cursor;
    if (!alloc_staging) return Status::OK;
    if (cudaHostAlloc(reinterpret_cast<void**>(&staging), table_bytes, cudaHostAllocDefault) != cudaSuccess) {
        staging = nullptr;
        return Status::CUDA_ERROR;
    }
    owns_staging = true;
    // Block counts of every launch are final once stage_tables has run.
    return Status::OK;
}

int Plan::knn_want_splits() const {
    int qtiles_total = 0;
    for (int i = 0; i < n; ++i) {
        const int dirs = pairs[i].s4.cross_check ? 2 : 1;
        const int k = pairs[i].s2.max_keypoints;
        qtiles_total += dirs * (k > 0 ? ceil_div(k, s4k::kQueryTile) : 0);
    }
    return std::max(1, ceil_div(2 * kSmCount, std::max(qtiles_total, 1)));
}

Plan::KnnShape Plan::knn_shape(int i, int dir, int want_splits) const {
    const int k = pairs[i].s2.max_keypoints;
    const auto& match = off[i].match;
    const int qt = k > 0 ? ceil_div(k, s4k::kQueryTile) : 0;
    const int stages = std::max(1, ceil_div(std::max(k, 1), s4k::kTrainStage));
    const int splits = std::min(want_splits, stages);
    const int rows = ceil_div(stages, splits) * s4k::kTrainStage;
    const int real_splits = ceil_div(std::max(k, 1), rows);
    // the partial buffer of the match layout holds fsplits/rsplits entries;
    // batch splits never exceed it (both come from the same capacities)
    const bool fits = real_splits <= (dir ? match.rsplits : match.fsplits) || real_splits == 1;
    KnnShape r;
    r.splits = fits ? real_splits : 1;
    r.rows = fits ? rows : std::max(s4k::kTrainStage, stages * s4k::kTrainStage);
    r.blocks = qt * r.splits;
    r.merge_blocks = (r.splits > 1 && k > 0) ? ceil_div(k, 256) : 0;
    return r;
}

void Plan::job_blocks(int i, int s, int l, int (&db)[s2s3::kDetectKinds], int (&sb)[s2s3::kDescribeKinds]) const {
    const auto& q = pairs[i];
    const auto& o = off[i];
    if (o.pyramid[s]) {
        s2s3::pyramid_detect_blocks(o.pyr[s], l, db);
        s2s3::pyramid_describe_blocks(o.pyr[s], l, sb);
        return;
    }
    const stitch_image_view& im = s ? q.image_b : q.image_a;
    const int k = q.s2.max_keypoints;
    const bool active = k > 0 && !small_image(im);
    db[s2s3::kFastKind] = active ? o.det[s].tiles : 0;
    db[s2s3::kSelectKind] = active ? o.det[s].select_blocks : 0;
    db[s2s3::kHarrisKind] = active ? ceil_div(o.det[s].candidates, s2s3::kHarrisThreads) : 0;
    db[s2s3::kSortKind] = active ? 1 : 0;
    sb[s2s3::kBlurKind] = 0;  // on demand: blur_tiles_kernel takes the flagged tiles from a list
    sb[s2s3::kDescKind] = k > 0 ? ceil_div(k, s2s3::kDescKeys) : 0;
}

Status Plan::stage_tables(void* ws) {
    if (staged_for == ws) return Status::OK;
    auto* T = staging;
    auto* dj = reinterpret_cast<DetectJob*>(T + offsets[kDetJobs]);
    auto* dp = reinterpret_cast<int*>(T + offsets[kDetPrefix]);
    auto* sj = reinterpret_cast<DescribeJob*>(T + offsets[kDesJobs]);
    auto* sp = reinterpret_cast<int*>(T + offsets[kDesPrefix]);
    auto* kj = reinterpret_cast<KnnJob*>(T + offsets[kKnnJobs]);
    auto* kp = reinterpret_cast<int*>(T + offsets[kKnnPrefix]);
    auto* mp = reinterpret_cast<int*>(T + offsets[kMergePrefix]);
    auto* aj = reinterpret_cast<AcceptJob*>(T + offsets[kAccJobs]);
    auto* ap = reinterpret_cast<int*>(T + offsets[kAccPrefix]);
    auto* pj = reinterpret_cast<PairIO*>(T + offsets[kPairJobs]);
    auto* pp = reinterpret_cast<int*>(T + offsets[kPairPrefix]);
    auto* rj = reinterpret_cast<SearchJob*>(T + offsets[kSearchJobs]);
    auto* rp = reinterpret_cast<int*>(T + offsets[kSearchPrefix]);
    auto* fp = reinterpret_cast<int*>(T + offsets[kFitPrefix]);
    auto* zj = reinterpret_cast<ResizeJob*>(T + offsets[kRsJobs]);
    auto* zp = reinterpret_cast<int*>(T + offsets[kRsPrefix]);
    std::uint32_t* hist_base = at<std::uint32_t>(ws, hists);
    std::uint32_t* mark_base = at<std::uint32_t>(ws, blur_flags);
    uint2* list = at<uint2>(ws, blur_list);
    std::uint32_t* list_count = at<std::uint32_t>(ws, queue) + 1;
    int* layer_counts = at<int>(ws, 0) + 3 * static_cast<std::size_t>(n);
    const int nd = n_det, nr = n_resize, rkinds = resize_kinds();
    int run_det[s2s3::kDetectKinds] = {}, run_des[s2s3::kDescribeKinds] = {};
    int run_rs[s2s3::kMaxLevels] = {};
    int rjob = 0;
    std::uint32_t* bmap = block_map ? reinterpret_cast<std::uint32_t*>(T + offsets[kBlockMap]) : nullptr;
    bool map_ok = true;  // every map entry lands inside its kind's range
    auto fill_map = [&](std::size_t first, int run, int total, int job, int blocks) {
        if (!bmap) return;
        if (run + blocks > total) {
            map_ok = false;
            return;
        }
        for (int b = 0; b < blocks; ++b)
            bmap[first + static_cast<std::size_t>(run + b)] = (static_cast<std::uint32_t>(job) << 16) | b;
    };
    auto add_job = [&](int idx, const DetectJob& d, const DescribeJob& e, const int (&db)[s2s3::kDetectKinds],
                       const int (&sb)[s2s3::kDescribeKinds]) {
        dj[idx] = d;
        sj[idx] = e;
        for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) {
            dp[kind * (nd + 1) + idx] = run_det[kind];
            fill_map(det_first[kind], run_det[kind], det_total[kind], idx, db[kind]);
            run_det[kind] += db[kind];
        }
        for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) {
            sp[kind * (nd + 1) + idx] = run_des[kind];
            fill_map(des_first[kind], run_des[kind], des_total[kind], idx, sb[kind]);
            run_des[kind] += sb[kind];
        }
    };
    const int want_splits = knn_want_splits();
    int knn = 0, run_knn = 0, run_merge = 0, run_search = 0, run_fit = 0;
    for (int i = 0; i < n; ++i) {
        const auto& q = pairs[i];
        const auto& o = off[i];
        const int k = q.s2.max_keypoints;
        Keypoints kps[2];
        Descriptors desc[2];
        for (int s = 0; s < 2; ++s) {
            const stitch_image_view& im = s ? q.image_b : q.image_a;
            kps[s] = Keypoints{at<float>(ws, o.kx[s]), at<float>(ws, o.ky[s]), at<float>(ws, o.kr[s]), k,
                               at<int>(ws, o.kcount[s])};
            desc[s] = Descriptors{DescriptorType::BINARY_U8, 32, 32, at<std::uint8_t>(ws, o.desc[s])};
            const auto& c2 = *reinterpret_cast<const s2::Config*>(&q.s2);
            const int idx = o.job0[s];
            if (o.pyramid[s]) {
                const auto& pl = o.pyr[s];
                s2s3::PyramidJobs pjobs;
                const s2s3::PyramidShared sh{layer_counts + o.layer0[s],
                                             hist_base + static_cast<std::size_t>(idx) * s2s3::kHistWords,
                                             mark_base + o.mark0[s], list, list_count, idx};
                s2s3::make_pyramid_jobs(view(im), c2, kps[s], desc[s], at<void>(ws, o.pyrws[s]), pl, sh, &pjobs);
                for (int l = 0; l < pl.plan.levels; ++l) {
                    int db[s2s3::kDetectKinds], sb[s2s3::kDescribeKinds];
                    job_blocks(i, s, l, db, sb);
                    add_job(idx + l, pjobs.detect[l], pjobs.describe[l], db, sb);
                }
                for (int l = 1; l < pl.plan.levels; ++l, ++rjob) {
                    zj[rjob] = pjobs.resize[l];
                    fill_map(rs_first[l - 1], run_rs[l - 1], rs_total[l - 1], rjob, pl.resize_tiles[l]);
                    for (int kind = 0; kind < rkinds; ++kind) {
                        zp[kind * (nr + 1) + rjob] = run_rs[kind];
                        run_rs[kind] += kind == l - 1 ? pl.resize_tiles[l] : 0;
                    }
                }
                continue;
            }
            DetectJob d = s2s3::make_detect_job(view(im), c2, kps[s], at<void>(ws, o.s2ws[s]), o.det[s]);
            d.hist = hist_base + static_cast<std::size_t>(idx) * s2s3::kHistWords;
            d.blur_marks = mark_base + o.mark0[s];
            d.blur_list = list;
            d.blur_count = list_count;
            d.job = idx;
            int db[s2s3::kDetectKinds], sb[s2s3::kDescribeKinds];
            job_blocks(i, s, 0, db, sb);
            const DescribeJob e =
                s2s3::make_describe_job(view(im), kps[s], desc[s], at<void>(ws, o.s3ws[s]), o.des[s]);
            add_job(idx, d, e, db, sb);
        }
        // S4 (forward, then reverse when the mutual check is on)
        auto* fwd = at<s4k::Top2>(ws, o.s4ws + o.match.forward);
        auto* rev = q.s4.cross_check ? at<s4k::Top2>(ws, o.s4ws + o.match.reverse) : nullptr;
        const int dirs = q.s4.cross_check ? 2 : 1;
        for (int dir = 0; dir < dirs; ++dir) {
            const int qs = dir ? 1 : 0, ts = dir ? 0 : 1;
            const int qt = k > 0 ? ceil_div(k, s4k::kQueryTile) : 0;
            const KnnShape sh = knn_shape(i, dir, want_splits);
            uint2* partial = at<uint2>(ws, o.s4ws + (dir ? o.match.rpartial : o.match.fpartial));
            kj[knn] = s4k::make_knn_job(kps[qs], desc[qs], kps[ts], desc[ts], std::max(qt, 1), sh.splits, sh.rows,
                                        partial, dir ? rev : fwd);
            kp[knn] = run_knn;
            mp[knn] = run_merge;
            fill_map(s45_first[kMapKnn], run_knn, s45_total[kMapKnn], knn, sh.blocks);
            fill_map(s45_first[kMapMerge], run_merge, s45_total[kMapMerge], knn, sh.merge_blocks);
            run_knn += sh.blocks;
            run_merge += sh.merge_blocks;
            ++knn;
        }
        AcceptJob a{};
        a.forward = fwd;
        a.reverse = rev;
        a.capacity = k;
        a.l2 = 0;
        a.ratio = q.s4.ratio_threshold;
        a.out = Matches{at<std::int32_t>(ws, o.ia), at<std::int32_t>(ws, o.ib), at<float>(ws, o.dist), k,
                        at<int>(ws, o.mcount)};
        aj[i] = a;
        ap[i] = i;
        fill_map(s45_first[kMapAccept], i, n, i, 1);
        fill_map(s45_first[kMapPair], i, n, i, 1);
        // S5
        PairIO io;
        const Status st = s5k::check_and_build(
            kps[0], kps[1], a.out, *reinterpret_cast<const ScaleInfo*>(&q.scale_a),
            *reinterpret_cast<const ScaleInfo*>(&q.scale_b), *reinterpret_cast<const s5::Config*>(&q.s5),
            at<std::uint8_t>(ws, o.mask), at<void>(ws, results), at<void>(ws, o.s5ws),
            s5k::estimate_workspace_bytes(), &io);
        if (st != Status::OK) return st;
        io.hpw = hpw;
        io.search_blocks = s5k::plan_search(q.s5.hypotheses, hpw);
        io.result_out = at<HomographyResult>(ws, results) + i;
        pj[i] = io;
        pp[i] = i;
        rj[i] = SearchJob{io, 0, q.s5.hypotheses, at<s5k::Model>(ws, o.models)};
        rp[i] = run_search;
        const int fit_b = io.search_blocks > 0 ? ceil_div(q.s5.hypotheses, s5k::kFitThreads) : 0;
        fill_map(s45_first[kMapSearch], run_search, s45_total[kMapSearch], i, io.search_blocks);
        fill_map(s45_first[kMapFit], run_fit, s45_total[kMapFit], i, fit_b);
        run_search += io.search_blocks;
        fp[i] = run_fit;
        run_fit += fit_b;
    }
    if (bmap) {  // the maps must cover exactly the blocks of every launch
        for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) map_ok = map_ok && run_det[kind] == det_total[kind];
        for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) map_ok = map_ok && run_des[kind] == des_total[kind];
        for (int kind = 0; kind < rkinds; ++kind) map_ok = map_ok && run_rs[kind] == rs_total[kind];
        map_ok = map_ok && run_knn == s45_total[kMapKnn] && run_merge == s45_total[kMapMerge] &&
                 run_search == s45_total[kMapSearch] && run_fit == s45_total[kMapFit];
        if (!map_ok) return Status::INVALID_ARGUMENT;
    }
    for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) dp[kind * (nd + 1) + nd] = run_det[kind];
    for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) sp[kind * (nd + 1) + nd] = run_des[kind];
    for (int kind = 0; kind < rkinds; ++kind) zp[kind * (nr + 1) + nr] = run_rs[kind];
    for (int kind = 0; kind < s2s3::kMaxLevels; ++kind) rs_blocks[kind] = kind < rkinds ? run_rs[kind] : 0;
    kp[n_knn] = run_knn;
    mp[n_knn] = run_merge;
    ap[n] = n;
    pp[n] = n;
    rp[n] = run_search;
    fp[n] = run_fit;
    knn_blocks = run_knn;
    merge_blocks = run_merge;
    search_blocks = run_search;
    fit_blocks = run_fit;
    for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) det_blocks[kind] = run_det[kind];
    for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) des_blocks[kind] = run_des[kind];
    staged_for = ws;
    return Status::OK;
}

Status Plan::enqueue(void* ws, std::size_t bytes, stitch_homography_result* host_results, cudaStream_t s,
                     const unsigned char* device_tables) {
    if (!ws || !aligned(ws, kWorkspaceAlign)) return Status::INVALID_ARGUMENT;
    if (bytes < total) return Status::INSUFFICIENT_WORKSPACE;
    set_attributes_once();
    const Status st = stage_tables(ws);
    if (st != Status::OK) return st;
    const unsigned char* T = device_tables;
    if (!T) {
        unsigned char* W = at<unsigned char>(ws, tables);
        if (cudaMemcpyAsync(W, staging, table_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
            return Status::CUDA_ERROR;
        T = W;
    }
    // counts and histograms: contiguous 32-bit words at the start, zeroed together
    const std::size_t words = zeroed / sizeof(std::uint32_t);
    const auto zero_blocks = static_cast<unsigned>(std::min<std::size_t>((words + 255) / 256, 148));
    zero_words_kernel<<<zero_blocks, 256, 0, s>>>(static_cast<std::uint32_t*>(ws), words);

    using DetSrc = s2s3::JobTable<DetectJob>;
    using DesSrc = s2s3::JobTable<DescribeJob>;
    using RsSrc = s2s3::JobTable<ResizeJob>;
    DetSrc det{reinterpret_cast<const DetectJob*>(T + offsets[kDetJobs]),
               reinterpret_cast<const int*>(T + offsets[kDetPrefix]), n_det};
    DesSrc des{reinterpret_cast<const DescribeJob*>(T + offsets[kDesJobs]),
               reinterpret_cast<const int*>(T + offsets[kDesPrefix]), n_det};
    RsSrc rs{reinterpret_cast<const ResizeJob*>(T + offsets[kRsJobs]),
             reinterpret_cast<const int*>(T + offsets[kRsPrefix]), n_resize};
    if (block_map) {
        const auto* M = reinterpret_cast<const std::uint32_t*>(T + offsets[kBlockMap]);
        for (int kind = 0; kind < s2s3::kDetectKinds; ++kind) {
            det.map[kind] = M + det_first[kind];
            det.map_blocks[kind] = det_total[kind];
        }
        for (int kind = 0; kind < s2s3::kDescribeKinds; ++kind) {
            des.map[kind] = M + des_first[kind];
            des.map_blocks[kind] = des_total[kind];
        }
        for (int kind = 0; kind < resize_kinds(); ++kind) {
            rs.map[kind] = M + rs_first[kind];
            rs.map_blocks[kind] = rs_total[kind];
        }
    }
    int launches = 1;  // zero_words_kernel
    int next_mark = 0;
    bool marks_ok = true;
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (marked && cudaStreamIsCapturing(s, &capturing) != cudaSuccess) return Status::CUDA_ERROR;
    auto go = [&](int blocks) { launches += blocks > 0; return blocks > 0; };
    auto mark = [&] {
        // Under stream capture the record must be external to become an
        // event-record node, so that replays of the graph record the mark.
        if (marked && marks[next_mark])
            marks_ok &= (capturing == cudaStreamCaptureStatusActive
                             ? cudaEventRecordWithFlags(marks[next_mark], s, cudaEventRecordExternal)
                             : cudaEventRecord(marks[next_mark], s)) == cudaSuccess;
        ++next_mark;
    };
    mark();  // tables uploaded, counts cleared
    for (int kind = 0; kind + 1 < max_levels; ++kind)  // layer kind + 1 of every pyramid image
        if (go(rs_blocks[kind])) {
            switch (tuning.resize_tile_h) {
                case 16: s2s3::resize_kernel<RsSrc, 16><<<rs_blocks[kind], 256, 0, s>>>(rs, kind); break;
                case 32: s2s3::resize_kernel<RsSrc, 32><<<rs_blocks[kind], 256, 0, s>>>(rs, kind); break;
                default: s2s3::resize_kernel<RsSrc, s2s3::kResizeTileH><<<rs_blocks[kind], 256, 0, s>>>(rs, kind);
            }
        }
    mark();
    std::uint32_t* q = at<std::uint32_t>(ws, queue);  // FAST tile queue, then the blur-list count
    const int tiles = det_blocks[s2s3::kFastKind];
    if (go(tiles))
        s2s3::fast_kernel<DetSrc><<<std::min(tiles, kSmCount * (tuning.fast_ctas_per_sm ? tuning.fast_ctas_per_sm
                                                                                      : s2s3::kFastCtasPerSm)),
                                    s2s3::kFastThreads, 0, s>>>(det, q, tiles);
    mark();
    if (go(det_blocks[s2s3::kSelectKind])) {
        s2s3::select_kernel<DetSrc><<<det_blocks[s2s3::kSelectKind], 256, 0, s>>>(det);
        s2s3::ties_kernel<DetSrc><<<det_blocks[s2s3::kSortKind], s2s3::kTieThreads, 0, s>>>(det);
        ++launches;
    }
    mark();
    if (go(det_blocks[s2s3::kHarrisKind]))
        s2s3::harris_kernel<DetSrc><<<det_blocks[s2s3::kHarrisKind], s2s3::kHarrisThreads, 0, s>>>(det);
    mark();
    if (go(det_blocks[s2s3::kSortKind]))
        s2s3::sort_topk_kernel<DetSrc><<<det_blocks[s2s3::kSortKind], s2s3::kSortThreads, sort_smem, s>>>(det);
    if (rank_fallback && go(det_blocks[s2s3::kHarrisKind]))
        s2s3::rank_topk_kernel<DetSrc><<<det_blocks[s2s3::kHarrisKind], s2s3::kHarrisThreads, 0, s>>>(det);
    mark();
    if (go(tiles > 0 && blur_total > 0 ? 1 : 0))
        s2s3::blur_tiles_kernel<DesSrc>
            <<<static_cast<int>(std::min<std::size_t>(
                   blur_total, kSmCount * (tuning.blur_ctas_per_sm ? tuning.blur_ctas_per_sm : s2s3::kBlurCtasPerSm))),
               256, 0, s>>>(des, at<uint2>(ws, blur_list), q + 1);
    mark();
    if (go(des_blocks[s2s3::kDescKind]))
        s2s3::describe_kernel<DesSrc><<<des_blocks[s2s3::kDescKind], s2s3::kDescWarps * 32, 0, s>>>(des);
    mark();

    // S4/S5 job tables, with their block maps when the plan has them
    const auto* M = block_map ? reinterpret_cast<const std::uint32_t*>(T + offsets[kBlockMap]) : nullptr;
    auto with_map = [&](auto src, int m) {
        if (M) {
            src.map = M + s45_first[m];
            src.map_blocks = s45_total[m];
        }
        return src;
    };
    using KnnSrc = s4k::JobTable<KnnJob>;
    const auto* kjobs = reinterpret_cast<const KnnJob*>(T + offsets[kKnnJobs]);
    if (go(knn_blocks)) {
        const KnnSrc ks = with_map(KnnSrc{kjobs, reinterpret_cast<const int*>(T + offsets[kKnnPrefix]), n_knn}, kMapKnn);
        if (s4k::is_tensor(matcher)) {
            if (!s4k::launch_tc(matcher, knn_blocks, ks, s)) return Status::CUDA_ERROR;
        } else {
            s4k::knn_popc_kernel<KnnSrc, s4k::kQueriesPerThread><<<knn_blocks, s4k::kQueryThreads, 0, s>>>(ks);
        }
    }
    mark();
    if (go(merge_blocks))
        s4k::knn_merge_kernel<KnnSrc><<<merge_blocks, 256, 0, s>>>(
            with_map(KnnSrc{kjobs, reinterpret_cast<const int*>(T + offsets[kMergePrefix]), n_knn}, kMapMerge));
    mark();
    using AccSrc = s4k::JobTable<AcceptJob>;
    if (go(n))
        s4k::accept_kernel<AccSrc><<<n, 1024, 0, s>>>(
            with_map(AccSrc{reinterpret_cast<const AcceptJob*>(T + offsets[kAccJobs]),
                            reinterpret_cast<const int*>(T + offsets[kAccPrefix]), n},
                     kMapAccept));
    mark();

    using PairSrc = s5k::JobTable<PairIO>;
    using SearchSrc = s5k::JobTable<SearchJob>;
    const PairSrc pairsrc = with_map(PairSrc{reinterpret_cast<const PairIO*>(T + offsets[kPairJobs]),
                                             reinterpret_cast<const int*>(T + offsets[kPairPrefix]), n},
                                     kMapPair);
    if (go(n)) s5k::prepare_kernel<PairSrc><<<n, 256, 0, s>>>(pairsrc);
    mark();
    if (go(fit_blocks))
        s5k::fit_kernel<SearchSrc><<<fit_blocks, s5k::kFitThreads, 0, s>>>(
            with_map(SearchSrc{reinterpret_cast<const SearchJob*>(T + offsets[kSearchJobs]),
                               reinterpret_cast<const int*>(T + offsets[kFitPrefix]), n},
                     kMapFit));
    if (go(search_blocks))
        s5k::search_kernel<SearchSrc, true><<<search_blocks, s5k::kSearchThreads, search_smem, s>>>(
            with_map(SearchSrc{reinterpret_cast<const SearchJob*>(T + offsets[kSearchJobs]),
                               reinterpret_cast<const int*>(T + offsets[kSearchPrefix]), n},
                     kMapSearch));
    mark();
    if (go(n)) s5k::finish_kernel<PairSrc><<<n, s5k::kFinishThreads, 0, s>>>(pairsrc);
    mark();
    if (!marks_ok) return Status::CUDA_ERROR;
    note_launches(launches);
    if (cudaGetLastError() != cudaSuccess) return Status::CUDA_ERROR;
    if (host_results &&
        cudaMemcpyAsync(host_results, at<void>(ws, results), n * sizeof(HomographyResult), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess)
        return Status::CUDA_ERROR;
    return Status::OK;
}

}  // namespace stitch::b200::batch

namespace stitch::b200::s4k {
int take_batch_tc_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)) != cudaSuccess) return -1;
    const int zero = 0;
    if (v && cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    return v;
}
}  // namespace stitch::b200::s4k

using stitch::Status;
using stitch::b200::batch::Plan;

struct stitch_batch {
    Plan plan;
    int launches_per_run = 0;
};

extern "C" {

int stitch_batch_create_tuned(int n_pairs, const stitch_pair_desc* pairs, const stitch_batch_tuning* tuning,
                              stitch_batch** out, size_t* bytes, int* bad_pair) {
    if (!out || !bytes) return static_cast<int>(Status::INVALID_ARGUMENT);
    *out = nullptr;
    *bytes = 0;
    if (tuning) {
        const auto& t = *tuning;
        const bool ok = t.fast_ctas_per_sm >= 0 && t.fast_ctas_per_sm <= stitch::b200::s2s3::kFastCtasPerSm &&
                        t.blur_ctas_per_sm >= 0 && t.blur_ctas_per_sm <= stitch::b200::s2s3::kBlurCtasPerSm &&
                        (t.matcher == 0 || stitch::b200::s4k::valid_matcher(t.matcher - 1)) &&
                        (t.search_hpw == 0 || t.search_hpw == 4 || t.search_hpw == 8 || t.search_hpw == 16 ||
                         t.search_hpw == 32) &&
                        (t.resize_tile_h == 0 || t.resize_tile_h == 16 || t.resize_tile_h == 32 ||
                         t.resize_tile_h == 64);
        if (!ok) return static_cast<int>(Status::INVALID_ARGUMENT);
    }
    auto* b = new (std::nothrow) stitch_batch;
    if (!b) return static_cast<int>(Status::CUDA_ERROR);
    if (tuning) b->plan.tuning = *tuning;
    const Status st = b->plan.build(n_pairs, pairs, bad_pair);
    if (st != Status::OK) {
        delete b;
        return static_cast<int>(st);
    }
    if (tuning && tuning->matcher > 0) b->plan.matcher = tuning->matcher - 1;
    *bytes = b->plan.total;
    *out = b;
    return 0;
}

int stitch_batch_create(int n_pairs, const stitch_pair_desc* pairs, stitch_batch** out, size_t* bytes,
                        int* bad_pair) {
    return stitch_batch_create_tuned(n_pairs, pairs, nullptr, out, bytes, bad_pair);
}

int stitch_batch_enqueue(stitch_batch* b, void* ws, size_t bytes, stitch_homography_result* results, void* stream) {
    if (!b) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(b->plan.enqueue(ws, bytes, results, static_cast<cudaStream_t>(stream)));
}

int stitch_batch_capture(stitch_batch* b, void* ws, size_t bytes, stitch_homography_result* results, void* stream) {
    if (!b) return static_cast<int>(Status::INVALID_ARGUMENT);
    auto& p = b->plan;
    if (!ws || bytes < p.total) return static_cast<int>(Status::INSUFFICIENT_WORKSPACE);
    const Status pre = p.stage_tables(ws);  // host work, before capture
    if (pre != Status::OK) return static_cast<int>(pre);
    const auto s = static_cast<cudaStream_t>(stream);
    if (p.graph_exec) {
        cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(p.graph_exec));
        p.graph_exec = nullptr;
    }
    if (p.graph) {
        cudaGraphDestroy(static_cast<cudaGraph_t>(p.graph));
        p.graph = nullptr;
    }
    // The first enqueue, outside capture, sets kernel attributes and uploads
    // the job tables into the workspace (it is a full run); they are then
    // copied, device to device, into the plan's own table buffer. Replays read
    // that buffer, so they start with a kernel rather than a host-to-device
    // copy, which would wait behind any other upload in flight on the same
    // copy engine, and depend on nothing left in the workspace.
    if (!p.graph_tables && cudaMalloc(reinterpret_cast<void**>(&p.graph_tables), p.table_bytes) != cudaSuccess) {
        p.graph_tables = nullptr;
        return static_cast<int>(Status::CUDA_ERROR);
    }
    const long long before = stitch_launch_count();
    Status st = p.enqueue(ws, bytes, results, s);
    if (st != Status::OK) return static_cast<int>(st);
    b->launches_per_run = static_cast<int>(stitch_launch_count() - before);
    if (cudaMemcpyAsync(p.graph_tables, static_cast<unsigned char*>(ws) + p.tables, p.table_bytes, cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)  // replays may go to any stream
        return static_cast<int>(Status::CUDA_ERROR);
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return static_cast<int>(Status::CUDA_ERROR);
    st = p.enqueue(ws, bytes, results, s, p.graph_tables);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s, &g);
    if (st != Status::OK || end != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        return static_cast<int>(st != Status::OK ? st : Status::CUDA_ERROR);
    }
    cudaGraphExec_t e = nullptr;
    if (cudaGraphInstantiate(&e, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return static_cast<int>(Status::CUDA_ERROR);
    }
    p.graph = g;
    p.graph_exec = e;
    return 0;
}

int stitch_batch_launch(stitch_batch* b, void* stream) {
    if (!b || !b->plan.graph_exec) return static_cast<int>(Status::INVALID_ARGUMENT);
    stitch::b200::note_launches(b->launches_per_run);
    return cudaGraphLaunch(static_cast<cudaGraphExec_t>(b->plan.graph_exec), static_cast<cudaStream_t>(stream)) ==
                   cudaSuccess
               ? 0
               : static_cast<int>(Status::CUDA_ERROR);
}

int stitch_batch_pair_outputs(const stitch_batch* b, void* ws, int i, stitch_keypoints* ka, stitch_keypoints* kb,
                              stitch_descriptors* da, stitch_descriptors* db, stitch_matches* m, uint8_t** mask,
                              stitch_homography_result** result) {
    if (!b || !ws || i < 0 || i >= b->plan.n) return static_cast<int>(Status::INVALID_ARGUMENT);
    const auto& p = b->plan;
    const auto& o = p.off[i];
    const int k = p.pairs[i].s2.max_keypoints;
    auto P = [&](std::size_t off) { return static_cast<char*>(ws) + off; };
    stitch_keypoints* ks[2] = {ka, kb};
    stitch_descriptors* ds[2] = {da, db};
    for (int s = 0; s < 2; ++s) {
        if (ks[s])
            *ks[s] = stitch_keypoints{reinterpret_cast<float*>(P(o.kx[s])), reinterpret_cast<float*>(P(o.ky[s])),
                                      reinterpret_cast<float*>(P(o.kr[s])), k, reinterpret_cast<int*>(P(o.kcount[s]))};
        if (ds[s]) *ds[s] = stitch_descriptors{0, 32, 32, P(o.desc[s])};
    }
    if (m)
        *m = stitch_matches{reinterpret_cast<int32_t*>(P(o.ia)), reinterpret_cast<int32_t*>(P(o.ib)),
                            reinterpret_cast<float*>(P(o.dist)), k, reinterpret_cast<int*>(P(o.mcount))};
    if (mask) *mask = reinterpret_cast<uint8_t*>(P(o.mask));
    if (result) *result = reinterpret_cast<stitch_homography_result*>(P(p.results)) + i;
    return 0;
}

void stitch_batch_destroy(stitch_batch* b) { delete b; }

int stitch_batch_set_matcher(stitch_batch* b, int kind) {
    if (!b || !stitch::b200::s4k::valid_matcher(kind)) return static_cast<int>(Status::INVALID_ARGUMENT);
    b->plan.matcher = kind;
    return 0;
}

int stitch_batch_set_marks(stitch_batch* b, void* const* events, int count) {
    if (!b || (events && count != STITCH_BATCH_MARKS)) return static_cast<int>(Status::INVALID_ARGUMENT);
    auto& p = b->plan;
    p.marked = events != nullptr;
    for (int i = 0; i < STITCH_BATCH_MARKS; ++i) p.marks[i] = events ? static_cast<cudaEvent_t>(events[i]) : nullptr;
    return 0;
}

}  // extern "C"
