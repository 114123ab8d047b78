// Host-only check that batch::Plan::build gives a fresh plan's layout when it
// is called again on the same object (every count, total, offset and
// block-map total reset). Built and run by tests/test_plan_rebuild.py on the
// CPU: build() with alloc_staging = false touches no device.
#include <cstdio>
#include <cstring>
#include <vector>

#include "batch.hpp"

using stitch::b200::batch::Plan;

namespace {

stitch_pair_desc pair(int wa, int ha, int wb, int hb, int k, int r, int levels, int cross) {
    static unsigned char fake[256];
    stitch_pair_desc d{};
    d.image_a = stitch_image_view{fake, wa, ha, (wa + 15) / 16 * 16, 1};
    d.image_b = stitch_image_view{fake, wb, hb, (wb + 15) / 16 * 16, 1};
    d.s2 = stitch_s2_config{20, k, 0.04f};
    d.s4.ratio_threshold = 0.8f;
    d.s4.cross_check = cross;
    d.s5 = stitch_s5_config{r, 0, 64, 1, 3.0, 7, 1};
    d.pyramid = stitch_pyramid_config{levels, 1.2f};
    return d;
}

bool same(const Plan& a, const Plan& b) {
    bool ok = a.n == b.n && a.total == b.total && a.table_bytes == b.table_bytes && a.tables == b.tables &&
              a.results == b.results && a.n_det == b.n_det && a.n_layers == b.n_layers &&
              a.n_resize == b.n_resize && a.max_levels == b.max_levels && a.hists == b.hists &&
              a.zeroed == b.zeroed && a.search_blocks == b.search_blocks && a.hpw == b.hpw &&
              a.sort_smem == b.sort_smem && a.search_smem == b.search_smem &&
              a.rank_fallback == b.rank_fallback && a.block_map == b.block_map;
    ok = ok && !std::memcmp(a.offsets, b.offsets, sizeof a.offsets) &&
         !std::memcmp(a.det_total, b.det_total, sizeof a.det_total) &&
         !std::memcmp(a.des_total, b.des_total, sizeof a.des_total) &&
         !std::memcmp(a.rs_total, b.rs_total, sizeof a.rs_total) &&
         !std::memcmp(a.det_first, b.det_first, sizeof a.det_first) &&
         !std::memcmp(a.des_first, b.des_first, sizeof a.des_first) &&
         !std::memcmp(a.rs_first, b.rs_first, sizeof a.rs_first) &&
         !std::memcmp(a.s45_total, b.s45_total, sizeof a.s45_total) &&
         !std::memcmp(a.s45_first, b.s45_first, sizeof a.s45_first);
    for (int i = 0; ok && i < a.n; ++i) {
        const auto& x = a.off[i];
        const auto& y = b.off[i];
        ok = !std::memcmp(x.kx, y.kx, sizeof x.kx) && !std::memcmp(x.desc, y.desc, sizeof x.desc) &&
             x.ia == y.ia && x.mask == y.mask && x.s4ws == y.s4ws && x.s5ws == y.s5ws && x.models == y.models &&
             !std::memcmp(x.pyrws, y.pyrws, sizeof x.pyrws) && !std::memcmp(x.job0, y.job0, sizeof x.job0) &&
             !std::memcmp(x.layer0, y.layer0, sizeof x.layer0);
    }
    return ok;
}

}  // namespace

int main() {
    const std::vector<stitch_pair_desc> big = {pair(640, 480, 640, 480, 500, 500, 8, 0),
                                               pair(1920, 1080, 1280, 720, 8000, 8000, 8, 1),
                                               pair(512, 512, 512, 512, 2000, 2000, 1, 0)};
    const std::vector<stitch_pair_desc> small = {pair(256, 256, 300, 200, 300, 256, 8, 0)};
    int bad = -1;
    Plan fresh_big, fresh_small, reused;
    if (fresh_big.build(3, big.data(), &bad, false) != stitch::Status::OK ||
        fresh_small.build(1, small.data(), &bad, false) != stitch::Status::OK)
        return 2;
    // the same object: big, small, big again
    if (reused.build(3, big.data(), &bad, false) != stitch::Status::OK || !same(reused, fresh_big)) return 3;
    if (reused.build(1, small.data(), &bad, false) != stitch::Status::OK || !same(reused, fresh_small)) return 4;
    if (reused.build(3, big.data(), &bad, false) != stitch::Status::OK || !same(reused, fresh_big)) return 5;
    std::printf("plan rebuild ok: %zu / %zu bytes\n", fresh_big.total, fresh_small.total);
    return 0;
}
