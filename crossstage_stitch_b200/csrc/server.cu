// Served form: a device-resident request loop with continuous batching.
//
// Requests (two host GRAY8 images and per-pair knobs) are queued by
// stitch_server_submit. One dispatcher thread admits them in arrival order
// into batches: a batch takes as many waiting requests as fit (in pairs and
// in one contiguous region of the caller's device arena, whose size is the
// HBM admission budget) and is launched on a free stream as soon as one is
// free, so a batch formed from requests that arrived while others were on
// the GPU overlaps them. Each batch copies its images into the arena, runs
// the batched registration chain (batch.cu: every kernel once for all of
// its pairs), and copies the homography results back; when its event
// completes the region and the stream return to the pool and the results
// are handed to stitch_server_poll. Two optional phases run on the same
// stream and region before that: the S5 extension retry of requests below
// their bar, then the S6 feather panorama of RGB requests that asked for one. A pair's result does not depend on the
// batch it ran in: the batched chain equals the per-pair stages bit for bit.
//
// No reference counterpart: the reference registers one pair at a time
// (harness/pipeline_runner.cu:335-416).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.hpp"
#include "s1_internal.hpp"

namespace stitch::b200::serve {

using batch::Plan;

namespace {

constexpr std::size_t kAlign = 256;
constexpr std::size_t kStagingPerPair = 16 << 10;  // pinned job-table bytes reserved per pair

std::size_t round_up(std::size_t v, std::size_t a) { return (v + a - 1) / a * a; }
int image_pitch(int w) { return (w + 15) / 16 * 16; }

// Device images of one request: the host copies (GRAY8, or RGB8 rows of 3w
// bytes) and, for RGB8, the working-size GRAY8 images S1 writes.
struct Geometry {
    bool rgb = false;
    int wa = 0, ha = 0, wb = 0, hb = 0;  // working (registered) sizes
    stitch_scale_info sa{}, sb{};
    std::size_t bytes() const { return host_a + host_b + (rgb ? work_a + work_b : 0); }
    std::size_t host_a = 0, host_b = 0, work_a = 0, work_b = 0;
};

std::size_t plane(int row_bytes, int rows) {
    return round_up(static_cast<std::size_t>(image_pitch(row_bytes)) * static_cast<std::size_t>(rows), kAlign);
}

Status geometry(const stitch_request& r, Geometry* g) {
    g->rgb = r.rgb != 0;
    if (!g->rgb) {
        if (r.pitch_a < r.width_a || r.pitch_b < r.width_b || (r.scale != 0.0 && r.scale != 1.0))
            return Status::INVALID_ARGUMENT;
        g->wa = r.width_a, g->ha = r.height_a, g->wb = r.width_b, g->hb = r.height_b;
        g->sa = r.scale_a;
        g->sb = r.scale_b;
        g->host_a = plane(r.width_a, r.height_a);
        g->host_b = plane(r.width_b, r.height_b);
        return Status::OK;
    }
    const double s = r.scale == 0.0 ? 1.0 : r.scale;
    if (r.width_a <= 0 || r.width_b <= 0 || r.pitch_a < 3 * r.width_a || r.pitch_b < 3 * r.width_b ||
        stitch_make_scale_info(r.width_a, r.height_a, s, &g->sa) != 0 ||
        stitch_make_scale_info(r.width_b, r.height_b, s, &g->sb) != 0)
        return Status::INVALID_ARGUMENT;
    g->wa = g->sa.work_w, g->ha = g->sa.work_h, g->wb = g->sb.work_w, g->hb = g->sb.work_h;
    g->host_a = plane(3 * r.width_a, r.height_a);
    g->host_b = plane(3 * r.width_b, r.height_b);
    g->work_a = plane(g->wa, g->ha);
    g->work_b = plane(g->wb, g->hb);
    return Status::OK;
}

// First-fit allocator over [0, size) with coalescing frees.
class Arena {
public:
    explicit Arena(std::size_t size) { free_[0] = size; }
    bool alloc(std::size_t bytes, std::size_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const std::size_t rest = it->second - bytes;
            const std::size_t next = it->first + bytes;
            free_.erase(it);
            if (rest) free_[next] = rest;
            return true;
        }
        return false;
    }
    void release(std::size_t off, std::size_t bytes) {
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    std::size_t largest() const {
        std::size_t m = 0;
        for (const auto& f : free_) m = std::max(m, f.second);
        return m;
    }

private:
    std::map<std::size_t, std::size_t> free_;
};

struct Request {
    stitch_request r;
    Geometry g;
    double submit_ms = 0.0;
    std::size_t footprint = 0;     // images + its share of a batch workspace, alone
    std::size_t render_bytes = 0;  // S6 canvas planes + counters (0: no panorama)
};

// S6 canvas planes of one request inside its batch region: packed RGB rows,
// packed mask rows, then the two uint64 counters.
std::size_t render_bytes(std::size_t capacity) {
    return round_up(3 * capacity, kAlign) + round_up(capacity, kAlign) + kAlign;
}

// Outcome of one request's panorama, reported in its result.
struct Panorama {
    int status = -1;  // not asked for
    int width = 0, height = 0, origin_x = 0, origin_y = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    unsigned char* staging = nullptr;           // pinned job tables
    unsigned char* s1_staging = nullptr;        // pinned S1 job table (2 jobs per pair) + prefix
    stitch_homography_result* results = nullptr;  // pinned, max_batch entries
    std::unique_ptr<Plan> plan;
    std::vector<Request> reqs;
    std::size_t offset = 0, bytes = 0;
    std::size_t ws_offset = 0;   // batch workspace inside the region
    double launch_ms = 0.0;
    bool busy = false;
    int phase = 0;               // 0 registering, 1 retries enqueued, 2 panoramas enqueued
    std::vector<int> attempts;   // per request
    std::vector<std::size_t> host_off;    // 2 per request: the copied images
    std::vector<std::size_t> render_off;  // per request: its S6 planes (panorama requests)
    std::vector<Panorama> panoramas;      // per request
    std::uint64_t* render_counts = nullptr;  // pinned, 2 per request slot
};

// Pair descriptor of a request whose registered (GRAY8) images start at
// `a` and `b`.
stitch_pair_desc pair_desc(const Request& q, const unsigned char* a, const unsigned char* b) {
    const stitch_request& r = q.r;
    const Geometry& g = q.g;
    stitch_pair_desc d{};
    d.image_a = stitch_image_view{const_cast<std::uint8_t*>(a), g.wa, g.ha, image_pitch(g.wa), 1};
    d.image_b = stitch_image_view{const_cast<std::uint8_t*>(b), g.wb, g.hb, image_pitch(g.wb), 1};
    d.scale_a = g.sa;
    d.scale_b = g.sb;
    d.s2 = r.s2;
    d.s4 = r.s4;
    d.s5 = r.s5;
    d.pyramid = r.pyramid;
    return d;
}

}  // namespace

// Checks a request and fills q (knobs, image geometry, footprint: the
// request alone in a batch, host layout only) and the job-table bytes.
Status prepare_request(const stitch_request& r, Request* q, std::size_t* table_bytes) {
    if (!r.host_a || !r.host_b) return Status::INVALID_ARGUMENT;
    if ((r.host_mask && !r.host_panorama) ||
        (r.host_panorama && (!r.rgb || r.panorama_capacity == 0 ||
                             r.panorama_capacity > std::numeric_limits<std::size_t>::max() / 8)))
        return Status::INVALID_ARGUMENT;
    q->r = r;
    Status st = geometry(r, &q->g);
    if (st != Status::OK) return st;
    q->render_bytes = r.host_panorama ? render_bytes(r.panorama_capacity) : 0;
    const auto* fake = reinterpret_cast<const unsigned char*>(kAlign);
    stitch_pair_desc d = pair_desc(*q, fake, fake);
    Plan p;
    int bad = -1;
    st = p.build(1, &d, &bad, false);
    if (st != Status::OK) return st;
    q->footprint = q->g.bytes() + round_up(p.total, kAlign) + (q->g.rgb ? kAlign : 0) + q->render_bytes;
    *table_bytes = p.table_bytes;
    return Status::OK;
}

class Server {
public:
    explicit Server(const stitch_server_config& c) : cfg_(c), arena_(c.arena_bytes) {
        t0_ = std::chrono::steady_clock::now();
        matcher_ = s4k::matcher();  // the creating thread's choice; the dispatcher thread builds the plans
    }
    ~Server() { shutdown(); }

    Status start() {
        if (cudaSetDevice(cfg_.device) != cudaSuccess) return Status::CUDA_ERROR;
        slots_.resize(cfg_.streams);
        for (auto& s : slots_) {
            if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess ||
                cudaHostAlloc(reinterpret_cast<void**>(&s.staging), staging_cap(), cudaHostAllocDefault) !=
                    cudaSuccess ||
                cudaHostAlloc(reinterpret_cast<void**>(&s.s1_staging), s1_staging_bytes(), cudaHostAllocDefault) !=
                    cudaSuccess ||
                cudaHostAlloc(reinterpret_cast<void**>(&s.results),
                              cfg_.max_batch * sizeof(stitch_homography_result), cudaHostAllocDefault) != cudaSuccess ||
                cudaHostAlloc(reinterpret_cast<void**>(&s.render_counts), 2 * cfg_.max_batch * sizeof(std::uint64_t),
                              cudaHostAllocDefault) != cudaSuccess)
                return Status::CUDA_ERROR;
        }
        worker_ = std::thread([this] { loop(); });
        return Status::OK;
    }

    Status submit(const stitch_request& r) {
        Request q;
        std::size_t table_bytes = 0;
        Status st = prepare_request(r, &q, &table_bytes);
        if (st != Status::OK) return st;
        if (q.footprint > cfg_.arena_bytes || table_bytes > staging_cap()) return Status::INSUFFICIENT_WORKSPACE;
        q.submit_ms = now_ms();
        {
            std::lock_guard<std::mutex> g(mu_);
            if (stopping_) return Status::INVALID_ARGUMENT;
            incoming_.push_back(q);
            ++outstanding_;
        }
        cv_.notify_one();
        return Status::OK;
    }

    int poll(stitch_server_result* out, int max) {
        std::lock_guard<std::mutex> g(mu_);
        const int n = std::min<int>(max, static_cast<int>(done_.size()));
        for (int i = 0; i < n; ++i) out[i] = done_[i];
        done_.erase(done_.begin(), done_.begin() + n);
        return n;
    }

    int outstanding() {
        std::lock_guard<std::mutex> g(mu_);
        return outstanding_;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (stopping_ && !worker_.joinable()) return;
            stopping_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
        for (auto& s : slots_) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            s.plan.reset();
            if (s.done) cudaEventDestroy(s.done);
            if (s.stream) cudaStreamDestroy(s.stream);
            if (s.staging) cudaFreeHost(s.staging);
            if (s.s1_staging) cudaFreeHost(s.s1_staging);
            if (s.results) cudaFreeHost(s.results);
            if (s.render_counts) cudaFreeHost(s.render_counts);
            s = Slot{};
        }
    }

private:
    std::size_t staging_cap() const { return kStagingPerPair * cfg_.max_batch + (64 << 10); }
    std::size_t s1_jobs_bytes() const { return round_up(2 * cfg_.max_batch * sizeof(b200::s1k::BatchJob), kAlign); }
    std::size_t s1_staging_bytes() const { return s1_jobs_bytes() + (2 * cfg_.max_batch + 1) * sizeof(int); }

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
    }

    void finish(Slot& s, Status launch_status) {
        const double t = now_ms();
        std::vector<stitch_server_result> out;
        for (std::size_t i = 0; i < s.reqs.size(); ++i) {
            stitch_server_result r{};
            r.tag = s.reqs[i].r.tag;
            r.submit_ms = s.reqs[i].submit_ms;
            r.launch_ms = s.launch_ms;
            r.done_ms = t;
            r.batch_pairs = static_cast<int>(s.reqs.size());
            r.status = static_cast<int>(launch_status);
            r.attempts = i < s.attempts.size() ? s.attempts[i] : 1;
            if (launch_status == Status::OK) r.result = s.results[i];
            r.render_status = -1;
            if (s.reqs[i].render_bytes) {
                const Panorama pano = i < s.panoramas.size() ? s.panoramas[i] : Panorama{};
                r.render_status = launch_status != Status::OK ? static_cast<int>(launch_status) : pano.status;
                if (r.render_status == static_cast<int>(Status::OK)) {
                    r.canvas_width = pano.width;
                    r.canvas_height = pano.height;
                    r.origin_x = pano.origin_x;
                    r.origin_y = pano.origin_y;
                    r.union_pixels = s.render_counts[2 * i];
                    r.overlap_pixels = s.render_counts[2 * i + 1];
                }
            }
            out.push_back(r);
        }
        if (s.bytes) arena_.release(s.offset, s.bytes);
        s.plan.reset();
        s.reqs.clear();
        s.attempts.clear();
        s.panoramas.clear();
        s.bytes = 0;
        s.busy = false;
        s.phase = 0;
        std::lock_guard<std::mutex> g(mu_);
        done_.insert(done_.end(), out.begin(), out.end());
        outstanding_ -= static_cast<int>(out.size());
    }

    // After a batch completes: requests whose result falls short of their
    // retry bar get their saved S5 search extended to retry_hypotheses on the
    // batch's resident buffers (src/controller/reuse.cpp:5-22). Returns true
    // when work was enqueued (the slot stays busy until it completes).
    bool retry(Slot& s) {
        bool any = false;
        auto* ws = static_cast<unsigned char*>(cfg_.arena) + s.offset + s.ws_offset;
        for (std::size_t i = 0; i < s.reqs.size(); ++i) {
            const stitch_request& r = s.reqs[i].r;
            const stitch_homography_result& res = s.results[i];
            if (r.retry_hypotheses <= r.s5.hypotheses) continue;
            if (res.status == static_cast<int>(Status::OK) && res.num_inliers >= r.retry_min_inliers) continue;
            if (res.status == static_cast<int>(Status::INVALID_ARGUMENT) ||
                res.status == static_cast<int>(Status::NOT_ENOUGH_POINTS))
                continue;  // no saved search to extend
            const auto& o = s.plan->off[i];
            const auto& q = s.plan->pairs[i];
            const int k = q.s2.max_keypoints;
            auto at = [&](std::size_t off) { return ws + off; };
            const Keypoints ka{reinterpret_cast<float*>(at(o.kx[0])), reinterpret_cast<float*>(at(o.ky[0])),
                               reinterpret_cast<float*>(at(o.kr[0])), k, reinterpret_cast<int*>(at(o.kcount[0]))};
            const Keypoints kb{reinterpret_cast<float*>(at(o.kx[1])), reinterpret_cast<float*>(at(o.ky[1])),
                               reinterpret_cast<float*>(at(o.kr[1])), k, reinterpret_cast<int*>(at(o.kcount[1]))};
            const Matches m{reinterpret_cast<std::int32_t*>(at(o.ia)), reinterpret_cast<std::int32_t*>(at(o.ib)),
                            reinterpret_cast<float*>(at(o.dist)), k, reinterpret_cast<int*>(at(o.mcount))};
            s5::Config c = *reinterpret_cast<const s5::Config*>(&q.s5);
            c.previous_hypotheses = c.hypotheses;
            c.hypotheses = r.retry_hypotheses;
            const Status st = s5::estimate(ka, kb, m, *reinterpret_cast<const ScaleInfo*>(&q.scale_a),
                                           *reinterpret_cast<const ScaleInfo*>(&q.scale_b), c, at(o.mask),
                                           reinterpret_cast<HomographyResult*>(&s.results[i]), at(o.s5ws),
                                           b200::s5k::estimate_workspace_bytes(), s.stream);
            if (st != Status::OK) continue;  // keep the first result
            s.attempts[i] = 2;
            any = true;
        }
        if (any && cudaEventRecord(s.done, s.stream) != cudaSuccess) {
            cudaStreamSynchronize(s.stream);
            return false;
        }
        return any;
    }

    // After registration (and retries): the S6 feather panorama of every
    // request that asked for one, from its registered H in original
    // coordinates (src/s6/geometry.cpp:106-200, src/s6/s6.cu:328-380), on the
    // batch's resident RGB images, then copied to the caller's host buffers.
    // Returns true when work was enqueued.
    bool render(Slot& s) {
        bool any = false;
        auto* base = static_cast<unsigned char*>(cfg_.arena) + s.offset;
        s.panoramas.assign(s.reqs.size(), Panorama{});
        for (std::size_t i = 0; i < s.reqs.size(); ++i) {
            const Request& q = s.reqs[i];
            if (!q.render_bytes) continue;
            Panorama& pano = s.panoramas[i];
            const stitch_homography_result& res = s.results[i];
            if (res.status != static_cast<int>(Status::OK)) {
                pano.status = res.status;
                continue;
            }
            s6::GeometryPolicy policy;
            policy.max_canvas_pixels = std::min(policy.max_canvas_pixels, q.r.panorama_capacity);
            s6::Geometry g;
            Status st = s6::prepare_geometry(q.r.width_a, q.r.height_a, q.r.width_b, q.r.height_b, res.H, policy, &g);
            pano.status = static_cast<int>(st);
            if (st != Status::OK) continue;
            const std::size_t px = static_cast<std::size_t>(g.width) * static_cast<std::size_t>(g.height);
            unsigned char* out = base + s.render_off[i];
            unsigned char* mask = out + round_up(3 * q.r.panorama_capacity, kAlign);
            auto* counts = reinterpret_cast<s6::RenderStatistics*>(mask + round_up(q.r.panorama_capacity, kAlign));
            const ImageView a{base + s.host_off[2 * i], q.r.width_a, q.r.height_a, image_pitch(3 * q.r.width_a),
                              PixelFormat::RGB8};
            const ImageView b{base + s.host_off[2 * i + 1], q.r.width_b, q.r.height_b, image_pitch(3 * q.r.width_b),
                              PixelFormat::RGB8};
            const ImageView vo{out, g.width, g.height, 3 * g.width, PixelFormat::RGB8};
            const ImageView vm{mask, g.width, g.height, g.width, PixelFormat::GRAY8};
            st = s6::render(a, b, g, s6::BlendMode::Feather, vo, vm, nullptr, 0, s.stream, counts);
            if (st == Status::OK &&
                (cudaMemcpyAsync(q.r.host_panorama, out, 3 * px, cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
                 (q.r.host_mask &&
                  cudaMemcpyAsync(q.r.host_mask, mask, px, cudaMemcpyDeviceToHost, s.stream) != cudaSuccess) ||
                 cudaMemcpyAsync(s.render_counts + 2 * i, counts, sizeof(s6::RenderStatistics),
                                 cudaMemcpyDeviceToHost, s.stream) != cudaSuccess))
                st = Status::CUDA_ERROR;
            pano.status = static_cast<int>(st);
            if (st != Status::OK) continue;
            pano.width = g.width;
            pano.height = g.height;
            pano.origin_x = g.origin_x;
            pano.origin_y = g.origin_y;
            any = true;
        }
        if (any && cudaEventRecord(s.done, s.stream) != cudaSuccess) {
            cudaStreamSynchronize(s.stream);
            return false;
        }
        return any;
    }

    // Forms a batch from the head of the queue and launches it on slot s.
    bool launch(Slot& s) {
        if (pending_.empty()) return false;
        const std::size_t room = arena_.largest();
        std::size_t need = 0;
        int n = 0;
        while (n < static_cast<int>(pending_.size()) && n < cfg_.max_batch &&
               need + pending_[n].footprint + (64 << 10) <= room) {
            need += pending_[n].footprint;
            ++n;
        }
        if (n == 0) return false;  // the head waits for memory to free up
        for (; n > 0; --n) {
            // host-copied images, S1 outputs, the S1 job table, then the batch workspace
            std::vector<std::size_t> host_off(2 * n), reg_off(2 * n);
            std::size_t images = 0;
            int rgb_images = 0;
            for (int i = 0; i < n; ++i) {
                const Geometry& g = pending_[i].g;
                host_off[2 * i] = images;
                images += g.host_a;
                host_off[2 * i + 1] = images;
                images += g.host_b;
            }
            for (int i = 0; i < n; ++i) {
                const Geometry& g = pending_[i].g;
                if (!g.rgb) {
                    reg_off[2 * i] = host_off[2 * i];
                    reg_off[2 * i + 1] = host_off[2 * i + 1];
                    continue;
                }
                reg_off[2 * i] = images;
                images += g.work_a;
                reg_off[2 * i + 1] = images;
                images += g.work_b;
                rgb_images += 2;
            }
            const std::size_t s1_tables = images;
            if (rgb_images) images += round_up(s1_staging_bytes(), kAlign);
            std::vector<std::size_t> render_off(n, 0);
            for (int i = 0; i < n; ++i) {
                render_off[i] = images;
                images += pending_[i].render_bytes;
            }
            // lay out with placeholder addresses to size the region
            auto plan = std::make_unique<Plan>();
            std::vector<stitch_pair_desc> descs(n);
            const auto* base0 = reinterpret_cast<const unsigned char*>(kAlign);
            for (int i = 0; i < n; ++i)
                descs[i] = pair_desc(pending_[i], base0 + reg_off[2 * i], base0 + reg_off[2 * i + 1]);
            int bad = -1;
            if (plan->build(n, descs.data(), &bad, false) != Status::OK) {
                // a request that passed submit cannot fail here; drop the head
                s.reqs.assign(pending_.begin(), pending_.begin() + 1);
                pending_.pop_front();
                finish(s, Status::INVALID_ARGUMENT);
                return true;
            }
            if (plan->table_bytes > staging_cap()) continue;
            const std::size_t bytes = images + round_up(plan->total, kAlign);
            std::size_t off = 0;
            if (!arena_.alloc(bytes, &off)) continue;
            auto* base = static_cast<unsigned char*>(cfg_.arena) + off;
            for (int i = 0; i < n; ++i)
                descs[i] = pair_desc(pending_[i], base + reg_off[2 * i], base + reg_off[2 * i + 1]);
            plan = std::make_unique<Plan>();
            if (plan->build(n, descs.data(), &bad, false) != Status::OK) {
                arena_.release(off, bytes);
                return false;
            }
            plan->use_staging(s.staging);
            plan->matcher = matcher_;
            s.reqs.assign(pending_.begin(), pending_.begin() + n);
            pending_.erase(pending_.begin(), pending_.begin() + n);
            s.offset = off;
            s.bytes = bytes;
            s.ws_offset = images;
            s.attempts.assign(n, 1);
            s.host_off = host_off;
            s.render_off = render_off;
            s.launch_ms = now_ms();
            s.busy = true;
            Status st = Status::OK;
            // host -> device copies (RGB8 rows are 3 * width bytes)
            for (int i = 0; i < n && st == Status::OK; ++i) {
                const auto& r = s.reqs[i].r;
                const int ca = (s.reqs[i].g.rgb ? 3 : 1) * r.width_a, cb = (s.reqs[i].g.rgb ? 3 : 1) * r.width_b;
                if (cudaMemcpy2DAsync(base + host_off[2 * i], image_pitch(ca), r.host_a, r.pitch_a, ca, r.height_a,
                                      cudaMemcpyHostToDevice, s.stream) != cudaSuccess ||
                    cudaMemcpy2DAsync(base + host_off[2 * i + 1], image_pitch(cb), r.host_b, r.pitch_b, cb,
                                      r.height_b, cudaMemcpyHostToDevice, s.stream) != cudaSuccess)
                    st = Status::CUDA_ERROR;
            }
            // S1 for the RGB8 requests: one launch over all their images
            if (st == Status::OK && rgb_images) {
                auto* jobs = reinterpret_cast<b200::s1k::BatchJob*>(s.s1_staging);
                auto* prefix = reinterpret_cast<int*>(s.s1_staging + s1_jobs_bytes());
                int k = 0, blocks = 0;
                for (int i = 0; i < n && st == Status::OK; ++i) {
                    const Request& q = s.reqs[i];
                    if (!q.g.rgb) continue;
                    for (int side = 0; side < 2 && st == Status::OK; ++side) {
                        const int w = side ? q.r.width_b : q.r.width_a, h = side ? q.r.height_b : q.r.height_a;
                        const ImageView in{base + host_off[2 * i + side], w, h, image_pitch(3 * w), PixelFormat::RGB8};
                        const stitch_scale_info& si = side ? q.g.sb : q.g.sa;
                        const ImageView out{base + reg_off[2 * i + side], si.work_w, si.work_h, image_pitch(si.work_w),
                                            PixelFormat::GRAY8};
                        st = b200::s1k::batch_job(in, out, *reinterpret_cast<const ScaleInfo*>(&si), &jobs[k]);
                        prefix[k] = blocks;
                        blocks += jobs[k].tiles;
                        ++k;
                    }
                }
                prefix[k] = blocks;
                auto* djobs = base + s1_tables;
                if (st == Status::OK &&
                    cudaMemcpyAsync(djobs, s.s1_staging, s1_staging_bytes(), cudaMemcpyHostToDevice, s.stream) !=
                        cudaSuccess)
                    st = Status::CUDA_ERROR;
                if (st == Status::OK)
                    st = b200::s1k::batch_enqueue(reinterpret_cast<const b200::s1k::BatchJob*>(djobs),
                                                  reinterpret_cast<const int*>(djobs + s1_jobs_bytes()), k, blocks,
                                                  s.stream);
            }
            if (st == Status::OK) st = plan->enqueue(base + images, bytes - images, s.results, s.stream);
            if (st == Status::OK && cudaEventRecord(s.done, s.stream) != cudaSuccess) st = Status::CUDA_ERROR;
            s.plan = std::move(plan);
            if (st != Status::OK) {
                cudaStreamSynchronize(s.stream);
                finish(s, st);
            }
            return true;
        }
        return false;
    }

    void loop() {
        cudaSetDevice(cfg_.device);
        for (;;) {
            bool busy = false;
            {
                std::unique_lock<std::mutex> g(mu_);
                for (const auto& s : slots_) busy |= s.busy;
                if (incoming_.empty() && pending_.empty() && !busy) {
                    if (stopping_) return;
                    cv_.wait(g, [&] { return stopping_ || !incoming_.empty(); });
                }
                while (!incoming_.empty()) {
                    pending_.push_back(incoming_.front());
                    incoming_.pop_front();
                }
            }
            bool progressed = false;
            for (auto& s : slots_) {
                if (s.busy && cudaEventQuery(s.done) == cudaSuccess) {
                    progressed = true;
                    if (s.phase == 0) {
                        s.phase = 1;
                        if (retry(s)) continue;
                    }
                    if (s.phase == 1) {
                        s.phase = 2;
                        if (render(s)) continue;
                    }
                    finish(s, Status::OK);
                }
            }
            for (auto& s : slots_) {
                if (!s.busy && launch(s)) progressed = true;
            }
            if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }

    stitch_server_config cfg_;
    int matcher_ = s4k::kMatcherTensor;  // S4 matcher of every plan this server builds
    Arena arena_;
    std::chrono::steady_clock::time_point t0_;
    std::vector<Slot> slots_;
    std::deque<Request> pending_;  // dispatcher thread only
    std::thread worker_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Request> incoming_;             // guarded by mu_
    std::vector<stitch_server_result> done_;   // guarded by mu_
    int outstanding_ = 0;                      // guarded by mu_
    bool stopping_ = false;                    // guarded by mu_
};

}  // namespace stitch::b200::serve

using stitch::Status;
using stitch::b200::serve::Server;

struct stitch_server {
    std::unique_ptr<Server> impl;
};

extern "C" {

int stitch_server_create(const stitch_server_config* config, stitch_server** out) {
    if (!config || !out || !config->arena || config->arena_bytes == 0 ||
        reinterpret_cast<std::uintptr_t>(config->arena) % 256 != 0 || config->max_batch < 0 || config->streams < 0)
        return static_cast<int>(Status::INVALID_ARGUMENT);
    *out = nullptr;
    stitch_server_config c = *config;
    if (c.max_batch == 0) c.max_batch = 64;
    if (c.streams == 0) c.streams = 2;
    auto* s = new (std::nothrow) stitch_server;
    if (!s) return static_cast<int>(Status::CUDA_ERROR);
    s->impl = std::make_unique<Server>(c);
    const Status st = s->impl->start();
    if (st != Status::OK) {
        delete s;
        return static_cast<int>(st);
    }
    *out = s;
    return 0;
}

int stitch_server_request_bytes(const stitch_request* r, size_t* bytes) {
    if (!r || !bytes) return static_cast<int>(Status::INVALID_ARGUMENT);
    stitch::b200::serve::Request q;
    std::size_t table_bytes = 0;
    const Status st = stitch::b200::serve::prepare_request(*r, &q, &table_bytes);
    *bytes = st == Status::OK ? q.footprint : 0;
    return static_cast<int>(st);
}

int stitch_server_submit(stitch_server* s, const stitch_request* r) {
    if (!s || !r) return static_cast<int>(Status::INVALID_ARGUMENT);
    return static_cast<int>(s->impl->submit(*r));
}

int stitch_server_poll(stitch_server* s, stitch_server_result* out, int max, int* count) {
    if (!s || !count || max < 0 || (max > 0 && !out)) return static_cast<int>(Status::INVALID_ARGUMENT);
    *count = s->impl->poll(out, max);
    return 0;
}

int stitch_server_outstanding(stitch_server* s) { return s ? s->impl->outstanding() : -1; }

void stitch_server_destroy(stitch_server* s) { delete s; }

}  // extern "C"
