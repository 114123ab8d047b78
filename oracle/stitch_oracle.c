/* CPU oracle for S4 (exact Hamming / L2 top-2, ratio test, compaction),
 * S5 (MSAC homography with counter-based sampling and refinement), S1
 * (integer gray and area resize) and S6 (canvas geometry, feather render).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA stages are compared against.
 * The product library never links this file.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp -shared -fPIC (oracle/Makefile).
 * -ffp-contract=off keeps every product and sum separately rounded, which is
 * the arithmetic the reference's host tests use for src/s5/s5_math.hpp.
 *
 * Reference semantics restated here, by file:line of the reference tree:
 *   S4 top-2 ......... src/s4/s4.cu:115-135 (insert/before: lower index wins,
 *                      second neighbour is a distinct index), :141-200 (byte
 *                      popcount summed as double; L2 as sum of rounded squares
 *                      in dimension order), tests/test_s4_cuda.cu:60-94
 *   S4 accept ........ src/s4/s4.cu:212-239 (second exists and
 *                      d1 == 0 ? d2 > 0 : d1 < ratio * d2; mutual check)
 *   S4 compaction .... src/s4/s4.cu:241-262 (query order, sqrt for L2, +inf
 *                      above FLT_MAX)
 *   S5 math .......... src/s5/s5_math.hpp:98-263 (finite, multiply, normalize,
 *                      residual_squared, SplitMix64 random_word, sample_four,
 *                      nondegenerate_four, fit, valid_domain)
 *   S5 search ........ src/s5/s5.cu:42-132 (prepare, generate, 128-lane
 *                      strided MSAC loss with a tree reduction, select_best)
 *   S5 finish ........ src/s5/s5.cu:139-212 (serial re-score, refinement
 *                      accepted only on a strictly lower loss, inlier mask
 *                      r^2 <= tau^2, telemetry, H = D_A^-1 H_s D_B)
 *   geometry ......... src/common/geometry.hpp:119-163
 *   S1 ............... src/s1/s1.cu:33-205
 *   S6 ............... src/s6/geometry.cpp:10-198, src/s6/s6.cu:147-215
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O_OK 0
#define O_INVALID_ARGUMENT 1
#define O_NOT_ENOUGH_POINTS 4
#define O_DEGENERATE 5

/* ------------------------------------------------------------------ S4 */

typedef struct {
    double first_distance, second_distance;
    int first_index, second_index;
} o_top2;

/* (d, i) precedes (e, j): lower distance, then lower index; missing entries
 * (index < 0) come last. */
static int precedes(double d, int i, double e, int j) {
    if (i < 0) return 0;
    if (j < 0) return 1;
    return d < e || (d == e && i < j);
}

static void top2_push(o_top2* t, double d, int i) {
    if (i < 0 || i == t->first_index || i == t->second_index) return;
    if (precedes(d, i, t->first_distance, t->first_index)) {
        t->second_distance = t->first_distance;
        t->second_index = t->first_index;
        t->first_distance = d;
        t->first_index = i;
    } else if (precedes(d, i, t->second_distance, t->second_index)) {
        t->second_distance = d;
        t->second_index = i;
    }
}

static o_top2 top2_empty(void) {
    o_top2 t = {INFINITY, INFINITY, -1, -1};
    return t;
}

/* type 0: bytes, Hamming; type 1: float32, squared L2. Rows [0, count) are
 * active; output has capacity_a rows. Counts outside [0, capacity] give all
 * rows empty, as the device path does. */
void oracle_s4_top2(int type, const void* a, int capacity_a, int count_a, int stride_a,
                    const void* b, int capacity_b, int count_b, int stride_b, int dim,
                    o_top2* out) {
    const int valid = count_a >= 0 && count_a <= capacity_a && count_b >= 0 && count_b <= capacity_b;
#pragma omp parallel for schedule(static)
    for (int q = 0; q < capacity_a; ++q) {
        o_top2 t = top2_empty();
        if (valid && q < count_a) {
            const unsigned char* qa = (const unsigned char*)a + (size_t)q * stride_a;
            for (int r = 0; r < count_b; ++r) {
                const unsigned char* rb = (const unsigned char*)b + (size_t)r * stride_b;
                double d = 0.0;
                if (type == 0) {
                    for (int k = 0; k < dim; ++k) d += (double)__builtin_popcount(qa[k] ^ rb[k]);
                } else {
                    const float* fa = (const float*)qa;
                    const float* fb = (const float*)rb;
                    for (int k = 0; k < dim; ++k) {
                        const double delta = (double)fa[k] - (double)fb[k];
                        d = d + delta * delta;
                    }
                }
                top2_push(&t, d, r);
            }
        }
        out[q] = t;
    }
}

/* Ratio test + optional mutual check + compaction in query order. Returns the
 * number of matches written. reverse may be NULL. */
int oracle_s4_accept(const o_top2* forward, int capacity_a, const o_top2* reverse,
                     double ratio_threshold, int l2, int32_t* idx_a, int32_t* idx_b,
                     float* distance) {
    const double ratio = l2 ? ratio_threshold * ratio_threshold : ratio_threshold;
    int n = 0;
    for (int q = 0; q < capacity_a; ++q) {
        const o_top2 p = forward[q];
        int ok = p.second_index >= 0 &&
                 (p.first_distance == 0 ? p.second_distance > 0
                                        : p.first_distance < ratio * p.second_distance);
        if (ok && reverse) ok = reverse[p.first_index].first_index == q;
        if (!ok) continue;
        idx_a[n] = q;
        idx_b[n] = p.first_index;
        const double d = l2 ? sqrt(p.first_distance) : p.first_distance;
        distance[n] = d > FLT_MAX ? INFINITY : (float)d;
        ++n;
    }
    return n;
}

/* ------------------------------------------------------------------ S5 */

typedef struct {
    double ax, ay, bx, by;
} o_point;

static int fin(double x) { return x == x && x <= DBL_MAX && x >= -DBL_MAX; }

static void mat3_mul(const double* a, const double* b, double* out) {
    double t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            t[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[j + 3] + a[3 * i + 2] * b[j + 6];
    memcpy(out, t, sizeof(t));
}

/* Scales by the largest magnitude; requires finite entries and |det| > 1e-15. */
static int h_normalize(double* h) {
    double scale = 0.0;
    for (int i = 0; i < 9; ++i) {
        if (!fin(h[i])) return 0;
        if (fabs(h[i]) > scale) scale = fabs(h[i]);
    }
    if (!(scale > 0.0)) return 0;
    for (int i = 0; i < 9; ++i) h[i] /= scale;
    const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                       h[2] * (h[3] * h[7] - h[4] * h[6]);
    return fin(det) && fabs(det) > 1e-15;
}

/* Forward B -> A reprojection error squared; DBL_MAX for a bad denominator. */
double oracle_residual2(const double* h, double ax, double ay, double bx, double by) {
    const double z = h[6] * bx + h[7] * by + h[8];
    if (!fin(z) || fabs(z) < 1e-15) return DBL_MAX;
    const double dx = (h[0] * bx + h[1] * by + h[2]) / z - ax;
    const double dy = (h[3] * bx + h[4] * by + h[5]) / z - ay;
    const double r = dx * dx + dy * dy;
    return fin(r) ? r : DBL_MAX;
}

/* SplitMix64 finaliser applied to a counter (public-domain algorithm by
 * Sebastiano Vigna). */
uint64_t oracle_splitmix64(uint64_t v) {
    v += 0x9e3779b97f4a7c15ULL;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
    return v ^ (v >> 31);
}

/* Four distinct indices in [0, n) for hypothesis h: draw k uses counter
 * seed ^ (4h + k), reduced mod (n - k), then skips over the already drawn
 * indices in ascending order. */
void oracle_sample_four(int n, uint64_t seed, int h, int* out) {
    for (int k = 0; k < 4; ++k) {
        int v = (int)(oracle_splitmix64(seed ^ ((uint64_t)h * 4 + (uint64_t)k)) % (uint64_t)(n - k));
        int sorted[4];
        for (int i = 0; i < k; ++i) sorted[i] = out[i];
        for (int i = 1; i < k; ++i)
            for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; --j) {
                const int t = sorted[j]; sorted[j] = sorted[j - 1]; sorted[j - 1] = t;
            }
        for (int i = 0; i < k; ++i)
            if (v >= sorted[i]) ++v;
        out[k] = v;
    }
}

static double coord(const o_point* p, int image, int axis) {
    return image ? (axis ? p->by : p->bx) : (axis ? p->ay : p->ax);
}

static int nondegenerate(const o_point* p) {
    for (int image = 0; image < 2; ++image) {
        double scale = 0.0;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < i; ++j) {
                const double dx = coord(&p[i], image, 0) - coord(&p[j], image, 0);
                const double dy = coord(&p[i], image, 1) - coord(&p[j], image, 1);
                const double d = dx * dx + dy * dy;
                if (d > scale) scale = d;
            }
        if (!(scale > 0.0) || !fin(scale)) return 0;
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j)
                for (int k = j + 1; k < 4; ++k) {
                    const double x1 = coord(&p[j], image, 0) - coord(&p[i], image, 0);
                    const double y1 = coord(&p[j], image, 1) - coord(&p[i], image, 1);
                    const double x2 = coord(&p[k], image, 0) - coord(&p[i], image, 0);
                    const double y2 = coord(&p[k], image, 1) - coord(&p[i], image, 1);
                    if (fabs(x1 * y2 - y1 * x2) <= 1e-8 * scale) return 0;
                }
    }
    return 1;
}

/* Normalised 8-unknown least squares (h33 = 1) over the points with
 * keep[i] != 0 (keep == NULL keeps all), Gauss-Jordan with partial pivoting,
 * then denormalised and scaled by its largest entry. */
static int fit(int n, const o_point* pts, const unsigned char* keep, double* out) {
    double cax = 0, cay = 0, cbx = 0, cby = 0;
    int count = 0;
    for (int i = 0; i < n; ++i) {
        if (keep && !keep[i]) continue;
        cax += pts[i].ax; cay += pts[i].ay; cbx += pts[i].bx; cby += pts[i].by;
        ++count;
    }
    if (count < 4) return 0;
    cax /= count; cay /= count; cbx /= count; cby /= count;
    double va = 0.0, vb = 0.0;
    for (int i = 0; i < n; ++i) {
        if (keep && !keep[i]) continue;
        const o_point p = pts[i];
        va += (p.ax - cax) * (p.ax - cax) + (p.ay - cay) * (p.ay - cay);
        vb += (p.bx - cbx) * (p.bx - cbx) + (p.by - cby) * (p.by - cby);
    }
    if (!(va > 0.0) || !(vb > 0.0) || !fin(va) || !fin(vb)) return 0;
    const double sa = sqrt(2.0 * count / va);
    const double sb = sqrt(2.0 * count / vb);
    double m[8][9];
    memset(m, 0, sizeof(m));
    for (int i = 0; i < n; ++i) {
        if (keep && !keep[i]) continue;
        const o_point p = pts[i];
        const double x = (p.bx - cbx) * sb, y = (p.by - cby) * sb;
        const double u = (p.ax - cax) * sa, v = (p.ay - cay) * sa;
        const double r0[9] = {x, y, 1, 0, 0, 0, -u * x, -u * y, u};
        const double r1[9] = {0, 0, 0, x, y, 1, -v * x, -v * y, v};
        for (int r = 0; r < 8; ++r)
            for (int c = 0; c < 9; ++c) m[r][c] += r0[r] * r0[c] + r1[r] * r1[c];
    }
    double max_entry = 0.0;
    for (int i = 0; i < 8; ++i)
        if (fabs(m[i][i]) > max_entry) max_entry = fabs(m[i][i]);
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        for (int r = c + 1; r < 8; ++r)
            if (fabs(m[r][c]) > fabs(m[piv][c])) piv = r;
        if (!fin(m[piv][c]) || fabs(m[piv][c]) <= 1e-12 * max_entry) return 0;
        for (int j = c; j < 9; ++j) {
            const double t = m[c][j]; m[c][j] = m[piv][j]; m[piv][j] = t;
        }
        const double div = m[c][c];
        for (int j = c; j < 9; ++j) m[c][j] /= div;
        for (int r = 0; r < 8; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
            for (int j = c; j < 9; ++j) m[r][j] -= f * m[c][j];
        }
    }
    double h[9];
    for (int i = 0; i < 8; ++i) h[i] = m[i][8];
    h[8] = 1.0;
    const double den_a[9] = {1.0 / sa, 0, cax, 0, 1.0 / sa, cay, 0, 0, 1};
    const double nrm_b[9] = {sb, 0, -sb * cbx, 0, sb, -sb * cby, 0, 0, 1};
    double tmp[9];
    mat3_mul(den_a, h, tmp);
    mat3_mul(tmp, nrm_b, out);
    return h_normalize(out);
}

/* The projective denominator keeps one sign, away from zero, on the corners
 * of a width x height frame. */
static int valid_domain(const double* h, int width, int height) {
    const double z[4] = {h[8], h[6] * (width - 1) + h[8], h[7] * (height - 1) + h[8],
                         h[6] * (width - 1) + h[7] * (height - 1) + h[8]};
    for (int i = 0; i < 4; ++i)
        if (!fin(z[i]) || fabs(z[i]) < 1e-15 || (z[i] > 0.0) != (z[0] > 0.0)) return 0;
    return 1;
}

/* Exported for host-side numerical tests. */
int oracle_fit(int n, const double* pts4, const unsigned char* keep, double* out) {
    return fit(n, (const o_point*)pts4, keep, out);
}
int oracle_nondegenerate(const double* pts4) { return nondegenerate((const o_point*)pts4); }
int oracle_valid_domain(const double* h, int w, int hgt) { return valid_domain(h, w, hgt); }
int oracle_mat3_inverse(const double* m, double* out) {
    const double c00 = m[4] * m[8] - m[5] * m[7];
    const double c01 = m[5] * m[6] - m[3] * m[8];
    const double c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (fabs(det) < 1e-300) return 0;
    const double inv = 1.0 / det;
    const double r[9] = {c00 * inv, (m[2] * m[7] - m[1] * m[8]) * inv, (m[1] * m[5] - m[2] * m[4]) * inv,
                         c01 * inv, (m[0] * m[8] - m[2] * m[6]) * inv, (m[2] * m[3] - m[0] * m[5]) * inv,
                         c02 * inv, (m[1] * m[6] - m[0] * m[7]) * inv, (m[0] * m[4] - m[1] * m[3]) * inv};
    memcpy(out, r, sizeof(r));
    return 1;
}

typedef struct {
    double h[9];
    double loss;
    int hypothesis;
    int valid;
} o_model;

typedef struct {
    double H[9];
    double H_s[9];
    int num_matches;
    int num_inliers;
    double inlier_ratio;
    double inlier_coverage;
    double reproj_residual;
    int status;
} o_result;

/* MSAC loss of one hypothesis in the device's summation order: 128 lanes,
 * lane l sums terms l, l+128, ... in index order, then a halving tree. */
static double tree_loss(int nm, const o_point* pts, const double* h, double thr2) {
    double lane[128];
    for (int l = 0; l < 128; ++l) {
        double v = 0.0;
        for (int i = l; i < nm; i += 128) {
            const double r = oracle_residual2(h, pts[i].ax, pts[i].ay, pts[i].bx, pts[i].by);
            v += r < thr2 ? r : thr2;
        }
        lane[l] = v;
    }
    for (int s = 64; s > 0; s /= 2)
        for (int l = 0; l < s; ++l) lane[l] += lane[l + s];
    return lane[0];
}

static double serial_loss(int nm, const o_point* pts, const double* h, double thr2) {
    double v = 0.0;
    for (int i = 0; i < nm; ++i) {
        const double r = oracle_residual2(h, pts[i].ax, pts[i].ay, pts[i].bx, pts[i].by);
        v += r < thr2 ? r : thr2;
    }
    return v;
}

static int better(const o_model* a, const o_model* b) {
    return a->valid && (!b->valid || a->loss < b->loss ||
                        (a->loss == b->loss && a->hypothesis < b->hypothesis));
}

/* Evaluates hypotheses [first, last) and folds them into *best (in/out,
 * zero-initialise for a fresh search). pts holds the nm matched points. */
void oracle_s5_search(int nm, const double* pts4, uint64_t seed, int first, int last,
                      int b_work_w, int b_work_h, double threshold, o_model* best) {
    const o_point* pts = (const o_point*)pts4;
    const double thr2 = threshold * threshold;
    const int count = last - first;
    if (count <= 0) return;
    o_model* models = (o_model*)calloc((size_t)count, sizeof(o_model));
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < count; ++k) {
        o_model m;
        memset(&m, 0, sizeof(m));
        m.hypothesis = first + k;
        int idx[4];
        oracle_sample_four(nm, seed, m.hypothesis, idx);
        o_point f[4];
        for (int j = 0; j < 4; ++j) f[j] = pts[idx[j]];
        m.valid = nondegenerate(f) && fit(4, f, NULL, m.h) && valid_domain(m.h, b_work_w, b_work_h);
        if (m.valid) {
            m.loss = tree_loss(nm, pts, m.h, thr2);
            if (!fin(m.loss)) m.valid = 0;
        }
        models[k] = m;
    }
    for (int k = 0; k < count; ++k)
        if (better(&models[k], best)) *best = models[k];
    free(models);
}

/* The reference's finish step: refine the raw winner, build mask and
 * telemetry, map to original coordinates. status_in is the search status
 * (OK, INVALID_ARGUMENT or NOT_ENOUGH_POINTS). inverse_a = D_A^-1 and d_b = D_B
 * are computed by the caller (oracle_mat3_inverse). */
void oracle_s5_finish(int nm, const double* pts4, int mask_capacity, const o_model* best,
                      int status_in, int refinement_steps, double threshold,
                      int a_work_w, int a_work_h, int b_work_w, int b_work_h,
                      int b_orig_w, int b_orig_h, const double* inverse_a, const double* d_b,
                      unsigned char* mask, o_result* out) {
    const o_point* pts = (const o_point*)pts4;
    o_result r;
    memset(&r, 0, sizeof(r));
    const double nanv = nan("");
    for (int i = 0; i < 9; ++i) r.H[i] = r.H_s[i] = nanv;
    r.reproj_residual = nanv;
    r.num_matches = (nm >= 0 && nm <= mask_capacity) ? nm : 0;
    r.status = status_in;
    for (int i = 0; i < mask_capacity; ++i) mask[i] = 0;
    if (r.status == O_OK && !best->valid) r.status = O_DEGENERATE;
    if (r.status == O_OK) {
        const double thr2 = threshold * threshold;
        o_model model = *best;
        model.loss = serial_loss(nm, pts, model.h, thr2);
        unsigned char* keep = (unsigned char*)malloc((size_t)(nm > 0 ? nm : 1));
        for (int step = 0; step < refinement_steps; ++step) {
            for (int i = 0; i < nm; ++i)
                keep[i] = oracle_residual2(model.h, pts[i].ax, pts[i].ay, pts[i].bx, pts[i].by) <= thr2;
            o_model cand;
            memset(&cand, 0, sizeof(cand));
            cand.valid = fit(nm, pts, keep, cand.h) && valid_domain(cand.h, b_work_w, b_work_h);
            if (!cand.valid) break;
            cand.loss = serial_loss(nm, pts, cand.h, thr2);
            if (!fin(cand.loss) || !(cand.loss < model.loss)) break;
            model = cand;
        }
        free(keep);
        double minx = DBL_MAX, miny = DBL_MAX, maxx = -DBL_MAX, maxy = -DBL_MAX, sum = 0.0;
        for (int i = 0; i < nm; ++i) {
            const double e = oracle_residual2(model.h, pts[i].ax, pts[i].ay, pts[i].bx, pts[i].by);
            if (e > thr2) continue;
            mask[i] = 1;
            ++r.num_inliers;
            sum += e;
            minx = fmin(minx, pts[i].ax); maxx = fmax(maxx, pts[i].ax);
            miny = fmin(miny, pts[i].ay); maxy = fmax(maxy, pts[i].ay);
        }
        if (r.num_inliers < 4) {
            r.status = O_DEGENERATE;
            for (int i = 0; i < mask_capacity; ++i) mask[i] = 0;
            r.num_inliers = 0;
        } else {
            r.inlier_ratio = (double)r.num_inliers / nm;
            r.reproj_residual = sqrt(sum / r.num_inliers);
            const double w = fmax(1.0, (double)(a_work_w - 1));
            const double h = fmax(1.0, (double)(a_work_h - 1));
            r.inlier_coverage = fmin(1.0, (maxx - minx) / w) * fmin(1.0, (maxy - miny) / h);
            for (int i = 0; i < 9; ++i) r.H_s[i] = model.h[i];
            double tmp[9];
            mat3_mul(inverse_a, model.h, tmp);
            mat3_mul(tmp, d_b, r.H);
            if (!h_normalize(r.H) || !valid_domain(r.H, b_orig_w, b_orig_h)) {
                r.status = O_DEGENERATE;
                for (int i = 0; i < mask_capacity; ++i) mask[i] = 0;
                r.num_inliers = 0;
                r.inlier_ratio = r.inlier_coverage = 0.0;
                r.reproj_residual = nanv;
                for (int i = 0; i < 9; ++i) r.H[i] = r.H_s[i] = nanv;
            }
        }
    }
    *out = r;
}

/* make_scale_info: working size lround(w * s) (at least 1), half-pixel D. */
int oracle_make_scale_info(int w, int h, double s, int* work_wh, double* sxy, double* d) {
    if (w <= 0 || h <= 0 || !(s > 0.0) || s > 1.0) return O_INVALID_ARGUMENT;
    long ww = lround((double)w * s), wh = lround((double)h * s);
    if (ww < 1) ww = 1;
    if (wh < 1) wh = 1;
    work_wh[0] = (int)ww;
    work_wh[1] = (int)wh;
    sxy[0] = (double)ww / w;
    sxy[1] = (double)wh / h;
    const double dd[9] = {sxy[0], 0, 0.5 * (sxy[0] - 1.0), 0, sxy[1], 0.5 * (sxy[1] - 1.0), 0, 0, 1};
    memcpy(d, dd, sizeof(dd));
    return O_OK;
}

/* ---------------------------------------------------------------- S1
 * src/s1/s1.cu:33-107, :116-141: 15-bit integer gray; S = 1 direct; exact
 * 2x2 ((sum + 2) >> 2) and 4x4 (float sum * 0.0625, round half to even)
 * averages; otherwise a float box filter whose weighted sum the reference's
 * nvcc build accumulates with a fused multiply-add (total += g * (wx * wy)),
 * restated with C99 fmaf. */
static int s1_gray(const uint8_t* p) { return (9798 * p[0] + 19235 * p[1] + 3735 * p[2] + 16384) >> 15; }

void oracle_s1(const uint8_t* rgb, int w, int h, int pitch, int work_w, int work_h, uint8_t* out) {
    const float inv_sx = (float)w / (float)work_w, inv_sy = (float)h / (float)work_h;
    const float scale_area = 1.0f / (inv_sx * inv_sy);
    const int mode = (w == work_w && h == work_h) ? 0
                     : (w == 2 * work_w && h == 2 * work_h) ? 1
                     : (w == 4 * work_w && h == 4 * work_h) ? 2 : 3;
    for (int yd = 0; yd < work_h; ++yd) {
        for (int xd = 0; xd < work_w; ++xd) {
            int v;
            if (mode == 0) {
                v = s1_gray(rgb + (size_t)yd * pitch + 3 * xd);
            } else if (mode == 1) {
                const uint8_t* r0 = rgb + (size_t)(2 * yd) * pitch + 6 * xd;
                const uint8_t* r1 = r0 + pitch;
                v = (s1_gray(r0) + s1_gray(r0 + 3) + s1_gray(r1) + s1_gray(r1 + 3) + 2) >> 2;
            } else if (mode == 2) {
                int sum = 0;
                for (int dy = 0; dy < 4; ++dy)
                    for (int dx = 0; dx < 4; ++dx) sum += s1_gray(rgb + (size_t)(4 * yd + dy) * pitch + 12 * xd + 3 * dx);
                v = (int)nearbyintf((float)sum * 0.0625f);
            } else {
                const float fsy1 = (float)yd * inv_sy, fsy2 = (float)(yd + 1) * inv_sy;
                const float fsx1 = (float)xd * inv_sx, fsx2 = (float)(xd + 1) * inv_sx;
                const int y0 = (int)floorf(fsy1), y1 = (int)ceilf(fsy2);
                const int x0 = (int)floorf(fsx1), x1 = (int)ceilf(fsx2);
                float total = 0.0f;
                for (int ys = y0; ys < y1 && ys < h; ++ys) {
                    const float wy = fmaxf(0.0f, fminf((float)(ys + 1), fsy2) - fmaxf((float)ys, fsy1));
                    if (wy <= 0.0f) continue;
                    for (int xs = x0; xs < x1 && xs < w; ++xs) {
                        const float wx = fmaxf(0.0f, fminf((float)(xs + 1), fsx2) - fmaxf((float)xs, fsx1));
                        if (wx <= 0.0f) continue;
                        const float ww = wx * wy;
                        total = fmaf((float)s1_gray(rgb + (size_t)ys * pitch + 3 * xs), ww, total);
                    }
                }
                v = (int)nearbyintf(total * scale_area);
            }
            out[(size_t)yd * work_w + xd] = (uint8_t)v;
        }
    }
}

/* src/s1/s1.cu:147-205: (sum |I(x+1,y) - I(x,y)| + sum |I(x,y+1) - I(x,y)|)
 * / (255 (h (w-1) + w (h-1))). */
double oracle_s1_gradient(const uint8_t* g, int w, int h, int pitch) {
    unsigned long long sum = 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const int c = g[(size_t)y * pitch + x];
            if (x + 1 < w) sum += (unsigned long long)abs(g[(size_t)y * pitch + x + 1] - c);
            if (y + 1 < h) sum += (unsigned long long)abs(g[(size_t)(y + 1) * pitch + x] - c);
        }
    const unsigned long long edges = (unsigned long long)h * (w - 1) + (unsigned long long)w * (h - 1);
    return edges ? (double)sum / (255.0 * (double)edges) : 0.0;
}

/* ---------------------------------------------------------------- S6
 * Geometry (src/s6/geometry.cpp:10-198) in x87 80-bit long double, the type
 * the reference's host build computes in: H scaled by its largest entry; the
 * four B corners on one side of the horizon with |w| above
 * denominator_tolerance * (|h6| (wb-1) + |h7| (hb-1) + |h8|); the inclusive
 * canvas floor(min) .. ceil(max) over A's pixel centres and B's projected
 * corners, each end snapped to an integer within
 * max(snap_tolerance, 16 eps max(1, |x|)); the pixel budget; the inverse
 * through size-normalised coordinates (A and B centred and divided by
 * max(1, w-1, h-1)), Gauss-Jordan with scaled partial pivoting, pivot score
 * and ||M||inf ||M^-1||inf checked against inverse_tolerance; the A -> B
 * inverse scaled by its largest entry.
 * Feather (src/s6/s6.cu:147-215), per canvas pixel, double arithmetic with
 * every product and sum rounded on its own: A sampled at the pixel, B through
 * the inverse when |den| > denominator_tolerance * den_scale; bilinear
 * interpolation of the pixel-centre grid (coordinates snapped as above),
 * converted to float after / 255; distance-to-edge scores; the score-weighted
 * mean where both cover the pixel; floor(clamp(255 c, 0, 255) + 0.5). */
typedef struct {
    double den_tol, inv_tol, snap_tol;
    size_t max_pixels;
} o_s6_policy;
typedef struct {
    int w, h, ox, oy, wa, ha, wb, hb;
    double den_tol, snap_tol;
    double inv[9];
} o_s6_geom;

typedef long double o_real;

static int lfin(o_real x) { return isfinite(x); }
static o_real lmaxr(o_real a, o_real b) { return a > b ? a : b; }

static void lmul3(const o_real* a, const o_real* b, o_real* out) {
    o_real t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            o_real s = 0;
            for (int k = 0; k < 3; ++k) s += a[3 * r + k] * b[3 * k + c];
            t[3 * r + c] = s;
        }
    memcpy(out, t, sizeof(t));
}

static int lscale(o_real* m) {
    o_real big = 0;
    for (int i = 0; i < 9; ++i) {
        if (!lfin(m[i])) return 0;
        big = lmaxr(big, fabsl(m[i]));
    }
    if (big == 0) return 0;
    for (int i = 0; i < 9; ++i) m[i] /= big;
    return 1;
}

static o_real linf(const o_real* m) {
    o_real n = 0;
    for (int r = 0; r < 3; ++r) {
        o_real s = 0;
        for (int c = 0; c < 3; ++c) s += fabsl(m[3 * r + c]);
        n = lmaxr(n, s);
    }
    return n;
}

static int linvert(const o_real* m, o_real tol, o_real* inv) {
    o_real a[3][6], rs[3];
    memset(a, 0, sizeof(a));
    for (int r = 0; r < 3; ++r) {
        rs[r] = 0;
        for (int c = 0; c < 3; ++c) {
            a[r][c] = m[3 * r + c];
            rs[r] = lmaxr(rs[r], fabsl(a[r][c]));
        }
        if (rs[r] == 0) return 0;
        a[r][3 + r] = 1;
    }
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        o_real best = 0;
        for (int r = col; r < 3; ++r) {
            const o_real sc = fabsl(a[r][col]) / rs[r];
            if (sc > best) {
                best = sc;
                piv = r;
            }
        }
        if (!lfin(best) || best <= tol) return 0;
        if (piv != col) {
            for (int c = 0; c < 6; ++c) {
                const o_real t = a[piv][c];
                a[piv][c] = a[col][c];
                a[col][c] = t;
            }
            const o_real t = rs[piv];
            rs[piv] = rs[col];
            rs[col] = t;
        }
        const o_real d = a[col][col];
        for (int c = 0; c < 6; ++c) a[col][c] /= d;
        for (int r = 0; r < 3; ++r) {
            if (r == col) continue;
            const o_real f = a[r][col];
            for (int c = 0; c < 6; ++c) a[r][c] -= f * a[col][c];
        }
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            if (!lfin(a[r][3 + c])) return 0;
            inv[3 * r + c] = a[r][3 + c];
        }
    const o_real cond = linf(m) * linf(inv);
    return lfin(cond) && cond * tol < 1;
}

static o_real lsnap(o_real x, double snap_tol) {
    const o_real near = roundl(x);
    const o_real floor_tol = 16 * (o_real)DBL_EPSILON * lmaxr(1, fabsl(x));
    return fabsl(x - near) <= lmaxr((o_real)snap_tol, floor_tol) ? near : x;
}

#define O_INSUFFICIENT_WORKSPACE 2

int oracle_s6_geometry(int wa, int ha, int wb, int hb, const double* h, const o_s6_policy* p, o_s6_geom* out) {
    o_real m[9];
    for (int i = 0; i < 9; ++i) m[i] = h ? h[i] : 0;
    memset(out, 0, sizeof(*out));
    out->den_tol = 1e-12;
    out->snap_tol = 1e-10;
    const int policy_ok = isfinite(p->den_tol) && p->den_tol > 0 && p->den_tol < 1 && isfinite(p->inv_tol) &&
                          p->inv_tol > 0 && p->inv_tol < 1 && isfinite(p->snap_tol) && p->snap_tol >= 0 &&
                          p->snap_tol < 0.5 && p->max_pixels > 0;
    if (!h || wa <= 0 || ha <= 0 || wb <= 0 || hb <= 0 || !policy_ok) return O_INVALID_ARGUMENT;
    if (!lscale(m)) return O_DEGENERATE;
    const o_real bx = (o_real)wb - 1, by = (o_real)hb - 1;
    const o_real dscale = fabsl(m[6]) * bx + fabsl(m[7]) * by + fabsl(m[8]);
    if (!(dscale > 0) || !lfin(dscale)) return O_DEGENERATE;
    const o_real dfloor = p->den_tol * dscale;
    o_real lo_x = 0, lo_y = 0, hi_x = (o_real)wa - 1, hi_y = (o_real)ha - 1;
    int side = 0;
    for (int k = 0; k < 4; ++k) {
        const o_real x = (k & 1) ? bx : 0, y = (k & 2) ? by : 0;
        const o_real w = m[6] * x + m[7] * y + m[8];
        if (!lfin(w) || fabsl(w) <= dfloor) return O_DEGENERATE;
        const int s = w > 0 ? 1 : -1;
        if (side != 0 && s != side) return O_DEGENERATE;
        side = s;
        const o_real px = (m[0] * x + m[1] * y + m[2]) / w;
        const o_real py = (m[3] * x + m[4] * y + m[5]) / w;
        if (!lfin(px) || !lfin(py)) return O_DEGENERATE;
        if (px < lo_x) lo_x = px;
        if (py < lo_y) lo_y = py;
        if (px > hi_x) hi_x = px;
        if (py > hi_y) hi_y = py;
    }
    lo_x = floorl(lsnap(lo_x, p->snap_tol));
    lo_y = floorl(lsnap(lo_y, p->snap_tol));
    hi_x = ceill(lsnap(hi_x, p->snap_tol));
    hi_y = ceill(lsnap(hi_y, p->snap_tol));
    const o_real cw = hi_x - lo_x + 1, ch = hi_y - lo_y + 1;
    if (lo_x < INT_MIN || lo_y < INT_MIN || lo_x > INT_MAX || lo_y > INT_MAX || !lfin(cw) || !lfin(ch) || cw < 1 ||
        ch < 1 || cw > INT_MAX || ch > INT_MAX)
        return O_INSUFFICIENT_WORKSPACE;
    const size_t uw = (size_t)cw, uh = (size_t)ch;
    if (uw > SIZE_MAX / uh || uw > p->max_pixels / uh) return O_INSUFFICIENT_WORKSPACE;
    const o_real sa = lmaxr(lmaxr(1, (o_real)wa - 1), (o_real)ha - 1);
    const o_real sb = lmaxr(lmaxr(1, bx), by);
    const o_real cax = ((o_real)wa - 1) / 2, cay = ((o_real)ha - 1) / 2;
    const o_real na[9] = {1 / sa, 0, -cax / sa, 0, 1 / sa, -cay / sa, 0, 0, 1};
    const o_real nb_inv[9] = {sb, 0, bx / 2, 0, sb, by / 2, 0, 0, 1};
    o_real t[9], hn[9], hn_inv[9], inv[9];
    lmul3(na, m, t);
    lmul3(t, nb_inv, hn);
    if (!lscale(hn) || !linvert(hn, p->inv_tol, hn_inv)) return O_DEGENERATE;
    lmul3(nb_inv, hn_inv, t);
    lmul3(t, na, inv);
    if (!lscale(inv)) return O_DEGENERATE;
    o_s6_geom g;
    memset(&g, 0, sizeof(g));
    g.w = (int)cw;
    g.h = (int)ch;
    g.ox = (int)lo_x;
    g.oy = (int)lo_y;
    g.wa = wa;
    g.ha = ha;
    g.wb = wb;
    g.hb = hb;
    g.den_tol = p->den_tol;
    g.snap_tol = p->snap_tol;
    for (int i = 0; i < 9; ++i) {
        g.inv[i] = (double)inv[i];
        if (!isfinite(g.inv[i])) return O_DEGENERATE;
    }
    *out = g;
    return O_OK;
}

static int s6_centre(double* x, int n, double tol) {
    if (!isfinite(*x)) return 0;
    const double near = nearbyint(*x);
    const double roundoff = 16 * DBL_EPSILON * fmax(1.0, fabs(*x));
    if (fabs(*x - near) <= fmax(tol, roundoff)) *x = near;
    return *x >= 0 && *x <= n - 1.0;
}

static int s6_sample(const uint8_t* im, int w, int h, int pitch, double x, double y, double tol, float* rgb,
                     double* score) {
    if (!s6_centre(&x, w, tol) || !s6_centre(&y, h, tol)) return 0;
    const int x0 = (int)floor(x), y0 = (int)floor(y);
    const int x1 = x0 < w - 1 ? x0 + 1 : x0, y1 = y0 < h - 1 ? y0 + 1 : y0;
    const double ax = x - x0, ay = y - y0;
    const uint8_t* r0 = im + (size_t)y0 * pitch;
    const uint8_t* r1 = im + (size_t)y1 * pitch;
    for (int c = 0; c < 3; ++c) {
        const double top = (1 - ax) * r0[3 * x0 + c] + ax * r0[3 * x1 + c];
        const double bottom = (1 - ax) * r1[3 * x0 + c] + ax * r1[3 * x1 + c];
        rgb[c] = (float)(((1 - ay) * top + ay * bottom) / 255.0);
    }
    const double left = (x + 0.5) / w, right = (w - 0.5 - x) / w;
    const double upper = (y + 0.5) / h, lower = (h - 0.5 - y) / h;
    *score = fmin(fmin(left, right), fmin(upper, lower));
    return 1;
}

static uint8_t s6_quantize(float c) {
    float v = 255.0f * c;
    v = fminf(255.0f, fmaxf(0.0f, v));
    return (uint8_t)floorf(v + 0.5f);
}

/* out: RGB8 canvas (pitch out_pitch), mask 0/1 (pitch mask_pitch);
 * stats (optional): {union, overlap}. */
void oracle_s6_feather(const uint8_t* a, int pitch_a, const uint8_t* b, int pitch_b, const o_s6_geom* g,
                       uint8_t* out, int out_pitch, uint8_t* mask, int mask_pitch, uint64_t* stats) {
    uint64_t n_union = 0, n_overlap = 0;
    const double* m = g->inv;
    for (int y = 0; y < g->h; ++y)
        for (int x = 0; x < g->w; ++x) {
            const double xa = (double)x + g->ox, ya = (double)y + g->oy;
            float ra[3] = {0, 0, 0}, rb[3] = {0, 0, 0};
            double sa = 0, sb = 0;
            const int ma = s6_sample(a, g->wa, g->ha, pitch_a, xa, ya, g->snap_tol, ra, &sa);
            int mb = 0;
            const double den = m[6] * xa + m[7] * ya + m[8];
            const double den_scale = fabs(m[6] * xa) + fabs(m[7] * ya) + fabs(m[8]);
            if (isfinite(den) && den_scale > 0 && fabs(den) > g->den_tol * den_scale) {
                const double xb = (m[0] * xa + m[1] * ya + m[2]) / den;
                const double yb = (m[3] * xa + m[4] * ya + m[5]) / den;
                mb = s6_sample(b, g->wb, g->hb, pitch_b, xb, yb, g->snap_tol, rb, &sb);
            }
            mask[(size_t)y * mask_pitch + x] = (uint8_t)(ma || mb);
            n_union += (uint64_t)(ma || mb);
            n_overlap += (uint64_t)(ma && mb);
            for (int c = 0; c < 3; ++c) {
                float col;
                if (ma && mb)
                    col = (float)((sa * ra[c] + sb * rb[c]) / (sa + sb));
                else
                    col = ma ? ra[c] : rb[c];
                out[(size_t)y * out_pitch + 3 * x + c] = s6_quantize(col);
            }
        }
    if (stats) {
        stats[0] = n_union;
        stats[1] = n_overlap;
    }
}
