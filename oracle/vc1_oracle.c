/*
 * vc1_oracle.c - CPU restatement of libvc1's encoder-analysis hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; never linked by the product).
 * Parity pinned against the reference compiled from its own sources (oracle/_ref) and
 * against the reference's fixtures: see tests/test_oracle_pin.py.
 *
 * Citations are file:line into blenheimears/libvc1 v0.2.69. Reference semantics that the
 * restatement keeps on purpose:
 *   - every cost is uint64; an illegal candidate costs UINT64_MAX/4;
 *   - the staged-refinement score sad + lambda*rate is computed in long double, as the
 *     reference does (x87 80-bit on x86-64);
 *   - FP64 transform arithmetic is evaluated in the reference's order with no contraction
 *     (compiled with -ffp-contract=off like the reference, CMakeLists.txt:251).
 */
#include "vc1_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BAD (UINT64_MAX / 4)

static vo_counts g_counts;
void vo_counts_reset(void) { memset(&g_counts, 0, sizeof g_counts); }
void vo_counts_get(vo_counts* out) { *out = g_counts; }

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int iabs(int v) { return v < 0 ? -v : v; }

/* ---- geometry helpers ------------------------------------------------------------- */

static int vis_w(const vc1cu_params* p) { return p->display_width > 0 ? p->display_width : p->width; }
static int vis_h(const vc1cu_params* p) { return p->display_height > 0 ? p->display_height : p->height; }
static int mbw_of(const vc1cu_params* p) { return (p->width + 15) / 16; }
static int mbh_of(const vc1cu_params* p) { return (p->height + 15) / 16; }
static int mode_halfpel(int m) { return m == VC1CU_MV_HPEL || m == VC1CU_MV_HPEL_BILINEAR; }
static int mode_bilinear(int m) { return m == VC1CU_MV_HPEL_BILINEAR; }

/* Vc1Encoder::floor_div4, encoder_motion_compensation.cpp:355-358 */
static int floor_div4(int v) { return v >= 0 ? v / 4 : -((-v + 3) / 4); }

/* Vc1Encoder::arshift, encoder_entropy.cpp:377-381 (floor division by 2^n) */
static int arshift(int v, int n) {
    if (v >= 0) return v >> n;
    const int d = 1 << n;
    return -((-v + d - 1) / d);
}

/* Vc1Encoder::sample_clamped, encoder_motion_compensation.cpp:350-353 */
static int sample_clamped(const uint8_t* p, int w, int h, int x, int y) {
    x = iclamp(x, 0, w - 1);
    y = iclamp(y, 0, h - 1);
    return p[(size_t)y * w + x];
}

/* Vc1Encoder::mspel_filter4, encoder_motion_compensation.cpp:360-365 */
static int mspel_filter4(int a, int b, int c, int d, int mode) {
    if (mode == 1) return -4 * a + 53 * b + 18 * c - 3 * d;
    if (mode == 2) return -a + 9 * b + 9 * c - d;
    if (mode == 3) return -3 * a + 18 * b + 53 * c - 4 * d;
    return b;
}

/* Vc1Encoder::luma_mc_sample, encoder_motion_compensation.cpp:367-396 */
static int luma_mc_sample(const uint8_t* p, int w, int h, int x, int y, int mvx, int mvy, int rnd) {
    const int ix = floor_div4(mvx), iy = floor_div4(mvy);
    const int hm = mvx - ix * 4, vm = mvy - iy * 4;
    const int sx = x + ix, sy = y + iy;
    if (!hm && !vm) return sample_clamped(p, w, h, sx, sy);
    int v;
    if (vm && hm) {
        static const int shift_value[4] = {0, 5, 1, 5};
        const int shift = (shift_value[hm] + shift_value[vm]) >> 1;
        const int r1 = (1 << (shift - 1)) + (rnd ? 1 : 0) - 1;
        int t[4];
        for (int k = -1; k <= 2; ++k) {
            const int raw = mspel_filter4(sample_clamped(p, w, h, sx + k, sy - 1), sample_clamped(p, w, h, sx + k, sy),
                                          sample_clamped(p, w, h, sx + k, sy + 1),
                                          sample_clamped(p, w, h, sx + k, sy + 2), vm);
            t[k + 1] = arshift(raw + r1, shift);
        }
        const int raw = mspel_filter4(t[0], t[1], t[2], t[3], hm);
        v = arshift(raw + 64 - (rnd ? 1 : 0), 7);
    } else if (vm) {
        const int raw = mspel_filter4(sample_clamped(p, w, h, sx, sy - 1), sample_clamped(p, w, h, sx, sy),
                                      sample_clamped(p, w, h, sx, sy + 1), sample_clamped(p, w, h, sx, sy + 2), vm);
        const int bias = (vm == 2) ? (7 + (rnd ? 1 : 0)) : (31 + (rnd ? 1 : 0));
        v = arshift(raw + bias, vm == 2 ? 4 : 6);
    } else {
        const int raw = mspel_filter4(sample_clamped(p, w, h, sx - 1, sy), sample_clamped(p, w, h, sx, sy),
                                      sample_clamped(p, w, h, sx + 1, sy), sample_clamped(p, w, h, sx + 2, sy), hm);
        const int bias = (hm == 2) ? (8 - (rnd ? 1 : 0)) : (32 - (rnd ? 1 : 0));
        v = arshift(raw + bias, hm == 2 ? 4 : 6);
    }
    return iclamp(v, 0, 255);
}

/* Vc1Encoder::luma_mc_sample_mode, encoder_motion_compensation.cpp:398-415 */
static int luma_mc_sample_mode(const uint8_t* p, int w, int h, int x, int y, int mvx, int mvy, int mode,
                               int rnd) {
    if (!mode_bilinear(mode)) return luma_mc_sample(p, w, h, x, y, mvx, mvy, rnd);
    const int ix = floor_div4(mvx), iy = floor_div4(mvy);
    const int fx = mvx - ix * 4, fy = mvy - iy * 4;
    const int sx = x + ix, sy = y + iy;
    const int a = sample_clamped(p, w, h, sx, sy);
    if (!fx && !fy) return a;
    const int b = sample_clamped(p, w, h, sx + 1, sy);
    const int c = sample_clamped(p, w, h, sx, sy + 1);
    if (fx && fy) {
        const int d = sample_clamped(p, w, h, sx + 1, sy + 1);
        return (a + b + c + d + (rnd ? 1 : 2)) >> 2;
    }
    if (fx) return (a + b + (rnd ? 0 : 1)) >> 1;
    return (a + c + (rnd ? 0 : 1)) >> 1;
}

/* Vc1Encoder::chroma_mc_sample, encoder_motion_compensation.cpp:417-447 */
static int chroma_mc_sample(const uint8_t* p, int w, int h, int x, int y, int mvx, int mvy, int future,
                            int rnd) {
    int uvx = arshift(mvx + ((mvx & 3) == 3), 1);
    int uvy = arshift(mvy + ((mvy & 3) == 3), 1);
    if (future) {
        if (uvx < 0) uvx -= (uvx & 1); else uvx += (uvx & 1);
        if (uvy < 0) uvy -= (uvy & 1); else uvy += (uvy & 1);
    } else {
        if (uvx < 0) uvx += (uvx & 1); else uvx -= (uvx & 1);
        if (uvy < 0) uvy += (uvy & 1); else uvy -= (uvy & 1);
    }
    const int ix = floor_div4(uvx), iy = floor_div4(uvy);
    const int fx = (uvx - ix * 4) * 2, fy = (uvy - iy * 4) * 2;
    const int sx = x + ix, sy = y + iy;
    const int a = sample_clamped(p, w, h, sx, sy);
    if (!fx && !fy) return a;
    const int b = sample_clamped(p, w, h, sx + 1, sy);
    const int cc = sample_clamped(p, w, h, sx, sy + 1);
    const int d = sample_clamped(p, w, h, sx + 1, sy + 1);
    const int value = a * (8 - fx) * (8 - fy) + b * fx * (8 - fy) + cc * (8 - fx) * fy + d * fx * fy;
    return (value + (rnd ? 28 : 32)) >> 6;
}

static void count_sample(int mvx, int mvy, int mode, uint64_t n) {
    const int hm = mvx & 3, vm = mvy & 3;
    if (!hm && !vm) g_counts.int_sad_samples += n;
    else if (mode_bilinear(mode)) g_counts.bilinear_samples += n;
    else if (hm && vm) g_counts.qpel2d_samples += n;
    else g_counts.qpel1d_samples += n;
}

/* ---- cropped-reference legality ----------------------------------------------------- */

/* Vc1Encoder::motion_uses_hidden_luma, encoder_motion.cpp:2143-2165 */
static int hidden_luma(const vc1cu_params* p, int x0, int y0, int bw, int bh, int xq, int yq, int mode) {
    const int vw = vis_w(p), vh = vis_h(p);
    const int right_padding = vw < mbw_of(p) * 16;
    const int bottom_padding = vh < mbh_of(p) * 16;
    if (!right_padding && !bottom_padding) return 0;
    const int aw = imax(0, imin(bw, vw - x0)), ah = imax(0, imin(bh, vh - y0));
    if (!aw || !ah) return 0;
    const int ix = floor_div4(xq), iy = floor_div4(yq);
    const int fx = xq - ix * 4, fy = yq - iy * 4;
    const int right = fx ? (mode_bilinear(mode) ? 1 : 2) : 0;
    const int bottom = fy ? (mode_bilinear(mode) ? 1 : 2) : 0;
    return (right_padding && x0 + aw - 1 + ix + right >= vw) || (bottom_padding && y0 + ah - 1 + iy + bottom >= vh);
}

/* Vc1Encoder::motion_uses_hidden_chroma, encoder_motion.cpp:2167-2189; future selects the
 * B future-reference rounding of the chroma vector (:2178-2181) */
static int hidden_chroma_f(const vc1cu_params* p, int x0, int y0, int bw, int bh, int xq, int yq, int future) {
    const int cw = (vis_w(p) + 1) / 2, ch = (vis_h(p) + 1) / 2;
    const int right_padding = cw < mbw_of(p) * 8;
    const int bottom_padding = ch < mbh_of(p) * 8;
    if (!right_padding && !bottom_padding) return 0;
    const int cx = x0 / 2, cy = y0 / 2;
    const int aw = imax(0, imin(bw / 2, cw - cx)), ah = imax(0, imin(bh / 2, ch - cy));
    if (!aw || !ah) return 0;
    int uvx = arshift(xq + ((xq & 3) == 3), 1);
    int uvy = arshift(yq + ((yq & 3) == 3), 1);
    if (future) {
        uvx = uvx < 0 ? uvx - (uvx & 1) : uvx + (uvx & 1);
        uvy = uvy < 0 ? uvy - (uvy & 1) : uvy + (uvy & 1);
    } else {
        uvx = uvx < 0 ? uvx + (uvx & 1) : uvx - (uvx & 1);
        uvy = uvy < 0 ? uvy + (uvy & 1) : uvy - (uvy & 1);
    }
    const int ix = floor_div4(uvx), iy = floor_div4(uvy);
    const int fx = (uvx - ix * 4) != 0, fy = (uvy - iy * 4) != 0;
    return (right_padding && cx + aw - 1 + ix + (fx ? 1 : 0) >= cw) ||
           (bottom_padding && cy + ah - 1 + iy + (fy ? 1 : 0) >= ch);
}
static int hidden_chroma(const vc1cu_params* p, int x0, int y0, int bw, int bh, int xq, int yq) {
    return hidden_chroma_f(p, x0, y0, bw, bh, xq, yq, 0);
}

/* Vc1Encoder::motion_uses_hidden_padding, encoder_motion.cpp:2191-2195 */
int vo_hidden_padding(const vc1cu_params* p, int x0, int y0, int bw, int bh, int xq, int yq, int mode,
                      int chroma) {
    return hidden_luma(p, x0, y0, bw, bh, xq, yq, mode) || (chroma && hidden_chroma(p, x0, y0, bw, bh, xq, yq));
}

static int chroma_gate(int x0, int y0, int bw, int bh) { return bw == 16 && bh == 16 && !(x0 & 15) && !(y0 & 15); }

/* ---- block costs -------------------------------------------------------------------- */

/* Vc1Encoder::mb_sad, encoder_motion.cpp:2197-2285 (scalar branch :2272-2283) */
uint64_t vo_mb_sad(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my, int dx,
                   int dy, int stride) {
    const int x0 = mx * 16, y0 = my * 16;
    if (vo_hidden_padding(p, x0, y0, 16, 16, dx * 4, dy * 4, VC1CU_MV_QPEL, 1)) return BAD;
    uint64_t sad = 0, n = 0;
    for (int y = 0; y < 16 && y0 + y < cur->h; y += stride) {
        const int sy = iclamp(y0 + y + dy, 0, ref->h - 1);
        for (int x = 0; x < 16 && x0 + x < cur->w; x += stride) {
            const int sx = iclamp(x0 + x + dx, 0, ref->w - 1);
            sad += (uint64_t)iabs((int)cur->y[(size_t)(y0 + y) * cur->w + x0 + x] - (int)ref->y[(size_t)sy * ref->w + sx]);
            ++n;
        }
    }
    g_counts.int_sad_samples += n;
    if (stride > 1) sad *= (uint64_t)(stride * stride);
    return sad;
}

/* Vc1Encoder::block_sad_qpel, encoder_motion.cpp:2286-2668 (scalar accumulate :2609-2667) */
uint64_t vo_block_sad_qpel(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                           int bw, int bh, int xq, int yq) {
    if (vo_hidden_padding(p, x0, y0, bw, bh, xq, yq, VC1CU_MV_QPEL, chroma_gate(x0, y0, bw, bh))) return BAD;
    const int aw = imax(0, imin(bw, cur->w - x0)), ah = imax(0, imin(bh, cur->h - y0));
    uint64_t sad = 0;
    for (int y = 0; y < ah; ++y)
        for (int x = 0; x < aw; ++x) {
            const int pred = luma_mc_sample(ref->y, ref->w, ref->h, x0 + x, y0 + y, xq, yq, p->rnd);
            sad += (uint64_t)iabs((int)cur->y[(size_t)(y0 + y) * cur->w + x0 + x] - pred);
        }
    count_sample(xq, yq, VC1CU_MV_QPEL, (uint64_t)aw * ah);
    return sad;
}

/* Vc1Encoder::block_sad_motion, encoder_motion.cpp:2670-2933 (scalar loop :2926-2932) */
uint64_t vo_block_sad_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                             int bw, int bh, int xq, int yq, int mode) {
    if (!mode_bilinear(mode)) return vo_block_sad_qpel(p, cur, ref, x0, y0, bw, bh, xq, yq);
    if (vo_hidden_padding(p, x0, y0, bw, bh, xq, yq, mode, chroma_gate(x0, y0, bw, bh))) return BAD;
    if ((xq & 1) || (yq & 1)) return BAD;
    const int aw = imax(0, imin(bw, cur->w - x0)), ah = imax(0, imin(bh, cur->h - y0));
    uint64_t sad = 0;
    for (int y = 0; y < ah; ++y)
        for (int x = 0; x < aw; ++x) {
            const int pred = luma_mc_sample_mode(ref->y, ref->w, ref->h, x0 + x, y0 + y, xq, yq, mode, p->rnd);
            sad += (uint64_t)iabs((int)cur->y[(size_t)(y0 + y) * cur->w + x0 + x] - pred);
        }
    count_sample(xq, yq, mode, (uint64_t)aw * ah);
    return sad;
}

/* satd4x4_scalar, encoder_motion.cpp:2936-2958 */
static uint64_t satd4x4(const uint8_t* c, int cs, const uint8_t* pr, int ps) {
    int d[4][4], t[4][4];
    for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x) d[y][x] = (int)c[y * cs + x] - (int)pr[y * ps + x];
    for (int y = 0; y < 4; ++y) {
        const int a0 = d[y][0] + d[y][3], a1 = d[y][1] + d[y][2];
        const int a2 = d[y][1] - d[y][2], a3 = d[y][0] - d[y][3];
        t[y][0] = a0 + a1;
        t[y][1] = a3 + a2;
        t[y][2] = a0 - a1;
        t[y][3] = a3 - a2;
    }
    uint64_t tile = 0;
    for (int x = 0; x < 4; ++x) {
        const int a0 = t[0][x] + t[3][x], a1 = t[1][x] + t[2][x];
        const int a2 = t[1][x] - t[2][x], a3 = t[0][x] - t[3][x];
        tile += (uint64_t)iabs(a0 + a1);
        tile += (uint64_t)iabs(a3 + a2);
        tile += (uint64_t)iabs(a0 - a1);
        tile += (uint64_t)iabs(a3 - a2);
    }
    g_counts.satd_tiles++;
    return (tile + 1) >> 1;
}

/* Vc1Encoder::predict_luma_motion_block, encoder_motion_compensation.cpp:449-472 (scalar) */
void vo_predict_luma(const vc1cu_params* p, const vo_frame* ref, int x0, int y0, int bw, int bh, int xq, int yq,
                     int mode, uint8_t* dst, int dst_stride) {
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x)
            dst[y * dst_stride + x] =
                (uint8_t)luma_mc_sample_mode(ref->y, ref->w, ref->h, x0 + x, y0 + y, xq, yq, mode, p->rnd);
}

/* Vc1Encoder::block_satd_motion, encoder_motion.cpp:2960-3042 */
uint64_t vo_block_satd_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                              int bw, int bh, int xq, int yq, int mode) {
    const int aw = imax(0, imin(bw, cur->w - x0)), ah = imax(0, imin(bh, cur->h - y0));
    if (!aw || !ah) return 0;
    if (mode_halfpel(mode) && ((xq & 1) || (yq & 1))) return BAD;
    uint8_t pred[16 * 16];
    memset(pred, 0, sizeof pred);
    vo_predict_luma(p, ref, x0, y0, aw, ah, xq, yq, mode, pred, 16);
    count_sample(xq, yq, mode, (uint64_t)aw * ah);
    uint64_t total = 0;
    for (int by = 0; by < bh; by += 4)
        for (int bx = 0; bx < bw; bx += 4) {
            const int tw = imax(0, imin(4, aw - bx)), th = imax(0, imin(4, ah - by));
            if (!tw || !th) continue;
            const uint8_t* cp = cur->y + (size_t)(y0 + by) * cur->w + x0 + bx;
            const uint8_t* pp = pred + by * 16 + bx;
            if (tw == 4 && th == 4) {
                total += satd4x4(cp, cur->w, pp, 16);
            } else {
                uint8_t ct[16] = {0}, pt[16] = {0};
                for (int yy = 0; yy < th; ++yy)
                    for (int xx = 0; xx < tw; ++xx) {
                        ct[yy * 4 + xx] = cp[yy * cur->w + xx];
                        pt[yy * 4 + xx] = pp[yy * 16 + xx];
                    }
                total += satd4x4(ct, 4, pt, 4);
            }
        }
    return total;
}

/* Vc1Encoder::frame_sad, encoder_motion.cpp:1499-1576 (scalar loop :1563-1575) */
uint64_t vo_frame_sad(const vo_frame* cur, const vo_frame* ref, int dx, int dy, int stride) {
    uint64_t sad = 0, n = 0;
    for (int y = 0; y < cur->h; y += stride) {
        const int sy = iclamp(y + dy, 0, ref->h - 1);
        for (int x = 0; x < cur->w; x += stride) {
            const int sx = iclamp(x + dx, 0, ref->w - 1);
            sad += (uint64_t)iabs((int)cur->y[(size_t)y * cur->w + x] - (int)ref->y[(size_t)sy * ref->w + sx]);
            ++n;
        }
    }
    g_counts.frame_sad_samples += n;
    if (stride > 1) sad *= (uint64_t)(stride * stride);
    return sad;
}

/* The Vulkan shader's cost law, vulkan_motion_cost.comp:58-176 (no legality gates). */
uint64_t vo_shader_cost(const vo_frame* cur, const vo_frame* ref, int x0, int y0, int bw, int bh,
                        int sample_stride, int bilinear, int rnd, int metric, int xq, int yq) {
    const int aw = imax(0, imin(bw, cur->w - x0)), ah = imax(0, imin(bh, cur->h - y0));
    const int mode = bilinear ? VC1CU_MV_HPEL_BILINEAR : VC1CU_MV_QPEL;
    if (metric == VC1CU_METRIC_SAD) {
        const int ss = imax(sample_stride, 1);
        uint32_t total = 0;
        for (int y = 0; y < ah; y += ss)
            for (int x = 0; x < aw; x += ss) {
                const int c = cur->y[(size_t)(y0 + y) * cur->w + x0 + x];
                const int pr = luma_mc_sample_mode(ref->y, ref->w, ref->h, x0 + x, y0 + y, xq, yq, mode, rnd);
                total += (uint32_t)iabs(c - pr);
            }
        if (ss > 1) total *= (uint32_t)(ss * ss);
        return total;
    }
    uint32_t total = 0;
    for (int by = 0; by < bh; by += 4)
        for (int bx = 0; bx < bw; bx += 4) {
            if (!(bx < aw && by < ah)) continue;
            uint8_t ct[16] = {0}, pt[16] = {0};
            for (int yy = 0; yy < 4; ++yy)
                for (int xx = 0; xx < 4; ++xx) {
                    const int px = bx + xx, py = by + yy;
                    if (px < aw && py < ah) {
                        ct[yy * 4 + xx] = cur->y[(size_t)(y0 + py) * cur->w + x0 + px];
                        pt[yy * 4 + xx] = (uint8_t)luma_mc_sample_mode(ref->y, ref->w, ref->h, x0 + px, y0 + py, xq,
                                                                       yq, mode, rnd);
                    }
                }
            total += (uint32_t)satd4x4(ct, 4, pt, 4);
        }
    return total;
}

/* ---- global motion ----------------------------------------------------------------- */

typedef struct cand { uint64_t cost; int dx, dy; } cand;

/* total order (cost, |dx|+|dy|, dy, dx), encoder_motion.cpp:1786-1792, :2027-2033, :2102-2108 */
static int cand_less(uint64_t ca, int ax, int ay, uint64_t cb, int bx, int by) {
    if (ca != cb) return ca < cb;
    const int am = iabs(ax) + iabs(ay), bm = iabs(bx) + iabs(by);
    if (am != bm) return am < bm;
    if (ay != by) return ay < by;
    return ax < bx;
}

static void sort_cands(cand* t, int n) {
    for (int i = 1; i < n; ++i) {
        cand v = t[i];
        int j = i - 1;
        while (j >= 0 && cand_less(v.cost, v.dx, v.dy, t[j].cost, t[j].dx, t[j].dy)) { t[j + 1] = t[j]; --j; }
        t[j + 1] = v;
    }
}

/* Vc1Encoder::global_motion_search_extended, encoder_motion.cpp:2025-2074 */
static void global_extended(const vo_frame* cur, const vo_frame* ref, int range, int* odx, int* ody, uint64_t* osad) {
    cand top[9];
    int n = 0;
#define GCONS(DX, DY, S)                                                                    \
    do {                                                                                    \
        const int dx_ = iclamp((DX), -range, range), dy_ = iclamp((DY), -range, range);    \
        const cand c_ = {vo_frame_sad(cur, ref, dx_, dy_, (S)), dx_, dy_};                  \
        int found_ = 0;                                                                     \
        for (int i_ = 0; i_ < n; ++i_)                                                      \
            if (top[i_].dx == dx_ && top[i_].dy == dy_) {                                   \
                if (c_.cost < top[i_].cost) top[i_] = c_;                                   \
                found_ = 1;                                                                 \
                break;                                                                      \
            }                                                                               \
        if (!found_) {                                                                      \
            top[n++] = c_;                                                                  \
            sort_cands(top, n);                                                             \
            if (n > 8) n = 8;                                                               \
        }                                                                                   \
    } while (0)
    GCONS(0, 0, 16);
    const int step = range >= 160 ? 16 : 8;
    for (int d = step; d <= range; d += step) {
        GCONS(-d, 0, 16); GCONS(d, 0, 16); GCONS(0, -d, 16); GCONS(0, d, 16);
    }
    for (int r = step; r <= range; r += step) {
        const int h = (r + 1) / 2;
        GCONS(-r, -h, 16); GCONS(-r, h, 16); GCONS(r, -h, 16); GCONS(r, h, 16);
        GCONS(-h, -r, 16); GCONS(h, -r, 16); GCONS(-h, r, 16); GCONS(h, r, 16);
    }
    cand coarse[8];
    const int ncoarse = n;
    memcpy(coarse, top, sizeof(cand) * (size_t)n);
    for (int i = 0; i < imin(4, ncoarse); ++i) {
        const cand c = coarse[i];
        for (int oy = -step; oy <= step; oy += 4)
            for (int ox = -step; ox <= step; ox += 4) GCONS(c.dx + ox, c.dy + oy, 8);
    }
    if (n == 0) GCONS(0, 0, 8);
    const cand mid = top[0];
    for (int oy = -4; oy <= 4; ++oy)
        for (int ox = -4; ox <= 4; ++ox) GCONS(mid.dx + ox, mid.dy + oy, 4);
    const cand fine = top[0];
#undef GCONS
    cand full = {UINT64_MAX, 0, 0};
    for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
            const int dx = iclamp(fine.dx + ox, -range, range), dy = iclamp(fine.dy + oy, -range, range);
            const uint64_t c = vo_frame_sad(cur, ref, dx, dy, 1);
            if (cand_less(c, dx, dy, full.cost, full.dx, full.dy)) { full.cost = c; full.dx = dx; full.dy = dy; }
        }
    *odx = full.dx;
    *ody = full.dy;
    *osad = full.cost;
}

/* Vc1Encoder::global_motion_search, encoder_motion.cpp:2076-2141 */
void vo_global_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int range, int* odx,
                      int* ody, uint64_t* osad) {
    (void)p;
    range = imin(range, 32);
    if (range <= 0) {
        *odx = 0;
        *ody = 0;
        *osad = vo_frame_sad(cur, ref, 0, 0, 1);
        return;
    }
    if (range > 31) {
        global_extended(cur, ref, range, odx, ody, osad);
        return;
    }
    const int stride = 4;
    const int coarse_step = range >= 4 ? 4 : (range >= 2 ? 2 : 1);
    cand top[9];
    int n = 0;
#define GPUSH(C, DX, DY)                     \
    do {                                     \
        top[n].cost = (C);                   \
        top[n].dx = (DX);                    \
        top[n].dy = (DY);                    \
        ++n;                                 \
        sort_cands(top, n);                  \
        if (n > 8) n = 8;                    \
    } while (0)
    for (int dy = -range; dy <= range; dy += coarse_step)
        for (int dx = -range; dx <= range; dx += coarse_step) GPUSH(vo_frame_sad(cur, ref, dx, dy, stride), dx, dy);
    GPUSH(vo_frame_sad(cur, ref, 0, 0, stride), 0, 0);
    for (int d = -range; d <= range; d += coarse_step) {
        GPUSH(vo_frame_sad(cur, ref, range, d, stride), range, d);
        GPUSH(vo_frame_sad(cur, ref, d, range, stride), d, range);
    }
#undef GPUSH
    cand best = {UINT64_MAX, 0, 0};
    static unsigned char seen[63 * 63];
    memset(seen, 0, sizeof seen);
    for (int i = 0; i < n; ++i) {
        const cand c = top[i];
        for (int dy = imax(-range, c.dy - coarse_step + 1); dy <= imin(range, c.dy + coarse_step - 1); ++dy)
            for (int dx = imax(-range, c.dx - coarse_step + 1); dx <= imin(range, c.dx + coarse_step - 1); ++dx) {
                const size_t key = (size_t)(dy + 31) * 63 + (size_t)(dx + 31);
                if (seen[key]) continue;
                seen[key] = 1;
                const uint64_t cost = vo_frame_sad(cur, ref, dx, dy, 2);
                const int cm = iabs(dx) + iabs(dy), bm = iabs(best.dx) + iabs(best.dy);
                if (cost < best.cost || (cost == best.cost && cm < bm)) { best.cost = cost; best.dx = dx; best.dy = dy; }
            }
    }
    *odx = best.dx;
    *ody = best.dy;
    *osad = vo_frame_sad(cur, ref, best.dx, best.dy, 1);
}

/* ---- MV syntax, bounds, predictors ------------------------------------------------- */

/* groupa::kMvDiffBits[0], vc1_groupa_tables.h:26 (the VC-1 MVDATA VLC lengths, table 0) */
static const uint8_t kMvDiffBits0[73] = {
    6, 7, 7, 8, 14, 6, 5, 6, 7, 14, 14, 6, 6, 6, 8, 9, 10, 9, 7, 7, 7, 14, 14, 10, 9, 10, 8, 10, 10, 14, 14, 14,
    13, 13, 13, 6, 3, 5, 6, 8, 9, 13, 5, 4, 4, 5, 7, 9, 6, 5, 5, 5, 6, 9, 8, 5, 5, 5, 7, 10, 7, 7, 7, 7,
    7, 8, 10, 9, 8, 9, 9, 9, 3};

typedef struct bounds { int xmin, xmax, ymin, ymax; } bounds;

/* Vc1Encoder::motion_search_bounds_px, encoder_motion.cpp:1236-1245 */
static bounds bounds_px(int requested) {
    const int r = iclamp(requested, 0, 1024);
    bounds b = {-imin(r, 1024), imin(r, 1023), -imin(r, 256), imin(r, 255)};
    return b;
}

/* Vc1Encoder::motion_search_bounds_qpel, encoder_motion.cpp:1247-1254 */
static bounds bounds_qpel(int requested) {
    const int r = iclamp(requested, 0, 1024);
    bounds b;
    b.xmin = -imin(r * 4, 4096);
    b.xmax = (r >= 1024) ? 4095 : imin(r * 4, 4095);
    b.ymin = -imin(r * 4, 1024);
    b.ymax = (r >= 256) ? 1023 : imin(r * 4, 1023);
    return b;
}

/* Vc1Encoder::motion_mvrange / mvrange_* , encoder_motion.cpp:1256-1287 */
static int mvrange(const vc1cu_params* p) {
    const int r = p->search_range;
    if (r <= 31) return 0;
    if (r <= 63) return 1;
    if (r <= 127) return 2;
    return 3;
}
static const int kMvrangeXq[4] = {256, 512, 2048, 4096};
static const int kMvrangeYq[4] = {128, 256, 512, 1024};
static const int kMvrangeKx[4] = {9, 10, 12, 13};
static const int kMvrangeKy[4] = {8, 9, 10, 11};

/* Vc1Encoder::median3 / round_qpel_to_pixel / modular distance, encoder_motion.cpp:1295-1310 */
static int median3(int a, int b, int c) { return a + b + c - imin(a, imin(b, c)) - imax(a, imax(b, c)); }
static int round_qpel_to_pixel(int q) { return q >= 0 ? (q + 2) / 4 : -((-q + 2) / 4); }
static int modular_component_distance(int a, int b, int range) {
    int d = a - b;
    const int span = range * 2;
    d = ((d + range) % span + span) % span - range;
    return iabs(d);
}
static int modular_mv_distance(const vc1cu_params* p, vc1cu_mv a, vc1cu_mv b) {
    const int r = mvrange(p);
    return modular_component_distance(a.xq, b.xq, kMvrangeXq[r]) + modular_component_distance(a.yq, b.yq, kMvrangeYq[r]);
}

/* Vc1Encoder::mv_cat / mv_symbol / mv_component_bits / mv_suffix_bits, encoder_motion.cpp:1150-1197 */
static int mv_cat(int v, int halfpel) {
    const int a = iabs(v);
    if (!a) return 0;
    if (a <= 2) return 1;
    if (a <= 6) return 2;
    if (a <= 14) return 3;
    if (a <= 30) return 4;
    if (a <= (halfpel ? 94 : 158)) return 5;
    return -1;
}
static int mv_component_bits(int cat, int halfpel) {
    static const int sz[6] = {0, 2, 3, 4, 5, 8};
    return sz[cat] - ((halfpel && cat == 5) ? 1 : 0);
}

/* Vc1Encoder::motion_vector_rate_bits, encoder_motion.cpp:3214-3225 (mvdata_for_mode :1099-1114) */
static uint64_t mv_rate_bits(const vc1cu_params* p, vc1cu_mv desired, vc1cu_mv pred, int mode, int more) {
    const int halfpel = mode_halfpel(mode);
    int dx = desired.xq - pred.xq, dy = desired.yq - pred.yq;
    if (halfpel) { dx /= 2; dy /= 2; }
    const int xc = mv_cat(dx, halfpel), yc = mv_cat(dy, halfpel);
    int sym;
    if (xc < 0 || yc < 0) sym = more ? 71 : 34;
    else {
        const int idx = yc * 6 + xc;
        if (!more && idx == 0) sym = 34;
        else sym = more ? idx + 36 : idx - 1;
    }
    int suffix;
    if (sym == 34 || sym == 71) {
        const int r = mvrange(p), hp = halfpel ? 1 : 0;
        suffix = (kMvrangeKx[r] - hp) + (kMvrangeKy[r] - hp);
    } else {
        suffix = mv_component_bits(xc, halfpel) + mv_component_bits(yc, halfpel);
    }
    return (uint64_t)kMvDiffBits0[sym] + (uint64_t)suffix;
}

typedef struct pinfo {
    vc1cu_mv pre, a, c;
    int a_valid, c_valid, hybrid;
} pinfo;

static void pullback(vc1cu_mv* pre, int qx, int qy, int X, int Y, int margin) {
    if (qx + pre->xq < margin) pre->xq = margin - qx;
    if (qx + pre->xq > X) pre->xq = X - qx;
    if (qy + pre->yq < margin) pre->yq = margin - qy;
    if (qy + pre->yq > Y) pre->yq = Y - qy;
}

/* Vc1Encoder::predictor_info, encoder_motion.cpp:1312-1352 */
static pinfo predictor_info(const vc1cu_mv* mv, int mbw, int mbh, int mx, int my) {
    pinfo o;
    memset(&o, 0, sizeof o);
    vc1cu_mv A = {0, 0}, B = {0, 0}, C = {0, 0};
    const int a_valid = my > 0, c_valid = mx > 0, b_valid = my > 0 && mbw > 1;
    if (a_valid) A = mv[(size_t)(my - 1) * mbw + mx];
    if (c_valid) C = mv[(size_t)my * mbw + mx - 1];
    if (b_valid) {
        const int bx = (mx == mbw - 1) ? mx - 1 : mx + 1;
        B = mv[(size_t)(my - 1) * mbw + bx];
    }
    vc1cu_mv pre = {0, 0};
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if (a_valid + b_valid + c_valid > 1) {
        pre.xq = median3(A.xq, B.xq, C.xq);
        pre.yq = median3(A.yq, B.yq, C.yq);
    }
    pullback(&pre, mx * 64, my * 64, mbw * 64 - 4, mbh * 64 - 4, -60);
    int hybrid = 0;
    if (a_valid && c_valid) {
        if (iabs(pre.xq - A.xq) + iabs(pre.yq - A.yq) > 32) hybrid = 1;
        else if (iabs(pre.xq - C.xq) + iabs(pre.yq - C.yq) > 32) hybrid = 1;
    }
    o.pre = pre; o.a = A; o.c = C; o.a_valid = a_valid; o.c_valid = c_valid; o.hybrid = hybrid;
    return o;
}

static vc1cu_mv field_get(const vc1cu_mv* bm, int mbw, int mbh, int x, int y) {
    vc1cu_mv z = {0, 0};
    if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return z;
    return bm[((size_t)(y >> 1) * mbw + (x >> 1)) * 4 + (((y & 1) << 1) | (x & 1))];
}
static int intra_at(const uint8_t* intra, int mbw, int mbh, int x, int y) {
    if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return 0;
    return intra[(size_t)(y >> 1) * mbw + (x >> 1)] != 0;
}

static int hybrid_of(vc1cu_mv pre, vc1cu_mv A, vc1cu_mv C, int a_intra, int c_intra) {
    const int suma = a_intra ? iabs(pre.xq) + iabs(pre.yq) : iabs(pre.xq - A.xq) + iabs(pre.yq - A.yq);
    if (suma > 32) return 1;
    const int sumc = c_intra ? iabs(pre.xq) + iabs(pre.yq) : iabs(pre.xq - C.xq) + iabs(pre.yq - C.yq);
    return sumc > 32;
}

/* Vc1Encoder::predictor_info_mixed_1mv, encoder_motion.cpp:1354-1406 */
static pinfo predictor_info_mixed_1mv(const vc1cu_mv* bm, const uint8_t* intra, int mbw, int mbh, int mx, int my) {
    pinfo o;
    memset(&o, 0, sizeof o);
    const int bx = mx * 2, by = my * 2;
    const int a_valid = my > 0, c_valid = mx > 0, b_valid = my > 0 && mbw > 1;
    vc1cu_mv z = {0, 0};
    vc1cu_mv A = a_valid ? field_get(bm, mbw, mbh, bx, by - 1) : z;
    vc1cu_mv C = c_valid ? field_get(bm, mbw, mbh, bx - 1, by) : z;
    vc1cu_mv B = z;
    if (b_valid) B = field_get(bm, mbw, mbh, bx + ((mx == mbw - 1) ? -1 : 2), by - 1);
    vc1cu_mv pre = z;
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if (a_valid + b_valid + c_valid > 1) {
        pre.xq = median3(A.xq, B.xq, C.xq);
        pre.yq = median3(A.yq, B.yq, C.yq);
    }
    pullback(&pre, mx * 64, my * 64, mbw * 64 - 4, mbh * 64 - 4, -60);
    int hybrid = 0;
    if (a_valid && c_valid)
        hybrid = hybrid_of(pre, A, C, intra_at(intra, mbw, mbh, bx, by - 1), intra_at(intra, mbw, mbh, bx - 1, by));
    o.pre = pre; o.a = A; o.c = C; o.a_valid = a_valid; o.c_valid = c_valid; o.hybrid = hybrid;
    return o;
}

/* Vc1Encoder::predictor_info_4mv, encoder_motion.cpp:1408-1466 */
static pinfo predictor_info_4mv(const vc1cu_mv* bm, const uint8_t* intra, int mbw, int mbh, int mx, int my, int n) {
    pinfo o;
    memset(&o, 0, sizeof o);
    const int bx = mx * 2 + (n & 1), by = my * 2 + ((n >> 1) & 1);
    const int a_valid = my > 0 || n == 2 || n == 3;
    const int c_valid = mx > 0 || n == 1 || n == 3;
    const int b_valid = a_valid;
    vc1cu_mv z = {0, 0};
    vc1cu_mv A = a_valid ? field_get(bm, mbw, mbh, bx, by - 1) : z;
    vc1cu_mv C = c_valid ? field_get(bm, mbw, mbh, bx - 1, by) : z;
    vc1cu_mv B = z;
    if (b_valid) {
        int bxx = bx;
        if (n == 0) bxx += mx ? -1 : 1;
        else if (n == 1) bxx += (mx == mbw - 1) ? -1 : 1;
        else if (n == 2) bxx += 1;
        else bxx -= 1;
        B = field_get(bm, mbw, mbh, bxx, by - 1);
    }
    vc1cu_mv pre = z;
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if (a_valid + b_valid + c_valid > 1) {
        pre.xq = median3(A.xq, B.xq, C.xq);
        pre.yq = median3(A.yq, B.yq, C.yq);
    }
    pullback(&pre, mx * 64 + ((n == 1 || n == 3) ? 32 : 0), my * 64 + ((n == 2 || n == 3) ? 32 : 0), mbw * 64 - 4,
             mbh * 64 - 4, -28);
    int hybrid = 0;
    if (a_valid && c_valid)
        hybrid = hybrid_of(pre, A, C, intra_at(intra, mbw, mbh, bx, by - 1), intra_at(intra, mbw, mbh, bx - 1, by));
    o.pre = pre; o.a = A; o.c = C; o.a_valid = a_valid; o.c_valid = c_valid; o.hybrid = hybrid;
    return o;
}

/* ---- integer searches ------------------------------------------------------------- */

static uint64_t active_mb_pixels(const vc1cu_params* p, int mx, int my) {
    const int x0 = mx * 16, y0 = my * 16;
    return (uint64_t)imax(0, imin(16, p->width - x0)) * (uint64_t)imax(0, imin(16, p->height - y0));
}

/* Vc1Encoder::motion_match_good, encoder_motion.cpp:1627-1635 */
static int motion_match_good(const vc1cu_params* p, uint64_t sad, int mx, int my) {
    const uint64_t px = active_mb_pixels(p, mx, my);
    if (!px || sad >= UINT64_MAX / 8) return 0;
    return sad <= px * 6u;
}

/* Vc1Encoder::distant_match_decision, encoder_motion.cpp:1637-1656 */
static int distant_match_decision(const vc1cu_params* p, uint64_t cand_sad, uint64_t local_sad, int mx, int my) {
    const uint64_t px = active_mb_pixels(p, mx, my);
    if (!px || cand_sad >= UINT64_MAX / 8) return 0;
    if (cand_sad <= px * 6u) return 2;
    const long double max_sad = (long double)px * (long double)p->distant_match_max_mae;
    if ((long double)cand_sad > max_sad) return 1;
    if (local_sad >= UINT64_MAX / 8) return 3;
    return cand_sad * 4u <= local_sad * 3u ? 3 : 1;
}

#define SEEN_R 64
#define SEEN_SIDE (2 * SEEN_R + 1)
typedef struct seenset { uint64_t w[(SEEN_SIDE * SEEN_SIDE + 63) / 64]; int active; } seenset;
static int seen_test_set(seenset* s, int dx, int dy) {
    if (!s->active) return 0;
    const size_t bit = (size_t)(dy + SEEN_R) * SEEN_SIDE + (size_t)(dx + SEEN_R);
    const uint64_t m = 1ull << (bit & 63);
    if (s->w[bit >> 6] & m) return 1;
    s->w[bit >> 6] |= m;
    return 0;
}

typedef struct umh_state {
    const vc1cu_params* p;
    const vo_frame *cur, *ref;
    int mx, my, range;
    cand best;
    cand top[8];
    int top_count;
    seenset seen;
} umh_state;

/* the `consider` lambda of integer_motion_umh, encoder_motion.cpp:1821-1839 */
static void umh_consider(umh_state* s, int dx, int dy) {
    dx = iclamp(dx, -s->range, s->range);
    dy = iclamp(dy, -s->range, s->range);
    if (seen_test_set(&s->seen, dx, dy)) return;
    const uint64_t cost = vo_mb_sad(s->p, s->cur, s->ref, s->mx, s->my, dx, dy, 2);
    if (cand_less(cost, dx, dy, s->best.cost, s->best.dx, s->best.dy)) { s->best.cost = cost; s->best.dx = dx; s->best.dy = dy; }
    for (int i = 0; i < s->top_count; ++i)
        if (s->top[i].dx == dx && s->top[i].dy == dy) {
            if (cost < s->top[i].cost) s->top[i].cost = cost;
            return;
        }
    int at = 0;
    while (at < s->top_count && !cand_less(cost, dx, dy, s->top[at].cost, s->top[at].dx, s->top[at].dy)) ++at;
    if (at < 8) {
        const int nc = imin(s->top_count + 1, 8);
        for (int j = nc - 1; j > at; --j) s->top[j] = s->top[j - 1];
        s->top[at].cost = cost; s->top[at].dx = dx; s->top[at].dy = dy;
        s->top_count = nc;
    }
}

/* Vc1Encoder::integer_motion_umh, encoder_motion.cpp:1781-2023 (CPU branch of every batch) */
static cand integer_motion_umh(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                               const pinfo* pi, int gdx, int gdy, int range) {
    umh_state s;
    memset(&s, 0, sizeof s);
    s.p = p; s.cur = cur; s.ref = ref; s.mx = mx; s.my = my; s.range = range;
    s.best.cost = UINT64_MAX;
    s.seen.active = range <= SEEN_R;
#define CL(v) iclamp((v), -range, range)
    umh_consider(&s, CL(round_qpel_to_pixel(pi->pre.xq)), CL(round_qpel_to_pixel(pi->pre.yq)));
    umh_consider(&s, 0, 0);
    umh_consider(&s, gdx, gdy);
    if (pi->a_valid) umh_consider(&s, round_qpel_to_pixel(pi->a.xq), round_qpel_to_pixel(pi->a.yq));
    if (pi->c_valid) umh_consider(&s, round_qpel_to_pixel(pi->c.xq), round_qpel_to_pixel(pi->c.yq));
    {
        const int cx = s.best.dx, cy = s.best.dy;
        for (int oy = -2; oy <= 2; ++oy)
            for (int ox = -2; ox <= 2; ++ox) umh_consider(&s, cx + ox, cy + oy);
    }
    if (range >= 8) {
        for (int dy = -range; dy <= range; dy += 8)
            for (int dx = -range; dx <= range; dx += 8) umh_consider(&s, dx, dy);
        for (int d = -range; d <= range; d += 8) { umh_consider(&s, range, d); umh_consider(&s, d, range); }
    }
    {
        const int cross_step = range >= 96 ? 8 : (range >= 32 ? 4 : 2);
        const int cx = s.best.dx, cy = s.best.dy;
        const int vlimit = imin(range, imax(8, range / 2));
        for (int d = cross_step; d <= range; d += cross_step) { umh_consider(&s, cx - d, cy); umh_consider(&s, cx + d, cy); }
        for (int d = cross_step; d <= vlimit; d += cross_step) { umh_consider(&s, cx, cy - d); umh_consider(&s, cx, cy + d); }
    }
    {
        const int hex_step = range >= 96 ? 8 : (range >= 24 ? 4 : 2);
        const int hx = s.best.dx, hy = s.best.dy;
        for (int r = hex_step; r <= range; r += hex_step) {
            const int h = (r + 1) / 2;
            umh_consider(&s, hx - r, hy); umh_consider(&s, hx + r, hy);
            umh_consider(&s, hx - h, hy - r); umh_consider(&s, hx + h, hy - r);
            umh_consider(&s, hx - h, hy + r); umh_consider(&s, hx + h, hy + r);
        }
    }
    for (int iter = 0; iter < 32; ++iter) {
        const int ox = s.best.dx, oy = s.best.dy;
        umh_consider(&s, ox - 2, oy); umh_consider(&s, ox + 2, oy);
        umh_consider(&s, ox - 1, oy - 2); umh_consider(&s, ox + 1, oy - 2);
        umh_consider(&s, ox - 1, oy + 2); umh_consider(&s, ox + 1, oy + 2);
        if (s.best.dx == ox && s.best.dy == oy) break;
    }
    {
        const int ox = s.best.dx, oy = s.best.dy;
        umh_consider(&s, ox - 1, oy); umh_consider(&s, ox + 1, oy);
        umh_consider(&s, ox, oy - 1); umh_consider(&s, ox, oy + 1);
    }
    cand full = {UINT64_MAX, 0, 0};
    seenset sf;
    memset(&sf, 0, sizeof sf);
    sf.active = range <= SEEN_R;
    const int finalists = imin(4, s.top_count);
    for (int i = 0; i < finalists; ++i) {
        const cand c = s.top[i];
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const int dx = CL(c.dx + ox), dy = CL(c.dy + oy);
                if (seen_test_set(&sf, dx, dy)) continue;
                const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
                if (cand_less(sad, dx, dy, full.cost, full.dx, full.dy)) { full.cost = sad; full.dx = dx; full.dy = dy; }
            }
    }
    if (full.cost == UINT64_MAX) {
        (void)seen_test_set(&sf, s.best.dx, s.best.dy);
        full.cost = vo_mb_sad(p, cur, ref, mx, my, s.best.dx, s.best.dy, 1);
        full.dx = s.best.dx;
        full.dy = s.best.dy;
    }
    if (range > 0 && !motion_match_good(p, full.cost, mx, my)) {
        cand coarse = {UINT64_MAX, 0, 0};
        const int step = range >= 8 ? 4 : (range >= 3 ? 2 : 1);
        for (int dy = -range; dy <= range; dy += step)
            for (int dx = -range; dx <= range; dx += step) {
                const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 4);
                if (cand_less(sad, dx, dy, coarse.cost, coarse.dx, coarse.dy)) { coarse.cost = sad; coarse.dx = dx; coarse.dy = dy; }
            }
        for (int d = -range; d <= range; d += step) {
            uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, range, d, 4);
            if (cand_less(sad, range, d, coarse.cost, coarse.dx, coarse.dy)) { coarse.cost = sad; coarse.dx = range; coarse.dy = d; }
            sad = vo_mb_sad(p, cur, ref, mx, my, d, range, 4);
            if (cand_less(sad, d, range, coarse.cost, coarse.dx, coarse.dy)) { coarse.cost = sad; coarse.dx = d; coarse.dy = range; }
        }
        cand rescue = {UINT64_MAX, coarse.dx, coarse.dy};
        const int rr = imax(1, step - 1);
        for (int dy = imax(-range, coarse.dy - rr); dy <= imin(range, coarse.dy + rr); ++dy)
            for (int dx = imax(-range, coarse.dx - rr); dx <= imin(range, coarse.dx + rr); ++dx) {
                if (seen_test_set(&sf, dx, dy)) continue;
                const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
                if (cand_less(sad, dx, dy, rescue.cost, rescue.dx, rescue.dy)) { rescue.cost = sad; rescue.dx = dx; rescue.dy = dy; }
            }
        if (cand_less(rescue.cost, rescue.dx, rescue.dy, full.cost, full.dx, full.dy)) full = rescue;
        const uint64_t pixels = active_mb_pixels(p, mx, my);
        if (pixels && full.cost > pixels * 24u && range <= 32) {
            cand dense = {UINT64_MAX, 0, 0};
            for (int dy = -range; dy <= range; dy += 2)
                for (int dx = -range; dx <= range; dx += 2) {
                    const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 2);
                    if (cand_less(sad, dx, dy, dense.cost, dense.dx, dense.dy)) { dense.cost = sad; dense.dx = dx; dense.dy = dy; }
                }
            cand df = {UINT64_MAX, dense.dx, dense.dy};
            for (int dy = imax(-range, dense.dy - 2); dy <= imin(range, dense.dy + 2); ++dy)
                for (int dx = imax(-range, dense.dx - 2); dx <= imin(range, dense.dx + 2); ++dx) {
                    if (seen_test_set(&sf, dx, dy)) continue;
                    const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
                    if (cand_less(sad, dx, dy, df.cost, df.dx, df.dy)) { df.cost = sad; df.dx = dx; df.dy = dy; }
                }
            if (cand_less(df.cost, df.dx, df.dy, full.cost, full.dx, full.dy)) full = df;
        }
    }
#undef CL
    return full;
}

/* Vc1Encoder::integer_motion_diamond, encoder_motion_diamond.cpp:13-73 */
static cand integer_motion_diamond(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                                   const pinfo* pi, int gdx, int gdy, int range) {
    cand best = {vo_mb_sad(p, cur, ref, mx, my, 0, 0, 1), 0, 0};
    if (best.cost == 0) return best;
    int sx[5] = {0}, sy[5] = {0}, sc = 1;
#define SEED(DX, DY)                                                                          \
    do {                                                                                      \
        const int dx_ = iclamp((DX), -range, range), dy_ = iclamp((DY), -range, range);      \
        int dup_ = 0;                                                                         \
        for (int i_ = 0; i_ < sc; ++i_) if (dx_ == sx[i_] && dy_ == sy[i_]) dup_ = 1;        \
        if (!dup_) {                                                                          \
            sx[sc] = dx_; sy[sc] = dy_; ++sc;                                                 \
            const uint64_t c_ = vo_mb_sad(p, cur, ref, mx, my, dx_, dy_, 1);                  \
            if (cand_less(c_, dx_, dy_, best.cost, best.dx, best.dy)) { best.cost = c_; best.dx = dx_; best.dy = dy_; } \
        }                                                                                     \
    } while (0)
    SEED(round_qpel_to_pixel(pi->pre.xq), round_qpel_to_pixel(pi->pre.yq));
    SEED(gdx, gdy);
    if (pi->a_valid) SEED(round_qpel_to_pixel(pi->a.xq), round_qpel_to_pixel(pi->a.yq));
    if (pi->c_valid) SEED(round_qpel_to_pixel(pi->c.xq), round_qpel_to_pixel(pi->c.yq));
#undef SEED
    int px = best.dx, py = best.dy, have_prev = 0;
    static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (int step = 0; step <= 4 * range + 1; ++step) {
        const cand center = best;
        cand winner = center;
        for (int k = 0; k < 4; ++k) {
            const int dx = center.dx + off[k][0], dy = center.dy + off[k][1];
            if (dx < -range || dx > range || dy < -range || dy > range) continue;
            if (have_prev && dx == px && dy == py) continue;
            const uint64_t c = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
            if (cand_less(c, dx, dy, winner.cost, winner.dx, winner.dy)) { winner.cost = c; winner.dx = dx; winner.dy = dy; }
        }
        if (winner.dx == center.dx && winner.dy == center.dy) break;
        px = center.dx; py = center.dy; have_prev = 1;
        best = winner;
        if (best.cost == 0) break;
    }
    return best;
}

void vo_integer_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                       const vc1cu_mv* field, int gdx, int gdy, int range, int* dx, int* dy, uint64_t* sad) {
    const pinfo pi = predictor_info(field, mbw_of(p), mbh_of(p), mx, my);
    const cand r = p->me_algorithm == 1 ? integer_motion_diamond(p, cur, ref, mx, my, &pi, gdx, gdy, range)
                                         : integer_motion_umh(p, cur, ref, mx, my, &pi, gdx, gdy, range);
    *dx = r.dx;
    *dy = r.dy;
    *sad = r.cost;
}

/* ---- long-range search (encoder_motion.cpp:1578-1779) -------------------------------- */

typedef struct lr_sig { uint8_t ydc[4], udc, vdc; } lr_sig;
typedef struct lr_cell { int x, y; lr_sig sig; } lr_cell;

/* Vc1Encoder::mean_region, encoder_motion.cpp:1578-1590 */
static uint8_t mean_region(const uint8_t* plane, int pw, int ph, int x0, int y0, int bw, int bh) {
    uint64_t sum = 0;
    int n = 0;
    for (int y = 0; y < bh && y0 + y < ph; ++y) {
        if (y0 + y < 0) continue;
        for (int x = 0; x < bw && x0 + x < pw; ++x) {
            if (x0 + x < 0) continue;
            sum += plane[(size_t)(y0 + y) * pw + x0 + x];
            ++n;
        }
    }
    return n ? (uint8_t)((sum + (uint64_t)(n / 2)) / (uint64_t)n) : 128;
}

/* Vc1Encoder::long_range_signature, encoder_motion.cpp:1592-1603 */
static lr_sig lr_signature(const vo_frame* f, int x0, int y0) {
    lr_sig s;
    s.ydc[0] = mean_region(f->y, f->w, f->h, x0, y0, 8, 8);
    s.ydc[1] = mean_region(f->y, f->w, f->h, x0 + 8, y0, 8, 8);
    s.ydc[2] = mean_region(f->y, f->w, f->h, x0, y0 + 8, 8, 8);
    s.ydc[3] = mean_region(f->y, f->w, f->h, x0 + 8, y0 + 8, 8, 8);
    const int cw = f->w / 2, ch = f->h / 2;
    s.udc = f->u ? mean_region(f->u, cw, ch, x0 / 2, y0 / 2, 8, 8) : 128;
    s.vdc = f->v ? mean_region(f->v, cw, ch, x0 / 2, y0 / 2, 8, 8) : 128;
    return s;
}

/* Vc1Encoder::long_range_signature_distance, encoder_motion.cpp:1605-1614 */
static unsigned lr_distance(const lr_sig* a, const lr_sig* b) {
    unsigned d = 0;
    for (int i = 0; i < 4; ++i) d += (unsigned)iabs((int)a->ydc[i] - (int)b->ydc[i]) * 2u;
    d += (unsigned)iabs((int)a->udc - (int)b->udc) * 3u;
    d += (unsigned)iabs((int)a->vdc - (int)b->vdc) * 3u;
    return d;
}

/* Vc1Encoder::propagated_long_range_motion, encoder_motion.cpp:1658-1694 */
static cand propagated_long_range(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                                  int mbw, const vc1cu_mv* field, const uint8_t* propagated, int requested_range) {
    cand best = {UINT64_MAX, 0, 0};
    const bounds b = bounds_px(requested_range);
    static const int offs[13][2] = {{0, 0}, {-1, 0}, {1, 0}, {0, -1}, {0, 1}, {-2, 0}, {2, 0},
                                    {0, -2}, {0, 2}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
    static const int nb[4][2] = {{-1, 0}, {0, -1}, {-1, -1}, {1, -1}};
    for (int k = 0; k < 4; ++k) {
        const int nx = mx + nb[k][0], ny = my + nb[k][1];
        if (nx < 0 || ny < 0 || nx >= mbw) continue;
        const size_t pos = (size_t)ny * mbw + nx;
        if (!propagated[pos]) continue;
        const int cx = round_qpel_to_pixel(field[pos].xq), cy = round_qpel_to_pixel(field[pos].yq);
        for (int o = 0; o < 13; ++o) {
            const int dx = iclamp(cx + offs[o][0], b.xmin, b.xmax), dy = iclamp(cy + offs[o][1], b.ymin, b.ymax);
            const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
            if (sad < best.cost || (sad == best.cost && iabs(dx) + iabs(dy) < iabs(best.dx) + iabs(best.dy))) {
                best.cost = sad; best.dx = dx; best.dy = dy;
            }
        }
        if (motion_match_good(p, best.cost, mx, my)) break;
    }
    return best;
}

typedef struct sigc { unsigned score; int dx, dy; } sigc;
static int sig_less(const sigc* a, const sigc* b) {
    if (a->score != b->score) return a->score < b->score;
    const int am = iabs(a->dx) + iabs(a->dy), bm = iabs(b->dx) + iabs(b->dy);
    if (am != bm) return am < bm;
    if (a->dy != b->dy) return a->dy < b->dy;
    return a->dx < b->dx;
}

/* Vc1Encoder::extended_content_motion, encoder_motion.cpp:1696-1779 (CPU branch of each batch) */
static cand extended_content(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                             int requested_range, const lr_cell* cells, int ncells, cand local,
                             uint64_t* cand_sad_out, int* decision_out) {
    sigc top[17];
    int nt = 0;
    const int x0 = mx * 16, y0 = my * 16;
    const lr_sig want = lr_signature(cur, x0, y0);
    const bounds b = bounds_px(requested_range);
    for (int i = 0; i < ncells; ++i) {
        const int dx = cells[i].x - x0, dy = cells[i].y - y0;
        if (dx < b.xmin || dx > b.xmax || dy < b.ymin || dy > b.ymax) continue;
        if (iabs(dx) <= 32 && iabs(dy) <= 32) continue;
        sigc c = {lr_distance(&want, &cells[i].sig), dx, dy};
        if (nt == 16 && !sig_less(&c, &top[15])) continue;
        int at = 0; /* std::lower_bound: first element not less than c */
        while (at < nt && sig_less(&top[at], &c)) ++at;
        for (int j = nt; j > at; --j) top[j] = top[j - 1];
        top[at] = c;
        if (++nt > 16) nt = 16;
    }
    cand best = {UINT64_MAX, 0, 0};
    for (int t = 0; t < nt; ++t) {
        const sigc c = top[t];
        int sx = c.dx, sy = c.dy;
        uint64_t sampled = UINT64_MAX;
        for (int oy = -8; oy <= 8; oy += 4)
            for (int ox = -8; ox <= 8; ox += 4) {
                const int dx = iclamp(c.dx + ox, b.xmin, b.xmax), dy = iclamp(c.dy + oy, b.ymin, b.ymax);
                const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 2);
                if (sad < sampled) { sampled = sad; sx = dx; sy = dy; }
            }
        cand full = {UINT64_MAX, sx, sy};
        for (int oy = -2; oy <= 2; ++oy)
            for (int ox = -2; ox <= 2; ++ox) {
                const int dx = iclamp(sx + ox, b.xmin, b.xmax), dy = iclamp(sy + oy, b.ymin, b.ymax);
                const uint64_t sad = vo_mb_sad(p, cur, ref, mx, my, dx, dy, 1);
                if (sad < full.cost || (sad == full.cost && iabs(dx) + iabs(dy) < iabs(full.dx) + iabs(full.dy))) {
                    full.cost = sad; full.dx = dx; full.dy = dy;
                }
            }
        if (full.cost < best.cost) best = full;
        if (motion_match_good(p, best.cost, mx, my)) break;
    }
    *cand_sad_out = best.cost;
    const int decision = best.cost < UINT64_MAX / 8 ? distant_match_decision(p, best.cost, local.cost, mx, my) : 0;
    *decision_out = decision;
    if (best.cost >= local.cost || decision < 2) return local;
    return best;
}

/* ---- sub-pel refinement ------------------------------------------------------------ */

typedef struct scand {
    vc1cu_mv mv;
    uint64_t sad, rate, satd;
    long double score;
    int eligible;
} scand;

/* tie_less, encoder_motion.cpp:3314-3319 */
static int tie_less(vc1cu_mv a, vc1cu_mv b) {
    const int am = iabs(a.xq) + iabs(a.yq), bm = iabs(b.xq) + iabs(b.yq);
    if (am != bm) return am < bm;
    if (a.yq != b.yq) return a.yq < b.yq;
    return a.xq < b.xq;
}
static int same_mv(vc1cu_mv a, vc1cu_mv b) { return a.xq == b.xq && a.yq == b.yq; }
static int make_even(int v) { return !(v & 1) ? v : (v > 0 ? v - 1 : v + 1); }

/* Vc1Encoder::refine_motion_integer_only, encoder_motion.cpp:3247-3269 */
static vc1cu_mv refine_integer_only(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                                    int bw, int bh, vc1cu_mv seed, int range, int mode, uint64_t* best_sad,
                                    uint64_t known) {
    const bounds qb = bounds_qpel(range);
#define SNAP(Q, LO, HI) ({ int q_ = iclamp((Q), (LO), (HI)); const int n_ = q_ >= 0 ? (q_ + 1) / 4 : (q_ - 1) / 4; iclamp(n_ * 4, (LO), (HI) / 4 * 4); })
    vc1cu_mv integer = {SNAP(seed.xq, qb.xmin, qb.xmax), SNAP(seed.yq, qb.ymin, qb.ymax)};
#undef SNAP
    if (vo_hidden_padding(p, x0, y0, bw, bh, integer.xq, integer.yq, mode, chroma_gate(x0, y0, bw, bh))) {
        integer.xq = 0;
        integer.yq = 0;
    }
    if (best_sad)
        *best_sad = (integer.xq == seed.xq && integer.yq == seed.yq && known != UINT64_MAX)
                        ? known : vo_block_sad_motion(p, cur, ref, x0, y0, bw, bh, integer.xq, integer.yq, mode);
    return integer;
}

typedef struct cands { scand c[24]; int n; } cands;

static scand* cands_find(cands* s, vc1cu_mv mv) {
    for (int i = 0; i < s->n; ++i) if (same_mv(s->c[i].mv, mv)) return &s->c[i];
    return NULL;
}

/* the `add` lambda, encoder_motion.cpp:3324-3337 */
static void cands_add(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, cands* s, int x0, int y0,
                      int bw, int bh, vc1cu_mv mv, int mode, uint64_t known) {
    if (cands_find(s, mv)) return;
    scand c;
    memset(&c, 0, sizeof c);
    c.mv = mv;
    c.sad = vo_hidden_padding(p, x0, y0, bw, bh, mv.xq, mv.yq, mode, chroma_gate(x0, y0, bw, bh))
                ? BAD : (known != UINT64_MAX ? known : vo_block_sad_motion(p, cur, ref, x0, y0, bw, bh, mv.xq, mv.yq, mode));
    s->c[s->n++] = c;
}

static void sort_scand(scand* a, int n, int (*less)(const scand*, const scand*)) {
    for (int i = 1; i < n; ++i) {
        scand v = a[i];
        int j = i - 1;
        while (j >= 0 && less(&v, &a[j])) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
}
static int sad_tie_less(const scand* a, const scand* b) {
    if (a->sad != b->sad) return a->sad < b->sad;
    return tie_less(a->mv, b->mv);
}
static int score_less(const scand* a, const scand* b) {
    if (a->score != b->score) return a->score < b->score;
    if (a->sad != b->sad) return a->sad < b->sad;
    return tie_less(a->mv, b->mv);
}
static int satd_order_less(const scand* a, const scand* b) {
    if (a->eligible != b->eligible) return a->eligible > b->eligible;
    if (a->score != b->score) return a->score < b->score;
    if (a->satd != b->satd) return a->satd < b->satd;
    if (a->sad != b->sad) return a->sad < b->sad;
    return tie_less(a->mv, b->mv);
}

static vc1cu_mv refine_qpel_block(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                                  int bw, int bh, vc1cu_mv seed, int range, uint64_t* best_sad, uint64_t known);
static vc1cu_mv refine_motion_block(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                                    int bw, int bh, vc1cu_mv seed, int range, int mode, uint64_t* best_sad,
                                    uint64_t known);

/* Vc1Encoder::refine_motion_block_staged, encoder_motion.cpp:3271-3594 (me_quality SAD, RATE, SATD) */
static vc1cu_mv refine_staged(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0, int bw,
                              int bh, vc1cu_mv seed, int range, int mode, const pinfo* pi, int more,
                              uint64_t* best_sad, uint64_t known) {
    const int limit_q = 4 * p->subpel_range;
    if (!p->subpel || limit_q == 0 || imax(iabs(seed.xq), iabs(seed.yq)) > limit_q)
        return refine_integer_only(p, cur, ref, x0, y0, bw, bh, seed, range, mode, best_sad, known);
    if (p->me_quality == 0) return refine_motion_block(p, cur, ref, x0, y0, bw, bh, seed, range, mode, best_sad, known);
    cands all;
    all.n = 0;
    const bounds qb = bounds_qpel(range);
    const int xmin = imax(qb.xmin, -limit_q), xmax = imin(qb.xmax, limit_q);
    const int ymin = imax(qb.ymin, -limit_q), ymax = imin(qb.ymax, limit_q);
    const int hp = mode_halfpel(mode);
    if (hp) {
        seed.xq = make_even(iclamp(seed.xq, xmin, xmax));
        seed.yq = make_even(iclamp(seed.yq, ymin, ymax));
    } else {
        seed.xq = iclamp(seed.xq, xmin, xmax);
        seed.yq = iclamp(seed.yq, ymin, ymax);
    }
    const int cg = chroma_gate(x0, y0, bw, bh);
    cands_add(p, cur, ref, &all, x0, y0, bw, bh, seed, mode, known);
    if (vo_hidden_padding(p, x0, y0, bw, bh, seed.xq, seed.yq, mode, cg)) {
        vc1cu_mv z = {0, 0};
        cands_add(p, cur, ref, &all, x0, y0, bw, bh, z, mode, UINT64_MAX);
    }
    vc1cu_mv half_best = seed;
    uint64_t half_sad = all.c[0].sad;
    vc1cu_mv batch[9];
    int nb = 0;
    const int fast = p->fast_subpel;
    if (fast) {
        static const int o4[4][2] = {{-2, 0}, {2, 0}, {0, -2}, {0, 2}};
        batch[nb++] = seed;
        for (int k = 0; k < 4; ++k) {
            vc1cu_mv mv = {iclamp(seed.xq + o4[k][0], xmin, xmax), iclamp(seed.yq + o4[k][1], ymin, ymax)};
            if (hp) { mv.xq = make_even(mv.xq); mv.yq = make_even(mv.yq); }
            batch[nb++] = mv;
        }
    } else {
        for (int oy = -2; oy <= 2; oy += 2)
            for (int ox = -2; ox <= 2; ox += 2) {
                vc1cu_mv mv = {iclamp(seed.xq + ox, xmin, xmax), iclamp(seed.yq + oy, ymin, ymax)};
                if (hp) { mv.xq = make_even(mv.xq); mv.yq = make_even(mv.yq); }
                batch[nb++] = mv;
            }
    }
    for (int i = 0; i < nb; ++i) cands_add(p, cur, ref, &all, x0, y0, bw, bh, batch[i], mode, UINT64_MAX);
    for (int i = 0; i < nb; ++i) {
        const scand* c = cands_find(&all, batch[i]);
        if (c && (c->sad < half_sad || (c->sad == half_sad && tie_less(c->mv, half_best)))) { half_sad = c->sad; half_best = c->mv; }
    }
    if (fast && !same_mv(half_best, seed)) {
        vc1cu_mv diag[2];
        int nd = 0;
        const int dx = half_best.xq - seed.xq, dy = half_best.yq - seed.yq;
        if (dx && !dy) {
            diag[nd].xq = half_best.xq; diag[nd].yq = iclamp(seed.yq - 2, ymin, ymax); ++nd;
            diag[nd].xq = half_best.xq; diag[nd].yq = iclamp(seed.yq + 2, ymin, ymax); ++nd;
        } else if (dy && !dx) {
            diag[nd].xq = iclamp(seed.xq - 2, xmin, xmax); diag[nd].yq = half_best.yq; ++nd;
            diag[nd].xq = iclamp(seed.xq + 2, xmin, xmax); diag[nd].yq = half_best.yq; ++nd;
        }
        if (hp) for (int i = 0; i < nd; ++i) { diag[i].xq = make_even(diag[i].xq); diag[i].yq = make_even(diag[i].yq); }
        for (int i = 0; i < nd; ++i) cands_add(p, cur, ref, &all, x0, y0, bw, bh, diag[i], mode, UINT64_MAX);
        for (int i = 0; i < nd; ++i) {
            const scand* c = cands_find(&all, diag[i]);
            if (c && (c->sad < half_sad || (c->sad == half_sad && tie_less(c->mv, half_best)))) { half_sad = c->sad; half_best = c->mv; }
        }
    }
    if (!hp) {
        if (fast) {
            static const int o4[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            const vc1cu_mv qc = half_best;
            vc1cu_mv qb5[5];
            int nq = 0;
            qb5[nq++] = qc;
            for (int k = 0; k < 4; ++k) {
                vc1cu_mv mv = {iclamp(qc.xq + o4[k][0], xmin, xmax), iclamp(qc.yq + o4[k][1], ymin, ymax)};
                qb5[nq++] = mv;
            }
            for (int i = 0; i < nq; ++i) cands_add(p, cur, ref, &all, x0, y0, bw, bh, qb5[i], mode, UINT64_MAX);
            vc1cu_mv qbmv = qc;
            uint64_t qcost = cands_find(&all, qc)->sad;
            for (int i = 0; i < nq; ++i) {
                const scand* c = cands_find(&all, qb5[i]);
                if (c && (c->sad < qcost || (c->sad == qcost && tie_less(c->mv, qbmv)))) { qbmv = c->mv; qcost = c->sad; }
            }
            vc1cu_mv q2[2];
            int n2 = 0;
            const int dx = qbmv.xq - qc.xq, dy = qbmv.yq - qc.yq;
            if (dx && !dy) {
                q2[n2].xq = qbmv.xq; q2[n2].yq = iclamp(qc.yq - 1, ymin, ymax); ++n2;
                q2[n2].xq = qbmv.xq; q2[n2].yq = iclamp(qc.yq + 1, ymin, ymax); ++n2;
            } else if (dy && !dx) {
                q2[n2].xq = iclamp(qc.xq - 1, xmin, xmax); q2[n2].yq = qbmv.yq; ++n2;
                q2[n2].xq = iclamp(qc.xq + 1, xmin, xmax); q2[n2].yq = qbmv.yq; ++n2;
            }
            for (int i = 0; i < n2; ++i) cands_add(p, cur, ref, &all, x0, y0, bw, bh, q2[i], mode, UINT64_MAX);
        } else {
            for (int oy = -1; oy <= 1; ++oy)
                for (int ox = -1; ox <= 1; ++ox) {
                    vc1cu_mv mv = {iclamp(half_best.xq + ox, xmin, xmax), iclamp(half_best.yq + oy, ymin, ymax)};
                    cands_add(p, cur, ref, &all, x0, y0, bw, bh, mv, mode, UINT64_MAX);
                }
        }
    }
    sort_scand(all.c, all.n, sad_tie_less);
    const uint64_t screen_sad = all.c[0].sad;
    const int keep = fast ? 4 : 8;
    if (all.n > keep) all.n = keep;
    const double lam_d = 0.35 * (double)p->pqindex;
    const long double lambda_me = (long double)(lam_d > 1.0 ? lam_d : 1.0);
    for (int i = 0; i < all.n; ++i) {
        scand* c = &all.c[i];
        vc1cu_mv pred = pi->pre;
        c->rate = 0;
        if (pi->hybrid) {
            pred = modular_mv_distance(p, c->mv, pi->a) <= modular_mv_distance(p, c->mv, pi->c) ? pi->a : pi->c;
            ++c->rate;
        }
        c->rate += mv_rate_bits(p, c->mv, pred, mode, more);
        c->score = (long double)c->sad + lambda_me * (long double)c->rate;
    }
    int rw = 0;
    for (int i = 1; i < all.n; ++i) if (score_less(&all.c[i], &all.c[rw])) rw = i;
    const scand rate_winner = all.c[rw];
    if (p->me_quality == 1) {
        if (best_sad) *best_sad = screen_sad;
        return rate_winner.mv;
    }
    const uint64_t pct3 = (rate_winner.sad / 100) * 3 + (((rate_winner.sad % 100) * 3 + 99) / 100);
    const uint64_t slack = pct3 > 4 ? pct3 : 4;
    const uint64_t limit = rate_winner.sad > UINT64_MAX - slack ? UINT64_MAX : rate_winner.sad + slack;
    for (int i = 0; i < all.n; ++i) {
        scand* c = &all.c[i];
        c->eligible = c->sad < UINT64_MAX / 8 && c->sad <= limit;
        c->satd = c->eligible ? vo_block_satd_motion(p, cur, ref, x0, y0, bw, bh, c->mv.xq, c->mv.yq, mode) : BAD;
        c->score = (long double)c->satd + lambda_me * (long double)c->rate;
    }
    sort_scand(all.c, all.n, satd_order_less);
    if (best_sad) *best_sad = screen_sad;
    return all.c[0].mv;
}

static int qbetter(uint64_t sad, vc1cu_mv mv, uint64_t best, vc1cu_mv bmv) {
    if (sad != best) return sad < best;
    return tie_less(mv, bmv);
}

/* Vc1Encoder::refine_qpel_block, encoder_motion.cpp:3596-3685 */
static vc1cu_mv refine_qpel_block(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                                  int bw, int bh, vc1cu_mv seed, int range, uint64_t* best_sad, uint64_t known) {
    const int limit_q = 4 * p->subpel_range;
    if (!p->subpel || limit_q == 0 || imax(iabs(seed.xq), iabs(seed.yq)) > limit_q)
        return refine_integer_only(p, cur, ref, x0, y0, bw, bh, seed, range, VC1CU_MV_QPEL, best_sad, known);
    const bounds qb = bounds_qpel(range);
    const int xmin = imax(qb.xmin, -limit_q), xmax = imin(qb.xmax, limit_q);
    const int ymin = imax(qb.ymin, -limit_q), ymax = imin(qb.ymax, limit_q);
    seed.xq = iclamp(seed.xq, xmin, xmax);
    seed.yq = iclamp(seed.yq, ymin, ymax);
    if (vo_hidden_padding(p, x0, y0, bw, bh, seed.xq, seed.yq, VC1CU_MV_QPEL, chroma_gate(x0, y0, bw, bh))) {
        seed.xq = 0; seed.yq = 0;
        known = UINT64_MAX;
    }
    vc1cu_mv best = seed;
    uint64_t cost = known != UINT64_MAX ? known : vo_block_sad_qpel(p, cur, ref, x0, y0, bw, bh, best.xq, best.yq);
    vc1cu_mv seen[20];
    int ns = 1;
    seen[0] = seed;
#define SEEN_BEFORE(MV) ({ int f_ = 0; for (int i_ = 0; i_ < ns; ++i_) if (same_mv(seen[i_], (MV))) { f_ = 1; break; } if (!f_ && ns < 20) seen[ns++] = (MV); f_; })
#define EVAL(X, Y) do { vc1cu_mv m_ = {iclamp((X), xmin, xmax), iclamp((Y), ymin, ymax)}; if (!SEEN_BEFORE(m_)) { const uint64_t s_ = vo_block_sad_qpel(p, cur, ref, x0, y0, bw, bh, m_.xq, m_.yq); if (qbetter(s_, m_, cost, best)) { cost = s_; best = m_; } } } while (0)
    if (p->fast_subpel) {
        if (cost == 0 && best.xq == 0 && best.yq == 0) {
            if (best_sad) *best_sad = 0;
            return best;
        }
        EVAL(seed.xq - 2, seed.yq); EVAL(seed.xq + 2, seed.yq); EVAL(seed.xq, seed.yq - 2); EVAL(seed.xq, seed.yq + 2);
        const vc1cu_mv axis = best;
        const int dx = axis.xq - seed.xq, dy = axis.yq - seed.yq;
        if (dx && !dy) { EVAL(axis.xq, axis.yq - 2); EVAL(axis.xq, axis.yq + 2); }
        else if (dy && !dx) { EVAL(axis.xq - 2, axis.yq); EVAL(axis.xq + 2, axis.yq); }
        const vc1cu_mv half = best;
        EVAL(half.xq - 1, half.yq); EVAL(half.xq + 1, half.yq); EVAL(half.xq, half.yq - 1); EVAL(half.xq, half.yq + 1);
        const vc1cu_mv qa = best;
        const int qdx = qa.xq - half.xq, qdy = qa.yq - half.yq;
        if (qdx && !qdy) { EVAL(qa.xq, qa.yq - 1); EVAL(qa.xq, qa.yq + 1); }
        else if (qdy && !qdx) { EVAL(qa.xq - 1, qa.yq); EVAL(qa.xq + 1, qa.yq); }
    } else {
        for (int oy = -2; oy <= 2; oy += 2)
            for (int ox = -2; ox <= 2; ox += 2) EVAL(seed.xq + ox, seed.yq + oy);
        const vc1cu_mv half = best;
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) EVAL(half.xq + ox, half.yq + oy);
    }
#undef EVAL
#undef SEEN_BEFORE
    if (best_sad) *best_sad = cost;
    return best;
}

/* Vc1Encoder::refine_motion_block, encoder_motion.cpp:3687-3749 */
static vc1cu_mv refine_motion_block(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0, int y0,
                                    int bw, int bh, vc1cu_mv seed, int range, int mode, uint64_t* best_sad,
                                    uint64_t known) {
    if (!mode_halfpel(mode)) return refine_qpel_block(p, cur, ref, x0, y0, bw, bh, seed, range, best_sad, known);
    const int limit_q = 4 * p->subpel_range;
    if (!p->subpel || limit_q == 0 || imax(iabs(seed.xq), iabs(seed.yq)) > limit_q)
        return refine_integer_only(p, cur, ref, x0, y0, bw, bh, seed, range, mode, best_sad, known);
    const bounds qb = bounds_qpel(range);
    const int xmin = imax(qb.xmin, -limit_q), xmax = imin(qb.xmax, limit_q);
    const int ymin = imax(qb.ymin, -limit_q), ymax = imin(qb.ymax, limit_q);
    seed.xq = make_even(iclamp(seed.xq, xmin, xmax));
    seed.yq = make_even(iclamp(seed.yq, ymin, ymax));
    if (vo_hidden_padding(p, x0, y0, bw, bh, seed.xq, seed.yq, mode, chroma_gate(x0, y0, bw, bh))) {
        seed.xq = 0; seed.yq = 0;
        known = UINT64_MAX;
    }
    vc1cu_mv best = seed;
    uint64_t cost = known != UINT64_MAX ? known : vo_block_sad_motion(p, cur, ref, x0, y0, bw, bh, seed.xq, seed.yq, mode);
    vc1cu_mv seen[9];
    int ns = 1;
    seen[0] = seed;
    if (p->fast_subpel && cost == 0 && best.xq == 0 && best.yq == 0) {
        if (best_sad) *best_sad = 0;
        return best;
    }
#define EVAL(X, Y) do { vc1cu_mv m_ = {make_even(iclamp((X), xmin, xmax)), make_even(iclamp((Y), ymin, ymax))}; int f_ = 0; for (int i_ = 0; i_ < ns; ++i_) if (same_mv(seen[i_], m_)) { f_ = 1; break; } if (!f_ && ns < 9) seen[ns++] = m_; if (!f_) { const uint64_t s_ = vo_block_sad_motion(p, cur, ref, x0, y0, bw, bh, m_.xq, m_.yq, mode); if (qbetter(s_, m_, cost, best)) { cost = s_; best = m_; } } } while (0)
    if (p->fast_subpel) {
        EVAL(seed.xq - 2, seed.yq); EVAL(seed.xq + 2, seed.yq); EVAL(seed.xq, seed.yq - 2); EVAL(seed.xq, seed.yq + 2);
        const vc1cu_mv axis = best;
        const int dx = axis.xq - seed.xq, dy = axis.yq - seed.yq;
        if (dx && !dy) { EVAL(axis.xq, axis.yq - 2); EVAL(axis.xq, axis.yq + 2); }
        else if (dy && !dx) { EVAL(axis.xq - 2, axis.yq); EVAL(axis.xq + 2, axis.yq); }
    } else {
        for (int oy = -2; oy <= 2; oy += 2)
            for (int ox = -2; ox <= 2; ox += 2) EVAL(seed.xq + ox, seed.yq + oy);
    }
#undef EVAL
    if (best_sad) *best_sad = cost;
    return best;
}

/* ---- the whole core pass ----------------------------------------------------------- */

/* Vc1Encoder::visible_block_mean, encoder_entropy.cpp:496-509 */
static int visible_block_mean(const uint8_t* p, int w, int h, int x0, int y0) {
    const int vw = imax(0, imin(8, w - x0)), vh = imax(0, imin(8, h - y0));
    if (!vw || !vh) return 128;
    uint64_t sum = 0;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) sum += p[(size_t)(y0 + y) * w + x0 + x];
    const uint64_t n = (uint64_t)vw * vh;
    return (int)((sum + n / 2) / n);
}

/* Vc1Encoder::median4 / chroma_mv_4mv, encoder_motion_compensation.cpp:522-534 */
static int median4(int a, int b, int c, int d) {
    if (a < b) {
        if (c < d) return (imin(b, d) + imax(a, c)) / 2;
        return (imin(b, c) + imax(a, d)) / 2;
    }
    if (c < d) return (imin(a, d) + imax(b, c)) / 2;
    return (imin(a, c) + imax(b, d)) / 2;
}

/* The integer search of an unseeded pass for one macroblock, encoder_motion.cpp:106-225: UMH or
 * diamond about the predictor / global seeds, the propagated and content-signature long-range
 * candidates, their distant_* records (dl, dc, dd: this macroblock's entries). The long-range
 * index is built on first use into *cells. */
static cand unseeded_integer(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, int mx, int my,
                             const vc1cu_mv* mvs, uint8_t* propagated, int gdx, int gdy, lr_cell** cells, int* ncells,
                             double* dl, double* dc, uint8_t* dd) {
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t pos = (size_t)my * mbw + mx;
    const int range = p->search_range;
    const int local_range = imin(range, imax(0, p->local_search_range));
    const pinfo pi = predictor_info(mvs, mbw, mbh, mx, my);
    cand im = {UINT64_MAX, 0, 0};
    int selected_distant = 0;
    const uint64_t pixels = active_mb_pixels(p, mx, my);
    if (p->long_range_mode == 2) {
        /* VC1_LONG_RANGE_LEGACY_DISTANT_FIRST, encoder_motion.cpp:144-160 */
        int short_circuit = 0;
        if (range > local_range) {
            const cand pr = propagated_long_range(p, f, ref, mx, my, mbw, mvs, propagated, range);
            if (motion_match_good(p, pr.cost, mx, my)) { im = pr; short_circuit = 1; selected_distant = 1; }
        }
        if (!short_circuit)
            im = p->me_algorithm == 1
                     ? integer_motion_diamond(p, f, ref, mx, my, &pi, gdx, gdy, local_range)
                     : integer_motion_umh(p, f, ref, mx, my, &pi, gdx, gdy, local_range);
    } else {
        /* encoder_motion.cpp:161-196 */
        im = p->me_algorithm == 1
                 ? integer_motion_diamond(p, f, ref, mx, my, &pi, gdx, gdy, local_range)
                 : integer_motion_umh(p, f, ref, mx, my, &pi, gdx, gdy, local_range);
        const uint64_t local_sad = im.cost;
        if (pixels) *dl = (double)local_sad / (double)pixels;
        const int skip_distant = p->long_range_mode == 1 && motion_match_good(p, im.cost, mx, my);
        if (range > local_range && !skip_distant) {
            const cand pr = propagated_long_range(p, f, ref, mx, my, mbw, mvs, propagated, range);
            const int decision = distant_match_decision(p, pr.cost, local_sad, mx, my);
            if (pixels && pr.cost < UINT64_MAX / 8) {
                const double mae = (double)pr.cost / (double)pixels;
                if (*dc < 0.0 || mae < *dc) { *dc = mae; *dd = (uint8_t)decision; }
            }
            if (cand_less(pr.cost, pr.dx, pr.dy, im.cost, im.dx, im.dy) && decision >= 2) {
                im = pr;
                selected_distant = 1;
            }
        }
    }
    if (range > local_range && !motion_match_good(p, im.cost, mx, my)) {
        /* encoder_motion.cpp:201-225 */
        if (!*cells) {
            const int nx = (ref->w + 7) / 8, ny = (ref->h + 7) / 8;
            *cells = (lr_cell*)malloc(sizeof(lr_cell) * (size_t)nx * ny);
            *ncells = 0;
            for (int yy = 0; yy < ref->h; yy += 8)
                for (int xx = 0; xx < ref->w; xx += 8) {
                    (*cells)[*ncells].x = xx;
                    (*cells)[*ncells].y = yy;
                    (*cells)[*ncells].sig = lr_signature(ref, xx, yy);
                    ++*ncells;
                }
        }
        uint64_t ext_sad = UINT64_MAX;
        int ext_dec = 0;
        const cand ext = extended_content(p, f, ref, mx, my, range, *cells, *ncells, im, &ext_sad, &ext_dec);
        if (p->long_range_mode != 2 && pixels && ext_sad < UINT64_MAX / 8) {
            const double mae = (double)ext_sad / (double)pixels;
            if (*dc < 0.0 || mae < *dc) { *dc = mae; *dd = (uint8_t)ext_dec; }
        }
        if (ext.dx != im.dx || ext.dy != im.dy) { im = ext; selected_distant = 1; }
    }
    if (selected_distant) propagated[pos] = 1;
    return im;
}

/* Vc1Encoder::analyze_p_picture_core, encoder_motion.cpp:47-442 (me_quality != RD) */
int vo_analyze_p_core(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, int mode, int allow_intra,
                      const vc1cu_mv* shared_seed, const vc1cu_panalysis* seed_distant, vc1cu_panalysis* out) {
    if (f->w != p->width || f->h != p->height || ref->w != p->width || ref->h != p->height) return 1;
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    const int allow_4mv = mode == VC1CU_MV_MIXED;
    const int one_mode = allow_4mv ? VC1CU_MV_QPEL : mode;
    vc1cu_mv* mvs = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_mv* bmv = (vc1cu_mv*)calloc(mbs * 4, sizeof(vc1cu_mv));
    uint8_t* use4 = (uint8_t*)calloc(mbs, 1);
    uint8_t* intra = (uint8_t*)calloc(mbs, 1);
    uint8_t* propagated = (uint8_t*)calloc(mbs, 1);
    uint64_t* screen = (uint64_t*)calloc(mbs, sizeof(uint64_t));
    double* ratio = (double*)malloc(mbs * sizeof(double));
    double* dl = (double*)malloc(mbs * sizeof(double));
    double* dc = (double*)malloc(mbs * sizeof(double));
    uint8_t* dd = (uint8_t*)calloc(mbs, 1);
    lr_cell* cells = NULL;
    int ncells = 0;
    for (size_t i = 0; i < mbs; ++i) { ratio[i] = -1.0; dl[i] = -1.0; dc[i] = -1.0; }
    uint64_t total_sad = 0, rate_sad_total = 0, total_pixels = 0;
    uint64_t moved = 0, frac = 0, four_count = 0, intra_count = 0;
    int gdx = 0, gdy = 0;
    uint64_t gsad = 0;
    g_counts.macroblocks += mbs;
    if (p->search_range == 0) {
        /* encoder_motion.cpp:72-85 */
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx) {
                const uint64_t z = vo_mb_sad(p, f, ref, mx, my, 0, 0, 1);
                total_sad += z;
                screen[(size_t)my * mbw + mx] = z;
                total_pixels += active_mb_pixels(p, mx, my);
            }
        out->mean_abs_residual = total_pixels ? (double)total_sad / (double)total_pixels : 0.0;
        out->rate_complexity = out->mean_abs_residual;
        out->motion_sad = 0;
        goto emit;
    }
    {
        const int configured_range = p->search_range;
        const int local_range = imin(configured_range, imax(0, p->local_search_range));
        if (!shared_seed) vo_global_motion(p, f, ref, local_range, &gdx, &gdy, &gsad);
        if (shared_seed && seed_distant) {
            for (size_t i = 0; i < mbs; ++i) {
                if (seed_distant->distant_local_mae) dl[i] = seed_distant->distant_local_mae[i];
                if (seed_distant->distant_candidate_mae) dc[i] = seed_distant->distant_candidate_mae[i];
                if (seed_distant->distant_match_decision) dd[i] = seed_distant->distant_match_decision[i];
            }
        }
        const double lam_d = 0.35 * (double)p->pqindex;
        const double lambda = lam_d > 1.0 ? lam_d : 1.0;
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx) {
                const size_t pos = (size_t)my * mbw + mx;
                const int range = configured_range;
                const int x0 = mx * 16, y0 = my * 16;
                const pinfo rate_pi = predictor_info_mixed_1mv(bmv, intra, mbw, mbh, mx, my);
                uint64_t one_sad = 0;
                vc1cu_mv one = {0, 0};
                if (shared_seed) {
                    vc1cu_mv seed = shared_seed[pos];
                    const bounds qb = bounds_qpel(range);
                    seed.xq = iclamp(seed.xq, qb.xmin, qb.xmax);
                    seed.yq = iclamp(seed.yq, qb.ymin, qb.ymax);
                    one = refine_staged(p, f, ref, x0, y0, 16, 16, seed, range, one_mode, &rate_pi, 1, &one_sad, UINT64_MAX);
                } else {
                    const cand im = unseeded_integer(p, f, ref, mx, my, mvs, propagated, gdx, gdy, &cells, &ncells,
                                                     &dl[pos], &dc[pos], &dd[pos]);
                    const vc1cu_mv s4 = {im.dx * 4, im.dy * 4};
                    one = refine_staged(p, f, ref, x0, y0, 16, 16, s4, range, one_mode, &rate_pi, 1, &one_sad, im.cost);
                }
                if (vo_hidden_padding(p, x0, y0, 16, 16, one.xq, one.yq, one_mode, 1)) {
                    one.xq = 0; one.yq = 0;
                    one_sad = vo_block_sad_motion(p, f, ref, x0, y0, 16, 16, 0, 0, one_mode);
                }
                const uint64_t one_screen_sad = one_sad;
                mvs[pos] = one;
                for (int k = 0; k < 4; ++k) bmv[pos * 4 + k] = one;
                uint64_t chosen_sad = one_sad, temporal_screen_sad = one_screen_sad;
                if (allow_4mv) {
                    /* encoder_motion.cpp:250-374 (me_quality != RD branch) */
                    vc1cu_mv four[4];
                    for (int k = 0; k < 4; ++k) four[k] = bmv[pos * 4 + k];
                    uint64_t four_sad = 0, four_screen = 0, extra_bits = 1;
                    const int limit = 4 * p->subpel_range;
                    for (int k = 0; k < 4; ++k) {
                        const pinfo pi4 = predictor_info_4mv(bmv, intra, mbw, mbh, mx, my, k);
                        const vc1cu_mv pred = pi4.pre;
                        const int bx = x0 + (k & 1) * 8, by = y0 + ((k >> 1) & 1) * 8;
#define WSR(M) do { if (imax(iabs((M).xq), iabs((M).yq)) > limit) { (M).xq = ((M).xq / 4) * 4; (M).yq = ((M).yq / 4) * 4; } } while (0)
                        vc1cu_mv best_seed = one;
                        WSR(best_seed);
                        uint64_t seed_cost = vo_block_sad_qpel(p, f, ref, bx, by, 8, 8, best_seed.xq, best_seed.yq);
                        const vc1cu_mv seeds[10] = {one, pred, {one.xq - 8, one.yq}, {one.xq + 8, one.yq},
                                                    {one.xq, one.yq - 8}, {one.xq, one.yq + 8}, {one.xq - 4, one.yq},
                                                    {one.xq + 4, one.yq}, {one.xq, one.yq - 4}, {one.xq, one.yq + 4}};
                        const bounds qb = bounds_qpel(range);
                        for (int s = 0; s < 10; ++s) {
                            vc1cu_mv sd = seeds[s];
                            sd.xq = iclamp(sd.xq, qb.xmin, qb.xmax);
                            sd.yq = iclamp(sd.yq, qb.ymin, qb.ymax);
                            WSR(sd);
                            if (same_mv(sd, best_seed)) continue;
                            const uint64_t c = vo_block_sad_qpel(p, f, ref, bx, by, 8, 8, sd.xq, sd.yq);
                            const int cm = iabs(sd.xq) + iabs(sd.yq), bm = iabs(best_seed.xq) + iabs(best_seed.yq);
                            if (c < seed_cost || (c == seed_cost && cm < bm)) { seed_cost = c; best_seed = sd; }
                        }
#undef WSR
                        uint64_t bsad = 0;
                        const vc1cu_mv mv = refine_staged(p, f, ref, bx, by, 8, 8, best_seed, range, VC1CU_MV_MIXED, &pi4,
                                                          1, &bsad, seed_cost);
                        four_screen += bsad;
                        four[k] = mv;
                        bmv[pos * 4 + k] = mv;
                        four_sad += bsad;
                        vc1cu_mv actual = pi4.pre;
                        if (pi4.hybrid) {
                            const int da = modular_mv_distance(p, mv, pi4.a), dcc = modular_mv_distance(p, mv, pi4.c);
                            actual = (da <= dcc) ? pi4.a : pi4.c;
                            ++extra_bits;
                        }
                        if (!same_mv(mv, actual)) {
                            /* MvDataSyntax est{dx,dy,false}: more=false, qpel */
                            extra_bits += mv_rate_bits(p, mv, actual, VC1CU_MV_MIXED, 0);
                        }
                    }
                    const vc1cu_mv cmv = {median4(four[0].xq, four[1].xq, four[2].xq, four[3].xq),
                                          median4(four[0].yq, four[1].yq, four[2].yq, four[3].yq)};
                    const int four_chroma_safe = !hidden_chroma(p, x0, y0, 16, 16, cmv.xq, cmv.yq);
                    int choose4 = 0;
                    if (four_chroma_safe)
                        choose4 = four_sad + (uint64_t)llround(lambda * (double)extra_bits) + 8 <
                                  (uint64_t)llround((double)one_sad * 0.985);
                    if (choose4) {
                        for (int k = 0; k < 4; ++k) bmv[pos * 4 + k] = four[k];
                        use4[pos] = 1;
                        mvs[pos] = four[0];
                        ++four_count;
                        chosen_sad = four_sad;
                        temporal_screen_sad = four_screen;
                    } else {
                        for (int k = 0; k < 4; ++k) bmv[pos * 4 + k] = one;
                        mvs[pos] = one;
                        temporal_screen_sad = one_screen_sad;
                    }
                }
                const uint64_t temporal_sad = chosen_sad;
                screen[pos] = temporal_screen_sad;
                if (allow_intra && !p->disable_p_intra) {
                    /* encoder_motion.cpp:384-415 */
                    uint64_t intra_sad = 0;
                    for (int k = 0; k < 4; ++k) {
                        const int bx = x0 + (k & 1) * 8, by = y0 + ((k >> 1) & 1) * 8;
                        const int mean = visible_block_mean(f->y, p->width, p->height, bx, by);
                        for (int yy = 0; yy < 8 && by + yy < p->height; ++yy)
                            for (int xx = 0; xx < 8 && bx + xx < p->width; ++xx)
                                intra_sad += (uint64_t)iabs((int)f->y[(size_t)(by + yy) * p->width + bx + xx] - mean);
                    }
                    const uint64_t intra_rate = (uint64_t)llround(lambda * 72.0);
                    ratio[pos] = temporal_screen_sad > 0 ? (double)(intra_sad + intra_rate) / (double)temporal_screen_sad
                                                         : HUGE_VAL;
                    if (intra_sad + intra_rate <
                        (uint64_t)llround((double)temporal_screen_sad * p->inter_intra_threshold)) {
                        intra[pos] = 1;
                        use4[pos] = 0;
                        mvs[pos].xq = mvs[pos].yq = 0;
                        for (int k = 0; k < 4; ++k) { bmv[pos * 4 + k].xq = 0; bmv[pos * 4 + k].yq = 0; }
                        ++intra_count;
                        chosen_sad = intra_sad;
                    }
                }
                int mv_moved = 0, mv_frac = 0;
                for (int k = 0; k < 4; ++k) {
                    const vc1cu_mv m = bmv[pos * 4 + k];
                    mv_moved |= m.xq != 0 || m.yq != 0;
                    mv_frac |= (m.xq % 8) != 0 || (m.yq % 8) != 0;
                }
                moved += mv_moved;
                frac += mv_frac;
                total_sad += chosen_sad;
                rate_sad_total += temporal_sad;
                total_pixels += active_mb_pixels(p, mx, my);
            }
        const double local_mad = total_pixels ? (double)total_sad / (double)total_pixels : 0.0;
        const double global_mad = shared_seed ? local_mad
                                              : ((p->width > 0 && p->height > 0)
                                                     ? (double)gsad / (double)((uint64_t)p->width * p->height) : 0.0);
        out->mean_abs_residual = local_mad < global_mad ? local_mad : global_mad;
        const double rate_local = total_pixels ? (double)rate_sad_total / (double)total_pixels : 0.0;
        out->rate_complexity = rate_local < global_mad ? rate_local : global_mad;
        out->motion_sad = total_sad;
    }
emit:
    for (size_t i = 0; i < mbs; ++i) {
        if (out->mvs) out->mvs[i] = mvs[i];
        if (out->block_mvs) for (int k = 0; k < 4; ++k) out->block_mvs[i * 4 + k] = bmv[i * 4 + k];
        if (out->use_4mv) out->use_4mv[i] = use4[i];
        if (out->use_intra) out->use_intra[i] = intra[i];
        if (out->screen_sads) out->screen_sads[i] = screen[i];
        if (out->inter_intra_cost_ratio) out->inter_intra_cost_ratio[i] = ratio[i];
        if (out->distant_local_mae) out->distant_local_mae[i] = dl[i];
        if (out->distant_candidate_mae) out->distant_candidate_mae[i] = dc[i];
        if (out->distant_match_decision) out->distant_match_decision[i] = dd[i];
    }
    out->moved_macroblocks = moved;
    out->fractional_chroma_macroblocks = frac;
    out->four_mv_macroblocks = four_count;
    out->intra_macroblocks = intra_count;
    out->global_dx = gdx;
    out->global_dy = gdy;
    out->global_full_sad = gsad;
    free(mvs); free(bmv); free(use4); free(intra); free(propagated); free(screen); free(ratio); free(dl); free(dc);
    free(dd); free(cells);
    return 0;
}

/* ---- prediction --------------------------------------------------------------------- */

/* motion_compensate_mb / motion_compensate_4mv, encoder_motion_compensation.cpp:474-600 */
void vo_motion_compensate(const vc1cu_params* p, const vo_frame* ref, const vc1cu_mv* mvs, const vc1cu_mv* block_mvs,
                          const uint8_t* use_4mv, int mode, uint8_t* dy, uint8_t* du, uint8_t* dv) {
    const int W = p->width, H = p->height, mbw = mbw_of(p), mbh = mbh_of(p);
    const int cw = W / 2, ch = H / 2;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = (size_t)my * mbw + mx;
            const int x0 = mx * 16, y0 = my * 16;
            vc1cu_mv cmv;
            if (use_4mv && use_4mv[pos]) {
                vc1cu_mv m4[4];
                for (int k = 0; k < 4; ++k) m4[k] = block_mvs[pos * 4 + k];
                for (int k = 0; k < 4; ++k) {
                    const int bx = x0 + (k & 1) * 8, by = y0 + ((k >> 1) & 1) * 8;
                    const int bw = imax(0, imin(8, W - bx)), bh = imax(0, imin(8, H - by));
                    for (int y = 0; y < bh; ++y)
                        for (int x = 0; x < bw; ++x)
                            dy[(size_t)(by + y) * W + bx + x] =
                                (uint8_t)luma_mc_sample(ref->y, W, H, bx + x, by + y, m4[k].xq, m4[k].yq, p->rnd);
                }
                cmv.xq = median4(m4[0].xq, m4[1].xq, m4[2].xq, m4[3].xq);
                cmv.yq = median4(m4[0].yq, m4[1].yq, m4[2].yq, m4[3].yq);
            } else {
                const vc1cu_mv mv = mvs[pos];
                const int vw = imax(0, imin(16, W - x0)), vh = imax(0, imin(16, H - y0));
                for (int y = 0; y < vh; ++y)
                    for (int x = 0; x < vw; ++x)
                        dy[(size_t)(y0 + y) * W + x0 + x] =
                            (uint8_t)luma_mc_sample_mode(ref->y, W, H, x0 + x, y0 + y, mv.xq, mv.yq, mode, p->rnd);
                cmv = mv;
            }
            const int cx0 = mx * 8, cy0 = my * 8;
            const int cvw = imax(0, imin(8, cw - cx0)), cvh = imax(0, imin(8, ch - cy0));
            for (int y = 0; y < cvh; ++y)
                for (int x = 0; x < cvw; ++x) {
                    const size_t off = (size_t)(cy0 + y) * cw + cx0 + x;
                    if (du) du[off] = (uint8_t)chroma_mc_sample(ref->u, cw, ch, cx0 + x, cy0 + y, cmv.xq, cmv.yq, 0, p->rnd);
                    if (dv) dv[off] = (uint8_t)chroma_mc_sample(ref->v, cw, ch, cx0 + x, cy0 + y, cmv.xq, cmv.yq, 0, p->rnd);
                }
        }
}

/* ---- forward transform + quantiser ------------------------------------------------ */

/* forward_transform::k4 / k8, forward_transform_tables.h:9-25 (inverse VC-1 basis) */
static const double k4[4][4] = {
    {0.0147058823529412, 0.0147058823529412, 0.0147058823529412, 0.0147058823529412},
    {0.0188356164383562, 0.0085616438356164, -0.0085616438356164, -0.0188356164383562},
    {0.0147058823529412, -0.0147058823529412, -0.0147058823529412, 0.0147058823529412},
    {0.0085616438356164, -0.0188356164383562, 0.0188356164383562, -0.0085616438356164}};
static const double k8[8][8] = {
    {0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667},
    {0.013840830450, 0.012975778547, 0.007785467128, 0.003460207612, -0.003460207612, -0.007785467128, -0.012975778547, -0.013840830450},
    {0.013698630137, 0.005136986301, -0.005136986301, -0.013698630137, -0.013698630137, -0.005136986301, 0.005136986301, 0.013698630137},
    {0.012975778547, -0.003460207612, -0.013840830450, -0.007785467128, 0.007785467128, 0.013840830450, 0.003460207612, -0.012975778547},
    {0.010416666667, -0.010416666667, -0.010416666667, 0.010416666667, 0.010416666667, -0.010416666667, -0.010416666667, 0.010416666667},
    {0.007785467128, -0.013840830450, 0.003460207612, 0.012975778547, -0.012975778547, -0.003460207612, 0.013840830450, -0.007785467128},
    {0.005136986301, -0.013698630137, 0.013698630137, -0.005136986301, -0.005136986301, 0.013698630137, -0.013698630137, 0.005136986301},
    {0.003460207612, -0.007785467128, 0.012975778547, -0.013840830450, 0.013840830450, -0.012975778547, 0.007785467128, -0.003460207612}};

/* forward_transform_residual (:797-913, scalar :881-912) and forward_transform_residual_part
 * (:935-1045, scalar :1011-1044), encoder_transform.cpp */
void vo_forward_part(const uint8_t* src, const uint8_t* pred, int w, int h, int x0, int y0, int bw, int bh,
                     double out[64]) {
    double r[8][8], tmp[8][8], xf[8][8];
    memset(r, 0, sizeof r);
    memset(tmp, 0, sizeof tmp);
    memset(xf, 0, sizeof xf);
    for (int i = 0; i < 64; ++i) out[i] = 0.0;
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) {
            const int sx = x0 + x, sy = y0 + y;
            if (sx < 0 || sy < 0 || sx >= w || sy >= h) { r[y][x] = 0.0; continue; }
            const size_t off = (size_t)sy * w + sx;
            r[y][x] = (double)((int)src[off] - (int)pred[off]);
        }
    for (int a = 0; a < bh; ++a)
        for (int x = 0; x < bw; ++x)
            for (int y = 0; y < bh; ++y) tmp[a][x] += (bh == 8 ? k8[a][y] : k4[a][y]) * r[y][x];
    for (int a = 0; a < bh; ++a)
        for (int b = 0; b < bw; ++b)
            for (int x = 0; x < bw; ++x) xf[a][b] += tmp[a][x] * (bw == 8 ? k8[b][x] : k4[b][x]);
    g_counts.xform_flops += (uint64_t)2 * (bh * bw * bh + bh * bw * bw);
    if (bw == 8 && bh == 8) {
        for (int row = 0; row < 8; ++row)
            for (int col = 0; col < 8; ++col) out[row * 8 + col] = 1024.0 * xf[col][row];
    } else {
        for (int row = 0; row < bh; ++row)
            for (int col = 0; col < bw; ++col) out[row * 8 + col] = 1024.0 * xf[row][col];
    }
}

/* Vc1Encoder::scalar_quantize_level, encoder_transform.cpp:1067-1085 (+picture_double_quant
 * :1052-1056, max_quantized_level encoder_entropy.cpp:208-218), mquant = PQINDEX */
int vo_quantize_level(const vc1cu_params* p, double coeff) {
    g_counts.quant_coeffs++;
    const int mq = p->pqindex;
    if (coeff == 0.0) return 0;
    const int sign = coeff < 0.0 ? -1 : 1;
    const double a = fabs(coeff);
    const double dq = (double)(2 * mq + (p->halfqp ? 1 : 0));
    const double offset = p->nonuniform ? (double)mq : 0.0;
    const int max_level = (1 << (p->pqindex < 8 ? 11 : 8)) - 1;
    int center = (int)llround((a - offset) / (dq > 1.0 ? dq : 1.0));
    center = iclamp(center, 1, max_level);
    int best = 0;
    double besterr = a * a;
    for (int n = imax(1, center - 1); n <= imin(max_level, center + 1); ++n) {
        const double recon = (double)n * dq + offset;
        const double e = a - recon;
        if (e * e < besterr) { besterr = e * e; best = n; }
    }
    return sign * best;
}

/* transform_part_geometry, encoder_transform.cpp:924-933 */
static void part_geometry(int t, int part, int* ox, int* oy, int* bw, int* bh) {
    *ox = *oy = 0; *bw = *bh = 8;
    if (t == 2) { *bw = 8; *bh = 4; *oy = part * 4; }
    else if (t == 3) { *bw = 4; *bh = 8; *ox = part * 4; }
    else if (t == 4) { *bw = 4; *bh = 4; *ox = (part & 1) * 4; *oy = (part >> 1) * 4; }
}

/* quantize_inter_part at trellis 0 for every MB / parent / type (evaluate_transform_parent,
 * encoder_transform.cpp:1555-1576; quantize_inter_part :1087-1171 scalar branch) */
void vo_forward_quant(const vc1cu_params* p, const vo_frame* src, const vo_frame* pred, int type_mask,
                      double* coeffs, int16_t* levels) {
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    size_t ti = 0;
    for (int t = 1; t <= 4; ++t) {
        if (!(type_mask & (1 << (t - 1)))) continue;
        const int np = t == 1 ? 1 : (t == 4 ? 4 : 2);
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx)
                for (int k = 0; k < 6; ++k) {
                    const int chroma = k >= 4;
                    const uint8_t* sp = chroma ? (k == 4 ? src->u : src->v) : src->y;
                    const uint8_t* pp = chroma ? (k == 4 ? pred->u : pred->v) : pred->y;
                    const int w = chroma ? p->width / 2 : p->width, h = chroma ? p->height / 2 : p->height;
                    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
                    const size_t base = ((ti * mbs + (size_t)my * mbw + mx) * 6 + (size_t)k) * 64;
                    double cc[64];
                    int16_t qq[64];
                    memset(cc, 0, sizeof cc);
                    memset(qq, 0, sizeof qq);
                    for (int part = 0; part < np; ++part) {
                        int ox, oy, bw, bh;
                        part_geometry(t, part, &ox, &oy, &bw, &bh);
                        const int px = bx * 8 + ox, py = by * 8 + oy;
                        if (px >= w || py >= h || px + bw <= 0 || py + bh <= 0) continue;
                        double co[64];
                        vo_forward_part(sp, pp, w, h, px, py, bw, bh, co);
                        for (int y = 0; y < bh; ++y)
                            for (int x = 0; x < bw; ++x) {
                                cc[(oy + y) * 8 + ox + x] = co[y * 8 + x];
                                qq[(oy + y) * 8 + ox + x] = (int16_t)vo_quantize_level(p, co[y * 8 + x]);
                            }
                    }
                    if (coeffs) memcpy(coeffs + base, cc, sizeof cc);
                    if (levels) memcpy(levels + base, qq, sizeof qq);
                }
        ++ti;
    }
}

/* ---- score emulation ---------------------------------------------------------------- */

/*
 * The staged refinement ranks candidates by sad + lambda*rate in long double
 * (encoder_motion.cpp:3458-3476, :3518-3524). lambda = max(1, 0.35*PQ) is a double, so
 * lambda = m * 2^-s exactly (m < 2^53) and the exact sum is (sad*2^s + m*rate) * 2^-s;
 * the long double value is that integer rounded to mant_bits significant bits (64 for
 * x87, 113 for binary128), nearest-even. All candidates of one call share s, so these
 * scaled integers order exactly like the reference's long doubles.
 */
void vo_score_key(uint64_t sad, double lambda, uint64_t rate, int mant_bits, uint64_t* hi, uint64_t* lo) {
    int e;
    const double fr = frexp(lambda, &e); /* lambda = fr * 2^e, fr in [0.5,1) */
    const uint64_t m = (uint64_t)ldexp(fr, 53);
    const int s = 53 - e;                /* lambda = m * 2^-s */
    unsigned __int128 v = ((unsigned __int128)sad << s) + (unsigned __int128)m * rate;
    /* round to mant_bits significant bits, ties to even */
    int nbits = 0;
    for (unsigned __int128 t = v; t; t >>= 1) ++nbits;
    if (nbits > mant_bits) {
        const int drop = nbits - mant_bits;
        const unsigned __int128 one = 1;
        const unsigned __int128 mask = (one << drop) - 1;
        const unsigned __int128 rem = v & mask, half = one << (drop - 1);
        v >>= drop;
        if (rem > half || (rem == half && (v & 1))) v += 1;
        v <<= drop;
    }
    *hi = (uint64_t)(v >> 64);
    *lo = (uint64_t)v;
}

/* ---- B-picture analysis ------------------------------------------------------------- */

/* scale_direct of Vc1Encoder::analyze_b_picture_mode, encoder_motion.cpp:819-833: the
 * direct-mode vector of a collocated anchor MV, BFRACTION-scaled and pulled into the
 * decoder's MV range */
static vc1cu_mv b_scale_direct(const vc1cu_params* p, vc1cu_mv col, int bfrac, int inverse, int mode, int mx,
                               int my) {
    const int n = inverse ? bfrac - 256 : bfrac;
    vc1cu_mv mv;
    if (mode_halfpel(mode)) {
        mv.xq = 2 * arshift(col.xq * n + 255, 9);
        mv.yq = 2 * arshift(col.yq * n + 255, 9);
    } else {
        mv.xq = arshift(col.xq * n + 128, 8);
        mv.yq = arshift(col.yq * n + 128, 8);
    }
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    mv.xq = iclamp(mv.xq, -60 - mx * 64, mbw * 64 - 4 - mx * 64);
    mv.yq = iclamp(mv.yq, -60 - my * 64, mbh * 64 - 4 - my * 64);
    return mv;
}

/* motion_uses_hidden_padding(x0, y0, 16, 16, mv, mode, chroma = true, future) */
static int b_unsafe(const vc1cu_params* p, int x0, int y0, vc1cu_mv mv, int mode, int future) {
    return hidden_luma(p, x0, y0, 16, 16, mv.xq, mv.yq, mode) || hidden_chroma_f(p, x0, y0, 16, 16, mv.xq, mv.yq, future);
}

/* The four candidate costs of one B macroblock (encoder_motion.cpp:844-888): SAD of the
 * forward, backward, interpolated ((pf+pb+1)>>1) and direct predictions over the coded
 * raster, each replaced by 2^54 when a reference it uses reads hidden padding. Also the
 * four-8x8 mean proxy of the B-intra decision (:936-943). */
void vo_b_costs(const vc1cu_params* p, const vo_frame* f, const vo_frame* past, const vo_frame* future, int mx,
                int my, vc1cu_mv fm, vc1cu_mv bm, vc1cu_mv df, vc1cu_mv db, int mode, uint64_t out[5]) {
    const int x0 = mx * 16, y0 = my * 16;
    const int vw = imin(16, p->width - x0), vh = imin(16, p->height - y0);
    uint8_t pf[256], pb[256], pdf[256], pdb[256];
    memset(pf, 0, sizeof pf); memset(pb, 0, sizeof pb); memset(pdf, 0, sizeof pdf); memset(pdb, 0, sizeof pdb);
    vo_predict_luma(p, past, x0, y0, vw, vh, fm.xq, fm.yq, mode, pf, 16);
    vo_predict_luma(p, future, x0, y0, vw, vh, bm.xq, bm.yq, mode, pb, 16);
    vo_predict_luma(p, past, x0, y0, vw, vh, df.xq, df.yq, mode, pdf, 16);
    vo_predict_luma(p, future, x0, y0, vw, vh, db.xq, db.yq, mode, pdb, 16);
    uint64_t cf = 0, cb = 0, ci = 0, cd = 0;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) {
            const int o = y * 16 + x;
            const int src = f->y[(size_t)(y0 + y) * p->width + x0 + x];
            cf += (uint64_t)iabs(src - pf[o]);
            cb += (uint64_t)iabs(src - pb[o]);
            ci += (uint64_t)iabs(src - ((pf[o] + pb[o] + 1) >> 1));
            cd += (uint64_t)iabs(src - ((pdf[o] + pdb[o] + 1) >> 1));
        }
    const uint64_t invalid = (uint64_t)1 << 54;
    const int safe_fm = !b_unsafe(p, x0, y0, fm, mode, 0), safe_bm = !b_unsafe(p, x0, y0, bm, mode, 1);
    const int safe_df = !b_unsafe(p, x0, y0, df, mode, 0), safe_db = !b_unsafe(p, x0, y0, db, mode, 1);
    if (!safe_fm) cf = invalid;
    if (!safe_bm) cb = invalid;
    if (!safe_fm || !safe_bm) ci = invalid;
    if (!safe_df || !safe_db) cd = invalid;
    uint64_t intra_sad = 0;
    for (int k = 0; k < 4; ++k) {
        const int bx = x0 + (k & 1) * 8, by = y0 + ((k >> 1) & 1) * 8;
        const int mean = visible_block_mean(f->y, p->width, p->height, bx, by);
        for (int yy = 0; yy < 8 && by + yy < p->height; ++yy)
            for (int xx = 0; xx < 8 && bx + xx < p->width; ++xx)
                intra_sad += (uint64_t)iabs((int)f->y[(size_t)(by + yy) * p->width + bx + xx] - mean);
    }
    out[0] = cf; out[1] = cb; out[2] = ci; out[3] = cd; out[4] = intra_sad;
}

/* Vc1Encoder::analyze_b_picture_mode, encoder_motion.cpp:753-1005 (Advanced Profile
 * predictors, no minimal zero-motion shortcut: that configuration check is the caller's). */
int vo_analyze_b(const vc1cu_params* p, const vo_frame* f, const vo_frame* past, const vo_frame* future,
                 const vc1cu_mv* anchor_mvs, const uint8_t* anchor_4mv, int fraction_num, int fraction_den,
                 int mode, vc1cu_banalysis* out) {
    if (!((fraction_den == 2 && fraction_num == 1) || (fraction_den == 3 && (fraction_num == 1 || fraction_num == 2))))
        return 1;
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    vc1cu_mv* fmv = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_mv* bmv = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    uint64_t* fscreen = (uint64_t*)calloc(mbs, sizeof(uint64_t));
    uint64_t* bscreen = (uint64_t*)calloc(mbs, sizeof(uint64_t));
    vc1cu_mv* ofm = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_mv* obm = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_panalysis fa, ba;
    memset(&fa, 0, sizeof fa);
    memset(&ba, 0, sizeof ba);
    fa.mvs = fmv; fa.screen_sads = fscreen;
    fa.distant_local_mae = out->forward_distant_local_mae;
    fa.distant_candidate_mae = out->forward_distant_candidate_mae;
    fa.distant_match_decision = out->forward_distant_match_decision;
    ba.mvs = bmv; ba.screen_sads = bscreen;
    ba.distant_local_mae = out->backward_distant_local_mae;
    ba.distant_candidate_mae = out->backward_distant_candidate_mae;
    ba.distant_match_decision = out->backward_distant_match_decision;
    int rc = vo_analyze_p_core(p, f, past, mode, 0, NULL, NULL, &fa);
    if (!rc) rc = vo_analyze_p_core(p, f, future, mode, 0, NULL, NULL, &ba);
    if (rc) goto done;
    {
        const int bfrac = fraction_den == 2 ? 128 : (fraction_num == 1 ? 85 : 170);
        const int below_half = 2 * fraction_num < fraction_den;
        const double lambda = fmax(1.0, 0.45 * (double)p->pqindex);
        const uint64_t intra_guard = (uint64_t)llround(lambda * 72.0);
        const uint64_t intra_marker_bits =
            (uint64_t)(kMvDiffBits0[35] > kMvDiffBits0[72] ? kMvDiffBits0[35] : kMvDiffBits0[72]) + 1u;
        const uint64_t ftype = below_half ? 1u : 2u, btype = below_half ? 2u : 1u;
        uint64_t sel_sad = 0, rate_sad = 0, sel_rate = 1, sel_pixels = 0;
        uint64_t nf = 0, nb = 0, ni = 0, nd = 0, nintra = 0, moved = 0, frac = 0;
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx) {
                const size_t pos = (size_t)my * mbw + mx;
                const vc1cu_mv df = b_scale_direct(p, anchor_mvs[pos], bfrac, 0, mode, mx, my);
                const vc1cu_mv db = b_scale_direct(p, anchor_mvs[pos], bfrac, 1, mode, mx, my);
                const vc1cu_mv fm = fmv[pos], bm = bmv[pos];
                uint64_t c[5];
                vo_b_costs(p, f, past, future, mx, my, fm, bm, df, db, mode, c);
                const vc1cu_mv fpred = predictor_info(ofm, mbw, mbh, mx, my).pre;
                const vc1cu_mv bpred = predictor_info(obm, mbw, mbh, mx, my).pre;
                const uint64_t fbits = mv_rate_bits(p, fm, fpred, mode, 0);
                const uint64_t bbits = mv_rate_bits(p, bm, bpred, mode, 0);
                const uint64_t ibits = mv_rate_bits(p, bm, bpred, mode, 1) + mv_rate_bits(p, fm, fpred, mode, 0) + 2;
                const uint64_t penalty = anchor_4mv[pos] ? 1000000000ull : 0ull;
                /* candidate order Direct, Forward, Backward, Interpolated (:920-925) */
                const int cmode[4] = {VC1CU_BMB_DIRECT, VC1CU_BMB_FORWARD, VC1CU_BMB_BACKWARD, VC1CU_BMB_INTERPOLATED};
                const uint64_t ccost[4] = {c[3] + penalty, c[0] + penalty, c[1] + penalty, c[2]};
                const uint64_t crate[4] = {0, fbits + ftype, bbits + btype, ibits};
                int best = 0;
                long double best_score = (long double)ccost[0] + (long double)(lambda * (double)crate[0]);
                for (int k = 1; k < 4; ++k) {
                    const long double sc = (long double)ccost[k] + (long double)(lambda * (double)crate[k]);
                    if (sc < best_score) { best_score = sc; best = k; }
                }
                const uint64_t intra_sad = c[4];
                uint64_t gate = ccost[best];
                if (fscreen[pos] < gate) gate = fscreen[pos];
                if (bscreen[pos] < gate) gate = bscreen[pos];
                if (out->inter_intra_cost_ratio)
                    out->inter_intra_cost_ratio[pos] =
                        gate > 0 ? (double)(intra_sad + intra_guard) / (double)gate : INFINITY;
                const int choose_intra =
                    !p->disable_b_intra &&
                    intra_sad + intra_guard < (uint64_t)llround((double)gate * p->inter_intra_threshold);
                sel_sad += choose_intra ? intra_sad : ccost[best];
                rate_sad += ccost[best];
                sel_rate += choose_intra ? intra_marker_bits : crate[best];
                sel_pixels += (uint64_t)imax(0, imin(16, p->width - mx * 16)) * (uint64_t)imax(0, imin(16, p->height - my * 16));
                int m;
                vc1cu_mv of, ob;
                if (choose_intra) {
                    m = VC1CU_BMB_INTRA;
                    of.xq = of.yq = ob.xq = ob.yq = 0;
                    ++nintra;
                } else {
                    m = cmode[best];
                    if (m == VC1CU_BMB_DIRECT) { of = df; ob = db; ++nd; }
                    else if (m == VC1CU_BMB_FORWARD) { of = fm; ob = db; ++nf; }
                    else if (m == VC1CU_BMB_BACKWARD) { of = df; ob = bm; ++nb; }
                    else { of = fm; ob = bm; ++ni; }
                }
                ofm[pos] = of;
                obm[pos] = ob;
                if (out->modes) out->modes[pos] = (uint8_t)m;
                if (of.xq || of.yq || ob.xq || ob.yq) ++moved;
#define VO_FRAC_CHROMA(v) (((v).xq & 3) || ((v).yq & 3) || (((v).xq / 4) & 1) || (((v).yq / 4) & 1))
                if (VO_FRAC_CHROMA(of) || VO_FRAC_CHROMA(ob)) ++frac;
#undef VO_FRAC_CHROMA
            }
        if (out->forward_mvs) memcpy(out->forward_mvs, ofm, mbs * sizeof(vc1cu_mv));
        if (out->backward_mvs) memcpy(out->backward_mvs, obm, mbs * sizeof(vc1cu_mv));
        out->forward_macroblocks = nf;
        out->backward_macroblocks = nb;
        out->interpolated_macroblocks = ni;
        out->direct_macroblocks = nd;
        out->intra_macroblocks = nintra;
        out->moved_macroblocks = moved;
        out->fractional_chroma_macroblocks = frac;
        out->mean_abs_residual = sel_pixels ? (double)sel_sad / (double)sel_pixels : 0.0;
        out->rate_complexity = sel_pixels ? (double)rate_sad / (double)sel_pixels : 0.0;
        out->motion_sad = sel_sad;
        out->motion_bits = sel_rate;
        out->mv_mode = mode;
    }
done:
    free(fmv); free(bmv); free(fscreen); free(bscreen); free(ofm); free(obm);
    return rc;
}

/* ---- intensity compensation --------------------------------------------------------- */

/* The LUMSCALE / LUMSHIFT luma law of Vc1Encoder::intensity_map_y,
 * encoder_motion_compensation.cpp:175-187 (scale and shift of (scale*v + shift + 32) >> 6) */
static void ic_luma_law(int lumscale, int lumshift, int* scale, int* shift) {
    if (lumscale == 0) {
        *scale = -64;
        *shift = (255 - lumshift * 2) * 64;
        if (lumshift > 31) *shift += 128 * 64;
    } else {
        *scale = lumscale + 32;
        *shift = (lumshift > 31 ? lumshift - 64 : lumshift) * 64;
    }
}
static int ic_map_y(int v, int scale, int shift) { return iclamp((scale * v + shift + 32) >> 6, 0, 255); }

/* Vc1Encoder::intensity_compensated_reference, encoder_motion_compensation.cpp:195-294, with
 * intensity_map_uv (:189-193) for chroma; a plain copy when the compensation is off */
void vo_intensity_compensate(const vo_frame* ref, const vc1cu_intensity* ic, uint8_t* y, uint8_t* u, uint8_t* v) {
    const size_t ny = (size_t)ref->w * ref->h, nc = (size_t)(ref->w / 2) * (ref->h / 2);
    if (!ic->enabled) {
        memcpy(y, ref->y, ny);
        if (ref->u) memcpy(u, ref->u, nc); else memset(u, 128, nc);
        if (ref->v) memcpy(v, ref->v, nc); else memset(v, 128, nc);
        return;
    }
    int scale, shift;
    ic_luma_law(ic->lumscale, ic->lumshift, &scale, &shift);
    for (size_t i = 0; i < ny; ++i) y[i] = (uint8_t)ic_map_y(ref->y[i], scale, shift);
    const int cs = ic->lumscale == 0 ? -64 : ic->lumscale + 32;
    for (size_t i = 0; i < nc; ++i) {
        const int cu = ref->u ? ref->u[i] : 128, cv = ref->v ? ref->v[i] : 128;
        u[i] = (uint8_t)iclamp((cs * (cu - 128) + 128 * 64 + 32) >> 6, 0, 255);
        v[i] = (uint8_t)iclamp((cs * (cv - 128) + 128 * 64 + 32) >> 6, 0, 255);
    }
}

/* Vc1Encoder::estimate_intensity_comp, encoder_motion_compensation.cpp:296-348: one sample per
 * 4x4 luma cell along the MV field, a long double least-squares fit cur ~ a*ref + b, then the
 * (LUMSCALE, shift) pair of smallest sample SAD in the fit's 7x7 neighbourhood. */
void vo_estimate_intensity_comp(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, const vc1cu_mv* mvs,
                                vc1cu_intensity* out) {
    const int mbw = mbw_of(p), mbh = mbh_of(p), W = p->width, H = p->height;
    out->enabled = 0;  /* IntensityComp{} (encoder_internal.h:341-345): off, LUMSCALE 32, LUMSHIFT 0 */
    out->lumscale = 32;
    out->lumshift = 0;
    const size_t cap = (size_t)((W + 3) / 4) * ((H + 3) / 4) + 16;
    uint8_t* rs = (uint8_t*)malloc(cap);
    uint8_t* cs = (uint8_t*)malloc(cap);
    long double sx = 0, sy = 0, sxx = 0, sxy = 0;
    uint64_t n = 0;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const vc1cu_mv mv = mvs[(size_t)my * mbw + mx];
            const int dx = round_qpel_to_pixel(mv.xq), dy = round_qpel_to_pixel(mv.yq);
            const int x0 = mx * 16, y0 = my * 16;
            for (int y = 0; y < 16 && y0 + y < H; y += 4)
                for (int x = 0; x < 16 && x0 + x < W; x += 4) {
                    const int px = x0 + x, py = y0 + y;
                    const int rv = sample_clamped(ref->y, W, H, px + dx, py + dy);
                    const int cv = f->y[(size_t)py * W + px];
                    rs[n] = (uint8_t)rv;
                    cs[n] = (uint8_t)cv;
                    sx += rv; sy += cv; sxx += (long double)rv * rv; sxy += (long double)rv * cv;
                    ++n;
                }
        }
    if (n >= 16) {
        const long double denom = (long double)n * sxx - sx * sx;
        long double a = 1.0L, b = 0.0L;
        if (fabsl(denom) > 1e-9L) {
            a = ((long double)n * sxy - sx * sy) / denom;
            b = (sy - a * sx) / (long double)n;
        } else {
            b = (sy - sx) / (long double)n;
        }
        const int ls = iclamp((int)llroundl(a * 64.0L - 32.0L), 1, 63);
        const int sh = iclamp((int)llroundl(b), -32, 31);
        uint64_t best = UINT64_MAX;
        int best_ls = 32, best_sh = 0;
        for (int l = imax(1, ls - 3); l <= imin(63, ls + 3); ++l)
            for (int z = imax(-32, sh - 3); z <= imin(31, sh + 3); ++z) {
                uint64_t sad = 0;
                for (uint64_t i = 0; i < n; ++i) sad += (uint64_t)iabs(cs[i] - ic_map_y(rs[i], l + 32, z * 64));
                if (sad < best || (sad == best && iabs(l - 32) + iabs(z) < iabs(best_ls - 32) + iabs(best_sh))) {
                    best = sad;
                    best_ls = l;
                    best_sh = z;
                }
            }
        if (!(best_ls == 32 && best_sh == 0)) {
            out->enabled = 1;
            out->lumscale = best_ls;
            out->lumshift = best_sh < 0 ? best_sh + 64 : best_sh;
        }
    }
    free(rs);
    free(cs);
}

/* ---- scene-change score ------------------------------------------------------------ */

/* The zoom-coherence test of Vc1Encoder::scene_change_score, encoder_motion.cpp:636-671:
 * the interior vectors fitted to translation + isotropic scale in long double; coherent when
 * 60% of them lie within 2.5 px of the fitted field and 0.005 <= |scale| <= 0.08. */
int vo_zoom_coherent(const vc1cu_mv* mvs, int mbw, int mbh) {
    long double mx = 0.0L, my = 0.0L, mdx = 0.0L, mdy = 0.0L;
    size_t samples = 0;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[(size_t)by * mbw + bx];
            mx += bx * 16.0L + 8.0L;
            my += by * 16.0L + 8.0L;
            mdx += mv.xq / 4.0L;
            mdy += mv.yq / 4.0L;
            ++samples;
        }
    if (samples < 12) return 0;
    mx /= samples; my /= samples; mdx /= samples; mdy /= samples;
    long double num = 0.0L, den = 0.0L;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[(size_t)by * mbw + bx];
            const long double x = bx * 16.0L + 8.0L - mx, y = by * 16.0L + 8.0L - my;
            const long double dx = mv.xq / 4.0L - mdx, dy = mv.yq / 4.0L - mdy;
            num += x * dx + y * dy;
            den += x * x + y * y;
        }
    const long double z = den > 0.0L ? num / den : 0.0L;
    size_t inliers = 0;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[(size_t)by * mbw + bx];
            const long double x = bx * 16.0L + 8.0L - mx, y = by * 16.0L + 8.0L - my;
            const long double ex = mv.xq / 4.0L - (mdx + z * x);
            const long double ey = mv.yq / 4.0L - (mdy + z * y);
            if (ex * ex + ey * ey <= 6.25L) ++inliers;
        }
    const long double az = fabsl(z);
    return inliers * 5 >= samples * 3 && az >= 0.005L && az <= 0.08L;
}

/* The learned analysis pass of this library (no counterpart in the reference; on the device:
 * learned_candidates / learned_descent in libvc1_b200/csrc/vc1cu_core.cu and the launches of
 * vc1cu_lp_analyze). Pass A, every macroblock independently: the best of its four integer-pixel
 * candidates (clamped to the search bounds) by exact mb_sad, a small-diamond descent of at most
 * 2 * reach steps within reach of it, the fallback flag (the match's mean absolute error is above
 * six levels and above the picture's mean error at the hint), then the staged
 * refinement, whose rate predictor takes the neighbours' first candidates as their vectors, as an
 * unseeded pass refines its integer vector (encoder_motion.cpp:226-230). Pass B (fallback != 0),
 * the flagged macroblocks independently: the unseeded pass's integer search with the hint as its
 * global vector and the finished pass-A field as neighbours, then the same refinement with that
 * field's predictor; its results replace pass A's. Totals as analyze_p_picture_core's, with the
 * hint's full-resolution frame SAD standing in for the global search's. */
int vo_analyze_p_learned(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, int mode, const vc1cu_mv* cands,
                         int hint_dx, int hint_dy, int fallback, uint8_t* flags, vc1cu_panalysis* out) {
    if (f->w != p->width || f->h != p->height || ref->w != p->width || ref->h != p->height) return 1;
    if (mode == VC1CU_MV_MIXED || p->search_range == 0) return 2;
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    const int range = p->search_range, reach = 4;
    const bounds b = bounds_px(range);
    vc1cu_mv* mvs = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_mv* bmv = (vc1cu_mv*)calloc(mbs * 4, sizeof(vc1cu_mv));
    uint8_t* intra = (uint8_t*)calloc(mbs, 1);
    uint8_t* propagated = (uint8_t*)calloc(mbs, 1);
    uint64_t* screen = (uint64_t*)calloc(mbs, sizeof(uint64_t));
    double* dl = (double*)malloc(mbs * sizeof(double));
    double* dc = (double*)malloc(mbs * sizeof(double));
    uint8_t* dd = (uint8_t*)calloc(mbs, 1);
    lr_cell* cells = NULL;
    int ncells = 0;
    /* the learned pass's neighbourhood: every macroblock's first candidate as its 1-MV vector
       (no wavefront); the fallback pass's: the finished learned field (smvs, sbmv), in which no
       macroblock took a distant match */
    vc1cu_mv* cbmv = (vc1cu_mv*)calloc(mbs * 4, sizeof(vc1cu_mv));
    vc1cu_mv* smvs = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
    vc1cu_mv* sbmv = (vc1cu_mv*)calloc(mbs * 4, sizeof(vc1cu_mv));
    for (size_t i = 0; i < mbs; ++i) {
        dl[i] = -1.0;
        dc[i] = -1.0;
        const vc1cu_mv c0 = {cands[i * 4].xq * 4, cands[i * 4].yq * 4};
        for (int k = 0; k < 4; ++k) cbmv[i * 4 + k] = c0;
    }
    const uint64_t hint_sad = vo_frame_sad(f, ref, hint_dx, hint_dy, 1);
    const uint64_t wh = (uint64_t)p->width * (uint64_t)p->height;
    for (int pass = 0; pass < (fallback ? 2 : 1); ++pass) {
        if (pass == 1) {
            memcpy(smvs, mvs, mbs * sizeof(vc1cu_mv));
            memcpy(sbmv, bmv, mbs * 4 * sizeof(vc1cu_mv));
        }
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx) {
                const size_t pos = (size_t)my * mbw + mx;
                if (pass == 1 && !flags[pos]) continue;
                const int x0 = mx * 16, y0 = my * 16;
                const uint64_t pixels = active_mb_pixels(p, mx, my);
                const pinfo rate_pi = predictor_info_mixed_1mv(pass == 0 ? cbmv : sbmv, intra, mbw, mbh, mx, my);
                cand best = {UINT64_MAX, 0, 0};
                if (pass == 0) {
                    for (int k = 0; k < 4; ++k) {
                        const int cx = iclamp(cands[pos * 4 + k].xq, b.xmin, b.xmax);
                        const int cy = iclamp(cands[pos * 4 + k].yq, b.ymin, b.ymax);
                        const uint64_t c = vo_mb_sad(p, f, ref, mx, my, cx, cy, 1);
                        if (k == 0 || cand_less(c, cx, cy, best.cost, best.dx, best.dy)) {
                            best.cost = c;
                            best.dx = cx;
                            best.dy = cy;
                        }
                    }
                    const int sx = best.dx, sy = best.dy;
                    for (int step = 0; step < 2 * reach; ++step) {
                        cand nb = {UINT64_MAX, 0, 0};
                        int any = 0;
                        for (int l = 0; l < 4; ++l) {
                            const int dx = best.dx + (l == 0) - (l == 1), dy = best.dy + (l == 2) - (l == 3);
                            if (dx < b.xmin || dx > b.xmax || dy < b.ymin || dy > b.ymax || iabs(dx - sx) > reach ||
                                iabs(dy - sy) > reach)
                                continue;
                            const uint64_t c = vo_mb_sad(p, f, ref, mx, my, dx, dy, 1);
                            if (!any || cand_less(c, dx, dy, nb.cost, nb.dx, nb.dy)) {
                                nb.cost = c;
                                nb.dx = dx;
                                nb.dy = dy;
                                any = 1;
                            }
                        }
                        if (!any || !cand_less(nb.cost, nb.dx, nb.dy, best.cost, best.dx, best.dy)) break;
                        best = nb;
                    }
                    if (flags) {
                        /* fallback when the match's mean absolute error is above both six levels
                           and the picture's mean error at the hint:
                           cost * W * H > pixels * max(6 * W * H, hint_sad) */
                        int fb = 1;
                        if (pixels && best.cost < UINT64_MAX / 8) {
                            const uint64_t a = 6 * wh;
                            fb = (unsigned __int128)best.cost * wh > (unsigned __int128)pixels * (a > hint_sad ? a : hint_sad);
                        }
                        flags[pos] = (uint8_t)fb;
                    }
                    if (pixels) dl[pos] = (double)best.cost / (double)pixels;
                } else {
                    dl[pos] = -1.0;
                    dc[pos] = -1.0;
                    dd[pos] = 0;
                    best = unseeded_integer(p, f, ref, mx, my, smvs, propagated, hint_dx, hint_dy, &cells, &ncells,
                                            &dl[pos], &dc[pos], &dd[pos]);
                    propagated[pos] = 0; /* the learned field holds no distant matches */
                }
                uint64_t one_sad = 0;
                const vc1cu_mv s4 = {best.dx * 4, best.dy * 4};
                vc1cu_mv one = refine_staged(p, f, ref, x0, y0, 16, 16, s4, range, mode, &rate_pi, 1, &one_sad, best.cost);
                if (vo_hidden_padding(p, x0, y0, 16, 16, one.xq, one.yq, mode, 1)) {
                    one.xq = 0;
                    one.yq = 0;
                    one_sad = vo_block_sad_motion(p, f, ref, x0, y0, 16, 16, 0, 0, mode);
                }
                mvs[pos] = one;
                for (int k = 0; k < 4; ++k) bmv[pos * 4 + k] = one;
                screen[pos] = one_sad;
            }
    }
    free(cbmv);
    free(smvs);
    free(sbmv);
    uint64_t total_sad = 0, total_pixels = 0, moved = 0, frac = 0;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = (size_t)my * mbw + mx;
            total_sad += screen[pos];
            total_pixels += active_mb_pixels(p, mx, my);
            moved += mvs[pos].xq != 0 || mvs[pos].yq != 0;
            frac += (mvs[pos].xq % 8) != 0 || (mvs[pos].yq % 8) != 0;
        }
    const uint64_t gsad = hint_sad;
    const double local_mad = total_pixels ? (double)total_sad / (double)total_pixels : 0.0;
    const double global_mad = (double)gsad / (double)((uint64_t)p->width * p->height);
    out->mean_abs_residual = local_mad < global_mad ? local_mad : global_mad;
    out->rate_complexity = out->mean_abs_residual;
    out->motion_sad = total_sad;
    for (size_t i = 0; i < mbs; ++i) {
        if (out->mvs) out->mvs[i] = mvs[i];
        if (out->block_mvs) for (int k = 0; k < 4; ++k) out->block_mvs[i * 4 + k] = bmv[i * 4 + k];
        if (out->use_4mv) out->use_4mv[i] = 0;
        if (out->use_intra) out->use_intra[i] = 0;
        if (out->screen_sads) out->screen_sads[i] = screen[i];
        if (out->inter_intra_cost_ratio) out->inter_intra_cost_ratio[i] = -1.0;
        if (out->distant_local_mae) out->distant_local_mae[i] = dl[i];
        if (out->distant_candidate_mae) out->distant_candidate_mae[i] = dc[i];
        if (out->distant_match_decision) out->distant_match_decision[i] = dd[i];
    }
    out->moved_macroblocks = moved;
    out->fractional_chroma_macroblocks = frac;
    out->four_mv_macroblocks = 0;
    out->intra_macroblocks = 0;
    out->global_dx = hint_dx;
    out->global_dy = hint_dy;
    out->global_full_sad = gsad;
    free(mvs);
    free(bmv);
    free(intra);
    free(propagated);
    free(screen);
    free(dl);
    free(dc);
    free(dd);
    free(cells);
    return 0;
}

/* Vc1Encoder::scene_change_score, encoder_motion.cpp:599-676: the whole-frame translation
 * SAD per pixel, the same after fade compensation along the uniform global field, and when
 * that still looks like a cut, a quarter-pel core pass whose field must fit a camera zoom. */
double vo_scene_change_score(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, int fade_compensation,
                             double scene_threshold) {
    const int W = p->width, H = p->height, mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    int gdx, gdy;
    uint64_t gsad;
    vo_global_motion(p, f, ref, p->search_range, &gdx, &gdy, &gsad);
    const uint64_t pixels = (uint64_t)W * H;
    double best = pixels ? (double)gsad / (double)pixels : 0.0;
    if (fade_compensation) {
        vc1cu_mv* uniform = (vc1cu_mv*)malloc(mbs * sizeof(vc1cu_mv));
        for (size_t i = 0; i < mbs; ++i) { uniform[i].xq = gdx * 4; uniform[i].yq = gdy * 4; }
        vc1cu_intensity ic;
        vo_estimate_intensity_comp(p, f, ref, uniform, &ic);
        free(uniform);
        if (ic.enabled) {
            const size_t ny = (size_t)W * H, nc = (size_t)(W / 2) * (H / 2);
            uint8_t* buf = (uint8_t*)malloc(ny + 2 * nc);
            vo_intensity_compensate(ref, &ic, buf, buf + ny, buf + ny + nc);
            const vo_frame weighted = {W, H, buf, buf + ny, buf + ny + nc};
            int wdx, wdy;
            uint64_t wsad;
            vo_global_motion(p, f, &weighted, p->search_range, &wdx, &wdy, &wsad);
            const double wm = pixels ? (double)wsad / (double)pixels : 0.0;
            if (wm < best) best = wm;
            free(buf);
        }
    }
    if (best >= scene_threshold) {
        vc1cu_panalysis a;
        memset(&a, 0, sizeof a);
        vc1cu_mv* mvs = (vc1cu_mv*)calloc(mbs, sizeof(vc1cu_mv));
        a.mvs = mvs;
        vo_analyze_p_core(p, f, ref, VC1CU_MV_QPEL, 0, NULL, NULL, &a);
        const double lm = a.mean_abs_residual;
        if (vo_zoom_coherent(mvs, mbw, mbh) && lm < best * 0.72 && lm < scene_threshold * 0.86) best = lm;
        free(mvs);
    }
    return best;
}

/* ---- B-picture prediction ------------------------------------------------------------ */

/* The prediction of a B analysis as sampled_b_mode_rd builds it for every macroblock
 * (encoder_motion.cpp:1030-1053): Forward from the past reference and Backward from the future
 * one with motion_compensate_mb (encoder_motion_compensation.cpp:474-525, chroma rounded as
 * for a P vector), Direct and Interpolated with motion_compensate_bi_mb (:659-711: the rounded
 * average of both, the future chroma vector rounded away from the even value), and B-intra
 * macroblocks filled with the visible mean of each source 8x8 block. */
void vo_b_predict(const vc1cu_params* p, const vo_frame* f, const vo_frame* past, const vo_frame* future,
                  const uint8_t* modes, const vc1cu_mv* fmv, const vc1cu_mv* bmv, int mode, uint8_t* dy, uint8_t* du,
                  uint8_t* dv) {
    const int W = p->width, H = p->height, mbw = mbw_of(p), mbh = mbh_of(p);
    const int cw = W / 2, ch = H / 2;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = (size_t)my * mbw + mx;
            const int m = modes[pos];
            const int x0 = mx * 16, y0 = my * 16, cx0 = mx * 8, cy0 = my * 8;
            const int vw = imax(0, imin(16, W - x0)), vh = imax(0, imin(16, H - y0));
            const int cvw = imax(0, imin(8, cw - cx0)), cvh = imax(0, imin(8, ch - cy0));
            if (m == VC1CU_BMB_INTRA) {
                for (int k = 0; k < 6; ++k) {
                    const uint8_t* src = k < 4 ? f->y : (k == 4 ? f->u : f->v);
                    uint8_t* dst = k < 4 ? dy : (k == 4 ? du : dv);
                    const int sw = k < 4 ? W : cw, sh = k < 4 ? H : ch;
                    const int bx = k < 4 ? mx * 2 + (k & 1) : mx, by = k < 4 ? my * 2 + ((k >> 1) & 1) : my;
                    const int mean = visible_block_mean(src, sw, sh, bx * 8, by * 8);
                    for (int yy = 0; yy < 8 && by * 8 + yy < sh; ++yy)
                        for (int xx = 0; xx < 8 && bx * 8 + xx < sw; ++xx)
                            dst[(size_t)(by * 8 + yy) * sw + bx * 8 + xx] = (uint8_t)mean;
                }
                continue;
            }
            if (m == VC1CU_BMB_FORWARD || m == VC1CU_BMB_BACKWARD) {
                const vo_frame* r = m == VC1CU_BMB_FORWARD ? past : future;
                const vc1cu_mv mv = m == VC1CU_BMB_FORWARD ? fmv[pos] : bmv[pos];
                for (int y = 0; y < vh; ++y)
                    for (int x = 0; x < vw; ++x)
                        dy[(size_t)(y0 + y) * W + x0 + x] =
                            (uint8_t)luma_mc_sample_mode(r->y, W, H, x0 + x, y0 + y, mv.xq, mv.yq, mode, p->rnd);
                for (int y = 0; y < cvh; ++y)
                    for (int x = 0; x < cvw; ++x) {
                        const size_t off = (size_t)(cy0 + y) * cw + cx0 + x;
                        du[off] = (uint8_t)chroma_mc_sample(r->u, cw, ch, cx0 + x, cy0 + y, mv.xq, mv.yq, 0, p->rnd);
                        dv[off] = (uint8_t)chroma_mc_sample(r->v, cw, ch, cx0 + x, cy0 + y, mv.xq, mv.yq, 0, p->rnd);
                    }
                continue;
            }
            const vc1cu_mv a = fmv[pos], b = bmv[pos];
            for (int y = 0; y < vh; ++y)
                for (int x = 0; x < vw; ++x) {
                    const int pa = luma_mc_sample_mode(past->y, W, H, x0 + x, y0 + y, a.xq, a.yq, mode, p->rnd);
                    const int pb = luma_mc_sample_mode(future->y, W, H, x0 + x, y0 + y, b.xq, b.yq, mode, p->rnd);
                    dy[(size_t)(y0 + y) * W + x0 + x] = (uint8_t)((pa + pb + 1) >> 1);
                }
            for (int y = 0; y < cvh; ++y)
                for (int x = 0; x < cvw; ++x) {
                    const size_t off = (size_t)(cy0 + y) * cw + cx0 + x;
                    const int au = chroma_mc_sample(past->u, cw, ch, cx0 + x, cy0 + y, a.xq, a.yq, 0, p->rnd);
                    const int bu = chroma_mc_sample(future->u, cw, ch, cx0 + x, cy0 + y, b.xq, b.yq, 1, p->rnd);
                    const int av = chroma_mc_sample(past->v, cw, ch, cx0 + x, cy0 + y, a.xq, a.yq, 0, p->rnd);
                    const int bv = chroma_mc_sample(future->v, cw, ch, cx0 + x, cy0 + y, b.xq, b.yq, 1, p->rnd);
                    du[off] = (uint8_t)((au + bu + 1) >> 1);
                    dv[off] = (uint8_t)((av + bv + 1) >> 1);
                }
        }
}

/* ---- inverse transform and reconstruction ------------------------------------------- */

/* Vc1Encoder::dequant_level, encoder_transform.cpp:1058-1065, at mquant = PQINDEX without
 * DQUANT (picture_double_quant :1052-1056: 2*PQ + HALFQP) */
static int dequant_level(const vc1cu_params* p, int level) {
    if (!level) return 0;
    long v = (long)level * (2 * p->pqindex + (p->halfqp ? 1 : 0));
    if (p->nonuniform) v += level > 0 ? p->pqindex : -p->pqindex;
    return (int)v;
}

/* The VC-1 8-point inverse butterfly of inverse_transform_8x8 (encoder_transform.cpp:566-609):
 * s[k*st] are the 8 inputs, bias and shift the stage's rounding; out[k*ot] the outputs; tail
 * adds the second stage's +1 to the lower half. */
static void inv8(const int* s, int st, int* o, int ot, int bias, int shift, int tail) {
    int t1 = 12 * (s[0] + s[4 * st]) + bias, t2 = 12 * (s[0] - s[4 * st]) + bias;
    int t3 = 16 * s[2 * st] + 6 * s[6 * st], t4 = 6 * s[2 * st] - 16 * s[6 * st];
    const int t5 = t1 + t3, t6 = t2 + t4, t7 = t2 - t4, t8 = t1 - t3;
    t1 = 16 * s[st] + 15 * s[3 * st] + 9 * s[5 * st] + 4 * s[7 * st];
    t2 = 15 * s[st] - 4 * s[3 * st] - 16 * s[5 * st] - 9 * s[7 * st];
    t3 = 9 * s[st] - 16 * s[3 * st] + 4 * s[5 * st] + 15 * s[7 * st];
    t4 = 4 * s[st] - 9 * s[3 * st] + 15 * s[5 * st] - 16 * s[7 * st];
    o[0] = arshift(t5 + t1, shift); o[ot] = arshift(t6 + t2, shift);
    o[2 * ot] = arshift(t7 + t3, shift); o[3 * ot] = arshift(t8 + t4, shift);
    o[4 * ot] = arshift(t8 - t4 + tail, shift); o[5 * ot] = arshift(t7 - t3 + tail, shift);
    o[6 * ot] = arshift(t6 - t2 + tail, shift); o[7 * ot] = arshift(t5 - t1 + tail, shift);
}
/* The 4-point one (inverse_partition's 8x4 / 4x8 / 4x4 stages, :1213-1272) */
static void inv4(const int* s, int st, int* o, int ot, int bias, int shift) {
    const int t1 = 17 * (s[0] + s[2 * st]) + bias, t2 = 17 * (s[0] - s[2 * st]) + bias;
    const int t3 = 22 * s[st] + 10 * s[3 * st], t4 = 22 * s[3 * st] - 10 * s[st];
    o[0] = arshift(t1 + t3, shift); o[ot] = arshift(t2 - t4, shift);
    o[2 * ot] = arshift(t2 + t4, shift); o[3 * ot] = arshift(t1 - t3, shift);
}

/* Vc1Encoder::inverse_partition, encoder_transform.cpp:1173-1274: dequantisation, the DC-only
 * shortcut of a partition whose only coefficient is its DC, then the type's inverse transform;
 * q and a are partition-local (row-major, stride 8). */
static void inverse_partition(const vc1cu_params* p, int t, const int q[64], int a[64]) {
    int ox, oy, bw, bh;
    part_geometry(t, 0, &ox, &oy, &bw, &bh);
    int nonzero = 0;
    memset(a, 0, 64 * sizeof(int));
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) {
            if (q[y * 8 + x]) ++nonzero;
            a[y * 8 + x] = dequant_level(p, q[y * 8 + x]);
        }
    if (nonzero == 1 && q[0] != 0) {
        int dc = a[0];
        if (t == 1) { dc = arshift(3 * dc + 1, 1); dc = arshift(3 * dc + 16, 5); }
        else if (t == 2) { dc = arshift(3 * dc + 1, 1); dc = arshift(17 * dc + 64, 7); }
        else if (t == 3) { dc = arshift(17 * dc + 4, 3); dc = arshift(12 * dc + 64, 7); }
        else { dc = arshift(17 * dc + 4, 3); dc = arshift(17 * dc + 64, 7); }
        memset(a, 0, 64 * sizeof(int));
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) a[y * 8 + x] = dc;
        return;
    }
    int tmp[64];
    memset(tmp, 0, sizeof tmp);
    if (t == 1) {
        /* columns first into rows of tmp, then columns of tmp (inverse_transform_8x8) */
        for (int col = 0; col < 8; ++col) inv8(a + col, 8, tmp + col * 8, 1, 4, 3, 0);
        for (int col = 0; col < 8; ++col) inv8(tmp + col, 8, a + col, 8, 64, 7, 1);
    } else if (t == 2) {
        for (int y = 0; y < 4; ++y) inv8(a + y * 8, 1, tmp + y * 8, 1, 4, 3, 0);
        for (int x = 0; x < 8; ++x) inv4(tmp + x, 8, a + x, 8, 64, 7);
    } else if (t == 3) {
        for (int y = 0; y < 8; ++y) inv4(a + y * 8, 1, tmp + y * 8, 1, 4, 3);
        for (int x = 0; x < 4; ++x) inv8(tmp + x, 8, a + x, 8, 64, 7, 1);
    } else {
        for (int y = 0; y < 4; ++y) inv4(a + y * 8, 1, tmp + y * 8, 1, 4, 3);
        for (int x = 0; x < 4; ++x) inv4(tmp + x, 8, a + x, 8, 64, 7);
    }
}

/* The reconstruction of evaluate_transform_parent, encoder_transform.cpp:1569-1585: every
 * partition of the chosen type inverse-transformed and added to the prediction, clamped to 8
 * bits. levels: vo_forward_quant's layout for type_mask; block_types: the TransformType (1..4)
 * of each (MB, parent). Pixels of MBs outside the raster are untouched. */
void vo_reconstruct(const vc1cu_params* p, const vo_frame* pred, const int16_t* levels, int type_mask,
                    const uint8_t* block_types, uint8_t* y, uint8_t* u, uint8_t* v) {
    const int mbw = mbw_of(p), mbh = mbh_of(p);
    const size_t mbs = (size_t)mbw * mbh;
    int tindex[5] = {-1, -1, -1, -1, -1}, nt = 0;
    for (int t = 1; t <= 4; ++t)
        if (type_mask & (1 << (t - 1))) tindex[t] = nt++;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx)
            for (int k = 0; k < 6; ++k) {
                const size_t mb = (size_t)my * mbw + mx;
                const int t = block_types[mb * 6 + k];
                const int16_t* q64 = levels + (((size_t)tindex[t] * mbs + mb) * 6 + k) * 64;
                const uint8_t* pp = k < 4 ? pred->y : (k == 4 ? pred->u : pred->v);
                uint8_t* dp = k < 4 ? y : (k == 4 ? u : v);
                const int w = k < 4 ? p->width : p->width / 2, h = k < 4 ? p->height : p->height / 2;
                const int bx = k < 4 ? mx * 2 + (k & 1) : mx, by = k < 4 ? my * 2 + ((k >> 1) & 1) : my;
                int residual[64];
                memset(residual, 0, sizeof residual);
                const int np = t == 1 ? 1 : (t == 4 ? 4 : 2);
                for (int part = 0; part < np; ++part) {
                    int ox, oy, bw, bh;
                    part_geometry(t, part, &ox, &oy, &bw, &bh);
                    int q[64], r[64];
                    memset(q, 0, sizeof q);
                    for (int yy = 0; yy < bh; ++yy)
                        for (int xx = 0; xx < bw; ++xx) q[yy * 8 + xx] = q64[(oy + yy) * 8 + ox + xx];
                    inverse_partition(p, t, q, r);
                    for (int yy = 0; yy < bh; ++yy)
                        for (int xx = 0; xx < bw; ++xx) residual[(oy + yy) * 8 + ox + xx] = r[yy * 8 + xx];
                }
                for (int yy = 0; yy < 8 && by * 8 + yy < h; ++yy)
                    for (int xx = 0; xx < 8 && bx * 8 + xx < w; ++xx) {
                        const size_t off = (size_t)(by * 8 + yy) * w + bx * 8 + xx;
                        dp[off] = (uint8_t)iclamp(pp[off] + residual[yy * 8 + xx], 0, 255);
                    }
            }
}

/* ---- in-loop deblocking --------------------------------------------------------------- */

/* Vc1Encoder::loop_filter_line, encoder_filter.cpp:366-395: one 8-sample line across an edge
 * between (x - cross) and (x, y); returns whether the line was eligible (its a0 test). */
static int lf_line(uint8_t* p, int w, int h, int x, int y, int cdx, int cdy, int pq) {
    for (int k = -4; k <= 3; ++k) {
        const int xx = x + k * cdx, yy = y + k * cdy;
        if (xx < 0 || yy < 0 || xx >= w || yy >= h) return 0;
    }
#define LFS(k) ((int)p[(size_t)(y + (k) * cdy) * w + x + (k) * cdx])
    int a0 = arshift(2 * (LFS(-2) - LFS(1)) - 5 * (LFS(-1) - LFS(0)) + 4, 3);
    const int a0_neg = a0 < 0;
    a0 = iabs(a0);
    if (a0 >= pq) return 0;
    const int a1 = iabs(arshift(2 * (LFS(-4) - LFS(-1)) - 5 * (LFS(-3) - LFS(-2)) + 4, 3));
    const int a2 = iabs(arshift(2 * (LFS(0) - LFS(3)) - 5 * (LFS(1) - LFS(2)) + 4, 3));
    if (!(a1 < a0 || a2 < a0)) return 0;
    const int edge = LFS(-1) - LFS(0);
#undef LFS
    const int limit = iabs(edge) >> 1;
    if (!limit) return 0;
    int delta = (5 * (a0 - imin(a1, a2))) >> 3;
    if (a0_neg != (edge < 0)) {
        delta = imin(delta, limit);
        if (edge < 0) delta = -delta;
        const size_t po = (size_t)(y - cdy) * w + x - cdx, qo = (size_t)y * w + x;
        p[po] = (uint8_t)iclamp((int)p[po] - delta, 0, 255);
        p[qo] = (uint8_t)iclamp((int)p[qo] + delta, 0, 255);
    }
    return 1;
}

/* Vc1Encoder::loop_filter_edge, encoder_filter.cpp:397-416 (scalar): groups of 4 lines, the
 * third line decides for its group */
static void lf_edge(uint8_t* p, int w, int h, int x, int y, int adx, int ady, int cdx, int cdy, int len, int pq) {
    for (int i = 0; i < len; i += 4) {
        const int bx = x + i * adx, by = y + i * ady;
        if (!lf_line(p, w, h, bx + 2 * adx, by + 2 * ady, cdx, cdy, pq)) continue;
        lf_line(p, w, h, bx, by, cdx, cdy, pq);
        lf_line(p, w, h, bx + adx, by + ady, cdx, cdy, pq);
        lf_line(p, w, h, bx + 3 * adx, by + 3 * ady, cdx, cdy, pq);
    }
}
static void lf_hborder(uint8_t* p, int w, int h, int x, int y, int len, int pq) { lf_edge(p, w, h, x, y, 1, 0, 0, 1, len, pq); }
static void lf_vborder(uint8_t* p, int w, int h, int x, int y, int len, int pq) { lf_edge(p, w, h, x, y, 0, 1, 1, 0, len, pq); }

/* overlap_arshift3, encoder_filter.cpp:162-164 */
static int ovl_arshift3(int v) { return v >= 0 ? (v >> 3) : -((-v + 7) >> 3); }

/* the four samples across one edge along one line, at line parity i
 * (overlap_vertical_edge :166-180 / overlap_horizontal_edge :182-199) */
static void ovl_line(int32_t* c, ptrdiff_t step, int i) {
    const int a = c[-2 * step], b = c[-step], cc = c[0], d = c[step];
    const int d1 = a - d, d2 = a - d + b - cc;
    const int r1 = (i & 1) ? 3 : 4, r2 = 7 - r1;
    c[-2 * step] = ovl_arshift3(8 * a - d1 + r1);
    c[-step] = ovl_arshift3(8 * b - d2 + r2);
    c[0] = ovl_arshift3(8 * cc + d2 + r1);
    c[step] = ovl_arshift3(8 * d + d1 + r2);
}

/* overlap_edge_enabled, encoder_filter.cpp:201-215 */
static int ovl_enabled(int luma, int bx0, int by0, int bx1, int by1, const uint8_t* flags, int mbw, int mbh, int all) {
    if (all) return 1;
    const int mx0 = luma ? bx0 >> 1 : bx0, my0 = luma ? by0 >> 1 : by0;
    const int mx1 = luma ? bx1 >> 1 : bx1, my1 = luma ? by1 >> 1 : by1;
    if (mx0 < 0 || my0 < 0 || mx0 >= mbw || my0 >= mbh || mx1 < 0 || my1 < 0 || mx1 >= mbw || my1 >= mbh) return 0;
    const int a = my0 * mbw + mx0, b = my1 * mbw + mx1;
    if (a == b) return flags[a] != 0;
    return flags[a] != 0 && flags[b] != 0;
}

/* apply_overlap_plane_signed, encoder_filter.cpp:217-243 */
static void ovl_plane(int32_t* p, int w, int h, int luma, const uint8_t* flags, int mbw, int mbh, int all) {
    if (w < 8 || h < 8) return;
    const int bw = w / 8, bh = h / 8;
    for (int bx = 1; bx < bw; ++bx)
        for (int by = 0; by < bh; ++by)
            if (ovl_enabled(luma, bx - 1, by, bx, by, flags, mbw, mbh, all))
                for (int i = 0; i < 8; ++i) ovl_line(p + (size_t)(by * 8 + i) * w + bx * 8, 1, i);
    for (int by = 1; by < bh; ++by)
        for (int bx = 0; bx < bw; ++bx)
            if (ovl_enabled(luma, bx, by - 1, bx, by, flags, mbw, mbh, all))
                for (int i = 0; i < 8; ++i) ovl_line(p + (size_t)(by * 8) * w + bx * 8 + i, w, i);
}

/* Vc1Encoder::apply_i_overlap / apply_p_overlap, encoder_filter.cpp:344-365 (the plan's
 * None mode and the picture-level condition are the caller's) */
void vo_overlap_smooth(int mbw, int mbh, int32_t* y, int32_t* u, int32_t* v, const uint8_t* flags, int all) {
    ovl_plane(y, mbw * 16, mbh * 16, 1, flags, mbw, mbh, all);
    ovl_plane(u, mbw * 8, mbh * 8, 0, flags, mbw, mbh, all);
    ovl_plane(v, mbw * 8, mbh * 8, 0, flags, mbw, mbh, all);
}

/* the store of reconstruct_i_picture_padded (clamp(s + bias) of every sample) and the intra
 * write-back after apply_p_overlap (encoder_encode.cpp:1425-1449, bias 128, intra MBs) */
void vo_store_signed(int mbw, int mbh, const int32_t* sy, const int32_t* su, const int32_t* sv, int bias,
                     const uint8_t* mask, int w, int h, uint8_t* y, uint8_t* u, uint8_t* v) {
    for (int k = 0; k < 3; ++k) {
        const int32_t* s = k == 0 ? sy : (k == 1 ? su : sv);
        uint8_t* d = k == 0 ? y : (k == 1 ? u : v);
        const int sw = k == 0 ? mbw * 16 : mbw * 8, sh = k == 0 ? mbh * 16 : mbh * 8;
        const int dw = k == 0 ? w : w / 2, dh = k == 0 ? h : h / 2, shift = k == 0 ? 4 : 3;
        for (int yy = 0; yy < dh && yy < sh; ++yy)
            for (int xx = 0; xx < dw && xx < sw; ++xx) {
                if (mask && !mask[(yy >> shift) * mbw + (xx >> shift)]) continue;
                const int t = s[(size_t)yy * sw + xx] + bias;
                d[(size_t)yy * dw + xx] = (uint8_t)(t < 0 ? 0 : (t > 255 ? 255 : t));
            }
    }
}

/* Vc1Encoder::apply_i_like_loop_filter_plane, encoder_filter.cpp:426-434 */
static void lf_i_plane(uint8_t* p, int w, int h, int pq) {
    for (int y = 8; y < h; y += 8)
        for (int x = 0; x < w; x += 16) lf_hborder(p, w, h, x, y, imin(16, w - x), pq);
    for (int x = 8; x < w; x += 8)
        for (int y = 0; y < h; y += 16) lf_vborder(p, w, h, x, y, imin(16, h - y), pq);
}

/* Vc1Encoder::apply_i_like_loop_filter, encoder_filter.cpp:436-441 (in place) */
void vo_loop_filter_i(const vc1cu_params* p, uint8_t* y, uint8_t* u, uint8_t* v) {
    lf_i_plane(y, p->width, p->height, p->pqindex);
    lf_i_plane(u, p->width / 2, p->height / 2, p->pqindex);
    lf_i_plane(v, p->width / 2, p->height / 2, p->pqindex);
}

typedef struct lf_meta {
    const vc1cu_mv* bmv;   /* 4 per MB */
    const uint8_t* cbp;    /* 6 per MB: loop_filter_pattern of each block */
    const uint8_t* tt;     /* 6 per MB: loop_filter_tt of each block */
    const uint8_t* intra;  /* per MB: bit k = block k intra */
    int mbw, mbh, luma, plane_k;
} lf_meta;

static void lf_at(const lf_meta* m, int bx, int by, int* mx, int* my, int* k) {
    if (m->luma) { *mx = bx >> 1; *my = by >> 1; *k = ((by & 1) << 1) | (bx & 1); }
    else { *mx = bx; *my = by; *k = m->plane_k; }
}
/* mv_at of apply_p_loop_filter_plane (encoder_filter.cpp:628-637): the block's vector, or for
 * chroma the pre-FASTUVMC representative of the 4-MV median */
static vc1cu_mv lf_mv(const lf_meta* m, int bx, int by) {
    int mx, my, k;
    lf_at(m, bx, by, &mx, &my, &k);
    const vc1cu_mv* b = m->bmv + ((size_t)my * m->mbw + mx) * 4;
    if (m->luma) return b[k];
    const int cx = median4(b[0].xq, b[1].xq, b[2].xq, b[3].xq), cy = median4(b[0].yq, b[1].yq, b[2].yq, b[3].yq);
    vc1cu_mv r;
    r.xq = arshift(cx + ((cx & 3) == 3), 1);
    r.yq = arshift(cy + ((cy & 3) == 3), 1);
    return r;
}
static int lf_cbp(const lf_meta* m, int bx, int by) { int mx, my, k; lf_at(m, bx, by, &mx, &my, &k); return m->cbp[((size_t)my * m->mbw + mx) * 6 + k]; }
static int lf_tt(const lf_meta* m, int bx, int by) { int mx, my, k; lf_at(m, bx, by, &mx, &my, &k); return m->tt[((size_t)my * m->mbw + mx) * 6 + k]; }
static int lf_intra(const lf_meta* m, int bx, int by) {
    int mx, my, k;
    lf_at(m, bx, by, &mx, &my, &k);
    return (m->intra[(size_t)my * m->mbw + mx] >> k) & 1;
}
static int lf_same_mv(vc1cu_mv a, vc1cu_mv b) { return a.xq == b.xq && a.yq == b.yq; }

/* process_v_parent, encoder_filter.cpp:654-676: the block's bottom border and its inner
 * horizontal 4-line edge */
static void lf_v_parent(const lf_meta* m, uint8_t* p, int w, int h, int bx, int by, int pq) {
    const int x0 = bx * 8, y0 = by * 8;
    if (x0 >= w || y0 >= h) return;
    const int grid_h = m->luma ? m->mbh * 2 : m->mbh;
    if (by + 1 < grid_h && y0 + 8 < h) {
        const int top = lf_cbp(m, bx, by), bottom = lf_cbp(m, bx, by + 1);
        if (lf_intra(m, bx, by) || lf_intra(m, bx, by + 1) || !lf_same_mv(lf_mv(m, bx, by), lf_mv(m, bx, by + 1))) {
            lf_hborder(p, w, h, x0, y0 + 8, imin(8, w - x0), pq);
        } else {
            const int mask = (top | (bottom >> 2)) & 3;
            if ((mask & 2) && x0 < w) lf_hborder(p, w, h, x0, y0 + 8, imin(4, w - x0), pq);
            if ((mask & 1) && x0 + 4 < w) lf_hborder(p, w, h, x0 + 4, y0 + 8, imin(4, w - (x0 + 4)), pq);
        }
    }
    const int kind = lf_tt(m, bx, by), pat = lf_cbp(m, bx, by);
    if ((kind == 7 || kind == 3) && y0 + 4 < h) {
        if ((pat & 10) && x0 < w) lf_hborder(p, w, h, x0, y0 + 4, imin(4, w - x0), pq);
        if ((pat & 5) && x0 + 4 < w) lf_hborder(p, w, h, x0 + 4, y0 + 4, imin(4, w - (x0 + 4)), pq);
    }
}
/* process_h_parent, encoder_filter.cpp:677-699: the block's right border and inner vertical edge */
static void lf_h_parent(const lf_meta* m, uint8_t* p, int w, int h, int bx, int by, int pq) {
    const int x0 = bx * 8, y0 = by * 8;
    if (x0 >= w || y0 >= h) return;
    const int grid_w = m->luma ? m->mbw * 2 : m->mbw;
    if (bx + 1 < grid_w && x0 + 8 < w) {
        const int left = lf_cbp(m, bx, by), right = lf_cbp(m, bx + 1, by);
        if (lf_intra(m, bx, by) || lf_intra(m, bx + 1, by) || !lf_same_mv(lf_mv(m, bx, by), lf_mv(m, bx + 1, by))) {
            lf_vborder(p, w, h, x0 + 8, y0, imin(8, h - y0), pq);
        } else {
            const int mask = (left | (right >> 1)) & 5;
            if ((mask & 4) && y0 < h) lf_vborder(p, w, h, x0 + 8, y0, imin(4, h - y0), pq);
            if ((mask & 1) && y0 + 4 < h) lf_vborder(p, w, h, x0 + 8, y0 + 4, imin(4, h - (y0 + 4)), pq);
        }
    }
    const int kind = lf_tt(m, bx, by), pat = lf_cbp(m, bx, by);
    if ((kind == 7 || kind == 6) && x0 + 4 < w) {
        if ((pat & 12) && y0 < h) lf_vborder(p, w, h, x0 + 4, y0, imin(4, h - y0), pq);
        if ((pat & 3) && y0 + 4 < h) lf_vborder(p, w, h, x0 + 4, y0 + 4, imin(4, h - (y0 + 4)), pq);
    }
}
static void lf_mb(const lf_meta* m, uint8_t* p, int w, int h, int mx, int my, int pq, int vertical) {
    if (m->luma) {
        for (int k = 0; k < 4; ++k) {
            const int bx = mx * 2 + (k & 1), by = my * 2 + (k >> 1);
            if (vertical) lf_v_parent(m, p, w, h, bx, by, pq); else lf_h_parent(m, p, w, h, bx, by, pq);
        }
    } else if (vertical) {
        lf_v_parent(m, p, w, h, mx, my, pq);
    } else {
        lf_h_parent(m, p, w, h, mx, my, pq);
    }
}

/* Vc1Encoder::apply_p_loop_filter (Advanced Profile), encoder_filter.cpp:610-738, in place: per
 * macroblock row, the horizontal edges of MB x before the vertical edges of MB x-1 */
void vo_loop_filter_p(const vc1cu_params* p, uint8_t* y, uint8_t* u, uint8_t* v, const vc1cu_mv* block_mvs,
                      const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra) {
    lf_meta m = {block_mvs, cbp, tt, intra, mbw_of(p), mbh_of(p), 1, 0};
    for (int plane = 0; plane < 3; ++plane) {
        uint8_t* pl = plane == 0 ? y : (plane == 1 ? u : v);
        const int w = plane ? p->width / 2 : p->width, h = plane ? p->height / 2 : p->height;
        m.luma = plane == 0;
        m.plane_k = plane == 0 ? 0 : 3 + plane;
        for (int my = 0; my < m.mbh; ++my) {
            for (int mx = 0; mx < m.mbw; ++mx) {
                lf_mb(&m, pl, w, h, mx, my, p->pqindex, 1);
                if (mx > 0) lf_mb(&m, pl, w, h, mx - 1, my, p->pqindex, 0);
            }
            if (m.mbw > 0) lf_mb(&m, pl, w, h, m.mbw - 1, my, p->pqindex, 0);
        }
    }
}

/* ---- transform type of the throughput preset --------------------------------------- */

/* transform_metrics::scalar, transform_residual_metrics.h:29-61: residual SAD, the 4-row and
 * 4-column inner-edge activity and the residual gradient of one MB's luma */
static void tx_metrics(const uint8_t* src, const uint8_t* pred, int stride, int height, int mx, int my, uint64_t m[4]) {
    m[0] = m[1] = m[2] = m[3] = 0;
    for (int py = 0; py < 16 && my * 16 + py < height; ++py)
        for (int px = 0; px < 16 && mx * 16 + px < stride; ++px) {
            const int x = mx * 16 + px, y = my * 16 + py;
            const size_t o = (size_t)y * stride + x;
            const int r = (int)src[o] - (int)pred[o];
            m[0] += (uint64_t)iabs(r);
            if ((py & 7) == 4 && py > 0) m[1] += (uint64_t)iabs(r - ((int)src[o - stride] - (int)pred[o - stride]));
            if ((px & 7) == 4 && px > 0) m[2] += (uint64_t)iabs(r - ((int)src[o - 1] - (int)pred[o - 1]));
            if (px > 0) m[3] += (uint64_t)iabs(r - ((int)src[o - 1] - (int)pred[o - 1]));
            if (py > 0) m[3] += (uint64_t)iabs(r - ((int)src[o - stride] - (int)pred[o - stride]));
        }
}

/* The TransformType choose_transform_mb returns with the throughput preset (fast transform RDO,
 * variable transforms, trellis 0, no DQUANT; encoder_transform.cpp:1605-1712): the candidate
 * list of the residual metrics (split shapes at a cropped raster edge), then the preset's pick. */
void vo_fast_transform_types(const vc1cu_params* p, const vo_frame* src, const vo_frame* pred, uint8_t* types) {
    const int mbw = mbw_of(p), mbh = mbh_of(p), mquant = p->pqindex;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            uint64_t m[4];
            tx_metrics(src->y, pred->y, p->width, p->height, mx, my, m);
            const uint64_t sad = m[0], hedge = m[1], vedge = m[2], grad = m[3];
            int list[4] = {1, 1, 1, 1}, count = 0;
            const int split_x = mx == mbw - 1 && (p->width & 15) != 0;
            const int split_y = my == mbh - 1 && (p->height & 15) != 0;
            if (split_x && split_y) {
                list[count++] = 4;
            } else if (split_x) {
                list[count++] = 3;
                if (sad > (uint64_t)(64 * mquant) && grad > sad * 2) list[count++] = 4;
            } else if (split_y) {
                list[count++] = 2;
                if (sad > (uint64_t)(64 * mquant) && grad > sad * 2) list[count++] = 4;
            } else {
                list[count++] = 1;
                if (sad > (uint64_t)(64 * mquant)) {
                    if (hedge * 5 > vedge * 6) list[count++] = 2;
                    else if (vedge * 5 > hedge * 6) list[count++] = 3;
                    else { list[count++] = 2; list[count++] = 3; }
                    if (count < 4 && grad > sad * 2) list[count++] = 4;
                }
            }
            int chosen = list[0];
            if (count > 1) {
                int index = count - 1;
                if (list[index] == 4 && grad * 2 <= sad * 5) --index;
                chosen = list[index];
                if (chosen == 3 && index > 0 && list[index - 1] == 2 && hedge >= vedge) chosen = 2;
            }
            types[(size_t)my * mbw + mx] = (uint8_t)chosen;
        }
}
