// vc1cu_common.cuh - device-side laws shared by the analysis kernels (sm_100a).
//
// Every function here restates one piece of libvc1 v0.2.69 with the same integer and
// IEEE-double results; the reference file:line is cited beside each. Costs are uint64 and
// an illegal candidate costs UINT64_MAX/4 exactly like the CPU law.
#pragma once

#include <cstdint>

#include "../../include/vc1cu.h"

namespace vc1cu {

constexpr uint64_t kBad = UINT64_MAX / 4;

// Geometry and knobs of one analysis configuration, derived on the host once per call.
struct DevParams {
    int W, H;            // internal raster (EncoderConfig::width/height)
    int vw, vh;          // visible raster
    int mbw, mbh;
    int cvw, cvh;        // visible chroma raster ((v+1)/2)
    int right_pad, bottom_pad, cright_pad, cbottom_pad;  // hidden-padding flags
    int pq, halfqp, nonuniform;
    int range;           // configured motion_search_range
    int local_range;     // min(range, local range)
    int me_algorithm, me_quality;
    int subpel, fast_subpel, subpel_range;
    int long_range_mode, rnd, disable_p_intra, disable_b_intra;
    int mvrange;         // motion_mvrange()
    double lambda;       // max(1, 0.35*PQ), the Mixed-MV / intra lambda
    uint64_t lam_m;      // lambda = lam_m * 2^-lam_s exactly
    int lam_s;
    int mant_bits;       // significand width of the host's long double (64: x87)
    double distant_match_max_mae;
    double inter_intra_threshold;
    int wait_log2;       // a wavefront wait gives up after 2^wait_log2 polls (default 24)
    uint32_t withhold;   // work item whose done flag is not published (test hook; 0xFFFFFFFF: none)
};

__host__ __device__ inline int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ inline int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ inline int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__host__ __device__ inline int iabs(int v) { return v < 0 ? -v : v; }

// Vc1Encoder::floor_div4, encoder_motion_compensation.cpp:355-358
__host__ __device__ inline int floor_div4(int v) { return v >= 0 ? v / 4 : -((-v + 3) / 4); }
// Vc1Encoder::arshift, encoder_entropy.cpp:377-381 (floor division by 2^n == arithmetic shift)
__host__ __device__ inline int arshift(int v, int n) { return v >> n; }
// Vc1Encoder::mspel_filter4, encoder_motion_compensation.cpp:360-365
__device__ __forceinline__ int mspel(int a, int b, int c, int d, int mode) {
    if (mode == 1) return -4 * a + 53 * b + 18 * c - 3 * d;
    if (mode == 2) return -a + 9 * b + 9 * c - d;
    return -3 * a + 18 * b + 53 * c - 4 * d;  // mode 3
}
__host__ __device__ inline bool mode_halfpel(int m) { return m == VC1CU_MV_HPEL || m == VC1CU_MV_HPEL_BILINEAR; }
__host__ __device__ inline bool mode_bilinear(int m) { return m == VC1CU_MV_HPEL_BILINEAR; }

// ---- cropped-reference legality (encoder_motion.cpp:2143-2195) -----------------------

// Vc1Encoder::motion_uses_hidden_luma, encoder_motion.cpp:2143-2165
__host__ __device__ inline bool hidden_luma(const DevParams& p, int x0, int y0, int bw, int bh, int xq, int yq, int mode) {
    if (!p.right_pad && !p.bottom_pad) return false;
    const int aw = imax(0, imin(bw, p.vw - x0)), ah = imax(0, imin(bh, p.vh - y0));
    if (!aw || !ah) return false;
    const int ix = floor_div4(xq), iy = floor_div4(yq);
    const int fx = xq - ix * 4, fy = yq - iy * 4;
    const int right = fx ? (mode_bilinear(mode) ? 1 : 2) : 0;
    const int bottom = fy ? (mode_bilinear(mode) ? 1 : 2) : 0;
    return (p.right_pad && x0 + aw - 1 + ix + right >= p.vw) || (p.bottom_pad && y0 + ah - 1 + iy + bottom >= p.vh);
}

// Vc1Encoder::motion_uses_hidden_chroma, encoder_motion.cpp:2167-2189. future: the B
// future-reference rounding of the chroma vector (away from zero instead of towards it).
__host__ __device__ inline bool hidden_chroma_f(const DevParams& p, int x0, int y0, int bw, int bh, int xq, int yq,
                                                bool future) {
    if (!p.cright_pad && !p.cbottom_pad) return false;
    const int cx = x0 / 2, cy = y0 / 2;
    const int aw = imax(0, imin(bw / 2, p.cvw - cx)), ah = imax(0, imin(bh / 2, p.cvh - cy));
    if (!aw || !ah) return false;
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
    const bool fx = (uvx - ix * 4) != 0, fy = (uvy - iy * 4) != 0;
    return (p.cright_pad && cx + aw - 1 + ix + (fx ? 1 : 0) >= p.cvw) ||
           (p.cbottom_pad && cy + ah - 1 + iy + (fy ? 1 : 0) >= p.cvh);
}
// P pictures: future = false
__host__ __device__ inline bool hidden_chroma(const DevParams& p, int x0, int y0, int bw, int bh, int xq, int yq) {
    return hidden_chroma_f(p, x0, y0, bw, bh, xq, yq, false);
}

// Vc1Encoder::motion_uses_hidden_padding, encoder_motion.cpp:2191-2195
__host__ __device__ inline bool hidden_padding(const DevParams& p, int x0, int y0, int bw, int bh, int xq, int yq, int mode,
                                               bool chroma) {
    return hidden_luma(p, x0, y0, bw, bh, xq, yq, mode) || (chroma && hidden_chroma(p, x0, y0, bw, bh, xq, yq));
}
__host__ __device__ inline bool chroma_gate(int x0, int y0, int bw, int bh) {
    return bw == 16 && bh == 16 && !(x0 & 15) && !(y0 & 15);
}

// ---- bounds, MV syntax, predictors (encoder_motion.cpp:1099-1466) --------------------

struct Bounds { int xmin, xmax, ymin, ymax; };

// Vc1Encoder::motion_search_bounds_px, encoder_motion.cpp:1236-1245
__host__ __device__ inline Bounds bounds_px(int requested) {
    const int r = iclamp(requested, 0, 1024);
    return {-imin(r, 1024), imin(r, 1023), -imin(r, 256), imin(r, 255)};
}
// Vc1Encoder::motion_search_bounds_qpel, encoder_motion.cpp:1247-1254
__host__ __device__ inline Bounds bounds_qpel(int requested) {
    const int r = iclamp(requested, 0, 1024);
    Bounds b;
    b.xmin = -imin(r * 4, 4096);
    b.xmax = (r >= 1024) ? 4095 : imin(r * 4, 4095);
    b.ymin = -imin(r * 4, 1024);
    b.ymax = (r >= 256) ? 1023 : imin(r * 4, 1023);
    return b;
}

__host__ __device__ inline int median3(int a, int b, int c) { return a + b + c - imin(a, imin(b, c)) - imax(a, imax(b, c)); }
__host__ __device__ inline int round_qpel_to_pixel(int q) { return q >= 0 ? (q + 2) / 4 : -((-q + 2) / 4); }

// Vc1Encoder::modular_component_distance / modular_mv_distance, encoder_motion.cpp:1298-1310
__device__ inline int modular_component_distance(int a, int b, int range) {
    int d = a - b;
    const int span = range * 2;
    d = ((d + range) % span + span) % span - range;
    return iabs(d);
}
// mvrange_x_qpel {256,512,2048,4096} / mvrange_y_qpel {128,256,512,1024} (:1263-1271)
__device__ __forceinline__ int mvrange_xq(int r) { return r < 2 ? (256 << r) : (2048 << (r - 2)); }
__device__ __forceinline__ int mvrange_yq(int r) { return 128 << r; }
__device__ inline int modular_mv_distance(const DevParams& p, int2 a, int2 b) {
    return modular_component_distance(a.x, b.x, mvrange_xq(p.mvrange)) +
           modular_component_distance(a.y, b.y, mvrange_yq(p.mvrange));
}

// groupa::kMvDiffBits[0], vc1_groupa_tables.h:26 (VC-1 MVDATA VLC lengths, table 0)
__constant__ static const uint8_t kMvDiffBits0[73] = {
    6, 7, 7, 8, 14, 6, 5, 6, 7, 14, 14, 6, 6, 6, 8, 9, 10, 9, 7, 7, 7, 14, 14, 10, 9, 10, 8, 10, 10, 14, 14, 14,
    13, 13, 13, 6, 3, 5, 6, 8, 9, 13, 5, 4, 4, 5, 7, 9, 6, 5, 5, 5, 6, 9, 8, 5, 5, 5, 7, 10, 7, 7, 7, 7,
    7, 8, 10, 9, 8, 9, 9, 9, 3};

// Vc1Encoder::mv_cat, encoder_motion.cpp:1150-1162
__device__ inline int mv_cat(int v, bool halfpel) {
    const int a = iabs(v);
    if (!a) return 0;
    if (a <= 2) return 1;
    if (a <= 6) return 2;
    if (a <= 14) return 3;
    if (a <= 30) return 4;
    if (a <= (halfpel ? 94 : 158)) return 5;
    return -1;
}
// {0,2,3,4,5,8}[cat] minus the half-pel category-5 bit (:1173-1176)
__device__ __forceinline__ int mv_component_bits(int cat, bool halfpel) {
    const int sz = cat == 5 ? 8 : (cat ? cat + 1 : 0);
    return sz - ((halfpel && cat == 5) ? 1 : 0);
}

// mvdata_for_mode (:1099-1114), mv_symbol (:1164-1171) and mv_suffix_bits (:1178-1197) of a
// non-intra MVDATA: the symbol (0..72), and in `suffix` the escape or category suffix bits. A
// half-pel mode codes the differential in half-pel units (callers keep it even).
__device__ inline int mv_symbol_suffix(const DevParams& p, int2 desired, int2 pred, int mode, bool more, int& suffix) {
    const bool hp = mode_halfpel(mode);
    int dx = desired.x - pred.x, dy = desired.y - pred.y;
    if (hp) { dx /= 2; dy /= 2; }
    const int xc = mv_cat(dx, hp), yc = mv_cat(dy, hp);
    int sym;
    if (xc < 0 || yc < 0) sym = more ? 71 : 34;
    else {
        const int idx = yc * 6 + xc;
        sym = (!more && idx == 0) ? 34 : (more ? idx + 36 : idx - 1);
    }
    if (sym == 34 || sym == 71) {
        // mvrange_kx {9,10,12,13} / mvrange_ky {8,9,10,11} (:1273-1281)
        const int kx = p.mvrange < 2 ? 9 + p.mvrange : 10 + p.mvrange, ky = 8 + p.mvrange;
        const int h = hp ? 1 : 0;
        suffix = (kx - h) + (ky - h);
    } else {
        suffix = mv_component_bits(xc, hp) + mv_component_bits(yc, hp);
    }
    return sym;
}

// Vc1Encoder::motion_vector_rate_bits, encoder_motion.cpp:3214-3225: the MVDATA length under
// table 0 (the reference's local proxy) plus the suffix.
__device__ inline uint32_t mv_rate_bits(const DevParams& p, int2 desired, int2 pred, int mode, bool more) {
    int suffix;
    const int sym = mv_symbol_suffix(p, desired, pred, mode, more, suffix);
    return (uint32_t)kMvDiffBits0[sym] + (uint32_t)suffix;
}

struct PInfo {
    int2 pre, a, c;
    bool a_valid, c_valid, hybrid;
};

__device__ inline void pullback(int2& pre, int qx, int qy, int X, int Y, int margin) {
    if (qx + pre.x < margin) pre.x = margin - qx;
    if (qx + pre.x > X) pre.x = X - qx;
    if (qy + pre.y < margin) pre.y = margin - qy;
    if (qy + pre.y > Y) pre.y = Y - qy;
}
__device__ inline bool hybrid_of(int2 pre, int2 A, int2 C, bool a_intra, bool c_intra) {
    const int suma = a_intra ? iabs(pre.x) + iabs(pre.y) : iabs(pre.x - A.x) + iabs(pre.y - A.y);
    if (suma > 32) return true;
    const int sumc = c_intra ? iabs(pre.x) + iabs(pre.y) : iabs(pre.x - C.x) + iabs(pre.y - C.y);
    return sumc > 32;
}

// Vc1Encoder::predictor_info_mixed_1mv, encoder_motion.cpp:1354-1406. F reads the block-MV field:
// get(x, y) the vector of 8x8 block (x, y) (zero outside the raster), intra(x, y) its MB's intra flag.
template <class F>
__device__ PInfo predictor_mixed_1mv(const DevParams& P, const F& f, int mx, int my) {
    PInfo r;
    const int bx = mx * 2, by = my * 2, mbw = P.mbw;
    const bool a_valid = my > 0, c_valid = mx > 0, b_valid = my > 0 && mbw > 1;
    const int2 z = make_int2(0, 0);
    const int2 A = a_valid ? f.get(bx, by - 1) : z;
    const int2 C = c_valid ? f.get(bx - 1, by) : z;
    int2 B = z;
    if (b_valid) B = f.get(bx + ((mx == mbw - 1) ? -1 : 2), by - 1);
    int2 pre = z;
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if ((int)a_valid + (int)b_valid + (int)c_valid > 1) {
        pre.x = median3(A.x, B.x, C.x);
        pre.y = median3(A.y, B.y, C.y);
    }
    pullback(pre, mx * 64, my * 64, mbw * 64 - 4, P.mbh * 64 - 4, -60);
    const bool hybrid = a_valid && c_valid && hybrid_of(pre, A, C, f.intra(bx, by - 1), f.intra(bx - 1, by));
    r.pre = pre; r.a = A; r.c = C; r.a_valid = a_valid; r.c_valid = c_valid; r.hybrid = hybrid;
    return r;
}

// Vc1Encoder::predictor_info_4mv, encoder_motion.cpp:1408-1466
template <class F>
__device__ PInfo predictor_4mv(const DevParams& P, const F& f, int mx, int my, int n) {
    PInfo r;
    const int mbw = P.mbw;
    const int bx = mx * 2 + (n & 1), by = my * 2 + ((n >> 1) & 1);
    const bool a_valid = my > 0 || n == 2 || n == 3;
    const bool c_valid = mx > 0 || n == 1 || n == 3;
    const bool b_valid = a_valid;
    const int2 z = make_int2(0, 0);
    const int2 A = a_valid ? f.get(bx, by - 1) : z;
    const int2 C = c_valid ? f.get(bx - 1, by) : z;
    int2 B = z;
    if (b_valid) {
        int bxx = bx;
        if (n == 0) bxx += mx ? -1 : 1;
        else if (n == 1) bxx += (mx == mbw - 1) ? -1 : 1;
        else if (n == 2) bxx += 1;
        else bxx -= 1;
        B = f.get(bxx, by - 1);
    }
    int2 pre = z;
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if ((int)a_valid + (int)b_valid + (int)c_valid > 1) {
        pre.x = median3(A.x, B.x, C.x);
        pre.y = median3(A.y, B.y, C.y);
    }
    pullback(pre, mx * 64 + ((n == 1 || n == 3) ? 32 : 0), my * 64 + ((n == 2 || n == 3) ? 32 : 0), mbw * 64 - 4,
             P.mbh * 64 - 4, -28);
    const bool hybrid = a_valid && c_valid && hybrid_of(pre, A, C, f.intra(bx, by - 1), f.intra(bx - 1, by));
    r.pre = pre; r.a = A; r.c = C; r.a_valid = a_valid; r.c_valid = c_valid; r.hybrid = hybrid;
    return r;
}

// ---- the x87 long double score (encoder_motion.cpp:3458-3476, :3518-3524) -------------
//
// score = (long double)sad + lambda_me * (long double)rate with lambda_me = max(1, 0.35*PQ).
// lambda_me = lam_m * 2^-lam_s exactly, so the exact sum is (sad << lam_s) + lam_m * rate,
// and the reference's long double is that integer rounded to mant_bits significant bits
// (round to nearest, ties to even). Candidates of one call share lam_s, so comparing the
// rounded integers orders them exactly as the reference's long double comparisons do.
__device__ inline unsigned __int128 score_key(const DevParams& p, uint64_t lam_m, int lam_s, uint64_t sad, uint32_t rate) {
    unsigned __int128 v = ((unsigned __int128)sad << lam_s) + (unsigned __int128)lam_m * rate;
    const uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    const int nbits = hi ? 128 - __clzll((long long)hi) : (lo ? 64 - __clzll((long long)lo) : 0);
    if (nbits > p.mant_bits) {
        const int drop = nbits - p.mant_bits;
        const unsigned __int128 one = 1;
        const unsigned __int128 rem = v & ((one << drop) - 1), half = one << (drop - 1);
        v >>= drop;
        if (rem > half || (rem == half && (v & 1))) v += 1;
        v <<= drop;
    }
    return v;
}

// tie_less, encoder_motion.cpp:3314-3319: (|x|+|y|, y, x)
__device__ __forceinline__ bool tie_less(int2 a, int2 b) {
    const int am = iabs(a.x) + iabs(a.y), bm = iabs(b.x) + iabs(b.y);
    if (am != bm) return am < bm;
    if (a.y != b.y) return a.y < b.y;
    return a.x < b.x;
}

// Total order (cost, |dx|+|dy|, dy, dx) of the integer searches (encoder_motion.cpp:1786-1792)
// packed into one comparable 64-bit key. Legal costs of a 16x16 block are < 2^17 (also
// after the stride^2 rescale); every illegal cost maps to the largest 20-bit value, and
// illegal candidates then order by (|d|, dy, dx) exactly like the reference.
__device__ __forceinline__ uint64_t int_key(uint64_t cost, int dx, int dy) {
    const uint64_t c = cost >= 0xFFFFFull ? 0xFFFFFull : cost;
    return (c << 44) | ((uint64_t)(iabs(dx) + iabs(dy)) << 32) | ((uint64_t)(dy + 2048) << 20) |
           ((uint64_t)(dx + 2048) << 8);
}
__device__ __forceinline__ int key_dx(uint64_t k) { return (int)((k >> 8) & 0xFFF) - 2048; }
__device__ __forceinline__ int key_dy(uint64_t k) { return (int)((k >> 20) & 0xFFF) - 2048; }
__device__ __forceinline__ uint64_t key_cost(uint64_t k) {
    const uint64_t c = k >> 44;
    return c == 0xFFFFFull ? kBad : c;
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace vc1cu
