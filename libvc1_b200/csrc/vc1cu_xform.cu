// vc1cu_xform.cu - decoder-equivalent prediction of a motion field and the forward
// 8x8/8x4/4x8/4x4 transform + scalar quantiser of its residual.
//
// Prediction follows motion_compensate_mb / motion_compensate_4mv
// (encoder_motion_compensation.cpp:474-600). The transform is the reference's FP64 law
// (forward_transform_residual[_part], encoder_transform.cpp:797-1045): residual rows
// multiplied by the k8/k4 matrices in the reference's loop order, every product and sum
// rounded separately (this translation unit is compiled with --fmad=false and spells the
// operations with __dmul_rn/__dadd_rn), then scalar_quantize_level (:1067-1085).
#include <cuda_runtime.h>

#include <climits>
#include <cstring>

#include "vc1cu_core.cuh"
#define VC1CU_ENT_TABLE __constant__ const
#include "vc1cu_entropy_lengths.h"
#include "vc1cu_pred.cuh"

namespace vc1cu {

// forward_transform::k4 / k8, forward_transform_tables.h:9-25 (inverse VC-1 basis)
__constant__ double c_k4[4][4] = {
    {0.0147058823529412, 0.0147058823529412, 0.0147058823529412, 0.0147058823529412},
    {0.0188356164383562, 0.0085616438356164, -0.0085616438356164, -0.0188356164383562},
    {0.0147058823529412, -0.0147058823529412, -0.0147058823529412, 0.0147058823529412},
    {0.0085616438356164, -0.0188356164383562, 0.0188356164383562, -0.0085616438356164}};
__constant__ double c_k8[8][8] = {
    {0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667, 0.010416666667},
    {0.013840830450, 0.012975778547, 0.007785467128, 0.003460207612, -0.003460207612, -0.007785467128, -0.012975778547, -0.013840830450},
    {0.013698630137, 0.005136986301, -0.005136986301, -0.013698630137, -0.013698630137, -0.005136986301, 0.005136986301, 0.013698630137},
    {0.012975778547, -0.003460207612, -0.013840830450, -0.007785467128, 0.007785467128, 0.013840830450, 0.003460207612, -0.012975778547},
    {0.010416666667, -0.010416666667, -0.010416666667, 0.010416666667, 0.010416666667, -0.010416666667, -0.010416666667, 0.010416666667},
    {0.007785467128, -0.013840830450, 0.003460207612, 0.012975778547, -0.012975778547, -0.003460207612, 0.013840830450, -0.007785467128},
    {0.005136986301, -0.013698630137, 0.013698630137, -0.005136986301, -0.005136986301, 0.013698630137, -0.013698630137, 0.005136986301},
    {0.003460207612, -0.007785467128, 0.012975778547, -0.013840830450, 0.013840830450, -0.012975778547, 0.007785467128, -0.003460207612}};

// Vc1Encoder::chroma_mc_sample, encoder_motion_compensation.cpp:417-447 (P: future = false)
__device__ __forceinline__ int chroma_sample(const uint8_t* p, int pitch, int w, int h, int x, int y, int mvx, int mvy,
                                             int rnd) {
    int uvx = arshift(mvx + ((mvx & 3) == 3), 1);
    int uvy = arshift(mvy + ((mvy & 3) == 3), 1);
    if (uvx < 0) uvx += (uvx & 1); else uvx -= (uvx & 1);
    if (uvy < 0) uvy += (uvy & 1); else uvy -= (uvy & 1);
    const int ix = floor_div4(uvx), iy = floor_div4(uvy);
    const int fx = (uvx - ix * 4) * 2, fy = (uvy - iy * 4) * 2;
    const int sx = x + ix, sy = y + iy;
    auto S = [&](int xx, int yy) { return (int)__ldg(p + (size_t)iclamp(yy, 0, h - 1) * pitch + iclamp(xx, 0, w - 1)); };
    const int a = S(sx, sy);
    if (!fx && !fy) return a;
    const int b = S(sx + 1, sy), c = S(sx, sy + 1), d = S(sx + 1, sy + 1);
    const int value = a * (8 - fx) * (8 - fy) + b * fx * (8 - fy) + c * (8 - fx) * fy + d * fx * fy;
    return (value + (rnd ? 28 : 32)) >> 6;
}

__device__ __forceinline__ int median4(int a, int b, int c, int d) {
    if (a < b) {
        if (c < d) return (imin(b, d) + imax(a, c)) / 2;
        return (imin(b, c) + imax(a, d)) / 2;
    }
    if (c < d) return (imin(a, d) + imax(b, c)) / 2;
    return (imin(a, c) + imax(b, d)) / 2;
}

// One thread per luma pixel (and, for even pixels, the co-sited chroma pair).
__global__ void mc_kernel(const __grid_constant__ DevParams P, DevFrame ref, const int2* mvs, const int2* bmv,
                          const uint8_t* use4, int mode, uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= P.W || y >= P.H) return;
    const int mx = x >> 4, my = y >> 4, pos = my * P.mbw + mx;
    const GlobSampler gs{ref.y, ref.pitch_y, P.W, P.H};
    int out[1];
    int2 cmv;
    if (use4[pos]) {
        const int k = ((y >> 3) & 1) * 2 + ((x >> 3) & 1);
        const int2 v = bmv[pos * 4 + k];
        predict_row<1>(gs, false, P.rnd, v.x, v.y, x, y, out);
        const int2 a = bmv[pos * 4 + 0], b = bmv[pos * 4 + 1], c = bmv[pos * 4 + 2], d = bmv[pos * 4 + 3];
        cmv = make_int2(median4(a.x, b.x, c.x, d.x), median4(a.y, b.y, c.y, d.y));
    } else {
        const int2 v = mvs[pos];
        predict_row<1>(gs, mode_bilinear(mode), P.rnd, v.x, v.y, x, y, out);
        cmv = v;
    }
    dy[(size_t)y * pitch_y + x] = (uint8_t)out[0];
    if (!(x & 1) && !(y & 1)) {
        const int cw = P.W / 2, ch = P.H / 2, cx = x >> 1, cy = y >> 1;
        if (cx < cw && cy < ch) {
            du[(size_t)cy * pitch_c + cx] = (uint8_t)chroma_sample(ref.u, ref.pitch_c, cw, ch, cx, cy, cmv.x, cmv.y, P.rnd);
            dv[(size_t)cy * pitch_c + cx] = (uint8_t)chroma_sample(ref.v, ref.pitch_c, cw, ch, cx, cy, cmv.x, cmv.y, P.rnd);
        }
    }
}

// Vc1Encoder::scalar_quantize_level, encoder_transform.cpp:1067-1085 (mquant = PQINDEX)
__device__ __forceinline__ int quantize_level(const DevParams& P, double coeff) {
    if (coeff == 0.0) return 0;
    const int sign = coeff < 0.0 ? -1 : 1;
    const double a = fabs(coeff);
    const double dq = (double)(2 * P.pq + (P.halfqp ? 1 : 0));
    const double offset = P.nonuniform ? (double)P.pq : 0.0;
    const int max_level = (1 << (P.pq < 8 ? 11 : 8)) - 1;
    int center = (int)llround(__ddiv_rn(__dsub_rn(a, offset), dq > 1.0 ? dq : 1.0));
    center = iclamp(center, 1, max_level);
    int best = 0;
    double besterr = __dmul_rn(a, a);
    for (int n = imax(1, center - 1); n <= imin(max_level, center + 1); ++n) {
        const double recon = __dadd_rn(__dmul_rn((double)n, dq), offset);
        const double e = __dsub_rn(a, recon);
        const double e2 = __dmul_rn(e, e);
        if (e2 < besterr) { besterr = e2; best = n; }
    }
    return sign * best;
}

// Threads per (MB, parent) of transform type t: one per partition row (partitions x rows).
__device__ __forceinline__ int xform_threads(int t) { return t == 1 || t == 2 ? 8 : 16; }

// One thread per (type, MB, parent, partition, transform row a): the row of the vertical stage
// and the outputs of frequency a (an 8x8 output column, transposed; a rectangle's row). Every
// product and sum is the reference's, in its order. Output layout [type][mb][parent][64].
__global__ void xform_kernel(const __grid_constant__ DevParams P, DevFrame src, DevFrame pred, int type_mask, double* coeffs,
                             int16_t* levels) {
    const int mbs = P.mbw * P.mbh;
    long off = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int ti = -1, t = 0, nt = 0;
    for (int tt = 1; tt <= 4; ++tt) {
        if (!(type_mask & (1 << (tt - 1)))) continue;
        const long n = (long)mbs * 6 * xform_threads(tt);
        if (ti < 0) {
            if (off < n) {
                ti = nt;
                t = tt;
            } else {
                off -= n;
            }
        }
        ++nt;
    }
    if (ti < 0) return;
    const int per = xform_threads(t);
    const int sub = (int)(off % per);
    const long pk = off / per;
    const int k = (int)(pk % 6), mb = (int)(pk / 6);
    const int bh = (t == 2 || t == 4) ? 4 : 8, bw = (t == 3 || t == 4) ? 4 : 8;
    const int part = sub / bh, a = sub % bh;
    int ox = 0, oy = 0;
    if (t == 2) oy = part * 4;
    else if (t == 3) ox = part * 4;
    else if (t == 4) { ox = (part & 1) * 4; oy = (part >> 1) * 4; }
    const int mx = mb % P.mbw, my = mb / P.mbw;
    const bool chroma = k >= 4;
    const uint8_t* sp = chroma ? (k == 4 ? src.u : src.v) : src.y;
    const uint8_t* pp = chroma ? (k == 4 ? pred.u : pred.v) : pred.y;
    const int spitch = chroma ? src.pitch_c : src.pitch_y, ppitch = chroma ? pred.pitch_c : pred.pitch_y;
    const int w = chroma ? P.W / 2 : P.W, h = chroma ? P.H / 2 : P.H;
    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
    const int x0 = bx * 8 + ox, y0 = by * 8 + oy;
    const size_t base = (((size_t)ti * mbs + mb) * 6 + k) * 64;
    // output b of this thread's frequency a: transposed for 8x8, row-major for rectangles
    auto out_pos = [&](int b) {
        return (bw == 8 && bh == 8) ? base + (size_t)(oy + b) * 8 + ox + a : base + (size_t)(oy + a) * 8 + ox + b;
    };
    if (x0 >= w || y0 >= h || x0 + bw <= 0 || y0 + bh <= 0) {
        // a partition wholly outside the crop codes nothing (encoder_transform.cpp:1097)
        for (int b = 0; b < bw; ++b) {
            if (coeffs) coeffs[out_pos(b)] = 0.0;
            if (levels) levels[out_pos(b)] = 0;
        }
        return;
    }
    double trow[8];
    for (int x = 0; x < bw; ++x) {
        double acc = 0.0;
        for (int y = 0; y < bh; ++y) {
            const int sx = x0 + x, sy = y0 + y;
            const double r = (sx < 0 || sy < 0 || sx >= w || sy >= h)
                                 ? 0.0
                                 : (double)((int)__ldg(sp + (size_t)sy * spitch + sx) - (int)__ldg(pp + (size_t)sy * ppitch + sx));
            acc = __dadd_rn(acc, __dmul_rn(bh == 8 ? c_k8[a][y] : c_k4[a][y], r));
        }
        trow[x] = acc;
    }
    for (int b = 0; b < bw; ++b) {
        double acc = 0.0;
        for (int x = 0; x < bw; ++x) acc = __dadd_rn(acc, __dmul_rn(trow[x], bw == 8 ? c_k8[b][x] : c_k4[b][x]));
        const double c = __dmul_rn(1024.0, acc);
        if (coeffs) coeffs[out_pos(b)] = c;
        if (levels) levels[out_pos(b)] = (int16_t)quantize_level(P, c);
    }
}

// ---- inverse transform and reconstruction (encoder_transform.cpp:1058-1274, :1569-1585) ----

// Vc1Encoder::dequant_level at mquant = PQINDEX without DQUANT (2*PQ + HALFQP, plus PQ away from
// zero for the non-uniform quantiser)
__device__ __forceinline__ int dequant(const DevParams& P, int level) {
    if (!level) return 0;
    const int v = level * (2 * P.pq + (P.halfqp ? 1 : 0));
    return P.nonuniform ? v + (level > 0 ? P.pq : -P.pq) : v;
}

// The VC-1 8-point inverse butterfly (inverse_transform_8x8, :566-609); tail adds the second
// stage's +1 to the lower four outputs.
__device__ __forceinline__ void inv8(const int* s, int st, int* o, int ot, int bias, int shift, int tail) {
    int t1 = 12 * (s[0] + s[4 * st]) + bias, t2 = 12 * (s[0] - s[4 * st]) + bias;
    int t3 = 16 * s[2 * st] + 6 * s[6 * st], t4 = 6 * s[2 * st] - 16 * s[6 * st];
    const int t5 = t1 + t3, t6 = t2 + t4, t7 = t2 - t4, t8 = t1 - t3;
    t1 = 16 * s[st] + 15 * s[3 * st] + 9 * s[5 * st] + 4 * s[7 * st];
    t2 = 15 * s[st] - 4 * s[3 * st] - 16 * s[5 * st] - 9 * s[7 * st];
    t3 = 9 * s[st] - 16 * s[3 * st] + 4 * s[5 * st] + 15 * s[7 * st];
    t4 = 4 * s[st] - 9 * s[3 * st] + 15 * s[5 * st] - 16 * s[7 * st];
    o[0] = arshift(t5 + t1, shift);
    o[ot] = arshift(t6 + t2, shift);
    o[2 * ot] = arshift(t7 + t3, shift);
    o[3 * ot] = arshift(t8 + t4, shift);
    o[4 * ot] = arshift(t8 - t4 + tail, shift);
    o[5 * ot] = arshift(t7 - t3 + tail, shift);
    o[6 * ot] = arshift(t6 - t2 + tail, shift);
    o[7 * ot] = arshift(t5 - t1 + tail, shift);
}
// The 4-point one of the 8x4 / 4x8 / 4x4 partitions (inverse_partition, :1213-1272)
__device__ __forceinline__ void inv4(const int* s, int st, int* o, int ot, int bias, int shift) {
    const int t1 = 17 * (s[0] + s[2 * st]) + bias, t2 = 17 * (s[0] - s[2 * st]) + bias;
    const int t3 = 22 * s[st] + 10 * s[3 * st], t4 = 22 * s[3 * st] - 10 * s[st];
    o[0] = arshift(t1 + t3, shift);
    o[ot] = arshift(t2 - t4, shift);
    o[2 * ot] = arshift(t2 + t4, shift);
    o[3 * ot] = arshift(t1 - t3, shift);
}

// dequant_level (encoder_transform.cpp:1052-1065) at an MB's MQUANT: a DQUANT-derived MQUANT, or one
// other than PQINDEX, takes no HALFQP half step
__device__ __forceinline__ int dequant_mq(const DevParams& P, int level, int mquant, bool derived) {
    if (!level) return 0;
    const int v = level * (2 * mquant + ((!derived && mquant == P.pq && P.halfqp) ? 1 : 0));
    return P.nonuniform ? v + (level > 0 ? mquant : -mquant) : v;
}

// One thread per (MB, parent): every partition of the block's chosen type dequantised at PQINDEX
// or at the MB's MQUANT (mquant / derived: per-MB device arrays, or nullptr), inverse-transformed
// (with the DC-only shortcut of a partition whose only level is its DC) and added to the
// prediction with 8-bit clamping. tindex[t] is type t's index in the levels layout
// [type][mb][parent][64] (-1 for a type the layout does not hold).
__global__ void recon_kernel(const __grid_constant__ DevParams P, DevFrame pred, const int16_t* levels, int4 tindex,
                             const uint8_t* block_types, uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c,
                             const uint8_t* mquant, const uint8_t* derived) {
    const int mbs = P.mbw * P.mbh;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= mbs * 6) return;
    const int mb = idx / 6, k = idx - mb * 6, mx = mb % P.mbw, my = mb / P.mbw;
    const int t = block_types[idx];
    const int ti = t == 1 ? tindex.x : (t == 2 ? tindex.y : (t == 3 ? tindex.z : tindex.w));
    const int16_t* q64 = levels + (((size_t)ti * mbs + mb) * 6 + k) * 64;
    const int mq = mquant ? (int)mquant[mb] : P.pq;
    const bool der = derived && derived[mb];
    int res[64];
#pragma unroll
    for (int i = 0; i < 64; ++i) res[i] = 0;
    const int np = t == 1 ? 1 : (t == 4 ? 4 : 2);
    for (int part = 0; part < np; ++part) {
        int ox = 0, oy = 0, bw = 8, bh = 8;
        if (t == 2) { bh = 4; oy = part * 4; }
        else if (t == 3) { bw = 4; ox = part * 4; }
        else if (t == 4) { bw = bh = 4; ox = (part & 1) * 4; oy = (part >> 1) * 4; }
        int a[64], tmp[64];
        int nonzero = 0, q0 = 0;
        for (int y = 0; y < 8; ++y)
            for (int x = 0; x < 8; ++x) {
                const int lv = (y < bh && x < bw) ? q64[(oy + y) * 8 + ox + x] : 0;
                nonzero += lv != 0;
                if (!y && !x) q0 = lv;
                a[y * 8 + x] = mquant ? dequant_mq(P, lv, mq, der) : dequant(P, lv);
                tmp[y * 8 + x] = 0;
            }
        if (nonzero == 1 && q0 != 0) {
            int dc = a[0];
            if (t == 1) { dc = arshift(3 * dc + 1, 1); dc = arshift(3 * dc + 16, 5); }
            else if (t == 2) { dc = arshift(3 * dc + 1, 1); dc = arshift(17 * dc + 64, 7); }
            else if (t == 3) { dc = arshift(17 * dc + 4, 3); dc = arshift(12 * dc + 64, 7); }
            else { dc = arshift(17 * dc + 4, 3); dc = arshift(17 * dc + 64, 7); }
            for (int y = 0; y < bh; ++y)
                for (int x = 0; x < bw; ++x) res[(oy + y) * 8 + ox + x] = dc;
            continue;
        }
        if (t == 1) {
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
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) res[(oy + y) * 8 + ox + x] = a[y * 8 + x];
    }
    const bool luma = k < 4;
    const int w = luma ? P.W : P.W / 2, h = luma ? P.H : P.H / 2;
    const int bx = luma ? mx * 2 + (k & 1) : mx, by = luma ? my * 2 + ((k >> 1) & 1) : my;
    const uint8_t* pp = luma ? pred.y : (k == 4 ? pred.u : pred.v);
    uint8_t* dp = luma ? dy : (k == 4 ? du : dv);
    const int pps = luma ? pred.pitch_y : pred.pitch_c, dps = luma ? pitch_y : pitch_c;
    for (int y = 0; y < 8 && by * 8 + y < h; ++y)
        for (int x = 0; x < 8 && bx * 8 + x < w; ++x) {
            const int v = pp[(size_t)(by * 8 + y) * pps + bx * 8 + x] + res[y * 8 + x];
            dp[(size_t)(by * 8 + y) * dps + bx * 8 + x] = (uint8_t)iclamp(v, 0, 255);
        }
}

void launch_recon(const DevParams& P, const DevFrame& pred, const int16_t* levels, int4 tindex, const uint8_t* block_types,
                  uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s, const uint8_t* mquant,
                  const uint8_t* derived) {
    const int n = P.mbw * P.mbh * 6;
    recon_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(P, pred, levels, tindex, block_types, dy, du, dv, pitch_y, pitch_c,
                                                             mquant, derived);
}

// ---- transform type of the throughput preset (encoder_transform.cpp:1605-1712) ----------------

// One warp per MB: transform_metrics::scalar (transform_residual_metrics.h:29-61) with each lane
// summing half a row, then choose_transform_mb's candidate list and the preset's pick.
__global__ void fast_tt_kernel(const __grid_constant__ DevParams P, DevFrame src, DevFrame pred, uint8_t* types) {
    const int mb = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (mb >= P.mbw * P.mbh) return;
    const int mx = mb % P.mbw, my = mb / P.mbw;
    const int py = lane >> 1, px0 = (lane & 1) * 8;
    uint32_t sad = 0, hedge = 0, vedge = 0, grad = 0;
    const int y = my * 16 + py;
    if (y < P.H) {
        auto R = [&](int xx, int yy) {
            return (int)src.y[(size_t)yy * src.pitch_y + xx] - (int)pred.y[(size_t)yy * pred.pitch_y + xx];
        };
        for (int px = px0; px < px0 + 8 && mx * 16 + px < P.W; ++px) {
            const int x = mx * 16 + px;
            const int r = R(x, y);
            sad += (uint32_t)iabs(r);
            if ((py & 7) == 4) hedge += (uint32_t)iabs(r - R(x, y - 1));
            if ((px & 7) == 4) vedge += (uint32_t)iabs(r - R(x - 1, y));
            if (px > 0) grad += (uint32_t)iabs(r - R(x - 1, y));
            if (py > 0) grad += (uint32_t)iabs(r - R(x, y - 1));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        sad += __shfl_xor_sync(0xffffffffu, sad, o);
        hedge += __shfl_xor_sync(0xffffffffu, hedge, o);
        vedge += __shfl_xor_sync(0xffffffffu, vedge, o);
        grad += __shfl_xor_sync(0xffffffffu, grad, o);
    }
    if (lane) return;
    const uint64_t S = sad, HE = hedge, VE = vedge, G = grad, lim = (uint64_t)(64 * P.pq);
    int list[4] = {1, 1, 1, 1}, count = 0;
    const bool split_x = mx == P.mbw - 1 && (P.W & 15) != 0, split_y = my == P.mbh - 1 && (P.H & 15) != 0;
    if (split_x && split_y) {
        list[count++] = 4;
    } else if (split_x || split_y) {
        list[count++] = split_x ? 3 : 2;
        if (S > lim && G > S * 2) list[count++] = 4;
    } else {
        list[count++] = 1;
        if (S > lim) {
            if (HE * 5 > VE * 6) list[count++] = 2;
            else if (VE * 5 > HE * 6) list[count++] = 3;
            else { list[count++] = 2; list[count++] = 3; }
            if (count < 4 && G > S * 2) list[count++] = 4;
        }
    }
    int chosen = list[0];
    if (count > 1) {
        int index = count - 1;
        if (list[index] == 4 && G * 2 <= S * 5) --index;
        chosen = list[index];
        if (chosen == 3 && index > 0 && list[index - 1] == 2 && HE >= VE) chosen = 2;
    }
    types[mb] = (uint8_t)chosen;
}

void launch_fast_tt(const DevParams& P, const DevFrame& src, const DevFrame& pred, uint8_t* types, cudaStream_t s) {
    const int mbs = P.mbw * P.mbh;
    fast_tt_kernel<<<(unsigned)((mbs + 3) / 4), 128, 0, s>>>(P, src, pred, types);
}

void launch_mc(const DevParams& P, const DevFrame& ref, const int2* mvs, const int2* bmv, const uint8_t* use4, int mode,
               uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s) {
    dim3 grid((P.W + 127) / 128, P.H);
    mc_kernel<<<grid, 128, 0, s>>>(P, ref, mvs, bmv, use4, mode, dy, du, dv, pitch_y, pitch_c);
}

void launch_xform(const DevParams& P, const DevFrame& src, const DevFrame& pred, int type_mask, double* coeffs,
                  int16_t* levels, cudaStream_t s) {
    long n = 0;
    for (int t = 1; t <= 4; ++t)
        if (type_mask & (1 << (t - 1))) n += (long)P.mbw * P.mbh * 6 * (t == 1 || t == 2 ? 8 : 16);
    if (!n) return;
    xform_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(P, src, pred, type_mask, coeffs, levels);
}


// ---- transform RD of the default presets (choose_transform_mb, encoder_transform.cpp:1605-1780) ----
//
// One warp per macroblock. The lanes evaluate the candidate types' 24 (type, parent) pairs at
// once (forward transform, scalar or trellis quantisation, inverse transform, reconstruction SSE,
// bit estimate); lane 0 then takes the macroblock- and block-level decisions in the reference's
// order; the trellis re-evaluation of the winners is again one parent per lane. Every double
// operation is the reference's, in its order (this file is compiled without contraction).

namespace {

// Dense rate tables built on the host from the VC-1 code lengths (vc1cu_entropy_lengths.h).
struct TrdTables {
    uint8_t ac_bits[8][2][64][64];  // direct AC code length (0: no direct code) [set][last][run][level]
    uint8_t max_level[8][2][64];    // max_direct_level
    int8_t max_run[8][2][64];       // max_direct_run (-1: none)
};

struct TrdArgs {
    DevParams P;
    DevFrame src, pred;
    const TrdTables* tab;
    const uint8_t* mquant;  // per MB, nullptr: PQINDEX
    vc1cu_trd_cfg cfg;
    double frame_mean;      // mean of the source luma plane (cached_luma_mean)
    vc1cu_tdecision* out;
    int16_t* levels;        // [mb][6][64] or nullptr
    const int* mb_list;     // nullptr: every MB; else entry i of out / levels is MB mb_list[i]
    int n_list;
};

__device__ __forceinline__ double dclamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

// picture_double_quant (:1052-1056), dequant_level (:1058-1065), scalar_quantize_level (:1067-1085)
__device__ __forceinline__ int trd_double_quant(const DevParams& P, int mquant, bool derived) {
    return 2 * mquant + ((!derived && mquant == P.pq && P.halfqp) ? 1 : 0);
}
__device__ __forceinline__ int trd_max_level(const DevParams& P) { return (1 << (P.pq < 8 ? 11 : 8)) - 1; }
__device__ int trd_dequant(const DevParams& P, int level, int mquant, bool derived) {
    if (!level) return 0;
    long long v = (long long)level * trd_double_quant(P, mquant, derived);
    if (P.nonuniform) v += level > 0 ? mquant : -mquant;
    return (int)(v < INT_MIN ? INT_MIN : (v > INT_MAX ? INT_MAX : v));
}
__device__ int trd_squant(const DevParams& P, double coeff, int mquant, bool derived) {
    if (coeff == 0.0) return 0;
    const int sign = coeff < 0.0 ? -1 : 1;
    const double a = fabs(coeff);
    const double dq = (double)trd_double_quant(P, mquant, derived);
    const double offset = P.nonuniform ? (double)mquant : 0.0;
    const int max_level = trd_max_level(P);
    int center = (int)llround(__ddiv_rn(__dsub_rn(a, offset), dq > 1.0 ? dq : 1.0));
    center = iclamp(center, 1, max_level);
    int best = 0;
    double besterr = __dmul_rn(a, a);
    for (int n = imax(1, center - 1); n <= imin(max_level, center + 1); ++n) {
        const double e = __dsub_rn(a, __dadd_rn(__dmul_rn((double)n, dq), offset));
        const double e2 = __dmul_rn(e, e);
        if (e2 < besterr) { besterr = e2; best = n; }
    }
    return sign * best;
}

__device__ __forceinline__ void part_geometry(int t, int part, int& ox, int& oy, int& bw, int& bh) {
    ox = 0; oy = 0; bw = 8; bh = 8;
    if (t == 2) { bh = 4; oy = part * 4; }
    else if (t == 3) { bw = 4; ox = part * 4; }
    else if (t == 4) { bw = bh = 4; ox = (part & 1) * 4; oy = (part >> 1) * 4; }
}
__device__ __forceinline__ int part_count(int t) { return t == 1 ? 1 : (t == 4 ? 4 : 2); }

// forward_transform_residual_part (:935-1045) into a partition-local 8-stride array: 8x8 output
// transposed, rectangles row-major; samples outside the visible w x h are zero.
__device__ void trd_forward(const uint8_t* sp, int spitch, const uint8_t* pp, int ppitch, int w, int h, int x0, int y0,
                            int bw, int bh, double* c) {
    double r[8][8];
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) {
            const int sx = x0 + x, sy = y0 + y;
            r[y][x] = (sx < 0 || sy < 0 || sx >= w || sy >= h)
                          ? 0.0
                          : (double)((int)__ldg(sp + (size_t)sy * spitch + sx) - (int)__ldg(pp + (size_t)sy * ppitch + sx));
        }
    double tmp[8][8];
    for (int a = 0; a < bh; ++a)
        for (int x = 0; x < bw; ++x) {
            double acc = 0.0;
            for (int y = 0; y < bh; ++y) acc = __dadd_rn(acc, __dmul_rn(bh == 8 ? c_k8[a][y] : c_k4[a][y], r[y][x]));
            tmp[a][x] = acc;
        }
    for (int i = 0; i < 64; ++i) c[i] = 0.0;
    for (int a = 0; a < bh; ++a)
        for (int b = 0; b < bw; ++b) {
            double acc = 0.0;
            for (int x = 0; x < bw; ++x) acc = __dadd_rn(acc, __dmul_rn(tmp[a][x], bw == 8 ? c_k8[b][x] : c_k4[b][x]));
            const double v = __dmul_rn(1024.0, acc);
            if (bw == 8 && bh == 8) c[b * 8 + a] = v;
            else c[a * 8 + b] = v;
        }
}

// inverse_partition (:1173-1274) of partition-local levels q into residuals a (8-stride)
__device__ void trd_inverse(const DevParams& P, int t, const int* q, int mquant, bool derived, int* a) {
    int bw, bh, ox, oy;
    part_geometry(t, 0, ox, oy, bw, bh);
    int nonzero = 0;
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) nonzero += q[y * 8 + x] != 0;
    for (int i = 0; i < 64; ++i) a[i] = 0;
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) a[y * 8 + x] = trd_dequant(P, q[y * 8 + x], mquant, derived);
    if (nonzero == 1 && q[0] != 0) {
        int dc = a[0];
        if (t == 1) { dc = arshift(3 * dc + 1, 1); dc = arshift(3 * dc + 16, 5); }
        else if (t == 2) { dc = arshift(3 * dc + 1, 1); dc = arshift(17 * dc + 64, 7); }
        else if (t == 3) { dc = arshift(17 * dc + 4, 3); dc = arshift(12 * dc + 64, 7); }
        else { dc = arshift(17 * dc + 4, 3); dc = arshift(17 * dc + 64, 7); }
        for (int i = 0; i < 64; ++i) a[i] = 0;
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) a[y * 8 + x] = dc;
        return;
    }
    int tmp[64];
    for (int i = 0; i < 64; ++i) tmp[i] = 0;
    if (t == 1) {
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

// ---- the perceptual lambda scale (perceptual_lambda_scale, encoder_aq.cpp:405-653) ----------

struct AqStats {
    double mean = 128.0, grad_avg = 0.0, residual_avg = 0.0;
    int mn = 255, mx = 0, edges = 0, n = 0;
};

__device__ AqStats aq_stats(const uint8_t* plane, int pitch, int pw, int ph, int sx, int sy, int sw, int sh,
                            const uint8_t* pp, int ppitch) {
    AqStats st;
    unsigned long long sum = 0, grad = 0, residual = 0;
    int grad_n = 0;
    for (int y = 0; y < sh && sy + y < ph; ++y)
        for (int x = 0; x < sw && sx + x < pw; ++x) {
            const int px = sx + x, py = sy + y;
            const int v = __ldg(plane + (size_t)py * pitch + px);
            sum += (unsigned long long)v;
            st.mn = imin(st.mn, v);
            st.mx = imax(st.mx, v);
            ++st.n;
            if (pp) residual += (unsigned long long)iabs(v - (int)__ldg(pp + (size_t)py * ppitch + px));
            if (x > 0) {
                const int d = iabs(v - (int)__ldg(plane + (size_t)py * pitch + px - 1));
                grad += (unsigned long long)d;
                ++grad_n;
                if (d >= 96) ++st.edges;
            }
            if (y > 0) {
                const int d = iabs(v - (int)__ldg(plane + (size_t)(py - 1) * pitch + px));
                grad += (unsigned long long)d;
                ++grad_n;
                if (d >= 96) ++st.edges;
            }
        }
    if (st.n) {
        st.mean = (double)sum / st.n;
        st.grad_avg = (double)grad / imax(1, grad_n);
        st.residual_avg = pp ? (double)residual / st.n : 0.0;
    }
    return st;
}

__device__ __forceinline__ double aq_activity(const AqStats& st) {
    const double range = (double)imax(0, st.mx - st.mn);
    const double g = dclamp((st.grad_avg - 0.35) / 5.0, 0.0, 1.0);
    const double r = dclamp((range - 1.5) / 18.0, 0.0, 1.0);
    return dmax(g, r);
}

// plane (pitch) of w x h; pp the prediction (or nullptr); luma: the picture's luma plane when the
// block is chroma (the luma context), else nullptr
// adjacency_out (luma blocks): the quiet-block-next-to-detail term, 0 when the scale is not
// computed (perceptual_lambda_scale's adjacency_out, encoder_aq.cpp:410, :641)
__device__ double aq_scale(const TrdArgs& A, const uint8_t* plane, int pitch, int w, int h, int x0, int y0, int bw, int bh,
                           const uint8_t* pp, int ppitch, const uint8_t* luma, int lpitch, double* adjacency_out = nullptr) {
    const vc1cu_trd_cfg& c = A.cfg;
    if (adjacency_out) *adjacency_out = 0.0;
    if (!c.adaptive_quality || c.aq_strength <= 0.0) return 1.0;
    const AqStats st = aq_stats(plane, pitch, w, h, x0, y0, bw, bh, pp, ppitch);
    if (!st.n) return 1.0;
    const double range = (double)imax(0, st.mx - st.mn);
    const double contrast = dclamp((range - 64.0) / 144.0, 0.0, 1.0) * dclamp((st.grad_avg - 7.0) / 40.0, 0.0, 1.0);
    const double edge_density = dclamp((double)st.edges / imax(1, st.n / 3), 0.0, 1.0);
    const double motion = dclamp((st.residual_avg - 5.0) / 30.0, 0.0, 1.0);
    if (luma) {
        const AqStats ly = aq_stats(luma, lpitch, A.P.W, A.P.H, x0 * 2, y0 * 2, bw * 2, bh * 2, nullptr, 0);
        const double chroma_detail =
            dmax(dclamp((st.grad_avg - 1.5) / 11.0, 0.0, 1.0), dclamp((range - 6.0) / 48.0, 0.0, 1.0));
        const double luma_activity = aq_activity(ly);
        const double luma_flat = dclamp((0.42 - luma_activity) / 0.42, 0.0, 1.0);
        const double luma_visibility = 0.20 + 0.80 * dclamp((ly.mean - 1.0) / 14.0, 0.0, 1.0);
        const double chroma_on_flat = luma_flat * chroma_detail * luma_visibility;
        const double frame_mean = A.frame_mean;
        const double dim_area = dclamp((132.0 - ly.mean) / 104.0, 0.0, 1.0);
        const double dim_frame = dclamp((132.0 - frame_mean) / 104.0, 0.0, 1.0);
        const double not_black = dclamp((ly.mean - 0.75) / 9.0, 0.0, 1.0);
        const double dim_detail = dmax(dim_area, 0.80 * dim_frame) * not_black * chroma_detail;
        const double protect = c.aq_strength * (1.90 * chroma_on_flat + 0.70 * dim_detail + 0.12 * contrast +
                                                0.08 * edge_density + 0.05 * motion);
        return dclamp(1.0 / (1.0 + protect), 0.24, 1.0);
    }
    unsigned long long dark_grad = 0;
    int dark_n = 0;
    for (int y = 0; y < bh && y0 + y < h; ++y)
        for (int x = 0; x < bw && x0 + x < w; ++x) {
            const int px = x0 + x, py = y0 + y;
            const int v = __ldg(plane + (size_t)py * pitch + px);
            if (x > 0 && v >= 2 && v <= 112) {
                dark_grad += (unsigned long long)iabs(v - (int)__ldg(plane + (size_t)py * pitch + px - 1));
                ++dark_n;
            }
            if (y > 0 && v >= 2 && v <= 112) {
                dark_grad += (unsigned long long)iabs(v - (int)__ldg(plane + (size_t)(py - 1) * pitch + px));
                ++dark_n;
            }
        }
    const double dark_avg = dark_n ? (double)dark_grad / dark_n : 0.0;
    const double dark_window = dclamp((118.0 - st.mean) / 96.0, 0.0, 1.0) * dclamp((st.mean - 1.0) / 13.0, 0.0, 1.0);
    const double dark_detail = dark_window * dclamp(dark_avg / 10.0, 0.0, 1.0);
    const double frame_mean = (w == A.P.W && h == A.P.H) ? A.frame_mean : st.mean;
    const double dim_area = dclamp((142.0 - st.mean) / 116.0, 0.0, 1.0);
    const double dim_frame = dclamp((142.0 - frame_mean) / 116.0, 0.0, 1.0);
    const double not_black = dclamp((st.mean - 0.75) / 9.0, 0.0, 1.0);
    const double dim_detail = dmax(dim_area, 0.82 * dim_frame) * not_black * aq_activity(st);
    const int pad = 4;
    const int cx0 = imax(0, x0 - pad), cy0 = imax(0, y0 - pad);
    const int cx1 = imin(w, x0 + bw + pad), cy1 = imin(h, y0 + bh + pad);
    unsigned long long ring_grad = 0;
    int ring_n = 0, ring_edges = 0;
    for (int py = cy0; py < cy1; ++py)
        for (int px = cx0; px < cx1; ++px) {
            if (px >= x0 && px < x0 + bw && py >= y0 && py < y0 + bh) continue;
            const int v = __ldg(plane + (size_t)py * pitch + px);
            if (px > cx0) {
                const int d = iabs(v - (int)__ldg(plane + (size_t)py * pitch + px - 1));
                ring_grad += d;
                if (d >= 64) ++ring_edges;
                ++ring_n;
            }
            if (py > cy0) {
                const int d = iabs(v - (int)__ldg(plane + (size_t)(py - 1) * pitch + px));
                ring_grad += d;
                if (d >= 64) ++ring_edges;
                ++ring_n;
            }
        }
    const double ring_grad_avg = ring_n ? (double)ring_grad / ring_n : 0.0;
    const double ring_edge_density = ring_n ? (double)ring_edges / ring_n : 0.0;
    const double context_activity = dclamp((ring_grad_avg - 10.0) / 36.0, 0.0, 1.0) +
                                    0.8 * dclamp((ring_edge_density - 0.04) / 0.24, 0.0, 1.0);
    const double quietness = dclamp((18.0 - st.grad_avg) / 14.0, 0.0, 1.0);
    const double neutral_window = dclamp((190.0 - st.mean) / 120.0, 0.0, 1.0) * dclamp((st.mean - 6.0) / 30.0, 0.0, 1.0);
    const double adjacency = quietness * neutral_window * dclamp(context_activity, 0.0, 1.5);
    if (adjacency_out) *adjacency_out = adjacency;
    double bright_field_detail = 0.0;
    if ((contrast > 0.15 || edge_density > 0.25) && w == A.P.W && h == A.P.H) {
        const double bright_field = dclamp((frame_mean - 165.0) / 55.0, 0.0, 1.0);
        bright_field_detail = bright_field * dmax(contrast, 0.65 * edge_density);
    }
    const double protect = c.aq_strength * (8.50 * dark_detail + 1.45 * dim_detail + 0.20 * contrast + 0.10 * edge_density +
                                            0.08 * motion + 1.00 * adjacency + 2.00 * bright_field_detail);
    return dclamp(1.0 / (1.0 + protect), 0.18, 1.0);
}

// ---- bit estimates (encoder_entropy.cpp:182-302, encoder_transform.cpp:1344-1553) ---------

__device__ __forceinline__ int ac_direct(const TrdTables* T, int set, int run, int level, bool last) {
    if (run < 0 || run > 63 || level < 0 || level >= 64) return 0;
    return __ldg(&T->ac_bits[set][last ? 1 : 0][run][level]);
}
__device__ __forceinline__ int ac_max_level(const TrdTables* T, int set, int run, bool last) {
    if (run < 0 || run > 63) return 0;
    return __ldg(&T->max_level[set][last ? 1 : 0][run]);
}
__device__ __forceinline__ int ac_max_run(const TrdTables* T, int set, int level, bool last) {
    if (level < 0 || level >= 64) return -1;
    return __ldg(&T->max_run[set][last ? 1 : 0][level]);
}
__device__ __forceinline__ int esc3_level_bits(const DevParams& P) { return P.pq < 8 ? 11 : 8; }

// trellis_rate_bits_for_set (encoder_transform.cpp:1811-1841)
__device__ int rate_for_set(const DevParams& P, const TrdTables* T, int run, int level, bool last, int set) {
    const int mag = iabs(level);
    if (run < 0 || run > 63 || level == 0 || mag > trd_max_level(P)) return 1000000;
    if (const int d = ac_direct(T, set, run, mag, last)) return d + 1;
    const int esc = ent::kAcEscapeBits[set];
    int best = 1000000;
    const int level_delta = ac_max_level(T, set, run, last);
    if (set != 3 && level_delta > 0 && mag > level_delta) {
        if (const int b = ac_direct(T, set, run, mag - level_delta, last)) best = esc + 1 + b + 1;
    }
    const int run_delta = ac_max_run(T, set, mag, last);
    if (run_delta >= 0 && run > run_delta) {
        if (const int b = ac_direct(T, set, run - run_delta - 1, mag, last)) best = imin(best, esc + 2 + b + 1);
    }
    return imin(best, esc + 2 + 1 + 6 + 1 + esc3_level_bits(P));
}

// trellis_rate_bits (:1843-1857): the lower envelope of coding sets 1, 3, 5 (inter family) or
// 0, 2, 4 (intra family)
__device__ int rate_family(const DevParams& P, const TrdTables* T, int run, int level, bool last, bool intra) {
    int bits = 1000000;
    for (int s = intra ? 0 : 1; s <= 5; s += 2) bits = imin(bits, rate_for_set(P, T, run, level, last, s));
    return bits;
}

// write_ac_coeff's length (encoder_entropy.cpp:246-302) with the Escape-3 length header state
__device__ int ac_coeff_bits(const TrdArgs& A, int run, int level, bool last, bool& esc3_written) {
    const DevParams& P = A.P;
    const int set = A.cfg.coding_set;
    const int mag = iabs(level);
    const int esc = ent::kAcEscapeBits[set];
    const int header = (P.pq < 8 || A.cfg.dquantfrm) ? 7 : 8;
    auto esc3 = [&]() {
        const int b = esc + 2 + 1 + (esc3_written ? 0 : header) + 6 + 1 + esc3_level_bits(P);
        esc3_written = true;
        return b;
    };
    if (!A.cfg.use_vlc) return esc3();
    if (const int d = ac_direct(A.tab, set, run, mag, last)) return d + 1;
    int best_bits = 1000000;
    bool have = false;
    const int level_delta = ac_max_level(A.tab, set, run, last);
    if (set != 3 && level_delta > 0 && mag > level_delta) {
        if (const int b = ac_direct(A.tab, set, run, mag - level_delta, last)) {
            best_bits = esc + 1 + b + 1;
            have = true;
        }
    }
    const int run_delta = ac_max_run(A.tab, set, mag, last);
    if (run_delta >= 0 && run > run_delta) {
        if (const int b = ac_direct(A.tab, set, run - run_delta - 1, mag, last)) {
            const int bits = esc + 2 + b + 1;
            if (bits < best_bits) {
                best_bits = bits;
                have = true;
            }
        }
    }
    const int esc3_bits = esc + 2 + 1 + 6 + 1 + esc3_level_bits(P) + (esc3_written ? 0 : header);
    if (have && best_bits < esc3_bits) return best_bits;
    return esc3();
}

__device__ __forceinline__ const uint8_t* inter_scan(int t, int& n) {
    if (t == 1) { n = 64; return ent::kInterScan; }
    if (t == 2) { n = 32; return ent::kInterScan8x4; }
    if (t == 3) { n = 32; return ent::kInterScan4x8; }
    n = 16;
    return ent::kInterScan4x4;
}

// write_inter_scan (:1414-1432) of partition-local levels
__device__ int inter_scan_bits(const TrdArgs& A, const int* q, int t, bool& esc3_written) {
    int n;
    const uint8_t* scan = inter_scan(t, n);
    int last = -1;
    for (int s = n - 1; s >= 0; --s)
        if (q[scan[s]]) { last = s; break; }
    if (last < 0) return 0;
    int bits = 0, previous = -1;
    for (int s = 0; s <= last; ++s) {
        const int level = q[scan[s]];
        if (!level) continue;
        bits += ac_coeff_bits(A, s - previous - 1, level, s == last, esc3_written);
        previous = s;
    }
    return bits;
}

__device__ __forceinline__ int tt_table(const DevParams& P) { return P.pq <= 4 ? 0 : (P.pq <= 12 ? 1 : 2); }
__device__ __forceinline__ int subblkpat_bits(const DevParams& P, int skip) { return ent::kSubblkBits[tt_table(P)][14 - skip]; }
__device__ __forceinline__ int rect_subblkpat_bits(int skip) { return skip == 0 ? 1 : 2; }  // decode012 of 0 / 2 / 1
__device__ int ttblk_bits(const DevParams& P, int t, int skip) {
    int variant;
    if (t == 1) variant = 0;
    else if (t == 4) variant = 7;
    else if (t == 2) variant = skip == 0 ? 1 : (skip == 1 ? 2 : 3);
    else variant = skip == 0 ? 4 : (skip == 1 ? 5 : 6);
    const int tab = tt_table(P);
    int symbol = 0;
    for (int s = 0; s < 8; ++s)
        if (ent::kTtSymbolVariant[tab][s] == variant) { symbol = s; break; }
    return ent::kTtblkBits[tab][symbol];
}
__device__ int ttmb_macro_bits(const DevParams& P, int t, int first_skip) {
    int symbol = 8;
    if (t == 2) symbol = first_skip == 1 ? 10 : (first_skip == 2 ? 9 : 11);
    else if (t == 3) symbol = first_skip == 1 ? 13 : (first_skip == 2 ? 12 : 14);
    else if (t == 4) symbol = 15;
    return ent::kTtmbBits[tt_table(P)][symbol];
}
__device__ int ttmb_block_bits(const DevParams& P, int t, int first_skip) {
    int value;
    if (t == 1) value = 0;
    else if (t == 4) value = 7;
    else if (t == 2) value = first_skip == 0 ? 3 : (first_skip == 1 ? 2 : 1);
    else value = first_skip == 0 ? 6 : (first_skip == 1 ? 5 : 4);
    return ent::kTtmbBits[tt_table(P)][value];
}

// A TransformParentDecision in shared memory
struct TParent {
    int16_t q[64];      // the partitions' levels in their sub-rectangles of the 8x8 grid
    double distortion;
    uint32_t bits;      // estimate_parent_payload_bits
    uint8_t type, skip;
};

__device__ __forceinline__ void load_part(const TParent& p, int t, int part, int* q) {
    int ox, oy, bw, bh;
    part_geometry(t, part, ox, oy, bw, bh);
    for (int i = 0; i < 64; ++i) q[i] = 0;
    for (int y = 0; y < bh; ++y)
        for (int x = 0; x < bw; ++x) q[y * 8 + x] = p.q[(oy + y) * 8 + ox + x];
}

// estimate_parent_payload_bits (:1528-1543)
__device__ uint32_t parent_payload_bits(const TrdArgs& A, const TParent& p) {
    const int np = part_count(p.type);
    const int allmask = (1 << np) - 1;
    if (p.skip == allmask) return 0;
    bool esc = false;
    int bits = 0;
    if (p.type == 4) bits += subblkpat_bits(A.P, p.skip);
    else if (p.type == 2 || p.type == 3) bits += rect_subblkpat_bits(p.skip);
    int q[64];
    for (int part = 0; part < np; ++part) {
        if (p.skip & (1 << (np - 1 - part))) continue;
        load_part(p, p.type, part, q);
        bits += inter_scan_bits(A, q, p.type, esc);
    }
    return (uint32_t)bits;
}

// estimate_ttblk_bits (:1545-1553)
__device__ uint32_t parent_ttblk_bits(const DevParams& P, const TParent& p) {
    const int np = part_count(p.type);
    if (p.skip == (1 << np) - 1) return 0;
    int bits = ttblk_bits(P, p.type, p.skip);
    if (p.type == 4) bits += subblkpat_bits(P, p.skip);
    return (uint32_t)bits;
}

// ---- trellis_quantize (:1873-2088) ---------------------------------------------------------

// trellis_coeff_weight (:1859-1871)
__device__ __forceinline__ double trellis_weight(int t, int index) {
    const double e8[8] = {1152, 1156, 1168, 1156, 1152, 1156, 1168, 1156};
    const double e4[4] = {1156, 1168, 1156, 1168};
    const int row = index / 8, col = index & 7;
    const bool x4 = t == 3 || t == 4, y4 = t == 2 || t == 4;
    const double ex = x4 ? e4[col] : e8[col], ey = y4 ? e4[row] : e8[row];
    return (ex * ey) / (1024.0 * 1024.0);
}

struct TState {
    double distortion, score;
    uint32_t bits;
    int last_scan;
    int from, level;  // the state of the previous position it extends, and this position's level
};

__device__ __forceinline__ bool tstate_less(const TState& a, const TState& b) {
    if (a.score != b.score) return a.score < b.score;
    if (a.bits != b.bits) return a.bits < b.bits;
    return a.distortion < b.distortion;
}

// Levels q (partition-local 8-stride) of coefficients c for transform type t along scan[0..n); the
// trellis decides positions first_scan..n-1 (1 for intra blocks, whose DC is coded apart, leaving
// q[scan[0]] zero) with the rates of the intra or inter family. The beam's paths are kept as
// back-pointers per scan position (the state each survivor extends, its level there).
__device__ void trellis_quantize(const TrdArgs& A, const double* c, int t, double lambda_scale, int mquant, int* q,
                                 const uint8_t* scan, int n, int first_scan, bool intra) {
    const DevParams& P = A.P;
    const bool derived = mquant != P.pq;
    const double qscale = (double)trd_double_quant(P, mquant, derived);
    const int max_level = trd_max_level(P);
    int scalar[64];
    for (int i = 0; i < 64; ++i) scalar[i] = 0;
    for (int s = 0; s < n; ++s) scalar[scan[s]] = trd_squant(P, c[scan[s]], mquant, derived);
    for (int i = 0; i < 64; ++i) q[i] = scalar[i];
    if (A.cfg.trellis <= 0 || (A.cfg.hrd_enabled && mquant == 1)) return;
    const int beam = A.cfg.trellis >= 2 ? 8 : 4;
    const double lambda = 0.15 * qscale * qscale * dclamp(lambda_scale, 0.20, 1.50);
    uint16_t bp[64][8];  // back-pointer: from state (3 bits) | level + 4096 (13 bits)
    TState states[8];
    int count = 1;
    states[0] = TState{0.0, 0.0, 0u, first_scan - 1, -1, 0};
    for (int s = first_scan; s < n; ++s) {
        const int idx = scan[s];
        const int q0 = scalar[idx];
        int cand[4], nc = 0;
        auto add = [&](int v) {
            v = iclamp(v, -max_level, max_level);
            for (int i = 0; i < nc; ++i)
                if (cand[i] == v) return;
            cand[nc++] = v;
        };
        add(0);
        if (q0 != 0) {
            const int sign = q0 > 0 ? 1 : -1;
            add(q0);
            add(q0 - sign);
            if (A.cfg.trellis >= 2) add(q0 + sign);
        }
        double cd[4];
        for (int ci = 0; ci < nc; ++ci) {
            const double e = c[idx] - (double)trd_dequant(P, cand[ci], mquant, derived);
            cd[ci] = e * e * trellis_weight(t, idx);
        }
        TState next[32];
        int nn = 0;
        for (int si = 0; si < count; ++si) {
            const TState& st = states[si];
            for (int ci = 0; ci < nc; ++ci) {
                const int level = cand[ci];
                TState ns = st;
                ns.distortion += cd[ci];
                ns.from = si;
                ns.level = level;
                if (level != 0) {
                    const int rb = rate_family(P, A.tab, s - st.last_scan - 1, level, false, intra);
                    if (rb >= 1000000) continue;
                    ns.bits += (uint32_t)rb;
                    ns.last_scan = s;
                }
                ns.score = ns.distortion + lambda * (double)ns.bits;
                next[nn++] = ns;
            }
        }
        for (int i = 1; i < nn; ++i) {
            const TState key = next[i];
            int j = i;
            while (j > 0 && tstate_less(key, next[j - 1])) {
                next[j] = next[j - 1];
                --j;
            }
            next[j] = key;
        }
        count = imin(nn, beam);
        for (int i = 0; i < count; ++i) {
            states[i] = next[i];
            bp[s][i] = (uint16_t)((next[i].from << 13) | (next[i].level + 4096));
        }
    }
    // the exact rate of each survivor (its last coefficient coded as last), then the least D + lambda R
    int best = 0;
    double best_rd = __longlong_as_double(0x7ff0000000000000LL);  // +infinity
    for (int si = 0; si < count; ++si) {
        uint32_t bits = 0;
        int next_pos = -1, next_level = 0;  // the coefficient after this one on the path (towards the end)
        int j = si;
        bool first = true;
        for (int s = n - 1; s >= first_scan; --s) {
            const int level = (int)(bp[s][j] & 0x1FFF) - 4096;
            const int from = bp[s][j] >> 13;
            if (level != 0) {
                if (next_pos >= 0)
                    bits += (uint32_t)rate_family(P, A.tab, next_pos - s - 1, next_level, first, intra);
                if (next_pos >= 0) first = false;
                next_pos = s;
                next_level = level;
            }
            j = from;
        }
        if (next_pos >= 0) bits += (uint32_t)rate_family(P, A.tab, next_pos - first_scan, next_level, first, intra);
        const double rd = states[si].distortion + lambda * (double)bits;
        if (rd < best_rd) {
            best = si;
            best_rd = rd;
        }
    }
    for (int i = 0; i < 64; ++i) q[i] = 0;
    int j = best;
    for (int s = n - 1; s >= first_scan; --s) {
        const int level = (int)(bp[s][j] & 0x1FFF) - 4096;
        if (level != 0) q[scan[s]] = level;
        j = bp[s][j] >> 13;
    }
}

// ---- evaluate_transform_parent (:1555-1590) --------------------------------------------------

__device__ void eval_parent(const TrdArgs& A, int mx, int my, int k, int t, bool allow_trellis, int mquant, TParent& out) {
    const DevParams& P = A.P;
    const bool chroma = k >= 4;
    const uint8_t* sp = chroma ? (k == 4 ? A.src.u : A.src.v) : A.src.y;
    const uint8_t* pp = chroma ? (k == 4 ? A.pred.u : A.pred.v) : A.pred.y;
    const int spitch = chroma ? A.src.pitch_c : A.src.pitch_y, ppitch = chroma ? A.pred.pitch_c : A.pred.pitch_y;
    const int w = chroma ? P.W / 2 : P.W, h = chroma ? P.H / 2 : P.H;
    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
    const bool derived = mquant != P.pq;
    out.type = (uint8_t)t;
    out.skip = 0;
    for (int i = 0; i < 64; ++i) out.q[i] = 0;
    int residual[64];
    for (int i = 0; i < 64; ++i) residual[i] = 0;
    const int np = part_count(t);
    for (int part = 0; part < np; ++part) {
        int ox, oy, bw, bh;
        part_geometry(t, part, ox, oy, bw, bh);
        const int x0 = bx * 8 + ox, y0 = by * 8 + oy;
        int q[64];
        for (int i = 0; i < 64; ++i) q[i] = 0;
        // quantize_inter_part (:1087-1171): nothing to code for a partition outside the crop
        if (!(x0 >= w || y0 >= h || x0 + bw <= 0 || y0 + bh <= 0)) {
            double c[64];
            trd_forward(sp, spitch, pp, ppitch, w, h, x0, y0, bw, bh, c);
            if (allow_trellis && A.cfg.trellis > 0) {
                const double ls = aq_scale(A, sp, spitch, w, h, x0, y0, bw, bh, pp, ppitch, chroma ? A.src.y : nullptr,
                                           A.src.pitch_y);
                int n;
                const uint8_t* scan = inter_scan(t, n);
                trellis_quantize(A, c, t, ls, mquant, q, scan, n, 0, false);
            } else {
                for (int y = 0; y < bh; ++y)
                    for (int x = 0; x < bw; ++x) q[y * 8 + x] = trd_squant(P, c[y * 8 + x], mquant, derived);
            }
        }
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) out.q[(oy + y) * 8 + ox + x] = (int16_t)q[y * 8 + x];
        bool any = false;
        for (int i = 0; i < 64; ++i) any |= q[i] != 0;
        if (!any) {
            out.skip |= (uint8_t)(1 << (np - 1 - part));
            continue;
        }
        int r[64];
        trd_inverse(P, t, q, mquant, A.cfg.dquantfrm != 0, r);  // the reference passes DQUANTFRM here
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) residual[(oy + y) * 8 + ox + x] = r[y * 8 + x];
    }
    unsigned long long sse = 0;
    for (int y = 0; y < 8 && by * 8 + y < h; ++y)
        for (int x = 0; x < 8 && bx * 8 + x < w; ++x) {
            const int px = bx * 8 + x, py = by * 8 + y;
            const int recon = iclamp((int)__ldg(pp + (size_t)py * ppitch + px) + residual[y * 8 + x], 0, 255);
            const int e = (int)__ldg(sp + (size_t)py * spitch + px) - recon;
            sse += (unsigned long long)(e * e);
        }
    out.distortion = (double)sse;
    out.bits = parent_payload_bits(A, out);
}

// An MbTransformDecision: parents by index into the warp's parent pool
struct TDec {
    int8_t parent[6];
    uint8_t type, level, cbp;
    double distortion;
    uint32_t bits;
};

// refresh_transform_estimate (:1496-1526) with write_transform_payload (:1434-1494)
__device__ void refresh(const TrdArgs& A, TDec& d, const TParent* pool) {
    const DevParams& P = A.P;
    d.cbp = 0;
    d.distortion = 0.0;
    int first = -1;
    for (int k = 0; k < 6; ++k) {
        const TParent& p = pool[d.parent[k]];
        d.distortion += p.distortion;
        const int np = part_count(p.type);
        if (p.skip != (1 << np) - 1) {
            d.cbp |= (uint8_t)(1 << (5 - k));
            if (first < 0) first = k;
        }
    }
    if (first >= 0 && d.level == 1) d.type = pool[d.parent[first]].type;
    d.bits = 0;
    if (!d.cbp) return;
    int bits = ent::kPcbpBits[d.cbp];
    bool esc = false;
    int q[64];
    if (!A.cfg.variable_transforms) {
        for (int k = 0; k < 6; ++k) {
            if (!(d.cbp & (1 << (5 - k)))) continue;
            load_part(pool[d.parent[k]], 1, 0, q);
            bits += inter_scan_bits(A, q, 1, esc);
        }
        d.bits = (uint32_t)bits;
        return;
    }
    const TParent& fp = pool[d.parent[first]];
    if (d.level == 0) bits += ttmb_macro_bits(P, d.type, fp.skip);
    else if (d.level == 1) bits += ttmb_block_bits(P, fp.type, fp.skip);
    for (int k = 0; k < 6; ++k) {
        if (!(d.cbp & (1 << (5 - k)))) continue;
        const TParent& p = pool[d.parent[k]];
        const int t = p.type;
        if (d.level == 1) {
            if (k != first) bits += ttblk_bits(P, t, p.skip);
            if (t == 4) bits += subblkpat_bits(P, p.skip);
        } else if (d.level == 0) {
            if (t == 4) bits += subblkpat_bits(P, p.skip);
            else if ((t == 2 || t == 3) && k != first) bits += rect_subblkpat_bits(p.skip);
        } else {
            if (t == 4) bits += subblkpat_bits(P, p.skip);
            else if (t == 2 || t == 3) bits += rect_subblkpat_bits(p.skip);
        }
        const int np = part_count(t);
        for (int part = 0; part < np; ++part) {
            if (p.skip & (1 << (np - 1 - part))) continue;
            load_part(p, t, part, q);
            bits += inter_scan_bits(A, q, t, esc);
        }
    }
    d.bits = (uint32_t)bits;
}

__device__ __forceinline__ double rd_of(const TDec& d, double lambda) { return d.distortion + lambda * (double)d.bits; }

constexpr int kTrdWarps = 4;
constexpr int kTrdPool = 36;  // 24 candidate parents, 6 trellis macro parents, 6 trellis block parents

__global__ void __launch_bounds__(32 * kTrdWarps) trd_kernel(const __grid_constant__ TrdArgs A) {
    __shared__ TParent pool_all[kTrdWarps][kTrdPool];
    __shared__ int list_all[kTrdWarps][8];  // [0..3] candidate types, [4] count, [5] macro type, [6..] scratch
    __shared__ uint8_t need_all[kTrdWarps][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * kTrdWarps + warp;
    const DevParams& P = A.P;
    if (item >= (A.mb_list ? A.n_list : P.mbw * P.mbh)) return;
    const int mb = A.mb_list ? A.mb_list[item] : item;
    TParent* pool = pool_all[warp];
    int* list = list_all[warp];
    uint8_t* need = need_all[warp];
    const int mx = mb % P.mbw, my = mb / P.mbw;
    const int mquant = (A.mquant && A.mquant[mb] >= 1) ? (int)A.mquant[mb] : P.pq;
    const vc1cu_trd_cfg& cfg = A.cfg;
    // ---- the candidate list ----
    if (!cfg.variable_transforms || cfg.frame_type) {
        if (lane == 0) {
            list[0] = cfg.variable_transforms ? cfg.frame_type : 1;
            list[4] = 1;
        }
    } else {
        // transform_metrics (transform_residual_metrics.h:29-61), each lane half a row
        const int py = lane >> 1, px0 = (lane & 1) * 8;
        uint32_t sad = 0, hedge = 0, vedge = 0, grad = 0;
        const int y = my * 16 + py;
        if (y < P.H) {
            auto R = [&](int xx, int yy) {
                return (int)A.src.y[(size_t)yy * A.src.pitch_y + xx] - (int)A.pred.y[(size_t)yy * A.pred.pitch_y + xx];
            };
            for (int px = px0; px < px0 + 8 && mx * 16 + px < P.W; ++px) {
                const int x = mx * 16 + px;
                const int r = R(x, y);
                sad += (uint32_t)iabs(r);
                if ((py & 7) == 4) hedge += (uint32_t)iabs(r - R(x, y - 1));
                if ((px & 7) == 4) vedge += (uint32_t)iabs(r - R(x - 1, y));
                if (px > 0) grad += (uint32_t)iabs(r - R(x - 1, y));
                if (py > 0) grad += (uint32_t)iabs(r - R(x, y - 1));
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            sad += __shfl_xor_sync(0xffffffffu, sad, o);
            hedge += __shfl_xor_sync(0xffffffffu, hedge, o);
            vedge += __shfl_xor_sync(0xffffffffu, vedge, o);
            grad += __shfl_xor_sync(0xffffffffu, grad, o);
        }
        if (lane == 0) {
            const uint64_t S = sad, HE = hedge, VE = vedge, G = grad, lim = (uint64_t)(64 * mquant);
            int l[4] = {1, 1, 1, 1}, count = 0;
            const bool split_x = mx == P.mbw - 1 && (P.W & 15) != 0, split_y = my == P.mbh - 1 && (P.H & 15) != 0;
            if (split_x && split_y) {
                l[count++] = 4;
            } else if (split_x || split_y) {
                l[count++] = split_x ? 3 : 2;
                if (S > lim && G > S * 2) l[count++] = 4;
            } else {
                l[count++] = 1;
                if (S > lim) {
                    if (HE * 5 > VE * 6) l[count++] = 2;
                    else if (VE * 5 > HE * 6) l[count++] = 3;
                    else { l[count++] = 2; l[count++] = 3; }
                    if (count < 4 && G > S * 2) l[count++] = 4;
                }
            }
            for (int i = 0; i < 4; ++i) list[i] = l[i];
            list[4] = count;
        }
    }
    __syncwarp();
    const int count = list[4];
    // candidates whose decision is final at once: the 8x8-only and frame-level forms (with trellis)
    const bool direct = !cfg.variable_transforms || cfg.frame_type;
    const bool scalar_search = cfg.trellis > 0;
    // ---- every candidate's six parents, one per lane ----
    if (lane < count * 6) {
        const int i = lane / 6, k = lane % 6;
        eval_parent(A, mx, my, k, list[i], direct ? true : !scalar_search, mquant, pool[i * 6 + k]);
    }
    __syncwarp();
    TDec macro{}, block{};
    double lambda = 0.0;
    if (lane == 0) {
        if (direct) {
            for (int k = 0; k < 6; ++k) macro.parent[k] = (int8_t)k;
            macro.type = (uint8_t)list[0];
            macro.level = cfg.variable_transforms ? 2 : 0;
            refresh(A, macro, pool);
        } else {
            TDec cand[4];
            for (int i = 0; i < count; ++i) {
                for (int k = 0; k < 6; ++k) cand[i].parent[k] = (int8_t)(i * 6 + k);
                cand[i].type = (uint8_t)list[i];
                cand[i].level = 0;
                refresh(A, cand[i], pool);
            }
            const double mb_lscale = aq_scale(A, A.src.y, A.src.pitch_y, P.W, P.H, mx * 16, my * 16, 16, 16, A.pred.y,
                                              A.pred.pitch_y, nullptr, 0);
            lambda = 0.75 * (double)(2 * mquant) * (double)(2 * mquant) * mb_lscale;
            int best_i = 0;
            double best_rd = rd_of(cand[0], lambda);
            for (int i = 1; i < count; ++i) {
                const double r = rd_of(cand[i], lambda);
                if (r < best_rd) {
                    best_rd = r;
                    best_i = i;
                }
            }
            block = cand[0];
            block.level = 1;
            for (int k = 0; k < 6; ++k) {
                int bi = 0;
                auto prd = [&](const TParent& p) {
                    return p.distortion + lambda * (double)(p.bits + parent_ttblk_bits(P, p));
                };
                double brd = prd(pool[cand[0].parent[k]]);
                for (int i = 1; i < count; ++i) {
                    const double r = prd(pool[cand[i].parent[k]]);
                    if (r < brd) {
                        brd = r;
                        bi = i;
                    }
                }
                block.parent[k] = cand[bi].parent[k];
            }
            refresh(A, block, pool);
            macro = cand[best_i];
            list[5] = macro.type;
            for (int k = 0; k < 6; ++k) need[k] = pool[block.parent[k]].type;
        }
    }
    __syncwarp();
    // ---- trellis re-evaluation of the macroblock winner and of the block winners of other types ----
    if (!direct && cfg.trellis > 0) {
        const int mt = list[5];
        if (lane < 6) eval_parent(A, mx, my, lane, mt, true, mquant, pool[24 + lane]);
        else if (lane < 12 && need[lane - 6] != mt) eval_parent(A, mx, my, lane - 6, need[lane - 6], true, mquant, pool[30 + lane - 6]);
        __syncwarp();
        if (lane == 0) {
            const uint8_t mtype = macro.type;
            for (int k = 0; k < 6; ++k) macro.parent[k] = (int8_t)(24 + k);
            macro.level = 0;
            refresh(A, macro, pool);
            for (int k = 0; k < 6; ++k) block.parent[k] = (int8_t)(need[k] == mtype ? 24 + k : 30 + k);
            block.level = 1;
            refresh(A, block, pool);
        }
    }
    __syncwarp();
    // ---- the signaling decision and the outputs ----
    __shared__ int chosen_all[kTrdWarps][6];
    if (lane == 0) {
        TDec d = macro;
        if (!direct && cfg.extended_transform_signaling && rd_of(block, lambda) < rd_of(macro, lambda) * 0.9999) d = block;
        vc1cu_tdecision o{};
        o.type = d.type;
        o.signal_level = d.level;
        o.cbp = d.cbp;
        o.estimated_bits = d.bits;
        o.distortion = d.distortion;
        for (int k = 0; k < 6; ++k) {
            const TParent& p = pool[d.parent[k]];
            o.parent_type[k] = p.type;
            o.skip_mask[k] = p.skip;
            o.parent_bits[k] = p.bits;
            o.parent_distortion[k] = p.distortion;
            chosen_all[warp][k] = d.parent[k];
        }
        A.out[item] = o;
    }
    __syncwarp();
    if (A.levels)
        for (int i = lane; i < 6 * 64; i += 32)
            A.levels[(size_t)item * 384 + i] = pool[chosen_all[warp][i >> 6]].q[i & 63];
}

// ---- I-picture intra reconstruction (reconstruct_i_signed_padded, encoder_encode.cpp:814-887) ----

// dc_scale (encoder_entropy.cpp:369-375): the DC step of MQUANT 1..31
__device__ __forceinline__ int intra_dc_scale(int q) {
    return q <= 0 ? 0 : (q == 1 ? 2 : (q == 2 ? 4 : (q <= 5 ? 8 : q / 2 + 6)));
}
// DQScale (SMPTE 421M 8.1.3.4, dqscale_value :434-447): round(2^18 / n) for n = index + 1
__device__ __forceinline__ int intra_dqscale(int index) {
    const int n = index + 1;
    return (0x40000 + n / 2) / n;
}
// reconstruct_dc_sample_with_bias (:383-389)
__device__ __forceinline__ int intra_dc_sample(int qdc, int mq, int bias) {
    int x = qdc * intra_dc_scale(mq);
    x = arshift(3 * x + 1, 1);
    x = arshift(3 * x + 16, 5);
    return min(255, max(0, bias + x));
}
// choose_dc_for_mean_with_bias (:395-412): the DC level whose reconstruction is nearest the mean
__device__ int intra_dc_for_mean(int mean, int mq, int bias) {
    const int bits = 8 + ((mq == 1 || mq == 2) ? 3 - mq : 0);
    const int maxq = (1 << bits) - 1;
    int lo = -maxq, hi = maxq;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (intra_dc_sample(mid, mq, bias) < mean) lo = mid + 1;
        else hi = mid;
    }
    int best = lo;
    if (lo > -maxq && iabs(intra_dc_sample(lo - 1, mq, bias) - mean) <= iabs(intra_dc_sample(lo, mq, bias) - mean)) best = lo - 1;
    return best;
}
// scale_dc_predictor (:449-456)
__device__ __forceinline__ int intra_scale_dc(int value, int from_q, int to_q) {
    from_q = iabs(from_q);
    to_q = iabs(to_q);
    if (!from_q || from_q == to_q) return value;
    const int idx = intra_dc_scale(to_q) - 1;
    if (idx < 0) return 0;
    const long long v = (long long)value * intra_dc_scale(from_q) * intra_dqscale(idx);
    return (int)((v + 0x20000) >> 18);
}

// The intra source, its MQUANT map and the per-block outputs of one I picture.
struct IntraArgs {
    DevParams P;
    const uint8_t* y;
    const uint8_t* u;
    const uint8_t* v;
    int pitch_y, pitch_c, sw, sh;  // the intra source's luma raster (the picture or its edge source)
    const uint8_t* mquant;         // per MB (nullptr: PQINDEX)
    const uint8_t* derived;        // per MB DQUANT-derived flag (nullptr: none)
    int16_t* q;                    // [mb][6][64] AC levels
    int* dc[3];                    // per plane block grid: the DC target, then the final DC
    int* qg[3];                    // per plane block grid: MQUANT, negative when derived
    TrdArgs trd;                   // P, tab, cfg (trellis, hrd_enabled, AQ) and the intra source's luma mean
};

__device__ __forceinline__ int intra_mq(const IntraArgs& A, int mb) {
    return (A.mquant && A.mquant[mb] >= 1) ? (int)A.mquant[mb] : A.P.pq;
}

// One thread per (MB, block): forward_transform (:672-795; samples outside the source read the
// pad value, 0 luma / 128 chroma, minus 128), the AC levels of quantize_ac (:2090-2144: scalar, or
// the trellis along the intra scan from position 1 with the intra-family rates and the perceptual
// lambda scale of the block, chroma weighed against the intra source's luma) and
// choose_dc_for_mean of the padded block mean.
__global__ void intra_fwd_kernel(const __grid_constant__ IntraArgs A) {
    const DevParams& P = A.P;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.mbw * P.mbh * 6) return;
    const int mb = i / 6, k = i % 6, mx = mb % P.mbw, my = mb / P.mbw;
    const bool chroma = k >= 4;
    const uint8_t* p = chroma ? (k == 4 ? A.u : A.v) : A.y;
    const int pitch = chroma ? A.pitch_c : A.pitch_y, w = chroma ? A.sw / 2 : A.sw, h = chroma ? A.sh / 2 : A.sh;
    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
    const int x0 = bx * 8, y0 = by * 8, pad = chroma ? 128 : 0;
    const int mq = intra_mq(A, mb);
    const bool derived = A.derived && A.derived[mb];
    int r[8][8];
    unsigned sum = 0;
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
            const int sx = x0 + x, sy = y0 + y;
            const int v = (sx < w && sy < h) ? (int)__ldg(p + (size_t)sy * pitch + sx) : pad;
            sum += (unsigned)v;
            r[y][x] = v - 128;
        }
    double tmp[8][8];
    for (int a = 0; a < 8; ++a)
        for (int x = 0; x < 8; ++x) {
            double acc = 0.0;
            for (int y = 0; y < 8; ++y) acc = __dadd_rn(acc, __dmul_rn(c_k8[a][y], (double)r[y][x]));
            tmp[a][x] = acc;
        }
    int16_t* q = A.q + (size_t)i * 64;
    q[0] = 0;
    const bool trellis = A.trd.cfg.trellis > 0 && !(A.trd.cfg.hrd_enabled && mq == 1);
    double c[64];
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            if (!a && !b) continue;
            double acc = 0.0;
            for (int x = 0; x < 8; ++x) acc = __dadd_rn(acc, __dmul_rn(tmp[a][x], c_k8[b][x]));
            c[b * 8 + a] = __dmul_rn(1024.0, acc);  // c[row*8+col] = xform[col][row]
            if (!trellis) q[b * 8 + a] = (int16_t)trd_squant(P, c[b * 8 + a], mq, derived);
        }
    if (trellis) {
        c[0] = 0.0;  // the DC stays out of the trellis (first_scan 1)
        // the luma context is read as a coded-width raster (stats(*luma_context, width, height, ...)):
        // an edge source of a cropped picture is a padded-width raster read at the coded width
        const int lpitch = A.sw == P.W ? A.pitch_y : P.W;
        const double ls = aq_scale(A.trd, p, pitch, w, h, x0, y0, 8, 8, nullptr, 0, chroma ? A.y : nullptr, lpitch);
        int lv[64];
        trellis_quantize(A.trd, c, 1, ls, mq, lv, ent::kIntraScan, 64, 1, !chroma);
        for (int j = 1; j < 64; ++j) q[j] = (int16_t)lv[j];
    }
    const int gw = chroma ? P.mbw : P.mbw * 2;
    A.dc[chroma ? k - 3 : 0][by * gw + bx] = intra_dc_for_mean((int)((sum + 32u) / 64u), mq, 128);
}

// predict_dc_dquant + clamp_dc_target_for_diff (encoder_entropy.cpp:549-571, :426-432) along the
// block grid of plane blockIdx.x (0 luma, 1 U, 2 V): a block's prediction reads its left, top
// and top-left neighbours' final DC, so the grid is walked by anti-diagonals.
__global__ void intra_dc_kernel(const __grid_constant__ IntraArgs A) {
    const DevParams& P = A.P;
    const int pl = blockIdx.x;
    const int gw = pl ? P.mbw : P.mbw * 2, gh = pl ? P.mbh : P.mbh * 2;
    int* g = A.dc[pl];
    int* qg = A.qg[pl];
    for (int d = 0; d < gw + gh - 1; ++d) {
        for (int y = max(0, d - gw + 1) + (int)threadIdx.x; y <= min(d, gh - 1); y += blockDim.x) {
            const int x = d - y;
            const int mb = pl ? y * P.mbw + x : (y >> 1) * P.mbw + (x >> 1);
            const int mq = intra_mq(A, mb);
            const bool a_avail = y > 0, c_avail = x > 0;
            int a = 0, b = 0, c = 0;
            if (a_avail) a = intra_scale_dc(g[(y - 1) * gw + x], qg[(y - 1) * gw + x], mq);
            if (c_avail) c = intra_scale_dc(g[y * gw + x - 1], qg[y * gw + x - 1], mq);
            if (a_avail && c_avail) b = intra_scale_dc(g[(y - 1) * gw + x - 1], qg[(y - 1) * gw + x - 1], mq);
            const bool left = c_avail && (!a_avail || iabs(a - b) <= iabs(b - c));
            const int pred = left ? c : (a_avail ? a : 0);
            const int bits = 8 + ((mq == 1 || mq == 2) ? 3 - mq : 0);
            const int maxv = (1 << bits) - 1;
            const int diff = min(maxv, max(-maxv, g[y * gw + x] - pred));
            g[y * gw + x] = min(maxv, max(-maxv, pred + diff));
            qg[y * gw + x] = (A.derived && A.derived[mb]) ? -mq : mq;
        }
        __syncthreads();
    }
}

// One thread per (MB, block): the coefficients (DC * dc_scale, dequant_level of the AC levels),
// inverse_transform_8x8 and the signed samples into the padded raster (rows packed).
__global__ void intra_inv_kernel(const __grid_constant__ IntraArgs A, int32_t* oy, int32_t* ou, int32_t* ov) {
    const DevParams& P = A.P;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.mbw * P.mbh * 6) return;
    const int mb = i / 6, k = i % 6, mx = mb % P.mbw, my = mb / P.mbw;
    const bool chroma = k >= 4;
    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
    const int gw = chroma ? P.mbw : P.mbw * 2;
    const int mq = intra_mq(A, mb);
    const bool derived = A.derived && A.derived[mb];
    const int16_t* q = A.q + (size_t)i * 64;
    int a[64], tmp[64];
    a[0] = A.dc[chroma ? k - 3 : 0][by * gw + bx] * intra_dc_scale(mq);
    for (int j = 1; j < 64; ++j) a[j] = trd_dequant(P, q[j], mq, derived);
    for (int j = 0; j < 64; ++j) tmp[j] = 0;
    for (int col = 0; col < 8; ++col) inv8(a + col, 8, tmp + col * 8, 1, 4, 3, 0);
    for (int col = 0; col < 8; ++col) inv8(tmp + col, 8, a + col, 8, 64, 7, 1);
    int32_t* o = chroma ? (k == 4 ? ou : ov) : oy;
    const int ow = chroma ? P.mbw * 8 : P.mbw * 16;
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) o[(size_t)(by * 8 + y) * ow + bx * 8 + x] = a[y * 8 + x];
}

// make_overlap_edge_source (encoder_encode.cpp:13-63): the picture on the coded (whole-MB)
// raster with the samples beyond the visible crop replaced by the nearest visible sample along an
// active overlap edge (all edges, or those between two flagged macroblocks). One thread per
// destination sample of one plane (blockIdx.y).
__host__ __device__ inline int ovl_border(int visible, int coded) {
    if (visible < 1 || visible >= coded) return -1;
    const int rem = visible & 7;
    const int edge = rem == 7 ? visible + 1 : (rem == 0 ? visible : (rem == 1 ? visible - 1 : -1));
    return edge > 0 && edge < coded ? edge : -1;
}

struct EdgeArgs {
    const uint8_t* in[3];
    int in_pitch[3], sw[3], sh[3];
    uint8_t* out[3];
    int out_pitch[3], dw[3], dh[3], vw[3], vh[3], ex[3], ey[3];
    const uint8_t* flags;
    int all, mbw, mbh;
};

__global__ void edge_source_kernel(const __grid_constant__ EdgeArgs E) {
    const int pl = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E.dw[pl] * E.dh[pl]) return;
    const int x = i % E.dw[pl], y = i / E.dw[pl];
    const bool luma = pl == 0;
    const int vw = E.vw[pl], vh = E.vh[pl];
    int v = (x < E.sw[pl] && y < E.sh[pl]) ? (int)E.in[pl][(size_t)y * E.in_pitch[pl] + x] : (luma ? 0 : 128);
    if (!(x < vw && y < vh)) {
        auto active = [&](int ax, int ay, int bx2, int by2) {
            if (E.all) return true;
            const int a = (luma ? ay / 2 : ay) * E.mbw + (luma ? ax / 2 : ax);
            const int b = (luma ? by2 / 2 : by2) * E.mbw + (luma ? bx2 / 2 : bx2);
            const int n = E.mbw * E.mbh;
            return a >= 0 && b >= 0 && a < n && b < n && E.flags[a] && E.flags[b];
        };
        const int ex = E.ex[pl], ey = E.ey[pl];
        const bool right = x >= vw && ex >= 0 && active(ex / 8 - 1, y / 8, ex / 8, y / 8);
        const bool bottom = y >= vh && ey >= 0 && active(x / 8, ey / 8 - 1, x / 8, ey / 8);
        if (right || bottom) {
            const int sx = min(max(x, 0), vw - 1), sy = min(max(y, 0), vh - 1);
            v = E.in[pl][(size_t)sy * E.in_pitch[pl] + sx];
        }
    }
    E.out[pl][(size_t)y * E.out_pitch[pl] + x] = (uint8_t)v;
}

// The DQUANT search's per-macroblock inputs (choose_dquant_transform_mb, encoder_aq.cpp:318-336):
// the perceptual lambda scale of the MB's luma against its prediction with its adjacency term,
// and the bright-detail-on-dark test of the source MB. One thread per MB.
__global__ void dquant_stats_kernel(const __grid_constant__ TrdArgs A, double* lscale, double* adjacency, uint8_t* bright) {
    const DevParams& P = A.P;
    const int mb = blockIdx.x * blockDim.x + threadIdx.x;
    if (mb >= P.mbw * P.mbh) return;
    const int x0 = (mb % P.mbw) * 16, y0 = (mb / P.mbw) * 16;
    double adj = 0.0;
    lscale[mb] = aq_scale(A, A.src.y, A.src.pitch_y, P.W, P.H, x0, y0, 16, 16, A.pred.y, A.pred.pitch_y, nullptr, 0, &adj);
    adjacency[mb] = adj;
    unsigned long long sum = 0;
    int n = 0, hi = 0, lo = 0;
    for (int y = 0; y < 16 && y0 + y < P.H; ++y)
        for (int x = 0; x < 16 && x0 + x < P.W; ++x) {
            const int v = A.src.y[(size_t)(y0 + y) * A.src.pitch_y + x0 + x];
            sum += (unsigned long long)v;
            ++n;
            hi += v >= 180;
            lo += v <= 48;
        }
    const double mean = n ? (double)sum / n : 128.0;
    bright[mb] = (n && mean < 90.0 && hi >= imax(2, n / 32) && lo >= n / 2) ? 1 : 0;
}

// mean of the source luma plane (cached_luma_mean, encoder_aq.cpp:506-545): one block's partial sums
__global__ void luma_sum_kernel(const uint8_t* y, int pitch, int W, int H, unsigned long long* sum) {
    unsigned long long s = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)W * H; i += (long)gridDim.x * blockDim.x)
        s += y[(size_t)(i / W) * pitch + i % W];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

}  // namespace

// The dense rate tables from the code lengths (host side).
size_t trd_tables_bytes() { return sizeof(TrdTables); }
void trd_fill_tables(void* host) {
    TrdTables& t = *static_cast<TrdTables*>(host);
    std::memset(&t, 0, sizeof t);
    std::memset(t.max_run, -1, sizeof t.max_run);
    for (int i = 0; i < ent::kAcEntries; ++i) {
        const uint8_t* e = ent::kAcEntry[i];
        const int set = e[0], run = e[1], level = e[2], last = e[3], bits = e[4];
        t.ac_bits[set][last][run][level] = (uint8_t)bits;
        if (level > t.max_level[set][last][run]) t.max_level[set][last][run] = (uint8_t)level;
        if (run > t.max_run[set][last][level]) t.max_run[set][last][level] = (int8_t)run;
    }
}

// The source luma mean the perceptual lambda scale reads (0 when the scale is off).
static cudaError_t frame_mean_for(const DevParams& P, const DevFrame& src, const vc1cu_trd_cfg& cfg,
                                  unsigned long long* d_sum, cudaStream_t s, double& mean) {
    mean = 0.0;
    if (!cfg.adaptive_quality || cfg.aq_strength <= 0.0 || P.W <= 0 || P.H <= 0) return cudaSuccess;
    cudaError_t e;
    unsigned long long sum = 0;
    if ((e = cudaMemsetAsync(d_sum, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
    luma_sum_kernel<<<148, 256, 0, s>>>(src.y, src.pitch_y, P.W, P.H, d_sum);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(&sum, d_sum, sizeof sum, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    mean = (double)sum / (double)((size_t)P.W * P.H);
    return cudaSuccess;
}

cudaError_t launch_trd(const DevParams& P, const DevFrame& src, const DevFrame& pred, const void* tables,
                       const uint8_t* mquant, const vc1cu_trd_cfg& cfg, unsigned long long* d_sum, vc1cu_tdecision* out,
                       int16_t* levels, cudaStream_t s, const int* mb_list, int n_list, double frame_mean) {
    cudaError_t e;
    if (frame_mean < 0.0 && (e = frame_mean_for(P, src, cfg, d_sum, s, frame_mean)) != cudaSuccess) return e;
    TrdArgs a;
    a.P = P;
    a.src = src;
    a.pred = pred;
    a.tab = static_cast<const TrdTables*>(tables);
    a.mquant = mquant;
    a.cfg = cfg;
    a.frame_mean = frame_mean < 0.0 ? 0.0 : frame_mean;
    a.out = out;
    a.levels = levels;
    a.mb_list = mb_list;
    a.n_list = n_list;
    const int items = mb_list ? n_list : P.mbw * P.mbh;
    if (items <= 0) return cudaSuccess;
    trd_kernel<<<(items + kTrdWarps - 1) / kTrdWarps, 32 * kTrdWarps, 0, s>>>(a);
    return cudaGetLastError();
}

// The source luma mean of the perceptual lambda scale (for launches that share it).
cudaError_t trd_frame_mean(const DevParams& P, const DevFrame& src, const vc1cu_trd_cfg& cfg, unsigned long long* d_sum,
                           cudaStream_t s, double* mean) {
    return frame_mean_for(P, src, cfg, d_sum, s, *mean);
}

// The DQUANT search's per-MB scale, adjacency and bright-on-dark flags.
cudaError_t launch_dquant_stats(const DevParams& P, const DevFrame& src, const DevFrame& pred, const vc1cu_trd_cfg& cfg,
                                double frame_mean, double* lscale, double* adjacency, uint8_t* bright, cudaStream_t s) {
    TrdArgs a{};
    a.P = P;
    a.src = src;
    a.pred = pred;
    a.cfg = cfg;
    a.frame_mean = frame_mean;
    const int mbs = P.mbw * P.mbh;
    if (mbs <= 0) return cudaSuccess;
    dquant_stats_kernel<<<(mbs + 127) / 128, 128, 0, s>>>(a, lscale, adjacency, bright);
    return cudaGetLastError();
}

// The signed intra reconstruction of an I picture: the optional overlap edge source (flags: per
// MB, nullptr with all = 0 for none), the forward transforms and AC levels, the DC chain, the
// inverse transforms into the int32 planes oy / ou / ov (padded raster, rows packed). scratch
// holds intra_scratch_bytes(P) bytes; edge: 1.5 * (mbw * 16) * (mbh * 16) bytes for the edge
// source. tables / cfg: the AC length tables and the trellis and perceptual settings (trellis 0:
// scalar levels); the trellis's lambda scale reads the intra source's luma mean, taken here.
size_t intra_scratch_bytes(const DevParams& P) {
    const size_t mbs = (size_t)P.mbw * P.mbh;
    return mbs * 6 * 64 * 2 + mbs * 6 * 4 * 2 + 256;
}

cudaError_t launch_intra_recon(const DevParams& P, const DevFrame& src, int overlap, const uint8_t* d_flags,
                               const uint8_t* d_mquant, const uint8_t* d_derived, void* scratch, uint8_t* edge,
                               int32_t* oy, int32_t* ou, int32_t* ov, const void* tables, const vc1cu_trd_cfg& cfg,
                               cudaStream_t s) {
    const int mbs = P.mbw * P.mbh;
    if (mbs <= 0) return cudaSuccess;
    IntraArgs A{};
    A.P = P;
    A.y = src.y;
    A.u = src.u;
    A.v = src.v;
    A.pitch_y = src.pitch_y;
    A.pitch_c = src.pitch_c;
    A.sw = P.W;
    A.sh = P.H;
    cudaError_t e;
    if (overlap) {
        const int cw = P.mbw * 16, ch = P.mbh * 16, ccw = cw / 2, cch = ch / 2;
        const int cvw = (P.vw + 1) / 2, cvh = (P.vh + 1) / 2;
        const int vx = ovl_border(P.vw, cw), vy = ovl_border(P.vh, ch), cx = ovl_border(cvw, ccw), cy = ovl_border(cvh, cch);
        if (vx >= 0 || vy >= 0 || cx >= 0 || cy >= 0) {
            EdgeArgs E{};
            const uint8_t* in[3] = {src.y, src.u, src.v};
            for (int k = 0; k < 3; ++k) {
                const bool l = k == 0;
                E.in[k] = in[k];
                E.in_pitch[k] = l ? src.pitch_y : src.pitch_c;
                E.sw[k] = l ? P.W : P.W / 2;
                E.sh[k] = l ? P.H : P.H / 2;
                E.dw[k] = l ? cw : ccw;
                E.dh[k] = l ? ch : cch;
                E.out_pitch[k] = E.dw[k];
                E.vw[k] = l ? P.vw : cvw;
                E.vh[k] = l ? P.vh : cvh;
                E.ex[k] = l ? vx : cx;
                E.ey[k] = l ? vy : cy;
            }
            E.out[0] = edge;
            E.out[1] = edge + (size_t)cw * ch;
            E.out[2] = edge + (size_t)cw * ch + (size_t)ccw * cch;
            E.flags = d_flags;
            E.all = overlap == 1;
            E.mbw = P.mbw;
            E.mbh = P.mbh;
            edge_source_kernel<<<dim3((unsigned)((cw * ch + 255) / 256), 3), 256, 0, s>>>(E);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            A.y = E.out[0];
            A.u = E.out[1];
            A.v = E.out[2];
            A.pitch_y = cw;
            A.pitch_c = ccw;
            A.sw = cw;
            A.sh = ch;
        }
    }
    A.mquant = d_mquant;
    A.derived = d_derived;
    uint8_t* p = static_cast<uint8_t*>(scratch);
    A.q = reinterpret_cast<int16_t*>(p);
    p += (size_t)mbs * 6 * 64 * 2;
    int* dc = reinterpret_cast<int*>(p);
    int* qg = dc + (size_t)mbs * 6;
    A.dc[0] = dc;
    A.dc[1] = dc + (size_t)mbs * 4;
    A.dc[2] = dc + (size_t)mbs * 5;
    A.qg[0] = qg;
    A.qg[1] = qg + (size_t)mbs * 4;
    A.qg[2] = qg + (size_t)mbs * 5;
    A.trd.P = P;
    A.trd.tab = static_cast<const TrdTables*>(tables);
    A.trd.cfg = cfg;
    A.trd.frame_mean = 0.0;
    if (cfg.trellis > 0) {  // cached_luma_mean of the intra source's luma (the picture or its edge source)
        DevParams sp = P;
        sp.W = A.sw;
        sp.H = A.sh;
        DevFrame sf{};
        sf.y = A.y;
        sf.pitch_y = A.pitch_y;
        unsigned long long* d_sum = reinterpret_cast<unsigned long long*>(qg + (size_t)mbs * 6);
        if ((e = frame_mean_for(sp, sf, cfg, d_sum, s, A.trd.frame_mean)) != cudaSuccess) return e;
    }
    const unsigned blocks = (unsigned)((mbs * 6 + 127) / 128);
    intra_fwd_kernel<<<blocks, 128, 0, s>>>(A);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    intra_dc_kernel<<<3, 256, 0, s>>>(A);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    intra_inv_kernel<<<blocks, 128, 0, s>>>(A, oy, ou, ov);
    return cudaGetLastError();
}

}  // namespace vc1cu
