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

#include "vc1cu_core.cuh"
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

// One thread per (type, MB, parent, partition). Output layout [type][mb][parent][64].
__global__ void xform_kernel(const __grid_constant__ DevParams P, DevFrame src, DevFrame pred, int type_mask, double* coeffs,
                             int16_t* levels) {
    const int mbs = P.mbw * P.mbh;
    // partitions per parent for each of the up-to-4 types, in type order
    int types[4], nt = 0;
    for (int t = 1; t <= 4; ++t)
        if (type_mask & (1 << (t - 1))) types[nt++] = t;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long per_type = (long)mbs * 6 * 4;  // up to 4 partitions
    if (idx >= per_type * nt) return;
    const int ti = (int)(idx / per_type);
    const long rem = idx % per_type;
    const int part = (int)(rem & 3);
    const int k = (int)((rem >> 2) % 6);
    const int mb = (int)((rem >> 2) / 6);
    const int t = types[ti];
    const int np = t == 1 ? 1 : (t == 4 ? 4 : 2);
    if (part >= np) return;
    int ox = 0, oy = 0, bw = 8, bh = 8;
    if (t == 2) { bh = 4; oy = part * 4; }
    else if (t == 3) { bw = 4; ox = part * 4; }
    else if (t == 4) { bw = 4; bh = 4; ox = (part & 1) * 4; oy = (part >> 1) * 4; }
    const int mx = mb % P.mbw, my = mb / P.mbw;
    const bool chroma = k >= 4;
    const uint8_t* sp = chroma ? (k == 4 ? src.u : src.v) : src.y;
    const uint8_t* pp = chroma ? (k == 4 ? pred.u : pred.v) : pred.y;
    const int spitch = chroma ? src.pitch_c : src.pitch_y, ppitch = chroma ? pred.pitch_c : pred.pitch_y;
    const int w = chroma ? P.W / 2 : P.W, h = chroma ? P.H / 2 : P.H;
    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
    const int x0 = bx * 8 + ox, y0 = by * 8 + oy;
    const size_t base = (((size_t)ti * mbs + mb) * 6 + k) * 64;
    if (x0 >= w || y0 >= h || x0 + bw <= 0 || y0 + bh <= 0) {
        // a partition wholly outside the crop codes nothing (encoder_transform.cpp:1097)
        for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) {
                if (coeffs) coeffs[base + (oy + y) * 8 + ox + x] = 0.0;
                if (levels) levels[base + (oy + y) * 8 + ox + x] = 0;
            }
        return;
    }
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
    for (int a = 0; a < bh; ++a)
        for (int b = 0; b < bw; ++b) {
            double acc = 0.0;
            for (int x = 0; x < bw; ++x) acc = __dadd_rn(acc, __dmul_rn(tmp[a][x], bw == 8 ? c_k8[b][x] : c_k4[b][x]));
            // 8x8 output is transposed (c[row*8+col] = 1024*xform[col][row]), rectangles are not
            const double c = __dmul_rn(1024.0, acc);
            int row, col;
            if (bw == 8 && bh == 8) { row = b; col = a; }
            else { row = a; col = b; }
            const size_t o = base + (size_t)(oy + row) * 8 + ox + col;
            if (coeffs) coeffs[o] = c;
            if (levels) levels[o] = (int16_t)quantize_level(P, c);
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

// One thread per (MB, parent): every partition of the block's chosen type dequantised,
// inverse-transformed (with the DC-only shortcut of a partition whose only level is its DC)
// and added to the prediction with 8-bit clamping. tindex[t] is type t's index in the levels
// layout [type][mb][parent][64] (-1 for a type the layout does not hold).
__global__ void recon_kernel(const __grid_constant__ DevParams P, DevFrame pred, const int16_t* levels, int4 tindex,
                             const uint8_t* block_types, uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c) {
    const int mbs = P.mbw * P.mbh;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= mbs * 6) return;
    const int mb = idx / 6, k = idx - mb * 6, mx = mb % P.mbw, my = mb / P.mbw;
    const int t = block_types[idx];
    const int ti = t == 1 ? tindex.x : (t == 2 ? tindex.y : (t == 3 ? tindex.z : tindex.w));
    const int16_t* q64 = levels + (((size_t)ti * mbs + mb) * 6 + k) * 64;
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
                a[y * 8 + x] = dequant(P, lv);
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
                  uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s) {
    const int n = P.mbw * P.mbh * 6;
    recon_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(P, pred, levels, tindex, block_types, dy, du, dv, pitch_y, pitch_c);
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
    int nt = 0;
    for (int t = 0; t < 4; ++t) nt += (type_mask >> t) & 1;
    const long n = (long)P.mbw * P.mbh * 6 * 4 * nt;
    if (!n) return;
    xform_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(P, src, pred, type_mask, coeffs, levels);
}

}  // namespace vc1cu
