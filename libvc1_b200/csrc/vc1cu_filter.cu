// vc1cu_filter.cu - VC-1 in-loop deblocking on the device: the I-like all-edges filter
// (Vc1Encoder::apply_i_like_loop_filter, encoder_filter.cpp:426-441) and the Advanced Profile
// P-picture filter of the coded blocks (apply_p_loop_filter, :610-738).
//
// Each edge filter works on groups of four lines across the edge (the third line decides for
// its group) and only reads and writes along its lines, so the groups of one edge are
// independent. The reference walks the picture in raster order (per macroblock row, the
// horizontal edges of MB x before the vertical edges of MB x-1). That order is equivalent to:
// every horizontal edge first, each 4-column strip walked top to bottom (a strip's edges read
// rows the edge above it wrote), then every vertical edge, each 4-row strip walked left to right
// (an inner 4x4 edge reads the column the block's left neighbour's border wrote); strips of one
// phase touch disjoint pixels. So one thread owns one strip:
//   lfp_h_kernel  one thread per 4-column strip of a plane: the horizontal edges, top to bottom;
//   lfp_v_kernel  one thread per 4-row strip: the vertical edges, left to right.
// The I-like filter has no order between its edges of one direction (8 pixels apart, each reads
// 4 on either side and writes 1): one thread per 4-line group of every edge.
//
// Overlap smoothing (apply_overlap_plane_signed, :217-243) of a signed reconstruction: each
// edge filter reads and writes the 2 samples on either side along one line, so the lines of
// one direction's edges (8 apart) touch disjoint samples; one thread per line of every edge,
// vertical edges in one launch, horizontal edges (which read the first stage's output) in a
// second.
#include <cuda_runtime.h>

#include "vc1cu_core.cuh"

namespace vc1cu {

struct LfPlane {
    uint8_t* p;
    int pitch, w, h;
};

// Vc1Encoder::loop_filter_line (encoder_filter.cpp:366-395): the line across the edge between
// (x - cross) and (x, y); false when ineligible.
__device__ bool lf_line(const LfPlane& pl, int x, int y, int cdx, int cdy, int pq) {
    if (x - 4 * cdx < 0 || y - 4 * cdy < 0 || x + 3 * cdx >= pl.w || y + 3 * cdy >= pl.h || x < 0 || y < 0 ||
        x >= pl.w || y >= pl.h)
        return false;
    const int step = cdy * pl.pitch + cdx;
    uint8_t* c = pl.p + (size_t)y * pl.pitch + x;
    auto S = [&](int k) { return (int)c[k * step]; };
    int a0 = arshift(2 * (S(-2) - S(1)) - 5 * (S(-1) - S(0)) + 4, 3);
    const bool a0_neg = a0 < 0;
    a0 = iabs(a0);
    if (a0 >= pq) return false;
    const int a1 = iabs(arshift(2 * (S(-4) - S(-1)) - 5 * (S(-3) - S(-2)) + 4, 3));
    const int a2 = iabs(arshift(2 * (S(0) - S(3)) - 5 * (S(1) - S(2)) + 4, 3));
    if (!(a1 < a0 || a2 < a0)) return false;
    const int edge = S(-1) - S(0);
    const int limit = iabs(edge) >> 1;
    if (!limit) return false;
    int delta = (5 * (a0 - imin(a1, a2))) >> 3;
    if (a0_neg != (edge < 0)) {
        delta = imin(delta, limit);
        if (edge < 0) delta = -delta;
        c[-step] = (uint8_t)iclamp(S(-1) - delta, 0, 255);
        c[0] = (uint8_t)iclamp(S(0) + delta, 0, 255);
    }
    return true;
}

// One 4-line group of loop_filter_edge (:397-416) starting at (x, y) along (adx, ady).
__device__ void lf_group(const LfPlane& pl, int x, int y, int adx, int ady, int cdx, int cdy, int pq) {
    if (!lf_line(pl, x + 2 * adx, y + 2 * ady, cdx, cdy, pq)) return;
    lf_line(pl, x, y, cdx, cdy, pq);
    lf_line(pl, x + adx, y + ady, cdx, cdy, pq);
    lf_line(pl, x + 3 * adx, y + 3 * ady, cdx, cdy, pq);
}
// the group of a horizontal edge (columns x..x+3, edge above row y) / of a vertical edge
__device__ __forceinline__ void lf_hgroup(const LfPlane& pl, int x, int y, int pq) { lf_group(pl, x, y, 1, 0, 0, 1, pq); }
__device__ __forceinline__ void lf_vgroup(const LfPlane& pl, int x, int y, int pq) { lf_group(pl, x, y, 0, 1, 1, 0, pq); }

// The three planes of a frame slot; strip index -> (plane, strip within it).
struct LfFrame {
    LfPlane pl[3];
};

// I-like filter, horizontal borders (apply_i_like_loop_filter_plane, :426-434): every row y = 8k
// (k >= 1), every 4-column group.
__global__ void lfi_h_kernel(LfFrame f, int pq) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < 3; ++k) {
        const LfPlane& pl = f.pl[k];
        const int gx = (pl.w + 3) / 4, ey = (pl.h - 1) / 8;  // edges at y = 8..8*ey
        if (idx < gx * ey) {
            lf_hgroup(pl, (idx % gx) * 4, (idx / gx + 1) * 8, pq);
            return;
        }
        idx -= gx * ey;
    }
}
// I-like filter, vertical borders: every column x = 8k (k >= 1), every 4-row group.
__global__ void lfi_v_kernel(LfFrame f, int pq) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < 3; ++k) {
        const LfPlane& pl = f.pl[k];
        const int gy = (pl.h + 3) / 4, ex = (pl.w - 1) / 8;
        if (idx < gy * ex) {
            lf_vgroup(pl, (idx / gy + 1) * 8, (idx % gy) * 4, pq);
            return;
        }
        idx -= gy * ex;
    }
}

// Coded-block metadata of the P filter: 4 block vectors, 6 loop_filter_pattern and 6
// loop_filter_tt codes and one intra bit per block, per macroblock.
struct LfMeta {
    const int2* bmv;
    const uint8_t* cbp;
    const uint8_t* tt;
    const uint8_t* intra;
    int mbw, mbh;
    int main_profile;  // the Main Profile rules (apply_p_loop_filter_plane_main, encoder_filter.cpp:465-608)
};

struct LfBlock {
    int cbp, tt;
    bool intra, mb_intra;  // this block intra; any block of its macroblock intra
    int2 mv;
};

// The block (bx, by) of plane k (luma 8x8 grid, chroma one block per MB), with mv_at's vector:
// the luma block vector, or for chroma the pre-FASTUVMC representative of the 4-MV median
// (encoder_filter.cpp:628-637).
__device__ LfBlock lf_block(const LfMeta& m, int k, int bx, int by) {
    const bool luma = k == 0;
    const int mx = luma ? bx >> 1 : bx, my = luma ? by >> 1 : by;
    const int bk = luma ? (((by & 1) << 1) | (bx & 1)) : 3 + k;
    const int mb = my * m.mbw + mx;
    LfBlock b;
    b.cbp = m.cbp[mb * 6 + bk];
    b.tt = m.tt[mb * 6 + bk];
    b.intra = (m.intra[mb] >> bk) & 1;
    b.mb_intra = m.intra[mb] != 0;
    const int2* v = m.bmv + mb * 4;
    if (luma) {
        b.mv = v[bk];
    } else {
        auto med4 = [](int a, int b2, int c, int d) {
            if (a < b2) {
                if (c < d) return (imin(b2, d) + imax(a, c)) / 2;
                return (imin(b2, c) + imax(a, d)) / 2;
            }
            if (c < d) return (imin(a, d) + imax(b2, c)) / 2;
            return (imin(a, c) + imax(b2, d)) / 2;
        };
        const int cx = med4(v[0].x, v[1].x, v[2].x, v[3].x), cy = med4(v[0].y, v[1].y, v[2].y, v[3].y);
        int x = arshift(cx + ((cx & 3) == 3), 1), y = arshift(cy + ((cy & 3) == 3), 1);
        if (m.main_profile) {
            // Main Profile exception 4 (:502-523): the FASTUVMC rounding towards zero and the
            // 8.3.6.5 range limit of the chroma vector that the decoder compares
            x = x < 0 ? x + (x & 1) : x - (x & 1);
            y = y < 0 ? y + (y & 1) : y - (y & 1);
            const int ox = mx * 8, oy = my * 8;
            const int px = ox + arshift(x, 2), py = oy + arshift(y, 2);
            if (px < -8) x = 4 * (-8 - ox) + (x & 3);
            else if (px > m.mbw * 8) x = 4 * (m.mbw * 8 - ox) + (x & 3);
            if (py < -8) y = 4 * (-8 - oy) + (y & 3);
            else if (py > m.mbh * 8) y = 4 * (m.mbh * 8 - oy) + (y & 3);
        }
        b.mv = make_int2(x, y);
    }
    return b;
}

// Horizontal edges of one 4-column strip, top to bottom (process_v_parent, :654-676): each
// block's bottom border, then its inner 4-row edge.
__global__ void lfp_h_kernel(LfFrame f, LfMeta m, int pq) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < 3; ++k) {
        const LfPlane& pl = f.pl[k];
        const int gx = (pl.w + 3) / 4;
        if (idx >= gx) {
            idx -= gx;
            continue;
        }
        const int cx = idx * 4, bx = cx >> 3, half = (cx >> 2) & 1;
        const int grid_h = k == 0 ? m.mbh * 2 : m.mbh;
        for (int by = 0; by < grid_h; ++by) {
            const int x0 = bx * 8, y0 = by * 8;
            if (x0 >= pl.w || y0 >= pl.h) break;
            const LfBlock b = lf_block(m, k, bx, by);
            if (by + 1 < grid_h && y0 + 8 < pl.h) {
                const LfBlock n = lf_block(m, k, bx, by + 1);
                // Main Profile exceptions 1 (block 0 of the first MB intra: every inter MB's top
                // border filtered whole) and 3 (a 4x4-transformed side: the whole border, :547-553)
                const bool ex = m.main_profile && (((m.intra[0] & 1) && !n.mb_intra) || b.tt == 7 || n.tt == 7);
                if (ex || b.intra || n.intra || b.mv.x != n.mv.x || b.mv.y != n.mv.y) {
                    if (half * 4 < imin(8, pl.w - x0)) lf_hgroup(pl, cx, y0 + 8, pq);
                } else {
                    const int mask = (b.cbp | (n.cbp >> 2)) & 3;
                    if (half == 0 ? (mask & 2) != 0 : ((mask & 1) && x0 + 4 < pl.w)) lf_hgroup(pl, cx, y0 + 8, pq);
                }
            }
            if ((b.tt == 7 || b.tt == 3) && y0 + 4 < pl.h) {
                if (half == 0 ? (b.cbp & 10) != 0 : ((b.cbp & 5) && x0 + 4 < pl.w)) lf_hgroup(pl, cx, y0 + 4, pq);
            }
        }
        return;
    }
}

// Vertical edges of one 4-row strip, left to right (process_h_parent, :677-699): each block's
// right border, then its inner 4-column edge.
__global__ void lfp_v_kernel(LfFrame f, LfMeta m, int pq) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < 3; ++k) {
        const LfPlane& pl = f.pl[k];
        const int gy = (pl.h + 3) / 4;
        if (idx >= gy) {
            idx -= gy;
            continue;
        }
        const int ry = idx * 4, by = ry >> 3, half = (ry >> 2) & 1;
        const int grid_w = k == 0 ? m.mbw * 2 : m.mbw;
        for (int bx = 0; bx < grid_w; ++bx) {
            const int x0 = bx * 8, y0 = by * 8;
            if (x0 >= pl.w || y0 >= pl.h) break;
            const LfBlock b = lf_block(m, k, bx, by);
            if (bx + 1 < grid_w && x0 + 8 < pl.w) {
                const LfBlock n = lf_block(m, k, bx + 1, by);
                // Main Profile exceptions 1 and 3, and 2: the luma edge between blocks 2 and 3
                // decides with block 1's pattern and kind on its left (:563-581)
                const LfBlock d = (m.main_profile && k == 0 && !(bx & 1) && (by & 1)) ? lf_block(m, k, bx + 1, by - 1) : b;
                const bool ex = m.main_profile && (((m.intra[0] & 1) && !n.mb_intra) || d.tt == 7 || n.tt == 7);
                if (ex || b.intra || n.intra || b.mv.x != n.mv.x || b.mv.y != n.mv.y) {
                    if (half * 4 < imin(8, pl.h - y0)) lf_vgroup(pl, x0 + 8, ry, pq);
                } else {
                    const int mask = (d.cbp | (n.cbp >> 1)) & 5;
                    if (half == 0 ? (mask & 4) != 0 : ((mask & 1) && y0 + 4 < pl.h)) lf_vgroup(pl, x0 + 8, ry, pq);
                }
            }
            if ((b.tt == 7 || b.tt == 6) && x0 + 4 < pl.w) {
                if (half == 0 ? (b.cbp & 12) != 0 : ((b.cbp & 3) && y0 + 4 < pl.h)) lf_vgroup(pl, x0 + 4, ry, pq);
            }
        }
        return;
    }
}

static LfFrame lf_frame(uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H) {
    LfFrame f;
    f.pl[0] = LfPlane{y, pitch_y, W, H};
    f.pl[1] = LfPlane{u, pitch_c, W / 2, H / 2};
    f.pl[2] = LfPlane{v, pitch_c, W / 2, H / 2};
    return f;
}

cudaError_t launch_loop_filter_i(uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H, int pq,
                                 cudaStream_t s) {
    const LfFrame f = lf_frame(y, u, v, pitch_y, pitch_c, W, H);
    int nh = 0, nv = 0;
    for (int k = 0; k < 3; ++k) {
        const LfPlane& pl = f.pl[k];
        nh += ((pl.w + 3) / 4) * imax(0, (pl.h - 1) / 8);
        nv += ((pl.h + 3) / 4) * imax(0, (pl.w - 1) / 8);
    }
    if (nh) lfi_h_kernel<<<(unsigned)((nh + 127) / 128), 128, 0, s>>>(f, pq);
    if (nv) lfi_v_kernel<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(f, pq);
    return cudaGetLastError();
}

cudaError_t launch_loop_filter_p(uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H, int pq,
                                 const int2* bmv, const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra,
                                 cudaStream_t s, int main_profile) {
    const LfFrame f = lf_frame(y, u, v, pitch_y, pitch_c, W, H);
    const LfMeta m{bmv, cbp, tt, intra, (W + 15) / 16, (H + 15) / 16, main_profile};
    const int nh = (W + 3) / 4 + 2 * ((W / 2 + 3) / 4), nv = (H + 3) / 4 + 2 * ((H / 2 + 3) / 4);
    lfp_h_kernel<<<(unsigned)((nh + 63) / 64), 64, 0, s>>>(f, m, pq);
    lfp_v_kernel<<<(unsigned)((nv + 63) / 64), 64, 0, s>>>(f, m, pq);
    return cudaGetLastError();
}

// ---- overlap smoothing --------------------------------------------------------------------

struct OvlPlanes {
    int32_t* p[3];
    int w[3], h[3];
    const uint8_t* flags;  // per macroblock, mbw * mbh (unused when all)
    int mbw, mbh, all;
};

// overlap_edge_enabled (encoder_filter.cpp:201-215) between 8x8 blocks (bx0, by0), (bx1, by1).
__device__ __forceinline__ bool ovl_enabled(const OvlPlanes& o, bool luma, int bx0, int by0, int bx1, int by1) {
    if (o.all) return true;
    const int mx0 = luma ? bx0 >> 1 : bx0, my0 = luma ? by0 >> 1 : by0;
    const int mx1 = luma ? bx1 >> 1 : bx1, my1 = luma ? by1 >> 1 : by1;
    if (mx0 < 0 || my0 < 0 || mx0 >= o.mbw || my0 >= o.mbh) return false;
    if (mx1 < 0 || my1 < 0 || mx1 >= o.mbw || my1 >= o.mbh) return false;
    const int a = my0 * o.mbw + mx0, b = my1 * o.mbw + mx1;
    if (a == b) return o.flags[a] != 0;
    return o.flags[a] != 0 && o.flags[b] != 0;
}

// overlap_arshift3 (:162-164): rounds v / 8 toward minus infinity.
__device__ __forceinline__ int ovl_shift3(int v) { return v >= 0 ? (v >> 3) : -((-v + 7) >> 3); }

// The 4 samples across an edge at line parity i (overlap_vertical_edge :166-180 and
// overlap_horizontal_edge :182-199 share it); step is the distance between the samples.
__device__ __forceinline__ void ovl_line(int32_t* c, int step, int i) {
    const int a = c[-2 * step], b = c[-step], cc = c[0], d = c[step];
    const int d1 = a - d, d2 = a - d + b - cc;
    const int r1 = (i & 1) ? 3 : 4, r2 = 7 - r1;
    c[-2 * step] = ovl_shift3(8 * a - d1 + r1);
    c[-step] = ovl_shift3(8 * b - d2 + r2);
    c[0] = ovl_shift3(8 * cc + d2 + r1);
    c[step] = ovl_shift3(8 * d + d1 + r2);
}

// Stage one: thread = (row y, vertical edge bx >= 1) of plane blockIdx.y.
__global__ void ovl_v_kernel(OvlPlanes o) {
    const int k = blockIdx.y;
    const int w = o.w[k], h = o.h[k], bw = w / 8;
    if (w < 8 || h < 8 || bw < 2) return;
    const long n = (long)(h / 8 * 8) * (bw - 1);
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const int y = (int)(t / (bw - 1)), bx = 1 + (int)(t % (bw - 1));
        if (!ovl_enabled(o, k == 0, bx - 1, y >> 3, bx, y >> 3)) continue;
        ovl_line(o.p[k] + (size_t)y * w + bx * 8, 1, y & 7);
    }
}

// Stage two: thread = (horizontal edge by >= 1, column x) of plane blockIdx.y.
__global__ void ovl_h_kernel(OvlPlanes o) {
    const int k = blockIdx.y;
    const int w = o.w[k], h = o.h[k], bh = h / 8, bw = w / 8;
    if (w < 8 || h < 8 || bh < 2) return;
    const long n = (long)(bh - 1) * (bw * 8);
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const int by = 1 + (int)(t / (bw * 8)), x = (int)(t % (bw * 8));
        if (!ovl_enabled(o, k == 0, x >> 3, by - 1, x >> 3, by)) continue;
        ovl_line(o.p[k] + (size_t)(by * 8) * w + x, w, x & 7);
    }
}

cudaError_t launch_overlap(int32_t* y, int32_t* u, int32_t* v, int mbw, int mbh, const uint8_t* d_flags, int all,
                           cudaStream_t s) {
    OvlPlanes o;
    o.p[0] = y;
    o.p[1] = u;
    o.p[2] = v;
    o.w[0] = mbw * 16;
    o.h[0] = mbh * 16;
    o.w[1] = o.w[2] = mbw * 8;
    o.h[1] = o.h[2] = mbh * 8;
    o.flags = d_flags;
    o.mbw = mbw;
    o.mbh = mbh;
    o.all = all;
    const long lines = (long)o.w[0] * o.h[0] / 8;  // edges per 8 samples, the most of any plane and stage
    const unsigned blocks = (unsigned)imin(4096, (int)((lines + 255) / 256));
    ovl_v_kernel<<<dim3(blocks, 3), 256, 0, s>>>(o);
    ovl_h_kernel<<<dim3(blocks, 3), 256, 0, s>>>(o);
    return cudaGetLastError();
}

// overlap_sse_region (encoder_filter.cpp:246-266) of every MB: the squared error of clamp(s + bias)
// of the padded signed planes against the source (coordinates clamped into it) over the MB's
// 16x16 luma and 8x8 chroma blocks. Integer sums, exact like the reference's long double ones.
// One thread per MB.
__global__ void overlap_sse_kernel(const int32_t* sy, const int32_t* su, const int32_t* sv, const uint8_t* oy,
                                   const uint8_t* ou, const uint8_t* ov, int pitch_y, int pitch_c, int W, int H, int mbw,
                                   int mbh, int bias, unsigned long long* sse) {
    const int mb = blockIdx.x * blockDim.x + threadIdx.x;
    if (mb >= mbw * mbh) return;
    const int mx = mb % mbw, my = mb / mbw;
    unsigned long long e = 0;
    auto plane = [&](const int32_t* rec, int rw, const uint8_t* org, int pitch, int ow, int oh, int x0, int y0, int n) {
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const int rx = x0 + x, ry = y0 + y;
                const int sx = imin(imax(rx, 0), ow - 1), sy = imin(imax(ry, 0), oh - 1);
                const int r = imin(255, imax(0, rec[(size_t)ry * rw + rx] + bias));
                const int d = r - (int)org[(size_t)sy * pitch + sx];
                e += (unsigned long long)(d * d);
            }
    };
    plane(sy, mbw * 16, oy, pitch_y, W, H, mx * 16, my * 16, 16);
    plane(su, mbw * 8, ou, pitch_c, W / 2, H / 2, mx * 8, my * 8, 8);
    plane(sv, mbw * 8, ov, pitch_c, W / 2, H / 2, mx * 8, my * 8, 8);
    sse[mb] = e;
}

cudaError_t launch_overlap_sse(const int32_t* sy, const int32_t* su, const int32_t* sv, const uint8_t* oy,
                               const uint8_t* ou, const uint8_t* ov, int pitch_y, int pitch_c, int W, int H, int bias,
                               unsigned long long* sse, cudaStream_t s) {
    const int mbw = (W + 15) / 16, mbh = (H + 15) / 16;
    if (mbw * mbh <= 0) return cudaSuccess;
    overlap_sse_kernel<<<(mbw * mbh + 127) / 128, 128, 0, s>>>(sy, su, sv, oy, ou, ov, pitch_y, pitch_c, W, H, mbw, mbh, bias,
                                                               sse);
    return cudaGetLastError();
}

// clamp(s + bias) of the padded signed planes into a frame (its visible w x h), all macroblocks
// or the flagged ones; thread = 4 samples of a row.
struct StoreArgs {
    const int32_t* s[3];
    uint8_t* d[3];
    int sw[3], dpitch[3], dw[3], dh[3];
    const uint8_t* mask;
    int mbw, bias;
};

__global__ void store_signed_kernel(StoreArgs a) {
    const int k = blockIdx.y;
    const int w = imin(a.sw[k], a.dw[k]), h = a.dh[k];
    const int shift = k == 0 ? 4 : 3;
    const int q = (w + 3) / 4;
    const long n = (long)q * h;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const int y = (int)(t / q), x0 = (int)(t % q) * 4;
        if (a.mask && !a.mask[(y >> shift) * a.mbw + (x0 >> shift)]) continue;
        const int32_t* src = a.s[k] + (size_t)y * a.sw[k];
        uint8_t* dst = a.d[k] + (size_t)y * a.dpitch[k];
        for (int x = x0; x < x0 + 4 && x < w; ++x) dst[x] = (uint8_t)iclamp(src[x] + a.bias, 0, 255);
    }
}

cudaError_t launch_store_signed(const int32_t* y, const int32_t* u, const int32_t* v, int mbw, int mbh, int bias,
                                const uint8_t* d_mask, uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c,
                                int W, int H, cudaStream_t s) {
    StoreArgs a;
    a.s[0] = y;
    a.s[1] = u;
    a.s[2] = v;
    a.d[0] = dy;
    a.d[1] = du;
    a.d[2] = dv;
    a.sw[0] = mbw * 16;
    a.sw[1] = a.sw[2] = mbw * 8;
    a.dpitch[0] = pitch_y;
    a.dpitch[1] = a.dpitch[2] = pitch_c;
    a.dw[0] = W;
    a.dw[1] = a.dw[2] = W / 2;
    a.dh[0] = imin(H, mbh * 16);
    a.dh[1] = a.dh[2] = imin(H / 2, mbh * 8);
    a.mask = d_mask;
    a.mbw = mbw;
    a.bias = bias;
    const long n = (long)((imin(W, mbw * 16) + 3) / 4) * imin(H, mbh * 16);
    const unsigned blocks = (unsigned)imax(1, imin(4096, (int)((n + 255) / 256)));
    store_signed_kernel<<<dim3(blocks, 3), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace vc1cu
