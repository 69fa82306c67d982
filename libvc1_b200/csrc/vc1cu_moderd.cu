// vc1cu_moderd.cu - the device counts of the P picture's motion-mode decision
// (Vc1Encoder::analyze_p_picture, src/encoder_motion.cpp:524-597).
//
// estimate_p_motion_bits (:444-486) charges a candidate analysis its MVTAB selector, MVMODE,
// the MVTYPEMB bitplane of a Mixed-MV picture and every macroblock's MVDATA under the cheapest
// of the four MV tables, plus one bit per hybrid-predicted vector. Here one thread per
// macroblock forms its MVDATA values (predictor, hybrid choice by modular distance, symbol and
// suffix) and adds their lengths under all four tables at once; one block scores the bitplane's
// raw, NORM-2, NORM-6, ROWSKIP and COLSKIP codings (plain and inverted, choose_bitplane,
// src/encoder_entropy.cpp:37-61). The host adds the picture-layer fields and takes the least
// table. The sampled transform RD of sampled_p_mode_rd (:488-522) runs trd_kernel on the
// sampled macroblocks; the host combines both in the reference's long double.
#include <cuda_runtime.h>

#include <cstdint>

#include "vc1cu_core.cuh"

#define VC1CU_ENT_TABLE __constant__ const
#include "vc1cu_entropy_lengths.h"

namespace vc1cu {
namespace {

constexpr unsigned FULLM = 0xffffffffu;

// The finished analysis's block-MV field as the predictors read it (predictor_info_4mv's `get`
// and `intra_at`, src/encoder_motion.cpp:1408-1466): zero and not intra outside the raster.
struct ResultField {
    const int2* bmv;
    const uint8_t* mb_intra;
    int mbw, mbh;
    __device__ int2 get(int x, int y) const {
        if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return make_int2(0, 0);
        return bmv[((size_t)(y >> 1) * mbw + (x >> 1)) * 4 + (((y & 1) << 1) | (x & 1))];
    }
    __device__ bool intra(int x, int y) const {
        if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return false;
        return mb_intra[(size_t)(y >> 1) * mbw + (x >> 1)] != 0;
    }
};

// acc: [0..3] MVDATA bits under tables 0..3, [4] hybrid-predictor bits, [5] half-pel
// differentials the syntax cannot represent (mvdata_for_mode throws for them).
__global__ void p_mv_bits_kernel(const __grid_constant__ DevParams P, DevResult r, int mode, unsigned long long* acc) {
    const int mbs = P.mbw * P.mbh;
    const bool mixed = mode == VC1CU_MV_MIXED;
    const ResultField f{r.bmv, r.intra, P.mbw, P.mbh};
    unsigned long long t0 = 0, t1 = 0, t2 = 0, t3 = 0, hyb = 0, bad = 0;
    auto add = [&](int2 d, int2 pred, int m) {
        if (mode_halfpel(m) && (((d.x - pred.x) & 1) || ((d.y - pred.y) & 1))) ++bad;
        int suffix;
        const int sym = mv_symbol_suffix(P, d, pred, m, true, suffix);
        t0 += ent::kMvDiffBits[0][sym] + suffix;
        t1 += ent::kMvDiffBits[1][sym] + suffix;
        t2 += ent::kMvDiffBits[2][sym] + suffix;
        t3 += ent::kMvDiffBits[3][sym] + suffix;
    };
    for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < mbs; pos += gridDim.x * blockDim.x) {
        const int mx = pos % P.mbw, my = pos / P.mbw;
        if (r.intra[pos]) {
            // the intra MVDATA with more = 1: symbol 72, no suffix
            t0 += ent::kMvDiffBits[0][72];
            t1 += ent::kMvDiffBits[1][72];
            t2 += ent::kMvDiffBits[2][72];
            t3 += ent::kMvDiffBits[3][72];
        } else if (mixed && r.use4[pos]) {
            for (int k = 0; k < 4; ++k) {
                const PInfo pi = predictor_4mv(P, f, mx, my, k);
                const int2 d = r.bmv[(size_t)pos * 4 + k];
                int2 pred = pi.pre;
                if (pi.hybrid) {
                    pred = modular_mv_distance(P, d, pi.a) <= modular_mv_distance(P, d, pi.c) ? pi.a : pi.c;
                    ++hyb;
                }
                add(d, pred, VC1CU_MV_MIXED);
            }
        } else {
            const PInfo pi = predictor_mixed_1mv(P, f, mx, my);
            const int2 d = r.mvs[pos];
            int2 pred = pi.pre;
            if (pi.hybrid) {
                pred = modular_mv_distance(P, d, pi.a) <= modular_mv_distance(P, d, pi.c) ? pi.a : pi.c;
                ++hyb;
            }
            add(d, pred, mode);
        }
    }
    unsigned long long v[6] = {t0, t1, t2, t3, hyb, bad};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(FULLM, v[i], o);
        if ((threadIdx.x & 31) == 0 && v[i]) atomicAdd(acc + i, v[i]);
    }
}

// The least total_bits of choose_bitplane over a w x h plane (nonzero = 1): raw, then IMODE
// 1 (NORM-2), 3 (NORM-6), 5 (ROWSKIP), 6 (COLSKIP), each plain and inverted; each coding costs
// the INVERT bit, its IMODE code and its payload (encode_norm2_bits / encode_norm6_bits /
// encode_rowskip_bits / encode_colskip_bits, src/encoder_encode.cpp:1878-1930). One block.
__global__ void bitplane_bits_kernel(const uint8_t* plane, int w, int h, unsigned long long* out) {
    // [0..1] NORM-2, [2..3] NORM-6, [4..5] ROWSKIP, [6..7] COLSKIP payloads, plain / inverted
    __shared__ unsigned int sum[8];
    if (threadIdx.x < 8) sum[threadIdx.x] = 0;
    __syncthreads();
    const int n = w * h;
    auto at = [&](int x, int y) -> unsigned { return plane[(size_t)y * w + x] != 0 ? 1u : 0u; };
    unsigned int s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // skip-coded run of `len` values starting at (x0, y0) stepping (dx, dy): the flag bit, then
    // the values when any is set (plain: any one; inverted: any zero)
    auto skip_bits = [&](int x0, int y0, int dx, int dy, int len, unsigned& plain, unsigned& inv) {
        unsigned ones = 0;
        for (int i = 0; i < len; ++i) ones += at(x0 + i * dx, y0 + i * dy);
        plain += 1u + (ones ? (unsigned)len : 0u);
        inv += 1u + (ones < (unsigned)len ? (unsigned)len : 0u);
    };
    // NORM-2: an odd plane's first value raw, then pairs in raster order
    const int off = n & 1;
    if (threadIdx.x == 0 && off) {
        s[0] += 1;
        s[1] += 1;
    }
    for (int i = off + 2 * threadIdx.x; i + 1 < n; i += 2 * blockDim.x) {
        const unsigned sym = (plane[i] != 0 ? 1u : 0u) | (plane[i + 1] != 0 ? 2u : 0u);
        s[0] += ent::kNorm2Bits[sym];
        s[1] += ent::kNorm2Bits[sym ^ 3u];
    }
    // NORM-6
    if (!(h % 3) && (w % 3)) {
        // 2x3 tiles from column w & 1, then the first column skip-coded when w is odd
        const int tx = (w - (w & 1)) / 2, ty = h / 3;
        for (int t = threadIdx.x; t < tx * ty; t += blockDim.x) {
            const int x = (w & 1) + 2 * (t % tx), y = 3 * (t / tx);
            const unsigned sym = at(x, y) | (at(x + 1, y) << 1) | (at(x, y + 1) << 2) | (at(x + 1, y + 1) << 3) |
                                 (at(x, y + 2) << 4) | (at(x + 1, y + 2) << 5);
            s[2] += ent::kNorm6Bits[sym];
            s[3] += ent::kNorm6Bits[sym ^ 63u];
        }
        if ((w & 1) && threadIdx.x == 0) skip_bits(0, 0, 0, 1, h, s[2], s[3]);
    } else {
        // 3x2 tiles from column w % 3 and row h & 1, then the lead columns skip-coded, then the
        // first row (right of the lead columns) skip-coded when h is odd
        const int lead = w % 3, tx = (w - lead) / 3, ty = (h - (h & 1)) / 2;
        for (int t = threadIdx.x; t < tx * ty; t += blockDim.x) {
            const int x = lead + 3 * (t % tx), y = (h & 1) + 2 * (t / tx);
            const unsigned sym = at(x, y) | (at(x + 1, y) << 1) | (at(x + 2, y) << 2) | (at(x, y + 1) << 3) |
                                 (at(x + 1, y + 1) << 4) | (at(x + 2, y + 1) << 5);
            s[2] += ent::kNorm6Bits[sym];
            s[3] += ent::kNorm6Bits[sym ^ 63u];
        }
        if ((int)threadIdx.x < lead) skip_bits(threadIdx.x, 0, 0, 1, h, s[2], s[3]);
        if ((h & 1) && threadIdx.x == 0) skip_bits(lead, 0, 1, 0, w - lead, s[2], s[3]);  // its flag even when empty
    }
    // ROWSKIP and COLSKIP
    for (int y = threadIdx.x; y < h; y += blockDim.x) skip_bits(0, y, 1, 0, w, s[4], s[5]);
    for (int x = threadIdx.x; x < w; x += blockDim.x) skip_bits(x, 0, 0, 1, h, s[6], s[7]);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        for (int o = 16; o; o >>= 1) s[i] += __shfl_xor_sync(FULLM, s[i], o);
        if ((threadIdx.x & 31) == 0 && s[i]) atomicAdd(&sum[i], s[i]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long best = 1ull + ent::kImodeBits[0] + (unsigned long long)n;  // raw
        const int imode[4] = {1, 3, 5, 6};
        for (int m = 0; m < 4; ++m)
            for (int inv = 0; inv < 2; ++inv) {
                const unsigned long long b = 1ull + ent::kImodeBits[imode[m]] + sum[2 * m + inv];
                if (b < best) best = b;
            }
        *out = best;
    }
}

}  // namespace

// acc: 7 counters (4 table sums, hybrid bits, unrepresentable differentials, the MVTYPEMB
// bitplane's bits when mode is Mixed-MV); zeroed here.
cudaError_t launch_p_motion_bits(const DevParams& P, const DevResult& r, int mode, unsigned long long* acc, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(acc, 0, 7 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const int mbs = P.mbw * P.mbh;
    if (mbs <= 0) return cudaSuccess;
    p_mv_bits_kernel<<<(mbs + 255) / 256, 256, 0, s>>>(P, r, mode, acc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (mode == VC1CU_MV_MIXED) {
        bitplane_bits_kernel<<<1, 512, 0, s>>>(r.use4, P.mbw, P.mbh, acc + 6);
        e = cudaGetLastError();
    }
    return e;
}

// choose_bitplane's least total bits of a w x h plane into *out (device).
cudaError_t launch_bitplane_bits(const uint8_t* plane, int w, int h, unsigned long long* out, cudaStream_t s) {
    bitplane_bits_kernel<<<1, 512, 0, s>>>(plane, w, h, out);
    return cudaGetLastError();
}

}  // namespace vc1cu
