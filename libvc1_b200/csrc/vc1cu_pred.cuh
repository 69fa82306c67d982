// vc1cu_pred.cuh - VC-1 luma interpolation and block costs on the device.
//
// Samplers read a reference plane either from a per-warp shared-memory window (fast path,
// WinSampler in vc1cu_core.cu) or from HBM with clamped coordinates (edge emulation, Vc1Encoder::sample_clamped,
// encoder_motion_compensation.cpp:350-353). Both return identical values wherever the
// window is defined, because the window is filled with the same clamped samples.
#pragma once

#include "vc1cu_common.cuh"

namespace vc1cu {

struct GlobSampler {
    const uint8_t* p;
    int pitch, W, H;
    __device__ __forceinline__ int operator()(int x, int y) const {
        x = iclamp(x, 0, W - 1);
        y = iclamp(y, 0, H - 1);
        return __ldg(p + (size_t)y * pitch + x);
    }
};

// N consecutive luma predictions of row py starting at px for quarter-pel MV (xq,yq):
// luma_mc_sample (VC-1 bicubic, encoder_motion_compensation.cpp:367-396) or, for the
// bilinear half-pel mode, luma_mc_sample_mode (:398-415).
template <int N, class S>
__device__ __forceinline__ void predict_row(const S& s, bool bilinear, int rnd, int xq, int yq, int px, int py,
                                            int out[N]) {
    const int ix = floor_div4(xq), iy = floor_div4(yq);
    const int hm = xq - ix * 4, vm = yq - iy * 4;
    const int sx = px + ix, sy = py + iy;
    if (bilinear) {
        if (!hm && !vm) {
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = s(sx + i, sy);
        } else if (hm && vm) {
#pragma unroll
            for (int i = 0; i < N; ++i)
                out[i] = (s(sx + i, sy) + s(sx + i + 1, sy) + s(sx + i, sy + 1) + s(sx + i + 1, sy + 1) + (rnd ? 1 : 2)) >> 2;
        } else if (hm) {
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = (s(sx + i, sy) + s(sx + i + 1, sy) + (rnd ? 0 : 1)) >> 1;
        } else {
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = (s(sx + i, sy) + s(sx + i, sy + 1) + (rnd ? 0 : 1)) >> 1;
        }
        return;
    }
    if (!hm && !vm) {
#pragma unroll
        for (int i = 0; i < N; ++i) out[i] = s(sx + i, sy);
        return;
    }
    if (hm && vm) {
        // shift_value {0,5,1,5}[m] of the reference (:375) is 1 for half-pel, 5 for quarter-pel
        const int shift = ((hm == 2 ? 1 : 5) + (vm == 2 ? 1 : 5)) >> 1;
        const int r1 = (1 << (shift - 1)) + (rnd ? 1 : 0) - 1;
        int t[N + 3];
#pragma unroll
        for (int k = -1; k <= N + 1; ++k) {
            const int raw = mspel(s(sx + k, sy - 1), s(sx + k, sy), s(sx + k, sy + 1), s(sx + k, sy + 2), vm);
            t[k + 1] = arshift(raw + r1, shift);
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const int raw = mspel(t[i], t[i + 1], t[i + 2], t[i + 3], hm);
            out[i] = iclamp(arshift(raw + 64 - (rnd ? 1 : 0), 7), 0, 255);
        }
        return;
    }
    if (vm) {
        const int bias = (vm == 2) ? (7 + (rnd ? 1 : 0)) : (31 + (rnd ? 1 : 0));
        const int sh = vm == 2 ? 4 : 6;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const int raw = mspel(s(sx + i, sy - 1), s(sx + i, sy), s(sx + i, sy + 1), s(sx + i, sy + 2), vm);
            out[i] = iclamp(arshift(raw + bias, sh), 0, 255);
        }
        return;
    }
    const int bias = (hm == 2) ? (8 - (rnd ? 1 : 0)) : (32 - (rnd ? 1 : 0));
    const int sh = hm == 2 ? 4 : 6;
    int r[N + 3];
#pragma unroll
    for (int k = -1; k <= N + 1; ++k) r[k + 1] = s(sx + k, sy);
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = iclamp(arshift(mspel(r[i], r[i + 1], r[i + 2], r[i + 3], hm) + bias, sh), 0, 255);
}

// mspel_filter4 taps of a quarter-pel phase (1: 1/4, 2: 1/2, 3: 3/4).
struct Taps {
    int w0, w1, w2, w3;
};
__device__ __forceinline__ Taps mspel_taps(int mode) {
    return mode == 1 ? Taps{-4, 53, 18, -3} : mode == 2 ? Taps{-1, 9, 9, -1} : Taps{-3, 18, 53, -4};
}
__device__ __forceinline__ int apply(const Taps& t, int a, int b, int c, int d) {
    return t.w0 * a + t.w1 * b + t.w2 * c + t.w3 * d;
}

template <int N>
struct PredRow {
    int v[N];
};

// predict_row over HBM with clamped coordinates, out of line: the rarely taken path of the
// shared-window scorers, kept out of their instruction stream.
template <int N>
__device__ __noinline__ PredRow<N> predict_row_glob(const uint8_t* p, int pitch, int W, int H, bool bilinear, int rnd, int xq,
                                                   int yq, int px, int py) {
    PredRow<N> r;
    predict_row<N>(GlobSampler{p, pitch, W, H}, bilinear, rnd, xq, yq, px, py, r.v);
    return r;
}

// Horizontal 4-point Hadamard of one residual row (the row stage of satd4x4_scalar).
__device__ __forceinline__ int4 hadamard_row(int d0, int d1, int d2, int d3) {
    const int a0 = d0 + d3, a1 = d1 + d2, a2 = d1 - d2, a3 = d0 - d3;
    return make_int4(a0 + a1, a3 + a2, a0 - a1, a3 - a2);
}

// Column stage of satd4x4_scalar over four row-transformed rows, with its (tile + 1) >> 1.
__device__ __forceinline__ uint32_t hadamard_cols(const int4& r0, const int4& r1, const int4& r2, const int4& r3) {
    auto col = [](int t0, int t1, int t2, int t3) {
        const int a0 = t0 + t3, a1 = t1 + t2, a2 = t1 - t2, a3 = t0 - t3;
        return (uint32_t)iabs(a0 + a1) + (uint32_t)iabs(a3 + a2) + (uint32_t)iabs(a0 - a1) + (uint32_t)iabs(a3 - a2);
    };
    const uint32_t tile = col(r0.x, r1.x, r2.x, r3.x) + col(r0.y, r1.y, r2.y, r3.y) + col(r0.z, r1.z, r2.z, r3.z) +
                          col(r0.w, r1.w, r2.w, r3.w);
    return (tile + 1) >> 1;
}

// 4x4 Hadamard SATD of a residual tile, satd4x4_scalar (encoder_motion.cpp:2936-2958).
__device__ __forceinline__ uint32_t satd4x4(const int d[16]) {
    int t[16];
#pragma unroll
    for (int y = 0; y < 4; ++y) {
        const int a0 = d[y * 4 + 0] + d[y * 4 + 3], a1 = d[y * 4 + 1] + d[y * 4 + 2];
        const int a2 = d[y * 4 + 1] - d[y * 4 + 2], a3 = d[y * 4 + 0] - d[y * 4 + 3];
        t[y * 4 + 0] = a0 + a1;
        t[y * 4 + 1] = a3 + a2;
        t[y * 4 + 2] = a0 - a1;
        t[y * 4 + 3] = a3 - a2;
    }
    uint32_t tile = 0;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        const int a0 = t[0 * 4 + x] + t[3 * 4 + x], a1 = t[1 * 4 + x] + t[2 * 4 + x];
        const int a2 = t[1 * 4 + x] - t[2 * 4 + x], a3 = t[0 * 4 + x] - t[3 * 4 + x];
        tile += (uint32_t)iabs(a0 + a1) + (uint32_t)iabs(a3 + a2) + (uint32_t)iabs(a0 - a1) + (uint32_t)iabs(a3 - a2);
    }
    return (tile + 1) >> 1;
}

}  // namespace vc1cu
