// vc1cu_lp.cuh - the learned motion-vector proposals: network geometry, buffers and launches.
//
// The network reads the current and reference pictures at quarter resolution (one sample per
// 4x4 luma block, so a macroblock is 4x4 samples) together with the picture's dominant
// translation g (a coarse-to-fine search: 1/16 resolution, then quarter resolution, then full
// resolution at stride 2, each about 4x the previous level's answer), runs four 3x3 convolutions of 32 channels with ReLU (BF16 operands, FP32
// accumulation in tensor memory, tcgen05.mma), mean-pools each macroblock's 16 samples and
// maps them (a 32 -> 8 projection) to two hypotheses: "the block moves with the zero vector"
// and "the block moves with g", each with a logit and a regressed offset. The K = 4
// candidates of a macroblock are both hypotheses' refined vectors and the two raw hints,
// ordered by the logits; an exact refinement on the full-resolution pictures follows.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vc1cu {

constexpr int kLpCin0 = 16;    // input feature channels (9 used, the rest zero)
constexpr int kLpC = 32;       // channels of every convolution's output
constexpr int kLpLayers = 4;   // 3x3 convolutions
constexpr int kLpHead = 8;     // projection outputs: logit0, logit1, d0x, d0y, d1x, d1y, 2 unused
constexpr int kLpK = 4;        // candidates per macroblock
constexpr int kLpTile = 128;   // output samples per convolution tile (a quarter-res row segment)
constexpr int kLpOffScale = 4; // a regressed offset of 1.0 is 4 full-resolution pixels
constexpr int kLpOffClip = 4;  // offsets are trained in [-4, 4] (+-16 pixels about the hint)

// Parameter counts (fp32 master copy order: for each layer W[co][tap][ci] then b[co]; then the
// projection Wh[j][c] and bh[j]).
constexpr int lp_cin(int l) { return l == 0 ? kLpCin0 : kLpC; }
constexpr int lp_wcount(int l) { return kLpC * 9 * lp_cin(l); }
constexpr int lp_param_count() {
    return lp_wcount(0) + lp_wcount(1) + lp_wcount(2) + lp_wcount(3) + 4 * kLpC + kLpHead * kLpC + kLpHead;
}

// Quarter-resolution raster of a picture: its macroblock raster times 4.
struct LpGeom {
    int W, H;      // full-resolution coding raster
    int W4, H4;    // 4 * mbw, 4 * mbh
    int mbw, mbh;
    int range;     // motion search range (pixels) the hint search covers
};

struct LpConvArgs {
    const void* x;        // A source: NHWC bf16 activations, CA channels
    const void* wb;       // B operand, packed [9][CA/8][32][8] bf16
    const float* bias;    // forward: per output channel
    void* y;              // output: NHWC bf16, 32 channels
    const void* act;      // dgrad: this layer's forward input (NHWC bf16, 32 ch): ReLU mask
    float* dbias;         // dgrad: the input layer's bias gradient accumulates here
    int W4, H4, frames;
    int* err;             // set when a bounded wait gives up
};

struct LpWgradArgs {
    const void* x;        // the layer's forward input, NHWC bf16, CIN channels
    const void* dz;       // gradient at the layer's pre-activation, NHWC bf16, 32 channels
    float* dw;            // [co][tap][ci] fp32, accumulated
    int W4, H4, frames;
    int* err;
};

// Per-sample state of the hint search and the features.
struct LpHeadArgs {
    const void* y4;       // last convolution's output, NHWC bf16 32 ch, `frames` pictures
    const float* wh;      // projection [8][32] and bias [8]
    const float* bh;
    const int2* hint;     // per picture: g (pixels)
    const int2* labels;   // per picture and MB: integer-pixel vector of the plain search (training)
    int2* cands;          // per picture and MB: K candidates (inference), may be null
    float* loss;          // training: summed loss
    float* dwh;           // training: projection gradients
    float* dbh;
    void* dz4;            // training: gradient at the last convolution's pre-activation (bf16)
    float* db4;           // training: its bias gradient
    int W4, H4, mbw, mbh, frames, range;
    float inv_count;      // 1 / (macroblocks in the batch)
};

cudaError_t lp_launch_downsample(const uint8_t* cur, int cur_pitch, const uint8_t* ref, int ref_pitch,
                                 const LpGeom& g, uint8_t* cur4, uint8_t* ref4, cudaStream_t s);
cudaError_t lp_launch_hint(const uint8_t* cur, int cur_pitch, const uint8_t* ref, int ref_pitch, const LpGeom& g,
                           const uint8_t* cur4, const uint8_t* ref4, unsigned long long* scratch, int2* hint,
                           unsigned long long* hint_sad, cudaStream_t s);
cudaError_t lp_launch_features(const uint8_t* ref, int ref_pitch, const LpGeom& g, const uint8_t* cur4,
                               const uint8_t* ref4, const int2* hint, void* x0, cudaStream_t s);
cudaError_t lp_launch_conv(int ca, bool dgrad, const LpConvArgs& a, int sm_count, cudaStream_t s);
cudaError_t lp_launch_wgrad(int cin, const LpWgradArgs& a, int sm_count, cudaStream_t s);
cudaError_t lp_launch_head(const LpHeadArgs& a, cudaStream_t s);
cudaError_t lp_launch_labels(const int2* mvs, int n, int2* labels, cudaStream_t s);
cudaError_t lp_launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                           float eps, int step, cudaStream_t s);
// fp32 master parameters -> the packed bf16 B operands of every layer (forward and dgrad).
cudaError_t lp_launch_pack(const float* master, void* fwd_b, void* dgrad_b, cudaStream_t s);
size_t lp_fwd_b_elems(int l);    // bf16 elements of layer l's forward B operand
size_t lp_dgrad_b_elems(int l);  // of its dgrad B operand (0 for the first layer)
size_t lp_conv_smem(int ca);     // dynamic shared memory of one convolution CTA
size_t lp_wgrad_smem(int cin);

}  // namespace vc1cu
