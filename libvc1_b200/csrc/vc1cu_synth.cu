// vc1cu_synth.cu - the seeded synthetic clip generator (vc1synth.c) on the device.
//
// Produces the same bytes as vc1synth_generate (the per-sample arithmetic is shared through
// vc1synth_math.h; IEEE doubles, no contraction), so training and evaluation workloads of the
// learned proposals are generated where they are consumed, with no host-to-device copy. The
// background normalisation is a sum over frame 0 in raster order: its terms are computed in
// parallel and added by one thread in that order, so the rounding matches the C generator.
#include <cuda_runtime.h>

#include <algorithm>

#include "vc1cu_synth.cuh"
#include "vc1synth_math.h"

namespace vc1cu {

// The normalisation samples of frame 0 (every 2nd pixel of every 2nd row, raster order).
__global__ void synth_norm_terms_kernel(const __grid_constant__ vc1synth_cfg c, double* terms) {
    const int sw = (c.width + 1) / 2, sh = (c.height + 1) / 2;
    const long n = (long)sw * sh;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int y = (int)(i / sw) * 2, x = (int)(i % sw) * 2;
        terms[i] = vs_value_noise(c.seed, (double)x, (double)y);
    }
}

// One thread adds the terms in raster order (sum and sum of squares), as vc1synth_normalisation.
__global__ void synth_norm_sum_kernel(const __grid_constant__ vc1synth_cfg c, const double* terms, double* mean_scale) {
    const int sw = (c.width + 1) / 2, sh = (c.height + 1) / 2;
    const long n = (long)sw * sh;
    double sum = 0.0, sumsq = 0.0;
    for (long i = 0; i < n; ++i) {
        const double v = terms[i];
        sum += v;
        sumsq += v * v;
    }
    const double mean = sum / (double)n;
    double var = sumsq / (double)n - mean * mean;
    if (var < 1e-12) var = 1e-12;
    mean_scale[0] = mean;
    mean_scale[1] = 40.0 / sqrt(var);
}

// One thread per luma sample of frames [first, first + count); chroma by the even rows' even
// columns. Frame i goes to out[i] (planes with the given pitches).
__global__ void synth_frames_kernel(const __grid_constant__ vc1synth_cfg c, const SynthArgs* a) {
    const int W = c.width, H = c.height;
    const long per = (long)W * H;
    const long total = per * a->count;
    const double mean = a->mean_scale[0], scale = a->mean_scale[1];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int f = (int)(i / per);
        const long r = i - (long)f * per;
        const int y = (int)(r / W), x = (int)(r % W);
        const int t = a->first + f;
        const SynthOut& o = a->out[f];
        o.y[(size_t)y * o.pitch_y + x] = vs_luma(&c, &a->plan, t, x, y, mean, scale, a->zinv[f], a->gx[f], a->gy[f]);
        if (!(y & 1) && !(x & 1)) {
            uint8_t uu, vv;
            vs_chroma(&c, &a->plan, t, x / 2, y / 2, &uu, &vv);
            o.u[(size_t)(y / 2) * o.pitch_c + x / 2] = uu;
            o.v[(size_t)(y / 2) * o.pitch_c + x / 2] = vv;
        }
    }
}

cudaError_t launch_synth(const vc1synth_cfg& c, const SynthArgs* d_args, double* d_terms, double* d_mean_scale,
                         int count, int sm_count, cudaStream_t s) {
    const long nterms = (long)((c.width + 1) / 2) * ((c.height + 1) / 2);
    synth_norm_terms_kernel<<<(int)std::min<long>((nterms + 255) / 256, 8L * sm_count), 256, 0, s>>>(c, d_terms);
    synth_norm_sum_kernel<<<1, 1, 0, s>>>(c, d_terms, d_mean_scale);
    const long total = (long)c.width * c.height * count;
    synth_frames_kernel<<<(int)std::min<long>((total + 255) / 256, 16L * sm_count), 256, 0, s>>>(c, d_args);
    return cudaGetLastError();
}

}  // namespace vc1cu
