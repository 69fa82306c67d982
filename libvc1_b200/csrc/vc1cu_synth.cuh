// vc1cu_synth.cuh - launch interface of the device-side synthetic clip generator.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vc1synth_math.h"

namespace vc1cu {

constexpr int kSynthMaxFrames = 64;  // frames per vc1cu_synth_frames call

struct SynthOut {
    uint8_t* y;
    uint8_t* u;
    uint8_t* v;
    int pitch_y, pitch_c;
};

// Everything one generation launch reads besides the configuration (device memory).
struct SynthArgs {
    vs_plan plan;
    int first, count;
    const double* mean_scale;  // the background normalisation, written by the launch itself
    double gx[kSynthMaxFrames], gy[kSynthMaxFrames], zinv[kSynthMaxFrames];
    SynthOut out[kSynthMaxFrames];
};

// Normalisation terms (d_terms: ((W+1)/2) * ((H+1)/2) doubles), their ordered sum into
// d_mean_scale, then the frames. d_args->mean_scale must point at d_mean_scale.
cudaError_t launch_synth(const vc1synth_cfg& c, const SynthArgs* d_args, double* d_terms, double* d_mean_scale,
                         int count, int sm_count, cudaStream_t s);

}  // namespace vc1cu
