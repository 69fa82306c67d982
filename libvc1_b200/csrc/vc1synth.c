/*
 * vc1synth.c - seeded synthetic 4:2:0 clip generator for the analysis workloads.
 *
 * Content (one clip):
 *   - background: 3-octave value noise (lattice pitches 64/16/4 px, amplitudes 1, 1/2, 1/4,
 *     smoothstep-weighted bilinear lattice interpolation), normalised to mean 128 and
 *     standard deviation 40 over frame 0, evaluated analytically at the translated (and
 *     optionally zoomed) canvas coordinate so quarter-pel motion needs no resampling;
 *   - a global translation per frame drawn uniformly on the quarter-pel grid
 *     (independent x/y ranges), accumulated over frames, plus a per-frame zoom factor;
 *   - opaque rectangles with their own noise texture and constant velocity, drawn in
 *     z-order, each with a constant chroma tint;
 *   - chroma: U = 128 + 40*x/W - 20, V = 128 + 40*y/H - 20 outside objects;
 *   - Gaussian sensor noise from an Irwin-Hall sum of 12 uniforms, then round and clip.
 * Only +, -, *, /, floor and sqrt enter, so the output is bit-identical on every IEEE
 * host; the random source is a counter-based splitmix64 hash, so rows can be generated
 * in any order or in parallel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vc1synth.h"
#include "vc1synth_math.h"

void vc1synth_default(vc1synth_cfg* c, int width, int height, int frames, uint64_t seed) {
    memset(c, 0, sizeof *c);
    c->width = width;
    c->height = height;
    c->frames = frames;
    c->seed = seed;
    c->global_range_x_px = 6.75;
    c->global_range_y_px = 6.75;
    c->n_objects = 4;
    c->obj_min = 32;
    c->obj_max = 96;
    c->obj_vel_px = 3.0;
    c->zoom = 1.0;
    c->noise_sigma = 2.0;
}

/* Mean of the background texture over frame 0 (every 2nd pixel, raster order) and the scale
 * that gives it standard deviation 40. */
void vc1synth_normalisation(const vc1synth_cfg* c, double* mean_out, double* scale_out) {
    const int W = c->width, H = c->height;
    double sum = 0.0, sumsq = 0.0;
    long cnt = 0;
    for (int y = 0; y < H; y += 2)
        for (int x = 0; x < W; x += 2) {
            const double v = vs_value_noise(c->seed, (double)x, (double)y);
            sum += v;
            sumsq += v * v;
            ++cnt;
        }
    const double mean = sum / (double)cnt;
    double var = sumsq / (double)cnt - mean * mean;
    if (var < 1e-12) var = 1e-12;
    *mean_out = mean;
    *scale_out = 40.0 / sqrt(var);
}

int vc1synth_generate(const vc1synth_cfg* c, uint8_t* Y, uint8_t* U, uint8_t* V) {
    const int W = c->width, H = c->height, T = c->frames;
    if (W <= 0 || H <= 0 || (W & 1) || (H & 1) || T <= 0 || c->n_objects < 0 || c->n_objects > 64)
        return 1;
    /* accumulated global translation per frame, quarter-pel grid */
    double* gx = (double*)malloc(sizeof(double) * (size_t)T);
    double* gy = (double*)malloc(sizeof(double) * (size_t)T);
    if (!gx || !gy) { free(gx); free(gy); return 2; }
    vs_global_track(c, T, gx, gy);
    vs_plan plan;
    vs_make_plan(c, &plan);
    double mean, scale;
    vc1synth_normalisation(c, &mean, &scale);
    const int CW = W / 2, CH = H / 2;
#pragma omp parallel for schedule(static)
    for (int row = 0; row < T * H; ++row) {
        const int t = row / H, y = row % H;
        double zinv = 1.0;
        for (int k = 0; k < t; ++k) zinv = zinv / c->zoom;
        uint8_t* out = Y + (size_t)t * W * H + (size_t)y * W;
        for (int x = 0; x < W; ++x) out[x] = vs_luma(c, &plan, t, x, y, mean, scale, zinv, gx[t], gy[t]);
        if ((y & 1) == 0 && (U || V)) {
            const int cy = y / 2;
            for (int cxp = 0; cxp < CW; ++cxp) {
                uint8_t uu, vv;
                vs_chroma(c, &plan, t, cxp, cy, &uu, &vv);
                if (U) U[(size_t)t * CW * CH + (size_t)cy * CW + cxp] = uu;
                if (V) V[(size_t)t * CW * CH + (size_t)cy * CW + cxp] = vv;
            }
        }
    }
    free(gx);
    free(gy);
    return 0;
}
