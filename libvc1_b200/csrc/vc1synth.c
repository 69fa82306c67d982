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

static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* uniform double in [0,1) from a 4-word key */
static double hash_unit(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t h = mix64(seed ^ mix64(a ^ mix64(b ^ mix64(c))));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

static double value_octave(uint64_t seed, int oct, double X, double Y, double pitch) {
    const double fx = floor(X / pitch), fy = floor(Y / pitch);
    const double tx = X / pitch - fx, ty = Y / pitch - fy;
    const int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    const double v00 = hash_unit(seed, (uint64_t)oct, (uint64_t)ix, (uint64_t)iy);
    const double v10 = hash_unit(seed, (uint64_t)oct, (uint64_t)(ix + 1), (uint64_t)iy);
    const double v01 = hash_unit(seed, (uint64_t)oct, (uint64_t)ix, (uint64_t)(iy + 1));
    const double v11 = hash_unit(seed, (uint64_t)oct, (uint64_t)(ix + 1), (uint64_t)(iy + 1));
    const double sx = smooth(tx), sy = smooth(ty);
    const double a = v00 + (v10 - v00) * sx;
    const double b = v01 + (v11 - v01) * sx;
    return a + (b - a) * sy;
}

static double value_noise(uint64_t seed, double X, double Y) {
    return value_octave(seed, 0, X, Y, 64.0) + 0.5 * value_octave(seed, 1, X, Y, 16.0) +
           0.25 * value_octave(seed, 2, X, Y, 4.0);
}

/* uniform integer in [-r, r] */
static int64_t uniform_int(uint64_t seed, uint64_t a, uint64_t b, int64_t r) {
    if (r <= 0) return 0;
    const uint64_t span = (uint64_t)(2 * r + 1);
    return (int64_t)(mix64(seed ^ mix64(a * 0x1000193ull + b)) % span) - r;
}

typedef struct obj {
    double x0, y0, vx, vy; /* top-left at frame 0 and velocity, pixels (quarter-pel grid) */
    int w, h;
    uint8_t u, v;
    uint64_t tex_seed;
} obj;

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

int vc1synth_generate(const vc1synth_cfg* c, uint8_t* Y, uint8_t* U, uint8_t* V) {
    const int W = c->width, H = c->height, T = c->frames;
    if (W <= 0 || H <= 0 || (W & 1) || (H & 1) || T <= 0 || c->n_objects < 0 || c->n_objects > 64)
        return 1;
    const uint64_t seed = c->seed;
    /* accumulated global translation per frame, quarter-pel grid */
    double* gx = (double*)malloc(sizeof(double) * (size_t)T);
    double* gy = (double*)malloc(sizeof(double) * (size_t)T);
    if (!gx || !gy) { free(gx); free(gy); return 2; }
    const int64_t rqx = (int64_t)floor(c->global_range_x_px * 4.0 + 0.5);
    const int64_t rqy = (int64_t)floor(c->global_range_y_px * 4.0 + 0.5);
    gx[0] = 0.0;
    gy[0] = 0.0;
    for (int t = 1; t < T; ++t) {
        gx[t] = gx[t - 1] + 0.25 * (double)uniform_int(seed, 11, (uint64_t)t, rqx);
        gy[t] = gy[t - 1] + 0.25 * (double)uniform_int(seed, 13, (uint64_t)t, rqy);
    }
    obj objs[64];
    const int64_t rv = (int64_t)floor(c->obj_vel_px * 4.0 + 0.5);
    for (int i = 0; i < c->n_objects; ++i) {
        obj* o = &objs[i];
        const int span = c->obj_max - c->obj_min + 1;
        o->w = c->obj_min + (int)(mix64(seed ^ mix64(1000 + (uint64_t)i)) % (uint64_t)(span > 0 ? span : 1));
        o->h = c->obj_min + (int)(mix64(seed ^ mix64(2000 + (uint64_t)i)) % (uint64_t)(span > 0 ? span : 1));
        o->x0 = (double)(mix64(seed ^ mix64(3000 + (uint64_t)i)) % (uint64_t)(W > o->w ? W - o->w : 1));
        o->y0 = (double)(mix64(seed ^ mix64(4000 + (uint64_t)i)) % (uint64_t)(H > o->h ? H - o->h : 1));
        o->vx = 0.25 * (double)uniform_int(seed, 5000, (uint64_t)i, rv);
        o->vy = 0.25 * (double)uniform_int(seed, 6000, (uint64_t)i, rv);
        o->u = (uint8_t)(64 + mix64(seed ^ mix64(7000 + (uint64_t)i)) % 129);
        o->v = (uint8_t)(64 + mix64(seed ^ mix64(8000 + (uint64_t)i)) % 129);
        o->tex_seed = mix64(seed ^ mix64(9000 + (uint64_t)i));
    }
    /* normalisation of the background texture over frame 0 (every 2nd pixel, raster order) */
    double sum = 0.0, sumsq = 0.0;
    long cnt = 0;
    for (int y = 0; y < H; y += 2)
        for (int x = 0; x < W; x += 2) {
            const double v = value_noise(seed, (double)x, (double)y);
            sum += v;
            sumsq += v * v;
            ++cnt;
        }
    const double mean = sum / (double)cnt;
    double var = sumsq / (double)cnt - mean * mean;
    if (var < 1e-12) var = 1e-12;
    const double scale = 40.0 / sqrt(var);
    const double cxm = 0.5 * (double)W, cym = 0.5 * (double)H;
    const int CW = W / 2, CH = H / 2;

#pragma omp parallel for schedule(static)
    for (int row = 0; row < T * H; ++row) {
        const int t = row / H, y = row % H;
        double zinv = 1.0;
        for (int k = 0; k < t; ++k) zinv = zinv / c->zoom;
        uint8_t* out = Y + (size_t)t * W * H + (size_t)y * W;
        for (int x = 0; x < W; ++x) {
            double v;
            int hit = -1;
            for (int i = c->n_objects - 1; i >= 0; --i) {
                const double ox = objs[i].x0 + objs[i].vx * t, oy = objs[i].y0 + objs[i].vy * t;
                if ((double)x >= ox && (double)x < ox + objs[i].w && (double)y >= oy && (double)y < oy + objs[i].h) {
                    hit = i;
                    break;
                }
            }
            if (hit >= 0) {
                const double ox = objs[hit].x0 + objs[hit].vx * t, oy = objs[hit].y0 + objs[hit].vy * t;
                v = 128.0 + (value_noise(objs[hit].tex_seed, (double)x - ox, (double)y - oy) - mean) * scale;
            } else {
                const double X = ((double)x - cxm) * zinv + cxm + gx[t];
                const double Yc = ((double)y - cym) * zinv + cym + gy[t];
                v = 128.0 + (value_noise(seed, X, Yc) - mean) * scale;
            }
            if (c->noise_sigma > 0.0) {
                double s = 0.0;
                const uint64_t key = ((uint64_t)t << 40) ^ ((uint64_t)y << 20) ^ (uint64_t)x;
                for (int k = 0; k < 12; ++k) s += hash_unit(seed ^ 0xA5A5A5A5ull, 77, key, (uint64_t)k);
                v += (s - 6.0) * c->noise_sigma;
            }
            double r = floor(v + 0.5);
            if (r < 0.0) r = 0.0;
            if (r > 255.0) r = 255.0;
            out[x] = (uint8_t)r;
        }
        if ((y & 1) == 0 && (U || V)) {
            const int cy = y / 2;
            for (int cxp = 0; cxp < CW; ++cxp) {
                const int x = cxp * 2;
                int hit = -1;
                for (int i = c->n_objects - 1; i >= 0; --i) {
                    const double ox = objs[i].x0 + objs[i].vx * t, oy = objs[i].y0 + objs[i].vy * t;
                    if ((double)x >= ox && (double)x < ox + objs[i].w && (double)y >= oy && (double)y < oy + objs[i].h) {
                        hit = i;
                        break;
                    }
                }
                uint8_t uu, vv;
                if (hit >= 0) {
                    uu = objs[hit].u;
                    vv = objs[hit].v;
                } else {
                    uu = (uint8_t)floor(128.0 + 40.0 * (double)x / (double)W - 20.0 + 0.5);
                    vv = (uint8_t)floor(128.0 + 40.0 * (double)y / (double)H - 20.0 + 0.5);
                }
                if (U) U[(size_t)t * CW * CH + (size_t)cy * CW + cxp] = uu;
                if (V) V[(size_t)t * CW * CH + (size_t)cy * CW + cxp] = vv;
            }
        }
    }
    free(gx);
    free(gy);
    return 0;
}
