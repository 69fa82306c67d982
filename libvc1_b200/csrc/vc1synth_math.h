/*
 * vc1synth_math.h - the per-sample arithmetic and the clip plan of the synthetic clip
 * generator, shared by the C generator (vc1synth.c) and its CUDA form (vc1cu_synth.cu) so
 * that both produce the same bytes. Only +, -, *, /, floor and sqrt of IEEE doubles and
 * 64-bit integer hashing enter (C: -ffp-contract=off; CUDA: --fmad=false).
 */
#ifndef VC1SYNTH_MATH_H
#define VC1SYNTH_MATH_H

#include <math.h>
#include <stdint.h>

#include "vc1synth.h"

#ifdef __CUDACC__
#define VC1SYNTH_FN static __host__ __device__ __forceinline__
#else
#define VC1SYNTH_FN static inline
#endif

VC1SYNTH_FN uint64_t vs_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* uniform double in [0,1) from a 4-word key */
VC1SYNTH_FN double vs_hash_unit(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t h = vs_mix64(seed ^ vs_mix64(a ^ vs_mix64(b ^ vs_mix64(c))));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

VC1SYNTH_FN double vs_smooth(double t) { return t * t * (3.0 - 2.0 * t); }

VC1SYNTH_FN double vs_value_octave(uint64_t seed, int oct, double X, double Y, double pitch) {
    const double fx = floor(X / pitch), fy = floor(Y / pitch);
    const double tx = X / pitch - fx, ty = Y / pitch - fy;
    const int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    const double v00 = vs_hash_unit(seed, (uint64_t)oct, (uint64_t)ix, (uint64_t)iy);
    const double v10 = vs_hash_unit(seed, (uint64_t)oct, (uint64_t)(ix + 1), (uint64_t)iy);
    const double v01 = vs_hash_unit(seed, (uint64_t)oct, (uint64_t)ix, (uint64_t)(iy + 1));
    const double v11 = vs_hash_unit(seed, (uint64_t)oct, (uint64_t)(ix + 1), (uint64_t)(iy + 1));
    const double sx = vs_smooth(tx), sy = vs_smooth(ty);
    const double a = v00 + (v10 - v00) * sx;
    const double b = v01 + (v11 - v01) * sx;
    return a + (b - a) * sy;
}

VC1SYNTH_FN double vs_value_noise(uint64_t seed, double X, double Y) {
    return vs_value_octave(seed, 0, X, Y, 64.0) + 0.5 * vs_value_octave(seed, 1, X, Y, 16.0) +
           0.25 * vs_value_octave(seed, 2, X, Y, 4.0);
}

/* uniform integer in [-r, r] */
VC1SYNTH_FN int64_t vs_uniform_int(uint64_t seed, uint64_t a, uint64_t b, int64_t r) {
    if (r <= 0) return 0;
    const uint64_t span = (uint64_t)(2 * r + 1);
    return (int64_t)(vs_mix64(seed ^ vs_mix64(a * 0x1000193ull + b)) % span) - r;
}

typedef struct vs_obj {
    double x0, y0, vx, vy; /* top-left at frame 0 and velocity, pixels (quarter-pel grid) */
    int w, h;
    uint8_t u, v;
    uint64_t tex_seed;
} vs_obj;

/* The moving objects of a clip. */
typedef struct vs_plan {
    vs_obj objs[64];
    int n_objects;
} vs_plan;

/* Accumulated global translation of frames 0..T-1 (quarter-pel grid), in frame order. */
VC1SYNTH_FN void vs_global_track(const vc1synth_cfg* c, int T, double* gx, double* gy) {
    const uint64_t seed = c->seed;
    const int64_t rqx = (int64_t)floor(c->global_range_x_px * 4.0 + 0.5);
    const int64_t rqy = (int64_t)floor(c->global_range_y_px * 4.0 + 0.5);
    gx[0] = 0.0;
    gy[0] = 0.0;
    for (int t = 1; t < T; ++t) {
        gx[t] = gx[t - 1] + 0.25 * (double)vs_uniform_int(seed, 11, (uint64_t)t, rqx);
        gy[t] = gy[t - 1] + 0.25 * (double)vs_uniform_int(seed, 13, (uint64_t)t, rqy);
    }
}

/* The object list of cfg. */
VC1SYNTH_FN void vs_make_plan(const vc1synth_cfg* c, vs_plan* p) {
    const uint64_t seed = c->seed;
    const int W = c->width, H = c->height;
    const int64_t rv = (int64_t)floor(c->obj_vel_px * 4.0 + 0.5);
    p->n_objects = c->n_objects;
    for (int i = 0; i < c->n_objects; ++i) {
        vs_obj* o = &p->objs[i];
        const int span = c->obj_max - c->obj_min + 1;
        o->w = c->obj_min + (int)(vs_mix64(seed ^ vs_mix64(1000 + (uint64_t)i)) % (uint64_t)(span > 0 ? span : 1));
        o->h = c->obj_min + (int)(vs_mix64(seed ^ vs_mix64(2000 + (uint64_t)i)) % (uint64_t)(span > 0 ? span : 1));
        o->x0 = (double)(vs_mix64(seed ^ vs_mix64(3000 + (uint64_t)i)) % (uint64_t)(W > o->w ? W - o->w : 1));
        o->y0 = (double)(vs_mix64(seed ^ vs_mix64(4000 + (uint64_t)i)) % (uint64_t)(H > o->h ? H - o->h : 1));
        o->vx = 0.25 * (double)vs_uniform_int(seed, 5000, (uint64_t)i, rv);
        o->vy = 0.25 * (double)vs_uniform_int(seed, 6000, (uint64_t)i, rv);
        o->u = (uint8_t)(64 + vs_mix64(seed ^ vs_mix64(7000 + (uint64_t)i)) % 129);
        o->v = (uint8_t)(64 + vs_mix64(seed ^ vs_mix64(8000 + (uint64_t)i)) % 129);
        o->tex_seed = vs_mix64(seed ^ vs_mix64(9000 + (uint64_t)i));
    }
}

/* The topmost object covering (x, y) at frame t, or -1. */
VC1SYNTH_FN int vs_hit(const vs_plan* p, int t, int x, int y) {
    for (int i = p->n_objects - 1; i >= 0; --i) {
        const double ox = p->objs[i].x0 + p->objs[i].vx * t, oy = p->objs[i].y0 + p->objs[i].vy * t;
        if ((double)x >= ox && (double)x < ox + p->objs[i].w && (double)y >= oy && (double)y < oy + p->objs[i].h)
            return i;
    }
    return -1;
}

/* Luma sample (x, y) of frame t; mean/scale normalise the background texture, zinv is
 * 1/zoom^t (accumulated by repeated division, as the generator does) and (gxt, gyt) the
 * frame's global translation. */
VC1SYNTH_FN uint8_t vs_luma(const vc1synth_cfg* c, const vs_plan* p, int t, int x, int y, double mean, double scale,
                            double zinv, double gxt, double gyt) {
    const uint64_t seed = c->seed;
    const double cxm = 0.5 * (double)c->width, cym = 0.5 * (double)c->height;
    double v;
    const int hit = vs_hit(p, t, x, y);
    if (hit >= 0) {
        const double ox = p->objs[hit].x0 + p->objs[hit].vx * t, oy = p->objs[hit].y0 + p->objs[hit].vy * t;
        v = 128.0 + (vs_value_noise(p->objs[hit].tex_seed, (double)x - ox, (double)y - oy) - mean) * scale;
    } else {
        const double X = ((double)x - cxm) * zinv + cxm + gxt;
        const double Yc = ((double)y - cym) * zinv + cym + gyt;
        v = 128.0 + (vs_value_noise(seed, X, Yc) - mean) * scale;
    }
    if (c->noise_sigma > 0.0) {
        double s = 0.0;
        const uint64_t key = ((uint64_t)t << 40) ^ ((uint64_t)y << 20) ^ (uint64_t)x;
        for (int k = 0; k < 12; ++k) s += vs_hash_unit(seed ^ 0xA5A5A5A5ull, 77, key, (uint64_t)k);
        v += (s - 6.0) * c->noise_sigma;
    }
    double r = floor(v + 0.5);
    if (r < 0.0) r = 0.0;
    if (r > 255.0) r = 255.0;
    return (uint8_t)r;
}

/* Chroma pair of chroma sample (cxp, cy) of frame t. */
VC1SYNTH_FN void vs_chroma(const vc1synth_cfg* c, const vs_plan* p, int t, int cxp, int cy, uint8_t* uu, uint8_t* vv) {
    const int x = cxp * 2, y = cy * 2;
    const int hit = vs_hit(p, t, x, y);
    if (hit >= 0) {
        *uu = p->objs[hit].u;
        *vv = p->objs[hit].v;
    } else {
        *uu = (uint8_t)floor(128.0 + 40.0 * (double)x / (double)c->width - 20.0 + 0.5);
        *vv = (uint8_t)floor(128.0 + 40.0 * (double)y / (double)c->height - 20.0 + 0.5);
    }
}

#endif
