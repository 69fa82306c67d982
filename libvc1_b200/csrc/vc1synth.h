/* vc1synth.h - seeded synthetic 4:2:0 clip generator (see vc1synth.c). */
#ifndef VC1SYNTH_H
#define VC1SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vc1synth_cfg {
    int32_t width;            /* even */
    int32_t height;           /* even */
    int32_t frames;
    int32_t n_objects;        /* 0..64 */
    uint64_t seed;
    double global_range_x_px; /* per-frame global translation drawn in [-r, r] at quarter-pel */
    double global_range_y_px;
    int32_t obj_min;          /* rectangle side range, pixels */
    int32_t obj_max;
    double obj_vel_px;        /* object velocity drawn in [-v, v] px/frame at quarter-pel */
    double zoom;              /* per-frame zoom factor about the frame centre, 1.0 = none */
    double noise_sigma;       /* Gaussian (Irwin-Hall) noise standard deviation */
} vc1synth_cfg;

void vc1synth_default(vc1synth_cfg* c, int width, int height, int frames, uint64_t seed);

/* Mean of the background texture over frame 0 and the scale giving it standard deviation 40
 * (the normalisation every sample uses). */
void vc1synth_normalisation(const vc1synth_cfg* c, double* mean, double* scale);

/* Writes frames*W*H luma bytes to y and frames*(W/2)*(H/2) bytes to u and v (either may
 * be NULL). Returns 0 on success. */
int vc1synth_generate(const vc1synth_cfg* c, uint8_t* y, uint8_t* u, uint8_t* v);

#ifdef __cplusplus
}
#endif

#endif
