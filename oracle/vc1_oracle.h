/*
 * vc1_oracle.h - CPU restatement of libvc1's encoder-analysis hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker, not the product: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it. Every function follows the reference
 * (blenheimears/libvc1 v0.2.69) line for line in behaviour; the file:line it restates is
 * cited beside each definition in vc1_oracle.c. Parity is pinned: tests/test_oracle_pin.py
 * compares this oracle with the reference's own code compiled from its sources
 * (oracle/_ref/libvc1ref.so) and with the reference's known-answer fixtures.
 */
#ifndef VC1_ORACLE_H
#define VC1_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/vc1cu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A frame as the reference holds it: tight planes, Y width x height, U/V (w/2) x (h/2). */
typedef struct vo_frame {
    int32_t w, h;
    const uint8_t* y;
    const uint8_t* u;
    const uint8_t* v;
} vo_frame;

/* Evaluation counters (the algorithmic op count of the roofline). */
typedef struct vo_counts {
    uint64_t int_sad_samples;     /* integer-MV SAD samples (mb_sad, integer qpel/bilinear) */
    uint64_t qpel1d_samples;      /* one-axis bicubic samples */
    uint64_t qpel2d_samples;      /* two-axis bicubic samples */
    uint64_t bilinear_samples;    /* fractional bilinear samples */
    uint64_t satd_tiles;          /* 4x4 Hadamard tiles */
    uint64_t frame_sad_samples;   /* whole-frame SAD samples of the global search */
    uint64_t xform_flops;         /* FP64 multiply+add of the forward transform */
    uint64_t quant_coeffs;        /* scalar_quantize_level calls */
    uint64_t macroblocks;         /* MBs analysed (one per MB per core pass) */
} vo_counts;

void vo_counts_reset(void);
void vo_counts_get(vo_counts* out);

/* primitives (CPU law; results equal the reference's scalar functions) */
uint64_t vo_mb_sad(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                   int dx, int dy, int stride);
uint64_t vo_block_sad_qpel(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0,
                           int y0, int bw, int bh, int xq, int yq);
uint64_t vo_block_sad_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0,
                             int y0, int bw, int bh, int xq, int yq, int mode);
uint64_t vo_block_satd_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int x0,
                              int y0, int bw, int bh, int xq, int yq, int mode);
uint64_t vo_frame_sad(const vo_frame* cur, const vo_frame* ref, int dx, int dy, int stride);
int vo_hidden_padding(const vc1cu_params* p, int x0, int y0, int bw, int bh, int xq, int yq, int mode,
                      int chroma);
/* shader law of src/shaders/vulkan_motion_cost.comp (no legality gates) */
uint64_t vo_shader_cost(const vo_frame* cur, const vo_frame* ref, int x0, int y0, int bw, int bh,
                        int sample_stride, int bilinear, int rnd, int metric, int xq, int yq);
void vo_predict_luma(const vc1cu_params* p, const vo_frame* ref, int x0, int y0, int bw, int bh, int xq,
                     int yq, int mode, uint8_t* dst, int dst_stride);

/* searches */
void vo_global_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int range,
                      int* dx, int* dy, uint64_t* sad);
void vo_integer_motion(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mx, int my,
                       const vc1cu_mv* field, int gdx, int gdy, int range, int* dx, int* dy,
                       uint64_t* sad);

/* whole core pass; seed NULL = unseeded */
int vo_analyze_p_core(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mode,
                      int allow_intra, const vc1cu_mv* seed, const vc1cu_panalysis* seed_distant,
                      vc1cu_panalysis* out);
/* This library's learned analysis pass (candidates, descent, fallback to the plain search). */
int vo_analyze_p_learned(const vc1cu_params* p, const vo_frame* cur, const vo_frame* ref, int mode, const vc1cu_mv* cands,
                         int hint_dx, int hint_dy, int fallback, uint8_t* flags, vc1cu_panalysis* out);

/* intensity compensation (fades) */
void vo_intensity_compensate(const vo_frame* ref, const vc1cu_intensity* ic, uint8_t* y, uint8_t* u, uint8_t* v);
void vo_estimate_intensity_comp(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, const vc1cu_mv* mvs,
                                vc1cu_intensity* out);

/* scene-change score (scene cut detection) */
int vo_zoom_coherent(const vc1cu_mv* mvs, int mbw, int mbh);
double vo_scene_change_score(const vc1cu_params* p, const vo_frame* f, const vo_frame* ref, int fade_compensation,
                             double scene_threshold);

/* B-picture analysis: the two core passes + the per-MB mode decision */
void vo_b_costs(const vc1cu_params* p, const vo_frame* f, const vo_frame* past, const vo_frame* future, int mx,
                int my, vc1cu_mv fm, vc1cu_mv bm, vc1cu_mv df, vc1cu_mv db, int mode, uint64_t out[5]);
void vo_b_predict(const vc1cu_params* p, const vo_frame* f, const vo_frame* past, const vo_frame* future,
                  const uint8_t* modes, const vc1cu_mv* fmv, const vc1cu_mv* bmv, int mode, uint8_t* dy, uint8_t* du,
                  uint8_t* dv);
int vo_analyze_b(const vc1cu_params* p, const vo_frame* cur, const vo_frame* past, const vo_frame* future,
                 const vc1cu_mv* anchor_mvs, const uint8_t* anchor_4mv, int fraction_num, int fraction_den,
                 int mode, vc1cu_banalysis* out);

/* prediction of an MV field (motion_compensate_mb / _4mv); dst planes tight */
void vo_motion_compensate(const vc1cu_params* p, const vo_frame* ref, const vc1cu_mv* mvs,
                          const vc1cu_mv* block_mvs, const uint8_t* use_4mv, int mode, uint8_t* dy,
                          uint8_t* du, uint8_t* dv);

/* transform + quantiser */
void vo_forward_part(const uint8_t* src, const uint8_t* pred, int w, int h, int x0, int y0, int bw,
                     int bh, double out[64]);
int vo_quantize_level(const vc1cu_params* p, double coeff);
void vo_forward_quant(const vc1cu_params* p, const vo_frame* src, const vo_frame* pred, int type_mask,
                      double* coeffs, int16_t* levels);

/* reconstruction: prediction + inverse-transformed dequantised levels of each block's type */
void vo_reconstruct(const vc1cu_params* p, const vo_frame* pred, const int16_t* levels, int type_mask,
                    const uint8_t* block_types, uint8_t* y, uint8_t* u, uint8_t* v);

/* in-loop deblocking (in place): the I-like all-edges filter and the P filter of the coded
 * blocks (block_mvs 4 per MB, cbp / tt 6 per MB, intra one bit per block) */
void vo_loop_filter_i(const vc1cu_params* p, uint8_t* y, uint8_t* u, uint8_t* v);
void vo_loop_filter_p(const vc1cu_params* p, uint8_t* y, uint8_t* u, uint8_t* v, const vc1cu_mv* block_mvs,
                      const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra);

/* overlap smoothing of a signed padded reconstruction in place (planes (mbw*16) x (mbh*16) luma,
 * half chroma, rows packed; flags per MB or all != 0), and its 8-bit store clamp(s + bias) into
 * a w x h frame (all MBs, or those mask flags) */
void vo_overlap_smooth(int mbw, int mbh, int32_t* y, int32_t* u, int32_t* v, const uint8_t* flags, int all);
void vo_store_signed(int mbw, int mbh, const int32_t* sy, const int32_t* su, const int32_t* sv, int bias,
                     const uint8_t* mask, int w, int h, uint8_t* y, uint8_t* u, uint8_t* v);

/* the throughput preset's transform type per MB (TransformType 1..4) */
void vo_fast_transform_types(const vc1cu_params* p, const vo_frame* src, const vo_frame* pred, uint8_t* types);

/* x87 extended-precision score emulation used by the GPU path, exposed for checking:
 * the long double value of sad + lambda*rate, as an integer scaled by 2^shift
 * (see vo_score_key in vc1_oracle.c). */
void vo_score_key(uint64_t sad, double lambda, uint64_t rate, int mant_bits, uint64_t* hi, uint64_t* lo);

#ifdef __cplusplus
}
#endif

#endif
