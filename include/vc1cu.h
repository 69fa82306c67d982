/*
 * vc1cu.h - C ABI of the B200 (sm_100a) backend for libvc1's encoder-analysis hot path.
 *
 * The library (libvc1_b200/libvc1cu.so) replaces these pieces of libvc1 (v0.2.69):
 *
 *   1. the motion-compute backend interface that the Vulkan path implements
 *      (src/vulkan_compute.h:26-60, class VulkanComputeContext), as vc1cu_open /
 *      vc1cu_close / vc1cu_device_name / vc1cu_device_index / vc1cu_score_motion_batch /
 *      vc1cu_counters / vc1cu_reset_counters;
 *   2. one whole-picture motion-analysis core pass,
 *      Vc1Encoder::analyze_p_picture_core (src/encoder_motion.cpp:47-442), as
 *      vc1cu_analyze_p_core (host buffers) and vc1cu_core_passes (device-resident batch);
 *   3. the forward 8x8/8x4/4x8/4x4 transform + scalar quantiser of a motion-compensated
 *      prediction, forward_transform_residual_part + scalar_quantize_level
 *      (src/encoder_transform.cpp:935-1045, :1067-1085), as vc1cu_forward_quant;
 *   4. the B-picture analysis, Vc1Encoder::analyze_b_picture_mode (encoder_motion.cpp:753-1005),
 *      as vc1cu_analyze_b_picture / vc1cu_b_decide;
 *   5. the fade and scene-cut analysis: estimate_intensity_comp and
 *      intensity_compensated_reference (encoder_motion_compensation.cpp:175-348) and
 *      scene_change_score (encoder_motion.cpp:599-676);
 *   6. the transform RD, Vc1Encoder::choose_transform_mb (encoder_transform.cpp:1605-1780), and
 *      its DQUANT search, choose_dquant_transform_mb (encoder_aq.cpp:280-404), as
 *      vc1cu_fast_transform_types / vc1cu_choose_transform / vc1cu_choose_dquant;
 *   7. the picture-level motion-mode decisions, analyze_p_picture (encoder_motion.cpp:524-597)
 *      with estimate_p_motion_bits and sampled_p_mode_rd, and the quarter-pel versus bilinear
 *      choice of analyze_b_picture (:1006-1095), as vc1cu_analyze_p_picture /
 *      vc1cu_p_motion_bits / vc1cu_b_mode_rd;
 *   8. the reconstruction side: the B prediction, the inverse transforms, the I picture's intra
 *      reconstruction (reconstruct_i_signed_padded, encoder_encode.cpp:814-887), the in-loop
 *      deblocking (Advanced and Main Profile) and overlap smoothing, as vc1cu_b_predict /
 *      vc1cu_reconstruct / vc1cu_reconstruct_intra / vc1cu_loop_filter_i / _p / _p_main /
 *      vc1cu_overlap_smooth / vc1cu_store_signed.
 *
 * Conventions: every function is extern "C", returns an int status (VC1CU_OK on
 * success), never throws, and records a message retrievable with vc1cu_last_error().
 * There is no CPU fallback: a CUDA failure is reported, not hidden. Motion vectors are
 * quarter-pel int32 pairs laid out exactly like VulkanMotionCandidate
 * (src/vulkan_compute.h:11-14). Costs are uint64 like the reference's CPU law.
 * Frames are 8-bit 4:2:0 planes with tight strides (Y: width, U/V: width/2), the
 * layout of libvc1::Frame (src/encoder_internal.h:68-71).
 *
 * A context is bound to one CUDA device and owns one CUDA stream for its work, plus one for
 * frame uploads (each after the last work that used its slot; later work waits for it) and one
 * for result reads (each after the launch that wrote its slot); calls on one context
 * are serialised by an internal mutex (the reference serialises its Vulkan context the
 * same way, src/vulkan_compute.cpp:385).
 */
#ifndef VC1CU_H
#define VC1CU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
enum {
    VC1CU_OK = 0,
    VC1CU_ERR_ARG = 1,         /* invalid argument (size, id, mode, null pointer) */
    VC1CU_ERR_CUDA = 2,        /* a CUDA runtime call or kernel launch failed */
    VC1CU_ERR_TIMEOUT = 3,     /* a bounded device-side wait gave up (wavefront dependency) */
    VC1CU_ERR_OOM = 4,         /* device or pinned host allocation failed */
    VC1CU_ERR_STATE = 5,       /* e.g. a frame id that was never uploaded */
    VC1CU_ERR_UNSUPPORTED = 6  /* a configuration this backend does not implement */
};

typedef struct vc1cu_ctx vc1cu_ctx;

/* Quarter-pel motion vector; same layout as VulkanMotionCandidate / Vc1Encoder::MotionVector. */
typedef struct vc1cu_mv {
    int32_t xq;
    int32_t yq;
} vc1cu_mv;

/* VulkanMotionMetric (src/vulkan_compute.h:16). */
enum { VC1CU_METRIC_SAD = 0, VC1CU_METRIC_SATD = 1 };

/* Vc1Encoder::ProgressiveMvMode (src/encoder_internal.h:335). */
enum {
    VC1CU_MV_QPEL = 0,
    VC1CU_MV_HPEL = 1,
    VC1CU_MV_HPEL_BILINEAR = 2,
    VC1CU_MV_MIXED = 3
};

/* Cost law for vc1cu_score_motion_batch_law. */
enum {
    VC1CU_LAW_SHADER = 0, /* exactly src/shaders/vulkan_motion_cost.comp: no legality gates */
    VC1CU_LAW_CPU = 1     /* the CPU law of block_sad_motion / mb_sad (encoder_motion.cpp:2197-2933):
                             hidden-padding and odd-half-pel candidates cost UINT64_MAX/4 */
};

/*
 * The subset of libvc1::EncoderConfig (src/encoder_internal.h:223-315) that the analysis
 * path reads. Field meanings and defaults follow vc1_param_default
 * (src/encoder_api_helpers.cpp:27-52); vc1cu_params_default fills them.
 * Only Advanced Profile progressive syntax is implemented.
 */
typedef struct vc1cu_params {
    int32_t width;              /* even internal coding raster, EncoderConfig::width */
    int32_t height;             /* EncoderConfig::height */
    int32_t display_width;      /* 0 = width; EncoderConfig::display_width */
    int32_t display_height;     /* 0 = height */
    int32_t pqindex;            /* 1..31 */
    int32_t halfqp;             /* HALFQP bit, 0/1 */
    int32_t nonuniform;         /* 0 = uniform quantiser, 1 = non-uniform */
    int32_t search_range;       /* motion_search_range, integer pixels, 0..1024 */
    int32_t local_search_range; /* motion_local_search_range */
    int32_t me_algorithm;       /* 0 = UMH, 1 = diamond (vc1_me_algorithm_e) */
    int32_t me_quality;         /* 0 SAD, 1 RATE, 2 SATD (vc1_me_quality_e); RD is not implemented */
    int32_t subpel;             /* subpixel_refinement */
    int32_t fast_subpel;        /* fast_subpixel_refinement */
    int32_t subpel_range;       /* subpixel_refinement_range, integer pixels */
    int32_t long_range_mode;    /* vc1_long_range_search_mode_e */
    int32_t rnd;                /* rndctrl */
    int32_t disable_p_intra;    /* debug_disable_p_intra */
    int32_t disable_b_intra;    /* debug_disable_b_intra */
    double distant_match_max_mae;  /* default 255.0 */
    double inter_intra_threshold;  /* default 0.80 */
} vc1cu_params;

/*
 * Per-macroblock result of one core pass (Vc1Encoder::PAnalysis, src/encoder_internal.h:346-370).
 * For vc1cu_analyze_p_core these are HOST arrays of mbw*mbh entries (block_mvs: 4 per MB,
 * raster order of the four luma blocks); any array pointer may be NULL to skip it.
 * The scalar fields are written by the call.
 */
typedef struct vc1cu_panalysis {
    vc1cu_mv* mvs;
    vc1cu_mv* block_mvs;
    uint8_t* use_4mv;
    uint8_t* use_intra;
    uint64_t* screen_sads;
    double* inter_intra_cost_ratio;
    double* distant_local_mae;
    double* distant_candidate_mae;
    uint8_t* distant_match_decision;
    double mean_abs_residual;
    double rate_complexity;
    uint64_t motion_sad;
    uint64_t moved_macroblocks;
    uint64_t fractional_chroma_macroblocks;
    uint64_t four_mv_macroblocks;
    uint64_t intra_macroblocks;
    int32_t global_dx;          /* whole-frame translation of the unseeded pass */
    int32_t global_dy;
    uint64_t global_full_sad;
} vc1cu_panalysis;

/* VulkanComputeCounters (src/vulkan_compute.h:18-24); device time instead of submit-wait. */
typedef struct vc1cu_counters {
    uint64_t dispatches;
    uint64_t candidates;
    uint64_t frame_uploads;
    uint64_t frame_upload_bytes;
    uint64_t submit_wait_nanoseconds;
    uint64_t macroblocks_analysed;
    uint64_t kernel_launches;   /* every kernel this library launched */
} vc1cu_counters;

/* Device time of each kernel family, summed over launches since the last reset, from CUDA
 * events recorded on the context's stream around every launch (vc1cu_set_timing(ctx, 1)). */
typedef struct vc1cu_timing {
    double core_ms;      /* core_pass_kernel */
    double global_ms;    /* global translation search (scoring + fold launches) */
    double totals_ms;    /* per-pass totals */
    double mc_ms;        /* motion compensation */
    double xform_ms;     /* forward transform + quantiser */
    uint64_t core_launches;
    uint64_t xform_launches;
    double b_ms;         /* B-picture decision (b_cost_kernel + b_decide_kernel) */
    double ic_ms;        /* intensity-compensation estimate */
} vc1cu_timing;

/* ---- context (VulkanComputeContext::create / device_name / device_index) ---------- */

/* Replaces VulkanComputeContext::create (src/vulkan_compute.h:28-29). device = -1 picks
 * the current CUDA device. */
int vc1cu_open(int device, vc1cu_ctx** out);
int vc1cu_close(vc1cu_ctx* ctx);
/* VulkanComputeContext::device_name / device_index (src/vulkan_compute.h:35-36). */
const char* vc1cu_device_name(const vc1cu_ctx* ctx);
int vc1cu_device_index(const vc1cu_ctx* ctx);
/* Message of the last failing call on this context (or of vc1cu_open when ctx is NULL). */
const char* vc1cu_last_error(const vc1cu_ctx* ctx);
/* VulkanComputeContext::counters / reset_counters (src/vulkan_compute.h:53-54). */
int vc1cu_counters_get(const vc1cu_ctx* ctx, vc1cu_counters* out);
int vc1cu_reset_counters(vc1cu_ctx* ctx);

/*
 * Test hooks of the wavefront waits' failure path (no counterpart in the reference, whose CPU
 * loop has no waits). A core-pass macroblock waits for its left, top-left, top and top-right
 * neighbours' done flags; a wait gives up after 2^log2_polls polls (default 24, a few seconds),
 * aborts the launch and makes the call that reads its results fail with VC1CU_ERR_TIMEOUT and a
 * message naming the first waiting work item ("pass P of its launch, macroblock M") and its
 * lanes still waiting. The context stays usable: the next call starts clean.
 * vc1cu_debug_set_wait_limit sets the limit (6..24) for every later core launch.
 * vc1cu_debug_withhold_publish makes the NEXT core launch skip publishing the done flag of one
 * work item (pass_index within that launch, macroblock index mb); (-1, -1) cancels it.
 */
int vc1cu_debug_set_wait_limit(vc1cu_ctx* ctx, int log2_polls);
int vc1cu_debug_withhold_publish(vc1cu_ctx* ctx, int pass_index, int mb);

/* Turns per-launch event timing on (1) or off (0); vc1cu_timing_get synchronises the
 * context stream and returns the sums; vc1cu_reset_counters clears them. */
int vc1cu_set_timing(vc1cu_ctx* ctx, int enable);
int vc1cu_timing_get(vc1cu_ctx* ctx, vc1cu_timing* out);
/* The CUDA stream (cudaStream_t) every launch of this context is ordered on. */
void* vc1cu_stream(const vc1cu_ctx* ctx);
/* Measures this device's 32-bit integer lane-op throughput (ops/s) with a dependency-free
 * add/xor kernel: the denominator of the analysis kernels' roofline. */
int vc1cu_measure_int32_peak(vc1cu_ctx* ctx, double* ops_per_second);
/* Measures this device's FP64 throughput (flops/s, a fused multiply-add counted as two) with a
 * dependency-free FMA kernel: the denominator of the transform kernel's roofline. */
int vc1cu_measure_fp64_peak(vc1cu_ctx* ctx, double* flops_per_second);
/* The index-checked build of this library (libvc1cu_checked.so, compiled with
 * -DVC1CU_INDEX_CHECK) tests every guarded access of the analysis kernels against its buffer
 * (search window, stage key array, first-visit bitset, neighbour, candidate and signature
 * tables, work items, window staging), counts violations and skips them. This returns the count
 * and the first violation (site << 40 | index, sites as in vc1cu_core.cu's IndexSite) since the
 * last reset, process-wide; with reset != 0 it clears them. Other builds return
 * VC1CU_ERR_UNSUPPORTED. */
int vc1cu_debug_index_faults(unsigned int* count, unsigned long long* first, int reset);

/* Fills the defaults of vc1_param_default for a width x height raster. */
void vc1cu_params_default(vc1cu_params* p, int width, int height);

/* ---- candidate scoring (VulkanComputeContext::score_motion_batch) ----------------- */

/*
 * Replaces VulkanComputeContext::score_motion_batch (src/vulkan_compute.h:42-51), with
 * the shader's law (src/shaders/vulkan_motion_cost.comp:109-183): SAD at sample_stride
 * (costs x stride^2) or 4x4 Hadamard SATD, VC-1 bicubic or bilinear interpolation with
 * rounding control, clamped edge sampling. cur/ref are host luma planes; they are copied
 * to the device when not already cached (key: pointer, size and a sampled fingerprint,
 * as the Vulkan backend does, src/vulkan_compute.cpp:30-45, :194-231). costs has n entries.
 * n == 0 is a no-op. Batches above 4,194,240 candidates are rejected like the reference.
 */
int vc1cu_score_motion_batch(vc1cu_ctx* ctx, const uint8_t* cur, const uint8_t* ref,
                             int width, int height, int x0, int y0, int bw, int bh,
                             int sample_stride, int bilinear, int rnd, int metric,
                             const vc1cu_mv* candidates, size_t n, uint64_t* costs);

/*
 * Same, choosing the cost law. With VC1CU_LAW_CPU, p supplies the display raster and the
 * results equal Vc1Encoder::block_sad_motion / block_satd_motion / mb_sad (the reference's
 * scalar path; encoder_motion.cpp:2197-2285, :2286-2933, :2962-3042).
 */
int vc1cu_score_motion_batch_law(vc1cu_ctx* ctx, const vc1cu_params* p, int law,
                                 const uint8_t* cur, const uint8_t* ref, int x0, int y0,
                                 int bw, int bh, int sample_stride, int mode, int metric,
                                 const vc1cu_mv* candidates, size_t n, uint64_t* costs);

/* ---- frames resident in HBM ---------------------------------------------------------- */

/* Copies one 4:2:0 frame (host planes, tight strides) into frame slot frame_id
 * (0 <= frame_id < 4096). u/v may be NULL (chroma then reads as 128). The copy runs on the
 * context's upload stream once the work already enqueued that uses the slot is done, so it
 * overlaps work on other slots; everything enqueued after this call sees the new frame. From
 * pinned host memory the call returns at once and the planes must stay unchanged until that
 * later work has started (or vc1cu_synchronize); from pageable memory it returns once staged. */
int vc1cu_upload_frame(vc1cu_ctx* ctx, int frame_id, const uint8_t* y, const uint8_t* u,
                       const uint8_t* v, int width, int height);
/*
 * Seeded synthetic clip content generated on the device (no counterpart in the reference): the
 * benchmark workloads' generator, bit-identical to the host generator of this library
 * (libvc1_b200/csrc/vc1synth.c): 3-octave value-noise background with a per-frame global
 * translation and zoom, moving textured rectangles, Irwin-Hall sensor noise. Layout mirrors
 * vc1synth_cfg.
 */
typedef struct vc1cu_synth_cfg {
    int32_t width;             /* even */
    int32_t height;            /* even */
    int32_t frames;            /* length of the clip the frames belong to */
    int32_t n_objects;         /* 0..64 */
    uint64_t seed;
    double global_range_x_px;  /* per-frame global translation drawn in [-r, r] at quarter-pel */
    double global_range_y_px;
    int32_t obj_min;           /* rectangle side range, pixels */
    int32_t obj_max;
    double obj_vel_px;         /* object velocity drawn in [-v, v] px/frame at quarter-pel */
    double zoom;               /* per-frame zoom about the frame centre, 1.0 = none */
    double noise_sigma;        /* Gaussian (Irwin-Hall) noise standard deviation */
} vc1cu_synth_cfg;

/* Frames first .. first+count-1 (count 1..64) of the clip cfg describes into frame slots
 * frame_id0 .. frame_id0+count-1. Asynchronous on the context stream. */
int vc1cu_synth_frames(vc1cu_ctx* ctx, const vc1cu_synth_cfg* cfg, int first, int count, int frame_id0);

/* Reads a frame slot back (for tests). */
int vc1cu_download_frame(vc1cu_ctx* ctx, int frame_id, uint8_t* y, uint8_t* u, uint8_t* v);

/* ---- whole-picture core pass (Vc1Encoder::analyze_p_picture_core) ------------------ */

/*
 * One analyze_p_picture_core pass of cur_id against ref_id, synchronous, host outputs.
 * mode: VC1CU_MV_*; allow_intra: the P-intra proxy (encoder_motion.cpp:387-414);
 * seed_mvs: NULL for the unseeded pass (global search + UMH/diamond + staged refinement),
 * else mbw*mbh host MVs of the shared qpel seed (encoder_motion.cpp:119-131). For a
 * seeded pass, seed_distant (may be NULL) carries the seed pass's distant_* arrays, which
 * the reference copies through unchanged (encoder_motion.cpp:100-104).
 */
int vc1cu_analyze_p_core(vc1cu_ctx* ctx, const vc1cu_params* p, int cur_id, int ref_id,
                         int mode, int allow_intra, const vc1cu_mv* seed_mvs,
                         const vc1cu_panalysis* seed_distant, vc1cu_panalysis* out);

/*
 * Device-resident batch form. Every pass in the batch is independent of the others; all
 * of them run in ONE persistent launch fed by a macroblock-row work queue (wavefront
 * order inside each picture). Results stay on the device in result slot out_slot
 * (0 <= slot < 4096); a seeded pass names the slot of its seed. Asynchronous on the
 * context's stream; vc1cu_synchronize waits for it.
 */
typedef struct vc1cu_pass {
    int32_t cur_id;
    int32_t ref_id;
    int32_t mode;
    int32_t allow_intra;
    int32_t seed_slot;   /* -1 = unseeded */
    int32_t out_slot;
    int32_t pqindex;     /* 0 = params->pqindex; else this picture's PQINDEX (1..31) */
} vc1cu_pass;

int vc1cu_core_passes(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_pass* passes, int n);
/*
 * Passes over pictures of different sizes (many clips) in ONE persistent launch: params holds one
 * parameter block per pass (its raster, display crop, PQINDEX, rounding control); the search
 * configuration (ranges, algorithm, quality, sub-pel and long-range settings, thresholds) must be
 * the same in all of them. A pass may be seeded by another pass of the same call (a picture's
 * seed pass, mode passes and final pass together), as in vc1cu_core_passes. The work queue
 * interleaves every pass's wavefront, so no picture waits for another. Asynchronous.
 */
int vc1cu_core_passes_multi(vc1cu_ctx* ctx, const vc1cu_params* params, const vc1cu_pass* passes, int n);

/*
 * CUDA graphs of the context's work (no counterpart in the reference, whose GOP workers call the
 * analysis per picture): vc1cu_graph_begin opens a capture of the context stream; the
 * asynchronous calls that follow (vc1cu_core_passes[_multi], vc1cu_motion_compensate,
 * vc1cu_forward_quant_device, vc1cu_reconstruct, vc1cu_synth_frames, ...) are recorded, not run;
 * vc1cu_graph_end instantiates them as graph *graph_id. vc1cu_graph_launch replays it on the
 * context stream (the result slots it writes become readable as after the recorded calls), so a
 * GOP's launches cost one host call. Each launch shape must have run once before it is captured
 * (the work-item tables and slots are built outside captures); calls that wait for the device
 * (reads, synchronous calls) fail inside a capture and close it. Core passes in a graph clear their
 * macroblock done flags at every replay.
 */
int vc1cu_graph_begin(vc1cu_ctx* ctx);
int vc1cu_graph_end(vc1cu_ctx* ctx, int* graph_id);
int vc1cu_graph_launch(vc1cu_ctx* ctx, int graph_id);
int vc1cu_graph_destroy(vc1cu_ctx* ctx, int graph_id);

/*
 * Launch-shape autotuner (no counterpart in the reference): runs the given passes as one launch
 * (per_pass_params: params holds one block per pass, as vc1cu_core_passes_multi; else one block)
 * under several shapes of the persistent core kernel - macroblocks (warps) per block 1..4 and
 * blocks per SM - and keeps the fastest for this raster, search configuration and kernel
 * instantiation; later launches of that key use it. The passes' result slots are overwritten.
 * Synchronous; *warps, *blocks (0 = as many as fit) and *ms (one launch) may be NULL.
 */
int vc1cu_autotune(vc1cu_ctx* ctx, const vc1cu_params* params, const vc1cu_pass* passes, int n, int per_pass_params,
                   int* warps, int* blocks, double* ms);
/* Copies a result slot to host arrays (and the scalar totals). Synchronous: returns once the
 * launch that last wrote the slot (as enqueued before this call) has finished and the copies have
 * landed; work enqueued after that launch keeps running (the copies use a second stream), so a
 * caller may enqueue its next picture's passes into other slots before reading this one. */
int vc1cu_read_result(vc1cu_ctx* ctx, int slot, vc1cu_panalysis* out);
int vc1cu_synchronize(vc1cu_ctx* ctx);

/* ---- B-picture analysis (Vc1Encoder::analyze_b_picture_mode) --------------------- */

/* Vc1Encoder::BMbMode (src/encoder_internal.h:407). */
enum {
    VC1CU_BMB_FORWARD = 0,
    VC1CU_BMB_BACKWARD = 1,
    VC1CU_BMB_INTERPOLATED = 2,
    VC1CU_BMB_DIRECT = 3,
    VC1CU_BMB_INTRA = 4
};

/*
 * Vc1Encoder::BAnalysis (src/encoder_internal.h:408-434). Per-macroblock HOST arrays of
 * mbw*mbh entries; any pointer may be NULL to skip it. The distant_* arrays are the two
 * core passes' own (PAnalysis::distant_*), copied through as the reference does
 * (encoder_motion.cpp:810-815). The scalar fields are written by the call.
 */
typedef struct vc1cu_banalysis {
    uint8_t* modes;                     /* VC1CU_BMB_* */
    vc1cu_mv* forward_mvs;              /* decoder forward MV state of every MB */
    vc1cu_mv* backward_mvs;             /* decoder backward MV state */
    double* inter_intra_cost_ratio;
    double* forward_distant_local_mae;
    double* forward_distant_candidate_mae;
    uint8_t* forward_distant_match_decision;
    double* backward_distant_local_mae;
    double* backward_distant_candidate_mae;
    uint8_t* backward_distant_match_decision;
    uint64_t forward_macroblocks;
    uint64_t backward_macroblocks;
    uint64_t interpolated_macroblocks;
    uint64_t direct_macroblocks;
    uint64_t intra_macroblocks;
    uint64_t moved_macroblocks;
    uint64_t fractional_chroma_macroblocks;
    double mean_abs_residual;
    double rate_complexity;
    uint64_t motion_sad;
    uint64_t motion_bits;
    int32_t mv_mode;
    int32_t reserved;
} vc1cu_banalysis;

/*
 * Replaces one Vc1Encoder::analyze_b_picture_mode call (src/encoder_motion.cpp:753-1005):
 * two unseeded core passes of cur_id (forward against past_id, backward against future_id,
 * allow_intra = 0, the given mode), then the per-macroblock Direct / Forward / Backward /
 * Interpolated / Intra decision with the direct vectors scaled from the future anchor's
 * collocated vectors. anchor_mvs / anchor_4mv: HOST arrays of mbw*mbh entries, the future
 * P anchor's MVs and Mixed-MV flags (future_anchor_mvs / future_anchor_4mv). fraction:
 * 1/2, 1/3 or 2/3. past_id holds the (already intensity-compensated, when the anchor
 * signals intensity compensation) past reference. The caller keeps the reference's two
 * encoder-level decisions around this call: the minimal zero-motion configuration
 * (encoder_motion.cpp:770-785, no analysis) and the qpel-versus-half-pel picture RD of
 * analyze_b_picture (:1062-1095). Synchronous.
 */
int vc1cu_analyze_b_picture(vc1cu_ctx* ctx, const vc1cu_params* p, int cur_id, int past_id,
                            int future_id, const vc1cu_mv* anchor_mvs, const uint8_t* anchor_4mv,
                            int fraction_num, int fraction_den, int mode, vc1cu_banalysis* out);

/*
 * Device-resident batch form: the decision stage for n B pictures whose two core passes
 * already ran (vc1cu_core_passes: unseeded, allow_intra 0, the same mode). anchor_slot
 * names the result slot whose mvs / use_4mv are the future anchor's. The B results go to
 * B-result slots (0 <= out_bslot < 4096, a namespace separate from the core result
 * slots). Asynchronous on the context stream.
 */
typedef struct vc1cu_bpass {
    int32_t cur_id;
    int32_t past_id;
    int32_t future_id;
    int32_t fwd_slot;      /* result slot of the forward core pass */
    int32_t bwd_slot;      /* result slot of the backward core pass */
    int32_t anchor_slot;   /* result slot holding the future anchor's MVs / Mixed-MV flags */
    int32_t fraction_num;
    int32_t fraction_den;
    int32_t mode;
    int32_t out_bslot;
    int32_t pqindex;       /* 0 = params->pqindex */
} vc1cu_bpass;

int vc1cu_b_decide(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_bpass* passes, int n);
/*
 * The prediction of the B analysis in bslot into frame slot pred_id, as the reference builds it
 * for every macroblock it codes or samples (encoder_motion.cpp:1030-1053): Forward and Backward
 * with motion_compensate_mb, Direct and Interpolated with motion_compensate_bi_mb
 * (encoder_motion_compensation.cpp:474-525, :659-711), B-intra macroblocks with the visible
 * mean of each source 8x8 block. vc1cu_forward_quant(_device) of (cur_id, pred_id) then gives
 * the B picture's coefficients and levels. Asynchronous.
 */
int vc1cu_b_predict(vc1cu_ctx* ctx, const vc1cu_params* p, int bslot, int cur_id, int past_id, int future_id,
                    int pred_id);
/* Copies a B-result slot to host arrays (and the scalar totals). Synchronous, waiting only for
 * the launch that last wrote the slot, like vc1cu_read_result. */
int vc1cu_read_bresult(vc1cu_ctx* ctx, int bslot, vc1cu_banalysis* out);

/* ---- intensity compensation (fades) ---------------------------------------------- */

/* Vc1Encoder::IntensityComp (src/encoder_internal.h:341-345): LUMSCALE / LUMSHIFT codes 0..63. */
typedef struct vc1cu_intensity {
    int32_t enabled;
    int32_t lumscale;
    int32_t lumshift;
} vc1cu_intensity;

/*
 * Replaces Vc1Encoder::estimate_intensity_comp (src/encoder_motion_compensation.cpp:296-348),
 * which analyze_p_picture runs on its chosen pass when fade compensation is on
 * (encoder_motion.cpp:570-573): the LUMSCALE/LUMSHIFT that map ref_id onto cur_id along the
 * 1-MV field mvs (HOST array of mbw*mbh vectors). The device samples one pixel per 4x4 luma
 * cell along the field and scores every (LUMSCALE, shift) pair; the least-squares fit and the
 * choice in its 7x7 neighbourhood follow the reference's long double arithmetic on the host.
 * When no fade is found out is {0, 32, 0}, the reference's IntensityComp{}. Synchronous.
 */
int vc1cu_estimate_intensity_comp(vc1cu_ctx* ctx, const vc1cu_params* p, int cur_id, int ref_id,
                                  const vc1cu_mv* mvs, vc1cu_intensity* out);

/* Batch form: picture i takes its field from the mvs of result slot passes[i].mv_slot; the
 * device work of all n pictures runs in one set of launches. out has n entries. Synchronous. */
typedef struct vc1cu_icpass {
    int32_t cur_id;
    int32_t ref_id;
    int32_t mv_slot;
} vc1cu_icpass;

int vc1cu_estimate_intensity_batch(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_icpass* passes, int n,
                                   vc1cu_intensity* out);

/* Two-phase form of vc1cu_estimate_intensity_batch for callers that pipeline pictures: _enqueue
 * puts the batch's device work on the context stream and returns at once with a ticket;
 * _collect waits for that work alone (not for work enqueued after it) and finishes the n
 * estimates on the host, with the same results as the batch form. Up to 4 batches may be
 * outstanding: the fifth enqueue reuses the oldest ticket's buffer, which then reports
 * VC1CU_ERR_STATE, as does a ticket collected twice. */
int vc1cu_estimate_intensity_enqueue(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_icpass* passes, int n,
                                     int64_t* ticket);
int vc1cu_estimate_intensity_collect(vc1cu_ctx* ctx, int64_t ticket, vc1cu_intensity* out, int n);

/*
 * Replaces Vc1Encoder::scene_change_score (src/encoder_motion.cpp:599-676), the scene-cut test
 * the encoder runs between consecutive frames (encoder_core.cpp:828): the whole-frame
 * translation SAD per pixel at min(search_range, 32); with fade_compensation, the same against
 * the fade-compensated reference found along the uniform translation field, keeping the
 * smaller; and when the score still reaches scene_threshold, an unseeded quarter-pel core pass
 * whose field, if it fits a camera zoom, may replace the score by its mean residual. The
 * searches and the pass run on the device; the fits use the reference's long double
 * arithmetic on the host. Synchronous.
 */
int vc1cu_scene_change_score(vc1cu_ctx* ctx, const vc1cu_params* p, int cur_id, int ref_id, int fade_compensation,
                             double scene_threshold, double* score);

/* Replaces Vc1Encoder::intensity_compensated_reference (encoder_motion_compensation.cpp:195-294):
 * frame slot out_id becomes ref_id with the luma and chroma maps of ic (intensity_map_y /
 * intensity_map_uv, :175-193), or a copy of it when ic->enabled is 0. Asynchronous. */
int vc1cu_intensity_compensate(vc1cu_ctx* ctx, int ref_id, const vc1cu_intensity* ic, int out_id);

/* ---- motion compensation + forward transform + quantisation ------------------------ */

/*
 * Builds the decoder-equivalent prediction of result slot mv_slot against ref_id into
 * frame slot pred_id (luma via luma_mc_sample[_mode] for 1-MV / 4-MV, chroma via
 * chroma_mc_sample with the 4-MV median chroma vector; motion_compensate_mb /
 * motion_compensate_4mv, src/encoder_motion_compensation.cpp:474-600). Intra MBs are
 * predicted with zero motion. Asynchronous.
 */
int vc1cu_motion_compensate(vc1cu_ctx* ctx, const vc1cu_params* p, int ref_id, int mv_slot,
                            int mv_mode, int pred_id);

/*
 * Forward transform and scalar quantisation of src_id - pred_id for every macroblock's
 * six 8x8 parents (Y0..Y3, U, V) and every transform type in type_mask
 * (bit (t-1) for TransformType t: 1 = 8x8, 2 = 8x4, 3 = 4x8, 4 = 4x4). Bit-exact with
 * quantize_inter_part at trellis 0 (src/encoder_transform.cpp:1087-1171 scalar branch).
 * Output layout: [type][mb][parent][64]; for type t the 64 entries hold the partitions
 * at the reference's storage (8x8 transposed, rectangles row-major with stride 8,
 * partition p at its transform_part_geometry offset, src/encoder_transform.cpp:915-933).
 * coeffs (double) and levels (int16) are HOST arrays of n_types*mbs*6*64 entries; either
 * may be NULL. Synchronous.
 */
int vc1cu_forward_quant(vc1cu_ctx* ctx, const vc1cu_params* p, int src_id, int pred_id,
                        int type_mask, double* coeffs, int16_t* levels);

/* Device-output form of vc1cu_forward_quant: d_coeffs/d_levels are device pointers
 * (either may be NULL). Asynchronous on the context stream. */
int vc1cu_forward_quant_device(vc1cu_ctx* ctx, const vc1cu_params* p, int src_id, int pred_id,
                               int type_mask, double* d_coeffs, int16_t* d_levels);

/*
 * The transform type (1 = 8x8, 2 = 8x4, 3 = 4x8, 4 = 4x4) that Vc1Encoder::choose_transform_mb
 * picks for each MB with the throughput preset (fast transform RDO with variable transforms,
 * trellis 0, no DQUANT; src/encoder_transform.cpp:1605-1712): the residual metrics of
 * transform_metrics (src/transform_residual_metrics.h:29-61) between src_id and pred_id, the
 * candidate list (split shapes where the coded raster crops an MB) and the preset's pick.
 * types: HOST array of mbw*mbh. The RD search of the other presets stays with the caller.
 * Synchronous.
 */
int vc1cu_fast_transform_types(vc1cu_ctx* ctx, const vc1cu_params* p, int src_id, int pred_id, uint8_t* types);

/* Configuration of the transform RD (the EncoderConfig fields and picture-level choices
 * Vc1Encoder::choose_transform_mb reads, src/encoder_internal.h:258-266). */
typedef struct {
    int32_t trellis;                      /* 0 scalar, 1 fast bounded trellis (beam 4), 2 wide (beam 8) */
    int32_t adaptive_quality;             /* perceptual lambda scale (src/encoder_aq.cpp:405-653) */
    double aq_strength;
    int32_t variable_transforms;          /* 0: every MB 8x8 */
    int32_t extended_transform_signaling; /* 0: macroblock signaling only (no TTBLK choice) */
    int32_t coding_set;                   /* the picture's inter AC coding set, 0..7 */
    int32_t use_vlc;                      /* 0: every AC coefficient as Escape-3 */
    int32_t dquantfrm;                    /* DQUANTFRM of the picture */
    int32_t hrd_enabled;                  /* keeps scalar levels at MQUANT 1 */
    int32_t frame_type;                   /* 0: per-MB choice; 1..4: frame-level TTFRM type */
} vc1cu_trd_cfg;

/* One macroblock's MbTransformDecision (src/encoder_internal.h:1013-1033). */
typedef struct {
    uint8_t type;                 /* 1 8x8, 2 8x4, 3 4x8, 4 4x4: the common type, or the first coded
                                     parent's at block signaling */
    uint8_t signal_level;         /* 0 macroblock (TTMB), 1 block (TTBLK), 2 frame (TTFRM) */
    uint8_t cbp;                  /* Y0 Y1 Y2 Y3 U V, bit 5 = Y0 */
    uint8_t parent_type[6];
    uint8_t skip_mask[6];
    uint8_t reserved;
    uint32_t estimated_bits;      /* CBPCY + transform syntax + coefficients */
    uint32_t parent_bits[6];      /* each parent's payload estimate (estimate_parent_payload_bits) */
    double distortion;            /* sum of the parents' reconstruction SSE */
    double parent_distortion[6];
} vc1cu_tdecision;

/*
 * The transform RD of the default presets (Vc1Encoder::choose_transform_mb without the
 * throughput shortcut, src/encoder_transform.cpp:1605-1780): for every MB of src_id against the
 * prediction pred_id, the candidate transform types from the residual metrics, each evaluated on
 * all six parents (forward transform, scalar or trellis quantisation (trellis_quantize,
 * :1873-2088) with the perceptual lambda scale, inverse transform, reconstruction SSE and the
 * coefficient/subblock bit estimate of the VC-1 VLC tables), the macroblock- against block-level
 * signaling decision by D + lambda R, and the trellis re-evaluation of the winners. mquant: HOST
 * array of mbw*mbh MQUANT values (NULL: PQINDEX everywhere). out: HOST array of mbw*mbh
 * decisions; levels: HOST int16 [mbw*mbh][6][64] of the chosen quantised coefficients (each
 * parent's partitions in their natural sub-rectangles of the 8x8 grid), or NULL. Synchronous.
 */
int vc1cu_choose_transform(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id, int pred_id,
                           const uint8_t* mquant, vc1cu_tdecision* out, int16_t* levels);

/*
 * Replaces Vc1Encoder::choose_dquant_transform_mb (src/encoder_aq.cpp:280-404) for every MB: the
 * transform RD at the MB's base MQUANT rate_base[mb] (HOST array of mbw*mbh values 1..31: the
 * caller's rate-control base, that is rate_weighted_mquant with the residual-priority adjustment
 * and the perceptual priority's boost, :284-310), then, with DQUANT and the perceptual scale on,
 * the finer absolute MQUANT of a quiet block next to detail, of bright detail on dark or of
 * predictable texture, kept when either decision codes coefficients (:318-370), else the up to
 * three coarser MQUANTs of an unprotected coded MB, each kept when its D + lambda R beats the
 * best so far by 0.05% (:372-403). cfg: as for vc1cu_choose_transform (dquantfrm is set per
 * evaluation as the reference does; the fixed-8x8 shortcut of the throughput preset is
 * vc1cu_fast_transform_types); dquant: EncoderConfig::dquant; predictable_texture:
 * EncoderConfig::aq_predictable_texture. out, mquant (HOST mbw*mbh) and levels (HOST int16
 * [mb][6][64] or NULL) take each MB's decision, MQUANT and levels. Synchronous.
 */
int vc1cu_choose_dquant(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int dquant,
                        int predictable_texture, int src_id, int pred_id, const uint8_t* rate_base, vc1cu_tdecision* out,
                        uint8_t* mquant, int16_t* levels);

/*
 * The reconstruction a transform decision implies (evaluate_transform_parent,
 * src/encoder_transform.cpp:1569-1585): for every MB and parent block (Y0..Y3, U, V), the levels
 * of its chosen type dequantised (dequant_level at PQINDEX, :1058-1065), inverse-transformed
 * (inverse_partition with its DC-only shortcuts, :1173-1274, the VC-1 inverse transforms) and
 * added to frame slot pred_id with 8-bit clamping, into frame slot out_id. d_levels: DEVICE
 * levels in vc1cu_forward_quant_device's layout for type_mask; block_types: HOST array of
 * mbw*mbh*6 TransformType codes (1 = 8x8, 2 = 8x4, 3 = 4x8, 4 = 4x4), each one of type_mask's
 * (the type decision itself, choose_transform_mb, stays with the caller). Asynchronous.
 */
int vc1cu_reconstruct(vc1cu_ctx* ctx, const vc1cu_params* p, int pred_id, const int16_t* d_levels, int type_mask,
                      const uint8_t* block_types, int out_id);

/*
 * vc1cu_reconstruct under a DQUANT plan: each MB's levels dequantised at its MQUANT (dequant_level,
 * :1058-1065; a derived MQUANT, or one other than PQINDEX, without the HALFQP half step), as the
 * picture coder reconstructs the decisions of vc1cu_choose_dquant. mquant: HOST mbw*mbh MQUANTs
 * (1..31); derived: HOST mbw*mbh DQUANT-derived flags, or NULL for none. Returns once the host
 * arrays are copied.
 */
int vc1cu_reconstruct_dquant(vc1cu_ctx* ctx, const vc1cu_params* p, int pred_id, const int16_t* d_levels,
                             int type_mask, const uint8_t* block_types, const uint8_t* mquant, const uint8_t* derived,
                             int out_id);

/* ---- the P picture's motion-mode decision (Vc1Encoder::analyze_p_picture) ---------- */

/*
 * Replaces Vc1Encoder::estimate_p_motion_bits (src/encoder_motion.cpp:444-486) for the analysis
 * in result slot `slot`, made in mv_mode: the MVTAB selector, MVMODE (with the
 * intensity-compensation fields when intensity != 0), the MVTYPEMB bitplane of a Mixed-MV
 * picture (choose_bitplane, src/encoder_entropy.cpp:37-61) and every macroblock's MVDATA under
 * the cheapest of the four MV tables (choose_mv_table, :1223-1234) with one bit per
 * hybrid-predicted vector. A half-pel differential the syntax cannot represent (the reference
 * throws) fails with VC1CU_ERR_STATE. Synchronous.
 */
int vc1cu_p_motion_bits(vc1cu_ctx* ctx, const vc1cu_params* p, int slot, int mv_mode, int intensity, uint64_t* bits);

/* The EncoderConfig fields analyze_p_picture reads beyond vc1cu_params. */
typedef struct {
    vc1cu_trd_cfg trd;           /* the encoder's trellis, variable_transforms,
                                    extended_transform_signaling, use_vlc and hrd_enabled; the mode
                                    RD evaluates AQ-neutrally at PQINDEX with the picture's decision
                                    coding set, per-MB types and no DQUANT (the other fields are
                                    ignored) */
    int32_t fast_transform_rdo;  /* EncoderConfig::fast_transform_rdo */
    int32_t dquant;              /* EncoderConfig::dquant */
    int32_t n_modes;             /* candidate modes in order qpel, half-pel, bilinear, Mixed-MV: 4 in
                                    Advanced Profile (1 or 3 in Main Profile) */
    int32_t fade_compensation;   /* EncoderConfig::fade_compensation */
    double fade_min_gain;        /* EncoderConfig::fade_min_gain */
} vc1cu_ppic_cfg;

/* What vc1cu_analyze_p_picture decided. Candidate i < n_modes is the plain analysis in mode i,
 * candidate 4 + i the fade-compensated one (when an estimate was enabled). */
typedef struct {
    int32_t mode;                /* the final pass's MV mode */
    int32_t weighted;            /* 1: the fade-compensated analysis was kept */
    vc1cu_intensity ic;          /* the fade estimate on the plain choice (enabled 0: none) */
    uint64_t motion_bits;        /* estimate_p_motion_bits of the returned analysis */
    uint64_t cand_bits[8];       /* the candidates' motion bits */
    double cand_score[8];        /* their sampled mode-RD scores (compared in long double; reported
                                    rounded to double) */
} vc1cu_ppic_info;

/*
 * The whole of Vc1Encoder::analyze_p_picture (src/encoder_motion.cpp:524-597) on the device: the
 * quarter-pel seed pass and the seeded mode passes, each candidate's motion bits and
 * sampled_p_mode_rd (:488-522: the prediction and the AQ-neutral transform RD of 32 evenly spaced
 * macroblocks, residual RD per MB plus lambda times motion bits per MB with lambda = 0.75 * (2 *
 * PQ + HALFQP)^2, in the host's long double), the final pass in the least-scoring mode into
 * out_slot, and with fade compensation the intensity estimate on it, the compensated reference,
 * the weighted seed and mode passes, their scores and the reference's acceptance test, the
 * weighted final pass replacing out_slot when it wins. scratch_slot .. scratch_slot + 7 are
 * result slots and scratch_frame, scratch_frame + 1 frame slots the call overwrites (the
 * prediction scratch and the compensated reference). info may be NULL. Synchronous.
 */
int vc1cu_analyze_p_picture(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_ppic_cfg* cfg, int cur_id, int ref_id,
                            int out_slot, int scratch_slot, int scratch_frame, vc1cu_ppic_info* info);

/*
 * The quarter-pel versus half-pel bilinear choice of Vc1Encoder::analyze_b_picture
 * (src/encoder_motion.cpp:1062-1095) for two analyses of one B picture already in B-result slots
 * (vc1cu_b_decide in quarter-pel and in bilinear mode): sampled_b_mode_rd (:1006-1060) of each,
 * the prediction of 32 evenly spaced macroblocks (B-intra ones from their blocks' visible means,
 * plus 72 bits of intra syntax) and their AQ-neutral transform RD, residual RD per MB plus lambda
 * times the analysis's motion bits per MB, in the host's long double. *choice = 1 when the
 * bilinear analysis scores strictly less, else 0. past_id is the forward reference the analyses
 * used (the compensated one under forward intensity compensation). cfg: the transform RD fields,
 * fast_transform_rdo and dquant of a vc1cu_ppic_cfg; the rest is ignored. pred_id is a frame slot
 * the call overwrites; scores (2 entries: quarter-pel, bilinear; rounded to double) may be NULL.
 * Synchronous.
 */
int vc1cu_b_mode_rd(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_ppic_cfg* cfg, int cur_id, int past_id,
                    int future_id, int bslot_qpel, int bslot_bilinear, int pred_id, int* choice, double* scores);

/*
 * In-loop deblocking of frame slot frame_id in place, at params->pqindex.
 * vc1cu_loop_filter_i: Vc1Encoder::apply_i_like_loop_filter (src/encoder_filter.cpp:426-441),
 * every 8-pixel block edge. vc1cu_loop_filter_p: the Advanced Profile apply_p_loop_filter
 * (:610-738) of a coded P picture, HOST arrays per macroblock: block_mvs (4 luma block vectors),
 * cbp (6 loop_filter_pattern codes, 4 bits each), tt (6 loop_filter_tt codes: 0, 3, 6, 7) and
 * intra (bit k set when block k is intra). The device result equals the reference's raster
 * order. The frame is the coding raster or the padded raster of whole macroblocks that the
 * reference's reconstruction holds (vc1cu_store_signed's output); the filter covers the frame's
 * own extent, as the reference's does. vc1cu_loop_filter_i is asynchronous; vc1cu_loop_filter_p
 * returns once its metadata copies are done.
 */
int vc1cu_loop_filter_i(vc1cu_ctx* ctx, const vc1cu_params* p, int frame_id);
int vc1cu_loop_filter_p(vc1cu_ctx* ctx, const vc1cu_params* p, int frame_id, const vc1cu_mv* block_mvs,
                        const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra);

/*
 * The Main Profile P-picture deblocking (apply_p_loop_filter_plane_main,
 * src/encoder_filter.cpp:465-608, what apply_p_loop_filter runs for WMV9 Main syntax): the
 * filter of vc1cu_loop_filter_p with SMPTE 421M 8.6.4.1's four Main Profile exceptions - block 0
 * of the first macroblock intra forces whole top and left borders of every inter macroblock; the
 * luma edge between blocks 2 and 3 decides with block 1's pattern and kind; a 4x4-transformed
 * side forces the whole border; chroma vectors compared after FASTUVMC rounding and the 8.3.6.5
 * range limit. Same arguments and return as vc1cu_loop_filter_p.
 */
int vc1cu_loop_filter_p_main(vc1cu_ctx* ctx, const vc1cu_params* p, int frame_id, const vc1cu_mv* block_mvs,
                             const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra);

/*
 * The signed intra reconstruction of an I picture, Vc1Encoder::reconstruct_i_signed_padded
 * (src/encoder_encode.cpp:814-887) with AC coding: for every 8x8 block of frame slot src_id the
 * intra forward transform (forward_transform, samples outside the source read 0 luma / 128
 * chroma), the AC levels at the MB's MQUANT (quantize_ac, src/encoder_transform.cpp:2090-2144:
 * scalar, or with cfg->trellis 1 / 2 the trellis along the intra scan with the intra-family rates
 * and, with cfg->adaptive_quality, the perceptual lambda scale of the block; cfg's other fields
 * are not read, NULL: scalar), the DC level whose
 * reconstruction is nearest the padded block mean, predicted from its neighbours and clamped to
 * the DC range (predict_dc_dquant with the DQUANT scaling, clamp_dc_target_for_diff), the
 * dequantised coefficients and the 8x8 inverse transform, into the DEVICE int32 planes d_y, d_u,
 * d_v of the padded raster, rows packed (the layout vc1cu_overlap_smooth and vc1cu_store_signed
 * take). overlap: 0 none, 1 all, 2 select with the HOST per-MB flags: the overlap plan whose edge
 * source (make_overlap_edge_source, :13-63) the transform reads. mquant / derived: HOST per-MB
 * MQUANT (1..31) and DQUANT-derived flags of the picture's DQUANT plan, or NULL for PQINDEX and
 * none. Returns once its inputs are copied.
 */
int vc1cu_reconstruct_intra(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id, int overlap,
                            const uint8_t* flags, const uint8_t* mquant, const uint8_t* derived, int32_t* d_y,
                            int32_t* d_u, int32_t* d_v);

/*
 * The I picture's overlap plan, Vc1Encoder::choose_i_overlap_plan (src/encoder_filter.cpp:277-343),
 * for an Advanced Profile picture whose sequence sets OVERLAP: at PQINDEX >= 9 every edge (ALL);
 * below, the intra reconstruction of frame slot src_id without smoothing and with every edge
 * smoothed (as vc1cu_reconstruct_intra and vc1cu_overlap_smooth), each macroblock flagged when
 * smoothing lowers its reconstruction error (overlap_sse_region, :246-266) by more than
 * 4 * PQINDEX^2, then NONE, ALL or SELECT by total error plus 8 * PQINDEX^2 per bit of syntax
 * (SELECT: its flags as the cheapest OVERFLAGS bitplane). cfg, mquant / derived: the AC
 * quantisation settings and the picture's DQUANT plan as for vc1cu_reconstruct_intra (NULL:
 * scalar levels, PQINDEX). *mode (0 none, 1 all, 2 select) and flags
 * (HOST mbw*mbh) take the plan as the reference returns it. Synchronous.
 */
int vc1cu_choose_i_overlap(vc1cu_ctx* ctx, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id,
                           const uint8_t* mquant, const uint8_t* derived, int* mode, uint8_t* flags);

/*
 * Overlap smoothing of a signed (unclamped, unbiased) reconstruction in place:
 * apply_overlap_plane_signed (src/encoder_filter.cpp:217-243) on each plane, as
 * Vc1Encoder::apply_i_overlap (:344-352) and apply_p_overlap (:354-365) call it. d_y, d_u, d_v
 * are DEVICE int32 planes of the padded raster, (mbh*16) x (mbw*16) luma and half that chroma,
 * rows packed (pitch = width). First every vertical 8x8 edge (4 samples across it, rows by
 * 8-row segment), then every horizontal edge, each enabled when all != 0 (CONDOVER ALL) or by
 * the HOST per-macroblock flags[mbw*mbh] (OVERFLAGS: an edge inside a macroblock needs its flag,
 * an edge between two needs both; apply_p_overlap passes the intra map). flags may be NULL when
 * all != 0. The picture-level condition (apply_p_overlap: OVERLAP on and PQINDEX >= 9; the I
 * plan's mode) stays with the caller. Returns once the flags are copied.
 */
int vc1cu_overlap_smooth(vc1cu_ctx* ctx, const vc1cu_params* p, int32_t* d_y, int32_t* d_u, int32_t* d_v,
                         const uint8_t* flags, int all);

/*
 * Stores a signed padded reconstruction (the planes of vc1cu_overlap_smooth) as 8-bit samples
 * clamp(s + bias, 0, 255) into frame slot out_id (src/encoder_filter.cpp reconstruct_i_picture_padded's
 * store, and the intra write-back after apply_p_overlap, src/encoder_encode.cpp:1425-1449). With
 * mb_mask NULL the slot becomes the whole padded raster ((mbw*16) x (mbh*16)); with a HOST
 * mb_mask[mbw*mbh] only the flagged macroblocks are written, into an existing slot (its samples
 * outside the slot's size are skipped). Returns once the mask is copied.
 */
int vc1cu_store_signed(vc1cu_ctx* ctx, const vc1cu_params* p, const int32_t* d_y, const int32_t* d_u,
                       const int32_t* d_v, int bias, const uint8_t* mb_mask, int out_id);

/* ---- learned motion-vector proposals ---------------------------------------------- */

/*
 * No counterpart in the reference: a small convolutional network that proposes, per macroblock,
 * K = 4 integer-pixel vectors which replace the integer search (UMH / diamond / long range,
 * encoder_motion.cpp:1781-2023, :1658-1779) of an unseeded analysis pass; the exact part of the
 * pass stays: the candidates' full-resolution SADs, a short descent about the best, and the
 * staged sub-pel refinement of refine_motion_block_staged (encoder_motion.cpp:3271-3594). A
 * macroblock whose best match is not good (motion_match_good, encoder_motion.cpp:1627-1635: more
 * than 6 levels of mean absolute error) falls back to the plain search.
 *
 * The network reads the current and reference pictures at quarter resolution plus the picture's
 * dominant translation (found by an exhaustive quarter-resolution search over the search range),
 * runs four 3x3 convolutions of 32 channels (BF16 weights, FP32 accumulation on the tensor
 * cores), pools each macroblock and projects to two hypotheses (zero vector, translation), each
 * with a logit and an offset. It is trained on the device by its own backward kernels on
 * (picture pair, plain-search vector) samples.
 *
 * A vc1cu_lp belongs to one context and one raster (width x height) and search range; it holds
 * `capacity` samples (features, hint, labels, candidates, fallback flags) and trains or proposes
 * on up to `max_batch` samples at once. Calls are asynchronous on the context stream unless noted.
 */
typedef struct vc1cu_lp vc1cu_lp;

/* Number of fp32 parameters (four conv layers W[32][9][Cin] + b[32], then the 8x32 projection
 * and its 8 biases, in that order). */
int vc1cu_lp_param_count(void);
int vc1cu_lp_create(vc1cu_ctx* ctx, int width, int height, int search_range, int capacity, int max_batch,
                    uint64_t seed, vc1cu_lp** out);
int vc1cu_lp_destroy(vc1cu_lp* net);
/* Synchronous copies of the fp32 parameters; set also restarts the optimiser. */
int vc1cu_lp_get_params(vc1cu_lp* net, float* out);
int vc1cu_lp_set_params(vc1cu_lp* net, const float* in);
/* Sample `sample` := the features and translation hint of the pair (cur_id, ref_id). */
int vc1cu_lp_prepare(vc1cu_lp* net, int cur_id, int ref_id, int sample);
/* Its labels := the integer-pixel vectors (nearest pixel) of a plain pass in result slot. */
int vc1cu_lp_set_labels(vc1cu_lp* net, int sample, int result_slot);
/* One Adam step (lr; betas 0.9 / 0.999) on the batch; *loss = the batch's mean loss before it.
 * Synchronous. */
int vc1cu_lp_train_step(vc1cu_lp* net, const int* samples, int n, float lr, float* loss);
/* The batch's loss and every parameter's gradient (host, vc1cu_lp_param_count floats), without
 * an update. Synchronous. */
int vc1cu_lp_gradients(vc1cu_lp* net, const int* samples, int n, float* grads, float* loss);
/* Inference on samples first .. first+n-1: their candidates. */
int vc1cu_lp_propose(vc1cu_lp* net, int first_sample, int n);
/* Reads a sample back (any pointer may be NULL): features (W4*H4*16 bf16 bit patterns, W4 =
 * 4*mbw, H4 = 4*mbh, sample-major, channel fastest), hint, candidates (4 per MB), fallback flags.
 * Synchronous. */
int vc1cu_lp_read_sample(vc1cu_lp* net, int sample, uint16_t* features, vc1cu_mv* hint, vc1cu_mv* candidates,
                         uint8_t* fallback);

/* One learned analysis pass (the counterpart of an unseeded 1-MV core pass without P-intra). */
typedef struct vc1cu_lp_pass {
    int32_t cur_id;
    int32_t ref_id;
    int32_t sample;     /* the sample holding this pair's candidates and hint */
    int32_t mode;       /* VC1CU_MV_QPEL, _HPEL or _HPEL_BILINEAR */
    int32_t out_slot;   /* result slot, read with vc1cu_read_result */
    int32_t pqindex;    /* 0 = params->pqindex */
} vc1cu_lp_pass;

/* n learned passes in one launch; with fallback != 0 a second launch runs the plain search
 * (params' algorithm and ranges, the hint as its global vector) on the macroblocks the first
 * flagged, in wavefront order over the learned field. */
int vc1cu_lp_analyze(vc1cu_lp* net, const vc1cu_params* p, const vc1cu_lp_pass* passes, int n, int fallback);

/* ---- allocation-free whole-frame translation search ------------------------------ */

/*
 * No counterpart in the reference: an addition of this library for callers that cannot
 * allocate device memory while they run (an encoder worker bound to a fixed device-memory
 * budget, or code on a path where cudaMalloc is not allowed because it would synchronise
 * the device). It needs no context and allocates nothing.
 *
 * Runs the whole-frame translation search of an unseeded analysis pass
 * (Vc1Encoder::global_motion_search, src/encoder_motion.cpp:2025-2141) for n pictures
 * and writes, per picture i, d_dxdy[2i], d_dxdy[2i+1] (integer pixels) and d_sad[i]
 * (the full-resolution frame SAD at that offset): the global_dx / global_dy /
 * global_full_sad that vc1cu_analyze_p_core reports for range =
 * min(search_range, local_search_range, 32).
 *
 * cur_y / ref_y: HOST arrays of n DEVICE pointers to 8-bit luma planes of width x height
 * with row pitch `pitch` bytes; d_dxdy (2n int32) and d_sad (n uint64) are DEVICE
 * buffers. stream is a cudaStream_t (NULL: the legacy default stream) of the current
 * device; the call only enqueues work on it and returns, so results are ready once that
 * stream has been synchronised.
 *
 * Limits: 1 <= n <= 16 pictures per call and 0 <= range <= 32; larger requests are
 * rejected with VC1CU_ERR_ARG. The search state lives in one fixed device array of
 * 168,192 bytes that every GPU loading this library holds until the process exits. All
 * calls on one device share that array: two calls whose GPU work can overlap (issued on
 * different streams, or from threads that do not order them) race on it and give wrong
 * results; calls issued in order on one stream are safe, and devices are independent.
 * Each call resets the state it reads, so nothing carries over from an earlier call.
 *
 * width and height may be odd (any coding size up to 16384); pitch >= width.
 *
 * Every call looks up the array's device address (cudaGetSymbolAddress, with the caller's
 * device current), so the address always belongs to the module loaded in the current context,
 * also after a cudaDeviceReset. The first call on a device may load the library's device code
 * into the context; make that first call before any stream capture begins.
 * On failure a message is written to err (err_len bytes, may be NULL).
 */
int vc1cu_global_motion_noalloc(const uint8_t* const* cur_y, const uint8_t* const* ref_y, int pitch,
                                int width, int height, int range, int n, int32_t* d_dxdy,
                                uint64_t* d_sad, void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* VC1CU_H */
