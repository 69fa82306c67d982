// encoder_cuda.cpp - libvc1's analysis entry points on the B200 backend (--compute cuda).
//
// Compiled into libvc1 together with libvc1_cuda.patch, which adds VC1_COMPUTE_CUDA to
// vc1_compute_backend_e (include/libvc1.h:62-66), EncoderConfig::cuda_compute beside
// vulkan_compute (src/encoder_internal.h:289), the selection in configure_compute_backend
// (src/encoder_compute.cpp:28-109), `--compute cuda` in the CLI, and one line at the top of each
// analysis function that hands the call to the member defined here:
//
//   Vc1Encoder::analyze_p_picture_core  (src/encoder_motion.cpp:47)  -> vc1cu_analyze_p_core
//   Vc1Encoder::analyze_b_picture_mode  (src/encoder_motion.cpp:753) -> vc1cu_analyze_b_picture
//   Vc1Encoder::estimate_intensity_comp (src/encoder_motion_compensation.cpp:296)
//                                                                    -> vc1cu_estimate_intensity_comp
//   Vc1Encoder::scene_change_score      (src/encoder_motion.cpp:599) -> vc1cu_scene_change_score
//
// Everything around them stays the reference's: the picture-level mode RD of analyze_p_picture
// and analyze_b_picture, transform RD, entropy coding and rate control consume the device's
// results exactly as they consume the CPU's. The results are bit-exact, so the elementary
// stream is byte-identical to a --compute cpu --simd none encode.
#include "cuda_compute.h"

#include <cstring>

#include "encoder_internal.h"

namespace libvc1 {

namespace {

// The subset of EncoderConfig the analysis reads (include/vc1cu.h, vc1cu_params).
vc1cu_params cuda_params(const EncoderConfig& c) {
    vc1cu_params p;
    vc1cu_params_default(&p, c.width, c.height);
    p.display_width = c.visible_width();
    p.display_height = c.visible_height();
    p.pqindex = c.pqindex;
    p.halfqp = c.halfqp ? 1 : 0;
    p.nonuniform = c.quantizer_type == QuantizerType::NonUniform ? 1 : 0;
    p.search_range = c.motion_search_range;
    p.local_search_range = c.motion_local_search_range;
    p.me_algorithm = static_cast<int>(c.me_algorithm);
    p.me_quality = static_cast<int>(c.me_quality);
    p.subpel = c.subpixel_refinement ? 1 : 0;
    p.fast_subpel = c.fast_subpixel_refinement ? 1 : 0;
    p.subpel_range = c.subpixel_refinement_range;
    p.long_range_mode = static_cast<int>(c.long_range_search_mode);
    p.rnd = c.rndctrl ? 1 : 0;
    p.disable_p_intra = c.debug_disable_p_intra ? 1 : 0;
    p.disable_b_intra = c.debug_disable_b_intra ? 1 : 0;
    p.distant_match_max_mae = c.distant_match_max_mae;
    p.inter_intra_threshold = c.inter_intra_threshold;
    return p;
}

// Frame slots this binding uses for the pictures of one call, and the result slot of a learned pass.
enum : int { kCur = 0, kRef = 1, kFuture = 2, kLearnedSlot = 3000 };

void upload(CudaComputeContext& cx, int id, const Frame& f) {
    cx.check(vc1cu_upload_frame(cx.handle(), id, f.y.data(), f.u.data(), f.v.data(), f.width, f.height),
             "vc1cu_upload_frame");
}

CudaComputeContext& context(const EncoderConfig& c) {
    if (!c.cuda_compute) throw std::runtime_error("CUDA analysis backend not configured");
    return *c.cuda_compute;
}

}  // namespace

void configure_cuda_backend(EncoderConfig& cfg, vc1_stats_t& stats, const vc1_param_t& p) {
    if (cfg.syntax != StreamSyntax::Advanced || cfg.interlaced())
        throw std::runtime_error("the CUDA analysis backend supports VC-1 Advanced Profile progressive coding only");
    if (cfg.me_quality == VC1_ME_RD)
        throw std::runtime_error("the CUDA analysis backend does not implement --me-quality rd");
    std::string error;
    auto cx = CudaComputeContext::create(p.i_compute_device, error);
    if (!cx) throw std::runtime_error("CUDA compute unavailable: " + error);
    stats.i_compute_selected = VC1_COMPUTE_CUDA;
    stats.i_compute_device = cx->device_index();
    std::strncpy(stats.sz_compute_device, cx->device_name().c_str(), sizeof(stats.sz_compute_device) - 1);
    stats.sz_compute_device[sizeof(stats.sz_compute_device) - 1] = '\0';
    cfg.cuda_compute = std::move(cx);
}

Vc1Encoder::PAnalysis Vc1Encoder::analyze_p_picture_core_cuda(const Frame& f, const Frame& ref,
                                                              ProgressiveMvMode mode, bool allow_intra,
                                                              const PAnalysis* shared_seed) const {
    CudaComputeContext& cx = context(c_);
    const vc1cu_params p = cuda_params(c_);
    const size_t mbs = static_cast<size_t>((c_.width + 15) / 16) * static_cast<size_t>((c_.height + 15) / 16);
    if (shared_seed && shared_seed->mvs.size() != mbs)
        throw std::runtime_error("shared P motion seed has the wrong macroblock count");
    PAnalysis out;
    out.mv_mode = mode;
    out.mvs.resize(mbs);
    out.block_mvs.resize(mbs);
    out.use_4mv.assign(mbs, 0);
    out.use_intra.assign(mbs, 0);
    out.screen_sads.assign(mbs, 0);
    out.inter_intra_cost_ratio.assign(mbs, -1.0);
    out.distant_local_mae.assign(mbs, -1.0);
    out.distant_candidate_mae.assign(mbs, -1.0);
    out.distant_match_decision.assign(mbs, 0);
    static_assert(sizeof(MotionVector) == sizeof(vc1cu_mv), "MotionVector and vc1cu_mv share one layout");
    static_assert(sizeof(std::array<MotionVector, 4>) == 4 * sizeof(vc1cu_mv), "four block vectors per MB");
    vc1cu_panalysis o{};
    o.mvs = reinterpret_cast<vc1cu_mv*>(out.mvs.data());
    o.block_mvs = reinterpret_cast<vc1cu_mv*>(out.block_mvs.data());
    o.use_4mv = out.use_4mv.data();
    o.use_intra = out.use_intra.data();
    o.screen_sads = reinterpret_cast<uint64_t*>(out.screen_sads.data());
    o.inter_intra_cost_ratio = out.inter_intra_cost_ratio.data();
    o.distant_local_mae = out.distant_local_mae.data();
    o.distant_candidate_mae = out.distant_candidate_mae.data();
    o.distant_match_decision = out.distant_match_decision.data();
    vc1cu_panalysis seed{};
    if (shared_seed) {
        // the seed pass's distant_* arrays, which a seeded pass copies through (encoder_motion.cpp:100-104)
        seed.distant_local_mae = const_cast<double*>(shared_seed->distant_local_mae.data());
        seed.distant_candidate_mae = const_cast<double*>(shared_seed->distant_candidate_mae.data());
        seed.distant_match_decision = const_cast<uint8_t*>(shared_seed->distant_match_decision.data());
    }
    {
        std::lock_guard<std::mutex> lock(cx.mutex());
        upload(cx, kCur, f);
        upload(cx, kRef, ref);
        vc1cu_lp* lp = (!shared_seed && !allow_intra && mode != ProgressiveMvMode::MixedMv && c_.motion_search_range > 0)
                           ? cx.learned(c_.width, c_.height, c_.motion_search_range)
                           : nullptr;
        if (lp) {
            // the learned proposals replace the integer search of this unseeded pass
            const vc1cu_lp_pass q{kCur, kRef, 0, static_cast<int>(mode), kLearnedSlot, 0};
            cx.check(vc1cu_lp_prepare(lp, kCur, kRef, 0), "vc1cu_lp_prepare");
            cx.check(vc1cu_lp_propose(lp, 0, 1), "vc1cu_lp_propose");
            cx.check(vc1cu_lp_analyze(lp, &p, &q, 1, 1), "vc1cu_lp_analyze");
            cx.check(vc1cu_read_result(cx.handle(), kLearnedSlot, &o), "vc1cu_read_result");
        } else
        cx.check(vc1cu_analyze_p_core(cx.handle(), &p, kCur, kRef, static_cast<int>(mode), allow_intra ? 1 : 0,
                                      shared_seed ? reinterpret_cast<const vc1cu_mv*>(shared_seed->mvs.data())
                                                  : nullptr,
                                      shared_seed ? &seed : nullptr, &o),
                 "vc1cu_analyze_p_core");
    }
    out.mean_abs_residual = o.mean_abs_residual;
    out.rate_complexity = o.rate_complexity;
    out.motion_sad = o.motion_sad;
    out.moved_macroblocks = static_cast<size_t>(o.moved_macroblocks);
    out.fractional_chroma_macroblocks = static_cast<size_t>(o.fractional_chroma_macroblocks);
    out.four_mv_macroblocks = static_cast<size_t>(o.four_mv_macroblocks);
    out.intra_macroblocks = static_cast<size_t>(o.intra_macroblocks);
    return out;
}

Vc1Encoder::BAnalysis Vc1Encoder::analyze_b_picture_mode_cuda(const Frame& f, const Frame& past_prediction,
                                                              const Frame& future,
                                                              const std::vector<MotionVector>& future_anchor_mvs,
                                                              const std::vector<uint8_t>& future_anchor_4mv,
                                                              int fraction_num, int fraction_den,
                                                              ProgressiveMvMode mode) const {
    CudaComputeContext& cx = context(c_);
    const vc1cu_params p = cuda_params(c_);
    const size_t mbs = static_cast<size_t>((c_.width + 15) / 16) * static_cast<size_t>((c_.height + 15) / 16);
    static_assert(sizeof(BMbMode) == 1, "BMbMode is one byte, VC1CU_BMB_* in the same order");
    BAnalysis out;
    out.mv_mode = mode;
    out.modes.assign(mbs, BMbMode::Forward);
    out.forward_mvs.resize(mbs);
    out.backward_mvs.resize(mbs);
    out.inter_intra_cost_ratio.assign(mbs, -1.0);
    out.forward_distant_local_mae.assign(mbs, -1.0);
    out.forward_distant_candidate_mae.assign(mbs, -1.0);
    out.forward_distant_match_decision.assign(mbs, 0);
    out.backward_distant_local_mae.assign(mbs, -1.0);
    out.backward_distant_candidate_mae.assign(mbs, -1.0);
    out.backward_distant_match_decision.assign(mbs, 0);
    vc1cu_banalysis o{};
    o.modes = reinterpret_cast<uint8_t*>(out.modes.data());
    o.forward_mvs = reinterpret_cast<vc1cu_mv*>(out.forward_mvs.data());
    o.backward_mvs = reinterpret_cast<vc1cu_mv*>(out.backward_mvs.data());
    o.inter_intra_cost_ratio = out.inter_intra_cost_ratio.data();
    o.forward_distant_local_mae = out.forward_distant_local_mae.data();
    o.forward_distant_candidate_mae = out.forward_distant_candidate_mae.data();
    o.forward_distant_match_decision = out.forward_distant_match_decision.data();
    o.backward_distant_local_mae = out.backward_distant_local_mae.data();
    o.backward_distant_candidate_mae = out.backward_distant_candidate_mae.data();
    o.backward_distant_match_decision = out.backward_distant_match_decision.data();
    {
        std::lock_guard<std::mutex> lock(cx.mutex());
        upload(cx, kCur, f);
        upload(cx, kRef, past_prediction);
        upload(cx, kFuture, future);
        cx.check(vc1cu_analyze_b_picture(cx.handle(), &p, kCur, kRef, kFuture,
                                         reinterpret_cast<const vc1cu_mv*>(future_anchor_mvs.data()),
                                         future_anchor_4mv.data(), fraction_num, fraction_den,
                                         static_cast<int>(mode), &o),
                 "vc1cu_analyze_b_picture");
    }
    out.forward_macroblocks = static_cast<size_t>(o.forward_macroblocks);
    out.backward_macroblocks = static_cast<size_t>(o.backward_macroblocks);
    out.interpolated_macroblocks = static_cast<size_t>(o.interpolated_macroblocks);
    out.direct_macroblocks = static_cast<size_t>(o.direct_macroblocks);
    out.intra_macroblocks = static_cast<size_t>(o.intra_macroblocks);
    out.moved_macroblocks = static_cast<size_t>(o.moved_macroblocks);
    out.fractional_chroma_macroblocks = static_cast<size_t>(o.fractional_chroma_macroblocks);
    out.mean_abs_residual = o.mean_abs_residual;
    out.rate_complexity = o.rate_complexity;
    out.motion_sad = o.motion_sad;
    out.motion_bits = o.motion_bits;
    return out;
}

Vc1Encoder::IntensityComp Vc1Encoder::estimate_intensity_comp_cuda(const Frame& f, const Frame& ref,
                                                                   const std::vector<MotionVector>& mvs) const {
    CudaComputeContext& cx = context(c_);
    const vc1cu_params p = cuda_params(c_);
    vc1cu_intensity ic{};
    {
        std::lock_guard<std::mutex> lock(cx.mutex());
        upload(cx, kCur, f);
        upload(cx, kRef, ref);
        cx.check(vc1cu_estimate_intensity_comp(cx.handle(), &p, kCur, kRef,
                                               reinterpret_cast<const vc1cu_mv*>(mvs.data()), &ic),
                 "vc1cu_estimate_intensity_comp");
    }
    IntensityComp out;
    out.enabled = ic.enabled != 0;
    out.lumscale = static_cast<uint8_t>(ic.lumscale);
    out.lumshift = static_cast<uint8_t>(ic.lumshift);
    return out;
}

double Vc1Encoder::scene_change_score_cuda(const Frame& f, const Frame& ref) const {
    CudaComputeContext& cx = context(c_);
    const vc1cu_params p = cuda_params(c_);
    double score = 0.0;
    std::lock_guard<std::mutex> lock(cx.mutex());
    upload(cx, kCur, f);
    upload(cx, kRef, ref);
    cx.check(vc1cu_scene_change_score(cx.handle(), &p, kCur, kRef, c_.fade_compensation ? 1 : 0, c_.scene_threshold,
                                      &score),
             "vc1cu_scene_change_score");
    return score;
}

}  // namespace libvc1
