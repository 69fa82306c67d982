// ref_harness.cpp - C entry points into the reference encoder's own analysis functions.
//
// Test infrastructure only: this file is compiled together with the reference's
// unmodified sources (see Makefile) into oracle/_ref/libvc1ref.so. It lets the tests,
// the oracle's self-check and bench.py's CPU baseline call the reference's scalar (or
// SIMD-dispatched) code directly, the way the reference's white-box tests do
// (tests/staged_motion_estimation.cpp, tests/vulkan_compute_runtime.cpp link vc1_static and
// call Vc1Encoder members). Nothing in the product links this library.
#include "encoder_internal.h"

#include <chrono>
#include <cstring>
#include <thread>

#include "../include/vc1cu.h"

using libvc1::EncoderConfig;
using libvc1::Frame;
using libvc1::Vc1Encoder;
using MV = Vc1Encoder::MotionVector;
using Mode = Vc1Encoder::ProgressiveMvMode;

namespace {

struct RefEncoder {
    EncoderConfig cfg;
    std::unique_ptr<Vc1Encoder> enc;
};

EncoderConfig make_config(const vc1cu_params* p, int simd) {
    EncoderConfig c;
    c.width = p->width;
    c.height = p->height;
    c.display_width = p->display_width > 0 ? p->display_width : p->width;
    c.display_height = p->display_height > 0 ? p->display_height : p->height;
    c.pqindex = p->pqindex;
    c.halfqp = p->halfqp != 0;
    c.quantizer_type = p->nonuniform ? libvc1::QuantizerType::NonUniform : libvc1::QuantizerType::Uniform;
    c.motion_search_range = p->search_range;
    c.motion_local_search_range = std::min(p->local_search_range, p->search_range);
    c.me_algorithm = static_cast<vc1_me_algorithm_e>(p->me_algorithm);
    c.me_quality = static_cast<vc1_me_quality_e>(p->me_quality);
    c.subpixel_refinement = p->subpel != 0;
    c.fast_subpixel_refinement = p->fast_subpel != 0;
    c.subpixel_refinement_range = p->subpel_range;
    c.long_range_search_mode = static_cast<vc1_long_range_search_mode_e>(p->long_range_mode);
    c.distant_match_max_mae = p->distant_match_max_mae;
    c.inter_intra_threshold = p->inter_intra_threshold;
    c.rndctrl = p->rnd != 0;
    c.debug_disable_p_intra = p->disable_p_intra != 0;
    c.debug_disable_b_intra = p->disable_b_intra != 0;
    c.syntax = libvc1::StreamSyntax::Advanced;
    c.trellis = 0;
    c.adaptive_quality = false;
    c.aq_strength = 0.0;
    c.dquant = false;
    if (simd) {
        // --simd auto: per-primitive startup benchmark (encoder_core.cpp:3240-3243), run once
        // per process and reused by every encoder this harness creates.
        static const libvc1::SimdDispatch dispatch = libvc1::auto_select_simd(true, true).dispatch;
        c.simd_dispatch = dispatch;
    } else {
        c.simd_dispatch.tier.fill(libvc1::SimdTier::None);
    }
    return c;
}

Mode to_mode(int m) { return static_cast<Mode>(m); }

void fill_out(const Vc1Encoder::PAnalysis& a, vc1cu_panalysis* out) {
    const size_t n = a.mvs.size();
    for (size_t i = 0; i < n; ++i) {
        if (out->mvs) out->mvs[i] = {a.mvs[i].xq, a.mvs[i].yq};
        if (out->block_mvs)
            for (int k = 0; k < 4; ++k) out->block_mvs[i * 4 + k] = {a.block_mvs[i][k].xq, a.block_mvs[i][k].yq};
        if (out->use_4mv) out->use_4mv[i] = a.use_4mv[i];
        if (out->use_intra) out->use_intra[i] = a.use_intra[i];
        if (out->screen_sads) out->screen_sads[i] = a.screen_sads[i];
        if (out->inter_intra_cost_ratio) out->inter_intra_cost_ratio[i] = a.inter_intra_cost_ratio[i];
        if (out->distant_local_mae) out->distant_local_mae[i] = a.distant_local_mae[i];
        if (out->distant_candidate_mae) out->distant_candidate_mae[i] = a.distant_candidate_mae[i];
        if (out->distant_match_decision) out->distant_match_decision[i] = a.distant_match_decision[i];
    }
    out->mean_abs_residual = a.mean_abs_residual;
    out->rate_complexity = a.rate_complexity;
    out->motion_sad = a.motion_sad;
    out->moved_macroblocks = a.moved_macroblocks;
    out->fractional_chroma_macroblocks = a.fractional_chroma_macroblocks;
    out->four_mv_macroblocks = a.four_mv_macroblocks;
    out->intra_macroblocks = a.intra_macroblocks;
}

}  // namespace

extern "C" {

void* ref_frame_new(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h) {
    auto* f = new Frame;
    f->width = w;
    f->height = h;
    const size_t ny = static_cast<size_t>(w) * h, nc = static_cast<size_t>(w / 2) * (h / 2);
    f->y.assign(y, y + ny);
    if (u) f->u.assign(u, u + nc); else f->u.assign(nc, 128);
    if (v) f->v.assign(v, v + nc); else f->v.assign(nc, 128);
    return f;
}

void ref_frame_free(void* f) { delete static_cast<Frame*>(f); }

void ref_frame_read(void* fp, uint8_t* y, uint8_t* u, uint8_t* v) {
    const Frame& f = *static_cast<Frame*>(fp);
    if (y) std::memcpy(y, f.y.data(), f.y.size());
    if (u) std::memcpy(u, f.u.data(), f.u.size());
    if (v) std::memcpy(v, f.v.data(), f.v.size());
}

void* ref_encoder_new(const vc1cu_params* p, int simd_auto) {
    auto* r = new RefEncoder;
    r->cfg = make_config(p, simd_auto);
    r->enc = std::make_unique<Vc1Encoder>(r->cfg);
    return r;
}

void ref_encoder_free(void* h) { delete static_cast<RefEncoder*>(h); }

static Vc1Encoder& E(void* h) { return *static_cast<RefEncoder*>(h)->enc; }
static const Frame& F(void* f) { return *static_cast<Frame*>(f); }

uint64_t ref_block_sad_motion(void* h, void* cur, void* ref, int x0, int y0, int bw, int bh,
                              int xq, int yq, int mode) {
    return E(h).block_sad_motion(F(cur), F(ref), x0, y0, bw, bh, MV{xq, yq}, to_mode(mode));
}

uint64_t ref_block_sad_qpel(void* h, void* cur, void* ref, int x0, int y0, int bw, int bh, int xq, int yq) {
    return E(h).block_sad_qpel(F(cur), F(ref), x0, y0, bw, bh, MV{xq, yq});
}

uint64_t ref_block_satd_motion(void* h, void* cur, void* ref, int x0, int y0, int bw, int bh,
                               int xq, int yq, int mode) {
    return E(h).block_satd_motion(F(cur), F(ref), x0, y0, bw, bh, MV{xq, yq}, to_mode(mode));
}

uint64_t ref_mb_sad(void* h, void* cur, void* ref, int mx, int my, int dx, int dy, int stride) {
    return E(h).mb_sad(F(cur), F(ref), mx, my, dx, dy, stride);
}

uint64_t ref_frame_sad(void* h, void* cur, void* ref, int dx, int dy, int stride) {
    return E(h).frame_sad(F(cur), F(ref), dx, dy, stride);
}

void ref_global_motion(void* h, void* cur, void* ref, int range, int* dx, int* dy, uint64_t* sad) {
    const auto g = E(h).global_motion_search(F(cur), F(ref), range);
    *dx = g.dx;
    *dy = g.dy;
    *sad = g.full_sad;
}

void ref_predict_luma(void* h, void* ref, int x0, int y0, int bw, int bh, int xq, int yq, int mode,
                      uint8_t* dst, int dst_stride) {
    E(h).predict_luma_motion_block(dst, dst_stride, F(ref), x0, y0, bw, bh, MV{xq, yq}, to_mode(mode));
}

// Integer motion search of one MB, given the spatial predictor state of a whole-pass
// MV field (mvs: mbw*mbh, the 1-MV field analyze_p_picture_core keeps).
void ref_integer_motion(void* h, void* cur, void* ref, int mx, int my, const vc1cu_mv* field,
                        int gdx, int gdy, int range, int* dx, int* dy, uint64_t* sad) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    std::vector<MV> mv(static_cast<size_t>(mbw) * mbh);
    for (size_t i = 0; i < mv.size(); ++i) mv[i] = MV{field[i].xq, field[i].yq};
    const auto pi = e.predictor_info(mv, mbw, mbh, mx, my);
    Vc1Encoder::GlobalMotionResult g{gdx, gdy, 0};
    const auto r = e.integer_motion_local(F(cur), F(ref), mx, my, pi, g, range);
    *dx = r.dx;
    *dy = r.dy;
    *sad = r.full_sad;
}

int ref_analyze_p_core(void* h, void* cur, void* ref, int mode, int allow_intra, const vc1cu_mv* seed,
                       const vc1cu_panalysis* seed_distant, vc1cu_panalysis* out) {
    try {
        auto& e = E(h);
        const auto& c = static_cast<RefEncoder*>(h)->cfg;
        const size_t mbs = static_cast<size_t>((c.width + 15) / 16) * ((c.height + 15) / 16);
        Vc1Encoder::PAnalysis s;
        if (seed) {
            s.mvs.resize(mbs);
            for (size_t i = 0; i < mbs; ++i) s.mvs[i] = MV{seed[i].xq, seed[i].yq};
            s.distant_local_mae.assign(mbs, -1.0);
            s.distant_candidate_mae.assign(mbs, -1.0);
            s.distant_match_decision.assign(mbs, 0);
            if (seed_distant) {
                for (size_t i = 0; i < mbs; ++i) {
                    if (seed_distant->distant_local_mae) s.distant_local_mae[i] = seed_distant->distant_local_mae[i];
                    if (seed_distant->distant_candidate_mae) s.distant_candidate_mae[i] = seed_distant->distant_candidate_mae[i];
                    if (seed_distant->distant_match_decision) s.distant_match_decision[i] = seed_distant->distant_match_decision[i];
                }
            }
        }
        const auto a = e.analyze_p_picture_core(F(cur), F(ref), to_mode(mode), allow_intra != 0, seed ? &s : nullptr);
        fill_out(a, out);
        out->global_dx = out->global_dy = 0;
        out->global_full_sad = 0;
        if (!seed && c.motion_search_range > 0) {
            const auto g = e.global_motion_search(F(cur), F(ref),
                                                  std::min(c.motion_search_range, std::max(0, c.motion_local_search_range)));
            out->global_dx = g.dx;
            out->global_dy = g.dy;
            out->global_full_sad = g.full_sad;
        }
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// One analyze_b_picture_mode call (forward + backward core passes and the per-MB B mode
// decision) with intensity compensation off and no search reuse cache.
int ref_analyze_b(void* h, void* cur, void* past, void* future, const vc1cu_mv* anchor_mvs, const uint8_t* anchor_4mv,
                  int fraction_num, int fraction_den, int mode, vc1cu_banalysis* out) {
    try {
        auto& e = E(h);
        const auto& c = static_cast<RefEncoder*>(h)->cfg;
        const size_t mbs = static_cast<size_t>((c.width + 15) / 16) * ((c.height + 15) / 16);
        std::vector<MV> amv(mbs);
        std::vector<uint8_t> a4(anchor_4mv, anchor_4mv + mbs);
        for (size_t i = 0; i < mbs; ++i) amv[i] = MV{anchor_mvs[i].xq, anchor_mvs[i].yq};
        const auto a = e.analyze_b_picture_mode(F(cur), F(past), F(future), amv, a4, Vc1Encoder::IntensityComp{},
                                                fraction_num, fraction_den, to_mode(mode), nullptr, nullptr, nullptr);
        for (size_t i = 0; i < mbs; ++i) {
            if (out->modes) out->modes[i] = static_cast<uint8_t>(a.modes[i]);
            if (out->forward_mvs) out->forward_mvs[i] = {a.forward_mvs[i].xq, a.forward_mvs[i].yq};
            if (out->backward_mvs) out->backward_mvs[i] = {a.backward_mvs[i].xq, a.backward_mvs[i].yq};
            if (out->inter_intra_cost_ratio) out->inter_intra_cost_ratio[i] = a.inter_intra_cost_ratio[i];
            if (out->forward_distant_local_mae) out->forward_distant_local_mae[i] = a.forward_distant_local_mae[i];
            if (out->forward_distant_candidate_mae) out->forward_distant_candidate_mae[i] = a.forward_distant_candidate_mae[i];
            if (out->forward_distant_match_decision) out->forward_distant_match_decision[i] = a.forward_distant_match_decision[i];
            if (out->backward_distant_local_mae) out->backward_distant_local_mae[i] = a.backward_distant_local_mae[i];
            if (out->backward_distant_candidate_mae) out->backward_distant_candidate_mae[i] = a.backward_distant_candidate_mae[i];
            if (out->backward_distant_match_decision) out->backward_distant_match_decision[i] = a.backward_distant_match_decision[i];
        }
        out->forward_macroblocks = a.forward_macroblocks;
        out->backward_macroblocks = a.backward_macroblocks;
        out->interpolated_macroblocks = a.interpolated_macroblocks;
        out->direct_macroblocks = a.direct_macroblocks;
        out->intra_macroblocks = a.intra_macroblocks;
        out->moved_macroblocks = a.moved_macroblocks;
        out->fractional_chroma_macroblocks = a.fractional_chroma_macroblocks;
        out->mean_abs_residual = a.mean_abs_residual;
        out->rate_complexity = a.rate_complexity;
        out->motion_sad = a.motion_sad;
        out->motion_bits = a.motion_bits;
        out->mv_mode = static_cast<int32_t>(a.mv_mode);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Vc1Encoder::estimate_intensity_comp along a host MV field.
void ref_estimate_ic(void* h, void* cur, void* ref, const vc1cu_mv* mvs, vc1cu_intensity* out) {
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const size_t mbs = static_cast<size_t>((c.width + 15) / 16) * ((c.height + 15) / 16);
    std::vector<MV> field(mbs);
    for (size_t i = 0; i < mbs; ++i) field[i] = MV{mvs[i].xq, mvs[i].yq};
    const auto ic = E(h).estimate_intensity_comp(F(cur), F(ref), field);
    out->enabled = ic.enabled ? 1 : 0;
    out->lumscale = ic.lumscale;
    out->lumshift = ic.lumshift;
}

// Vc1Encoder::intensity_compensated_reference into dst (a frame handle of the same size).
void ref_ic_reference(void* h, void* ref, const vc1cu_intensity* ic, void* dst) {
    Vc1Encoder::IntensityComp k{ic->enabled != 0, static_cast<uint8_t>(ic->lumscale), static_cast<uint8_t>(ic->lumshift)};
    *static_cast<Frame*>(dst) = E(h).intensity_compensated_reference(F(ref), k);
}

// Vc1Encoder::scene_change_score with the given fade-compensation switch and threshold.
double ref_scene_change_score(void* h, void* cur, void* ref, int fade_compensation, double scene_threshold) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.fade_compensation = fade_compensation != 0;
    c.scene_threshold = scene_threshold;
    Vc1Encoder enc(c);
    return enc.scene_change_score(F(cur), F(ref));
}

// The B prediction of an analysis (modes, forward/backward MV state) exactly as
// sampled_b_mode_rd builds it for a macroblock (encoder_motion.cpp:1030-1053), for every MB.
void ref_b_predict(void* h, void* cur, void* past, void* future, const uint8_t* modes, const vc1cu_mv* fmv,
                   const vc1cu_mv* bmv, int mode, void* dst) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const Frame& f = F(cur);
    Frame& pred = *static_cast<Frame*>(dst);
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            const MV fm{fmv[pos].xq, fmv[pos].yq}, bm{bmv[pos].xq, bmv[pos].yq};
            const auto m = static_cast<Vc1Encoder::BMbMode>(modes[pos]);
            if (m == Vc1Encoder::BMbMode::Intra) {
                for (int k = 0; k < 6; ++k) {
                    const std::vector<uint8_t>* src = nullptr;
                    std::vector<uint8_t>* d = nullptr;
                    int sw = 0, sh = 0, dw = 0, dh = 0, bx = 0, by = 0;
                    if (k < 4) {
                        src = &f.y; d = &pred.y; sw = c.width; sh = c.height; dw = pred.width; dh = pred.height;
                        bx = mx * 2 + (k & 1); by = my * 2 + ((k >> 1) & 1);
                    } else {
                        src = (k == 4) ? &f.u : &f.v; d = (k == 4) ? &pred.u : &pred.v;
                        sw = c.width / 2; sh = c.height / 2; dw = pred.width / 2; dh = pred.height / 2; bx = mx; by = my;
                    }
                    const int mean = Vc1Encoder::visible_block_mean(*src, sw, sh, bx * 8, by * 8);
                    for (int yy = 0; yy < 8 && by * 8 + yy < dh; ++yy)
                        for (int xx = 0; xx < 8 && bx * 8 + xx < dw; ++xx)
                            (*d)[static_cast<size_t>(by * 8 + yy) * dw + bx * 8 + xx] = static_cast<uint8_t>(mean);
                }
            } else if (m == Vc1Encoder::BMbMode::Forward) {
                e.motion_compensate_mb(pred, F(past), mx, my, fm, to_mode(mode));
            } else if (m == Vc1Encoder::BMbMode::Backward) {
                e.motion_compensate_mb(pred, F(future), mx, my, bm, to_mode(mode));
            } else {
                e.motion_compensate_bi_mb(pred, F(past), F(future), mx, my, fm, bm, to_mode(mode));
            }
        }
}

// Reconstruction of each (MB, parent) with its chosen transform type as
// evaluate_transform_parent forms it (encoder_transform.cpp:1569-1585): inverse_partition of
// every partition's levels (layout of ref_forward_quant for type_mask) added to the prediction;
// dequantised at PQINDEX, or at per-MB mquant with the derived flags (either may be null).
void ref_reconstruct(void* h, void* pred, const int16_t* levels, int type_mask, const uint8_t* block_types,
                     const uint8_t* mquant, const uint8_t* derived, void* dst) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const size_t mbs = static_cast<size_t>(mbw) * mbh;
    int tindex[5] = {-1, -1, -1, -1, -1}, nt = 0;
    for (int t = 1; t <= 4; ++t)
        if (type_mask & (1 << (t - 1))) tindex[t] = nt++;
    const Frame& pf = F(pred);
    Frame& out = *static_cast<Frame*>(dst);
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx)
            for (int k = 0; k < 6; ++k) {
                const size_t mb = static_cast<size_t>(my) * mbw + mx;
                const int t = block_types[mb * 6 + k];
                const auto type = static_cast<Vc1Encoder::TransformType>(t);
                const int16_t* q64 = levels + ((static_cast<size_t>(tindex[t]) * mbs + mb) * 6 + k) * 64;
                const std::vector<uint8_t>& pp = k < 4 ? pf.y : (k == 4 ? pf.u : pf.v);
                std::vector<uint8_t>& dp = k < 4 ? out.y : (k == 4 ? out.u : out.v);
                const int w = k < 4 ? c.width : c.width / 2, hh = k < 4 ? c.height : c.height / 2;
                const int bx = k < 4 ? mx * 2 + (k & 1) : mx, by = k < 4 ? my * 2 + ((k >> 1) & 1) : my;
                std::array<int, 64> residual{};
                for (int part = 0; part < Vc1Encoder::transform_part_count(type); ++part) {
                    int ox, oy, bw, bh;
                    Vc1Encoder::transform_part_geometry(type, part, ox, oy, bw, bh);
                    std::array<int, 64> q{};
                    for (int y = 0; y < bh; ++y)
                        for (int x = 0; x < bw; ++x) q[y * 8 + x] = q64[(oy + y) * 8 + ox + x];
                    const auto r = e.inverse_partition(type, q, mquant ? mquant[mb] : c.pqindex,
                                                       derived ? derived[mb] != 0 : false);
                    for (int y = 0; y < bh; ++y)
                        for (int x = 0; x < bw; ++x) residual[(oy + y) * 8 + ox + x] = r[y * 8 + x];
                }
                for (int yy = 0; yy < 8 && by * 8 + yy < hh; ++yy)
                    for (int xx = 0; xx < 8 && bx * 8 + xx < w; ++xx) {
                        const size_t off = static_cast<size_t>(by * 8 + yy) * w + bx * 8 + xx;
                        dp[off] = static_cast<uint8_t>(std::clamp(static_cast<int>(pp[off]) + residual[yy * 8 + xx], 0, 255));
                    }
            }
}

// In-place loop filters of a frame handle: apply_i_like_loop_filter, or apply_p_loop_filter
// with per-MB block vectors (4), coded-block patterns and transform kinds (6) and intra bits.
void ref_loop_filter_i(void* h, void* frame) { E(h).apply_i_like_loop_filter(*static_cast<Frame*>(frame)); }

void ref_loop_filter_p(void* h, void* frame, const vc1cu_mv* bmv, const uint8_t* cbp, const uint8_t* tt,
                       const uint8_t* intra, int main_profile) {
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const size_t mbs = static_cast<size_t>(mbw) * mbh;
    std::vector<std::array<MV, 4>> b(mbs);
    std::vector<std::array<uint8_t, 6>> cb(mbs), t(mbs);
    std::vector<uint8_t> in(intra, intra + mbs);
    for (size_t i = 0; i < mbs; ++i) {
        for (int k = 0; k < 4; ++k) b[i][k] = MV{bmv[i * 4 + k].xq, bmv[i * 4 + k].yq};
        for (int k = 0; k < 6; ++k) {
            cb[i][k] = cbp[i * 6 + k];
            t[i][k] = tt[i * 6 + k];
        }
    }
    if (main_profile) {
        // the Main Profile branch of apply_p_loop_filter_plane (encoder_filter.cpp:616-619)
        EncoderConfig mc = c;
        mc.syntax = libvc1::StreamSyntax::Wmv9Main;
        Vc1Encoder(mc).apply_p_loop_filter(*static_cast<Frame*>(frame), b, cb, t, in, mbw, mbh);
        return;
    }
    E(h).apply_p_loop_filter(*static_cast<Frame*>(frame), b, cb, t, in, mbw, mbh);
}

// Vc1Encoder::apply_i_overlap (mode 0 None, 1 All, 2 Select with flags) or, with p_picture set,
// apply_p_overlap (flags = the intra map; OVERLAP on), on a signed padded frame held as int32
// planes (in place).
void ref_overlap(void* h, int p_picture, int mode, const uint8_t* flags, int32_t* y, int32_t* u, int32_t* v) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.overlap = true;
    Vc1Encoder enc(c);
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const size_t mbs = static_cast<size_t>(mbw) * mbh;
    Vc1Encoder::SignedFrame f;
    f.width = mbw * 16;
    f.height = mbh * 16;
    const size_t ny = static_cast<size_t>(f.width) * f.height, nc = ny / 4;
    f.y.assign(y, y + ny);
    f.u.assign(u, u + nc);
    f.v.assign(v, v + nc);
    if (p_picture) {
        enc.apply_p_overlap(f, std::vector<uint8_t>(flags, flags + mbs), mbw, mbh);
    } else {
        Vc1Encoder::OverlapPlan plan;
        plan.mode = static_cast<Vc1Encoder::OverlapMode>(mode);
        plan.flags.assign(mbs, 0);
        if (flags) plan.flags.assign(flags, flags + mbs);
        enc.apply_i_overlap(f, plan);
    }
    std::copy(f.y.begin(), f.y.end(), y);
    std::copy(f.u.begin(), f.u.end(), u);
    std::copy(f.v.begin(), f.v.end(), v);
}

// The transform type choose_transform_mb picks per MB with the throughput preset
// (fast_transform_rdo, variable transforms, trellis 0, no DQUANT).
void ref_fast_transform_types(void* h, void* src, void* pred, uint8_t* types) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.fast_transform_rdo = true;
    c.variable_transforms = true;
    c.trellis = 0;
    c.dquant = false;
    Vc1Encoder enc(c);
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx)
            types[my * mbw + mx] =
                static_cast<uint8_t>(enc.choose_transform_mb(F(src), F(pred), mx, my, 0, true, c.pqindex, false).type);
}

// The whole analyze_p_picture (qpel seed pass, seeded mode passes, sampled-RD mode
// decision, final pass, optional fade passes). Reports the chosen mode and IC state.
int ref_analyze_p_picture(void* h, void* cur, void* ref, vc1cu_panalysis* out, int* chosen_mode, int* ic_enabled) {
    try {
        const auto a = E(h).analyze_p_picture(F(cur), F(ref));
        fill_out(a, out);
        *chosen_mode = static_cast<int>(a.mv_mode);
        *ic_enabled = a.intensity.enabled ? 1 : 0;
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// The harness encoder's configuration with the mode decision's fields of a vc1cu_ppic_cfg.
static EncoderConfig ppic_config(void* h, const vc1cu_ppic_cfg* pc) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.trellis = pc->trd.trellis;
    c.variable_transforms = pc->trd.variable_transforms != 0;
    c.extended_transform_signaling = pc->trd.extended_transform_signaling != 0;
    c.ac_mode = pc->trd.use_vlc ? libvc1::AcMode::Auto : libvc1::AcMode::Esc3;
    c.hrd_enabled = pc->trd.hrd_enabled != 0;
    c.fast_transform_rdo = pc->fast_transform_rdo != 0;
    c.dquant = pc->dquant != 0;
    c.fade_compensation = pc->fade_compensation != 0;
    c.fade_min_gain = pc->fade_min_gain;
    return c;
}

// analyze_p_picture under a vc1cu_ppic_cfg, with the returned analysis's motion bits.
int ref_analyze_p_picture_cfg(void* h, const vc1cu_ppic_cfg* pc, void* cur, void* ref, vc1cu_panalysis* out,
                              int* chosen_mode, int* ic_enabled, uint64_t* motion_bits) {
    try {
        const Vc1Encoder e(ppic_config(h, pc));
        const auto a = e.analyze_p_picture(F(cur), F(ref));
        fill_out(a, out);
        *chosen_mode = static_cast<int>(a.mv_mode);
        *ic_enabled = a.intensity.enabled ? 1 : 0;
        *motion_bits = a.motion_bits;
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// The plain candidates of analyze_p_picture (encoder_motion.cpp:541-566): each of the four modes'
// analysis, its estimate_p_motion_bits and its sampled_p_mode_rd score, as the reference computes
// them (scores in long double).
int ref_p_mode_scores(void* h, const vc1cu_ppic_cfg* pc, void* cur, void* ref, uint64_t* bits, long double* scores) {
    try {
        const EncoderConfig c = ppic_config(h, pc);
        const Vc1Encoder e(c);
        EncoderConfig nc = c;
        nc.adaptive_quality = false;
        nc.aq_strength = 0.0;
        const Vc1Encoder neutral(nc);
        const Mode modes[4] = {Mode::OneMvQpel, Mode::OneMvHpel, Mode::OneMvHpelBilinear, Mode::MixedMv};
        Frame pred = e.empty_frame();
        const auto qseed = e.analyze_p_picture_core(F(cur), F(ref), Mode::OneMvQpel, false, nullptr);
        for (int i = 0; i < 4; ++i) {
            auto cand = i == 0 ? qseed : e.analyze_p_picture_core(F(cur), F(ref), modes[i], false, &qseed);
            cand.motion_bits = e.estimate_p_motion_bits(cand, false);
            bits[i] = cand.motion_bits;
            scores[i] = e.sampled_p_mode_rd(F(cur), F(ref), cand, cand.motion_bits, pred, neutral);
        }
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// analyze_b_picture's two analyses (encoder_motion.cpp:1066-1088) and their sampled_b_mode_rd
// scores (:1089-1094) in long double, no forward intensity compensation; *chosen = 1 when the
// bilinear analysis wins.
int ref_b_mode_scores(void* h, const vc1cu_ppic_cfg* pc, void* cur, void* past, void* future, const vc1cu_mv* anchor_mvs,
                      const uint8_t* anchor_4mv, int fraction_num, int fraction_den, long double* scores, int* chosen) {
    try {
        const EncoderConfig c = ppic_config(h, pc);
        const Vc1Encoder e(c);
        EncoderConfig nc = c;
        nc.adaptive_quality = false;
        nc.aq_strength = 0.0;
        const Vc1Encoder neutral(nc);
        const size_t mbs = static_cast<size_t>((c.width + 15) / 16) * ((c.height + 15) / 16);
        std::vector<MV> amv(mbs);
        std::vector<uint8_t> a4(anchor_4mv, anchor_4mv + mbs);
        for (size_t i = 0; i < mbs; ++i) amv[i] = MV{anchor_mvs[i].xq, anchor_mvs[i].yq};
        const Vc1Encoder::IntensityComp none{};
        auto q = e.analyze_b_picture_mode(F(cur), F(past), F(future), amv, a4, none, fraction_num, fraction_den,
                                          Mode::OneMvQpel, nullptr, nullptr, nullptr);
        auto hh = e.analyze_b_picture_mode(F(cur), F(past), F(future), amv, a4, none, fraction_num, fraction_den,
                                           Mode::OneMvHpelBilinear, nullptr, nullptr, &q.compensated_past);
        Frame pred = e.empty_frame();
        scores[0] = e.sampled_b_mode_rd(F(cur), F(past), F(future), q, pred, neutral);
        scores[1] = e.sampled_b_mode_rd(F(cur), F(past), F(future), hh, pred, neutral);
        const auto whole = e.analyze_b_picture(F(cur), F(past), F(future), amv, a4, none, fraction_num, fraction_den);
        *chosen = whole.mv_mode == Mode::OneMvHpelBilinear ? 1 : 0;
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// reconstruct_i_signed_padded (encoder_encode.cpp:814-887) at the given trellis (0 scalar, 1, 2),
// DQUANT on or off, the perceptual scale at aq_strength (0: off), with the overlap plan (mode 0 none, 1 all, 2 select
// with flags) whose edge source it reads; the signed planes of the padded raster go to y, u, v.
// mquant / derived (when set) receive the DQUANT plan the function forms (choose_intra_mquant,
// make_dquant_plan, dquant_mb_derived; :826-833).
void ref_reconstruct_intra(void* h, int dquant, double aq_strength, int trellis, void* src, int overlap,
                           const uint8_t* flags, int32_t* y, int32_t* u, int32_t* v, uint8_t* mquant, uint8_t* derived) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.trellis = trellis;
    c.dquant = dquant != 0;
    c.adaptive_quality = aq_strength > 0.0;
    c.aq_strength = aq_strength;
    const Vc1Encoder e(c);
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const size_t mbs = static_cast<size_t>(mbw) * mbh;
    Vc1Encoder::OverlapPlan plan;
    plan.mode = overlap == 1 ? Vc1Encoder::OverlapMode::All : (overlap == 2 ? Vc1Encoder::OverlapMode::Select : Vc1Encoder::OverlapMode::None);
    plan.flags.assign(mbs, overlap == 1 ? 1 : 0);
    if (overlap == 2) plan.flags.assign(flags, flags + mbs);
    const auto sf = e.reconstruct_i_signed_padded(F(src), &plan);
    std::copy(sf.y.begin(), sf.y.end(), y);
    std::copy(sf.u.begin(), sf.u.end(), u);
    std::copy(sf.v.begin(), sf.v.end(), v);
    if (mquant || derived) {
        std::vector<int> desired(mbs, c.pqindex);
        if (c.dquant)
            for (int my = 0; my < mbh; ++my)
                for (int mx = 0; mx < mbw; ++mx) desired[static_cast<size_t>(my) * mbw + mx] = e.choose_intra_mquant(F(src), mx, my);
        const auto dplan = e.make_dquant_plan(desired, mbw, mbh);
        for (size_t i = 0; i < mbs; ++i) {
            if (mquant) mquant[i] = static_cast<uint8_t>(dplan.mquant.empty() ? c.pqindex : dplan.mquant[i]);
            if (derived) derived[i] = Vc1Encoder::dquant_mb_derived(dplan, i, mbw) ? 1 : 0;
        }
    }
}

// choose_i_overlap_plan (encoder_filter.cpp:277-343) with OVERLAP on, the given trellis, DQUANT on or
// off, the perceptual scale at aq_strength (0: off): the plan's mode (0 none, 1 all, 2 select) and flags.
void ref_choose_i_overlap(void* h, int dquant, double aq_strength, int trellis, void* src, int* mode, uint8_t* flags) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.trellis = trellis;
    c.overlap = true;
    c.dquant = dquant != 0;
    c.adaptive_quality = aq_strength > 0.0;
    c.aq_strength = aq_strength;
    const Vc1Encoder e(c);
    const auto plan = e.choose_i_overlap_plan(F(src));
    *mode = static_cast<int>(plan.mode);
    std::copy(plan.flags.begin(), plan.flags.end(), flags);
}

// estimate_p_motion_bits of an analysis given as host arrays (mbw*mbh vectors, 4 block vectors
// per MB, the 4-MV and intra flags) made in `mode`; UINT64_MAX when the reference throws.
uint64_t ref_estimate_p_motion_bits(void* h, const vc1cu_mv* mvs, const vc1cu_mv* block_mvs, const uint8_t* use_4mv,
                                    const uint8_t* use_intra, int mode, int intensity) {
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const size_t mbs = static_cast<size_t>((c.width + 15) / 16) * ((c.height + 15) / 16);
    Vc1Encoder::PAnalysis a;
    a.mv_mode = to_mode(mode);
    a.mvs.resize(mbs);
    a.block_mvs.resize(mbs);
    a.use_4mv.assign(use_4mv, use_4mv + mbs);
    a.use_intra.assign(use_intra, use_intra + mbs);
    for (size_t i = 0; i < mbs; ++i) {
        a.mvs[i] = MV{mvs[i].xq, mvs[i].yq};
        for (int k = 0; k < 4; ++k) a.block_mvs[i][k] = MV{block_mvs[i * 4 + k].xq, block_mvs[i * 4 + k].yq};
    }
    try {
        return E(h).estimate_p_motion_bits(a, intensity != 0);
    } catch (const std::exception&) {
        return UINT64_MAX;
    }
}

// Prediction of a PAnalysis-like MV field (motion_compensate_mb / _4mv), intra MBs at zero
// motion, into dst (a frame handle of the same size).
void ref_motion_compensate(void* h, void* ref, const vc1cu_mv* mvs, const vc1cu_mv* block_mvs,
                           const uint8_t* use_4mv, int mode, void* dst) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    Frame& d = *static_cast<Frame*>(dst);
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            if (use_4mv && use_4mv[pos]) {
                std::array<MV, 4> four;
                for (int k = 0; k < 4; ++k) four[k] = MV{block_mvs[pos * 4 + k].xq, block_mvs[pos * 4 + k].yq};
                e.motion_compensate_4mv(d, F(ref), mx, my, four);
            } else {
                e.motion_compensate_mb(d, F(ref), mx, my, MV{mvs[pos].xq, mvs[pos].yq}, to_mode(mode));
            }
        }
}

// The padded-raster prediction of the picture coder's reconstruction loop
// (motion_compensate_mb_padded / motion_compensate_4mv_padded, encoder_motion_compensation.cpp:573-660;
// encoder_encode.cpp:1183-1195): every whole macroblock of a (mbw*16) x (mbh*16) destination from
// a padded reference, intra MBs at zero motion.
void ref_motion_compensate_padded(void* h, void* ref, const vc1cu_mv* mvs, const vc1cu_mv* block_mvs,
                                  const uint8_t* use_4mv, int mode, void* dst) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    Frame& d = *static_cast<Frame*>(dst);
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            if (use_4mv && use_4mv[pos]) {
                std::array<MV, 4> four;
                for (int k = 0; k < 4; ++k) four[k] = MV{block_mvs[pos * 4 + k].xq, block_mvs[pos * 4 + k].yq};
                e.motion_compensate_4mv_padded(d, F(ref), mx, my, four);
            } else {
                e.motion_compensate_mb_padded(d, F(ref), mx, my, MV{mvs[pos].xq, mvs[pos].yq}, to_mode(mode));
            }
        }
}

// The B picture's padded-raster prediction (encoder_encode.cpp:1679-1688): Backward from the
// future reference, Forward from the past, Direct and Interpolated with
// motion_compensate_bi_mb_padded (:712-763); B-intra macroblocks are left as they are.
void ref_b_predict_padded(void* h, void* past, void* future, const uint8_t* modes, const vc1cu_mv* fmv,
                          const vc1cu_mv* bmv, int mode, void* dst) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    Frame& d = *static_cast<Frame*>(dst);
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            const MV f{fmv[pos].xq, fmv[pos].yq}, b{bmv[pos].xq, bmv[pos].yq};
            switch (modes[pos]) {
                case VC1CU_BMB_INTRA: break;
                case VC1CU_BMB_BACKWARD: e.motion_compensate_mb_padded(d, F(future), mx, my, b, to_mode(mode)); break;
                case VC1CU_BMB_FORWARD: e.motion_compensate_mb_padded(d, F(past), mx, my, f, to_mode(mode)); break;
                default: e.motion_compensate_bi_mb_padded(d, F(past), F(future), mx, my, f, b, to_mode(mode)); break;
            }
        }
}

// Forward transform + scalar quantisation (trellis off) of src - pred for all MBs, parents
// and the transform types in type_mask. Layout [type][mb][parent][64] over the set bits.
void ref_forward_quant(void* h, void* src, void* pred, int type_mask, double* coeffs, int16_t* levels) {
    auto& e = E(h);
    const auto& c = static_cast<RefEncoder*>(h)->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    const size_t mbs = static_cast<size_t>(mbw) * mbh;
    const Frame& s = F(src);
    const Frame& p = F(pred);
    size_t ti = 0;
    for (int t = 1; t <= 4; ++t) {
        if (!(type_mask & (1 << (t - 1)))) continue;
        const auto type = static_cast<Vc1Encoder::TransformType>(t);
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx)
                for (int k = 0; k < 6; ++k) {
                    const bool chroma = k >= 4;
                    const auto& sp = chroma ? (k == 4 ? s.u : s.v) : s.y;
                    const auto& pp = chroma ? (k == 4 ? p.u : p.v) : p.y;
                    const int w = chroma ? c.width / 2 : c.width, hh = chroma ? c.height / 2 : c.height;
                    const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
                    const size_t base = ((ti * mbs + static_cast<size_t>(my) * mbw + mx) * 6 + k) * 64;
                    double cc[64] = {0};
                    int16_t qq[64] = {0};
                    for (int part = 0; part < Vc1Encoder::transform_part_count(type); ++part) {
                        int ox, oy, bw, bh;
                        Vc1Encoder::transform_part_geometry(type, part, ox, oy, bw, bh);
                        const int px = bx * 8 + ox, py = by * 8 + oy;
                        std::array<double, 64> co{};
                        if (!(px >= w || py >= hh || px + bw <= 0 || py + bh <= 0))
                            co = e.forward_transform_residual_part(sp, pp, w, hh, px, py, bw, bh);
                        const auto q = e.quantize_inter_part(sp, pp, w, hh, px, py, bw, bh, false);
                        for (int y = 0; y < bh; ++y)
                            for (int x = 0; x < bw; ++x) {
                                cc[(oy + y) * 8 + ox + x] = co[y * 8 + x];
                                qq[(oy + y) * 8 + ox + x] = static_cast<int16_t>(q[y * 8 + x]);
                            }
                    }
                    if (coeffs) std::memcpy(coeffs + base, cc, sizeof cc);
                    if (levels) std::memcpy(levels + base, qq, sizeof qq);
                }
        ++ti;
    }
}

int ref_scalar_quantize_level(void* h, double coeff) { return E(h).scalar_quantize_level(coeff); }

// Vc1Encoder::choose_transform_mb (encoder_transform.cpp:1605-1780) for every MB of src against
// pred, with the handle's configuration and the transform RD fields of t (trellis, AQ, variable
// transforms, extended signaling, HRD; the throughput shortcut off); mquant per MB (NULL: PQINDEX).
// The harness encoder's configuration with a vc1cu_trd_cfg's EncoderConfig fields.
static EncoderConfig trd_config(void* h, const vc1cu_trd_cfg* t) {
    EncoderConfig c = static_cast<RefEncoder*>(h)->cfg;
    c.trellis = t->trellis;
    c.adaptive_quality = t->adaptive_quality != 0;
    c.aq_strength = t->aq_strength;
    c.variable_transforms = t->variable_transforms != 0;
    c.extended_transform_signaling = t->extended_transform_signaling != 0;
    c.hrd_enabled = t->hrd_enabled != 0;
    c.fast_transform_rdo = false;
    return c;
}

// An MbTransformDecision as a vc1cu_tdecision (and its 6 x 64 levels when levels is set).
static void fill_tdecision(const Vc1Encoder::MbTransformDecision& d, vc1cu_tdecision* out, int16_t* levels) {
    vc1cu_tdecision& o = *out;
    std::memset(&o, 0, sizeof o);
    o.type = static_cast<uint8_t>(d.type);
    o.signal_level = static_cast<uint8_t>(d.signal_level == Vc1Encoder::TransformSignalLevel::Macroblock
                                              ? 0
                                              : (d.signal_level == Vc1Encoder::TransformSignalLevel::Block ? 1 : 2));
    o.cbp = d.cbp;
    o.estimated_bits = static_cast<uint32_t>(d.estimated_bits);
    o.distortion = d.distortion;
    for (int k = 0; k < 6; ++k) {
        const auto& p = d.parents[static_cast<size_t>(k)];
        o.parent_type[k] = static_cast<uint8_t>(p.type);
        o.skip_mask[k] = p.skip_mask;
        o.parent_bits[k] = static_cast<uint32_t>(p.estimated_bits);
        o.parent_distortion[k] = p.distortion;
        if (levels)
            for (int i = 0; i < 64; ++i) levels[k * 64 + i] = p.qcoeff[static_cast<size_t>(i)];
    }
}

void ref_choose_transform(void* h, const vc1cu_trd_cfg* t, void* src, void* pred, const uint8_t* mquant,
                          vc1cu_tdecision* out, int16_t* levels) {
    const EncoderConfig c = trd_config(h, t);
    Vc1Encoder e(c);
    Vc1Encoder::TransformPicturePlan plan;
    plan.frame_level = t->frame_type > 0;
    plan.frame_type = static_cast<Vc1Encoder::TransformType>(t->frame_type > 0 ? t->frame_type : 1);
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            const auto d = e.choose_transform_mb(F(src), F(pred), mx, my, t->coding_set, t->use_vlc != 0,
                                                 mquant ? mquant[pos] : 0, t->dquantfrm != 0,
                                                 t->frame_type > 0 ? &plan : nullptr);
            fill_tdecision(d, out + pos, levels ? levels + pos * 384 : nullptr);
        }
}


// choose_dquant_transform_mb (encoder_aq.cpp:280-404) of every MB under a transform configuration,
// the DQUANT switches and the rate-control hooks it reads (rc_inter_block_weight,
// rc_prediction_residual_mean). rate_base receives each MB's base MQUANT as the function forms it
// (:284-310, restated here from the same member functions) for the device search to start from.
void ref_choose_dquant(void* h, const vc1cu_trd_cfg* t, int dquant, int predictable, double block_weight,
                       double residual_mean, void* src, void* pred, uint8_t* rate_base, vc1cu_tdecision* out,
                       uint8_t* mquant, int16_t* levels) {
    EncoderConfig c = trd_config(h, t);
    c.dquant = dquant != 0;
    c.aq_predictable_texture = predictable != 0;
    c.rc_inter_block_weight = block_weight;
    c.rc_prediction_residual_mean = residual_mean;
    const Vc1Encoder e(c);
    Vc1Encoder::TransformPicturePlan plan;
    plan.frame_level = t->frame_type > 0;
    plan.frame_type = static_cast<Vc1Encoder::TransformType>(t->frame_type > 0 ? t->frame_type : 1);
    const Frame& s = F(src);
    const Frame& pr = F(pred);
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    for (int my = 0; my < mbh; ++my)
        for (int mx = 0; mx < mbw; ++mx) {
            const size_t pos = static_cast<size_t>(my) * mbw + mx;
            int rb = e.rate_weighted_mquant(c.rc_inter_block_weight);
            if (c.rc_prediction_residual_mean > 0.0) {
                const int x0 = mx * 16, y0 = my * 16;
                const int bw = std::max(0, std::min(16, c.visible_width() - x0));
                const int bh = std::max(0, std::min(16, c.visible_height() - y0));
                uint64_t sad = 0;
                for (int y = 0; y < bh; ++y)
                    for (int x = 0; x < bw; ++x) {
                        const size_t o = static_cast<size_t>(y0 + y) * c.width + x0 + x;
                        sad += static_cast<uint64_t>(std::abs(static_cast<int>(s.y[o]) - static_cast<int>(pr.y[o])));
                    }
                const double local_mae = (bw > 0 && bh > 0) ? static_cast<double>(sad) / static_cast<double>(bw * bh) : 0.0;
                rb = e.residual_priority_mquant(rb, local_mae, c.rc_prediction_residual_mean);
            }
            if (c.adaptive_quality && c.aq_strength > 0.0 && c.dquant && rb > 1) {
                const auto priority = e.perceptual_mb_priority(s, mx, my, false);
                const int delta = std::clamp(static_cast<int>(std::lround(priority.requested_q_boost)), 0, std::min(2, rb - 1));
                rb = std::max(1, rb - delta);
            }
            rate_base[pos] = static_cast<uint8_t>(rb);
            const auto q = e.choose_dquant_transform_mb(s, pr, mx, my, t->coding_set, t->use_vlc != 0,
                                                        t->frame_type > 0 ? &plan : nullptr);
            mquant[pos] = static_cast<uint8_t>(q.mquant);
            fill_tdecision(q.tx, out + pos, levels ? levels + pos * 384 : nullptr);
        }
}

// The direct AC code length (0: none) of (run, level, last) in coding set `set`
// (Vc1Encoder::find_ac_vlc, encoder_entropy.cpp:182-192), and write_ac_coeff's lower envelope
// used by the trellis (trellis_rate_bits_for_set, encoder_transform.cpp:1811-1841).
int ref_ac_direct_bits(int set, int run, int level, int last) {
    const auto* e = Vc1Encoder::find_ac_vlc(set, run, level, last != 0);
    return e ? e->bits : 0;
}
int ref_ac_rate_bits(void* h, int set, int run, int level, int last) {
    return E(h).trellis_rate_bits_for_set(run, level, last != 0, set);
}

// CPU baseline over pairs that each carry their own encoder configuration (e.g. per-picture
// PQINDEX): analyze_p_picture + choose_transform_mb of the chosen prediction for every MB,
// one pair per worker thread at a time. Returns wall ns.
uint64_t ref_bench_analysis_multi(void** handles, void** curs, void** refs, int n_pairs, int threads) {
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n_pairs) break;
            auto* r = static_cast<RefEncoder*>(handles[i]);
            const auto& c = r->cfg;
            const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
            Vc1Encoder enc(c);
            Frame pred;
            pred.width = c.width;
            pred.height = c.height;
            pred.y.assign(static_cast<size_t>(c.width) * c.height, 0);
            pred.u.assign(static_cast<size_t>(c.width / 2) * (c.height / 2), 128);
            pred.v = pred.u;
            const Frame& cur = F(curs[i]);
            const Frame& ref = F(refs[i]);
            const auto a = enc.analyze_p_picture(cur, ref);
            for (int my = 0; my < mbh; ++my)
                for (int mx = 0; mx < mbw; ++mx) {
                    const size_t pos = static_cast<size_t>(my) * mbw + mx;
                    if (a.use_4mv[pos]) enc.motion_compensate_4mv(pred, ref, mx, my, a.block_mvs[pos]);
                    else enc.motion_compensate_mb(pred, ref, mx, my, a.mvs[pos], a.mv_mode);
                    (void)enc.choose_transform_mb(cur, pred, mx, my, 0, true, c.pqindex, false);
                }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    const auto t1 = std::chrono::steady_clock::now();
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
}

// CPU baseline of one GOP-planned step: first every P picture (analyze_p_picture +
// choose_transform_mb of its chosen prediction), then every B picture (analyze_b_picture
// against its two anchors, with the future anchor's MVs, Mixed-MV flags and intensity
// compensation from that P picture's analysis, as encoder_core.cpp:1086-1097 passes them),
// each phase one picture per worker thread at a time. Returns wall ns.
uint64_t ref_bench_gop_multi(void** p_handles, void** p_curs, void** p_refs, int n_p, void** b_handles, void** b_curs,
                             void** b_pasts, void** b_futures, const int* b_anchor, const int* b_num, const int* b_den,
                             int n_b, int threads) {
    std::vector<Vc1Encoder::PAnalysis> anchors(static_cast<size_t>(std::max(0, n_p)));
    std::atomic<int> next{0};
    auto p_worker = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n_p) break;
            const auto& c = static_cast<RefEncoder*>(p_handles[i])->cfg;
            const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
            Vc1Encoder enc(c);
            Frame pred;
            pred.width = c.width;
            pred.height = c.height;
            pred.y.assign(static_cast<size_t>(c.width) * c.height, 0);
            pred.u.assign(static_cast<size_t>(c.width / 2) * (c.height / 2), 128);
            pred.v = pred.u;
            const Frame& cur = F(p_curs[i]);
            const Frame& ref = F(p_refs[i]);
            anchors[i] = enc.analyze_p_picture(cur, ref);
            const auto& a = anchors[i];
            for (int my = 0; my < mbh; ++my)
                for (int mx = 0; mx < mbw; ++mx) {
                    const size_t pos = static_cast<size_t>(my) * mbw + mx;
                    if (a.use_4mv[pos]) enc.motion_compensate_4mv(pred, ref, mx, my, a.block_mvs[pos]);
                    else enc.motion_compensate_mb(pred, ref, mx, my, a.mvs[pos], a.mv_mode);
                    (void)enc.choose_transform_mb(cur, pred, mx, my, 0, true, c.pqindex, false);
                }
        }
    };
    std::atomic<int> bnext{0};
    auto b_worker = [&]() {
        for (;;) {
            const int i = bnext.fetch_add(1);
            if (i >= n_b) break;
            const auto& c = static_cast<RefEncoder*>(b_handles[i])->cfg;
            Vc1Encoder enc(c);
            const auto& a = anchors[static_cast<size_t>(b_anchor[i])];
            (void)enc.analyze_b_picture(F(b_curs[i]), F(b_pasts[i]), F(b_futures[i]), a.mvs, a.use_4mv, a.intensity,
                                        b_num[i], b_den[i]);
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(p_worker);
        for (auto& t : pool) t.join();
    }
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(b_worker);
        for (auto& t : pool) t.join();
    }
    const auto t1 = std::chrono::steady_clock::now();
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
}

// CPU baseline doing the GPU arm's work with the reference's own functions, one job pool for
// the P and the B pictures. Per P picture: the five core passes analyze_p_picture chains
// (quarter-pel seed pass, the half-pel, bilinear and Mixed-MV passes seeded by it, the final
// Mixed-MV pass with P-intra seeded by the Mixed-MV pass; encoder_motion.cpp:524-597), the fade
// estimate along the final vectors, the prediction of the final field and quantize_inter_part
// (forward transform + quantiser) of every partition of all four transform types. Per B picture:
// analyze_b_picture_mode in quarter-pel and in half-pel bilinear mode against its anchors, with
// the future anchor's final vectors (intensity compensation off). A B job waits for its anchor's
// P job; every P job is taken before any B job, so the pool cannot deadlock. Returns wall ns.
uint64_t ref_bench_gop_same(void** p_handles, void** p_curs, void** p_refs, int n_p, void** b_handles, void** b_curs,
                            void** b_pasts, void** b_futures, const int* b_anchor, const int* b_num, const int* b_den,
                            int n_b, int threads) {
    const size_t np = static_cast<size_t>(std::max(0, n_p));
    std::vector<Vc1Encoder::PAnalysis> finals(np);
    std::unique_ptr<std::atomic<int>[]> done(new std::atomic<int>[np > 0 ? np : 1]);
    for (size_t i = 0; i < np; ++i) done[i].store(0);
    std::atomic<long long> sink{0};
    std::atomic<int> next{0};
    auto p_job = [&](int i) {
        const auto& c = static_cast<RefEncoder*>(p_handles[i])->cfg;
        const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
        Vc1Encoder enc(c);
        const Frame& cur = F(p_curs[i]);
        const Frame& ref = F(p_refs[i]);
        const auto seed = enc.analyze_p_picture_core(cur, ref, Mode::OneMvQpel, false, nullptr);
        (void)enc.analyze_p_picture_core(cur, ref, Mode::OneMvHpel, false, &seed);
        (void)enc.analyze_p_picture_core(cur, ref, Mode::OneMvHpelBilinear, false, &seed);
        const auto mixed = enc.analyze_p_picture_core(cur, ref, Mode::MixedMv, false, &seed);
        finals[i] = enc.analyze_p_picture_core(cur, ref, Mode::MixedMv, true, &mixed);
        const auto& a = finals[i];
        const auto ic = enc.estimate_intensity_comp(cur, ref, a.mvs);
        Frame pred;
        pred.width = c.width;
        pred.height = c.height;
        pred.y.assign(static_cast<size_t>(c.width) * c.height, 0);
        pred.u.assign(static_cast<size_t>(c.width / 2) * (c.height / 2), 128);
        pred.v = pred.u;
        for (int my = 0; my < mbh; ++my)
            for (int mx = 0; mx < mbw; ++mx) {
                const size_t pos = static_cast<size_t>(my) * mbw + mx;
                if (a.use_4mv[pos]) enc.motion_compensate_4mv(pred, ref, mx, my, a.block_mvs[pos]);
                else enc.motion_compensate_mb(pred, ref, mx, my, a.mvs[pos], Mode::MixedMv);
            }
        long long acc = ic.enabled ? 1 : 0;
        for (int t = 1; t <= 4; ++t) {
            const auto type = static_cast<Vc1Encoder::TransformType>(t);
            for (int my = 0; my < mbh; ++my)
                for (int mx = 0; mx < mbw; ++mx)
                    for (int k = 0; k < 6; ++k) {
                        const bool chroma = k >= 4;
                        const auto& sp = chroma ? (k == 4 ? cur.u : cur.v) : cur.y;
                        const auto& pp = chroma ? (k == 4 ? pred.u : pred.v) : pred.y;
                        const int w = chroma ? c.width / 2 : c.width, hh = chroma ? c.height / 2 : c.height;
                        const int bx = chroma ? mx : mx * 2 + (k & 1), by = chroma ? my : my * 2 + ((k >> 1) & 1);
                        for (int part = 0; part < Vc1Encoder::transform_part_count(type); ++part) {
                            int ox, oy, bw, bh;
                            Vc1Encoder::transform_part_geometry(type, part, ox, oy, bw, bh);
                            const auto q = enc.quantize_inter_part(sp, pp, w, hh, bx * 8 + ox, by * 8 + oy, bw, bh, false);
                            acc += q[0];
                        }
                    }
        }
        sink.fetch_add(acc);
        done[i].store(1, std::memory_order_release);
    };
    auto b_job = [&](int i) {
        const auto& c = static_cast<RefEncoder*>(b_handles[i])->cfg;
        const size_t a_idx = static_cast<size_t>(b_anchor[i]);
        while (!done[a_idx].load(std::memory_order_acquire)) std::this_thread::yield();
        const auto& a = finals[a_idx];
        Vc1Encoder enc(c);
        for (const Mode m : {Mode::OneMvQpel, Mode::OneMvHpelBilinear}) {
            const auto r = enc.analyze_b_picture_mode(F(b_curs[i]), F(b_pasts[i]), F(b_futures[i]), a.mvs, a.use_4mv,
                                                      Vc1Encoder::IntensityComp{}, b_num[i], b_den[i], m, nullptr,
                                                      nullptr, nullptr);
            sink.fetch_add(static_cast<long long>(r.motion_sad));
        }
    };
    auto worker = [&]() {
        for (;;) {
            const int j = next.fetch_add(1);
            if (j >= n_p + n_b) break;
            if (j < n_p) p_job(j);
            else b_job(j - n_p);
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    const auto t1 = std::chrono::steady_clock::now();
    static std::atomic<long long> keep{0};
    keep.fetch_add(sink.load());
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
}

// CPU baseline: analyze_p_picture + choose_transform_mb of the chosen prediction for every
// MB of every (cur, ref) pair, one pair per worker thread at a time. Returns wall ns.
uint64_t ref_bench_analysis(void* h, void** curs, void** refs, int n_pairs, int threads) {
    auto* r = static_cast<RefEncoder*>(h);
    const auto& c = r->cfg;
    const int mbw = (c.width + 15) / 16, mbh = (c.height + 15) / 16;
    std::atomic<int> next{0};
    auto worker = [&]() {
        Vc1Encoder enc(c);
        Frame pred;
        pred.width = c.width;
        pred.height = c.height;
        pred.y.assign(static_cast<size_t>(c.width) * c.height, 0);
        pred.u.assign(static_cast<size_t>(c.width / 2) * (c.height / 2), 128);
        pred.v = pred.u;
        const int coding_set = 0;
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n_pairs) break;
            const Frame& cur = F(curs[i]);
            const Frame& ref = F(refs[i]);
            const auto a = enc.analyze_p_picture(cur, ref);
            for (int my = 0; my < mbh; ++my)
                for (int mx = 0; mx < mbw; ++mx) {
                    const size_t pos = static_cast<size_t>(my) * mbw + mx;
                    if (a.use_4mv[pos]) enc.motion_compensate_4mv(pred, ref, mx, my, a.block_mvs[pos]);
                    else enc.motion_compensate_mb(pred, ref, mx, my, a.mvs[pos], a.mv_mode);
                    (void)enc.choose_transform_mb(cur, pred, mx, my, coding_set, true, c.pqindex, false);
                }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    const auto t1 = std::chrono::steady_clock::now();
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
}

}  // extern "C"
