// vc1cu_core.cuh - device-side descriptors shared by the core-pass, global-search and
// transform kernels and the host shim.
#pragma once

#include <cstdint>

#include "vc1cu_common.cuh"

namespace vc1cu {

// A frame slot in HBM: three planes with 16-byte-aligned row pitches.
struct DevFrame {
    const uint8_t* y;
    const uint8_t* u;
    const uint8_t* v;
    int pitch_y, pitch_c;
};

// One result slot (Vc1Encoder::PAnalysis) in HBM, structure of arrays over macroblocks.
struct DevResult {
    int2* mvs;
    int2* bmv;             // 4 per MB
    uint8_t* use4;
    uint8_t* intra;
    uint64_t* screen;
    double* ratio;
    double* dl;
    double* dc;
    uint8_t* dd;
    uint64_t* chosen;      // per-MB chosen SAD (motion_sad summand)
    uint64_t* temporal;    // per-MB temporal SAD (rate_complexity summand)
    uint8_t* flags;        // bit0 moved, bit1 fractional chroma, bit2 long-range vector, bit3 4MV chosen
    uint32_t* done;        // wavefront flags (== epoch when the MB is final)
    int* global;           // [dx, dy] of the unseeded pass
    unsigned long long* gsad;
    double* totals;        // mean_abs_residual, rate_complexity
    unsigned long long* itotals;  // motion_sad, moved, frac, four, intra
};

struct alignas(64) PassDesc {
    unsigned char ref_tmap[128];  // TMA descriptor (CUtensorMap) of ref's luma plane, box = the
                                  // launch's window (wp x wh bytes); valid when ref_tma != 0
    int ref_tma;
    // Sub-pel prediction planes of ref for this pass's filter and rounding (nullptr: none): the
    // prediction of phase (hm, vm) whose integer origin is (x, y), for x in [-sp_border, W +
    // sp_border) and y likewise, at sp_planes + (vm * 4 + hm) * sp_stride + (y + sp_border) *
    // sp_pitch + x + sp_border.
    const uint8_t* sp_planes;
    int sp_pitch, sp_border;
    long long sp_stride;
    DevFrame cur, ref;
    int mode, allow_intra;
    int pq;                // this picture's PQINDEX
    double lambda;         // max(1, 0.35*pq)
    uint64_t lam_m;        // lambda = lam_m * 2^-lam_s exactly
    int lam_s;
    int seeded;            // 1: seed fields below are valid
    int seed_pass;         // index of the seeding pass in the same launch, -1 if produced earlier
    const int2* seed_mvs;
    const int2* seed_bmv;        // the seed pass's block vectors and P-intra flags (only used to
    const uint8_t* seed_intra;   // guess this pass's predictors before the wavefront wait)
    const uint64_t* lr_sig;      // long-range signature index of `ref` (long-range passes only)
    int lr_nx, lr_ny;            // its 8-pixel lattice
    const double* seed_dl;
    const double* seed_dc;
    const uint8_t* seed_dd;
    const int2* cands;           // learned passes: kLearnK integer-pixel candidates per MB
    uint8_t* fallback;           // learned passes: 1 where the candidates' best match is not good
    const uint8_t* only;         // non-null: only the MBs flagged here are computed (the others
                                 // keep the slot's contents and just publish their done flag)
    DevResult out;
    DevResult nb;                // no_wait passes: the field the neighbours' vectors are read from
    int no_wait;                 // 1: no wavefront waits; neighbours from `nb`, a finished field
    DevParams geom;              // this pass's picture geometry and configuration (read by the
                                 // kCoreMulti instantiation and the totals; the others take the
                                 // launch's parameter block)
};
constexpr int kLearnK = 4;       // candidates per macroblock of a learned pass
constexpr int kLearnRw = 8;      // window radius of a learned pass around its best candidate

// core_pass_kernel instantiations, as flags: each flag compiles out code that the launch's
// passes cannot reach (the launches are bound by instruction fetch, so a smaller footprint pays).
constexpr int kCoreSeededOnly = 1;    // every pass seeded: no integer-search code
constexpr int kCoreUnseededOnly = 2;  // every pass unseeded: no seeded refinement or speculation
constexpr int kCoreUmhLocal = 4;      // (with kCoreUnseededOnly) UMH with the search range equal to
                                      // the local range: no diamond or long-range code
constexpr int kCoreNoMixed = 8;       // (with kCoreSeededOnly or kCoreUmhLocal) no Mixed-MV pass: no 4-MV code
constexpr int kCoreWide = 16;         // one block per SM, all 255 registers (search windows that large
                                      // leave room for one block anyway); not with kCoreSeededOnly
constexpr int kCoreDefaultRefine = 32;  // (with kCoreSeededOnly or kCoreUmhLocal) me_quality SATD and the
                                        // full sub-pel stencils: no SAD-only, RATE or fast refinement code
constexpr int kCoreNoIntra = 64;        // (with kCoreDefaultRefine) no pass allows P-intra: no intra code
constexpr int kCoreLearned = 128;       // (with kCoreUnseededOnly) the integer search is the learned
                                        // candidates' exact costs and a short descent about the best
constexpr int kCoreMulti = 256;         // passes of pictures of different sizes in one launch: each
                                        // work item takes its pass's own geometry
constexpr int kCoreAny = 0;
constexpr int kCoreSeeded = kCoreSeededOnly;

// Shared-memory window geometry for one launch.
struct WinCfg {
    int rw;        // window radius in integer pixels around its centre MV
    int wh;        // window height = 16 + 2*rw + 3
    int wp;        // window row pitch = width: wh + 15 rounded up to 16 (16-byte-aligned origin)
    int seen_r;    // radius of the first-visit bitsets (0 = none)
    int seen_words;
    int keys_cap;  // capacity of the per-stage key array
    int warp_bytes;
    int tma;       // 1: windows wholly inside the picture are staged by one TMA tensor copy
};

// Arguments of one candidate-scoring launch (vc1cu_score_motion_batch[_law]).
struct ScoreArgs {
    const uint8_t* cur;
    const uint8_t* ref;
    int pitch, W, H;
    int x0, y0, bw, bh, stride, mode, rnd, metric, law;
};

struct LaunchStatus {
    int error;          // 0 ok, VC1CU_ERR_TIMEOUT
    int abort;
    unsigned int queue;
    unsigned int timeouts;
    unsigned int tcode;  // 1 + the work item of the first wait that gave up (0: none)
    unsigned int tmask;  // its lanes still waiting (lanes 0-3: left, top-left, top, top-right; lane 0: seed)
};

// A pass that reuses another pass's whole-frame search (same picture pair) takes its result.
struct GlobalCopy {
    const int* src_global;
    const unsigned long long* src_sad;
    int* dst_global;
    unsigned long long* dst_sad;
};

// One B-result slot (Vc1Encoder::BAnalysis) in HBM, structure of arrays over macroblocks.
struct DevBResult {
    uint8_t* modes;
    int2* fmv;                 // decoder forward / backward MV state
    int2* bmv;
    double* ratio;
    double* fdl;               // the core passes' distant_* arrays, copied through
    double* fdc;
    uint8_t* fdd;
    double* bdl;
    double* bdc;
    uint8_t* bdd;
    uint4* cost;               // per MB: forward, backward, interpolated, direct SAD (kBCostInvalid: 2^54)
    uint32_t* intra;           // per MB: the four-8x8 mean proxy
    unsigned long long* itotals;  // kBTot* below
    double* totals;            // mean_abs_residual, rate_complexity
};
constexpr uint32_t kBCostInvalid = 0xFFFFFFFFu;
enum {
    kBTotForward = 0, kBTotBackward, kBTotInterpolated, kBTotDirect, kBTotIntra, kBTotMoved, kBTotFrac,
    kBTotSelSad, kBTotRateSad, kBTotSelRate, kBTotPixels, kBTotCount
};

// One B picture's decision stage (encoder_motion.cpp:817-1001).
struct BDesc {
    DevFrame cur, past, future;
    const int2* fmv;           // forward / backward core passes
    const int2* bmv;
    const uint64_t* fscreen;
    const uint64_t* bscreen;
    const double* fdl;
    const double* fdc;
    const uint8_t* fdd;
    const double* bdl;
    const double* bdc;
    const uint8_t* bdd;
    const int2* anchor;        // the future anchor's MVs and Mixed-MV flags
    const uint8_t* anchor4;
    int bfrac;                 // BFRACTION scale: 128 (1/2), 85 (1/3), 170 (2/3)
    int below_half;
    int mode;
    uint64_t lam_m;            // B lambda max(1, 0.45*PQ) = lam_m * 2^-lam_s exactly
    int lam_s;
    uint64_t intra_guard;      // llround(lambda * 72)
    DevBResult out;
};

}  // namespace vc1cu
