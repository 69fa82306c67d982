// vc1cu_bpic.cu - the B-picture macroblock decision on the device
// (Vc1Encoder::analyze_b_picture_mode, encoder_motion.cpp:753-1005).
//
// The two core passes (forward against the past anchor, backward against the future anchor,
// P-intra off) run as ordinary core passes. Two kernels follow them:
//   b_cost_kernel    one CTA of 256 threads per (picture, macroblock), one thread per luma
//                    pixel: the four candidate predictions (forward, backward and the direct
//                    pair scaled from the anchor's collocated vector), their SADs and the
//                    four-8x8 mean intra proxy. Fully parallel; reads the frames through L2.
//   b_decide_kernel  one CTA per picture walking the macroblocks in wavefront order
//                    (t = x + 2y). The MV predictors read the decisions already made for the
//                    left, top and top-right neighbours, so the macroblocks of one t are
//                    independent and one __syncthreads separates consecutive t.
#include <cuda_runtime.h>

#include "vc1cu_core.cuh"
#include "vc1cu_pred.cuh"

namespace vc1cu {

constexpr unsigned FULL = 0xffffffffu;

// scale_direct (encoder_motion.cpp:819-833): the direct-mode vector of a collocated anchor
// MV, BFRACTION-scaled and pulled into the decoder's MV range.
__device__ __forceinline__ int2 scale_direct(const DevParams& P, int2 col, int bfrac, bool inverse, int mode, int mx,
                                             int my) {
    const int n = inverse ? bfrac - 256 : bfrac;
    int2 mv;
    if (mode_halfpel(mode)) {
        mv.x = 2 * arshift(col.x * n + 255, 9);
        mv.y = 2 * arshift(col.y * n + 255, 9);
    } else {
        mv.x = arshift(col.x * n + 128, 8);
        mv.y = arshift(col.y * n + 128, 8);
    }
    mv.x = iclamp(mv.x, -60 - mx * 64, P.mbw * 64 - 4 - mx * 64);
    mv.y = iclamp(mv.y, -60 - my * 64, P.mbh * 64 - 4 - my * 64);
    return mv;
}

// motion_uses_hidden_padding(x0, y0, 16, 16, mv, mode, chroma = true, future)
__device__ __forceinline__ bool b_unsafe(const DevParams& P, int x0, int y0, int2 mv, int mode, bool future) {
    return hidden_luma(P, x0, y0, 16, 16, mv.x, mv.y, mode) || hidden_chroma_f(P, x0, y0, 16, 16, mv.x, mv.y, future);
}

// Candidate costs of one macroblock (encoder_motion.cpp:844-888) and its B-intra proxy
// (:936-943). Thread = pixel (tx, ty) of the macroblock; warp w holds rows 2w and 2w+1.
__global__ void __launch_bounds__(256) b_cost_kernel(const __grid_constant__ DevParams P, const BDesc* descs) {
    const BDesc& d = descs[blockIdx.y];
    const int pos = blockIdx.x, mx = pos % P.mbw, my = pos / P.mbw;
    const int x0 = mx * 16, y0 = my * 16;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ uint32_t s_sum[3][8];
    __shared__ uint32_t s_abs[8];
    const int2 col = d.anchor[pos];
    const int2 df = scale_direct(P, col, d.bfrac, false, d.mode, mx, my);
    const int2 db = scale_direct(P, col, d.bfrac, true, d.mode, mx, my);
    const int2 fm = d.fmv[pos], bm = d.bmv[pos];
    const int vw = imin(16, P.W - x0), vh = imin(16, P.H - y0);
    const bool in = tx < vw && ty < vh;
    const bool bil = mode_bilinear(d.mode);
    uint32_t fb = 0, id = 0, q = 0;  // packed 16-bit sums: forward|backward, interpolated|direct, left|right
    int src = 0;
    if (in) {
        const GlobSampler sp{d.past.y, d.past.pitch_y, P.W, P.H};
        const GlobSampler sf{d.future.y, d.future.pitch_y, P.W, P.H};
        int pf[1], pb[1], pdf[1], pdb[1];
        predict_row<1>(sp, bil, P.rnd, fm.x, fm.y, x0 + tx, y0 + ty, pf);
        predict_row<1>(sf, bil, P.rnd, bm.x, bm.y, x0 + tx, y0 + ty, pb);
        predict_row<1>(sp, bil, P.rnd, df.x, df.y, x0 + tx, y0 + ty, pdf);
        predict_row<1>(sf, bil, P.rnd, db.x, db.y, x0 + tx, y0 + ty, pdb);
        src = d.cur.y[(size_t)(y0 + ty) * d.cur.pitch_y + x0 + tx];
        fb = (uint32_t)iabs(src - pf[0]) | ((uint32_t)iabs(src - pb[0]) << 16);
        id = (uint32_t)iabs(src - ((pf[0] + pb[0] + 1) >> 1)) | ((uint32_t)iabs(src - ((pdf[0] + pdb[0] + 1) >> 1)) << 16);
        q = tx < 8 ? (uint32_t)src : ((uint32_t)src << 16);
    }
    // 16-bit fields cannot carry: a macroblock sums at most 256 * 255 < 2^16 per field
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        fb += __shfl_xor_sync(FULL, fb, o);
        id += __shfl_xor_sync(FULL, id, o);
        q += __shfl_xor_sync(FULL, q, o);
    }
    if (lane == 0) {
        s_sum[0][warp] = fb;
        s_sum[1][warp] = id;
        s_sum[2][warp] = q;
    }
    __syncthreads();
    // visible_block_mean (encoder_entropy.cpp:496-509) of this pixel's 8x8 block
    const int half = ty >> 3, right = tx >> 3;
    uint32_t qs = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w) qs += s_sum[2][half * 4 + w];
    qs = right ? (qs >> 16) : (qs & 0xFFFFu);
    const int bx = x0 + right * 8, by = y0 + half * 8;
    const uint32_t bw8 = (uint32_t)imax(0, imin(8, P.W - bx)), bh8 = (uint32_t)imax(0, imin(8, P.H - by));
    const uint32_t nn = bw8 * bh8;
    const int mean = nn ? (int)((qs + nn / 2) / nn) : 128;
    uint32_t a = in ? (uint32_t)iabs(src - mean) : 0u;
#pragma unroll
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
    if (lane == 0) s_abs[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sfb = 0, sid = 0, intra = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            sfb += s_sum[0][w];
            sid += s_sum[1][w];
            intra += s_abs[w];
        }
        const bool safe_fm = !b_unsafe(P, x0, y0, fm, d.mode, false), safe_bm = !b_unsafe(P, x0, y0, bm, d.mode, true);
        const bool safe_df = !b_unsafe(P, x0, y0, df, d.mode, false), safe_db = !b_unsafe(P, x0, y0, db, d.mode, true);
        uint4 c;
        c.x = safe_fm ? (sfb & 0xFFFFu) : kBCostInvalid;
        c.y = safe_bm ? (sfb >> 16) : kBCostInvalid;
        c.z = (safe_fm && safe_bm) ? (sid & 0xFFFFu) : kBCostInvalid;
        c.w = (safe_df && safe_db) ? (sid >> 16) : kBCostInvalid;
        d.out.cost[pos] = c;
        d.out.intra[pos] = intra;
    }
}

// v rounded to `bits` significant bits, nearest-even
__device__ __forceinline__ unsigned __int128 round_sig(unsigned __int128 v, int bits) {
    const uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    const int nbits = hi ? 128 - __clzll((long long)hi) : (lo ? 64 - __clzll((long long)lo) : 0);
    if (nbits <= bits) return v;
    const int drop = nbits - bits;
    const unsigned __int128 one = 1;
    const unsigned __int128 rem = v & ((one << drop) - 1), halfv = one << (drop - 1);
    v >>= drop;
    if (rem > halfv || (rem == halfv && (v & 1))) v += 1;
    return v << drop;
}

// The candidate score static_cast<long double>(cost) + lambda * rate_bits
// (encoder_motion.cpp:927): lambda * rate is a double product (53 significant bits), the
// sum a long double. With lambda = lam_m * 2^-lam_s both are integers scaled by 2^lam_s,
// so the scaled, rounded integers order exactly like the reference's long doubles.
__device__ __forceinline__ unsigned __int128 b_score(const BDesc& d, int mant_bits, uint64_t cost, uint32_t rate) {
    const unsigned __int128 prod = round_sig((unsigned __int128)d.lam_m * rate, 53);
    return round_sig(((unsigned __int128)cost << d.lam_s) + prod, mant_bits);
}

// predictor_info(field, mbw, mbh, mx, my).pre (encoder_motion.cpp:1312-1352) over a
// decoder MV field in HBM whose earlier wavefront positions are final.
__device__ int2 b_predictor(const DevParams& P, const int2* field, int mx, int my) {
    const int mbw = P.mbw;
    int2 A = make_int2(0, 0), B = A, C = A;
    const bool a_valid = my > 0, c_valid = mx > 0, b_valid = my > 0 && mbw > 1;
    if (a_valid) A = field[(my - 1) * mbw + mx];
    if (c_valid) C = field[my * mbw + mx - 1];
    if (b_valid) B = field[(my - 1) * mbw + ((mx == mbw - 1) ? mx - 1 : mx + 1)];
    int2 pre = make_int2(0, 0);
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if ((int)a_valid + (int)b_valid + (int)c_valid > 1) {
        pre.x = median3(A.x, B.x, C.x);
        pre.y = median3(A.y, B.y, C.y);
    }
    pullback(pre, mx * 64, my * 64, mbw * 64 - 4, P.mbh * 64 - 4, -60);
    return pre;
}

__device__ __forceinline__ bool frac_chroma(int2 v) {
    return (v.x & 3) || (v.y & 3) || ((v.x / 4) & 1) || ((v.y / 4) & 1);
}

// The decision of one macroblock (encoder_motion.cpp:889-996).
__device__ void b_decide_mb(const DevParams& P, const BDesc& d, int mx, int my, uint64_t tot[kBTotCount]) {
    const int pos = my * P.mbw + mx;
    const int2 col = d.anchor[pos];
    const int2 df = scale_direct(P, col, d.bfrac, false, d.mode, mx, my);
    const int2 db = scale_direct(P, col, d.bfrac, true, d.mode, mx, my);
    const int2 fm = d.fmv[pos], bm = d.bmv[pos];
    const uint4 c4 = d.out.cost[pos];
    auto dec = [](uint32_t v) -> uint64_t { return v == kBCostInvalid ? (1ull << 54) : (uint64_t)v; };
    const int2 fpred = b_predictor(P, d.out.fmv, mx, my), bpred = b_predictor(P, d.out.bmv, mx, my);
    const uint32_t fbits = mv_rate_bits(P, fm, fpred, d.mode, false);
    const uint32_t bbits = mv_rate_bits(P, bm, bpred, d.mode, false);
    const uint32_t ibits = mv_rate_bits(P, bm, bpred, d.mode, true) + mv_rate_bits(P, fm, fpred, d.mode, false) + 2;
    const uint32_t ftype = d.below_half ? 1u : 2u, btype = d.below_half ? 2u : 1u;
    const uint64_t penalty = d.anchor4[pos] ? 1000000000ull : 0ull;
    // Direct, Forward, Backward, Interpolated: the reference's candidate order (:920-925)
    const uint64_t cost[4] = {dec(c4.w) + penalty, dec(c4.x) + penalty, dec(c4.y) + penalty, dec(c4.z)};
    const uint32_t rate[4] = {0u, fbits + ftype, bbits + btype, ibits};
    int best = 0;
    unsigned __int128 best_key = b_score(d, P.mant_bits, cost[0], rate[0]);
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        const unsigned __int128 key = b_score(d, P.mant_bits, cost[k], rate[k]);
        if (key < best_key) { best_key = key; best = k; }
    }
    const uint64_t intra_sad = d.out.intra[pos];
    uint64_t gate = cost[best];
    const uint64_t fs = d.fscreen[pos], bs = d.bscreen[pos];
    if (fs < gate) gate = fs;
    if (bs < gate) gate = bs;
    const uint64_t ig = intra_sad + d.intra_guard;
    d.out.ratio[pos] = gate > 0 ? __ddiv_rn(__ull2double_rn(ig), __ull2double_rn(gate)) : __longlong_as_double(0x7ff0000000000000ll);
    const bool intra =
        !P.disable_b_intra && ig < (uint64_t)llround(__dmul_rn(__ull2double_rn(gate), P.inter_intra_threshold));
    const uint32_t marker = (uint32_t)(kMvDiffBits0[35] > kMvDiffBits0[72] ? kMvDiffBits0[35] : kMvDiffBits0[72]) + 1u;
    tot[kBTotSelSad] += intra ? intra_sad : cost[best];
    tot[kBTotRateSad] += cost[best];
    tot[kBTotSelRate] += intra ? marker : rate[best];
    tot[kBTotPixels] += (uint64_t)imax(0, imin(16, P.W - mx * 16)) * (uint64_t)imax(0, imin(16, P.H - my * 16));
    int mode;
    int2 of, ob;
    if (intra) {
        mode = VC1CU_BMB_INTRA;
        of = ob = make_int2(0, 0);
        tot[kBTotIntra]++;
    } else if (best == 0) {
        mode = VC1CU_BMB_DIRECT; of = df; ob = db; tot[kBTotDirect]++;
    } else if (best == 1) {
        mode = VC1CU_BMB_FORWARD; of = fm; ob = db; tot[kBTotForward]++;
    } else if (best == 2) {
        mode = VC1CU_BMB_BACKWARD; of = df; ob = bm; tot[kBTotBackward]++;
    } else {
        mode = VC1CU_BMB_INTERPOLATED; of = fm; ob = bm; tot[kBTotInterpolated]++;
    }
    d.out.modes[pos] = (uint8_t)mode;
    d.out.fmv[pos] = of;
    d.out.bmv[pos] = ob;
    if (of.x || of.y || ob.x || ob.y) tot[kBTotMoved]++;
    if (frac_chroma(of) || frac_chroma(ob)) tot[kBTotFrac]++;
}

__global__ void __launch_bounds__(128) b_decide_kernel(const __grid_constant__ DevParams P, const BDesc* descs) {
    const BDesc& d = descs[blockIdx.x];
    const int mbw = P.mbw, mbh = P.mbh, mbs = mbw * mbh;
    __shared__ unsigned long long s_tot[kBTotCount];
    if (threadIdx.x < kBTotCount) s_tot[threadIdx.x] = 0;
    // the core passes' distant_* arrays, carried through (encoder_motion.cpp:810-815)
    for (int i = threadIdx.x; i < mbs; i += blockDim.x) {
        d.out.fdl[i] = d.fdl[i];
        d.out.fdc[i] = d.fdc[i];
        d.out.fdd[i] = d.fdd[i];
        d.out.bdl[i] = d.bdl[i];
        d.out.bdc[i] = d.bdc[i];
        d.out.bdd[i] = d.bdd[i];
    }
    uint64_t tot[kBTotCount];
#pragma unroll
    for (int k = 0; k < kBTotCount; ++k) tot[k] = 0;
    const int tmax = (mbw - 1) + 2 * (mbh - 1);
    for (int t = 0; t <= tmax; ++t) {
        const int ylo = imax(0, (t - (mbw - 1) + 1) / 2), yhi = imin(mbh - 1, t / 2);
        for (int my = ylo + (int)threadIdx.x; my <= yhi; my += (int)blockDim.x) b_decide_mb(P, d, t - 2 * my, my, tot);
        __syncthreads();  // this wavefront's decisions are the next ones' predictors
    }
#pragma unroll
    for (int k = 0; k < kBTotCount; ++k)
        if (tot[k]) atomicAdd(&s_tot[k], (unsigned long long)tot[k]);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < kBTotCount; ++k) d.out.itotals[k] = s_tot[k];
        const unsigned long long px = s_tot[kBTotPixels];
        d.out.totals[0] = px ? __ddiv_rn(__ull2double_rn(s_tot[kBTotSelSad]), __ull2double_rn(px)) : 0.0;
        d.out.totals[1] = px ? __ddiv_rn(__ull2double_rn(s_tot[kBTotRateSad]), __ull2double_rn(px)) : 0.0;
        d.out.itotals[kBTotSelRate] = s_tot[kBTotSelRate] + 1;  // the progressive B MVMODE bit
    }
}

// Vc1Encoder::chroma_mc_sample (encoder_motion_compensation.cpp:417-447): future selects the
// B future-reference rounding of the chroma vector (away from the even value).
__device__ __forceinline__ int chroma_mc(const uint8_t* p, int pitch, int w, int h, int x, int y, int mvx, int mvy,
                                         bool future, int rnd) {
    int uvx = arshift(mvx + ((mvx & 3) == 3), 1);
    int uvy = arshift(mvy + ((mvy & 3) == 3), 1);
    if (future) {
        uvx = uvx < 0 ? uvx - (uvx & 1) : uvx + (uvx & 1);
        uvy = uvy < 0 ? uvy - (uvy & 1) : uvy + (uvy & 1);
    } else {
        uvx = uvx < 0 ? uvx + (uvx & 1) : uvx - (uvx & 1);
        uvy = uvy < 0 ? uvy + (uvy & 1) : uvy - (uvy & 1);
    }
    const int ix = floor_div4(uvx), iy = floor_div4(uvy);
    const int fx = (uvx - ix * 4) * 2, fy = (uvy - iy * 4) * 2;
    const int sx = x + ix, sy = y + iy;
    auto S = [&](int xx, int yy) { return (int)__ldg(p + (size_t)iclamp(yy, 0, h - 1) * pitch + iclamp(xx, 0, w - 1)); };
    const int a = S(sx, sy);
    if (!fx && !fy) return a;
    const int b = S(sx + 1, sy), c = S(sx, sy + 1), d = S(sx + 1, sy + 1);
    return (a * (8 - fx) * (8 - fy) + b * fx * (8 - fy) + c * (8 - fx) * fy + d * fx * fy + (rnd ? 28 : 32)) >> 6;
}

// Vc1Encoder::visible_block_mean (encoder_entropy.cpp:496-509) of the 8x8 block at (x0, y0)
__device__ int block_mean(const uint8_t* p, int pitch, int w, int h, int x0, int y0) {
    const int vw = imax(0, imin(8, w - x0)), vh = imax(0, imin(8, h - y0));
    if (!vw || !vh) return 128;
    uint32_t sum = 0;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) sum += __ldg(p + (size_t)(y0 + y) * pitch + x0 + x);
    const uint32_t n = (uint32_t)(vw * vh);
    return (int)((sum + n / 2) / n);
}

// The B prediction of an analysis (encoder_motion.cpp:1030-1053): one thread per luma pixel and,
// for even coordinates, the co-sited chroma pair. Forward / Backward: motion_compensate_mb
// (encoder_motion_compensation.cpp:474-525); Direct / Interpolated: motion_compensate_bi_mb
// (:659-711); Intra: the visible mean of each source 8x8 block.
__global__ void b_mc_kernel(const __grid_constant__ DevParams P, DevFrame cur, DevFrame past, DevFrame fut,
                            const uint8_t* modes, const int2* fmv, const int2* bmv, int mode, uint8_t* dy, uint8_t* du,
                            uint8_t* dv, int pitch_y, int pitch_c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= P.W || y >= P.H) return;
    const int pos = (y >> 4) * P.mbw + (x >> 4);
    const int m = modes[pos];
    const int cw = P.W / 2, ch = P.H / 2, cx = x >> 1, cy = y >> 1;
    const bool chroma = !(x & 1) && !(y & 1) && cx < cw && cy < ch;
    if (m == VC1CU_BMB_INTRA) {
        dy[(size_t)y * pitch_y + x] = (uint8_t)block_mean(cur.y, cur.pitch_y, P.W, P.H, x & ~7, y & ~7);
        if (chroma) {
            du[(size_t)cy * pitch_c + cx] = (uint8_t)block_mean(cur.u, cur.pitch_c, cw, ch, cx & ~7, cy & ~7);
            dv[(size_t)cy * pitch_c + cx] = (uint8_t)block_mean(cur.v, cur.pitch_c, cw, ch, cx & ~7, cy & ~7);
        }
        return;
    }
    const bool bil = mode_bilinear(mode);
    if (m == VC1CU_BMB_FORWARD || m == VC1CU_BMB_BACKWARD) {
        const DevFrame& r = m == VC1CU_BMB_FORWARD ? past : fut;
        const int2 mv = m == VC1CU_BMB_FORWARD ? fmv[pos] : bmv[pos];
        int o[1];
        predict_row<1>(GlobSampler{r.y, r.pitch_y, P.W, P.H}, bil, P.rnd, mv.x, mv.y, x, y, o);
        dy[(size_t)y * pitch_y + x] = (uint8_t)o[0];
        if (chroma) {
            du[(size_t)cy * pitch_c + cx] = (uint8_t)chroma_mc(r.u, r.pitch_c, cw, ch, cx, cy, mv.x, mv.y, false, P.rnd);
            dv[(size_t)cy * pitch_c + cx] = (uint8_t)chroma_mc(r.v, r.pitch_c, cw, ch, cx, cy, mv.x, mv.y, false, P.rnd);
        }
        return;
    }
    const int2 a = fmv[pos], b = bmv[pos];
    int pa[1], pb[1];
    predict_row<1>(GlobSampler{past.y, past.pitch_y, P.W, P.H}, bil, P.rnd, a.x, a.y, x, y, pa);
    predict_row<1>(GlobSampler{fut.y, fut.pitch_y, P.W, P.H}, bil, P.rnd, b.x, b.y, x, y, pb);
    dy[(size_t)y * pitch_y + x] = (uint8_t)((pa[0] + pb[0] + 1) >> 1);
    if (chroma) {
        const int au = chroma_mc(past.u, past.pitch_c, cw, ch, cx, cy, a.x, a.y, false, P.rnd);
        const int bu = chroma_mc(fut.u, fut.pitch_c, cw, ch, cx, cy, b.x, b.y, true, P.rnd);
        const int av = chroma_mc(past.v, past.pitch_c, cw, ch, cx, cy, a.x, a.y, false, P.rnd);
        const int bv = chroma_mc(fut.v, fut.pitch_c, cw, ch, cx, cy, b.x, b.y, true, P.rnd);
        du[(size_t)cy * pitch_c + cx] = (uint8_t)((au + bu + 1) >> 1);
        dv[(size_t)cy * pitch_c + cx] = (uint8_t)((av + bv + 1) >> 1);
    }
}

cudaError_t launch_b_mc(const DevParams& P, const DevFrame& cur, const DevFrame& past, const DevFrame& fut,
                        const uint8_t* modes, const int2* fmv, const int2* bmv, int mode, uint8_t* dy, uint8_t* du,
                        uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s) {
    b_mc_kernel<<<dim3((unsigned)((P.W + 127) / 128), (unsigned)P.H), 128, 0, s>>>(P, cur, past, fut, modes, fmv, bmv, mode,
                                                                                  dy, du, dv, pitch_y, pitch_c);
    return cudaGetLastError();
}

cudaError_t launch_bpictures(const DevParams& P, const BDesc* d_descs, int n, cudaStream_t s) {
    const unsigned mbs = (unsigned)(P.mbw * P.mbh);
    b_cost_kernel<<<dim3(mbs, (unsigned)n), 256, 0, s>>>(P, d_descs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    b_decide_kernel<<<(unsigned)n, 128, 0, s>>>(P, d_descs);
    return cudaGetLastError();
}

}  // namespace vc1cu
