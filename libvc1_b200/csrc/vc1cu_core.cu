// vc1cu_core.cu - one Vc1Encoder::analyze_p_picture_core pass per picture, many pictures
// per launch (encoder_motion.cpp:47-442).
//
// Execution model (sm_100a):
//   * persistent grid; each warp owns one macroblock at a time, taken from a global work
//     queue that interleaves the pictures of the batch in raster order, so every
//     dependency of an item was handed out before it;
//   * the raster-order dependency of the reference (left, top-left, top, top-right MVs of
//     the same pass, encoder_motion.cpp:1312-1466) is a wavefront: a warp waits on the
//     four neighbours' done flags (acquire loads, bounded spin that flags
//     VC1CU_ERR_TIMEOUT instead of hanging) and publishes its own MB with a release store;
//   * the reference search window of the MB is staged once into the warp's shared memory
//     with 128-bit loads on a 16-byte-aligned grid (edge-replicated outside the picture);
//     candidates outside it read HBM with clamping;
//   * integer stages score one candidate per lane; sub-pel stages split each candidate's
//     block into 8-pixel row segments across lanes; every selection uses the reference's
//     total orders, so the parallel evaluation returns the reference's exact choice.
#include <cuda_runtime.h>

#include "vc1cu_core.cuh"
#include "vc1cu_pred.cuh"

namespace vc1cu {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kListCap = 24;

// Optional per-phase SM-clock accounting of the core kernel, compiled only with
// -DVC1CU_PHASE_CLOCKS (a profiling build): slot [kind * 16 + phase] accumulates the cycles
// lane 0 of each warp spent in that phase, kind = seeded + 2 * Mixed-MV.
#ifdef VC1CU_PHASE_CLOCKS
__device__ unsigned long long g_phase_clk[64];
__device__ unsigned long long g_phase_cnt[64];
#define PHASE_START(kind) long long phase_t = clock64(); const int phase_kind = (kind)
#define PHASE_MARK(k)                                                                 \
    do {                                                                              \
        const long long phase_n = clock64();                                          \
        if (m.lane == 0) {                                                            \
            atomicAdd(&g_phase_clk[phase_kind * 16 + (k)], (unsigned long long)(phase_n - phase_t)); \
            atomicAdd(&g_phase_cnt[phase_kind * 16 + (k)], 1ull);                     \
        }                                                                             \
        phase_t = phase_n;                                                            \
    } while (0)
#else
#define PHASE_START(kind)
#define PHASE_MARK(k)
#endif

// The kernel's dynamic shared memory. Every per-warp buffer is addressed as an offset from
// this symbol, so all of its accesses compile to shared-space loads and stores (a pointer
// kept in a struct would otherwise degrade to generic addressing).
extern __shared__ __align__(16) uint8_t g_smem[];
extern __shared__ __align__(16) uint32_t g_smem32[];  // the same memory, 32-bit words

// Reference-window sampler: bytes read by direct index into the shared array (so always
// shared-space loads). off: byte offset of the window; ww: row pitch; (wx0, wy0): origin.
// ---- the index-checked build (-DVC1CU_INDEX_CHECK) ----------------------------------------
// Every guarded access tests its index against the buffer it addresses. A violation is counted
// with its site and index (the first one is kept) and the access is skipped: a read returns 0,
// a write is dropped, a work item is abandoned. vc1cu_debug_index_faults reads the record. In
// the default build the guards are the constant true.
enum IndexSite : int {
    kSiteWorkItem = 1,   // work item: pass index < npass, macroblock < the pass's raster
    kSiteWindow = 2,     // search-window read (x, y) inside the staged window
    kSiteKeys = 3,       // a stage's key slot < the key array's capacity
    kSiteSeen = 4,       // first-visit bitset: (dx, dy) inside the bitset's square
    kSiteNeighbour = 5,  // neighbour macroblock inside the raster
    kSiteCands = 6,      // learned candidate of a macroblock inside the raster
    kSiteSignature = 7,  // long-range signature cell inside the reference's lattice
    kSiteStage = 8,      // window staging write inside the window
};
#ifdef VC1CU_INDEX_CHECK
__device__ unsigned int g_index_faults;
__device__ unsigned long long g_index_first;  // site << 40 | (index & (2^40 - 1)) of the first violation
__device__ __noinline__ void index_fault(int site, long long index) {
    if (atomicAdd(&g_index_faults, 1u) == 0)
        atomicExch(&g_index_first, ((unsigned long long)site << 40) | ((unsigned long long)index & 0xFFFFFFFFFFull));
}
#define IDX_OK(cond, site, index) ((cond) || (index_fault((site), (long long)(index)), false))
#else
#define IDX_OK(cond, site, index) true
#endif

struct WinSampler {
    uint32_t off;
    int ww, wx0, wy0;
    int wh = 1 << 30;  // rows staged (checked builds test reads against it)
    __device__ __forceinline__ int operator()(int x, int y) const {
        const int rx = x - wx0, ry = y - wy0;
        if (!IDX_OK(rx >= 0 && ry >= 0 && rx < ww && ry < wh, kSiteWindow, (long long)ry * 65536 + rx)) return 0;
        return g_smem[off + (uint32_t)(ry * ww + rx)];
    }
};

template <class T>
struct SPtr {
    uint32_t off;
    __device__ __forceinline__ T* get() const { return reinterpret_cast<T*>(g_smem + off); }
    __device__ __forceinline__ operator T*() const { return get(); }
    __device__ __forceinline__ T& operator[](int i) const { return get()[i]; }
};

struct SpecBlk;

// Per-warp shared-memory carve.
struct WarpMem {
    SPtr<uint8_t> cur;          // 16x16 current MB (zero outside the visible raster)
    SPtr<uint8_t> win;          // reference window
    SPtr<uint32_t> seen;        // first-visit bitset of the sampled UMH stages
    SPtr<uint32_t> seen_full;   // first-visit bitset of the full-resolution stages
    SPtr<uint64_t> keys;        // per-stage candidate keys
    SPtr<int2> list_mv;         // staged-refinement candidate list
    SPtr<uint64_t> list_sad;
    SPtr<uint64_t> list_satd;
    SPtr<uint32_t> list_rate;
    SPtr<unsigned __int128> list_key;
    SPtr<int2> batch;           // scratch MV batch
    SPtr<uint64_t> batch_cost;
    SPtr<int2> stencil;         // sub-pel stencil MVs of the current refinement stage
    SPtr<uint64_t> top;         // sorted top-8 keys of the UMH search
    SPtr<uint32_t> cur2;        // current MB, even columns packed 4 per word: [row][2]
    SPtr<uint32_t> cur4;        // current MB, every 4th column packed: [row]
    SPtr<int> misc;             // small scalars: [0] top count, [1] compaction count
    SPtr<int2> cur_bmv;         // the current MB's four block MVs while it is searched
    SPtr<int2> nb_mv;           // 1-MV field of the left, top-left, top, top-right neighbours
    SPtr<int2> nb_bmv;          // their block MVs [4][4]
    SPtr<int> nb_intra;         // their P-intra flags
    SPtr<int2> spec_mv;         // shortlists kept across the wavefront wait [5][8]
    SPtr<uint64_t> spec_cost;   //   slot 0: the 16x16 refinement, slot k + 1: 8x8 block k
    SPtr<uint64_t> spec_satd;
    SPtr<SpecBlk> spec_blk;     // [5]
    SPtr<uint8_t> ctx;          // the macroblock's MbCtx
    SPtr<uint64_t> tma_bar;     // mbarrier of the window's TMA copy
};

struct Mb {
    int lane;
    uint64_t lam_m;   // this pass's lambda_me = lam_m * 2^-lam_s
    int lam_s;
    int mx, my, x0, y0, pos, aw, ah;  // aw/ah: visible wrt the internal raster (cur.width)
    const PassDesc* d;
    WarpMem sm;
    int wx0, wy0, wp, wh;  // window origin (wx0 a multiple of 16), row pitch = width, height
    GlobSampler gref;
    uint32_t tma_phase;    // parity of the window mbarrier's next phase
    bool tma_pending;      // a TMA window copy is in flight
#ifdef VC1CU_INDEX_CHECK
    int keys_cap;  // capacity of m.sm.keys
#endif
};

__device__ __forceinline__ bool win_inside(const Mb& m, int xa, int ya, int xb, int yb) {
    return xa >= m.wx0 && ya >= m.wy0 && xb < m.wx0 + m.wp && yb < m.wy0 + m.wh;
}

// SAD of one row segment of n <= 8 visible pixels against the current block at shared
// byte offset `cur`: the same predictions as predict_row<8> (sx = px + floor(xq/4) ...),
// evaluated with rolled loops and sliding windows so that each interpolation case is a few
// dozen instructions rather than an unrolled block.
template <class S>
__device__ __forceinline__ uint32_t sad_row8(const S& s, bool bilinear, int rnd, int xq, int yq, int px, int py, uint32_t cur,
                                             int n) {
    const int ix = floor_div4(xq), iy = floor_div4(yq);
    const int hm = xq - ix * 4, vm = yq - iy * 4;
    const int sx = px + ix, sy = py + iy;
    uint32_t acc = 0;
    if (!hm && !vm) {
#pragma unroll 1
        for (int i = 0; i < n; ++i) acc += (uint32_t)iabs((int)g_smem[cur + i] - s(sx + i, sy));
        return acc;
    }
    if (bilinear) {
        if (hm && vm) {
            const int r = rnd ? 1 : 2;
            int a0 = s(sx, sy) + s(sx, sy + 1);
#pragma unroll 1
            for (int i = 0; i < n; ++i) {
                const int a1 = s(sx + i + 1, sy) + s(sx + i + 1, sy + 1);
                acc += (uint32_t)iabs((int)g_smem[cur + i] - ((a0 + a1 + r) >> 2));
                a0 = a1;
            }
        } else if (hm) {
            const int r = rnd ? 0 : 1;
            int a0 = s(sx, sy);
#pragma unroll 1
            for (int i = 0; i < n; ++i) {
                const int a1 = s(sx + i + 1, sy);
                acc += (uint32_t)iabs((int)g_smem[cur + i] - ((a0 + a1 + r) >> 1));
                a0 = a1;
            }
        } else {
            const int r = rnd ? 0 : 1;
#pragma unroll 1
            for (int i = 0; i < n; ++i)
                acc += (uint32_t)iabs((int)g_smem[cur + i] - ((s(sx + i, sy) + s(sx + i, sy + 1) + r) >> 1));
        }
        return acc;
    }
    if (hm && vm) {
        const int shift = ((hm == 2 ? 1 : 5) + (vm == 2 ? 1 : 5)) >> 1;
        const int r1 = (1 << (shift - 1)) + (rnd ? 1 : 0) - 1;
        const Taps tv = mspel_taps(vm), th = mspel_taps(hm);
        auto col = [&](int x) { return arshift(apply(tv, s(x, sy - 1), s(x, sy), s(x, sy + 1), s(x, sy + 2)) + r1, shift); };
        int t0 = col(sx - 1), t1 = col(sx), t2 = col(sx + 1);
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            const int t3 = col(sx + i + 2);
            const int v = iclamp(arshift(apply(th, t0, t1, t2, t3) + 64 - (rnd ? 1 : 0), 7), 0, 255);
            acc += (uint32_t)iabs((int)g_smem[cur + i] - v);
            t0 = t1;
            t1 = t2;
            t2 = t3;
        }
        return acc;
    }
    if (vm) {
        const int bias = (vm == 2) ? (7 + (rnd ? 1 : 0)) : (31 + (rnd ? 1 : 0));
        const int sh = vm == 2 ? 4 : 6;
        const Taps tv = mspel_taps(vm);
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            const int x = sx + i;
            const int v = iclamp(arshift(apply(tv, s(x, sy - 1), s(x, sy), s(x, sy + 1), s(x, sy + 2)) + bias, sh), 0, 255);
            acc += (uint32_t)iabs((int)g_smem[cur + i] - v);
        }
        return acc;
    }
    const int bias = (hm == 2) ? (8 - (rnd ? 1 : 0)) : (32 - (rnd ? 1 : 0));
    const int sh = hm == 2 ? 4 : 6;
    const Taps th = mspel_taps(hm);
    int r0 = s(sx - 1, sy), r1 = s(sx, sy), r2 = s(sx + 1, sy);
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
        const int r3 = s(sx + i + 2, sy);
        const int v = iclamp(arshift(apply(th, r0, r1, r2, r3) + bias, sh), 0, 255);
        acc += (uint32_t)iabs((int)g_smem[cur + i] - v);
        r0 = r1;
        r1 = r2;
        r2 = r3;
    }
    return acc;
}

// The four predictions of predict_row<4>, evaluated like sad_row8 (rolled loops with
// sliding windows), delivered through a four-register queue.
template <class S>
__device__ __forceinline__ int4 pred_row4(const S& s, bool bilinear, int rnd, int xq, int yq, int px, int py) {
    const int ix = floor_div4(xq), iy = floor_div4(yq);
    const int hm = xq - ix * 4, vm = yq - iy * 4;
    const int sx = px + ix, sy = py + iy;
    int q0 = 0, q1 = 0, q2 = 0, q3 = 0;
    auto push = [&](int v) {
        q0 = q1;
        q1 = q2;
        q2 = q3;
        q3 = v;
    };
    if (!hm && !vm) {
#pragma unroll 1
        for (int i = 0; i < 4; ++i) push(s(sx + i, sy));
    } else if (bilinear) {
        const int r2 = rnd ? 1 : 2, r1 = rnd ? 0 : 1;
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int x = sx + i;
            push(hm && vm ? (s(x, sy) + s(x + 1, sy) + s(x, sy + 1) + s(x + 1, sy + 1) + r2) >> 2
                 : hm     ? (s(x, sy) + s(x + 1, sy) + r1) >> 1
                          : (s(x, sy) + s(x, sy + 1) + r1) >> 1);
        }
    } else if (hm && vm) {
        const int shift = ((hm == 2 ? 1 : 5) + (vm == 2 ? 1 : 5)) >> 1;
        const int r1 = (1 << (shift - 1)) + (rnd ? 1 : 0) - 1;
        const Taps tv = mspel_taps(vm), th = mspel_taps(hm);
        auto col = [&](int x) { return arshift(apply(tv, s(x, sy - 1), s(x, sy), s(x, sy + 1), s(x, sy + 2)) + r1, shift); };
        int t0 = col(sx - 1), t1 = col(sx), t2 = col(sx + 1);
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int t3 = col(sx + i + 2);
            push(iclamp(arshift(apply(th, t0, t1, t2, t3) + 64 - (rnd ? 1 : 0), 7), 0, 255));
            t0 = t1;
            t1 = t2;
            t2 = t3;
        }
    } else if (vm) {
        const int bias = (vm == 2) ? (7 + (rnd ? 1 : 0)) : (31 + (rnd ? 1 : 0));
        const int sh = vm == 2 ? 4 : 6;
        const Taps tv = mspel_taps(vm);
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int x = sx + i;
            push(iclamp(arshift(apply(tv, s(x, sy - 1), s(x, sy), s(x, sy + 1), s(x, sy + 2)) + bias, sh), 0, 255));
        }
    } else {
        const int bias = (hm == 2) ? (8 - (rnd ? 1 : 0)) : (32 - (rnd ? 1 : 0));
        const int sh = hm == 2 ? 4 : 6;
        const Taps th = mspel_taps(hm);
        int r0 = s(sx - 1, sy), r1 = s(sx, sy), r2 = s(sx + 1, sy);
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int r3 = s(sx + i + 2, sy);
            push(iclamp(arshift(apply(th, r0, r1, r2, r3) + bias, sh), 0, 255));
            r0 = r1;
            r1 = r2;
            r2 = r3;
        }
    }
    return make_int4(q0, q1, q2, q3);
}

// 16 shared-memory bytes starting at byte offset `off`, as four little-endian words.
__device__ __forceinline__ void win_load16(uint32_t off, uint32_t r[4]) {
    const uint32_t w = off >> 2;
    const uint32_t sh = (off & 3) * 8;
    const uint32_t w0 = g_smem32[w], w1 = g_smem32[w + 1], w2 = g_smem32[w + 2], w3 = g_smem32[w + 3],
                   w4 = g_smem32[w + 4];
    r[0] = __funnelshift_r(w0, w1, sh);
    r[1] = __funnelshift_r(w1, w2, sh);
    r[2] = __funnelshift_r(w2, w3, sh);
    r[3] = __funnelshift_r(w3, w4, sh);
}

// mb_sad of a full 16x16 MB from the window with packed byte SADs (__vsadu4), strides 1/2/4.
template <int STRIDE>
__device__ __forceinline__ uint32_t sad_packed(uint32_t cur_off, uint32_t cur2_off, uint32_t cur4_off, int wp, uint32_t base) {
    uint32_t acc = 0;
    const uint32_t c = cur_off >> 2, c2 = cur2_off >> 2, c4 = cur4_off >> 2;
#pragma unroll 4
    for (int y = 0; y < 16; y += STRIDE) {
        uint32_t r[4];
        win_load16(base + (uint32_t)(y * wp), r);
        if (STRIDE == 1) {
            acc += __vsadu4(r[0], g_smem32[c + y * 4 + 0]) + __vsadu4(r[1], g_smem32[c + y * 4 + 1]) +
                   __vsadu4(r[2], g_smem32[c + y * 4 + 2]) + __vsadu4(r[3], g_smem32[c + y * 4 + 3]);
        } else if (STRIDE == 2) {
            acc += __vsadu4(__byte_perm(r[0], r[1], 0x6420), g_smem32[c2 + y * 2 + 0]) +
                   __vsadu4(__byte_perm(r[2], r[3], 0x6420), g_smem32[c2 + y * 2 + 1]);
        } else {
            const uint32_t e = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
            acc += __vsadu4(e, g_smem32[c4 + y]);
        }
    }
    return acc;
}

// 16 bytes of a frame row starting at `p` (any alignment), as four little-endian words: five
// aligned word loads through the read-only path and funnel shifts. The fifth word can reach up
// to three bytes past the row's 16, which stay inside the frame's allocation (the next row, or
// the chroma planes after the last luma row).
__device__ __forceinline__ void glob_load16(const uint8_t* p, uint32_t r[4]) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(3));
    const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 3) * 8;
    const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3);
    const uint32_t w4 = sh ? __ldg(w + 4) : 0u;
    r[0] = __funnelshift_r(w0, w1, sh);
    r[1] = __funnelshift_r(w1, w2, sh);
    r[2] = __funnelshift_r(w2, w3, sh);
    r[3] = __funnelshift_r(w3, w4, sh);
}

// mb_sad of a full 16x16 MB whose reference block lies inside the frame, read from global
// memory (the frames stay in L2) with the same packed byte SADs as sad_packed.
template <int STRIDE>
__device__ __forceinline__ uint32_t sad_packed_glob(uint32_t cur_off, uint32_t cur2_off, uint32_t cur4_off,
                                                    const uint8_t* ref, int pitch) {
    uint32_t acc = 0;
    const uint32_t c = cur_off >> 2, c2 = cur2_off >> 2, c4 = cur4_off >> 2;
#pragma unroll 4
    for (int y = 0; y < 16; y += STRIDE) {
        uint32_t r[4];
        glob_load16(ref + (size_t)y * pitch, r);
        if (STRIDE == 1) {
            acc += __vsadu4(r[0], g_smem32[c + y * 4 + 0]) + __vsadu4(r[1], g_smem32[c + y * 4 + 1]) +
                   __vsadu4(r[2], g_smem32[c + y * 4 + 2]) + __vsadu4(r[3], g_smem32[c + y * 4 + 3]);
        } else if (STRIDE == 2) {
            acc += __vsadu4(__byte_perm(r[0], r[1], 0x6420), g_smem32[c2 + y * 2 + 0]) +
                   __vsadu4(__byte_perm(r[2], r[3], 0x6420), g_smem32[c2 + y * 2 + 1]);
        } else {
            const uint32_t e = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
            acc += __vsadu4(e, g_smem32[c4 + y]);
        }
    }
    return acc;
}

// ---- integer SAD of the 16x16 MB, mb_sad (encoder_motion.cpp:2197-2285) ----------------

template <int STRIDE, class S>
__device__ __forceinline__ uint32_t sad_int_loop(const S& s, uint32_t cur, int x0, int y0, int dx, int dy, int aw,
                                                 int ah) {
    uint32_t acc = 0;
#pragma unroll 1
    for (int y = 0; y < ah; y += STRIDE) {
#pragma unroll 1
        for (int x = 0; x < 16; x += STRIDE) {
            if (x < aw) acc += (uint32_t)iabs((int)g_smem[cur + y * 16 + x] - s(x0 + x + dx, y0 + y + dy));
        }
    }
    return acc;
}

// The picture geometry the scorers read (raster, rounding, cropped-padding flags), by value:
// passing the kernel's parameter block by address would make every parameter read of the
// kernel a generic load.
struct ScoreGeo {
    int W, H, vw, vh, cvw, cvh, rnd, pads;  // pads: right, bottom, chroma right, chroma bottom
};

__device__ __forceinline__ ScoreGeo score_geo(const DevParams& P) {
    return ScoreGeo{P.W, P.H, P.vw, P.vh, P.cvw, P.cvh, P.rnd,
                    (P.right_pad ? 1 : 0) | (P.bottom_pad ? 2 : 0) | (P.cright_pad ? 4 : 0) | (P.cbottom_pad ? 8 : 0)};
}

// A parameter block holding just the scorer's fields (the rest stay zero).
__device__ __forceinline__ DevParams geo_params(const ScoreGeo& g) {
    DevParams P{};
    P.W = g.W;
    P.H = g.H;
    P.vw = g.vw;
    P.vh = g.vh;
    P.cvw = g.cvw;
    P.cvh = g.cvh;
    P.rnd = g.rnd;
    P.right_pad = g.pads & 1;
    P.bottom_pad = (g.pads >> 1) & 1;
    P.cright_pad = (g.pads >> 2) & 1;
    P.cbottom_pad = (g.pads >> 3) & 1;
    return P;
}

// The per-macroblock values the out-of-line search routines read. It lives in the warp's
// shared memory (written once per macroblock, after its window is staged), and the routines
// take only its offset, so no structure travels through the stack on a call.
struct MbCtx {
    ScoreGeo g;
    uint32_t win_off, cur_off, cur2_off, cur4_off;
    int wp, wx0, wy0, wh, x0, y0, aw, ah;
    const uint8_t* gref;
    int gpitch;
    int subpel, fast_subpel, subpel_range, me_quality, mvrange, mant_bits, lam_s;
    uint64_t lam_m;
    uint32_t batch, cost, satd;  // the warp's shortlist buffers
    const uint8_t* sp;           // the pass's sub-pel prediction planes (nullptr: none)
    int sp_pitch, sp_border;
    long long sp_stride;
};
constexpr int kMbCtxBytes = 192;
static_assert(sizeof(MbCtx) <= kMbCtxBytes, "MbCtx layout");

__device__ __forceinline__ const MbCtx& mbctx(uint32_t off) { return *reinterpret_cast<const MbCtx*>(g_smem + off); }

// mb_sad at integer offset (dx, dy) and sampling stride 1/2/4 (encoder_motion.cpp:2197-2285);
// one out-of-line copy serves every search stage.
__device__ __noinline__ uint64_t mb_sad_core(uint32_t ctx, int dx, int dy, int stride) {
    const MbCtx& c = mbctx(ctx);
    const DevParams P = geo_params(c.g);
    if (hidden_padding(P, c.x0, c.y0, 16, 16, dx * 4, dy * 4, VC1CU_MV_QPEL, true)) return kBad;
    uint32_t s;
    const int xa = c.x0 + dx, ya = c.y0 + dy;
    const bool fast = xa >= c.wx0 && ya >= c.wy0 && xa + 15 < c.wx0 + c.wp && ya + 15 < c.wy0 + c.wh;
    if (fast && c.aw == 16 && c.ah == 16) {
        const uint32_t base = c.win_off + (uint32_t)((ya - c.wy0) * c.wp + (xa - c.wx0));
        if (stride == 1) s = sad_packed<1>(c.cur_off, c.cur2_off, c.cur4_off, c.wp, base);
        else if (stride == 2) s = sad_packed<2>(c.cur_off, c.cur2_off, c.cur4_off, c.wp, base);
        else s = sad_packed<4>(c.cur_off, c.cur2_off, c.cur4_off, c.wp, base);
    } else if (fast) {
        const WinSampler ws{c.win_off, c.wp, c.wx0, c.wy0, c.wh};
        if (stride == 1) s = sad_int_loop<1>(ws, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
        else if (stride == 2) s = sad_int_loop<2>(ws, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
        else s = sad_int_loop<4>(ws, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
    } else if (c.aw == 16 && c.ah == 16 && xa >= 0 && ya >= 0 && xa + 16 <= P.W && ya + 16 <= P.H) {
        // outside the staged window but inside the frame: no clamping, packed rows from L2
        const uint8_t* base = c.gref + (size_t)ya * c.gpitch + xa;
        if (stride == 1) s = sad_packed_glob<1>(c.cur_off, c.cur2_off, c.cur4_off, base, c.gpitch);
        else if (stride == 2) s = sad_packed_glob<2>(c.cur_off, c.cur2_off, c.cur4_off, base, c.gpitch);
        else s = sad_packed_glob<4>(c.cur_off, c.cur2_off, c.cur4_off, base, c.gpitch);
    } else {
        const GlobSampler gs{c.gref, c.gpitch, P.W, P.H};
        if (stride == 1) s = sad_int_loop<1>(gs, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
        else if (stride == 2) s = sad_int_loop<2>(gs, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
        else s = sad_int_loop<4>(gs, c.cur_off, c.x0, c.y0, dx, dy, c.aw, c.ah);
    }
    return stride > 1 ? (uint64_t)s * (uint64_t)(stride * stride) : (uint64_t)s;
}

__device__ __forceinline__ uint64_t mb_sad(const DevParams&, const Mb& m, int dx, int dy, int stride) {
    return mb_sad_core(m.sm.ctx.off, dx, dy, stride);
}

// ---- sub-pel SAD / SATD batches (block_sad_motion :2670-2933, block_satd_motion :2960-3042)

__device__ __forceinline__ uint32_t soff(const void* p) {
    return (uint32_t)(reinterpret_cast<const uint8_t*>(p) - g_smem);
}

__device__ __forceinline__ bool ctx_inside(const MbCtx& c, int xa, int ya, int xb, int yb) {
    return xa >= c.wx0 && ya >= c.wy0 && xb < c.wx0 + c.wp && yb < c.wy0 + c.wh;
}

// The sub-pel plane row of phase (hm, vm) at integer origin (sx, sy), when its n samples lie in
// the planes (nullptr otherwise).
__device__ __forceinline__ const uint8_t* sp_row(const MbCtx& c, int hm, int vm, int sx, int sy, int n) {
    if (!c.sp || !(hm | vm)) return nullptr;
    const int b = c.sp_border;
    if (sx < -b || sx + n > c.g.W + b || sy < -b || sy >= c.g.H + b) return nullptr;
    return c.sp + (long long)(vm * 4 + hm) * c.sp_stride + (long long)(sy + b) * c.sp_pitch + (sx + b);
}

// n <= 8 bytes of a plane row as two little-endian words (aligned loads and funnel shifts; the
// row continues at least 3 bytes past any origin sp_row accepts)
__device__ __forceinline__ void sp_load8(const uint8_t* p, uint32_t& lo, uint32_t& hi) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(3));
    const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 3) * 8;
    const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = sh ? __ldg(w + 2) : 0u;
    lo = __funnelshift_r(w0, w1, sh);
    hi = __funnelshift_r(w1, w2, sh);
}

// SAD of n candidates of block (bx,by,bw,bh) (bw,bh in {8,16}) under the CPU law, written
// to out[]. Each candidate's block is split into 8-pixel row segments over bh*bw/8 lanes.
// One out-of-line copy serves every call site. Sub-pel rows come from the pass's prediction
// planes where they cover them, else are interpolated from the window or the frame.
__device__ __noinline__ void sad_batch_core(uint32_t ctx, uint32_t mvs_off, int n, int bx, int by,
                                            int bw, int bh, int mode, uint32_t out_off) {
    const MbCtx& c = mbctx(ctx);
    const int lane = threadIdx.x & 31;
    const DevParams P = geo_params(c.g);
    const int2* mvs = reinterpret_cast<const int2*>(g_smem + mvs_off);
    uint64_t* out = reinterpret_cast<uint64_t*>(g_smem + out_off);
    const int spr = bw >> 3;
    const int segs = bh * spr;  // 32 (16x16) or 8 (8x8)
    const int per_iter = 32 / segs;
    const int aw = imax(0, imin(bw, P.W - bx)), ah = imax(0, imin(bh, P.H - by));
    const bool bil = mode_bilinear(mode);
    const bool cg = chroma_gate(bx, by, bw, bh);
    const int cx = bx - c.x0, cy = by - c.y0;
    for (int base = 0; base < n; base += per_iter) {
        const int ci = base + lane / segs;
        const int sidx = lane % segs;
        const int r = sidx / spr, c0 = (sidx % spr) * 8;
        const bool valid = ci < n;
        const int2 mv = valid ? mvs[ci] : make_int2(0, 0);
        bool bad = false;
        uint32_t part = 0;
        if (valid) {
            bad = hidden_padding(P, bx, by, bw, bh, mv.x, mv.y, mode, cg) || (bil && ((mv.x & 1) || (mv.y & 1)));
            if (!bad && r < ah && c0 < aw) {
                const int ix = floor_div4(mv.x), iy = floor_div4(mv.y);
                const uint32_t cp = c.cur_off + (uint32_t)((cy + r) * 16 + cx + c0);
                const int nvis = imin(8, aw - c0);
                const uint8_t* pr = nvis == 8 ? sp_row(c, mv.x - 4 * ix, mv.y - 4 * iy, bx + c0 + ix, by + r + iy, 8) : nullptr;
                if (pr) {
                    uint32_t lo, hi;
                    sp_load8(pr, lo, hi);
                    part = __vsadu4(lo, g_smem32[cp >> 2]) + __vsadu4(hi, g_smem32[(cp >> 2) + 1]);
                } else if (ctx_inside(c, bx + ix - 1, by + iy - 1, bx + ix + bw + 1, by + iy + bh + 1)) {
                    part = sad_row8(WinSampler{c.win_off, c.wp, c.wx0, c.wy0, c.wh}, bil, P.rnd, mv.x, mv.y, bx + c0, by + r, cp, nvis);
                } else {
                    const PredRow<8> g8 = predict_row_glob<8>(c.gref, c.gpitch, P.W, P.H, bil, P.rnd, mv.x, mv.y, bx + c0, by + r);
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (i < nvis) part += (uint32_t)iabs((int)g_smem[cp + i] - g8.v[i]);
                }
            }
        }
        for (int o = segs >> 1; o; o >>= 1) part += __shfl_xor_sync(FULL, part, o);
        if (valid && sidx == 0) out[ci] = bad ? kBad : (uint64_t)part;
    }
    __syncwarp();
}

__device__ __noinline__ void satd_batch_core(uint32_t ctx, uint32_t mvs_off, int n, int bx, int by,
                                             int bw, int bh, int mode, uint32_t out_off) {
    const MbCtx& c = mbctx(ctx);
    const int lane = threadIdx.x & 31;
    const DevParams P = geo_params(c.g);
    const int2* mvs = reinterpret_cast<const int2*>(g_smem + mvs_off);
    uint64_t* out = reinterpret_cast<uint64_t*>(g_smem + out_off);
    const int tpr = bw >> 2;
    const int tiles = tpr * (bh >> 2);  // 16 or 4
    const int per_iter = 32 / tiles;
    const int aw = imax(0, imin(bw, P.W - bx)), ah = imax(0, imin(bh, P.H - by));
    const bool bil = mode_bilinear(mode);
    const int cx = bx - c.x0, cy = by - c.y0;
    for (int base = 0; base < n; base += per_iter) {
        const int ci = base + lane / tiles;
        const int t = lane % tiles;
        const int tx = (t % tpr) * 4, ty = (t / tpr) * 4;
        const bool valid = ci < n;
        const int2 mv = valid ? mvs[ci] : make_int2(0, 0);
        const bool bad = valid && mode_halfpel(mode) && ((mv.x & 1) || (mv.y & 1));
        uint32_t part = 0;
        const int tw = imax(0, imin(4, aw - tx)), th = imax(0, imin(4, ah - ty));
        if (valid && !bad && tw && th) {
            const int ix = floor_div4(mv.x), iy = floor_div4(mv.y);
            const bool fast = ctx_inside(c, bx + ix - 1, by + iy - 1, bx + ix + bw + 1, by + iy + bh + 1);
            // rows one at a time (one copy of the interpolation code), row-transformed and
            // rotated through four registers for the column stage
            int4 r0 = make_int4(0, 0, 0, 0), r1 = r0, r2 = r0, r3 = r0;
            const uint8_t* pr = sp_row(c, mv.x - 4 * ix, mv.y - 4 * iy, bx + tx + ix, by + ty + iy, 4);
            if (pr && !sp_row(c, mv.x - 4 * ix, mv.y - 4 * iy, bx + tx + ix, by + ty + iy + 3, 4)) pr = nullptr;
#pragma unroll 1
            for (int yy = 0; yy < 4; ++yy) {
                int pred[4];
                if (pr) {
                    uint32_t lo, hi;
                    sp_load8(pr + (long long)yy * c.sp_pitch, lo, hi);
                    pred[0] = lo & 255;
                    pred[1] = (lo >> 8) & 255;
                    pred[2] = (lo >> 16) & 255;
                    pred[3] = lo >> 24;
                } else if (fast) {
                    const int4 w4 = pred_row4(WinSampler{c.win_off, c.wp, c.wx0, c.wy0, c.wh}, bil, P.rnd, mv.x, mv.y, bx + tx, by + ty + yy);
                    pred[0] = w4.x;
                    pred[1] = w4.y;
                    pred[2] = w4.z;
                    pred[3] = w4.w;
                } else {
                    const PredRow<4> g4 = predict_row_glob<4>(c.gref, c.gpitch, P.W, P.H, bil, P.rnd, mv.x, mv.y, bx + tx,
                                                              by + ty + yy);
#pragma unroll
                    for (int i = 0; i < 4; ++i) pred[i] = g4.v[i];
                }
                int d[4];
                const uint32_t crow = c.cur_off + (uint32_t)((cy + ty + yy) * 16 + cx + tx);
#pragma unroll
                for (int xx = 0; xx < 4; ++xx) d[xx] = (xx < tw && yy < th) ? (int)g_smem[crow + xx] - pred[xx] : 0;
                r0 = r1;
                r1 = r2;
                r2 = r3;
                r3 = hadamard_row(d[0], d[1], d[2], d[3]);
            }
            part = hadamard_cols(r0, r1, r2, r3);
        }
        for (int o = tiles >> 1; o; o >>= 1) part += __shfl_xor_sync(FULL, part, o);
        if (valid && t == 0) out[ci] = (!aw || !ah) ? 0 : (bad ? kBad : (uint64_t)part);
    }
    __syncwarp();
}

// mvs and out point into the warp's shared-memory buffers.
__device__ __forceinline__ void sad_batch(const DevParams& P, const Mb& m, const int2* mvs, int n, int bx, int by, int bw,
                                          int bh, int mode, uint64_t* out) {
    sad_batch_core(m.sm.ctx.off, soff(mvs), n, bx, by, bw, bh, mode, soff(out));
}

__device__ __forceinline__ void satd_batch(const DevParams& P, const Mb& m, const int2* mvs, int n, int bx, int by, int bw,
                                           int bh, int mode, uint64_t* out) {
    satd_batch_core(m.sm.ctx.off, soff(mvs), n, bx, by, bw, bh, mode, soff(out));
}

// ---- first-visit bitsets ----------------------------------------------------------------

__device__ __forceinline__ bool seen_test_set(uint32_t* bits, int r, int dx, int dy) {
    const int side = 2 * r + 1;
    if (!IDX_OK(dx >= -r && dx <= r && dy >= -r && dy <= r, kSiteSeen, (long long)dy * 65536 + dx)) return true;
    const int bit = (dy + r) * side + (dx + r);
    const uint32_t mask = 1u << (bit & 31);
    return (atomicOr(&bits[bit >> 5], mask) & mask) != 0;
}

// ---- integer UMH (encoder_motion.cpp:1781-2023) -----------------------------------------

// Merges the n keys of m.sm.keys (UINT64_MAX = skipped) into the sorted top-8 list
// m.sm.top / m.sm.misc[0]. Keys below the current 8th entry are compacted with a ballot
// first; the few survivors are ranked and merged on every lane identically.
__device__ __noinline__ void top8_merge_core(int lane, uint32_t keys_off, uint32_t top_off, uint32_t misc_off,
                                             uint32_t out8_off, int n) {
    uint64_t* keys = reinterpret_cast<uint64_t*>(g_smem + keys_off);
    uint64_t* top = reinterpret_cast<uint64_t*>(g_smem + top_off);
    int* misc = reinterpret_cast<int*>(g_smem + misc_off);
    const int tn = misc[0];
    const uint64_t bound = tn == 8 ? top[7] : UINT64_MAX;
    int cnt = 0;
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const uint64_t k = i < n ? keys[i] : UINT64_MAX;
        const bool take = k < bound;
        const unsigned b = __ballot_sync(FULL, take);
        if (take) keys[cnt + __popc(b & ((1u << lane) - 1))] = k;
        cnt += __popc(b);
        __syncwarp();
    }
    if (!cnt) return;
    const uint64_t* sel;
    int ns = 0;
    if (cnt <= 32) {
        // rank of each survivor (keys are distinct), the 8 lowest ranks in order
        const uint64_t k = lane < cnt ? keys[lane] : UINT64_MAX;
        int rank = 0;
        for (int j = 0; j < cnt; ++j) rank += keys[j] < k;
        __syncwarp();
        if (lane < cnt && rank < 8) keys[rank] = k;
        __syncwarp();
        ns = cnt < 8 ? cnt : 8;
        sel = keys;
    } else {
        uint64_t* out8 = reinterpret_cast<uint64_t*>(g_smem + out8_off);  // idle during the integer search
        for (int r = 0; r < 8; ++r) {
            uint64_t lm = UINT64_MAX;
            for (int i = lane; i < cnt; i += 32) lm = keys[i] < lm ? keys[i] : lm;
            const uint64_t g = warp_min_u64(lm);
            if (lane == 0) out8[r] = g;
            for (int i = lane; i < cnt; i += 32)
                if (keys[i] == g) keys[i] = UINT64_MAX;
            __syncwarp();
        }
        ns = 8;
        sel = out8;
    }
    uint64_t out[8];
    int a = 0, b = 0, o = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (a < tn || b < ns) {
            const uint64_t ta = a < tn ? top[a] : UINT64_MAX, tb = b < ns ? sel[b] : UINT64_MAX;
            if (ta < tb) { out[q] = ta; ++a; } else { out[q] = tb; ++b; }
            ++o;
        }
    }
    __syncwarp();
    if (lane < o) {
        uint64_t v = out[0];
#pragma unroll
        for (int q = 1; q < 8; ++q) if (lane == q) v = out[q];
        top[lane] = v;
    }
    if (lane == 0) misc[0] = o;
    __syncwarp();
}

__device__ __forceinline__ void top8_merge(const Mb& m, int n) {
    top8_merge_core(m.lane, m.sm.keys.off, m.sm.top.off, m.sm.misc.off, m.sm.list_sad.off, n);
}

// Scores the candidates produced by gen(i) for i < n at sampled stride 2 (the UMH
// `consider` lambda, encoder_motion.cpp:1821-1839) and merges them into top.
template <class Gen>
__device__ void umh_stage(const DevParams& P, const Mb& m, int n, int range, Gen gen) {
    for (int i = m.lane; i < n; i += 32) {
        int2 c = gen(i);
        c.x = iclamp(c.x, -range, range);
        c.y = iclamp(c.y, -range, range);
        uint64_t key = UINT64_MAX;
        if (!seen_test_set(m.sm.seen, range, c.x, c.y)) key = int_key(mb_sad(P, m, c.x, c.y, 2), c.x, c.y);
        if (IDX_OK(i < m.keys_cap, kSiteKeys, i)) m.sm.keys[i] = key;
    }
    __syncwarp();
    top8_merge(m, n);
}

// Minimum key over full-resolution candidates (no top list), optional first-visit filter.
template <class Gen>
__device__ uint64_t full_stage(const DevParams& P, const Mb& m, int n, int range, int stride, bool use_seen, Gen gen) {
    uint64_t best = UINT64_MAX;
    for (int i = m.lane; i < n; i += 32) {
        bool ok;
        int2 c = gen(i, ok);
        if (!ok) continue;
        if (use_seen && seen_test_set(m.sm.seen_full, range, c.x, c.y)) continue;
        const uint64_t k = int_key(mb_sad(P, m, c.x, c.y, stride), c.x, c.y);
        best = k < best ? k : best;
    }
    return warp_min_u64(best);
}

__device__ __forceinline__ bool match_good(const DevParams& P, uint64_t sad, uint64_t pixels) {
    if (!pixels || sad >= UINT64_MAX / 8) return false;
    return sad <= pixels * 6u;
}

struct IntRes {
    int dx, dy;
    uint64_t cost;
};

__device__ IntRes umh(const DevParams& P, const Mb& m, const PInfo& pi, int gdx, int gdy, int range, uint64_t pixels) {
    // clear bitsets
    const int words = ((2 * range + 1) * (2 * range + 1) + 31) >> 5;
    for (int i = m.lane; i < words; i += 32) {
        m.sm.seen[i] = 0;
        m.sm.seen_full[i] = 0;
    }
    if (m.lane == 0) m.sm.misc[0] = 0;
    __syncwarp();
    const uint64_t* top = m.sm.top;
    // predictor seeds (:1843-1850)
    {
        // predictor, zero, global, then A and C where they exist
        const int2 sp = make_int2(iclamp(round_qpel_to_pixel(pi.pre.x), -range, range),
                                  iclamp(round_qpel_to_pixel(pi.pre.y), -range, range));
        const int2 sa = make_int2(round_qpel_to_pixel(pi.a.x), round_qpel_to_pixel(pi.a.y));
        const int2 sc = make_int2(round_qpel_to_pixel(pi.c.x), round_qpel_to_pixel(pi.c.y));
        const int ns = 3 + (pi.a_valid ? 1 : 0) + (pi.c_valid ? 1 : 0);
        umh_stage(P, m, ns, range, [&](int i) {
            return i == 0 ? sp : i == 1 ? make_int2(0, 0) : i == 2 ? make_int2(gdx, gdy) : (i == 3 && pi.a_valid) ? sa : sc;
        });
    }
    // 5x5 around best (:1855-1859)
    {
        const int cx = key_dx(top[0]), cy = key_dy(top[0]);
        umh_stage(P, m, 25, range, [&](int i) { return make_int2(cx + i % 5 - 2, cy + i / 5 - 2); });
    }
    // sparse lattice over the whole window (:1865-1870)
    if (range >= 8) {
        const int L = (2 * range) / 8 + 1;
        umh_stage(P, m, L * L + 2 * L, range, [&](int i) {
            if (i < L * L) return make_int2(-range + (i % L) * 8, -range + (i / L) * 8);
            const int j = i - L * L;
            const int d = -range + (j >> 1) * 8;
            return (j & 1) ? make_int2(d, range) : make_int2(range, d);
        });
    }
    // uneven cross (:1875-1884)
    {
        const int cs = range >= 96 ? 8 : (range >= 32 ? 4 : 2);
        const int cx = key_dx(top[0]), cy = key_dy(top[0]);
        const int vlimit = imin(range, imax(8, range / 2));
        const int nh = range / cs, nv = vlimit / cs;
        umh_stage(P, m, 2 * nh + 2 * nv, range, [&](int i) {
            if (i < 2 * nh) {
                const int d = cs * (i / 2 + 1);
                return (i & 1) ? make_int2(cx + d, cy) : make_int2(cx - d, cy);
            }
            const int j = i - 2 * nh;
            const int d = cs * (j / 2 + 1);
            return (j & 1) ? make_int2(cx, cy + d) : make_int2(cx, cy - d);
        });
    }
    // multi-hexagon rings (:1889-1897)
    {
        const int hs = range >= 96 ? 8 : (range >= 24 ? 4 : 2);
        const int hx = key_dx(top[0]), hy = key_dy(top[0]);
        const int nr = range / hs;
        umh_stage(P, m, 6 * nr, range, [&](int i) {
            const int r = hs * (i / 6 + 1), h = (r + 1) / 2;
            switch (i % 6) {
                case 0: return make_int2(hx - r, hy);
                case 1: return make_int2(hx + r, hy);
                case 2: return make_int2(hx - h, hy - r);
                case 3: return make_int2(hx + h, hy - r);
                case 4: return make_int2(hx - h, hy + r);
                default: return make_int2(hx + h, hy + r);
            }
        });
    }
    // iterative small hexagon (:1902-1908)
    for (int iter = 0; iter < 32; ++iter) {
        const uint64_t before = top[0];
        const int ox = key_dx(before), oy = key_dy(before);
        umh_stage(P, m, 6, range, [&](int i) {
            // (-2,0) (2,0) (-1,-2) (1,-2) (-1,2) (1,2)
            return i < 2 ? make_int2(ox + (i ? 2 : -2), oy) : make_int2(ox + ((i & 1) ? 1 : -1), oy + (i < 4 ? -2 : 2));
        });
        if (key_dx(top[0]) == ox && key_dy(top[0]) == oy) break;
    }
    // closing diamond (:1909-1913)
    {
        const int ox = key_dx(top[0]), oy = key_dy(top[0]);
        umh_stage(P, m, 4, range, [&](int i) {
            // (-1,0) (1,0) (0,-1) (0,1)
            return i < 2 ? make_int2(ox + (i ? 1 : -1), oy) : make_int2(ox, oy + (i == 3 ? 1 : -1));
        });
    }
    // full-resolution finalists (:1929-1952)
    const int nf = imin(4, m.sm.misc[0]);
    uint64_t fk = full_stage(P, m, nf * 9, range, 1, true, [&](int i, bool& ok) {
        ok = true;
        const uint64_t t = top[i / 9];
        return make_int2(iclamp(key_dx(t) + (i % 9) % 3 - 1, -range, range),
                         iclamp(key_dy(t) + (i % 9) / 3 - 1, -range, range));
    });
    IntRes full{key_dx(fk), key_dy(fk), key_cost(fk)};
    if (fk == UINT64_MAX) {  // unreachable in practice (:1948-1951)
        full.dx = key_dx(top[0]);
        full.dy = key_dy(top[0]);
        full.cost = mb_sad(P, m, full.dx, full.dy, 1);
        fk = int_key(full.cost, full.dx, full.dy);
    }
    // bounded rescue on a poor match (:1958-2020)
    if (range > 0 && !match_good(P, full.cost, pixels)) {
        const int step = range >= 8 ? 4 : (range >= 3 ? 2 : 1);
        const int L = (2 * range) / step + 1;
        const uint64_t ck = full_stage(P, m, L * L + 2 * L, range, 4, false, [&](int i, bool& ok) {
            ok = true;
            if (i < L * L) return make_int2(-range + (i % L) * step, -range + (i / L) * step);
            const int j = i - L * L;
            const int d = -range + (j >> 1) * step;
            return (j & 1) ? make_int2(d, range) : make_int2(range, d);
        });
        const int cdx = key_dx(ck), cdy = key_dy(ck);
        const int rr = imax(1, step - 1);
        const int ylo = imax(-range, cdy - rr), yhi = imin(range, cdy + rr);
        const int xlo = imax(-range, cdx - rr), xhi = imin(range, cdx + rr);
        const int nx = xhi - xlo + 1, ny = yhi - ylo + 1;
        const uint64_t rk = full_stage(P, m, nx * ny, range, 1, true, [&](int i, bool& ok) {
            ok = true;
            return make_int2(xlo + i % nx, ylo + i / nx);
        });
        if (rk < fk) fk = rk;
        full = IntRes{key_dx(fk), key_dy(fk), key_cost(fk)};
        if (pixels && full.cost > pixels * 24u && range <= 32) {
            const int Ld = range + 1;  // -range..range step 2
            const uint64_t dk = full_stage(P, m, Ld * Ld, range, 2, false, [&](int i, bool& ok) {
                ok = true;
                return make_int2(-range + (i % Ld) * 2, -range + (i / Ld) * 2);
            });
            const int ddx = key_dx(dk), ddy = key_dy(dk);
            const int y0 = imax(-range, ddy - 2), y1 = imin(range, ddy + 2);
            const int x0 = imax(-range, ddx - 2), x1 = imin(range, ddx + 2);
            const int mx = x1 - x0 + 1, my = y1 - y0 + 1;
            const uint64_t dfk = full_stage(P, m, mx * my, range, 1, true, [&](int i, bool& ok) {
                ok = true;
                return make_int2(x0 + i % mx, y0 + i / mx);
            });
            if (dfk < fk) fk = dfk;
            full = IntRes{key_dx(fk), key_dy(fk), key_cost(fk)};
        }
    }
    return full;
}

// integer_motion_diamond, encoder_motion_diamond.cpp:13-73
__device__ IntRes diamond(const DevParams& P, const Mb& m, const PInfo& pi, int gdx, int gdy, int range) {
    uint64_t best = int_key(mb_sad(P, m, 0, 0, 1), 0, 0);
    if (key_cost(best) == 0) return IntRes{0, 0, 0};
    // predictor, global, then A and C where they exist
    const int ns = 2 + (pi.a_valid ? 1 : 0) + (pi.c_valid ? 1 : 0);
    {
        uint64_t k = UINT64_MAX;
        if (m.lane < ns) {
            const int l = m.lane;
            const int2 v = l == 0 ? make_int2(round_qpel_to_pixel(pi.pre.x), round_qpel_to_pixel(pi.pre.y))
                         : l == 1 ? make_int2(gdx, gdy)
                         : (l == 2 && pi.a_valid) ? make_int2(round_qpel_to_pixel(pi.a.x), round_qpel_to_pixel(pi.a.y))
                                                  : make_int2(round_qpel_to_pixel(pi.c.x), round_qpel_to_pixel(pi.c.y));
            const int dx = iclamp(v.x, -range, range), dy = iclamp(v.y, -range, range);
            k = int_key(mb_sad(P, m, dx, dy, 1), dx, dy);
        }
        k = warp_min_u64(k);
        best = k < best ? k : best;
    }
    int px = key_dx(best), py = key_dy(best);
    bool have_prev = false;
    for (int step = 0; step <= 4 * range + 1; ++step) {
        const uint64_t center = best;
        const int cx = key_dx(center), cy = key_dy(center);
        uint64_t k = UINT64_MAX;
        if (m.lane < 4) {
            const int l = m.lane;  // (-1,0) (1,0) (0,-1) (0,1)
            const int dx = cx + (l < 2 ? (l ? 1 : -1) : 0), dy = cy + (l < 2 ? 0 : (l == 3 ? 1 : -1));
            if (!(dx < -range || dx > range || dy < -range || dy > range) && !(have_prev && dx == px && dy == py))
                k = int_key(mb_sad(P, m, dx, dy, 1), dx, dy);
        }
        k = warp_min_u64(k);
        const uint64_t winner = k < center ? k : center;
        if (winner == center) break;
        px = cx;
        py = cy;
        have_prev = true;
        best = winner;
        if (key_cost(best) == 0) break;
    }
    return IntRes{key_dx(best), key_dy(best), key_cost(best)};
}

// ---- staged sub-pel refinement (encoder_motion.cpp:3247-3594) ---------------------------

// ---- long-range search (encoder_motion.cpp:1578-1779) -------------------------------------

// motion_match_good, encoder_motion.cpp:1627-1635
__device__ __forceinline__ bool match_good(const Mb& m, uint64_t sad) {
    const uint64_t px = (uint64_t)m.aw * (uint64_t)m.ah;
    return px && sad < UINT64_MAX / 8 && sad <= px * 6u;
}

// sad > px * mae, exactly: the reference compares in long double, where the product of a
// pixel count and a double is exact. mae = mant * 2^k with a 53-bit integer mant.
__device__ bool sad_above(uint64_t sad, uint64_t px, double mae) {
    if (isnan(mae)) return false;
    if (mae < 0.0) return true;
    if (isinf(mae)) return false;
    if (mae == 0.0) return sad > 0;
    int e = 0;
    const double fr = frexp(mae, &e);                 // mae = fr * 2^e, fr in [0.5, 1)
    const uint64_t mant = (uint64_t)ldexp(fr, 53);    // exact
    const int k = e - 53;
    const unsigned __int128 rhs0 = (unsigned __int128)px * mant;  // < 2^62
    if (k >= 0) {
        if (k > 64) return false;
        return (unsigned __int128)sad > (rhs0 << k);
    }
    if (-k > 64) return sad > 0;
    return ((unsigned __int128)sad << (-k)) > rhs0;
}

// distant_match_decision, encoder_motion.cpp:1637-1656
__device__ int distant_decision(const DevParams& P, const Mb& m, uint64_t cand, uint64_t local) {
    const uint64_t px = (uint64_t)m.aw * (uint64_t)m.ah;
    if (!px || cand >= UINT64_MAX / 8) return 0;
    if (cand <= px * 6u) return 2;
    if (sad_above(cand, px, P.distant_match_max_mae)) return 1;
    if (local >= UINT64_MAX / 8) return 3;
    return cand * 4u <= local * 3u ? 3 : 1;
}

// Least (sad, |dx|+|dy|, lane) over the lanes with `valid`, on every lane.
__device__ void warp_argmin_int(bool& valid, uint64_t& sad, int& dx, int& dy, int& idx) {
#pragma unroll 1
    for (int o = 16; o; o >>= 1) {
        const bool ov = __shfl_xor_sync(FULL, valid, o);
        const uint64_t os = __shfl_xor_sync(FULL, sad, o);
        const int ox = __shfl_xor_sync(FULL, dx, o), oy = __shfl_xor_sync(FULL, dy, o);
        const int oi = __shfl_xor_sync(FULL, idx, o);
        bool take = ov && !valid;
        if (ov && valid) {
            const int l1 = iabs(ox) + iabs(oy), l0 = iabs(dx) + iabs(dy);
            take = os != sad ? os < sad : (l1 != l0 ? l1 < l0 : oi < idx);
        }
        if (take) {
            valid = true;
            sad = os;
            dx = ox;
            dy = oy;
            idx = oi;
        }
    }
}

// The 13 offsets of propagated_long_range_motion (:1671-1673), by lane.
__device__ __forceinline__ int2 lr_prop_offset(int l) {
    if (l == 0) return make_int2(0, 0);
    if (l <= 8) {
        const int a = (l - 1) & 3, d = l <= 4 ? 1 : 2;  // (-d,0) (d,0) (0,-d) (0,d)
        return a == 0 ? make_int2(-d, 0) : a == 1 ? make_int2(d, 0) : a == 2 ? make_int2(0, -d) : make_int2(0, d);
    }
    const int a = l - 9;  // (-1,-1) (1,-1) (-1,1) (1,1)
    return make_int2((a & 1) ? 1 : -1, (a & 2) ? 1 : -1);
}

// Vc1Encoder::propagated_long_range_motion, encoder_motion.cpp:1658-1694: around the integer
// vectors of the left, top, top-left and top-right neighbours whose search took a long-range
// vector (flags bit 2), in that order, stopping once the match is good.
__device__ IntRes lr_propagated(const DevParams& P, const Mb& m, const DevResult& o, int range) {
    IntRes best{0, 0, UINT64_MAX};
    const Bounds b = bounds_px(range);
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const int nx = m.mx + (k == 0 || k == 2 ? -1 : (k == 3 ? 1 : 0)), ny = m.my - (k == 0 ? 0 : 1);
        if (nx < 0 || ny < 0 || nx >= P.mbw) continue;
        const int pos = ny * P.mbw + nx;
        if (!(__ldcg(&o.flags[pos]) & 4)) continue;
        const int2 f = __ldcg(&o.mvs[pos]);
        const int cx = round_qpel_to_pixel(f.x), cy = round_qpel_to_pixel(f.y);
        bool valid = m.lane < 13;
        uint64_t sad = UINT64_MAX;
        int dx = 0, dy = 0, idx = m.lane;
        if (valid) {
            const int2 of = lr_prop_offset(m.lane);
            dx = iclamp(cx + of.x, b.xmin, b.xmax);
            dy = iclamp(cy + of.y, b.ymin, b.ymax);
            sad = mb_sad(P, m, dx, dy, 1);
        }
        warp_argmin_int(valid, sad, dx, dy, idx);
        if (sad < best.cost || (sad == best.cost && iabs(dx) + iabs(dy) < iabs(best.dx) + iabs(best.dy))) {
            best.cost = sad;
            best.dx = dx;
            best.dy = dy;
        }
        if (match_good(m, best.cost)) break;
    }
    return best;
}

// mean_region (:1578-1590) of an 8x8 region of a plane, by the warp (two samples per lane).
__device__ uint32_t warp_mean8(const uint8_t* plane, int pitch, int pw, int ph, int x0, int y0, int lane) {
    uint32_t sum = 0, n = 0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int i = lane * 2 + j, x = x0 + (i & 7), y = y0 + (i >> 3);
        if (x >= 0 && y >= 0 && x < pw && y < ph) {
            sum += __ldg(plane + (size_t)y * pitch + x);
            ++n;
        }
    }
    for (int o = 16; o; o >>= 1) {
        sum += __shfl_xor_sync(FULL, sum, o);
        n += __shfl_xor_sync(FULL, n, o);
    }
    return n ? (sum + n / 2) / n : 128;
}

// long_range_signature (:1592-1603) packed as bytes ydc0..3, udc, vdc.
__device__ uint64_t warp_signature(const DevFrame& f, int W, int H, int x0, int y0, int lane) {
    uint64_t s = 0;
    s |= (uint64_t)warp_mean8(f.y, f.pitch_y, W, H, x0, y0, lane);
    s |= (uint64_t)warp_mean8(f.y, f.pitch_y, W, H, x0 + 8, y0, lane) << 8;
    s |= (uint64_t)warp_mean8(f.y, f.pitch_y, W, H, x0, y0 + 8, lane) << 16;
    s |= (uint64_t)warp_mean8(f.y, f.pitch_y, W, H, x0 + 8, y0 + 8, lane) << 24;
    s |= (uint64_t)warp_mean8(f.u, f.pitch_c, W / 2, H / 2, x0 / 2, y0 / 2, lane) << 32;
    s |= (uint64_t)warp_mean8(f.v, f.pitch_c, W / 2, H / 2, x0 / 2, y0 / 2, lane) << 40;
    return s;
}

// long_range_signature_distance (:1605-1614)
__device__ __forceinline__ uint32_t sig_distance(uint64_t a, uint64_t b) {
    uint32_t d = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) d += (uint32_t)iabs((int)((a >> (8 * i)) & 255) - (int)((b >> (8 * i)) & 255)) * 2u;
    d += (uint32_t)iabs((int)((a >> 32) & 255) - (int)((b >> 32) & 255)) * 3u;
    d += (uint32_t)iabs((int)((a >> 40) & 255) - (int)((b >> 40) & 255)) * 3u;
    return d;
}

// Vc1Encoder::extended_content_motion, encoder_motion.cpp:1696-1779: the 16 lattice cells
// whose signature is nearest the macroblock's (order (distance, |d|, dy, dx), cells within
// 32 pixels excluded), each refined by a 5x5 grid of step 4 at stride 2 and a 5x5 full
// search; `local` stands unless the best is both cheaper and a good enough distant match.
__device__ IntRes lr_extended(const DevParams& P, const Mb& m, const PassDesc& d, int range, const IntRes& local,
                              uint64_t& cand_sad, int& decision) {
    const Bounds b = bounds_px(range);
    const uint64_t want = warp_signature(d.cur, P.W, P.H, m.x0, m.y0, m.lane);
    uint64_t* top = m.sm.list_sad;  // 16 sorted keys (idle after the integer search)
    uint64_t* stage = m.sm.keys;
    int tn = 0;
    const int n = d.lr_nx * d.lr_ny;
#pragma unroll 1
    for (int base = 0; base < n; base += 32) {
        const int i = base + m.lane;
        uint64_t key = UINT64_MAX;
        if (i < n) {
            const int dx = (i % d.lr_nx) * 8 - m.x0, dy = (i / d.lr_nx) * 8 - m.y0;
            if (dx >= b.xmin && dx <= b.xmax && dy >= b.ymin && dy <= b.ymax && !(iabs(dx) <= 32 && iabs(dy) <= 32) &&
                IDX_OK(d.lr_sig != nullptr, kSiteSignature, i)) {
                const uint64_t dist = sig_distance(want, __ldg(&d.lr_sig[i]));
                key = (dist << 36) | ((uint64_t)(iabs(dx) + iabs(dy)) << 24) | ((uint64_t)(dy + 2048) << 12) |
                      (uint64_t)(dx + 2048);
            }
        }
        const uint64_t bound = tn == 16 ? top[15] : UINT64_MAX;
        const bool take = key < bound;
        const unsigned tm = __ballot_sync(FULL, take);
        if (!tm) continue;
        if (take) stage[__popc(tm & ((1u << m.lane) - 1))] = key;
        __syncwarp();
        if (m.lane == 0) {
            const int cnt = __popc(tm);
            for (int j = 0; j < cnt; ++j) {
                const uint64_t k = stage[j];
                if (tn == 16 && k >= top[15]) continue;
                int at = tn < 16 ? tn : 15;
                while (at > 0 && top[at - 1] > k) {
                    top[at] = top[at - 1];
                    --at;
                }
                top[at] = k;
                if (tn < 16) ++tn;
            }
        }
        tn = __shfl_sync(FULL, tn, 0);
        __syncwarp();
    }
    IntRes best{0, 0, UINT64_MAX};
#pragma unroll 1
    for (int t = 0; t < tn; ++t) {
        const uint64_t key = top[t];
        const int cdx = (int)(key & 0xFFF) - 2048, cdy = (int)((key >> 12) & 0xFFF) - 2048;
        // 5x5 at step 4, stride 2: the first least SAD in scan order
        bool valid = m.lane < 25;
        uint64_t sad = UINT64_MAX;
        int dx = 0, dy = 0, idx = m.lane;
        if (valid) {
            dx = iclamp(cdx - 8 + 4 * (m.lane % 5), b.xmin, b.xmax);
            dy = iclamp(cdy - 8 + 4 * (m.lane / 5), b.ymin, b.ymax);
            sad = mb_sad(P, m, dx, dy, 2);
        }
        {
            uint64_t s = sad;
            const uint64_t mn = warp_min_u64(valid ? s : UINT64_MAX);
            const unsigned at = __ballot_sync(FULL, valid && s == mn);
            const int src = __ffs(at) - 1;
            dx = __shfl_sync(FULL, dx, src);
            dy = __shfl_sync(FULL, dy, src);
        }
        const int sx = dx, sy = dy;
        // 5x5 full search around it: least (sad, |d|), first in scan order
        valid = m.lane < 25;
        sad = UINT64_MAX;
        idx = m.lane;
        if (valid) {
            dx = iclamp(sx + m.lane % 5 - 2, b.xmin, b.xmax);
            dy = iclamp(sy + m.lane / 5 - 2, b.ymin, b.ymax);
            sad = mb_sad(P, m, dx, dy, 1);
        }
        warp_argmin_int(valid, sad, dx, dy, idx);
        if (sad < best.cost) {
            best.cost = sad;
            best.dx = dx;
            best.dy = dy;
        }
        if (match_good(m, best.cost)) break;
    }
    cand_sad = best.cost;
    decision = best.cost < UINT64_MAX / 8 ? distant_decision(P, m, best.cost, local.cost) : 0;
    __syncwarp();
    if (best.cost >= local.cost || decision < 2) return local;
    return best;
}

// ---- learned passes: candidates and a short integer descent ----------------------------

// (cost, |dx|+|dy|, dy, dx) lexicographic (better_integer, encoder_motion.cpp:127-133).
__device__ __forceinline__ bool int_better(uint64_t ca, int ax, int ay, uint64_t cb, int bx, int by) {
    if (ca != cb) return ca < cb;
    const int ma = iabs(ax) + iabs(ay), mb = iabs(bx) + iabs(by);
    if (ma != mb) return ma < mb;
    if (ay != by) return ay < by;
    return ax < bx;
}

// Exact full-resolution 16x16 SAD (mb_sad at stride 1, clamped sampling of the reference in
// HBM) of the pass's kLearnK candidates, clamped to the search bounds; hidden-padding vectors
// are illegal. Eight lanes per candidate, two rows each. The best by int_better, on every lane.
__device__ IntRes learned_candidates(const DevParams& P, const Mb& m, const PassDesc& d, int range) {
    const Bounds b = bounds_px(range);
    const int k = m.lane >> 3, part = m.lane & 7;
    int2 c = make_int2(0, 0);
    if (IDX_OK(m.pos >= 0 && m.pos < P.mbw * P.mbh, kSiteCands, m.pos)) c = __ldg(&d.cands[(size_t)m.pos * kLearnK + k]);
    c.x = iclamp(c.x, b.xmin, b.xmax);
    c.y = iclamp(c.y, b.ymin, b.ymax);
    uint32_t s = 0;
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int y = 2 * part + rr;
        if (y < m.ah) {
            const uint8_t* row = d.ref.y + (size_t)iclamp(m.y0 + y + c.y, 0, P.H - 1) * d.ref.pitch_y;
            const uint8_t* cur = m.sm.cur.get() + 16 * y;
#pragma unroll 4
            for (int x = 0; x < 16; ++x)
                if (x < m.aw) s += (uint32_t)iabs((int)cur[x] - (int)__ldg(row + iclamp(m.x0 + x + c.x, 0, P.W - 1)));
        }
    }
#pragma unroll
    for (int o = 4; o; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    uint64_t cost = s;
    if (hidden_padding(P, m.x0, m.y0, 16, 16, c.x * 4, c.y * 4, VC1CU_MV_QPEL, true)) cost = kBad;
    IntRes best{c.x, c.y, cost};
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
        const uint64_t oc = __shfl_xor_sync(FULL, best.cost, o);
        const int ox = __shfl_xor_sync(FULL, best.dx, o), oy = __shfl_xor_sync(FULL, best.dy, o);
        if (int_better(oc, ox, oy, best.cost, best.dx, best.dy)) best = IntRes{ox, oy, oc};
    }
    return best;
}

// Small-diamond descent from `best` (window staged about it): the four +-1 neighbours, move
// while one is int_better, at most 2 * reach steps and never farther than reach from the start.
__device__ IntRes learned_descent(const DevParams& P, const Mb& m, IntRes best, int range, int reach) {
    const Bounds b = bounds_px(range);
    const int cx = best.dx, cy = best.dy;
#pragma unroll 1
    for (int step = 0; step < 2 * reach; ++step) {
        int dx = best.dx + (m.lane == 0 ? 1 : (m.lane == 1 ? -1 : 0));
        int dy = best.dy + (m.lane == 2 ? 1 : (m.lane == 3 ? -1 : 0));
        bool valid = m.lane < 4 && dx >= b.xmin && dx <= b.xmax && dy >= b.ymin && dy <= b.ymax &&
                     iabs(dx - cx) <= reach && iabs(dy - cy) <= reach;
        uint64_t s = valid ? mb_sad(P, m, dx, dy, 1) : UINT64_MAX;
#pragma unroll 1
        for (int o = 1; o < 4; o <<= 1) {
            const bool ov = __shfl_xor_sync(FULL, valid, o);
            const uint64_t os = __shfl_xor_sync(FULL, s, o);
            const int ox = __shfl_xor_sync(FULL, dx, o), oy = __shfl_xor_sync(FULL, dy, o);
            if (ov && (!valid || int_better(os, ox, oy, s, dx, dy))) {
                valid = true;
                s = os;
                dx = ox;
                dy = oy;
            }
        }
        valid = __shfl_sync(FULL, valid, 0);
        s = __shfl_sync(FULL, s, 0);
        dx = __shfl_sync(FULL, dx, 0);
        dy = __shfl_sync(FULL, dy, 0);
        if (!valid || !int_better(s, dx, dy, best.cost, best.dx, best.dy)) break;
        best = IntRes{dx, dy, s};
    }
    return best;
}

// The learned pass's fallback test: the best match's mean absolute error is above both
// motion_match_good's six levels and the picture's mean error at the translation hint
// (global_full_sad / pixels, in o.gsad), so that sensor noise alone sends no macroblock to the
// plain search. Exact in integers: cost * W * H > px * max(6 * W * H, hint_sad).
__device__ __forceinline__ bool learned_falls_back(const DevParams& P, const Mb& m, const DevResult& o, uint64_t cost) {
    const uint64_t px = (uint64_t)m.aw * (uint64_t)m.ah;
    if (!px || cost >= UINT64_MAX / 8) return true;
    const uint64_t wh = (uint64_t)P.W * (uint64_t)P.H, hs = __ldcg(o.gsad);
    const uint64_t a = 6 * wh;
    return (unsigned __int128)cost * wh > (unsigned __int128)px * (a > hs ? a : hs);
}

struct RefineOut {
    int2 mv;
    uint64_t screen_sad;
};

// A refinement worked out before the wavefront wait under a guessed predictor and parked in
// shared memory (slot 0: the 16x16 refinement; slot k + 1: 8x8 block k): its shortlist,
// the 4MV seed it was refined from (with and without the predictor slot), the guessed
// predictor and the result under it.
struct SpecBlk {
    int2 seed;
    uint64_t seed_cost;
    int seed_slot, nk, direct, satd_done;
    uint64_t screen;
    RefineOut out;
    int2 b10;            // the seed chosen without the predictor slot
    uint64_t b10_cost;
    int b10_slot;
    RefineOut res;       // refine_select under `pi`
    PInfo pi;
};
constexpr int kSpecBlkBytes = 160;
static_assert(sizeof(SpecBlk) <= kSpecBlkBytes, "SpecBlk layout");

__device__ __forceinline__ int make_even(int v) { return !(v & 1) ? v : (v > 0 ? v - 1 : v + 1); }

// ---- the refinement's candidate list, held across the warp's lanes -------------------------
//
// Lane j < n holds list entry j (vector, CPU-law SAD). Entries are distinct vectors; their
// order is immaterial because every selection over them uses a total order, so membership
// tests, minima and ranks are warp votes and shuffles instead of serial scans.
struct RegList {
    int n;  // warp-uniform entry count (<= 32)
    int2 mv;
    uint64_t sad;
};

__device__ __forceinline__ bool sad_tie_less(uint64_t sa, int2 a, uint64_t sb, int2 b) {
    if (sa != sb) return sa < sb;
    return tie_less(a, b);
}

// Minimum over the lanes with `valid` of (s, v) under (sad, tie_less); the result on every lane.
__device__ __forceinline__ void warp_argmin_sad(bool& valid, uint64_t& s, int2& v) {
#pragma unroll 1
    for (int o = 16; o; o >>= 1) {
        const bool ov = __shfl_xor_sync(FULL, valid, o);
        const uint64_t os = __shfl_xor_sync(FULL, s, o);
        const int ox = __shfl_xor_sync(FULL, v.x, o), oy = __shfl_xor_sync(FULL, v.y, o);
        if (ov && (!valid || sad_tie_less(os, make_int2(ox, oy), s, v))) {
            valid = true;
            s = os;
            v = make_int2(ox, oy);
        }
    }
}

// Adds the candidates that lanes i < nb hold in `c` and the list lacks, in lane order, and
// scores the new ones with the CPU law in one batch (the `add` lambda, :3324-3337).
__device__ __forceinline__ void reg_add(const DevParams& P, const Mb& m, RegList& L, int2 c, int nb, int bx, int by,
                                        int bw, int bh, int mode) {
    const bool act = m.lane < nb;
    bool listed = false;
#pragma unroll 1
    for (int i = 0; i < nb; ++i) {
        const int cx = __shfl_sync(FULL, c.x, i), cy = __shfl_sync(FULL, c.y, i);
        const bool hit = __any_sync(FULL, m.lane < L.n && L.mv.x == cx && L.mv.y == cy);
        if (m.lane == i) listed = hit;
    }
    bool first = false;
    const unsigned amask = __ballot_sync(FULL, act);
    if (act) {
        const unsigned long long key = ((unsigned long long)(uint32_t)c.x << 32) | (uint32_t)c.y;
        first = (__ffs(__match_any_sync(amask, key)) - 1) == m.lane;
    }
    const bool fresh = act && !listed && first;
    const unsigned fm = __ballot_sync(FULL, fresh);
    const int nn = __popc(fm);
    if (!nn) return;
    if (fresh) m.sm.batch[__popc(fm & ((1u << m.lane) - 1))] = c;
    __syncwarp();
    sad_batch(P, m, m.sm.batch, nn, bx, by, bw, bh, mode, m.sm.batch_cost);  // hidden padding costs BAD
    if (m.lane >= L.n && m.lane < L.n + nn) {
        L.mv = m.sm.batch[m.lane - L.n];
        L.sad = m.sm.batch_cost[m.lane - L.n];
    }
    L.n += nn;
    __syncwarp();
}

// The entry equal to the stencil vectors of lanes i < nb with the least (sad, tie_less),
// folded into (best, best_sad) by the same order (every stencil vector is in the list).
__device__ __forceinline__ void reg_update_min(const Mb& m, const RegList& L, int2 c, int nb, int2& best,
                                               uint64_t& best_sad) {
    bool in_st = false;
#pragma unroll 1
    for (int i = 0; i < nb; ++i) {
        const int cx = __shfl_sync(FULL, c.x, i), cy = __shfl_sync(FULL, c.y, i);
        in_st |= m.lane < L.n && L.mv.x == cx && L.mv.y == cy;
    }
    bool valid = in_st;
    uint64_t s = L.sad;
    int2 v = L.mv;
    warp_argmin_sad(valid, s, v);
    if (valid && sad_tie_less(s, v, best_sad, best)) {
        best = v;
        best_sad = s;
    }
}

// SAD of the listed vector v (warp-uniform; it must be listed).
__device__ __forceinline__ uint64_t reg_find(const RegList& L, int lane, int2 v) {
    const unsigned hit = __ballot_sync(FULL, lane < L.n && L.mv.x == v.x && L.mv.y == v.y);
    return __shfl_sync(FULL, L.sad, __ffs(hit) - 1);
}

// refine_motion_integer_only, encoder_motion.cpp:3247-3269
__device__ RefineOut refine_integer_only(const DevParams& P, const Mb& m, int bx, int by, int bw, int bh, int2 seed,
                                         int range, int mode, uint64_t known) {
    const Bounds qb = bounds_qpel(range);
    auto snap = [](int q, int lo, int hi) {
        q = iclamp(q, lo, hi);
        const int nr = q >= 0 ? (q + 1) / 4 : (q - 1) / 4;
        return iclamp(nr * 4, lo, hi / 4 * 4);
    };
    int2 integer = make_int2(snap(seed.x, qb.xmin, qb.xmax), snap(seed.y, qb.ymin, qb.ymax));
    if (hidden_padding(P, bx, by, bw, bh, integer.x, integer.y, mode, chroma_gate(bx, by, bw, bh))) integer = make_int2(0, 0);
    uint64_t s;
    if (integer.x == seed.x && integer.y == seed.y && known != UINT64_MAX) {
        s = known;
    } else {
        if (m.lane == 0) m.sm.batch[8] = integer;
        __syncwarp();
        sad_batch(P, m, m.sm.batch + 8, 1, bx, by, bw, bh, mode, m.sm.batch_cost + 8);
        s = m.sm.batch_cost[8];
    }
    return RefineOut{integer, s};
}

// refine_qpel_block / refine_motion_block (me_quality SAD), encoder_motion.cpp:3596-3749
__device__ __forceinline__ RefineOut refine_sad_only(const DevParams& P, const Mb& m, int bx, int by, int bw, int bh,
                                                     int2 seed, int range, int mode, uint64_t known) {
    const int limit_q = 4 * P.subpel_range;
    if (!P.subpel || limit_q == 0 || imax(iabs(seed.x), iabs(seed.y)) > limit_q)
        return refine_integer_only(P, m, bx, by, bw, bh, seed, range, mode, known);
    const Bounds qb = bounds_qpel(range);
    const int xmin = imax(qb.xmin, -limit_q), xmax = imin(qb.xmax, limit_q);
    const int ymin = imax(qb.ymin, -limit_q), ymax = imin(qb.ymax, limit_q);
    const bool hp = mode_halfpel(mode);
    const int emode = hp ? mode : VC1CU_MV_QPEL;
    seed.x = iclamp(seed.x, xmin, xmax);
    seed.y = iclamp(seed.y, ymin, ymax);
    if (hp) { seed.x = make_even(seed.x); seed.y = make_even(seed.y); }
    if (hidden_padding(P, bx, by, bw, bh, seed.x, seed.y, emode, chroma_gate(bx, by, bw, bh))) {
        seed = make_int2(0, 0);
        known = UINT64_MAX;
    }
    RegList L{0, make_int2(0, 0), 0};
    if (known != UINT64_MAX) {
        L.n = 1;
        L.mv = seed;
        L.sad = known;
    } else {
        reg_add(P, m, L, seed, 1, bx, by, bw, bh, emode);
    }
    int2 best = seed;
    uint64_t cost = __shfl_sync(FULL, L.sad, 0);
    auto fix = [&](int2 v) {
        v.x = iclamp(v.x, xmin, xmax);
        v.y = iclamp(v.y, ymin, ymax);
        if (hp) { v.x = make_even(v.x); v.y = make_even(v.y); }
        return v;
    };
    // one stencil stage: gen(i) for i < np, clamped, scored and folded into (cost, best)
    auto stage = [&](int np, auto gen) {
        const int2 c = m.lane < np ? fix(gen(m.lane)) : make_int2(0, 0);
        reg_add(P, m, L, c, np, bx, by, bw, bh, emode);
        reg_update_min(m, L, c, np, best, cost);
    };
    // the two candidates beside an axis move: (c.x, c.y -/+ d) or (c.x -/+ d, c.y)
    auto side = [](int2 c, int d, bool vertical) {
        return [=](int i) { const int o = i ? d : -d; return vertical ? make_int2(c.x, c.y + o) : make_int2(c.x + o, c.y); };
    };
    auto cross = [](int2 c, int d) {
        return [=](int i) {
            return i == 0 ? make_int2(c.x - d, c.y) : i == 1 ? make_int2(c.x + d, c.y) : i == 2 ? make_int2(c.x, c.y - d)
                                                                                                   : make_int2(c.x, c.y + d);
        };
    };
    if (P.fast_subpel) {
        if (cost == 0 && best.x == 0 && best.y == 0) return RefineOut{best, 0};
        stage(4, cross(seed, 2));
        const int2 axis = best;
        const int dx = axis.x - seed.x, dy = axis.y - seed.y;
        if (dx && !dy) stage(2, side(axis, 2, true));
        else if (dy && !dx) stage(2, side(axis, 2, false));
        if (!hp) {
            const int2 half = best;
            stage(4, cross(half, 1));
            const int2 qa = best;
            const int qdx = qa.x - half.x, qdy = qa.y - half.y;
            if (qdx && !qdy) stage(2, side(qa, 1, true));
            else if (qdy && !qdx) stage(2, side(qa, 1, false));
        }
    } else {
        const int2 sd = seed;
        stage(9, [=](int i) { return make_int2(sd.x + (i % 3 - 1) * 2, sd.y + (i / 3 - 1) * 2); });
        if (!hp) {
            const int2 half = best;
            stage(9, [=](int i) { return make_int2(half.x + i % 3 - 1, half.y + i / 3 - 1); });
        }
    }
    return RefineOut{best, cost};
}

// The SAD shortlist of one staged refinement, kept in the warp's shared memory between the
// neighbour-independent half (candidate discovery, SAD, sort, and for me_quality SATD the
// SATD of every shortlisted vector) and the half that needs the MV predictor (rate term,
// score, SAD envelope, final order).
struct Shortlist {
    int direct;        // 1: the refinement needs no predictor; the result is `out`
    int nk;            // shortlisted candidates in m.sm.batch / batch_cost [0, nk)
    int satd_done;     // m.sm.list_satd[i] holds the SATD of shortlist entry i
    uint64_t screen;   // best SAD discovered (best_sad of the reference)
    RefineOut out;
};

// Vc1Encoder::refine_motion_block_staged up to the rate term (encoder_motion.cpp:3271-3456).
__device__ __forceinline__ Shortlist refine_prepare(const DevParams& P, const Mb& m, int bx, int by, int bw, int bh, int2 seed, int range,
                                    int mode, uint64_t known, bool satd_all) {
    Shortlist sl;
    sl.direct = 1;
    sl.nk = 0;
    sl.satd_done = 0;
    sl.screen = 0;
    const int limit_q = 4 * P.subpel_range;
    if (!P.subpel || limit_q == 0 || imax(iabs(seed.x), iabs(seed.y)) > limit_q) {
        sl.out = refine_integer_only(P, m, bx, by, bw, bh, seed, range, mode, known);
        return sl;
    }
    if (P.me_quality == 0) {
        sl.out = refine_sad_only(P, m, bx, by, bw, bh, seed, range, mode, known);
        return sl;
    }
    const Bounds qb = bounds_qpel(range);
    const int xmin = imax(qb.xmin, -limit_q), xmax = imin(qb.xmax, limit_q);
    const int ymin = imax(qb.ymin, -limit_q), ymax = imin(qb.ymax, limit_q);
    const bool hp = mode_halfpel(mode);
    const bool cg = chroma_gate(bx, by, bw, bh);
    seed.x = iclamp(seed.x, xmin, xmax);
    seed.y = iclamp(seed.y, ymin, ymax);
    if (hp) { seed.x = make_even(seed.x); seed.y = make_even(seed.y); }
    RegList L{0, seed, 0};
    // add(seed, known)
    if (known != UINT64_MAX) {
        L.n = 1;
        L.sad = hidden_padding(P, bx, by, bw, bh, seed.x, seed.y, mode, cg) ? kBad : known;
    } else {
        reg_add(P, m, L, seed, 1, bx, by, bw, bh, mode);
    }
    if (hidden_padding(P, bx, by, bw, bh, seed.x, seed.y, mode, cg)) reg_add(P, m, L, make_int2(0, 0), 1, bx, by, bw, bh, mode);
    int2 half_best = seed;
    uint64_t half_sad = __shfl_sync(FULL, L.sad, 0);
    const bool fast = P.fast_subpel;
    auto clampmv = [&](int x, int y) {
        int2 v = make_int2(iclamp(x, xmin, xmax), iclamp(y, ymin, ymax));
        if (hp) { v.x = make_even(v.x); v.y = make_even(v.y); }
        return v;
    };
    const int i = m.lane;
    {
        const int nb = fast ? 5 : 9;
        const int2 c = fast ? (i == 0 ? seed : i == 1 ? clampmv(seed.x - 2, seed.y) : i == 2 ? clampmv(seed.x + 2, seed.y)
                                             : i == 3 ? clampmv(seed.x, seed.y - 2) : clampmv(seed.x, seed.y + 2))
                            : clampmv(seed.x + (i % 3 - 1) * 2, seed.y + (i / 3 - 1) * 2);
        reg_add(P, m, L, c, nb, bx, by, bw, bh, mode);
        reg_update_min(m, L, c, nb, half_best, half_sad);
    }
    if (fast && !(half_best.x == seed.x && half_best.y == seed.y)) {
        const int dx = half_best.x - seed.x, dy = half_best.y - seed.y;
        const int2 hbv = half_best;
        int nd = 0;
        int2 c = make_int2(0, 0);
        if (dx && !dy) {
            nd = 2;
            c = make_int2(hbv.x, iclamp(seed.y + (i ? 2 : -2), ymin, ymax));
        } else if (dy && !dx) {
            nd = 2;
            c = make_int2(iclamp(seed.x + (i ? 2 : -2), xmin, xmax), hbv.y);
        }
        if (hp) { c.x = make_even(c.x); c.y = make_even(c.y); }
        if (nd) {
            reg_add(P, m, L, c, nd, bx, by, bw, bh, mode);
            reg_update_min(m, L, c, nd, half_best, half_sad);
        }
    }
    if (!hp) {
        if (fast) {
            const int2 qc = half_best;
            const int2 c = i == 0 ? qc : i == 1 ? make_int2(iclamp(qc.x - 1, xmin, xmax), qc.y)
                         : i == 2 ? make_int2(iclamp(qc.x + 1, xmin, xmax), qc.y)
                         : i == 3 ? make_int2(qc.x, iclamp(qc.y - 1, ymin, ymax))
                                  : make_int2(qc.x, iclamp(qc.y + 1, ymin, ymax));
            reg_add(P, m, L, c, 5, bx, by, bw, bh, mode);
            uint64_t qcost = reg_find(L, m.lane, qc);
            int2 qbmv = qc;
            reg_update_min(m, L, c, 5, qbmv, qcost);
            const int dx = qbmv.x - qc.x, dy = qbmv.y - qc.y;
            if (dx && !dy) {
                reg_add(P, m, L, make_int2(qbmv.x, iclamp(qc.y + (i ? 1 : -1), ymin, ymax)), 2, bx, by, bw, bh, mode);
            } else if (dy && !dx) {
                reg_add(P, m, L, make_int2(iclamp(qc.x + (i ? 1 : -1), xmin, xmax), qbmv.y), 2, bx, by, bw, bh, mode);
            }
        } else {
            const int2 hbv = half_best;
            reg_add(P, m, L, make_int2(iclamp(hbv.x + i % 3 - 1, xmin, xmax), iclamp(hbv.y + i / 3 - 1, ymin, ymax)), 9,
                    bx, by, bw, bh, mode);
        }
    }
    // sort by (sad, tie_less), keep 8 / 4 (:3445-3456): rank of each entry by shuffles
    const int keep = fast ? 4 : 8;
    int rank = 0;
#pragma unroll 1
    for (int k = 0; k < L.n; ++k) {
        const uint64_t sk = __shfl_sync(FULL, L.sad, k);
        const int kx = __shfl_sync(FULL, L.mv.x, k), ky = __shfl_sync(FULL, L.mv.y, k);
        rank += sad_tie_less(sk, make_int2(kx, ky), L.sad, L.mv) ? 1 : 0;
    }
    const uint64_t screen = warp_min_u64(m.lane < L.n ? L.sad : UINT64_MAX);
    const int nk = imin(L.n, keep);
    if (m.lane < L.n && rank < nk) {
        m.sm.batch[rank] = L.mv;
        m.sm.batch_cost[rank] = L.sad;
    }
    __syncwarp();
    sl.direct = 0;
    sl.nk = nk;
    sl.screen = screen;
    sl.out = RefineOut{make_int2(0, 0), screen};
    if (satd_all && P.me_quality != 1) {
        // SATD of every shortlisted vector; the eligible subset is chosen after the rate
        // term, and an eligible vector's SATD does not depend on which others are eligible
        satd_batch(P, m, m.sm.batch, nk, bx, by, bw, bh, mode, m.sm.list_satd);
        sl.satd_done = 1;
    }
    return sl;
}

// 128-bit value exchanged with the lane `o` positions away (xor).
__device__ __forceinline__ unsigned __int128 shfl_xor_u128(unsigned __int128 x, int o) {
    const uint64_t lo = __shfl_xor_sync(FULL, (uint64_t)x, o), hi = __shfl_xor_sync(FULL, (uint64_t)(x >> 64), o);
    return ((unsigned __int128)hi << 64) | lo;
}

// One shortlisted candidate in a lane's registers during the final selection.
struct SelCand {
    bool valid, elig;
    unsigned __int128 key;
    uint64_t satd, sad;
    int2 mv;
};

__device__ __forceinline__ SelCand shfl_xor_cand(const SelCand& c, int o) {
    SelCand r;
    r.valid = __shfl_xor_sync(FULL, c.valid, o);
    r.elig = __shfl_xor_sync(FULL, c.elig, o);
    r.key = shfl_xor_u128(c.key, o);
    r.satd = __shfl_xor_sync(FULL, c.satd, o);
    r.sad = __shfl_xor_sync(FULL, c.sad, o);
    r.mv = make_int2(__shfl_xor_sync(FULL, c.mv.x, o), __shfl_xor_sync(FULL, c.mv.y, o));
    return r;
}

// Rate winner order (:3477-3488): (score, sad, tie_less).
__device__ __forceinline__ bool rate_less(const SelCand& a, const SelCand& b) {
    if (a.valid != b.valid) return a.valid;
    if (a.key != b.key) return a.key < b.key;
    return sad_tie_less(a.sad, a.mv, b.sad, b.mv);
}

// Final order (:3526-3531): eligible first, then (score, satd, sad, tie_less).
__device__ __forceinline__ bool final_less(const SelCand& a, const SelCand& b) {
    if (a.valid != b.valid) return a.valid;
    if (a.elig != b.elig) return a.elig;
    if (a.key != b.key) return a.key < b.key;
    if (a.satd != b.satd) return a.satd < b.satd;
    return sad_tie_less(a.sad, a.mv, b.sad, b.mv);
}

// Least candidate of lanes 0..7 under `less`, on every lane.
template <class Less>
__device__ __forceinline__ SelCand warp_min8(SelCand c, Less less) {
#pragma unroll 1
    for (int o = 4; o; o >>= 1) {
        const SelCand d = shfl_xor_cand(c, o);
        if (less(d, c)) c = d;
    }
    SelCand r;
    r.valid = __shfl_sync(FULL, c.valid, 0);
    r.elig = __shfl_sync(FULL, c.elig, 0);
    r.key = ((unsigned __int128)__shfl_sync(FULL, (uint64_t)(c.key >> 64), 0) << 64) | __shfl_sync(FULL, (uint64_t)c.key, 0);
    r.satd = __shfl_sync(FULL, c.satd, 0);
    r.sad = __shfl_sync(FULL, c.sad, 0);
    r.mv = make_int2(__shfl_sync(FULL, c.mv.x, 0), __shfl_sync(FULL, c.mv.y, 0));
    return r;
}

// The rest of refine_motion_block_staged (encoder_motion.cpp:3458-3535) given the predictor.
// Lane i < nk holds shortlist entry i; both selections are warp reductions.
__device__ RefineOut refine_select(const DevParams& P, const Mb& m, const Shortlist& sl, int bx, int by, int bw, int bh,
                                   int mode, const PInfo& pi, bool more) {
    if (sl.direct) return sl.out;
    const int nk = sl.nk;  // <= 8
    SelCand c;
    c.valid = m.lane < nk;
    c.elig = false;
    c.mv = c.valid ? m.sm.batch[m.lane] : make_int2(0, 0);
    c.sad = c.valid ? m.sm.batch_cost[m.lane] : UINT64_MAX;
    c.satd = kBad;
    uint32_t rate = 0;
    c.key = 0;
    if (c.valid) {
        // rate + score (:3458-3476)
        int2 pred = pi.pre;
        if (pi.hybrid) {
            pred = modular_mv_distance(P, c.mv, pi.a) <= modular_mv_distance(P, c.mv, pi.c) ? pi.a : pi.c;
            ++rate;
        }
        rate += mv_rate_bits(P, c.mv, pred, mode, more);
        c.key = score_key(P, m.lam_m, m.lam_s, c.sad, rate);
    }
    const SelCand rw = warp_min8(c, rate_less);
    if (P.me_quality == 1) {
        __syncwarp();
        return RefineOut{rw.mv, sl.screen};
    }
    const uint64_t rws = rw.sad;
    const uint64_t pct3 = (rws / 100) * 3 + (((rws % 100) * 3 + 99) / 100);
    const uint64_t slack = pct3 > 4 ? pct3 : 4;
    const uint64_t limit = rws > UINT64_MAX - slack ? UINT64_MAX : rws + slack;
    c.elig = c.valid && c.sad < UINT64_MAX / 8 && c.sad <= limit;
    // SATD of the eligible shortlist (:3507-3524), unless already known for every entry
    if (sl.satd_done) {
        if (c.elig) c.satd = m.sm.list_satd[m.lane];
    } else {
        const unsigned em = __ballot_sync(FULL, c.elig);
        const int pos = __popc(em & ((1u << m.lane) - 1));
        int2* el = m.sm.batch + 16;
        if (c.elig) el[pos] = c.mv;
        __syncwarp();
        satd_batch(P, m, el, __popc(em), bx, by, bw, bh, mode, m.sm.list_satd + 8);
        if (c.elig) c.satd = m.sm.list_satd[8 + pos];
    }
    if (c.valid) c.key = score_key(P, m.lam_m, m.lam_s, c.satd, rate);
    const SelCand best = warp_min8(c, final_less);
    __syncwarp();
    return RefineOut{best.mv, sl.screen};
}

// ---- out-of-line refinement ---------------------------------------------------------------
//
// The staged refinement is reached from several places of the kernel; one out-of-line copy
// of each half keeps the kernel's instruction footprint small enough for the instruction
// cache. Only values cross the call (never the address of the kernel's parameter block or
// of the macroblock state), so the caller's state stays in registers.

// Writes the macroblock's MbCtx (lane 0) once its window geometry is known.
__device__ void publish_ctx(const DevParams& P, const Mb& m) {
    if (m.lane == 0) {
        MbCtx& r = *reinterpret_cast<MbCtx*>(g_smem + m.sm.ctx.off);
        r.g = score_geo(P);
        r.win_off = m.sm.win.off;
        r.cur_off = m.sm.cur.off;
        r.cur2_off = m.sm.cur2.off;
        r.cur4_off = m.sm.cur4.off;
        r.wp = m.wp;
        r.wx0 = m.wx0;
        r.wy0 = m.wy0;
        r.wh = m.wh;
        r.x0 = m.x0;
        r.y0 = m.y0;
        r.aw = m.aw;
        r.ah = m.ah;
        r.gref = m.gref.p;
        r.gpitch = m.gref.pitch;
        r.subpel = P.subpel;
        r.fast_subpel = P.fast_subpel;
        r.subpel_range = P.subpel_range;
        r.me_quality = P.me_quality;
        r.mvrange = P.mvrange;
        r.mant_bits = P.mant_bits;
        r.lam_s = m.lam_s;
        r.lam_m = m.lam_m;
        r.batch = m.sm.batch.off;
        r.cost = m.sm.batch_cost.off;
        r.satd = m.sm.list_satd.off;
        r.sp = m.d->sp_planes;
        r.sp_pitch = m.d->sp_pitch;
        r.sp_border = m.d->sp_border;
        r.sp_stride = m.d->sp_stride;
    }
    __syncwarp();
}

// The parameter block and macroblock state the refinement reads, rebuilt from the MbCtx.
__device__ __forceinline__ void ref_unpack(uint32_t ctx, DevParams& P, Mb& m) {
    const MbCtx& r = mbctx(ctx);
    P = geo_params(r.g);
    P.subpel = r.subpel;
    P.fast_subpel = r.fast_subpel;
    P.subpel_range = r.subpel_range;
    P.me_quality = r.me_quality;
    P.mvrange = r.mvrange;
    P.mant_bits = r.mant_bits;
    m.lane = threadIdx.x & 31;
    m.lam_m = r.lam_m;
    m.lam_s = r.lam_s;
    m.x0 = r.x0;
    m.y0 = r.y0;
    m.aw = r.aw;
    m.ah = r.ah;
    m.wx0 = r.wx0;
    m.wy0 = r.wy0;
    m.wp = r.wp;
    m.wh = r.wh;
    m.gref = GlobSampler{r.gref, r.gpitch, P.W, P.H};
    m.sm.ctx.off = ctx;
    m.sm.win.off = r.win_off;
    m.sm.cur.off = r.cur_off;
    m.sm.cur2.off = r.cur2_off;
    m.sm.cur4.off = r.cur4_off;
    m.sm.batch.off = r.batch;
    m.sm.batch_cost.off = r.cost;
    m.sm.list_satd.off = r.satd;
}

// DR: the launch runs the default refinement (me_quality SATD, the full stencils); fixing those
// parameters lets the compiler drop the other refinements from these hot functions.
template <bool DR>
__device__ __forceinline__ void refine_defaults(DevParams& P) {
    if (DR) {
        P.me_quality = 2;
        P.fast_subpel = 0;
    }
}

template <bool DR>
__device__ __noinline__ Shortlist refine_prepare_ool(uint32_t ctx, int bx, int by, int bw, int bh, int2 seed, int range,
                                                     int mode, uint64_t known, bool satd_all) {
    DevParams P;
    Mb m{};
    ref_unpack(ctx, P, m);
    refine_defaults<DR>(P);
    return refine_prepare(P, m, bx, by, bw, bh, seed, range, mode, known, satd_all);
}

template <bool DR>
__device__ __noinline__ RefineOut refine_select_ool(uint32_t ctx, const Shortlist sl, int bx, int by, int bw, int bh,
                                                    int mode, const PInfo pi, bool more) {
    DevParams P;
    Mb m{};
    ref_unpack(ctx, P, m);
    refine_defaults<DR>(P);
    return refine_select(P, m, sl, bx, by, bw, bh, mode, pi, more);
}

template <bool DR>
__device__ __forceinline__ RefineOut refine_staged(const DevParams& P, const Mb& m, int bx, int by, int bw, int bh, int2 seed,
                                                   int range, int mode, const PInfo& pi, bool more, uint64_t known) {
    const uint32_t r = m.sm.ctx.off;
    const Shortlist sl = refine_prepare_ool<DR>(r, bx, by, bw, bh, seed, range, mode, known, false);
    return refine_select_ool<DR>(r, sl, bx, by, bw, bh, mode, pi, more);
}

// ---- shortlists parked across the wavefront wait -----------------------------------------

__device__ __forceinline__ void shortlist_save(const Mb& m, int slot, const Shortlist& sl, int2 seed, uint64_t seed_cost,
                                               int seed_slot) {
    if (!sl.direct && m.lane < sl.nk) {
        m.sm.spec_mv[slot * 8 + m.lane] = m.sm.batch[m.lane];
        m.sm.spec_cost[slot * 8 + m.lane] = m.sm.batch_cost[m.lane];
        m.sm.spec_satd[slot * 8 + m.lane] = m.sm.list_satd[m.lane];
    }
    if (m.lane == 0) {
        SpecBlk& b = m.sm.spec_blk[slot];
        b.seed = seed;
        b.seed_cost = seed_cost;
        b.seed_slot = seed_slot;
        b.nk = sl.nk;
        b.direct = sl.direct;
        b.satd_done = sl.satd_done;
        b.screen = sl.screen;
        b.out = sl.out;
    }
    __syncwarp();
}

// Puts a parked shortlist back into the working buffers refine_select reads.
__device__ __forceinline__ Shortlist shortlist_restore(const Mb& m, int slot) {
    const SpecBlk& b = m.sm.spec_blk[slot];
    Shortlist sl;
    sl.direct = b.direct;
    sl.nk = b.nk;
    sl.satd_done = b.satd_done;
    sl.screen = b.screen;
    sl.out = b.out;
    if (!sl.direct && m.lane < sl.nk) {
        m.sm.batch[m.lane] = m.sm.spec_mv[slot * 8 + m.lane];
        m.sm.batch_cost[m.lane] = m.sm.spec_cost[slot * 8 + m.lane];
        m.sm.list_satd[m.lane] = m.sm.spec_satd[slot * 8 + m.lane];
    }
    __syncwarp();
    return sl;
}

// ---- Mixed-MV block seeds (encoder_motion.cpp:250-374) -----------------------------------

// The eleven seed slots of one 8x8 block in m.sm.batch[0..10]: slot 0 the within-radius
// `one`, then the reference's ten seeds {one, pred, one -/+8 x, one -/+8 y, one -/+4 x,
// one -/+4 y}, clamped to the quarter-pel bounds.
__device__ __forceinline__ void put_4mv_seeds(const DevParams& P, const Mb& m, int2 one, int2 pred, const Bounds& qb) {
    const int limit = 4 * P.subpel_range;
    if (m.lane < 11) {
        int2 v;
        if (m.lane <= 1) v = one;
        else if (m.lane == 2) v = pred;
        else {
            const int t = m.lane - 3, d4 = t < 4 ? 8 : 4, dir = t & 3;
            v = dir == 0 ? make_int2(one.x - d4, one.y) : dir == 1 ? make_int2(one.x + d4, one.y)
              : dir == 2 ? make_int2(one.x, one.y - d4) : make_int2(one.x, one.y + d4);
        }
        if (m.lane > 0) v = make_int2(iclamp(v.x, qb.xmin, qb.xmax), iclamp(v.y, qb.ymin, qb.ymax));
        if (imax(iabs(v.x), iabs(v.y)) > limit) { v.x = (v.x / 4) * 4; v.y = (v.y / 4) * 4; }
        m.sm.batch[m.lane] = v;
    }
    __syncwarp();
}

struct SeedPick {
    int2 v;
    uint64_t cost;
    int slot;
};

__device__ __forceinline__ int l1_norm(int2 v) { return iabs(v.x) + iabs(v.y); }

// The reference's seed choice over the scored slots: the first slot that attains the least
// (SAD, |mv|_1); with skip_pred the predictor slot 2 takes no part. A warp reduction over
// lanes 0..10 by (SAD, |mv|_1, slot).
__device__ __forceinline__ SeedPick pick_4mv_seed(const Mb& m, bool skip_pred) {
    const int l = m.lane;
    bool valid = l <= 10 && !(skip_pred && l == 2);
    int2 v = valid ? m.sm.batch[l] : make_int2(0, 0);
    uint64_t c = valid ? m.sm.batch_cost[l] : 0;
    int slot = l;
#pragma unroll 1
    for (int o = 8; o; o >>= 1) {
        const bool ov = __shfl_xor_sync(FULL, valid, o);
        const uint64_t oc = __shfl_xor_sync(FULL, c, o);
        const int ox = __shfl_xor_sync(FULL, v.x, o), oy = __shfl_xor_sync(FULL, v.y, o);
        const int os = __shfl_xor_sync(FULL, slot, o);
        const int2 ovv = make_int2(ox, oy);
        bool take = false;
        if (ov && !valid) take = true;
        else if (ov) {
            if (oc != c) take = oc < c;
            else if (l1_norm(ovv) != l1_norm(v)) take = l1_norm(ovv) < l1_norm(v);
            else take = os < slot;
        }
        if (take) {
            valid = true;
            c = oc;
            v = ovv;
            slot = os;
        }
    }
    SeedPick b{make_int2(__shfl_sync(FULL, v.x, 0), __shfl_sync(FULL, v.y, 0)), __shfl_sync(FULL, c, 0),
               __shfl_sync(FULL, slot, 0)};
    __syncwarp();
    return b;
}

// True when slot `slot` holding (v, c) would have been chosen over the pick b.
__device__ __forceinline__ bool seed_before(int2 v, uint64_t c, int slot, const SeedPick& b) {
    if (v.x == b.v.x && v.y == b.v.y) return false;
    if (c != b.cost) return c < b.cost;
    const int lv = l1_norm(v), lb = l1_norm(b.v);
    if (lv != lb) return lv < lb;
    return slot < b.slot;
}

// ---- predictor state of the current pass --------------------------------------------------
//
// Every predictor of the reference reads only the left, top-left, top and top-right
// macroblocks and the current one (encoder_motion.cpp:1312-1466). Their state is fetched
// into shared memory once, after the wavefront wait, with one load per lane.

__device__ void load_neighbours(const DevParams& P, const Mb& m, const DevResult& o) {
    const int q = m.lane < 16 ? (m.lane >> 2) : (m.lane & 3);
    const int nx = m.mx + (q == 0 || q == 1 ? -1 : (q == 2 ? 0 : 1)), ny = m.my - (q == 0 ? 0 : 1);
    bool valid = nx >= 0 && ny >= 0 && nx < P.mbw;
    const int nb = ny * P.mbw + nx;
    valid = valid && IDX_OK(nb >= 0 && nb < P.mbw * P.mbh, kSiteNeighbour, nb);
    if (m.lane < 16) m.sm.nb_bmv[m.lane] = valid ? __ldcg(&o.bmv[nb * 4 + (m.lane & 3)]) : make_int2(0, 0);
    else if (m.lane < 20) m.sm.nb_mv[q] = valid ? __ldcg(&o.mvs[nb]) : make_int2(0, 0);
    else if (m.lane < 24) m.sm.nb_intra[q] = valid ? (int)__ldcg(&o.intra[nb]) : 0;
    __syncwarp();
}

// The neighbourhood a learned pass refines under: each neighbour's first candidate (the
// network's top proposal, integer pixels) as its 1-MV vector, no P-intra. It is known before any
// macroblock is analysed, so a learned pass has no wavefront.
__device__ void load_cand_neighbours(const DevParams& P, const Mb& m, const PassDesc& d) {
    const int q = m.lane < 16 ? (m.lane >> 2) : (m.lane & 3);
    const int nx = m.mx + (q == 0 || q == 1 ? -1 : (q == 2 ? 0 : 1)), ny = m.my - (q == 0 ? 0 : 1);
    const bool valid = nx >= 0 && ny >= 0 && nx < P.mbw;
    const int nb = ny * P.mbw + nx;
    int2 v = make_int2(0, 0);
    if (valid && m.lane < 20) {
        v = __ldg(&d.cands[(size_t)nb * kLearnK]);
        v = make_int2(4 * v.x, 4 * v.y);
    }
    if (m.lane < 16) m.sm.nb_bmv[m.lane] = v;
    else if (m.lane < 20) m.sm.nb_mv[q] = v;
    else if (m.lane < 24) m.sm.nb_intra[q] = 0;
    __syncwarp();
}

// A stand-in neighbourhood for guessing before the wavefront wait: the seed pass's final
// vectors and P-intra flags of the same four neighbours (that pass is complete), and a
// zero current MB.
__device__ void guess_neighbours(const DevParams& P, const Mb& m, const PassDesc& d) {
    const int q = m.lane < 16 ? (m.lane >> 2) : (m.lane & 3);
    const int nx = m.mx + (q == 0 || q == 1 ? -1 : (q == 2 ? 0 : 1)), ny = m.my - (q == 0 ? 0 : 1);
    const bool valid = nx >= 0 && ny >= 0 && nx < P.mbw;
    const int nb = ny * P.mbw + nx;
    if (m.lane < 16) m.sm.nb_bmv[m.lane] = valid ? __ldcg(&d.seed_bmv[nb * 4 + (m.lane & 3)]) : make_int2(0, 0);
    else if (m.lane < 20) m.sm.nb_mv[q] = valid ? __ldcg(&d.seed_mvs[nb]) : make_int2(0, 0);
    else if (m.lane < 24) m.sm.nb_intra[q] = valid ? (int)__ldcg(&d.seed_intra[nb]) : 0;
    else if (m.lane < 28) m.sm.cur_bmv[m.lane - 24] = make_int2(0, 0);
    __syncwarp();
}

__device__ __forceinline__ bool pinfo_equal(const PInfo& a, const PInfo& b) {
    return a.pre.x == b.pre.x && a.pre.y == b.pre.y && a.a.x == b.a.x && a.a.y == b.a.y && a.c.x == b.c.x &&
           a.c.y == b.c.y && a.a_valid == b.a_valid && a.c_valid == b.c_valid && a.hybrid == b.hybrid;
}

// Parks the guessed predictor and the result under it in slot `slot`.
__device__ __forceinline__ void spec_result_save(const Mb& m, int slot, const PInfo& pi, const RefineOut& res) {
    if (m.lane == 0) {
        SpecBlk& b = m.sm.spec_blk[slot];
        b.pi = pi;
        b.res = res;
    }
    __syncwarp();
}

// Vc1Encoder::predictor_info, encoder_motion.cpp:1312-1352 (reads the pass's 1-MV field)
__device__ PInfo predictor_info(const DevParams& P, const Mb& m) {
    PInfo r;
    const int mbw = P.mbw, mx = m.mx, my = m.my;
    int2 A = make_int2(0, 0), B = A, C = A;
    const bool a_valid = my > 0, c_valid = mx > 0, b_valid = my > 0 && mbw > 1;
    if (a_valid) A = m.sm.nb_mv[2];
    if (c_valid) C = m.sm.nb_mv[0];
    if (b_valid) B = (mx == mbw - 1) ? m.sm.nb_mv[1] : m.sm.nb_mv[3];
    int2 pre = make_int2(0, 0);
    if (a_valid) pre = A;
    else if (c_valid) pre = C;
    else if (b_valid) pre = B;
    if ((int)a_valid + (int)b_valid + (int)c_valid > 1) {
        pre.x = median3(A.x, B.x, C.x);
        pre.y = median3(A.y, B.y, C.y);
    }
    pullback(pre, mx * 64, my * 64, mbw * 64 - 4, P.mbh * 64 - 4, -60);
    bool hybrid = false;
    if (a_valid && c_valid) {
        if (iabs(pre.x - A.x) + iabs(pre.y - A.y) > 32) hybrid = true;
        else if (iabs(pre.x - C.x) + iabs(pre.y - C.y) > 32) hybrid = true;
    }
    r.pre = pre; r.a = A; r.c = C; r.a_valid = a_valid; r.c_valid = c_valid; r.hybrid = hybrid;
    return r;
}

// Block-MV field accessor over the current MB (shared memory) and its prefetched neighbours.
struct Field {
    const int2* cur4;
    const int2* nb_bmv;
    const int* nb_intra;
    int mbw, mbh, mx, my;
    __device__ __forceinline__ int nb_index(int bxm, int bym) const {
        return bym == my ? 0 : (bxm < mx ? 1 : (bxm == mx ? 2 : 3));
    }
    __device__ int2 get(int x, int y) const {
        if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return make_int2(0, 0);
        const int bxm = x >> 1, bym = y >> 1, k = ((y & 1) << 1) | (x & 1);
        if (bxm == mx && bym == my) return cur4[k];
        return nb_bmv[nb_index(bxm, bym) * 4 + k];
    }
    __device__ bool intra(int x, int y) const {
        if (x < 0 || y < 0 || x >= mbw * 2 || y >= mbh * 2) return false;
        const int bxm = x >> 1, bym = y >> 1;
        if (bxm == mx && bym == my) return false;  // the current MB is never intra while it is searched
        return nb_intra[nb_index(bxm, bym)] != 0;
    }
};

__device__ __forceinline__ int median4(int a, int b, int c, int d) {
    if (a < b) {
        if (c < d) return (imin(b, d) + imax(a, c)) / 2;
        return (imin(b, c) + imax(a, d)) / 2;
    }
    if (c < d) return (imin(a, d) + imax(b, c)) / 2;
    return (imin(a, c) + imax(b, d)) / 2;
}

// ---- wavefront synchronisation ----------------------------------------------------------

__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Waits (bounded) until each lane's flag equals epoch (a macroblock of this launch was
// published; a lane with a null flag waits for nothing). The flags are polled with relaxed
// loads, all lanes at once, and one acquire fence follows the last poll, so a poll costs
// no L1 invalidation. Every lane calls it. After 2^log2_limit polls it gives up: it raises
// the launch's error and abort flags and returns false (a wait that sees the abort flag
// returns false at once).
// code: the waiting work item, recorded (with the lanes still waiting) by the first wait
// that gives up.
__device__ bool wait_flags(const uint32_t* flag, uint32_t epoch, LaunchStatus* st, uint32_t code, int log2_limit) {
    bool mine = flag == nullptr;
    const long limit = 1L << log2_limit;
    for (long it = 0; it < limit; ++it) {
        if (!mine) mine = ld_relaxed(flag) == epoch;
        if (__all_sync(FULL, mine)) {
            // the observing lanes acquire; the warp barrier orders the other lanes' reads after it
            fence_acquire();
            __syncwarp();
            return true;
        }
        if ((it & 15) == 15) {
            const int ab = __shfl_sync(FULL, (int)ld_relaxed(reinterpret_cast<const uint32_t*>(&st->abort)), 0);
            if (ab) return false;
        }
        __nanosleep(64);
    }
    const unsigned waiting = __ballot_sync(FULL, !mine);
    if ((threadIdx.x & 31) == 0) {
        if (atomicCAS(&st->tcode, 0u, code + 1u) == 0u) st->tmask = waiting;
        atomicExch(&st->error, (int)VC1CU_ERR_TIMEOUT);
        atomicExch(&st->abort, 1);
        atomicAdd(&st->timeouts, 1u);
    }
    return false;
}

// Waits for the left, top-left, top and top-right macroblocks of the same pass (lanes 0..3;
// positions outside the raster need no wait).
__device__ bool wait_neighbours(const DevParams& P, const DevResult& o, int mx, int my, int lane, uint32_t epoch,
                                LaunchStatus* st, uint32_t code) {
    const uint32_t* f = nullptr;
    if (lane < 4) {
        const int x = mx + (lane == 3 ? 1 : (lane == 2 ? 0 : -1)), y = my - (lane == 0 ? 0 : 1);
        if (x >= 0 && y >= 0 && x < P.mbw) f = &o.done[y * P.mbw + x];
    }
    return wait_flags(f, epoch, st, code, P.wait_log2);
}

// ---- the kernel ---------------------------------------------------------------------------

// Carves one warp's buffers from byte offset `base` of the dynamic shared memory.
__device__ void carve(WarpMem& s, uint32_t base, const WinCfg& wc) {
    uint32_t p = base;
    auto take = [&](uint32_t bytes) {
        const uint32_t q = p;
        p += (bytes + 15) & ~15u;
        return q;
    };
    s.list_key.off = take(sizeof(unsigned __int128) * kListCap);
    s.list_sad.off = take(8 * kListCap);
    s.list_satd.off = take(8 * kListCap);
    s.batch_cost.off = take(8 * 32);
    s.keys.off = take(8 * (uint32_t)wc.keys_cap);
    s.top.off = take(8 * 8);
    s.list_mv.off = take(8 * kListCap);
    s.batch.off = take(8 * 32);
    s.stencil.off = take(8 * 16);
    s.list_rate.off = take(4 * kListCap);
    s.cur2.off = take(4 * 32);
    s.cur4.off = take(4 * 16);
    s.misc.off = take(4 * 16);
    s.cur_bmv.off = take(8 * 4);
    s.nb_mv.off = take(8 * 4);
    s.nb_bmv.off = take(8 * 16);
    s.nb_intra.off = take(4 * 4);
    s.spec_mv.off = take(8 * 40);
    s.spec_cost.off = take(8 * 40);
    s.spec_satd.off = take(8 * 40);
    s.spec_blk.off = take(kSpecBlkBytes * 5);
    s.ctx.off = take(kMbCtxBytes);
    s.seen.off = take(4 * (uint32_t)wc.seen_words);
    s.seen_full.off = take(4 * (uint32_t)wc.seen_words);
    s.cur.off = take(256);
    s.tma_bar.off = take(8);
    // the window starts on a 128-byte boundary of the shared address space (a TMA destination)
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(g_smem);
    p = ((sbase + p + 127) & ~127u) - sbase;
    s.win.off = take((uint32_t)(wc.wp * wc.wh + 32));
}

__host__ __device__ inline int warp_bytes_for(const WinCfg& wc) {
    auto r = [](int b) { return (b + 15) & ~15; };
    return r(16 * kListCap) + r(8 * kListCap) * 2 + r(8 * 32) + r(8 * wc.keys_cap) + r(64) + r(8 * kListCap) +
           r(8 * 32) + r(128) + r(4 * kListCap) + r(128) + r(64) + r(64) + r(32) + r(32) + r(128) + r(16) +
           3 * r(8 * 40) + r(kSpecBlkBytes * 5) + r(kMbCtxBytes) +
           2 * r(4 * wc.seen_words) + r(256) + r(8) + 128 +
           r(wc.wp * wc.wh + 32);
}

int warp_bytes_for_host(const WinCfg& wc) { return warp_bytes_for(wc); }

// 16 bytes from global to shared memory without a register round trip (cp.async; both
// addresses 16-byte aligned). The copy lands by the next window_wait().
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}

// ---- the window's TMA copy (cp.async.bulk.tensor on the reference's tensor map) ----------
__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Lane 0: orders the warp's earlier generic reads of the window before the async write, arms
// the barrier with the box's bytes and issues the 2-D tensor copy of the box at (x, y).
__device__ __forceinline__ void tma_window(uint32_t dst, const void* tmap, int x, int y, uint32_t bar, uint32_t bytes) {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ bool tma_bar_test(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits (bounded) for the window's TMA copy; on timeout records VC1CU_ERR_TIMEOUT with the work
// item, aborts the launch and leaves the copy marked pending (drained before the kernel exits).
__device__ void tma_wait(Mb& m, LaunchStatus* st, uint32_t code, int log2_limit) {
    if (!m.tma_pending) return;
    const uint32_t bar = m.sm.tma_bar.off + sh_addr(g_smem);
    const long limit = 1L << log2_limit;
    for (long it = 0; it < limit; ++it) {
        if (tma_bar_test(bar, m.tma_phase)) {
            m.tma_phase ^= 1u;
            m.tma_pending = false;
            __syncwarp();
            return;
        }
        if (it > 64) __nanosleep(32);
    }
    if (m.lane == 0 && st) {
        if (atomicCAS(&st->tcode, 0u, code + 1u) == 0u) st->tmask = 0x100u;  // 0x100: the window copy
        atomicExch(&st->error, (int)VC1CU_ERR_TIMEOUT);
        atomicExch(&st->abort, 1);
        atomicAdd(&st->timeouts, 1u);
    }
}

// Completes this thread's cp.async copies; the warp barrier makes every lane's copies
// visible to the whole warp.
__device__ __forceinline__ void window_wait(Mb& m, LaunchStatus* st, uint32_t code, int log2_limit) {
    tma_wait(m, st, code, log2_limit);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
}

// Stages the reference window around MV (cdx, cdy) integer pixels: rows wy0 .. wy0+wh-1,
// columns from the 16-byte-aligned wx0. Chunks inside the raster are asynchronous 16-byte
// copies (all of a lane's in flight at once) that land at the next window_wait(); edge
// chunks clamp per byte and are stored at once.
__device__ void load_window(const DevParams& P, Mb& m, const DevFrame& ref, int cdx, int cdy, const WinCfg& wc) {
    m.wh = wc.wh;
    m.wp = wc.wp;
    m.wx0 = (m.x0 + cdx - wc.rw - 1) & ~15;
    m.wy0 = m.y0 + cdy - wc.rw - 1;
    // a window wholly inside the picture: one tensor copy (its x is a multiple of 16 bytes)
    if (wc.tma && m.d->ref_tma && m.wx0 >= 0 && m.wy0 >= 0 && m.wx0 + m.wp <= P.W && m.wy0 + m.wh <= P.H &&
        !m.tma_pending) {
        __syncwarp();  // every lane's reads of the previous window are done
        if (m.lane == 0)
            tma_window(sh_addr(m.sm.win.get()), m.d->ref_tmap, m.wx0, m.wy0, sh_addr(m.sm.tma_bar.get()),
                       (uint32_t)(m.wp * m.wh));
        m.tma_pending = true;
        return;
    }
    const int cpr = m.wp >> 4;
    const int total = m.wh * cpr;
#pragma unroll 4
    for (int j = m.lane; j < total; j += 32) {
        const int r = j / cpr, c = j - r * cpr;
        const int gy = iclamp(m.wy0 + r, 0, P.H - 1), gx = m.wx0 + 16 * c;
        const uint8_t* row = ref.y + (size_t)gy * ref.pitch_y;
        uint8_t* dst = m.sm.win.get() + r * m.wp + 16 * c;
        if (!IDX_OK(r < m.wh && 16 * c + 16 <= m.wp, kSiteStage, j)) continue;
        if (gx >= 0 && gx + 16 <= P.W) {
            cp_async16(dst, row + gx);
        } else {
            uint32_t w[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t x = 0;
#pragma unroll
                for (int i = 0; i < 4; ++i) x |= (uint32_t)__ldg(row + iclamp(gx + 4 * k + i, 0, P.W - 1)) << (8 * i);
                w[k] = x;
            }
            *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Current MB into shared memory (zero outside the raster) plus its packed column subsets.
__device__ void load_cur(const DevParams& P, Mb& m, const DevFrame& cur) {
    if (m.aw == 16) {
        if (m.lane < 16) {
            uint4 v = make_uint4(0, 0, 0, 0);
            if (m.lane < m.ah) v = __ldg(reinterpret_cast<const uint4*>(cur.y + (size_t)(m.y0 + m.lane) * cur.pitch_y + m.x0));
            *reinterpret_cast<uint4*>(m.sm.cur.get() + 16 * m.lane) = v;
        }
    } else {
        for (int i = m.lane; i < 256; i += 32) {
            const int y = i >> 4, x = i & 15;
            m.sm.cur[i] = (x < m.aw && y < m.ah) ? __ldg(cur.y + (size_t)(m.y0 + y) * cur.pitch_y + m.x0 + x) : 0;
        }
    }
    __syncwarp();
    const uint32_t* c32 = reinterpret_cast<const uint32_t*>(m.sm.cur.get());
    {
        const int row = m.lane >> 1, k = m.lane & 1;
        m.sm.cur2[row * 2 + k] = __byte_perm(c32[row * 4 + 2 * k], c32[row * 4 + 2 * k + 1], 0x6420);
    }
    if (m.lane < 16) {
        const int row = m.lane;
        m.sm.cur4[row] = __byte_perm(__byte_perm(c32[row * 4 + 0], c32[row * 4 + 1], 0x0040),
                                     __byte_perm(c32[row * 4 + 2], c32[row * 4 + 3], 0x0040), 0x5410);
    }
    __syncwarp();
}

// P-intra proxy of the current MB (encoder_motion.cpp:384-396): sum over its four 8x8
// blocks of |pixel - visible block mean|. Lane = block k * 8 + row.
__device__ uint64_t intra_proxy(const DevParams& P, const Mb& m) {
    uint32_t part = 0;
    const int k = m.lane >> 3, row = m.lane & 7;
    const int bx = (k & 1) * 8, by = ((k >> 1) & 1) * 8;
    const int vw = imax(0, imin(8, P.W - (m.x0 + bx))), vh = imax(0, imin(8, P.H - (m.y0 + by)));
    uint32_t rs = 0;
    if (row < vh)
        for (int x = 0; x < vw; ++x) rs += m.sm.cur[(by + row) * 16 + bx + x];
    for (int o2 = 4; o2; o2 >>= 1) rs += __shfl_xor_sync(FULL, rs, o2);
    const uint32_t nn = (uint32_t)vw * (uint32_t)vh;
    const int mean = (!vw || !vh) ? 128 : (int)((rs + nn / 2) / nn);  // visible_block_mean (encoder_entropy.cpp:496)
    if (row < vh)
        for (int x = 0; x < vw; ++x) part += (uint32_t)iabs((int)m.sm.cur[(by + row) * 16 + bx + x] - mean);
    return warp_sum_u64(part);
}

// items[k] = (pass << 20) | macroblock: the launch's work queue. Inside one pass the
// macroblocks come in wavefront order (t = x + 2y, then y), so every same-pass dependency
// (left, top-left, top, top-right) of an item precedes it and the items of one t are
// independent; a pass seeded by another pass of the launch is delayed behind it, so its
// seed macroblock precedes it too. Items are handed out in order, hence no wait can
// depend on an item that no running warp holds.
// Instantiations (the kCore* flags): kCoreAny runs any mix of passes; the flags compile out what
// a launch's passes cannot reach (seeded-only launches also need fewer registers and hold more
// resident warps). Four warps per block; at most 65536 / (128 * min blocks) registers per thread.
#ifndef VC1CU_CORE_MIN_BLOCKS
#define VC1CU_CORE_MIN_BLOCKS 3
#endif
#ifndef VC1CU_SEEDED_MIN_BLOCKS
#define VC1CU_SEEDED_MIN_BLOCKS 4
#endif
template <int KIND>
// The wide-register instantiation (one block per SM) takes up to 8 warps per block: 255
// registers x 256 threads is the SM's register file.
__global__ void __launch_bounds__((KIND & kCoreWide) ? 256 : 128,
                                  (KIND & (kCoreSeededOnly | kCoreLearned)) ? VC1CU_SEEDED_MIN_BLOCKS
                                                                           : ((KIND & kCoreWide) ? 1 : VC1CU_CORE_MIN_BLOCKS))
    core_pass_kernel(const __grid_constant__ DevParams P0, const PassDesc* passes, int npass, const uint32_t* items,
                     unsigned nitems, WinCfg wc, uint32_t epoch, LaunchStatus* st) {
    Mb m;
    m.lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    carve(m.sm, (uint32_t)(warp * wc.warp_bytes), wc);
#ifdef VC1CU_INDEX_CHECK
    m.keys_cap = wc.keys_cap;
#endif
    m.tma_phase = 0;
    m.tma_pending = false;
    if (wc.tma && m.lane == 0) tma_bar_init(sh_addr(m.sm.tma_bar.get()));
    __syncwarp();
    const int range = P0.range, local_range = P0.local_range;  // one search configuration per launch
    for (;;) {
        unsigned item = 0;
        if (m.lane == 0) item = atomicAdd(&st->queue, 1u);
        item = __shfl_sync(FULL, item, 0);
        if (item >= nitems) break;
        const uint32_t code = __ldg(&items[item]);
        const int pi_idx = (int)(code >> 20);
        const int mbi = (int)(code & 0xFFFFFu);
        if (!IDX_OK(pi_idx < npass, kSiteWorkItem, code)) continue;
        const PassDesc& d = passes[pi_idx];
        // the picture geometry of this item (every pass of a kCoreMulti launch has its own)
        const DevParams& P = (KIND & kCoreMulti) ? d.geom : P0;
        if (!IDX_OK(mbi < P.mbw * P.mbh, kSiteWorkItem, code)) continue;
        m.d = &d;
        m.mx = mbi % P.mbw;
        m.my = mbi / P.mbw;
        m.pos = mbi;
        m.x0 = m.mx * 16;
        m.y0 = m.my * 16;
        m.aw = imax(0, imin(16, P.W - m.x0));
        m.ah = imax(0, imin(16, P.H - m.y0));
        m.gref = GlobSampler{d.ref.y, d.ref.pitch_y, P.W, P.H};
        m.lam_m = d.lam_m;
        m.lam_s = d.lam_s;
        const DevResult& o = d.out;
        constexpr bool kUmhOnly = (KIND & kCoreUmhLocal) != 0;
        constexpr bool kDR = (KIND & kCoreDefaultRefine) != 0;
        const int mode = d.mode,
                  seeded = (KIND & kCoreSeededOnly) ? 1 : ((KIND & kCoreUnseededOnly) ? 0 : d.seeded);
        const bool allow_intra = !(KIND & kCoreNoIntra) && d.allow_intra && !P.disable_p_intra;
        const bool allow_4mv = !(KIND & kCoreNoMixed) && mode == VC1CU_MV_MIXED;
        const int one_mode = allow_4mv ? VC1CU_MV_QPEL : mode;
        PHASE_START((seeded ? 1 : 0) + (allow_4mv ? 2 : 0));
        bool ok = !*(volatile int*)&st->abort;
        if (d.only && !__ldcg(&d.only[mbi])) ok = false;  // keeps the slot's result, publishes at once
        // a seed produced by another pass of this launch
        if (ok && d.seed_pass >= 0)
            ok = wait_flags(m.lane == 0 ? &passes[d.seed_pass].out.done[mbi] : nullptr, epoch, st, code, P.wait_log2);
        PHASE_MARK(0);
        if (ok) load_cur(P, m, d.cur);
        PHASE_MARK(1);
        if (ok && range == 0) {
            // --search-range 0 is a real no-search mode (encoder_motion.cpp:72-85)
            m.wp = m.wh = 0;
            m.wx0 = m.wy0 = 0;
            publish_ctx(P, m);
            const uint64_t z = mb_sad(P, m, 0, 0, 1);
            if (m.lane == 0) {
                o.mvs[m.pos] = make_int2(0, 0);
                for (int k = 0; k < 4; ++k) o.bmv[m.pos * 4 + k] = make_int2(0, 0);
                o.use4[m.pos] = 0;
                o.intra[m.pos] = 0;
                o.screen[m.pos] = z;
                o.ratio[m.pos] = -1.0;
                o.dl[m.pos] = -1.0;  // the zero path returns before the seed's distant fields are copied
                o.dc[m.pos] = -1.0;
                o.dd[m.pos] = 0;
                o.chosen[m.pos] = z;
                o.temporal[m.pos] = z;
                o.flags[m.pos] = 0;
            }
            ok = false;
        }
        // ---- neighbour-independent work: staging, the seeded SAD shortlist, intra proxy ----
        Shortlist sl;
        sl.direct = 1;
        double dl = -1.0, dc = -1.0;
        uint8_t dd = 0;
        uint64_t intra_sad = 0;
        // Mixed-MV speculation: the 4MV block work for a guessed 1-MV vector runs before the
        // wait and is kept when the vector chosen after it matches (seeds from earlier launches)
        // Speculation: with the seed pass's neighbourhood standing in for this pass's, the
        // refinements (and for Mixed-MV every block's) run before the wait; after it each
        // result is kept where the real predictor equals the guessed one (seeds produced by
        // earlier launches only)
        const bool spec = seeded && d.seed_pass < 0;
        const bool spec4 = allow_4mv && spec;
        int2 one_g = make_int2(0, 0);
        IntRes learned{0, 0, UINT64_MAX};  // learned passes: the integer vector before refinement
        if (ok) {
            if (seeded) {
                int2 seed = __ldcg(&d.seed_mvs[m.pos]);
                const Bounds qb = bounds_qpel(range);
                seed.x = iclamp(seed.x, qb.xmin, qb.xmax);
                seed.y = iclamp(seed.y, qb.ymin, qb.ymax);
                load_window(P, m, d.ref, floor_div4(seed.x), floor_div4(seed.y), wc);
                publish_ctx(P, m);
                window_wait(m, st, code, P.wait_log2);
                PHASE_MARK(2);
                sl = refine_prepare_ool<kDR>(m.sm.ctx.off, m.x0, m.y0, 16, 16, seed, range, one_mode, UINT64_MAX, true);
                PHASE_MARK(3);
                dl = __ldcg(&d.seed_dl[m.pos]);
                dc = __ldcg(&d.seed_dc[m.pos]);
                dd = __ldcg(&d.seed_dd[m.pos]);
                if (spec) {
                    guess_neighbours(P, m, d);
                    int2* cur4g = m.sm.cur_bmv;
                    const Field fg{cur4g, m.sm.nb_bmv, m.sm.nb_intra, P.mbw, P.mbh, m.mx, m.my};
                    const PInfo pig = predictor_mixed_1mv(P, fg, m.mx, m.my);
                    shortlist_save(m, 0, sl, seed, 0, 0);
                    const RefineOut og = refine_select_ool<kDR>(m.sm.ctx.off, sl, m.x0, m.y0, 16, 16, one_mode, pig, true);
                    spec_result_save(m, 0, pig, og);
                    one_g = og.mv;
                    if (hidden_padding(P, m.x0, m.y0, 16, 16, one_g.x, one_g.y, one_mode, true)) one_g = make_int2(0, 0);
                    if (spec4) {
                        if (m.lane < 4) cur4g[m.lane] = one_g;
                        __syncwarp();
                        for (int k = 0; k < 4; ++k) {
                            const int bx = m.x0 + (k & 1) * 8, by = m.y0 + ((k >> 1) & 1) * 8;
                            const PInfo pi4g = predictor_4mv(P, fg, m.mx, m.my, k);
                            put_4mv_seeds(P, m, one_g, pi4g.pre, qb);
                            sad_batch(P, m, m.sm.batch, 11, bx, by, 8, 8, VC1CU_MV_QPEL, m.sm.batch_cost);
                            const SeedPick b10 = pick_4mv_seed(m, true);
                            const SeedPick bf = pick_4mv_seed(m, false);
                            const uint32_t rc = m.sm.ctx.off;
                            const Shortlist sk = refine_prepare_ool<kDR>(rc, bx, by, 8, 8, bf.v, range, VC1CU_MV_MIXED, bf.cost, true);
                            shortlist_save(m, k + 1, sk, bf.v, bf.cost, bf.slot);
                            const RefineOut rk = refine_select_ool<kDR>(rc, sk, bx, by, 8, 8, VC1CU_MV_MIXED, pi4g, true);
                            if (m.lane == 0) {
                                SpecBlk& sb = m.sm.spec_blk[k + 1];
                                sb.b10 = b10.v;
                                sb.b10_cost = b10.cost;
                                sb.b10_slot = b10.slot;
                                cur4g[k] = rk.mv;
                            }
                            spec_result_save(m, k + 1, pi4g, rk);
                        }
                    }
                    PHASE_MARK(12);
                }
            } else if constexpr ((KIND & kCoreLearned) != 0) {
                // the candidates' exact costs on the full-resolution picture, then a short descent
                // in a small window about the best (neighbour-independent, before the wait)
                const IntRes best = learned_candidates(P, m, d, range);
                load_window(P, m, d.ref, best.dx, best.dy, wc);
                publish_ctx(P, m);
                window_wait(m, st, code, P.wait_log2);
                learned = learned_descent(P, m, best, range, kLearnRw - 4);
                if (m.lane == 0 && d.fallback) d.fallback[m.pos] = learned_falls_back(P, m, o, learned.cost) ? 1 : 0;
                PHASE_MARK(2);
            } else {
                load_window(P, m, d.ref, 0, 0, wc);
                publish_ctx(P, m);
                PHASE_MARK(2);
            }
            if (allow_intra) intra_sad = intra_proxy(P, m);
            PHASE_MARK(4);
        }
        // ---- wavefront: left, top-left, top, top-right of the same pass ----
        // learned passes and no_wait passes read a field that is already complete: no wavefront
        constexpr bool kLearned = (KIND & kCoreLearned) != 0;
        const bool no_wait = kLearned || d.no_wait;
        if (ok && !no_wait) ok = wait_neighbours(P, o, m.mx, m.my, m.lane, epoch, st, code);
        window_wait(m, st, code, P.wait_log2);  // an unseeded pass's window copies (none pending otherwise)
        PHASE_MARK(5);
        if (ok) {
            if constexpr (kLearned) load_cand_neighbours(P, m, d);
            else load_neighbours(P, m, d.no_wait ? d.nb : o);
            int2* cur4 = m.sm.cur_bmv;
            if (m.lane < 4) cur4[m.lane] = make_int2(0, 0);
            __syncwarp();
            Field field{cur4, m.sm.nb_bmv, m.sm.nb_intra, P.mbw, P.mbh, m.mx, m.my};
            const PInfo rate_pi = predictor_mixed_1mv(P, field, m.mx, m.my);
            const uint64_t pixels = (uint64_t)m.aw * (uint64_t)m.ah;
            RefineOut one;
            bool distant = false;  // the integer vector came from a long-range search
            PHASE_MARK(6);
            if (seeded) {
                if (spec && pinfo_equal(rate_pi, m.sm.spec_blk[0].pi)) {
                    one = m.sm.spec_blk[0].res;
                } else {
                    if (spec) shortlist_restore(m, 0);
                    one = refine_select_ool<kDR>(m.sm.ctx.off, sl, m.x0, m.y0, 16, 16, one_mode, rate_pi, true);
                }
            } else if constexpr ((KIND & kCoreLearned) != 0) {
                if (pixels) dl = (double)learned.cost / (double)pixels;
                PHASE_MARK(7);
                one = refine_staged<kDR>(P, m, m.x0, m.y0, 16, 16, make_int2(learned.dx * 4, learned.dy * 4), range,
                                         one_mode, rate_pi, true, learned.cost);
            } else {
                const PInfo pi = predictor_info(P, m);
                const int gdx = __ldcg(&o.global[0]), gdy = __ldcg(&o.global[1]);
                auto local_search = [&]() {
                    return !kUmhOnly && P.me_algorithm == 1 ? diamond(P, m, pi, gdx, gdy, local_range)
                                                            : umh(P, m, pi, gdx, gdy, local_range, pixels);
                };
                // a distant candidate's MAE, kept when it is the least seen (record_distant, :176-183)
                auto record = [&](uint64_t s, int decision) {
                    if (!pixels || s >= UINT64_MAX / 8) return;
                    const double mae = (double)s / (double)pixels;
                    if (dc < 0.0 || mae < dc) {
                        dc = mae;
                        dd = (uint8_t)decision;
                    }
                };
                const bool long_range = !kUmhOnly && range > local_range;
                IntRes im{0, 0, UINT64_MAX};
                if (P.long_range_mode == 2) {
                    // legacy distant-first policy (:144-160)
                    bool short_circuit = false;
                    if (long_range) {
                        const IntRes pr = lr_propagated(P, m, d.no_wait ? d.nb : o, range);
                        if (match_good(m, pr.cost)) {
                            im = pr;
                            short_circuit = true;
                            distant = true;
                        }
                    }
                    if (!short_circuit) im = local_search();
                } else {
                    // local search first, then the propagated distant candidate (:161-196)
                    im = local_search();
                    const uint64_t local_sad = im.cost;
                    if (pixels) dl = (double)local_sad / (double)pixels;
                    const bool skip = P.long_range_mode == 1 && match_good(m, im.cost);
                    if (long_range && !skip) {
                        const IntRes pr = lr_propagated(P, m, d.no_wait ? d.nb : o, range);
                        const int decision = distant_decision(P, m, pr.cost, local_sad);
                        record(pr.cost, decision);
                        const bool less = pr.cost != im.cost ? pr.cost < im.cost
                                        : (iabs(pr.dx) + iabs(pr.dy) != iabs(im.dx) + iabs(im.dy)
                                               ? iabs(pr.dx) + iabs(pr.dy) < iabs(im.dx) + iabs(im.dy)
                                               : (pr.dy != im.dy ? pr.dy < im.dy : pr.dx < im.dx));
                        if (less && decision >= 2) {
                            im = pr;
                            distant = true;
                        }
                    }
                }
                if (long_range && !match_good(m, im.cost)) {
                    // content-signature search (:201-225)
                    uint64_t ext_sad = UINT64_MAX;
                    int ext_decision = 0;
                    const IntRes ext = lr_extended(P, m, d, range, im, ext_sad, ext_decision);
                    if (P.long_range_mode != 2) record(ext_sad, ext_decision);
                    if (ext.dx != im.dx || ext.dy != im.dy) {
                        im = ext;
                        distant = true;
                    }
                }
                PHASE_MARK(7);
                one = refine_staged<kDR>(P, m, m.x0, m.y0, 16, 16, make_int2(im.dx * 4, im.dy * 4), range, one_mode, rate_pi,
                                    true, im.cost);
            }
            PHASE_MARK(8);
            if (hidden_padding(P, m.x0, m.y0, 16, 16, one.mv.x, one.mv.y, one_mode, true)) {
                if (m.lane == 0) m.sm.batch[31] = make_int2(0, 0);
                __syncwarp();
                sad_batch(P, m, m.sm.batch + 31, 1, m.x0, m.y0, 16, 16, one_mode, m.sm.batch_cost + 31);
                one.mv = make_int2(0, 0);
                one.screen_sad = m.sm.batch_cost[31];
            }
            const uint64_t one_sad = one.screen_sad;
            int2 out4[4] = {one.mv, one.mv, one.mv, one.mv};
            int2 out_mv = one.mv;
            uint8_t use4 = 0, intra = 0;
            bool chose4 = false;
            uint64_t chosen = one_sad, temporal_screen = one_sad;
            const double lambda = d.lambda;
            if (allow_4mv) {
                // progressive Mixed-MV (:250-374, me_quality != RD)
                if (m.lane < 4) cur4[m.lane] = one.mv;
                __syncwarp();
                uint64_t four_sad = 0, four_screen = 0, extra_bits = 1;
                const Bounds qb = bounds_qpel(range);
                const bool hit = spec4 && one.mv.x == one_g.x && one.mv.y == one_g.y;
                for (int k = 0; k < 4; ++k) {
                    const PInfo pi4 = predictor_4mv(P, field, m.mx, m.my, k);
                    const int bx = m.x0 + (k & 1) * 8, by = m.y0 + ((k >> 1) & 1) * 8;
                    RefineOut r;
                    bool have = false;
                    int2 best_seed;
                    uint64_t seed_cost;
                    const SpecBlk& sb = m.sm.spec_blk[k + 1];
                    if (hit && pinfo_equal(pi4, sb.pi)) {
                        // same seeds, same shortlist, same predictor: the parked result
                        r = sb.res;
                        have = true;
                    } else if (hit) {
                        // the parked seed search covered every slot but the predictor's
                        put_4mv_seeds(P, m, one.mv, pi4.pre, qb);
                        const int2 v2 = m.sm.batch[2];
                        sad_batch(P, m, m.sm.batch + 2, 1, bx, by, 8, 8, VC1CU_MV_QPEL, m.sm.batch_cost + 2);
                        const uint64_t c2 = m.sm.batch_cost[2];
                        const SeedPick b{sb.b10, sb.b10_cost, sb.b10_slot};
                        if (seed_before(v2, c2, 2, b)) {
                            best_seed = v2;
                            seed_cost = c2;
                        } else if (sb.seed_slot != 2) {
                            // the parked shortlist was refined from this same seed
                            const Shortlist sk = shortlist_restore(m, k + 1);
                            r = refine_select_ool<kDR>(m.sm.ctx.off, sk, bx, by, 8, 8, VC1CU_MV_MIXED, pi4, true);
                            have = true;
                        } else {
                            best_seed = b.v;
                            seed_cost = b.cost;
                        }
                    } else {
                        put_4mv_seeds(P, m, one.mv, pi4.pre, qb);
                        sad_batch(P, m, m.sm.batch, 11, bx, by, 8, 8, VC1CU_MV_QPEL, m.sm.batch_cost);
                        const SeedPick b = pick_4mv_seed(m, false);
                        best_seed = b.v;
                        seed_cost = b.cost;
                    }
                    PHASE_MARK(9);
                    if (!have) r = refine_staged<kDR>(P, m, bx, by, 8, 8, best_seed, range, VC1CU_MV_MIXED, pi4, true, seed_cost);
                    PHASE_MARK(10);
                    four_screen += r.screen_sad;
                    if (m.lane == 0) cur4[k] = r.mv;
                    __syncwarp();
                    four_sad += r.screen_sad;
                    int2 actual = pi4.pre;
                    if (pi4.hybrid) {
                        const int da = modular_mv_distance(P, r.mv, pi4.a), dcc = modular_mv_distance(P, r.mv, pi4.c);
                        actual = (da <= dcc) ? pi4.a : pi4.c;
                        ++extra_bits;
                    }
                    if (!(r.mv.x == actual.x && r.mv.y == actual.y)) extra_bits += mv_rate_bits(P, r.mv, actual, VC1CU_MV_MIXED, false);
                }
                int2 four[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) four[k] = cur4[k];
                const int cmx = median4(four[0].x, four[1].x, four[2].x, four[3].x);
                const int cmy = median4(four[0].y, four[1].y, four[2].y, four[3].y);
                const bool four_chroma_safe = !hidden_chroma(P, m.x0, m.y0, 16, 16, cmx, cmy);
                bool choose4 = false;
                if (four_chroma_safe)
                    choose4 = four_sad + (uint64_t)llround(__dmul_rn(lambda, (double)extra_bits)) + 8 <
                              (uint64_t)llround(__dmul_rn((double)one_sad, 0.985));
                chose4 = choose4;
                if (choose4) {
                    for (int k = 0; k < 4; ++k) out4[k] = four[k];
                    use4 = 1;
                    out_mv = four[0];
                    chosen = four_sad;
                    temporal_screen = four_screen;
                } else {
                    temporal_screen = one_sad;
                }
            }
            const uint64_t temporal = chosen;
            double ratio = -1.0;
            if (allow_intra) {
                // P-intra decision (:396-414)
                const uint64_t intra_rate = (uint64_t)llround(__dmul_rn(lambda, 72.0));
                ratio = temporal_screen > 0 ? __ddiv_rn((double)(intra_sad + intra_rate), (double)temporal_screen)
                                            : __longlong_as_double(0x7ff0000000000000ll);
                if (intra_sad + intra_rate < (uint64_t)llround(__dmul_rn((double)temporal_screen, P.inter_intra_threshold))) {
                    intra = 1;
                    use4 = 0;
                    out_mv = make_int2(0, 0);
                    for (int k = 0; k < 4; ++k) out4[k] = make_int2(0, 0);
                    chosen = intra_sad;
                }
            }
            bool moved = false, frac = false;
            for (int k = 0; k < 4; ++k) {
                moved |= out4[k].x != 0 || out4[k].y != 0;
                frac |= (out4[k].x % 8) != 0 || (out4[k].y % 8) != 0;
            }
            if (m.lane == 0) {
                o.mvs[m.pos] = out_mv;
                for (int k = 0; k < 4; ++k) o.bmv[m.pos * 4 + k] = out4[k];
                o.use4[m.pos] = use4;
                o.intra[m.pos] = intra;
                o.screen[m.pos] = temporal_screen;
                o.ratio[m.pos] = ratio;
                o.dl[m.pos] = dl;
                o.dc[m.pos] = dc;
                o.dd[m.pos] = dd;
                o.chosen[m.pos] = chosen;
                o.temporal[m.pos] = temporal;
                o.flags[m.pos] = (uint8_t)((moved ? 1 : 0) | (frac ? 2 : 0) | (distant ? 4 : 0) | (chose4 ? 8 : 0));
            }
        }
        __syncwarp();
        if (m.lane == 0 && code != P.withhold) {
            __threadfence();
            st_release(&o.done[m.pos], epoch);
        }
        __syncwarp();
        PHASE_MARK(11);
    }
    // a window copy still in flight after a timed-out wait lands before the block's shared
    // memory is released (bounded again)
    if (m.tma_pending) tma_wait(m, nullptr, 0, 22);
}

// mean_region (:1578-1590) of one 8x8 region, by one thread.
__device__ uint32_t mean8(const uint8_t* plane, int pitch, int pw, int ph, int x0, int y0) {
    uint32_t sum = 0, n = 0;
    for (int y = 0; y < 8 && y0 + y < ph; ++y) {
        if (y0 + y < 0) continue;
        for (int x = 0; x < 8 && x0 + x < pw; ++x) {
            if (x0 + x < 0) continue;
            sum += __ldg(plane + (size_t)(y0 + y) * pitch + x0 + x);
            ++n;
        }
    }
    return n ? (sum + n / 2) / n : 128;
}

// build_long_range_index (:1616-1625): the signature of every 8-pixel lattice cell of a
// reference picture, one thread per cell, raster order.
__global__ void lr_index_kernel(DevFrame ref, int W, int H, int nx, int ny, uint64_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    const int x0 = (i % nx) * 8, y0 = (i / nx) * 8;
    uint64_t s = (uint64_t)mean8(ref.y, ref.pitch_y, W, H, x0, y0);
    s |= (uint64_t)mean8(ref.y, ref.pitch_y, W, H, x0 + 8, y0) << 8;
    s |= (uint64_t)mean8(ref.y, ref.pitch_y, W, H, x0, y0 + 8) << 16;
    s |= (uint64_t)mean8(ref.y, ref.pitch_y, W, H, x0 + 8, y0 + 8) << 24;
    s |= (uint64_t)mean8(ref.u, ref.pitch_c, W / 2, H / 2, x0 / 2, y0 / 2) << 32;
    s |= (uint64_t)mean8(ref.v, ref.pitch_c, W / 2, H / 2, x0 / 2, y0 / 2) << 40;
    out[i] = s;
}

cudaError_t launch_lr_index(const DevFrame& ref, int W, int H, uint64_t* out, cudaStream_t s) {
    const int nx = (W + 7) / 8, ny = (H + 7) / 8;
    lr_index_kernel<<<(nx * ny + 255) / 256, 256, 0, s>>>(ref, W, H, nx, ny, out);
    return cudaGetLastError();
}

// Host-side handles of the instantiations (attributes, occupancy, launch): the flag sets the
// host selects.
#define VC1CU_CORE_KINDS(X)                                                                      \
    X(kCoreAny) X(kCoreAny | kCoreWide) X(kCoreSeededOnly) X(kCoreSeededOnly | kCoreNoMixed)     \
    X(kCoreUnseededOnly) X(kCoreUnseededOnly | kCoreWide) X(kCoreUnseededOnly | kCoreUmhLocal)   \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreWide) X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed) \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed | kCoreWide)                                \
    X(kCoreSeededOnly | kCoreDefaultRefine) X(kCoreSeededOnly | kCoreNoMixed | kCoreDefaultRefine)   \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreDefaultRefine)                                      \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreWide | kCoreDefaultRefine)                          \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed | kCoreDefaultRefine)                       \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed | kCoreWide | kCoreDefaultRefine)                 \
    X(kCoreSeededOnly | kCoreDefaultRefine | kCoreNoIntra)                                              \
    X(kCoreSeededOnly | kCoreNoMixed | kCoreDefaultRefine | kCoreNoIntra)                               \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreDefaultRefine | kCoreNoIntra)                            \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreWide | kCoreDefaultRefine | kCoreNoIntra)                \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed | kCoreDefaultRefine | kCoreNoIntra)             \
    X(kCoreUnseededOnly | kCoreUmhLocal | kCoreNoMixed | kCoreWide | kCoreDefaultRefine | kCoreNoIntra)    \
    X(kCoreUnseededOnly | kCoreLearned | kCoreNoMixed | kCoreNoIntra)                                   \
    X(kCoreUnseededOnly | kCoreLearned | kCoreNoMixed | kCoreNoIntra | kCoreDefaultRefine)                 \
    X(kCoreMulti) X(kCoreMulti | kCoreWide)

const void* core_kernel(int kind) {
    switch (kind) {
#define VC1CU_KERNEL_CASE(k) \
    case (k): return reinterpret_cast<const void*>(&core_pass_kernel<(k)>);
        VC1CU_CORE_KINDS(VC1CU_KERNEL_CASE)
#undef VC1CU_KERNEL_CASE
        default: return nullptr;
    }
}

// The fallback macroblocks of a learned pass, from the fallback pass's slot into the learned one.
__global__ void learned_merge_kernel(DevResult dst, DevResult src, const uint8_t* only, int mbs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mbs || !only[i]) return;
    dst.mvs[i] = src.mvs[i];
    for (int k = 0; k < 4; ++k) dst.bmv[4 * i + k] = src.bmv[4 * i + k];
    dst.use4[i] = src.use4[i];
    dst.intra[i] = src.intra[i];
    dst.dd[i] = src.dd[i];
    dst.flags[i] = src.flags[i];
    dst.screen[i] = src.screen[i];
    dst.chosen[i] = src.chosen[i];
    dst.temporal[i] = src.temporal[i];
    dst.ratio[i] = src.ratio[i];
    dst.dl[i] = src.dl[i];
    dst.dc[i] = src.dc[i];
}

// The 4x4 clamped neighbourhood of an integer origin (columns x-1..x+2, rows y-1..y+2), which
// holds every tap any phase of predict_row<1> reads there.
struct NbrSampler {
    int v[4][4];
    int x0, y0;
    __device__ __forceinline__ int operator()(int x, int y) const { return v[y - y0][x - x0]; }
};

// The sub-pel prediction planes of a reference picture: plane (vm * 4 + hm) holds, at (y + border)
// * opitch + x + border, the prediction of phase (hm, vm) whose integer origin is (x, y) (predict_row,
// clamped sampling), for the phases in phase_mask. One thread per origin loads its neighbourhood
// once and evaluates every phase from it.
template <bool BILINEAR>
__global__ void subpel_plane_kernel(const uint8_t* ref, int pitch, int W, int H, int rnd, uint32_t phase_mask,
                                    uint8_t* out, int opitch, int border, long long stride) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= W + 2 * border) return;
    const int x = px - border, y = py - border;
    NbrSampler n;
    n.x0 = x - 1;
    n.y0 = y - 1;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint8_t* row = ref + (size_t)iclamp(y - 1 + r, 0, H - 1) * pitch;
#pragma unroll
        for (int k = 0; k < 4; ++k) n.v[r][k] = __ldg(row + iclamp(x - 1 + k, 0, W - 1));
    }
    uint8_t* o = out + (long long)py * opitch + px;
#pragma unroll
    for (int ph = 1; ph < 16; ++ph) {
        if (!((phase_mask >> ph) & 1)) continue;
        int v[1];
        predict_row<1>(n, BILINEAR, rnd, ph & 3, ph >> 2, x, y, v);
        o[ph * stride] = (uint8_t)v[0];
    }
}

cudaError_t launch_subpel_planes(const uint8_t* ref, int pitch, int W, int H, int rnd, int bilinear, uint32_t phase_mask,
                                 uint8_t* out, int opitch, int border, long long stride, cudaStream_t s) {
    const dim3 grid((unsigned)((W + 2 * border + 127) / 128), (unsigned)(H + 2 * border));
    if (bilinear) subpel_plane_kernel<true><<<grid, 128, 0, s>>>(ref, pitch, W, H, rnd, phase_mask, out, opitch, border, stride);
    else subpel_plane_kernel<false><<<grid, 128, 0, s>>>(ref, pitch, W, H, rnd, phase_mask, out, opitch, border, stride);
    return cudaGetLastError();
}

cudaError_t launch_learned_merge(const DevResult& dst, const DevResult& src, const uint8_t* only, int mbs,
                                 cudaStream_t s) {
    learned_merge_kernel<<<(mbs + 255) / 256, 256, 0, s>>>(dst, src, only, mbs);
    return cudaGetLastError();
}

cudaError_t launch_core(int kind, int grid, int block, size_t smem, cudaStream_t s, const DevParams& P,
                        const PassDesc* passes, int npass, const uint32_t* items, unsigned nitems, const WinCfg& wc,
                        uint32_t epoch, LaunchStatus* st) {
    switch (kind) {
#define VC1CU_LAUNCH_CASE(k)                                                                              \
    case (k):                                                                                          \
        core_pass_kernel<(k)><<<grid, block, smem, s>>>(P, passes, npass, items, nitems, wc, epoch, st); \
        break;
        VC1CU_CORE_KINDS(VC1CU_LAUNCH_CASE)
#undef VC1CU_LAUNCH_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Picture totals of each pass (encoder_motion.cpp:428-441): integer sums, then the
// reference's double expressions. One block per pass.
__global__ void totals_kernel(const __grid_constant__ DevParams P0, const PassDesc* passes, int npass) {
    const PassDesc& d = passes[blockIdx.x];
    const DevParams& P = d.geom;  // every pass carries its own geometry
    (void)P0;
    const DevResult& o = d.out;
    const int mbs = P.mbw * P.mbh;
    uint64_t ts = 0, rs = 0, mv = 0, fr = 0, f4 = 0, in = 0, px = 0;
    for (int i = threadIdx.x; i < mbs; i += blockDim.x) {
        ts += o.chosen[i];
        rs += o.temporal[i];
        mv += o.flags[i] & 1;
        fr += (o.flags[i] >> 1) & 1;
        f4 += (o.flags[i] >> 3) & 1;  // 4MV chosen, also where P-intra then replaced it (:370)
        in += o.intra[i];
        const int mx = i % P.mbw, my = i / P.mbw;
        px += (uint64_t)imax(0, imin(16, P.W - mx * 16)) * (uint64_t)imax(0, imin(16, P.H - my * 16));
    }
    __shared__ unsigned long long red[7][32];
    uint64_t v[7] = {ts, rs, mv, fr, f4, in, px};
    for (int k = 0; k < 7; ++k) {
        uint64_t x = warp_sum_u64(v[k]);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t s[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 7; ++k)
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s[k] += red[k][w];
        const uint64_t total_pixels = s[6];
        const double local_mad = total_pixels ? __ddiv_rn((double)s[0], (double)total_pixels) : 0.0;
        double global_mad;
        if (d.seeded) global_mad = local_mad;
        else global_mad = (P.W > 0 && P.H > 0) ? __ddiv_rn((double)*o.gsad, (double)((uint64_t)P.W * P.H)) : 0.0;
        const double rate_local = total_pixels ? __ddiv_rn((double)s[1], (double)total_pixels) : 0.0;
        if (P.range == 0) {
            o.totals[0] = local_mad;
            o.totals[1] = local_mad;
        } else {
            o.totals[0] = local_mad < global_mad ? local_mad : global_mad;
            o.totals[1] = rate_local < global_mad ? rate_local : global_mad;
        }
        o.itotals[0] = P.range == 0 ? 0 : s[0];
        o.itotals[1] = s[2];
        o.itotals[2] = s[3];
        o.itotals[3] = s[4];
        o.itotals[4] = s[5];
    }
}

}  // namespace vc1cu

namespace vc1cu {
// The index-checked build's record (count, first site << 40 | index); -1 in other builds.
int index_fault_record(unsigned int* count, unsigned long long* first, int reset) {
#ifdef VC1CU_INDEX_CHECK
    unsigned int n = 0;
    unsigned long long f = 0;
    if (cudaMemcpyFromSymbol(&n, g_index_faults, sizeof n) != cudaSuccess) return 1;
    if (cudaMemcpyFromSymbol(&f, g_index_first, sizeof f) != cudaSuccess) return 1;
    if (count) *count = n;
    if (first) *first = f;
    if (reset) {
        const unsigned int z = 0;
        const unsigned long long zf = 0;
        if (cudaMemcpyToSymbol(g_index_faults, &z, sizeof z) != cudaSuccess) return 1;
        if (cudaMemcpyToSymbol(g_index_first, &zf, sizeof zf) != cudaSuccess) return 1;
    }
    return 0;
#else
    (void)count;
    (void)first;
    (void)reset;
    return -1;
#endif
}
}  // namespace vc1cu

#ifdef VC1CU_PHASE_CLOCKS
// Profiling build only: copies (and with reset != 0 clears) the phase accumulators.
extern "C" int vc1cu_phase_clocks(unsigned long long* clk, unsigned long long* cnt, int reset) {
    if (cudaMemcpyFromSymbol(clk, vc1cu::g_phase_clk, sizeof vc1cu::g_phase_clk) != cudaSuccess) return -1;
    if (cudaMemcpyFromSymbol(cnt, vc1cu::g_phase_cnt, sizeof vc1cu::g_phase_cnt) != cudaSuccess) return -1;
    if (reset) {
        static const unsigned long long z[64] = {};
        if (cudaMemcpyToSymbol(vc1cu::g_phase_clk, z, sizeof z) != cudaSuccess) return -1;
        if (cudaMemcpyToSymbol(vc1cu::g_phase_cnt, z, sizeof z) != cudaSuccess) return -1;
    }
    return 0;
}
#endif
