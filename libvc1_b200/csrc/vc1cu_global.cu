// vc1cu_global.cu - whole-frame translation search, Vc1Encoder::global_motion_search and
// global_motion_search_extended (encoder_motion.cpp:2025-2141), for many pictures at once.
//
// Each stage of the reference is a fixed candidate list (given the previous stage) scored
// with frame_sad (encoder_motion.cpp:1499-1576) and then folded by a sequential rule
// (top-8 insertion with truncation, first-visit tie breaks). Here every stage is one
// parallel scoring launch (one block per candidate x row slab, partial sums combined with
// integer atomics, so the order of summation does not matter) followed by a one-thread
// replay of the reference's sequential fold over the precomputed costs.
#include <cuda_runtime.h>

#include <cstdio>

#include "vc1cu_core.cuh"

namespace vc1cu {

constexpr int kGMaxCand = 512;  // largest stage: range 31 refine, 8 x 7 x 7 = 392

struct GCand {
    int dx, dy, stride;
};

struct GState {
    // inputs
    DevFrame cur, ref;
    int range;                 // min(local range, 32)
    int* out_global;           // [dx, dy]
    unsigned long long* out_sad;
    // stage scratch
    int n;                     // candidates of the current stage
    GCand cand[kGMaxCand];
    unsigned long long cost[kGMaxCand];
    // fold state
    int top_n;
    unsigned long long top_cost[9];
    int top_dx[9], top_dy[9];
    int best_dx, best_dy;
    unsigned long long best_cost;
    int phase;
};

__device__ __forceinline__ bool gless(unsigned long long ca, int ax, int ay, unsigned long long cb, int bx, int by) {
    if (ca != cb) return ca < cb;
    const int am = iabs(ax) + iabs(ay), bm = iabs(bx) + iabs(by);
    if (am != bm) return am < bm;
    if (ay != by) return ay < by;
    return ax < bx;
}

// frame_sad of every candidate of every state: grid (slab, candidate, state)
__global__ void gsad_kernel(GState* states, int W, int H, int rows_per_slab) {
    GState& s = states[blockIdx.z];
    const int ci = blockIdx.y;
    if (ci >= s.n) return;
    const GCand c = s.cand[ci];
    const int st = c.stride;
    const int nrows = (H + st - 1) / st;
    const int r0 = blockIdx.x * rows_per_slab;
    if (r0 >= nrows) return;
    const int r1 = imin(nrows, r0 + rows_per_slab);
    const int ncols = (W + st - 1) / st;
    uint64_t acc = 0;
    for (int r = r0; r < r1; ++r) {
        const int y = r * st;
        const int sy = iclamp(y + c.dy, 0, H - 1);
        const uint8_t* cp = s.cur.y + (size_t)y * s.cur.pitch_y;
        const uint8_t* rp = s.ref.y + (size_t)sy * s.ref.pitch_y;
        for (int k = threadIdx.x; k < ncols; k += blockDim.x) {
            const int x = k * st;
            const int sx = iclamp(x + c.dx, 0, W - 1);
            acc += (uint64_t)iabs((int)__ldg(cp + x) - (int)__ldg(rp + sx));
        }
    }
    acc = warp_sum_u64(acc);
    __shared__ unsigned long long red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(&s.cost[ci], t);
    }
}

__device__ unsigned long long scaled(const GState& s, int i) {
    const int st = s.cand[i].stride;
    return st > 1 ? s.cost[i] * (unsigned long long)(st * st) : s.cost[i];
}

// sort-and-truncate insertion of global_motion_search (:2086-2098): multiset top-8
__device__ void push_plain(GState& s, unsigned long long c, int dx, int dy) {
    int at = s.top_n;
    while (at > 0 && gless(c, dx, dy, s.top_cost[at - 1], s.top_dx[at - 1], s.top_dy[at - 1])) --at;
    for (int j = s.top_n; j > at; --j) {
        s.top_cost[j] = s.top_cost[j - 1];
        s.top_dx[j] = s.top_dx[j - 1];
        s.top_dy[j] = s.top_dy[j - 1];
    }
    s.top_cost[at] = c;
    s.top_dx[at] = dx;
    s.top_dy[at] = dy;
    if (++s.top_n > 8) s.top_n = 8;
}

// `consider` of global_motion_search_extended (:2034-2039): keep-min per vector, sorted, 8
__device__ void push_ext(GState& s, unsigned long long c, int dx, int dy) {
    for (int i = 0; i < s.top_n; ++i)
        if (s.top_dx[i] == dx && s.top_dy[i] == dy) {
            if (c < s.top_cost[i]) {
                s.top_cost[i] = c;
                // re-sort (the reference sorts only on insertion; a lowered cost stays in place
                // until the next insertion sorts the list, which yields the same order)
            }
            return;
        }
    // insertion then sort then truncate; sorting an almost-sorted list by insertion
    s.top_cost[s.top_n] = c;
    s.top_dx[s.top_n] = dx;
    s.top_dy[s.top_n] = dy;
    ++s.top_n;
    for (int i = 1; i < s.top_n; ++i) {
        const unsigned long long vc = s.top_cost[i];
        const int vx = s.top_dx[i], vy = s.top_dy[i];
        int j = i - 1;
        while (j >= 0 && gless(vc, vx, vy, s.top_cost[j], s.top_dx[j], s.top_dy[j])) {
            s.top_cost[j + 1] = s.top_cost[j];
            s.top_dx[j + 1] = s.top_dx[j];
            s.top_dy[j + 1] = s.top_dy[j];
            --j;
        }
        s.top_cost[j + 1] = vc;
        s.top_dx[j + 1] = vx;
        s.top_dy[j + 1] = vy;
    }
    if (s.top_n > 8) s.top_n = 8;
}

__device__ void add_cand(GState& s, int dx, int dy, int stride) {
    s.cand[s.n].dx = dx;
    s.cand[s.n].dy = dy;
    s.cand[s.n].stride = stride;
    s.cost[s.n] = 0;
    ++s.n;
}

// One thread per state: fold the costs of the finished stage and plan the next one.
// phase 0: plan the first stage. Returns via s.phase = -1 when the result is written.
__global__ void gplan_kernel(GState* states, int nstates) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nstates) return;
    GState& s = states[i];
    const int R = s.range;
    if (s.phase < 0) return;
    if (R <= 0) {
        // range 0: frame_sad(0,0,1) (:2082-2085)
        if (s.phase == 0) {
            s.n = 0;
            add_cand(s, 0, 0, 1);
            s.phase = 100;
        } else {
            s.out_global[0] = 0;
            s.out_global[1] = 0;
            *s.out_sad = s.cost[0];
            s.phase = -1;
            s.n = 0;
        }
        return;
    }
    if (R <= 31) {
        const int cs = R >= 4 ? 4 : (R >= 2 ? 2 : 1);
        if (s.phase == 0) {
            // coarse grid + zero + edges at stride 4 (:2110-2124)
            s.n = 0;
            for (int dy = -R; dy <= R; dy += cs)
                for (int dx = -R; dx <= R; dx += cs) add_cand(s, dx, dy, 4);
            add_cand(s, 0, 0, 4);
            for (int d = -R; d <= R; d += cs) {
                add_cand(s, R, d, 4);
                add_cand(s, d, R, 4);
            }
            s.phase = 1;
            return;
        }
        if (s.phase == 1) {
            s.top_n = 0;
            for (int k = 0; k < s.n; ++k) push_plain(s, scaled(s, k), s.cand[k].dx, s.cand[k].dy);
            // refinement visit list around each top entry at stride 2 (:2129-2140)
            bool seen[63 * 63];
            for (int k = 0; k < 63 * 63; ++k) seen[k] = false;
            const int tn = s.top_n;
            int tdx[8], tdy[8];
            for (int k = 0; k < tn; ++k) { tdx[k] = s.top_dx[k]; tdy[k] = s.top_dy[k]; }
            s.n = 0;
            for (int k = 0; k < tn; ++k)
                for (int dy = imax(-R, tdy[k] - cs + 1); dy <= imin(R, tdy[k] + cs - 1); ++dy)
                    for (int dx = imax(-R, tdx[k] - cs + 1); dx <= imin(R, tdx[k] + cs - 1); ++dx) {
                        const int key = (dy + 31) * 63 + (dx + 31);
                        if (seen[key]) continue;
                        seen[key] = true;
                        add_cand(s, dx, dy, 2);
                    }
            s.phase = 2;
            return;
        }
        if (s.phase == 2) {
            unsigned long long bc = ~0ull;
            int bx = 0, by = 0;
            for (int k = 0; k < s.n; ++k) {
                const unsigned long long c = scaled(s, k);
                const int dx = s.cand[k].dx, dy = s.cand[k].dy;
                const int cm = iabs(dx) + iabs(dy), bm = iabs(bx) + iabs(by);
                if (c < bc || (c == bc && cm < bm)) { bc = c; bx = dx; by = dy; }
            }
            s.best_dx = bx;
            s.best_dy = by;
            s.n = 0;
            add_cand(s, bx, by, 1);
            s.phase = 3;
            return;
        }
        s.out_global[0] = s.best_dx;
        s.out_global[1] = s.best_dy;
        *s.out_sad = s.cost[0];
        s.phase = -1;
        s.n = 0;
        return;
    }
    // extended search (range 32 after the min(range, 32) clamp), :2025-2074
    const int step = R >= 160 ? 16 : 8;
    if (s.phase == 0) {
        s.n = 0;
        add_cand(s, 0, 0, 16);
        for (int d = step; d <= R; d += step) {
            add_cand(s, iclamp(-d, -R, R), 0, 16);
            add_cand(s, iclamp(d, -R, R), 0, 16);
            add_cand(s, 0, iclamp(-d, -R, R), 16);
            add_cand(s, 0, iclamp(d, -R, R), 16);
        }
        for (int r = step; r <= R; r += step) {
            const int h = (r + 1) / 2;
            const int xs[8] = {-r, -r, r, r, -h, h, -h, h}, ys[8] = {-h, h, -h, h, -r, -r, r, r};
            for (int k = 0; k < 8; ++k) add_cand(s, iclamp(xs[k], -R, R), iclamp(ys[k], -R, R), 16);
        }
        s.top_n = 0;
        s.phase = 1;
        return;
    }
    if (s.phase == 1) {
        for (int k = 0; k < s.n; ++k) push_ext(s, scaled(s, k), s.cand[k].dx, s.cand[k].dy);
        const int nc = imin(4, s.top_n);
        int cx[4], cy[4];
        for (int k = 0; k < nc; ++k) { cx[k] = s.top_dx[k]; cy[k] = s.top_dy[k]; }
        s.n = 0;
        for (int k = 0; k < nc; ++k)
            for (int oy = -step; oy <= step; oy += 4)
                for (int ox = -step; ox <= step; ox += 4)
                    add_cand(s, iclamp(cx[k] + ox, -R, R), iclamp(cy[k] + oy, -R, R), 8);
        s.phase = 2;
        return;
    }
    if (s.phase == 2) {
        for (int k = 0; k < s.n; ++k) push_ext(s, scaled(s, k), s.cand[k].dx, s.cand[k].dy);
        if (s.top_n == 0) {  // (:2059) unreachable with a non-empty coarse stage
            s.n = 0;
            add_cand(s, 0, 0, 8);
            s.phase = 20;
            return;
        }
        const int mdx = s.top_dx[0], mdy = s.top_dy[0];
        s.n = 0;
        for (int oy = -4; oy <= 4; ++oy)
            for (int ox = -4; ox <= 4; ++ox) add_cand(s, iclamp(mdx + ox, -R, R), iclamp(mdy + oy, -R, R), 4);
        s.phase = 3;
        return;
    }
    if (s.phase == 20) {
        push_ext(s, scaled(s, 0), 0, 0);
        const int mdx = s.top_dx[0], mdy = s.top_dy[0];
        s.n = 0;
        for (int oy = -4; oy <= 4; ++oy)
            for (int ox = -4; ox <= 4; ++ox) add_cand(s, iclamp(mdx + ox, -R, R), iclamp(mdy + oy, -R, R), 4);
        s.phase = 3;
        return;
    }
    if (s.phase == 3) {
        for (int k = 0; k < s.n; ++k) push_ext(s, scaled(s, k), s.cand[k].dx, s.cand[k].dy);
        const int fdx = s.top_dx[0], fdy = s.top_dy[0];
        s.n = 0;
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) add_cand(s, iclamp(fdx + ox, -R, R), iclamp(fdy + oy, -R, R), 1);
        s.phase = 4;
        return;
    }
    // phase 4: full 3x3, min by the total order
    unsigned long long bc = ~0ull;
    int bx = 0, by = 0;
    for (int k = 0; k < s.n; ++k) {
        const unsigned long long c = s.cost[k];
        if (gless(c, s.cand[k].dx, s.cand[k].dy, bc, bx, by)) { bc = c; bx = s.cand[k].dx; by = s.cand[k].dy; }
    }
    s.out_global[0] = bx;
    s.out_global[1] = by;
    *s.out_sad = bc;
    s.phase = -1;
    s.n = 0;
}

size_t gstate_bytes() { return sizeof(GState); }

// Host driver: runs the staged search for n states already initialised in device memory
// (cur, ref, range, outputs, phase = 0). Every stage is one scoring launch sized to the
// stage's largest candidate list and sampling stride, bracketed by plan/fold launches.
// Passes that share one search take its result: one thread per copy (dx, dy and the SAD).
__global__ void global_fanout_kernel(const GlobalCopy* copies, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const GlobalCopy c = copies[i];
    c.dst_global[0] = c.src_global[0];
    c.dst_global[1] = c.src_global[1];
    *c.dst_sad = *c.src_sad;
}

cudaError_t launch_global_fanout(const GlobalCopy* d_copies, int n, cudaStream_t s) {
    if (n > 0) global_fanout_kernel<<<(n + 127) / 128, 128, 0, s>>>(d_copies, n);
    return cudaGetLastError();
}

int run_global_search(GState* d_states, int n, int R, int W, int H, cudaStream_t stream) {
    struct Stage { int maxc, stride; };
    Stage st[4];
    int ns = 0;
    if (R <= 0) {
        st[ns++] = {1, 1};
    } else if (R <= 31) {
        const int cs = R >= 4 ? 4 : (R >= 2 ? 2 : 1);
        const int L = (2 * R) / cs + 1;
        st[ns++] = {L * L + 1 + 2 * L, 4};
        st[ns++] = {imin(kGMaxCand, 8 * (2 * cs - 1) * (2 * cs - 1)), 2};
        st[ns++] = {1, 1};
    } else {
        const int step = R >= 160 ? 16 : 8;
        const int k = R / step;
        const int g = (2 * step) / 4 + 1;
        st[ns++] = {1 + 4 * k + 8 * k, 16};
        st[ns++] = {4 * g * g, 8};
        st[ns++] = {81, 4};
        st[ns++] = {9, 1};
    }
    const int rows_per_slab = 64;
    gplan_kernel<<<(n + 63) / 64, 64, 0, stream>>>(d_states, n);
    for (int i = 0; i < ns; ++i) {
        const int rows = (H + st[i].stride - 1) / st[i].stride;
        dim3 grid((rows + rows_per_slab - 1) / rows_per_slab, st[i].maxc, n);
        gsad_kernel<<<grid, 256, 0, stream>>>(d_states, W, H, rows_per_slab);
        gplan_kernel<<<(n + 63) / 64, 64, 0, stream>>>(d_states, n);
    }
    return 1 + 2 * ns;
}

void init_gstate(GState* h, const DevFrame& cur, const DevFrame& ref, int range, int* out_global,
                 unsigned long long* out_sad) {
    h->cur = cur;
    h->ref = ref;
    h->range = range;
    h->out_global = out_global;
    h->out_sad = out_sad;
    h->n = 0;
    h->top_n = 0;
    h->phase = 0;
}


// ---- allocation-free form (vc1cu_global_motion_noalloc) ---------------------------------
//
// Some callers cannot allocate device memory while they run: an encoder thread working out
// of a fixed device-memory budget, or code that runs where a cudaMalloc would synchronise
// the device or is not permitted. For them the search state of up to
// kNoAllocMaxPictures pictures lives in this fixed array, which every GPU that loads the
// library holds until the process exits (16 states of 10,512 bytes: 168,192 bytes).
// Every call shares it.
constexpr int kNoAllocMaxPictures = 16;
static __device__ __align__(256) GState g_noalloc_states[kNoAllocMaxPictures];
static_assert(sizeof(GState) * kNoAllocMaxPictures <= 192 * 1024, "no-alloc scratch stays modest");

struct NoAllocInit {
    DevFrame cur[kNoAllocMaxPictures], ref[kNoAllocMaxPictures];
    int* out_global;
    unsigned long long* out_sad;
    int range, n;
};

// Resets the fields the staged search reads before it writes them (the planner zeroes each
// stage's costs itself), so a call never sees the previous call's state.
__global__ void noalloc_init_kernel(GState* states, const __grid_constant__ NoAllocInit a) {
    const int i = threadIdx.x;
    if (i >= a.n) return;
    GState& s = states[i];
    s.cur = a.cur[i];
    s.ref = a.ref[i];
    s.range = a.range;
    s.out_global = a.out_global + 2 * i;
    s.out_sad = a.out_sad + i;
    s.n = 0;
    s.top_n = 0;
    s.best_dx = s.best_dy = 0;
    s.best_cost = 0;
    s.phase = 0;
}

}  // namespace vc1cu

namespace {

int noalloc_fail(char* err, size_t err_len, int code, const char* msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
    return code;
}

}  // namespace

extern "C" int vc1cu_global_motion_noalloc(const uint8_t* const* cur_y, const uint8_t* const* ref_y, int pitch,
                                           int width, int height, int range, int n, int32_t* d_dxdy,
                                           uint64_t* d_sad, void* stream, char* err, size_t err_len) {
    using namespace vc1cu;
    if (err && err_len) err[0] = 0;
    if (n < 1 || n > kNoAllocMaxPictures)
        return noalloc_fail(err, err_len, VC1CU_ERR_ARG,
                            "vc1cu_global_motion_noalloc: n must be 1..16 pictures per call (the fixed scratch size)");
    if (width <= 0 || height <= 0 || width > 16384 || height > 16384 || pitch < width)
        return noalloc_fail(err, err_len, VC1CU_ERR_ARG,
                            "vc1cu_global_motion_noalloc: width/height must be 1..16384 and pitch >= width");
    if (range < 0 || range > 32)
        return noalloc_fail(err, err_len, VC1CU_ERR_ARG, "vc1cu_global_motion_noalloc: range must be 0..32");
    if (!cur_y || !ref_y || !d_dxdy || !d_sad)
        return noalloc_fail(err, err_len, VC1CU_ERR_ARG, "vc1cu_global_motion_noalloc: null pointer argument");
    NoAllocInit a{};
    for (int i = 0; i < n; ++i) {
        if (!cur_y[i] || !ref_y[i])
            return noalloc_fail(err, err_len, VC1CU_ERR_ARG, "vc1cu_global_motion_noalloc: null frame pointer");
        a.cur[i] = DevFrame{cur_y[i], nullptr, nullptr, pitch, 0};
        a.ref[i] = DevFrame{ref_y[i], nullptr, nullptr, pitch, 0};
    }
    a.out_global = reinterpret_cast<int*>(d_dxdy);
    a.out_sad = reinterpret_cast<unsigned long long*>(d_sad);
    a.range = range;
    a.n = n;
    // The host-side name of a __device__ array is not a device address. The address is looked
    // up on every call, with the caller's device current, so it is always the one of the module
    // loaded in the current context (a cached value would dangle after cudaDeviceReset).
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_states);
    if (e != cudaSuccess || !ptr)
        return noalloc_fail(err, err_len, VC1CU_ERR_CUDA,
                            e != cudaSuccess ? cudaGetErrorString(e) : "cudaGetSymbolAddress returned null");
    GState* states = static_cast<GState*>(ptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_init_kernel<<<1, 32, 0, s>>>(states, a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(err, err_len, VC1CU_ERR_CUDA, cudaGetErrorString(e));
    run_global_search(states, n, range, width, height, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(err, err_len, VC1CU_ERR_CUDA, cudaGetErrorString(e));
    return VC1CU_OK;
}
