// vc1cu_lp.cu - kernels of the learned motion-vector proposals (see vc1cu_lp.cuh).
//
// The three convolution kernels (forward, data gradient, weight gradient) are implicit GEMMs on
// the fifth-generation tensor cores: operands staged in shared memory in the canonical
// no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix), one elected thread issues
// tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) into a tensor-memory accumulator, tcgen05.commit
// arrives on an mbarrier, and the epilogue reads the accumulator back with tcgen05.ld.
//
//  forward   D[pixel][co] = sum_tap sum_ci X[pixel + off(tap)][ci] W[co][tap][ci]   (M=128, N=32)
//            A = the tile's input halo (K-major: a pixel's 8 channels are one 16-byte row, so
//            the A operand of tap (ty, tx) is the halo at a 16-byte offset: no im2col copy);
//  dgrad     D[pixel][ci] = sum_tap sum_co dZ[pixel - off(tap)][co] W[co][tap][ci]   (same A
//            geometry over the gradient halo, B = the flipped, transposed weights);
//  wgrad     D[(tap, ci)][co] = sum_pixel X[pixel + off(tap)][ci] dZ[pixel][co]       (M = taps x
//            channels in blocks of 128, K = pixels; both operands MN-major, so each core matrix
//            is 8 pixels of one 8-channel chunk: 16-byte copies of activation rows).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "vc1cu_lp.cuh"

namespace vc1cu {

namespace {

constexpr unsigned FULLM = 0xffffffffu;

// ---- tcgen05 / mbarrier primitives ------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), descriptor version 1.
// lbo: byte distance between core matrices adjacent in the leading (K for K-major operands)
// direction; sbo: in the stride (M / N) direction.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the mbarrier phase with parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Tensor-memory allocation by warp 0 of the CTA (ncols a power of two >= 32).
__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive fp32 columns of this thread's tensor-memory lane (32x32b shape, 32 repeats).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// ---- shared-memory geometry ---------------------------------------------------------------

constexpr int kHaloW = kLpTile + 2;  // a tile's input row segment with one sample either side

// Convolution CTA: B operand [9][CA/8][32][16 B], then the halo [CA/8][3][kHaloW][16 B], then
// the mbarrier and the tensor-memory address slot.
__host__ __device__ constexpr int conv_b_bytes(int ca) { return 9 * (ca / 8) * 32 * 16; }
__host__ __device__ constexpr int conv_a_bytes(int ca) { return (ca / 8) * 3 * kHaloW * 16; }
__host__ __device__ constexpr int conv_smem_bytes(int ca) {
    return conv_b_bytes(ca) + conv_a_bytes(ca) + 64;
}

constexpr int kWgK = 64;  // pixels per weight-gradient chunk
__host__ __device__ constexpr int wg_groups(int cin) { return 9 * cin / 8; }
__host__ __device__ constexpr int wg_groups_padded(int cin) { return (wg_groups(cin) + 15) / 16 * 16; }
__host__ __device__ constexpr int wg_a_bytes(int cin) { return (kWgK / 8) * wg_groups_padded(cin) * 128; }
__host__ __device__ constexpr int wg_b_bytes() { return (kWgK / 8) * 4 * 128; }
__host__ __device__ constexpr int wg_smem_bytes(int cin) { return wg_a_bytes(cin) + wg_b_bytes() + 64; }

}  // namespace

size_t lp_conv_smem(int ca) { return (size_t)conv_smem_bytes(ca); }
// At least 50 KB, so that no more than four weight-gradient CTAs share an SM: each holds 128 of
// the SM's 512 tensor-memory columns.
size_t lp_wgrad_smem(int cin) { return std::max<size_t>((size_t)wg_smem_bytes(cin), 50 * 1024); }
size_t lp_fwd_b_elems(int l) { return (size_t)9 * lp_cin(l) * kLpC; }
size_t lp_dgrad_b_elems(int l) { return l == 0 ? 0 : (size_t)9 * kLpC * kLpC; }

namespace {

// ---- quarter-resolution pictures and the translation hint -------------------------------

__global__ void lp_down_kernel(const uint8_t* cur, int cp, const uint8_t* ref, int rp, LpGeom g, uint8_t* cur4,
                               uint8_t* ref4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.W4 * g.H4) return;
    const int x = i % g.W4, y = i / g.W4;
    int sc = 0, sr = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int yy = min(4 * y + a, g.H - 1);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int xx = min(4 * x + b, g.W - 1);
            sc += cur[(size_t)yy * cp + xx];
            sr += ref[(size_t)yy * rp + xx];
        }
    }
    cur4[i] = (uint8_t)((sc + 8) >> 4);
    ref4[i] = (uint8_t)((sr + 8) >> 4);
}

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v, unsigned long long* red) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULLM, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    unsigned long long t = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    __syncthreads();
    return t;
}

// The translation hint, coarse to fine (each stage's least SAD by hint_less):
//  A  1/16 resolution (one sample per macroblock, the rounded mean of its 4x4 quarter-res
//     samples): every displacement in [-R16, R16]^2, R16 = min(16, ceil(range / 16));
//  B  1/4 resolution: the 7x7 displacements about 4x A's, within +-ceil(range / 4);
//  C  full resolution, frame SAD at stride 2: the 5x5 vectors about 4x B's, within +-range.
// Clamped reference sampling at every level; one block per candidate.
__device__ __forceinline__ int hint_r16(const LpGeom& g) { return min(16, (g.range + 15) / 16); }
__device__ __forceinline__ int hint_na(const LpGeom& g) { return (2 * hint_r16(g) + 1) * (2 * hint_r16(g) + 1); }

// (cost, |dx|+|dy|, dy, dx) lexicographic order.
__device__ __forceinline__ bool hint_less(unsigned long long ca, int ax, int ay, unsigned long long cb, int bx, int by) {
    if (ca != cb) return ca < cb;
    const int ma = abs(ax) + abs(ay), mb = abs(bx) + abs(by);
    if (ma != mb) return ma < mb;
    if (ay != by) return ay < by;
    return ax < bx;
}

__device__ __forceinline__ int2 vec_a(const LpGeom& g, int i) {
    const int R = hint_r16(g), n = 2 * R + 1;
    return make_int2(i % n - R, i / n - R);
}
__device__ __forceinline__ int2 vec_b(const LpGeom& g, int2 a, int k) {
    const int r = (g.range + 3) / 4;
    return make_int2(min(max(4 * a.x + k % 7 - 3, -r), r), min(max(4 * a.y + k / 7 - 3, -r), r));
}
__device__ __forceinline__ int2 vec_c(const LpGeom& g, int2 b, int k) {
    return make_int2(min(max(4 * b.x + k % 5 - 2, -g.range), g.range), min(max(4 * b.y + k / 5 - 2, -g.range), g.range));
}

// The winners of the finished stages (cost layout: A's, then B's 49, then C's 25).
__device__ int2 best_a(const unsigned long long* cost, const LpGeom& g) {
    unsigned long long bc = ~0ull;
    int2 b = make_int2(0, 0);
    for (int i = 0; i < hint_na(g); ++i) {
        const int2 v = vec_a(g, i);
        if (hint_less(cost[i], v.x, v.y, bc, b.x, b.y)) {
            bc = cost[i];
            b = v;
        }
    }
    return b;
}
__device__ int2 best_b(const unsigned long long* cost, const LpGeom& g, int2 a) {
    const unsigned long long* cb = cost + hint_na(g);
    unsigned long long bc = ~0ull;
    int2 b = make_int2(0, 0);
    for (int k = 0; k < 49; ++k) {
        const int2 v = vec_b(g, a, k);
        if (hint_less(cb[k], v.x, v.y, bc, b.x, b.y)) {
            bc = cb[k];
            b = v;
        }
    }
    return b;
}

// 1/16-resolution pictures: the rounded mean of each macroblock's 4x4 quarter-res samples.
__global__ void lp_down16_kernel(const uint8_t* cur4, const uint8_t* ref4, LpGeom g, uint8_t* cur16, uint8_t* ref16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mbw * g.mbh) return;
    const int x = i % g.mbw, y = i / g.mbw;
    int sc = 0, sr = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            sc += cur4[(4 * y + a) * g.W4 + 4 * x + b];
            sr += ref4[(4 * y + a) * g.W4 + 4 * x + b];
        }
    cur16[i] = (uint8_t)((sc + 8) >> 4);
    ref16[i] = (uint8_t)((sr + 8) >> 4);
}

__global__ void lp_hint_a_kernel(const uint8_t* cur16, const uint8_t* ref16, LpGeom g, unsigned long long* cost) {
    __shared__ unsigned long long red[8];
    const int2 v = vec_a(g, blockIdx.x);
    unsigned long long s = 0;
    for (int i = threadIdx.x; i < g.mbw * g.mbh; i += blockDim.x) {
        const int x = i % g.mbw, y = i / g.mbw;
        const int rx = min(max(x + v.x, 0), g.mbw - 1), ry = min(max(y + v.y, 0), g.mbh - 1);
        s += (unsigned)abs((int)cur16[i] - (int)ref16[ry * g.mbw + rx]);
    }
    s = block_sum_u64(s, red);
    if (threadIdx.x == 0) cost[blockIdx.x] = s;
}

__global__ void lp_hint_b_kernel(const uint8_t* cur4, const uint8_t* ref4, LpGeom g, unsigned long long* cost) {
    __shared__ unsigned long long red[8];
    __shared__ int2 a;
    if (threadIdx.x == 0) a = best_a(cost, g);
    __syncthreads();
    const int2 v = vec_b(g, a, blockIdx.x);
    unsigned long long s = 0;
    for (int i = threadIdx.x; i < g.W4 * g.H4; i += blockDim.x) {
        const int x = i % g.W4, y = i / g.W4;
        const int rx = min(max(x + v.x, 0), g.W4 - 1), ry = min(max(y + v.y, 0), g.H4 - 1);
        s += (unsigned)abs((int)cur4[i] - (int)ref4[ry * g.W4 + rx]);
    }
    s = block_sum_u64(s, red);
    if (threadIdx.x == 0) cost[hint_na(g) + blockIdx.x] = s;
}

__global__ void lp_hint_c_kernel(const uint8_t* cur, int cp, const uint8_t* ref, int rp, LpGeom g,
                                 unsigned long long* cost) {
    __shared__ unsigned long long red[8];
    __shared__ int2 b;
    if (threadIdx.x == 0) b = best_b(cost, g, best_a(cost, g));
    __syncthreads();
    const int2 v = vec_c(g, b, blockIdx.x);
    const int sw = (g.W + 1) / 2, sh = (g.H + 1) / 2;
    unsigned long long s = 0;
    for (int i = threadIdx.x; i < sw * sh; i += blockDim.x) {
        const int x = 2 * (i % sw), y = 2 * (i / sw);
        const int rx = min(max(x + v.x, 0), g.W - 1), ry = min(max(y + v.y, 0), g.H - 1);
        s += (unsigned)abs((int)cur[(size_t)y * cp + x] - (int)ref[(size_t)ry * rp + rx]);
    }
    s = block_sum_u64(s, red);
    if (threadIdx.x == 0) cost[hint_na(g) + 49 + blockIdx.x] = s;
}

__global__ void lp_pick_kernel(const unsigned long long* cost, LpGeom g, int2* hint) {
    const int2 b = best_b(cost, g, best_a(cost, g));
    const unsigned long long* cc = cost + hint_na(g) + 49;
    unsigned long long bc = ~0ull;
    int2 best = make_int2(0, 0);
    for (int k = 0; k < 25; ++k) {
        const int2 v = vec_c(g, b, k);
        if (hint_less(cc[k], v.x, v.y, bc, best.x, best.y)) {
            bc = cc[k];
            best = v;
        }
    }
    *hint = best;
}

// The full-resolution frame SAD at the hint (stride 1, clamped sampling): the analysis pass's
// global_full_sad when the hint stands in for the global search. `sad` is zeroed by the launcher.
__global__ void lp_hint_sad_kernel(const uint8_t* cur, int cp, const uint8_t* ref, int rp, LpGeom g, const int2* hint,
                                   unsigned long long* sad) {
    __shared__ unsigned long long red[8];
    const int2 h = *hint;
    unsigned long long s = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)g.W * g.H; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % g.W), y = (int)(i / g.W);
        const int rx = min(max(x + h.x, 0), g.W - 1), ry = min(max(y + h.y, 0), g.H - 1);
        s += (unsigned)abs((int)cur[(size_t)y * cp + x] - (int)ref[(size_t)ry * rp + rx]);
    }
    s = block_sum_u64(s, red);
    if (threadIdx.x == 0) atomicAdd(sad, s);
}

// ---- input features ----------------------------------------------------------------------

// Per quarter-res sample, 16 bf16 channels: cur, ref, ref shifted by the hint, the two
// differences, cur's horizontal and vertical gradients, the hint (/64), zeros.
__global__ void lp_feat_kernel(const uint8_t* ref, int rp, LpGeom g, const uint8_t* cur4, const uint8_t* ref4,
                               const int2* hint, uint4* x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.W4 * g.H4) return;
    const int x = i % g.W4, y = i / g.W4;
    const int2 h = *hint;
    int sg = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int yy = min(max(4 * y + a + h.y, 0), g.H - 1);
#pragma unroll
        for (int b = 0; b < 4; ++b) sg += ref[(size_t)yy * rp + min(max(4 * x + b + h.x, 0), g.W - 1)];
    }
    const int c = cur4[i], r = ref4[i], rg = (sg + 8) >> 4;
    const int gx = (int)cur4[y * g.W4 + min(x + 1, g.W4 - 1)] - (int)cur4[y * g.W4 + max(x - 1, 0)];
    const int gy = (int)cur4[min(y + 1, g.H4 - 1) * g.W4 + x] - (int)cur4[max(y - 1, 0) * g.W4 + x];
    const float k = 1.0f / 64.0f;
    uint4 lo, hi;
    lo.x = pack_bf16x2((float)(c - 128) * k, (float)(r - 128) * k);
    lo.y = pack_bf16x2((float)(rg - 128) * k, (float)(c - r) * k);
    lo.z = pack_bf16x2((float)(c - rg) * k, (float)gx * k);
    lo.w = pack_bf16x2((float)gy * k, (float)h.x * k);
    hi.x = pack_bf16x2((float)h.y * k, 0.0f);
    hi.y = hi.z = hi.w = 0u;
    x0[2 * (size_t)i] = lo;
    x0[2 * (size_t)i + 1] = hi;
}

// ---- the convolutions on the tensor cores --------------------------------------------------

// One CTA (4 warps = the 128 tensor-memory lanes) per 128-sample row segment, persistent over
// tiles. CA: channels of the A operand (16 or 32). DGRAD: the data gradient (flipped taps,
// ReLU mask of the layer input) instead of the forward pass (bias + ReLU).
template <int CA, bool DGRAD>
__global__ void __launch_bounds__(128) lp_conv_kernel(const __grid_constant__ LpConvArgs a) {
    extern __shared__ __align__(128) uint8_t sm[];
    uint8_t* sB = sm;
    uint8_t* sA = sm + conv_b_bytes(CA);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + conv_smem_bytes(CA) - 64);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + conv_smem_bytes(CA) - 48);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int CH = CA / 8;  // 16-byte chunks per sample
    // weights: one flat copy of the packed B operand
    {
        const uint4* src = static_cast<const uint4*>(a.wb);
        uint4* dst = reinterpret_cast<uint4*>(sB);
        for (int i = tid; i < conv_b_bytes(CA) / 16; i += 128) dst[i] = __ldg(src + i);
    }
    if (warp == 0) tmem_alloc(smem_addr(tslot), 32);
    if (tid == 0) mbar_init(smem_addr(mbar), 1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int segs = (a.W4 + kLpTile - 1) / kLpTile;
    const int tiles = segs * a.H4 * a.frames;
    constexpr uint32_t idesc = idesc_bf16(128, 32, false, false);
    uint32_t phase = 0;
    bool ok = true;
    const uint4* X = static_cast<const uint4*>(a.x);
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int seg = t % segs, row = (t / segs) % a.H4, f = t / (segs * a.H4);
        const int x0 = seg * kLpTile;
        // the input halo: rows row-1..row+1, samples x0-1..x0+128, zero outside the picture
        for (int i = tid; i < 3 * kHaloW * CH; i += 128) {
            const int j = i % CH, p = (i / CH) % kHaloW, r = i / (CH * kHaloW);
            const int xx = x0 - 1 + p, yy = row - 1 + r;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (xx >= 0 && xx < a.W4 && yy >= 0 && yy < a.H4)
                v = __ldg(X + (((size_t)f * a.H4 + yy) * a.W4 + xx) * CH + j);
            *reinterpret_cast<uint4*>(sA + ((j * 3 + r) * kHaloW + p) * 16) = v;
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
#pragma unroll 1
            for (int tap = 0; tap < 9; ++tap) {
                const int ty = tap / 3, tx = tap % 3;
#pragma unroll
                for (int s = 0; s < CA / 16; ++s) {
                    const uint64_t ad = umma_desc(a0 + (uint32_t)(((2 * s * 3 + ty) * kHaloW + tx) * 16),
                                                  (uint32_t)(3 * kHaloW * 16), 128u);
                    const uint64_t bd = umma_desc(b0 + (uint32_t)((tap * CH + 2 * s) * 32 * 16), 32u * 16u, 128u);
                    umma_bf16(tmem, ad, bd, idesc, (tap | s) != 0);
                }
            }
            umma_commit(smem_addr(mbar));
        }
        ok = mbar_wait(smem_addr(mbar), phase);
        phase ^= 1;
        tc_fence_after();
        if (ok) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16), v);
            const int x = x0 + warp * 32 + lane;
            const bool valid = x < a.W4;
            const size_t pix = ((size_t)f * a.H4 + row) * a.W4 + x;
            uint32_t w[16];
            if (!DGRAD) {
#pragma unroll
                for (int c = 0; c < 32; c += 2)
                    w[c / 2] = pack_bf16x2(fmaxf(v[c] + a.bias[c], 0.0f), fmaxf(v[c + 1] + a.bias[c + 1], 0.0f));
            } else {
                uint4 m[4] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0),
                              make_uint4(0, 0, 0, 0)};
                if (valid) {
                    const uint4* act = static_cast<const uint4*>(a.act) + pix * 4;
#pragma unroll
                    for (int k = 0; k < 4; ++k) m[k] = __ldg(act + k);
                }
                const uint32_t* mw = reinterpret_cast<const uint32_t*>(m);
#pragma unroll
                for (int c = 0; c < 32; c += 2) {
                    const float g0 = bf16_lo(mw[c / 2]) > 0.0f ? v[c] : 0.0f;
                    const float g1 = bf16_hi(mw[c / 2]) > 0.0f ? v[c + 1] : 0.0f;
                    w[c / 2] = pack_bf16x2(g0, g1);
                }
                // the input layer's bias gradient: the stored (rounded) values, summed over the warp
#pragma unroll
                for (int c = 0; c < 32; c += 2) {
                    float s0 = valid ? bf16_lo(w[c / 2]) : 0.0f, s1 = valid ? bf16_hi(w[c / 2]) : 0.0f;
#pragma unroll
                    for (int o = 16; o; o >>= 1) {
                        s0 += __shfl_xor_sync(FULLM, s0, o);
                        s1 += __shfl_xor_sync(FULLM, s1, o);
                    }
                    if (lane == 0) {
                        atomicAdd(a.dbias + c, s0);
                        atomicAdd(a.dbias + c + 1, s1);
                    }
                }
            }
            if (valid) {
                uint4* y = static_cast<uint4*>(a.y) + pix * 4;
#pragma unroll
                for (int k = 0; k < 4; ++k) y[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
            }
        } else if (tid == 0) {
            atomicExch(a.err, 1);
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, 32);
}

// Weight gradient: persistent CTAs, each accumulating its share of 64-pixel row chunks in
// tensor memory (one 128 x 32 fp32 accumulator per 128 stacked (tap, channel) rows), then one
// atomic add per weight.
template <int CIN>
__global__ void __launch_bounds__(128) lp_wgrad_kernel(const __grid_constant__ LpWgradArgs a) {
    extern __shared__ __align__(128) uint8_t sm[];
    constexpr int G = wg_groups(CIN), GP = wg_groups_padded(CIN), NB = GP / 16, CH = CIN / 8;
    constexpr int KG = kWgK / 8;
    uint8_t* sA = sm;                       // [KG][GP][8 pixels][16 B]
    uint8_t* sB = sm + wg_a_bytes(CIN);     // [KG][4][8 pixels][16 B]
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + wg_smem_bytes(CIN) - 64);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + wg_smem_bytes(CIN) - 48);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < wg_a_bytes(CIN) / 16; i += 128) reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) tmem_alloc(smem_addr(tslot), 128);
    if (tid == 0) mbar_init(smem_addr(mbar), 1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int segs = (a.W4 + kWgK - 1) / kWgK;
    const int chunks = segs * a.H4 * a.frames;
    constexpr uint32_t idesc = idesc_bf16(128, 32, true, true);
    const uint4* X = static_cast<const uint4*>(a.x);
    const uint4* DZ = static_cast<const uint4*>(a.dz);
    uint32_t phase = 0;
    bool ok = true, first = true;
    for (int t = blockIdx.x; t < chunks && ok; t += gridDim.x) {
        const int seg = t % segs, row = (t / segs) % a.H4, f = t / (segs * a.H4);
        const int x0 = seg * kWgK;
        // A: for every (k-group, tap/chunk group, pixel) the 8 channels of the shifted input
        for (int i = tid; i < KG * G * 8; i += 128) {
            const int r = i % 8, g = (i / 8) % G, kg = i / (8 * G);
            const int tap = g / CH, j = g % CH, ty = tap / 3, tx = tap % 3;
            const int p = x0 + 8 * kg + r;
            const int xx = p + tx - 1, yy = row + ty - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < a.W4 && xx >= 0 && xx < a.W4 && yy >= 0 && yy < a.H4)
                v = __ldg(X + (((size_t)f * a.H4 + yy) * a.W4 + xx) * CH + j);
            *reinterpret_cast<uint4*>(sA + ((kg * GP + g) * 8 + r) * 16) = v;
        }
        for (int i = tid; i < KG * 4 * 8; i += 128) {
            const int r = i % 8, j = (i / 8) % 4, kg = i / 32;
            const int p = x0 + 8 * kg + r;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < a.W4) v = __ldg(DZ + (((size_t)f * a.H4 + row) * a.W4 + p) * 4 + j);
            *reinterpret_cast<uint4*>(sB + ((kg * 4 + j) * 8 + r) * 16) = v;
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
#pragma unroll 1
            for (int b = 0; b < NB; ++b)
#pragma unroll
                for (int s = 0; s < KG / 2; ++s) {
                    const uint64_t ad = umma_desc(a0 + (uint32_t)(((2 * s) * GP + 16 * b) * 128), (uint32_t)(GP * 128), 128u);
                    const uint64_t bd = umma_desc(b0 + (uint32_t)((2 * s) * 4 * 128), 4u * 128u, 128u);
                    umma_bf16(tmem + (uint32_t)(32 * b), ad, bd, idesc, (first && s == 0) ? 0u : 1u);
                }
            umma_commit(smem_addr(mbar));
        }
        first = false;
        ok = mbar_wait(smem_addr(mbar), phase);
        phase ^= 1;
        if (!ok && tid == 0) atomicExch(a.err, 1);
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (ok && !first) {
#pragma unroll 1
        for (int b = 0; b < NB; ++b) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(32 * b), v);
            const int m = 128 * b + 32 * warp + lane, g = m / 8;
            if (g < G) {
                const int tap = g / CH, ci = (g % CH) * 8 + m % 8;
#pragma unroll 4
                for (int co = 0; co < 32; ++co) atomicAdd(a.dw + ((size_t)co * 9 + tap) * CIN + ci, v[co]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, 128);
}

// ---- pooling, projection, candidates and the training loss ----------------------------------

__device__ __forceinline__ float softplus(float s) { return s > 0.0f ? s + log1pf(expf(-s)) : log1pf(expf(s)); }
__device__ __forceinline__ float sigm(float s) { return 1.0f / (1.0f + expf(-s)); }
__device__ __forceinline__ float smooth_l1(float e) { return fabsf(e) < 1.0f ? 0.5f * e * e : fabsf(e) - 0.5f; }

// One warp per macroblock (lane = channel), 8 macroblocks per block.
__global__ void __launch_bounds__(256) lp_head_kernel(const __grid_constant__ LpHeadArgs a) {
    __shared__ float s_dwh[kLpHead * kLpC];
    __shared__ float s_dbh[kLpHead];
    __shared__ float s_db4[kLpC];
    __shared__ float s_loss;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool train = a.labels != nullptr;
    if (train) {
        for (int i = threadIdx.x; i < kLpHead * kLpC; i += blockDim.x) s_dwh[i] = 0.0f;
        if (threadIdx.x < kLpHead) s_dbh[threadIdx.x] = 0.0f;
        if (threadIdx.x < kLpC) s_db4[threadIdx.x] = 0.0f;
        if (threadIdx.x == 0) s_loss = 0.0f;
        __syncthreads();
    }
    const int mbs = a.mbw * a.mbh;
    const int gm = blockIdx.x * 8 + warp;  // macroblock of the batch
    if (gm < mbs * a.frames) {
        const int f = gm / mbs, mb = gm % mbs, mx = mb % a.mbw, my = mb / a.mbw;
        const __nv_bfloat16* y4 = static_cast<const __nv_bfloat16*>(a.y4);
        float vals[16];
        float pooled = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const size_t pix = ((size_t)f * a.H4 + 4 * my + k / 4) * a.W4 + 4 * mx + k % 4;
            vals[k] = __bfloat162float(y4[pix * kLpC + lane]);
            pooled += vals[k];
        }
        pooled *= (1.0f / 16.0f);
        float out[kLpHead];
#pragma unroll
        for (int j = 0; j < kLpHead; ++j) {
            float p = a.wh[j * kLpC + lane] * pooled;
#pragma unroll
            for (int o = 16; o; o >>= 1) p += __shfl_xor_sync(FULLM, p, o);
            out[j] = p + a.bh[j];
        }
        const int2 g = a.hint[f];
        const int2 h[2] = {make_int2(0, 0), g};
        if (a.cands) {
            int2 r[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const float ox = fminf(fmaxf(out[2 + 2 * k], -(float)kLpOffClip), (float)kLpOffClip);
                const float oy = fminf(fmaxf(out[3 + 2 * k], -(float)kLpOffClip), (float)kLpOffClip);
                r[k] = make_int2(min(max(h[k].x + __float2int_rn(ox * kLpOffScale), -a.range), a.range),
                                 min(max(h[k].y + __float2int_rn(oy * kLpOffScale), -a.range), a.range));
            }
            const int first = out[1] > out[0] ? 1 : 0;
            if (lane < kLpK) {
                const int k = lane;
                const int2 v = k == 0 ? r[first] : (k == 1 ? r[1 - first] : (k == 2 ? h[first] : h[1 - first]));
                a.cands[(size_t)gm * kLpK + k] = v;
            }
        }
        if (train) {
            const int2 L = a.labels[gm];
            const int d0 = abs(L.x - h[0].x) + abs(L.y - h[0].y), d1 = abs(L.x - h[1].x) + abs(L.y - h[1].y);
            const int hs = d0 <= d1 ? 0 : 1;
            float dout[kLpHead];
            float loss = 0.0f;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const float tgt = k == hs ? 1.0f : 0.0f;
                loss += softplus(out[k]) - tgt * out[k];
                dout[k] = (sigm(out[k]) - tgt) * a.inv_count;
                const bool m = max(abs(L.x - h[k].x), abs(L.y - h[k].y)) <= kLpOffClip * kLpOffScale;
                const float tx = fminf(fmaxf((float)(L.x - h[k].x) / kLpOffScale, -(float)kLpOffClip), (float)kLpOffClip);
                const float ty = fminf(fmaxf((float)(L.y - h[k].y) / kLpOffScale, -(float)kLpOffClip), (float)kLpOffClip);
                const float ex = out[2 + 2 * k] - tx, ey = out[3 + 2 * k] - ty;
                loss += m ? smooth_l1(ex) + smooth_l1(ey) : 0.0f;
                dout[2 + 2 * k] = m ? fminf(fmaxf(ex, -1.0f), 1.0f) * a.inv_count : 0.0f;
                dout[3 + 2 * k] = m ? fminf(fmaxf(ey, -1.0f), 1.0f) * a.inv_count : 0.0f;
            }
            dout[6] = dout[7] = 0.0f;
            float dp = 0.0f;
#pragma unroll
            for (int j = 0; j < kLpHead; ++j) {
                dp += a.wh[j * kLpC + lane] * dout[j];
                atomicAdd(&s_dwh[j * kLpC + lane], dout[j] * pooled);
            }
            if (lane < kLpHead) atomicAdd(&s_dbh[lane], dout[lane]);
            if (lane == 0) atomicAdd(&s_loss, loss * a.inv_count);
            const float dy = dp * (1.0f / 16.0f);
            __nv_bfloat16* dz4 = static_cast<__nv_bfloat16*>(a.dz4);
            float db = 0.0f;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const size_t pix = ((size_t)f * a.H4 + 4 * my + k / 4) * a.W4 + 4 * mx + k % 4;
                const __nv_bfloat16 z = __float2bfloat16_rn(vals[k] > 0.0f ? dy : 0.0f);
                dz4[pix * kLpC + lane] = z;
                db += __bfloat162float(z);
            }
            atomicAdd(&s_db4[lane], db);
        }
    }
    if (train) {
        __syncthreads();
        for (int i = threadIdx.x; i < kLpHead * kLpC; i += blockDim.x) atomicAdd(a.dwh + i, s_dwh[i]);
        if (threadIdx.x < kLpHead) atomicAdd(a.dbh + threadIdx.x, s_dbh[threadIdx.x]);
        if (threadIdx.x < kLpC) atomicAdd(a.db4 + threadIdx.x, s_db4[threadIdx.x]);
        if (threadIdx.x == 0) atomicAdd(a.loss, s_loss);
    }
}

// Integer-pixel label of a plain pass's quarter-pel vector: the nearest pixel (ties upward).
__global__ void lp_labels_kernel(const int2* mvs, int n, int2* labels) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) labels[i] = make_int2((mvs[i].x + 2) >> 2, (mvs[i].y + 2) >> 2);
}

__global__ void lp_adam_kernel(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                               float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Packs layer l's fp32 W[co][tap][ci] into the forward B operand [tap][ci/8][co][8] and (l >= 1)
// the data-gradient B operand [tap'][co/8][ci][8] with tap' = 8 - tap.
__global__ void lp_pack_kernel(const float* w, int cin, __nv_bfloat16* fwd, __nv_bfloat16* dgr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 32 * 9 * cin) return;
    const int ci = i % cin, tap = (i / cin) % 9, co = i / (9 * cin);
    const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
    fwd[((tap * (cin / 8) + ci / 8) * 32 + co) * 8 + ci % 8] = b;
    if (dgr) dgr[(((8 - tap) * 4 + co / 8) * cin + ci) * 8 + co % 8] = b;
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------------

cudaError_t lp_launch_downsample(const uint8_t* cur, int cur_pitch, const uint8_t* ref, int ref_pitch,
                                 const LpGeom& g, uint8_t* cur4, uint8_t* ref4, cudaStream_t s) {
    const int n = g.W4 * g.H4;
    lp_down_kernel<<<(n + 255) / 256, 256, 0, s>>>(cur, cur_pitch, ref, ref_pitch, g, cur4, ref4);
    return cudaGetLastError();
}

cudaError_t lp_launch_hint(const uint8_t* cur, int cur_pitch, const uint8_t* ref, int ref_pitch, const LpGeom& g,
                           const uint8_t* cur4, const uint8_t* ref4, unsigned long long* scratch, int2* hint,
                           unsigned long long* hint_sad, cudaStream_t s) {
    const int R = std::min(16, (g.range + 15) / 16), na = (2 * R + 1) * (2 * R + 1);
    uint8_t* cur16 = const_cast<uint8_t*>(cur4) + (size_t)g.W4 * g.H4;  // the buffers hold both levels
    uint8_t* ref16 = const_cast<uint8_t*>(ref4) + (size_t)g.W4 * g.H4;
    lp_down16_kernel<<<(g.mbw * g.mbh + 255) / 256, 256, 0, s>>>(cur4, ref4, g, cur16, ref16);
    lp_hint_a_kernel<<<na, 256, 0, s>>>(cur16, ref16, g, scratch);
    lp_hint_b_kernel<<<49, 256, 0, s>>>(cur4, ref4, g, scratch);
    lp_hint_c_kernel<<<25, 256, 0, s>>>(cur, cur_pitch, ref, ref_pitch, g, scratch);
    lp_pick_kernel<<<1, 1, 0, s>>>(scratch, g, hint);
    cudaError_t e = cudaMemsetAsync(hint_sad, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const long px = (long)g.W * g.H;
    lp_hint_sad_kernel<<<(int)std::min<long>((px + 255) / 256, 1184L), 256, 0, s>>>(cur, cur_pitch, ref, ref_pitch, g,
                                                                                  hint, hint_sad);
    return cudaGetLastError();
}

cudaError_t lp_launch_features(const uint8_t* ref, int ref_pitch, const LpGeom& g, const uint8_t* cur4,
                               const uint8_t* ref4, const int2* hint, void* x0, cudaStream_t s) {
    const int n = g.W4 * g.H4;
    lp_feat_kernel<<<(n + 255) / 256, 256, 0, s>>>(ref, ref_pitch, g, cur4, ref4, hint, static_cast<uint4*>(x0));
    return cudaGetLastError();
}

cudaError_t lp_launch_conv(int ca, bool dgrad, const LpConvArgs& a, int sm_count, cudaStream_t s) {
    const int tiles = ((a.W4 + kLpTile - 1) / kLpTile) * a.H4 * a.frames;
    const size_t smem = lp_conv_smem(ca);
    const void* k = nullptr;
    if (ca == 16 && !dgrad) k = reinterpret_cast<const void*>(&lp_conv_kernel<16, false>);
    else if (ca == 32 && !dgrad) k = reinterpret_cast<const void*>(&lp_conv_kernel<32, false>);
    else if (ca == 32 && dgrad) k = reinterpret_cast<const void*>(&lp_conv_kernel<32, true>);
    else return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, smem);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, std::min(tiles, std::max(per_sm, 1) * sm_count));
    if (ca == 16) lp_conv_kernel<16, false><<<grid, 128, smem, s>>>(a);
    else if (!dgrad) lp_conv_kernel<32, false><<<grid, 128, smem, s>>>(a);
    else lp_conv_kernel<32, true><<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t lp_launch_wgrad(int cin, const LpWgradArgs& a, int sm_count, cudaStream_t s) {
    const int chunks = ((a.W4 + kWgK - 1) / kWgK) * a.H4 * a.frames;
    const size_t smem = lp_wgrad_smem(cin);
    const void* k = cin == 16 ? reinterpret_cast<const void*>(&lp_wgrad_kernel<16>)
                              : reinterpret_cast<const void*>(&lp_wgrad_kernel<32>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, smem);
    if (e != cudaSuccess) return e;
    // at most four CTAs per SM: each holds 128 of the SM's 512 tensor-memory columns
    const int grid = std::max(1, std::min(chunks, std::min(std::max(per_sm, 1), 4) * sm_count));
    if (cin == 16) lp_wgrad_kernel<16><<<grid, 128, smem, s>>>(a);
    else lp_wgrad_kernel<32><<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t lp_launch_head(const LpHeadArgs& a, cudaStream_t s) {
    const int n = a.mbw * a.mbh * a.frames;
    lp_head_kernel<<<(n + 7) / 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t lp_launch_labels(const int2* mvs, int n, int2* labels, cudaStream_t s) {
    lp_labels_kernel<<<(n + 255) / 256, 256, 0, s>>>(mvs, n, labels);
    return cudaGetLastError();
}

cudaError_t lp_launch_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                           float eps, int step, cudaStream_t s) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    lp_adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t lp_launch_pack(const float* master, void* fwd_b, void* dgrad_b, cudaStream_t s) {
    size_t off = 0, fo = 0, dof = 0;
    for (int l = 0; l < kLpLayers; ++l) {
        const int cin = lp_cin(l), n = lp_wcount(l);
        lp_pack_kernel<<<(n + 255) / 256, 256, 0, s>>>(
            master + off, cin, static_cast<__nv_bfloat16*>(fwd_b) + fo,
            l ? static_cast<__nv_bfloat16*>(dgrad_b) + dof : nullptr);
        off += (size_t)n + kLpC;
        fo += lp_fwd_b_elems(l);
        dof += lp_dgrad_b_elems(l);
    }
    return cudaGetLastError();
}

}  // namespace vc1cu
