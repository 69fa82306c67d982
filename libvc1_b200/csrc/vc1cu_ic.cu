// vc1cu_ic.cu - intensity compensation on the device: the fade estimate of
// Vc1Encoder::estimate_intensity_comp (encoder_motion_compensation.cpp:296-348) and the
// compensated reference of intensity_compensated_reference (:195-294).
//
// The estimate samples one luma pixel per 4x4 cell along the picture's 1-MV field (the
// reference pixel at the vector rounded to whole pixels, clamped at the edges). Every sample
// cost the reference evaluates, |cur - map(ref; LUMSCALE, shift)|, depends on the sample only
// through its (ref, cur) pair, so three small kernels turn the samples into the SAD of every
// (LUMSCALE 1..63, shift -32..31) pair:
//   ic_hist_kernel  one thread per sample: the 256x256 joint histogram of (ref, cur) and the
//                   exact integer sums n, sum ref, sum cur, sum ref^2, sum ref*cur;
//   ic_row_kernel   S[r][m] = sum over c of hist[r][c] * |c - m|, one CTA per ref value r;
//   ic_sad_kernel   SAD(l, z) = sum over r of S[r][map_lz(r)], one thread per pair.
// The host then reproduces the reference's long double least-squares fit from the exact sums
// and picks, from the table, the pair of the fit's 7x7 neighbourhood exactly as the reference
// does (smallest SAD, ties to the smaller |l - 32| + |z|, in the reference's scan order).
#include <cuda_runtime.h>

#include "vc1cu_core.cuh"

namespace vc1cu {

constexpr int kIcLumScales = 63;  // LUMSCALE 1..63 (the estimate never produces 0)
constexpr int kIcShifts = 64;     // shift -32..31

// Per-picture scratch of the estimate (one contiguous block per picture).
struct IcScratch {
    unsigned int hist[256 * 256];
    unsigned long long row[256 * 256];
    unsigned long long table[kIcLumScales * kIcShifts];
    unsigned long long sums[5];  // n, sum r, sum c, sum r^2, sum r*c
};

struct IcDesc {
    DevFrame cur, ref;
    const int2* mvs;
    IcScratch* s;
};

size_t ic_scratch_bytes() { return (sizeof(IcScratch) + 255) & ~size_t(255); }

// Vc1Encoder::round_qpel_to_pixel, encoder_motion.cpp:1295-1297
__device__ __forceinline__ int qpel_to_pixel(int q) { return q >= 0 ? (q + 2) / 4 : -((-q + 2) / 4); }

__global__ void __launch_bounds__(256) ic_hist_kernel(const IcDesc* descs, int W, int H, int mbw) {
    const IcDesc& d = descs[blockIdx.y];
    const int cw = (W + 3) / 4, ch = (H + 3) / 4;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v[5] = {0, 0, 0, 0, 0};
    if (s < cw * ch) {
        const int px = (s % cw) * 4, py = (s / cw) * 4;
        const int2 mv = d.mvs[(py >> 4) * mbw + (px >> 4)];
        const int rx = iclamp(px + qpel_to_pixel(mv.x), 0, W - 1), ry = iclamp(py + qpel_to_pixel(mv.y), 0, H - 1);
        const unsigned r = d.ref.y[(size_t)ry * d.ref.pitch_y + rx];
        const unsigned c = d.cur.y[(size_t)py * d.cur.pitch_y + px];
        atomicAdd(&d.s->hist[r * 256 + c], 1u);
        v[0] = 1;
        v[1] = r;
        v[2] = c;
        v[3] = r * r;
        v[4] = r * c;
    }
    __shared__ unsigned long long part[8][5];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        unsigned long long x = v[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) part[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        unsigned long long x = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) x += part[w][threadIdx.x];
        if (x) atomicAdd(&d.s->sums[threadIdx.x], x);
    }
}

__global__ void __launch_bounds__(256) ic_row_kernel(const IcDesc* descs) {
    const IcDesc& d = descs[blockIdx.y];
    const int r = blockIdx.x, m = threadIdx.x;
    __shared__ unsigned int h[256];
    h[m] = d.s->hist[r * 256 + m];
    __syncthreads();
    unsigned long long acc = 0;
    for (int c = 0; c < 256; ++c) acc += (unsigned long long)h[c] * (unsigned)iabs(c - m);
    d.s->row[r * 256 + m] = acc;
}

// intensity_map_y with LUMSCALE l (1..63) and shift z (-32..31): (scale*v + shift + 32) >> 6
__global__ void __launch_bounds__(64) ic_sad_kernel(const IcDesc* descs) {
    const IcDesc& d = descs[blockIdx.y];
    const int l = blockIdx.x + 1, z = (int)threadIdx.x - 32;
    const int scale = l + 32, shift = z * 64;
    unsigned long long acc = 0;
    for (int r = 0; r < 256; ++r) acc += d.s->row[r * 256 + iclamp((scale * r + shift + 32) >> 6, 0, 255)];
    d.s->table[(l - 1) * kIcShifts + (z + 32)] = acc;
}

cudaError_t launch_ic_estimate(const IcDesc* d_descs, int n, int W, int H, cudaStream_t s) {
    const int mbw = (W + 15) / 16;
    const int samples = ((W + 3) / 4) * ((H + 3) / 4);
    ic_hist_kernel<<<dim3((unsigned)((samples + 255) / 256), (unsigned)n), 256, 0, s>>>(d_descs, W, H, mbw);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ic_row_kernel<<<dim3(256, (unsigned)n), 256, 0, s>>>(d_descs);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ic_sad_kernel<<<dim3(kIcLumScales, (unsigned)n), kIcShifts, 0, s>>>(d_descs);
    return cudaGetLastError();
}

// Offsets of the fields the host reads back.
size_t ic_table_offset() { return offsetof(IcScratch, table); }
size_t ic_sums_offset() { return offsetof(IcScratch, sums); }
size_t ic_hist_bytes() { return sizeof(((IcScratch*)nullptr)->hist); }

// intensity_compensated_reference (encoder_motion_compensation.cpp:195-294): one thread per
// luma pixel, and for the pixels of even coordinates the co-sited chroma pair. scale/shift
// are the luma law of intensity_map_y (:175-187), cscale the chroma scale of intensity_map_uv.
__global__ void ic_map_kernel(DevFrame ref, uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H,
                              int enabled, int scale, int shift, int cscale) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y;
    if (x >= W || yy >= H) return;
    const int a = ref.y[(size_t)yy * ref.pitch_y + x];
    y[(size_t)yy * pitch_y + x] = (uint8_t)(enabled ? iclamp((scale * a + shift + 32) >> 6, 0, 255) : a);
    if (!(x & 1) && !(yy & 1)) {
        const int cx = x >> 1, cy = yy >> 1;
        if (cx < W / 2 && cy < H / 2) {
            const int b = ref.u[(size_t)cy * ref.pitch_c + cx], c = ref.v[(size_t)cy * ref.pitch_c + cx];
            u[(size_t)cy * pitch_c + cx] = (uint8_t)(enabled ? iclamp((cscale * (b - 128) + 128 * 64 + 32) >> 6, 0, 255) : b);
            v[(size_t)cy * pitch_c + cx] = (uint8_t)(enabled ? iclamp((cscale * (c - 128) + 128 * 64 + 32) >> 6, 0, 255) : c);
        }
    }
}

cudaError_t launch_ic_map(const DevFrame& ref, uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H,
                          int enabled, int scale, int shift, int cscale, cudaStream_t s) {
    ic_map_kernel<<<dim3((unsigned)((W + 255) / 256), (unsigned)H), 256, 0, s>>>(ref, y, u, v, pitch_y, pitch_c, W, H, enabled,
                                                                                scale, shift, cscale);
    return cudaGetLastError();
}

// The descriptor is opaque to the host shim: it fills one through this helper.
void ic_fill_desc(void* desc, const DevFrame& cur, const DevFrame& ref, const int2* mvs, void* scratch) {
    IcDesc* d = static_cast<IcDesc*>(desc);
    d->cur = cur;
    d->ref = ref;
    d->mvs = mvs;
    d->s = static_cast<IcScratch*>(scratch);
}
size_t ic_desc_bytes() { return sizeof(IcDesc); }

}  // namespace vc1cu
