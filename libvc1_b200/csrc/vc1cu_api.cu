// vc1cu_api.cu - host shim exporting the C ABI of include/vc1cu.h.
//
// Owns the CUDA context state: one stream per context, frame slots and result slots in
// HBM, the pointer+fingerprint frame cache of the Vulkan-compatible scoring entry point
// (src/vulkan_compute.cpp:30-45, :194-231), launch descriptors and counters. Every entry
// point returns a status code and never throws; failures are reported, never replaced by a
// CPU computation.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is reached through the runtime's entry point)
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstddef>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "vc1cu_core.cuh"
#include "vc1cu_lp.cuh"
#include "vc1cu_synth.cuh"

namespace vc1cu {
// kernels and drivers of the other translation units
const void* core_kernel(int kind);
cudaError_t launch_lr_index(const DevFrame& ref, int W, int H, uint64_t* out, cudaStream_t s);
cudaError_t launch_core(int kind, int grid, int block, size_t smem, cudaStream_t s, const DevParams& P,
                        const PassDesc* passes, int npass, const uint32_t* items, unsigned nitems, const WinCfg& wc,
                        uint32_t epoch, LaunchStatus* st);
__global__ void totals_kernel(const __grid_constant__ DevParams P, const PassDesc* passes, int npass);
cudaError_t launch_learned_merge(const DevResult& dst, const DevResult& src, const uint8_t* only, int mbs,
                                 cudaStream_t s);
cudaError_t launch_subpel_planes(const uint8_t* ref, int pitch, int W, int H, int rnd, int bilinear, uint32_t phase_mask,
                                 uint8_t* out, int opitch, int border, long long stride, cudaStream_t s);
int warp_bytes_for_host(const WinCfg& wc);
struct GState;
size_t gstate_bytes();
int run_global_search(GState* d_states, int n, int R, int W, int H, cudaStream_t stream);
cudaError_t launch_global_fanout(const GlobalCopy* d_copies, int n, cudaStream_t s);
void init_gstate(GState* h, const DevFrame& cur, const DevFrame& ref, int range, int* out_global,
                 unsigned long long* out_sad);
void launch_mc(const DevParams& P, const DevFrame& ref, const int2* mvs, const int2* bmv, const uint8_t* use4, int mode,
               uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s);
void launch_xform(const DevParams& P, const DevFrame& src, const DevFrame& pred, int type_mask, double* coeffs,
                  int16_t* levels, cudaStream_t s);
void launch_score(const DevParams& P, const ScoreArgs& a, const int2* cands, int n, unsigned long long* out,
                  cudaStream_t s);
double measure_int32_peak(cudaStream_t s, int sms);
int index_fault_record(unsigned int* count, unsigned long long* first, int reset);
double measure_fp64_peak(cudaStream_t s, int sms);
size_t trd_tables_bytes();
void trd_fill_tables(void* host);
cudaError_t launch_trd(const DevParams& P, const DevFrame& src, const DevFrame& pred, const void* tables,
                       const uint8_t* mquant, const vc1cu_trd_cfg& cfg, unsigned long long* d_sum, vc1cu_tdecision* out,
                       int16_t* levels, cudaStream_t s, const int* mb_list, int n_list, double frame_mean);
cudaError_t trd_frame_mean(const DevParams& P, const DevFrame& src, const vc1cu_trd_cfg& cfg, unsigned long long* d_sum,
                           cudaStream_t s, double* mean);
size_t intra_scratch_bytes(const DevParams& P);
cudaError_t launch_overlap_sse(const int32_t* sy, const int32_t* su, const int32_t* sv, const uint8_t* oy,
                               const uint8_t* ou, const uint8_t* ov, int pitch_y, int pitch_c, int W, int H, int bias,
                               unsigned long long* sse, cudaStream_t s);
cudaError_t launch_bitplane_bits(const uint8_t* plane, int w, int h, unsigned long long* out, cudaStream_t s);
cudaError_t launch_intra_recon(const DevParams& P, const DevFrame& src, int overlap, const uint8_t* d_flags,
                               const uint8_t* d_mquant, const uint8_t* d_derived, void* scratch, uint8_t* edge,
                               int32_t* oy, int32_t* ou, int32_t* ov, const void* tables, const vc1cu_trd_cfg& cfg,
                               cudaStream_t s);
cudaError_t launch_dquant_stats(const DevParams& P, const DevFrame& src, const DevFrame& pred, const vc1cu_trd_cfg& cfg,
                                double frame_mean, double* lscale, double* adjacency, uint8_t* bright, cudaStream_t s);
cudaError_t launch_bpictures(const DevParams& P, const BDesc* d_descs, int n, cudaStream_t s);
cudaError_t launch_p_motion_bits(const DevParams& P, const DevResult& r, int mode, unsigned long long* acc, cudaStream_t s);
cudaError_t launch_loop_filter_i(uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H, int pq,
                                 cudaStream_t s);
cudaError_t launch_loop_filter_p(uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H, int pq,
                                 const int2* bmv, const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra,
                                 cudaStream_t s, int main_profile);
cudaError_t launch_overlap(int32_t* y, int32_t* u, int32_t* v, int mbw, int mbh, const uint8_t* d_flags, int all,
                           cudaStream_t s);
cudaError_t launch_store_signed(const int32_t* y, const int32_t* u, const int32_t* v, int mbw, int mbh, int bias,
                                const uint8_t* d_mask, uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c,
                                int W, int H, cudaStream_t s);
void launch_fast_tt(const DevParams& P, const DevFrame& src, const DevFrame& pred, uint8_t* types, cudaStream_t s);
void launch_recon(const DevParams& P, const DevFrame& pred, const int16_t* levels, int4 tindex, const uint8_t* block_types,
                  uint8_t* dy, uint8_t* du, uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s,
                  const uint8_t* mquant = nullptr, const uint8_t* derived = nullptr);
cudaError_t launch_b_mc(const DevParams& P, const DevFrame& cur, const DevFrame& past, const DevFrame& fut,
                        const uint8_t* modes, const int2* fmv, const int2* bmv, int mode, uint8_t* dy, uint8_t* du,
                        uint8_t* dv, int pitch_y, int pitch_c, cudaStream_t s);
struct IcDesc;
size_t ic_scratch_bytes();
size_t ic_table_offset();
size_t ic_sums_offset();
size_t ic_hist_bytes();
size_t ic_desc_bytes();
void ic_fill_desc(void* desc, const DevFrame& cur, const DevFrame& ref, const int2* mvs, void* scratch);
cudaError_t launch_ic_estimate(const IcDesc* d_descs, int n, int W, int H, cudaStream_t s);
cudaError_t launch_ic_map(const DevFrame& ref, uint8_t* y, uint8_t* u, uint8_t* v, int pitch_y, int pitch_c, int W, int H,
                          int enabled, int scale, int shift, int cscale, cudaStream_t s);
}  // namespace vc1cu

using namespace vc1cu;

namespace {

constexpr int kMaxSlot = 4096;
constexpr int kInternalOut = kMaxSlot + 1;   // result slot of vc1cu_analyze_p_core
constexpr int kInternalSeed = kMaxSlot + 2;  // its seed
constexpr int kInternalFwd = kMaxSlot + 3;   // the forward / backward core passes and the anchor
constexpr int kInternalBwd = kMaxSlot + 4;   // of vc1cu_analyze_b_picture
constexpr int kInternalAnchor = kMaxSlot + 5;
constexpr int kInternalIc = kMaxSlot + 6;     // MV field of vc1cu_estimate_intensity_comp
constexpr int kInternalLpFb = kMaxSlot + 7;   // + i: the fallback results of vc1cu_lp_analyze's pass i
constexpr int kMaxLpPasses = 256;
constexpr int kInternalLast = kInternalLpFb + kMaxLpPasses - 1;
constexpr int kInternalB = kMaxSlot + 1;     // B-result slot of vc1cu_analyze_b_picture
constexpr int kInternalFrame = kMaxSlot + 1; // frame slot of the scene score's compensated reference
constexpr size_t kMaxBatch = 64u * 65535u;   // VulkanComputeContext's candidate limit
#ifndef VC1CU_SEEDED_MIXED_RW
#define VC1CU_SEEDED_MIXED_RW 8
#endif
constexpr int kSeededMixedRw = VC1CU_SEEDED_MIXED_RW;  // window radius of seeded Mixed-MV launches
constexpr int kMinUnseededRw = 24;  // smallest window radius a tuned unseeded launch shrinks to
#ifndef VC1CU_WINDOW_TMA
#define VC1CU_WINDOW_TMA 1
#endif
#ifndef VC1CU_SUBPEL_PLANES
#define VC1CU_SUBPEL_PLANES 1
#endif
constexpr int kSubpelBorder = 32;  // sub-pel planes extend this far beyond the picture

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// The tensor map of a frame's luma plane (W x H bytes, row pitch `pitch`) with a box of one
// search window (wp x wh bytes). Requirements checked here: base 16-byte aligned, pitch a
// multiple of 16, box sides 1..256, box width a multiple of 16 bytes; the kernel only issues a
// copy whose x is a multiple of 16 and whose box lies inside the plane.
bool encode_window_map(void* out128, const uint8_t* luma, int W, int H, int pitch, int wp, int wh) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || (reinterpret_cast<uintptr_t>(luma) & 15) || (pitch & 15) || wp < 16 || wp > 256 || (wp & 15) ||
        wh < 1 || wh > 256 || W < wp || H < wh)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch};
    const cuuint32_t box[2] = {(cuuint32_t)wp, (cuuint32_t)wh};
    const cuuint32_t estr[2] = {1, 1};
    CUtensorMap map;
    const CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(luma), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    static_assert(sizeof(CUtensorMap) == 128, "CUtensorMap size");
    std::memcpy(out128, &map, 128);
    return true;
}

struct Status {
    int code;
    std::string msg;
};

struct Fail {
    int code;
    std::string msg;
};

inline void ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    // reset the runtime's last error, so a later launch check does not report this one again
    (void)cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) throw Fail{VC1CU_ERR_OOM, std::string(what) + ": out of device memory"};
    if (e != cudaSuccess) throw Fail{VC1CU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// The event recorded on the context stream after the work of the API call that last wrote a
// slot: reads of the slot wait for it alone, on the read stream.
struct Written {
    cudaEvent_t e = nullptr;
    Written() = default;
    Written(const Written&) = delete;
    Written& operator=(const Written&) = delete;
    ~Written() {
        if (e) cudaEventDestroy(e);
    }
};

struct FrameSlot {
    uint8_t* d = nullptr;
    size_t cap = 0;
    int w = 0, h = 0, pitch_y = 0, pitch_c = 0;
    bool valid = false;
    std::shared_ptr<Written> last_use;  // after the last call whose work read or wrote the frame
    cudaEvent_t uploaded = nullptr;     // the last upload into the slot, on the upload stream
    DevFrame view() const {
        DevFrame f;
        f.y = d;
        f.pitch_y = pitch_y;
        f.pitch_c = pitch_c;
        f.u = d + (size_t)pitch_y * h;
        f.v = f.u + (size_t)pitch_c * (h / 2);
        return f;
    }
};

struct ResultSlot {
    void* d = nullptr;
    size_t bytes = 0;  // the slot's one allocation, all fields
    std::shared_ptr<Written> written;
    int mbs = 0;
    DevResult r{};
    bool valid = false;
    int mode = -1;         // how the slot's last pass ran (-1: uploaded, not computed)
    bool seeded = false;
    bool allow_intra = false;
};

struct BSlot {
    void* d = nullptr;
    size_t bytes = 0;
    std::shared_ptr<Written> written;
    int mbs = 0;
    DevBResult r{};
    bool valid = false;
    int mode = 0;
};

struct CacheSlot {
    const uint8_t* host = nullptr;
    int w = 0, h = 0;
    uint64_t fp = 0, age = 0;
    uint8_t* d = nullptr;
    size_t cap = 0;
    bool valid = false;
};

// frame_fingerprint, src/vulkan_compute.cpp:30-45 (cache-invalidation tag, not a hash)
uint64_t frame_fingerprint(const uint8_t* p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    if (!p || !n) return h;
    constexpr size_t samples = 97;
    for (size_t i = 0; i < samples; ++i) {
        const size_t pos = (i * (n - 1)) / (samples - 1);
        h ^= static_cast<uint64_t>(p[pos]);
        h *= 1099511628211ull;
    }
    h ^= static_cast<uint64_t>(n);
    h *= 1099511628211ull;
    return h;
}

thread_local std::string t_open_error;

}  // namespace

struct vc1cu_ctx {
    int device = 0;
    std::string name;
    cudaStream_t stream = nullptr;
    cudaStream_t rstream = nullptr;  // result reads (waits on the slot's Written event only)
    void* h_read = nullptr;          // pinned landing buffer of a result read (one slot)
    size_t read_cap = 0;
    std::vector<int> dirty_results, dirty_bresults;  // slots written by the current call
    std::vector<int> used_frames;                     // frame slots the current call's work uses
    cudaStream_t ustream = nullptr;  // frame uploads (each waits for the last use of its slot)
    std::mutex mu;
    std::string err;
    std::unordered_map<int, FrameSlot> frames;
    std::unordered_map<int, ResultSlot> results;
    std::unordered_map<int, BSlot> bresults;
    CacheSlot cache[8];
    uint64_t age = 0;
    vc1cu_counters counters{};
    LaunchStatus* d_status = nullptr;
    PassDesc* d_passes = nullptr;
    int passes_cap = 0;
    BDesc* d_bdescs = nullptr;
    int bdescs_cap = 0;
    void* d_lf = nullptr;      // coded-block metadata of vc1cu_loop_filter_p
    size_t lf_cap = 0;
    void* d_btypes = nullptr;  // per-block transform types of vc1cu_reconstruct
    size_t btypes_cap = 0;
    void* d_sp = nullptr;       // sub-pel prediction planes of the current launch's references
    size_t sp_cap = 0;
    void* d_trd_tab = nullptr;  // the transform RD's dense rate tables (built once)
    void* d_trd = nullptr;      // its per-call buffers: MQUANT, decisions, levels, luma sum
    size_t trd_cap = 0;
    void* d_mrd = nullptr;      // the P mode decision's counters, sampled MB list and decisions
    size_t mrd_cap = 0;
    void* d_dq = nullptr;       // the DQUANT search's rounds (MB lists, MQUANTs, decisions, levels, statistics)
    size_t dq_cap = 0;
    void* d_intra = nullptr;    // the intra reconstruction's levels, DC grids, maps and edge source
    size_t intra_cap = 0;
    void* d_iovl = nullptr;     // the I overlap plan's three signed reconstructions and error sums
    size_t iovl_cap = 0;
    void* d_ic = nullptr;      // intensity-estimate scratch (one block per picture) and descriptors
    size_t ic_cap = 0;
    void* d_icdesc = nullptr;
    // Outstanding fade-estimate batches (vc1cu_estimate_intensity_enqueue / _collect): each has
    // a pinned landing buffer for its tables and sums and the event after their copy.
    static constexpr int kIcTickets = 4;
    struct IcTicket {
        void* h = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;
        int n = 0;
        int64_t id = 0;  // 0: free
    } ic_tickets[kIcTickets], ic_sync;  // ic_sync: the synchronous entry points' buffer
    int64_t ic_next_id = 1;
    void* d_gcopy = nullptr;   // GlobalCopy list of a launch's passes that share a global search
    size_t gcopy_cap = 0;
    void* d_ovl = nullptr;     // per-macroblock overlap flags / store mask
    size_t ovl_cap = 0;
    size_t icdesc_cap = 0;
    GState* d_gstates = nullptr;
    int gstates_cap = 0;
    void* d_lr = nullptr;      // long-range signature indexes of a launch's reference pictures
    size_t lr_cap = 0;
    void* d_scratch = nullptr;
    size_t scratch_cap = 0;
    void* d_synth = nullptr;   // vc1cu_synth_frames: launch arguments, normalisation terms and sums
    size_t synth_cap = 0;
    // Pinned staging of launch descriptors: a ring, so that the host can enqueue up to
    // kStagingRing launches ahead of the device (each copy out of a buffer is ordered behind
    // the launches before it on the stream, and its buffer is reused once that copy is done).
    static constexpr int kStagingRing = 8;
    struct StagingBuf {
        void* h = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;  // the H2D copy out of h
    } staging_ring[kStagingRing];
    int staging_next = 0, staging_cur = 0;
    uint32_t epoch = 0;
    // CUDA-graph capture (vc1cu_graph_begin / _end): while capturing, launch descriptors go to
    // pinned buffers the graph keeps, core launches clear their done flags and use a fixed epoch,
    // and the slots the captured work writes are recorded for the graph's launches.
    bool capturing = false;
    std::vector<void*> capture_hold;
    std::vector<int> capture_results, capture_bresults, capture_frames;
    struct Graph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<void*> hold;
        std::vector<int> results, bresults, frames;
    };
    std::map<int, Graph> graphs;
    int graph_next = 1;
    // launch shapes chosen by vc1cu_autotune: key (W, H, range, local range, instantiation) ->
    // (warps per block, blocks per SM; 0 = the occupancy limit)
    std::map<std::vector<int>, std::pair<int, int>> tuned;
    std::pair<int, int> tune_force{0, 0};  // a shape under trial (vc1cu_autotune), (0, 0) otherwise
    std::vector<int> last_tune_key;        // the key of the last core launch
    int wait_log2 = 24;                  // vc1cu_debug_set_wait_limit
    uint32_t withhold_next = 0xFFFFFFFFu;  // vc1cu_debug_withhold_publish (next core launch only)
    int sm_count = 0;
    int max_smem = 0;
    int max_smem_sm = 0;  // shared memory per SM
    // per-launch event timing
    bool timing = false;
    struct Timed { cudaEvent_t a, b; int family; };
    std::vector<Timed> pending;
    std::vector<cudaEvent_t> event_pool;
    vc1cu_timing tsum{};
    // work-queue tables per launch shape (raster, pass levels)
    std::map<std::vector<int>, std::pair<uint32_t*, unsigned>> items;
};

namespace {

void* ensure(void*& p, size_t& cap, size_t bytes, const char* what) {
    if (cap >= bytes && p) return p;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    ck(cudaMalloc(&p, bytes), what);
    cap = bytes;
    return p;
}

int fail(vc1cu_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else t_open_error = msg;
    return code;
}

void stamp_written(vc1cu_ctx* c);

void abort_capture(vc1cu_ctx* c);

template <class F>
int guarded(vc1cu_ctx* c, F&& f) {
    if (!c) return fail(nullptr, VC1CU_ERR_ARG, "null context");
    std::lock_guard<std::mutex> lock(c->mu);
    try {
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        const int rc = f();
        stamp_written(c);
        return rc;
    } catch (const Fail& e) {
        try {
            stamp_written(c);  // slots the failed call wrote before its error
        } catch (const Fail&) {
        }
        abort_capture(c);
        return fail(c, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(c, VC1CU_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(c, VC1CU_ERR_CUDA, e.what());
    }
}

// Validates p and derives the device-side parameter block.
int make_dev_params(const vc1cu_params* p, DevParams& P, std::string& why) {
    if (!p) { why = "null params"; return VC1CU_ERR_ARG; }
    if (p->width <= 0 || p->height <= 0 || (p->width & 1) || (p->height & 1) || p->width > 16384 || p->height > 16384) {
        why = "width/height must be positive, even and <= 16384 (the internal 4:2:0 raster)";
        return VC1CU_ERR_ARG;
    }
    if (p->pqindex < 1 || p->pqindex > 31) { why = "pqindex must be 1..31"; return VC1CU_ERR_ARG; }
    if (p->search_range < 0 || p->search_range > 1024 || p->local_search_range < 0) {
        why = "search_range must be 0..1024 and local_search_range >= 0";
        return VC1CU_ERR_ARG;
    }
    if (p->me_quality == 3) { why = "me_quality RD (codec-aware finalists) is not implemented on the device"; return VC1CU_ERR_UNSUPPORTED; }
    if (p->me_quality < 0 || p->me_quality > 3 || p->me_algorithm < 0 || p->me_algorithm > 1 || p->long_range_mode < 0 ||
        p->long_range_mode > 2 || p->subpel_range < 0) {
        why = "invalid me_quality / me_algorithm / long_range_mode / subpel_range";
        return VC1CU_ERR_ARG;
    }
    P.W = p->width;
    P.H = p->height;
    P.vw = p->display_width > 0 ? p->display_width : p->width;
    P.vh = p->display_height > 0 ? p->display_height : p->height;
    if (P.vw > P.W || P.vh > P.H) { why = "display raster larger than the coding raster"; return VC1CU_ERR_ARG; }
    P.mbw = (P.W + 15) / 16;
    P.mbh = (P.H + 15) / 16;
    P.cvw = (P.vw + 1) / 2;
    P.cvh = (P.vh + 1) / 2;
    P.right_pad = P.vw < P.mbw * 16;
    P.bottom_pad = P.vh < P.mbh * 16;
    P.cright_pad = P.cvw < P.mbw * 8;
    P.cbottom_pad = P.cvh < P.mbh * 8;
    P.pq = p->pqindex;
    P.halfqp = p->halfqp != 0;
    P.nonuniform = p->nonuniform != 0;
    P.range = p->search_range;
    P.local_range = std::min(p->search_range, std::max(0, p->local_search_range));
    P.me_algorithm = p->me_algorithm;
    P.me_quality = p->me_quality;
    P.subpel = p->subpel != 0;
    P.fast_subpel = p->fast_subpel != 0;
    P.subpel_range = p->subpel_range;
    P.long_range_mode = p->long_range_mode;
    P.rnd = p->rnd != 0;
    P.disable_p_intra = p->disable_p_intra != 0;
    P.disable_b_intra = p->disable_b_intra != 0;
    const int r = p->search_range;
    P.mvrange = r <= 31 ? 0 : (r <= 63 ? 1 : (r <= 127 ? 2 : 3));
    P.wait_log2 = 24;
    P.withhold = 0xFFFFFFFFu;
    const double lam = 0.35 * static_cast<double>(p->pqindex);
    P.lambda = std::max(1.0, lam);
    int e = 0;
    const double fr = std::frexp(P.lambda, &e);
    P.lam_m = static_cast<uint64_t>(std::ldexp(fr, 53));
    P.lam_s = 53 - e;
    // the reference scores in long double; its significand width is the host ABI's
    P.mant_bits = std::numeric_limits<long double>::digits;
    P.distant_match_max_mae = p->distant_match_max_mae;
    P.inter_intra_threshold = p->inter_intra_threshold;
    return VC1CU_OK;
}

// lambda_me = max(1, 0.35*PQ) (encoder_motion.cpp:3459), split as lam_m * 2^-lam_s exactly
void set_lambda(PassDesc& d, int pq) {
    d.pq = pq;
    d.lambda = std::max(1.0, 0.35 * static_cast<double>(pq));
    int e = 0;
    const double fr = std::frexp(d.lambda, &e);
    d.lam_m = static_cast<uint64_t>(std::ldexp(fr, 53));
    d.lam_s = 53 - e;
}

// Work-queue table of a launch: (pass << 20) | macroblock. Inside a pass the macroblocks
// follow the wavefront order (t = x + 2y, then y); a pass at seed level L (seeded by a pass
// of the same launch at level L-1) is delayed by L * lag positions, so each item follows all
// of its dependencies. Cached per (raster, pass levels).
const uint32_t* work_items(vc1cu_ctx* c, const std::vector<int>& mbw, const std::vector<int>& mbh,
                           const std::vector<int>& level, unsigned& nitems) {
    const int n = (int)level.size();
    std::vector<int> key;
    for (int p = 0; p < n; ++p) {
        key.push_back(mbw[p]);
        key.push_back(mbh[p]);
        key.push_back(level[p]);
    }
    auto it = c->items.find(key);
    if (it != c->items.end()) {
        nitems = it->second.second;
        return it->second.first;
    }
    // Each pass's macroblocks in its own wavefront order (t = x + 2y, then y); a seeded pass runs
    // about two wavefront steps (one raster row of macroblocks) behind its seed pass. The passes'
    // lists are merged by that step, so every item's dependencies (its neighbours and its seed)
    // are handed out before it, whatever the passes' raster sizes.
    std::vector<std::vector<int>> order(n);
    long steps = 0;
    for (int p = 0; p < n; ++p) {
        const int w = mbw[p], hh = mbh[p];
        order[p].reserve((size_t)w * hh);
        for (int t = 0; t <= (w - 1) + 2 * (hh - 1); ++t)
            for (int y = 0; y < hh; ++y) {
                const int x = t - 2 * y;
                if (x >= 0 && x < w) order[p].push_back(y * w + x);
            }
        steps = std::max(steps, (long)w * hh + (long)w * level[p]);
    }
    if (c->capturing)
        throw Fail{VC1CU_ERR_STATE, "run a launch of this shape once before capturing it (its work-item table is "
                                    "built and uploaded outside the capture)"};
    std::vector<uint32_t> items;
    for (long sstep = 0; sstep < steps; ++sstep)
        for (int p = 0; p < n; ++p) {
            const long j = sstep - (long)mbw[p] * level[p];
            if (j >= 0 && j < (long)order[p].size()) items.push_back(((uint32_t)p << 20) | (uint32_t)order[p][j]);
        }
    void* d = nullptr;
    ck(cudaMalloc(&d, items.size() * sizeof(uint32_t)), "cudaMalloc(work items)");
    // Ordered on the context stream, which does not synchronise with the legacy default stream:
    // a plain cudaMemcpy from pageable memory may return before its DMA lands, and the kernel
    // that reads the table could then start first.
    ck(cudaMemcpyAsync(d, items.data(), items.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream),
       "cudaMemcpyAsync(work items)");
    ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize(work items)");  // `items` is freed on return
    nitems = (unsigned)items.size();
    c->items[key] = {static_cast<uint32_t*>(d), nitems};
    return static_cast<uint32_t*>(d);
}

int stage_max(int R) {
    int m = 32;
    const int L = (2 * R) / 8 + 1;
    if (R >= 8) m = std::max(m, L * L + 2 * L);
    const int cs = R >= 96 ? 8 : (R >= 32 ? 4 : 2);
    const int vlimit = std::min(R, std::max(8, R / 2));
    m = std::max(m, 2 * (R / cs) + 2 * (vlimit / cs));
    const int hs = R >= 96 ? 8 : (R >= 24 ? 4 : 2);
    m = std::max(m, 6 * (R / hs));
    return m;
}

FrameSlot& frame_slot(vc1cu_ctx* c, int id) {
    c->used_frames.push_back(id);
    auto it = c->frames.find(id);
    if (it == c->frames.end() || !it->second.valid) throw Fail{VC1CU_ERR_STATE, "frame slot " + std::to_string(id) + " was never uploaded"};
    return it->second;
}

ResultSlot& result_slot(vc1cu_ctx* c, int id, int mbs, bool create) {
    if (create) c->dirty_results.push_back(id);  // create: the caller writes the slot
    auto& s = c->results[id];
    if (s.valid && s.mbs == mbs) return s;
    if (!create) throw Fail{VC1CU_ERR_STATE, "result slot " + std::to_string(id) + " holds no result of this size"};
    if (s.d) cudaFree(s.d);
    s = ResultSlot{};
    const size_t n = (size_t)mbs;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = al(8 * n) + al(32 * n) + al(n) * 2 + al(8 * n) * 4 + al(n) + al(8 * n) * 2 + al(n) + al(4 * n) +
                         al(8) + al(8) + al(16) + al(40);
    ck(cudaMalloc(&s.d, bytes), "cudaMalloc(result slot)");
    s.bytes = bytes;
    ck(cudaMemsetAsync(s.d, 0, bytes, c->stream), "cudaMemsetAsync(result slot)");
    uint8_t* p = static_cast<uint8_t*>(s.d);
    auto take = [&](size_t b) { uint8_t* q = p; p += al(b); return q; };
    s.r.mvs = (int2*)take(8 * n);
    s.r.bmv = (int2*)take(32 * n);
    s.r.use4 = take(n);
    s.r.intra = take(n);
    s.r.screen = (uint64_t*)take(8 * n);
    s.r.ratio = (double*)take(8 * n);
    s.r.dl = (double*)take(8 * n);
    s.r.dc = (double*)take(8 * n);
    s.r.dd = take(n);
    s.r.chosen = (uint64_t*)take(8 * n);
    s.r.temporal = (uint64_t*)take(8 * n);
    s.r.flags = take(n);
    s.r.done = (uint32_t*)take(4 * n);
    s.r.global = (int*)take(8);
    s.r.gsad = (unsigned long long*)take(8);
    s.r.totals = (double*)take(16);
    s.r.itotals = (unsigned long long*)take(40);
    s.mbs = mbs;
    s.valid = true;
    return s;
}

// by_upload: the caller writes the slot on the upload stream (else work on the context stream
// writes it, a use of the slot).
FrameSlot& alloc_frame(vc1cu_ctx* c, int id, int w, int h, bool by_upload = false) {
    if (!by_upload) c->used_frames.push_back(id);
    auto& f = c->frames[id];
    const int py = (w + 15) & ~15, pc = (w / 2 + 15) & ~15;
    const size_t bytes = (size_t)py * h + 2 * (size_t)pc * (h / 2);
    if (!f.d || f.cap < bytes) {
        if (f.d) cudaFree(f.d);
        f.d = nullptr;
        f.cap = 0;
        void* d = nullptr;
        ck(cudaMalloc(&d, bytes), "cudaMalloc(frame)");
        f.d = static_cast<uint8_t*>(d);
        f.cap = bytes;
    }
    f.w = w;
    f.h = h;
    f.pitch_y = py;
    f.pitch_c = pc;
    f.valid = true;
    return f;
}

uint8_t* cache_frame(vc1cu_ctx* c, const uint8_t* data, int w, int h) {
    const size_t bytes = (size_t)w * h;
    const uint64_t fp = frame_fingerprint(data, bytes);
    for (auto& s : c->cache)
        if (s.valid && s.host == data && s.w == w && s.h == h && s.fp == fp) {
            s.age = ++c->age;
            return s.d;
        }
    CacheSlot* slot = &c->cache[0];
    for (auto& s : c->cache) {
        if (!s.valid) { slot = &s; break; }
        if (s.age < slot->age) slot = &s;
    }
    void* d = slot->d;
    ensure(d, slot->cap, bytes, "cudaMalloc(cached frame)");
    slot->d = static_cast<uint8_t*>(d);
    ck(cudaMemcpyAsync(slot->d, data, bytes, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(frame)");
    slot->host = data;
    slot->w = w;
    slot->h = h;
    slot->fp = fp;
    slot->age = ++c->age;
    slot->valid = true;
    c->counters.frame_uploads++;
    c->counters.frame_upload_bytes += bytes;
    return slot->d;
}

void sync_checked(vc1cu_ctx* c) {
    ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    ck(cudaGetLastError(), "kernel");
}

// kCoreAux: work timed with the core passes without counting as a core launch (sub-pel planes)
enum Family { kCore = 0, kGlobal = 1, kTotals = 2, kMc = 3, kXform = 4, kScore = 5, kB = 6, kIc = 7, kCoreAux = 8 };

cudaEvent_t take_event(vc1cu_ctx* c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    ck(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

// Brackets the launches of one kernel family with CUDA events on the context stream
// when timing is on, and counts the launches.
struct Timer {
    vc1cu_ctx* c;
    int family;
    cudaEvent_t a = nullptr;
    Timer(vc1cu_ctx* cc, int f) : c(cc), family(f) {
        if (c->timing && !c->capturing) {
            a = take_event(c);
            ck(cudaEventRecord(a, c->stream), "cudaEventRecord");
        }
    }
    void stop(int launches) {
        c->counters.kernel_launches += (uint64_t)launches;
        if (!a) return;
        cudaEvent_t b = take_event(c);
        ck(cudaEventRecord(b, c->stream), "cudaEventRecord");
        c->pending.push_back({a, b, family});
        a = nullptr;
    }
};

void collect_timing(vc1cu_ctx* c) {
    if (c->pending.empty()) return;
    ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    for (auto& t : c->pending) {
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, t.a, t.b), "cudaEventElapsedTime");
        switch (t.family) {
            case kCore: c->tsum.core_ms += ms; c->tsum.core_launches++; break;
            case kCoreAux: c->tsum.core_ms += ms; break;
            case kGlobal: c->tsum.global_ms += ms; break;
            case kTotals: c->tsum.totals_ms += ms; break;
            case kMc: c->tsum.mc_ms += ms; break;
            case kXform: c->tsum.xform_ms += ms; c->tsum.xform_launches++; break;
            case kB: c->tsum.b_ms += ms; break;
            case kIc: c->tsum.ic_ms += ms; break;
            default: break;
        }
        c->event_pool.push_back(t.a);
        c->event_pool.push_back(t.b);
    }
    c->pending.clear();
}

// Pinned staging for host->device launch descriptors: the next buffer of the ring, once its
// previous copy is done. The caller copies out of it on the context stream, then staging_mark.
void* staging(vc1cu_ctx* c, size_t bytes) {
    if (c->capturing) {
        // a captured copy reads its source at every launch of the graph: a buffer of its own
        void* h = nullptr;
        ck(cudaMallocHost(&h, bytes), "cudaMallocHost(captured staging)");
        c->capture_hold.push_back(h);
        return h;
    }
    const int i = c->staging_next;
    c->staging_next = (i + 1) % vc1cu_ctx::kStagingRing;
    auto& b = c->staging_ring[i];
    if (b.done) ck(cudaEventSynchronize(b.done), "cudaEventSynchronize(staging)");
    if (b.cap < bytes) {
        if (b.h) cudaFreeHost(b.h);
        b.h = nullptr;
        b.cap = 0;
        ck(cudaMallocHost(&b.h, bytes), "cudaMallocHost(staging)");
        b.cap = bytes;
    }
    if (!b.done) ck(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming), "cudaEventCreate(staging)");
    c->staging_cur = i;
    return b.h;
}

// Records the copy out of the buffer the last staging() call handed out.
void staging_mark(vc1cu_ctx* c) {
    if (c->capturing) return;
    ck(cudaEventRecord(c->staging_ring[c->staging_cur].done, c->stream), "cudaEventRecord(staging)");
}

int score_common(vc1cu_ctx* c, const DevParams& P, const ScoreArgs& a, const vc1cu_mv* cands, size_t n, uint64_t* costs) {
    const size_t cb = n * sizeof(int2), ob = n * sizeof(unsigned long long);
    ensure(c->d_scratch, c->scratch_cap, cb + ob + 256, "cudaMalloc(candidates)");
    int2* dc = static_cast<int2*>(c->d_scratch);
    unsigned long long* dout = reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(c->d_scratch) + ((cb + 255) & ~size_t(255)));
    const auto t0 = std::chrono::steady_clock::now();
    ck(cudaMemcpyAsync(dc, cands, cb, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(candidates)");
    Timer tm(c, kScore);
    launch_score(P, a, dc, (int)n, dout, c->stream);
    ck(cudaGetLastError(), "score_kernel launch");
    tm.stop(1);
    ck(cudaMemcpyAsync(costs, dout, ob, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(costs)");
    sync_checked(c);
    const auto t1 = std::chrono::steady_clock::now();
    c->counters.dispatches++;
    c->counters.candidates += n;
    c->counters.submit_wait_nanoseconds += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    return VC1CU_OK;
}

// Launches a batch of independent core passes (global search first for unseeded ones).
// globals_ready: the unseeded passes' global translation results are already in their slots.
// Per-pass additions of the learned form (all null for the plain passes): the candidates of a
// learned pass and where it flags its fallback macroblocks, or the flags a fallback pass
// computes (only those macroblocks), and the translation hint that replaces the global search.
struct PassExtra {
    const int2* cands = nullptr;
    uint8_t* fallback = nullptr;
    const uint8_t* only = nullptr;
    const int2* hint = nullptr;
    const unsigned long long* hint_sad = nullptr;  // the frame SAD at the hint (global_full_sad)
    const DevResult* nb = nullptr;  // no-wait pass: read the neighbours from this finished field
};

// The search configuration every pass of one launch shares (the kernel's window, bitsets and
// instantiation depend on it); the picture geometry, rounding control and quantiser may differ.
void same_search_config(const DevParams& a, const DevParams& b) {
    if (a.range != b.range || a.local_range != b.local_range || a.me_algorithm != b.me_algorithm ||
        a.me_quality != b.me_quality || a.subpel != b.subpel || a.fast_subpel != b.fast_subpel ||
        a.subpel_range != b.subpel_range || a.long_range_mode != b.long_range_mode ||
        a.disable_p_intra != b.disable_p_intra || a.distant_match_max_mae != b.distant_match_max_mae ||
        a.inter_intra_threshold != b.inter_intra_threshold)
        throw Fail{VC1CU_ERR_ARG, "passes of one launch must share the search configuration (ranges, algorithm, "
                                  "quality, sub-pel and long-range settings, thresholds)"};
}

// The autotuner's cache key of a launch: raster, ranges, algorithm and the instantiation.
std::vector<int> tune_key(const DevParams& P, int kind) { return {P.W, P.H, P.range, P.local_range, P.me_algorithm, kind}; }

// per_pass: null, or n parameter blocks (pictures of different sizes in one kCoreMulti launch).
int launch_group(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_pass* passes, int n, bool globals_ready = false,
                 const PassExtra* extra = nullptr, const vc1cu_params* per_pass = nullptr,
                 std::vector<PassDesc>* descs = nullptr) {
    DevParams P;
    std::string why;
    int rc = make_dev_params(per_pass ? per_pass : p, P, why);
    if (rc) throw Fail{rc, why};
    if (n <= 0) return VC1CU_OK;
    const bool multi = per_pass != nullptr;
    bool any_unseeded = false;
    std::vector<PassDesc> h(n);
    std::vector<int> unseeded;
    for (int i = 0; i < n; ++i) {
        const vc1cu_pass& q = passes[i];
        if (q.mode < 0 || q.mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        if (q.out_slot < 0 || q.out_slot > kInternalLast || q.seed_slot == q.out_slot)
            throw Fail{VC1CU_ERR_ARG, "invalid result slot"};
        PassDesc& d = h[i];
        d.geom = P;
        if (multi) {
            rc = make_dev_params(per_pass + i, d.geom, why);
            if (rc) throw Fail{rc, why};
            same_search_config(P, d.geom);
        }
        const int mbs = d.geom.mbw * d.geom.mbh;
        FrameSlot& fc = frame_slot(c, q.cur_id);
        FrameSlot& fr = frame_slot(c, q.ref_id);
        if (fc.w != d.geom.W || fc.h != d.geom.H || fr.w != d.geom.W || fr.h != d.geom.H)
            throw Fail{VC1CU_ERR_ARG, "P-picture reference dimensions do not match the configuration"};
        d.cur = fc.view();
        d.ref = fr.view();
        d.mode = q.mode;
        d.allow_intra = q.allow_intra != 0;
        if (q.pqindex < 0 || q.pqindex > 31) throw Fail{VC1CU_ERR_ARG, "pass pqindex must be 0 (params) or 1..31"};
        set_lambda(d, q.pqindex ? q.pqindex : d.geom.pq);
        d.seeded = q.seed_slot >= 0;
        d.seed_pass = -1;
        for (int j = 0; j < n; ++j)
            if (q.seed_slot >= 0 && passes[j].out_slot == q.seed_slot) d.seed_pass = j;
        if (d.seeded && d.seed_pass < 0) {
            ResultSlot& s = result_slot(c, q.seed_slot, mbs, false);
            d.seed_mvs = s.r.mvs;
            d.seed_bmv = s.r.bmv;
            d.seed_intra = s.r.intra;
            d.seed_dl = s.r.dl;
            d.seed_dc = s.r.dc;
            d.seed_dd = s.r.dd;
        } else if (d.seeded) {
            d.seed_mvs = nullptr;  // bound to the seeding pass's result below
        } else {
            d.seed_mvs = nullptr;
            d.seed_dl = d.seed_dc = nullptr;
            d.seed_dd = nullptr;
            any_unseeded = true;
            unseeded.push_back(i);
        }
    }
    bool learned = false;
    for (int i = 0; i < n; ++i) {
        ResultSlot& o = result_slot(c, passes[i].out_slot, h[i].geom.mbw * h[i].geom.mbh, true);
        o.mode = passes[i].mode;
        o.seeded = passes[i].seed_slot >= 0;
        o.allow_intra = passes[i].allow_intra != 0;
        h[i].out = o.r;
        h[i].cands = extra ? extra[i].cands : nullptr;
        h[i].fallback = extra ? extra[i].fallback : nullptr;
        h[i].only = extra ? extra[i].only : nullptr;
        h[i].no_wait = (extra && extra[i].nb) ? 1 : 0;
        if (h[i].no_wait) h[i].nb = *extra[i].nb;
        learned |= h[i].cands != nullptr;
    }
    if (learned) {
        for (int i = 0; i < n; ++i)
            if (!h[i].cands || h[i].seeded || h[i].mode == VC1CU_MV_MIXED || h[i].allow_intra)
                throw Fail{VC1CU_ERR_ARG, "a learned launch takes unseeded 1-MV passes without P-intra only"};
    }
    // the translation hint stands in for the global search of passes that carry one
    if (extra) {
        bool any_hint = false;
        for (int i = 0; i < n; ++i)
            if (extra[i].hint) {
                any_hint = true;
                ck(cudaMemcpyAsync(h[i].out.global, extra[i].hint, sizeof(int2), cudaMemcpyDeviceToDevice, c->stream),
                   "cudaMemcpyAsync(hint)");
                if (extra[i].hint_sad)
                    ck(cudaMemcpyAsync(h[i].out.gsad, extra[i].hint_sad, 8, cudaMemcpyDeviceToDevice, c->stream),
                       "cudaMemcpyAsync(hint sad)");
                else
                    ck(cudaMemsetAsync(h[i].out.gsad, 0, 8, c->stream), "cudaMemsetAsync(hint sad)");
            }
        if (any_hint) globals_ready = true;
    }
    // seed levels of in-launch seeds (a chain, never a cycle)
    std::vector<int> level(n, 0);
    for (int i = 0; i < n; ++i) {
        int l = 0, j = i;
        while (h[j].seed_pass >= 0) {
            j = h[j].seed_pass;
            if (++l > n) throw Fail{VC1CU_ERR_ARG, "passes of one launch seed each other in a cycle"};
        }
        level[i] = l;
        if (h[i].seed_pass >= 0) {
            const DevResult& so = h[h[i].seed_pass].out;
            h[i].seed_mvs = so.mvs;
            h[i].seed_bmv = so.bmv;
            h[i].seed_intra = so.intra;
            h[i].seed_dl = so.dl;
            h[i].seed_dc = so.dc;
            h[i].seed_dd = so.dd;
        }
    }
    // global translation search of the unseeded passes (none at --search-range 0)
    if (!globals_ready && !unseeded.empty() && P.range == 0)
        for (int k : unseeded) {
            ck(cudaMemsetAsync(h[k].out.global, 0, 8, c->stream), "cudaMemsetAsync(global)");
            ck(cudaMemsetAsync(h[k].out.gsad, 0, 8, c->stream), "cudaMemsetAsync(global)");
        }
    if (!globals_ready && !unseeded.empty() && P.range > 0) {
        const int nu = (int)unseeded.size();
        const size_t gb = gstate_bytes();
        if (c->gstates_cap < nu) {
            if (c->d_gstates) cudaFree(c->d_gstates);
            c->d_gstates = nullptr;
            c->gstates_cap = 0;
            void* d = nullptr;
            ck(cudaMalloc(&d, gb * nu), "cudaMalloc(global search state)");
            c->d_gstates = static_cast<GState*>(d);
            c->gstates_cap = nu;
        }
        uint8_t* hs = static_cast<uint8_t*>(staging(c, gb * nu));
        const int grange = std::min(P.local_range, 32);
        // states in raster-size order, so that every size's searches are one contiguous run
        std::vector<int> order(unseeded);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return h[x].geom.W != h[y].geom.W ? h[x].geom.W < h[y].geom.W : h[x].geom.H < h[y].geom.H;
        });
        for (int k = 0; k < nu; ++k) {
            const PassDesc& d = h[order[k]];
            init_gstate(reinterpret_cast<GState*>(hs + gb * k), d.cur, d.ref, grange, d.out.global, d.out.gsad);
        }
        ck(cudaMemcpyAsync(c->d_gstates, hs, gb * nu, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(gstate)");
        staging_mark(c);
        Timer tm(c, kGlobal);
        int launches = 0;
        for (int k0 = 0; k0 < nu;) {
            int k1 = k0 + 1;
            const DevParams& g0 = h[order[k0]].geom;
            while (k1 < nu && h[order[k1]].geom.W == g0.W && h[order[k1]].geom.H == g0.H) ++k1;
            launches += run_global_search(reinterpret_cast<GState*>(reinterpret_cast<uint8_t*>(c->d_gstates) + gb * k0),
                                          k1 - k0, grange, g0.W, g0.H, c->stream);
            k0 = k1;
        }
        ck(cudaGetLastError(), "global search launch");
        tm.stop(launches);
    }
    // long-range signature index of each long-range pass's reference (build_long_range_index)
    if (!unseeded.empty() && P.range > P.local_range && !learned) {
        size_t per = 0;
        for (size_t k = 0; k < unseeded.size(); ++k)
            per = std::max(per, sizeof(uint64_t) * (size_t)((h[unseeded[k]].geom.W + 7) / 8) *
                                    (size_t)((h[unseeded[k]].geom.H + 7) / 8));
        uint64_t* base = static_cast<uint64_t*>(ensure(c->d_lr, c->lr_cap, per * unseeded.size(), "cudaMalloc(long-range index)"));
        for (size_t k = 0; k < unseeded.size(); ++k) {
            PassDesc& d = h[unseeded[k]];
            const int nx = (d.geom.W + 7) / 8, ny = (d.geom.H + 7) / 8;
            d.lr_sig = base + per / sizeof(uint64_t) * k;
            d.lr_nx = nx;
            d.lr_ny = ny;
            ck(launch_lr_index(d.ref, d.geom.W, d.geom.H, const_cast<uint64_t*>(d.lr_sig), c->stream),
               "lr_index_kernel launch");
            c->counters.kernel_launches++;
        }
    }
    // window / bitset geometry
    WinCfg wc;
    if (learned) {
        wc.rw = kLearnRw;
        wc.seen_r = 0;
        wc.seen_words = 1;
        wc.keys_cap = 32;
    } else if (any_unseeded) {
        wc.rw = P.local_range + 1;
        wc.seen_r = P.local_range;
        wc.seen_words = ((2 * P.local_range + 1) * (2 * P.local_range + 1) + 31) / 32;
        wc.keys_cap = std::max(stage_max(P.local_range), 32);  // >= one warp of staged long-range keys
    } else {
        // seeded refinement stays within 3 quarter-pels of the seed; the Mixed-MV block seeds
        // add up to 8 more and their refinement 3 (samples outside the window read HBM)
        bool any_mixed = false;
        for (int i = 0; i < n; ++i) any_mixed |= passes[i].mode == VC1CU_MV_MIXED;
        wc.rw = any_mixed ? kSeededMixedRw : 4;
        wc.seen_r = 0;
        wc.seen_words = 1;
        wc.keys_cap = 32;
    }
    wc.wh = 16 + 2 * wc.rw + 3;
    wc.wp = (wc.wh + 15 + 15) & ~15;
    wc.warp_bytes = warp_bytes_for_host(wc);
    int warps = 4;
    while (warps > 1 && (size_t)warps * wc.warp_bytes > (size_t)c->max_smem) --warps;
    size_t smem = (size_t)warps * wc.warp_bytes;
    if (smem > (size_t)c->max_smem)
        throw Fail{VC1CU_ERR_UNSUPPORTED, "search window does not fit in shared memory (local range too large)"};
    // the instantiation: the code this launch's passes can reach (the kCore* flags)
    bool any_mixed_pass = false;
    for (int i = 0; i < n; ++i) any_mixed_pass |= passes[i].mode == VC1CU_MV_MIXED;
    int kind = kCoreAny;
    if (!any_unseeded) {
        kind = kCoreSeededOnly;
    } else if ((int)unseeded.size() == n) {
        kind = kCoreUnseededOnly;
        if (P.me_algorithm == 0 && P.range == P.local_range) kind |= kCoreUmhLocal;
    }
    if (!any_mixed_pass && (kind & (kCoreSeededOnly | kCoreUmhLocal))) kind |= kCoreNoMixed;
    if (P.me_quality == 2 && !P.fast_subpel && (kind & (kCoreSeededOnly | kCoreUmhLocal))) kind |= kCoreDefaultRefine;
    bool any_intra_pass = false;
    for (int i = 0; i < n; ++i) any_intra_pass |= passes[i].allow_intra != 0;
    if (!any_intra_pass && (kind & kCoreDefaultRefine)) kind |= kCoreNoIntra;
    if (learned)
        kind = kCoreUnseededOnly | kCoreLearned | kCoreNoMixed | kCoreNoIntra |
               ((P.me_quality == 2 && !P.fast_subpel) ? kCoreDefaultRefine : 0);
    if (multi) kind = kCoreMulti;
    // windows so large that a second 4-warp block cannot fit: the wide-register build costs no occupancy
    if (!(kind & kCoreSeededOnly) && 2 * 4 * (size_t)wc.warp_bytes > (size_t)c->max_smem_sm) kind |= kCoreWide;
    const void* kern = core_kernel(kind);
    // a launch shape chosen by vc1cu_autotune for this raster, search configuration and instantiation
    int tuned_blocks = 0;
    {
        c->last_tune_key = tune_key(P, kind);
        auto t = c->tuned.find(c->last_tune_key);
        if (c->tune_force.first) {
            warps = c->tune_force.first;
            tuned_blocks = c->tune_force.second;
        } else if (t != c->tuned.end()) {
            warps = t->second.first;
            tuned_blocks = t->second.second;
        }
        // a wider block of unseeded passes: their windows shrink until `warps` of them fit; a
        // candidate outside its window reads the frame in global memory, at the same result
        if ((kind & kCoreWide) && any_unseeded && !learned)
            while ((size_t)warps * wc.warp_bytes > (size_t)c->max_smem && wc.rw > kMinUnseededRw) {
                --wc.rw;
                wc.wh = 16 + 2 * wc.rw + 3;
                wc.wp = (wc.wh + 15 + 15) & ~15;
                wc.warp_bytes = warp_bytes_for_host(wc);
            }
        if (warps < 1 || warps > ((kind & kCoreWide) ? 8 : 4) || (size_t)warps * wc.warp_bytes > (size_t)c->max_smem)
            throw Fail{VC1CU_ERR_ARG, "tuned warps do not fit this instantiation"};
        smem = (size_t)warps * wc.warp_bytes;
    }
    // the windows' tensor maps (the box is this launch's final window)
    wc.tma = 0;
    if (VC1CU_WINDOW_TMA && wc.wp <= 256 && wc.wh <= 256) {
        wc.tma = 1;
        for (int i = 0; i < n; ++i)
            h[i].ref_tma = encode_window_map(h[i].ref_tmap, h[i].ref.y, h[i].geom.W, h[i].geom.H, h[i].ref.pitch_y, wc.wp,
                                             wc.wh)
                               ? 1
                               : 0;
    }
    // Sub-pel prediction planes, one set per (reference, rounding, filter) of the launch, built
    // before it on the context stream: every candidate's interpolated rows are then read, not
    // recomputed per candidate and macroblock (the phases each set needs: all 15 for the bicubic
    // modes, whose SAD batches may score odd seeds; the three half-pel ones for the bilinear mode,
    // which rejects odd vectors).
    if (VC1CU_SUBPEL_PLANES && P.subpel) {
        struct Key {
            const uint8_t* ref;
            int W, H, pitch, rnd, bil;
            uint32_t mask;
            size_t off, stride;
            int opitch;
        };
        std::vector<Key> keys;
        std::vector<int> key_of(n);
        for (int i = 0; i < n; ++i) {
            const int bil = h[i].mode == VC1CU_MV_HPEL_BILINEAR ? 1 : 0;
            const uint32_t mask = bil ? 0x504u : 0xFFFEu;
            int k = 0;
            while (k < (int)keys.size() && !(keys[k].ref == h[i].ref.y && keys[k].rnd == h[i].geom.rnd && keys[k].bil == bil))
                ++k;
            if (k == (int)keys.size())
                keys.push_back(Key{h[i].ref.y, h[i].geom.W, h[i].geom.H, h[i].ref.pitch_y, h[i].geom.rnd, bil, 0u, 0, 0, 0});
            keys[k].mask |= mask;
            key_of[i] = k;
        }
        size_t total = 0;
        for (auto& k : keys) {
            k.opitch = ((k.W + 2 * kSubpelBorder + 15) & ~15) + 16;
            k.stride = (size_t)k.opitch * (size_t)(k.H + 2 * kSubpelBorder);
            k.off = total;
            total += 16 * k.stride;
        }
        if (c->capturing && c->sp_cap < total)
            throw Fail{VC1CU_ERR_STATE, "run this launch once before capturing it (sub-pel plane pool too small)"};
        uint8_t* pool = static_cast<uint8_t*>(ensure(c->d_sp, c->sp_cap, total, "cudaMalloc(sub-pel planes)"));
        // timed with the core passes: the planes carry part of their interpolation work
        Timer tm(c, kCoreAux);
        for (const auto& k : keys)
            ck(launch_subpel_planes(k.ref, k.pitch, k.W, k.H, k.rnd, k.bil, k.mask, pool + k.off, k.opitch, kSubpelBorder,
                                    (long long)k.stride, c->stream),
               "subpel_plane_kernel launch");
        c->counters.kernel_launches += keys.size();
        tm.stop(0);
        for (int i = 0; i < n; ++i) {
            const Key& k = keys[key_of[i]];
            h[i].sp_planes = pool + k.off;
            h[i].sp_pitch = k.opitch;
            h[i].sp_border = kSubpelBorder;
            h[i].sp_stride = (long long)k.stride;
        }
    }
    // pass descriptors, ordered on the context stream after any launch still reading the
    // previous ones
    if (c->passes_cap < n) {
        if (c->d_passes) cudaFree(c->d_passes);
        c->d_passes = nullptr;
        c->passes_cap = 0;
        void* d = nullptr;
        ck(cudaMalloc(&d, sizeof(PassDesc) * n), "cudaMalloc(pass descriptors)");
        c->d_passes = static_cast<PassDesc*>(d);
        c->passes_cap = n;
    }
    {
        void* hp = staging(c, sizeof(PassDesc) * n);
        std::memcpy(hp, h.data(), sizeof(PassDesc) * n);
        ck(cudaMemcpyAsync(c->d_passes, hp, sizeof(PassDesc) * n, cudaMemcpyHostToDevice, c->stream),
           "cudaMemcpyAsync(pass descriptors)");
        staging_mark(c);
    }
    ck(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "cudaFuncSetAttribute");
    int per_sm = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem), "occupancy");
    per_sm = std::max(per_sm, 1);
    if (tuned_blocks > 0) per_sm = std::min(per_sm, tuned_blocks);
    long items = 0;
    for (int i = 0; i < n; ++i) items += (long)h[i].geom.mbw * h[i].geom.mbh;
    const long need = (items + warps - 1) / warps;
    const int grid = (int)std::max(1L, std::min<long>((long)per_sm * c->sm_count, need));
    uint32_t epoch = 0;
    if (c->capturing) {
        // a replayed graph cannot count epochs: the flags restart from zero at every launch
        epoch = 0xFFFFFFFFu;
        for (int i = 0; i < n; ++i)
            ck(cudaMemsetAsync(h[i].out.done, 0, sizeof(uint32_t) * h[i].geom.mbw * h[i].geom.mbh, c->stream),
               "cudaMemsetAsync(done flags)");
    } else {
        if (++c->epoch == 0 || c->epoch == 0xFFFFFFFFu) c->epoch = 1;
        epoch = c->epoch;
    }
    // only the work counter restarts: an error (and its abort flag) stays until check_status reports it
    ck(cudaMemsetAsync(reinterpret_cast<char*>(c->d_status) + offsetof(LaunchStatus, queue), 0, sizeof(unsigned int),
                       c->stream),
       "cudaMemsetAsync(status)");
    {
        Timer tm(c, kCore);
        unsigned nitems = 0;
        std::vector<int> mbw(n), mbh(n);
        for (int i = 0; i < n; ++i) {
            mbw[i] = h[i].geom.mbw;
            mbh[i] = h[i].geom.mbh;
        }
        const uint32_t* items = work_items(c, mbw, mbh, level, nitems);
        P.wait_log2 = c->wait_log2;
        P.withhold = c->withhold_next;
        c->withhold_next = 0xFFFFFFFFu;
        ck(launch_core(kind, grid, 32 * warps, smem, c->stream, P, c->d_passes, n, items, nitems, wc, epoch,
                       c->d_status),
           "core_pass_kernel launch");
        tm.stop(1);
    }
    {
        Timer tm(c, kTotals);
        totals_kernel<<<n, 256, 0, c->stream>>>(P, c->d_passes, n);
        ck(cudaGetLastError(), "totals_kernel launch");
        tm.stop(1);
    }
    c->counters.dispatches++;
    c->counters.macroblocks_analysed += (uint64_t)items;
    if (descs) *descs = h;
    return VC1CU_OK;
}

// Launches a batch of core passes. Passes of different kinds (seeded or not, MV mode, P-intra)
// run as separate launches in the order the kinds first appear: each launch then executes
// one code path, whose instructions stay in the SMs' instruction caches. A batch in which a
// pass is seeded by another pass of the same batch runs as one launch.
int launch_passes(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_pass* passes, int n) {
    bool chained = false;
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            if (j < i && passes[j].out_slot == passes[i].out_slot)
                throw Fail{VC1CU_ERR_ARG, "two passes write one result slot"};
            if (passes[i].seed_slot >= 0 && passes[j].out_slot == passes[i].seed_slot) chained = true;
        }
    }
    if (n <= 1 || chained) return launch_group(c, p, passes, n);
    std::vector<int> keys;
    std::vector<std::vector<vc1cu_pass>> groups;
    for (int i = 0; i < n; ++i) {
        const int key = (passes[i].seed_slot >= 0 ? 8 : 0) + 2 * passes[i].mode + (passes[i].allow_intra ? 1 : 0);
        size_t g = 0;
        while (g < keys.size() && keys[g] != key) ++g;
        if (g == keys.size()) {
            keys.push_back(key);
            groups.emplace_back();
        }
        groups[g].push_back(passes[i]);
    }
    // The global translation search depends only on (cur, ref) at the call's range, so passes of
    // one picture pair in different groups (a B picture's quarter-pel and bilinear passes) share
    // one search, as the reference shares it through BSearchReuse (encoder_motion.cpp:90-95).
    DevParams P;
    std::string why;
    const int rc = make_dev_params(p, P, why);
    if (rc) throw Fail{rc, why};
    const int mbs = P.mbw * P.mbh;
    std::vector<int> first_of;  // per unseeded pass: index of the pass whose search it reuses
    std::vector<int> un;
    for (int i = 0; i < n; ++i) {
        if (passes[i].seed_slot >= 0) continue;
        int f = i;
        for (int j : un)
            if (passes[j].cur_id == passes[i].cur_id && passes[j].ref_id == passes[i].ref_id) {
                f = j;
                break;
            }
        if (f == i) un.push_back(i);
        first_of.push_back(f);
    }
    std::vector<int> unseeded_idx;
    for (int i = 0; i < n; ++i)
        if (passes[i].seed_slot < 0) unseeded_idx.push_back(i);
    if (!un.empty()) {
        std::vector<DevResult*> outs(n, nullptr);
        for (int i : unseeded_idx) outs[i] = &result_slot(c, passes[i].out_slot, mbs, true).r;
        if (P.range == 0) {
            for (int i : unseeded_idx) {
                ck(cudaMemsetAsync(outs[i]->global, 0, 8, c->stream), "cudaMemsetAsync(global)");
                ck(cudaMemsetAsync(outs[i]->gsad, 0, 8, c->stream), "cudaMemsetAsync(global)");
            }
        } else {
            const int nu = (int)un.size();
            const size_t gb = gstate_bytes();
            if (c->gstates_cap < nu) {
                if (c->d_gstates) cudaFree(c->d_gstates);
                c->d_gstates = nullptr;
                c->gstates_cap = 0;
                void* d = nullptr;
                ck(cudaMalloc(&d, gb * nu), "cudaMalloc(global search state)");
                c->d_gstates = static_cast<GState*>(d);
                c->gstates_cap = nu;
            }
            uint8_t* hs = static_cast<uint8_t*>(staging(c, gb * nu));
            const int grange = std::min(P.local_range, 32);
            for (int k = 0; k < nu; ++k) {
                const vc1cu_pass& q = passes[un[k]];
                FrameSlot& fc = frame_slot(c, q.cur_id);
                FrameSlot& fr = frame_slot(c, q.ref_id);
                if (fc.w != P.W || fc.h != P.H || fr.w != P.W || fr.h != P.H)
                    throw Fail{VC1CU_ERR_ARG, "P-picture reference dimensions do not match the configuration"};
                init_gstate(reinterpret_cast<GState*>(hs + gb * k), fc.view(), fr.view(), grange, outs[un[k]]->global,
                            outs[un[k]]->gsad);
            }
            ck(cudaMemcpyAsync(c->d_gstates, hs, gb * nu, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(gstate)");
            staging_mark(c);
            Timer tm(c, kGlobal);
            const int launches = run_global_search(c->d_gstates, nu, grange, P.W, P.H, c->stream);
            ck(cudaGetLastError(), "global search launch");
            tm.stop(launches);
            // the passes that reuse a search take its result, in one launch (not one copy each)
            std::vector<GlobalCopy> copies;
            for (size_t k = 0; k < unseeded_idx.size(); ++k) {
                const int i = unseeded_idx[k], f = first_of[k];
                if (f != i) copies.push_back(GlobalCopy{outs[f]->global, outs[f]->gsad, outs[i]->global, outs[i]->gsad});
            }
            if (!copies.empty()) {
                const size_t cb = sizeof(GlobalCopy) * copies.size();
                void* dcp = ensure(c->d_gcopy, c->gcopy_cap, cb, "cudaMalloc(global copies)");
                void* hc = staging(c, cb);
                std::memcpy(hc, copies.data(), cb);
                ck(cudaMemcpyAsync(dcp, hc, cb, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(global copies)");
                staging_mark(c);
                Timer tf(c, kGlobal);
                ck(launch_global_fanout(static_cast<const GlobalCopy*>(dcp), (int)copies.size(), c->stream),
                   "global copy launch");
                tf.stop(1);
            }
        }
    }
    for (const auto& g : groups) launch_group(c, p, g.data(), (int)g.size(), true);
    return VC1CU_OK;
}

// Records one event after the work the current call enqueued and hands it to every slot the
// call wrote.
void stamp_written(vc1cu_ctx* c) {
    if (c->capturing) {
        // the graph's launches stamp these slots (vc1cu_graph_launch)
        auto add = [](std::vector<int>& to, std::vector<int>& from) {
            to.insert(to.end(), from.begin(), from.end());
            from.clear();
        };
        add(c->capture_results, c->dirty_results);
        add(c->capture_bresults, c->dirty_bresults);
        add(c->capture_frames, c->used_frames);
        return;
    }
    if (c->dirty_results.empty() && c->dirty_bresults.empty() && c->used_frames.empty()) return;
    auto w = std::make_shared<Written>();
    ck(cudaEventCreateWithFlags(&w->e, cudaEventDisableTiming), "cudaEventCreate(slot)");
    ck(cudaEventRecord(w->e, c->stream), "cudaEventRecord(slot)");
    for (int id : c->dirty_results) {
        auto it = c->results.find(id);
        if (it != c->results.end()) it->second.written = w;
    }
    for (int id : c->dirty_bresults) {
        auto it = c->bresults.find(id);
        if (it != c->bresults.end()) it->second.written = w;
    }
    for (int id : c->used_frames) {
        auto it = c->frames.find(id);
        if (it != c->frames.end()) it->second.last_use = w;
    }
    c->dirty_results.clear();
    c->dirty_bresults.clear();
    c->used_frames.clear();
}

// Ends an open capture after a failed call and drops what it held, so the stream is usable again.
void abort_capture(vc1cu_ctx* c) {
    if (!c || !c->capturing) return;
    c->capturing = false;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c->stream, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    for (void* h : c->capture_hold) cudaFreeHost(h);
    c->capture_hold.clear();
    c->capture_results.clear();
    c->capture_bresults.clear();
    c->capture_frames.clear();
}

// Orders the read stream after the work that last wrote a slot (after everything enqueued so far
// when the slot has no record).
void read_after(vc1cu_ctx* c, const std::shared_ptr<Written>& w) {
    if (w) {
        ck(cudaStreamWaitEvent(c->rstream, w->e, 0), "cudaStreamWaitEvent(read)");
        return;
    }
    cudaEvent_t e = take_event(c);
    ck(cudaEventRecord(e, c->stream), "cudaEventRecord(read)");
    ck(cudaStreamWaitEvent(c->rstream, e, 0), "cudaStreamWaitEvent(read)");
    c->event_pool.push_back(e);
}

// A whole slot allocation copied to the pinned read buffer in one transfer (on the read stream,
// after read_after); the fields are then unpacked on the host.
const uint8_t* read_slot_bytes(vc1cu_ctx* c, const void* d, size_t bytes) {
    if (c->read_cap < bytes) {
        if (c->h_read) cudaFreeHost(c->h_read);
        c->h_read = nullptr;
        c->read_cap = 0;
        ck(cudaMallocHost(&c->h_read, bytes), "cudaMallocHost(read buffer)");
        c->read_cap = bytes;
    }
    ck(cudaMemcpyAsync(c->h_read, d, bytes, cudaMemcpyDeviceToHost, c->rstream), "cudaMemcpyAsync(result)");
    return static_cast<const uint8_t*>(c->h_read);
}

void read_sync(vc1cu_ctx* c);

void read_sync(vc1cu_ctx* c) {
    ck(cudaStreamSynchronize(c->rstream), "cudaStreamSynchronize(read)");
    ck(cudaGetLastError(), "kernel");
}

int check_status(vc1cu_ctx* c);

// The launch status as of the slot's writer (later launches may already have added to it); a
// recorded error is reported and cleared as check_status does.
void check_status_read(vc1cu_ctx* c, const std::shared_ptr<Written>& w) {
    read_after(c, w);
    LaunchStatus st{};
    ck(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->rstream), "cudaMemcpyAsync(status)");
    read_sync(c);
    if (st.error) check_status(c);
}

int check_status(vc1cu_ctx* c) {
    LaunchStatus st{};
    ck(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(status)");
    sync_checked(c);
    if (st.error) {
        ck(cudaMemsetAsync(c->d_status, 0, sizeof(LaunchStatus), c->stream), "cudaMemsetAsync(status)");
        sync_checked(c);
        std::string where;
        if (st.tcode) {
            const unsigned code = st.tcode - 1u;
            where = "; first: pass " + std::to_string(code >> 20) + " of its launch, macroblock " +
                    std::to_string(code & 0xFFFFFu) + ", lanes still waiting 0x" + [&] {
                        char b[16];
                        std::snprintf(b, sizeof b, "%x", st.tmask);
                        return std::string(b);
                    }();
        }
        throw Fail{st.error, "a wavefront wait timed out on the device (" + std::to_string(st.timeouts) + " waits" +
                                 where + ")"};
    }
    return VC1CU_OK;
}

void read_result(vc1cu_ctx* c, const ResultSlot& s, vc1cu_panalysis* out) {
    const size_t n = (size_t)s.mbs;
    stamp_written(c);  // slots this call wrote
    read_after(c, s.written);
    const uint8_t* hb = read_slot_bytes(c, s.d, s.bytes);
    read_sync(c);
    const uint8_t* base = static_cast<const uint8_t*>(s.d);
    auto cp = [&](void* dst, const void* src, size_t b) {
        if (dst) std::memcpy(dst, hb + (static_cast<const uint8_t*>(src) - base), b);
    };
    cp(out->mvs, s.r.mvs, 8 * n);
    cp(out->block_mvs, s.r.bmv, 32 * n);
    cp(out->use_4mv, s.r.use4, n);
    cp(out->use_intra, s.r.intra, n);
    cp(out->screen_sads, s.r.screen, 8 * n);
    cp(out->inter_intra_cost_ratio, s.r.ratio, 8 * n);
    cp(out->distant_local_mae, s.r.dl, 8 * n);
    cp(out->distant_candidate_mae, s.r.dc, 8 * n);
    cp(out->distant_match_decision, s.r.dd, n);
    double tot[2];
    unsigned long long it[5], gsad;
    int g[2];
    cp(tot, s.r.totals, 16);
    cp(it, s.r.itotals, 40);
    cp(g, s.r.global, 8);
    cp(&gsad, s.r.gsad, 8);
    out->mean_abs_residual = tot[0];
    out->rate_complexity = tot[1];
    out->motion_sad = it[0];
    out->moved_macroblocks = it[1];
    out->fractional_chroma_macroblocks = it[2];
    out->four_mv_macroblocks = it[3];
    out->intra_macroblocks = it[4];
    out->global_dx = g[0];
    out->global_dy = g[1];
    out->global_full_sad = gsad;
}

BSlot& bresult_slot(vc1cu_ctx* c, int id, int mbs) {
    c->dirty_bresults.push_back(id);
    auto& s = c->bresults[id];
    if (s.d && s.mbs == mbs) {
        s.valid = true;
        return s;
    }
    if (s.d) cudaFree(s.d);
    s = BSlot{};
    const size_t n = (size_t)mbs;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = al(n) * 3 + al(8 * n) * 7 + al(16 * n) + al(4 * n) + al(8 * kBTotCount) + al(16);
    ck(cudaMalloc(&s.d, bytes), "cudaMalloc(B result slot)");
    s.bytes = bytes;
    ck(cudaMemsetAsync(s.d, 0, bytes, c->stream), "cudaMemsetAsync(B result slot)");
    uint8_t* p = static_cast<uint8_t*>(s.d);
    auto take = [&](size_t b) { uint8_t* q = p; p += al(b); return q; };
    s.r.modes = take(n);
    s.r.fmv = (int2*)take(8 * n);
    s.r.bmv = (int2*)take(8 * n);
    s.r.ratio = (double*)take(8 * n);
    s.r.fdl = (double*)take(8 * n);
    s.r.fdc = (double*)take(8 * n);
    s.r.fdd = take(n);
    s.r.bdl = (double*)take(8 * n);
    s.r.bdc = (double*)take(8 * n);
    s.r.bdd = take(n);
    s.r.cost = (uint4*)take(16 * n);
    s.r.intra = (uint32_t*)take(4 * n);
    s.r.itotals = (unsigned long long*)take(8 * kBTotCount);
    s.r.totals = (double*)take(16);
    s.mbs = mbs;
    s.valid = true;
    return s;
}

// A core result slot usable as one direction of a B picture: an unseeded pass with P-intra
// off in the B picture's mode (analyze_b_picture_mode, encoder_motion.cpp:800-801).
const ResultSlot& b_direction(vc1cu_ctx* c, int slot, int mbs, int mode, const char* what) {
    const ResultSlot& s = result_slot(c, slot, mbs, false);
    if (s.mode != mode || s.seeded || s.allow_intra)
        throw Fail{VC1CU_ERR_ARG, std::string(what) + " slot does not hold an unseeded, P-intra-off core pass of this mode"};
    return s;
}

// Decision stage of a batch of B pictures (b_cost_kernel + b_decide_kernel).
void launch_b(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_bpass* b, int n, int max_out) {
    DevParams P;
    std::string why;
    const int rc = make_dev_params(p, P, why);
    if (rc) throw Fail{rc, why};
    if (n <= 0) return;
    const int mbs = P.mbw * P.mbh;
    std::vector<BDesc> h(n);
    for (int i = 0; i < n; ++i) {
        const vc1cu_bpass& q = b[i];
        if (!((q.fraction_den == 2 && q.fraction_num == 1) ||
              (q.fraction_den == 3 && (q.fraction_num == 1 || q.fraction_num == 2))))
            throw Fail{VC1CU_ERR_ARG, "unsupported B-picture temporal fraction (1/2, 1/3 and 2/3 are)"};
        if (q.mode < 0 || q.mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        if (q.pqindex < 0 || q.pqindex > 31) throw Fail{VC1CU_ERR_ARG, "pass pqindex must be 0 (params) or 1..31"};
        if (q.out_bslot < 0 || q.out_bslot > max_out) throw Fail{VC1CU_ERR_ARG, "B-result slot out of range"};
        for (int j = 0; j < i; ++j)
            if (b[j].out_bslot == q.out_bslot) throw Fail{VC1CU_ERR_ARG, "two B pictures of one call share a result slot"};
        FrameSlot& fc = frame_slot(c, q.cur_id);
        FrameSlot& fp = frame_slot(c, q.past_id);
        FrameSlot& ff = frame_slot(c, q.future_id);
        if (fc.w != P.W || fc.h != P.H || fp.w != P.W || fp.h != P.H || ff.w != P.W || ff.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "B-picture reference dimensions do not match the configuration"};
        const ResultSlot& fs = b_direction(c, q.fwd_slot, mbs, q.mode, "forward");
        const ResultSlot& bs = b_direction(c, q.bwd_slot, mbs, q.mode, "backward");
        const ResultSlot& as = result_slot(c, q.anchor_slot, mbs, false);
        BDesc& d = h[i];
        d.cur = fc.view();
        d.past = fp.view();
        d.future = ff.view();
        d.fmv = fs.r.mvs;
        d.bmv = bs.r.mvs;
        d.fscreen = fs.r.screen;
        d.bscreen = bs.r.screen;
        d.fdl = fs.r.dl;
        d.fdc = fs.r.dc;
        d.fdd = fs.r.dd;
        d.bdl = bs.r.dl;
        d.bdc = bs.r.dc;
        d.bdd = bs.r.dd;
        d.anchor = as.r.mvs;
        d.anchor4 = as.r.use4;
        d.bfrac = q.fraction_den == 2 ? 128 : (q.fraction_num == 1 ? 85 : 170);
        d.below_half = 2 * q.fraction_num < q.fraction_den;
        d.mode = q.mode;
        // lambda = max(1, 0.45*PQ) (encoder_motion.cpp:919), split as lam_m * 2^-lam_s exactly
        const int pq = q.pqindex ? q.pqindex : P.pq;
        const double lambda = std::max(1.0, 0.45 * static_cast<double>(pq));
        int e = 0;
        const double fr = std::frexp(lambda, &e);
        d.lam_m = static_cast<uint64_t>(std::ldexp(fr, 53));
        d.lam_s = 53 - e;
        d.intra_guard = static_cast<uint64_t>(std::llround(lambda * 72.0));
    }
    for (int i = 0; i < n; ++i) {
        BSlot& o = bresult_slot(c, b[i].out_bslot, mbs);
        o.mode = b[i].mode;
        h[i].out = o.r;
    }
    if (c->bdescs_cap < n) {
        if (c->d_bdescs) cudaFree(c->d_bdescs);
        c->d_bdescs = nullptr;
        c->bdescs_cap = 0;
        void* d = nullptr;
        ck(cudaMalloc(&d, sizeof(BDesc) * n), "cudaMalloc(B descriptors)");
        c->d_bdescs = static_cast<BDesc*>(d);
        c->bdescs_cap = n;
    }
    void* hp = staging(c, sizeof(BDesc) * n);
    std::memcpy(hp, h.data(), sizeof(BDesc) * n);
    ck(cudaMemcpyAsync(c->d_bdescs, hp, sizeof(BDesc) * n, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(B descriptors)");
    staging_mark(c);
    Timer tm(c, kB);
    ck(launch_bpictures(P, c->d_bdescs, n, c->stream), "B-picture kernel launch");
    tm.stop(2);
    c->counters.macroblocks_analysed += (uint64_t)mbs * (uint64_t)n;
}

// The host half of Vc1Encoder::estimate_intensity_comp (encoder_motion_compensation.cpp:321-347):
// the long double least-squares fit from the exact integer sums, then the pair of smallest
// sample SAD in the fit's 7x7 neighbourhood, read from the device's table of every pair.
vc1cu_intensity ic_decide(const unsigned long long sums[5], const unsigned long long* table) {
    vc1cu_intensity out{0, 32, 0};  // IntensityComp{}: off, LUMSCALE 32, LUMSHIFT 0
    const uint64_t n = sums[0];
    if (n < 16) return out;
    const long double sx = (long double)sums[1], sy = (long double)sums[2], sxx = (long double)sums[3],
                      sxy = (long double)sums[4];
    const long double denom = static_cast<long double>(n) * sxx - sx * sx;
    long double a = 1.0L, b = 0.0L;
    if (std::fabs(denom) > 1e-9L) {
        a = (static_cast<long double>(n) * sxy - sx * sy) / denom;
        b = (sy - a * sx) / static_cast<long double>(n);
    } else {
        b = (sy - sx) / static_cast<long double>(n);
    }
    const int ls = std::clamp(static_cast<int>(std::llround(a * 64.0L - 32.0L)), 1, 63);
    const int sh = std::clamp(static_cast<int>(std::llround(b)), -32, 31);
    uint64_t best = std::numeric_limits<uint64_t>::max();
    int best_ls = 32, best_sh = 0;
    for (int l = std::max(1, ls - 3); l <= std::min(63, ls + 3); ++l)
        for (int z = std::max(-32, sh - 3); z <= std::min(31, sh + 3); ++z) {
            const uint64_t sad = table[(l - 1) * 64 + (z + 32)];
            if (sad < best || (sad == best && std::abs(l - 32) + std::abs(z) < std::abs(best_ls - 32) + std::abs(best_sh))) {
                best = sad;
                best_ls = l;
                best_sh = z;
            }
        }
    if (best_ls == 32 && best_sh == 0) return out;
    out.enabled = 1;
    out.lumscale = best_ls;
    out.lumshift = best_sh < 0 ? best_sh + 64 : best_sh;
    return out;
}

struct IcJob {
    DevFrame cur, ref;
    const int2* mvs;
};

constexpr size_t kIcTable = 63 * 64;                              // SAD of every (LUMSCALE, LUMSHIFT)
constexpr size_t kIcHostBytes = (kIcTable + 5) * sizeof(unsigned long long);  // one picture's table + sums

// Device part of the estimate for a batch of pictures (one set of launches) on the context
// stream, its tables and sums copied into ticket t's pinned buffer; t.done follows the copies.
void ic_enqueue(vc1cu_ctx* c, const DevParams& P, const std::vector<IcJob>& jobs, vc1cu_ctx::IcTicket& t) {
    const int n = (int)jobs.size();
    t.n = n;
    if (!n) return;
    const size_t sb = ic_scratch_bytes(), db = (ic_desc_bytes() + 15) & ~size_t(15);
    uint8_t* scratch = static_cast<uint8_t*>(ensure(c->d_ic, c->ic_cap, sb * n, "cudaMalloc(intensity scratch)"));
    void* ddesc = ensure(c->d_icdesc, c->icdesc_cap, db * n, "cudaMalloc(intensity descriptors)");
    if (t.cap < kIcHostBytes * n) {
        if (t.done) ck(cudaEventSynchronize(t.done), "cudaEventSynchronize(intensity)");
        if (t.h) cudaFreeHost(t.h);
        t.h = nullptr;
        t.cap = 0;
        ck(cudaMallocHost(&t.h, kIcHostBytes * n), "cudaMallocHost(intensity results)");
        t.cap = kIcHostBytes * n;
    }
    if (!t.done) ck(cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming), "cudaEventCreate(intensity)");
    uint8_t* hp = static_cast<uint8_t*>(staging(c, db * n));
    for (int i = 0; i < n; ++i) ic_fill_desc(hp + db * i, jobs[i].cur, jobs[i].ref, jobs[i].mvs, scratch + sb * i);
    ck(cudaMemcpyAsync(ddesc, hp, db * n, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(intensity descriptors)");
    staging_mark(c);
    // every picture's histogram and sums start at zero (one fill of the whole scratch)
    ck(cudaMemsetAsync(scratch, 0, sb * n, c->stream), "cudaMemsetAsync(intensity scratch)");
    {
        Timer tm(c, kIc);
        ck(launch_ic_estimate(static_cast<const IcDesc*>(ddesc), n, P.W, P.H, c->stream), "intensity estimate launch");
        tm.stop(3);
    }
    uint8_t* hb = static_cast<uint8_t*>(t.h);
    for (int i = 0; i < n; ++i) {
        ck(cudaMemcpyAsync(hb + kIcHostBytes * i, scratch + sb * i + ic_table_offset(), kIcTable * 8,
                           cudaMemcpyDeviceToHost, c->stream),
           "cudaMemcpyAsync(intensity table)");
        ck(cudaMemcpyAsync(hb + kIcHostBytes * i + kIcTable * 8, scratch + sb * i + ic_sums_offset(), 40,
                           cudaMemcpyDeviceToHost, c->stream),
           "cudaMemcpyAsync(intensity sums)");
    }
    ck(cudaEventRecord(t.done, c->stream), "cudaEventRecord(intensity)");
}

// The host part, once ticket t's copies are done: the long double fit and the 7x7 choice.
void ic_finish(vc1cu_ctx* c, vc1cu_ctx::IcTicket& t, vc1cu_intensity* out) {
    if (!t.n) return;
    ck(cudaEventSynchronize(t.done), "cudaEventSynchronize(intensity)");
    ck(cudaGetLastError(), "kernel");
    const uint8_t* hb = static_cast<const uint8_t*>(t.h);
    for (int i = 0; i < t.n; ++i) {
        const auto* table = reinterpret_cast<const unsigned long long*>(hb + kIcHostBytes * i);
        out[i] = ic_decide(table + kIcTable, table);
    }
}

// Device part of the estimate for a batch of pictures (one set of launches), then the host part.
void ic_estimate(vc1cu_ctx* c, const DevParams& P, const std::vector<IcJob>& jobs, vc1cu_intensity* out) {
    ic_enqueue(c, P, jobs, c->ic_sync);  // the call waits for its own copies before returning
    ic_finish(c, c->ic_sync, out);
}

// Vc1Encoder::global_motion_search (encoder_motion.cpp:2076-2141) of one picture pair at
// min(range, 32), on the device; the result lands in result slot `slot`'s global fields.
void global_search_one(vc1cu_ctx* c, const DevFrame& cur, const DevFrame& ref, int range, int W, int H, int slot, int mbs,
                       int* dx, int* dy, uint64_t* sad) {
    ResultSlot& s = result_slot(c, slot, mbs, true);
    const size_t gb = gstate_bytes();
    if (c->gstates_cap < 1) {
        void* d = nullptr;
        ck(cudaMalloc(&d, gb), "cudaMalloc(global search state)");
        c->d_gstates = static_cast<GState*>(d);
        c->gstates_cap = 1;
    }
    uint8_t* hs = static_cast<uint8_t*>(staging(c, gb));
    const int grange = std::min(range, 32);
    init_gstate(reinterpret_cast<GState*>(hs), cur, ref, grange, s.r.global, s.r.gsad);
    ck(cudaMemcpyAsync(c->d_gstates, hs, gb, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(gstate)");
    staging_mark(c);
    {
        Timer tm(c, kGlobal);
        const int launches = run_global_search(c->d_gstates, 1, grange, W, H, c->stream);
        ck(cudaGetLastError(), "global search launch");
        tm.stop(launches);
    }
    int g[2];
    unsigned long long gs = 0;
    ck(cudaMemcpyAsync(g, s.r.global, 8, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(global)");
    ck(cudaMemcpyAsync(&gs, s.r.gsad, 8, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(global)");
    sync_checked(c);
    *dx = g[0];
    *dy = g[1];
    *sad = gs;
}

// The zoom-coherence test of Vc1Encoder::scene_change_score (encoder_motion.cpp:636-671), in
// the reference's long double arithmetic.
bool zoom_coherent(const std::vector<vc1cu_mv>& mvs, int mbw, int mbh) {
    long double mx = 0.0L, my = 0.0L, mdx = 0.0L, mdy = 0.0L;
    size_t samples = 0;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[static_cast<size_t>(by) * mbw + bx];
            mx += bx * 16.0L + 8.0L;
            my += by * 16.0L + 8.0L;
            mdx += mv.xq / 4.0L;
            mdy += mv.yq / 4.0L;
            ++samples;
        }
    if (samples < 12) return false;
    mx /= samples;
    my /= samples;
    mdx /= samples;
    mdy /= samples;
    long double num = 0.0L, den = 0.0L;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[static_cast<size_t>(by) * mbw + bx];
            const long double x = bx * 16.0L + 8.0L - mx, y = by * 16.0L + 8.0L - my;
            const long double dx = mv.xq / 4.0L - mdx, dy = mv.yq / 4.0L - mdy;
            num += x * dx + y * dy;
            den += x * x + y * y;
        }
    const long double z = den > 0.0L ? num / den : 0.0L;
    size_t inliers = 0;
    for (int by = 1; by < mbh - 1; ++by)
        for (int bx = 1; bx < mbw - 1; ++bx) {
            const vc1cu_mv mv = mvs[static_cast<size_t>(by) * mbw + bx];
            const long double x = bx * 16.0L + 8.0L - mx, y = by * 16.0L + 8.0L - my;
            const long double ex = mv.xq / 4.0L - (mdx + z * x);
            const long double ey = mv.yq / 4.0L - (mdy + z * y);
            if (ex * ex + ey * ey <= 6.25L) ++inliers;
        }
    const long double az = std::fabs(z);
    return inliers * 5 >= samples * 3 && az >= 0.005L && az <= 0.08L;
}

void read_bresult(vc1cu_ctx* c, const BSlot& s, vc1cu_banalysis* out) {
    const size_t n = (size_t)s.mbs;
    stamp_written(c);
    read_after(c, s.written);
    const uint8_t* hb = read_slot_bytes(c, s.d, s.bytes);
    read_sync(c);
    const uint8_t* base = static_cast<const uint8_t*>(s.d);
    auto cp = [&](void* dst, const void* src, size_t b) {
        if (dst) std::memcpy(dst, hb + (static_cast<const uint8_t*>(src) - base), b);
    };
    cp(out->modes, s.r.modes, n);
    cp(out->forward_mvs, s.r.fmv, 8 * n);
    cp(out->backward_mvs, s.r.bmv, 8 * n);
    cp(out->inter_intra_cost_ratio, s.r.ratio, 8 * n);
    cp(out->forward_distant_local_mae, s.r.fdl, 8 * n);
    cp(out->forward_distant_candidate_mae, s.r.fdc, 8 * n);
    cp(out->forward_distant_match_decision, s.r.fdd, n);
    cp(out->backward_distant_local_mae, s.r.bdl, 8 * n);
    cp(out->backward_distant_candidate_mae, s.r.bdc, 8 * n);
    cp(out->backward_distant_match_decision, s.r.bdd, n);
    unsigned long long it[kBTotCount];
    double tot[2];
    cp(it, s.r.itotals, sizeof it);
    cp(tot, s.r.totals, sizeof tot);
    out->forward_macroblocks = it[kBTotForward];
    out->backward_macroblocks = it[kBTotBackward];
    out->interpolated_macroblocks = it[kBTotInterpolated];
    out->direct_macroblocks = it[kBTotDirect];
    out->intra_macroblocks = it[kBTotIntra];
    out->moved_macroblocks = it[kBTotMoved];
    out->fractional_chroma_macroblocks = it[kBTotFrac];
    out->mean_abs_residual = tot[0];
    out->rate_complexity = tot[1];
    out->motion_sad = it[kBTotSelSad];
    out->motion_bits = it[kBTotSelRate];
    out->mv_mode = s.mode;
    out->reserved = 0;
}

}  // namespace

// ---- C ABI -------------------------------------------------------------------------------

extern "C" {

void vc1cu_params_default(vc1cu_params* p, int width, int height) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->width = width;
    p->height = height;
    p->pqindex = 8;
    p->search_range = 1024;
    p->local_search_range = 32;
    p->me_algorithm = 0;
    p->me_quality = 2;
    p->subpel = 1;
    p->subpel_range = 1024;
    p->distant_match_max_mae = 255.0;
    p->inter_intra_threshold = 0.80;
}

int vc1cu_open(int device, vc1cu_ctx** out) {
    if (!out) return fail(nullptr, VC1CU_ERR_ARG, "null output pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(nullptr, VC1CU_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0) {
        e = cudaGetDevice(&device);
        if (e != cudaSuccess) return fail(nullptr, VC1CU_ERR_CUDA, cudaGetErrorString(e));
    }
    if (device >= count) return fail(nullptr, VC1CU_ERR_ARG, "device ordinal out of range");
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return fail(nullptr, VC1CU_ERR_CUDA, cudaGetErrorString(e));
    if (prop.major < 10) return fail(nullptr, VC1CU_ERR_UNSUPPORTED, "this library is built for sm_100a (B200)");
    auto* c = new (std::nothrow) vc1cu_ctx;
    if (!c) return fail(nullptr, VC1CU_ERR_OOM, "host allocation failed");
    c->device = device;
    c->name = prop.name;
    c->sm_count = prop.multiProcessorCount;
    c->max_smem = (int)prop.sharedMemPerBlockOptin;
    c->max_smem_sm = (int)prop.sharedMemPerMultiprocessor;
    try {
        ck(cudaSetDevice(device), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaStreamCreateWithFlags(&c->rstream, cudaStreamNonBlocking), "cudaStreamCreate(read)");
        ck(cudaStreamCreateWithFlags(&c->ustream, cudaStreamNonBlocking), "cudaStreamCreate(upload)");
        void* d = nullptr;
        ck(cudaMalloc(&d, sizeof(LaunchStatus)), "cudaMalloc(status)");
        c->d_status = static_cast<LaunchStatus*>(d);
        ck(cudaMemsetAsync(c->d_status, 0, sizeof(LaunchStatus), c->stream), "cudaMemsetAsync(status)");
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    } catch (const Fail& f) {
        const int code = f.code;
        t_open_error = f.msg;
        vc1cu_close(c);
        return code;
    }
    *out = c;
    return VC1CU_OK;
}

int vc1cu_close(vc1cu_ctx* c) {
    if (!c) return VC1CU_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->ustream) cudaStreamSynchronize(c->ustream);
    for (auto& kv : c->frames) {
        if (kv.second.d) cudaFree(kv.second.d);
        if (kv.second.uploaded) cudaEventDestroy(kv.second.uploaded);
    }
    for (auto& kv : c->results)
        if (kv.second.d) cudaFree(kv.second.d);
    for (auto& kv : c->bresults)
        if (kv.second.d) cudaFree(kv.second.d);
    if (c->d_bdescs) cudaFree(c->d_bdescs);
    if (c->d_ic) cudaFree(c->d_ic);
    if (c->d_icdesc) cudaFree(c->d_icdesc);
    if (c->d_btypes) cudaFree(c->d_btypes);
    if (c->d_trd_tab) cudaFree(c->d_trd_tab);
    if (c->d_sp) cudaFree(c->d_sp);
    if (c->d_trd) cudaFree(c->d_trd);
    if (c->d_mrd) cudaFree(c->d_mrd);
    if (c->d_dq) cudaFree(c->d_dq);
    if (c->d_intra) cudaFree(c->d_intra);
    if (c->d_iovl) cudaFree(c->d_iovl);
    if (c->d_lf) cudaFree(c->d_lf);
    if (c->d_ovl) cudaFree(c->d_ovl);
    if (c->d_gcopy) cudaFree(c->d_gcopy);
    auto free_ticket = [](vc1cu_ctx::IcTicket& t) {
        if (t.h) cudaFreeHost(t.h);
        if (t.done) cudaEventDestroy(t.done);
    };
    for (auto& t : c->ic_tickets) free_ticket(t);
    free_ticket(c->ic_sync);
    for (auto& s : c->cache)
        if (s.d) cudaFree(s.d);
    if (c->d_status) cudaFree(c->d_status);
    if (c->d_passes) cudaFree(c->d_passes);
    if (c->d_gstates) cudaFree(c->d_gstates);
    if (c->d_lr) cudaFree(c->d_lr);
    if (c->d_scratch) cudaFree(c->d_scratch);
    if (c->d_synth) cudaFree(c->d_synth);
    for (auto& kv : c->graphs) {
        cudaGraphExecDestroy(kv.second.exec);
        cudaGraphDestroy(kv.second.g);
        for (void* h : kv.second.hold) cudaFreeHost(h);
    }
    for (auto& kv : c->items) cudaFree(kv.second.first);
    if (c->h_read) cudaFreeHost(c->h_read);
    for (auto& b : c->staging_ring) {
        if (b.h) cudaFreeHost(b.h);
        if (b.done) cudaEventDestroy(b.done);
    }
    for (auto& t : c->pending) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->rstream) {
        cudaStreamSynchronize(c->rstream);
        cudaStreamDestroy(c->rstream);
    }
    if (c->ustream) cudaStreamDestroy(c->ustream);
    delete c;
    return VC1CU_OK;
}

const char* vc1cu_device_name(const vc1cu_ctx* c) { return c ? c->name.c_str() : ""; }
int vc1cu_device_index(const vc1cu_ctx* c) { return c ? c->device : -1; }
const char* vc1cu_last_error(const vc1cu_ctx* c) { return c ? c->err.c_str() : t_open_error.c_str(); }

int vc1cu_counters_get(const vc1cu_ctx* c, vc1cu_counters* out) {
    if (!c || !out) return VC1CU_ERR_ARG;
    *out = c->counters;
    return VC1CU_OK;
}

int vc1cu_reset_counters(vc1cu_ctx* c) {
    return guarded(c, [&]() -> int {
        collect_timing(c);
        c->counters = vc1cu_counters{};
        c->tsum = vc1cu_timing{};
        return VC1CU_OK;
    });
}

int vc1cu_debug_set_wait_limit(vc1cu_ctx* c, int log2_polls) {
    return guarded(c, [&]() -> int {
        if (log2_polls < 6 || log2_polls > 24) throw Fail{VC1CU_ERR_ARG, "log2_polls must be 6..24"};
        c->wait_log2 = log2_polls;
        return VC1CU_OK;
    });
}

int vc1cu_debug_withhold_publish(vc1cu_ctx* c, int pass_index, int mb) {
    return guarded(c, [&]() -> int {
        if (pass_index < 0 && mb < 0) {
            c->withhold_next = 0xFFFFFFFFu;
            return VC1CU_OK;
        }
        if (pass_index < 0 || pass_index > 0x7FF || mb < 0 || mb > 0xFFFFF)
            throw Fail{VC1CU_ERR_ARG, "pass_index must be 0..2047 and mb 0..2^20-1 (or both -1)"};
        c->withhold_next = ((uint32_t)pass_index << 20) | (uint32_t)mb;
        return VC1CU_OK;
    });
}

int vc1cu_set_timing(vc1cu_ctx* c, int enable) {
    return guarded(c, [&]() -> int {
        collect_timing(c);
        c->timing = enable != 0;
        return VC1CU_OK;
    });
}

int vc1cu_timing_get(vc1cu_ctx* c, vc1cu_timing* out) {
    return guarded(c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        collect_timing(c);
        *out = c->tsum;
        return VC1CU_OK;
    });
}

void* vc1cu_stream(const vc1cu_ctx* c) { return c ? (void*)c->stream : nullptr; }

int vc1cu_measure_int32_peak(vc1cu_ctx* c, double* ops_per_second) {
    return guarded(c, [&]() -> int {
        if (!ops_per_second) throw Fail{VC1CU_ERR_ARG, "null output"};
        *ops_per_second = measure_int32_peak(c->stream, c->sm_count);
        ck(cudaGetLastError(), "int32_peak_kernel");
        if (*ops_per_second <= 0.0) throw Fail{VC1CU_ERR_CUDA, "calibration kernel failed"};
        return VC1CU_OK;
    });
}

int vc1cu_debug_index_faults(unsigned int* count, unsigned long long* first, int reset) {
    const int rc = index_fault_record(count, first, reset);
    if (rc < 0) return fail(nullptr, VC1CU_ERR_UNSUPPORTED, "not an index-checked build (libvc1cu_checked.so)");
    if (rc > 0) return fail(nullptr, VC1CU_ERR_CUDA, "reading the index-check record failed");
    return VC1CU_OK;
}

int vc1cu_measure_fp64_peak(vc1cu_ctx* c, double* flops_per_second) {
    return guarded(c, [&]() -> int {
        if (!flops_per_second) throw Fail{VC1CU_ERR_ARG, "null output"};
        *flops_per_second = measure_fp64_peak(c->stream, c->sm_count);
        ck(cudaGetLastError(), "fp64_peak_kernel");
        if (*flops_per_second <= 0.0) throw Fail{VC1CU_ERR_CUDA, "calibration kernel failed"};
        return VC1CU_OK;
    });
}

int vc1cu_score_motion_batch(vc1cu_ctx* c, const uint8_t* cur, const uint8_t* ref, int width, int height, int x0, int y0,
                             int bw, int bh, int sample_stride, int bilinear, int rnd, int metric,
                             const vc1cu_mv* candidates, size_t n, uint64_t* costs) {
    return guarded(c, [&]() -> int {
        // src/vulkan_compute.cpp:375-382: empty or degenerate batches are a successful no-op
        if (!cur || !ref || width <= 0 || height <= 0 || bw <= 0 || bh <= 0 || !candidates || !n) return VC1CU_OK;
        if (!costs) throw Fail{VC1CU_ERR_ARG, "null costs"};
        if (n > kMaxBatch) throw Fail{VC1CU_ERR_ARG, "motion batches above 4,194,240 candidates are not supported"};
        if (metric != VC1CU_METRIC_SAD && metric != VC1CU_METRIC_SATD) throw Fail{VC1CU_ERR_ARG, "invalid metric"};
        if (x0 < 0 || y0 < 0 || sample_stride < 0) throw Fail{VC1CU_ERR_ARG, "block origin must lie in the picture"};
        uint8_t* dcur = cache_frame(c, cur, width, height);
        uint8_t* dref = cache_frame(c, ref, width, height);
        DevParams P{};
        P.W = width;
        P.H = height;
        ScoreArgs a{dcur, dref, width, width, height, x0, y0, bw, bh, sample_stride,
                    bilinear ? VC1CU_MV_HPEL_BILINEAR : VC1CU_MV_QPEL, rnd != 0, metric, VC1CU_LAW_SHADER};
        return score_common(c, P, a, candidates, n, costs);
    });
}

int vc1cu_score_motion_batch_law(vc1cu_ctx* c, const vc1cu_params* p, int law, const uint8_t* cur, const uint8_t* ref,
                                 int x0, int y0, int bw, int bh, int sample_stride, int mode, int metric,
                                 const vc1cu_mv* candidates, size_t n, uint64_t* costs) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        if (!cur || !ref || bw <= 0 || bh <= 0 || !candidates || !n) return VC1CU_OK;
        if (!costs) throw Fail{VC1CU_ERR_ARG, "null costs"};
        if (n > kMaxBatch) throw Fail{VC1CU_ERR_ARG, "motion batches above 4,194,240 candidates are not supported"};
        if (law != VC1CU_LAW_SHADER && law != VC1CU_LAW_CPU) throw Fail{VC1CU_ERR_ARG, "invalid law"};
        if (mode < 0 || mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        if (metric != VC1CU_METRIC_SAD && metric != VC1CU_METRIC_SATD) throw Fail{VC1CU_ERR_ARG, "invalid metric"};
        if (x0 < 0 || y0 < 0 || sample_stride < 0) throw Fail{VC1CU_ERR_ARG, "block origin must lie in the picture"};
        if (law == VC1CU_LAW_CPU && metric == VC1CU_METRIC_SAD && sample_stride > 1 &&
            (bw != 16 || bh != 16 || (x0 & 15) || (y0 & 15)))
            throw Fail{VC1CU_ERR_ARG, "sampled SAD is defined for macroblock-aligned 16x16 blocks (mb_sad)"};
        uint8_t* dcur = cache_frame(c, cur, p->width, p->height);
        uint8_t* dref = cache_frame(c, ref, p->width, p->height);
        ScoreArgs a{dcur, dref, p->width, p->width, p->height, x0, y0, bw, bh, sample_stride, mode, p->rnd != 0, metric, law};
        return score_common(c, P, a, candidates, n, costs);
    });
}

int vc1cu_upload_frame(vc1cu_ctx* c, int id, const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h) {
    return guarded(c, [&]() -> int {
        if (id < 0 || id >= kMaxSlot) throw Fail{VC1CU_ERR_ARG, "frame id out of range"};
        if (!y || w <= 0 || h <= 0 || (w & 1) || (h & 1)) throw Fail{VC1CU_ERR_ARG, "invalid frame"};
        // On the upload stream after the last work that used the slot; work enqueued on the
        // context stream from here on waits for it, work enqueued before keeps running.
        FrameSlot& f = alloc_frame(c, id, w, h, true);
        if (f.last_use) ck(cudaStreamWaitEvent(c->ustream, f.last_use->e, 0), "cudaStreamWaitEvent(upload)");
        const DevFrame d = f.view();
        cudaStream_t us = c->ustream;
        ck(cudaMemcpy2DAsync((void*)d.y, f.pitch_y, y, w, w, h, cudaMemcpyHostToDevice, us), "upload Y");
        const int cw = w / 2, ch = h / 2;
        if (u) ck(cudaMemcpy2DAsync((void*)d.u, f.pitch_c, u, cw, cw, ch, cudaMemcpyHostToDevice, us), "upload U");
        else ck(cudaMemset2DAsync((void*)d.u, f.pitch_c, 128, cw, ch, us), "fill U");
        if (v) ck(cudaMemcpy2DAsync((void*)d.v, f.pitch_c, v, cw, cw, ch, cudaMemcpyHostToDevice, us), "upload V");
        else ck(cudaMemset2DAsync((void*)d.v, f.pitch_c, 128, cw, ch, us), "fill V");
        if (!f.uploaded) ck(cudaEventCreateWithFlags(&f.uploaded, cudaEventDisableTiming), "cudaEventCreate(upload)");
        ck(cudaEventRecord(f.uploaded, us), "cudaEventRecord(upload)");
        ck(cudaStreamWaitEvent(c->stream, f.uploaded, 0), "cudaStreamWaitEvent(upload)");
        c->counters.frame_uploads++;
        c->counters.frame_upload_bytes += (size_t)w * h + 2 * (size_t)cw * ch;
        return VC1CU_OK;
    });
}

static_assert(sizeof(vc1cu_synth_cfg) == sizeof(vc1synth_cfg) &&
                  offsetof(vc1cu_synth_cfg, noise_sigma) == offsetof(vc1synth_cfg, noise_sigma) &&
                  offsetof(vc1cu_synth_cfg, seed) == offsetof(vc1synth_cfg, seed),
              "vc1cu_synth_cfg mirrors vc1synth_cfg");

int vc1cu_synth_frames(vc1cu_ctx* c, const vc1cu_synth_cfg* cfg, int first, int count, int frame_id0) {
    return guarded(c, [&]() -> int {
        if (!cfg) throw Fail{VC1CU_ERR_ARG, "null configuration"};
        vc1synth_cfg s;
        std::memcpy(&s, cfg, sizeof s);
        if (s.width <= 0 || s.height <= 0 || (s.width & 1) || (s.height & 1) || s.width > 16384 || s.height > 16384)
            throw Fail{VC1CU_ERR_ARG, "width/height must be positive, even and <= 16384"};
        if (s.n_objects < 0 || s.n_objects > 64) throw Fail{VC1CU_ERR_ARG, "n_objects must be 0..64"};
        if (count < 1 || count > kSynthMaxFrames || first < 0 || first + count > s.frames)
            throw Fail{VC1CU_ERR_ARG, "count must be 1..64 and first + count <= frames"};
        if (frame_id0 < 0 || frame_id0 + count > kMaxSlot) throw Fail{VC1CU_ERR_ARG, "frame id out of range"};
        const size_t nterms = (size_t)((s.width + 1) / 2) * ((s.height + 1) / 2);
        const size_t args_bytes = (sizeof(SynthArgs) + 255) & ~size_t(255);
        uint8_t* d = static_cast<uint8_t*>(
            ensure(c->d_synth, c->synth_cap, args_bytes + 256 + nterms * sizeof(double), "cudaMalloc(synth)"));
        SynthArgs* da = reinterpret_cast<SynthArgs*>(d);
        double* d_ms = reinterpret_cast<double*>(d + args_bytes);
        double* d_terms = reinterpret_cast<double*>(d + args_bytes + 256);
        SynthArgs* ha = static_cast<SynthArgs*>(staging(c, sizeof(SynthArgs)));
        std::memset(ha, 0, sizeof(SynthArgs));
        vs_make_plan(&s, &ha->plan);
        std::vector<double> gx(first + count), gy(first + count);
        vs_global_track(&s, first + count, gx.data(), gy.data());
        ha->first = first;
        ha->count = count;
        ha->mean_scale = d_ms;
        for (int i = 0; i < count; ++i) {
            const int t = first + i;
            double zinv = 1.0;
            for (int k = 0; k < t; ++k) zinv = zinv / s.zoom;
            ha->zinv[i] = zinv;
            ha->gx[i] = gx[t];
            ha->gy[i] = gy[t];
            FrameSlot& f = alloc_frame(c, frame_id0 + i, s.width, s.height);
            const DevFrame v = f.view();
            ha->out[i] = SynthOut{const_cast<uint8_t*>(v.y), const_cast<uint8_t*>(v.u), const_cast<uint8_t*>(v.v),
                                  f.pitch_y, f.pitch_c};
        }
        ck(cudaMemcpyAsync(da, ha, sizeof(SynthArgs), cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(synth)");
        staging_mark(c);
        ck(launch_synth(s, da, d_terms, d_ms, count, c->sm_count, c->stream), "synth launch");
        c->counters.kernel_launches += 3;
        return VC1CU_OK;
    });
}

int vc1cu_download_frame(vc1cu_ctx* c, int id, uint8_t* y, uint8_t* u, uint8_t* v) {
    return guarded(c, [&]() -> int {
        FrameSlot& f = frame_slot(c, id);
        const DevFrame d = f.view();
        const int cw = f.w / 2, ch = f.h / 2;
        if (y) ck(cudaMemcpy2DAsync(y, f.w, d.y, f.pitch_y, f.w, f.h, cudaMemcpyDeviceToHost, c->stream), "download Y");
        if (u) ck(cudaMemcpy2DAsync(u, cw, d.u, f.pitch_c, cw, ch, cudaMemcpyDeviceToHost, c->stream), "download U");
        if (v) ck(cudaMemcpy2DAsync(v, cw, d.v, f.pitch_c, cw, ch, cudaMemcpyDeviceToHost, c->stream), "download V");
        sync_checked(c);
        return VC1CU_OK;
    });
}

int vc1cu_core_passes(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_pass* passes, int n) {
    return guarded(c, [&]() -> int {
        if (n < 0 || (n > 0 && !passes)) throw Fail{VC1CU_ERR_ARG, "invalid pass list"};
        for (int i = 0; i < n; ++i)
            if (passes[i].out_slot < 0 || passes[i].out_slot >= kMaxSlot || passes[i].seed_slot >= kMaxSlot)
                throw Fail{VC1CU_ERR_ARG, "result slot out of range"};
        return launch_passes(c, p, passes, n);
    });
}

int vc1cu_core_passes_multi(vc1cu_ctx* c, const vc1cu_params* params, const vc1cu_pass* passes, int n) {
    return guarded(c, [&]() -> int {
        if (n <= 0 || !passes || !params) throw Fail{VC1CU_ERR_ARG, "invalid pass list"};
        for (int i = 0; i < n; ++i) {
            if (passes[i].out_slot < 0 || passes[i].out_slot >= kMaxSlot || passes[i].seed_slot >= kMaxSlot)
                throw Fail{VC1CU_ERR_ARG, "result slot out of range"};
            for (int j = 0; j < i; ++j)
                if (passes[j].out_slot == passes[i].out_slot) throw Fail{VC1CU_ERR_ARG, "two passes write one result slot"};
        }
        return launch_group(c, params, passes, n, false, nullptr, params);
    });
}

int vc1cu_graph_begin(vc1cu_ctx* c) {
    return guarded(c, [&]() -> int {
        if (c->capturing) throw Fail{VC1CU_ERR_STATE, "a capture is already open on this context"};
        if (c->timing) throw Fail{VC1CU_ERR_STATE, "turn per-launch timing off before capturing"};
        stamp_written(c);
        ck(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
        c->capturing = true;
        c->capture_hold.clear();
        c->capture_results.clear();
        c->capture_bresults.clear();
        c->capture_frames.clear();
        return VC1CU_OK;
    });
}

int vc1cu_graph_end(vc1cu_ctx* c, int* graph_id) {
    return guarded(c, [&]() -> int {
        if (!c->capturing) throw Fail{VC1CU_ERR_STATE, "no capture is open on this context"};
        if (!graph_id) throw Fail{VC1CU_ERR_ARG, "null output"};
        stamp_written(c);
        vc1cu_ctx::Graph g;
        c->capturing = false;
        ck(cudaStreamEndCapture(c->stream, &g.g), "cudaStreamEndCapture");
        g.hold.swap(c->capture_hold);
        g.results.swap(c->capture_results);
        g.bresults.swap(c->capture_bresults);
        g.frames.swap(c->capture_frames);
        const cudaError_t e = cudaGraphInstantiate(&g.exec, g.g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g.g);
            for (void* h : g.hold) cudaFreeHost(h);
            throw Fail{VC1CU_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
        }
        const int id = c->graph_next++;
        c->graphs[id] = std::move(g);
        *graph_id = id;
        return VC1CU_OK;
    });
}

int vc1cu_graph_launch(vc1cu_ctx* c, int graph_id) {
    return guarded(c, [&]() -> int {
        auto it = c->graphs.find(graph_id);
        if (it == c->graphs.end()) throw Fail{VC1CU_ERR_ARG, "unknown graph id"};
        if (c->capturing) throw Fail{VC1CU_ERR_STATE, "a capture is open on this context"};
        // frames the graph reads may have uploads in flight on the upload stream
        for (int id : it->second.frames) {
            auto f = c->frames.find(id);
            if (f != c->frames.end() && f->second.uploaded)
                ck(cudaStreamWaitEvent(c->stream, f->second.uploaded, 0), "cudaStreamWaitEvent(upload)");
        }
        ck(cudaGraphLaunch(it->second.exec, c->stream), "cudaGraphLaunch");
        c->dirty_results = it->second.results;
        c->dirty_bresults = it->second.bresults;
        c->used_frames = it->second.frames;
        c->counters.dispatches++;
        return VC1CU_OK;
    });
}

int vc1cu_graph_destroy(vc1cu_ctx* c, int graph_id) {
    return guarded(c, [&]() -> int {
        auto it = c->graphs.find(graph_id);
        if (it == c->graphs.end()) throw Fail{VC1CU_ERR_ARG, "unknown graph id"};
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        cudaGraphExecDestroy(it->second.exec);
        cudaGraphDestroy(it->second.g);
        for (void* h : it->second.hold) cudaFreeHost(h);
        c->graphs.erase(it);
        return VC1CU_OK;
    });
}

int vc1cu_autotune(vc1cu_ctx* c, const vc1cu_params* params, const vc1cu_pass* passes, int n, int per_pass_params,
                   int* warps_out, int* blocks_out, double* ms_out) {
    return guarded(c, [&]() -> int {
        if (n <= 0 || !passes || !params) throw Fail{VC1CU_ERR_ARG, "invalid pass list"};
        if (c->capturing) throw Fail{VC1CU_ERR_STATE, "cannot tune during a capture"};
        const vc1cu_params* pp = per_pass_params ? params : nullptr;
        auto run = [&]() { launch_group(c, params, passes, n, false, nullptr, pp); };
        cudaEvent_t a = take_event(c), b = take_event(c);
        double best = -1.0;
        std::pair<int, int> best_shape{0, 0};
        std::vector<int> key;
        // warps (macroblocks) per block and blocks per SM (0: as many as fit); shapes that do not fit
        // the launch's instantiation or shared memory are skipped
        const std::pair<int, int> shapes[] = {{4, 0}, {4, 1}, {4, 2}, {2, 0}, {2, 2}, {1, 0}, {1, 4}, {3, 0},
                                              {5, 1}, {6, 1}, {7, 1}, {8, 1}};
        for (const auto& s : shapes) {
            c->tune_force = s;
            try {
                run();  // warm-up (and the shape's work-item table)
                ck(cudaEventRecord(a, c->stream), "cudaEventRecord");
                run();
                run();
                ck(cudaEventRecord(b, c->stream), "cudaEventRecord");
                check_status(c);
            } catch (const Fail& f) {
                if (f.code != VC1CU_ERR_ARG) {  // a shape that does not fit is skipped, anything else fails
                    c->tune_force = {0, 0};
                    c->event_pool.push_back(a);
                    c->event_pool.push_back(b);
                    throw;
                }
                continue;
            }
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
            key = c->last_tune_key;
            if (best < 0.0 || ms < best) {
                best = ms;
                best_shape = s;
            }
        }
        c->tune_force = {0, 0};
        c->event_pool.push_back(a);
        c->event_pool.push_back(b);
        if (best < 0.0) throw Fail{VC1CU_ERR_UNSUPPORTED, "no launch shape fits"};
        c->tuned[key] = best_shape;
        if (warps_out) *warps_out = best_shape.first;
        if (blocks_out) *blocks_out = best_shape.second;
        if (ms_out) *ms_out = best / 2.0;
        return VC1CU_OK;
    });
}

int vc1cu_synchronize(vc1cu_ctx* c) {
    return guarded(c, [&]() -> int { return check_status(c); });
}

int vc1cu_read_result(vc1cu_ctx* c, int slot, vc1cu_panalysis* out) {
    return guarded(c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        auto it = c->results.find(slot);
        if (it == c->results.end() || !it->second.valid) throw Fail{VC1CU_ERR_STATE, "empty result slot"};
        check_status_read(c, it->second.written);
        read_result(c, it->second, out);
        return VC1CU_OK;
    });
}

int vc1cu_analyze_p_core(vc1cu_ctx* c, const vc1cu_params* p, int cur_id, int ref_id, int mode, int allow_intra,
                         const vc1cu_mv* seed_mvs, const vc1cu_panalysis* seed_distant, vc1cu_panalysis* out) {
    return guarded(c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const int mbs = P.mbw * P.mbh;
        vc1cu_pass q{cur_id, ref_id, mode, allow_intra, -1, kInternalOut, 0};
        if (seed_mvs) {
            ResultSlot& s = result_slot(c, kInternalSeed, mbs, true);
            ck(cudaMemcpyAsync(s.r.mvs, seed_mvs, 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload seed");
            std::vector<double> neg(mbs, -1.0);
            std::vector<uint8_t> zero(mbs, 0);
            const double* dl = seed_distant && seed_distant->distant_local_mae ? seed_distant->distant_local_mae : neg.data();
            const double* dc = seed_distant && seed_distant->distant_candidate_mae ? seed_distant->distant_candidate_mae : neg.data();
            const uint8_t* dd = seed_distant && seed_distant->distant_match_decision ? seed_distant->distant_match_decision : zero.data();
            ck(cudaMemcpyAsync(s.r.dl, dl, 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload seed");
            ck(cudaMemcpyAsync(s.r.dc, dc, 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload seed");
            ck(cudaMemcpyAsync(s.r.dd, dd, (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload seed");
            ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
            q.seed_slot = kInternalSeed;
        }
        launch_passes(c, p, &q, 1);
        check_status(c);
        read_result(c, c->results[kInternalOut], out);
        if (seed_mvs) {
            out->global_dx = out->global_dy = 0;
            out->global_full_sad = 0;
        }
        return VC1CU_OK;
    });
}

int vc1cu_b_decide(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_bpass* passes, int n) {
    return guarded(c, [&]() -> int {
        if (n < 0 || (n > 0 && !passes)) throw Fail{VC1CU_ERR_ARG, "invalid B pass list"};
        for (int i = 0; i < n; ++i) {
            const vc1cu_bpass& q = passes[i];
            if (q.fwd_slot < 0 || q.fwd_slot >= kMaxSlot || q.bwd_slot < 0 || q.bwd_slot >= kMaxSlot ||
                q.anchor_slot < 0 || q.anchor_slot >= kMaxSlot)
                throw Fail{VC1CU_ERR_ARG, "result slot out of range"};
        }
        launch_b(c, p, passes, n, kMaxSlot - 1);
        return VC1CU_OK;
    });
}

int vc1cu_read_bresult(vc1cu_ctx* c, int bslot, vc1cu_banalysis* out) {
    return guarded(c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        auto it = c->bresults.find(bslot);
        if (it == c->bresults.end() || !it->second.valid) throw Fail{VC1CU_ERR_STATE, "empty B-result slot"};
        check_status_read(c, it->second.written);
        read_bresult(c, it->second, out);
        return VC1CU_OK;
    });
}

int vc1cu_b_predict(vc1cu_ctx* c, const vc1cu_params* p, int bslot, int cur_id, int past_id, int future_id, int pred_id) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        auto it = c->bresults.find(bslot);
        if (it == c->bresults.end() || !it->second.valid || it->second.mbs != P.mbw * P.mbh)
            throw Fail{VC1CU_ERR_STATE, "B-result slot holds no analysis of this size"};
        if (pred_id < 0 || pred_id >= kMaxSlot || pred_id == cur_id || pred_id == past_id || pred_id == future_id)
            throw Fail{VC1CU_ERR_ARG, "invalid prediction slot"};
        FrameSlot& fc = frame_slot(c, cur_id);
        FrameSlot& fp = frame_slot(c, past_id);
        FrameSlot& ff = frame_slot(c, future_id);
        if (fc.w != P.W || fc.h != P.H || fp.w != P.W || fp.h != P.H || ff.w != P.W || ff.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "B-picture reference dimensions do not match the configuration"};
        const DevFrame cur = fc.view(), past = fp.view(), fut = ff.view();
        FrameSlot& fo = alloc_frame(c, pred_id, P.W, P.H);
        const DevFrame o = fo.view();
        const BSlot& b = it->second;
        Timer tm(c, kMc);
        ck(launch_b_mc(P, cur, past, fut, b.r.modes, b.r.fmv, b.r.bmv, b.mode, (uint8_t*)o.y, (uint8_t*)o.u, (uint8_t*)o.v,
                       fo.pitch_y, fo.pitch_c, c->stream),
           "B prediction launch");
        tm.stop(1);
        return VC1CU_OK;
    });
}

int vc1cu_analyze_b_picture(vc1cu_ctx* c, const vc1cu_params* p, int cur_id, int past_id, int future_id,
                            const vc1cu_mv* anchor_mvs, const uint8_t* anchor_4mv, int fraction_num, int fraction_den,
                            int mode, vc1cu_banalysis* out) {
    return guarded(c, [&]() -> int {
        if (!out || !anchor_mvs || !anchor_4mv) throw Fail{VC1CU_ERR_ARG, "null output or anchor field"};
        if (!((fraction_den == 2 && fraction_num == 1) || (fraction_den == 3 && (fraction_num == 1 || fraction_num == 2))))
            throw Fail{VC1CU_ERR_ARG, "unsupported B-picture temporal fraction (1/2, 1/3 and 2/3 are)"};
        if (mode < 0 || mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const int mbs = P.mbw * P.mbh;
        // the direct-mode scaling multiplies anchor components by at most 256 in 32-bit ints
        for (int i = 0; i < mbs; ++i)
            if (anchor_mvs[i].xq < -65536 || anchor_mvs[i].xq > 65536 || anchor_mvs[i].yq < -65536 || anchor_mvs[i].yq > 65536)
                throw Fail{VC1CU_ERR_ARG, "anchor MV component outside +-65536 quarter pixels"};
        ResultSlot& as = result_slot(c, kInternalAnchor, mbs, true);
        as.mode = -1;
        ck(cudaMemcpyAsync(as.r.mvs, anchor_mvs, 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload anchor");
        ck(cudaMemcpyAsync(as.r.use4, anchor_4mv, (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload anchor");
        const vc1cu_pass q[2] = {{cur_id, past_id, mode, 0, -1, kInternalFwd, 0}, {cur_id, future_id, mode, 0, -1, kInternalBwd, 0}};
        launch_passes(c, p, q, 2);
        const vc1cu_bpass b{cur_id, past_id, future_id, kInternalFwd, kInternalBwd, kInternalAnchor,
                            fraction_num, fraction_den, mode, kInternalB, 0};
        launch_b(c, p, &b, 1, kInternalB);
        check_status(c);
        read_bresult(c, c->bresults[kInternalB], out);
        return VC1CU_OK;
    });
}

int vc1cu_estimate_intensity_comp(vc1cu_ctx* c, const vc1cu_params* p, int cur_id, int ref_id, const vc1cu_mv* mvs,
                                  vc1cu_intensity* out) {
    return guarded(c, [&]() -> int {
        if (!out || !mvs) throw Fail{VC1CU_ERR_ARG, "null output or MV field"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const int mbs = P.mbw * P.mbh;
        FrameSlot& fc = frame_slot(c, cur_id);
        FrameSlot& fr = frame_slot(c, ref_id);
        if (fc.w != P.W || fc.h != P.H || fr.w != P.W || fr.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "intensity estimate frame dimensions do not match the configuration"};
        ResultSlot& s = result_slot(c, kInternalIc, mbs, true);
        s.mode = -1;
        ck(cudaMemcpyAsync(s.r.mvs, mvs, 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload MV field");
        ic_estimate(c, P, {IcJob{fc.view(), fr.view(), s.r.mvs}}, out);
        return VC1CU_OK;
    });
}

// The jobs of a batch of fade estimates, each along the mvs of its result slot.
static std::vector<IcJob> ic_jobs(vc1cu_ctx* c, const DevParams& P, const vc1cu_icpass* passes, int n) {
    const int mbs = P.mbw * P.mbh;
    std::vector<IcJob> jobs;
    for (int i = 0; i < n; ++i) {
        FrameSlot& fc = frame_slot(c, passes[i].cur_id);
        FrameSlot& fr = frame_slot(c, passes[i].ref_id);
        if (fc.w != P.W || fc.h != P.H || fr.w != P.W || fr.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "intensity estimate frame dimensions do not match the configuration"};
        if (passes[i].mv_slot < 0 || passes[i].mv_slot >= kMaxSlot) throw Fail{VC1CU_ERR_ARG, "result slot out of range"};
        jobs.push_back(IcJob{fc.view(), fr.view(), result_slot(c, passes[i].mv_slot, mbs, false).r.mvs});
    }
    return jobs;
}

int vc1cu_estimate_intensity_batch(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_icpass* passes, int n,
                                   vc1cu_intensity* out) {
    return guarded(c, [&]() -> int {
        if (n < 0 || (n > 0 && (!passes || !out))) throw Fail{VC1CU_ERR_ARG, "invalid intensity batch"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        check_status(c);
        ic_estimate(c, P, ic_jobs(c, P, passes, n), out);
        return VC1CU_OK;
    });
}

int vc1cu_estimate_intensity_enqueue(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_icpass* passes, int n,
                                     int64_t* ticket) {
    return guarded(c, [&]() -> int {
        if (!ticket || n < 0 || (n > 0 && !passes)) throw Fail{VC1CU_ERR_ARG, "invalid intensity batch"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const std::vector<IcJob> jobs = ic_jobs(c, P, passes, n);
        const int64_t id = c->ic_next_id++;
        auto& t = c->ic_tickets[id % vc1cu_ctx::kIcTickets];
        t.id = 0;  // not collectable until its work is enqueued
        ic_enqueue(c, P, jobs, t);
        t.id = id;
        *ticket = id;
        return VC1CU_OK;
    });
}

int vc1cu_estimate_intensity_collect(vc1cu_ctx* c, int64_t ticket, vc1cu_intensity* out, int n) {
    return guarded(c, [&]() -> int {
        auto& t = c->ic_tickets[(ticket > 0 ? ticket : 0) % vc1cu_ctx::kIcTickets];
        if (ticket <= 0 || t.id != ticket)
            throw Fail{VC1CU_ERR_STATE, "intensity ticket unknown, already collected or overwritten"};
        if (n != t.n || (n > 0 && !out)) throw Fail{VC1CU_ERR_ARG, "collect n differs from the enqueued batch"};
        // a wavefront timeout recorded by the launches before it is reported here
        ck(cudaStreamWaitEvent(c->rstream, t.done, 0), "cudaStreamWaitEvent(intensity)");
        LaunchStatus st{};
        ck(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->rstream), "cudaMemcpyAsync(status)");
        read_sync(c);
        if (st.error) check_status(c);
        ic_finish(c, t, out);
        t.id = 0;
        return VC1CU_OK;
    });
}

int vc1cu_scene_change_score(vc1cu_ctx* c, const vc1cu_params* p, int cur_id, int ref_id, int fade_compensation,
                             double scene_threshold, double* score) {
    return guarded(c, [&]() -> int {
        if (!score) throw Fail{VC1CU_ERR_ARG, "null output"};
        if (!(scene_threshold >= 0.0 && scene_threshold <= 255.0)) throw Fail{VC1CU_ERR_ARG, "scene threshold must be 0..255"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const int mbs = P.mbw * P.mbh;
        check_status(c);
        FrameSlot& fc = frame_slot(c, cur_id);
        FrameSlot& fr = frame_slot(c, ref_id);
        if (fc.w != P.W || fc.h != P.H || fr.w != P.W || fr.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "scene-analysis dimensions do not match the configuration"};
        const DevFrame cur = fc.view(), ref = fr.view();
        int gdx = 0, gdy = 0;
        uint64_t gsad = 0;
        global_search_one(c, cur, ref, P.range, P.W, P.H, kInternalIc, mbs, &gdx, &gdy, &gsad);
        const uint64_t pixels = static_cast<uint64_t>(P.W) * P.H;
        double best = pixels ? static_cast<double>(gsad) / static_cast<double>(pixels) : 0.0;
        if (fade_compensation) {
            // the fade estimate along the uniform global field (encoder_motion.cpp:606-616)
            std::vector<vc1cu_mv> uniform(mbs, vc1cu_mv{gdx * 4, gdy * 4});
            ResultSlot& s = result_slot(c, kInternalIc, mbs, true);
            ck(cudaMemcpyAsync(s.r.mvs, uniform.data(), 8 * (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload field");
            vc1cu_intensity ic{};
            ic_estimate(c, P, {IcJob{cur, ref, s.r.mvs}}, &ic);
            if (ic.enabled) {
                FrameSlot& fw = alloc_frame(c, kInternalFrame, P.W, P.H);
                const DevFrame w = fw.view();
                const int scale = ic.lumscale + 32, shift = (ic.lumshift > 31 ? ic.lumshift - 64 : ic.lumshift) * 64;
                ck(launch_ic_map(ref, (uint8_t*)w.y, (uint8_t*)w.u, (uint8_t*)w.v, fw.pitch_y, fw.pitch_c, P.W, P.H, 1, scale,
                                 shift, ic.lumscale + 32, c->stream),
                   "intensity map launch");
                c->counters.kernel_launches++;
                int wdx = 0, wdy = 0;
                uint64_t wsad = 0;
                global_search_one(c, cur, w, P.range, P.W, P.H, kInternalIc, mbs, &wdx, &wdy, &wsad);
                const double wm = pixels ? static_cast<double>(wsad) / static_cast<double>(pixels) : 0.0;
                best = std::min(best, wm);
            }
        }
        if (best >= scene_threshold) {
            // a local quarter-pel core pass may rescue a camera zoom (encoder_motion.cpp:627-674)
            const vc1cu_pass q{cur_id, ref_id, VC1CU_MV_QPEL, 0, -1, kInternalOut, 0};
            launch_passes(c, p, &q, 1);
            check_status(c);
            std::vector<vc1cu_mv> mvs(mbs);
            vc1cu_panalysis a{};
            a.mvs = mvs.data();
            read_result(c, c->results[kInternalOut], &a);
            const double lm = a.mean_abs_residual;
            if (zoom_coherent(mvs, P.mbw, P.mbh) && lm < best * 0.72 && lm < scene_threshold * 0.86) best = lm;
        }
        *score = best;
        return VC1CU_OK;
    });
}

// intensity_compensated_reference (encoder_motion_compensation.cpp:175-193, :195-294) of frame
// slot ref_id into out_id, on the context stream.
static void ic_compensate(vc1cu_ctx* c, int ref_id, const vc1cu_intensity* ic, int out_id) {
    FrameSlot& fr = frame_slot(c, ref_id);
    const int W = fr.w, H = fr.h;
    const DevFrame ref = fr.view();
    FrameSlot& fo = alloc_frame(c, out_id, W, H);
    const DevFrame o = fo.view();
    // the luma law of intensity_map_y and the chroma scale of intensity_map_uv
    // (encoder_motion_compensation.cpp:175-193)
    int scale, shift;
    if (ic->lumscale == 0) {
        scale = -64;
        shift = (255 - ic->lumshift * 2) * 64;
        if (ic->lumshift > 31) shift += 128 * 64;
    } else {
        scale = ic->lumscale + 32;
        shift = (ic->lumshift > 31 ? ic->lumshift - 64 : ic->lumshift) * 64;
    }
    const int cscale = ic->lumscale == 0 ? -64 : ic->lumscale + 32;
    Timer tm(c, kMc);
    ck(launch_ic_map(ref, (uint8_t*)o.y, (uint8_t*)o.u, (uint8_t*)o.v, fo.pitch_y, fo.pitch_c, W, H, ic->enabled != 0, scale,
                     shift, cscale, c->stream),
       "intensity map launch");
    tm.stop(1);
}

int vc1cu_intensity_compensate(vc1cu_ctx* c, int ref_id, const vc1cu_intensity* ic, int out_id) {
    return guarded(c, [&]() -> int {
        if (!ic) throw Fail{VC1CU_ERR_ARG, "null intensity parameters"};
        if (ic->lumscale < 0 || ic->lumscale > 63 || ic->lumshift < 0 || ic->lumshift > 63)
            throw Fail{VC1CU_ERR_ARG, "LUMSCALE and LUMSHIFT are 6-bit codes (0..63)"};
        if (out_id < 0 || out_id >= kMaxSlot || out_id == ref_id) throw Fail{VC1CU_ERR_ARG, "invalid output frame slot"};
        ic_compensate(c, ref_id, ic, out_id);
        return VC1CU_OK;
    });
}

int vc1cu_motion_compensate(vc1cu_ctx* c, const vc1cu_params* p, int ref_id, int mv_slot, int mv_mode, int pred_id) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        if (mv_mode < 0 || mv_mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        if (pred_id < 0 || pred_id >= kMaxSlot || pred_id == ref_id) throw Fail{VC1CU_ERR_ARG, "invalid prediction slot"};
        FrameSlot& fr = frame_slot(c, ref_id);
        if (fr.w != P.W || fr.h != P.H) throw Fail{VC1CU_ERR_ARG, "reference size mismatch"};
        const DevFrame ref = fr.view();
        ResultSlot& s = result_slot(c, mv_slot, P.mbw * P.mbh, false);
        FrameSlot& fp = alloc_frame(c, pred_id, P.W, P.H);
        const DevFrame pd = fp.view();
        Timer tm(c, kMc);
        launch_mc(P, ref, s.r.mvs, s.r.bmv, s.r.use4, mv_mode, (uint8_t*)pd.y, (uint8_t*)pd.u, (uint8_t*)pd.v, fp.pitch_y,
                  fp.pitch_c, c->stream);
        ck(cudaGetLastError(), "mc_kernel launch");
        tm.stop(1);
        return VC1CU_OK;
    });
}

int vc1cu_fast_transform_types(vc1cu_ctx* c, const vc1cu_params* p, int src_id, int pred_id, uint8_t* types) {
    return guarded(c, [&]() -> int {
        if (!types) throw Fail{VC1CU_ERR_ARG, "null output"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& fs = frame_slot(c, src_id);
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fs.w != P.W || fs.h != P.H || fp.w != P.W || fp.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
        const size_t mbs = (size_t)P.mbw * P.mbh;
        uint8_t* d = static_cast<uint8_t*>(ensure(c->d_btypes, c->btypes_cap, std::max<size_t>(mbs * 6, 256), "cudaMalloc(types)"));
        Timer tm(c, kXform);
        launch_fast_tt(P, fs.view(), fp.view(), d, c->stream);
        ck(cudaGetLastError(), "transform type launch");
        tm.stop(1);
        ck(cudaMemcpyAsync(types, d, mbs, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(types)");
        sync_checked(c);
        return VC1CU_OK;
    });
}

// The transform RD's dense rate tables on the device, built once per context.
static const void* trd_tables(vc1cu_ctx* c) {
    if (!c->d_trd_tab) {
        std::vector<uint8_t> h(trd_tables_bytes());
        trd_fill_tables(h.data());
        void* d = nullptr;
        ck(cudaMalloc(&d, h.size()), "cudaMalloc(transform RD tables)");
        c->d_trd_tab = d;
        ck(cudaMemcpyAsync(d, h.data(), h.size(), cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(tables)");
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize(tables)");  // h is freed on return
    }
    return c->d_trd_tab;
}

int vc1cu_choose_transform(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id, int pred_id,
                           const uint8_t* mquant, vc1cu_tdecision* out, int16_t* levels) {
    return guarded(c, [&]() -> int {
        if (!cfg || !out) throw Fail{VC1CU_ERR_ARG, "null configuration or output"};
        if (cfg->trellis < 0 || cfg->trellis > 2 || cfg->coding_set < 0 || cfg->coding_set > 7 || cfg->frame_type < 0 ||
            cfg->frame_type > 4)
            throw Fail{VC1CU_ERR_ARG, "invalid transform RD configuration"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& fs = frame_slot(c, src_id);
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fs.w != P.W || fs.h != P.H || fp.w != P.W || fp.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
        const size_t mbs = (size_t)P.mbw * P.mbh;
        if (mquant)
            for (size_t i = 0; i < mbs; ++i)
                if (mquant[i] > 31) throw Fail{VC1CU_ERR_ARG, "MQUANT must be 0 (PQINDEX) or 1..31"};
        trd_tables(c);
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t b_sum = 256, b_mq = al(mbs), b_out = al(mbs * sizeof(vc1cu_tdecision)), b_lv = al(mbs * 384 * 2);
        uint8_t* base = static_cast<uint8_t*>(ensure(c->d_trd, c->trd_cap, b_sum + b_mq + b_out + b_lv,
                                                     "cudaMalloc(transform RD buffers)"));
        auto* d_sum = reinterpret_cast<unsigned long long*>(base);
        uint8_t* d_mq = base + b_sum;
        auto* d_out = reinterpret_cast<vc1cu_tdecision*>(base + b_sum + b_mq);
        auto* d_lv = reinterpret_cast<int16_t*>(base + b_sum + b_mq + b_out);
        if (mquant) ck(cudaMemcpyAsync(d_mq, mquant, mbs, cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(mquant)");
        Timer tm(c, kXform);
        ck(launch_trd(P, fs.view(), fp.view(), c->d_trd_tab, mquant ? d_mq : nullptr, *cfg, d_sum, d_out,
                      levels ? d_lv : nullptr, c->stream, nullptr, 0, -1.0),
           "transform RD launch");
        tm.stop(2);
        ck(cudaMemcpyAsync(out, d_out, mbs * sizeof(vc1cu_tdecision), cudaMemcpyDeviceToHost, c->stream),
           "cudaMemcpyAsync(decisions)");
        if (levels)
            ck(cudaMemcpyAsync(levels, d_lv, mbs * 384 * 2, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(levels)");
        sync_checked(c);
        return VC1CU_OK;
    });
}

// ---- the DQUANT MQUANT search (choose_dquant_transform_mb, encoder_aq.cpp:280-404) ----------

// Evaluation rounds of the search: the base MQUANT at PQINDEX (DQUANTFRM 0) and elsewhere
// (DQUANTFRM 1), the finer adjacency candidate, the three coarser candidates.
constexpr int kDqRounds = 6;

int vc1cu_choose_dquant(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int dquant, int predictable_texture,
                        int src_id, int pred_id, const uint8_t* rate_base, vc1cu_tdecision* out, uint8_t* mquant_out,
                        int16_t* levels) {
    return guarded(c, [&]() -> int {
        if (!cfg || !rate_base || !out || !mquant_out) throw Fail{VC1CU_ERR_ARG, "null configuration, base MQUANT or output"};
        if (cfg->trellis < 0 || cfg->trellis > 2 || cfg->coding_set < 0 || cfg->coding_set > 7 || cfg->frame_type < 0 ||
            cfg->frame_type > 4)
            throw Fail{VC1CU_ERR_ARG, "invalid transform RD configuration"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& fs = frame_slot(c, src_id);
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fs.w != P.W || fs.h != P.H || fp.w != P.W || fp.h != P.H)
            throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
        const int mbs = P.mbw * P.mbh;
        for (int i = 0; i < mbs; ++i)
            if (rate_base[i] < 1 || rate_base[i] > 31) throw Fail{VC1CU_ERR_ARG, "base MQUANT must be 1..31"};
        const void* tab = trd_tables(c);
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t b_mq = al(mbs), b_list = al(4 * (size_t)mbs), b_out = al(mbs * sizeof(vc1cu_tdecision)),
                     b_lv = levels ? al((size_t)mbs * 768) : 0, b_stat = al(8 * (size_t)mbs);
        const size_t round_bytes = b_mq + b_list + b_out + b_lv;
        uint8_t* base = static_cast<uint8_t*>(
            ensure(c->d_dq, c->dq_cap, 256 + kDqRounds * round_bytes + 2 * b_stat + al(mbs), "cudaMalloc(DQUANT search)"));
        auto* d_sum = reinterpret_cast<unsigned long long*>(base);
        auto rb_at = [&](int r) { return base + 256 + (size_t)r * round_bytes; };
        auto* d_lscale = reinterpret_cast<double*>(base + 256 + kDqRounds * round_bytes);
        auto* d_adj = reinterpret_cast<double*>(base + 256 + kDqRounds * round_bytes + b_stat);
        uint8_t* d_bright = base + 256 + kDqRounds * round_bytes + 2 * b_stat;
        double frame_mean = 0.0;
        ck(trd_frame_mean(P, fs.view(), *cfg, d_sum, c->stream, &frame_mean), "frame mean");
        std::vector<std::vector<int>> lists(kDqRounds);
        std::vector<std::vector<uint8_t>> mqs(kDqRounds, std::vector<uint8_t>((size_t)mbs, 0));
        std::vector<std::vector<vc1cu_tdecision>> res(kDqRounds);
        // round r: the transform RD of lists[r] at MQUANT mqs[r] with DQUANTFRM dqf, decisions back
        auto run = [&](int r, int dqf) {
            const int n = (int)lists[r].size();
            if (!n) return;
            uint8_t* b = rb_at(r);
            auto* d_list = reinterpret_cast<int*>(b + b_mq);
            auto* d_out = reinterpret_cast<vc1cu_tdecision*>(b + b_mq + b_list);
            auto* d_lv = levels ? reinterpret_cast<int16_t*>(b + b_mq + b_list + b_out) : nullptr;
            ck(cudaMemcpyAsync(b, mqs[r].data(), (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload MQUANT");
            ck(cudaMemcpyAsync(d_list, lists[r].data(), 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream), "upload MB list");
            vc1cu_trd_cfg t = *cfg;
            t.dquantfrm = dqf;
            {
                Timer tm(c, kXform);
                ck(launch_trd(P, fs.view(), fp.view(), tab, b, t, d_sum, d_out, d_lv, c->stream, d_list, n, frame_mean),
                   "transform RD launch");
                tm.stop(1);
            }
            res[r].resize(n);
            ck(cudaMemcpyAsync(res[r].data(), d_out, n * sizeof(vc1cu_tdecision), cudaMemcpyDeviceToHost, c->stream),
               "cudaMemcpyAsync(decisions)");
            sync_checked(c);
        };
        // the base decision (:308-309): DQUANTFRM set where the base MQUANT is not PQINDEX
        std::vector<vc1cu_tdecision> dec((size_t)mbs);
        std::vector<int> mq_out((size_t)mbs), src_round((size_t)mbs), src_pos((size_t)mbs);
        for (int mb = 0; mb < mbs; ++mb) {
            const int r = rate_base[mb] == P.pq ? 0 : 1;
            lists[r].push_back(mb);
            mqs[r][mb] = rate_base[mb];
        }
        run(0, 0);
        run(1, 1);
        for (int r = 0; r < 2; ++r)
            for (size_t i = 0; i < lists[r].size(); ++i) {
                const int mb = lists[r][i];
                dec[mb] = res[r][i];
                mq_out[mb] = rate_base[mb];
                src_round[mb] = r;
                src_pos[mb] = (int)i;
            }
        if (dquant && cfg->adaptive_quality && cfg->aq_strength > 0.0) {
            ck(launch_dquant_stats(P, fs.view(), fp.view(), *cfg, frame_mean, d_lscale, d_adj, d_bright, c->stream),
               "DQUANT statistics launch");
            std::vector<double> lscale((size_t)mbs), adj((size_t)mbs);
            std::vector<uint8_t> bright((size_t)mbs);
            ck(cudaMemcpyAsync(lscale.data(), d_lscale, 8 * (size_t)mbs, cudaMemcpyDeviceToHost, c->stream), "read scales");
            ck(cudaMemcpyAsync(adj.data(), d_adj, 8 * (size_t)mbs, cudaMemcpyDeviceToHost, c->stream), "read adjacency");
            ck(cudaMemcpyAsync(bright.data(), d_bright, (size_t)mbs, cudaMemcpyDeviceToHost, c->stream), "read flags");
            sync_checked(c);
            // the finer absolute MQUANT (:318-370)
            std::vector<uint8_t> done((size_t)mbs, 0);
            for (int mb = 0; mb < mbs; ++mb) {
                const int rb = rate_base[mb];
                if (rb <= 2 || rb < 12 || !(adj[mb] >= 0.80 || bright[mb] || predictable_texture)) continue;
                const int implied = std::clamp(
                    static_cast<int>(std::lround(static_cast<double>(rb) * std::sqrt(std::clamp(lscale[mb], 0.18, 1.0)))), 1, rb);
                const int cap = adj[mb] >= 0.80 ? 16 : (bright[mb] ? 2 : 1);
                const int protected_implied = adj[mb] >= 0.80 ? std::max(1, implied - 4) : implied;
                const int mq = predictable_texture ? std::max(1, rb - 1) : std::max(protected_implied, rb - cap);
                if (mq < rb) {
                    lists[2].push_back(mb);
                    mqs[2][mb] = (uint8_t)mq;
                }
            }
            run(2, 1);
            for (size_t i = 0; i < lists[2].size(); ++i) {
                const int mb = lists[2][i];
                if (res[2][i].cbp || dec[mb].cbp) {
                    dec[mb] = res[2][i];
                    mq_out[mb] = mqs[2][mb];
                    src_round[mb] = 2;
                    src_pos[mb] = (int)i;
                    done[mb] = 1;
                }
            }
            // the coarser candidates of an unprotected coded MB (:372-403), each MQUANT evaluated
            // once; the acceptance below keeps the reference's order and 0.9995 rule
            std::vector<int> eligible;
            std::vector<std::array<int, 3>> cand_mq;
            std::vector<std::array<int, 3>> cand_pos;
            for (int mb = 0; mb < mbs; ++mb) {
                const int rb = rate_base[mb];
                if (rb <= 2 || done[mb] || !dec[mb].cbp || rb >= 31 || lscale[mb] < 1.0 - 1e-12) continue;
                const int md = std::min(4, 31 - rb);
                const std::array<int, 3> deltas = P.halfqp ? std::array<int, 3>{1, 1, 1}
                                                           : std::array<int, 3>{std::max(1, md / 2), md, std::max(1, md - 1)};
                std::array<int, 3> mq{}, pos{-1, -1, -1};
                for (int k = 0; k < 3; ++k) {
                    mq[k] = std::min(31, rb + deltas[k]);
                    bool dup = false;
                    for (int j = 0; j < k; ++j) dup |= mq[j] == mq[k];
                    if (dup) continue;
                    pos[k] = (int)lists[3 + k].size();
                    lists[3 + k].push_back(mb);
                    mqs[3 + k][mb] = (uint8_t)mq[k];
                }
                eligible.push_back(mb);
                cand_mq.push_back(mq);
                cand_pos.push_back(pos);
            }
            for (int k = 0; k < 3; ++k) run(3 + k, 1);
            for (size_t e = 0; e < eligible.size(); ++e) {
                const int mb = eligible[e], rb = rate_base[mb];
                const double base_q = static_cast<double>(2 * rb + ((rb == P.pq && P.halfqp) ? 1 : 0));
                const double lambda = 0.75 * base_q * base_q * lscale[mb];
                auto rd = [&](const vc1cu_tdecision& t) {
                    return t.distortion + lambda * static_cast<double>(static_cast<uint64_t>(t.estimated_bits) + (t.cbp ? 3u : 0u));
                };
                double best_rd = rd(dec[mb]);
                int tried[3], n_tried = 0;
                for (int k = 0; k < 3; ++k) {
                    const int mq = cand_mq[e][k];
                    if (mq <= mq_out[mb]) continue;
                    bool again = false;
                    for (int i = 0; i < n_tried; ++i) again |= tried[i] == mq;
                    if (again) continue;
                    tried[n_tried++] = mq;
                    int r = 3 + k, pos = cand_pos[e][k];
                    for (int j = 0; pos < 0 && j < k; ++j)  // a repeated MQUANT was evaluated at its first index
                        if (cand_mq[e][j] == mq) {
                            r = 3 + j;
                            pos = cand_pos[e][j];
                        }
                    const double crd = rd(res[r][pos]);
                    if (crd < best_rd * 0.9995) {
                        dec[mb] = res[r][pos];
                        mq_out[mb] = mq;
                        best_rd = crd;
                        src_round[mb] = r;
                        src_pos[mb] = pos;
                    }
                }
            }
        }
        for (int mb = 0; mb < mbs; ++mb) {
            out[mb] = dec[mb];
            mquant_out[mb] = (uint8_t)mq_out[mb];
        }
        if (levels) {
            std::vector<int16_t> lv;
            for (int r = 0; r < kDqRounds; ++r) {
                const int n = (int)lists[r].size();
                if (!n) continue;
                lv.resize((size_t)n * 384);
                ck(cudaMemcpyAsync(lv.data(), rb_at(r) + b_mq + b_list + b_out, (size_t)n * 768, cudaMemcpyDeviceToHost,
                                   c->stream),
                   "cudaMemcpyAsync(levels)");
                sync_checked(c);
                for (int mb = 0; mb < mbs; ++mb)
                    if (src_round[mb] == r) std::memcpy(levels + (size_t)mb * 384, lv.data() + (size_t)src_pos[mb] * 384, 768);
            }
        }
        return VC1CU_OK;
    });
}

// ---- the P picture's motion-mode decision (analyze_p_picture, encoder_motion.cpp:524-597) ----

// unary_mode_bits and p_mv_mode_index (encoder_motion.cpp:1116-1143): the MVMODE (and, with
// intensity compensation, MVMODE2) unary codes of a progressive P picture.
static int unary_mode_bits(int index, int maximum) { return index < maximum ? index + 1 : maximum; }
static int p_mv_mode_index(int mode, int pq, bool secondary) {
    if (secondary) {
        if (pq <= 12) return mode == VC1CU_MV_QPEL ? 0 : mode == VC1CU_MV_MIXED ? 1 : mode == VC1CU_MV_HPEL ? 2 : 3;
        return mode == VC1CU_MV_HPEL_BILINEAR ? 0 : mode == VC1CU_MV_QPEL ? 1 : mode == VC1CU_MV_HPEL ? 2 : 3;
    }
    if (pq <= 12) {
        if (mode == VC1CU_MV_QPEL) return 0;
        if (mode == VC1CU_MV_MIXED) return 1;
        if (mode == VC1CU_MV_HPEL) return 2;
        if (mode == VC1CU_MV_HPEL_BILINEAR) return 4;
    } else {
        if (mode == VC1CU_MV_HPEL_BILINEAR) return 0;
        if (mode == VC1CU_MV_QPEL) return 1;
        if (mode == VC1CU_MV_HPEL) return 2;
        if (mode == VC1CU_MV_MIXED) return 4;
    }
    return 3;
}

// The mode decision's device buffer: 7 counters, the sampled MB list, their decisions.
constexpr int kModeRdSamples = 32;
static uint8_t* mrd_buffer(vc1cu_ctx* c) {
    return static_cast<uint8_t*>(ensure(c->d_mrd, c->mrd_cap, 256 + 256 + kModeRdSamples * sizeof(vc1cu_tdecision),
                                        "cudaMalloc(mode decision buffers)"));
}

// estimate_p_motion_bits (encoder_motion.cpp:444-486) of result slot s, analysed in `mode`.
static uint64_t p_motion_bits(vc1cu_ctx* c, const DevParams& P, const ResultSlot& s, int mode, bool intensity) {
    auto* acc = reinterpret_cast<unsigned long long*>(mrd_buffer(c));
    Timer tm(c, kMc);
    ck(launch_p_motion_bits(P, s.r, mode, acc, c->stream), "motion-bit launch");
    tm.stop(mode == VC1CU_MV_MIXED ? 2 : 1);
    unsigned long long h[7];
    ck(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync(motion bits)");
    sync_checked(c);
    if (h[5]) throw Fail{VC1CU_ERR_STATE, "a half-pel MV differential is not representable from its predictor"};
    uint64_t bits = 2;  // MVTAB
    if (intensity)
        bits += (uint64_t)unary_mode_bits(3, 4) + (uint64_t)unary_mode_bits(p_mv_mode_index(mode, P.pq, true), 3) + 12;
    else
        bits += (uint64_t)unary_mode_bits(p_mv_mode_index(mode, P.pq, false), 4);
    if (mode == VC1CU_MV_MIXED) bits += h[6];  // MVTYPEMB
    bits += h[4];                              // hybrid-predictor flags
    uint64_t table = h[0];                     // choose_mv_table: the least of the four
    for (int t = 1; t < 4; ++t) table = h[t] < table ? h[t] : table;
    return bits + table;
}

// The mode RD's sample (sampled_p_mode_rd :504-508, sampled_b_mode_rd :1024-1028): up to 32
// macroblocks evenly spaced in raster order.
static std::vector<int> mode_rd_sample(const DevParams& P) {
    const int total = P.mbw * P.mbh;
    std::vector<int> list;
    if (total <= 0) return list;
    const int wanted = std::min(kModeRdSamples, total);
    const int stride = std::max(1, total / wanted);
    for (int linear = 0; linear < total && (int)list.size() < wanted; linear += stride) list.push_back(linear);
    return list;
}

// lambda = 0.75 * q^2 with q = picture_double_quant(PQINDEX, false)
static double mode_rd_lambda(const DevParams& P) {
    const int q = 2 * P.pq + (P.halfqp ? 1 : 0);
    return 0.75 * static_cast<double>(q) * static_cast<double>(q);
}

// The fixed-8x8 shortcut of choose_transform_mb (encoder_transform.cpp:1610-1634): an empty
// decision, no distortion and no bits.
static bool fixed_8x8_shortcut(const vc1cu_ppic_cfg& cfg) {
    return !cfg.trd.variable_transforms && cfg.fast_transform_rdo && !cfg.dquant && cfg.trd.trellis == 0;
}

// The AQ-neutral transform RD (at PQINDEX, no DQUANT, per-MB types, the picture's decision
// coding set) of the listed macroblocks of cur_id against the prediction in frame slot pred_id.
static std::vector<vc1cu_tdecision> sampled_decisions(vc1cu_ctx* c, const DevParams& P, const vc1cu_ppic_cfg& cfg,
                                                      int cur_id, int pred_id, const std::vector<int>& list) {
    const int n = (int)list.size();
    FrameSlot& fc = frame_slot(c, cur_id);
    FrameSlot& fp = frame_slot(c, pred_id);
    uint8_t* base = mrd_buffer(c);
    auto* d_list = reinterpret_cast<int*>(base + 256);
    auto* d_out = reinterpret_cast<vc1cu_tdecision*>(base + 512);
    ck(cudaMemcpyAsync(d_list, list.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync(list)");
    vc1cu_trd_cfg t = cfg.trd;
    t.adaptive_quality = 0;
    t.aq_strength = 0.0;
    t.coding_set = P.pq <= 8 ? 1 : 3;  // chroma_coding_set(PQINDEX <= 8 ? 1 : 0, PQINDEX)
    t.dquantfrm = 0;
    t.frame_type = 0;
    {
        Timer tm(c, kXform);
        ck(launch_trd(P, fc.view(), fp.view(), trd_tables(c), nullptr, t, nullptr, d_out, nullptr, c->stream, d_list, n, -1.0),
           "transform RD launch");
        tm.stop(1);
    }
    std::vector<vc1cu_tdecision> dec(n);
    ck(cudaMemcpyAsync(dec.data(), d_out, n * sizeof(vc1cu_tdecision), cudaMemcpyDeviceToHost, c->stream),
       "cudaMemcpyAsync(decisions)");
    sync_checked(c);
    return dec;
}

// sampled_p_mode_rd (encoder_motion.cpp:488-522): the prediction of slot s against pred_ref and
// the AQ-neutral transform RD of the sampled macroblocks, combined with the motion bits in long
// double exactly as the reference does.
static long double sampled_mode_rd(vc1cu_ctx* c, const DevParams& P, const vc1cu_ppic_cfg& cfg, int cur_id, int pred_ref_id,
                                   const ResultSlot& s, int mode, uint64_t motion_bits, int pred_id) {
    const int total = P.mbw * P.mbh;
    const std::vector<int> list = mode_rd_sample(P);
    if (list.empty()) return 0.0L;
    const double lambda = mode_rd_lambda(P);
    long double rd = 0.0L;
    if (!fixed_8x8_shortcut(cfg)) {
        FrameSlot& fr = frame_slot(c, pred_ref_id);
        FrameSlot& fp = alloc_frame(c, pred_id, P.W, P.H);
        {
            Timer tm(c, kMc);
            launch_mc(P, fr.view(), s.r.mvs, s.r.bmv, s.r.use4, mode, (uint8_t*)fp.view().y, (uint8_t*)fp.view().u,
                      (uint8_t*)fp.view().v, fp.pitch_y, fp.pitch_c, c->stream);
            ck(cudaGetLastError(), "mc_kernel launch");
            tm.stop(1);
        }
        for (const vc1cu_tdecision& d : sampled_decisions(c, P, cfg, cur_id, pred_id, list))
            rd += static_cast<long double>(d.distortion) + lambda * static_cast<long double>(d.estimated_bits);
    }
    const long double residual_per_mb = rd / static_cast<long double>(list.size());
    const long double motion_per_mb = static_cast<long double>(motion_bits) / static_cast<long double>(total);
    return residual_per_mb + lambda * motion_per_mb;
}

// sampled_b_mode_rd (encoder_motion.cpp:1006-1060) of the B analysis in b: the B prediction of
// the sampled macroblocks (B-intra ones from their blocks' visible means), their AQ-neutral
// transform RD, 72 bits of intra syntax per B-intra sample, and the analysis's motion bits.
static long double sampled_b_rd(vc1cu_ctx* c, const DevParams& P, const vc1cu_ppic_cfg& cfg, int cur_id, int past_id,
                                int future_id, const BSlot& b, int pred_id) {
    const int total = P.mbw * P.mbh;
    const std::vector<int> list = mode_rd_sample(P);
    if (list.empty()) return 0.0L;
    std::vector<uint8_t> modes((size_t)total);
    vc1cu_banalysis ba{};
    ba.modes = modes.data();
    read_bresult(c, b, &ba);
    const double lambda = mode_rd_lambda(P);
    std::vector<vc1cu_tdecision> dec(list.size());  // the shortcut's empty decisions
    if (!fixed_8x8_shortcut(cfg)) {
        FrameSlot& fc = frame_slot(c, cur_id);
        FrameSlot& fp = frame_slot(c, past_id);
        FrameSlot& ff = frame_slot(c, future_id);
        FrameSlot& fo = alloc_frame(c, pred_id, P.W, P.H);
        {
            Timer tm(c, kMc);
            ck(launch_b_mc(P, fc.view(), fp.view(), ff.view(), b.r.modes, b.r.fmv, b.r.bmv, b.mode, (uint8_t*)fo.view().y,
                           (uint8_t*)fo.view().u, (uint8_t*)fo.view().v, fo.pitch_y, fo.pitch_c, c->stream),
               "B prediction launch");
            tm.stop(1);
        }
        dec = sampled_decisions(c, P, cfg, cur_id, pred_id, list);
    }
    long double rd = 0.0L;
    for (size_t i = 0; i < list.size(); ++i) {
        rd += static_cast<long double>(dec[i].distortion) + lambda * static_cast<long double>(dec[i].estimated_bits);
        if (modes[(size_t)list[i]] == VC1CU_BMB_INTRA) rd += lambda * 72.0L;
    }
    const long double residual_per_mb = rd / static_cast<long double>(list.size());
    const long double motion_per_mb = static_cast<long double>(ba.motion_bits) / static_cast<long double>(total);
    return residual_per_mb + lambda * motion_per_mb;
}

int vc1cu_p_motion_bits(vc1cu_ctx* c, const vc1cu_params* p, int slot, int mv_mode, int intensity, uint64_t* bits) {
    return guarded(c, [&]() -> int {
        if (!bits) throw Fail{VC1CU_ERR_ARG, "null output"};
        if (mv_mode < 0 || mv_mode > 3) throw Fail{VC1CU_ERR_ARG, "invalid MV mode"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        ResultSlot& s = result_slot(c, slot, P.mbw * P.mbh, false);
        check_status(c);
        *bits = p_motion_bits(c, P, s, mv_mode, intensity != 0);
        return VC1CU_OK;
    });
}

int vc1cu_analyze_p_picture(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_ppic_cfg* cfg, int cur_id, int ref_id,
                            int out_slot, int scratch_slot, int scratch_frame, vc1cu_ppic_info* info) {
    return guarded(c, [&]() -> int {
        if (!cfg) throw Fail{VC1CU_ERR_ARG, "null configuration"};
        const int n = cfg->n_modes;
        if (n != 1 && n != 3 && n != 4) throw Fail{VC1CU_ERR_ARG, "n_modes must be 1, 3 or 4"};
        if (cfg->trd.trellis < 0 || cfg->trd.trellis > 2) throw Fail{VC1CU_ERR_ARG, "invalid trellis"};
        if (out_slot < 0 || out_slot >= kMaxSlot || scratch_slot < 0 || scratch_slot + 8 > kMaxSlot ||
            (out_slot >= scratch_slot && out_slot < scratch_slot + 8))
            throw Fail{VC1CU_ERR_ARG, "result slots out of range or overlapping"};
        if (scratch_frame < 0 || scratch_frame + 2 > kMaxSlot || cur_id == scratch_frame || cur_id == scratch_frame + 1 ||
            ref_id == scratch_frame || ref_id == scratch_frame + 1)
            throw Fail{VC1CU_ERR_ARG, "scratch frame slots out of range or overlapping the pictures"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        {
            FrameSlot& fc = frame_slot(c, cur_id);
            FrameSlot& fr = frame_slot(c, ref_id);
            if (fc.w != P.W || fc.h != P.H || fr.w != P.W || fr.h != P.H)
                throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
        }
        const int mbs = P.mbw * P.mbh;
        const int modes[4] = {VC1CU_MV_QPEL, VC1CU_MV_HPEL, VC1CU_MV_HPEL_BILINEAR, VC1CU_MV_MIXED};
        const int pred_id = scratch_frame, comp_id = scratch_frame + 1;
        vc1cu_ppic_info inf{};
        auto mean_abs_residual = [&](int slot) {
            vc1cu_panalysis a{};
            ResultSlot& s = result_slot(c, slot, mbs, false);
            check_status_read(c, s.written);
            read_result(c, s, &a);
            return a.mean_abs_residual;
        };
        // the seed pass and the seeded mode passes over reference r into slots base..base+n-1,
        // each scored; returns the candidate index with the strictly least score
        auto candidates = [&](int r, int base, bool intensity, long double& best_score) {
            std::vector<vc1cu_pass> passes;
            passes.push_back(vc1cu_pass{cur_id, r, VC1CU_MV_QPEL, 0, -1, base, 0});
            for (int i = 1; i < n; ++i) passes.push_back(vc1cu_pass{cur_id, r, modes[i], 0, base, base + i, 0});
            launch_passes(c, p, passes.data(), n);
            stamp_written(c);
            check_status(c);
            int best = 0;
            best_score = std::numeric_limits<long double>::infinity();
            for (int i = 0; i < n; ++i) {
                ResultSlot& s = result_slot(c, base + i, mbs, false);
                const uint64_t bits = p_motion_bits(c, P, s, modes[i], intensity);
                const long double sc = sampled_mode_rd(c, P, *cfg, cur_id, r, s, modes[i], bits, pred_id);
                const int k = (intensity ? 4 : 0) + i;
                inf.cand_bits[k] = bits;
                inf.cand_score[k] = static_cast<double>(sc);
                if (sc < best_score) {
                    best_score = sc;
                    best = i;
                }
            }
            return best;
        };
        long double best_score;
        const int best = candidates(ref_id, scratch_slot, false, best_score);
        const vc1cu_pass fin{cur_id, ref_id, modes[best], 1, scratch_slot + best, out_slot, 0};
        launch_passes(c, p, &fin, 1);
        stamp_written(c);
        check_status(c);
        inf.mode = modes[best];
        inf.motion_bits = p_motion_bits(c, P, result_slot(c, out_slot, mbs, false), modes[best], false);
        if (cfg->fade_compensation) {
            // estimate_intensity_comp on the chosen analysis, then the weighted candidates
            const vc1cu_icpass icp{cur_id, ref_id, out_slot};
            ic_estimate(c, P, ic_jobs(c, P, &icp, 1), &inf.ic);
            if (inf.ic.enabled) {
                ic_compensate(c, ref_id, &inf.ic, comp_id);
                long double w_score;
                const int wbest = candidates(comp_id, scratch_slot + 4, true, w_score);
                const double mar = mean_abs_residual(out_slot);
                const double need = std::max(0.25, mar * cfg->fade_min_gain);
                if (!(mean_abs_residual(scratch_slot + 4 + wbest) + need >= mar || w_score >= best_score)) {
                    const vc1cu_pass wfin{cur_id, comp_id, modes[wbest], 1, scratch_slot + 4 + wbest, out_slot, 0};
                    launch_passes(c, p, &wfin, 1);
                    stamp_written(c);
                    check_status(c);
                    inf.mode = modes[wbest];
                    inf.weighted = 1;
                    inf.motion_bits = p_motion_bits(c, P, result_slot(c, out_slot, mbs, false), modes[wbest], true);
                }
            }
        }
        if (info) *info = inf;
        return VC1CU_OK;
    });
}

int vc1cu_b_mode_rd(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_ppic_cfg* cfg, int cur_id, int past_id,
                    int future_id, int bslot_qpel, int bslot_bilinear, int pred_id, int* choice, double* scores) {
    return guarded(c, [&]() -> int {
        if (!cfg || !choice) throw Fail{VC1CU_ERR_ARG, "null configuration or output"};
        if (cfg->trd.trellis < 0 || cfg->trd.trellis > 2) throw Fail{VC1CU_ERR_ARG, "invalid trellis"};
        if (pred_id < 0 || pred_id >= kMaxSlot || pred_id == cur_id || pred_id == past_id || pred_id == future_id)
            throw Fail{VC1CU_ERR_ARG, "invalid prediction slot"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        auto slot = [&](int id, int mode) -> const BSlot& {
            auto it = c->bresults.find(id);
            if (it == c->bresults.end() || !it->second.valid || it->second.mbs != P.mbw * P.mbh)
                throw Fail{VC1CU_ERR_STATE, "B-result slot holds no analysis of this size"};
            if (it->second.mode != mode) throw Fail{VC1CU_ERR_ARG, "B-result slot analysed in another mode"};
            return it->second;
        };
        const BSlot& q = slot(bslot_qpel, VC1CU_MV_QPEL);
        const BSlot& h = slot(bslot_bilinear, VC1CU_MV_HPEL_BILINEAR);
        for (int id : {cur_id, past_id, future_id}) {
            FrameSlot& f = frame_slot(c, id);
            if (f.w != P.W || f.h != P.H) throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
        }
        check_status(c);
        const long double qs = sampled_b_rd(c, P, *cfg, cur_id, past_id, future_id, q, pred_id);
        const long double hs = sampled_b_rd(c, P, *cfg, cur_id, past_id, future_id, h, pred_id);
        *choice = hs < qs ? 1 : 0;
        if (scores) {
            scores[0] = static_cast<double>(qs);
            scores[1] = static_cast<double>(hs);
        }
        return VC1CU_OK;
    });
}

// The deblocking filters take the coding raster or the padded raster the reference's
// reconstruction uses (whole macroblocks); they filter the frame's own extent.
static bool filter_size_ok(const DevParams& P, const FrameSlot& f) {
    return (f.w == P.W && f.h == P.H) || (f.w == P.mbw * 16 && f.h == P.mbh * 16);
}

int vc1cu_loop_filter_i(vc1cu_ctx* c, const vc1cu_params* p, int frame_id) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& f = frame_slot(c, frame_id);
        if (!filter_size_ok(P, f)) throw Fail{VC1CU_ERR_ARG, "frame size is neither the raster nor the padded raster"};
        const DevFrame d = f.view();
        Timer tm(c, kMc);
        ck(launch_loop_filter_i((uint8_t*)d.y, (uint8_t*)d.u, (uint8_t*)d.v, f.pitch_y, f.pitch_c, f.w, f.h, P.pq, c->stream),
           "loop filter launch");
        tm.stop(2);
        return VC1CU_OK;
    });
}

// The P-picture deblocking of vc1cu_loop_filter_p (main_profile 0) and
// vc1cu_loop_filter_p_main (1).
static int loop_filter_p(vc1cu_ctx* c, const vc1cu_params* p, int frame_id, const vc1cu_mv* block_mvs, const uint8_t* cbp,
                         const uint8_t* tt, const uint8_t* intra, int main_profile) {
    return guarded(c, [&]() -> int {
        if (!block_mvs || !cbp || !tt || !intra) throw Fail{VC1CU_ERR_ARG, "null block metadata"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& f = frame_slot(c, frame_id);
        if (!filter_size_ok(P, f)) throw Fail{VC1CU_ERR_ARG, "frame size is neither the raster nor the padded raster"};
        const size_t mbs = (size_t)P.mbw * P.mbh;
        for (size_t i = 0; i < mbs * 6; ++i)
            if (cbp[i] > 15 || !(tt[i] == 0 || tt[i] == 3 || tt[i] == 6 || tt[i] == 7))
                throw Fail{VC1CU_ERR_ARG, "block patterns are 4-bit and transform kinds 0, 3, 6 or 7"};
        const size_t bm = 32 * mbs, al = (bm + 255) & ~size_t(255);
        uint8_t* d = static_cast<uint8_t*>(ensure(c->d_lf, c->lf_cap, al + 13 * mbs + 256, "cudaMalloc(loop filter metadata)"));
        ck(cudaMemcpyAsync(d, block_mvs, bm, cudaMemcpyHostToDevice, c->stream), "upload block vectors");
        ck(cudaMemcpyAsync(d + al, cbp, 6 * mbs, cudaMemcpyHostToDevice, c->stream), "upload block patterns");
        ck(cudaMemcpyAsync(d + al + 6 * mbs, tt, 6 * mbs, cudaMemcpyHostToDevice, c->stream), "upload transform kinds");
        ck(cudaMemcpyAsync(d + al + 12 * mbs, intra, mbs, cudaMemcpyHostToDevice, c->stream), "upload intra bits");
        const DevFrame fr = f.view();
        Timer tm(c, kMc);
        ck(launch_loop_filter_p((uint8_t*)fr.y, (uint8_t*)fr.u, (uint8_t*)fr.v, f.pitch_y, f.pitch_c, f.w, f.h, P.pq,
                                reinterpret_cast<const int2*>(d), d + al, d + al + 6 * mbs, d + al + 12 * mbs, c->stream,
                                main_profile),
           "loop filter launch");
        tm.stop(2);
        // the metadata copies read the caller's pageable arrays; finish before returning
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        return VC1CU_OK;
    });
}

int vc1cu_loop_filter_p(vc1cu_ctx* c, const vc1cu_params* p, int frame_id, const vc1cu_mv* block_mvs, const uint8_t* cbp,
                        const uint8_t* tt, const uint8_t* intra) {
    return loop_filter_p(c, p, frame_id, block_mvs, cbp, tt, intra, 0);
}

int vc1cu_loop_filter_p_main(vc1cu_ctx* c, const vc1cu_params* p, int frame_id, const vc1cu_mv* block_mvs,
                             const uint8_t* cbp, const uint8_t* tt, const uint8_t* intra) {
    return loop_filter_p(c, p, frame_id, block_mvs, cbp, tt, intra, 1);
}

// The signed intra reconstruction of frame slot src_id (HOST flags / mquant / derived, copied on the
// context stream) into the device planes d_y, d_u, d_v, with the trellis and perceptual settings of cfg.
static void intra_recon(vc1cu_ctx* c, const DevParams& P, const vc1cu_trd_cfg& cfg, FrameSlot& fs, int overlap,
                        const uint8_t* flags, const uint8_t* mquant, const uint8_t* derived, int32_t* d_y, int32_t* d_u,
                        int32_t* d_v) {
    const size_t mbs = (size_t)P.mbw * P.mbh;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_scr = al(intra_scratch_bytes(P)), b_edge = al(mbs * 256 * 3 / 2), b_map = al(mbs);
    uint8_t* base = static_cast<uint8_t*>(
        ensure(c->d_intra, c->intra_cap, b_scr + b_edge + 3 * b_map, "cudaMalloc(intra reconstruction)"));
    uint8_t* d_flags = base + b_scr + b_edge;
    uint8_t* d_mq = d_flags + b_map;
    uint8_t* d_der = d_mq + b_map;
    if (overlap == 2) ck(cudaMemcpyAsync(d_flags, flags, mbs, cudaMemcpyHostToDevice, c->stream), "upload overlap flags");
    if (mquant) ck(cudaMemcpyAsync(d_mq, mquant, mbs, cudaMemcpyHostToDevice, c->stream), "upload MQUANT");
    if (derived) ck(cudaMemcpyAsync(d_der, derived, mbs, cudaMemcpyHostToDevice, c->stream), "upload derived flags");
    Timer tm(c, kXform);
    ck(launch_intra_recon(P, fs.view(), overlap, overlap == 2 ? d_flags : nullptr, mquant ? d_mq : nullptr,
                          derived ? d_der : nullptr, base, base + b_scr, d_y, d_u, d_v,
                          cfg.trellis > 0 ? trd_tables(c) : nullptr, cfg, c->stream),
       "intra reconstruction launch");
    tm.stop(overlap ? 4 : 3);
}

// The intra settings of cfg (NULL: scalar levels, no perceptual scale).
static vc1cu_trd_cfg intra_cfg(const vc1cu_trd_cfg* cfg) {
    vc1cu_trd_cfg k{};
    if (cfg) {
        if (cfg->trellis < 0 || cfg->trellis > 2) throw Fail{VC1CU_ERR_ARG, "trellis is 0, 1 or 2"};
        k.trellis = cfg->trellis;
        k.adaptive_quality = cfg->adaptive_quality;
        k.aq_strength = cfg->aq_strength;
        k.hrd_enabled = cfg->hrd_enabled;
    }
    return k;
}

static void check_intra_args(const DevParams& P, FrameSlot& fs, const uint8_t* mquant) {
    if (fs.w != P.W || fs.h != P.H) throw Fail{VC1CU_ERR_ARG, "frame size does not match the configuration"};
    if (mquant)
        for (size_t i = 0; i < (size_t)P.mbw * P.mbh; ++i)
            if (mquant[i] < 1 || mquant[i] > 31) throw Fail{VC1CU_ERR_ARG, "MQUANT must be 1..31"};
}

int vc1cu_reconstruct_intra(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id, int overlap,
                            const uint8_t* flags, const uint8_t* mquant, const uint8_t* derived, int32_t* d_y,
                            int32_t* d_u, int32_t* d_v) {
    return guarded(c, [&]() -> int {
        if (!d_y || !d_u || !d_v) throw Fail{VC1CU_ERR_ARG, "null signed plane"};
        if (overlap < 0 || overlap > 2) throw Fail{VC1CU_ERR_ARG, "overlap is 0 none, 1 all or 2 select"};
        if (overlap == 2 && !flags) throw Fail{VC1CU_ERR_ARG, "null overlap flags"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& fs = frame_slot(c, src_id);
        check_intra_args(P, fs, mquant);
        intra_recon(c, P, intra_cfg(cfg), fs, overlap, flags, mquant, derived, d_y, d_u, d_v);
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");  // the copies read the caller's arrays
        return VC1CU_OK;
    });
}

int vc1cu_choose_i_overlap(vc1cu_ctx* c, const vc1cu_params* p, const vc1cu_trd_cfg* cfg, int src_id,
                           const uint8_t* mquant, const uint8_t* derived, int* mode, uint8_t* flags) {
    return guarded(c, [&]() -> int {
        if (!mode || !flags) throw Fail{VC1CU_ERR_ARG, "null output"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& fs = frame_slot(c, src_id);
        check_intra_args(P, fs, mquant);
        const vc1cu_trd_cfg icfg = intra_cfg(cfg);
        const size_t mbs = (size_t)P.mbw * P.mbh;
        std::fill(flags, flags + mbs, (uint8_t)0);
        if (P.pq >= 9) {  // unconditional overlap above the CONDOVER range (:290-294)
            *mode = 1;
            return VC1CU_OK;
        }
        // three signed reconstructions (no smoothing, every edge, the selected edges), their
        // per-MB errors, the flags and the OVERFLAGS bitplane's bits
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t ny = mbs * 256, nc = mbs * 64, b_rec = al(4 * (ny + 2 * nc)), b_sse = al(8 * mbs);
        uint8_t* base = static_cast<uint8_t*>(
            ensure(c->d_iovl, c->iovl_cap, 3 * b_rec + 3 * b_sse + al(mbs) + 256, "cudaMalloc(overlap plan)"));
        auto rec = [&](int k, int pl) {
            int32_t* r = reinterpret_cast<int32_t*>(base + (size_t)k * b_rec);
            return pl == 0 ? r : (pl == 1 ? r + ny : r + ny + nc);
        };
        auto* sse = reinterpret_cast<unsigned long long*>(base + 3 * b_rec);
        uint8_t* d_flags = base + 3 * b_rec + 3 * b_sse;
        auto* d_bits = reinterpret_cast<unsigned long long*>(d_flags + al(mbs));
        const DevFrame src = fs.view();
        auto errors = [&](int k) {
            ck(launch_overlap_sse(rec(k, 0), rec(k, 1), rec(k, 2), src.y, src.u, src.v, src.pitch_y, src.pitch_c, P.W, P.H,
                                  128, sse + (size_t)k * mbs, c->stream),
               "overlap error launch");
        };
        intra_recon(c, P, icfg, fs, 0, nullptr, mquant, derived, rec(0, 0), rec(0, 1), rec(0, 2));
        ck(cudaMemcpyAsync(rec(1, 0), rec(0, 0), 4 * (ny + 2 * nc), cudaMemcpyDeviceToDevice, c->stream), "copy reconstruction");
        ck(launch_overlap(rec(1, 0), rec(1, 1), rec(1, 2), P.mbw, P.mbh, nullptr, 1, c->stream), "overlap launch");
        errors(0);
        errors(1);
        std::vector<unsigned long long> e((size_t)2 * mbs);
        ck(cudaMemcpyAsync(e.data(), sse, 16 * mbs, cudaMemcpyDeviceToHost, c->stream), "read errors");
        sync_checked(c);
        const long double pq2 = static_cast<long double>(P.pq * P.pq);
        bool any = false, every = true;
        for (size_t i = 0; i < mbs; ++i) {
            const bool on = static_cast<long double>(e[mbs + i]) + pq2 * 4.0L < static_cast<long double>(e[i]);
            flags[i] = on ? 1 : 0;
            any |= on;
            every &= on;
        }
        if (!any) {
            *mode = 0;
            return VC1CU_OK;
        }
        if (every) {
            *mode = 1;
            return VC1CU_OK;
        }
        ck(cudaMemcpyAsync(d_flags, flags, mbs, cudaMemcpyHostToDevice, c->stream), "upload flags");
        ck(launch_bitplane_bits(d_flags, P.mbw, P.mbh, d_bits, c->stream), "bitplane launch");
        ck(cudaMemcpyAsync(rec(2, 0), rec(0, 0), 4 * (ny + 2 * nc), cudaMemcpyDeviceToDevice, c->stream), "copy reconstruction");
        ck(launch_overlap(rec(2, 0), rec(2, 1), rec(2, 2), P.mbw, P.mbh, d_flags, 0, c->stream), "overlap launch");
        errors(2);
        std::vector<unsigned long long> e2(mbs);
        unsigned long long bits = 0;
        ck(cudaMemcpyAsync(e2.data(), sse + 2 * mbs, 8 * mbs, cudaMemcpyDeviceToHost, c->stream), "read errors");
        ck(cudaMemcpyAsync(&bits, d_bits, 8, cudaMemcpyDeviceToHost, c->stream), "read bitplane bits");
        sync_checked(c);
        long double t0 = 0.0L, t1 = 0.0L, t2 = 0.0L;
        for (size_t i = 0; i < mbs; ++i) {
            t0 += static_cast<long double>(e[i]);
            t1 += static_cast<long double>(e[mbs + i]);
            t2 += static_cast<long double>(e2[i]);
        }
        const long double lambda = pq2 * 8.0L;
        const long double nscore = t0 + lambda, ascore = t1 + 2.0L * lambda;
        const long double sscore = t2 + lambda * (2.0L + static_cast<long double>(bits));
        if (nscore <= ascore && nscore <= sscore) {
            *mode = 0;
            std::fill(flags, flags + mbs, (uint8_t)0);
        } else if (ascore <= sscore) {
            *mode = 1;
            std::fill(flags, flags + mbs, (uint8_t)1);
        } else {
            *mode = 2;
        }
        return VC1CU_OK;
    });
}

// The per-macroblock byte map of an overlap call on the device (stream-ordered after any launch
// still reading the previous one).
static const uint8_t* upload_mb_map(vc1cu_ctx* c, const uint8_t* map, size_t mbs) {
    uint8_t* d = static_cast<uint8_t*>(ensure(c->d_ovl, c->ovl_cap, mbs, "cudaMalloc(macroblock map)"));
    ck(cudaMemcpyAsync(d, map, mbs, cudaMemcpyHostToDevice, c->stream), "upload macroblock map");
    return d;
}

int vc1cu_overlap_smooth(vc1cu_ctx* c, const vc1cu_params* p, int32_t* d_y, int32_t* d_u, int32_t* d_v,
                         const uint8_t* flags, int all) {
    return guarded(c, [&]() -> int {
        if (!d_y || !d_u || !d_v) throw Fail{VC1CU_ERR_ARG, "null signed plane"};
        if (!all && !flags) throw Fail{VC1CU_ERR_ARG, "null overlap flags"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const uint8_t* df = all ? nullptr : upload_mb_map(c, flags, (size_t)P.mbw * P.mbh);
        Timer tm(c, kMc);
        ck(launch_overlap(d_y, d_u, d_v, P.mbw, P.mbh, df, all ? 1 : 0, c->stream), "overlap launch");
        tm.stop(2);
        return VC1CU_OK;
    });
}

int vc1cu_store_signed(vc1cu_ctx* c, const vc1cu_params* p, const int32_t* d_y, const int32_t* d_u, const int32_t* d_v,
                       int bias, const uint8_t* mb_mask, int out_id) {
    return guarded(c, [&]() -> int {
        if (!d_y || !d_u || !d_v) throw Fail{VC1CU_ERR_ARG, "null signed plane"};
        if (out_id < 0 || out_id >= kMaxSlot) throw Fail{VC1CU_ERR_ARG, "invalid output frame slot"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        FrameSlot& f = mb_mask ? frame_slot(c, out_id) : alloc_frame(c, out_id, P.mbw * 16, P.mbh * 16);
        const uint8_t* dm = mb_mask ? upload_mb_map(c, mb_mask, (size_t)P.mbw * P.mbh) : nullptr;
        const DevFrame o = f.view();
        Timer tm(c, kMc);
        ck(launch_store_signed(d_y, d_u, d_v, P.mbw, P.mbh, bias, dm, (uint8_t*)o.y, (uint8_t*)o.u, (uint8_t*)o.v,
                               f.pitch_y, f.pitch_c, f.w, f.h, c->stream),
           "signed store launch");
        tm.stop(1);
        return VC1CU_OK;
    });
}

static int reconstruct(vc1cu_ctx* c, const vc1cu_params* p, int pred_id, const int16_t* d_levels, int type_mask,
                       const uint8_t* block_types, const uint8_t* mquant, const uint8_t* derived, int out_id) {
    return guarded(c, [&]() -> int {
        if (!d_levels || !block_types) throw Fail{VC1CU_ERR_ARG, "null levels or block types"};
        if (type_mask < 1 || type_mask > 15) throw Fail{VC1CU_ERR_ARG, "type_mask must select 1..4 transform types"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        const int mbs = P.mbw * P.mbh;
        for (int i = 0; i < mbs * 6; ++i) {
            const int t = block_types[i];
            if (t < 1 || t > 4 || !(type_mask & (1 << (t - 1))))
                throw Fail{VC1CU_ERR_ARG, "a block's transform type is not one of type_mask's"};
        }
        if (out_id < 0 || out_id >= kMaxSlot || out_id == pred_id) throw Fail{VC1CU_ERR_ARG, "invalid output frame slot"};
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fp.w != P.W || fp.h != P.H) throw Fail{VC1CU_ERR_ARG, "prediction size does not match the configuration"};
        const DevFrame pred = fp.view();
        FrameSlot& fo = alloc_frame(c, out_id, P.W, P.H);
        const DevFrame o = fo.view();
        if (mquant)
            for (int i = 0; i < mbs; ++i)
                if (mquant[i] < 1 || mquant[i] > 31) throw Fail{VC1CU_ERR_ARG, "MQUANT must be 1..31"};
        // block types, then the per-MB MQUANT and derived flags (8 bytes per MB in all)
        uint8_t* dt = static_cast<uint8_t*>(ensure(c->d_btypes, c->btypes_cap, (size_t)mbs * 8, "cudaMalloc(block types)"));
        ck(cudaMemcpyAsync(dt, block_types, (size_t)mbs * 6, cudaMemcpyHostToDevice, c->stream), "upload block types");
        uint8_t* dmq = dt + (size_t)mbs * 6;
        uint8_t* dder = dmq + mbs;
        if (mquant) ck(cudaMemcpyAsync(dmq, mquant, (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload MQUANT");
        if (derived) ck(cudaMemcpyAsync(dder, derived, (size_t)mbs, cudaMemcpyHostToDevice, c->stream), "upload derived flags");
        int ti[4], n = 0;
        for (int t = 0; t < 4; ++t) ti[t] = (type_mask >> t) & 1 ? n++ : -1;
        Timer tm(c, kXform);
        launch_recon(P, pred, d_levels, make_int4(ti[0], ti[1], ti[2], ti[3]), dt, (uint8_t*)o.y, (uint8_t*)o.u, (uint8_t*)o.v,
                     fo.pitch_y, fo.pitch_c, c->stream, mquant ? dmq : nullptr, mquant && derived ? dder : nullptr);
        ck(cudaGetLastError(), "reconstruction launch");
        tm.stop(1);
        if (mquant) ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");  // the copies read the caller's arrays
        return VC1CU_OK;
    });
}

int vc1cu_reconstruct(vc1cu_ctx* c, const vc1cu_params* p, int pred_id, const int16_t* d_levels, int type_mask,
                      const uint8_t* block_types, int out_id) {
    return reconstruct(c, p, pred_id, d_levels, type_mask, block_types, nullptr, nullptr, out_id);
}

int vc1cu_reconstruct_dquant(vc1cu_ctx* c, const vc1cu_params* p, int pred_id, const int16_t* d_levels, int type_mask,
                             const uint8_t* block_types, const uint8_t* mquant, const uint8_t* derived, int out_id) {
    if (!mquant) return guarded(c, [&]() -> int { throw Fail{VC1CU_ERR_ARG, "null MQUANT"}; });
    return reconstruct(c, p, pred_id, d_levels, type_mask, block_types, mquant, derived, out_id);
}

int vc1cu_forward_quant_device(vc1cu_ctx* c, const vc1cu_params* p, int src_id, int pred_id, int type_mask,
                               double* d_coeffs, int16_t* d_levels) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        if (type_mask <= 0 || type_mask > 15) throw Fail{VC1CU_ERR_ARG, "type_mask must select 1..4 transform types"};
        FrameSlot& fs = frame_slot(c, src_id);
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fs.w != P.W || fs.h != P.H || fp.w != P.W || fp.h != P.H) throw Fail{VC1CU_ERR_ARG, "frame size mismatch"};
        Timer tm(c, kXform);
        launch_xform(P, fs.view(), fp.view(), type_mask, d_coeffs, d_levels, c->stream);
        ck(cudaGetLastError(), "xform_kernel launch");
        tm.stop(1);
        return VC1CU_OK;
    });
}

int vc1cu_forward_quant(vc1cu_ctx* c, const vc1cu_params* p, int src_id, int pred_id, int type_mask, double* coeffs,
                        int16_t* levels) {
    return guarded(c, [&]() -> int {
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        if (type_mask <= 0 || type_mask > 15) throw Fail{VC1CU_ERR_ARG, "type_mask must select 1..4 transform types"};
        int nt = 0;
        for (int t = 0; t < 4; ++t) nt += (type_mask >> t) & 1;
        const size_t n = (size_t)nt * P.mbw * P.mbh * 6 * 64;
        const size_t cb = n * 8, lb = n * 2;
        ensure(c->d_scratch, c->scratch_cap, cb + lb + 256, "cudaMalloc(transform output)");
        double* dco = static_cast<double*>(c->d_scratch);
        int16_t* dlv = reinterpret_cast<int16_t*>(static_cast<uint8_t*>(c->d_scratch) + ((cb + 255) & ~size_t(255)));
        FrameSlot& fs = frame_slot(c, src_id);
        FrameSlot& fp = frame_slot(c, pred_id);
        if (fs.w != P.W || fs.h != P.H || fp.w != P.W || fp.h != P.H) throw Fail{VC1CU_ERR_ARG, "frame size mismatch"};
        Timer tm(c, kXform);
        launch_xform(P, fs.view(), fp.view(), type_mask, dco, dlv, c->stream);
        ck(cudaGetLastError(), "xform_kernel launch");
        tm.stop(1);
        if (coeffs) ck(cudaMemcpyAsync(coeffs, dco, cb, cudaMemcpyDeviceToHost, c->stream), "download coefficients");
        if (levels) ck(cudaMemcpyAsync(levels, dlv, lb, cudaMemcpyDeviceToHost, c->stream), "download levels");
        sync_checked(c);
        return VC1CU_OK;
    });
}


}  // extern "C"

// ---- learned motion-vector proposals ---------------------------------------------------------

struct vc1cu_lp {
    vc1cu_ctx* c = nullptr;
    LpGeom g{};
    int capacity = 0, max_batch = 0;
    size_t xelems = 0, aelems = 0;  // bf16 elements of one sample's input / one layer's output
    float* w = nullptr;             // fp32 master parameters
    float* gr = nullptr;            // their gradients
    float* m1 = nullptr;            // Adam moments
    float* m2 = nullptr;
    void* fwd_b = nullptr;          // packed bf16 B operands
    void* dgr_b = nullptr;
    int step = 0;
    void* x0 = nullptr;             // dataset: per sample the input features
    int2* hints = nullptr;          // per sample the translation hint
    unsigned long long* hint_sads = nullptr;  // per sample the frame SAD at the hint
    int2* labels = nullptr;         // per sample and MB the plain search's integer vector
    int2* cands = nullptr;          // per sample and MB the K candidates
    uint8_t* fallback = nullptr;    // per sample and MB the learned pass's fallback flags
    void* act[kLpLayers] = {};      // a batch's layer outputs
    void* dz[2] = {};               // gradient ping-pong
    void* xb = nullptr;             // a training batch's gathered inputs
    int2* bhint = nullptr;          // its hints
    int2* blabel = nullptr;         // its labels
    uint8_t* cur4 = nullptr;
    uint8_t* ref4 = nullptr;
    unsigned long long* hs = nullptr;  // hint search costs
    float* loss = nullptr;
    int* err = nullptr;
    std::vector<void*> owned;
};

namespace {

size_t lp_off_w(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += (size_t)lp_wcount(k) + kLpC;
    return o;
}
size_t lp_off_b(int l) { return lp_off_w(l) + (size_t)lp_wcount(l); }
size_t lp_off_head() { return lp_off_w(kLpLayers); }

template <class T>
T* lp_alloc(vc1cu_lp* n, size_t bytes, const char* what) {
    void* d = nullptr;
    ck(cudaMalloc(&d, bytes ? bytes : 16), what);
    n->owned.push_back(d);
    return static_cast<T*>(d);
}

void lp_check_sample(const vc1cu_lp* n, int s) {
    if (s < 0 || s >= n->capacity) throw Fail{VC1CU_ERR_ARG, "sample index out of range"};
}

void lp_pack(vc1cu_lp* n) { ck(lp_launch_pack(n->w, n->fwd_b, n->dgr_b, n->c->stream), "lp pack"); }

size_t lp_fwd_off(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += lp_fwd_b_elems(k);
    return o;
}
size_t lp_dgr_off(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += lp_dgrad_b_elems(k);
    return o;
}

// The four convolutions of `frames` pictures starting at x (bf16 elements).
void lp_forward(vc1cu_lp* n, const void* x, int frames) {
    const auto* bf = static_cast<const uint16_t*>(n->fwd_b);
    for (int l = 0; l < kLpLayers; ++l) {
        LpConvArgs a{};
        a.x = l == 0 ? x : n->act[l - 1];
        a.wb = bf + lp_fwd_off(l);
        a.bias = n->w + lp_off_b(l);
        a.y = n->act[l];
        a.W4 = n->g.W4;
        a.H4 = n->g.H4;
        a.frames = frames;
        a.err = n->err;
        ck(lp_launch_conv(lp_cin(l), false, a, n->c->sm_count, n->c->stream), "lp conv forward");
    }
    n->c->counters.kernel_launches += kLpLayers;
}

// Forward, loss and every gradient of a gathered batch (xb, bhint, blabel) into gr; returns the
// loss (synchronous).
float lp_backward(vc1cu_lp* n, int frames) {
    vc1cu_ctx* c = n->c;
    const int mbs = n->g.mbw * n->g.mbh;
    ck(cudaMemsetAsync(n->gr, 0, sizeof(float) * lp_param_count(), c->stream), "lp zero grads");
    ck(cudaMemsetAsync(n->loss, 0, sizeof(float), c->stream), "lp zero loss");
    lp_forward(n, n->xb, frames);
    LpHeadArgs h{};
    h.y4 = n->act[kLpLayers - 1];
    h.wh = n->w + lp_off_head();
    h.bh = h.wh + kLpHead * kLpC;
    h.hint = n->bhint;
    h.labels = n->blabel;
    h.cands = nullptr;
    h.loss = n->loss;
    h.dwh = n->gr + lp_off_head();
    h.dbh = h.dwh + kLpHead * kLpC;
    h.dz4 = n->dz[0];
    h.db4 = n->gr + lp_off_b(kLpLayers - 1);
    h.W4 = n->g.W4;
    h.H4 = n->g.H4;
    h.mbw = n->g.mbw;
    h.mbh = n->g.mbh;
    h.frames = frames;
    h.range = n->g.range;
    h.inv_count = 1.0f / (float)(mbs * frames);
    ck(lp_launch_head(h, c->stream), "lp head");
    const auto* db = static_cast<const uint16_t*>(n->dgr_b);
    int cur = 0;  // dz[cur] holds the gradient at layer l's pre-activation
    for (int l = kLpLayers - 1; l >= 0; --l) {
        LpWgradArgs wa{};
        wa.x = l == 0 ? n->xb : n->act[l - 1];
        wa.dz = n->dz[cur];
        wa.dw = n->gr + lp_off_w(l);
        wa.W4 = n->g.W4;
        wa.H4 = n->g.H4;
        wa.frames = frames;
        wa.err = n->err;
        ck(lp_launch_wgrad(lp_cin(l), wa, c->sm_count, c->stream), "lp wgrad");
        if (l > 0) {
            LpConvArgs a{};
            a.x = n->dz[cur];
            a.wb = db + lp_dgr_off(l);
            a.y = n->dz[1 - cur];
            a.act = n->act[l - 1];
            a.dbias = n->gr + lp_off_b(l - 1);
            a.W4 = n->g.W4;
            a.H4 = n->g.H4;
            a.frames = frames;
            a.err = n->err;
            ck(lp_launch_conv(kLpC, true, a, c->sm_count, c->stream), "lp conv dgrad");
            cur = 1 - cur;
        }
    }
    c->counters.kernel_launches += 1 + 2 * kLpLayers - 1;
    float loss = 0.0f;
    int err = 0;
    ck(cudaMemcpyAsync(&loss, n->loss, sizeof loss, cudaMemcpyDeviceToHost, c->stream), "lp loss");
    ck(cudaMemcpyAsync(&err, n->err, sizeof err, cudaMemcpyDeviceToHost, c->stream), "lp err");
    sync_checked(c);
    if (err) {
        ck(cudaMemsetAsync(n->err, 0, sizeof(int), c->stream), "lp err reset");
        throw Fail{VC1CU_ERR_TIMEOUT, "a tensor-core wait of the proposal network timed out"};
    }
    return loss;
}

void lp_gather(vc1cu_lp* n, const int* samples, int count) {
    vc1cu_ctx* c = n->c;
    if (count < 1 || count > n->max_batch) throw Fail{VC1CU_ERR_ARG, "batch must be 1..max_batch samples"};
    const int mbs = n->g.mbw * n->g.mbh;
    for (int i = 0; i < count; ++i) {
        lp_check_sample(n, samples[i]);
        const size_t s = (size_t)samples[i];
        ck(cudaMemcpyAsync(static_cast<uint16_t*>(n->xb) + n->xelems * i, static_cast<const uint16_t*>(n->x0) + n->xelems * s,
                           n->xelems * 2, cudaMemcpyDeviceToDevice, c->stream), "lp gather");
        ck(cudaMemcpyAsync(n->bhint + i, n->hints + s, sizeof(int2), cudaMemcpyDeviceToDevice, c->stream), "lp gather");
        ck(cudaMemcpyAsync(n->blabel + (size_t)mbs * i, n->labels + (size_t)mbs * s, sizeof(int2) * mbs,
                           cudaMemcpyDeviceToDevice, c->stream), "lp gather");
    }
}

// He-uniform initial weights from a counter-based hash (no libm), biases zero.
void lp_init(vc1cu_lp* n, uint64_t seed) {
    std::vector<float> h(lp_param_count(), 0.0f);
    auto unit = [&](uint64_t i) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    uint64_t k = 0;
    for (int l = 0; l < kLpLayers; ++l) {
        const double a = std::sqrt(6.0 / (9.0 * lp_cin(l)));
        for (int i = 0; i < lp_wcount(l); ++i) h[lp_off_w(l) + i] = (float)(a * unit(k++));
    }
    const double ah = 0.1 * std::sqrt(6.0 / kLpC);
    for (int i = 0; i < kLpHead * kLpC; ++i) h[lp_off_head() + i] = (float)(ah * unit(k++));
    ck(cudaMemcpyAsync(n->w, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, n->c->stream), "lp init");
    ck(cudaMemsetAsync(n->m1, 0, sizeof(float) * h.size(), n->c->stream), "lp init");
    ck(cudaMemsetAsync(n->m2, 0, sizeof(float) * h.size(), n->c->stream), "lp init");
    n->step = 0;
    lp_pack(n);
    sync_checked(n->c);
}

}  // namespace

extern "C" {

int vc1cu_lp_param_count(void) { return lp_param_count(); }

int vc1cu_lp_create(vc1cu_ctx* c, int width, int height, int search_range, int capacity, int max_batch, uint64_t seed,
                    vc1cu_lp** out) {
    return guarded(c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        *out = nullptr;
        if (width <= 0 || height <= 0 || (width & 1) || (height & 1) || width > 16384 || height > 16384)
            throw Fail{VC1CU_ERR_ARG, "width/height must be positive, even and <= 16384"};
        if (search_range < 0 || search_range > 1024) throw Fail{VC1CU_ERR_ARG, "search_range must be 0..1024"};
        if (capacity < 1 || capacity > (1 << 20) || max_batch < 1 || max_batch > 64)
            throw Fail{VC1CU_ERR_ARG, "capacity must be >= 1 and max_batch 1..64"};
        std::unique_ptr<vc1cu_lp> n(new vc1cu_lp);
        n->c = c;
        n->g.W = width;
        n->g.H = height;
        n->g.mbw = (width + 15) / 16;
        n->g.mbh = (height + 15) / 16;
        n->g.W4 = 4 * n->g.mbw;
        n->g.H4 = 4 * n->g.mbh;
        n->g.range = search_range;
        n->capacity = capacity;
        n->max_batch = max_batch;
        const size_t px = (size_t)n->g.W4 * n->g.H4, mbs = (size_t)n->g.mbw * n->g.mbh;
        n->xelems = px * kLpCin0;
        n->aelems = px * kLpC;
        try {
            const size_t np = (size_t)lp_param_count();
            n->w = lp_alloc<float>(n.get(), 4 * np, "cudaMalloc(lp params)");
            n->gr = lp_alloc<float>(n.get(), 4 * np, "cudaMalloc(lp grads)");
            n->m1 = lp_alloc<float>(n.get(), 4 * np, "cudaMalloc(lp adam)");
            n->m2 = lp_alloc<float>(n.get(), 4 * np, "cudaMalloc(lp adam)");
            size_t fb = 0, db = 0;
            for (int l = 0; l < kLpLayers; ++l) {
                fb += lp_fwd_b_elems(l);
                db += lp_dgrad_b_elems(l);
            }
            n->fwd_b = lp_alloc<void>(n.get(), 2 * fb, "cudaMalloc(lp packed weights)");
            n->dgr_b = lp_alloc<void>(n.get(), 2 * db, "cudaMalloc(lp packed weights)");
            n->x0 = lp_alloc<void>(n.get(), 2 * n->xelems * capacity, "cudaMalloc(lp dataset)");
            n->hints = lp_alloc<int2>(n.get(), sizeof(int2) * capacity, "cudaMalloc(lp hints)");
            n->hint_sads = lp_alloc<unsigned long long>(n.get(), 8 * (size_t)capacity, "cudaMalloc(lp hints)");
            n->labels = lp_alloc<int2>(n.get(), sizeof(int2) * mbs * capacity, "cudaMalloc(lp labels)");
            n->cands = lp_alloc<int2>(n.get(), sizeof(int2) * kLpK * mbs * capacity, "cudaMalloc(lp candidates)");
            n->fallback = lp_alloc<uint8_t>(n.get(), mbs * capacity, "cudaMalloc(lp fallback flags)");
            for (int l = 0; l < kLpLayers; ++l)
                n->act[l] = lp_alloc<void>(n.get(), 2 * n->aelems * max_batch, "cudaMalloc(lp activations)");
            for (int k = 0; k < 2; ++k) n->dz[k] = lp_alloc<void>(n.get(), 2 * n->aelems * max_batch, "cudaMalloc(lp grads)");
            n->xb = lp_alloc<void>(n.get(), 2 * n->xelems * max_batch, "cudaMalloc(lp batch)");
            n->bhint = lp_alloc<int2>(n.get(), sizeof(int2) * max_batch, "cudaMalloc(lp batch)");
            n->blabel = lp_alloc<int2>(n.get(), sizeof(int2) * mbs * max_batch, "cudaMalloc(lp batch)");
            // quarter-resolution pictures, then their 1/16-resolution level (the hint search's)
            n->cur4 = lp_alloc<uint8_t>(n.get(), px + mbs, "cudaMalloc(lp quarter-res)");
            n->ref4 = lp_alloc<uint8_t>(n.get(), px + mbs, "cudaMalloc(lp quarter-res)");
            n->hs = lp_alloc<unsigned long long>(n.get(), 8 * (65 * 65 + 32), "cudaMalloc(lp hint search)");
            n->loss = lp_alloc<float>(n.get(), 16, "cudaMalloc(lp loss)");
            n->err = lp_alloc<int>(n.get(), 16, "cudaMalloc(lp err)");
            ck(cudaMemsetAsync(n->err, 0, 16, c->stream), "lp err");
            ck(cudaMemsetAsync(n->labels, 0, sizeof(int2) * mbs * capacity, c->stream), "lp labels");
            lp_init(n.get(), seed);
        } catch (...) {
            for (void* d : n->owned) cudaFree(d);
            throw;
        }
        *out = n.release();
        return VC1CU_OK;
    });
}

int vc1cu_lp_destroy(vc1cu_lp* n) {
    if (!n) return VC1CU_OK;
    cudaSetDevice(n->c->device);
    cudaStreamSynchronize(n->c->stream);
    for (void* d : n->owned) cudaFree(d);
    delete n;
    return VC1CU_OK;
}

int vc1cu_lp_get_params(vc1cu_lp* n, float* out) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    return guarded(n->c, [&]() -> int {
        if (!out) throw Fail{VC1CU_ERR_ARG, "null output"};
        ck(cudaMemcpyAsync(out, n->w, sizeof(float) * lp_param_count(), cudaMemcpyDeviceToHost, n->c->stream), "lp params");
        sync_checked(n->c);
        return VC1CU_OK;
    });
}

int vc1cu_lp_set_params(vc1cu_lp* n, const float* in) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    return guarded(n->c, [&]() -> int {
        if (!in) throw Fail{VC1CU_ERR_ARG, "null input"};
        const size_t b = sizeof(float) * lp_param_count();
        ck(cudaMemcpyAsync(n->w, in, b, cudaMemcpyHostToDevice, n->c->stream), "lp params");
        ck(cudaMemsetAsync(n->m1, 0, b, n->c->stream), "lp adam");
        ck(cudaMemsetAsync(n->m2, 0, b, n->c->stream), "lp adam");
        n->step = 0;
        lp_pack(n);
        sync_checked(n->c);
        return VC1CU_OK;
    });
}

int vc1cu_lp_prepare(vc1cu_lp* n, int cur_id, int ref_id, int sample) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        lp_check_sample(n, sample);
        FrameSlot& fc = frame_slot(c, cur_id);
        FrameSlot& fr = frame_slot(c, ref_id);
        if (fc.w != n->g.W || fc.h != n->g.H || fr.w != n->g.W || fr.h != n->g.H)
            throw Fail{VC1CU_ERR_ARG, "frame size differs from the network's raster"};
        c->used_frames.push_back(cur_id);
        c->used_frames.push_back(ref_id);
        const DevFrame cf = fc.view(), rf = fr.view();
        ck(lp_launch_downsample(cf.y, cf.pitch_y, rf.y, rf.pitch_y, n->g, n->cur4, n->ref4, c->stream), "lp downsample");
        ck(lp_launch_hint(cf.y, cf.pitch_y, rf.y, rf.pitch_y, n->g, n->cur4, n->ref4, n->hs, n->hints + sample,
                          n->hint_sads + sample, c->stream),
           "lp hint search");
        ck(lp_launch_features(rf.y, rf.pitch_y, n->g, n->cur4, n->ref4, n->hints + sample,
                              static_cast<uint16_t*>(n->x0) + n->xelems * sample, c->stream),
           "lp features");
        c->counters.kernel_launches += 8;
        return VC1CU_OK;
    });
}

int vc1cu_lp_set_labels(vc1cu_lp* n, int sample, int result_slot_id) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        lp_check_sample(n, sample);
        const int mbs = n->g.mbw * n->g.mbh;
        ResultSlot& s = result_slot(c, result_slot_id, mbs, false);
        ck(lp_launch_labels(s.r.mvs, mbs, n->labels + (size_t)mbs * sample, c->stream), "lp labels");
        c->counters.kernel_launches++;
        return VC1CU_OK;
    });
}

int vc1cu_lp_train_step(vc1cu_lp* n, const int* samples, int count, float lr, float* loss) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        if (!samples) throw Fail{VC1CU_ERR_ARG, "null sample list"};
        lp_gather(n, samples, count);
        const float l = lp_backward(n, count);
        ++n->step;
        ck(lp_launch_adam(n->w, n->gr, n->m1, n->m2, lp_param_count(), lr, 0.9f, 0.999f, 1e-8f, n->step, c->stream),
           "lp adam");
        lp_pack(n);
        c->counters.kernel_launches += 1 + kLpLayers;
        if (loss) *loss = l;
        return VC1CU_OK;
    });
}

int vc1cu_lp_gradients(vc1cu_lp* n, const int* samples, int count, float* grads, float* loss) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        if (!samples) throw Fail{VC1CU_ERR_ARG, "null sample list"};
        lp_gather(n, samples, count);
        const float l = lp_backward(n, count);
        if (grads) {
            ck(cudaMemcpyAsync(grads, n->gr, sizeof(float) * lp_param_count(), cudaMemcpyDeviceToHost, c->stream),
               "lp grads");
            sync_checked(c);
        }
        if (loss) *loss = l;
        return VC1CU_OK;
    });
}

int vc1cu_lp_propose(vc1cu_lp* n, int first_sample, int count) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        if (count < 1 || count > n->max_batch) throw Fail{VC1CU_ERR_ARG, "count must be 1..max_batch"};
        lp_check_sample(n, first_sample);
        lp_check_sample(n, first_sample + count - 1);
        const int mbs = n->g.mbw * n->g.mbh;
        lp_forward(n, static_cast<const uint16_t*>(n->x0) + n->xelems * first_sample, count);
        LpHeadArgs h{};
        h.y4 = n->act[kLpLayers - 1];
        h.wh = n->w + lp_off_head();
        h.bh = h.wh + kLpHead * kLpC;
        h.hint = n->hints + first_sample;
        h.cands = n->cands + (size_t)kLpK * mbs * first_sample;
        h.W4 = n->g.W4;
        h.H4 = n->g.H4;
        h.mbw = n->g.mbw;
        h.mbh = n->g.mbh;
        h.frames = count;
        h.range = n->g.range;
        ck(lp_launch_head(h, c->stream), "lp head");
        c->counters.kernel_launches++;
        return VC1CU_OK;
    });
}

int vc1cu_lp_read_sample(vc1cu_lp* n, int sample, uint16_t* features, vc1cu_mv* hint, vc1cu_mv* candidates,
                         uint8_t* fallback) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        lp_check_sample(n, sample);
        const size_t mbs = (size_t)n->g.mbw * n->g.mbh;
        if (features)
            ck(cudaMemcpyAsync(features, static_cast<const uint16_t*>(n->x0) + n->xelems * sample, 2 * n->xelems,
                               cudaMemcpyDeviceToHost, c->stream), "lp read");
        if (hint) ck(cudaMemcpyAsync(hint, n->hints + sample, 8, cudaMemcpyDeviceToHost, c->stream), "lp read");
        if (candidates)
            ck(cudaMemcpyAsync(candidates, n->cands + kLpK * mbs * sample, 8 * kLpK * mbs, cudaMemcpyDeviceToHost,
                               c->stream), "lp read");
        if (fallback)
            ck(cudaMemcpyAsync(fallback, n->fallback + mbs * sample, mbs, cudaMemcpyDeviceToHost, c->stream), "lp read");
        sync_checked(c);
        return VC1CU_OK;
    });
}

int vc1cu_lp_analyze(vc1cu_lp* n, const vc1cu_params* p, const vc1cu_lp_pass* passes, int count, int fallback) {
    if (!n) return fail(nullptr, VC1CU_ERR_ARG, "null network");
    vc1cu_ctx* c = n->c;
    return guarded(c, [&]() -> int {
        if (count < 1 || !passes) throw Fail{VC1CU_ERR_ARG, "invalid pass list"};
        DevParams P;
        std::string why;
        const int rc = make_dev_params(p, P, why);
        if (rc) throw Fail{rc, why};
        if (P.W != n->g.W || P.H != n->g.H || P.range != n->g.range)
            throw Fail{VC1CU_ERR_ARG, "params differ from the network's raster or search range"};
        const size_t mbs = (size_t)P.mbw * P.mbh;
        std::vector<vc1cu_pass> q(count);
        std::vector<PassExtra> ex(count);
        for (int i = 0; i < count; ++i) {
            const vc1cu_lp_pass& a = passes[i];
            lp_check_sample(n, a.sample);
            if (a.mode == VC1CU_MV_MIXED) throw Fail{VC1CU_ERR_ARG, "learned passes are 1-MV"};
            if (a.out_slot < 0 || a.out_slot >= kMaxSlot) throw Fail{VC1CU_ERR_ARG, "result slot out of range"};
            q[i] = vc1cu_pass{a.cur_id, a.ref_id, a.mode, 0, -1, a.out_slot, a.pqindex};
            ex[i].cands = n->cands + kLpK * mbs * a.sample;
            ex[i].fallback = n->fallback + mbs * a.sample;
            ex[i].hint = n->hints + a.sample;
            ex[i].hint_sad = n->hint_sads + a.sample;
        }
        for (int i = 0; i < count; ++i)
            for (int j = 0; j < i; ++j)
                if (q[i].out_slot == q[j].out_slot) throw Fail{VC1CU_ERR_ARG, "two passes write one result slot"};
        if (fallback && count > kMaxLpPasses) throw Fail{VC1CU_ERR_ARG, "too many learned passes in one call"};
        std::vector<PassDesc> learned;
        launch_group(c, p, q.data(), count, true, ex.data(), nullptr, &learned);
        if (!fallback) return VC1CU_OK;
        // The macroblocks whose best learned match is not good: the plain search, all of them at
        // once, with the finished learned field as their neighbourhood, into scratch slots; then
        // their results replace the learned ones and the totals are taken again.
        std::vector<vc1cu_pass> qb(q);
        std::vector<PassExtra> eb(count);
        std::vector<DevResult> snap(count);
        for (int i = 0; i < count; ++i) {
            snap[i] = learned[i].out;
            qb[i].out_slot = kInternalLpFb + i;
            eb[i].only = ex[i].fallback;
            eb[i].hint = ex[i].hint;
            eb[i].hint_sad = ex[i].hint_sad;
            eb[i].nb = &snap[i];
        }
        launch_group(c, p, qb.data(), count, true, eb.data());
        for (int i = 0; i < count; ++i) {
            const ResultSlot& s = result_slot(c, kInternalLpFb + i, (int)mbs, false);
            ck(launch_learned_merge(learned[i].out, s.r, ex[i].fallback, (int)mbs, c->stream), "learned merge launch");
            c->counters.kernel_launches++;
        }
        void* hp = staging(c, sizeof(PassDesc) * count);
        std::memcpy(hp, learned.data(), sizeof(PassDesc) * count);
        ck(cudaMemcpyAsync(c->d_passes, hp, sizeof(PassDesc) * count, cudaMemcpyHostToDevice, c->stream),
           "cudaMemcpyAsync(pass descriptors)");
        staging_mark(c);
        totals_kernel<<<count, 256, 0, c->stream>>>(learned[0].geom, c->d_passes, count);
        ck(cudaGetLastError(), "totals_kernel launch");
        return VC1CU_OK;
    });
}

}  // extern "C"
