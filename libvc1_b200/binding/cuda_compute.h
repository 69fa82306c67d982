// cuda_compute.h - libvc1's handle on the B200 analysis backend (libvc1cu, include/vc1cu.h).
//
// Compiled into libvc1 itself, beside src/vulkan_compute.h (whose VulkanComputeContext this
// mirrors: create / device_name / device_index / score_motion_batch / counters /
// reset_counters, src/vulkan_compute.h:26-60). EncoderConfig::cuda_compute holds one
// std::shared_ptr to it, copied into every GOP worker's config like vulkan_compute
// (src/encoder_internal.h:289); every call runs under the context's own mutex, so the
// workers share it safely. A failing call throws std::runtime_error with the library's
// message: the CUDA backend has no CPU fallback (the reference's --vulkan-force behaviour,
// src/encoder_compute.cpp:63-64).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "vc1cu.h"
#include "vulkan_compute.h"

namespace libvc1 {

class CudaComputeContext {
public:
    // VulkanComputeContext::create (src/vulkan_compute.h:28-29); device -1: the current device.
    static std::shared_ptr<CudaComputeContext> create(int device, std::string& error) {
        vc1cu_ctx* h = nullptr;
        if (vc1cu_open(device, &h) != VC1CU_OK) {
            error = vc1cu_last_error(nullptr);
            return nullptr;
        }
        return std::shared_ptr<CudaComputeContext>(new CudaComputeContext(h));
    }
    ~CudaComputeContext() {
        if (lp_) vc1cu_lp_destroy(lp_);
        vc1cu_close(h_);
    }
    CudaComputeContext(const CudaComputeContext&) = delete;
    CudaComputeContext& operator=(const CudaComputeContext&) = delete;

    const std::string& device_name() const { return name_; }
    int device_index() const { return vc1cu_device_index(h_); }

    // VulkanComputeContext::score_motion_batch (src/vulkan_compute.h:42-51): the shader's law.
    bool score_motion_batch(const uint8_t* cur, const uint8_t* ref, int width, int height, int x0, int y0, int bw,
                            int bh, int sample_stride, bool bilinear, bool rnd, VulkanMotionMetric metric,
                            const VulkanMotionCandidate* c, size_t n, std::vector<uint64_t>& costs,
                            std::string* error = nullptr) {
        std::lock_guard<std::mutex> lock(mu_);
        costs.resize(n);
        const int rc = vc1cu_score_motion_batch(h_, cur, ref, width, height, x0, y0, bw, bh, sample_stride, bilinear,
                                                rnd, static_cast<int>(metric),
                                                reinterpret_cast<const vc1cu_mv*>(c), n, costs.data());
        if (rc != VC1CU_OK && error) *error = vc1cu_last_error(h_);
        return rc == VC1CU_OK;
    }
    VulkanComputeCounters counters() const {
        vc1cu_counters k{};
        vc1cu_counters_get(h_, &k);
        VulkanComputeCounters out{};
        out.dispatches = k.dispatches;
        out.candidates = k.candidates;
        out.frame_uploads = k.frame_uploads;
        out.frame_upload_bytes = k.frame_upload_bytes;
        out.submit_wait_nanoseconds = k.submit_wait_nanoseconds;
        return out;
    }
    void reset_counters() { vc1cu_reset_counters(h_); }

    // The analysis entry points run a sequence of library calls (uploads, the pass, the read)
    // that must not interleave with another worker's: they hold this lock around it.
    std::mutex& mutex() { return mu_; }
    vc1cu_ctx* handle() const { return h_; }
    // The learned proposals for the encoder's raster, when LIBVC1_CUDA_LEARNED names a file of
    // vc1cu_lp_param_count() little-endian float32 parameters: unseeded 1-MV analysis passes
    // without P-intra then use the learned pass (vc1cu_lp_analyze) instead of the plain search.
    // Created on first use; call with the mutex held.
    vc1cu_lp* learned(int width, int height, int search_range) {
        if (lp_tried_) return lp_;
        lp_tried_ = true;
        const char* path = std::getenv("LIBVC1_CUDA_LEARNED");
        if (!path || !*path) return nullptr;
        std::vector<float> w(static_cast<size_t>(vc1cu_lp_param_count()));
        std::FILE* f = std::fopen(path, "rb");
        if (!f) throw std::runtime_error(std::string("cannot open learned parameters ") + path);
        const size_t got = std::fread(w.data(), sizeof(float), w.size(), f);
        std::fclose(f);
        if (got != w.size()) throw std::runtime_error(std::string("short learned parameter file ") + path);
        check(vc1cu_lp_create(h_, width, height, search_range, 1, 1, 1, &lp_), "vc1cu_lp_create");
        check(vc1cu_lp_set_params(lp_, w.data()), "vc1cu_lp_set_params");
        return lp_;
    }
    // Throws with the library's message when rc is not VC1CU_OK.
    void check(int rc, const char* what) const {
        if (rc != VC1CU_OK) throw std::runtime_error(std::string("CUDA analysis backend: ") + what + ": " +
                                                     vc1cu_last_error(h_));
    }

private:
    explicit CudaComputeContext(vc1cu_ctx* h) : h_(h), name_(vc1cu_device_name(h)) {}
    vc1cu_ctx* h_;
    std::string name_;
    std::mutex mu_;
    vc1cu_lp* lp_ = nullptr;
    bool lp_tried_ = false;
};

}  // namespace libvc1
