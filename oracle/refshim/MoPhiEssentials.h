// Minimal stand-in for the parts of MoPhiEssentials that the TLFEA element and solver
// sources use (the submodule external/MoPhiEssentials is not vendored with the reference).
//
// Test infrastructure only: it lets the reference's unchanged CUDA sources compile and run
// as a parity harness on the GPU. Nothing in the product library includes it.
//
// Provided:
//   mophi::DualArray<T>   a host array paired with a device array of the same length;
//                         resize / BindDevicePointer (keeps a caller's raw device pointer
//                         in step with the allocation) / host / ToDevice / ToHost / SetVal
//                         (host values) / MakeReadyDevice (host -> device) / free / size.
//   MOPHI_GPU_CALL(call)  evaluates a CUDA runtime call and records the first failure.
//   MOPHI_ERROR(...)      logs a misuse message and records it (the caller then returns,
//                         as the reference's code does after each MOPHI_ERROR).
//   MOPHI_INFO(...)       logs at info verbosity (silent unless enabled).
//   mophi::Logger         verbosity switch used by the reference's example drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mophi {

enum Verbosity { VERBOSITY_QUIET = 0, VERBOSITY_ERROR = 1, VERBOSITY_WARNING = 2, VERBOSITY_INFO = 3 };

class Logger {
  public:
    static Logger& GetInstance() {
        static Logger l;
        return l;
    }
    void SetVerbosity(int v) { verbosity_ = v; }
    int Verbosity() const { return verbosity_; }

  private:
    int verbosity_ = VERBOSITY_QUIET;
};

// First CUDA failure and the number of MOPHI_ERROR reports since the last reset;
// the harness reads and clears them around every reference call.
struct ShimStatus {
    int cuda_error = 0;
    int n_errors = 0;
    char where[256] = {0};
};
inline ShimStatus& shim_status() {
    static ShimStatus s;
    return s;
}

inline void shim_cuda_fail(cudaError_t e, const char* file, int line, const char* expr) {
    ShimStatus& s = shim_status();
    if (s.cuda_error == 0) {
        s.cuda_error = static_cast<int>(e);
        std::snprintf(s.where, sizeof(s.where), "%s:%d %s", file, line, expr);
    }
    std::fprintf(stderr, "[refshim] CUDA error %d (%s) at %s:%d: %s\n", static_cast<int>(e), cudaGetErrorString(e),
                 file, line, expr);
}

inline void shim_vlog(const char* tag, const char* fmt, va_list ap) {
    std::fprintf(stderr, "[refshim %s] ", tag);
    std::vfprintf(stderr, fmt, ap);
    std::fprintf(stderr, "\n");
}
inline void shim_error(const char* fmt, ...) {
    shim_status().n_errors++;
    va_list ap;
    va_start(ap, fmt);
    shim_vlog("error", fmt, ap);
    va_end(ap);
}
inline void shim_error(const std::string& msg) { shim_error("%s", msg.c_str()); }
inline void shim_info(const char* fmt, ...) {
    if (Logger::GetInstance().Verbosity() < VERBOSITY_INFO)
        return;
    va_list ap;
    va_start(ap, fmt);
    shim_vlog("info", fmt, ap);
    va_end(ap);
}
inline void shim_info(const std::string& msg) { shim_info("%s", msg.c_str()); }

template <typename T>
class DualArray {
  public:
    DualArray() = default;
    DualArray(const DualArray&) = delete;
    DualArray& operator=(const DualArray&) = delete;
    ~DualArray() { free(); }

    void resize(size_t n) {
        if (n == n_ && dev_ != nullptr)
            return;
        free();
        n_ = n;
        host_.assign(n, T(0));
        if (n > 0) {
            cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dev_), n * sizeof(T));
            if (e != cudaSuccess) {
                shim_cuda_fail(e, __FILE__, __LINE__, "cudaMalloc(DualArray)");
                dev_ = nullptr;
            }
        }
        if (bound_)
            *bound_ = dev_;
    }
    void BindDevicePointer(T** p) {
        bound_ = p;
        if (bound_)
            *bound_ = dev_;
    }
    T* host() { return host_.data(); }
    const T* host() const { return host_.data(); }
    T* device() { return dev_; }
    size_t size() const { return n_; }
    T* data() { return host_.data(); }

    void ToDevice() {
        if (n_ == 0 || dev_ == nullptr)
            return;
        cudaError_t e = cudaMemcpy(dev_, host_.data(), n_ * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess)
            shim_cuda_fail(e, __FILE__, __LINE__, "DualArray::ToDevice");
    }
    void ToHost() {
        if (n_ == 0 || dev_ == nullptr)
            return;
        cudaError_t e = cudaMemcpy(host_.data(), dev_, n_ * sizeof(T), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            shim_cuda_fail(e, __FILE__, __LINE__, "DualArray::ToHost");
    }
    void SetVal(const T& v) { std::fill(host_.begin(), host_.end(), v); }
    void MakeReadyDevice() { ToDevice(); }
    void MakeReadyHost() { ToHost(); }

    void free() {
        if (dev_ != nullptr)
            cudaFree(dev_);
        dev_ = nullptr;
        n_ = 0;
        host_.clear();
        host_.shrink_to_fit();
        if (bound_)
            *bound_ = nullptr;
    }

  private:
    std::vector<T> host_;
    T* dev_ = nullptr;
    size_t n_ = 0;
    T** bound_ = nullptr;
};

}  // namespace mophi

#define MOPHI_GPU_CALL(call)                                                      \
    do {                                                                          \
        cudaError_t mophi_shim_e_ = (call);                                       \
        if (mophi_shim_e_ != cudaSuccess)                                         \
            ::mophi::shim_cuda_fail(mophi_shim_e_, __FILE__, __LINE__, #call);    \
    } while (0)

#define MOPHI_ERROR(...) ::mophi::shim_error(__VA_ARGS__)
#define MOPHI_INFO(...) ::mophi::shim_info(__VA_ARGS__)
#define MOPHI_WARNING(...) ::mophi::shim_info(__VA_ARGS__)
