// Shared host/device helpers for the fftsvd_b200 library: error status
// plumbing (thread-local last error, never exit), RAII device buffers and
// small numeric traits for the FP32/FP64 operator variants.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fftsvd_b200.h"

namespace fftsvd {

// Error carried from the point of failure to the C-ABI boundary, where it is
// turned into a status code and a message for fftsvd_b200_last_error().
struct Error : std::runtime_error {
   int code;
   Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

// Runs f and turns exceptions into a status code (and the last-error text).
template <typename F>
inline int guarded(F&& f) {
   try {
      f();
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   } catch (const std::bad_alloc&) {
      set_last_error("host allocation failed");
      return FFTSVD_ERR_ARGUMENT;
   } catch (const std::exception& e) {
      set_last_error(e.what());
      return FFTSVD_ERR_ARGUMENT;
   }
}

#define FFTSVD_CUDA(call)                                                                              \
   do {                                                                                               \
      cudaError_t err_ = (call);                                                                      \
      if (err_ != cudaSuccess)                                                                        \
         throw ::fftsvd::Error(FFTSVD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
   } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts the launch (fftsvd_b200_launch_count).
extern std::atomic<long long> g_kernel_launches;
// Device allocations (cudaMalloc) made by the library (fftsvd_b200_device_alloc_count).
extern std::atomic<long long> g_device_allocs;
#define FFTSVD_CHECK_LAUNCH()                                        \
   do {                                                              \
      ::fftsvd::g_kernel_launches.fetch_add(1, std::memory_order_relaxed); \
      FFTSVD_CUDA(cudaGetLastError());                              \
   } while (0)

#define FFTSVD_REQUIRE(cond, msg)                                        \
   do {                                                                 \
      if (!(cond)) throw ::fftsvd::Error(FFTSVD_ERR_ARGUMENT, (msg));  \
   } while (0)

// Owning device allocation.
template <typename T>
class DevBuf {
 public:
   DevBuf() = default;
   explicit DevBuf(size_t n) { alloc(n); }
   ~DevBuf() { release(); }
   DevBuf(const DevBuf&) = delete;
   DevBuf& operator=(const DevBuf&) = delete;
   DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
   DevBuf& operator=(DevBuf&& o) noexcept {
      if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
      return *this;
   }
   void alloc(size_t n) {
      release();
      n_ = n;
      if (n) {
         g_device_allocs.fetch_add(1, std::memory_order_relaxed);
         FFTSVD_CUDA(cudaMalloc(&p_, n * sizeof(T)));
      }
   }
   void upload(const T* host, size_t n) {
      alloc(n);
      if (n) FFTSVD_CUDA(cudaMemcpy(p_, host, n * sizeof(T), cudaMemcpyHostToDevice));
   }
   void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
   void zero(cudaStream_t s = 0) {
      if (n_) FFTSVD_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
   }
   void release() {
      if (p_) cudaFree(p_);
      p_ = nullptr;
      n_ = 0;
   }
   T* get() const { return p_; }
   size_t size() const { return n_; }
   size_t bytes() const { return n_ * sizeof(T); }

 private:
   T* p_ = nullptr;
   size_t n_ = 0;
};

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

template <typename T>
inline const char* type_name();
template <> inline const char* type_name<float>() { return "f32"; }
template <> inline const char* type_name<double>() { return "f64"; }

}  // namespace fftsvd
