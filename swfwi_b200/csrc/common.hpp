// Status codes, errors and a small device buffer type for the host layer.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include "swfwi_gpu.h"

namespace swfwi {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string &m);
std::string last_error();

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    int st = (e == cudaErrorMemoryAllocation) ? SWFWI_ERR_OOM : SWFWI_ERR_CUDA;
    throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

#define SWFWI_CUDA(call) ::swfwi::cuda_check((call), #call)
#define SWFWI_REQUIRE(cond, msg)                                  \
  do {                                                            \
    if (!(cond)) throw ::swfwi::Error(SWFWI_ERR_BAD_ARG, (msg));  \
  } while (0)

// Runs f, converting exceptions into a status code and a last-error text.
template <typename F>
int guarded(F &&f) {
  try {
    f();
    return SWFWI_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return SWFWI_ERR_OOM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SWFWI_ERR_CUDA;
  }
}

// Owning device allocation (cudaMalloc / cudaFree).
template <typename T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(size_t n) { resize(n); }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p_(o.p_), n_(o.n_), cap_(o.cap_) {
    o.p_ = nullptr;
    o.n_ = o.cap_ = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_; n_ = o.n_; cap_ = o.cap_;
      o.p_ = nullptr;
      o.n_ = o.cap_ = 0;
    }
    return *this;
  }
  // Grows the allocation when needed; shrinking keeps the capacity.
  void resize(size_t n) {
    if (n > cap_) {
      release();
      SWFWI_CUDA(cudaMalloc(&p_, n * sizeof(T)));
      cap_ = n;
    }
    n_ = n;
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = cap_ = 0;
  }
  size_t capacity() const { return cap_; }
  T *get() const { return p_; }
  size_t size() const { return n_; }
  void upload(const T *h, size_t n, cudaStream_t st) {
    resize(n);
    if (n) SWFWI_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T> &h, cudaStream_t st) { upload(h.data(), h.size(), st); }
  void zero(cudaStream_t st) {
    if (n_) SWFWI_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), st));
  }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
  size_t cap_ = 0;
};

}  // namespace swfwi
