// Shared definitions of the B200 ED solver: errors, CUDA checks, device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "qed_b200.h"

namespace qed {

// Exception carrying a C-ABI status code. The C layer converts it into a
// return value; a C++ adapter on the reference side rethrows it as qcm_error
// (the reference's qcm_ED_throw, src_util/parser.cpp:323-328).
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? QED_ERR_MEMORY : QED_ERR_CUDA;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = QED_ERR_NO_DEVICE;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                   std::to_string(line) + ")");
  }
}
#define QED_CUDA(x) ::qed::cuda_check((x), #x, __FILE__, __LINE__)
#define QED_LAUNCH() ::qed::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Stream used for stream-ordered allocation by the calling host thread: the
// stream of that thread's Workspace (legacy default stream before one exists).
cudaStream_t alloc_stream();

// Owning device allocation, stream-ordered (cudaMallocAsync / cudaFreeAsync on
// the calling thread's stream, served from the device's memory pool), so that
// allocating and freeing never synchronises the whole device and host threads
// driving different instances do not serialise each other. Library calls
// synchronise their stream before returning, so a buffer may be freed from any
// thread once the call that used it has returned.
template <class T> struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    if (count) QED_CUDA(cudaMallocAsync((void **)&p, count * sizeof(T), alloc_stream()));
    n = count;
  }
  void release() {
    if (p) cudaFreeAsync(p, alloc_stream());
    p = nullptr;
    n = 0;
  }
  void upload(const T *h, size_t count, cudaStream_t s) {
    if (count > n) alloc(count);
    if (count) QED_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T> &h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void download(T *h, size_t count, cudaStream_t s) const {
    if (count) QED_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Binomial coefficient C(n, k) for n <= 64 in 64-bit arithmetic.
inline uint64_t binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  if (k > n - k) k = n - k;
  uint64_t r = 1;
  for (int i = 1; i <= k; ++i) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
  return r;
}

}  // namespace qed
