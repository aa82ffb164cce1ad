// Minimal check harness for the C++ API tests: failed checks are counted and
// printed; main returns non-zero if any failed.  Device helpers for tests.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace tcheck {

inline int& failures() {
  static int n = 0;
  return n;
}

inline void report(bool ok, const char* what, const char* file, int line, const std::string& detail = {}) {
  if (ok) return;
  ++failures();
  std::fprintf(stderr, "FAIL %s:%d: %s%s%s\n", file, line, what, detail.empty() ? "" : " -- ", detail.c_str());
}

inline bool near(double a, double b, double tol) { return !std::isnan(a) && !std::isnan(b) && std::fabs(a - b) <= tol; }

inline int finish(const char* name) {
  if (failures() == 0) {
    std::printf("ok %s\n", name);
    return 0;
  }
  std::fprintf(stderr, "FAILED %s: %d check(s)\n", name, failures());
  return 1;
}

// Owning device buffer of T.
template <typename T>
struct Dev {
  T* p = nullptr;
  std::size_t n = 0;
  explicit Dev(std::size_t count) : n(count) {
    if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
      std::fprintf(stderr, "cudaMalloc failed\n");
      std::exit(2);
    }
    cudaMemset(p, 0, sizeof(T) * (count ? count : 1));
  }
  Dev(const std::vector<T>& host) : Dev(host.size()) { upload(host); }
  ~Dev() { cudaFree(p); }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  void upload(const std::vector<T>& host) { cudaMemcpy(p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice); }
  std::vector<T> download(std::size_t count = 0) const {
    std::vector<T> h(count ? count : n);
    cudaMemcpy(h.data(), p, sizeof(T) * h.size(), cudaMemcpyDeviceToHost);
    return h;
  }
};

}  // namespace tcheck

#define CHECK(expr) ::tcheck::report((expr), #expr, __FILE__, __LINE__)
#define CHECK_CLOSE(a, b, tol)                                                                 \
  ::tcheck::report(::tcheck::near((a), (b), (tol)), #a " ~= " #b, __FILE__, __LINE__,          \
                   std::to_string(static_cast<double>(a)) + " vs " + std::to_string(static_cast<double>(b)))
#define CHECK_CUDA(expr)                                                                       \
  do {                                                                                         \
    const cudaError_t e_ = (expr);                                                             \
    ::tcheck::report(e_ == cudaSuccess, #expr, __FILE__, __LINE__, cudaGetErrorString(e_));    \
  } while (0)
