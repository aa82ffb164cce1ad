// Grow-only per-stream scratch for the drop-in launchers (workspace.hpp).
#include "workspace.hpp"

#include <mutex>
#include <vector>

#include "hsi/sam_cuda.hpp"

namespace hsi {
namespace detail {
namespace {

struct Scratch {
  int device;
  unsigned long long stream_id;
  void* ptr;
  std::size_t bytes;
};

std::mutex g_mutex;
std::vector<Scratch> g_scratch;

}  // namespace

cudaError_t stream_scratch(cudaStream_t stream, std::size_t bytes, void** out) {
  *out = nullptr;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  unsigned long long id = 0;
  e = cudaStreamGetId(stream, &id);
  if (e != cudaSuccess) return e;
  if (bytes == 0) bytes = 256;
  std::lock_guard<std::mutex> lock(g_mutex);
  Scratch* s = nullptr;
  for (Scratch& x : g_scratch)
    if (x.device == device && x.stream_id == id) s = &x;
  if (s && s->bytes >= bytes) {
    *out = s->ptr;
    return cudaSuccess;
  }
  void* p = nullptr;
  e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return e;
  if (s) {
    // the old buffer may still be read by work queued on this stream
    e = cudaFreeAsync(s->ptr, stream);
    if (e != cudaSuccess) {
      cudaFree(p);
      return e;
    }
    s->ptr = p;
    s->bytes = bytes;
  } else {
    g_scratch.push_back(Scratch{device, id, p, bytes});
  }
  *out = p;
  return cudaSuccess;
}

}  // namespace detail

cudaError_t release_launch_workspaces() {
  std::lock_guard<std::mutex> lock(detail::g_mutex);
  int current = 0;
  cudaError_t first = cudaGetDevice(&current);
  for (const detail::Scratch& s : detail::g_scratch) {
    cudaError_t e = cudaSetDevice(s.device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaFree(s.ptr);
    if (first == cudaSuccess) first = e;
  }
  detail::g_scratch.clear();
  cudaSetDevice(current);
  return first;
}

}  // namespace hsi
