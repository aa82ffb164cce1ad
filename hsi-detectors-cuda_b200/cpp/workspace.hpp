// Scratch for the drop-in launchers whose reference signatures carry no
// workspace argument (launch_detect, the moment accumulators, launch_rx_ace).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace hsi {
namespace detail {

// Device scratch of at least `bytes` for work queued on `stream`.  One buffer
// per (device, stream), kept between calls and grown only when a call needs
// more than any earlier call on that stream did, so steady-state calls
// allocate nothing.  Work on one stream runs in order, so calls on the same
// stream reuse the buffer safely; different streams never share one.  A grown
// buffer's predecessor is released in stream order (after the work already
// queued on that stream).  Growth calls cudaMalloc, which a stream that is
// being captured into a graph does not allow: make one call at the largest
// size before capturing.  Streams are told apart by their process-unique id
// (cudaStreamGetId), so a new stream that reuses a destroyed stream's handle
// does not inherit its buffer.
cudaError_t stream_scratch(cudaStream_t stream, std::size_t bytes, void** out);

}  // namespace detail
}  // namespace hsi
