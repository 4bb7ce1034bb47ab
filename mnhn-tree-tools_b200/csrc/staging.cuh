// Host <-> device transfers through two pinned staging chunks kept by a
// context, with host threads assembling or scattering each chunk while the
// other one is in flight.  Used by the k-mer tables and the point uploads.
#pragma once
#include <algorithm>
#include <thread>
#include <vector>

#include "engine_ctx.cuh"

namespace swgpu {

struct Staging {
  HostPinned<char> pin[2];
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Staging() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

constexpr size_t STAGE_CHUNK = size_t(8) << 20;  // bytes per pinned staging chunk

// The context's staging with both chunks of at least `chunk` bytes.
swe_status staging_ready(swe_ctx* ctx, size_t chunk, Staging** out);

// Chunk size of a context's transfers (the k-mer test hook shrinks it).
inline size_t stage_chunk(const swe_ctx* ctx) {
  const size_t c = ctx->kmer_batch_bytes ? std::min(ctx->kmer_batch_bytes, STAGE_CHUNK) : STAGE_CHUNK;
  return std::max<size_t>(16, c & ~size_t(15));
}

// f(t) for t in [0, tasks) on up to `threads` host threads.
template <class F>
void host_parallel(int64_t tasks, int threads, F&& f) {
  threads = (int)std::min<int64_t>(std::max(threads, 1), tasks);
  if (threads <= 1) {
    for (int64_t t = 0; t < tasks; ++t) f(t);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(threads);
  for (int w = 0; w < threads; ++w)
    th.emplace_back([&, w]() {
      for (int64_t t = w; t < tasks; t += threads) f(t);
    });
  for (auto& x : th) x.join();
}

// Host threads for a copy of `bytes` (about 1 MB each, at most 8).
inline int copy_threads(size_t bytes) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)std::min(hw, 8), bytes >> 20));
}

// copy(a, b) over [a, b) split into one sub-range per host thread.
template <class F>
void split_copy(size_t a, size_t b, F&& copy) {
  const int T = copy_threads(b - a);
  const size_t step = (b - a + T - 1) / T;
  host_parallel(T, T, [&](int64_t t) {
    const size_t x = a + (size_t)t * step, y = std::min(b, x + step);
    if (x < y) copy(x, y);
  });
}

// Host -> device copy of `total` bytes assembled by gather(dst, a, b) (source
// bytes [a, b) into dst), chunk by chunk through the two pinned buffers: the
// gather of one chunk overlaps the copy of the previous one.
template <class G>
swe_status staged_h2d(swe_ctx* ctx, Staging* sg, size_t chunk, void* d_dst, size_t total, G&& gather) {
  size_t j = 0;
  for (size_t a = 0; a < total; a += chunk, ++j) {
    const int slot = (int)(j & 1);
    const size_t b = std::min(total, a + chunk);
    CK(cudaEventSynchronize(sg->ev[slot]));  // the copy that last read this buffer
    gather(sg->pin[slot].p, a, b);
    CK(cpy(ctx, static_cast<char*>(d_dst) + a, sg->pin[slot].p, b - a, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaEventRecord(sg->ev[slot], ctx->st));
  }
  return SWE_OK;
}

// Device -> host copy of `total` bytes of d_src, handed to consume(src, a, b)
// (host bytes [a, b)) in order; the copy of the next chunk overlaps the
// consumer.  A consumer returning false stops the transfer (SWE_ERR_IO).
template <class C>
swe_status staged_d2h(swe_ctx* ctx, Staging* sg, size_t chunk, const void* d_src, size_t total, C&& consume) {
  if (total == 0) return SWE_OK;
  const size_t nch = (total + chunk - 1) / chunk;
  auto issue = [&](size_t j) -> cudaError_t {
    const size_t a = j * chunk, b = std::min(total, a + chunk);
    cudaError_t e = cpy(ctx, sg->pin[j & 1].p, static_cast<const char*>(d_src) + a, b - a,
                        cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaEventRecord(sg->ev[j & 1], ctx->st);
    return e;
  };
  CK(issue(0));
  for (size_t j = 0; j < nch; ++j) {
    if (j + 1 < nch) CK(issue(j + 1));
    CK(cudaEventSynchronize(sg->ev[j & 1]));
    const size_t a = j * chunk, b = std::min(total, a + chunk);
    if (!consume(sg->pin[j & 1].p, a, b)) {
      CK(cudaStreamSynchronize(ctx->st));
      return fail(ctx, SWE_ERR_IO, "transfer stopped by its consumer");
    }
  }
  return SWE_OK;
}

}  // namespace swgpu
